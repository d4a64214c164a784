// Tabulated layer phase factors exp(omega_k * i eta h) for uniform frequency grids.
//
// The frequency axis is cut into tiles of 128 (tile u holds k = 128 u + t, t < 128).  When
// every frequency of tile u lies on the grid's line omega_k = omega_0 + k delta,
// delta = (omega_{n-1} - omega_0) / (n - 1), to within kUniformTol * max|omega| (rounding of
// an arange-built grid is ~1 ulp), then for each layer phase c (i eta h or i neta h)
//
//     exp(omega_k c) = (hi[u] * mid[t / 16]) * lo[t % 16],
//     lo[j] = exp(j delta c) (j < 16),  mid[m] = exp(16 m delta c) (m < 8),
//     hi[u] = exp(omega_{128 u} c)       (the tile's own first frequency),
//
// each entry one direct exp of an exactly formed argument: two complex products and three
// shared-memory reads replace an exp and a sincos per layer, phase and frequency.  A tile
// whose frequencies leave the line, or whose entries exceed 1e100 in magnitude (so that no
// product can overflow), evaluates its phases directly.  The per-tile decision depends only
// on the grid, so every kernel that uses this table gives bit-identical results.
#pragma once

#include "kr_internal.cuh"

namespace kr {

constexpr int kPhTile = 128;
constexpr int kPhLo = 16;
constexpr int kPhMid = kPhTile / kPhLo;
constexpr int kPhHead = kPhLo + kPhMid;  // lo + mid entries ahead of the hi entries
constexpr int kPhMaxTiles = 31;         // tiles per table (bit 31 of the mask: lo / mid bad)
constexpr double kUniformTol = 2e-15;
constexpr double kPhMaxMag = 1e100;

// Entries per phase for tables of up to `tiles` hi entries; bytes for a model of L layers.
__host__ __device__ inline int phase_entries(int tiles) { return kPhHead + tiles; }
__host__ __device__ inline size_t phase_table_bytes(int n_layers, int tiles) {
  return sizeof(cd) * (size_t)phase_entries(tiles) * 2 * (size_t)(n_layers - 1);
}

// Which models tabulate: those whose forward-kernel block (prologue + a table of 16 tiles)
// stays within 50 KB of shared memory, i.e. up to 30 layers.  Every kernel applies the same
// per-model rule, so a model's phases come from the same source everywhere.
constexpr int kFwdTabTiles = 16;
constexpr size_t kFwdTabSmemMax = 50 * 1024;
__host__ __device__ inline bool phase_table_model(int n_layers) {
  return prologue_smem_bytes(n_layers) + phase_table_bytes(n_layers, kFwdTabTiles) <=
         kFwdTabSmemMax;
}
inline int phase_table_max_layers() {
  int L = 1;
  while (L < kMaxLayers && phase_table_model(L + 1)) ++L;
  return L;
}

struct GridLine {
  double2 w0;
  cd d;
  double tol;
};

__device__ __forceinline__ GridLine grid_line(const double2* __restrict__ omega, int n_w) {
  const double2 a = omega[0], b = omega[n_w - 1];
  GridLine g;
  g.w0 = a;
  g.d = n_w > 1 ? mk((b.x - a.x) / (n_w - 1), (b.y - a.y) / (n_w - 1)) : mk(0.0, 0.0);
  g.tol = kUniformTol * fmax(fmax(fabs(a.x), fabs(a.y)), fmax(fabs(b.x), fabs(b.y)));
  return g;
}

// Phase factors of one frequency from the table (same a(l) / b(l) interface as PhaseDirect).
struct PhaseTable {
  const cd* tab;  // [2 (L - 1)][entries]: phase 2 l (P) and 2 l + 1 (S) of layer l
  int entries, lo, mid, hi;
  __device__ __forceinline__ cd at(int id) const {
    const cd* q = tab + id * entries;
    return (q[hi] * q[mid]) * q[lo];
  }
  __device__ __forceinline__ cd a(int l) const { return at(2 * l); }
  __device__ __forceinline__ cd b(int l) const { return at(2 * l + 1); }
  __device__ __forceinline__ bool cheap() const { return true; }
};

// Either source, chosen per block (a uniform branch), so that callers compile once.
struct PhaseAuto {
  bool tab;
  PhaseTable t;
  PhaseDirect d;
  __device__ __forceinline__ cd a(int l) const { return tab ? t.a(l) : d.a(l); }
  __device__ __forceinline__ cd b(int l) const { return tab ? t.b(l) : d.b(l); }
  __device__ __forceinline__ bool cheap() const { return tab; }
};

// The same factors with the per-tile products hi[u] * mid[m] formed once per tile
// (phase_hm_warp): one complex product per lookup instead of two, the same roundings in the
// same order, so the values are bit-identical to PhaseTable's.  A warp's 32 consecutive
// frequencies use two mid entries, so each warp forms its own products (no block barrier).
struct PhaseTableHM {
  const cd* tab;
  const cd* hm;  // [2 (L - 1)][2] products of the warp's current tile
  int entries, lo, m;  // m: which of the warp's two mid entries
  __device__ __forceinline__ cd at(int id) const {
    return hm[2 * id + m] * tab[id * entries + lo];
  }
  __device__ __forceinline__ cd a(int l) const { return at(2 * l); }
  __device__ __forceinline__ cd b(int l) const { return at(2 * l + 1); }
};

// Warp-cooperative: s_hm[2 id + k] = hi[hi_entry] * mid[m0 + k] (k = 0, 1) for the n_phase
// phases, followed by __syncwarp.
__device__ __forceinline__ void phase_hm_warp(const cd* s_ph, int entries, int n_phase,
                                              int hi_entry, int m0, cd* s_hm) {
  for (int e = threadIdx.x & 31; e < 2 * n_phase; e += 32) {
    const cd* q = s_ph + (e >> 1) * entries;
    s_hm[e] = q[hi_entry] * q[kPhLo + m0 + (e & 1)];
  }
  __syncwarp();
}

__device__ __forceinline__ PhaseTable phase_at(const cd* s_ph, int entries, int k, int u0) {
  const int t = k & (kPhTile - 1);
  return PhaseTable{s_ph, entries, t & (kPhLo - 1), kPhLo + (t >> 4), kPhHead + (k >> 7) - u0};
}

// Block-cooperative: checks tiles [u0, u0 + n_tiles) (n_tiles <= kPhMaxTiles) against the
// grid line, fills the table for the model's 2 (L - 1) phases and returns the mask of tiles
// that use it (bit u - u0).  `s_bad` is one shared word; the caller guarantees no thread
// still reads it from a previous use.  Contains block barriers; all threads must call it.
__device__ inline unsigned build_phase_table(const double2* __restrict__ omega, int n_w,
                                      const GridLine& g, int u0, int n_tiles, int entries,
                                      int n_layers, const LayerP* lay, cd* s_ph,
                                      unsigned* s_bad) {
  if (threadIdx.x == 0) *s_bad = 0u;
  __syncthreads();
  unsigned bad = 0u;
  const int k_end = min(n_w, (u0 + n_tiles) * kPhTile);
  for (int k = u0 * kPhTile + threadIdx.x; k < k_end; k += blockDim.x) {
    const double2 w = omega[k];
    const double m = (double)k;
    const bool ok = fabs(w.x - fma(m, g.d.x, g.w0.x)) <= g.tol &&
                    fabs(w.y - fma(m, g.d.y, g.w0.y)) <= g.tol;
    if (!ok) bad |= 1u << ((k >> 7) - u0);
  }
  const int n_ent = 2 * (n_layers - 1) * entries;
  for (int e = threadIdx.x; e < n_ent; e += blockDim.x) {
    const int id = e / entries, j = e - id * entries;
    const LayerP& lp = lay[id >> 1];
    const cd c = (id & 1) ? lp.cb : lp.ca;
    cd z;
    unsigned bit;
    if (j < kPhLo) {
      z = (double)j * g.d;
      bit = 1u << 31;
    } else if (j < kPhHead) {
      z = (double)((j - kPhLo) * kPhLo) * g.d;
      bit = 1u << 31;
    } else {
      const int u = u0 + (j - kPhHead);
      if (j - kPhHead >= n_tiles) {
        s_ph[e] = mk(0.0, 0.0);
        continue;
      }
      const double2 ws = omega[u * kPhTile];
      z = mk(ws.x, ws.y);
      bit = 1u << (u - u0);
    }
    const cd v = cexp_(z * c);
    if (!(fabs(v.x) <= kPhMaxMag && fabs(v.y) <= kPhMaxMag)) bad |= bit;
    s_ph[e] = v;
  }
  if (bad) atomicOr(s_bad, bad);
  __syncthreads();
  const unsigned b = *s_bad;
  return (b >> 31) ? 0u : ~b;
}

// The same table built in two block-cooperative pieces, for kernels that hold the hi entries
// of one or two tiles at a time (kPhHead + slots entries per phase): build_phase_lomid fills
// the lo and mid entries of every phase and returns whether all of them are usable;
// phase_hi_tile fills tile u's hi entry in hi slot `slot` and returns whether tile u uses
// the table.  Every entry and every decision is formed exactly as build_phase_table forms it,
// so the phase factors are bit-identical to it.  Each contains a block barrier and reads
// omega / lay only; all threads must call them.
__device__ inline bool build_phase_lomid(const GridLine& g, int entries, int n_layers,
                                         const LayerP* lay, cd* s_ph) {
  bool bad = false;
  const int n_phase = 2 * (n_layers - 1);
  for (int e = threadIdx.x; e < n_phase * kPhHead; e += blockDim.x) {
    const int id = e / kPhHead, j = e - id * kPhHead;
    const LayerP& lp = lay[id >> 1];
    const cd c = (id & 1) ? lp.cb : lp.ca;
    const cd z = j < kPhLo ? (double)j * g.d : (double)((j - kPhLo) * kPhLo) * g.d;
    const cd v = cexp_(z * c);
    if (!(fabs(v.x) <= kPhMaxMag && fabs(v.y) <= kPhMaxMag)) bad = true;
    s_ph[id * entries + j] = v;
  }
  return __syncthreads_or(bad) == 0;
}

__device__ inline bool phase_hi_tile(const double2* __restrict__ omega, int n_w,
                                     const GridLine& g, int u, int slot, int entries,
                                     int n_layers, const LayerP* lay, cd* s_ph) {
  bool bad = false;
  const int k_end = min(n_w, (u + 1) * kPhTile);
  for (int k = u * kPhTile + threadIdx.x; k < k_end; k += blockDim.x) {
    const double2 w = omega[k];
    const double m = (double)k;
    const bool ok = fabs(w.x - fma(m, g.d.x, g.w0.x)) <= g.tol &&
                    fabs(w.y - fma(m, g.d.y, g.w0.y)) <= g.tol;
    if (!ok) bad = true;
  }
  const int n_phase = 2 * (n_layers - 1);
  const double2 ws = omega[u * kPhTile];
  for (int id = threadIdx.x; id < n_phase; id += blockDim.x) {
    const LayerP& lp = lay[id >> 1];
    const cd c = (id & 1) ? lp.cb : lp.ca;
    const cd v = cexp_(mk(ws.x, ws.y) * c);
    if (!(fabs(v.x) <= kPhMaxMag && fabs(v.y) <= kPhMaxMag)) bad = true;
    s_ph[id * entries + kPhHead + slot] = v;
  }
  return __syncthreads_or(bad) == 0;
}

}  // namespace kr
