// Fused forward reflectivity kernel: one thread per (omega, p), one slowness per block.
//
// Block prologue: layer slownesses and the interface coefficients of this block's slowness
// go to shared memory (computed once per block, read as broadcasts).  Each thread then runs
// the whole bottom-up Kennett sweep for its frequency with the cumulative reflection
// matrix in registers, applies the ocean phase / free-surface operator and writes
// R[p][omega] (coalesced along omega).  FP64 CUDA cores; no tensor-core work exists here
// (2x2 complex algebra per thread is not a contraction).
#include <stdlib.h>

#include "kr_phase.cuh"

namespace kr {

constexpr int kFwdThreads = 128;

// Phase factors come from a per-block table (kr_phase.cuh) for the block's frequency tiles
// when the grid is uniform, from direct exponentials otherwise.
constexpr int kTabTiles = kFwdTabTiles;  // frequency tiles per block on the table path
static_assert(kFwdThreads == kPhTile, "one forward tile is one phase-table tile");

// Bytes of the per-warp products hi * mid of the current tile (PhaseTableHM).
constexpr int kFwdWarps = kFwdThreads / 32;
inline size_t phase_hm_bytes(int n_layers) {
  return sizeof(cd) * (size_t)kFwdWarps * 2 * 2 * (size_t)(n_layers - 1);
}

template <int MINB>
__global__ void __launch_bounds__(kFwdThreads, MINB)
reflectivity_kernel(const double* __restrict__ tab, int n_layers, const double* __restrict__ p,
                    int n_p, const double2* __restrict__ omega, int n_w, int n_wtiles,
                    int tiles_per_block, int free_surface, int use_table, int use_hm,
                    double2* __restrict__ R) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned s_bad;
  LayerP* s_layer = reinterpret_cast<LayerP*>(smem);
  Iface* s_iface = reinterpret_cast<Iface*>(smem + sizeof(LayerP) * n_layers);
  cd* s_ph = reinterpret_cast<cd*>(smem + prologue_smem_bytes(n_layers));
  const int n_phase = 2 * (n_layers - 1);
  cd* s_hm = reinterpret_cast<cd*>(smem + prologue_smem_bytes(n_layers) +
                                   phase_table_bytes(n_layers, kTabTiles));
  const int groups = (n_wtiles + tiles_per_block - 1) / tiles_per_block;
  const int ip = blockIdx.x / groups;
  const int t0 = (blockIdx.x % groups) * tiles_per_block;
  const int t1 = min(n_wtiles, t0 + tiles_per_block);
  block_prologue(tab, n_layers, p[ip], s_layer, s_iface);
  unsigned mask = 0u;
  const int entries = phase_entries(kTabTiles);
  if (use_table)
    mask = build_phase_table(omega, n_w, grid_line(omega, n_w), t0, t1 - t0, entries,
                             n_layers, s_layer, s_ph, &s_bad);
  const bool fs = free_surface != 0;
  double2* Rp = R + (size_t)ip * n_w;
  if (use_table && use_hm) {
    // per-tile products hi * mid, formed by each warp for its own two mid entries: the tile
    // loop has no block barrier, so the warps drift apart and hide each other's latencies
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lo = lane & (kPhLo - 1), m = lane >> 4;
    cd* hmw = s_hm + warp * 2 * n_phase;
    for (int t = t0; t < t1; ++t) {
      const int iw = t * kFwdThreads + threadIdx.x;
      const bool tab_tile = (mask >> (t - t0)) & 1u;
      if (tab_tile) phase_hm_warp(s_ph, entries, n_phase, kPhHead + t - t0, 2 * warp, hmw);
      if (iw < n_w) {
        cd e0, rpp;
        if (tab_tile) {
          rpp = sweep_ph(n_layers, s_iface, PhaseTableHM{s_ph, hmw, entries, lo, m}, &e0);
        } else {
          const double2 wv = omega[iw];
          rpp = sweep(mk(wv.x, wv.y), n_layers, s_layer, s_iface, &e0);
        }
        const cd out = pp_surface(rpp, e0, fs);
        Rp[iw] = make_double2(out.x, out.y);
      }
      __syncwarp();  // the warp's products are read before the next tile's overwrite them
    }
    return;
  }
  for (int t = t0; t < t1; ++t) {
    const int iw = t * kFwdThreads + threadIdx.x;
    if (iw >= n_w) break;
    cd e0, rpp;
    if ((mask >> (t - t0)) & 1u) {
      rpp = sweep_ph(n_layers, s_iface, phase_at(s_ph, entries, iw, t0), &e0);
    } else {
      const double2 wv = omega[iw];
      rpp = sweep(mk(wv.x, wv.y), n_layers, s_layer, s_iface, &e0);
    }
    const cd out = pp_surface(rpp, e0, fs);
    Rp[iw] = make_double2(out.x, out.y);
  }
}

// Frequency tiles one block sweeps after its prologue: enough to amortise the prologue
// (the block's threads wait at its barrier while ~L of them compute coefficients) while
// keeping at least ~8 waves of blocks on 148 SMs.
static int tiles_per_block(long long n_p, int n_wtiles) {
  const long long target_blocks = 148LL * 6 * 8;
  long long t = (n_p * n_wtiles) / target_blocks;
  if (t < 1) t = 1;
  if (t > n_wtiles) t = n_wtiles;
  return (int)t;
}

// Register budget of the forward kernel: blocks of 128 threads resident per SM the compiler
// must allow (4 -> 128 registers, 5 -> 96, 6 -> 80).  Set by kr_set_forward_variant or the
// KR_FWD_MINB environment variable; otherwise 5 for models on the phase-table path (21-layer
// gather grid: 3.34 ms at 5, 3.45 ms at 4, 3.37 ms at 6) and 4 for direct phases, whose
// exponentials need the registers.
static int g_fwd_minb = -1;  // -1: not read yet, 0: automatic

static int forward_minb(bool table) {
  if (g_fwd_minb < 0) {
    const char* e = getenv("KR_FWD_MINB");
    const int v = e ? atoi(e) : 0;
    g_fwd_minb = (v >= 4 && v <= 6) ? v : 0;
  }
  if (g_fwd_minb > 0) return g_fwd_minb;
  return table ? 5 : 4;
}

template <int MINB>
static kr_status launch_forward(const double* layers, int n_layers, const double* p, int n_p,
                                const double* omega, int n_w, int n_wtiles, uint32_t flags,
                                double* R, cudaStream_t st) {
  size_t smem = prologue_smem_bytes(n_layers);
  int tpb = tiles_per_block(n_p, n_wtiles);
  const bool table = phase_table_model(n_layers);  // <= 50 KB: 4 blocks of 128 per SM
  bool hm = false;
  if (table) {
    smem += phase_table_bytes(n_layers, kTabTiles);
    tpb = tpb < kTabTiles ? tpb : kTabTiles;
    // the per-tile products only where they keep the block within the same budget
    hm = smem + phase_hm_bytes(n_layers) <= kFwdTabSmemMax;
    if (hm) smem += phase_hm_bytes(n_layers);
  }
  const long long blocks = (long long)n_p * ((n_wtiles + tpb - 1) / tpb);
  if (blocks > 0x7fffffffLL) return KR_ERR_TOO_LARGE;
  static SmemLimit lim;
  if (smem > 48 * 1024) {
    const kr_status a = raise_smem_limit((const void*)reflectivity_kernel<MINB>, smem, lim,
                                         "kr_reflectivity: smem attribute");
    if (a != KR_OK) return a;
  }
  reflectivity_kernel<MINB><<<(unsigned)blocks, kFwdThreads, smem, st>>>(
      layers, n_layers, p, n_p, reinterpret_cast<const double2*>(omega), n_w, n_wtiles, tpb,
      (flags & KR_FREE_SURFACE) ? 1 : 0, table ? 1 : 0, hm ? 1 : 0,
      reinterpret_cast<double2*>(R));
  return check_launch("kr_reflectivity");
}

}  // namespace kr

using namespace kr;

extern "C" void kr_set_forward_variant(int32_t min_blocks_per_sm) {
  g_fwd_minb = (min_blocks_per_sm >= 4 && min_blocks_per_sm <= 6) ? min_blocks_per_sm : 0;
}

extern "C" kr_status kr_reflectivity(const double* layers, int32_t n_layers, const double* p,
                                     int32_t n_p, const double* omega, int32_t n_w,
                                     uint32_t flags, double* R, void* stream) {
  if (n_p < 0 || n_w < 0 || (flags & ~KR_FREE_SURFACE)) return KR_ERR_INVALID_ARGUMENT;
  if (n_layers < 2) return KR_ERR_INVALID_MODEL;
  if (n_layers > kMaxLayers) return KR_ERR_TOO_LARGE;
  if (n_p == 0 || n_w == 0) return KR_OK;
  if (!layers || !p || !omega || !R) return KR_ERR_INVALID_ARGUMENT;
  if (!aligned16(omega) || !aligned16(R)) return KR_ERR_INVALID_ARGUMENT;
  const int n_wtiles = (n_w + kFwdThreads - 1) / kFwdThreads;
  cudaStream_t st = (cudaStream_t)stream;
  switch (forward_minb(phase_table_model(n_layers))) {
    case 6:
      return launch_forward<6>(layers, n_layers, p, n_p, omega, n_w, n_wtiles, flags, R, st);
    case 5:
      return launch_forward<5>(layers, n_layers, p, n_p, omega, n_w, n_wtiles, flags, R, st);
    default:
      return launch_forward<4>(layers, n_layers, p, n_p, omega, n_w, n_wtiles, flags, R, st);
  }
}
