// Batched evaluation of many earth models of uneven size in persistent launches.
//
// A batch is a list of models, each with its own layer count, slowness grid and frequency
// grid, asking for the forward reflectivity or forward + misfit gradient.  kr_batch_plan
// (host) builds, once per batch shape:
//   * a pair table: one entry per (model, slowness) with the offset of its coefficient block
//     in the plan buffer;
//   * two work lists (forward items, gradient items), item = (pair, first frequency, count),
//     sorted by descending cost (layers x frequencies, x4 for gradients) so the dynamic
//     scheduler hands out the longest items first (LPT);
// and uploads them into the caller's plan buffer.  kr_batch_launch (device only, capturable
// in a CUDA graph) then runs:
//   1. batch_prep_kernel: one block per pair -> layer terms and interface coefficients (and,
//      for gradient models, layer derivative factors) into the plan;
//   2. batch_tan_kernel: the gradient models' coefficient tangents, one thread per interface
//      and tangent column, alongside the forward kernel (its programmatic dependent);
//   3. batch_forward_kernel and batch_grad_sums_kernel (batch_gradient_kernel where a model's
//      frequency sums exceed shared memory): persistent grids (resident blocks only) that
//      pull items with an atomic counter until the list is exhausted.
// Gradient items reduce their contributions per block in a fixed order and add them to the
// model's chi_grad with FP64 atomics (the order of those additions across blocks is not
// fixed: results agree to rounding, ~1e-16 relative, run to run).
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "kr_adjoint.cuh"
#include "kr_adjsum.cuh"
#include "kr_internal.cuh"
#include "kr_phase.cuh"

namespace kr {

struct PairRec {
  int32_t model;
  int32_t j;
  int64_t coef_off;  // bytes into the plan buffer
};

struct ItemRec {
  int32_t pair;
  int32_t w0;
  int32_t nw;
  int32_t pad;
};

struct PlanHeader {
  int32_t n_models, n_pairs, n_fwd, n_grad;
  int32_t threads, tile_w, grid_fwd, grid_grad;
  int64_t off_models, off_pairs, off_fwd, off_grad, total_bytes;
  int32_t counters[4];  // [0] forward item counter, [1] gradient item counter
};

__host__ __device__ inline size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

static size_t pair_bytes(const kr_model_desc& d) {
  const int L = d.n_layers, I = d.n_layers - 1;
  size_t b = a256(sizeof(LayerP) * L) + a256(sizeof(Iface) * I);
  if (d.flags & KR_BATCH_GRADIENT) b += a256(sizeof(LayerD) * L) + a256(sizeof(ScatTan) * I);
  return b;
}

struct PairView {
  const LayerP* lay;
  const Iface* coef;
  const LayerD* dlay;
  const ScatTan* tan;
};

__device__ __forceinline__ PairView pair_view(const unsigned char* plan, const PairRec& pr,
                                              const kr_model_desc& d) {
  const int L = d.n_layers, I = d.n_layers - 1;
  const unsigned char* b = plan + pr.coef_off;
  PairView v;
  v.lay = reinterpret_cast<const LayerP*>(b);
  b += a256(sizeof(LayerP) * L);
  v.coef = reinterpret_cast<const Iface*>(b);
  b += a256(sizeof(Iface) * I);
  v.dlay = reinterpret_cast<const LayerD*>(b);
  b += a256(sizeof(LayerD) * L);
  v.tan = reinterpret_cast<const ScatTan*>(b);
  return v;
}

__global__ void batch_prep_kernel(unsigned char* plan, const double* __restrict__ layers,
                                  const double* __restrict__ p_all) {
  const PlanHeader* h = reinterpret_cast<const PlanHeader*>(plan);
  const kr_model_desc* models = reinterpret_cast<const kr_model_desc*>(plan + h->off_models);
  const PairRec* pairs = reinterpret_cast<const PairRec*>(plan + h->off_pairs);
  for (int q = blockIdx.x; q < h->n_pairs; q += gridDim.x) {
    const PairRec pr = pairs[q];
    const kr_model_desc d = models[pr.model];
    const int L = d.n_layers, I = L - 1;
    const double* tab = layers + d.layers_off;
    const double pj = p_all[d.p_off + pr.j];
    unsigned char* b = plan + pr.coef_off;
    LayerP* lay = reinterpret_cast<LayerP*>(b);
    b += a256(sizeof(LayerP) * L);
    Iface* coef = reinterpret_cast<Iface*>(b);
    b += a256(sizeof(Iface) * I);
    LayerD* dlay = reinterpret_cast<LayerD*>(b);
    const bool grad = (d.flags & KR_BATCH_GRADIENT) != 0;
    for (int l = threadIdx.x; l < L; l += blockDim.x) {
      lay[l] = layer_terms(tab, L, l, pj);
      if (grad) dlay[l] = layer_derivs(tab, L, l, pj, lay[l]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < I; i += blockDim.x)
      coef[i] = interface_coeffs(pj, i, lay[i], lay[i + 1]);
    __syncthreads();
  }
}

// Coefficient tangents of the gradient models' pairs, one thread per (interface, tangent
// column), from the layer terms and derivative factors batch_prep_kernel left in the plan.
// Only the gradient kernel reads them, so the forward kernel is launched as this kernel's
// programmatic dependent (released on entry) and runs alongside it; the forward kernel
// waits for this grid before it exits, so the gradient kernel after it sees the tangents.
__global__ void __launch_bounds__(64)
batch_tan_kernel(unsigned char* plan, const double* __restrict__ p_all) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const PlanHeader* h = reinterpret_cast<const PlanHeader*>(plan);
  const kr_model_desc* models = reinterpret_cast<const kr_model_desc*>(plan + h->off_models);
  const PairRec* pairs = reinterpret_cast<const PairRec*>(plan + h->off_pairs);
  for (int q = blockIdx.x; q < h->n_pairs; q += gridDim.x) {
    const PairRec pr = pairs[q];
    const kr_model_desc d = models[pr.model];
    if (!(d.flags & KR_BATCH_GRADIENT)) continue;
    const int L = d.n_layers, I = L - 1;
    const double pj = p_all[d.p_off + pr.j];
    unsigned char* b = plan + pr.coef_off;
    const LayerP* lay = reinterpret_cast<const LayerP*>(b);
    b += a256(sizeof(LayerP) * L) + a256(sizeof(Iface) * I);
    const LayerD* dlay = reinterpret_cast<const LayerD*>(b);
    b += a256(sizeof(LayerD) * L);
    ScatTan* tan = reinterpret_cast<ScatTan*>(b);
    for (int t = threadIdx.x; t < 6 * I; t += blockDim.x) {
      const int i = t / 6, col = t % 6;
      cd c[10];
      interface_tangent_col(pj, i, lay[i], dlay[i], lay[i + 1], dlay[i + 1], col, c);
      for (int k = 0; k < 10; ++k) tan[i].t[k][col] = c[k];
    }
  }
}

// Zeroes chi_grad of gradient models and the item counters (first node of a launch).
__global__ void batch_reset_kernel(unsigned char* plan, double* chi_grad) {
  PlanHeader* h = reinterpret_cast<PlanHeader*>(plan);
  const kr_model_desc* models = reinterpret_cast<const kr_model_desc*>(plan + h->off_models);
  if (blockIdx.x == 0 && threadIdx.x < 4) h->counters[threadIdx.x] = 0;
  for (int b = blockIdx.x; b < h->n_models; b += gridDim.x) {
    const kr_model_desc d = models[b];
    if (!(d.flags & KR_BATCH_GRADIENT)) continue;
    for (int k = threadIdx.x; k < 4 * d.n_layers + 1; k += blockDim.x) chi_grad[d.grad_off + k] = 0.0;
  }
}

__device__ __forceinline__ int next_item(int* counter) {
  __shared__ int s_item;
  __syncthreads();
  if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
  __syncthreads();
  return s_item;
}

// Forward items: one (model, slowness) pair and a frequency range [w0, w0 + nw).  With
// tab_entries > 0 (kPhHead + 2: lo, mid and two hi slots) models that tabulate take their
// phase factors from a table holding one tile's hi entry at a time (kr_phase.cuh; same
// entries and decisions as kr_reflectivity, so the results are bit-identical to a per-model
// call): ~37 KB of shared memory for the deepest such model, six blocks per SM.
template <int THREADS>
__global__ void __launch_bounds__(THREADS)
batch_forward_kernel(unsigned char* plan, const double2* __restrict__ omega_all,
                     double2* __restrict__ R_all, int tab_entries) {
  extern __shared__ __align__(16) unsigned char s_pair[];  // layer terms + coefficients + table
  PlanHeader* h = reinterpret_cast<PlanHeader*>(plan);
  const kr_model_desc* models = reinterpret_cast<const kr_model_desc*>(plan + h->off_models);
  const PairRec* pairs = reinterpret_cast<const PairRec*>(plan + h->off_pairs);
  const ItemRec* items = reinterpret_cast<const ItemRec*>(plan + h->off_fwd);
  const int n_items = h->n_fwd;
  for (;;) {
    const int it = next_item(&h->counters[0]);
    if (it >= n_items) break;
    const ItemRec item = items[it];
    const PairRec pr = pairs[item.pair];
    const kr_model_desc d = models[pr.model];
    const PairView v = pair_view(plan, pr, d);
    const bool fs = (d.flags & KR_FREE_SURFACE) != 0;
    LayerP* lay = reinterpret_cast<LayerP*>(s_pair);
    Iface* coef = reinterpret_cast<Iface*>(s_pair + sizeof(LayerP) * d.n_layers);
    cd* s_ph = reinterpret_cast<cd*>(s_pair + prologue_smem_bytes(d.n_layers));
    copy16(lay, v.lay, sizeof(LayerP) * d.n_layers);
    copy16(coef, v.coef, sizeof(Iface) * (d.n_layers - 1));
    __syncthreads();
    const double2* om = omega_all + d.omega_off;
    const GridLine g = grid_line(om, d.n_w);
    // block-uniform conditions: every thread takes the same branches through the barriers
    const bool tab = tab_entries > 0 && phase_table_model(d.n_layers);
    const bool lomid = tab && build_phase_lomid(g, tab_entries, d.n_layers, lay, s_ph);
    const int u_end = (item.w0 + item.nw - 1) / kPhTile;
    for (int u = item.w0 / kPhTile; u <= u_end; ++u) {
      // tile u's hi entry goes to slot u & 1, last read by tile u - 2, whose readers passed
      // the barrier inside phase_hi_tile for tile u - 1
      const bool tile_tab =
          lomid && phase_hi_tile(om, d.n_w, g, u, u & 1, tab_entries, d.n_layers, lay, s_ph);
      const int k_lo = max(item.w0, u * kPhTile);
      const int k_hi = min(item.w0 + item.nw, (u + 1) * kPhTile);
      for (int iw = k_lo + threadIdx.x; iw < k_hi; iw += THREADS) {
        cd e0, rpp;
        if (tile_tab) {
          rpp = sweep_ph(d.n_layers, coef, phase_at(s_ph, tab_entries, iw, u - (u & 1)), &e0);
        } else {
          const double2 wv = om[iw];
          rpp = sweep(mk(wv.x, wv.y), d.n_layers, lay, coef, &e0);
        }
        const cd out = pp_surface(rpp, e0, fs);
        R_all[d.R_off + (size_t)pr.j * d.n_w + iw] = make_double2(out.x, out.y);
      }
    }
  }
  // launched as batch_tan_kernel's programmatic dependent: this grid completes only after
  // that one has, so the gradient kernel launched after it reads finished tangents
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Per-thread sink for gradient items: 2 Re(conj(res) dR/dtheta) per layer, reduced over the
// warp by shuffles into the warp's own accumulator row (no block barrier inside the sweep).
template <int THREADS>
struct BatchGradSink {
  typedef AccR AccT;  // reverse sweep seeded with 2 conj(res): real contributions only
  static constexpr bool kSeeded = true;
  bool valid;
  cd res;
  const double2* obs;
  double2* R_out;
  double* row;  // this warp's [4L + 1] accumulators
  int L;
  __device__ cd reflectivity(cd R) {
    res = mk(0.0, 0.0);
    if (!valid) return mk(0.0, 0.0);
    if (R_out) *R_out = make_double2(R.x, R.y);
    const double2 o = *obs;
    res = mk(R.x - o.x, R.y - o.y);
    return mk(2.0 * res.x, -2.0 * res.y);  // 2 conj(res)
  }
  __device__ void layer(int l, const AccR& a) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (valid) {
      v[0] = a.a;
      v[1] = a.b;
      v[2] = a.r;
      v[3] = a.h;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0)
      for (int k = 0; k < 4; ++k) row[k * L + l] += v[k];
  }
};

template <int THREADS>
__global__ void __launch_bounds__(THREADS)
batch_gradient_kernel(unsigned char* plan, const double2* __restrict__ omega_all,
                      const double2* __restrict__ obs_all, double2* __restrict__ R_all,
                      double* __restrict__ chi_grad, int stage, int tab_entries) {
  // [THREADS / 32][4L + 1] accumulators (padded to 16 bytes), then the item's slowness data,
  // then (tab_entries > 0, models that tabulate) the phase table of the item's tiles
  extern __shared__ __align__(16) double s_wacc[];
  __shared__ unsigned s_bad;
  PlanHeader* h = reinterpret_cast<PlanHeader*>(plan);
  const kr_model_desc* models = reinterpret_cast<const kr_model_desc*>(plan + h->off_models);
  const PairRec* pairs = reinterpret_cast<const PairRec*>(plan + h->off_pairs);
  const ItemRec* items = reinterpret_cast<const ItemRec*>(plan + h->off_grad);
  const int n_items = h->n_grad;
  for (;;) {
    const int it = next_item(&h->counters[1]);
    if (it >= n_items) break;
    const ItemRec item = items[it];
    const PairRec pr = pairs[item.pair];
    const kr_model_desc d = models[pr.model];
    PairView v = pair_view(plan, pr, d);
    const int L = d.n_layers;
    const int nv = 4 * L + 1;
    for (int k = threadIdx.x; k < (THREADS / 32) * nv; k += THREADS) s_wacc[k] = 0.0;
    if (stage) {
      unsigned char* b = reinterpret_cast<unsigned char*>(s_wacc + ((THREADS / 32) * nv + 1) / 2 * 2);
      ScatTan* st = reinterpret_cast<ScatTan*>(b);
      Iface* sc = reinterpret_cast<Iface*>(b + sizeof(ScatTan) * (L - 1));
      LayerP* sl = reinterpret_cast<LayerP*>(b + (sizeof(ScatTan) + sizeof(Iface)) * (L - 1));
      LayerD* sd = reinterpret_cast<LayerD*>(reinterpret_cast<unsigned char*>(sl) +
                                             sizeof(LayerP) * L);
      copy16(st, v.tan, sizeof(ScatTan) * (L - 1));
      copy16(sc, v.coef, sizeof(Iface) * (L - 1));
      copy16(sl, v.lay, sizeof(LayerP) * L);
      copy16(sd, v.dlay, sizeof(LayerD) * L);
      v.tan = st;
      v.coef = sc;
      v.lay = sl;
      v.dlay = sd;
    }
    __syncthreads();
    const double2* om = omega_all + d.omega_off;
    const int u0 = item.w0 / kPhTile;
    cd* s_ph = reinterpret_cast<cd*>(
        reinterpret_cast<unsigned char*>(s_wacc + ((THREADS / 32) * nv + 1) / 2 * 2) +
        pair_smem_bytes(L));
    unsigned mask = 0u;
    if (stage && tab_entries > 0 && phase_table_model(L))
      mask = build_phase_table(om, d.n_w, grid_line(om, d.n_w), u0,
                               (item.w0 + item.nw - 1) / kPhTile - u0 + 1, tab_entries, L,
                               v.lay, s_ph, &s_bad);
    double* row = s_wacc + (threadIdx.x >> 5) * nv;
    const int seg = checkpoint_spacing(L - 2 > 0 ? L - 2 : 1);
    const bool fs = (d.flags & KR_FREE_SURFACE) != 0;
    for (int k0 = 0; k0 < item.nw; k0 += THREADS) {
      const int iw = item.w0 + k0 + threadIdx.x;
      const bool valid = k0 + threadIdx.x < item.nw;
      cd w = mk(0.0, 0.0);
      if (valid) {
        const double2 wv = omega_all[d.omega_off + iw];
        w = mk(wv.x, wv.y);
      }
      BatchGradSink<THREADS> sink;
      sink.valid = valid;
      sink.L = L;
      sink.row = row;
      const size_t e = (size_t)pr.j * d.n_w + (valid ? iw : 0);
      sink.obs = obs_all + d.obs_off + e;
      sink.R_out = (d.flags & KR_BATCH_STORE_R) ? R_all + d.R_off + e : nullptr;
      const int iwt = valid ? iw : item.w0;
      const PhaseAuto ph{((mask >> (iwt / kPhTile - u0)) & 1u) != 0,
                         phase_at(s_ph, tab_entries, iwt, u0), PhaseDirect{w, v.lay}};
      jacobian_pair(L, w, fs, seg, v.lay, v.dlay, v.coef, v.tan, ph, sink);
      double c2 = valid ? (sink.res.x * sink.res.x + sink.res.y * sink.res.y) : 0.0;
      for (int o = 16; o > 0; o >>= 1) c2 += __shfl_down_sync(0xffffffffu, c2, o);
      if ((threadIdx.x & 31) == 0) row[4 * L] += c2;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nv; k += THREADS) {
      double t = 0.0;
      for (int wi = 0; wi < THREADS / 32; ++wi) t += s_wacc[wi * nv + k];
      atomicAdd(chi_grad + d.grad_off + k, t);
    }
  }
}

// Gradient items with the contraction moved out of the frequency loop (kr_adjsum.cuh): the
// block's warps sum the per-step adjoints of every frequency of the item, then contract once
// per (pair, interface).  Dynamic smem: per-warp sum rows (sized for max_layers) and staging
// tiles (which then hold the item's [4L] result), then the item's interface coefficients and
// layer terms and (models that tabulate) the phase table of its tiles.  Register budget: 256 threads per SM
// (its shared memory admits two 128-thread blocks per SM; a 168-register cap only spills).
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 256 / THREADS)
batch_grad_sums_kernel(unsigned char* plan, const double2* __restrict__ omega_all,
                       const double2* __restrict__ obs_all, double2* __restrict__ R_all,
                       double* __restrict__ chi_grad, int max_layers, int tab_entries) {
  constexpr int W = THREADS / 32;
  extern __shared__ __align__(16) double s_raw[];
  __shared__ unsigned s_bad;
  __shared__ double s_chi[W];
  PlanHeader* h = reinterpret_cast<PlanHeader*>(plan);
  const kr_model_desc* models = reinterpret_cast<const kr_model_desc*>(plan + h->off_models);
  const PairRec* pairs = reinterpret_cast<const PairRec*>(plan + h->off_pairs);
  const ItemRec* items = reinterpret_cast<const ItemRec*>(plan + h->off_grad);
  const int n_items = h->n_grad;
  const int warp = threadIdx.x >> 5;
  constexpr int RS = 2;  // two staging rounds: half the tile, two blocks per SM
  cd* acc = reinterpret_cast<cd*>(s_raw);
  cd* stage = acc + (size_t)W * sum_rows(max_layers) * kSumVals;
  // the item's [4L] result reuses the staging tiles once the sweeps are done
  double* s_out = reinterpret_cast<double*>(stage);
  unsigned char* area = reinterpret_cast<unsigned char*>(stage + W * 32 * stage_stride<RS>());
  for (;;) {
    const int it = next_item(&h->counters[1]);
    if (it >= n_items) break;
    const ItemRec item = items[it];
    const PairRec pr = pairs[item.pair];
    const kr_model_desc d = models[pr.model];
    const PairView v = pair_view(plan, pr, d);
    const int L = d.n_layers, I = L - 1;
    Iface* sc = reinterpret_cast<Iface*>(area);
    LayerP* sl = reinterpret_cast<LayerP*>(area + sizeof(Iface) * I);
    cd* s_ph = reinterpret_cast<cd*>(area + prologue_smem_bytes(L));
    sums_zero(acc, L, W);
    copy16(sc, v.coef, sizeof(Iface) * I);
    copy16(sl, v.lay, sizeof(LayerP) * L);
    __syncthreads();
    const double2* om = omega_all + d.omega_off;
    const int u0 = item.w0 / kPhTile;
    unsigned mask = 0u;
    if (tab_entries > 0 && phase_table_model(L))
      mask = build_phase_table(om, d.n_w, grid_line(om, d.n_w), u0,
                               (item.w0 + item.nw - 1) / kPhTile - u0 + 1, tab_entries, L, sl,
                               s_ph, &s_bad);
    const int seg = checkpoint_spacing(L - 2 > 0 ? L - 2 : 1);
    const bool fs = (d.flags & KR_FREE_SURFACE) != 0;
    double c2 = 0.0;
    for (int k0 = 0; k0 < item.nw; k0 += THREADS) {
      const int iw = item.w0 + k0 + threadIdx.x;
      const bool valid = k0 + threadIdx.x < item.nw;
      cd w = mk(0.0, 0.0);
      if (valid) {
        const double2 wv = om[iw];
        w = mk(wv.x, wv.y);
      }
      const size_t e = (size_t)pr.j * d.n_w + (valid ? iw : 0);
      SumSink<RS> sink;
      sink.valid = valid;
      sink.vjp = false;
      sink.obs = obs_all + d.obs_off + e;
      sink.R_out = (d.flags & KR_BATCH_STORE_R) ? R_all + d.R_off + e : nullptr;
      sink.acc = acc + (size_t)warp * L * kSumVals;
      sink.stage = stage + warp * 32 * stage_stride<RS>();
      sink.I = I;
      const int iwt = valid ? iw : item.w0;
      const PhaseAuto ph{((mask >> (iwt / kPhTile - u0)) & 1u) != 0,
                         phase_at(s_ph, tab_entries, iwt, u0), PhaseDirect{w, sl}};
      adjoint_pair_sums(L, w, fs, seg, sc, ph, sink);
      if (valid) c2 += sink.res.x * sink.res.x + sink.res.y * sink.res.y;
    }
    for (int o = 16; o > 0; o >>= 1) c2 += __shfl_down_sync(0xffffffffu, c2, o);
    if ((threadIdx.x & 31) == 0) s_chi[warp] = c2;
    sums_finish(acc, L, W, v.tan, v.dlay, s_out);
    __syncthreads();
    for (int k = threadIdx.x; k < 4 * L; k += THREADS) atomicAdd(chi_grad + d.grad_off + k, s_out[k]);
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int wi = 0; wi < W; ++wi) t += s_chi[wi];
      atomicAdd(chi_grad + d.grad_off + 4 * L, t);
    }
  }
}

static int occupancy_grid(const void* fn, int threads, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return per_sm * sms;
}

static bool valid_config(const kr_batch_config* c) {
  return c && (c->threads == 32 || c->threads == 64 || c->threads == 128) && c->tile_w >= 32 &&
         c->tile_w <= 8192;
}

struct PlanLayout {
  PlanHeader h;
  size_t bytes;
};

static kr_status layout(const kr_model_desc* descs, int n_models, const kr_batch_config* cfg,
                        PlanLayout* out, std::vector<PairRec>* pairs,
                        std::vector<ItemRec>* fwd, std::vector<ItemRec>* grad) {
  PlanHeader h{};
  h.n_models = n_models;
  h.threads = cfg->threads;
  h.tile_w = cfg->tile_w;
  size_t off = a256(sizeof(PlanHeader));
  h.off_models = (int64_t)off;
  off = a256(off + sizeof(kr_model_desc) * (size_t)n_models);
  long long n_pairs = 0;
  for (int b = 0; b < n_models; ++b) {
    const kr_model_desc& d = descs[b];
    if (d.n_layers < 2) return KR_ERR_INVALID_MODEL;
    if (d.n_layers > kMaxLayers) return KR_ERR_TOO_LARGE;
    if (d.n_p < 0 || d.n_w < 0 || (d.flags & ~(KR_FREE_SURFACE | KR_BATCH_GRADIENT |
                                               KR_BATCH_STORE_R)))
      return KR_ERR_INVALID_ARGUMENT;
    n_pairs += d.n_p;
  }
  if (n_pairs > 0x7fffffffLL) return KR_ERR_TOO_LARGE;
  h.n_pairs = (int)n_pairs;
  h.off_pairs = (int64_t)off;
  off = a256(off + sizeof(PairRec) * (size_t)n_pairs);
  // item lists (count first)
  struct Costed {
    double cost;
    ItemRec it;
  };
  std::vector<Costed> cf, cg;
  int q = 0;
  for (int b = 0; b < n_models; ++b) {
    const kr_model_desc& d = descs[b];
    const bool gr = (d.flags & KR_BATCH_GRADIENT) != 0;
    for (int j = 0; j < d.n_p; ++j, ++q) {
      for (int w0 = 0; w0 < d.n_w; w0 += cfg->tile_w) {
        ItemRec it{q, w0, std::min(cfg->tile_w, d.n_w - w0), 0};
        const double cost = (double)(d.n_layers - 1) * it.nw * (gr ? 4.0 : 1.0);
        (gr ? cg : cf).push_back({cost, it});
      }
    }
  }
  auto by_cost = [](const Costed& a, const Costed& b) { return a.cost > b.cost; };
  std::stable_sort(cf.begin(), cf.end(), by_cost);
  std::stable_sort(cg.begin(), cg.end(), by_cost);
  h.n_fwd = (int)cf.size();
  h.n_grad = (int)cg.size();
  h.off_fwd = (int64_t)off;
  off = a256(off + sizeof(ItemRec) * cf.size());
  h.off_grad = (int64_t)off;
  off = a256(off + sizeof(ItemRec) * cg.size());
  if (pairs) {
    pairs->clear();
    pairs->reserve((size_t)n_pairs);
  }
  for (int b = 0; b < n_models; ++b) {
    const size_t pb = pair_bytes(descs[b]);
    for (int j = 0; j < descs[b].n_p; ++j) {
      if (pairs) pairs->push_back(PairRec{b, j, (int64_t)off});
      off += pb;
    }
  }
  h.total_bytes = (int64_t)off;
  if (fwd) {
    fwd->clear();
    for (auto& c : cf) fwd->push_back(c.it);
  }
  if (grad) {
    grad->clear();
    for (auto& c : cg) grad->push_back(c.it);
  }
  out->h = h;
  out->bytes = off;
  return KR_OK;
}

constexpr size_t kBatchStageMax = 160 * 1024;

static size_t fwd_smem(int max_layers) {
  return sizeof(LayerP) * (size_t)max_layers + sizeof(Iface) * (size_t)(max_layers - 1);
}

// Phase-table entries per phase for items of tile_w frequencies (0: direct exponentials for
// every model).  Only models that tabulate in kr_reflectivity (phase_table_model) use the
// table, so the smem reserved is that of the largest such model.
static int fwd_table_entries(int tile_w) {
  const int tiles = (tile_w + kPhTile - 1) / kPhTile + 1;
  return tiles > kPhMaxTiles ? 0 : phase_entries(tiles);
}

// gradient kernel dynamic smem, whether the slowness data is staged, and the phase-table
// entries (0: none).  The table of a model that tabulates (at most phase_table_max_layers()
// layers) sits after that model's own staged data, inside the staging area sized for the
// largest model where it fits.
static size_t grad_smem(int threads, int max_layers, int tab_entries, int* stage, int* tab) {
  const size_t acc = sizeof(double) * (((size_t)(threads / 32) * (4 * max_layers + 1) + 1) / 2 * 2);
  const size_t pair = pair_smem_bytes(max_layers);
  *stage = (acc + pair <= kBatchStageMax) ? 1 : 0;
  *tab = 0;
  if (!*stage) return acc;
  size_t area = pair;
  if (tab_entries > 0) {
    const int lt = std::min(max_layers, phase_table_max_layers());
    const size_t need = pair_smem_bytes(lt) + sizeof(cd) * (size_t)tab_entries * 2 * (lt - 1);
    if (acc + std::max(area, need) <= kBatchStageMax) {
      area = std::max(area, need);
      *tab = tab_entries;
    }
  }
  return acc + area;
}

// Dynamic smem of batch_grad_sums_kernel (0 if it does not fit) and the phase-table entries it
// uses (0: none), for blocks of THREADS threads.
static size_t sums_smem(int threads, int max_layers, int tab_entries, int* tab) {
  size_t area = prologue_smem_bytes(max_layers);
  *tab = 0;
  if (tab_entries > 0) {
    const int lt = std::min(max_layers, phase_table_max_layers());
    area = std::max(area, prologue_smem_bytes(lt) +
                              sizeof(cd) * (size_t)tab_entries * 2 * (size_t)(lt - 1));
    *tab = tab_entries;
  }
  // the staging tiles hold the item's [4L] result after its sweeps
  if (adjsum_stage_bytes(threads / 32, 2) < sizeof(double) * 4 * (size_t)max_layers) return 0;
  const size_t smem = adjsum_smem_bytes(max_layers, threads / 32, 2) + area;
  return smem <= kBatchStageMax ? smem : 0;
}

// KR_DERIV_SUMS=0 keeps the per-step contraction for gradient items (comparison runs).
static bool batch_sums_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("KR_DERIV_SUMS");
    v = (e && atoi(e) == 0) ? 0 : 1;
  }
  return v == 1;
}

template <int THREADS>
static kr_status grids(PlanHeader& h, int max_layers, int tab_entries, int ftab, size_t* fsm,
                       size_t* gsm, int* stage, int* gtab, bool* sums) {
  const int lt = std::min(max_layers, phase_table_max_layers());
  // a model's table sits right after its own layer terms and coefficients, so the block needs
  // the larger of the deepest model's prologue and the deepest tabulating model's prologue
  // plus table (not their sum: 51 instead of 66 KB for 64- and 30-layer models, four blocks
  // per SM instead of three)
  *fsm = std::max(fwd_smem(max_layers),
                  fwd_smem(lt) + (ftab ? sizeof(cd) * (size_t)ftab * 2 * (size_t)(lt - 1) : 0));
  int stab = 0;
  const size_t ssm = batch_sums_enabled() ? sums_smem(THREADS, max_layers, tab_entries, &stab) : 0;
  *sums = ssm > 0;
  if (*sums) {
    *gsm = ssm;
    *gtab = stab;
    *stage = 1;
  } else {
    *gsm = grad_smem(THREADS, max_layers, tab_entries, stage, gtab);
  }
  // limits only ever rise (raise_smem_limit), so batches of different shapes launched from
  // several host threads at once never find a kernel's limit lowered under them
  static SmemLimit flim, slim, glim;
  if (*fsm > 48 * 1024 && raise_smem_limit((const void*)batch_forward_kernel<THREADS>, *fsm, flim,
                                           "kr_batch_launch: forward smem") != KR_OK)
    return KR_ERR_CUDA;
  const void* gk = *sums ? (const void*)batch_grad_sums_kernel<THREADS>
                        : (const void*)batch_gradient_kernel<THREADS>;
  if (*gsm > 48 * 1024 && raise_smem_limit(gk, *gsm, *sums ? slim : glim,
                                           "kr_batch_launch: gradient smem") != KR_OK)
    return KR_ERR_CUDA;
  h.grid_fwd = occupancy_grid((const void*)batch_forward_kernel<THREADS>, THREADS, *fsm);
  h.grid_grad = occupancy_grid(gk, THREADS, *gsm);
  return KR_OK;
}

}  // namespace kr

using namespace kr;

extern "C" size_t kr_batch_plan_bytes(const kr_model_desc* descs, int32_t n_models,
                                      const kr_batch_config* cfg) {
  if (!descs || n_models < 0 || !valid_config(cfg)) return 0;
  PlanLayout lay;
  if (layout(descs, n_models, cfg, &lay, nullptr, nullptr, nullptr) != KR_OK) return 0;
  return lay.bytes;
}

// Fills the plan's metadata image (header, model table, pair table, work lists) in host
// memory; returns its size in *meta_bytes.  Host only: no CUDA call.
static kr_status plan_image(const kr_model_desc* descs, int n_models, const kr_batch_config* cfg,
                            std::vector<unsigned char>* img, size_t* total_bytes) {
  PlanLayout lay;
  std::vector<PairRec> pairs;
  std::vector<ItemRec> fwd, grad;
  kr_status s = layout(descs, n_models, cfg, &lay, &pairs, &fwd, &grad);
  if (s != KR_OK) return s;
  const size_t meta = (size_t)(lay.h.off_grad + sizeof(ItemRec) * grad.size());
  img->assign(meta, 0);
  memcpy(img->data(), &lay.h, sizeof(PlanHeader));
  memcpy(img->data() + lay.h.off_models, descs, sizeof(kr_model_desc) * (size_t)n_models);
  if (!pairs.empty())
    memcpy(img->data() + lay.h.off_pairs, pairs.data(), sizeof(PairRec) * pairs.size());
  if (!fwd.empty()) memcpy(img->data() + lay.h.off_fwd, fwd.data(), sizeof(ItemRec) * fwd.size());
  if (!grad.empty())
    memcpy(img->data() + lay.h.off_grad, grad.data(), sizeof(ItemRec) * grad.size());
  *total_bytes = lay.bytes;
  return KR_OK;
}

extern "C" size_t kr_batch_plan_meta_bytes(const kr_model_desc* descs, int32_t n_models,
                                           const kr_batch_config* cfg) {
  if (!descs || n_models < 0 || !valid_config(cfg)) return 0;
  std::vector<unsigned char> img;
  size_t total = 0;
  if (plan_image(descs, n_models, cfg, &img, &total) != KR_OK) return 0;
  return img.size();
}

extern "C" kr_status kr_batch_plan_host(const kr_model_desc* descs, int32_t n_models,
                                        const kr_batch_config* cfg, void* image,
                                        size_t image_bytes) {
  if (!descs || n_models < 0 || !image) return KR_ERR_INVALID_ARGUMENT;
  if (!valid_config(cfg)) return KR_ERR_INVALID_ARGUMENT;
  std::vector<unsigned char> img;
  size_t total = 0;
  kr_status s = plan_image(descs, n_models, cfg, &img, &total);
  if (s != KR_OK) return s;
  if (image_bytes < img.size()) return KR_ERR_WORKSPACE;
  memcpy(image, img.data(), img.size());
  return KR_OK;
}

extern "C" kr_status kr_batch_plan(const kr_model_desc* descs, int32_t n_models,
                                   const kr_batch_config* cfg, void* plan, size_t plan_bytes,
                                   void* stream) {
  if (!descs || n_models < 0 || !plan) return KR_ERR_INVALID_ARGUMENT;
  if (!valid_config(cfg)) return KR_ERR_INVALID_ARGUMENT;
  std::vector<unsigned char> img;
  size_t total = 0;
  kr_status s = plan_image(descs, n_models, cfg, &img, &total);
  if (s != KR_OK) return s;
  if (plan_bytes < total) return KR_ERR_WORKSPACE;
  // Pageable source: synchronise before the vector goes out of scope.
  cudaError_t e = cudaMemcpyAsync(plan, img.data(), img.size(), cudaMemcpyHostToDevice,
                                  (cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) {
    set_last_error("kr_batch_plan: upload", e);
    return KR_ERR_CUDA;
  }
  return KR_OK;
}

namespace kr {

// One batch launch for a block size of THREADS (32: one warp per work item, i.e. per
// (model, slowness) pair and frequency range; 64 / 128: two / four warps per item).
template <int THREADS>
static kr_status launch_batch(unsigned char* pl, const kr_batch_config* cfg, int max_layers,
                              const double* layers, const double* p, const double* omega,
                              const double* R_obs, double* R, double* chi_grad,
                              cudaStream_t st) {
  // Grid sizes from an occupancy query (host-side, capture-safe).
  PlanHeader h{};
  size_t fsm = 0, gsm = 0;
  int stage = 0;
  const int tab = fwd_table_entries(cfg->tile_w);
  // the forward kernel holds lo / mid and two tiles' hi entries per phase (kPhHead + 2)
  const int ftab = kPhHead + 2;
  int gtab = 0;
  bool sums = false;
  kr_status s = grids<THREADS>(h, max_layers, tab, ftab, &fsm, &gsm, &stage, &gtab, &sums);
  if (s != KR_OK) {
    set_last_error_msg("kr_batch_launch: shared-memory attribute");
    return s;
  }
  batch_reset_kernel<<<148, 128, 0, st>>>(pl, chi_grad);
  s = check_launch("kr_batch_launch: reset");
  if (s != KR_OK) return s;
  batch_prep_kernel<<<148 * 16, 64, 0, st>>>(pl, layers, p);
  s = check_launch("kr_batch_launch: prep");
  if (s != KR_OK) return s;
  // tangents on a resident-sized grid (every block starts at once and releases the forward
  // kernel), the forward kernel as its programmatic dependent
  batch_tan_kernel<<<148 * 4, 64, 0, st>>>(pl, p);
  s = check_launch("kr_batch_launch: tangents");
  if (s != KR_OK) return s;
  const double2* w = reinterpret_cast<const double2*>(omega);
  {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(h.grid_fwd);
    lc.blockDim = dim3(THREADS);
    lc.dynamicSmemBytes = fsm;
    lc.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&lc, batch_forward_kernel<THREADS>, pl, w,
                                             reinterpret_cast<double2*>(R), ftab);
    if (e != cudaSuccess) {
      set_last_error("kr_batch_launch: forward", e);
      return KR_ERR_CUDA;
    }
  }
  if (sums)
    batch_grad_sums_kernel<THREADS><<<h.grid_grad, THREADS, gsm, st>>>(
        pl, w, reinterpret_cast<const double2*>(R_obs), reinterpret_cast<double2*>(R), chi_grad,
        max_layers, gtab);
  else
    batch_gradient_kernel<THREADS><<<h.grid_grad, THREADS, gsm, st>>>(
        pl, w, reinterpret_cast<const double2*>(R_obs), reinterpret_cast<double2*>(R), chi_grad,
        stage, gtab);
  return check_launch("kr_batch_launch: gradient");
}

}  // namespace kr

extern "C" kr_status kr_batch_launch(void* plan, const kr_batch_config* cfg, int32_t max_layers,
                                     const double* layers, const double* p, const double* omega,
                                     const double* R_obs, double* R, double* chi_grad,
                                     void* stream) {
  if (!plan || !valid_config(cfg) || !layers || !p || !omega) return KR_ERR_INVALID_ARGUMENT;
  if (!aligned16(omega) || (R && !aligned16(R)) || (R_obs && !aligned16(R_obs)))
    return KR_ERR_INVALID_ARGUMENT;
  if (max_layers < 2 || max_layers > kMaxLayers) return KR_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char* pl = static_cast<unsigned char*>(plan);
  switch (cfg->threads) {
    case 32:
      return launch_batch<32>(pl, cfg, max_layers, layers, p, omega, R_obs, R, chi_grad, st);
    case 64:
      return launch_batch<64>(pl, cfg, max_layers, layers, p, omega, R_obs, R, chi_grad, st);
    default:
      return launch_batch<128>(pl, cfg, max_layers, layers, p, omega, R_obs, R, chi_grad, st);
  }
}
