// Jacobian and misfit gradient of the reflectivity with respect to every layer's
// (alpha, beta, rho, h): the hand-written adjoint of the Kennett recursion.
//
// Kernels (stream-ordered, no host synchronisation):
//   deriv_prep_kernel  : per (p, interface, tangent column or coefficients): layer terms and
//                        derivative factors, interface coefficients and their 10 x 6 tangents
//                        -> workspace (JAC, and GRAD / VJP on the per-step path)
//   deriv_coef_kernel, deriv_tan_kernel : the same in two kernels for the frequency-sum sweep,
//                        which is launched as the tangent kernel's programmatic dependent and
//                        waits for the tangents only before its contraction
//   deriv_sum_kernel   : GRAD / VJP, per (omega, p): forward sweep with a tape of up to 64
//                        steps (deeper models checkpoint and recompute segments), seed
//                        2 conj(R - R_obs) (GRAD) or conj(gR) (VJP), reverse sweep; the per-step
//                        adjoints are summed over the block's frequencies and contracted with
//                        the tangents once per (p, interface) -> per-block partials
//   deriv_sweep_kernel : the same sweep with the contraction per (omega, p): JAC mode writes
//                        dR/dtheta (J[p][k*L + l][omega], k = alpha, beta, rho, h); GRAD / VJP
//                        for models whose frequency sums exceed shared memory
//   reduce_partials_kernel : adds the block partials in a fixed order (deterministic)
// Replaces the torch autograd graph of kennett_reflectivity_torch (kennett_torch.py:312-480),
// jacobian (:611-641), its reverse pass under torch.autograd.grad, and the per-slowness
// gradient of taup_misfit_grad_hessian (taup_inversion.py:112-187).
#include <stdlib.h>

#include <type_traits>

#include "kr_adjoint.cuh"
#include "kr_adjsum.cuh"
#include "kr_internal.cuh"
#include "kr_phase.cuh"

namespace kr {

constexpr int kDerThreads = 128;
static_assert((kMaxLayers - 2 + kSegMax - 1) / kSegMax <= kCpMax,
              "checkpoints must cover the deepest model");

static size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

struct DerivWs {
  LayerP* lay;
  LayerD* dlay;
  Iface* coef;
  ScatTan* tan;
  double* partial;  // [blocks][4L + 1] (gradient mode)
  size_t bytes;
};

static DerivWs deriv_ws(void* base, int L, int n_p, size_t n_blocks) {
  DerivWs w;
  const int I = L - 1;
  size_t off = 0;
  unsigned char* b = static_cast<unsigned char*>(base);
  w.lay = reinterpret_cast<LayerP*>(b + off);
  off = a256(off + sizeof(LayerP) * (size_t)n_p * L);
  w.dlay = reinterpret_cast<LayerD*>(b + off);
  off = a256(off + sizeof(LayerD) * (size_t)n_p * L);
  w.coef = reinterpret_cast<Iface*>(b + off);
  off = a256(off + sizeof(Iface) * (size_t)n_p * I);
  w.tan = reinterpret_cast<ScatTan*>(b + off);
  off = a256(off + sizeof(ScatTan) * (size_t)n_p * I);
  w.partial = reinterpret_cast<double*>(b + off);
  off = a256(off + sizeof(double) * n_blocks * (size_t)(4 * L + 1));
  w.bytes = off;
  return w;
}

// One block per (slowness, chunk of kPrepThreads interface items): the layer terms and
// derivative factors of the chunk's layers go to shared memory, then one thread per
// (interface, item): items 0..5 form one tangent column each, item 6 the interface's
// coefficients and the workspace copy of its upper layer (and of the half-space, for the last
// interface), so no lane of a warp waits on another's extra work.  The coefficients read the
// layer terms back from shared memory after a barrier, as the forward kernel's prologue
// does, so they round exactly as there (R bit-identical across entry points).
constexpr int kPrepThreads = 128;
constexpr int kPrepItems = 7;                                  // per interface
constexpr int kPrepLayers = kPrepThreads / kPrepItems + 3;     // layers one chunk touches

__global__ void __launch_bounds__(kPrepThreads)
deriv_prep_kernel(const double* __restrict__ tab, int L, const double* __restrict__ p,
                  int n_chunks, LayerP* lay, LayerD* dlay, Iface* coef, ScatTan* tan) {
  __shared__ LayerP s_lp[kPrepLayers];
  __shared__ LayerD s_ld[kPrepLayers];
  const int I = L - 1;
  const int j = blockIdx.x / n_chunks;
  const int t0 = (blockIdx.x % n_chunks) * kPrepThreads;
  const int t1 = min(t0 + kPrepThreads, kPrepItems * I);
  const int l0 = t0 / kPrepItems, l1 = (t1 - 1) / kPrepItems + 1;  // the chunk's layers
  const double pj = p[j];
  for (int l = l0 + threadIdx.x; l <= l1; l += blockDim.x) {
    const LayerP lp = layer_terms(tab, L, l, pj);
    s_lp[l - l0] = lp;
    s_ld[l - l0] = layer_derivs(tab, L, l, pj, lp);
  }
  __syncthreads();
  const int t = t0 + threadIdx.x;
  if (t >= t1) return;
  const int i = t / kPrepItems, item = t % kPrepItems;
  const size_t idx = (size_t)j * I + i, e = (size_t)j * L + i;
  const LayerP& up = s_lp[i - l0];
  const LayerP& lo = s_lp[i + 1 - l0];
  if (item == 6) {
    lay[e] = up;
    dlay[e] = s_ld[i - l0];
    if (i == I - 1) {
      lay[e + 1] = lo;
      dlay[e + 1] = s_ld[i + 1 - l0];
    }
    coef[idx] = interface_coeffs(pj, i, up, lo);
    return;
  }
  cd c[10];
  interface_tangent_col(pj, i, up, s_ld[i - l0], lo, s_ld[i + 1 - l0], item, c);
  for (int k = 0; k < 10; ++k) tan[idx].t[k][item] = c[k];
}

// The same preparation in two kernels, for the frequency-sum sweep, which needs the
// coefficients from its first step but the tangents only in its final contraction:
// deriv_coef_kernel (block per slowness and chunk of kPrepThreads interfaces: layer terms
// staged in shared memory, then one thread per interface for the coefficients, exactly as in
// deriv_prep_kernel) and deriv_tan_kernel (one thread per (slowness, interface, tangent
// column), from the layer terms deriv_coef_kernel wrote), which lets the sweep launch at once
// (griddepcontrol.launch_dependents) so that the tangents overlap the sweep.
__global__ void __launch_bounds__(kPrepThreads)
deriv_coef_kernel(const double* __restrict__ tab, int L, const double* __restrict__ p,
                  int n_chunks, LayerP* lay, LayerD* dlay, Iface* coef) {
  __shared__ LayerP s_lp[kPrepThreads + 1];
  const int I = L - 1;
  const int j = blockIdx.x / n_chunks;
  const int i0 = (blockIdx.x % n_chunks) * kPrepThreads;
  const int i1 = min(i0 + kPrepThreads, I);  // the chunk's interfaces [i0, i1), layers i0 .. i1
  const double pj = p[j];
  for (int l = i0 + threadIdx.x; l <= i1; l += blockDim.x) {
    const LayerP lp = layer_terms(tab, L, l, pj);
    s_lp[l - i0] = lp;
    if (l < i1 || i1 == I) {  // each layer written by one block
      lay[(size_t)j * L + l] = lp;
      dlay[(size_t)j * L + l] = layer_derivs(tab, L, l, pj, lp);
    }
  }
  __syncthreads();
  const int i = i0 + threadIdx.x;
  if (i < i1) coef[(size_t)j * I + i] = interface_coeffs(pj, i, s_lp[i - i0], s_lp[i + 1 - i0]);
}

__global__ void __launch_bounds__(kPrepThreads)
deriv_tan_kernel(const double* __restrict__ p, int n_p, int L, const LayerP* __restrict__ lay,
                 const LayerD* __restrict__ dlay, ScatTan* tan) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int I = L - 1;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n_p * I * 6) return;
  const int col = (int)(t % 6);
  const size_t idx = t / 6;
  const int j = (int)(idx / I), i = (int)(idx % I);
  const size_t e = (size_t)j * L + i;
  cd c[10];
  interface_tangent_col(p[j], i, lay[e], dlay[e], lay[e + 1], dlay[e + 1], col, c);
  for (int k = 0; k < 10; ++k) tan[idx].t[k][col] = c[k];
}

// Jacobian mode: writes dR/dtheta of layer l.
__device__ __forceinline__ void finalize_layer(int l, int L, const Acc& acc, bool valid, int ip,
                                               int iw, int n_w, double2* __restrict__ J) {
  if (valid) {
    const size_t base = ((size_t)ip * 4 * L) * n_w + iw;
    J[base + (size_t)(0 * L + l) * n_w] = make_double2(acc.a.x, acc.a.y);
    J[base + (size_t)(1 * L + l) * n_w] = make_double2(acc.b.x, acc.b.y);
    J[base + (size_t)(2 * L + l) * n_w] = make_double2(acc.r.x, acc.r.y);
    J[base + (size_t)(3 * L + l) * n_w] = make_double2(acc.h.x, acc.h.y);
  }
}

// Gradient mode: acc already holds 2 Re(conj(res) dR/dtheta) (the reverse sweep was seeded
// with 2 conj(res)); reduced over the warp by shuffles and added to this warp's own
// accumulator row (no block barrier).
__device__ __forceinline__ void finalize_layer(int l, int L, const AccR& acc, bool valid,
                                               double* s_wacc) {
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (valid) {
    v[0] = acc.a;
    v[1] = acc.b;
    v[2] = acc.r;
    v[3] = acc.h;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0) {
    double* row = s_wacc + (threadIdx.x >> 5) * (4 * L + 1);
    for (int k = 0; k < 4; ++k) row[k * L + l] += v[k];
  }
}

// Sweep modes: JAC writes dR/dtheta per (omega, p); GRAD seeds the reverse sweep with
// 2 conj(R - R_obs) (misfit gradient, plus chi); VJP seeds it with conj(gR) for a caller's
// cotangent gR (Re sum conj(gR) dR/dtheta, no chi).  GRAD and VJP accumulate real parts only.
constexpr int kModeJac = 0;
constexpr int kModeGrad = 1;
constexpr int kModeVjp = 2;

// Receives R and the per-layer derivatives of one thread's (omega, p) pair.
template <int MODE>
struct PairSink {
  typedef typename std::conditional<MODE != kModeJac, AccR, Acc>::type AccT;
  static constexpr bool kSeeded = MODE != kModeJac;
  int L, ip, iw, n_w;
  bool valid;
  const double2* R_obs;  // GRAD: observed R; VJP: the cotangent gR
  double2* R_out;
  double2* J;
  double* s_wacc;
  cd res;
  __device__ cd reflectivity(cd R) {
    res = mk(0.0, 0.0);
    if (!valid) return mk(0.0, 0.0);
    if (R_out) R_out[(size_t)ip * n_w + iw] = make_double2(R.x, R.y);
    if (MODE == kModeJac) return mk(1.0, 0.0);
    const double2 o = R_obs[(size_t)ip * n_w + iw];
    if (MODE == kModeVjp) return mk(o.x, -o.y);  // conj(gR)
    res = mk(R.x - o.x, R.y - o.y);
    return mk(2.0 * res.x, -2.0 * res.y);  // 2 conj(res)
  }
  __device__ void layer(int l, const AccT& acc) {
    if constexpr (MODE != kModeJac)
      finalize_layer(l, L, acc, valid, s_wacc);
    else
      finalize_layer(l, L, acc, valid, ip, iw, n_w, J);
  }
};

template <int MODE, int MINB>
__global__ void __launch_bounds__(kDerThreads, MINB)
deriv_sweep_kernel(int L, const double* __restrict__ p, int n_p,
                   const double2* __restrict__ omega, int n_w, int n_wtiles, int free_surface,
                   int seg, int stage, int table, const LayerP* __restrict__ lay_all,
                   const LayerD* __restrict__ dlay_all, const Iface* __restrict__ coef_all,
                   const ScatTan* __restrict__ tan_all, const double2* __restrict__ R_obs,
                   double2* __restrict__ R_out, double2* __restrict__ J,
                   double* __restrict__ partial) {
  // dynamic smem: [warps][4L + 1] per-warp accumulators (GRAD), then, if `stage`, this
  // block's slowness data (tangents, coefficients, layer terms, layer derivatives), then, if
  // `table`, the phase-factor table of this block's frequency tile (kr_phase.cuh)
  constexpr bool GRAD = MODE != kModeJac;
  extern __shared__ __align__(16) double s_wacc[];
  __shared__ unsigned s_bad;
  const int ip = blockIdx.x / n_wtiles;
  const int iw = (blockIdx.x % n_wtiles) * kDerThreads + threadIdx.x;
  const bool valid = iw < n_w;
  const int I = L - 1;
  const int nv = 4 * L + 1;
  if (GRAD) {
    for (int k = threadIdx.x; k < (kDerThreads / 32) * nv; k += blockDim.x) s_wacc[k] = 0.0;
    __syncthreads();
  }
  cd w = mk(0.0, 0.0);
  if (valid) {
    const double2 wv = omega[iw];
    w = mk(wv.x, wv.y);
  }
  const ScatTan* tan = tan_all + (size_t)ip * I;
  const Iface* coef = coef_all + (size_t)ip * I;
  const LayerP* lay = lay_all + (size_t)ip * L;
  const LayerD* dlay = dlay_all + (size_t)ip * L;
  if (stage) {
    unsigned char* b = reinterpret_cast<unsigned char*>(s_wacc) +
                       (GRAD ? sizeof(double) * (((kDerThreads / 32) * nv + 1) / 2 * 2) : 0);
    ScatTan* st = reinterpret_cast<ScatTan*>(b);
    Iface* sc = reinterpret_cast<Iface*>(b + sizeof(ScatTan) * I);
    LayerP* sl = reinterpret_cast<LayerP*>(b + (sizeof(ScatTan) + sizeof(Iface)) * I);
    LayerD* sd = reinterpret_cast<LayerD*>(b + (sizeof(ScatTan) + sizeof(Iface)) * I +
                                           sizeof(LayerP) * L);
    copy16(st, tan, sizeof(ScatTan) * I);
    copy16(sc, coef, sizeof(Iface) * I);
    copy16(sl, lay, sizeof(LayerP) * L);
    copy16(sd, dlay, sizeof(LayerD) * L);
    __syncthreads();
    tan = st;
    coef = sc;
    lay = sl;
    dlay = sd;
  }
  const int tile = blockIdx.x % n_wtiles;
  const size_t acc_bytes = GRAD ? sizeof(double) * (((kDerThreads / 32) * nv + 1) / 2 * 2) : 0;
  cd* s_ph = reinterpret_cast<cd*>(reinterpret_cast<unsigned char*>(s_wacc) + acc_bytes +
                                   pair_smem_bytes(L));
  bool use_tab = false;
  if (table)
    use_tab = (build_phase_table(omega, n_w, grid_line(omega, n_w), tile, 1, kPhHead + 1, L, lay,
                                 s_ph, &s_bad) &
               1u) != 0;
  const PhaseAuto ph{use_tab, phase_at(s_ph, kPhHead + 1, valid ? iw : tile * kDerThreads, tile),
                     PhaseDirect{w, lay}};
  PairSink<MODE> sink;
  sink.L = L;
  sink.ip = ip;
  sink.iw = iw;
  sink.n_w = n_w;
  sink.valid = valid;
  sink.R_obs = R_obs;
  sink.R_out = R_out;
  sink.J = J;
  sink.s_wacc = s_wacc;
  jacobian_pair(L, w, free_surface != 0, seg, lay, dlay, coef, tan, ph, sink);
  if (GRAD) {
    const cd res = sink.res;
    double c2 = valid ? (res.x * res.x + res.y * res.y) : 0.0;
    for (int o = 16; o > 0; o >>= 1) c2 += __shfl_down_sync(0xffffffffu, c2, o);
    if ((threadIdx.x & 31) == 0) s_wacc[(threadIdx.x >> 5) * nv + 4 * L] += c2;
    __syncthreads();
    double* dst = partial + (size_t)blockIdx.x * nv;
    for (int k = threadIdx.x; k < nv; k += blockDim.x) {
      double t = 0.0;
      for (int wi = 0; wi < kDerThreads / 32; ++wi) t += s_wacc[wi * nv + k];
      dst[k] = t;
    }
  }
}

// out[k] = sum_b partial[b][k] for k < gridDim.x (rows of `stride` doubles): one block per
// k, fixed-shape tree (deterministic).
__global__ void __launch_bounds__(256)
reduce_partials_kernel(const double* __restrict__ partial, int n_blocks, int stride,
                       double* __restrict__ out) {
  // after the frequency-sum sweep this kernel is launched as the sweep's programmatic
  // dependent: wait for that grid and its partials (a no-op after an ordinary launch)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  __shared__ double s[256];
  const int k = blockIdx.x;
  double t = 0.0;
  for (int b = threadIdx.x; b < n_blocks; b += 256) t += partial[(size_t)b * stride + k];
  s[threadIdx.x] = t;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[k] = s[0];
}

// GRAD / VJP with the contraction moved out of the frequency loop (kr_adjsum.cuh): block =
// one slowness x 128 frequencies; dynamic smem: per-warp sum rows and staging tiles, then the
// slowness's interface coefficients and layer terms, then (table models) the phase table.
// Writes the block's [4L] contributions and chi to partial[block][4L + 1].
template <int MINB>
__global__ void __launch_bounds__(kDerThreads, MINB)
deriv_sum_kernel(int L, int n_p, const double2* __restrict__ omega, int n_w, int n_wtiles,
                 int free_surface, int vjp, int seg, int table, const LayerP* __restrict__ lay_all,
                 const LayerD* __restrict__ dlay_all, const Iface* __restrict__ coef_all,
                 const ScatTan* __restrict__ tan_all, const double2* __restrict__ obs,
                 double2* __restrict__ R_out, double* __restrict__ partial) {
  // the reduction after this kernel may launch as soon as every block of it has started
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  constexpr int W = kDerThreads / 32;
  extern __shared__ __align__(16) double s_raw[];
  __shared__ unsigned s_bad;
  __shared__ double s_chi[W];
  const int I = L - 1;
  const int ip = blockIdx.x / n_wtiles;
  const int tile = blockIdx.x % n_wtiles;
  const int iw = tile * kDerThreads + threadIdx.x;
  const bool valid = iw < n_w;
  const int warp = threadIdx.x >> 5;
  constexpr int RS = 1;  // one staging round: registers, not shared memory, bound residency
  cd* acc = reinterpret_cast<cd*>(s_raw);
  cd* stage = acc + (size_t)W * sum_rows(L) * kSumVals;
  unsigned char* b = reinterpret_cast<unsigned char*>(stage + W * 32 * stage_stride<RS>());
  Iface* sc = reinterpret_cast<Iface*>(b);
  LayerP* sl = reinterpret_cast<LayerP*>(b + sizeof(Iface) * I);
  cd* s_ph = reinterpret_cast<cd*>(b + sizeof(Iface) * I + sizeof(LayerP) * L);
  sums_zero(acc, L, W);
  copy16(sc, coef_all + (size_t)ip * I, sizeof(Iface) * I);
  copy16(sl, lay_all + (size_t)ip * L, sizeof(LayerP) * L);
  __syncthreads();
  cd w = mk(0.0, 0.0);
  if (valid) {
    const double2 wv = omega[iw];
    w = mk(wv.x, wv.y);
  }
  bool use_tab = false;
  if (table)
    use_tab = (build_phase_table(omega, n_w, grid_line(omega, n_w), tile, 1, kPhHead + 1, L, sl,
                                 s_ph, &s_bad) & 1u) != 0;
  const PhaseAuto ph{use_tab, phase_at(s_ph, kPhHead + 1, valid ? iw : tile * kDerThreads, tile),
                     PhaseDirect{w, sl}};
  const size_t e = (size_t)ip * n_w + (valid ? iw : 0);
  SumSink<RS> sink;
  sink.valid = valid;
  sink.vjp = vjp != 0;
  sink.obs = obs + e;
  sink.R_out = R_out ? R_out + e : nullptr;
  sink.acc = acc + (size_t)warp * sum_rows(L) * kSumVals;
  sink.stage = stage + warp * 32 * stage_stride<RS>();
  sink.I = I;
  adjoint_pair_sums(L, w, free_surface != 0, seg, sc, ph, sink);
  double c2 = valid ? (sink.res.x * sink.res.x + sink.res.y * sink.res.y) : 0.0;
  for (int o = 16; o > 0; o >>= 1) c2 += __shfl_down_sync(0xffffffffu, c2, o);
  if ((threadIdx.x & 31) == 0) s_chi[warp] = c2;
  double* dst = partial + (size_t)blockIdx.x * (4 * L + 1);
  // the tangents may still be in the making (deriv_tan_kernel, launched ahead of this kernel
  // as its programmatic prerequisite): wait for that grid's completion and its writes; a
  // no-op when the kernel was launched without the dependency
  asm volatile("griddepcontrol.wait;" ::: "memory");
  sums_finish(acc, L, W, tan_all + (size_t)ip * I, dlay_all + (size_t)ip * L, dst);
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int wi = 0; wi < W; ++wi) t += s_chi[wi];
    dst[4 * L] = t;
  }
}

// Shared memory the sweep may use for staging one slowness's data (per block).
constexpr size_t kStageSmemMax = 160 * 1024;

// Register budget of the sweep kernels: blocks of 128 threads per SM (2 -> up to 255
// registers, 3 -> 168).  KR_DERIV_MINB or kr_set_deriv_variant; default 2.  (The
// frequency-sum kernel fits 168 registers without spills, but three of its blocks leave too
// little L1 for the tape: 0.154 ms vs 0.138 ms per 64 x 1024 gradient.)
static int g_deriv_minb = -1;

static int deriv_minb_setting() {
  if (g_deriv_minb < 0) {
    const char* e = getenv("KR_DERIV_MINB");
    const int v = e ? atoi(e) : 0;
    g_deriv_minb = (v == 2 || v == 3) ? v : 0;
  }
  return g_deriv_minb;
}
static int deriv_minb() { return deriv_minb_setting() == 3 ? 3 : 2; }
static int sum_minb() { return deriv_minb(); }

template <int MODE, int MINB>
static kr_status launch_sweep_v(unsigned blocks, size_t smem, cudaStream_t st, int L,
                                const double* p, int n_p, const double2* omega, int n_w,
                                int n_wtiles, int fs, int seg, int stage, int table,
                                const LayerP* lay, const LayerD* dlay, const Iface* coef,
                                const ScatTan* tan, const double2* R_obs, double2* R, double2* J,
                                double* partial) {
  static SmemLimit lim;
  if (smem > 48 * 1024) {
    const kr_status a = raise_smem_limit((const void*)deriv_sweep_kernel<MODE, MINB>, smem, lim,
                                         "kr_deriv: smem attribute");
    if (a != KR_OK) return a;
  }
  deriv_sweep_kernel<MODE, MINB><<<blocks, kDerThreads, smem, st>>>(
      L, p, n_p, omega, n_w, n_wtiles, fs, seg, stage, table, lay, dlay, coef, tan, R_obs, R, J,
      partial);
  return KR_OK;
}

template <int MODE>
static kr_status launch_sweep(int minb, unsigned blocks, size_t smem, cudaStream_t st, int L,
                              const double* p, int n_p, const double2* omega, int n_w,
                              int n_wtiles, int fs, int seg, int stage, int table,
                              const LayerP* lay, const LayerD* dlay, const Iface* coef,
                              const ScatTan* tan, const double2* R_obs, double2* R, double2* J,
                              double* partial) {
  if (minb == 3)
    return launch_sweep_v<MODE, 3>(blocks, smem, st, L, p, n_p, omega, n_w, n_wtiles, fs, seg,
                                   stage, table, lay, dlay, coef, tan, R_obs, R, J, partial);
  return launch_sweep_v<MODE, 2>(blocks, smem, st, L, p, n_p, omega, n_w, n_wtiles, fs, seg,
                                 stage, table, lay, dlay, coef, tan, R_obs, R, J, partial);
}

// Dynamic smem of deriv_sum_kernel for a model of L layers (0 if it does not fit).
static size_t sum_kernel_smem(int L, int table) {
  const size_t smem = adjsum_smem_bytes(L, kDerThreads / 32, 1) + prologue_smem_bytes(L) +
                      (table ? phase_table_bytes(L, 1) : 0);
  return smem <= kStageSmemMax ? smem : 0;
}

// KR_DERIV_SUMS=0 keeps the per-step contraction for GRAD / VJP (comparison runs).
static bool deriv_sums_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("KR_DERIV_SUMS");
    v = (e && atoi(e) == 0) ? 0 : 1;
  }
  return v == 1;
}

template <int MINB>
static kr_status launch_sum_v(unsigned blocks, size_t smem, cudaStream_t st, int L, int n_p,
                              const double2* omega, int n_w, int n_wtiles, int fs, int vjp,
                              int seg, int table, const LayerP* lay, const LayerD* dlay,
                              const Iface* coef, const ScatTan* tan, const double2* obs,
                              double2* R, double* partial) {
  static SmemLimit lim;
  if (smem > 48 * 1024) {
    const kr_status a = raise_smem_limit((const void*)deriv_sum_kernel<MINB>, smem, lim,
                                         "kr_deriv: smem attribute");
    if (a != KR_OK) return a;
  }
  // programmatic dependent launch: the sweep may start while the tangent kernel ahead of it
  // on the stream still runs; it waits for it (griddepcontrol.wait) only before contracting
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(kDerThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, deriv_sum_kernel<MINB>, L, n_p, omega, n_w,
                                           n_wtiles, fs, vjp, seg, table, lay, dlay, coef, tan,
                                           obs, R, partial);
  if (e != cudaSuccess) {
    set_last_error("kr_deriv: sweep launch", e);
    return KR_ERR_CUDA;
  }
  return KR_OK;
}

template <int MODE>
static kr_status launch_deriv(const double* layers, int L, const double* p, int n_p,
                              const double* omega, int n_w, uint32_t flags, const double* R_obs,
                              double* R, double* J, double* chi_grad, void* ws, size_t ws_bytes,
                              cudaStream_t st) {
  constexpr bool GRAD = MODE != kModeJac;
  const int n_wtiles = (n_w + kDerThreads - 1) / kDerThreads;
  const size_t n_blocks = (size_t)n_p * n_wtiles;
  if (n_blocks > 0x7fffffffULL) return KR_ERR_TOO_LARGE;
  DerivWs w = deriv_ws(ws, L, n_p, GRAD ? n_blocks : 0);
  if (!ws || ws_bytes < w.bytes) return KR_ERR_WORKSPACE;
  const int I = L - 1;
  const int seg = checkpoint_spacing(I - 1 > 0 ? I - 1 : 1);
  const int sum_table = phase_table_model(L) ? 1 : 0;
  const size_t sum_smem = (GRAD && deriv_sums_enabled()) ? sum_kernel_smem(L, sum_table) : 0;
  kr_status s = KR_OK;
  if (sum_smem) {
    // coefficients first; the tangents then overlap the frequency-sum sweep
    const int n_cc = (I + kPrepThreads - 1) / kPrepThreads;
    const size_t n_tan = (size_t)n_p * I * 6;
    if ((size_t)n_p * n_cc > 0x7fffffffULL || (n_tan + kPrepThreads - 1) / kPrepThreads > 0x7fffffffULL)
      return KR_ERR_TOO_LARGE;
    deriv_coef_kernel<<<(unsigned)(n_p * n_cc), kPrepThreads, 0, st>>>(layers, L, p, n_cc, w.lay,
                                                                       w.dlay, w.coef);
    s = check_launch("kr_deriv: layers and coefficients");
    if (s != KR_OK) return s;
    deriv_tan_kernel<<<(unsigned)((n_tan + kPrepThreads - 1) / kPrepThreads), kPrepThreads, 0,
                       st>>>(p, n_p, L, w.lay, w.dlay, w.tan);
    s = check_launch("kr_deriv: tangents");
    if (s != KR_OK) return s;
  } else {
    const int n_chunks = (kPrepItems * I + kPrepThreads - 1) / kPrepThreads;
    if ((size_t)n_p * n_chunks > 0x7fffffffULL) return KR_ERR_TOO_LARGE;
    deriv_prep_kernel<<<(unsigned)(n_p * n_chunks), kPrepThreads, 0, st>>>(
        layers, L, p, n_chunks, w.lay, w.dlay, w.coef, w.tan);
    s = check_launch("kr_deriv: layers and interfaces");
    if (s != KR_OK) return s;
  }
  if (sum_smem) {
    const int fs = (flags & KR_FREE_SURFACE) ? 1 : 0;
    const int vjp = MODE == kModeVjp ? 1 : 0;
    const double2* o = reinterpret_cast<const double2*>(R_obs);
    const double2* w2 = reinterpret_cast<const double2*>(omega);
    double2* R2 = reinterpret_cast<double2*>(R);
    s = sum_minb() == 3
            ? launch_sum_v<3>((unsigned)n_blocks, sum_smem, st, L, n_p, w2, n_w, n_wtiles, fs,
                              vjp, seg, sum_table, w.lay, w.dlay, w.coef, w.tan, o, R2, w.partial)
            : launch_sum_v<2>((unsigned)n_blocks, sum_smem, st, L, n_p, w2, n_w, n_wtiles, fs,
                              vjp, seg, sum_table, w.lay, w.dlay, w.coef, w.tan, o, R2, w.partial);
    if (s != KR_OK) return s;
    s = check_launch("kr_deriv: sweep");
    if (s != KR_OK) return s;
    const int nv = 4 * L + 1;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(MODE == kModeGrad ? nv : nv - 1);
    lc.blockDim = dim3(256);
    lc.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&lc, reduce_partials_kernel,
                                             (const double*)w.partial, (int)n_blocks, nv, chi_grad);
    if (e != cudaSuccess) {
      set_last_error("kr_deriv: reduce launch", e);
      return KR_ERR_CUDA;
    }
    return KR_OK;
  }
  // accumulators: [warps][4L + 1] doubles, padded to 16 bytes
  const size_t acc = GRAD ? sizeof(double) * (((size_t)(kDerThreads / 32) * (4 * L + 1) + 1) / 2 * 2) : 0;
  const size_t pair = pair_smem_bytes(L);
  const int stage = (acc + pair <= kStageSmemMax) ? 1 : 0;
  // phase table of the block's tile after the staged slowness data (models that tabulate in
  // kr_reflectivity, so R here is bit-identical to the forward kernel's)
  const int table = (stage && phase_table_model(L)) ? 1 : 0;
  const size_t smem = acc + (stage ? pair : 0) + (table ? phase_table_bytes(L, 1) : 0);
  s = launch_sweep<MODE>(deriv_minb(), (unsigned)n_blocks, smem, st, L, p, n_p,
                         reinterpret_cast<const double2*>(omega), n_w, n_wtiles,
                         (flags & KR_FREE_SURFACE) ? 1 : 0, seg, stage, table, w.lay, w.dlay, w.coef,
                         w.tan, reinterpret_cast<const double2*>(R_obs),
                         reinterpret_cast<double2*>(R), reinterpret_cast<double2*>(J), w.partial);
  if (s != KR_OK) return s;
  s = check_launch("kr_deriv: sweep");
  if (s != KR_OK || !GRAD) return s;
  // GRAD: gradient then chi (4L + 1 values); VJP: the gradient only (4L)
  const int nv = 4 * L + 1;
  reduce_partials_kernel<<<MODE == kModeGrad ? nv : nv - 1, 256, 0, st>>>(w.partial, (int)n_blocks,
                                                                          nv, chi_grad);
  return check_launch("kr_deriv: reduce");
}

static kr_status deriv_args(const double* layers, int L, const double* p, int n_p,
                            const double* omega, int n_w, uint32_t flags) {
  if (n_p < 0 || n_w < 0 || (flags & ~KR_FREE_SURFACE)) return KR_ERR_INVALID_ARGUMENT;
  if (L < 2) return KR_ERR_INVALID_MODEL;
  if (L > kMaxLayers) return KR_ERR_TOO_LARGE;
  if (n_p > 0 && n_w > 0 && (!layers || !p || !omega)) return KR_ERR_INVALID_ARGUMENT;
  if (!aligned16(omega)) return KR_ERR_INVALID_ARGUMENT;
  return KR_OK;
}

}  // namespace kr

using namespace kr;

extern "C" void kr_set_deriv_variant(int32_t min_blocks_per_sm) {
  g_deriv_minb = (min_blocks_per_sm == 2 || min_blocks_per_sm == 3) ? min_blocks_per_sm : 0;
}

extern "C" size_t kr_jacobian_workspace_bytes(int32_t n_layers, int32_t n_p, int32_t n_w) {
  if (n_layers < 2 || n_p <= 0 || n_w <= 0) return 0;
  (void)n_w;
  return deriv_ws(nullptr, n_layers, n_p, 0).bytes;
}

extern "C" kr_status kr_jacobian(const double* layers, int32_t n_layers, const double* p,
                                 int32_t n_p, const double* omega, int32_t n_w, uint32_t flags,
                                 double* R, double* J, void* workspace, size_t workspace_bytes,
                                 void* stream) {
  kr_status s = deriv_args(layers, n_layers, p, n_p, omega, n_w, flags);
  if (s != KR_OK) return s;
  if (n_p == 0 || n_w == 0) return KR_OK;
  if (!J || !aligned16(J) || (R && !aligned16(R))) return KR_ERR_INVALID_ARGUMENT;
  return launch_deriv<kModeJac>(layers, n_layers, p, n_p, omega, n_w, flags, nullptr, R, J, nullptr,
                             workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" size_t kr_misfit_gradient_workspace_bytes(int32_t n_layers, int32_t n_p, int32_t n_w) {
  if (n_layers < 2 || n_p <= 0 || n_w <= 0) return 0;
  const size_t n_blocks = (size_t)n_p * ((n_w + kDerThreads - 1) / kDerThreads);
  return deriv_ws(nullptr, n_layers, n_p, n_blocks).bytes;
}

extern "C" kr_status kr_misfit_gradient(const double* layers, int32_t n_layers, const double* p,
                                        int32_t n_p, const double* omega, int32_t n_w,
                                        uint32_t flags, const double* R_obs, double* R,
                                        double* chi_grad, void* workspace,
                                        size_t workspace_bytes, void* stream) {
  kr_status s = deriv_args(layers, n_layers, p, n_p, omega, n_w, flags);
  if (s != KR_OK) return s;
  if (!chi_grad) return KR_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (n_p == 0 || n_w == 0) {
    cudaError_t e = cudaMemsetAsync(chi_grad, 0, sizeof(double) * (4 * (size_t)n_layers + 1), st);
    if (e != cudaSuccess) set_last_error("kr_misfit_gradient: memset", e);
    return cuda_status(e);
  }
  if (!R_obs || !aligned16(R_obs) || (R && !aligned16(R))) return KR_ERR_INVALID_ARGUMENT;
  return launch_deriv<kModeGrad>(layers, n_layers, p, n_p, omega, n_w, flags, R_obs, R, nullptr,
                            chi_grad, workspace, workspace_bytes, st);
}

extern "C" size_t kr_vjp_workspace_bytes(int32_t n_layers, int32_t n_p, int32_t n_w) {
  return kr_misfit_gradient_workspace_bytes(n_layers, n_p, n_w);
}

extern "C" kr_status kr_vjp(const double* layers, int32_t n_layers, const double* p, int32_t n_p,
                            const double* omega, int32_t n_w, uint32_t flags, const double* gR,
                            double* R, double* grad, void* workspace, size_t workspace_bytes,
                            void* stream) {
  kr_status s = deriv_args(layers, n_layers, p, n_p, omega, n_w, flags);
  if (s != KR_OK) return s;
  if (!grad) return KR_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (n_p == 0 || n_w == 0) {
    cudaError_t e = cudaMemsetAsync(grad, 0, sizeof(double) * 4 * (size_t)n_layers, st);
    if (e != cudaSuccess) set_last_error("kr_vjp: memset", e);
    return cuda_status(e);
  }
  if (!gR || !aligned16(gR) || (R && !aligned16(R))) return KR_ERR_INVALID_ARGUMENT;
  return launch_deriv<kModeVjp>(layers, n_layers, p, n_p, omega, n_w, flags, gR, R, nullptr, grad,
                                workspace, workspace_bytes, st);
}
