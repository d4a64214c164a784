// Exact second derivatives of the reflectivity path: Hessian-vector products of the misfit
// and directional derivatives of the Jacobian, by the tangent of the adjoint (kr_hvp.cuh).
//
// Kernels (all stream-ordered, no host synchronisation):
//   hvp_layer_kernel : per (p, layer)            layer terms, first and second derivative
//                                                 factors -> workspace
//   hvp_iface_kernel : per (p, interface, column) coefficients + 10x6 tangents
//   hvp_ldot_kernel  : per (direction, p, layer) layer values with tangents along v
//   hvp_idot_kernel  : per (direction, p, iface, column) coefficients with tangents along v and the
//                                                 tangents of the 10x6 coefficient tangents
//   hvp_sum_kernel   : per (direction, p, omega) forward sweep, seed and reverse sweep in dual
//                                                 numbers, the per-step dual adjoints summed over
//                                                 the block's frequencies and contracted once
//                                                 (HV mode)
//   hvp_sweep_kernel : the same with the contraction per (omega, p): HV mode for models whose
//                                                 sums exceed shared memory, JDOT mode (writes
//                                                 d/dv of dR/dtheta per frequency)
//   hvp_reduce_kernel: per (direction, parameter) adds the block partials in a fixed order
// Replaces torch.func.hessian of the reference's tau-p misfit (taup_inversion.py:177,
// kennett_torch.py:644-684) and the second-order derivative graph it differentiates.
#include "kr_adjsum.cuh"
#include "kr_hvp.cuh"
#include "kr_internal.cuh"

namespace kr {

constexpr int kHvpThreads = 128;
constexpr int kHvpModeHv = 0;
constexpr int kHvpModeJdot = 1;

static size_t a256h(size_t x) { return (x + 255) & ~(size_t)255; }

struct HvpWs {
  LayerP* lay;      // [n_p][L]
  LayerD* dlay;     // [n_p][L]
  LayerD2* d2;      // [n_p][L]
  Iface* coef;      // [n_p][I]
  ScatTan* tan;     // [n_p][I]
  LayerV* lv;       // [n_dir][n_p][L]
  IfS<DC>* ifs;     // [n_dir][n_p][I]
  ScatTan* tant;    // [n_dir][n_p][I]
  double* partial;  // [n_dir][n_p * n_wtiles][4L] (HV mode)
  size_t bytes;
};

static HvpWs hvp_ws(void* base, int L, int n_p, int n_dir, size_t blocks_per_dir, bool hv) {
  HvpWs w;
  const int I = L - 1;
  size_t off = 0;
  unsigned char* b = static_cast<unsigned char*>(base);
  const size_t np = (size_t)n_p, nd = (size_t)n_dir;
  w.lay = reinterpret_cast<LayerP*>(b + off);
  off = a256h(off + sizeof(LayerP) * np * L);
  w.dlay = reinterpret_cast<LayerD*>(b + off);
  off = a256h(off + sizeof(LayerD) * np * L);
  w.d2 = reinterpret_cast<LayerD2*>(b + off);
  off = a256h(off + sizeof(LayerD2) * np * L);
  w.coef = reinterpret_cast<Iface*>(b + off);
  off = a256h(off + sizeof(Iface) * np * I);
  w.tan = reinterpret_cast<ScatTan*>(b + off);
  off = a256h(off + sizeof(ScatTan) * np * I);
  w.lv = reinterpret_cast<LayerV*>(b + off);
  off = a256h(off + sizeof(LayerV) * nd * np * L);
  w.ifs = reinterpret_cast<IfS<DC>*>(b + off);
  off = a256h(off + sizeof(IfS<DC>) * nd * np * I);
  w.tant = reinterpret_cast<ScatTan*>(b + off);
  off = a256h(off + sizeof(ScatTan) * nd * np * I);
  w.partial = reinterpret_cast<double*>(b + off);
  if (hv) off = a256h(off + sizeof(double) * nd * blocks_per_dir * (size_t)(4 * L));
  w.bytes = off;
  return w;
}

__global__ void hvp_layer_kernel(const double* __restrict__ tab, int L,
                                 const double* __restrict__ p, int n_p, LayerP* lay, LayerD* dlay,
                                 LayerD2* d2) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_p * L) return;
  const int j = idx / L, l = idx % L;
  const LayerP lp = layer_terms(tab, L, l, p[j]);
  const LayerD d = layer_derivs(tab, L, l, p[j], lp);
  lay[idx] = lp;
  dlay[idx] = d;
  d2[idx] = layer_derivs2(tab, L, l, lp, d);
}

__global__ void hvp_iface_kernel(const double* __restrict__ p, int n_p, int L,
                                 const LayerP* __restrict__ lay, const LayerD* __restrict__ dlay,
                                 Iface* coef, ScatTan* tan) {
  const int I = L - 1;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n_p * I * 6) return;
  const int col = (int)(t % 6);
  const size_t idx = t / 6;
  const int j = (int)(idx / I), i = (int)(idx % I);
  const size_t e = (size_t)j * L + i;
  const LayerP up = lay[e], lo = lay[e + 1];
  if (col == 0) coef[idx] = interface_coeffs(p[j], i, up, lo);
  cd c[10];
  interface_tangent_col(p[j], i, up, dlay[e], lo, dlay[e + 1], col, c);
  for (int k = 0; k < 10; ++k) tan[idx].t[k][col] = c[k];
}

// V: [n_dir][4L] directions, theta order k*L + l (alpha, beta, rho, h)
__global__ void hvp_ldot_kernel(const double* __restrict__ tab, int L, int n_p, int n_dir,
                                const double* __restrict__ V, const LayerP* __restrict__ lay,
                                const LayerD* __restrict__ dlay, const LayerD2* __restrict__ d2,
                                LayerV* lv) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)n_dir * n_p * L) return;
  const int l = (int)(idx % L);
  const size_t jd = idx / L;
  const int j = (int)(jd % n_p);
  const int dir = (int)(jd / n_p);
  const double* v = V + (size_t)dir * 4 * L;
  const double vl[4] = {v[l], v[L + l], v[2 * L + l], v[3 * L + l]};
  const size_t e = (size_t)j * L + l;
  lv[idx] = layer_dot(tab, L, l, lay[e], dlay[e], d2[e], vl);
}

__global__ void hvp_idot_kernel(const double* __restrict__ p, int L, int n_p, int n_dir,
                                const Iface* __restrict__ coef, const LayerV* __restrict__ lv,
                                IfS<DC>* ifs, ScatTan* tant) {
  const int I = L - 1;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n_dir * n_p * I * 6) return;
  const int col = (int)(t % 6);
  const size_t idx = t / 6;
  const int i = (int)(idx % I);
  const size_t jd = idx / I;
  const int j = (int)(jd % n_p);
  const LayerV* l0 = lv + jd * L;
  IfS<DC> c;
  cd tc[10];
  interface_dot_col(p[j], i, l0[i], l0[i + 1], col, col == 0 ? &c : nullptr, tc);
  for (int k = 0; k < 10; ++k) tant[idx].t[k][col] = tc[k];
  if (col == 0) ifs[idx] = iface_dual(coef[(size_t)j * I + i], c);
}

template <int MODE>
struct HvpSink {
  int L;
  bool valid;
  cd robs;           // HV: observed R at this (p, omega)
  double* row;       // HV: this warp's [4L] accumulators
  double2* jd;       // JDOT: d/dv J for this (direction, p), [4L][n_w], at this omega
  int n_w;
  DC res;
  __device__ DC reflectivity(const DC& R) {
    res = dc(mk(0.0, 0.0));
    if (!valid) return dc(mk(0.0, 0.0));
    if (MODE == kHvpModeJdot) return dc(mk(1.0, 0.0));
    res = dc(R.v - robs, R.t);
    return dc(mk(2.0 * res.v.x, -2.0 * res.v.y), mk(2.0 * res.t.x, -2.0 * res.t.y));
  }
  __device__ void layer(int l, const AccD& a) {
    if (MODE == kHvpModeJdot) {
      if (valid) {
        jd[(size_t)(0 * L + l) * n_w] = make_double2(a.a.t.x, a.a.t.y);
        jd[(size_t)(1 * L + l) * n_w] = make_double2(a.b.t.x, a.b.t.y);
        jd[(size_t)(2 * L + l) * n_w] = make_double2(a.r.t.x, a.r.t.y);
        jd[(size_t)(3 * L + l) * n_w] = make_double2(a.h.t.x, a.h.t.y);
      }
      return;
    }
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (valid) {
      v[0] = a.a.t.x;
      v[1] = a.b.t.x;
      v[2] = a.r.t.x;
      v[3] = a.h.t.x;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0)
      for (int k = 0; k < 4; ++k) row[k * L + l] += v[k];
  }
};

// grid: n_dir * n_p * n_wtiles blocks of kHvpThreads; block -> (dir, p, frequency tile)
template <int MODE>
__global__ void __launch_bounds__(kHvpThreads, 1)
hvp_sweep_kernel(int L, int n_p, int n_dir, const double2* __restrict__ omega, int n_w,
                 int n_wtiles, int free_surface, const LayerV* __restrict__ lv_all,
                 const IfS<DC>* __restrict__ ifs_all, const ScatTan* __restrict__ tan_all,
                 const ScatTan* __restrict__ tant_all, const double2* __restrict__ R_obs,
                 double2* __restrict__ Jdot, double* __restrict__ partial) {
  extern __shared__ __align__(16) double s_acc[];  // HV: [warps][4L]
  const int I = L - 1;
  const int nv = 4 * L;
  const int tile = blockIdx.x % n_wtiles;
  const size_t pd = blockIdx.x / n_wtiles;  // dir * n_p + p
  const int ip = (int)(pd % n_p);
  const int iw = tile * kHvpThreads + threadIdx.x;
  const bool valid = iw < n_w;
  if (MODE == kHvpModeHv) {
    for (int k = threadIdx.x; k < (kHvpThreads / 32) * nv; k += blockDim.x) s_acc[k] = 0.0;
    __syncthreads();
  }
  cd w = mk(0.0, 0.0);
  if (valid) {
    const double2 wv = omega[iw];
    w = mk(wv.x, wv.y);
  }
  HvpSink<MODE> sink;
  sink.L = L;
  sink.valid = valid;
  sink.n_w = n_w;
  sink.row = s_acc + (threadIdx.x >> 5) * nv;
  sink.robs = mk(0.0, 0.0);
  if (MODE == kHvpModeHv && valid) {
    const double2 o = R_obs[(size_t)ip * n_w + iw];
    sink.robs = mk(o.x, o.y);
  }
  sink.jd = (MODE == kHvpModeJdot) ? Jdot + pd * (size_t)nv * n_w + (valid ? iw : 0) : nullptr;
  hvp_pair(L, w, free_surface != 0, lv_all + pd * L, ifs_all + pd * I, tan_all + (size_t)ip * I,
           tant_all + pd * I, sink);
  if (MODE == kHvpModeHv) {
    __syncthreads();
    double* dst = partial + (size_t)blockIdx.x * nv;  // blocks of one direction are contiguous
    for (int k = threadIdx.x; k < nv; k += blockDim.x) {
      double t = 0.0;
      for (int wi = 0; wi < kHvpThreads / 32; ++wi) t += s_acc[wi * nv + k];
      dst[k] = t;
    }
  }
}

// HV mode with the contraction moved out of the frequency loop: each warp sums the value and
// tangent parts of its lanes' per-step dual adjoints into its own rows (two row sets), the
// block contracts the summed rows once per (direction, p, interface).  Dynamic smem: per-warp
// value rows, tangent rows, staging tiles.
struct DualSumSink {
  bool valid;
  cd robs;
  cd* accv;  // this warp's value rows
  cd* acct;  // this warp's tangent rows
  cd* stage;
  int I;
  __device__ DC reflectivity(const DC& R) {
    if (!valid) return dc(mk(0.0, 0.0));
    const cd r = R.v - robs;
    return dc(mk(2.0 * r.x, -2.0 * r.y), mk(2.0 * R.t.x, -2.0 * R.t.y));
  }
  __device__ void add(int row, const DC v[kSumVals]) {
    cd x[kSumVals];
#pragma unroll
    for (int k = 0; k < kSumVals; ++k) x[k] = v[k].v;
    warp_add12<1>(x, stage, accv + (size_t)row * kSumVals);
#pragma unroll
    for (int k = 0; k < kSumVals; ++k) x[k] = v[k].t;
    warp_add12<1>(x, stage, acct + (size_t)row * kSumVals);
  }
  __device__ void top(const DC& f0) {
    DC v[kSumVals];
#pragma unroll
    for (int k = 0; k < kSumVals; ++k) v[k] = dc(mk(0.0, 0.0));
    v[10] = f0;
    add(I, v);
  }
  __device__ void step(int i, const DC cbar[10], const DC& fa, const DC& fb) {
    DC v[kSumVals];
#pragma unroll
    for (int k = 0; k < 10; ++k) v[k] = cbar[k];
    v[10] = fa;
    v[11] = fb;
    add(i, v);
  }
};

__global__ void __launch_bounds__(kHvpThreads, 1)
hvp_sum_kernel(int L, int n_p, const double2* __restrict__ omega, int n_w, int n_wtiles,
               int free_surface, const LayerV* __restrict__ lv_all,
               const IfS<DC>* __restrict__ ifs_all, const ScatTan* __restrict__ tan_all,
               const ScatTan* __restrict__ tant_all, const double2* __restrict__ R_obs,
               double* __restrict__ partial) {
  constexpr int W = kHvpThreads / 32;
  extern __shared__ __align__(16) double s_raw[];
  const int I = L - 1;
  const int nrow = (int)sum_rows(L) * kSumVals;
  const int tile = blockIdx.x % n_wtiles;
  const size_t pd = blockIdx.x / n_wtiles;  // dir * n_p + p
  const int ip = (int)(pd % n_p);
  const int iw = tile * kHvpThreads + threadIdx.x;
  const bool valid = iw < n_w;
  const int warp = threadIdx.x >> 5;
  cd* accv = reinterpret_cast<cd*>(s_raw);
  cd* acct = accv + (size_t)W * nrow;
  cd* stage = acct + (size_t)W * nrow;
  for (int k = threadIdx.x; k < 2 * W * nrow; k += blockDim.x) accv[k] = mk(0.0, 0.0);
  __syncthreads();
  cd w = mk(0.0, 0.0);
  if (valid) {
    const double2 wv = omega[iw];
    w = mk(wv.x, wv.y);
  }
  DualSumSink sink;
  sink.valid = valid;
  sink.robs = mk(0.0, 0.0);
  if (valid) {
    const double2 o = R_obs[(size_t)ip * n_w + iw];
    sink.robs = mk(o.x, o.y);
  }
  sink.accv = accv + (size_t)warp * nrow;
  sink.acct = acct + (size_t)warp * nrow;
  sink.stage = stage + warp * 32 * stage_stride<1>();
  sink.I = I;
  const LayerV* lv = lv_all + pd * L;
  hvp_pair_sums(L, w, free_surface != 0, lv, ifs_all + pd * I, sink);
  __syncthreads();
  for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
    cd a = accv[k], b = acct[k];
    for (int wi = 1; wi < W; ++wi) {
      a = a + accv[wi * nrow + k];
      b = b + acct[wi * nrow + k];
    }
    accv[k] = a;
    acct[k] = b;
  }
  __syncthreads();
  double* dst = partial + (size_t)blockIdx.x * (4 * L);
  for (int l = threadIdx.x; l < L; l += blockDim.x) {
    double v[4];
    hvp_sums_contract_layer(l, L, accv, acct, tan_all + (size_t)ip * I, tant_all + pd * I, lv, v);
    dst[0 * L + l] = v[0];
    dst[1 * L + l] = v[1];
    dst[2 * L + l] = v[2];
    dst[3 * L + l] = v[3];
  }
}

// Dynamic smem of hvp_sum_kernel (0 if it does not fit).
static size_t hvp_sum_smem(int L) {
  const size_t smem = sizeof(cd) * (size_t)(kHvpThreads / 32) *
                      (2 * sum_rows(L) * kSumVals + 32 * stage_stride<1>());
  return smem <= 160 * 1024 ? smem : 0;
}

// out[dir][k] = sum_b partial[dir][b][k]; grid (nv, n_dir), fixed-shape tree.
__global__ void __launch_bounds__(256)
hvp_reduce_kernel(const double* __restrict__ partial, int blocks_per_dir, int nv,
                  double* __restrict__ out) {
  __shared__ double s[256];
  const int k = blockIdx.x;
  const size_t dir = blockIdx.y;
  const double* src = partial + dir * (size_t)blocks_per_dir * nv;
  double t = 0.0;
  for (int b = threadIdx.x; b < blocks_per_dir; b += 256) t += src[(size_t)b * nv + k];
  s[threadIdx.x] = t;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[dir * nv + k] = s[0];
}

static kr_status hvp_args(const double* layers, int L, const double* p, int n_p,
                          const double* omega, int n_w, uint32_t flags, const double* V,
                          int n_dir) {
  if (n_p < 0 || n_w < 0 || n_dir < 0 || (flags & ~KR_FREE_SURFACE)) return KR_ERR_INVALID_ARGUMENT;
  if (L < 2) return KR_ERR_INVALID_MODEL;
  if (L > kMaxLayers) return KR_ERR_TOO_LARGE;
  if (L - 2 > kHvpSeg * kHvpCp) return KR_ERR_TOO_LARGE;
  if (n_p > 0 && n_w > 0 && n_dir > 0 && (!layers || !p || !omega || !V))
    return KR_ERR_INVALID_ARGUMENT;
  if (!aligned16(omega)) return KR_ERR_INVALID_ARGUMENT;
  return KR_OK;
}

template <int MODE>
static kr_status launch_hvp(const double* layers, int L, const double* p, int n_p,
                            const double* omega, int n_w, uint32_t flags, const double* R_obs,
                            const double* V, int n_dir, double* out, void* ws, size_t ws_bytes,
                            cudaStream_t st) {
  const int I = L - 1;
  const int n_wtiles = (n_w + kHvpThreads - 1) / kHvpThreads;
  const size_t per_dir = (size_t)n_p * n_wtiles;
  const size_t blocks = per_dir * n_dir;
  if (blocks > 0x7fffffffULL || per_dir > 0x7fffffffULL || n_dir > 65535) return KR_ERR_TOO_LARGE;
  HvpWs w = hvp_ws(ws, L, n_p, n_dir, per_dir, MODE == kHvpModeHv);
  if (!ws || ws_bytes < w.bytes) return KR_ERR_WORKSPACE;
  int nb = (n_p * L + 127) / 128;
  hvp_layer_kernel<<<nb, 128, 0, st>>>(layers, L, p, n_p, w.lay, w.dlay, w.d2);
  kr_status s = check_launch("kr_hvp: layers");
  if (s != KR_OK) return s;
  const unsigned nbi = (unsigned)(((size_t)n_p * I * 6 + 127) / 128);
  hvp_iface_kernel<<<nbi, 128, 0, st>>>(p, n_p, L, w.lay, w.dlay, w.coef, w.tan);
  s = check_launch("kr_hvp: interfaces");
  if (s != KR_OK) return s;
  size_t n = (size_t)n_dir * n_p * L;
  hvp_ldot_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(layers, L, n_p, n_dir, V, w.lay,
                                                               w.dlay, w.d2, w.lv);
  s = check_launch("kr_hvp: layer tangents");
  if (s != KR_OK) return s;
  n = (size_t)n_dir * n_p * I * 6;
  hvp_idot_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(p, L, n_p, n_dir, w.coef, w.lv, w.ifs,
                                                            w.tant);
  s = check_launch("kr_hvp: interface tangents");
  if (s != KR_OK) return s;
  if (MODE == kHvpModeHv) {
    const size_t ssm = hvp_sum_smem(L);
    if (ssm) {
      static SmemLimit slim;
      if (ssm > 48 * 1024) {
        s = raise_smem_limit((const void*)hvp_sum_kernel, ssm, slim, "kr_hvp: smem attribute");
        if (s != KR_OK) return s;
      }
      hvp_sum_kernel<<<(unsigned)blocks, kHvpThreads, ssm, st>>>(
          L, n_p, reinterpret_cast<const double2*>(omega), n_w, n_wtiles,
          (flags & KR_FREE_SURFACE) ? 1 : 0, w.lv, w.ifs, w.tan, w.tant,
          reinterpret_cast<const double2*>(R_obs), w.partial);
      s = check_launch("kr_hvp: sweep");
      if (s != KR_OK) return s;
      hvp_reduce_kernel<<<dim3(4 * L, n_dir), 256, 0, st>>>(w.partial, (int)per_dir, 4 * L, out);
      return check_launch("kr_hvp: reduce");
    }
  }
  const size_t smem = MODE == kHvpModeHv ? sizeof(double) * (kHvpThreads / 32) * 4 * (size_t)L : 0;
  static SmemLimit lim;
  if (smem > 48 * 1024) {
    s = raise_smem_limit((const void*)hvp_sweep_kernel<MODE>, smem, lim, "kr_hvp: smem attribute");
    if (s != KR_OK) return s;
  }
  hvp_sweep_kernel<MODE><<<(unsigned)blocks, kHvpThreads, smem, st>>>(
      L, n_p, n_dir, reinterpret_cast<const double2*>(omega), n_w, n_wtiles,
      (flags & KR_FREE_SURFACE) ? 1 : 0, w.lv, w.ifs, w.tan, w.tant,
      reinterpret_cast<const double2*>(R_obs),
      MODE == kHvpModeJdot ? reinterpret_cast<double2*>(out) : nullptr, w.partial);
  s = check_launch("kr_hvp: sweep");
  if (s != KR_OK || MODE != kHvpModeHv) return s;
  hvp_reduce_kernel<<<dim3(4 * L, n_dir), 256, 0, st>>>(w.partial, (int)per_dir, 4 * L, out);
  return check_launch("kr_hvp: reduce");
}

}  // namespace kr

using namespace kr;

extern "C" size_t kr_misfit_hvp_workspace_bytes(int32_t n_layers, int32_t n_p, int32_t n_w,
                                                int32_t n_dir) {
  if (n_layers < 2 || n_p <= 0 || n_w <= 0 || n_dir <= 0) return 0;
  const size_t per_dir = (size_t)n_p * ((n_w + kHvpThreads - 1) / kHvpThreads);
  return hvp_ws(nullptr, n_layers, n_p, n_dir, per_dir, true).bytes;
}

extern "C" kr_status kr_misfit_hvp(const double* layers, int32_t n_layers, const double* p,
                                   int32_t n_p, const double* omega, int32_t n_w, uint32_t flags,
                                   const double* R_obs, const double* V, int32_t n_dir, double* HV,
                                   void* workspace, size_t workspace_bytes, void* stream) {
  kr_status s = hvp_args(layers, n_layers, p, n_p, omega, n_w, flags, V, n_dir);
  if (s != KR_OK) return s;
  if (n_dir == 0) return KR_OK;
  if (!HV) return KR_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (n_p == 0 || n_w == 0) {
    cudaError_t e = cudaMemsetAsync(HV, 0, sizeof(double) * 4 * (size_t)n_layers * n_dir, st);
    if (e != cudaSuccess) set_last_error("kr_misfit_hvp: memset", e);
    return cuda_status(e);
  }
  if (!R_obs || !aligned16(R_obs)) return KR_ERR_INVALID_ARGUMENT;
  return launch_hvp<kHvpModeHv>(layers, n_layers, p, n_p, omega, n_w, flags, R_obs, V, n_dir, HV,
                                workspace, workspace_bytes, st);
}

extern "C" size_t kr_jacobian_dot_workspace_bytes(int32_t n_layers, int32_t n_p, int32_t n_w,
                                                  int32_t n_dir) {
  if (n_layers < 2 || n_p <= 0 || n_w <= 0 || n_dir <= 0) return 0;
  return hvp_ws(nullptr, n_layers, n_p, n_dir, 0, false).bytes;
}

extern "C" kr_status kr_jacobian_dot(const double* layers, int32_t n_layers, const double* p,
                                     int32_t n_p, const double* omega, int32_t n_w,
                                     uint32_t flags, const double* V, int32_t n_dir, double* Jdot,
                                     void* workspace, size_t workspace_bytes, void* stream) {
  kr_status s = hvp_args(layers, n_layers, p, n_p, omega, n_w, flags, V, n_dir);
  if (s != KR_OK) return s;
  if (n_dir == 0 || n_p == 0 || n_w == 0) return KR_OK;
  if (!Jdot || !aligned16(Jdot)) return KR_ERR_INVALID_ARGUMENT;
  return launch_hvp<kHvpModeJdot>(layers, n_layers, p, n_p, omega, n_w, flags, nullptr, V, n_dir,
                                  Jdot, workspace, workspace_bytes, (cudaStream_t)stream);
}
