// Discrete-wavenumber gather: Bessel-weighted slowness sum and the omega -> t step.
//
// kr_bessel_sum: one thread per (offset, omega) and slowness slice.  Blocks are
// 32 frequencies x 8 offsets; the slowness range is split into slices (grid.x) so the grid
// fills the 148 SMs several times over; each slice writes its partial U to the workspace and
// a second kernel adds the slices in a fixed order (bit-reproducible).  J0 is evaluated on
// the fly in registers (FP64): Hankel's asymptotic expansion above x = 25 with cos/sin
// carried along the slowness loop by rotation (exact anchors every 32 steps), a piecewise
// Taylor table below; R[p][omega] arrives through shared memory in tiles of 32 slownesses
// x 32 frequencies (cp.async, a ring of three) shared by the block's 8 offsets.
//
// kr_traces: builds the half spectrum conj(U S) (DC and Nyquist zero) and runs a batched
// cuFFT Z2D: for a Hermitian spectrum H, the forward DFT the reference applies
// (np.fft.fft) equals the inverse real transform of conj(H).  The decay exp(-gamma t) is
// applied by a last elementwise kernel.
#include <cufft.h>
#include <stdio.h>

#include <mutex>
#include <vector>

#include "kr_internal.cuh"
#include "kr_j0_table.h"

namespace kr {

constexpr int kBsW = 32;  // frequencies per block
constexpr int kBsR = 8;   // offsets per block

// ---------------------------------------------------------------------------------------
// J0 for large arguments: Hankel's asymptotic expansion (Abramowitz & Stegun 9.2.5,
// 9.2.9-9.2.10) with the coefficients a_k(0) = prod_{j=1..k} (-(2j-1)^2) / (k! 8^k):
//   J0(x) = sqrt(2 / (pi x)) [P(x) cos(x - pi/4) - Q(x) sin(x - pi/4)]
//         = sqrt(1 / (pi x)) [(P + Q) cos x + (P - Q) sin x],
//   P = sum_m (-1)^m a_{2m} x^{-2m},  Q = sum_m (-1)^m a_{2m+1} x^{-2m-1}.
// With 7 terms each the truncation error is below 7e-16 absolute for x >= 25 (checked
// against SciPy's j0); below 25 the kernel uses the Taylor table of kr_j0_table.h.
// ---------------------------------------------------------------------------------------
constexpr double kJ0X0 = 25.0;
constexpr int kJ0Terms = 7;

__host__ __device__ constexpr double hankel_a(int k) {
  double num = 1.0, den = 1.0;
  for (int j = 1; j <= k; ++j) {
    num *= -(double)((2 * j - 1) * (2 * j - 1));
    den *= 8.0 * j;
  }
  return num / den;
}
__host__ __device__ constexpr double hankel_p(int m) { return (m % 2 ? -1.0 : 1.0) * hankel_a(2 * m); }
__host__ __device__ constexpr double hankel_q(int m) { return (m % 2 ? -1.0 : 1.0) * hankel_a(2 * m + 1); }

// sqrt(pi x) J0(x) = P u + Q v with u = cos x + sin x, v = cos x - sin x, y = 1 / x and
// the first NT terms of P and Q.  The first omitted terms bound the truncation error
// (A&S 9.2.10); the absolute J0 error is below 7e-16 for NT = 7 at x >= 25 and below 1e-16
// for NT = 5 at x >= 60, NT = 4 at x >= 100, NT = 3 at x >= 300 and NT = 2 at x >= 3000.
template <int NT>
__device__ __forceinline__ double j0_asym_scaled(double y, double u, double v) {
  const double q = y * y;
  double P = hankel_p(NT - 1), Qs = hankel_q(NT - 1);
#pragma unroll
  for (int m = NT - 2; m >= 0; --m) {
    P = fma(P, q, hankel_p(m));
    Qs = fma(Qs, q, hankel_q(m));
  }
  return fma(P, u, Qs * (y * v));
}

// J0(x) for x >= kJ0X0 given c = cos x, s = sin x.
__device__ __forceinline__ double j0_asymptotic(double x, double c, double s) {
  const double amp = rsqrt(3.14159265358979323846 * x);  // sqrt(1 / (pi x))
  const double y = 3.14159265358979323846 * (amp * amp);  // 1 / x
  const double q = y * y;
  double P = hankel_p(kJ0Terms - 1), Q = hankel_q(kJ0Terms - 1);
#pragma unroll
  for (int m = kJ0Terms - 2; m >= 0; --m) {
    P = fma(P, q, hankel_p(m));
    Q = fma(Q, q, hankel_q(m));
  }
  Q *= y;
  return amp * fma(P + Q, c, (P - Q) * s);
}

// J0(x) for 0 <= x < 25 from the piecewise Taylor table (kr_j0_table.h, staged in shared
// memory with rows padded to kJ0Row doubles so that lanes on different intervals fall on
// different banks): interval k = floor(x), t = x - (k + 1/2), degree-15 Horner in t.
// Absolute error below 5e-16 against SciPy's j0 on [0, 25).
constexpr int kJ0Row = kJ0TabDegree + 2;
__device__ __forceinline__ double j0_table(const double* s_j0, double x) {
  const int k = min((int)x, kJ0TabIntervals - 1);
  const double t = x - ((double)k + 0.5);
  const double* a = s_j0 + k * kJ0Row;
  double v = a[kJ0TabDegree];
#pragma unroll
  for (int n = kJ0TabDegree - 1; n >= 0; --n) v = fma(v, t, a[n]);
  return v;
}

// Slowness steps between exact sincos anchors when p is an arithmetic progression.
constexpr int kRotSteps = 32;
// Slownesses staged per shared-memory chunk: (p_j, pw_j dp) and (1 / p_j, pw_j dp / sqrt p_j).
constexpr int kChunk = 128;

// R rows are staged through shared memory in tiles of kSub slownesses x 32 frequencies
// (16 KB) in a ring of three with cp.async: the 8 offset warps of a block read each R
// element from shared memory instead of each loading it from L1 / L2, two tiles are in
// flight while one is summed, and one block barrier per tile suffices (the barrier that
// publishes tile t also shows every warp done with tile t - 1, whose buffer then takes
// tile t + 2).  kSub equals the rotation anchor spacing.
constexpr int kSub = kRotSteps;
constexpr int kRing = 3;
constexpr size_t kRingBytes = sizeof(double2) * kRing * kSub * kBsW;  // dynamic shared memory

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gmem),
               "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::); }

// Block-cooperative: R rows [j0, j0 + ns) x frequencies [iw0, iw0 + 32) into `tile`,
// zero-filled (no global read) outside the grid.  Warp ty copies rows ty, ty + 8, ...;
// lane copies frequency iw0 + lane (one coalesced 512-byte row per warp and copy).
__device__ __forceinline__ void stage_R(double2 (*tile)[kBsW], const double2* __restrict__ R,
                                        int j0, int ns, int iw0, int n_w) {
  const int ty = threadIdx.y, lane = threadIdx.x;
  const bool col_ok = iw0 + lane < n_w;
  const double2* src = R + (size_t)(j0 + ty) * n_w + iw0 + lane;
  const size_t stride = (size_t)kBsR * n_w;
#pragma unroll
  for (int i = 0; i < kSub / kBsR; ++i) {
    const int row = ty + i * kBsR;
    const bool ok = col_ok && row < ns;
    cp_async16(&tile[row][lane], ok ? src + i * stride : R, ok ? 16 : 0);
  }
}

// Terms of one staged tile for one thread on the fast path: exact cos / sin anchor at the
// tile's first slowness, rotation of (u, v) = (cos + sin, cos - sin) in between.  The
// amplitude 1 / sqrt(pi omega r) is common to the thread and applied to (ax, ay) by the
// caller; 1 / sqrt(p_j) is staged.
template <int NT, int M>
__device__ __forceinline__ void fast_terms(const double2* __restrict__ ig_p,
                                           const double2* __restrict__ r_p, int m, double inv_omr,
                                           double cdl, double sd, double& u, double& v,
                                           double& ax, double& ay) {
#pragma unroll 8
  for (int k = 0; k < (M > 0 ? M : m); ++k) {
    const double2 ig = ig_p[k];
    const double2 rv = r_p[k * kBsW];
    const double t = j0_asym_scaled<NT>(ig.x * inv_omr, u, v) * ig.y;
    const double u2 = fma(u, cdl, v * sd);
    v = fma(v, cdl, -u * sd);
    u = u2;
    ax = fma(t, rv.x, ax);
    ay = fma(t, rv.y, ay);
  }
}

template <int NT>
__device__ __forceinline__ void fast_tile(const double2* s_pf, const double2* s_ig,
                                          const double2 (*tile)[kBsW], int k0, int m, int lane,
                                          double om, double r, double inv_omr, double cdl,
                                          double sd, double& ax, double& ay) {
  double s, c;
  sincos((om * s_pf[k0].x) * r, &s, &c);
  double u = c + s, v = c - s;
  // full tiles run a loop of compile-time length (no remainder handling)
  if (m == kSub)
    fast_terms<NT, kSub>(s_ig + k0, &tile[0][lane], kSub, inv_omr, cdl, sd, u, v, ax, ay);
  else
    fast_terms<NT, 0>(s_ig + k0, &tile[0][lane], m, inv_omr, cdl, sd, u, v, ax, ay);
}

// One thread per (omega, offset) and slowness slice.  Grid: x = slowness slice, y = offset
// group, z = frequency tile, so the hardware starts the low-frequency tiles (small J0
// arguments, the slowest blocks) first and the cheap high-frequency tiles fill the tail.
// Per chunk of the slice the block stages (p_j, pw_j dp) and (1 / p_j, pw_j dp / sqrt p_j)
// in shared memory and checks once whether the chunk continues the slice's arithmetic
// progression (to 4.5 ulp); inside such a chunk cos / sin of x_j = (omega p_j) r advance by
// one rotation per slowness, with an exact sincos anchor every kRotSteps.  R arrives in
// tiles through a ring of three buffers (stage_R).  omega is factored out of the weight:
// U = omega * sum_j J0(x_j) (pw_j dp) R_j.  Four blocks of 256 threads per SM (64 registers,
// 40 bytes of spills; 128-slowness chunks keep four blocks' shared memory within the SM's
// 228 KB): the kernel is bound by each warp's dependency chains, so more resident warps
// help despite the spills (21-layer gather grid: 2.98 ms at two blocks and 124 registers,
// 2.65 at three and 80, 2.635 at four, U bit-identical).
__global__ void __launch_bounds__(kBsW * kBsR, 4)
bessel_partial_kernel(const double2* __restrict__ R, const double* __restrict__ p,
                      const double* __restrict__ pw, int n_p, double dp,
                      const double* __restrict__ omega, int n_w,
                      const double* __restrict__ offsets, int n_r, int p_per_slice,
                      double2* __restrict__ partial) {
  __shared__ double2 s_pf[kChunk];  // (p_j, pw_j dp)
  __shared__ double2 s_ig[kChunk];  // (1 / p_j, pw_j dp / sqrt(p_j))
  __shared__ double s_j0[kJ0TabIntervals * kJ0Row];
  extern __shared__ __align__(16) unsigned char s_dyn[];
  double2(*s_R)[kSub][kBsW] = reinterpret_cast<double2(*)[kSub][kBsW]>(s_dyn);  // [kRing]
  const int tid = threadIdx.y * kBsW + threadIdx.x;
  for (int e = tid; e < kJ0TabIntervals * kJ0Row; e += kBsW * kBsR) {
    const int k = e / kJ0Row, n = e - k * kJ0Row;
    s_j0[e] = n <= kJ0TabDegree ? kJ0Taylor[k][n] : 0.0;  // made visible by the chunk barrier
  }
  const int lane = threadIdx.x;
  const int iw0 = blockIdx.z * kBsW;
  const int iw = iw0 + lane;
  const int ir = blockIdx.y * kBsR + threadIdx.y;
  const int j_begin = blockIdx.x * p_per_slice;
  const int j_end = min(n_p, j_begin + p_per_slice);
  const bool active = iw < n_w && ir < n_r;
  const double om = active ? omega[iw] : 0.0;
  const double r = active ? offsets[ir] : 0.0;
  const double omr = om * r;
  // per-thread factors of 1 / x and sqrt(1 / (pi x)) with x = omr p (used where x >= 25)
  const double inv_omr = omr > 0.0 ? 1.0 / omr : 0.0;
  const double isq_pomr = omr > 0.0 ? rsqrt(3.14159265358979323846 * omr) : 0.0;
  // Linear model of the slice's slownesses: p_j ~ p0 + (j - j_begin) * step.
  const double p0 = __ldg(p + j_begin);
  const double step =
      (j_end - j_begin >= 2) ? (__ldg(p + j_end - 1) - p0) / (double)(j_end - 1 - j_begin) : 0.0;
  double sd, cdl;
  sincos(omr * step, &sd, &cdl);
  double c = 0.0, s = 0.0;
  int since = kRotSteps;  // steps since the last exact anchor (kRotSteps: none valid)
  double ax = 0.0, ay = 0.0;  // fast-path terms, without the factor 1 / sqrt(pi omega r)
  double bx = 0.0, by = 0.0;  // other terms, complete
  for (int jc = j_begin; jc < j_end; jc += kChunk) {
    const int n = min(kChunk, j_end - jc);
    __syncthreads();  // the previous chunk's readers of s_pf, s_ig, s_R are done
    bool ok = true;
    if (tid < n) {
      const int j = jc + tid;
      const double pj = __ldg(p + j);
      const double f = __ldg(pw + j) * dp;
      s_pf[tid] = make_double2(pj, f);
      s_ig[tid] = make_double2(1.0 / pj, f * rsqrt(pj));
      const double lin = fma((double)(j - j_begin), step, p0);
      ok = fabs(pj - lin) <= 1e-15 * fabs(pj);
    }
    const int nsub = (n + kSub - 1) / kSub;
    // tiles 0 and 1 now, tile sb + 2 in iteration sb; every thread commits one group per
    // step (empty ones included), so wait_group 1 at iteration sb means tile sb has landed
    stage_R(s_R[0], R, jc, min(kSub, n), iw0, n_w);
    cp_async_commit();
    if (nsub > 1) stage_R(s_R[1], R, jc + kSub, min(kSub, n - kSub), iw0, n_w);
    cp_async_commit();
    const bool uniform = __syncthreads_and(ok) != 0;
    if (!uniform) since = kRotSteps;
    const bool rising = active && uniform && step > 0.0 && omr > 0.0;
    for (int sb = 0; sb < nsub; ++sb) {
      cp_async_wait_1();  // this thread's copies of tile sb have landed
      __syncthreads();    // ... and every thread's; every thread is done with tile sb - 1
      if (sb + 2 < nsub)
        stage_R(s_R[(sb + 2) % kRing], R, jc + (sb + 2) * kSub,
                min(kSub, n - (sb + 2) * kSub), iw0, n_w);
      cp_async_commit();
      const double2(*tile)[kBsW] = s_R[sb % kRing];
      const int k0 = sb * kSub, m = min(kSub, n - k0);
      // Fast tile: slownesses in arithmetic progression with x increasing from >= 25, so
      // every term takes the asymptotic branch with the anchor / rotation scheme (no
      // data-dependent branches in the inner loop).  The number of expansion terms follows
      // from the tile's smallest argument.
      const double x_first = (om * s_pf[k0].x) * r;
      const bool fast = rising && x_first >= kJ0X0;
      const int nt = x_first >= 3000.0 ? 2 : x_first >= 300.0 ? 3 : x_first >= 100.0 ? 4
                   : x_first >= 60.0 ? 5 : 7;
      if (fast) {
        since = kRotSteps;
        switch (nt) {
          case 2: fast_tile<2>(s_pf, s_ig, tile, k0, m, lane, om, r, inv_omr, cdl, sd, ax, ay); break;
          case 3: fast_tile<3>(s_pf, s_ig, tile, k0, m, lane, om, r, inv_omr, cdl, sd, ax, ay); break;
          case 4: fast_tile<4>(s_pf, s_ig, tile, k0, m, lane, om, r, inv_omr, cdl, sd, ax, ay); break;
          case 5: fast_tile<5>(s_pf, s_ig, tile, k0, m, lane, om, r, inv_omr, cdl, sd, ax, ay); break;
          default: fast_tile<7>(s_pf, s_ig, tile, k0, m, lane, om, r, inv_omr, cdl, sd, ax, ay); break;
        }
      } else if (active) {
        // not unrolled: fewer spills at 64 registers, 2.593 vs 2.615 ms (unroll 4) and
        // 2.723 (unroll 8) on the 21-layer gather grid, U bit-identical
#pragma unroll 1
        for (int k = 0; k < m; ++k) {
          const double2 pf = s_pf[k0 + k];
          const double2 rv = tile[k][lane];
          const double x = (om * pf.x) * r;
          double jv;
          if (x < kJ0X0) {
            jv = x > -kJ0X0 ? j0_table(s_j0, fabs(x)) : j0(x);
            since = kRotSteps;
          } else {
            if (since < kRotSteps) {
              const double c2 = fma(c, cdl, -s * sd);
              s = fma(s, cdl, c * sd);
              c = c2;
              ++since;
            } else {
              sincos(x, &s, &c);
              since = uniform ? 1 : kRotSteps;
            }
            jv = j0_asymptotic(x, c, s);
          }
          const double t = jv * pf.y;
          bx = fma(t, rv.x, bx);
          by = fma(t, rv.y, by);
        }
      }
    }
  }
  if (active)
    partial[((size_t)blockIdx.x * n_r + ir) * n_w + iw] =
        make_double2(fma(ax, isq_pomr, bx) * om, fma(ay, isq_pomr, by) * om);
}

__global__ void reduce_slices_kernel(const double2* __restrict__ partial, int n_slices,
                                     size_t n_elem, double2* __restrict__ U) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_elem;
       i += (size_t)gridDim.x * blockDim.x) {
    double x = 0.0, y = 0.0;
    for (int s = 0; s < n_slices; ++s) {
      double2 v = partial[(size_t)s * n_elem + i];
      x += v.x;
      y += v.y;
    }
    U[i] = make_double2(x, y);
  }
}

// The R ring lives in dynamic shared memory above the 48 KB default (with the static arrays
// ~56 KB per block, four blocks per SM); the limit is raised once per device.
static SmemLimit g_ring_limit;
static kr_status bessel_ring_attribute(const char* where) {
  return raise_smem_limit((const void*)bessel_partial_kernel, kRingBytes, g_ring_limit, where);
}

struct BesselPlan {
  int n_slices;
  int p_per_slice;
  size_t partial_bytes;
};

static BesselPlan bessel_plan(int n_p, int n_w, int n_r) {
  BesselPlan b;
  const long long tiles = (long long)((n_w + kBsW - 1) / kBsW) * ((n_r + kBsR - 1) / kBsR);
  // About 96 blocks of 256 threads per SM in total (~24 waves at 4 resident blocks per SM:
  // shorter blocks even out the slow low-frequency tiles; on the 21-layer gather grid
  // 2.612 ms against 2.633 at 64 and 2.623 at 128; with three resident blocks 2.65 at 64,
  // 2.73 at 32, 2.85 at 16), but no slice shorter than 64 slownesses.
  const long long target = 148LL * 96;
  long long s = (target + tiles - 1) / (tiles > 0 ? tiles : 1);
  long long smax = (n_p + 63) / 64;
  if (s > smax) s = smax;
  if (s < 1) s = 1;
  if (s > 65535) s = 65535;
  b.p_per_slice = (int)((n_p + s - 1) / s);
  b.n_slices = (int)((n_p + b.p_per_slice - 1) / b.p_per_slice);
  if (b.n_slices < 1) b.n_slices = 1;
  b.partial_bytes = (size_t)b.n_slices * n_r * n_w * sizeof(double2);
  return b;
}

// ---------------------------------------------------------------------------------------
// Traces
// ---------------------------------------------------------------------------------------
__global__ void half_spectrum_kernel(const double2* __restrict__ U, const double2* __restrict__ S,
                                     int n_r, int nw, double2* __restrict__ X) {
  const int nh = nw + 1;
  const size_t n = (size_t)n_r * nh;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / nh);
    const int k = (int)(i % nh);
    double2 v = make_double2(0.0, 0.0);
    if (k >= 1 && k <= nw - 1) {
      double2 u = U[(size_t)r * (nw - 1) + (k - 1)];
      if (S) {
        double2 s = S[k - 1];
        cd y = mk(u.x, u.y) * mk(s.x, s.y);
        u = make_double2(y.x, y.y);
      }
      v = make_double2(u.x, -u.y);
    }
    X[i] = v;
  }
}

__global__ void decay_kernel(double* __restrict__ tr, const double* __restrict__ decay, int n_r,
                             int nt) {
  const size_t n = (size_t)n_r * nt;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    tr[i] *= decay[i % nt];
}

struct FftEntry {
  int device;
  int nt;
  int batch;
  cufftHandle plan;
  size_t work;
};

static std::mutex g_fft_mu;
static std::vector<FftEntry> g_fft;

// Returns a cached C2R plan (auto work-area allocation off) for nt-point transforms.
static kr_status get_fft_plan(int nt, int batch, FftEntry** out) {
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) {
    set_last_error("kr_traces: cudaGetDevice", ce);
    return KR_ERR_CUDA;
  }
  for (auto& e : g_fft)
    if (e.device == dev && e.nt == nt && e.batch == batch) {
      *out = &e;
      return KR_OK;
    }
  FftEntry e;
  e.device = dev;
  e.nt = nt;
  e.batch = batch;
  if (cufftCreate(&e.plan) != CUFFT_SUCCESS) return KR_ERR_CUFFT;
  if (cufftSetAutoAllocation(e.plan, 0) != CUFFT_SUCCESS) {
    cufftDestroy(e.plan);
    return KR_ERR_CUFFT;
  }
  int n = nt;
  if (cufftMakePlanMany(e.plan, 1, &n, nullptr, 1, nt / 2 + 1, nullptr, 1, nt, CUFFT_Z2D, batch,
                        &e.work) != CUFFT_SUCCESS) {
    cufftDestroy(e.plan);
    set_last_error_msg("kr_traces: cufftMakePlanMany failed");
    return KR_ERR_CUFFT;
  }
  g_fft.push_back(e);
  *out = &g_fft.back();
  return KR_OK;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace kr

using namespace kr;

extern "C" size_t kr_bessel_sum_workspace_bytes(int32_t n_p, int32_t n_w, int32_t n_r) {
  if (n_p <= 0 || n_w <= 0 || n_r <= 0) return 0;
  return bessel_plan(n_p, n_w, n_r).partial_bytes;
}

extern "C" kr_status kr_bessel_sum(const double* R, const double* p, const double* pw,
                                   int32_t n_p, double dp, const double* omega, int32_t n_w,
                                   const double* offsets, int32_t n_r, double* U,
                                   void* workspace, size_t workspace_bytes, void* stream) {
  if (n_p < 0 || n_w < 0 || n_r < 0) return KR_ERR_INVALID_ARGUMENT;
  if (n_w == 0 || n_r == 0) return KR_OK;
  if (!U || !omega || !offsets) return KR_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (n_p == 0) {
    cudaError_t e = cudaMemsetAsync(U, 0, (size_t)n_r * n_w * sizeof(double2), st);
    if (e != cudaSuccess) set_last_error("kr_bessel_sum: memset", e);
    return cuda_status(e);
  }
  if (!R || !p || !pw) return KR_ERR_INVALID_ARGUMENT;
  if (!aligned16(R) || !aligned16(U)) return KR_ERR_INVALID_ARGUMENT;
  if ((n_r + kBsR - 1) / kBsR > 65535 || (n_w + kBsW - 1) / kBsW > 65535)
    return KR_ERR_TOO_LARGE;
  BesselPlan b = bessel_plan(n_p, n_w, n_r);
  if (!workspace || workspace_bytes < b.partial_bytes) return KR_ERR_WORKSPACE;
  double2* partial = reinterpret_cast<double2*>(workspace);
  dim3 grid(b.n_slices, (n_r + kBsR - 1) / kBsR, (n_w + kBsW - 1) / kBsW);
  kr_status a = bessel_ring_attribute("kr_bessel_sum");
  if (a != KR_OK) return a;
  bessel_partial_kernel<<<grid, dim3(kBsW, kBsR), kRingBytes, st>>>(
      reinterpret_cast<const double2*>(R), p, pw, n_p, dp, omega, n_w, offsets, n_r,
      b.p_per_slice, partial);
  kr_status s = check_launch("kr_bessel_sum: partial");
  if (s != KR_OK) return s;
  const size_t n_elem = (size_t)n_r * n_w;
  int blocks = (int)((n_elem + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  reduce_slices_kernel<<<blocks, 256, 0, st>>>(partial, b.n_slices, n_elem,
                                               reinterpret_cast<double2*>(U));
  return check_launch("kr_bessel_sum: reduce");
}

extern "C" size_t kr_traces_workspace_bytes(int32_t n_r, int32_t nw) {
  if (n_r <= 0 || nw <= 1) return 0;
  std::lock_guard<std::mutex> lk(g_fft_mu);
  FftEntry* e = nullptr;
  if (get_fft_plan(2 * nw, n_r, &e) != KR_OK) return 0;
  return align256((size_t)n_r * (nw + 1) * sizeof(double2)) + e->work;
}

extern "C" kr_status kr_traces(const double* U, const double* S, int32_t n_r, int32_t nw,
                               const double* decay, double* traces, void* workspace,
                               size_t workspace_bytes, void* stream) {
  if (n_r < 0 || nw < 0) return KR_ERR_INVALID_ARGUMENT;
  if (n_r == 0) return KR_OK;
  if (nw < 2) return KR_ERR_INVALID_ARGUMENT;
  if (!U || !traces) return KR_ERR_INVALID_ARGUMENT;
  if (!aligned16(U) || (S && !aligned16(S))) return KR_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  std::lock_guard<std::mutex> lk(g_fft_mu);
  FftEntry* e = nullptr;
  kr_status s = get_fft_plan(2 * nw, n_r, &e);
  if (s != KR_OK) return s;
  const size_t xbytes = align256((size_t)n_r * (nw + 1) * sizeof(double2));
  if (!workspace || workspace_bytes < xbytes + e->work) return KR_ERR_WORKSPACE;
  double2* X = reinterpret_cast<double2*>(workspace);
  void* work = static_cast<unsigned char*>(workspace) + xbytes;
  const size_t nx = (size_t)n_r * (nw + 1);
  int blocks = (int)((nx + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  half_spectrum_kernel<<<blocks, 256, 0, st>>>(reinterpret_cast<const double2*>(U),
                                               reinterpret_cast<const double2*>(S), n_r, nw, X);
  s = check_launch("kr_traces: half spectrum");
  if (s != KR_OK) return s;
  if (cufftSetStream(e->plan, st) != CUFFT_SUCCESS) return KR_ERR_CUFFT;
  if (e->work && cufftSetWorkArea(e->plan, work) != CUFFT_SUCCESS) return KR_ERR_CUFFT;
  if (cufftExecZ2D(e->plan, reinterpret_cast<cufftDoubleComplex*>(X), traces) != CUFFT_SUCCESS) {
    set_last_error_msg("kr_traces: cufftExecZ2D failed");
    return KR_ERR_CUFFT;
  }
  if (decay) {
    const size_t nt_all = (size_t)n_r * 2 * nw;
    int b2 = (int)((nt_all + 255) / 256);
    if (b2 > 148 * 16) b2 = 148 * 16;
    decay_kernel<<<b2, 256, 0, st>>>(traces, decay, n_r, 2 * nw);
    return check_launch("kr_traces: decay");
  }
  return KR_OK;
}

// ---------------------------------------------------------------------------------------
// Allocation-free variant of kr_bessel_sum.
//
// Some callers cannot allocate device memory at all: a host application that reserved the
// whole GPU in its own pool at start-up and hands out only pointers, a processing system
// that reaches this library through a C/Fortran FFI with device buffers owned by another
// component, or a loop that must not hit cudaMalloc's implicit device synchronisation.
// They pass inputs and the output only; the slice partials live in this file-scope device
// array instead of a caller workspace.  Every GPU that loads the library holds the array
// (16 MiB) until the process exits.
// ---------------------------------------------------------------------------------------
namespace kr {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_bessel_scratch[kNoAllocScratchBytes];

static std::mutex g_scratch_mu;
struct ScratchSlot {
  void* ctx;   // the context the address belongs to
  void* addr;  // device address of g_bessel_scratch in that context
};
static ScratchSlot g_scratch[kMaxDevices];

// cuCtxGetCurrent through the runtime's driver entry-point table (no link against libcuda).
typedef int (*CtxGetCurrentFn)(void**);
static CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(f);
  }
  return fn;
}

// Device address of g_bessel_scratch in the current device's current context.  The
// host-side symbol is only a stand-in, so the address is looked up (with that device
// current) on the first call per device and again whenever the device's context has changed
// since (cudaDeviceReset makes a new primary context, in which the array lives elsewhere).
static kr_status scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error("kr_bessel_sum_noalloc: cudaGetDevice", e);
    return KR_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_last_error_msg("kr_bessel_sum_noalloc: device index beyond 63");
    return KR_ERR_TOO_LARGE;
  }
  void* ctx = nullptr;
  CtxGetCurrentFn get = ctx_get_current();
  if (get) get(&ctx);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  ScratchSlot& slot = g_scratch[dev];
  if (!slot.addr || !ctx || slot.ctx != ctx) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_bessel_scratch);
    if (e != cudaSuccess || !ptr) {
      set_last_error("kr_bessel_sum_noalloc: cudaGetSymbolAddress", e);
      return KR_ERR_CUDA;
    }
    if (!ctx && get) get(&ctx);  // the lookup made the primary context current
    slot.addr = ptr;
    slot.ctx = ctx;
  }
  *out = slot.addr;
  return KR_OK;
}

}  // namespace kr

extern "C" size_t kr_bessel_sum_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

extern "C" kr_status kr_bessel_sum_noalloc(const double* R, const double* p, const double* pw,
                                           int32_t n_p, double dp, const double* omega,
                                           int32_t n_w, const double* offsets, int32_t n_r,
                                           double* U, void* stream) {
  if (n_p < 0 || n_w < 0 || n_r < 0) return KR_ERR_INVALID_ARGUMENT;
  if (n_w == 0 || n_r == 0) return KR_OK;
  if (!U || !omega || !offsets) return KR_ERR_INVALID_ARGUMENT;
  const size_t slice_bytes = (size_t)n_r * n_w * sizeof(double2);
  if (slice_bytes > kNoAllocScratchBytes) {
    char buf[200];
    snprintf(buf, sizeof buf,
             "kr_bessel_sum_noalloc: n_r * n_w = %lld exceeds the static scratch "
             "(16 MiB holds n_r * n_w <= %lld)",
             (long long)n_r * n_w, (long long)(kNoAllocScratchBytes / sizeof(double2)));
    set_last_error_msg(buf);
    return KR_ERR_TOO_LARGE;
  }
  if ((n_r + kBsR - 1) / kBsR > 65535 || (n_w + kBsW - 1) / kBsW > 65535)
    return KR_ERR_TOO_LARGE;
  cudaStream_t st = (cudaStream_t)stream;
  if (n_p == 0) {
    cudaError_t e = cudaMemsetAsync(U, 0, (size_t)n_r * n_w * sizeof(double2), st);
    if (e != cudaSuccess) set_last_error("kr_bessel_sum_noalloc: memset", e);
    return cuda_status(e);
  }
  if (!R || !p || !pw) return KR_ERR_INVALID_ARGUMENT;
  if (!aligned16(R) || !aligned16(U)) return KR_ERR_INVALID_ARGUMENT;
  void* scratch = nullptr;
  kr_status s = scratch_address(&scratch);
  if (s != KR_OK) return s;
  // As many slowness slices as the occupancy target asks for and the scratch holds.  Each
  // slice element is written by exactly one thread before the reduction reads it, so the
  // array needs no clearing between calls.
  BesselPlan b = bessel_plan(n_p, n_w, n_r);
  const int cap = (int)(kNoAllocScratchBytes / slice_bytes);
  int n_slices = b.n_slices < cap ? b.n_slices : cap;
  const int p_per_slice = (n_p + n_slices - 1) / n_slices;
  n_slices = (n_p + p_per_slice - 1) / p_per_slice;
  double2* partial = reinterpret_cast<double2*>(scratch);
  dim3 grid(n_slices, (n_r + kBsR - 1) / kBsR, (n_w + kBsW - 1) / kBsW);
  s = bessel_ring_attribute("kr_bessel_sum_noalloc");
  if (s != KR_OK) return s;
  bessel_partial_kernel<<<grid, dim3(kBsW, kBsR), kRingBytes, st>>>(
      reinterpret_cast<const double2*>(R), p, pw, n_p, dp, omega, n_w, offsets, n_r,
      p_per_slice, partial);
  s = check_launch("kr_bessel_sum_noalloc: partial");
  if (s != KR_OK) return s;
  const size_t n_elem = (size_t)n_r * n_w;
  int blocks = (int)((n_elem + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  reduce_slices_kernel<<<blocks, 256, 0, st>>>(partial, n_slices, n_elem,
                                               reinterpret_cast<double2*>(U));
  return check_launch("kr_bessel_sum_noalloc: reduce");
}
