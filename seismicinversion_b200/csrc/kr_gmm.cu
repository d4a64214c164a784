// Global Matrix Method reflectivity with the block-Riccati sweep: an independent FP64
// evaluation of R(omega, p) behind the same boundary as kr_reflectivity.
//
// Follows tmnestor/SeismicInversion, GlobalMatrix/:
//   layer eigenvectors     layer_matrix.py:201-258 (E_d, E_u 4x2; ocean e_d, e_u)
//   Riccati sweep          riccati_solver.py:200-283 (E_eff = E_d + E_u diag(ph) Y,
//                          F = [E_u | -E_eff], F X = -E_d diag(ph), Y = X[0:2])
//   ocean extraction       riccati_solver.py:297-330
//   entry point            gmm_torch.py:229-305 (R / (1 + R) with the free surface)
//
// One thread per (omega, p), one slowness per block (the layout of reflectivity_kernel):
// the block prologue puts the layer terms, the eigenvector terms of every layer and the
// phase table in shared memory.  The 4x4 complex systems are solved by Gaussian elimination
// with partial pivoting on |Re| + |Im| (the pivot rule of the LAPACK solve the reference
// calls), fully unrolled so that row exchanges are register selects, not indexed memory.
#include <stdlib.h>

#include "kr_phase.cuh"

namespace kr {

constexpr int kGmmThreads = 128;
static_assert(kGmmThreads == kPhTile, "one tile is one phase-table tile");

// Eigenvector terms of one solid layer (p real):
//   E_d = [[p, neta], [eta, -p], [-gamma, a], [b, gamma]],
//   E_u = [[p, -neta], [-eta, -p], [-gamma, -a], [-b, gamma]],
// gamma = rho (1 - 2 beta_c^2 p^2), a = 2 mu p neta, b = 2 mu p eta, mu = rho beta_c^2.
struct LayerG {
  cd eta, neta, gamma, a, b;
};

KR_HD LayerG gmm_layer(const LayerP& lp, double p) {
  const cd cp = mk(p, 0.0);
  const cd crho = mk(lp.rho, 0.0);
  const cd mu = (crho * lp.betac) * lp.betac;
  LayerG g;
  g.eta = lp.eta;
  g.neta = lp.neta;
  g.gamma = crho * (1.0 - ((2.0 * lp.betac) * lp.betac) * cp * cp);
  g.a = ((2.0 * mu) * cp) * lp.neta;
  g.b = ((2.0 * mu) * cp) * lp.eta;
  return g;
}

__device__ __forceinline__ void e_down(const LayerG& g, double p, cd E[4][2]) {
  E[0][0] = mk(p, 0.0);
  E[0][1] = g.neta;
  E[1][0] = g.eta;
  E[1][1] = mk(-p, 0.0);
  E[2][0] = -g.gamma;
  E[2][1] = g.a;
  E[3][0] = g.b;
  E[3][1] = g.gamma;
}

__device__ __forceinline__ void e_up(const LayerG& g, double p, cd E[4][2]) {
  E[0][0] = mk(p, 0.0);
  E[0][1] = -g.neta;
  E[1][0] = -g.eta;
  E[1][1] = mk(-p, 0.0);
  E[2][0] = -g.gamma;
  E[2][1] = -g.a;
  E[3][0] = -g.b;
  E[3][1] = g.gamma;
}

KR_HD double cabs1(cd z) { return fabs(z.x) + fabs(z.y); }

__device__ __forceinline__ void swap_rows(cd (&A)[4][4], cd (&B)[4][2], int c, int piv) {
  // rows c and piv (piv >= c); compile-time indices only
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    if (r <= c) continue;
    const bool s = (piv == r);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const cd t = A[c][j];
      A[c][j] = s ? A[r][j] : t;
      A[r][j] = s ? t : A[r][j];
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const cd t = B[c][j];
      B[c][j] = s ? B[r][j] : t;
      B[r][j] = s ? t : B[r][j];
    }
  }
}

// Solves A X = B (4x4, two right-hand sides) in place: on return B holds X.
__device__ __forceinline__ void solve4x2(cd (&A)[4][4], cd (&B)[4][2]) {
  cd inv[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    double best = cabs1(A[c][c]);
#pragma unroll
    for (int r = c + 1; r < 4; ++r) {
      const double m = cabs1(A[r][c]);
      if (m > best) {
        best = m;
        piv = r;
      }
    }
    swap_rows(A, B, c, piv);
    inv[c] = recip(A[c][c]);
#pragma unroll
    for (int r = c + 1; r < 4; ++r) {
      const cd l = A[r][c] * inv[c];
#pragma unroll
      for (int j = c + 1; j < 4; ++j) A[r][j] = cmac(A[r][j], -l, A[c][j]);
#pragma unroll
      for (int j = 0; j < 2; ++j) B[r][j] = cmac(B[r][j], -l, B[c][j]);
    }
  }
#pragma unroll
  for (int c = 3; c >= 0; --c) {
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      cd s = B[c][j];
#pragma unroll
      for (int k = c + 1; k < 4; ++k) s = cmac(s, -A[c][k], B[k][j]);
      B[c][j] = s * inv[c];
    }
  }
}

// Riccati sweep for one (omega, p); returns R without the free-surface operator.
template <class Ph>
__device__ __forceinline__ cd gmm_sweep(int L, double p, const LayerG* g, const Ph& ph,
                                        double rho0) {
  const int M = L - 2;
  cd Y[2][2] = {{mk(0.0, 0.0), mk(0.0, 0.0)}, {mk(0.0, 0.0), mk(0.0, 0.0)}};
  for (int k = M; k >= 1; --k) {
    // E_eff of the layer below interface k
    cd Ee[4][2];
    e_down(g[k + 1], p, Ee);
    if (k < M) {
      cd Eu[4][2];
      e_up(g[k + 1], p, Eu);
      const cd pa = ph.a(k + 1), pb = ph.b(k + 1);
      const cd Z00 = pa * Y[0][0], Z01 = pa * Y[0][1], Z10 = pb * Y[1][0], Z11 = pb * Y[1][1];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        Ee[r][0] = cmac2(Ee[r][0], Eu[r][0], Z00, Eu[r][1], Z10);
        Ee[r][1] = cmac2(Ee[r][1], Eu[r][0], Z01, Eu[r][1], Z11);
      }
    }
    // F = [E_u(k) | -E_eff], right-hand side -E_d(k) diag(ph(k))
    cd F[4][4], B[4][2];
    {
      cd Eu[4][2], Ed[4][2];
      e_up(g[k], p, Eu);
      e_down(g[k], p, Ed);
      const cd pa = ph.a(k), pb = ph.b(k);
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        F[r][0] = Eu[r][0];
        F[r][1] = Eu[r][1];
        F[r][2] = -Ee[r][0];
        F[r][3] = -Ee[r][1];
        B[r][0] = -(Ed[r][0] * pa);
        B[r][1] = -(Ed[r][1] * pb);
      }
    }
    solve4x2(F, B);
    Y[0][0] = B[0][0];
    Y[0][1] = B[0][1];
    Y[1][0] = B[1][0];
    Y[1][1] = B[1][1];
  }
  // ocean extraction at the ocean bottom
  cd E1[4][2];
  e_down(g[1], p, E1);
  if (M >= 1) {
    cd Eu[4][2];
    e_up(g[1], p, Eu);
    const cd pa = ph.a(1), pb = ph.b(1);
    const cd Z00 = pa * Y[0][0], Z01 = pa * Y[0][1], Z10 = pb * Y[1][0], Z11 = pb * Y[1][1];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      E1[r][0] = cmac2(E1[r][0], Eu[r][0], Z00, Eu[r][1], Z10);
      E1[r][1] = cmac2(E1[r][1], Eu[r][0], Z01, Eu[r][1], Z11);
    }
  }
  const cd eta0 = g[0].eta;
  const cd e0 = ph.a(0);
  const cd crho = mk(rho0, 0.0);
  // e_d = (eta0, -rho0), e_u = (-eta0, -rho0)
  const cd eu0 = -eta0, eu1 = -crho, ed0 = eta0, ed1 = -crho;
  cd m00 = cdot2(eu0, E1[2][0], -eu1, E1[1][0]);
  cd m01 = cdot2(eu0, E1[2][1], -eu1, E1[1][1]);
  cd m10 = E1[3][0], m11 = E1[3][1];
  cd r0 = cdot2(eu0, ed1, -eu1, ed0) * e0, r1 = mk(0.0, 0.0);
  // 2x2 solve with partial pivoting
  if (cabs1(m10) > cabs1(m00)) {
    cd t = m00; m00 = m10; m10 = t;
    t = m01; m01 = m11; m11 = t;
    t = r0; r0 = r1; r1 = t;
  }
  const cd i00 = recip(m00);
  const cd l = m10 * i00;
  const cd u11 = cmac(m11, -l, m01);
  const cd y1 = cmac(r1, -l, r0);
  const cd d1 = y1 * recip(u11);
  const cd d0 = cmac(r0, -m01, d1) * i00;
  const cd uz = cdot2(E1[1][0], d0, E1[1][1], d1);
  const cd U0 = cmac(uz, -ed0, e0) * recip(eu0);
  return e0 * U0;
}

constexpr int kGmmTabTiles = 16;

// Shared memory: LayerP[L], LayerG[L], phase table (when the model tabulates).
static size_t gmm_smem(int L, bool table) {
  return sizeof(LayerP) * (size_t)L + sizeof(LayerG) * (size_t)L +
         (table ? phase_table_bytes(L, kGmmTabTiles) : 0);
}

// Four blocks of 128 threads per SM (128 registers): 13.34 ms on the 21-layer gather grid
// against 13.47 at the compiler's 134 registers (three blocks) and 13.59 at five (96).
__global__ void __launch_bounds__(kGmmThreads, 4)
gmm_kernel(const double* __restrict__ tab, int L, const double* __restrict__ p, int n_p,
           const double2* __restrict__ omega, int n_w, int n_wtiles, int tiles_per_block,
           int free_surface, int use_table, double2* __restrict__ R) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned s_bad;
  LayerP* s_layer = reinterpret_cast<LayerP*>(smem);
  LayerG* s_g = reinterpret_cast<LayerG*>(smem + sizeof(LayerP) * L);
  cd* s_ph = reinterpret_cast<cd*>(smem + sizeof(LayerP) * L + sizeof(LayerG) * L);
  const int groups = (n_wtiles + tiles_per_block - 1) / tiles_per_block;
  const int ip = blockIdx.x / groups;
  const int t0 = (blockIdx.x % groups) * tiles_per_block;
  const int t1 = min(n_wtiles, t0 + tiles_per_block);
  const double pj = p[ip];
  for (int l = threadIdx.x; l < L; l += blockDim.x) {
    const LayerP lp = layer_terms(tab, L, l, pj);
    s_layer[l] = lp;
    s_g[l] = gmm_layer(lp, pj);
  }
  __syncthreads();
  unsigned mask = 0u;
  const int entries = phase_entries(kGmmTabTiles);
  if (use_table)
    mask = build_phase_table(omega, n_w, grid_line(omega, n_w), t0, t1 - t0, entries, L,
                             s_layer, s_ph, &s_bad);
  const double rho0 = s_layer[0].rho;
  double2* Rp = R + (size_t)ip * n_w;
  for (int t = t0; t < t1; ++t) {
    const int iw = t * kGmmThreads + threadIdx.x;
    if (iw >= n_w) break;
    const double2 wv = omega[iw];
    const PhaseAuto ph{((mask >> (t - t0)) & 1u) != 0, phase_at(s_ph, entries, iw, t0),
                       PhaseDirect{mk(wv.x, wv.y), s_layer}};
    cd r = gmm_sweep(L, pj, s_g, ph, rho0);
    if (free_surface) r = r * recip(1.0 + r);
    Rp[iw] = make_double2(r.x, r.y);
  }
}

}  // namespace kr

using namespace kr;

extern "C" kr_status kr_gmm_reflectivity(const double* layers, int32_t n_layers, const double* p,
                                         int32_t n_p, const double* omega, int32_t n_w,
                                         uint32_t flags, double* R, void* stream) {
  if (n_p < 0 || n_w < 0 || (flags & ~KR_FREE_SURFACE)) return KR_ERR_INVALID_ARGUMENT;
  if (n_layers < 2) return KR_ERR_INVALID_MODEL;
  if (n_layers > kMaxLayers) return KR_ERR_TOO_LARGE;
  if (n_p == 0 || n_w == 0) return KR_OK;
  if (!layers || !p || !omega || !R) return KR_ERR_INVALID_ARGUMENT;
  if (!aligned16(omega) || !aligned16(R)) return KR_ERR_INVALID_ARGUMENT;
  const int n_wtiles = (n_w + kGmmThreads - 1) / kGmmThreads;
  // tiles per block: enough slownesses x tile groups for ~8 waves, at most kGmmTabTiles
  long long tpb = ((long long)n_p * n_wtiles) / (148LL * 4 * 8);
  if (tpb < 1) tpb = 1;
  if (tpb > kGmmTabTiles) tpb = kGmmTabTiles;
  if (tpb > n_wtiles) tpb = n_wtiles;
  const long long blocks = (long long)n_p * ((n_wtiles + tpb - 1) / tpb);
  if (blocks > 0x7fffffffLL) return KR_ERR_TOO_LARGE;
  const bool table = phase_table_model(n_layers);
  const size_t smem = gmm_smem(n_layers, table);
  cudaStream_t st = (cudaStream_t)stream;
  static SmemLimit lim;
  if (smem > 48 * 1024) {
    const kr_status a = raise_smem_limit((const void*)gmm_kernel, smem, lim,
                                         "kr_gmm_reflectivity: smem attribute");
    if (a != KR_OK) return a;
  }
  gmm_kernel<<<(unsigned)blocks, kGmmThreads, smem, st>>>(
      layers, n_layers, p, n_p, reinterpret_cast<const double2*>(omega), n_w, n_wtiles, (int)tpb,
      (flags & KR_FREE_SURFACE) ? 1 : 0, table ? 1 : 0, reinterpret_cast<double2*>(R));
  return check_launch("kr_gmm_reflectivity");
}
