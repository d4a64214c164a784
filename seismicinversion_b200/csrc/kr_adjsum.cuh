// Device side of the frequency sums of the adjoint (adjoint_pair_sums in kr_adjoint.cuh):
// every warp adds its 32 lanes' 12 per-step values into its own rows of shared memory through
// a padded staging tile (a transposed, fixed-order reduction: deterministic), and the block
// contracts the summed rows with the coefficient tangents and phase-derivative factors once.
#pragma once

#include "kr_adjoint.cuh"

namespace kr {

// Staging of the warp sums: ROUNDS = 1 stages all 12 values in one 32 x 13 tile (fewest
// instructions); ROUNDS = 2 stages 6 at a time in a 32 x 7 tile (half the shared memory, for
// kernels whose residency shared memory limits).  Tile row stride in complex values:
template <int ROUNDS>
__host__ __device__ constexpr int stage_stride() { return kSumVals / ROUNDS + 1; }

// Shared memory of the sums for `warps` warps: per warp L rows of 12 complex values and its
// staging tile.
__host__ __device__ inline size_t adjsum_smem_bytes(int L, int warps, int rounds) {
  const int stride = kSumVals / rounds + 1;
  return sizeof(cd) * (size_t)warps * (sum_rows(L) * kSumVals + 32 * (size_t)stride);
}

// Bytes of the warps' staging tiles (the region a block may reuse once its sweeps are done).
__host__ __device__ inline size_t adjsum_stage_bytes(int warps, int rounds) {
  return sizeof(cd) * (size_t)warps * 32 * (size_t)(kSumVals / rounds + 1);
}

// acc_row[c] += sum over the warp's lanes of v[c], c < 12.  Per round, lanes (c, g) add the
// rows of row group g in column c (2 groups of 16 rows for one round, 4 of 8 for two), then
// shuffles combine the groups; a fixed order (deterministic).  All 32 lanes call it.
template <int ROUNDS>
__device__ __forceinline__ void warp_add12(const cd v[kSumVals], cd* stage, cd* acc_row) {
  constexpr int P = kSumVals / ROUNDS, S = P + 1, G = 2 * ROUNDS, RG = 32 / G;
  const int lane = threadIdx.x & 31;
  cd* mine = stage + lane * S;
#pragma unroll
  for (int h = 0; h < ROUNDS; ++h) {
#pragma unroll
    for (int k = 0; k < P; ++k) mine[k] = v[h * P + k];
    __syncwarp();
    if (lane < G * P) {  // 24 lanes
      const int c = lane % P, g = lane / P;
      cd s = stage[(RG * g) * S + c];
#pragma unroll
      for (int r = 1; r < RG; ++r) s = s + stage[(RG * g + r) * S + c];
      if (G == 4) {
        s.x += __shfl_down_sync(0x00ffffffu, s.x, 2 * P);
        s.y += __shfl_down_sync(0x00ffffffu, s.y, 2 * P);
      }
      if (lane < 2 * P) {
        const unsigned m = (2 * P == 24) ? 0x00ffffffu : 0x00000fffu;
        s.x += __shfl_down_sync(m, s.x, P);
        s.y += __shfl_down_sync(m, s.y, P);
        if (lane < P) acc_row[h * P + c] = acc_row[h * P + c] + s;
      }
    }
    __syncwarp();
  }
}

// The summing sink of one lane: seed 2 conj(R - R_obs) (misfit) or conj(gR) (cotangent gR).
template <int ROUNDS>
struct SumSink {
  bool valid;
  bool vjp;          // seed with conj(gR) instead of 2 conj(R - R_obs)
  const double2* obs;  // R_obs or gR at this (p, omega)
  double2* R_out;      // R at this (p, omega), or nullptr
  cd* acc;             // this warp's sum rows
  cd* stage;           // this warp's staging tile
  int I;
  cd res;
  __device__ cd reflectivity(cd R) {
    res = mk(0.0, 0.0);
    if (!valid) return mk(0.0, 0.0);
    if (R_out) *R_out = make_double2(R.x, R.y);
    const double2 o = *obs;
    if (vjp) return mk(o.x, -o.y);  // conj(gR)
    res = mk(R.x - o.x, R.y - o.y);
    return mk(2.0 * res.x, -2.0 * res.y);  // 2 conj(res)
  }
  __device__ void top(cd f0) {
    cd v[kSumVals];
#pragma unroll
    for (int k = 0; k < kSumVals; ++k) v[k] = mk(0.0, 0.0);
    v[10] = f0;
    warp_add12<ROUNDS>(v, stage, acc + (size_t)I * kSumVals);
  }
  __device__ void step(int i, const cd cbar[10], cd fa, cd fb) {
    cd v[kSumVals];
#pragma unroll
    for (int k = 0; k < 10; ++k) v[k] = cbar[k];
    v[10] = fa;
    v[11] = fb;
    warp_add12<ROUNDS>(v, stage, acc + (size_t)i * kSumVals);
  }
};

// Zeroes the warps' sum rows (block-cooperative; the caller synchronises afterwards).
__device__ __forceinline__ void sums_zero(cd* acc_all, int L, int warps) {
  const int n = warps * (int)sum_rows(L) * kSumVals;
  for (int k = threadIdx.x; k < n; k += blockDim.x) acc_all[k] = mk(0.0, 0.0);
}

// Adds the warps' rows into warp 0's (fixed order), then thread l < L contracts layer l into
// out[k L + l] (k = alpha, beta, rho, h).  Contains block barriers; all threads call it.
__device__ __forceinline__ void sums_finish(cd* acc_all, int L, int warps,
                                            const ScatTan* __restrict__ tan,
                                            const LayerD* __restrict__ dlay, double* out) {
  const int n = (int)sum_rows(L) * kSumVals;
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    cd s = acc_all[k];
    for (int wi = 1; wi < warps; ++wi) s = s + acc_all[wi * n + k];
    acc_all[k] = s;
  }
  __syncthreads();
  for (int l = threadIdx.x; l < L; l += blockDim.x) {
    double v[4];
    sums_contract_layer(l, L, acc_all, tan, dlay, v);
    out[0 * L + l] = v[0];
    out[1 * L + l] = v[1];
    out[2 * L + l] = v[2];
    out[3 * L + l] = v[3];
  }
}

}  // namespace kr
