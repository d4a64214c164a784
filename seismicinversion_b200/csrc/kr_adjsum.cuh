// Device side of the frequency sums of the adjoint (adjoint_pair_sums in kr_adjoint.cuh):
// every warp adds its 32 lanes' 12 per-step values into its own rows of shared memory through
// a padded staging tile (a transposed, fixed-order reduction: deterministic), and the block
// contracts the summed rows with the coefficient tangents and phase-derivative factors once.
#pragma once

#include "kr_adjoint.cuh"

namespace kr {

constexpr int kSumHalf = 6;     // values staged per round (two rounds per step)
constexpr int kSumStride = 7;   // staging row stride in complex values

// Shared memory of the sums for `warps` warps: per warp L rows of 12 complex values and a
// 32 x 7 staging tile.
__host__ __device__ inline size_t adjsum_smem_bytes(int L, int warps) {
  return sizeof(cd) * (size_t)warps * (sum_rows(L) * kSumVals + 32 * kSumStride);
}

// Bytes of one warp's staging tile (the region a block may reuse once its sweeps are done).
__host__ __device__ inline size_t adjsum_stage_bytes(int warps) {
  return sizeof(cd) * (size_t)warps * 32 * kSumStride;
}

// acc_row[c] += sum over the warp's lanes of v[c], c < 12, in two rounds of 6 values: lanes
// (c, g) add rows 8 g .. 8 g + 7 of column c, then the four row groups by shuffles.  All 32
// lanes call it.
__device__ __forceinline__ void warp_add12(const cd v[kSumVals], cd* stage, cd* acc_row) {
  const int lane = threadIdx.x & 31;
  cd* mine = stage + lane * kSumStride;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
#pragma unroll
    for (int k = 0; k < kSumHalf; ++k) mine[k] = v[h * kSumHalf + k];
    __syncwarp();
    if (lane < 4 * kSumHalf) {
      const int c = lane % kSumHalf, g = lane / kSumHalf;
      cd s = stage[(8 * g) * kSumStride + c];
#pragma unroll
      for (int r = 1; r < 8; ++r) s = s + stage[(8 * g + r) * kSumStride + c];
      s.x += __shfl_down_sync(0x00ffffffu, s.x, 2 * kSumHalf);
      s.y += __shfl_down_sync(0x00ffffffu, s.y, 2 * kSumHalf);
      if (lane < 2 * kSumHalf) {
        s.x += __shfl_down_sync(0x00000fffu, s.x, kSumHalf);
        s.y += __shfl_down_sync(0x00000fffu, s.y, kSumHalf);
        if (lane < kSumHalf) acc_row[h * kSumHalf + c] = acc_row[h * kSumHalf + c] + s;
      }
    }
    __syncwarp();
  }
}

// The summing sink of one lane: seed 2 conj(R - R_obs) (misfit) or conj(gR) (cotangent gR).
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
    warp_add12(v, stage, acc + (size_t)I * kSumVals);
  }
  __device__ void step(int i, const cd cbar[10], cd fa, cd fb) {
    cd v[kSumVals];
#pragma unroll
    for (int k = 0; k < 10; ++k) v[k] = cbar[k];
    v[10] = fa;
    v[11] = fb;
    warp_add12(v, stage, acc + (size_t)i * kSumVals);
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
