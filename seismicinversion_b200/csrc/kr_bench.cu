// Benchmark support: FP64 CUDA-core throughput probe (the roofline denominator of the FP64
// kernels).  Each thread runs 8 independent DFMA chains.
#include "../../include/kennett_b200_bench.h"
#include "kr_internal.cuh"

namespace kr {

__global__ void __launch_bounds__(256) fp64_fma_probe(int iters, double seed, double* out) {
  double a0 = seed + threadIdx.x * 1e-12, a1 = a0 + 1e-3, a2 = a0 + 2e-3, a3 = a0 + 3e-3;
  double a4 = a0 + 4e-3, a5 = a0 + 5e-3, a6 = a0 + 6e-3, a7 = a0 + 7e-3;
  const double b = 0.9999999999, c = 1e-12;
#pragma unroll 4
  for (int i = 0; i < iters; ++i) {
    a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
    a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
  }
  double s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (s == 12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace kr

extern "C" kr_status kr_bench_fp64_fma(int32_t blocks, int32_t iters, double* out, void* stream) {
  if (blocks <= 0 || iters <= 0 || !out) return KR_ERR_INVALID_ARGUMENT;
  kr::fp64_fma_probe<<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, 1.0, out);
  return kr::check_launch("kr_bench_fp64_fma");
}

extern "C" double kr_bench_fp64_fma_flops(int32_t blocks, int32_t iters) {
  return 16.0 * 256.0 * (double)blocks * (double)iters;
}
