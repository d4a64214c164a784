/*
 * kennett_b200 benchmark support (no counterpart in the reference): an FP64 CUDA-core
 * throughput probe used as the measured roofline denominator of the FP64 kernels.
 */
#ifndef KENNETT_B200_BENCH_H
#define KENNETT_B200_BENCH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Launches `blocks` x 256 threads, each running 8 independent chains of `iters` DFMAs.
 * `out` is a device float64 buffer of blocks*256 elements (written only to keep the
 * chains live).  Time it with events on `stream`; flops = kr_bench_fp64_fma_flops(). */
int32_t kr_bench_fp64_fma(int32_t blocks, int32_t iters, double* out, void* stream);

/* FLOPs of one kr_bench_fp64_fma launch (2 per DFMA). */
double kr_bench_fp64_fma_flops(int32_t blocks, int32_t iters);

#ifdef __cplusplus
}
#endif

#endif /* KENNETT_B200_BENCH_H */
