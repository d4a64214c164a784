// Internal declarations shared by the library's translation units (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <mutex>

#include "../../include/kennett_b200.h"
#include "kr_math.cuh"

namespace kr {

constexpr int kMaxLayers = KR_MAX_LAYERS;

// Dynamic shared memory of the per-slowness prologue: layer terms + interface coefficients.
__host__ __device__ inline size_t prologue_smem_bytes(int n_layers) {
  return sizeof(LayerP) * (size_t)n_layers + sizeof(Iface) * (size_t)(n_layers - 1);
}

inline kr_status cuda_status(cudaError_t e) { return e == cudaSuccess ? KR_OK : KR_ERR_CUDA; }

// Complex arrays are read and written as 16-byte units (vector loads, cp.async): every
// complex pointer of the C ABI must be 16-byte aligned.  Null passes (checked separately).
inline bool aligned16(const void* ptr) { return ((uintptr_t)ptr & 15u) == 0; }

// Remembers the last CUDA error string for kr_last_error().
void set_last_error(const char* where, cudaError_t e);
void set_last_error_msg(const char* msg);

// Raises a kernel's dynamic shared-memory limit to `bytes` on the current device, calling the
// runtime only when the limit recorded for that device is lower: after the first call per
// device (and larger size) a launcher makes no runtime call but the launch, so it can be
// captured into a CUDA graph.  `lim` is the launcher's own per-kernel table (zero-initialised
// static storage).
constexpr int kMaxDevices = 64;
struct SmemLimit {
  int bytes[kMaxDevices];
};
// One lock for every kernel's limit: host threads that launch concurrently (two servers, a
// server and a direct call) must not interleave the check, the attribute call and the
// record, or one could lower a limit another thread's launch relies on.  Under the lock a
// limit only ever rises.
inline std::mutex& smem_limit_mutex() {
  static std::mutex m;
  return m;
}

inline kr_status raise_smem_limit(const void* fn, size_t bytes, SmemLimit& lim,
                                  const char* where) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(where, e);
    return KR_ERR_CUDA;
  }
  const bool known = dev >= 0 && dev < kMaxDevices;
  std::lock_guard<std::mutex> g(smem_limit_mutex());
  if (known && lim.bytes[dev] >= (int)bytes) return KR_OK;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) {
    set_last_error(where, e);
    return KR_ERR_CUDA;
  }
  if (known) lim.bytes[dev] = (int)bytes;
  return KR_OK;
}

inline kr_status check_launch(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(where, e);
    return KR_ERR_CUDA;
  }
  return KR_OK;
}

// Computes the layer terms and interface coefficients of one slowness into shared memory
// (threads of the block cooperate: one layer / one interface per thread).  Ends with a
// block barrier.
__device__ __forceinline__ void block_prologue(const double* __restrict__ tab, int n_layers,
                                               double p, LayerP* s_layer, Iface* s_iface) {
  for (int l = threadIdx.x; l < n_layers; l += blockDim.x) s_layer[l] = layer_terms(tab, n_layers, l, p);
  __syncthreads();
  for (int i = threadIdx.x; i < n_layers - 1; i += blockDim.x)
    s_iface[i] = interface_coeffs(p, i, s_layer[i], s_layer[i + 1]);
  __syncthreads();
}

// The full upward sweep for one (omega, p) with coefficients in shared memory; `ph` supplies
// the layer phase factors (PhaseDirect, or a tabulated source with the same a(l) / b(l)).
// Returns RRd_PP below the ocean and the ocean phase factor e0.  The phase factors of the
// next layer are fetched one step ahead, so their latency overlaps the current step's
// algebra; the last (ocean-bottom) step forms only RRd_00.
template <class Ph>
__device__ __forceinline__ cd sweep_ph(int n_layers, const Iface* s_iface, const Ph& ph,
                                       cd* e0_out) {
  const int I = n_layers - 1;
  // Bottom interface: RRd below it is 0, so RRd = Rd.
  M2 r;
  r.a = s_iface[I - 1].rd11;
  r.b = s_iface[I - 1].rd12;
  r.c = s_iface[I - 1].rd12;
  r.d = s_iface[I - 1].rd22;
  if (I == 1) {
    *e0_out = ph.a(0);
    return r.a;
  }
  cd ea = ph.a(I - 1), eb = ph.b(I - 1);
  for (int i = I - 2; i >= 1; --i) {
    const cd ea_n = ph.a(i), eb_n = ph.b(i);
    r = kennett_step(r, ea, eb, s_iface[i]);
    ea = ea_n;
    eb = eb_n;
  }
  *e0_out = ph.a(0);
  return kennett_last_step_pp(r, ea, eb, s_iface[0]);
}

__device__ __forceinline__ cd sweep(cd w, int n_layers, const LayerP* s_layer,
                                    const Iface* s_iface, cd* e0_out) {
  return sweep_ph(n_layers, s_iface, PhaseDirect{w, s_layer}, e0_out);
}

// Block-cooperative copy of n bytes (multiple of 16, 16-byte aligned) into shared memory.
__device__ __forceinline__ void copy16(void* dst, const void* src, size_t n) {
  double2* d = reinterpret_cast<double2*>(dst);
  const double2* s = reinterpret_cast<const double2*>(src);
  for (size_t k = threadIdx.x; k < n / 16; k += blockDim.x) d[k] = s[k];
}

}  // namespace kr
