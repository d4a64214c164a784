// Fused forward reflectivity kernel: one thread per (omega, p), one slowness per block.
//
// Block prologue: layer slownesses and the interface coefficients of this block's slowness
// go to shared memory (computed once per block, read as broadcasts).  Each thread then runs
// the whole bottom-up Kennett sweep for its frequency with the cumulative reflection
// matrix in registers, applies the ocean phase / free-surface operator and writes
// R[p][omega] (coalesced along omega).  FP64 CUDA cores; no tensor-core work exists here
// (2x2 complex algebra per thread is not a contraction).
#include "kr_internal.cuh"

namespace kr {

constexpr int kFwdThreads = 128;

__global__ void __launch_bounds__(kFwdThreads)
reflectivity_kernel(const double* __restrict__ tab, int n_layers, const double* __restrict__ p,
                    int n_p, const double2* __restrict__ omega, int n_w, int n_wtiles,
                    int free_surface, double2* __restrict__ R) {
  extern __shared__ __align__(16) unsigned char smem[];
  LayerP* s_layer = reinterpret_cast<LayerP*>(smem);
  Iface* s_iface = reinterpret_cast<Iface*>(smem + sizeof(LayerP) * n_layers);
  const int ip = blockIdx.x / n_wtiles;
  const int iw = (blockIdx.x % n_wtiles) * kFwdThreads + threadIdx.x;
  const double pj = p[ip];
  block_prologue(tab, n_layers, pj, s_layer, s_iface);
  if (iw >= n_w) return;
  const double2 wv = omega[iw];
  const cd w = mk(wv.x, wv.y);
  cd rpp = sweep(w, n_layers, s_layer, s_iface);
  cd e0 = cexp_(w * s_layer[0].ca);
  cd out = pp_surface(rpp, e0, free_surface != 0);
  R[(size_t)ip * n_w + iw] = make_double2(out.x, out.y);
}

}  // namespace kr

using namespace kr;

extern "C" kr_status kr_reflectivity(const double* layers, int32_t n_layers, const double* p,
                                     int32_t n_p, const double* omega, int32_t n_w,
                                     uint32_t flags, double* R, void* stream) {
  if (n_p < 0 || n_w < 0 || (flags & ~KR_FREE_SURFACE)) return KR_ERR_INVALID_ARGUMENT;
  if (n_layers < 2) return KR_ERR_INVALID_MODEL;
  if (n_layers > kMaxLayers) return KR_ERR_TOO_LARGE;
  if (n_p == 0 || n_w == 0) return KR_OK;
  if (!layers || !p || !omega || !R) return KR_ERR_INVALID_ARGUMENT;
  const int n_wtiles = (n_w + kFwdThreads - 1) / kFwdThreads;
  const long long blocks = (long long)n_p * n_wtiles;
  if (blocks > 0x7fffffffLL) return KR_ERR_TOO_LARGE;
  const size_t smem = prologue_smem_bytes(n_layers);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(reflectivity_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
      set_last_error("kr_reflectivity: smem attribute", e);
      return KR_ERR_CUDA;
    }
  }
  reflectivity_kernel<<<(unsigned)blocks, kFwdThreads, smem, (cudaStream_t)stream>>>(
      layers, n_layers, p, n_p, reinterpret_cast<const double2*>(omega), n_w, n_wtiles,
      (flags & KR_FREE_SURFACE) ? 1 : 0, reinterpret_cast<double2*>(R));
  return check_launch("kr_reflectivity");
}
