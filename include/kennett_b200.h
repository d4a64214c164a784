/*
 * kennett_b200 -- C ABI of the B200 (sm_100a) Kennett reflectivity library.
 *
 * Plain pointers and sizes only.  Unless stated otherwise every array argument is a DEVICE
 * pointer owned by the caller; the library never allocates or frees caller memory, and
 * every call is enqueued on the caller's CUDA stream (`stream`, a cudaStream_t passed as
 * void*, NULL = legacy default stream).  Calls return a kr_status; no C++ exception
 * crosses this boundary.  Complex numbers are interleaved (re, im) float64 pairs, and every
 * complex array must start on a 16-byte boundary (the kernels move complex values as
 * 16-byte units); a misaligned complex pointer is rejected with KR_ERR_INVALID_ARGUMENT.
 *
 * Layer table: float64 [6][n_layers], rows alpha (P velocity), beta (S velocity, 0 in the
 * acoustic ocean = layer 0), rho, thickness (+inf or >= 1e30 marks the half-space), Q_alpha,
 * Q_beta.  Layer 0 is the ocean, layer n_layers-1 the half-space.
 *
 * Stream capture: the launch entry points (kr_reflectivity, kr_gmm_reflectivity,
 * kr_bessel_sum[_noalloc], kr_traces, kr_jacobian, kr_misfit_gradient, kr_vjp,
 * kr_misfit_hvp, kr_jacobian_dot, kr_batch_launch) make
 * no CUDA runtime call besides their launches once they have been called on that device with
 * the same sizes (the first call raises kernel shared-memory limits, creates the cuFFT plan
 * or looks up static scratch), so later calls can be recorded into a CUDA graph.
 *
 * Each entry point names the reference (tmnestor/SeismicInversion) interface it replaces.
 */
#ifndef KENNETT_B200_H
#define KENNETT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t kr_status;

#define KR_OK 0
#define KR_ERR_INVALID_ARGUMENT 1   /* null or misaligned pointer, negative size, bad flags */
#define KR_ERR_INVALID_MODEL 2      /* layer table violates the model rules                 */
#define KR_ERR_CUDA 3               /* a CUDA runtime call or kernel launch failed          */
#define KR_ERR_CUFFT 4              /* a cuFFT call failed                                  */
#define KR_ERR_WORKSPACE 5          /* workspace pointer NULL or smaller than required      */
#define KR_ERR_TOO_LARGE 6          /* a size exceeds a documented limit                    */

#define KR_MAX_LAYERS 256           /* layers per model (shared-memory prologue)            */

/* flags */
#define KR_FREE_SURFACE 0x1u        /* include free-surface multiples (R_fs = -1)           */

/* Human-readable name of a status code (static string). */
const char* kr_status_string(kr_status status);

/* Detail of the most recent error in the calling thread ("" if none). */
const char* kr_last_error(void);

/* Library version as major*10000 + minor*100 + patch. */
int32_t kr_version(void);

/*
 * Validates a HOST layer table against the rules of LayerModel
 * (Kennett_Reflectivity/layer_model.py:105-123: alpha > 0, beta >= 0, rho > 0) plus what the
 * kernels need: 2 <= n_layers <= KR_MAX_LAYERS, beta[0] == 0 (acoustic ocean,
 * scattering_matrices.py:164-296), finite positive Q, non-negative thickness.
 * Returns KR_OK or KR_ERR_INVALID_MODEL (detail in kr_last_error()).
 */
kr_status kr_validate_layers(const double* layers_host, int32_t n_layers);

/*
 * Plane-wave PP reflectivity R(p, omega) for one model on a slowness x frequency grid.
 * Replaces kennett_reflectivity (Kennett_Reflectivity/kennett_reflectivity.py:73-78) and
 * kennett_reflectivity_batch (Kennett_Reflectivity/kennett_reflectivity_gpu.py:88-93).
 *   layers : device float64 [6][n_layers]
 *   p      : device float64 [n_p] horizontal slownesses (s/km)
 *   omega  : device complex [n_w] angular frequencies (imaginary part = damping, may be 0)
 *   R      : device complex [n_p][n_w] output
 *   flags  : KR_FREE_SURFACE or 0
 * One fused kernel: slownesses, interface coefficients (shared memory, per slowness) and
 * the Kennett sweep, one thread per (omega, p).  n_p == 0 or n_w == 0 is a no-op.
 */
kr_status kr_reflectivity(const double* layers, int32_t n_layers, const double* p, int32_t n_p,
                          const double* omega, int32_t n_w, uint32_t flags, double* R,
                          void* stream);

/*
 * The same R(p, omega) by the Global Matrix Method with the block-Riccati sweep, an
 * independent FP64 evaluation of the reflectivity.  Replaces gmm_reflectivity
 * (GlobalMatrix/global_matrix.py:297-348) and the forward of gmm_reflectivity_torch
 * (GlobalMatrix/gmm_torch.py:229-305, riccati_solver.py:200-330).  Arguments and errors as
 * kr_reflectivity; with KR_FREE_SURFACE the result is R / (1 + R).  One thread per
 * (omega, p); per interface a 4x4 complex solve with partial pivoting.
 */
kr_status kr_gmm_reflectivity(const double* layers, int32_t n_layers, const double* p,
                              int32_t n_p, const double* omega, int32_t n_w, uint32_t flags,
                              double* R, void* stream);

/* Bytes of device workspace kr_jacobian needs. */
size_t kr_jacobian_workspace_bytes(int32_t n_layers, int32_t n_p, int32_t n_w);

/*
 * Reflectivity and its Jacobian with respect to every layer's alpha, beta, rho, h.
 * Replaces the autograd graph of kennett_reflectivity_torch
 * (Kennett_Reflectivity/kennett_torch.py:312-480) and jacobian (kennett_torch.py:611-641,
 * jacrev of Re and Im).  Hand-written adjoint: one reverse sweep per (omega, p) over a
 * tape of up to 64 steps (deeper models checkpoint and recompute segments); interface-
 * coefficient tangents by forward-mode dual numbers once per (p, interface).
 *   layers, p, omega, flags : as kr_reflectivity
 *   R : device complex [n_p][n_w] output, or NULL
 *   J : device complex [n_p][4*n_layers][n_w] output, J[j][k*L + l][w] = dR(p_j, w)/d theta,
 *       theta = alpha_l (k=0), beta_l (1), rho_l (2), h_l (3).  Derivatives through the
 *       ocean's S quantities, layers with beta = 0 and the half-space phase are zero.
 *   workspace : >= kr_jacobian_workspace_bytes(n_layers, n_p, n_w) bytes
 */
kr_status kr_jacobian(const double* layers, int32_t n_layers, const double* p, int32_t n_p,
                      const double* omega, int32_t n_w, uint32_t flags, double* R, double* J,
                      void* workspace, size_t workspace_bytes, void* stream);

/* Bytes of device workspace kr_misfit_gradient needs. */
size_t kr_misfit_gradient_workspace_bytes(int32_t n_layers, int32_t n_p, int32_t n_w);

/*
 * Misfit chi = sum_{p, w} |R - R_obs|^2 and its gradient with respect to every layer's
 * alpha, beta, rho, h, without forming the Jacobian (block-reduced in a fixed order).
 * Replaces the per-slowness misfit + torch.autograd.grad of taup_misfit_grad_hessian
 * (Kennett_Reflectivity/taup_inversion.py:112-187) for the gradient part.
 *   R_obs    : device complex [n_p][n_w]
 *   R        : device complex [n_p][n_w] output (the forward result), or NULL
 *   chi_grad : device float64 [4*n_layers + 1] output: gradient (index k*L + l as in
 *              kr_jacobian) followed by chi.
 */
kr_status kr_misfit_gradient(const double* layers, int32_t n_layers, const double* p,
                             int32_t n_p, const double* omega, int32_t n_w, uint32_t flags,
                             const double* R_obs, double* R, double* chi_grad, void* workspace,
                             size_t workspace_bytes, void* stream);

/* Bytes of device workspace kr_vjp needs. */
size_t kr_vjp_workspace_bytes(int32_t n_layers, int32_t n_p, int32_t n_w);

/*
 * Vector-Jacobian product of the reflectivity for a caller's cotangent, without forming the
 * Jacobian:  grad[k*L + l] = Re sum_{p, w} conj(gR[p][w]) * dR(p, w) / d theta  (theta as in
 * kr_jacobian; PyTorch's convention for real inputs of a complex output).  Replaces the
 * reverse pass of kennett_reflectivity_torch's autograd graph
 * (Kennett_Reflectivity/kennett_torch.py:312-480) as torch.autograd.grad / backward() drive
 * it with an arbitrary upstream gradient (taup_inversion.py:169-171).  The reverse sweep of
 * kr_misfit_gradient seeded with conj(gR), per-layer recomputation instead of a stored tape of
 * every (p, w, layer) intermediate; block partials reduced in a fixed order (deterministic).
 *   gR   : device complex [n_p][n_w] cotangent
 *   R    : device complex [n_p][n_w] output (the forward result), or NULL
 *   grad : device float64 [4*n_layers] output
 *   workspace : >= kr_vjp_workspace_bytes(n_layers, n_p, n_w) bytes
 */
kr_status kr_vjp(const double* layers, int32_t n_layers, const double* p, int32_t n_p,
                 const double* omega, int32_t n_w, uint32_t flags, const double* gR, double* R,
                 double* grad, void* workspace, size_t workspace_bytes, void* stream);

/* Bytes of device workspace kr_misfit_hvp needs for n_dir directions. */
size_t kr_misfit_hvp_workspace_bytes(int32_t n_layers, int32_t n_p, int32_t n_w, int32_t n_dir);

/*
 * Exact Hessian-vector products of the misfit chi = sum_{p, w} |R - R_obs|^2:
 *   HV[d][j] = sum_i (d^2 chi / d theta_j d theta_i) V[d][i],   d = 0 .. n_dir-1,
 * theta = (alpha_l, beta_l, rho_l, h_l) in the order of kr_jacobian (index k*L + l).
 * Replaces torch.func.hessian of the reference's misfit (Kennett_Reflectivity/
 * taup_inversion.py:177, kennett_torch.py:644-684): the tangent of the adjoint -- the
 * forward sweep, the seed 2 conj(R - R_obs) and the reverse sweep of kr_misfit_gradient
 * carried in dual numbers along each direction, with second derivatives of the interface
 * coefficients from nested dual numbers -- so no step size enters.  One launch for all
 * directions; block partials reduced in a fixed order (deterministic).
 *   R_obs : device complex [n_p][n_w];  V : device float64 [n_dir][4*n_layers]
 *   HV    : device float64 [n_dir][4*n_layers] output
 *   workspace : >= kr_misfit_hvp_workspace_bytes(n_layers, n_p, n_w, n_dir) bytes
 * Limits: n_dir <= 65535, n_layers <= 258 (KR_ERR_TOO_LARGE).
 */
kr_status kr_misfit_hvp(const double* layers, int32_t n_layers, const double* p, int32_t n_p,
                        const double* omega, int32_t n_w, uint32_t flags, const double* R_obs,
                        const double* V, int32_t n_dir, double* HV, void* workspace,
                        size_t workspace_bytes, void* stream);

/* Bytes of device workspace kr_jacobian_dot needs for n_dir directions. */
size_t kr_jacobian_dot_workspace_bytes(int32_t n_layers, int32_t n_p, int32_t n_w,
                                       int32_t n_dir);

/*
 * Directional derivatives of the Jacobian: Jdot[d][j][k*L + l][w] = sum_i
 * (d^2 R(p_j, w) / d theta_{k*L+l} d theta_i) V[d][i] (complex), the second derivative of
 * the reflectivity along each direction.  Replaces the forward-over-reverse derivative that
 * torch.func.hessian takes through kennett_reflectivity_torch (kennett_torch.py:644-684), so
 * that a Hessian built on the differentiable forward is exact rather than Gauss-Newton.
 * Same method and limits as kr_misfit_hvp (seed 1 instead of the misfit's).
 *   V    : device float64 [n_dir][4*n_layers]
 *   Jdot : device complex [n_dir][n_p][4*n_layers][n_w] output
 */
kr_status kr_jacobian_dot(const double* layers, int32_t n_layers, const double* p, int32_t n_p,
                          const double* omega, int32_t n_w, uint32_t flags, const double* V,
                          int32_t n_dir, double* Jdot, void* workspace, size_t workspace_bytes,
                          void* stream);

/* Bytes of device workspace kr_bessel_sum needs for these sizes. */
size_t kr_bessel_sum_workspace_bytes(int32_t n_p, int32_t n_w, int32_t n_r);

/*
 * Discrete-wavenumber (Bessel) summation over slowness, float64 throughout:
 *   U[r][w] = sum_j R[j][w] * ((pw[j] * omega[w]) * dp) * J0((omega[w] * p[j]) * offsets[r])
 * Replaces _gpu_bessel_summation (Kennett_Reflectivity/kennett_gather_gpu.py:56-166) and the
 * per-slowness accumulation of compute_gather (Kennett_Reflectivity/kennett_gather.py:112-124,
 * :274-288).  pw[j] is the per-slowness weight taper_j * p_j.
 *   R       : device complex [n_p][n_w]
 *   p, pw   : device float64 [n_p]
 *   omega   : device float64 [n_w] (real parts of the frequencies)
 *   offsets : device float64 [n_r] (km)
 *   U       : device complex [n_r][n_w] output
 *   workspace: device, >= kr_bessel_sum_workspace_bytes(n_p, n_w, n_r) bytes
 * The slowness sum is split over blocks and reduced in a fixed order (deterministic).
 */
kr_status kr_bessel_sum(const double* R, const double* p, const double* pw, int32_t n_p,
                        double dp, const double* omega, int32_t n_w, const double* offsets,
                        int32_t n_r, double* U, void* workspace, size_t workspace_bytes,
                        void* stream);

/*
 * Allocation-free variant of kr_bessel_sum.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory -- an application that reserved the GPU in
 * its own pool and hands out only pointers, a C/Fortran system whose device buffers are owned
 * by another component, or a loop that must avoid cudaMalloc's implicit synchronisation.  The
 * caller passes inputs and U only (same meaning as kr_bessel_sum); the slice partials live in
 * a 16 MiB file-scope device array that every GPU loading the library holds until exit.
 * Limit: n_r * n_w <= 1048576 (one slice must fit), else KR_ERR_TOO_LARGE.  No cudaMalloc,
 * cudaFree or allocating library call is made.  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress), and so does the first call after the
 * device's context changed (cudaDeviceReset); make such a first call before any stream
 * capture.  All calls share the array: calls that overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller.
 */
kr_status kr_bessel_sum_noalloc(const double* R, const double* p, const double* pw,
                                int32_t n_p, double dp, const double* omega, int32_t n_w,
                                const double* offsets, int32_t n_r, double* U, void* stream);

/* Size in bytes of the static scratch array used by kr_bessel_sum_noalloc (16 MiB). */
size_t kr_bessel_sum_noalloc_scratch_bytes(void);

/* Bytes of device workspace kr_traces needs. */
size_t kr_traces_workspace_bytes(int32_t n_r, int32_t nw);

/*
 * Time traces from spectra at omega_k = k*dw, k = 1..nw-1 (nt = 2*nw samples):
 *   traces[r][t] = Re( FFT_forward( H[r] ) )[t] * decay[t]
 * where H[r] is the Hermitian length-nt spectrum with H[k] = U[r][k-1]*S[k-1] (k = 1..nw-1),
 * H[0] = H[nw] = 0, H[nt-k] = conj(H[k]).  Replaces the trace assembly of compute_seismogram
 * (Kennett_Reflectivity/kennett_seismogram.py:124-144) and the per-trace FFT loops of
 * compute_gather / compute_gather_gpu (kennett_gather.py:294-303, kennett_gather_gpu.py:272-282).
 * Uses a cuFFT complex-to-real transform.
 *   U      : device complex [n_r][nw-1]
 *   S      : device complex [nw-1] source spectrum, or NULL for S = 1
 *   decay  : device float64 [2*nw] (e.g. exp(-gamma t)), or NULL for 1
 *   traces : device float64 [n_r][2*nw] output
 *   workspace: device, >= kr_traces_workspace_bytes(n_r, nw) bytes
 */
kr_status kr_traces(const double* U, const double* S, int32_t n_r, int32_t nw,
                    const double* decay, double* traces, void* workspace,
                    size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------------------- *
 * Batched evaluation of many models of uneven size (no single reference counterpart: the
 * reference evaluates one model per call -- kennett_reflectivity / kennett_reflectivity_torch
 * -- and the batch replaces loops of those calls, e.g. the per-slowness loops of
 * taup_misfit_grad_hessian, Kennett_Reflectivity/taup_inversion.py:153-178).
 * ------------------------------------------------------------------------------------- */

#define KR_BATCH_GRADIENT 0x2u  /* model asks for chi and d chi / d(alpha, beta, rho, h)     */
#define KR_BATCH_STORE_R 0x4u   /* gradient model also writes its R grid                      */

/* One model of a batch.  Offsets index caller-owned packed device buffers:
 *   layers_off : doubles into `layers` (the model's [6][n_layers] table)
 *   p_off      : doubles into `p`;  omega_off : complex elements into `omega`
 *   R_off      : complex elements into `R` ([n_p][n_w], forward models and KR_BATCH_STORE_R)
 *   obs_off    : complex elements into `R_obs` ([n_p][n_w], gradient models)
 *   grad_off   : doubles into `chi_grad` ([4*n_layers + 1]: gradient as in
 *                kr_misfit_gradient, then chi; gradient models)
 * flags: KR_FREE_SURFACE | KR_BATCH_GRADIENT | KR_BATCH_STORE_R. */
typedef struct {
  int32_t n_layers;
  int32_t n_p;
  int32_t n_w;
  uint32_t flags;
  int64_t layers_off;
  int64_t p_off;
  int64_t omega_off;
  int64_t R_off;
  int64_t obs_off;
  int64_t grad_off;
} kr_model_desc;

/* Schedule of a batch: threads per block (32: one warp per work item; 64 or 128) and
 * frequencies per work item. */
typedef struct {
  int32_t threads;
  int32_t tile_w;
  int32_t reserved0;
  int32_t reserved1;
} kr_batch_config;

/* Device bytes of the plan buffer for this batch shape and schedule (0 if invalid). */
size_t kr_batch_plan_bytes(const kr_model_desc* descs_host, int32_t n_models,
                           const kr_batch_config* cfg);

/*
 * Builds the plan of a batch on the host (pair table, work lists sorted by descending cost)
 * and uploads it into `plan` (device, >= kr_batch_plan_bytes).  Synchronises `stream` once.
 * The plan depends only on the batch SHAPE (layer counts, grid sizes, flags, offsets), not on
 * parameter values: relaunching after updating `layers` / `p` / `omega` / `R_obs` in place is
 * valid.
 */
kr_status kr_batch_plan(const kr_model_desc* descs_host, int32_t n_models,
                        const kr_batch_config* cfg, void* plan, size_t plan_bytes, void* stream);

/* Size of the plan's metadata image (the first bytes of the plan buffer). */
size_t kr_batch_plan_meta_bytes(const kr_model_desc* descs_host, int32_t n_models,
                                const kr_batch_config* cfg);

/*
 * Host-only variant of kr_batch_plan: writes the metadata image into HOST memory `image`
 * (>= kr_batch_plan_meta_bytes); the caller copies it to the start of a plan buffer of
 * kr_batch_plan_bytes (e.g. asynchronously from pinned memory) -- no CUDA call, no stream
 * synchronisation.
 */
kr_status kr_batch_plan_host(const kr_model_desc* descs_host, int32_t n_models,
                             const kr_batch_config* cfg, void* image, size_t image_bytes);

/*
 * Runs a planned batch: reset -> per-(model, slowness) coefficient prep -> persistent
 * forward kernel -> persistent gradient kernel, all enqueued on `stream` with no host
 * synchronisation or allocation (capturable in a CUDA graph).  `cfg` must be the plan's
 * schedule and `max_layers` the largest n_layers of the batch.
 */
kr_status kr_batch_launch(void* plan, const kr_batch_config* cfg, int32_t max_layers,
                          const double* layers, const double* p, const double* omega,
                          const double* R_obs, double* R, double* chi_grad, void* stream);

/*
 * Tuning knob (no counterpart in the reference): register budget of the kr_reflectivity
 * kernel as the number of 128-thread blocks each SM must fit (4 -> 128 registers per thread,
 * 5 -> 96, 6 -> 80; other values restore the automatic choice: 5 for models whose phases
 * come from the frequency-grid table, 4 otherwise).  Process-wide; results are identical for
 * every setting, only speed changes.
 */
void kr_set_forward_variant(int32_t min_blocks_per_sm);

/*
 * Tuning knob (no counterpart in the reference): register budget of the kr_jacobian /
 * kr_misfit_gradient / kr_vjp sweep kernels as 128-thread blocks per SM (2 -> up to 255
 * registers, 3 -> 168; other values select 2).  Process-wide; results do not depend on it.
 */
void kr_set_deriv_variant(int32_t min_blocks_per_sm);

#ifdef __cplusplus
}
#endif

#endif /* KENNETT_B200_H */
