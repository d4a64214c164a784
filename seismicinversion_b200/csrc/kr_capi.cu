// C-ABI housekeeping: status strings, per-thread error detail, version, host-side model
// validation (the rules of Kennett_Reflectivity/layer_model.py:105-123 plus kernel limits).
#include <math.h>
#include <stdio.h>

#include <string>

#include "kr_internal.cuh"

namespace kr {

static thread_local std::string g_last_error;

void set_last_error(const char* where, cudaError_t e) {
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
}
void set_last_error_msg(const char* msg) { g_last_error = msg; }

}  // namespace kr

extern "C" const char* kr_status_string(kr_status s) {
  switch (s) {
    case KR_OK: return "KR_OK";
    case KR_ERR_INVALID_ARGUMENT: return "KR_ERR_INVALID_ARGUMENT";
    case KR_ERR_INVALID_MODEL: return "KR_ERR_INVALID_MODEL";
    case KR_ERR_CUDA: return "KR_ERR_CUDA";
    case KR_ERR_CUFFT: return "KR_ERR_CUFFT";
    case KR_ERR_WORKSPACE: return "KR_ERR_WORKSPACE";
    case KR_ERR_TOO_LARGE: return "KR_ERR_TOO_LARGE";
    default: return "KR_ERR_UNKNOWN";
  }
}

extern "C" const char* kr_last_error(void) { return kr::g_last_error.c_str(); }

extern "C" int32_t kr_version(void) { return 1 * 10000 + 0 * 100 + 0; }

extern "C" kr_status kr_validate_layers(const double* tab, int32_t n) {
  char buf[160];
  if (!tab) return KR_ERR_INVALID_ARGUMENT;
  if (n < 2 || n > KR_MAX_LAYERS) {
    snprintf(buf, sizeof buf, "n_layers must be in [2, %d], got %d", KR_MAX_LAYERS, n);
    kr::set_last_error_msg(buf);
    return KR_ERR_INVALID_MODEL;
  }
  const double* alpha = tab;
  const double* beta = tab + n;
  const double* rho = tab + 2 * n;
  const double* h = tab + 3 * n;
  const double* qa = tab + 4 * n;
  const double* qb = tab + 5 * n;
  for (int l = 0; l < n; ++l) {
    const char* why = nullptr;
    if (!(alpha[l] > 0.0) || !isfinite(alpha[l])) why = "alpha must be positive and finite";
    else if (!(beta[l] >= 0.0) || !isfinite(beta[l])) why = "beta must be non-negative and finite";
    else if (!(rho[l] > 0.0) || !isfinite(rho[l])) why = "rho must be positive and finite";
    else if (!(h[l] >= 0.0)) why = "thickness must be non-negative (inf for the half-space)";
    else if (!(qa[l] > 0.0) || !isfinite(qa[l])) why = "Q_alpha must be positive and finite";
    else if (beta[l] > 0.0 && (!(qb[l] > 0.0) || !isfinite(qb[l])))
      why = "Q_beta must be positive and finite where beta > 0";
    else if (l == 0 && beta[0] != 0.0) why = "layer 0 must be the acoustic ocean (beta = 0)";
    if (why) {
      snprintf(buf, sizeof buf, "layer %d: %s", l, why);
      kr::set_last_error_msg(buf);
      return KR_ERR_INVALID_MODEL;
    }
  }
  return KR_OK;
}
