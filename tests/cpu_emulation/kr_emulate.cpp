// Test-only CPU build of the device math in seismicinversion_b200/csrc/kr_math.cuh: the
// per-(omega, p) sweep exactly as the kernels run it, compiled with g++ so the CPU test
// suite can check the kernel arithmetic against the oracle without a GPU.  Not a fallback:
// nothing in the package loads this.
#include "../../seismicinversion_b200/csrc/kr_math.cuh"

using namespace kr;

extern "C" void emu_reflectivity(const double* tab, int L, const double* p, int n_p,
                                 const double* w, int nw, int fs, double* out) {
  LayerP lay[512];
  Iface f[512];
  for (int j = 0; j < n_p; ++j) {
    for (int l = 0; l < L; ++l) lay[l] = layer_terms(tab, L, l, p[j]);
    for (int i = 0; i < L - 1; ++i) f[i] = interface_coeffs(p[j], i, lay[i], lay[i + 1]);
    for (int k = 0; k < nw; ++k) {
      cd om = mk(w[2 * k], w[2 * k + 1]);
      const int I = L - 1;
      M2 r;
      r.a = f[I - 1].rd11; r.b = f[I - 1].rd12; r.c = f[I - 1].rd12; r.d = f[I - 1].rd22;
      for (int i = I - 2; i >= 0; --i)
        r = kennett_step(r, cexp_(om * lay[i + 1].ca), cexp_(om * lay[i + 1].cb), f[i]);
      cd o = pp_surface(r.a, cexp_(om * lay[0].ca), fs != 0);
      out[2 * ((size_t)j * nw + k)] = o.x;
      out[2 * ((size_t)j * nw + k) + 1] = o.y;
    }
  }
}
