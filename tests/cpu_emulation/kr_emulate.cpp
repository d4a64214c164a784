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

// ---- derivatives (kr_adjoint.cuh), same per-pair code the deriv_sweep_kernel runs ----
#include "../../seismicinversion_b200/csrc/kr_adjoint.cuh"

namespace {
struct HostSink {
  typedef Acc AccT;
  static constexpr bool kSeeded = false;
  int L, nw, k;
  double* R;
  double* J;  // [4L][nw] complex for this slowness
  cd reflectivity(cd r) {
    R[2 * k] = r.x;
    R[2 * k + 1] = r.y;
    return mk(1.0, 0.0);
  }
  void layer(int l, const Acc& a) {
    const cd v[4] = {a.a, a.b, a.r, a.h};
    for (int q = 0; q < 4; ++q) {
      J[2 * ((size_t)(q * L + l) * nw + k)] = v[q].x;
      J[2 * ((size_t)(q * L + l) * nw + k) + 1] = v[q].y;
    }
  }
};
}  // namespace

extern "C" void emu_jacobian(const double* tab, int L, const double* p, int n_p, const double* w,
                             int nw, int fs, double* R, double* J) {
  static LayerP lay[512];
  static LayerD dlay[512];
  static Iface f[512];
  static ScatTan t[512];
  const int I = L - 1;
  for (int j = 0; j < n_p; ++j) {
    for (int l = 0; l < L; ++l) {
      lay[l] = layer_terms(tab, L, l, p[j]);
      dlay[l] = layer_derivs(tab, L, l, p[j], lay[l]);
    }
    for (int i = 0; i < I; ++i) {
      f[i] = interface_coeffs(p[j], i, lay[i], lay[i + 1]);
      interface_tangents(p[j], i, lay[i], dlay[i], lay[i + 1], dlay[i + 1], t[i]);
    }
    const int seg = checkpoint_spacing(I - 1 > 0 ? I - 1 : 1);
    for (int k = 0; k < nw; ++k) {
      HostSink s{L, nw, k, R + 2 * (size_t)j * nw, J + 2 * (size_t)j * 4 * L * nw};
      jacobian_pair(L, mk(w[2 * k], w[2 * k + 1]), fs != 0, seg, lay, dlay, f, t,
                    PhaseDirect{mk(w[2 * k], w[2 * k + 1]), lay}, s);
    }
  }
}
