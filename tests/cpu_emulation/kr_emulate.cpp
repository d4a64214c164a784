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

// ---- second derivatives (kr_hvp.cuh): the per-pair dual-number code the hvp kernels run ----
#include "../../seismicinversion_b200/csrc/kr_hvp.cuh"

namespace {
struct HostDualSink {
  int L, nw, k, mode;  // mode 0: misfit H v (seed 2 conj(R - R_obs)), 1: d/dv of dR/dtheta
  cd robs;
  double* hv;   // [4L] accumulated H v (mode 0)
  double* jd;   // [4L][nw] complex for this slowness (mode 1)
  DC reflectivity(const DC& R) {
    if (mode == 1) return dc(mk(1.0, 0.0));
    const cd r = R.v - robs;
    return dc(mk(2.0 * r.x, -2.0 * r.y), mk(2.0 * R.t.x, -2.0 * R.t.y));
  }
  void layer(int l, const AccD& a) {
    const DC v[4] = {a.a, a.b, a.r, a.h};
    for (int q = 0; q < 4; ++q) {
      if (mode == 0) {
        hv[q * L + l] += v[q].t.x;
      } else {
        jd[2 * ((size_t)(q * L + l) * nw + k)] = v[q].t.x;
        jd[2 * ((size_t)(q * L + l) * nw + k) + 1] = v[q].t.y;
      }
    }
  }
};
}  // namespace

// mode 0: hv[4L] += H v of chi = sum |R - R_obs|^2 (R_obs [n_p][nw] complex);
// mode 1: jd [n_p][4L][nw] complex = d/dv of dR/dtheta.  v: [4L] direction.
extern "C" void emu_hvp(const double* tab, int L, const double* p, int n_p, const double* w,
                        int nw, int fs, const double* v, int mode, const double* R_obs,
                        double* hv, double* jd) {
  static LayerP lay[512];
  static LayerD dlay[512];
  static LayerD2 d2[512];
  static LayerV lv[512];
  static Iface f[512];
  static IfS<DC> ifs[512];
  static ScatTan t[512], tt[512];
  const int I = L - 1;
  for (int q = 0; q < 4 * L && mode == 0; ++q) hv[q] = 0.0;
  for (int j = 0; j < n_p; ++j) {
    for (int l = 0; l < L; ++l) {
      lay[l] = layer_terms(tab, L, l, p[j]);
      dlay[l] = layer_derivs(tab, L, l, p[j], lay[l]);
      d2[l] = layer_derivs2(tab, L, l, lay[l], dlay[l]);
      const double vl[4] = {v[l], v[L + l], v[2 * L + l], v[3 * L + l]};
      lv[l] = layer_dot(tab, L, l, lay[l], dlay[l], d2[l], vl);
    }
    for (int i = 0; i < I; ++i) {
      f[i] = interface_coeffs(p[j], i, lay[i], lay[i + 1]);
      interface_tangents(p[j], i, lay[i], dlay[i], lay[i + 1], dlay[i + 1], t[i]);
      IfS<DC> c;
      interface_dot(p[j], i, lv[i], lv[i + 1], c, tt[i]);
      ifs[i] = iface_dual(f[i], c);
    }
    for (int k = 0; k < nw; ++k) {
      HostDualSink s;
      s.L = L;
      s.nw = nw;
      s.k = k;
      s.mode = mode;
      s.robs = mode == 0 ? mk(R_obs[2 * ((size_t)j * nw + k)], R_obs[2 * ((size_t)j * nw + k) + 1])
                         : mk(0.0, 0.0);
      s.hv = hv;
      s.jd = mode == 1 ? jd + 2 * (size_t)j * 4 * L * nw : nullptr;
      hvp_pair(L, mk(w[2 * k], w[2 * k + 1]), fs != 0, lv, ifs, t, tt, s);
    }
  }
}

// ---- frequency sums of the adjoint (adjoint_pair_sums + sums_contract_layer), the path of
// the gradient / vector-Jacobian-product kernels ----
namespace {
struct HostSumSink {
  cd* sums;  // [L][12] of this slowness, summed over the frequencies
  int I;
  bool vjp;
  cd obs;
  cd res;
  cd reflectivity(cd R) {
    if (vjp) { res = mk(0.0, 0.0); return mk(obs.x, -obs.y); }
    res = R - obs;
    return mk(2.0 * res.x, -2.0 * res.y);
  }
  void top(cd f0) { sums[(size_t)I * kSumVals + 10] = sums[(size_t)I * kSumVals + 10] + f0; }
  void step(int i, const cd cbar[10], cd fa, cd fb) {
    cd* row = sums + (size_t)i * kSumVals;
    for (int k = 0; k < 10; ++k) row[k] = row[k] + cbar[k];
    row[10] = row[10] + fa;
    row[11] = row[11] + fb;
  }
};
}  // namespace

// out[4L + 1]: the misfit gradient (vjp = 0, obs = R_obs) or Re sum conj(gR) dR/dtheta
// (vjp = 1, obs = gR) over all slownesses and frequencies, then chi.
extern "C" void emu_gradient_sums(const double* tab, int L, const double* p, int n_p,
                                  const double* w, int nw, int fs, int vjp, const double* obs,
                                  double* out) {
  static LayerP lay[512];
  static LayerD dlay[512];
  static Iface f[512];
  static ScatTan t[512];
  static cd sums[512 * kSumVals];
  const int I = L - 1;
  for (int q = 0; q < 4 * L + 1; ++q) out[q] = 0.0;
  for (int j = 0; j < n_p; ++j) {
    for (int l = 0; l < L; ++l) {
      lay[l] = layer_terms(tab, L, l, p[j]);
      dlay[l] = layer_derivs(tab, L, l, p[j], lay[l]);
    }
    for (int i = 0; i < I; ++i) {
      f[i] = interface_coeffs(p[j], i, lay[i], lay[i + 1]);
      interface_tangents(p[j], i, lay[i], dlay[i], lay[i + 1], dlay[i + 1], t[i]);
    }
    for (size_t q = 0; q < sum_rows(L) * kSumVals; ++q) sums[q] = mk(0.0, 0.0);
    const int seg = checkpoint_spacing(I - 1 > 0 ? I - 1 : 1);
    for (int k = 0; k < nw; ++k) {
      const cd om = mk(w[2 * k], w[2 * k + 1]);
      HostSumSink s{sums, I, vjp != 0, mk(obs[2 * ((size_t)j * nw + k)],
                                          obs[2 * ((size_t)j * nw + k) + 1]), mk(0.0, 0.0)};
      adjoint_pair_sums(L, om, fs != 0, seg, f, PhaseDirect{om, lay}, s);
      out[4 * L] += s.res.x * s.res.x + s.res.y * s.res.y;
    }
    for (int l = 0; l < L; ++l) {
      double v[4];
      sums_contract_layer(l, L, sums, t, dlay, v);
      for (int q = 0; q < 4; ++q) out[q * L + l] += v[q];
    }
  }
}

// ---- frequency sums of the dual adjoint (hvp_pair_sums + hvp_sums_contract_layer), the path
// of the misfit Hessian-vector-product kernel ----
namespace {
struct HostDualSumSink {
  cd* sv;  // [L][12] value parts, summed over frequency
  cd* st;  // [L][12] tangent parts
  int I;
  cd robs;
  DC reflectivity(const DC& R) {
    const cd r = R.v - robs;
    return dc(mk(2.0 * r.x, -2.0 * r.y), mk(2.0 * R.t.x, -2.0 * R.t.y));
  }
  void add(int row, int k, const DC& x) {
    sv[(size_t)row * kSumVals + k] = sv[(size_t)row * kSumVals + k] + x.v;
    st[(size_t)row * kSumVals + k] = st[(size_t)row * kSumVals + k] + x.t;
  }
  void top(const DC& f0) { add(I, 10, f0); }
  void step(int i, const DC cbar[10], const DC& fa, const DC& fb) {
    for (int k = 0; k < 10; ++k) add(i, k, cbar[k]);
    add(i, 10, fa);
    add(i, 11, fb);
  }
};
}  // namespace

// hv[4L] = H v of chi = sum |R - R_obs|^2 by the frequency-sum dual path.
extern "C" void emu_hvp_sums(const double* tab, int L, const double* p, int n_p, const double* w,
                             int nw, int fs, const double* v, const double* R_obs, double* hv) {
  static LayerP lay[512];
  static LayerD dlay[512];
  static LayerD2 d2[512];
  static LayerV lv[512];
  static Iface f[512];
  static IfS<DC> ifs[512];
  static ScatTan t[512], tt[512];
  static cd sv[512 * kSumVals], st[512 * kSumVals];
  const int I = L - 1;
  for (int q = 0; q < 4 * L; ++q) hv[q] = 0.0;
  for (int j = 0; j < n_p; ++j) {
    for (int l = 0; l < L; ++l) {
      lay[l] = layer_terms(tab, L, l, p[j]);
      dlay[l] = layer_derivs(tab, L, l, p[j], lay[l]);
      d2[l] = layer_derivs2(tab, L, l, lay[l], dlay[l]);
      const double vl[4] = {v[l], v[L + l], v[2 * L + l], v[3 * L + l]};
      lv[l] = layer_dot(tab, L, l, lay[l], dlay[l], d2[l], vl);
    }
    for (int i = 0; i < I; ++i) {
      f[i] = interface_coeffs(p[j], i, lay[i], lay[i + 1]);
      interface_tangents(p[j], i, lay[i], dlay[i], lay[i + 1], dlay[i + 1], t[i]);
      IfS<DC> c;
      interface_dot(p[j], i, lv[i], lv[i + 1], c, tt[i]);
      ifs[i] = iface_dual(f[i], c);
    }
    for (size_t q = 0; q < (size_t)L * kSumVals; ++q) sv[q] = st[q] = mk(0.0, 0.0);
    for (int k = 0; k < nw; ++k) {
      HostDualSumSink s{sv, st, I, mk(R_obs[2 * ((size_t)j * nw + k)],
                                      R_obs[2 * ((size_t)j * nw + k) + 1])};
      hvp_pair_sums(L, mk(w[2 * k], w[2 * k + 1]), fs != 0, lv, ifs, s);
    }
    for (int l = 0; l < L; ++l) {
      double o[4];
      hvp_sums_contract_layer(l, L, sv, st, t, tt, lv, o);
      for (int q = 0; q < 4; ++q) hv[q * L + l] += o[q];
    }
  }
}
