// Complex FP64 arithmetic, layer slownesses, interface scattering coefficients and the
// Kennett 2x2 addition step, shared by every kernel of the library.
//
// Physics follows tmnestor/SeismicInversion, Kennett_Reflectivity/:
//   complex slowness      layer_model.py:15-45
//   vertical slowness     layer_model.py:48-74   (Im(eta) > 0 branch, flip when Im <= 0)
//   solid-solid coeffs    scattering_matrices.py:42-161
//   ocean-bottom coeffs   scattering_matrices.py:164-296
//   Kennett step          kennett_reflectivity.py:227-256
//   PP + free surface     kennett_reflectivity.py:264-326
//
// Storage choices (ours): Rd and Ru are symmetric and Tu = Td^T (reciprocity,
// scattering_matrices.py:150), so an interface is 10 complex numbers.  The 2x2 inverse is
// one reciprocal of the determinant times the adjugate.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define KR_HD __host__ __device__ __forceinline__
#else
#define KR_HD inline
#endif

namespace kr {

struct alignas(16) cd {  // 16-byte aligned: one 128-bit load / store per complex value
  double x, y;
};

KR_HD cd mk(double x, double y) { cd r; r.x = x; r.y = y; return r; }
KR_HD cd operator+(cd a, cd b) { return mk(a.x + b.x, a.y + b.y); }
KR_HD cd operator-(cd a, cd b) { return mk(a.x - b.x, a.y - b.y); }
KR_HD cd operator-(cd a) { return mk(-a.x, -a.y); }
KR_HD cd operator*(cd a, cd b) {
  return mk(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
KR_HD cd operator*(double s, cd a) { return mk(s * a.x, s * a.y); }
KR_HD cd operator*(cd a, double s) { return mk(s * a.x, s * a.y); }
KR_HD cd operator+(cd a, double s) { return mk(a.x + s, a.y); }
KR_HD cd operator+(double s, cd a) { return mk(a.x + s, a.y); }
KR_HD cd operator-(double s, cd a) { return mk(s - a.x, -a.y); }
KR_HD cd operator-(cd a, double s) { return mk(a.x - s, a.y); }
KR_HD cd conj(cd a) { return mk(a.x, -a.y); }
// Fused complex multiply-accumulate: s + a b with two FMAs per component (one rounding per
// FMA, no separate product and sum), and a b + c d as one multiply and three FMAs per
// component.  Operand negations are free in an FMA, so s - a b is cmac(s, -a, b).
KR_HD cd cmac(cd s, cd a, cd b) {
  return mk(fma(a.x, b.x, fma(-a.y, b.y, s.x)), fma(a.x, b.y, fma(a.y, b.x, s.y)));
}
KR_HD cd cdot2(cd a, cd b, cd c, cd d) {
  return mk(fma(a.x, b.x, fma(-a.y, b.y, fma(c.x, d.x, -(c.y * d.y)))),
            fma(a.x, b.y, fma(a.y, b.x, fma(c.x, d.y, c.y * d.x))));
}
KR_HD cd cmac2(cd s, cd a, cd b, cd c, cd d) { return cmac(cmac(s, c, d), a, b); }
KR_HD double abs2(cd a) { return fma(a.x, a.x, a.y * a.y); }

// 1/z via the conjugate over |z|^2, with a prescale by 1e-150 or 1e150 so that |z|^2 neither
// overflows nor underflows for the magnitudes met here (down to ~1e-150).
KR_HD cd recip(cd z) {
  double m = fmax(fabs(z.x), fabs(z.y));
  double s = 1.0;
  if (m > 1e150) s = 1e-150; else if (m < 1e-150 && m > 0.0) s = 1e150;
  double zx = z.x * s, zy = z.y * s;
  double inv = 1.0 / fma(zx, zx, zy * zy);
  return mk(zx * inv * s, -zy * inv * s);
}
KR_HD cd operator/(cd a, cd b) { return a * recip(b); }
KR_HD cd operator/(cd a, double s) { return mk(a.x / s, a.y / s); }

// Principal square root, branch cut on the negative real axis, sqrt(conj z) = conj sqrt z
// (C99 csqrt semantics, the convention NumPy and torch use).
KR_HD cd csqrt(cd z) {
  if (z.x == 0.0 && z.y == 0.0) return mk(0.0, z.y);
  double t = sqrt(0.5 * (fabs(z.x) + hypot(z.x, z.y)));
  if (z.x >= 0.0) return mk(t, z.y / (2.0 * t));
  return mk(fabs(z.y) / (2.0 * t), copysign(t, z.y));
}

KR_HD cd cexp_(cd z) {
  double e = exp(z.x);
  double s, c;
#ifdef __CUDA_ARCH__
  sincos(z.y, &s, &c);
#else
  s = sin(z.y);
  c = cos(z.y);
#endif
  return mk(e * c, e * s);
}

// Complex slowness of a layer with velocity v and quality factor Q.
KR_HD cd complex_slowness(double v, double Q) {
  double q2 = 2.0 * Q;
  double q2sq = q2 * q2;
  double den = (1.0 + q2sq) * v;
  return mk(q2sq / den, q2 / den);
}

// eta = sqrt((s + p)(s - p)) with Im(eta) > 0.
KR_HD cd vertical_slowness(cd s, double p) {
  cd t = (s + p) * (s - p);
  cd e = csqrt(t);
  if (e.y <= 0.0) e = -e;
  return e;
}

KR_HD bool is_half_space(double h) { return !(h < 1e30); }  // +inf, >= 1e30 (and NaN)

// ---------------------------------------------------------------------------------------
// Per-layer quantities for one slowness.
// ---------------------------------------------------------------------------------------
struct LayerP {
  cd eta;    // vertical P slowness
  cd neta;   // vertical S slowness (0 in the ocean)
  cd betac;  // complex S velocity 1/s_s (0 where beta = 0)
  cd ca;     // i * eta * h   (0 for the half-space: phase factor exactly 1)
  cd cb;     // i * neta * h
  double rho;
  double pad;  // 96 bytes: arrays of LayerP are whole 16-byte units (vector copies)
};

// Phase factors exp(omega * i eta h) and exp(omega * i neta h) of layer l, evaluated directly
// (kernels on uniform frequency grids use a tabulated source with the same a(l) / b(l)).
struct PhaseDirect {
  cd w;
  const LayerP* lay;
  KR_HD cd a(int l) const { return cexp_(w * lay[l].ca); }
  KR_HD cd b(int l) const { return cexp_(w * lay[l].cb); }
};

// Layer table layout (device or host): 6 rows of n_layers doubles:
// alpha, beta, rho, thickness, Q_alpha, Q_beta.
KR_HD LayerP layer_terms(const double* tab, int n_layers, int l, double p) {
  const double alpha = tab[l];
  const double beta = tab[n_layers + l];
  const double rho = tab[2 * n_layers + l];
  const double h = tab[3 * n_layers + l];
  const double qa = tab[4 * n_layers + l];
  const double qb = tab[5 * n_layers + l];
  LayerP o;
  cd sp = complex_slowness(alpha, qa);
  cd ss = beta > 0.0 ? complex_slowness(beta, qb) : mk(0.0, 0.0);
  o.betac = (ss.x != 0.0 || ss.y != 0.0) ? recip(ss) : mk(0.0, 0.0);
  o.eta = vertical_slowness(sp, p);
  o.neta = (l == 0) ? mk(0.0, 0.0) : vertical_slowness(ss, p);
  if (is_half_space(h)) {
    o.ca = mk(0.0, 0.0);
    o.cb = mk(0.0, 0.0);
  } else {
    o.ca = mk(-o.eta.y * h, o.eta.x * h);
    o.cb = mk(-o.neta.y * h, o.neta.x * h);
  }
  o.rho = rho;
  o.pad = 0.0;
  return o;
}

// ---------------------------------------------------------------------------------------
// Interface coefficients: Rd, Ru symmetric (3 entries each), Td full (Tu = Td^T).
// ---------------------------------------------------------------------------------------
template <class T>
struct IfaceT {
  T rd11, rd12, rd22;
  T ru11, ru12, ru22;
  T td11, td12, td21, td22;
};
typedef IfaceT<cd> Iface;

// Scalar-generic so that the same code yields values (T = cd) and forward-mode tangents
// (T = a dual number).  rho enters as T so its tangent can be seeded.
template <class T>
KR_HD void solid_solid(double p, T eta1, T neta1, T rho1, T beta1, T eta2, T neta2, T rho2,
                       T beta2, IfaceT<T>& o) {
  T rteta1 = csqrt(eta1), rteta2 = csqrt(eta2);
  T rtneta1 = csqrt(neta1), rtneta2 = csqrt(neta2);
  T rtrho1 = csqrt(rho1), rtrho2 = csqrt(rho2);
  T rtza1 = rteta1 * rtrho1, rtza2 = rteta2 * rtrho2;
  T rtzb1 = rtneta1 * rtrho1, rtzb2 = rtneta2 * rtrho2;
  const double psq = p * p;
  T dmu = rho2 * beta2 * beta2 - rho1 * beta1 * beta1;
  T d = 2.0 * dmu;
  T psqd = psq * d;
  T a = (rho2 - rho1) - psqd;
  T b = rho2 - psqd;
  T c = rho1 + psqd;
  T E = b * eta1 + c * eta2;
  T F = b * neta1 + c * neta2;
  T G = a - d * eta1 * neta2;
  T H = a - d * eta2 * neta1;
  T det = E * F + G * H * psq;
  T idet = recip(det);
  E = E * idet;
  F = F * idet;
  G = G * idet;
  H = H * idet;
  T Qv = (b * eta1 - c * eta2) * F;
  T Rv = (a + d * eta1 * neta2) * H * psq;
  T Sv = (a * b + c * d * eta2 * neta2) * p * idet;
  T Tv = (b * neta1 - c * neta2) * E;
  T Uv = (a + d * eta2 * neta1) * G * psq;
  T Vv = (a * c + b * d * eta1 * neta1) * p * idet;
  const cd m2i = mk(0.0, -2.0);
  o.rd11 = Qv - Rv;
  o.rd12 = m2i * (rteta1 * rtneta1 * Sv);
  o.rd22 = Tv - Uv;
  o.ru11 = -(Qv + Uv);
  o.ru12 = m2i * (rteta2 * rtneta2 * Vv);
  o.ru22 = -(Tv + Rv);
  o.td11 = 2.0 * (rtza1 * rtza2 * F);
  o.td12 = m2i * (rtzb1 * rtza2 * G * p);
  o.td21 = m2i * (rtza1 * rtzb2 * H * p);
  o.td22 = 2.0 * (rtzb1 * rtzb2 * E);
}

template <class T>
KR_HD void ocean_bottom(double p, T eta1, T rho1, T eta2, T neta2, T rho2, T beta2,
                        IfaceT<T>& o) {
  T rteta1 = csqrt(eta1), rteta2 = csqrt(eta2), rtneta2 = csqrt(neta2);
  T rtrho1 = csqrt(rho1), rtrho2 = csqrt(rho2);
  T rtza1 = rtrho1 * rteta1, rtza2 = rtrho2 * rteta2, rtzb2 = rtrho2 * rtneta2;
  const double psq = p * p;
  T d = 2.0 * (rho2 * beta2 * beta2);
  T psqd = psq * d;
  T a = (rho2 - rho1) - psqd;
  T b = rho2 - psqd;
  T c = rho1 + psqd;
  T E = b * eta1 + c * eta2;
  T F = b;
  T G = a - d * eta1 * neta2;
  T H = -(d * eta2);
  T det = E * F + G * H * psq;
  T idet = recip(det);
  E = E * idet;
  F = F * idet;
  G = G * idet;
  H = H * idet;
  T T1 = (b * eta1 - c * eta2) * F;
  T T2 = (a + d * eta1 * neta2) * H * psq;
  T T4 = b * E;
  T T5 = d * eta2 * G * psq;
  T T6 = b * d * eta1 * p * idet;
  const cd mi = mk(0.0, -1.0);
  T zero = 0.0 * rho1;
  o.rd11 = T1 - T2;
  o.rd12 = zero;
  o.rd22 = zero;
  o.ru11 = -(T1 + T5);
  o.ru12 = mi * (2.0 * (rteta2 * rtneta2 * T6));
  o.ru22 = -(T2 + T4);
  o.td11 = 2.0 * (rtza1 * rtza2 * F);
  o.td12 = zero;
  o.td21 = mi * (2.0 * (rtza1 * rtzb2 * H * p));
  o.td22 = zero;
}

KR_HD cd to_c(double r) { return mk(r, 0.0); }

// Coefficients of interface `iface` (between layers iface and iface+1) from layer terms.
KR_HD Iface interface_coeffs(double p, int iface, const LayerP& up, const LayerP& lo) {
  Iface o;
  if (iface == 0)
    ocean_bottom<cd>(p, up.eta, to_c(up.rho), lo.eta, lo.neta, to_c(lo.rho), lo.betac, o);
  else
    solid_solid<cd>(p, up.eta, up.neta, to_c(up.rho), up.betac, lo.eta, lo.neta, to_c(lo.rho),
                    lo.betac, o);
  return o;
}

// ---------------------------------------------------------------------------------------
// One Kennett addition step: RRd <- Rd + Tu MT (I - Ru MT)^-1 Td with MT = E RRd E,
// E = diag(ea, eb) of the layer below the interface.  RRd = [[a, b], [c, d]].
//
// RRd is symmetric in exact arithmetic, but the two off-diagonal entries carry different
// rounding, and at large slowness (evanescent layers, near-cancelling interface
// determinants) the recursion amplifies rounding by ~1e6-1e8: carrying one off-diagonal
// for both positions loses 1e-8 relative accuracy against an extended-precision
// evaluation, the full matrix keeps the reference's ~1e-10.  So the step carries all four
// entries, in the reference's product order (kennett_reflectivity.py:235-256).
// ---------------------------------------------------------------------------------------
struct M2 {
  cd a, b, c, d;
};

KR_HD M2 kennett_step(const M2& r, cd ea, cd eb, const Iface& f) {
  cd eaea = ea * ea, ebeb = eb * eb, eaeb = ea * eb;
  cd m11 = eaea * r.a, m12 = eaeb * r.b, m21 = eaeb * r.c, m22 = ebeb * r.d;
  // N = I - Ru MT
  const cd one = mk(1.0, 0.0);
  cd n11 = cmac2(one, -f.ru11, m11, -f.ru12, m21);
  cd n12 = cdot2(-f.ru11, m12, -f.ru12, m22);
  cd n21 = cdot2(-f.ru12, m11, -f.ru22, m21);
  cd n22 = cmac2(one, -f.ru12, m12, -f.ru22, m22);
  cd idet = recip(cdot2(n11, n22, -n12, n21));
  cd u11 = n22 * idet, u12 = -(n12 * idet), u21 = -(n21 * idet), u22 = n11 * idet;
  cd x11 = cdot2(m11, u11, m12, u21), x12 = cdot2(m11, u12, m12, u22);
  cd x21 = cdot2(m21, u11, m22, u21), x22 = cdot2(m21, u12, m22, u22);
  // Tu X with Tu = Td^T
  cd z11 = cdot2(f.td11, x11, f.td21, x21), z12 = cdot2(f.td11, x12, f.td21, x22);
  cd z21 = cdot2(f.td12, x11, f.td22, x21), z22 = cdot2(f.td12, x12, f.td22, x22);
  M2 o;
  o.a = cmac2(f.rd11, z11, f.td11, z12, f.td21);
  o.b = cmac2(f.rd12, z11, f.td12, z12, f.td22);
  o.c = cmac2(f.rd12, z21, f.td11, z22, f.td21);
  o.d = cmac2(f.rd22, z21, f.td12, z22, f.td22);
  return o;
}

// The last (ocean-bottom) step, returning only RRd_00: that interface's Rd has one entry and
// Td one column (Td = [[t11, 0], [t21, 0]]), so RRd_00 = rd11 + t11 (x11 t11 + x12 t21)
// + t21 (x21 t11 + x22 t21) with X = MT (I - Ru MT)^-1 (same products as kennett_step).
KR_HD cd kennett_last_step_pp(const M2& r, cd ea, cd eb, const Iface& f) {
  cd eaea = ea * ea, ebeb = eb * eb, eaeb = ea * eb;
  cd m11 = eaea * r.a, m12 = eaeb * r.b, m21 = eaeb * r.c, m22 = ebeb * r.d;
  const cd one = mk(1.0, 0.0);
  cd n11 = cmac2(one, -f.ru11, m11, -f.ru12, m21);
  cd n12 = cdot2(-f.ru11, m12, -f.ru12, m22);
  cd n21 = cdot2(-f.ru12, m11, -f.ru22, m21);
  cd n22 = cmac2(one, -f.ru12, m12, -f.ru22, m22);
  cd idet = recip(cdot2(n11, n22, -n12, n21));
  cd u11 = n22 * idet, u12 = -(n12 * idet), u21 = -(n21 * idet), u22 = n11 * idet;
  cd x11 = cdot2(m11, u11, m12, u21), x12 = cdot2(m11, u12, m12, u22);
  cd x21 = cdot2(m21, u11, m22, u21), x22 = cdot2(m21, u12, m22, u22);
  cd z11 = cdot2(f.td11, x11, f.td21, x21), z12 = cdot2(f.td11, x12, f.td21, x22);
  return cmac2(f.rd11, z11, f.td11, z12, f.td21);
}

// PP reflectivity at the surface from RRd_PP below the ocean and the ocean phase e0.
KR_HD cd pp_surface(cd rpp, cd e0, bool free_surface) {
  cd y = (e0 * e0) * rpp;
  if (!free_surface) return y;
  return y * recip(1.0 + y);
}

}  // namespace kr
