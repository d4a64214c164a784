// Second derivatives of the Kennett path by forward-mode differentiation of the adjoint
// ("tangent of the adjoint").
//
// Every quantity of the reflectivity's reverse sweep (kr_adjoint.cuh) is carried as a dual
// complex number DC = (value, tangent), the tangent being its derivative along one direction
// v of the layer parameters theta = (alpha_l, beta_l, rho_l, h_l).  Running the forward sweep,
// the seed and the reverse sweep in DC gives, besides the adjoints of kr_adjoint.cuh, their
// derivatives along v; contracting those with the coefficient tangents ScatTan (first
// derivatives) and their own derivatives along v (second derivatives of the interface
// coefficients, from nested dual numbers through the same coefficient formulas) yields
//   * d/dv of the misfit gradient, i.e. the Hessian-vector product H v of
//     chi = sum |R - R_obs|^2 (seed 2 conj(R - R_obs) with tangent 2 conj(dR/dv)), exactly,
//     with no step size;
//   * d/dv of the Jacobian dR/dtheta (seed 1), which makes torch.func.hessian through the
//     differentiable forward exact.
// This is the exact second derivative the reference obtains with torch.func.hessian
// (reverse over reverse through its autograd graph, Kennett_Reflectivity/kennett_torch.py:644-684,
// taup_inversion.py:177) computed here as forward over reverse.
//
// Second derivatives of the per-layer primitives (closed forms, zero in the half-space and for
// the ocean's S quantities, as the first derivatives):
//   eta^2 = s^2 - p^2, s = c / alpha:  eta_a = -s^2 / (alpha eta),
//                                      eta_aa = (3 s^2 / alpha^2 - eta_a^2) / eta,
// likewise neta with beta; beta_c = beta / c_s is linear in beta (second derivative 0).
#pragma once

#include "kr_adjoint.cuh"

namespace kr {

// ------------------------------------------------------------------------------------
// Dual complex numbers: value and tangent along the direction v.
// ------------------------------------------------------------------------------------
struct DC {
  cd v, t;
};

KR_HD DC dc(cd v, cd t) { DC r; r.v = v; r.t = t; return r; }
KR_HD DC dc(cd v) { return dc(v, mk(0.0, 0.0)); }
KR_HD DC operator+(const DC& a, const DC& b) { return dc(a.v + b.v, a.t + b.t); }
KR_HD DC operator-(const DC& a, const DC& b) { return dc(a.v - b.v, a.t - b.t); }
KR_HD DC operator-(const DC& a) { return dc(-a.v, -a.t); }
KR_HD DC operator*(const DC& a, const DC& b) { return dc(a.v * b.v, cdot2(a.t, b.v, a.v, b.t)); }
KR_HD DC operator*(double s, const DC& a) { return dc(s * a.v, s * a.t); }
KR_HD DC operator*(const DC& a, double s) { return dc(s * a.v, s * a.t); }
KR_HD DC operator*(cd s, const DC& a) { return dc(s * a.v, s * a.t); }
KR_HD DC operator*(const DC& a, cd s) { return dc(a.v * s, a.t * s); }
KR_HD DC operator+(const DC& a, double s) { return dc(a.v + s, a.t); }
KR_HD DC operator+(double s, const DC& a) { return dc(a.v + s, a.t); }
KR_HD DC operator-(double s, const DC& a) { return dc(s - a.v, -a.t); }
KR_HD DC operator-(const DC& a, double s) { return dc(a.v - s, a.t); }
KR_HD DC conj(const DC& a) { return dc(conj(a.v), conj(a.t)); }
KR_HD DC recip(const DC& a) {
  const cd r = recip(a.v);
  return dc(r, -(a.t * (r * r)));
}
KR_HD DC csqrt(const DC& a) {
  const cd r = csqrt(a.v);
  // A zero tangent stays zero even where sqrt has an infinite derivative (sqrt(0)).
  const cd t = (a.t.x == 0.0 && a.t.y == 0.0) ? mk(0.0, 0.0) : a.t * recip(2.0 * r);
  return dc(r, t);
}
KR_HD DC cexp_(const DC& a) {
  const cd e = cexp_(a.v);
  return dc(e, e * a.t);
}
// s + a b and a b + c d, value parts rounded exactly as the complex versions
KR_HD DC cmac(const DC& s, const DC& a, const DC& b) {
  return dc(cmac(s.v, a.v, b.v), cmac(cmac(s.t, a.t, b.v), a.v, b.t));
}
KR_HD DC cdot2(const DC& a, const DC& b, const DC& c, const DC& d) {
  return dc(cdot2(a.v, b.v, c.v, d.v), cmac(cmac(cdot2(a.t, b.v, a.v, b.t), c.t, d.v), c.v, d.t));
}

// Scalar constants of either type.
template <class S> KR_HD S sconst(cd v);
template <> KR_HD cd sconst<cd>(cd v) { return v; }
template <> KR_HD DC sconst<DC>(cd v) { return dc(v); }

// ------------------------------------------------------------------------------------
// Nested dual numbers over a base scalar S (S = DC: first derivatives with respect to the six
// parameters of an interface, each carried with its own derivative along v).
// ------------------------------------------------------------------------------------
template <int N, class S>
struct DualG {
  S v;
  S d[N];
};

template <int N, class S>
KR_HD DualG<N, S> gconst(S v) {
  DualG<N, S> r;
  r.v = v;
  for (int k = 0; k < N; ++k) r.d[k] = sconst<S>(mk(0.0, 0.0));
  return r;
}
template <int N, class S>
KR_HD DualG<N, S> operator+(const DualG<N, S>& a, const DualG<N, S>& b) {
  DualG<N, S> r;
  r.v = a.v + b.v;
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int N, class S>
KR_HD DualG<N, S> operator-(const DualG<N, S>& a, const DualG<N, S>& b) {
  DualG<N, S> r;
  r.v = a.v - b.v;
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int N, class S>
KR_HD DualG<N, S> operator-(const DualG<N, S>& a) {
  DualG<N, S> r;
  r.v = -a.v;
  for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int N, class S>
KR_HD DualG<N, S> operator*(const DualG<N, S>& a, const DualG<N, S>& b) {
  DualG<N, S> r;
  r.v = a.v * b.v;
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int N, class S>
KR_HD DualG<N, S> operator*(cd s, const DualG<N, S>& a) {
  DualG<N, S> r;
  r.v = s * a.v;
  for (int k = 0; k < N; ++k) r.d[k] = s * a.d[k];
  return r;
}
template <int N, class S>
KR_HD DualG<N, S> operator*(double s, const DualG<N, S>& a) {
  DualG<N, S> r;
  r.v = s * a.v;
  for (int k = 0; k < N; ++k) r.d[k] = s * a.d[k];
  return r;
}
template <int N, class S>
KR_HD DualG<N, S> operator*(const DualG<N, S>& a, double s) { return s * a; }
template <int N, class S>
KR_HD DualG<N, S> operator+(const DualG<N, S>& a, double s) {
  DualG<N, S> r = a;
  r.v = a.v + s;
  return r;
}
template <int N, class S>
KR_HD DualG<N, S> operator-(double s, const DualG<N, S>& a) { return -a + s; }
template <int N, class S>
KR_HD DualG<N, S> recip(const DualG<N, S>& a) {
  DualG<N, S> r;
  r.v = recip(a.v);
  const S m = -(r.v * r.v);
  for (int k = 0; k < N; ++k) r.d[k] = m * a.d[k];
  return r;
}
KR_HD bool is_zero(const cd& x) { return x.x == 0.0 && x.y == 0.0; }
KR_HD bool is_zero(const DC& x) { return is_zero(x.v) && is_zero(x.t); }
template <int N, class S>
KR_HD DualG<N, S> csqrt(const DualG<N, S>& a) {
  DualG<N, S> r;
  r.v = csqrt(a.v);
  const S h = recip(2.0 * r.v);
  for (int k = 0; k < N; ++k) r.d[k] = is_zero(a.d[k]) ? sconst<S>(mk(0.0, 0.0)) : h * a.d[k];
  return r;
}

// ------------------------------------------------------------------------------------
// The Kennett step and its reverse on a generic scalar (the arithmetic of kennett_step and
// kennett_step_reverse, written once for cd and DC).
// ------------------------------------------------------------------------------------
template <class S>
struct IfS {  // interface coefficients and the step's derived constants (as Iface)
  S rd11, rd12, rd22, ru11, ru12, ru22, td11, td12, td21, td22;
  S ru12x2, dru;
  S q[9];
};
template <class S>
struct SymS {  // symmetric 2x2 state (a, b; b, d)
  S a, b, d;
};

template <class S>
KR_HD void iface_derived(IfS<S>& o) {
  const S t11 = o.td11, t12 = o.td12, t21 = o.td21, t22 = o.td22;
  o.ru12x2 = 2.0 * o.ru12;
  o.dru = cdot2(o.ru11, o.ru22, -o.ru12, o.ru12);
  o.q[0] = t11 * t11;
  o.q[1] = 2.0 * (t11 * t21);
  o.q[2] = t21 * t21;
  o.q[3] = t11 * t12;
  o.q[4] = cdot2(t11, t22, t21, t12);
  o.q[5] = t21 * t22;
  o.q[6] = t12 * t12;
  o.q[7] = 2.0 * (t12 * t22);
  o.q[8] = t22 * t22;
}

template <class S>
KR_HD SymS<S> step_s(const SymS<S>& r, const S& ea, const S& eb, const IfS<S>& f) {
  const S eaea = ea * ea, ebeb = eb * eb, eaeb = ea * eb;
  const S m11 = eaea * r.a, m12 = eaeb * r.b, m22 = ebeb * r.d;
  const S dm = cdot2(m11, m22, -m12, m12);
  const S one = sconst<S>(mk(1.0, 0.0));
  const S idet = recip(cmac(cmac(cmac(cmac(one, -f.ru11, m11), -f.ru12x2, m12), -f.ru22, m22),
                            f.dru, dm));
  const S x11 = cmac(m11, -f.ru22, dm) * idet;
  const S x12 = cmac(m12, f.ru12, dm) * idet;
  const S x22 = cmac(m22, -f.ru11, dm) * idet;
  SymS<S> o;
  o.a = cmac(cmac(cmac(f.rd11, f.q[0], x11), f.q[1], x12), f.q[2], x22);
  o.b = cmac(cmac(cmac(f.rd12, f.q[3], x11), f.q[4], x12), f.q[5], x22);
  o.d = cmac(cmac(cmac(f.rd22, f.q[6], x11), f.q[7], x12), f.q[8], x22);
  return o;
}

// Reverse of step_s (see kennett_step_reverse for the forward it differentiates).  ob: the
// adjoint of the step's output (ob.b = the one off-diagonal value's); outputs rbar (adjoint
// of the input state), eabar, ebbar and the 10 coefficient adjoints in ScatTan order.
template <class S>
KR_HD void step_reverse_s(const SymS<S>& r, const S& ea, const S& eb, const IfS<S>& f,
                          const SymS<S>& ob, SymS<S>& rbar, S& eabar, S& ebbar, S cbar[10]) {
  const S P = ea * ea, Q = eb * eb, Sx = ea * eb;
  const S m11 = P * r.a, m12 = Sx * r.b, m22 = Q * r.d;
  const S dm = cdot2(m11, m22, -m12, m12);
  const S one = sconst<S>(mk(1.0, 0.0));
  const S idet = recip(cmac(cmac(cmac(cmac(one, -f.ru11, m11), -f.ru12x2, m12), -f.ru22, m22),
                            f.dru, dm));
  const S a11 = cmac(m11, -f.ru22, dm), a12 = cmac(m12, f.ru12, dm), a22 = cmac(m22, -f.ru11, dm);
  const S x11 = a11 * idet, x12 = a12 * idet, x22 = a22 * idet;
  const S o11 = ob.a, o12 = ob.b, o22 = ob.d;
  const S xb11 = cmac(cmac(f.q[0] * o11, f.q[3], o12), f.q[6], o22);
  const S xb12 = cmac(cmac(f.q[1] * o11, f.q[4], o12), f.q[7], o22);
  const S xb22 = cmac(cmac(f.q[2] * o11, f.q[5], o12), f.q[8], o22);
  const S w1 = cdot2(f.td11, x11, f.td21, x12), w2 = cdot2(f.td11, x12, f.td21, x22);
  const S w3 = cdot2(f.td12, x11, f.td22, x12), w4 = cdot2(f.td12, x12, f.td22, x22);
  const S o11x2 = 2.0 * o11, o22x2 = 2.0 * o22;
  cbar[0] = o11;
  cbar[1] = o12;
  cbar[2] = o22;
  cbar[6] = cdot2(o11x2, w1, o12, w3);
  cbar[7] = cdot2(o12, w1, o22x2, w3);
  cbar[8] = cdot2(o11x2, w2, o12, w4);
  cbar[9] = cdot2(o12, w2, o22x2, w4);
  const S ab11 = xb11 * idet, ab12 = xb12 * idet, ab22 = xb22 * idet;
  const S Db = -(cmac(cdot2(xb11, a11, xb12, a12), xb22, a22) * (idet * idet));
  const S dmb = cmac(cmac(cmac(f.dru * Db, -f.ru22, ab11), f.ru12, ab12), -f.ru11, ab22);
  const S mb11 = cmac(cmac(ab11, -f.ru11, Db), m22, dmb);
  const S mb22 = cmac(cmac(ab22, -f.ru22, Db), m11, dmb);
  const S mb12 = cmac(cmac(ab12, -f.ru12x2, Db), -2.0 * m12, dmb);
  const S dDb = Db * dm;
  cbar[3] = cmac(cmac(-(m11 * Db), f.ru22, dDb), -ab22, dm);
  cbar[4] = cmac(cmac(-2.0 * (m12 * Db), -f.ru12x2, dDb), ab12, dm);
  cbar[5] = cmac(cmac(-(m22 * Db), f.ru11, dDb), -ab11, dm);
  rbar.a = mb11 * P;
  rbar.b = mb12 * Sx;
  rbar.d = mb22 * Q;
  const S Sb = r.b * mb12;
  eabar = cmac(eb * Sb, 2.0 * ea, r.a * mb11);
  ebbar = cmac(ea * Sb, 2.0 * eb, r.d * mb22);
}

// ------------------------------------------------------------------------------------
// Per-(slowness, direction) derivative data.
// ------------------------------------------------------------------------------------
// Second-derivative factors of one layer: d(eta_alpha)/d alpha and d(neta_beta)/d beta
// (zero for the ocean's S quantities and where beta = 0).
struct LayerD2 {
  cd eta_aa, neta_bb;
};

KR_HD LayerD2 layer_derivs2(const double* tab, int n_layers, int l, const LayerP& lp,
                            const LayerD& d) {
  const double alpha = tab[l];
  const double beta = tab[n_layers + l];
  const double qa = tab[4 * n_layers + l];
  const double qb = tab[5 * n_layers + l];
  LayerD2 o;
  const cd sp = complex_slowness(alpha, qa);
  // (3 s^2 / alpha^2 - eta_a^2) / eta
  o.eta_aa = (((3.0 / (alpha * alpha)) * (sp * sp)) - d.eta_alpha * d.eta_alpha) * recip(lp.eta);
  if (beta > 0.0 && l > 0) {
    const cd ss = complex_slowness(beta, qb);
    o.neta_bb = (((3.0 / (beta * beta)) * (ss * ss)) - d.neta_beta * d.neta_beta) * recip(lp.neta);
  } else {
    o.neta_bb = mk(0.0, 0.0);
  }
  return o;
}

// One layer's values and tangents along v: the layer terms used by the coefficients and the
// phases, and the derivative factors used by the phase contributions.
struct LayerV {
  DC eta, neta, betac, rho;  // rho as a complex scalar (value, tangent v_rho)
  DC ca, cb;                 // phase exponents i eta h, i neta h (0 in the half-space)
  DC ca_alpha, cb_beta, ca_h, cb_h;  // derivative factors of the phases and their tangents
  DC eta_alpha, neta_beta, betac_beta;  // first derivatives of the primitives and tangents
};

// vl = (v_alpha, v_beta, v_rho, v_h) of layer l.
KR_HD LayerV layer_dot(const double* tab, int n_layers, int l, const LayerP& lp, const LayerD& d,
                       const LayerD2& d2, const double vl[4]) {
  const double h = tab[3 * n_layers + l];
  const double va = vl[0], vb = vl[1], vr = vl[2], vh = vl[3];
  LayerV o;
  const cd eta_a_t = va * d2.eta_aa, neta_b_t = vb * d2.neta_bb;
  o.eta = dc(lp.eta, va * d.eta_alpha);
  o.neta = dc(lp.neta, vb * d.neta_beta);
  o.betac = dc(lp.betac, vb * d.betac_beta);
  o.rho = dc(to_c(lp.rho), to_c(vr));
  o.eta_alpha = dc(d.eta_alpha, eta_a_t);
  o.neta_beta = dc(d.neta_beta, neta_b_t);
  o.betac_beta = dc(d.betac_beta);
  if (is_half_space(h)) {
    const DC z = dc(mk(0.0, 0.0));
    o.ca = o.cb = o.ca_alpha = o.cb_beta = o.ca_h = o.cb_h = z;
  } else {
    // ca = i eta h: tangent i (eta_a v_a h + eta v_h)
    o.ca = dc(lp.ca, cmac(va * d.ca_alpha, d.ca_h, to_c(vh)));
    o.cb = dc(lp.cb, cmac(vb * d.cb_beta, d.cb_h, to_c(vh)));
    const cd i1 = mk(0.0, 1.0);
    // ca_alpha = i h eta_a: tangent i (v_h eta_a + h eta_aa v_a); ca_h = i eta: i eta_a v_a
    o.ca_alpha = dc(d.ca_alpha, i1 * cmac(vh * d.eta_alpha, to_c(h), eta_a_t));
    o.cb_beta = dc(d.cb_beta, i1 * cmac(vh * d.neta_beta, to_c(h), neta_b_t));
    o.ca_h = dc(d.ca_h, i1 * (va * d.eta_alpha));
    o.cb_h = dc(d.cb_h, i1 * (vb * d.neta_beta));
  }
  return o;
}

// Coefficient tangents along v and their own derivatives: out_c[k] = coefficient k as DC
// (value, d/dv), out_t.t[k][j] = d coefficient_k / d theta_j along v (the tangent of the
// ScatTan entry), for the interface between layers `iface` (upper) and iface + 1 (lower).
// interface_dot_col computes column j alone (nested duals with one outer direction, the
// component-wise arithmetic of the six-direction pass) and, given out_c, the coefficients.
KR_HD void interface_dot_col(double p, int iface, const LayerV& up, const LayerV& lo, int j,
                             IfS<DC>* out_c, cd col[10]) {
  typedef DualG<1, DC> G;
  G eta1 = gconst<1>(up.eta), neta1 = gconst<1>(up.neta), rho1 = gconst<1>(up.rho);
  G betac1 = gconst<1>(up.betac);
  G eta2 = gconst<1>(lo.eta), neta2 = gconst<1>(lo.neta), rho2 = gconst<1>(lo.rho);
  G betac2 = gconst<1>(lo.betac);
  switch (j) {
    case 0: eta1.d[0] = up.eta_alpha; break;
    case 1: neta1.d[0] = up.neta_beta; betac1.d[0] = up.betac_beta; break;
    case 2: rho1.d[0] = dc(mk(1.0, 0.0)); break;
    case 3: eta2.d[0] = lo.eta_alpha; break;
    case 4: neta2.d[0] = lo.neta_beta; betac2.d[0] = lo.betac_beta; break;
    default: rho2.d[0] = dc(mk(1.0, 0.0)); break;
  }
  IfaceT<G> f;
  if (iface == 0)
    ocean_bottom<G>(p, eta1, rho1, eta2, neta2, rho2, betac2, f);
  else
    solid_solid<G>(p, eta1, neta1, rho1, betac1, eta2, neta2, rho2, betac2, f);
  const G* c[10] = {&f.rd11, &f.rd12, &f.rd22, &f.ru11, &f.ru12,
                    &f.ru22, &f.td11, &f.td12, &f.td21, &f.td22};
  for (int k = 0; k < 10; ++k) col[k] = c[k]->d[0].t;
  if (out_c) {
    DC* oc[10] = {&out_c->rd11, &out_c->rd12, &out_c->rd22, &out_c->ru11, &out_c->ru12,
                  &out_c->ru22, &out_c->td11, &out_c->td12, &out_c->td21, &out_c->td22};
    for (int k = 0; k < 10; ++k) *oc[k] = c[k]->v;
    iface_derived(*out_c);
  }
}

KR_HD void interface_dot(double p, int iface, const LayerV& up, const LayerV& lo, IfS<DC>& out_c,
                         ScatTan& out_t) {
  for (int j = 0; j < 6; ++j) {
    cd col[10];
    interface_dot_col(p, iface, up, lo, j, j == 0 ? &out_c : nullptr, col);
    for (int k = 0; k < 10; ++k) out_t.t[k][j] = col[k];
  }
}

// The interface as IfS<DC> from the value coefficients and the value-plus-tangent ones
// (values from the exact Iface the first-order kernels use, tangents from interface_dot).
KR_HD IfS<DC> iface_dual(const Iface& f, const IfS<DC>& d) {
  IfS<DC> o;
  o.rd11 = dc(f.rd11, d.rd11.t);
  o.rd12 = dc(f.rd12, d.rd12.t);
  o.rd22 = dc(f.rd22, d.rd22.t);
  o.ru11 = dc(f.ru11, d.ru11.t);
  o.ru12 = dc(f.ru12, d.ru12.t);
  o.ru22 = dc(f.ru22, d.ru22.t);
  o.td11 = dc(f.td11, d.td11.t);
  o.td12 = dc(f.td12, d.td12.t);
  o.td21 = dc(f.td21, d.td21.t);
  o.td22 = dc(f.td22, d.td22.t);
  o.ru12x2 = dc(f.ru12x2, d.ru12x2.t);
  o.dru = dc(f.dru, d.dru.t);
  for (int k = 0; k < 9; ++k) o.q[k] = dc(f.q[k], d.q[k].t);
  return o;
}

// ------------------------------------------------------------------------------------
// One (omega, p, direction): forward sweep in DC with a tape of the step inputs, seed, reverse
// sweep in DC.  The sink receives, per layer l in order 0..L-1, the DC contributions
// (value = first derivative, tangent = its derivative along v) of the layer's alpha, beta,
// rho, h, with the coefficient contraction sum_k cbar_k t_kj done per pair.
// ------------------------------------------------------------------------------------
constexpr int kHvpSeg = 32;   // tape steps held at once
constexpr int kHvpCp = 8;     // checkpoints: models of up to 258 layers

struct AccD {
  DC a, b, r, h;
};

KR_HD void accd_zero(AccD& z) { z.a = z.b = z.r = z.h = dc(mk(0.0, 0.0)); }

// z += x y on DC
KR_HD void accd_add(DC& s, const DC& x, const DC& y) { s = cmac(s, x, y); }

// coefficient contraction of one interface: up / lo get sum_k cbar_k t_kj (as DC, the tangent
// from cbar's tangent with t and cbar's value with t's tangent)
KR_HD void contract_dual(const ScatTan& t, const ScatTan& tt, const DC cbar[10], AccD& up,
                         AccD& lo) {
  DC s[6];
  for (int j = 0; j < 6; ++j) s[j] = dc(mk(0.0, 0.0));
  for (int k = 0; k < 10; ++k) {
    if (is_zero(cbar[k])) continue;
    for (int j = 0; j < 6; ++j) {
      s[j].v = cmac(s[j].v, cbar[k].v, t.t[k][j]);
      s[j].t = cmac(cmac(s[j].t, cbar[k].t, t.t[k][j]), cbar[k].v, tt.t[k][j]);
    }
  }
  up.a = up.a + s[0];
  up.b = up.b + s[1];
  up.r = up.r + s[2];
  lo.a = lo.a + s[3];
  lo.b = lo.b + s[4];
  lo.r = lo.r + s[5];
}

KR_HD int hvp_spacing(int nsteps) {
  if (nsteps <= kHvpSeg) return nsteps > 0 ? nsteps : 1;
  const int nseg = (nsteps + kHvpSeg - 1) / kHvpSeg;
  return (nsteps + nseg - 1) / nseg;
}

// lv: per-layer LayerV (values and tangents), coef: value interfaces (Iface), cdot: the
// interfaces as IfS<DC> (value + tangent), tan / tant: ScatTan and its tangent per interface.
// seed(R) returns the DC seed of the reverse sweep (1 for the Jacobian, 2 conj(R - R_obs) for
// the misfit gradient); sink.layer(l, AccD) as in jacobian_pair.
#ifdef __CUDACC__
#pragma nv_exec_check_disable
#endif
template <class Sink>
KR_HD void hvp_pair(int L, cd w, bool free_surface, const LayerV* lv, const IfS<DC>* ifs,
                    const ScatTan* tan, const ScatTan* tant, Sink& sink) {
  const int I = L - 1;
  const int nsteps = I - 1;  // step s applies interface i = I - 2 - s
  const int seg = hvp_spacing(nsteps);
  const int ncp = nsteps > 0 ? (nsteps + seg - 1) / seg : 0;
  const DC W = dc(w);
  SymS<DC> cp[kHvpCp];
  SymS<DC> sg[kHvpSeg];
  DC sea[kHvpSeg], seb[kHvpSeg];  // the steps' phase factors, kept for the reverse sweep
  SymS<DC> r;
  r.a = ifs[I - 1].rd11;
  r.b = ifs[I - 1].rd12;
  r.d = ifs[I - 1].rd22;
  for (int s = 0; s < nsteps; ++s) {
    if (s % seg == 0) cp[s / seg] = r;
    const int i = I - 2 - s;
    const DC ea = cexp_(W * lv[i + 1].ca), eb = cexp_(W * lv[i + 1].cb);
    if (s >= (ncp - 1) * seg) {
      const int k = s - (ncp - 1) * seg;
      sg[k] = r;
      sea[k] = ea;
      seb[k] = eb;
    }
    r = step_s(r, ea, eb, ifs[i]);
  }
  const DC e0 = cexp_(W * lv[0].ca);
  // top: R = y or y / (1 + y), y = e0^2 RRd_00
  const DC y = (e0 * e0) * r.a;
  DC g = dc(mk(1.0, 0.0));
  DC R = y;
  if (free_surface) {
    const DC q = recip(1.0 + y);
    R = y * q;
    g = q * q;
  }
  const DC seed = sink.reflectivity(R);
  const DC ob0 = ((e0 * e0) * g) * seed;
  const DC f0 = ((2.0 * (e0 * r.a)) * g) * ((e0 * W) * seed);
  SymS<DC> ob;
  ob.a = ob0;
  ob.b = ob.d = dc(mk(0.0, 0.0));
  AccD cur, nxt;
  accd_zero(cur);
  accd_zero(nxt);
  accd_add(cur.a, f0, lv[0].ca_alpha);
  accd_add(cur.h, f0, lv[0].ca_h);
  for (int q = ncp - 1; q >= 0; --q) {
    const int s0 = q * seg;
    const int s1 = s0 + seg < nsteps ? s0 + seg : nsteps;
    if (q != ncp - 1) {
      SymS<DC> x = cp[q];
      for (int s = s0; s < s1; ++s) {
        const int i = I - 2 - s;
        const DC ea = cexp_(W * lv[i + 1].ca), eb = cexp_(W * lv[i + 1].cb);
        sg[s - s0] = x;
        sea[s - s0] = ea;
        seb[s - s0] = eb;
        if (s + 1 < s1) x = step_s(x, ea, eb, ifs[i]);
      }
    }
    for (int s = s1 - 1; s >= s0; --s) {
      const int i = I - 2 - s;
      const DC ea = sea[s - s0], eb = seb[s - s0];
      SymS<DC> rb;
      DC eab, ebb, cbar[10];
      step_reverse_s(sg[s - s0], ea, eb, ifs[i], ob, rb, eab, ebb, cbar);
      contract_dual(tan[i], tant[i], cbar, cur, nxt);
      const LayerV& d = lv[i + 1];
      const DC fa = eab * (ea * W), fb = ebb * (eb * W);
      accd_add(nxt.a, fa, d.ca_alpha);
      accd_add(nxt.b, fb, d.cb_beta);
      accd_add(nxt.h, fa, d.ca_h);
      accd_add(nxt.h, fb, d.cb_h);
      sink.layer(i, cur);
      cur = nxt;
      accd_zero(nxt);
      ob = rb;
    }
  }
  DC cbar[10];
  cbar[0] = ob.a;
  cbar[1] = ob.b;
  cbar[2] = ob.d;
  for (int k = 3; k < 10; ++k) cbar[k] = dc(mk(0.0, 0.0));
  contract_dual(tan[I - 1], tant[I - 1], cbar, cur, nxt);
  sink.layer(I - 1, cur);
  sink.layer(L - 1, nxt);
}

}  // namespace kr

namespace kr {

// ------------------------------------------------------------------------------------------
// Frequency sums of the dual adjoint (misfit Hessian-vector products): as adjoint_pair_sums,
// the sink receives per step the dual coefficient adjoints and phase terms, and the
// contraction with the (frequency-independent) coefficient tangents, their derivatives along
// v and the phase-derivative factors runs once per (p, direction, interface) on the sums:
//   (H v)_j = Re( sum_w dcbar_k(w) t_kj + sum_w cbar_k(w) dt_kj ) + phase terms alike.
// ------------------------------------------------------------------------------------------
#ifdef __CUDACC__
#pragma nv_exec_check_disable
#endif
template <class Sink>
KR_HD void hvp_pair_sums(int L, cd w, bool free_surface, const LayerV* lv, const IfS<DC>* ifs,
                         Sink& sink) {
  const int I = L - 1;
  const int nsteps = I - 1;
  const int seg = hvp_spacing(nsteps);
  const int ncp = nsteps > 0 ? (nsteps + seg - 1) / seg : 0;
  const DC W = dc(w);
  SymS<DC> cp[kHvpCp];
  SymS<DC> sg[kHvpSeg];
  DC sea[kHvpSeg], seb[kHvpSeg];  // the steps' phase factors, kept for the reverse sweep
  SymS<DC> r;
  r.a = ifs[I - 1].rd11;
  r.b = ifs[I - 1].rd12;
  r.d = ifs[I - 1].rd22;
  for (int s = 0; s < nsteps; ++s) {
    if (s % seg == 0) cp[s / seg] = r;
    const int i = I - 2 - s;
    const DC ea = cexp_(W * lv[i + 1].ca), eb = cexp_(W * lv[i + 1].cb);
    if (s >= (ncp - 1) * seg) {
      const int k = s - (ncp - 1) * seg;
      sg[k] = r;
      sea[k] = ea;
      seb[k] = eb;
    }
    r = step_s(r, ea, eb, ifs[i]);
  }
  const DC e0 = cexp_(W * lv[0].ca);
  const DC y = (e0 * e0) * r.a;
  DC g = dc(mk(1.0, 0.0));
  DC R = y;
  if (free_surface) {
    const DC q = recip(1.0 + y);
    R = y * q;
    g = q * q;
  }
  const DC seed = sink.reflectivity(R);
  const DC ob0 = ((e0 * e0) * g) * seed;
  const DC f0 = ((2.0 * (e0 * r.a)) * g) * ((e0 * W) * seed);
  sink.top(f0);
  SymS<DC> ob;
  ob.a = ob0;
  ob.b = ob.d = dc(mk(0.0, 0.0));
  for (int q = ncp - 1; q >= 0; --q) {
    const int s0 = q * seg;
    const int s1 = s0 + seg < nsteps ? s0 + seg : nsteps;
    if (q != ncp - 1) {
      SymS<DC> x = cp[q];
      for (int s = s0; s < s1; ++s) {
        const int i = I - 2 - s;
        const DC ea = cexp_(W * lv[i + 1].ca), eb = cexp_(W * lv[i + 1].cb);
        sg[s - s0] = x;
        sea[s - s0] = ea;
        seb[s - s0] = eb;
        if (s + 1 < s1) x = step_s(x, ea, eb, ifs[i]);
      }
    }
    for (int s = s1 - 1; s >= s0; --s) {
      const int i = I - 2 - s;
      const DC ea = sea[s - s0], eb = seb[s - s0];
      SymS<DC> rb;
      DC eab, ebb, cbar[10];
      step_reverse_s(sg[s - s0], ea, eb, ifs[i], ob, rb, eab, ebb, cbar);
      sink.step(i, cbar, eab * (ea * W), ebb * (eb * W));
      ob = rb;
    }
  }
  DC cbar[10];
  cbar[0] = ob.a;
  cbar[1] = ob.b;
  cbar[2] = ob.d;
  for (int k = 3; k < 10; ++k) cbar[k] = dc(mk(0.0, 0.0));
  sink.step(I - 1, cbar, dc(mk(0.0, 0.0)), dc(mk(0.0, 0.0)));
}

// Re of the tangent of the alpha, beta, rho, h contributions of layer l from the summed rows
// (sv: value parts, st: tangent parts, the row layout of sums_contract_layer): t / tt are the
// coefficient tangents and their derivatives along v, lv the layer's values and tangents.
KR_HD void hvp_sums_contract_layer(int l, int L, const cd* sv, const cd* st, const ScatTan* t,
                                   const ScatTan* tt, const LayerV* lv, double out[4]) {
  const int I = L - 1;
  double a = 0.0, b = 0.0, r = 0.0, h = 0.0;
  if (l < I) {
    const cd* V = sv + (size_t)l * kSumVals;
    const cd* T = st + (size_t)l * kSumVals;
    for (int k = 0; k < 10; ++k) {
      acc_add(a, T[k], t[l].t[k][0]);
      acc_add(b, T[k], t[l].t[k][1]);
      acc_add(r, T[k], t[l].t[k][2]);
      acc_add(a, V[k], tt[l].t[k][0]);
      acc_add(b, V[k], tt[l].t[k][1]);
      acc_add(r, V[k], tt[l].t[k][2]);
    }
  }
  DC A = dc(mk(0.0, 0.0)), B = dc(mk(0.0, 0.0));
  if (l > 0) {
    const cd* V = sv + (size_t)(l - 1) * kSumVals;
    const cd* T = st + (size_t)(l - 1) * kSumVals;
    for (int k = 0; k < 10; ++k) {
      acc_add(a, T[k], t[l - 1].t[k][3]);
      acc_add(b, T[k], t[l - 1].t[k][4]);
      acc_add(r, T[k], t[l - 1].t[k][5]);
      acc_add(a, V[k], tt[l - 1].t[k][3]);
      acc_add(b, V[k], tt[l - 1].t[k][4]);
      acc_add(r, V[k], tt[l - 1].t[k][5]);
    }
    A = dc(V[10], T[10]);
    B = dc(V[11], T[11]);
  } else {
    A = dc(sv[(size_t)I * kSumVals + 10], st[(size_t)I * kSumVals + 10]);
  }
  const LayerV& d = lv[l];
  // Re of the tangent of A ca_alpha etc.: dA ca_alpha + A dca_alpha
  acc_add(a, A.t, d.ca_alpha.v);
  acc_add(a, A.v, d.ca_alpha.t);
  acc_add(b, B.t, d.cb_beta.v);
  acc_add(b, B.v, d.cb_beta.t);
  acc_add(h, A.t, d.ca_h.v);
  acc_add(h, A.v, d.ca_h.t);
  acc_add(h, B.t, d.cb_h.v);
  acc_add(h, B.v, d.cb_h.t);
  out[0] = a;
  out[1] = b;
  out[2] = r;
  out[3] = h;
}

}  // namespace kr
