// Derivatives of the Kennett path.
//
// R is a holomorphic function of every complex intermediate (coefficients, phase factors,
// the 2x2 matrices), so one reverse sweep per (omega, p) carries "adjoints"
// Zbar = dR/dZ (complex partial derivatives, no conjugation) from R down to
//   * the 10 independent coefficients of each interface (Rd, Ru symmetric, Td; Tu = Td^T),
//   * the two phase factors ea, eb of each layer.
// dR/dtheta for a real layer parameter theta is then sum_z zbar * dz/dtheta, with
// dz/dtheta from (i) forward-mode tangents of the coefficients (ScatTan, omega independent,
// once per slowness and interface) and (ii) closed-form phase derivatives:
//   ea = exp(omega * i eta h):  dea/dalpha = ea * omega * (i h deta/dalpha),
//                               dea/dh     = ea * omega * (i eta),        likewise eb.
// Primitive chains: ds/dv = -s/v (complex slowness), deta/dv = -s^2 / (eta v),
// d(beta_c)/dbeta = beta_c / beta (beta_c = 1/s_s); zero where beta = 0 and for the ocean
// S quantities; phase derivatives are zero in the half-space (phase fixed to 1), as in the
// reference's torch forward (kennett_torch.py:369-390, torch.where masks).
#pragma once

#include "kr_dual.cuh"
#include "kr_math.cuh"

namespace kr {

// ---------------- 2x2 complex matrix helpers ([[a, b], [c, d]]) ----------------
KR_HD M2 m2(cd a, cd b, cd c, cd d) { M2 r; r.a = a; r.b = b; r.c = c; r.d = d; return r; }
// A symmetric state as its three entries (the tape's storage) and back.
struct S3 {
  cd a, b, d;
};
KR_HD S3 s3(const M2& x) { S3 r; r.a = x.a; r.b = x.b; r.d = x.d; return r; }
KR_HD M2 m2(const S3& x) { return m2(x.a, x.b, x.b, x.d); }

// Per-layer derivative factors for one slowness.
struct LayerD {
  cd ca_alpha;  // d(ca)/d alpha = i h deta/dalpha      (0 in the half-space)
  cd cb_beta;   // d(cb)/d beta  = i h dneta/dbeta      (0 in the half-space / beta = 0)
  cd ca_h;      // d(ca)/d h     = i eta                (0 in the half-space)
  cd cb_h;      // d(cb)/d h     = i neta
  cd eta_alpha; // deta/dalpha
  cd neta_beta; // dneta/dbeta
  cd betac_beta;// dbeta_c/dbeta
};

KR_HD LayerD layer_derivs(const double* tab, int n_layers, int l, double p, const LayerP& lp) {
  const double alpha = tab[l];
  const double beta = tab[n_layers + l];
  const double h = tab[3 * n_layers + l];
  const double qa = tab[4 * n_layers + l];
  const double qb = tab[5 * n_layers + l];
  LayerD o;
  cd sp = complex_slowness(alpha, qa);
  o.eta_alpha = -((sp * sp) * recip(lp.eta * alpha));
  if (beta > 0.0 && l > 0) {
    cd ss = complex_slowness(beta, qb);
    o.neta_beta = -((ss * ss) * recip(lp.neta * beta));
    o.betac_beta = lp.betac * (1.0 / beta);
  } else {
    o.neta_beta = mk(0.0, 0.0);
    o.betac_beta = (beta > 0.0) ? lp.betac * (1.0 / beta) : mk(0.0, 0.0);
  }
  if (is_half_space(h)) {
    o.ca_alpha = o.cb_beta = o.ca_h = o.cb_h = mk(0.0, 0.0);
  } else {
    const cd ih = mk(0.0, h);
    o.ca_alpha = ih * o.eta_alpha;
    o.cb_beta = ih * o.neta_beta;
    o.ca_h = mk(-lp.eta.y, lp.eta.x);
    o.cb_h = mk(-lp.neta.y, lp.neta.x);
  }
  return o;
}

// Tangents of the 10 independent coefficients of interface `iface` with respect to
// (alpha_u, beta_u, rho_u, alpha_l, beta_l, rho_l) of the upper (u = iface) and lower
// (l = iface + 1) layer: t[k][j], k in coefficient order rd11 rd12 rd22 ru11 ru12 ru22
// td11 td12 td21 td22.
struct ScatTan {
  cd t[10][6];
};

// Column j of t (one tangent direction: forward mode with a single dual component).  The dual
// arithmetic acts on each tangent component separately, so the column is the one a pass over
// all six directions computes, with a sixth of the live state: the kernels run one thread per
// (slowness, interface, column) and nothing spills.
KR_HD void interface_tangent_col(double p, int iface, const LayerP& up, const LayerD& dup,
                                 const LayerP& lo, const LayerD& dlo, int j, cd col[10]) {
  typedef Dual<1> D;
  D eta1 = dconst<1>(up.eta), neta1 = dconst<1>(up.neta), rho1 = dconst<1>(to_c(up.rho));
  D betac1 = dconst<1>(up.betac);
  D eta2 = dconst<1>(lo.eta), neta2 = dconst<1>(lo.neta), rho2 = dconst<1>(to_c(lo.rho));
  D betac2 = dconst<1>(lo.betac);
  switch (j) {
    case 0: eta1.d[0] = dup.eta_alpha; break;
    case 1: neta1.d[0] = dup.neta_beta; betac1.d[0] = dup.betac_beta; break;
    case 2: rho1.d[0] = mk(1.0, 0.0); break;
    case 3: eta2.d[0] = dlo.eta_alpha; break;
    case 4: neta2.d[0] = dlo.neta_beta; betac2.d[0] = dlo.betac_beta; break;
    default: rho2.d[0] = mk(1.0, 0.0); break;
  }
  IfaceT<D> f;
  if (iface == 0)
    ocean_bottom<D>(p, eta1, rho1, eta2, neta2, rho2, betac2, f);
  else
    solid_solid<D>(p, eta1, neta1, rho1, betac1, eta2, neta2, rho2, betac2, f);
  col[0] = f.rd11.d[0];
  col[1] = f.rd12.d[0];
  col[2] = f.rd22.d[0];
  col[3] = f.ru11.d[0];
  col[4] = f.ru12.d[0];
  col[5] = f.ru22.d[0];
  col[6] = f.td11.d[0];
  col[7] = f.td12.d[0];
  col[8] = f.td21.d[0];
  col[9] = f.td22.d[0];
}

KR_HD void interface_tangents(double p, int iface, const LayerP& up, const LayerD& dup,
                              const LayerP& lo, const LayerD& dlo, ScatTan& out) {
  for (int j = 0; j < 6; ++j) {
    cd col[10];
    interface_tangent_col(p, iface, up, dup, lo, dlo, j, col);
    for (int k = 0; k < 10; ++k) out.t[k][j] = col[k];
  }
}

// Reverse of kennett_step, differentiating its symmetric adjugate form.  States and their
// adjoints are symmetric: the adjoint of an off-diagonal entry is that of the one value both
// positions share (ob.b; ob.c is not read and rbar.c is 0).  Inputs: the step's input state
// r, the phase factors, the interface, and ob = dR/d(step output).  Outputs:
// rbar = dR/d(step input), dR/dea, dR/deb and the 10 coefficient adjoints cbar (same order
// as ScatTan).  Forward, with P = ea^2, Q = eb^2, S = ea eb:
//   m = (P r11, S r12, Q r22),  dm = m11 m22 - m12^2,  dru = ru11 ru22 - ru12^2,
//   D = 1 - ru11 m11 - 2 ru12 m12 - ru22 m22 + dru dm,
//   A = (m11 - ru22 dm, m12 + ru12 dm, m22 - ru11 dm),  X = A / D,
//   out = Rd + Td^T X Td = Rd + q(Td) . X.
KR_HD void kennett_step_reverse(const M2& r, cd ea, cd eb, const Iface& f, const M2& ob,
                                M2& rbar, cd& eabar, cd& ebbar, cd cbar[10]) {
  // forward quantities, formed exactly as in kennett_step
  const cd P = ea * ea, Q = eb * eb, S = ea * eb;
  const cd m11 = P * r.a, m12 = S * r.b, m22 = Q * r.d;
  const cd dm = cdot2(m11, m22, -m12, m12);
  const cd one = mk(1.0, 0.0);
  const cd idet = recip(cmac(cmac(cmac(cmac(one, -f.ru11, m11), -f.ru12x2, m12), -f.ru22, m22),
                             f.dru, dm));
  const cd a11 = cmac(m11, -f.ru22, dm), a12 = cmac(m12, f.ru12, dm),
           a22 = cmac(m22, -f.ru11, dm);
  const cd x11 = a11 * idet, x12 = a12 * idet, x22 = a22 * idet;
  const cd o11 = ob.a, o12 = ob.b, o22 = ob.d;
  // out = Rd + q . X: adjoints of X, and of Td through the quadratic forms (W = X Td)
  const cd xb11 = cmac(cmac(f.q[0] * o11, f.q[3], o12), f.q[6], o22);
  const cd xb12 = cmac(cmac(f.q[1] * o11, f.q[4], o12), f.q[7], o22);
  const cd xb22 = cmac(cmac(f.q[2] * o11, f.q[5], o12), f.q[8], o22);
  const cd w1 = cdot2(f.td11, x11, f.td21, x12), w2 = cdot2(f.td11, x12, f.td21, x22);
  const cd w3 = cdot2(f.td12, x11, f.td22, x12), w4 = cdot2(f.td12, x12, f.td22, x22);
  const cd o11x2 = 2.0 * o11, o22x2 = 2.0 * o22;
  cbar[0] = o11;
  cbar[1] = o12;
  cbar[2] = o22;
  cbar[6] = cdot2(o11x2, w1, o12, w3);  // td11
  cbar[7] = cdot2(o12, w1, o22x2, w3);  // td12
  cbar[8] = cdot2(o11x2, w2, o12, w4);  // td21
  cbar[9] = cdot2(o12, w2, o22x2, w4);  // td22
  // X = A / D
  const cd ab11 = xb11 * idet, ab12 = xb12 * idet, ab22 = xb22 * idet;
  const cd Db = -(cmac(cdot2(xb11, a11, xb12, a12), xb22, a22) * (idet * idet));
  // A and D from m, dm and Ru
  const cd dmb = cmac(cmac(cmac(f.dru * Db, -f.ru22, ab11), f.ru12, ab12), -f.ru11, ab22);
  const cd mb11 = cmac(cmac(ab11, -f.ru11, Db), m22, dmb);
  const cd mb22 = cmac(cmac(ab22, -f.ru22, Db), m11, dmb);
  const cd mb12 = cmac(cmac(ab12, -f.ru12x2, Db), -2.0 * m12, dmb);
  const cd dDb = Db * dm;  // adjoint of dru
  cbar[3] = cmac(cmac(-(m11 * Db), f.ru22, dDb), -ab22, dm);                 // ru11
  cbar[4] = cmac(cmac(-2.0 * (m12 * Db), -f.ru12x2, dDb), ab12, dm);         // ru12
  cbar[5] = cmac(cmac(-(m22 * Db), f.ru11, dDb), -ab11, dm);                 // ru22
  // m = (P r11, S r12, Q r22)
  rbar = m2(mb11 * P, mb12 * S, mk(0.0, 0.0), mb22 * Q);
  const cd Sb = r.b * mb12;
  eabar = cmac(eb * Sb, 2.0 * ea, r.a * mb11);
  ebbar = cmac(ea * Sb, 2.0 * eb, r.d * mb22);
}

// Bytes of one slowness's derivative data in shared memory (layer terms, layer derivative
// factors, interface coefficients, coefficient tangents), 16-byte aligned sections.
KR_HD size_t pair_smem_bytes(int L) {
  return sizeof(LayerP) * (size_t)L + sizeof(LayerD) * (size_t)L +
         sizeof(Iface) * (size_t)(L - 1) + sizeof(ScatTan) * (size_t)(L - 1);
}

// dR/d(alpha, beta, rho, h) of one layer (Jacobian mode: complex), or, when the reverse
// sweep is seeded with 2 conj(R - R_obs), the misfit gradient's real contributions
// 2 Re(conj(R - R_obs) dR/dtheta) (gradient mode: only real parts are ever formed).
struct Acc {
  cd a, b, r, h;
};
struct AccR {
  double a, b, r, h;
};

KR_HD void set_zero(cd& x) { x = mk(0.0, 0.0); }
KR_HD void set_zero(double& x) { x = 0.0; }
KR_HD void acc_zero(Acc& z) { z.a = z.b = z.r = z.h = mk(0.0, 0.0); }
KR_HD void acc_zero(AccR& z) { z.a = z.b = z.r = z.h = 0.0; }
KR_HD Acc acc_zero() {
  Acc z;
  acc_zero(z);
  return z;
}
// s += x y (complex), or s += Re(x y) (real: 2 FP64 operations instead of 4)
KR_HD void acc_add(cd& s, cd x, cd y) { s = s + x * y; }
KR_HD void acc_add(double& s, cd x, cd y) { s = fma(x.x, y.x, fma(-x.y, y.y, s)); }

// Adds the coefficient-tangent contractions of one interface to its upper / lower layer.
template <class AccT>
KR_HD void contract(const ScatTan& t, const cd cbar[10], AccT& up, AccT& lo) {
  decltype(up.a) s[6];
  for (int j = 0; j < 6; ++j) set_zero(s[j]);
  for (int k = 0; k < 10; ++k) {
    if (cbar[k].x == 0.0 && cbar[k].y == 0.0) continue;
    for (int j = 0; j < 6; ++j) acc_add(s[j], cbar[k], t.t[k][j]);
  }
  up.a = up.a + s[0];
  up.b = up.b + s[1];
  up.r = up.r + s[2];
  lo.a = lo.a + s[3];
  lo.b = lo.b + s[4];
  lo.r = lo.r + s[5];
}

// Tape of one (omega, p) pair, in local memory: up to kSegMax steps of inputs (the three
// entries of the symmetric state) and phase factors (80 B per step; 48 B where the phases
// come from a table) plus kCpMax checkpoints.  64 steps hold every model of up to 66 layers
// outright, so those run without any recomputation; measured on an uneven batch of 3-64-layer
// models with the per-step contraction, the larger per-thread stack (~7 KB) cost far less
// than recomputing segments did (24 steps: 1080 ms, 40: 1049 ms, 64: 963 ms per batch).
// KR_TAPE_STEPS changes the length at build time.
#ifndef KR_TAPE_STEPS
#define KR_TAPE_STEPS 64
#endif
constexpr int kSegMax = KR_TAPE_STEPS;
constexpr int kCpMax = (256 - 2 + kSegMax - 1) / kSegMax;  // segments of the deepest model

// Steps per segment: one segment (a full tape, no recomputation) when the pair's steps fit
// the buffer, else the fewest segments of at most kSegMax steps, of balanced length.
KR_HD int checkpoint_spacing(int nsteps) {
  if (nsteps <= kSegMax) return nsteps > 0 ? nsteps : 1;
  const int nseg = (nsteps + kSegMax - 1) / kSegMax;
  return (nsteps + nseg - 1) / nseg;
}

// R and dR/dtheta for one (omega, p) pair; `ph` supplies the layer phase factors at omega
// (PhaseDirect or a tabulated source), `w` itself enters the phase derivatives.  The sink's
// reflectivity(R) returns the seed of the reverse sweep (1 for dR/dtheta itself,
// 2 conj(R - R_obs) for the misfit gradient) and its AccT picks complex or real
// accumulation.  Forward sweep storing the state every `seg` steps (and recording the top
// segment's step inputs and phases outright), then the reverse sweep top-down, every other
// segment recomputed from its checkpoint (no recomputation at all when the steps fit one
// segment).  sink.reflectivity(R) is called once before the reverse pass, sink.layer(l, acc)
// once per layer l (in order 0, 1, ..., L-1) with the finished dR/d(alpha_l, beta_l, rho_l,
// h_l).
#ifdef __CUDACC__
#pragma nv_exec_check_disable
#endif
template <class Sink, class Ph>
KR_HD void jacobian_pair(int L, cd w, bool free_surface, int seg, const LayerP* lay,
                         const LayerD* dlay, const Iface* coef, const ScatTan* tan, const Ph& ph,
                         Sink& sink) {
  const int I = L - 1;
  const int nsteps = I - 1;  // step s applies interface i = I - 2 - s
  const int ncp = nsteps > 0 ? (nsteps + seg - 1) / seg : 0;
  const int top0 = (ncp - 1) * seg;  // first step of the top segment (reversed first)
  S3 cp[kCpMax];
  S3 sg[kSegMax];
  cd sea[kSegMax], seb[kSegMax];
  // tabulated phase factors are recomputed in the reverse sweep (two products each) instead of
  // kept on the tape, as in adjoint_pair_sums
  const bool keep_ph = !ph.cheap();
  M2 r = m2(coef[I - 1].rd11, coef[I - 1].rd12, coef[I - 1].rd12, coef[I - 1].rd22);
  for (int s = 0; s < nsteps; ++s) {
    if (s % seg == 0) cp[s / seg] = s3(r);
    const int i = I - 2 - s;
    const cd ea = ph.a(i + 1), eb = ph.b(i + 1);
    if (s >= top0) {  // the top segment is recorded now and never recomputed
      sg[s - top0] = s3(r);
      if (keep_ph) {
        sea[s - top0] = ea;
        seb[s - top0] = eb;
      }
    }
    r = kennett_step(r, ea, eb, coef[i]);
  }
  typedef typename Sink::AccT AccT;
  const cd e0 = ph.a(0);
  const cd seed = sink.reflectivity(pp_surface(r.a, e0, free_surface));
  // top: R = E0^2 RRd_00, or y / (1 + y) with y = E0^2 RRd_00
  cd g = mk(1.0, 0.0);
  if (free_surface) {
    cd q = recip(1.0 + (e0 * e0) * r.a);
    g = q * q;
  }
  cd ob0 = (e0 * e0) * g;
  cd f0 = 2.0 * (e0 * r.a) * g * e0 * w;
  if (Sink::kSeeded) {
    ob0 = ob0 * seed;
    f0 = f0 * seed;
  }
  M2 ob = m2(ob0, mk(0.0, 0.0), mk(0.0, 0.0), mk(0.0, 0.0));
  AccT cur, nxt;
  acc_zero(cur);
  acc_zero(nxt);
  acc_add(cur.a, f0, dlay[0].ca_alpha);
  acc_add(cur.h, f0, dlay[0].ca_h);
  for (int q = ncp - 1; q >= 0; --q) {
    const int s0 = q * seg;
    const int s1 = s0 + seg < nsteps ? s0 + seg : nsteps;
    if (q != ncp - 1) {
      // recompute this segment's step inputs and phase factors from its checkpoint
      M2 x = m2(cp[q]);
      for (int s = s0; s < s1; ++s) {
        const int i = I - 2 - s;
        const cd ea = ph.a(i + 1), eb = ph.b(i + 1);
        sg[s - s0] = s3(x);
        if (keep_ph) {
          sea[s - s0] = ea;
          seb[s - s0] = eb;
        }
        if (s + 1 < s1) x = kennett_step(x, ea, eb, coef[i]);
      }
    }
    for (int s = s1 - 1; s >= s0; --s) {
      const int i = I - 2 - s;  // interface i, lower layer i + 1
      const cd ea = keep_ph ? sea[s - s0] : ph.a(i + 1);
      const cd eb = keep_ph ? seb[s - s0] : ph.b(i + 1);
      M2 rb;
      cd eab, ebb, cbar[10];
      kennett_step_reverse(m2(sg[s - s0]), ea, eb, coef[i], ob, rb, eab, ebb, cbar);
      contract(tan[i], cbar, cur, nxt);
      const LayerD& d = dlay[i + 1];
      const cd fa = eab * ea * w, fb = ebb * eb * w;
      acc_add(nxt.a, fa, d.ca_alpha);
      acc_add(nxt.b, fb, d.cb_beta);
      acc_add(nxt.h, fa, d.ca_h);
      acc_add(nxt.h, fb, d.cb_h);
      sink.layer(i, cur);
      cur = nxt;
      acc_zero(nxt);
      ob = rb;
    }
  }
  // bottom interface I-1 initialises RRd = Rd (ob.b: the symmetric off-diagonal's adjoint)
  cd cbar[10];
  cbar[0] = ob.a;
  cbar[1] = ob.b;
  cbar[2] = ob.d;
  for (int k = 3; k < 10; ++k) cbar[k] = mk(0.0, 0.0);
  contract(tan[I - 1], cbar, cur, nxt);
  sink.layer(I - 1, cur);
  sink.layer(L - 1, nxt);
}

}  // namespace kr

namespace kr {

// ------------------------------------------------------------------------------------------
// Frequency sums of the adjoint (misfit gradient, vector-Jacobian products).
//
// When only sum over (p, omega) of Re(seed dR/dtheta) is wanted, the contraction with the
// frequency-independent coefficient tangents and phase-derivative factors can wait until the
// per-step adjoints are summed over the frequencies:
//   sum_w Re(cbar_k(w) t_kj) = Re((sum_w cbar_k(w)) t_kj),
//   sum_w Re(fa(w) ca_alpha) = Re((sum_w fa(w)) ca_alpha),  fa = eabar ea w (likewise eb),
// so per (omega, p) and step the sweep only hands 12 complex values (the 10 coefficient
// adjoints of the interface and the phase terms fa, fb of the layer below it) to a summing
// sink, and one contraction per (p, interface) replaces the per-step 10 x 6 one.
// ------------------------------------------------------------------------------------------
constexpr int kSumVals = 12;  // per step: 10 coefficient adjoints, fa, fb

// Sum rows: row i < I holds interface i's 10 coefficient adjoints and the phase terms of
// layer i + 1 (slots 10, 11); row I holds the top phase term of layer 0 (slot 10).
KR_HD size_t sum_rows(int L) { return (size_t)L; }

// One (omega, p) pair: forward sweep with the tape of jacobian_pair, seed, reverse sweep; per
// step sink.step(i, cbar, fa, fb), once sink.top(f0) (the ocean phase term of layer 0).
#ifdef __CUDACC__
#pragma nv_exec_check_disable
#endif
template <class Sink, class Ph>
KR_HD void adjoint_pair_sums(int L, cd w, bool free_surface, int seg, const Iface* coef,
                             const Ph& ph, Sink& sink) {
  const int I = L - 1;
  const int nsteps = I - 1;  // step s applies interface i = I - 2 - s
  const int ncp = nsteps > 0 ? (nsteps + seg - 1) / seg : 0;
  const int top0 = (ncp - 1) * seg;
  S3 cp[kCpMax];
  S3 sg[kSegMax];
  cd sea[kSegMax], seb[kSegMax];
  // tabulated phase factors are recomputed in the reverse sweep (two products each) instead of
  // kept on the tape: 48 instead of 80 bytes of local memory per step
  const bool keep_ph = !ph.cheap();
  M2 r = m2(coef[I - 1].rd11, coef[I - 1].rd12, coef[I - 1].rd12, coef[I - 1].rd22);
  for (int s = 0; s < nsteps; ++s) {
    if (s % seg == 0) cp[s / seg] = s3(r);
    const int i = I - 2 - s;
    const cd ea = ph.a(i + 1), eb = ph.b(i + 1);
    if (s >= top0) {
      sg[s - top0] = s3(r);
      if (keep_ph) {
        sea[s - top0] = ea;
        seb[s - top0] = eb;
      }
    }
    r = kennett_step(r, ea, eb, coef[i]);
  }
  const cd e0 = ph.a(0);
  const cd seed = sink.reflectivity(pp_surface(r.a, e0, free_surface));
  cd g = mk(1.0, 0.0);
  if (free_surface) {
    cd q = recip(1.0 + (e0 * e0) * r.a);
    g = q * q;
  }
  const cd ob0 = ((e0 * e0) * g) * seed;
  const cd f0 = (2.0 * (e0 * r.a) * g * e0 * w) * seed;
  sink.top(f0);
  M2 ob = m2(ob0, mk(0.0, 0.0), mk(0.0, 0.0), mk(0.0, 0.0));
  for (int q = ncp - 1; q >= 0; --q) {
    const int s0 = q * seg;
    const int s1 = s0 + seg < nsteps ? s0 + seg : nsteps;
    if (q != ncp - 1) {
      M2 x = m2(cp[q]);
      for (int s = s0; s < s1; ++s) {
        const int i = I - 2 - s;
        const cd ea = ph.a(i + 1), eb = ph.b(i + 1);
        sg[s - s0] = s3(x);
        if (keep_ph) {
          sea[s - s0] = ea;
          seb[s - s0] = eb;
        }
        if (s + 1 < s1) x = kennett_step(x, ea, eb, coef[i]);
      }
    }
    for (int s = s1 - 1; s >= s0; --s) {
      const int i = I - 2 - s;
      const cd ea = keep_ph ? sea[s - s0] : ph.a(i + 1);
      const cd eb = keep_ph ? seb[s - s0] : ph.b(i + 1);
      M2 rb;
      cd eab, ebb, cbar[10];
      kennett_step_reverse(m2(sg[s - s0]), ea, eb, coef[i], ob, rb, eab, ebb, cbar);
      sink.step(i, cbar, eab * ea * w, ebb * eb * w);
      ob = rb;
    }
  }
  // bottom interface I-1 initialises RRd = Rd (ob.b: the symmetric off-diagonal's adjoint)
  cd cbar[10];
  cbar[0] = ob.a;
  cbar[1] = ob.b;
  cbar[2] = ob.d;
  for (int k = 3; k < 10; ++k) cbar[k] = mk(0.0, 0.0);
  sink.step(I - 1, cbar, mk(0.0, 0.0), mk(0.0, 0.0));
}

// The contraction of the summed rows for layer l: out[0..3] = Re of the alpha, beta, rho, h
// contributions (the interface above layer l contributes through its lower-layer tangents,
// the one below through its upper-layer tangents, plus the layer's phase terms).
KR_HD void sums_contract_layer(int l, int L, const cd* sums, const ScatTan* tan,
                               const LayerD* dlay, double out[4]) {
  const int I = L - 1;
  double a = 0.0, b = 0.0, r = 0.0, h = 0.0;
  if (l < I) {  // interface l: layer l is its upper layer (tangent columns 0..2)
    const cd* S = sums + (size_t)l * kSumVals;
    for (int k = 0; k < 10; ++k) {
      acc_add(a, S[k], tan[l].t[k][0]);
      acc_add(b, S[k], tan[l].t[k][1]);
      acc_add(r, S[k], tan[l].t[k][2]);
    }
  }
  cd A = mk(0.0, 0.0), B = mk(0.0, 0.0);
  if (l > 0) {  // interface l - 1: layer l is its lower layer (columns 3..5)
    const cd* S = sums + (size_t)(l - 1) * kSumVals;
    for (int k = 0; k < 10; ++k) {
      acc_add(a, S[k], tan[l - 1].t[k][3]);
      acc_add(b, S[k], tan[l - 1].t[k][4]);
      acc_add(r, S[k], tan[l - 1].t[k][5]);
    }
    A = S[10];
    B = S[11];
  } else {
    A = sums[(size_t)I * kSumVals + 10];
  }
  const LayerD& d = dlay[l];
  acc_add(a, A, d.ca_alpha);
  acc_add(b, B, d.cb_beta);
  acc_add(h, A, d.ca_h);
  acc_add(h, B, d.cb_h);
  out[0] = a;
  out[1] = b;
  out[2] = r;
  out[3] = h;
}

}  // namespace kr
