// Test-only references for the conditioning of the Kennett recursion: the reference's
// full-matrix step (kennett_reflectivity.py:235-256: MT = E RRd E, U = (I - Ru MT)^-1,
// RRd = Rd + Tu MT U Td, all four entries carried) evaluated
//   mode 0: in 80-bit extended precision (x86 long double) from the layer table up, the
//           stand-in for exact arithmetic;
//   mode 1: in double, as the reference evaluates it.
// The interface coefficients come from the same scalar-generic formulas as the kernels'
// (kr_math.cuh solid_solid / ocean_bottom), instantiated on an extended complex type.
#include <math.h>

#include "../../seismicinversion_b200/csrc/kr_math.cuh"

using namespace kr;

namespace {

template <class R>
struct C {
  R x, y;
};
template <class R> C<R> mkc(R x, R y) { C<R> r; r.x = x; r.y = y; return r; }
template <class R> C<R> operator+(C<R> a, C<R> b) { return mkc<R>(a.x + b.x, a.y + b.y); }
template <class R> C<R> operator-(C<R> a, C<R> b) { return mkc<R>(a.x - b.x, a.y - b.y); }
template <class R> C<R> operator-(C<R> a) { return mkc<R>(-a.x, -a.y); }
template <class R> C<R> operator*(C<R> a, C<R> b) {
  return mkc<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class R> C<R> operator*(double s, C<R> a) { return mkc<R>(s * a.x, s * a.y); }
template <class R> C<R> operator*(C<R> a, double s) { return mkc<R>(s * a.x, s * a.y); }
template <class R> C<R> operator*(cd s, C<R> a) { return mkc<R>(s.x, s.y) * a; }
template <class R> C<R> operator+(C<R> a, double s) { return mkc<R>(a.x + s, a.y); }
template <class R> C<R> operator+(double s, C<R> a) { return mkc<R>(a.x + s, a.y); }
template <class R> C<R> operator-(double s, C<R> a) { return mkc<R>(s - a.x, -a.y); }
template <class R> C<R> recip(C<R> z) {
  const R d = z.x * z.x + z.y * z.y;
  return mkc<R>(z.x / d, -z.y / d);
}
template <class R> C<R> csqrt(C<R> z) {  // principal branch, C99 csqrt conventions
  if (z.x == 0 && z.y == 0) return mkc<R>(0, z.y);
  const R t = std::sqrt((R)0.5 * (std::fabs(z.x) + std::hypot(z.x, z.y)));
  if (z.x >= 0) return mkc<R>(t, z.y / (2 * t));
  return mkc<R>(std::fabs(z.y) / (2 * t), std::copysign(t, z.y));
}
template <class R> C<R> cexpc(C<R> z) {
  const R e = std::exp(z.x);
  return mkc<R>(e * std::cos(z.y), e * std::sin(z.y));
}

template <class R>
C<R> slowness(R v, R Q) {
  const R q2 = 2 * Q, q2sq = q2 * q2, den = (1 + q2sq) * v;
  return mkc<R>(q2sq / den, q2 / den);
}

template <class R>
C<R> vertical(C<R> s, R p) {
  C<R> e = csqrt((s + mkc<R>(p, 0)) * (s - mkc<R>(p, 0)));
  if (e.y <= 0) e = -e;
  return e;
}

template <class R>
C<R> reflect(const double* tab, int L, double p, double wr, double wi, bool fs) {
  typedef C<R> T;
  const int I = L - 1;
  T eta[512], neta[512], bc[512], rho[512];
  for (int l = 0; l < L; ++l) {
    const R a = tab[l], b = tab[L + l], qa = tab[4 * L + l], qb = tab[5 * L + l];
    const T sp = slowness<R>(a, qa);
    const T ss = b > 0 ? slowness<R>(b, qb) : mkc<R>(0, 0);
    bc[l] = (ss.x != 0 || ss.y != 0) ? recip(ss) : mkc<R>(0, 0);
    eta[l] = vertical<R>(sp, (R)p);
    neta[l] = l == 0 ? mkc<R>(0, 0) : vertical<R>(ss, (R)p);
    rho[l] = mkc<R>(tab[2 * L + l], 0);
  }
  const T W = mkc<R>(wr, wi);
  auto phase = [&](int l, bool s) {
    const double h = tab[3 * L + l];
    if (!(h < 1e30)) return mkc<R>(1, 0);
    const T e = s ? neta[l] : eta[l];
    return cexpc(W * mkc<R>(-e.y * (R)h, e.x * (R)h));
  };
  IfaceT<T> f;
  auto coeffs = [&](int i) {
    if (i == 0)
      ocean_bottom<T>(p, eta[0], rho[0], eta[1], neta[1], rho[1], bc[1], f);
    else
      solid_solid<T>(p, eta[i], neta[i], rho[i], bc[i], eta[i + 1], neta[i + 1], rho[i + 1],
                     bc[i + 1], f);
  };
  coeffs(I - 1);
  T a = f.rd11, b = f.rd12, c = f.rd12, d = f.rd22;
  for (int i = I - 2; i >= 0; --i) {
    coeffs(i);
    const T ea = phase(i + 1, false), eb = phase(i + 1, true);
    const T m11 = ea * ea * a, m12 = ea * eb * b, m21 = ea * eb * c, m22 = eb * eb * d;
    const T n11 = 1.0 - (f.ru11 * m11 + f.ru12 * m21), n12 = -(f.ru11 * m12 + f.ru12 * m22);
    const T n21 = -(f.ru12 * m11 + f.ru22 * m21), n22 = 1.0 - (f.ru12 * m12 + f.ru22 * m22);
    const T id = recip(n11 * n22 - n12 * n21);
    const T u11 = n22 * id, u12 = -(n12 * id), u21 = -(n21 * id), u22 = n11 * id;
    const T x11 = m11 * u11 + m12 * u21, x12 = m11 * u12 + m12 * u22;
    const T x21 = m21 * u11 + m22 * u21, x22 = m21 * u12 + m22 * u22;
    const T z11 = f.td11 * x11 + f.td21 * x21, z12 = f.td11 * x12 + f.td21 * x22;
    const T z21 = f.td12 * x11 + f.td22 * x21, z22 = f.td12 * x12 + f.td22 * x22;
    a = f.rd11 + z11 * f.td11 + z12 * f.td21;
    b = f.rd12 + z11 * f.td12 + z12 * f.td22;
    c = f.rd12 + z21 * f.td11 + z22 * f.td21;
    d = f.rd22 + z21 * f.td12 + z22 * f.td22;
  }
  const T e0 = phase(0, false);
  const T y = e0 * e0 * a;
  return fs ? y * recip(1.0 + y) : y;
}

}  // namespace

extern "C" void emu_reflectivity_reference_form(const double* tab, int L, const double* p,
                                                int n_p, const double* w, int nw, int fs,
                                                int extended, double* out) {
  for (int j = 0; j < n_p; ++j)
    for (int k = 0; k < nw; ++k) {
      double x, y;
      if (extended) {
        const C<long double> r = reflect<long double>(tab, L, p[j], w[2 * k], w[2 * k + 1], fs);
        x = (double)r.x;
        y = (double)r.y;
      } else {
        const C<double> r = reflect<double>(tab, L, p[j], w[2 * k], w[2 * k + 1], fs);
        x = r.x;
        y = r.y;
      }
      out[2 * ((size_t)j * nw + k)] = x;
      out[2 * ((size_t)j * nw + k) + 1] = y;
    }
}
