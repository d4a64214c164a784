// Forward-mode dual numbers over complex doubles with N tangent directions, used to
// differentiate the interface coefficients (functions of the two adjacent layers' alpha,
// beta, rho) once per (slowness, interface).  The coefficient code in kr_math.cuh is
// templated on its scalar type, so the same source yields values and tangents.
#pragma once

#include "kr_math.cuh"

namespace kr {

template <int N>
struct Dual {
  cd v;
  cd d[N];
};

template <int N>
KR_HD Dual<N> dconst(cd v) {
  Dual<N> r;
  r.v = v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = mk(0.0, 0.0);
  return r;
}

template <int N>
KR_HD Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int N>
KR_HD Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int N>
KR_HD Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int N>
KR_HD Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int N>
KR_HD Dual<N> operator*(cd s, const Dual<N>& a) {
  Dual<N> r;
  r.v = s * a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = s * a.d[k];
  return r;
}
template <int N>
KR_HD Dual<N> operator*(double s, const Dual<N>& a) {
  Dual<N> r;
  r.v = s * a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = s * a.d[k];
  return r;
}
template <int N>
KR_HD Dual<N> operator*(const Dual<N>& a, double s) { return s * a; }
template <int N>
KR_HD Dual<N> operator+(const Dual<N>& a, double s) {
  Dual<N> r = a;
  r.v = a.v + s;
  return r;
}
template <int N>
KR_HD Dual<N> operator-(double s, const Dual<N>& a) { return -a + s; }
template <int N>
KR_HD Dual<N> recip(const Dual<N>& a) {
  Dual<N> r;
  r.v = recip(a.v);
  cd m = -(r.v * r.v);
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = m * a.d[k];
  return r;
}
template <int N>
KR_HD Dual<N> csqrt(const Dual<N>& a) {
  Dual<N> r;
  r.v = csqrt(a.v);
  cd h = recip(2.0 * r.v);
  // A zero tangent stays zero even where sqrt has an infinite derivative (sqrt(0)).
#pragma unroll
  for (int k = 0; k < N; ++k)
    r.d[k] = (a.d[k].x == 0.0 && a.d[k].y == 0.0) ? mk(0.0, 0.0) : h * a.d[k];
  return r;
}

}  // namespace kr
