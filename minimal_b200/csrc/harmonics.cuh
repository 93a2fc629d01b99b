// Device helpers for the complex spherical-harmonic expansions of the 3D
// Laplace kernel, in the reference's normalisation (3d/kernel.h:43-116):
//   regular   Y_n^m  = (-1)^n rho^n     P_n^m(cos a) e^{i m b} / (n+m)!
//   irregular Z_n^m  = (-1)^n (n-m)!    P_n^m(cos a) e^{i m b} / rho^(n+1)
// with P_n^m carrying the Condon-Shortley phase and Y_n^{-m} = conj(Y_n^m).
// Coefficients are stored for m >= 0 at index n(n+1)/2 + m (NTERM = P(P+1)/2).
//
// Work is split by order m: one lane builds the column n = m..P-1 of its m
// with the associated-Legendre recurrences (the same recurrences as
// evalMultipole/evalLocal), so a warp forms all P columns in parallel.
// Angles are never formed: cos a, sin a and e^{ib} come straight from the
// Cartesian offset (the reference's acos/atan2 followed by cos/sin give the
// same values up to rounding).
#pragma once
#include <cuda_runtime.h>

namespace fmm {

struct Sph {
  double r, c, s, inv_s;  // radius, cos(alpha), sin(alpha), 1/sin (0 if sin==0)
  double2 e;              // e^{i beta}
};

__device__ __forceinline__ Sph sph_of(double dx, double dy, double dz) {
  Sph o;
  const double rxy2 = dx * dx + dy * dy;
  o.r = sqrt(rxy2 + dz * dz);
  const double rxy = sqrt(rxy2);
  if (o.r == 0) {
    o.c = 1; o.s = 0;
  } else {
    o.c = dz / o.r; o.s = rxy / o.r;
  }
  o.inv_s = o.s == 0 ? 0 : 1 / o.s;
  if (rxy == 0) o.e = make_double2(1, 0);
  else o.e = make_double2(dx / rxy, dy / rxy);
  return o;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// e^{i m b} by binary powering of e^{ib}.
__device__ __forceinline__ double2 cpow_int(double2 e, int m) {
  double2 r = make_double2(1, 0), b = e;
  while (m) {
    if (m & 1) r = cmul(r, b);
    m >>= 1;
    if (m) b = cmul(b, b);
  }
  return r;
}

// P_m^m(c) = (-1)^m (2m-1)!! s^m
__device__ __forceinline__ double legendre_mm(int m, double s) {
  double p = 1, odd = 1;
  for (int k = 0; k < m; k++) { p = -p * odd * s; odd += 2; }
  return p;
}

// Regular column m (n = m..P-1): calls f(n, Y_nm, dY_nm) with dY the alpha
// derivative (3d/kernel.h:60,72).  Negate beta by passing conj(e).
template <class F>
__device__ __forceinline__ void regular_column(int m, int P, double rho, const Sph &g, double2 e, F f) {
  const double2 em = cpow_int(e, m);
  double c = 1;  // (-1)^m rho^m / (2m)! -> updated to (-1)^n rho^n/(n+m)!
  for (int k = 0; k < m; k++) c *= rho / (double)(-(2 * k + 2) * (2 * k + 1));
  double p = legendre_mm(m, g.s), p1 = 0;
  for (int n = m; n < P; n++) {
    double pn1;  // P_{n+1}^m
    if (n == m) pn1 = g.c * (2 * m + 1) * p;
    else pn1 = (g.c * (2 * n + 1) * p - (n + m) * p1) / (n - m + 1);
    const double2 Y = cscale(em, c * p);
    const double2 dY = cscale(em, c * ((n - m + 1) * pn1 - (n + 1) * g.c * p) * g.inv_s);
    f(n, Y, dY);
    p1 = p;
    p = pn1;
    c *= rho / (double)(-(n + 1 + m));
  }
}

// Irregular column m (n = m..P-1): calls f(n, Z_nm) (3d/kernel.h:83-116).
template <class F>
__device__ __forceinline__ void irregular_column(int m, int P, double rho, const Sph &g, F f) {
  const double2 em = cpow_int(g.e, m);
  const double inv = -1.0 / rho;
  double c = 1.0 / rho;  // (1/rho)(-1/rho)^m (n-m)! (-1)^? -> see below
  for (int k = 0; k < m; k++) c *= inv;
  double p = legendre_mm(m, g.s), p1 = 0;
  for (int n = m; n < P; n++) {
    f(n, cscale(em, c * p));
    double pn1;
    if (n == m) pn1 = g.c * (2 * m + 1) * p;
    else pn1 = (g.c * (2 * n + 1) * p - (n + m) * p1) / (n - m + 1);
    p1 = p;
    p = pn1;
    c *= inv * (double)(n - m + 1);
  }
}

__host__ __device__ __forceinline__ int tri(int n) { return n * (n + 1) / 2; }

}  // namespace fmm
