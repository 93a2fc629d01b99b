// Translation formulas shared by the expansion, M2L and periodic kernels:
// one output coefficient (j,k) of M2M, L2L or M2L from a staged input
// expansion and staged offset harmonics (3d/kernel.h:204-291).  All three are
// linear in the harmonics, so a sum of harmonics over several offsets gives
// the sum of the translations.
#pragma once
#include "harmonics.cuh"

namespace fmm {

// Y(deg, o) for any sign of o from the m>=0 table.
__device__ __forceinline__ double2 ylook(const double2 *Y, int n, int o) {
  return o >= 0 ? Y[tri(n) + o] : cconj(Y[tri(n) - o]);
}

__device__ __forceinline__ int sgn(int n) { return (n & 1) ? -1 : 1; }

__device__ __forceinline__ int octant_of(const double4 &child, const double4 &parent) {
  return (child.x > parent.x) | ((child.y > parent.y) << 1) | ((child.z > parent.z) << 2);
}

__device__ __forceinline__ int order_of(int ci) {
  int n = 0;
  while (tri(n + 1) <= ci) n++;
  return n;
}

__host__ __device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ int sgn_hd(int n) { return (n & 1) ? -1 : 1; }

// The terms of one M2M output (j,k), in the reference's order: each is
// emit(ia, conjugate input?, n, o, sign) for  sign * A[ia]' * Y(n, o), with
// A the child's multipole and Y(n, o) the offset harmonic (ylook).
template <class E>
__host__ __device__ inline void m2m_terms(int j, int k, E emit) {
  for (int n = 0; n <= j; n++) {
    const int lo = imax(-n, -j + k + n), hi = imin(k - 1, n);
    for (int m = lo; m <= hi; m++) emit(tri(j - n) + k - m, false, n, -m, (m >= 0 ? 1 : sgn_hd(m)) * sgn_hd(n));
    const int hi2 = imin(n, j + k - n);
    for (int m = k; m <= hi2; m++) emit(tri(j - n) - k + m, true, n, -m, sgn_hd(k + n + m));
  }
}

// The terms of one L2L output (j,k): A = the parent's local expansion.
template <class E>
__host__ __device__ inline void l2l_terms(int j, int k, int P, E emit) {
  for (int n = j; n < P; n++) {
    for (int m = j + k - n; m < 0; m++) emit(tri(n) - m, true, n - j, m - k, sgn_hd(k));
    for (int m = 0; m <= n; m++)
      if (n - j >= (m - k < 0 ? k - m : m - k)) emit(tri(n) + m, false, n - j, m - k, sgn_hd((m - k) * (m < k)));
  }
}

// M2M output (j,k) from one child's multipole Mc and the offset harmonics Y
// (offset parent - child).
__device__ inline double2 m2m_coeff(int j, int k, const double2 *Mc, const double2 *Y) {
  double2 s = make_double2(0, 0);
  m2m_terms(j, k, [&](int ia, bool ca, int n, int o, int f) {
    const double2 a = cmul(ca ? cconj(Mc[ia]) : Mc[ia], ylook(Y, n, o));
    s.x += a.x * (double)f;
    s.y += a.y * (double)f;
  });
  return s;
}

// L2L output (j,k) from the parent's local Lp and the offset harmonics Y
// (offset child - parent).
__device__ inline double2 l2l_coeff(int j, int k, int P, const double2 *Lp, const double2 *Y) {
  double2 s = make_double2(0, 0);
  l2l_terms(j, k, P, [&](int ia, bool ca, int n, int o, int f) {
    const double2 a = cmul(ca ? cconj(Lp[ia]) : Lp[ia], ylook(Y, n, o));
    s.x += a.x * (double)f;
    s.y += a.y * (double)f;
  });
  return s;
}

// Packed term of a translation table: input index (10 bits), conjugate
// input, harmonic index tri(n) + |o| (10 bits), conjugate harmonic (o < 0),
// negative sign.
__host__ __device__ __forceinline__ unsigned pack_term(int ia, bool ca, int n, int o, int f) {
  const int iy = tri(n) + (o < 0 ? -o : o);
  return (unsigned)ia | ((unsigned)ca << 10) | ((unsigned)iy << 11) | ((unsigned)(o < 0) << 21) |
         ((unsigned)(f < 0) << 22);
}

// One output from a packed term list: the same products in the same order as
// the formulas above.
__device__ __forceinline__ double2 apply_terms(const unsigned *t, int nterms, const double2 *A, const double2 *Y) {
  double2 s = make_double2(0, 0);
  for (int q = 0; q < nterms; q++) {
    const unsigned e = t[q];
    double2 a = A[e & 1023u], y = Y[(e >> 11) & 1023u];
    if (e & (1u << 10)) a.y = -a.y;
    if (e & (1u << 21)) y.y = -y.y;
    const double2 p = cmul(a, y);
    const double f = (e & (1u << 22)) ? -1.0 : 1.0;
    s.x += p.x * f;
    s.y += p.y * f;
  }
  return s;
}

// M2L output (j,k) (3d/kernel.h:233-260) from the source multipole A and the
// irregular harmonics Z of the offset target - source; only degrees j+n < P
// contribute, as in the reference (its harmonics table is zero beyond).
__device__ inline double2 m2l_coeff(int j, int k, int P, const double2 *A, const double2 *Z) {
  double sx = 0, sy = 0;
  for (int n = 0; n <= P - 1 - j; n++) {
    const int d = j + n;
    for (int m = -n; m <= n; m++) {
      const double2 a = m >= 0 ? A[tri(n) + m] : cconj(A[tri(n) - m]);
      const int om = m - k;
      const double2 z = om >= 0 ? Z[tri(d) + om] : cconj(Z[tri(d) - om]);
      const int e2 = m < 0 ? 0 : (m <= k ? m : k);
      const double f = ((j + e2) & 1) ? -1.0 : 1.0;
      sx += f * (a.x * z.x - a.y * z.y);
      sy += f * (a.x * z.y + a.y * z.x);
    }
  }
  return make_double2(sx, sy);
}

}  // namespace fmm
