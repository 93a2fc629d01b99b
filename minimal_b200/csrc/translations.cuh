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

// M2M output (j,k) from one child's multipole Mc and the offset harmonics Y
// (offset parent - child).
__device__ inline double2 m2m_coeff(int j, int k, const double2 *Mc, const double2 *Y) {
  double2 s = make_double2(0, 0);
  for (int n = 0; n <= j; n++) {
    const int lo = max(-n, -j + k + n), hi = min(k - 1, n);
    for (int m = lo; m <= hi; m++) {
      const double2 a = cmul(Mc[tri(j - n) + k - m], ylook(Y, n, -m));
      const double f = (double)((m >= 0 ? 1 : sgn(m)) * sgn(n));
      s.x += a.x * f;
      s.y += a.y * f;
    }
    const int hi2 = min(n, j + k - n);
    for (int m = k; m <= hi2; m++) {
      const double2 a = cmul(cconj(Mc[tri(j - n) - k + m]), ylook(Y, n, -m));
      const double f = (double)sgn(k + n + m);
      s.x += a.x * f;
      s.y += a.y * f;
    }
  }
  return s;
}

// L2L output (j,k) from the parent's local Lp and the offset harmonics Y
// (offset child - parent).
__device__ inline double2 l2l_coeff(int j, int k, int P, const double2 *Lp, const double2 *Y) {
  double2 s = make_double2(0, 0);
  for (int n = j; n < P; n++) {
    for (int m = j + k - n; m < 0; m++) {
      const double2 a = cmul(cconj(Lp[tri(n) - m]), ylook(Y, n - j, m - k));
      const double f = (double)sgn(k);
      s.x += a.x * f;
      s.y += a.y * f;
    }
    for (int m = 0; m <= n; m++) {
      if (n - j >= abs(m - k)) {
        const double2 a = cmul(Lp[tri(n) + m], ylook(Y, n - j, m - k));
        const double f = (double)sgn((m - k) * (m < k));
        s.x += a.x * f;
        s.y += a.y * f;
      }
    }
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
