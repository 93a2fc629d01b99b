// Group key of an M2L entry: the translation operator of a same-image pair
// depends only on the level difference and on the centre offset in units of
// the smaller cell radius (an integer vector), so entries with equal keys
// share one operator.  Key layout: (dl + KEY_DL) << 18 | (vx + KEY_V) << 12 |
// (vy + KEY_V) << 6 | (vz + KEY_V); entries outside that range (and periodic
// images) have no key (-1) and go to the direct-form kernel.
#pragma once
#include "fmm.cuh"

namespace fmm {

constexpr int KEY_DL = 4;   // level difference lt - ls in [-4, 3]
constexpr int KEY_V = 32;   // offset components in [-32, 31]
constexpr int KEY_SPACE = 8 << 18;

// X target, Y source (centre, radius); dl = level(target) - level(source).
__device__ __forceinline__ int m2l_group_key(const double4 &X, const double4 &Y, int dl) {
  // the quotients are integers up to rounding: an FP32 reciprocal (relative
  // error < 2^-22) leaves them within 1e-5 of the integer for |v| <= 32
  // (radii far outside the normal FP32 range take the FP64 division)
  const double m = fmin(X.w, Y.w);
  const double inv = m > 1e-30 && m < 1e30 ? (double)__frcp_rn((float)m) : 1.0 / m;
  const double vx = rint((X.x - Y.x) * inv), vy = rint((X.y - Y.y) * inv), vz = rint((X.z - Y.z) * inv);
  if (dl >= -KEY_DL && dl < KEY_DL && vx >= -KEY_V && vx < KEY_V && vy >= -KEY_V && vy < KEY_V && vz >= -KEY_V &&
      vz < KEY_V)
    return ((dl + KEY_DL) << 18) | (((int)vx + KEY_V) << 12) | (((int)vy + KEY_V) << 6) | ((int)vz + KEY_V);
  return -1;
}

// Marks a key and a target as present.  A few hundred keys (and every
// target) take millions of entries: store only what this SM has not seen
// set, so the L1-cached reads keep the stores off a few hot L2 lines.
__device__ __forceinline__ void m2l_mark_key(int key, int t, int *occ, int *gflag) {
  if (occ[key] == 0) occ[key] = 1;
  if (gflag[t] == 0) gflag[t] = 1;
}

}  // namespace fmm
