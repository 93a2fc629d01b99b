// Group key of an M2L entry: the translation operator of a same-image pair
// depends only on the level difference and on the centre offset in units of
// the smaller cell radius (an integer vector), so entries with equal keys
// share one operator.  Key layout: (dl + KEY_DL) << 18 | (vx + KEY_V) << 12 |
// (vy + KEY_V) << 6 | (vz + KEY_V); entries outside that range have no key
// (-1) and go to the direct-form kernel.  Periodic image entries take the
// image keys below.
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

// Periodic image entries (3dp): the offset in units of the finer radius r
// is n0 - iX * C with n0 = (X_t - X_s) / r an integer vector and
// C = cycle / r = cycle * 2^lf / R0 (lf the finer cell's level, R0 the root
// radius) the same for every entry of one (image, lf).  The key keeps the
// integer part v = n0 - rint(iX * C) and the slot (image, lf); the operator
// adds back rint(iX * C) - iX * C, computed the same way (image_shift_units),
// so every entry of a key has exactly the key's offset.  Key layout: above
// KEY_SPACE, slot * IKEY_SPACE + ((dl + 2) << 15 | (vx + 16) << 10 |
// (vy + 16) << 5 | (vz + 16)) with slot = image' * nlev + (lf - 1), image' the
// image index 0..26 without the unshifted 13, lf in [1, nlev].
constexpr int IKEY_DL = 2;   // level difference in [-2, 1]
constexpr int IKEY_V = 16;   // offset components in [-16, 15]
constexpr int IKEY_SPACE = 1 << 17;

// Key space of a tree: the free-space keys, and for a periodic system the
// image slots of its levels 1..depth.
__host__ __device__ __forceinline__ long key_space(int images, int depth) {
  return images > 0 ? (long)KEY_SPACE + 26L * (depth > 0 ? depth : 1) * IKEY_SPACE : (long)KEY_SPACE;
}

// The image shift of image index img (x + 1) + 3 (y + 1) + 9 (z + 1) in units
// of a level-lf radius: C = cycle * 2^lf / R0 per unit shift.
__device__ __forceinline__ double image_shift_units(int i, int lf, double R0, double cycle) {
  return (double)i * scalbn(cycle / R0, lf);
}

__device__ __forceinline__ int m2l_image_key(const double4 &X, const double4 &Y, int dl, int img, double R0,
                                             double cycle, int depth) {
  if (dl < -IKEY_DL || dl >= IKEY_DL) return -1;
  const double m = fmin(X.w, Y.w);
  const int lf = ilogb(R0) - ilogb(m);
  if (lf < 1 || lf > depth) return -1;
  const int ix = img % 3 - 1, iy = (img / 3) % 3 - 1, iz = img / 9 - 1;
  const double inv = 1.0 / m;
  const double sx = image_shift_units(ix, lf, R0, cycle), sy = image_shift_units(iy, lf, R0, cycle),
               sz = image_shift_units(iz, lf, R0, cycle);
  const double vx = rint((X.x - Y.x) * inv) - rint(sx), vy = rint((X.y - Y.y) * inv) - rint(sy),
               vz = rint((X.z - Y.z) * inv) - rint(sz);
  if (vx < -IKEY_V || vx >= IKEY_V || vy < -IKEY_V || vy >= IKEY_V || vz < -IKEY_V || vz >= IKEY_V) return -1;
  const int slot = (img < 13 ? img : img - 1) * depth + (lf - 1);
  const long key = (long)KEY_SPACE + (long)slot * IKEY_SPACE +
                   (((dl + IKEY_DL) << 15) | (((int)vx + IKEY_V) << 10) | (((int)vy + IKEY_V) << 5) | ((int)vz + IKEY_V));
  return (int)key;
}

// Decodes a key into the level difference and the (possibly fractional)
// offset in units of the finer radius.
__device__ __forceinline__ int m2l_key_offset(int key, double R0, double cycle, int depth, double &vx, double &vy,
                                              double &vz) {
  if (key < KEY_SPACE) {
    vx = ((key >> 12) & 63) - KEY_V;
    vy = ((key >> 6) & 63) - KEY_V;
    vz = (key & 63) - KEY_V;
    return (key >> 18) - KEY_DL;
  }
  const int k = key - KEY_SPACE, slot = k / IKEY_SPACE, loc = k % IKEY_SPACE;
  const int ic = slot / depth, lf = slot % depth + 1, img = ic < 13 ? ic : ic + 1;
  const int ix = img % 3 - 1, iy = (img / 3) % 3 - 1, iz = img / 9 - 1;
  const double sx = image_shift_units(ix, lf, R0, cycle), sy = image_shift_units(iy, lf, R0, cycle),
               sz = image_shift_units(iz, lf, R0, cycle);
  vx = ((loc >> 10) & 31) - IKEY_V + (rint(sx) - sx);
  vy = ((loc >> 5) & 31) - IKEY_V + (rint(sy) - sy);
  vz = (loc & 31) - IKEY_V + (rint(sz) - sz);
  return (loc >> 15) - IKEY_DL;
}

// Ghost sources (mixed form).  An image entry whose fractional offset f (the
// offset's distance from the integer vector v) is tiny can use the
// free-space operator of (dl, v) instead of an image key of its own: its
// source multipole is moved by the exact M2M shift f * r onto a "ghost"
// centre at the integer offset, X_t - v r.  M2M keeps every retained order
// exact, and with |f| <= GHOST_MAX_FRAC the shifted multipole's extent grows
// by less than one percent of the cell radius, so the M2L's truncation error
// barely changes.  Bodies that fill a periodic box give |f| ~ 1e-3 or less
// (the root radius is the bounds' half-extent times 1.00001); other entries
// keep their image keys.  A ghost is one (source cell, image, finer level)
// triple: gslot = (s * 26 + image') * 4 + (lf - ls).
constexpr double GHOST_MAX_FRAC = 0.005;
constexpr int GHOST_SLOTS = 26 * 4;  // ghost slots per source cell

// Returns the free-space key of the entry's ghost (or -1: no ghost), its
// slot, and the shift f r from the image source's centre to the ghost's.
__device__ __forceinline__ int m2l_ghost_key(const double4 &X, const double4 &Y, int dl, int img, int s, double R0,
                                             double cycle, int depth, long *gslot, double3 *shift) {
  if (img == 13 || dl < -KEY_DL || dl >= KEY_DL) return -1;
  const double m = fmin(X.w, Y.w);
  const int lf = ilogb(R0) - ilogb(m), dlf = ilogb(Y.w) - ilogb(m);
  if (lf < 1 || lf > depth || dlf < 0 || dlf > 3) return -1;
  const int ix = img % 3 - 1, iy = (img / 3) % 3 - 1, iz = img / 9 - 1;
  const double sx = image_shift_units(ix, lf, R0, cycle), sy = image_shift_units(iy, lf, R0, cycle),
               sz = image_shift_units(iz, lf, R0, cycle);
  const double fx = rint(sx) - sx, fy = rint(sy) - sy, fz = rint(sz) - sz;
  if (fabs(fx) > GHOST_MAX_FRAC || fabs(fy) > GHOST_MAX_FRAC || fabs(fz) > GHOST_MAX_FRAC) return -1;
  const double inv = 1.0 / m;
  const double vx = rint((X.x - Y.x) * inv) - rint(sx), vy = rint((X.y - Y.y) * inv) - rint(sy),
               vz = rint((X.z - Y.z) * inv) - rint(sz);
  if (vx < -KEY_V || vx >= KEY_V || vy < -KEY_V || vy >= KEY_V || vz < -KEY_V || vz >= KEY_V) return -1;
  *gslot = ((long)s * 26 + (img < 13 ? img : img - 1)) * 4 + dlf;
  *shift = make_double3(fx * m, fy * m, fz * m);
  return ((dl + KEY_DL) << 18) | (((int)vx + KEY_V) << 12) | (((int)vy + KEY_V) << 6) | ((int)vz + KEY_V);
}

// Marks a key and a target as present.  A few hundred keys (and every
// target) take millions of entries: store only what this SM has not seen
// set, so the L1-cached reads keep the stores off a few hot L2 lines.
__device__ __forceinline__ void m2l_mark_key(int key, int t, int *occ, int *gflag) {
  if (occ[key] == 0) occ[key] = 1;
  if (gflag[t] == 0) gflag[t] = 1;
}

}  // namespace fmm
