// The 2D variants (2d/, 2dp/): Laplace FMM in the plane with the log kernel
// and complex power-series expansions of P terms (2d/kernel.h:12-126), FP64.
//
// Bodies sit at z = 0 in the handle's double4 arrays (x, y, 0, q) and the
// tree and the interaction lists come from the 3D machinery: on bodies in one
// plane the octree's z digit is the same for every body of a level, so the
// octree is the reference's quadtree cell for cell (2d/build_tree.h: quadrant
// (x > X) + ((y > Y) << 1), the same centre recurrence and leaf rule); with
// the cells' z centres set to zero the dual walk's distance test and branch
// rules are the 2D ones (2d/traverse_lazy.h:27-44), and a 2dp system seeds
// the nine in-plane images (2dp/traverse_lazy.h:124-141).  What is new here
// is the arithmetic:
//   P2M, L2P   warp per leaf, lane per body, z^n/n! generated as in the
//              reference (powZ *= Z / n);
//   M2M, L2L   per level, thread per (cell, coefficient);
//   M2L        warp per target cell over its ordered M2L list, lane n owns
//              L[n]: lane 0 the log term and 1/z^k series, lane 1 the 1/z^(k+1)
//              series, lane n >= 2 the (n+k-1)!/z^(n+k) series
//              (2d/kernel.h:61-90; the 2dp image shift :63);
//   P2P        warp per target leaf over its ordered P2P list, lane per
//              target body, q log(1/R) and q dX / R^2 (2d/kernel.h:12-31);
//   periodic   one warp: the 72 root M2Ls and the 8-copy M2M per image level
//              (2dp/traverse_eager.h:46-93).
#include <type_traits>

#include "fmm.cuh"
#include "harmonics.cuh"

namespace fmm {

namespace {

constexpr int W2 = 4;  // warps per block
constexpr int IMG_SHIFT = 26;
constexpr u32 IDX_MASK = (1u << IMG_SHIFT) - 1;

__device__ __forceinline__ double2 cdivr(double2 a, double r) { return make_double2(a.x / r, a.y / r); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmulr(double2 a, double r) { return make_double2(a.x * r, a.y * r); }

// 1/z with Smith's scaling (no overflow for large or small |z|).
__device__ __forceinline__ double2 crecip(double2 z) {
  if (fabs(z.x) >= fabs(z.y)) {
    const double r = z.y / z.x, d = z.x + z.y * r;
    return make_double2(1.0 / d, -r / d);
  }
  const double r = z.x / z.y, d = z.x * r + z.y;
  return make_double2(r / d, -1.0 / d);
}

__device__ __forceinline__ double2 clog2(double2 z) { return make_double2(log(hypot(z.x, z.y)), atan2(z.y, z.x)); }

// Image shift of a list entry: periodic1D of the 3D walk with z = 0.
__device__ __forceinline__ void img_shift(u32 img, double cycle, double &sx, double &sy) {
  const int ix = (int)(img % 3) - 1, iy = (int)((img / 3) % 3) - 1;
  sx = ix * cycle;
  sy = iy * cycle;
}

// P2M (2d/kernel.h:34-45): M[n] += q z^n / n!, z = X_body - X_cell.
__global__ void __launch_bounds__(W2 * 32) k2_p2m(const int *leaves, int nleaves, const int *begin, const int *count,
                                                  const double4 *xr, const double4 *src, double2 *M, int P) {
  extern __shared__ double2 sh[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * W2 + wid;
  if (w >= nleaves) return;
  double2 *acc = sh + wid * P;
  for (int k = lane; k < P; k += 32) acc[k] = make_double2(0, 0);
  __syncwarp();
  const int c = leaves[w];
  const double4 C = xr[c];
  const int b0 = begin[c], nb = count[c];
  for (int t = 0; t < nb; t += 32) {
    const bool ok = t + lane < nb;
    const double4 B = ok ? src[b0 + t + lane] : make_double4(C.x, C.y, 0, 0.0);
    const double2 Z = make_double2(B.x - C.x, B.y - C.y);
    double2 pz = make_double2(1, 0);
    for (int n = 0; n < P; n++) {
      if (n > 0) pz = cmul(pz, cdivr(Z, (double)n));
      double x = n == 0 ? B.w : pz.x * B.w, y = n == 0 ? 0.0 : pz.y * B.w;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
      }
      if (lane == 0) {
        acc[n].x += x;
        acc[n].y += y;
      }
    }
  }
  __syncwarp();
  for (int k = lane; k < P; k += 32) M[(long)c * P + k] = acc[k];
}

// M2M (2d/kernel.h:48-59) for the parents of one level: thread per
// (parent, k); M[k] = sum over children of M_c[k] + sum_n M_c[k-n] z^n/n!,
// z = X_child - X_parent.  Leaves keep their P2M.
__global__ void k2_m2m(int c0, int ncell, const int *child, const int *nchild, const double4 *xr, double2 *M, int P) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)ncell * P) return;
  const int c = c0 + (int)(i / P), k = (int)(i % P);
  const int nc = nchild[c];
  if (nc == 0) return;
  const double4 X = xr[c];
  double2 s = make_double2(0, 0);
  for (int j = child[c]; j < child[c] + nc; j++) {
    const double4 Y = xr[j];
    const double2 Z = make_double2(Y.x - X.x, Y.y - X.y);
    const double2 *Mc = M + (long)j * P;
    double2 pz = make_double2(1, 0);
    s = cadd(s, Mc[k]);
    for (int n = 1; n <= k; n++) {
      pz = cmul(pz, cdivr(Z, (double)n));
      s = cadd(s, cmul(Mc[k - n], pz));
    }
  }
  M[(long)c * P + k] = s;
}

// One M2L (2d/kernel.h:61-90) of source multipole M (lane k holds M[k]) into
// lane n's coefficient L[n], offset Z = X_target - X_source - shift.
__device__ __forceinline__ double2 m2l_term(double2 Z, double2 Mk, int lane, int P) {
  const double2 invZ = crecip(Z);
  const double2 M0 = make_double2(__shfl_sync(0xffffffffu, Mk.x, 0), __shfl_sync(0xffffffffu, Mk.y, 0));
  double2 acc = make_double2(0, 0);
  if (lane == 0) {
    acc = csub(acc, cmul(M0, clog2(Z)));
  } else if (lane == 1) {
    acc = csub(acc, cmul(M0, invZ));
  }
  // lane 0: + M1/z + sum_{k>=2} M_k (k-1)!/z^k; lane 1: - sum_{k>=1} M_k k!/z^(k+1);
  // lane n >= 2: sum_{k>=0} M_k (-1)^n (n+k-1)!/z^(n+k)
  double2 pw;
  if (lane == 0 || lane == 1) {
    pw = invZ;
  } else {
    double2 pnk = make_double2(1, 0);  // (n-2)!/z^(n-1), as the reference builds it over n
    for (int m = 2; m <= lane; m++) {
      pnk = cmul(pnk, invZ);
      if (m < lane) pnk = cmulr(pnk, (double)(m - 1));
    }
    pw = cmulr(pnk, (lane & 1) ? -1.0 : 1.0);
  }
  for (int k = 0; k < P; k++) {
    const double2 m = make_double2(__shfl_sync(0xffffffffu, Mk.x, k), __shfl_sync(0xffffffffu, Mk.y, k));
    if (lane == 0) {
      if (k == 1) acc = cadd(acc, cmul(m, invZ));
      if (k >= 2) {
        pw = cmul(cmulr(invZ, (double)(k - 1)), pw);
        acc = cadd(acc, cmul(m, pw));
      }
    } else if (lane == 1) {
      if (k >= 1) {
        pw = cmul(cmulr(invZ, (double)k), pw);
        acc = csub(acc, cmul(m, pw));
      }
    } else if (lane < P) {
      pw = cmul(cmulr(invZ, (double)(lane + k - 1)), pw);
      acc = cadd(acc, cmul(m, pw));
    }
  }
  return acc;
}

// M2L over the ordered lists: warp per target cell; L[t] = the sum of its
// entries (the first writer of L).
__global__ void __launch_bounds__(W2 * 32) k2_m2l(int ncells, const int *off, const u32 *ent, const double4 *xr,
                                                  const double2 *M, double2 *L, int P, double cycle) {
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * W2 + wid;
  if (t >= ncells) return;
  const double4 X = xr[t];
  double2 acc = make_double2(0, 0);
  for (int e = off[t]; e < off[t + 1]; e++) {
    const u32 en = ent[e];
    const int s = (int)(en & IDX_MASK);
    double sx, sy;
    img_shift(en >> IMG_SHIFT, cycle, sx, sy);
    const double4 Y = xr[s];
    const double2 Z = make_double2(X.x - Y.x - sx, X.y - Y.y - sy);
    const double2 Mk = lane < P ? M[(long)s * P + lane] : make_double2(0, 0);
    acc = cadd(acc, m2l_term(Z, Mk, lane, P));
  }
  if (lane < P) L[(long)t * P + lane] = acc;
}

// The same M2L with a lane per list entry (orders P <= 16): with
// q_m = (m-1)!/z^m, the terms of m2l_term are L[n] += (-1)^n M_k q_(n+k) for
// n + k >= 1 and L[0] -= M_0 log z, so one lane evaluates a whole entry --
// one reciprocal, one logarithm, the q_m by the recurrence
// q_(m+1) = q_m m / z and P^2 complex products, summed along n + k = m --
// with every coefficient in registers (P is a compile-time constant), while
// the warp's lanes take the target's entries 32 at a time.  The lanes' sums
// are then added in a fixed butterfly order (deterministic).  The operations
// are those of m2l_term in another order: the expansions agree with it, and
// with the reference, to rounding.
template <int P>
__global__ void __launch_bounds__(W2 * 32) k2_m2l_lane(int ncells, const int *off, const u32 *ent, const double4 *xr,
                                                       const double2 *M, double2 *L, double cycle) {
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * W2 + wid;
  if (t >= ncells) return;  // warp-uniform
  const double4 X = xr[t];
  double2 acc[P];
#pragma unroll
  for (int n = 0; n < P; n++) acc[n] = make_double2(0, 0);
  for (int e = off[t] + lane; e < off[t + 1]; e += 32) {
    const u32 en = ent[e];
    const int s = (int)(en & IDX_MASK);
    double sx, sy;
    img_shift(en >> IMG_SHIFT, cycle, sx, sy);
    const double4 Y = xr[s];
    const double2 Z = make_double2(X.x - Y.x - sx, X.y - Y.y - sy);
    double2 Mk[P];
#pragma unroll
    for (int k = 0; k < P; k++) Mk[k] = M[(long)s * P + k];
    const double2 iz = crecip(Z);
    acc[0] = csub(acc[0], cmul(Mk[0], clog2(Z)));
    double2 q = iz;  // q_1
#pragma unroll
    for (int m = 1; m <= 2 * P - 2; m++) {
#pragma unroll
      for (int n = 0; n < P; n++) {
        const int k = m - n;
        if (k < 0 || k >= P) continue;
        const double2 term = cmul(Mk[k], q);
        acc[n] = (n & 1) ? csub(acc[n], term) : cadd(acc[n], term);
      }
      if (m < 2 * P - 2) q = cmulr(cmul(q, iz), (double)m);
    }
  }
#pragma unroll
  for (int n = 0; n < P; n++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      acc[n].x += __shfl_xor_sync(0xffffffffu, acc[n].x, o);
      acc[n].y += __shfl_xor_sync(0xffffffffu, acc[n].y, o);
    }
    if (lane == (n & 31)) L[(long)t * P + n] = acc[n];
  }
}

// Far periodic images of a 2dp system (2dp/traverse_eager.h:46-93): per
// image level, the 72 M2Ls from the super-cell (the root's multipole, at the
// root's centre) shifted by (3 ix + cx, 3 iy + cy) cycles into the root's L,
// then the super-cell's multipole gathers its 8 copies (M2M), and the cycle
// triples.  One warp.
__global__ void k2_periodic(const double4 *xr, const double2 *M, double2 *L, int P, int images, double cycle) {
  __shared__ double2 Ms[32];
  const int lane = threadIdx.x;
  const double4 X = xr[0];
  if (lane < P) Ms[lane] = M[lane];
  __syncwarp();
  double2 acc = make_double2(0, 0);
  double cyc = cycle;
  for (int level = 0; level < images - 1; level++) {
    const double2 Mk = lane < P ? Ms[lane] : make_double2(0, 0);
    for (int ix = -1; ix <= 1; ix++)
      for (int iy = -1; iy <= 1; iy++) {
        if (ix == 0 && iy == 0) continue;
        for (int cx = -1; cx <= 1; cx++)
          for (int cy = -1; cy <= 1; cy++) {
            const double sx = (3 * ix + cx) * cyc, sy = (3 * iy + cy) * cyc;
            const double2 Z = make_double2(X.x - X.x - sx, X.y - X.y - sy);
            acc = cadd(acc, m2l_term(Z, Mk, lane, P));
          }
      }
    // M2M of the 8 copies at the super-cell's centre +- cycle into Ms
    double2 s = make_double2(0, 0);
    if (lane < P) {
      s = Mk;
      for (int ix = -1; ix <= 1; ix++)
        for (int iy = -1; iy <= 1; iy++) {
          if (ix == 0 && iy == 0) continue;
          const double2 Z = make_double2((X.x + ix * cyc) - X.x, (X.y + iy * cyc) - X.y);
          double2 pz = make_double2(1, 0);
          s = cadd(s, Ms[lane]);
          for (int n = 1; n <= lane; n++) {
            pz = cmul(pz, cdivr(Z, (double)n));
            s = cadd(s, cmul(Ms[lane - n], pz));
          }
        }
    }
    __syncwarp();
    if (lane < P) Ms[lane] = s;
    __syncwarp();
    cyc *= 3;
  }
  if (lane < P) L[lane] = cadd(L[lane], acc);
}

// L2L (2d/kernel.h:93-106) from the parents of one level to their children:
// thread per (child, l); L_c[l] += L_p[l] + sum_k L_p[l+k] z^k/k!,
// z = X_child - X_parent.
__global__ void k2_l2l(int c0, int ncell, const int *child, const int *nchild, const double4 *xr, double2 *L, int P) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)ncell * 8 * P) return;  // up to 4 children (8 octants) per parent
  const int c = c0 + (int)(i / (8 * P)), r = (int)(i % (8 * P)), q = r / P, l = r % P;
  if (q >= nchild[c]) return;
  const int j = child[c] + q;
  const double4 X = xr[c], Y = xr[j];
  const double2 Z = make_double2(Y.x - X.x, Y.y - X.y);
  const double2 *Lp = L + (long)c * P;
  double2 s = cadd(L[(long)j * P + l], Lp[l]), pz = make_double2(1, 0);
  for (int k = 1; k < P - l; k++) {
    pz = cmul(pz, cdivr(Z, (double)k));
    s = cadd(s, cmul(Lp[l + k], pz));
  }
  L[(long)j * P + l] = s;
}

// L2P (2d/kernel.h:109-126): p += Re sum L[n] z^n/n!, F += (Re, -Im) of
// sum L[n+1] z^n/n!.  Adds into the near-field sums.
__global__ void __launch_bounds__(W2 * 32) k2_l2p(const int *leaves, int nleaves, const int *begin, const int *count,
                                                  const double4 *xr, const double4 *src, const double2 *L,
                                                  double4 *out, int P) {
  extern __shared__ double2 sh[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * W2 + wid;
  if (w >= nleaves) return;
  const int c = leaves[w];
  double2 *Lc = sh + wid * P;
  for (int k = lane; k < P; k += 32) Lc[k] = L[(long)c * P + k];
  __syncwarp();
  const double4 C = xr[c];
  const int b0 = begin[c], nb = count[c];
  for (int t = lane; t < nb; t += 32) {
    const double4 B = src[b0 + t];
    const double2 Z = make_double2(B.x - C.x, B.y - C.y);
    double p = Lc[0].x, fx = P > 1 ? Lc[1].x : 0.0, fy = P > 1 ? -Lc[1].y : 0.0;
    double2 pz = make_double2(1, 0);
    for (int n = 1; n < P; n++) {
      pz = cmul(pz, cdivr(Z, (double)n));
      p += cmul(Lc[n], pz).x;
      if (n < P - 1) {
        const double2 f = cmul(Lc[n + 1], pz);
        fx += f.x;
        fy -= f.y;
      }
    }
    double4 &o = out[b0 + t];
    o.x += p;
    o.y += fx;
    o.z += fy;
  }
}

// P2P (2d/kernel.h:12-31; 2dp: the image shift of each list entry):
// p += q log(1/r), F -= q (dx, dy) / r^2 over the target leaf's ordered near
// list, each source leaf's sums added to the body as one term, as the
// reference's per-pair calls do; writes out (the first writer).  A warp per
// target leaf.  For leaves of up to 16
// bodies the lanes are (target i, entry group g), G = floor(32 / nb) groups
// taking the list entries round-robin, and the groups' sums are added in
// group order at the end (deterministic); larger leaves take a lane per
// target.  log(1/r) is formed as -log(r^2) / 2 and the force with one
// reciprocal of r^2 (the reference's quantities, to rounding).
__global__ void __launch_bounds__(W2 * 32) k2_p2p(const int *leaves, int nleaves, const int *begin, const int *count,
                                                  const int *off, const u32 *ent, const double4 *src, double4 *out,
                                                  double cycle) {
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * W2 + wid;
  if (w >= nleaves) return;  // warp-uniform
  const int c = leaves[w], b0 = begin[c], nb = count[c];
  const int e0 = off[c], e1 = off[c + 1];
  const int G = nb <= 16 ? 32 / nb : 1;  // entry groups
  const int span = nb <= 16 ? nb : 32;   // targets per pass
  const int i = lane % span, g = lane / span;
  const bool lane_ok = g < G;
  for (int tb = 0; tb < nb; tb += span) {
    const int t = tb + i;
    const bool ok = lane_ok && t < nb;
    const double4 T = ok ? src[b0 + t] : make_double4(0, 0, 0, 0);
    double p = 0, fx = 0, fy = 0;
    if (lane_ok) {
      for (int e = e0 + g; e < e1; e += G) {
        const u32 en = ent[e];
        const int s = (int)(en & IDX_MASK);
        double sx, sy;
        img_shift(en >> IMG_SHIFT, cycle, sx, sy);
        double pp = 0, px = 0, py = 0;
        for (int j = begin[s]; j < begin[s] + count[s]; j++) {
          const double4 S = src[j];
          const double dx = T.x - S.x - sx, dy = T.y - S.y - sy;
          const double R2 = dx * dx + dy * dy;
          if (R2 != 0) {
            const double invR2 = 1 / R2;
            pp -= 0.5 * S.w * log(R2);
            px += dx * S.w * invR2;
            py += dy * S.w * invR2;
          }
        }
        p += pp;
        fx -= px;
        fy -= py;
      }
    }
    // group 0 adds the other groups' sums in group order
    for (int gg = 1; gg < G; gg++) {
      const int from = (gg * span + i) & 31;
      const double vp = __shfl_sync(0xffffffffu, p, from), vx = __shfl_sync(0xffffffffu, fx, from),
                   vy = __shfl_sync(0xffffffffu, fy, from);
      if (g == 0) {
        p += vp;
        fx += vx;
        fy += vy;
      }
    }
    if (ok && g == 0) out[b0 + t] = make_double4(p, fx, fy, 0.0);
  }
}

// Direct summation (2d/traverse_eager.h:69-80 direct; 2dp with the
// (2 prange + 1)^2 images, 2dp/traverse_eager.h:124-143): one thread per
// target, sources in shared tiles; p, F add into out.
constexpr int DT2 = 256;
__global__ void __launch_bounds__(DT2) k2_direct(const double4 *tgt, long nt, const double4 *src, long ns,
                                                 double4 *out, int prange, double cycle) {
  __shared__ double4 tile[DT2];
  const long i = (long)blockIdx.x * DT2 + threadIdx.x;
  const double4 T = i < nt ? tgt[i] : make_double4(0, 0, 0, 0);
  double p = 0, fx = 0, fy = 0;
  for (long b = 0; b < ns; b += DT2) {
    __syncthreads();
    if (b + threadIdx.x < ns) tile[threadIdx.x] = src[b + threadIdx.x];
    __syncthreads();
    const int m = (int)min((long)DT2, ns - b);
    for (int ix = -prange; ix <= prange; ix++)
      for (int iy = -prange; iy <= prange; iy++) {
        const double sx = ix * cycle, sy = iy * cycle;
        for (int k = 0; k < m; k++) {
          const double4 S = tile[k];
          const double dx = T.x - S.x - sx, dy = T.y - S.y - sy;
          const double R2 = dx * dx + dy * dy;
          if (R2 != 0) {
            const double invR = 1 / sqrt(R2);
            p += S.w * log(invR);
            fx += dx * S.w / R2;
            fy += dy * S.w / R2;
          }
        }
      }
  }
  if (i < nt) {
    out[i].x += p;
    out[i].y -= fx;
    out[i].z -= fy;
  }
}

// Cells of a 2D tree lie in the plane z = 0.
__global__ void k2_flatten(double4 *xr, int ncells) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncells) xr[c].z = 0.0;
}

}  // namespace

void flatten_tree_2d(Handle &h) {
  k2_flatten<<<grid_for(h.ncells, 256), 256, 0, h.stream>>>(h.c_xr.as<double4>(), h.ncells);
  h.launches++;
  FMM_LAUNCH();
}

void upward_pass_2d(Handle &h, cudaStream_t s) {
  const int P = h.prm.P;
  h.M.need((size_t)h.ncells * P * sizeof(double2));
  h.L.need((size_t)h.ncells * P * sizeof(double2));
  k2_p2m<<<grid_for(h.nleaves, W2), W2 * 32, W2 * P * sizeof(double2), s>>>(
      h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(), h.c_xr.as<double4>(),
      h.src.as<double4>(), h.M.as<double2>(), P);
  h.launches++;
  FMM_LAUNCH();
  for (int l = h.depth - 1; l >= 0; l--) {
    const int c0 = h.level_base[l], c1 = h.level_base[l + 1];
    if (c1 <= c0) continue;
    k2_m2m<<<grid_for((long)(c1 - c0) * P, 256), 256, 0, s>>>(c0, c1 - c0, h.c_child.as<int>(), h.c_nchild.as<int>(),
                                                             h.c_xr.as<double4>(), h.M.as<double2>(), P);
    h.launches++;
    FMM_LAUNCH();
  }
}

void m2l_pass_2d(Handle &h) {
  const int P = h.prm.P;
  h.L.need((size_t)h.ncells * P * sizeof(double2));
  order_m2l_lists(h);
  const double cyc = h.prm.images ? h.prm.cycle : 0.0;
  const int g = grid_for(h.ncells, W2);
  auto lane_form = [&](auto pc) {
    constexpr int PP = decltype(pc)::value;
    k2_m2l_lane<PP><<<g, W2 * 32, 0, h.stream>>>(h.ncells, h.m2l_off.as<int>(), h.m2l_ent.as<u32>(),
                                                h.c_xr.as<double4>(), h.M.as<double2>(), h.L.as<double2>(), cyc);
  };
  switch (P) {
    case 2: lane_form(std::integral_constant<int, 2>{}); break;
    case 3: lane_form(std::integral_constant<int, 3>{}); break;
    case 4: lane_form(std::integral_constant<int, 4>{}); break;
    case 5: lane_form(std::integral_constant<int, 5>{}); break;
    case 6: lane_form(std::integral_constant<int, 6>{}); break;
    case 7: lane_form(std::integral_constant<int, 7>{}); break;
    case 8: lane_form(std::integral_constant<int, 8>{}); break;
    case 9: lane_form(std::integral_constant<int, 9>{}); break;
    case 10: lane_form(std::integral_constant<int, 10>{}); break;
    case 11: lane_form(std::integral_constant<int, 11>{}); break;
    case 12: lane_form(std::integral_constant<int, 12>{}); break;
    case 13: lane_form(std::integral_constant<int, 13>{}); break;
    case 14: lane_form(std::integral_constant<int, 14>{}); break;
    case 15: lane_form(std::integral_constant<int, 15>{}); break;
    case 16: lane_form(std::integral_constant<int, 16>{}); break;
    default:  // larger orders: a warp per entry, a lane per coefficient
      k2_m2l<<<g, W2 * 32, 0, h.stream>>>(h.ncells, h.m2l_off.as<int>(), h.m2l_ent.as<u32>(), h.c_xr.as<double4>(),
                                          h.M.as<double2>(), h.L.as<double2>(), P, cyc);
  }
  h.launches++;
  FMM_LAUNCH();
}

void periodic_pass_2d(Handle &h) {
  if (h.prm.images < 2) return;
  k2_periodic<<<1, 32, 0, h.stream>>>(h.c_xr.as<double4>(), h.M.as<double2>(), h.L.as<double2>(), h.prm.P,
                                      h.prm.images, h.prm.cycle);
  h.launches++;
  FMM_LAUNCH();
}

void p2p_pass_2d(Handle &h, cudaStream_t s) {
  h.out.need((size_t)h.n * sizeof(double4));
  k2_p2p<<<grid_for(h.nleaves, W2), W2 * 32, 0, s>>>(h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(),
                                                     h.c_count.as<int>(), h.p2p_off.as<int>(), h.p2p_ent.as<u32>(),
                                                     h.src.as<double4>(), h.out.as<double4>(),
                                                     h.prm.images ? h.prm.cycle : 0.0);
  h.launches++;
  FMM_LAUNCH();
}

void downward_pass_2d(Handle &h, cudaStream_t s, cudaEvent_t before_l2p) {
  const int P = h.prm.P;
  for (int l = 0; l < h.depth; l++) {
    const int c0 = h.level_base[l], c1 = h.level_base[l + 1];
    if (c1 <= c0) continue;
    k2_l2l<<<grid_for((long)(c1 - c0) * 8 * P, 256), 256, 0, s>>>(c0, c1 - c0, h.c_child.as<int>(),
                                                                  h.c_nchild.as<int>(), h.c_xr.as<double4>(),
                                                                  h.L.as<double2>(), P);
    h.launches++;
    FMM_LAUNCH();
  }
  if (before_l2p) FMM_CUDA(cudaStreamWaitEvent(s, before_l2p, 0));
  k2_l2p<<<grid_for(h.nleaves, W2), W2 * 32, W2 * P * sizeof(double2), s>>>(
      h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(), h.c_xr.as<double4>(),
      h.src.as<double4>(), h.L.as<double2>(), h.out.as<double4>(), P);
  h.launches++;
  FMM_LAUNCH();
}

void direct_sum_2d(Handle &h, double4 *targets, double4 *out, long nt) {
  int prange = 0;  // r = sum_{i < images} 3^i (2dp/traverse_eager.h:131-134)
  for (int i = 0, p3 = 1; i < h.prm.images; i++, p3 *= 3) prange += p3;
  k2_direct<<<grid_for(nt, DT2), DT2, 0, h.stream>>>(targets, nt, h.src.as<double4>(), h.n, out, prange,
                                                     h.prm.images ? h.prm.cycle : 0.0);
  h.launches++;
  FMM_LAUNCH();
}

}  // namespace fmm
