// Upward and downward passes in FP64: P2M at the leaves, M2M bottom-up one
// level per launch, L2L top-down one level per launch, L2P at the leaves
// (3d/kernel.h:187-323; traversal order 3d/traverse_eager.h:127-190, which
// the level-synchronous launches respect: a cell's children are complete
// before its M2M, and its parent's local is final before its L2L).
//
// Mapping: P2M and L2P take one warp per leaf and one lane per body.  M2M
// and L2L take one thread per (cell, output coefficient (j,k)); the offset
// harmonics they need depend only on level and octant and come from a
// table built once per upward pass.
#include <algorithm>
#include <vector>

#include "fmm.cuh"
#include "harmonics.cuh"
#include "translations.cuh"

namespace fmm {

namespace {

constexpr int WARPS = 4;

// 1/k for the Legendre and factorial recurrences (k = 1..2*EXAFMM_MAX_P+2).
__constant__ double c_recip[2 * EXAFMM_MAX_P + 4];

// All regular harmonics of one offset, generated order by order: calls
// f(n, m, Y_n^m, dY_n^m) for m = 0..P-1, n = m..P-1, in that (uniform) order
// so that lanes working on different bodies stay in lock step.
template <bool WITH_DY, class F>
__device__ __forceinline__ void regular_all(int P, const Sph &g, double2 e1, F f) {
  double2 em = make_double2(1, 0);
  double pmm = 1, odd = 1, cm = 1;
  for (int m = 0; m < P; m++) {
    double p = pmm, p1 = 0, cn = cm;
    for (int n = m; n < P; n++) {
      const double pn1 = n == m ? g.c * (2 * m + 1) * p : (g.c * (2 * n + 1) * p - (n + m) * p1) * c_recip[n - m + 1];
      const double2 Y = cscale(em, cn * p);
      double2 dY = make_double2(0, 0);
      if (WITH_DY) dY = cscale(em, cn * ((n - m + 1) * pn1 - (n + 1) * g.c * p) * g.inv_s);
      f(n, m, Y, dY);
      p1 = p;
      p = pn1;
      cn *= -g.r * c_recip[n + 1 + m];
    }
    cm *= -g.r * c_recip[2 * m + 2] * c_recip[2 * m + 1];
    pmm = -pmm * odd * g.s;
    odd += 2;
    em = cmul(em, e1);
  }
}

// P2M (3d/kernel.h:187-202): M[n][m] += q * Y_n^m(rho, alpha, -beta).  One
// warp per leaf, one lane per body; each coefficient is summed over the
// warp's bodies with a butterfly and added by lane 0.
__global__ void __launch_bounds__(WARPS * 32) k_p2m(const int *leaves, int nleaves, const int *begin,
                                                    const int *count, const double4 *xr, const double4 *src,
                                                    double2 *M, int P) {
  extern __shared__ double2 sh[];
  const int nt = tri(P);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * WARPS + wid;
  if (w >= nleaves) return;
  double2 *acc = sh + wid * nt;
  for (int k = lane; k < nt; k += 32) acc[k] = make_double2(0, 0);
  __syncwarp();
  const int c = leaves[w];
  const double4 C = xr[c];
  const int b0 = begin[c], nb = count[c];
  for (int t = 0; t < nb; t += 32) {
    const bool ok = t + lane < nb;
    const double4 B = ok ? src[b0 + t + lane] : make_double4(C.x, C.y, C.z, 0.0);
    const Sph g = sph_of(B.x - C.x, B.y - C.y, B.z - C.z);
    regular_all<false>(P, g, cconj(g.e), [&](int n, int m, double2 Y, double2) {
      double x = B.w * Y.x, y = B.w * Y.y;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
      }
      if (lane == 0) {
        acc[tri(n) + m].x += x;
        acc[tri(n) + m].y += y;
      }
    });
  }
  __syncwarp();
  for (int k = lane; k < nt; k += 32) M[(long)c * nt + k] = acc[k];
}

// M2M (3d/kernel.h:204-231), one warp per parent at one level.
// ---- mixed form: P2M and L2P in FP32 (bodies relative to their leaf centre,
// the FP32 copy the near field uses), same lock-step generator in float;
// expansions stay FP64 in memory.
__constant__ float c_recip_f[2 * EXAFMM_MAX_P + 4];
#ifndef P2M_TRANSPOSE
#define P2M_TRANSPOSE 1
#endif
#ifndef L2P_F32_MIN_BLOCKS
#define L2P_F32_MIN_BLOCKS 6  // 128-thread blocks per SM: up to 80 registers a thread
#endif
// orders with unrolled FP32 P2M / L2P kernels (others take the runtime-order ones)
#define EXAFMM_UNROLLED_ORDERS(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

struct SphF {
  float r, c, s, inv_s;
  float2 e;
};

__device__ __forceinline__ SphF sph_of_f(float dx, float dy, float dz) {
  SphF o;
  const float rxy2 = dx * dx + dy * dy;
  o.r = sqrtf(rxy2 + dz * dz);
  const float rxy = sqrtf(rxy2);
  if (o.r == 0.f) {
    o.c = 1.f;
    o.s = 0.f;
  } else {
    o.c = dz / o.r;
    o.s = rxy / o.r;
  }
  o.inv_s = o.s == 0.f ? 0.f : 1.f / o.s;
  if (rxy == 0.f) o.e = make_float2(1.f, 0.f);
  else o.e = make_float2(dx / rxy, dy / rxy);
  return o;
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// PT > 0: the order as a compile-time constant -- the loops unroll and the
// integer factors and reciprocals become immediates; PT = 0: runtime order Prt.
template <int PT, bool WITH_DY, class F>
__device__ __forceinline__ void regular_all_f(int Prt, const SphF &g, float2 e1, F f) {
  const int P = PT > 0 ? PT : Prt;
  auto rcp = [](int k) { return PT > 0 ? 1.0f / (float)k : c_recip_f[k]; };
  float2 em = make_float2(1.f, 0.f);
  float pmm = 1.f, odd = 1.f, cm = 1.f;
#pragma unroll
  for (int m = 0; m < P; m++) {
    float p = pmm, p1 = 0.f, cn = cm;
#pragma unroll
    for (int n = m; n < P; n++) {
      const float pn1 =
          n == m ? g.c * (float)(2 * m + 1) * p : (g.c * (float)(2 * n + 1) * p - (float)(n + m) * p1) * rcp(n - m + 1);
      const float2 Y = make_float2(em.x * cn * p, em.y * cn * p);
      float2 dY = make_float2(0.f, 0.f);
      if (WITH_DY) {
        const float d = cn * ((float)(n - m + 1) * pn1 - (float)(n + 1) * g.c * p) * g.inv_s;
        dY = make_float2(em.x * d, em.y * d);
      }
      f(n, m, Y, dY);
      p1 = p;
      p = pn1;
      cn *= -g.r * rcp(n + 1 + m);
    }
    cm *= -g.r * rcp(2 * m + 2) * rcp(2 * m + 1);
    pmm = -pmm * odd * g.s;
    odd += 2.f;
    em = cmulf(em, e1);
  }
}

// Binary exponent of a leaf radius (clamped): the FP32 expansion kernels work
// in units of 2^e, where the radius lies in [1, 2).
__device__ __forceinline__ int leaf_exponent(double R) { return R > 0 ? max(-100, min(100, ilogb(R))) : 0; }

// P2M in FP32: lane per body, each coefficient reduced over the warp by a
// float butterfly, chunks of 32 bodies summed in FP64.
template <int PT>
__global__ void __launch_bounds__(WARPS * 32) k_p2m_f32(const int *leaves, int nleaves, const int *begin,
                                                        const int *count, const double4 *xr, const float4 *srcf,
                                                        double2 *M, int Prt) {
  extern __shared__ double2 sh[];
  const int P = PT > 0 ? PT : Prt;
  const int nt = tri(P);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * WARPS + wid;
  if (w >= nleaves) return;
  double2 *acc = sh + wid * nt;
  for (int k = lane; k < nt; k += 32) acc[k] = make_double2(0, 0);
  __syncwarp();
  const int c = leaves[w];
  const int ex = leaf_exponent(xr[c].w);
  const float sc = exp2f((float)-ex);  // coordinates in units where the leaf radius is in [1, 2)
  const int b0 = begin[c], nb = count[c];
  for (int t = 0; t < nb; t += 32) {
    const bool ok = t + lane < nb;
    const float4 B = ok ? srcf[b0 + t + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
    const SphF g = sph_of_f(B.x * sc, B.y * sc, B.z * sc);
    regular_all_f<PT, false>(P, g, make_float2(g.e.x, -g.e.y), [&](int n, int m, float2 Y, float2) {
      float x = B.w * Y.x, y = B.w * Y.y;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
      }
      if (lane == 0) {
        acc[tri(n) + m].x += (double)x;
        acc[tri(n) + m].y += (double)y;
      }
    });
  }
  __syncwarp();
  for (int k = lane; k < nt; k += 32) {  // back to the input units: M_n = M~_n R_s^n (exact)
    const int n = order_of(k);
    M[(long)c * nt + k] = make_double2(scalbn(acc[k].x, ex * n), scalbn(acc[k].y, ex * n));
  }
}

// P2M in FP32 for a compile-time order: each lane writes its body's q Y
// terms to shared memory 32 terms at a time, then lane k sums term k of the
// batch over the 32 bodies (rows padded to 33 entries: conflict-free), and
// the sums are added in FP64.  The batch buffer (8 KB per warp) keeps
// enough warps resident to hide the recurrence's latency.
constexpr int P2M_ROW = 33;
constexpr size_t p2m_t_smem(int nt) { return WARPS * (nt * sizeof(double2) + 32 * P2M_ROW * sizeof(float2) + 32 * sizeof(int)); }

template <int PT>
__global__ void __launch_bounds__(WARPS * 32) k_p2m_f32t(const int *leaves, int nleaves, const int *begin,
                                                         const int *count, const double4 *xr, const float4 *srcf,
                                                         double2 *M) {
  constexpr int NT = PT * (PT + 1) / 2, ROW = P2M_ROW;
  extern __shared__ double2 sh[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * WARPS + wid;
  if (w >= nleaves) return;
  double2 *acc = sh + wid * NT;
  float2 *buf = (float2 *)(sh + WARPS * NT) + wid * 32 * ROW;
  int *rowidx = (int *)((float2 *)(sh + WARPS * NT) + WARPS * 32 * ROW) + wid * 32;
  for (int k = lane; k < NT; k += 32) acc[k] = make_double2(0, 0);
  const int c = leaves[w];
  const int ex = leaf_exponent(xr[c].w);
  const float sc = exp2f((float)-ex);  // coordinates in units where the leaf radius is in [1, 2)
  const int b0 = begin[c], nb = count[c];
  for (int t = 0; t < nb; t += 32) {
    const bool ok = t + lane < nb;
    const float4 B = ok ? srcf[b0 + t + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
    const SphF g = sph_of_f(B.x * sc, B.y * sc, B.z * sc);
    int gen = 0;  // terms generated so far (a constant at every unrolled step)
    __syncwarp();
    regular_all_f<PT, false>(PT, g, make_float2(g.e.x, -g.e.y), [&](int n, int m, float2 Y, float2) {
      const int slot = gen & 31;
      buf[slot * ROW + lane] = make_float2(B.w * Y.x, B.w * Y.y);
      if (lane == 0) rowidx[slot] = tri(n) + m;
      gen++;
      if ((gen & 31) == 0 || gen == NT) {  // sum the batch over the bodies
        __syncwarp();
        if (lane <= ((gen - 1) & 31)) {
          float sx = 0.f, sy = 0.f;
#pragma unroll 8
          for (int b = 0; b < 32; b++) {
            const float2 v = buf[lane * ROW + b];
            sx += v.x;
            sy += v.y;
          }
          double2 &a = acc[rowidx[lane]];
          a.x += (double)sx;
          a.y += (double)sy;
        }
        __syncwarp();
      }
    });
  }
  __syncwarp();
  for (int k = lane; k < NT; k += 32) {  // back to the input units: M_n = M~_n R_s^n (exact)
    const int n = order_of(k);
    M[(long)c * NT + k] = make_double2(scalbn(acc[k].x, ex * n), scalbn(acc[k].y, ex * n));
  }
}

// L2P in FP32, in two parts.  k_l2p_prep (before the wait for the near
// field): per leaf, the local expansion in the leaf's units, L~_n = L_n R^n
// with R the leaf radius rounded down to a power of two (exact), as FP32,
// and the scale 1/R for the coordinates -- so the FP32 terms stay in range
// at any domain size.  k_l2p_f32: a thread per body over all bodies (tree
// order, every lane busy whatever the leaf sizes), its leaf's expansion
// read through L1 (the lanes of a warp share one or two leaves); p and F
// added to the FP64 results.
__global__ void k_l2p_prep(const int *leaves, int nleaves, const double4 *xr, const double2 *L, int nt, float2 *Lf,
                           float *lsc) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)nleaves * nt) return;
  const int w = (int)(i / nt), k = (int)(i - (long)w * nt), c = leaves[w];
  const int ex = leaf_exponent(xr[c].w), n = order_of(k);
  const double2 l = L[(long)c * nt + k];
  Lf[i] = make_float2((float)scalbn(l.x, ex * n), (float)scalbn(l.y, ex * n));
  if (k == 0) lsc[w] = exp2f((float)-ex);
}

template <int PT>
__global__ void __launch_bounds__(128, L2P_F32_MIN_BLOCKS) k_l2p_f32(long nbodies, const int *body_leaf,
                                                                   const float4 *srcf, const float2 *Lf,
                                                                   const float *lsc, double4 *out, int Prt) {
  const int P = PT > 0 ? PT : Prt;
  const int nt = tri(P);
  const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbodies) return;
  const int w = body_leaf[b];
  const float sc = lsc[w];
  const float2 *Lw = Lf + (size_t)w * nt;
  const float4 B = srcf[b];
  const SphF g = sph_of_f(B.x * sc, B.y * sc, B.z * sc);
  float pot = 0.f, s0 = 0.f, s1 = 0.f, s2 = 0.f;
  regular_all_f<PT, true>(P, g, g.e, [&](int n, int m, float2 Y, float2 dY) {
    const float2 l = __ldg(Lw + tri(n) + m);
    const float w2 = m == 0 ? 1.f : 2.f;
    const float re = l.x * Y.x - l.y * Y.y;
    const float red = l.x * dY.x - l.y * dY.y;
    const float rei = -(l.x * Y.y + l.y * Y.x);
    pot += w2 * re;
    s0 += w2 * re * (float)n;
    s1 += w2 * red;
    s2 += w2 * rei * (float)m;
  });
  s0 = g.r != 0.f ? s0 / g.r : 0.f;
  const float st = g.s, ct = g.c, cp = g.e.x, sp = g.e.y, r = g.r;
  float fx = st * cp * s0, fy = st * sp * s0, fz = ct * s0;
  if (r != 0.f) {
    fx += ct * cp / r * s1;
    fy += ct * sp / r * s1;
    fz -= st / r * s1;
    if (st != 0.f) {
      fx -= sp / r / st * s2;
      fy += cp / r / st * s2;
    }
  }
  double4 &d = out[b];  // the gradient back to the input units
  d.x += pot;
  d.y += fx * sc;
  d.z += fy * sc;
  d.w += fz * sc;
}

// M2M and L2L.  A child sits at its parent's centre +-R_child on every
// axis, so the offset harmonics depend only on the octant and, through
// rho = R_child, on the level: Y_n = rho^n Yhat_n with Yhat the harmonics of
// the unit offset (+-1, +-1, +-1).  The 16 unit tables (M2M: parent - child,
// L2L: child - parent; octant bit b set = child on the + side of axis b) are
// built once per order P; each launch scales them for its level.
// ytab[(dir * 8 + oct) * nt + tri(n) + m], dir 0 = M2M, 1 = L2L.
// Both kernels take one CTA per parent and one thread per (octant, output
// coefficient (j,k)), all inputs staged in shared memory.

__global__ void k_unit_tables(int P, double2 *ytab) {
  const int nt = tri(P);
  const int oct = blockIdx.x & 7, dir = blockIdx.x >> 3;
  const double sx = (oct & 1) ? 1.0 : -1.0, sy = (oct & 2) ? 1.0 : -1.0, sz = (oct & 4) ? 1.0 : -1.0;
  const double f = dir == 0 ? -1.0 : 1.0;  // M2M: parent - child; L2L: child - parent
  const Sph g = sph_of(sx * f, sy * f, sz * f);
  double2 *Y = ytab + (size_t)blockIdx.x * nt;
  const int m = threadIdx.x;
  if (m < P) regular_column(m, P, g.r, g, g.e, [&](int n, double2 v, double2) { Y[tri(n) + m] = v; });
}

constexpr int SH_O = 64;          // threads per octant (outputs; more loop for P > 10)
constexpr int SH_T = 8 * SH_O;    // threads per CTA

// Y[oct][idx] = rho^n * Yhat[dir][oct][idx] into shared memory.
__device__ void stage_tables(double2 *Y, const double2 *ytab, int dir, double rho, int P) {
  const int nt = tri(P);
  for (int e = threadIdx.x; e < 8 * nt; e += blockDim.x) {
    const int oct = e / nt, idx = e - oct * nt;
    const int n = order_of(idx);
    double sc = 1;
    for (int q = 0; q < n; q++) sc *= rho;
    Y[e] = cscale(ytab[(size_t)(dir * 8 + oct) * nt + idx], sc);
  }
}

// M2M of one level: thread (oct, o) translates the child in octant oct (if
// any); the eight contributions are summed in octant order.
// Term table of one translation for order P: output slot r computes
// output perm[r] from terms[off[r], off[r+1]); slots sorted by descending
// term count so the lanes of a warp do similar work.
struct TermTable {
  const int *perm, *off;
  const unsigned *terms;
};

__global__ void __launch_bounds__(SH_T) k_m2m(int c0, const int *child, const int *nchild, const double4 *xr,
                                             const double2 *ytab, TermTable tab, double2 *M, int P) {
  extern __shared__ double2 sm2[];  // Y[8][nt], Mc[8][nt], part[8][nt]
  __shared__ int cho[8];
  const int nt = tri(P), c = c0 + blockIdx.x;
  const int nk = nchild[c];
  if (nk == 0) return;
  double2 *Y = sm2, *Mc = Y + 8 * nt, *part = Mc + 8 * nt;
  const double4 X = xr[c];
  if (threadIdx.x < 8) cho[threadIdx.x] = -1;
  __syncthreads();
  if (threadIdx.x < nk) {
    const int q = child[c] + threadIdx.x;
    cho[octant_of(xr[q], X)] = q;
  }
  stage_tables(Y, ytab, 0, X.w * 0.5, P);
  __syncthreads();
  for (int e = threadIdx.x; e < 8 * nt; e += SH_T) {
    const int oct = e / nt, q = cho[oct];
    Mc[e] = q >= 0 ? M[(long)q * nt + (e - oct * nt)] : make_double2(0, 0);
  }
  __syncthreads();
  const int oct = threadIdx.x / SH_O;
  for (int r = threadIdx.x % SH_O; r < nt; r += SH_O) {  // outputs by descending term count
    const int o = tab.perm[r];
    part[oct * nt + o] = cho[oct] >= 0 ? apply_terms(tab.terms + tab.off[r], tab.off[r + 1] - tab.off[r],
                                                     Mc + oct * nt, Y + oct * nt)
                                       : make_double2(0, 0);
  }
  __syncthreads();
  for (int o = threadIdx.x; o < nt; o += SH_T) {
    double2 sum = make_double2(0, 0);
    for (int q = 0; q < 8; q++) {
      sum.x += part[q * nt + o].x;
      sum.y += part[q * nt + o].y;
    }
    M[(long)c * nt + o] = sum;
  }
}

// L2L of one level of parents: thread (oct, o) adds the parent's local,
// shifted, into output o of its child in octant oct.
__global__ void __launch_bounds__(SH_T) k_l2l(int c0, const int *child, const int *nchild, const double4 *xr,
                                             const double2 *ytab, TermTable tab, double2 *L, int P) {
  extern __shared__ double2 sm2[];  // Y[8][nt], Lp[nt]
  __shared__ int cho[8];
  const int nt = tri(P), c = c0 + blockIdx.x;
  const int nk = nchild[c];
  if (nk == 0) return;
  double2 *Y = sm2, *Lp = Y + 8 * nt;
  const double4 X = xr[c];
  if (threadIdx.x < 8) cho[threadIdx.x] = -1;
  __syncthreads();
  if (threadIdx.x < nk) {
    const int q = child[c] + threadIdx.x;
    cho[octant_of(xr[q], X)] = q;
  }
  stage_tables(Y, ytab, 1, X.w * 0.5, P);
  for (int e = threadIdx.x; e < nt; e += SH_T) Lp[e] = L[(long)c * nt + e];
  __syncthreads();
  const int oct = threadIdx.x / SH_O, q = cho[oct];
  if (q < 0) return;
  for (int r = threadIdx.x % SH_O; r < nt; r += SH_O) {  // outputs by descending term count
    const int o = tab.perm[r];
    const double2 v = apply_terms(tab.terms + tab.off[r], tab.off[r + 1] - tab.off[r], Lp, Y + oct * nt);
    double2 &d = L[(long)q * nt + o];
    d.x += v.x;
    d.y += v.y;
  }
}

// ---- octant-batched L2L (orders P <= OB_MAXP).  One thread per output
// coefficient walks that output's term list once for all eight children:
// the parent's input and the term's index arithmetic are shared, and the
// signs live in the tables -- the parent's local expansion is staged as
// (conjugate / negated) copies and the unit harmonics as conjugate
// variants, so a term is two plain index offsets.  A scaled expansion keeps
// both parents of a CTA on the same unit tables: the kernel stages
// L(n) * rho^n and multiplies output degree j by rho^-j (rho = the child
// radius), each by repeated multiplication so no intermediate leaves the
// range of the scaled values.  (In FP64 the per-octant M2M kernel above is
// as fast as an octant-batched one: its eight children bring eight
// different inputs; the mixed form uses the octant-batched k_m2m_ob32.)
constexpr int OB_PAR = 2;    // parents per CTA
constexpr int OB_T = 64;     // threads per parent (outputs)
constexpr int OB_MAXP = 16;

// degree of coefficient index ci
__device__ __forceinline__ int deg_of(int ci) {
  int n = (int)((sqrtf(8.0f * ci + 1.0f) - 1.0f) * 0.5f);
  while (tri(n) > ci) n--;
  while (tri(n + 1) <= ci) n++;
  return n;
}

template <class V>
__device__ __forceinline__ void cfma(V &acc, const V a, const V y) {
  acc.x = fma(a.x, y.x, fma(-a.y, y.y, acc.x));
  acc.y = fma(a.x, y.y, fma(a.y, y.x, acc.y));
}

// complex value type of a compute precision
template <bool F32>
struct Cplx {
  typedef double2 V;
  typedef double R;
};
template <>
struct Cplx<true> {
  typedef float2 V;
  typedef float R;
};

// Unit harmonic variants into shared memory: Yv[v][oct][idx], v bit 0
// conjugate, bit 1 negate (nv = 2 or 4 variants).
template <class V>
__device__ void stage_unit_variants(V *Yv, const double2 *ytab, int dir, int nt, int nv) {
  for (int e = threadIdx.x; e < nv * 8 * nt; e += blockDim.x) {
    const int v = e / (8 * nt), r = e - v * 8 * nt;
    double2 y = ytab[(size_t)dir * 8 * nt + r];
    if (v & 1) y.y = -y.y;
    if (v & 2) y = make_double2(-y.x, -y.y);
    Yv[e].x = y.x;
    Yv[e].y = y.y;
  }
}

// Octant-batched M2M for the mixed form: one thread per output coefficient
// sums all eight children in one walk of the output's term list; children
// staged as scaled multipoles M(d) / rho^d (plain and conjugate copies, zero
// for an absent child), the unit harmonics in four sign variants, products
// in FP32 on these order-one values, the output rescaled by rho^j in FP64.
__global__ void __launch_bounds__(OB_PAR * OB_T) k_m2m_ob32(int c0, int np, const int *child, const int *nchild,
                                                         const double4 *xr, const double2 *ytab, TermTable tab,
                                                         double2 *M, int P) {
  extern __shared__ __align__(16) unsigned char smraw[];
  float2 *sm2 = (float2 *)smraw;
  const int nt = tri(P);
  float2 *Yv = sm2;           // [4][8][nt] unit harmonics (parent - child)
  float2 *A = Yv + 32 * nt;   // [OB_PAR][8][2][nt] scaled child multipoles, plain and conjugate
  __shared__ int cho[OB_PAR][8];
  const int slot = threadIdx.x / OB_T, tl = threadIdx.x % OB_T;
  const int pi = blockIdx.x * OB_PAR + slot, c = c0 + pi;
  const bool has = pi < np && nchild[c] > 0;  // a leaf keeps its P2M multipole
  if (tl < 8) cho[slot][tl] = -1;
  __syncthreads();
  if (has && tl < nchild[c]) {
    const int q = child[c] + tl;
    cho[slot][octant_of(xr[q], xr[c])] = q;
  }
  stage_unit_variants(Yv, ytab, 0, nt, 4);
  __syncthreads();
  const double inv = has ? 1.0 / (xr[c].w * 0.5) : 0.0;  // 1 / R_child
  for (int e = tl; e < 8 * nt; e += OB_T) {
    const int oct = e / nt, ci = e - oct * nt, q = cho[slot][oct];
    double2 v = make_double2(0, 0);
    if (has && q >= 0) {
      v = M[(long)q * nt + ci];
      for (int d = deg_of(ci); d > 0; d--) v = make_double2(v.x * inv, v.y * inv);
    }
    float2 *a = A + ((size_t)slot * 8 + oct) * 2 * nt;
    a[ci] = make_float2((float)v.x, (float)v.y);
    a[nt + ci] = make_float2((float)v.x, (float)-v.y);
  }
  __syncthreads();
  if (!has) return;
  const float2 *As = A + (size_t)slot * 8 * 2 * nt;
  const double rho = xr[c].w * 0.5;
  for (int r = tl; r < nt; r += OB_T) {
    const int o = tab.perm[r];
    const unsigned *t = tab.terms + tab.off[r];
    const int nterm = tab.off[r + 1] - tab.off[r];
    float2 acc[8];  // one chain per octant
#pragma unroll
    for (int oct = 0; oct < 8; oct++) acc[oct] = make_float2(0.f, 0.f);
    for (int qq = 0; qq < nterm; qq++) {
      const unsigned e = t[qq];
      const int ia = (int)(e & 2047u), iy = (int)(e >> 11);
#pragma unroll
      for (int oct = 0; oct < 8; oct++) cfma(acc[oct], As[oct * 2 * nt + ia], Yv[iy + oct * nt]);
    }
    double2 v = make_double2(0, 0);
#pragma unroll
    for (int oct = 0; oct < 8; oct++) {
      v.x += acc[oct].x;
      v.y += acc[oct].y;
    }
    for (int d = deg_of(o); d > 0; d--) v = make_double2(v.x * rho, v.y * rho);
    M[(long)c * nt + o] = v;
  }
}

// F32 (mixed form): the products in FP32 on the scaled (order-one) values;
// staging, the rescaling and the sums into L stay FP64.
template <bool F32>
__global__ void __launch_bounds__(OB_PAR * OB_T) k_l2l_ob(int c0, int np, const int *child, const int *nchild,
                                                       const double4 *xr, const double2 *ytab, TermTable tab,
                                                       double2 *L, int P) {
  typedef typename Cplx<F32>::V V;
  extern __shared__ __align__(16) unsigned char smraw[];
  V *sm2 = (V *)smraw;
  const int nt = tri(P);
  V *Yv = sm2;          // [2][8][nt] unit harmonics (child - parent)
  V *A = Yv + 16 * nt;  // [OB_PAR][4][nt] scaled parent local: plain, conjugate, negated, both
  __shared__ int cho[OB_PAR][8];
  const int slot = threadIdx.x / OB_T, tl = threadIdx.x % OB_T;
  const int pi = blockIdx.x * OB_PAR + slot, c = c0 + pi;
  const bool has = pi < np && nchild[c] > 0;  // a leaf has no children to shift to
  if (tl < 8) cho[slot][tl] = -1;
  __syncthreads();
  if (has && tl < nchild[c]) {
    const int q = child[c] + tl;
    cho[slot][octant_of(xr[q], xr[c])] = q;
  }
  stage_unit_variants(Yv, ytab, 1, nt, 2);
  const double rho = has ? xr[c].w * 0.5 : 0.0;  // R_child
  for (int ci = tl; ci < nt; ci += OB_T) {
    double2 v = make_double2(0, 0);
    if (has) {
      v = L[(long)c * nt + ci];
      for (int d = deg_of(ci); d > 0; d--) v = make_double2(v.x * rho, v.y * rho);
    }
    V *a = A + (size_t)slot * 4 * nt;
    a[ci].x = v.x;
    a[ci].y = v.y;
    a[nt + ci].x = v.x;
    a[nt + ci].y = -v.y;
    a[2 * nt + ci].x = -v.x;
    a[2 * nt + ci].y = -v.y;
    a[3 * nt + ci].x = -v.x;
    a[3 * nt + ci].y = v.y;
  }
  __syncthreads();
  if (!has) return;
  const V *As = A + (size_t)slot * 4 * nt;
  const double inv = 1.0 / rho;
  int kids[8];
#pragma unroll
  for (int oct = 0; oct < 8; oct++) kids[oct] = cho[slot][oct];
  for (int r = tl; r < nt; r += OB_T) {
    const int o = tab.perm[r];
    const unsigned *t = tab.terms + tab.off[r];
    const int nterm = tab.off[r + 1] - tab.off[r];
    V acc[8];
#pragma unroll
    for (int oct = 0; oct < 8; oct++) acc[oct].x = acc[oct].y = 0;
    for (int qq = 0; qq < nterm; qq++) {
      const unsigned e = t[qq];
      const V a = As[e & 2047u];
      const int iy = (int)(e >> 11);
#pragma unroll
      for (int oct = 0; oct < 8; oct++) cfma(acc[oct], a, Yv[iy + oct * nt]);
    }
    const int dj = deg_of(o);
#pragma unroll
    for (int oct = 0; oct < 8; oct++) {
      if (kids[oct] < 0) continue;
      double2 v = make_double2(acc[oct].x, acc[oct].y);
      for (int d = dj; d > 0; d--) v = make_double2(v.x * inv, v.y * inv);
      double2 &dst = L[(long)kids[oct] * nt + o];
      dst.x += v.x;
      dst.y += v.y;
    }
  }
}

// L2P (3d/kernel.h:293-323): potential and force at each body of a leaf.
__global__ void __launch_bounds__(WARPS * 32) k_l2p(const int *leaves, int nleaves, const int *begin,
                                                    const int *count, const double4 *xr, const double4 *src,
                                                    const double2 *L, double4 *out, int P) {
  extern __shared__ double2 sh[];
  const int nt = tri(P);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * WARPS + wid;
  if (w >= nleaves) return;
  const int c = leaves[w];
  double2 *Lc = sh + wid * nt;
  for (int k = lane; k < nt; k += 32) Lc[k] = L[(long)c * nt + k];
  __syncwarp();
  const double4 C = xr[c];
  const int b0 = begin[c], nb = count[c];
  for (int t = 0; t < nb; t += 32) {
    const int b = b0 + t + lane;
    const bool ok = t + lane < nb;
    const double4 B = ok ? src[b] : make_double4(C.x + 1, C.y, C.z, 0.0);
    const Sph g = sph_of(B.x - C.x, B.y - C.y, B.z - C.z);
    double pot = 0, s0 = 0, s1 = 0, s2 = 0;
    regular_all<true>(P, g, g.e, [&](int n, int m, double2 Y, double2 dY) {
      const double2 l = Lc[tri(n) + m];  // same coefficient on every lane: broadcast
      const double w2 = m == 0 ? 1.0 : 2.0;
      const double re = l.x * Y.x - l.y * Y.y;        // Re(L Y)
      const double red = l.x * dY.x - l.y * dY.y;     // Re(L dY)
      const double rei = -(l.x * Y.y + l.y * Y.x);    // Re(L Y i)
      pot += w2 * re;
      s0 += w2 * re * (float)n;
      s1 += w2 * red;
      s2 += w2 * rei * (float)m;
    });
    s0 = g.r != 0 ? s0 / g.r : 0.0;
    if (ok) {
      // sph2cart (3d/kernel.h:31-40); the 1/sin(theta) term is dropped on the
      // polar axis, where every m>0 term (s2) vanishes.
      const double st = g.s, ct = g.c, cp = g.e.x, sp = g.e.y, r = g.r;
      double fx = st * cp * s0, fy = st * sp * s0, fz = ct * s0;
      if (r != 0) {
        fx += ct * cp / r * s1;
        fy += ct * sp / r * s1;
        fz -= st / r * s1;
        if (st != 0) {
          fx -= sp / r / st * s2;
          fy += cp / r / st * s2;
        }
      }
      double4 &d = out[b];
      d.x += pot;
      d.y += fx;
      d.z += fy;
      d.w += fz;
    }
  }
}

}  // namespace

// One cell's P2M or L2P with the FP64 pass kernels, for the single-operator
// entry points: `mini` holds the one-cell tree (leaves = {0}, begin = {0},
// count = {nb}) in device memory, xr the cell, src the bodies (x,y,z,q).
void op_p2m(const int *mini, const double4 *xr, const double4 *src, double2 *M, int P, cudaStream_t s) {
  const int nt = tri(P);
  k_p2m<<<1, WARPS * 32, WARPS * nt * sizeof(double2), s>>>(mini, 1, mini + 1, mini + 2, xr, src, M, P);
  FMM_LAUNCH();
}

void op_l2p(const int *mini, const double4 *xr, const double4 *src, const double2 *L, double4 *out, int P,
            cudaStream_t s) {
  const int nt = tri(P);
  k_l2p<<<1, WARPS * 32, WARPS * nt * sizeof(double2), s>>>(mini, 1, mini + 1, mini + 2, xr, src, L, out, P);
  FMM_LAUNCH();
}

void expansions_set_attributes() {
  double rc[2 * EXAFMM_MAX_P + 4];
  rc[0] = 0;
  for (int k = 1; k < 2 * EXAFMM_MAX_P + 4; k++) rc[k] = 1.0 / k;
  FMM_CUDA(cudaMemcpyToSymbol(c_recip, rc, sizeof(rc)));
  float rf[2 * EXAFMM_MAX_P + 4];
  for (int k = 0; k < 2 * EXAFMM_MAX_P + 4; k++) rf[k] = (float)rc[k];
  FMM_CUDA(cudaMemcpyToSymbol(c_recip_f, rf, sizeof(rf)));
  cudaFuncSetAttribute(k_p2m, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_l2p, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
#define EXAFMM_F32_ATTR(p)                                                                     \
  cudaFuncSetAttribute(k_p2m_f32<p>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024); \
  cudaFuncSetAttribute(k_p2m_f32t<p>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_p2m_f32<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  EXAFMM_UNROLLED_ORDERS(EXAFMM_F32_ATTR)
#undef EXAFMM_F32_ATTR
  cudaFuncSetAttribute(k_m2m, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_l2l_ob<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_m2m_ob32, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_l2l_ob<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_l2l, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

// Term tables of M2M and L2L for order P, built on the host from the same
// enumerators the formulas use.  Layout (ints): per direction perm[nt],
// off[nt + 1], terms[...].
// Term tables of M2M (dir 0) and L2L (dir 1) for the per-octant kernels, and
// (dirs 2, 3, orders up to OB_MAXP) for the octant-batched ones, whose terms
// are ia' | iy' << 11: the input index in its variant plane (M2M: conjugate;
// L2L: conjugate + 2 * negate) and the harmonic index in its variant plane
// of 8 octant tables (M2M: conjugate + 2 * negate; L2L: conjugate).
std::vector<int> term_tables(int P, size_t at[4]) {
  const int nt = tri(P);
  std::vector<int> out;
  for (int dir = 0; dir < 4; dir++) {
    at[dir] = out.size();
    if (dir >= 2 && P > OB_MAXP) continue;
    std::vector<std::vector<unsigned>> per(nt);
    for (int j = 0; j < P; j++)
      for (int k = 0; k <= j; k++) {
        auto emit = [&](int ia, bool ca, int n, int o, int f) {
          unsigned t;
          if (dir < 2) {
            t = pack_term(ia, ca, n, o, f);
          } else {
            const int iy = tri(n) + (o < 0 ? -o : o);
            const int cy = o < 0, neg = f < 0;
            const int va = dir == 2 ? (int)ca : (int)ca + 2 * neg, vy = dir == 2 ? cy + 2 * neg : cy;
            t = (unsigned)(ia + va * nt) | ((unsigned)(iy + vy * 8 * nt) << 11);
          }
          per[tri(j) + k].push_back(t);
        };
        if (dir % 2 == 0) m2m_terms(j, k, emit);
        else l2l_terms(j, k, P, emit);
      }
    std::vector<int> perm(nt);
    for (int o = 0; o < nt; o++) perm[o] = o;
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return per[a].size() > per[b].size(); });
    const size_t base = out.size();
    out.resize(base + 2 * nt + 1);
    int acc = 0;
    for (int r = 0; r < nt; r++) {
      out[base + r] = perm[r];
      out[base + nt + r] = acc;
      acc += (int)per[perm[r]].size();
    }
    out[base + 2 * nt] = acc;
    for (int r = 0; r < nt; r++)
      for (unsigned t : per[perm[r]]) out.push_back((int)t);
  }
  return out;
}

TermTable table_view(const Handle &h, int P, int dir) {
  const int nt = tri(P);
  const int *b = h.shift_terms.as<int>() + h.shift_at[dir];
  return TermTable{b, b + nt, (const unsigned *)(b + 2 * nt + 1)};
}

// Unit offset harmonics and term tables for order P (cached per handle).
void unit_tables(Handle &h, cudaStream_t s) {
  const int P = h.prm.P;
  if (h.shift_P == P) return;
  h.shift_ops.need((size_t)16 * tri(P) * sizeof(double2));
  k_unit_tables<<<16, 32, 0, s>>>(P, h.shift_ops.as<double2>());
  h.launches++;
  FMM_LAUNCH();
  const std::vector<int> t = term_tables(P, h.shift_at);
  h.shift_terms.need(t.size() * sizeof(int));
  FMM_CUDA(cudaMemcpy(h.shift_terms.p, t.data(), t.size() * sizeof(int), cudaMemcpyHostToDevice));
  h.shift_P = P;
}

void upward_pass(Handle &h, cudaStream_t s) {
  if (h.prm.dim == 2) return upward_pass_2d(h, s);
  const int P = h.prm.P, nt = tri(P);
  h.M.need((size_t)h.ncells * nt * sizeof(double2));
  h.L.need((size_t)h.ncells * nt * sizeof(double2));
  if (h.prm.precision == EXAFMM_MIXED) {
    if (s != h.stream && !h.srcf_ready) throw Error{EXAFMM_ERR_STATE, "upward pass on a side stream before its sources"};
    make_srcf(h);
    const dim3 grid(grid_for(h.nleaves, WARPS)), block(WARPS * 32);
    const size_t sm = WARPS * nt * sizeof(double2);
    auto args = [&](auto kernel) {
      kernel<<<grid, block, sm, s>>>(h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(),
                                     h.c_xr.as<double4>(), h.srcf.as<float4>(), h.M.as<double2>(), P);
    };
    const size_t smt = p2m_t_smem(nt);
    auto argst = [&](auto kernel) {
      kernel<<<grid, block, smt, s>>>(h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(),
                                      h.c_xr.as<double4>(), h.srcf.as<float4>(), h.M.as<double2>());
    };
    switch (P) {
#define EXAFMM_P2M_CASE(p) \
  case p:                  \
    if (P2M_TRANSPOSE) argst(k_p2m_f32t<p>); else args(k_p2m_f32<p>); \
    break;
      EXAFMM_UNROLLED_ORDERS(EXAFMM_P2M_CASE)
#undef EXAFMM_P2M_CASE
      default:
        args(k_p2m_f32<0>);
    }
  } else {
    k_p2m<<<grid_for(h.nleaves, WARPS), WARPS * 32, WARPS * nt * sizeof(double2), s>>>(
        h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(), h.c_xr.as<double4>(),
        h.src.as<double4>(), h.M.as<double2>(), P);
  }
  h.launches++;
  FMM_LAUNCH();
  unit_tables(h, s);
  for (int l = h.depth - 1; l >= 0; l--) {
    const int c0 = h.level_base[l], c1 = h.level_base[l + 1];
    if (c1 <= c0) continue;
    if (P <= OB_MAXP && h.prm.precision == EXAFMM_MIXED)
      k_m2m_ob32<<<(c1 - c0 + OB_PAR - 1) / OB_PAR, OB_PAR * OB_T, (32 + OB_PAR * 16) * nt * sizeof(float2), s>>>(
          c0, c1 - c0, h.c_child.as<int>(), h.c_nchild.as<int>(), h.c_xr.as<double4>(), h.shift_ops.as<double2>(),
          table_view(h, P, 2), h.M.as<double2>(), P);
    else
      k_m2m<<<c1 - c0, SH_T, 24 * nt * sizeof(double2), s>>>(c0, h.c_child.as<int>(), h.c_nchild.as<int>(),
                                                            h.c_xr.as<double4>(), h.shift_ops.as<double2>(),
                                                            table_view(h, P, 0), h.M.as<double2>(), P);
    h.launches++;
    FMM_LAUNCH();
  }
}

void downward_pass(Handle &h, cudaStream_t s, cudaEvent_t before_l2p) {
  if (h.prm.dim == 2) return downward_pass_2d(h, s, before_l2p);
  const int P = h.prm.P, nt = tri(P);
  unit_tables(h, s);
  for (int l = 0; l < h.depth; l++) {  // parents at level l push to their children
    const int c0 = h.level_base[l], c1 = h.level_base[l + 1];
    if (c1 <= c0) continue;
    const dim3 grid((c1 - c0 + OB_PAR - 1) / OB_PAR), block(OB_PAR * OB_T);
    if (P <= OB_MAXP && h.prm.precision == EXAFMM_MIXED)
      k_l2l_ob<true><<<grid, block, (16 + OB_PAR * 4) * nt * sizeof(float2), s>>>(
          c0, c1 - c0, h.c_child.as<int>(), h.c_nchild.as<int>(), h.c_xr.as<double4>(), h.shift_ops.as<double2>(),
          table_view(h, P, 3), h.L.as<double2>(), P);
    else if (P <= OB_MAXP)
      k_l2l_ob<false><<<grid, block, (16 + OB_PAR * 4) * nt * sizeof(double2), s>>>(
          c0, c1 - c0, h.c_child.as<int>(), h.c_nchild.as<int>(), h.c_xr.as<double4>(), h.shift_ops.as<double2>(),
          table_view(h, P, 3), h.L.as<double2>(), P);
    else
      k_l2l<<<c1 - c0, SH_T, 9 * nt * sizeof(double2), s>>>(c0, h.c_child.as<int>(), h.c_nchild.as<int>(),
                                                           h.c_xr.as<double4>(), h.shift_ops.as<double2>(),
                                                           table_view(h, P, 1), h.L.as<double2>(), P);
    h.launches++;
    FMM_LAUNCH();
  }
  // L2P adds into the near-field sums; the mixed form's leaf expansions are
  // prepared before the wait for the near field
  float2 *Lf = nullptr;
  float *lsc = nullptr;
  if (h.prm.precision == EXAFMM_MIXED) {
    make_srcf(h);
    const size_t nlf = (size_t)h.nleaves * nt;
    h.l2p_f.need(nlf * sizeof(float2) + (size_t)h.nleaves * sizeof(float) + 16);
    Lf = h.l2p_f.as<float2>();
    lsc = (float *)(Lf + nlf);
    k_l2p_prep<<<grid_for((long)nlf, 256), 256, 0, s>>>(h.leaves.as<int>(), h.nleaves, h.c_xr.as<double4>(),
                                                         h.L.as<double2>(), nt, Lf, lsc);
    h.launches++;
  }
  if (before_l2p) FMM_CUDA(cudaStreamWaitEvent(s, before_l2p, 0));
  if (h.prm.precision == EXAFMM_MIXED) {
    auto args = [&](auto kernel) {
      kernel<<<grid_for(h.n, 128), 128, 0, s>>>((long)h.n, h.body_leaf.as<int>(), h.srcf.as<float4>(), Lf, lsc,
                                                h.out.as<double4>(), P);
    };
    switch (P) {
#define EXAFMM_L2P_CASE(p) \
  case p:                  \
    args(k_l2p_f32<p>);    \
    break;
      EXAFMM_UNROLLED_ORDERS(EXAFMM_L2P_CASE)
#undef EXAFMM_L2P_CASE
      default:
        args(k_l2p_f32<0>);
    }
  } else {
    k_l2p<<<grid_for(h.nleaves, WARPS), WARPS * 32, WARPS * nt * sizeof(double2), s>>>(
        h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(), h.c_xr.as<double4>(),
        h.src.as<double4>(), h.L.as<double2>(), h.out.as<double4>(), P);
  }
  h.launches++;
  FMM_LAUNCH();
}

}  // namespace fmm
