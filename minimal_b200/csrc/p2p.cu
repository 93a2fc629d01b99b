// Near field in FP64 (3d/kernel.h:122-150; periodic shift 3dp/kernel.h:133)
// and the direct-summation check (3d/traverse_eager.h:193-202).
//
// P2P: k_p2p_cta (target leaves of up to 256 bodies, both forms) -- one CTA
// per target leaf: the leaf's P2P list is taken in chunks of whole source
// leaves staged into shared memory, shifted into the target leaf's frame
// (the FP32 form scaled and interleaved into source pairs for packed FP32x2
// sweeps), and the threads, two targets each, sweep contiguous parts of the
// chunk; their partial sums are reduced in a fixed order.  Larger leaves take
// k_p2p / k_p2p_f32: one warp per target leaf streaming every source leaf
// through a 32-body shared-memory tile (coalesced loads, then a broadcast).
// Pairs at distance zero are skipped as in the reference.  P2P is the first
// writer of the outputs, so it stores p and F; L2P adds to them later.
#include <type_traits>

#include "fmm.cuh"

namespace fmm {

namespace {

constexpr int WARPS = 4;
constexpr int IMG_SHIFT = 26;
constexpr u32 IDX_MASK = (1u << IMG_SHIFT) - 1;

__device__ __forceinline__ void pair(double xi, double yi, double zi, const double4 s, double &pot, double &ax,
                                     double &ay, double &az) {
  const double dx = xi - s.x, dy = yi - s.y, dz = zi - s.z;
  const double r2 = dx * dx + dy * dy + dz * dz;
  const double ir = r2 > 0 ? rsqrt(r2) : 0.0;
  const double qir = s.w * ir;
  const double qir3 = qir * ir * ir;
  pot += qir;
  ax += dx * qir3;
  ay += dy * qir3;
  az += dz * qir3;
}

__global__ void __launch_bounds__(WARPS * 32) k_p2p(const int *leaves, int nleaves, const int *begin,
                                                    const int *count, const int *off, const u32 *ent,
                                                    const double4 *src, double4 *out, double cycle) {
  __shared__ double4 tile[WARPS][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * WARPS + wid;
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int tb = begin[c], tn = count[c];
  for (int t0 = 0; t0 < tn; t0 += 64) {
    const int ia = tb + t0 + lane, ib = ia + 32;
    const bool va = t0 + lane < tn, vb = t0 + lane + 32 < tn;
    const double4 A = va ? src[ia] : make_double4(0, 0, 0, 0);
    const double4 B = vb ? src[ib] : make_double4(0, 0, 0, 0);
    double pa = 0, xa = 0, ya = 0, za = 0, pb = 0, xb = 0, yb = 0, zb = 0;
    for (int e = off[c]; e < off[c + 1]; e++) {
      const u32 en = ent[e];
      const int sc = (int)(en & IDX_MASK), img = (int)(en >> IMG_SHIFT);
      const double sx = (img % 3 - 1) * cycle, sy = ((img / 3) % 3 - 1) * cycle, sz = (img / 9 - 1) * cycle;
      const double axa = A.x - sx, aya = A.y - sy, aza = A.z - sz;
      const double axb = B.x - sx, ayb = B.y - sy, azb = B.z - sz;
      const int sb = begin[sc], sn = count[sc];
      for (int s0 = 0; s0 < sn; s0 += 32) {
        const int m = min(32, sn - s0);
        __syncwarp();
        if (lane < m) tile[wid][lane] = src[sb + s0 + lane];
        __syncwarp();
        if (vb) {
          for (int k = 0; k < m; k++) {
            const double4 s = tile[wid][k];
            pair(axa, aya, aza, s, pa, xa, ya, za);
            pair(axb, ayb, azb, s, pb, xb, yb, zb);
          }
        } else {
          for (int k = 0; k < m; k++) pair(axa, aya, aza, tile[wid][k], pa, xa, ya, za);
        }
      }
    }
    if (va) out[ia] = make_double4(pa, -xa, -ya, -za);
    if (vb) out[ib] = make_double4(pb, -xb, -yb, -zb);
  }
}

// Direct sum: block = 256 targets x one chunk of sources; partial results
// are added with FP64 atomics.
constexpr int DT = 256;
constexpr int DCHUNK = 8192;

__global__ void __launch_bounds__(DT) k_direct(const double4 *tgt, long nt, const double4 *src, long ns,
                                               double4 *out, int prange, double cycle) {
  __shared__ double4 tile[DT];
  const long i = (long)blockIdx.x * DT + threadIdx.x;
  const long s0 = (long)blockIdx.y * DCHUNK, s1 = min(ns, s0 + DCHUNK);
  const double4 T = i < nt ? tgt[i] : make_double4(0, 0, 0, 0);
  double p = 0, ax = 0, ay = 0, az = 0;
  for (long b = s0; b < s1; b += DT) {
    __syncthreads();
    if (b + threadIdx.x < s1) tile[threadIdx.x] = src[b + threadIdx.x];
    __syncthreads();
    const int m = (int)min((long)DT, s1 - b);
    for (int ix = -prange; ix <= prange; ix++)
      for (int iy = -prange; iy <= prange; iy++)
        for (int iz = -prange; iz <= prange; iz++) {
          const double tx = T.x - ix * cycle, ty = T.y - iy * cycle, tz = T.z - iz * cycle;
          for (int k = 0; k < m; k++) pair(tx, ty, tz, tile[k], p, ax, ay, az);
        }
  }
  if (i < nt) {
    atomicAdd(&out[i].x, p);
    atomicAdd(&out[i].y, -ax);
    atomicAdd(&out[i].z, -ay);
    atomicAdd(&out[i].w, -az);
  }
}

// ---------------------------------------------------------------- mixed form
// Bodies as float offsets from their own leaf centre (FP64 subtraction, one
// rounding), so the pair offset dx = (xi - ci) + (ci - cj) - (xj - cj) keeps
// the bits that an FP32 copy of the absolute coordinates would lose.
__global__ void k_make_srcf(const int *leaves, int nleaves, const int *begin, const int *count, const double4 *xr,
                            const double4 *src, float4 *srcf, int *body_leaf) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nleaves) return;
  const int c = leaves[w];
  const double4 C = xr[c];
  for (int b = begin[c] + lane; b < begin[c] + count[c]; b += 32) {
    const double4 B = src[b];
    srcf[b] = make_float4((float)(B.x - C.x), (float)(B.y - C.y), (float)(B.z - C.z), (float)B.w);
    body_leaf[b] = w;
  }
}

// Error-free sum s + p = t + e (Knuth's TwoSum), accumulated as (s, e).
__device__ __forceinline__ void two_sum_acc(float &s, float &e, float p) {
  const float t = s + p;
  const float bp = t - s;
  e += (s - (t - bp)) + (p - bp);
  s = t;
}

// 1/sqrt(r2) from the hardware approximation (relative error below 2^-22),
// 0 for r2 = 0; subnormal r2 counts as 0 (flush to zero), so pairs closer
// than ~1e-19 in the leaf frame are skipped like coincident ones.
__device__ __forceinline__ float rsqrt_or_zero(float r2) {
  float y;
  asm("{\n\t.reg .pred p;\n\t"
      "setp.gt.ftz.f32 p, %1, 0f00000000;\n\t"
      "rsqrt.approx.ftz.f32 %0, %1;\n\t"
      "@!p mov.f32 %0, 0f00000000;\n\t}"
      : "=f"(y)
      : "f"(r2));
  return y;
}

// r2 floor of the unchecked pair, in units where the target leaf's radius is
// in [1, 2): 2^-64, far below the FP32 resolution of that frame (~2^-20), so
// it changes no resolved pair; two distinct bodies whose FP32 offsets
// coincide get 1/r = 2^32 instead of an infinity, and q / r^3 stays finite
// for |q| < 2^32.
constexpr float NEAR_TINY = 5.421010862427522e-20f;  // 2^-64

// CHECK: pairs at distance zero contribute nothing (3d/kernel.h:131); the
// unchecked form serves source leaves other than the target's own, where a
// zero offset can only come from FP32 rounding.
template <bool CHECK = true>
__device__ __forceinline__ void pair_f32(float xi, float yi, float zi, const float4 s, float &pot, float &ax,
                                         float &ay, float &az) {
  const float dx = xi - s.x, dy = yi - s.y, dz = zi - s.z;
  float ir;
  if constexpr (CHECK) {
    ir = rsqrt_or_zero(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
  } else {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, NEAR_TINY)));
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(ir) : "f"(r2));
  }
  const float qir = s.w * ir;
  const float qir3 = qir * ir * ir;
  pot += qir;
  ax = fmaf(dx, qir3, ax);
  ay = fmaf(dy, qir3, ay);
  az = fmaf(dz, qir3, az);
}

// ---- packed FP32x2 arithmetic (sm_100a): two FP32 lanes per 64-bit value,
// one instruction for both.  The packed near field evaluates one target
// against two sources at a time, with the sources staged in pairs:
// slot 2p = {x_2p, x_2p+1, y_2p, y_2p+1}, slot 2p+1 = {z.., z.., q.., q..}.
typedef unsigned long long f2x;
__device__ __forceinline__ f2x pk2(float a, float b) {
  f2x r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void upk2(f2x v, float &a, float &b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ f2x sub2(f2x a, f2x b) {
  f2x r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2x add2(f2x a, f2x b) {
  f2x r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2x mul2(f2x a, f2x b) {
  f2x r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c) {
  f2x r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// A staged source that adds nothing: zero charge, far from every target.
constexpr float NEAR_DUMMY = 1e15f;

// One target (X, Y, Z = the coordinate in both lanes) against a staged
// source pair (sx, sy from the first slot, sz, sq from the second); the same
// arithmetic as pair_f32 in each lane.
template <bool CHECK>
__device__ __forceinline__ void pair_x2(f2x X, f2x Y, f2x Z, f2x sx, f2x sy, f2x sz, f2x sq, f2x &pot, f2x &ax,
                                        f2x &ay, f2x &az) {
  const f2x dx = sub2(X, sx), dy = sub2(Y, sy), dz = sub2(Z, sz);
  float r0, r1;
  f2x ir;
  if constexpr (CHECK) {
    upk2(fma2(dx, dx, fma2(dy, dy, mul2(dz, dz))), r0, r1);
    ir = pk2(rsqrt_or_zero(r0), rsqrt_or_zero(r1));
  } else {
    const f2x tiny = pk2(NEAR_TINY, NEAR_TINY);
    upk2(fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, tiny))), r0, r1);
    ir = pk2(rsqrt_approx(r0), rsqrt_approx(r1));
  }
  const f2x qir = mul2(sq, ir);
  const f2x qir3 = mul2(qir, mul2(ir, ir));
  pot = add2(pot, qir);
  ax = fma2(dx, qir3, ax);
  ay = fma2(dy, qir3, ay);
  az = fma2(dz, qir3, az);
}

// FP32 P2P: same mapping as k_p2p; FP32 partial sums per source leaf, then a
// compensated (TwoSum) accumulation per target across the source leaves.
__global__ void __launch_bounds__(WARPS * 32) k_p2p_f32(const int *leaves, int nleaves, const int *begin,
                                                        const int *count, const int *off, const u32 *ent,
                                                        const double4 *xr, const float4 *srcf, double4 *out,
                                                        double cycle) {
  __shared__ float4 tile[WARPS][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * WARPS + wid;
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int tb = begin[c], tn = count[c];
  const double4 CA = xr[c];
  for (int t0 = 0; t0 < tn; t0 += 64) {
    const int ia = tb + t0 + lane, ib = ia + 32;
    const bool va = t0 + lane < tn, vb = t0 + lane + 32 < tn;
    const float4 A = va ? srcf[ia] : make_float4(0, 0, 0, 0);
    const float4 B = vb ? srcf[ib] : make_float4(0, 0, 0, 0);
    float sa[4] = {0, 0, 0, 0}, ea[4] = {0, 0, 0, 0}, sb[4] = {0, 0, 0, 0}, eb[4] = {0, 0, 0, 0};
    for (int e = off[c]; e < off[c + 1]; e++) {
      const u32 en = ent[e];
      const int sc = (int)(en & IDX_MASK), img = (int)(en >> IMG_SHIFT);
      const double4 CB = xr[sc];
      const float ox = (float)(CA.x - CB.x - (img % 3 - 1) * cycle);
      const float oy = (float)(CA.y - CB.y - ((img / 3) % 3 - 1) * cycle);
      const float oz = (float)(CA.z - CB.z - (img / 9 - 1) * cycle);
      const float xa = A.x + ox, ya = A.y + oy, za = A.z + oz;
      const float xb = B.x + ox, yb = B.y + oy, zb = B.z + oz;
      float pa = 0, qa = 0, ra = 0, ta = 0, pb = 0, qb = 0, rb = 0, tb2 = 0;
      const int sbeg = begin[sc], sn = count[sc];
      for (int s0 = 0; s0 < sn; s0 += 32) {
        const int m = min(32, sn - s0);
        __syncwarp();
        if (lane < m) tile[wid][lane] = srcf[sbeg + s0 + lane];
        __syncwarp();
        if (vb) {
          for (int k = 0; k < m; k++) {
            const float4 s = tile[wid][k];
            pair_f32(xa, ya, za, s, pa, qa, ra, ta);
            pair_f32(xb, yb, zb, s, pb, qb, rb, tb2);
          }
        } else {
          for (int k = 0; k < m; k++) pair_f32(xa, ya, za, tile[wid][k], pa, qa, ra, ta);
        }
      }
      two_sum_acc(sa[0], ea[0], pa);
      two_sum_acc(sa[1], ea[1], qa);
      two_sum_acc(sa[2], ea[2], ra);
      two_sum_acc(sa[3], ea[3], ta);
      two_sum_acc(sb[0], eb[0], pb);
      two_sum_acc(sb[1], eb[1], qb);
      two_sum_acc(sb[2], eb[2], rb);
      two_sum_acc(sb[3], eb[3], tb2);
    }
    if (va)
      out[ia] = make_double4((double)sa[0] + ea[0], -((double)sa[1] + ea[1]), -((double)sa[2] + ea[2]),
                             -((double)sa[3] + ea[3]));
    if (vb)
      out[ib] = make_double4((double)sb[0] + eb[0], -((double)sb[1] + eb[1]), -((double)sb[2] + eb[2]),
                             -((double)sb[3] + eb[3]));
  }
}

// ------------------------------------------------ CTA-per-leaf near field
// One CTA per target leaf.  The P2P list is taken in chunks of whole source
// leaves (up to 32) that fit the staging buffer.  Every warp reads the
// metadata of the chunk's leaves lane-parallel (lane k: leaf k's first body,
// size and shift into the target frame) and scans the sizes; the warps then
// copy the chunk's bodies into shared memory, already shifted into the
// target's frame, in 32-body blocks (a body finds its leaf with two warp
// votes), so the inner loop is a plain (target, source) sweep.  Thread t
// takes the targets i and i+H with i = t % H, H = ceil(tn/2), and the G-th
// part of the staged sources, g = t / H, G = floor(128/H): for leaves of 20-64
// bodies nearly all 128 threads are busy, and each staged source is read once
// per two pairs.  Partial sums of the G source parts are combined in a fixed
// order at the end.  Target leaves up to 256 bodies (ncrit <= 256) use this
// kernel, larger ones the warp kernels above.
//
// FP32 form: coordinates are scaled by a power of two (exact) so that the
// target leaf's radius is in [1, 2); the target leaf's own bodies (its list
// always holds it: the acceptance test never accepts a cell with itself) go
// first, in slots [0, tn) of the first chunk, and only they are swept with
// the zero-distance check; every group takes its share of both parts, so the
// warps stay converged.  FP64 form: list order, every pair checked.
constexpr int CT = 128;           // threads per CTA
// bodies staged at once (the source tile): a template parameter, chosen at
// run time among 1024, 1536 and 2048 (exafmm_b200_set_tile / the
// autotuner); the defaults, FP32 1536 (7 CTAs per SM, register-bound) and
// FP64 1024 (5 CTAs per SM), were tuned on B200 at 1M uniform bodies
template <bool F32>
constexpr int ct_cap() { return F32 ? 1536 : 1024; }
constexpr int CT_MAXTGT = 256;    // target-leaf bodies: two per thread
constexpr int CT_TPT = 2;         // targets per thread (register blocking)
constexpr int CT_BLOCK = 256;     // sources summed in FP32 before one compensated addition
// 32-body blocks a warp loads before storing them (register-bound)
template <bool F32>
constexpr int ct_unroll() { return F32 ? 2 : 1; }

template <bool F32>
struct NearBody;
template <>
struct NearBody<false> {
  typedef double4 T;
  typedef double R;
};
template <>
struct NearBody<true> {
  typedef float4 T;
  typedef float R;
};

template <bool F32, int CAP>
__global__ void __launch_bounds__(CT, F32 ? 7 : 5) k_p2p_cta(const int *leaves, const int *begin, const int *count,
                                                const int *off, const u32 *ent, const double4 *xr,
                                                const typename NearBody<F32>::T *bodies, double4 *out,
                                                double cycle) {
  typedef typename NearBody<F32>::T BT;
  typedef typename NearBody<F32>::R RT;
  constexpr int CT_UNROLL = ct_unroll<F32>();
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char stage_raw[];  // CAP bodies
  BT *stage = (BT *)stage_raw;
  double *red = (double *)stage_raw;  // after the last chunk: CT * CT_TPT * 4 partial sums
  const int c = leaves[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int tb = begin[c], tn = count[c];
  const int H = (tn + CT_TPT - 1) / CT_TPT, G = CT / H;
  const int i = tid % H, g = tid / H;
  // x / G for the FP32 form's part bounds of every chunk, without an integer
  // division: a float estimate (x < 2^24) corrected by one step
  const float rG = 1.0f / (float)G;
  auto divG = [&](int x) {
    int q = (int)((float)x * rG);
    q -= q * G > x;
    q += (q + 1) * G <= x;
    return q;
  };
  const bool act = g < G;
  const double4 CA = xr[c];
  const int sexp = CA.w > 0 ? max(-100, min(100, ilogb(CA.w))) : 0;
  const float scale = F32 ? exp2f((float)-sexp) : 1.0f;  // FP32: R * scale in [1, 2)
  BT A[CT_TPT];
#pragma unroll
  for (int u = 0; u < CT_TPT; u++) {
    A[u] = act && i + u * H < tn ? bodies[tb + i + u * H] : BT{};
    if constexpr (F32) {
      A[u].x *= scale;
      A[u].y *= scale;
      A[u].z *= scale;
    }
  }
  // accumulators: FP64 form plain; FP32 form compensated (s, e) per quantity
  RT sacc[CT_TPT][4], eacc[CT_TPT][4];
#pragma unroll
  for (int u = 0; u < CT_TPT; u++)
#pragma unroll
    for (int q = 0; q < 4; q++) sacc[u][q] = eacc[u][q] = 0;
  const int eb = off[c], ee = off[c + 1];
  // slots [0, pre) of the first chunk: the target leaf itself (FP32), padded
  // to an even count (the FP32 stage holds sources in pairs)
  int pre = F32 ? tn + (tn & 1) : 0;
  for (int e0i = eb; e0i < ee;) {
    // lane k: source leaf k of the chunk candidates
    const int cand = min(32, ee - e0i);
    // FP32: the shift (ox, oy, oz) from the source leaf's frame into the
    // target leaf's, scaled; FP64: absolute positions, shifted by the
    // periodic image `img` (the shift is formed per body from it)
    int n = 0, base = 0, img = 13;
    bool self = false;  // FP32: the target leaf's own entry (staged first, so here of size 0)
    float ox = 0, oy = 0, oz = 0;
    if (lane < cand) {
      const u32 en = ent[e0i + lane];
      const int sc = (int)(en & IDX_MASK);
      img = (int)(en >> IMG_SHIFT);
      n = count[sc];
      base = begin[sc];
      if constexpr (F32) {
        self = sc == c && img == 13;
        if (self) n = 0;
        const double sx = (img % 3 - 1) * cycle, sy = ((img / 3) % 3 - 1) * cycle, sz = (img / 9 - 1) * cycle;
        const double4 CB = xr[sc];
        ox = (float)(CA.x - CB.x - sx) * scale;  // exact: scale is a power of two
        oy = (float)(CA.y - CB.y - sy) * scale;
        oz = (float)(CA.z - CB.z - sz) * scale;
      }
    }
    int inc = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, inc, o);
      if (lane >= o) inc += t;
    }
    inc += pre;
    // the running sums grow, so the leaves that fit are a prefix (at least
    // one: no leaf exceeds the buffer less the target leaf)
    const int nl = __popc(__ballot_sync(FULL, lane < cand && inc <= CAP));
    const int T = __shfl_sync(FULL, inc, nl - 1);
    const int start = inc - n;  // first staging slot of leaf `lane`
    base -= start;              // body index = base + staging slot
    const bool inchunk = lane < nl;
    // the size-0 self entry shares its start with the next leaf
    const unsigned zm = __ballot_sync(FULL, inchunk && self);
    const int zs = zm ? __shfl_sync(FULL, start, __ffs(zm) - 1) : -1;
    __syncthreads();  // the previous chunk's sweep is done with the buffer
    if constexpr (F32) {
      for (int pp = tid; 2 * pp < pre; pp += CT) {  // the target leaf, in slots [0, tn), in pairs
        float4 a = bodies[tb + 2 * pp], b = make_float4(NEAR_DUMMY, NEAR_DUMMY, NEAR_DUMMY, 0.f);
        a.x *= scale;
        a.y *= scale;
        a.z *= scale;
        if (2 * pp + 1 < tn) {
          b = bodies[tb + 2 * pp + 1];
          b.x *= scale;
          b.y *= scale;
          b.z *= scale;
        }
        stage[2 * pp] = make_float4(a.x, b.x, a.y, b.y);
        stage[2 * pp + 1] = make_float4(a.z, b.z, a.w, b.w);
      }
    }
    for (int j0 = pre + wid * 32; j0 < T; j0 += CT * CT_UNROLL) {
      BT v[CT_UNROLL];
      int kk[CT_UNROLL];
#pragma unroll
      for (int u = 0; u < CT_UNROLL; u++) {
        const int jb = j0 + u * CT, j = jb + lane;
        // leaf of slot j: the last leaf starting at or before jb, plus the
        // leaves starting in (jb, j] (a size-0 leaf counts as well: the
        // leaf after it starts at the same slot)
        const int k0 = __popc(__ballot_sync(FULL, inchunk && start <= jb)) - 1;
        const unsigned st = __reduce_or_sync(FULL, inchunk && start > jb && start < jb + 32 ? 1u << (start - jb) : 0u);
        const int k = k0 + __popc(st & (FULL >> (31 - lane))) + (zs > jb && zs <= j);
        kk[u] = k;
        const int bk = __shfl_sync(FULL, base, k);
        if (j < T) v[u] = bodies[bk + j];
      }
#pragma unroll
      for (int u = 0; u < CT_UNROLL; u++) {
        const int j = j0 + u * CT + lane;
        RT sx, sy, sz;
        if constexpr (F32) {
          sx = __shfl_sync(FULL, ox, kk[u]);
          sy = __shfl_sync(FULL, oy, kk[u]);
          sz = __shfl_sync(FULL, oz, kk[u]);
        } else {
          const int im = __shfl_sync(FULL, img, kk[u]);
          sx = -(im % 3 - 1) * cycle;
          sy = -((im / 3) % 3 - 1) * cycle;
          sz = -(im / 9 - 1) * cycle;
        }
        if constexpr (F32) {  // into the target frame, scaled (exact); stored in source pairs
          float4 t = make_float4(NEAR_DUMMY, NEAR_DUMMY, NEAR_DUMMY, 0.f);
          if (j < T) t = make_float4(fmaf(v[u].x, scale, -sx), fmaf(v[u].y, scale, -sy), fmaf(v[u].z, scale, -sz), v[u].w);
          const float4 o = make_float4(__shfl_xor_sync(FULL, t.x, 1), __shfl_xor_sync(FULL, t.y, 1),
                                       __shfl_xor_sync(FULL, t.z, 1), __shfl_xor_sync(FULL, t.w, 1));
          if (j < T) {
            if ((j & 1) == 0) {  // the pair's first slot (its partner, or a dummy past the end)
              stage[j] = make_float4(t.x, o.x, t.y, o.y);
              if (j + 1 == T) stage[j + 1] = make_float4(t.z, NEAR_DUMMY, t.w, 0.f);
            } else {
              stage[j] = make_float4(o.z, t.z, o.w, t.w);
            }
          }
        } else if (j < T) {
          BT t;
          t.x = v[u].x - sx;
          t.y = v[u].y - sy;
          t.z = v[u].z - sz;
          t.w = v[u].w;
          stage[j] = t;
        }
      }
    }
    __syncthreads();
    if (act) {
      // FP64: a slot range, CT_BLOCK sources at a time, four per iteration
      auto sweep = [&](int from, int to, auto check) {
        constexpr bool CHECK = decltype(check)::value;
        const BT *sp = stage + from;
        for (int c0 = from; c0 < to; c0 += CT_BLOCK) {
          RT p[CT_TPT][4];
#pragma unroll
          for (int u = 0; u < CT_TPT; u++)
#pragma unroll
            for (int q = 0; q < 4; q++) p[u][q] = 0;
          const int cend = min(to, c0 + CT_BLOCK);
          int cs = c0;
          auto acc = [&](const BT &sv) {
#pragma unroll
            for (int u = 0; u < CT_TPT; u++) {
              if constexpr (F32) pair_f32<CHECK>(A[u].x, A[u].y, A[u].z, sv, p[u][0], p[u][1], p[u][2], p[u][3]);
              else pair(A[u].x, A[u].y, A[u].z, sv, p[u][0], p[u][1], p[u][2], p[u][3]);
            }
          };
          for (; cs + 4 <= cend; cs += 4) {
            const BT s0 = sp[0], s1 = sp[1], s2 = sp[2], s3 = sp[3];
            sp += 4;
            acc(s0);
            acc(s1);
            acc(s2);
            acc(s3);
          }
          for (; cs < cend; cs++) {
            const BT s0 = sp[0];
            sp += 1;
            acc(s0);
          }
#pragma unroll
          for (int u = 0; u < CT_TPT; u++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
              if constexpr (F32) two_sum_acc(sacc[u][q], eacc[u][q], p[u][q]);  // compensated per block
              else sacc[u][q] += p[u][q];
            }
        }
      };
      if constexpr (F32) {
        // packed FP32x2: one target against a staged source pair per step;
        // the target leaf's own pairs (a few per thread) with the
        // zero-distance check, summed into the first block of the others
        // (without the check).  Lane partial sums are combined at each
        // block's compensated addition.
        f2x X[CT_TPT], Y[CT_TPT], Z[CT_TPT], acc[CT_TPT][4];
#pragma unroll
        for (int u = 0; u < CT_TPT; u++) {
          X[u] = pk2(A[u].x, A[u].x);
          Y[u] = pk2(A[u].y, A[u].y);
          Z[u] = pk2(A[u].z, A[u].z);
#pragma unroll
          for (int q = 0; q < 4; q++) acc[u][q] = 0ull;
        }
        const f2x *sp2 = (const f2x *)stage;  // pair p: sp2[4p .. 4p + 3] = x, y, z, q pairs
        auto step = [&](int pp, auto check) {
          constexpr bool CHECK = decltype(check)::value;
          const ulonglong2 s0 = ((const ulonglong2 *)sp2)[2 * pp], s1 = ((const ulonglong2 *)sp2)[2 * pp + 1];
#pragma unroll
          for (int u = 0; u < CT_TPT; u++)
            pair_x2<CHECK>(X[u], Y[u], Z[u], s0.x, s0.y, s1.x, s1.y, acc[u][0], acc[u][1], acc[u][2], acc[u][3]);
        };
        auto flush = [&]() {  // one compensated addition per block
#pragma unroll
          for (int u = 0; u < CT_TPT; u++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
              float lo, hi;
              upk2(acc[u][q], lo, hi);
              two_sum_acc(sacc[u][q], eacc[u][q], lo + hi);
              acc[u][q] = 0ull;
            }
        };
        const int nps = pre / 2, npt = (T + 1) / 2;  // pairs of the target leaf, of the chunk
        for (int pp = divG(g * nps), pe = divG((g + 1) * nps); pp < pe; pp++) step(pp, std::true_type{});
        const int rest = npt - nps, from = nps + divG(g * rest), to = nps + divG((g + 1) * rest);
        for (int c0 = from; c0 < to; c0 += CT_BLOCK / 2) {
          const int cend = min(to, c0 + CT_BLOCK / 2);
          int pp = c0;
          for (; pp + 2 <= cend; pp += 2) {
            step(pp, std::false_type{});
            step(pp + 1, std::false_type{});
          }
          if (pp < cend) step(pp, std::false_type{});
          flush();
        }
        if (from == to && nps) flush();  // only the target leaf's pairs
      } else {
        sweep(g * T / G, (g + 1) * T / G, std::true_type{});
      }
    }
    e0i += nl;
    pre = 0;
  }
  __syncthreads();
  if (act) {
#pragma unroll
    for (int u = 0; u < CT_TPT; u++)
#pragma unroll
      for (int q = 0; q < 4; q++) red[(g * CT_TPT * H + i + u * H) * 4 + q] = (double)sacc[u][q] + (double)eacc[u][q];
  }
  __syncthreads();
  // a target leaf holds up to CT_TPT * CT bodies: every thread writes
  // targets tid, tid + CT, ...
  for (int t = tid; t < tn; t += CT) {
    double r[4] = {0, 0, 0, 0};
    for (int gg = 0; gg < G; gg++)
#pragma unroll
      for (int q = 0; q < 4; q++) r[q] += red[(gg * CT_TPT * H + t) * 4 + q];
    const double s1 = scale, s2 = s1 * s1;  // back to the input units
    out[tb + t] = make_double4(r[0] * s1, -r[1] * s2, -r[2] * s2, -r[3] * s2);
  }
}

}  // namespace

// The FP32 leaf-relative copy of the bodies (mixed form) and each body's
// leaf slot, once per tree (and charge set).
void make_srcf(Handle &h) {
  if (h.srcf_ready) return;
  h.srcf.need((size_t)h.n * sizeof(float4));
  h.body_leaf.need((size_t)h.n * sizeof(int));
  k_make_srcf<<<grid_for((long)h.nleaves * 32, 256), 256, 0, h.stream>>>(
      h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(), h.c_xr.as<double4>(),
      h.src.as<double4>(), h.srcf.as<float4>(), h.body_leaf.as<int>());
  h.launches++;
  FMM_LAUNCH();
  h.srcf_ready = true;
}

// The near-field CTA kernel with source tile `cap` (1024, 1536 or 2048).
template <bool F32, class... A>
void launch_p2p_cta(int cap, int nleaves, cudaStream_t s, A... args) {
  typedef typename NearBody<F32>::T BT;
  switch (cap) {
    case 1024: k_p2p_cta<F32, 1024><<<nleaves, CT, 1024 * sizeof(BT), s>>>(args...); break;
    case 2048: k_p2p_cta<F32, 2048><<<nleaves, CT, 2048 * sizeof(BT), s>>>(args...); break;
    default: k_p2p_cta<F32, 1536><<<nleaves, CT, 1536 * sizeof(BT), s>>>(args...);
  }
}

template <bool F32>
void set_p2p_attributes() {
  typedef typename NearBody<F32>::T BT;
  cudaFuncSetAttribute(k_p2p_cta<F32, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, 1024 * (int)sizeof(BT));
  cudaFuncSetAttribute(k_p2p_cta<F32, 1536>, cudaFuncAttributeMaxDynamicSharedMemorySize, 1536 * (int)sizeof(BT));
  cudaFuncSetAttribute(k_p2p_cta<F32, 2048>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2048 * (int)sizeof(BT));
}

void p2p_set_attributes() {
  set_p2p_attributes<false>();
  set_p2p_attributes<true>();
}

int p2p_tile(const Handle &h) {
  if (h.tile_p2p_stage > 0) return h.tile_p2p_stage;
  return h.prm.precision == EXAFMM_MIXED ? ct_cap<true>() : ct_cap<false>();
}

void p2p_pass(Handle &h, cudaStream_t s) {
  if (h.prm.dim == 2) return p2p_pass_2d(h, s);
  h.out.need((size_t)h.n * sizeof(double4));
  const double cyc = h.prm.images ? h.prm.cycle : 0.0;
  const bool cta = h.prm.ncrit <= CT_MAXTGT;  // every leaf fits two targets per thread and the buffer
  if (h.prm.precision == EXAFMM_MIXED) {
    if (s != h.stream && !h.srcf_ready) throw Error{EXAFMM_ERR_STATE, "near field on a side stream before its sources"};
    make_srcf(h);
    if (cta)
      launch_p2p_cta<true>(p2p_tile(h), h.nleaves, s, h.leaves.as<int>(), h.c_begin.as<int>(), h.c_count.as<int>(),
                           h.p2p_off.as<int>(), h.p2p_ent.as<u32>(), h.c_xr.as<double4>(), h.srcf.as<float4>(),
                           h.out.as<double4>(), cyc);
    else
      k_p2p_f32<<<grid_for(h.nleaves, WARPS), WARPS * 32, 0, s>>>(
          h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(), h.p2p_off.as<int>(),
          h.p2p_ent.as<u32>(), h.c_xr.as<double4>(), h.srcf.as<float4>(), h.out.as<double4>(), cyc);
    h.launches++;
    FMM_LAUNCH();
    return;
  }
  if (cta)
    launch_p2p_cta<false>(p2p_tile(h), h.nleaves, s, h.leaves.as<int>(), h.c_begin.as<int>(), h.c_count.as<int>(),
                          h.p2p_off.as<int>(), h.p2p_ent.as<u32>(), h.c_xr.as<double4>(), h.src.as<double4>(),
                          h.out.as<double4>(), cyc);
  else
    k_p2p<<<grid_for(h.nleaves, WARPS), WARPS * 32, 0, s>>>(
        h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(), h.p2p_off.as<int>(),
        h.p2p_ent.as<u32>(), h.src.as<double4>(), h.out.as<double4>(), cyc);
  h.launches++;
  FMM_LAUNCH();
}

void direct_sum(Handle &h, double4 *targets, double4 *out, long nt) {
  dim3 grid(grid_for(nt, DT), grid_for(h.n, DCHUNK));
  int prange = 0;  // periodic images: r = sum_{i < images} 3^i (3dp/traverse_eager.h:139-142)
  for (int i = 0, p3 = 1; i < h.prm.images; i++, p3 *= 3) prange += p3;
  k_direct<<<grid, DT, 0, h.stream>>>(targets, nt, h.src.as<double4>(), h.n, out, prange,
                                      h.prm.images ? h.prm.cycle : 0.0);
  h.launches++;
  FMM_LAUNCH();
}

}  // namespace fmm
