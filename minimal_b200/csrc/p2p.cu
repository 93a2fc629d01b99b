// Near field in FP64 (3d/kernel.h:122-150; periodic shift 3dp/kernel.h:133)
// and the direct-summation check (3d/traverse_eager.h:193-202).
//
// P2P: one warp per target leaf; each lane keeps up to two target bodies in
// registers while the warp streams every source leaf of the target's P2P
// list through a 32-body shared-memory tile (coalesced 32-byte loads, all
// lanes then read the same body: a broadcast).  Pairs at distance zero are
// skipped as in the reference.  P2P is the first writer of the outputs, so it
// stores p and F; L2P adds to them later.
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
                                               double4 *out) {
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
    for (int k = 0; k < m; k++) pair(T.x, T.y, T.z, tile[k], p, ax, ay, az);
  }
  if (i < nt) {
    atomicAdd(&out[i].x, p);
    atomicAdd(&out[i].y, -ax);
    atomicAdd(&out[i].z, -ay);
    atomicAdd(&out[i].w, -az);
  }
}

}  // namespace

void p2p_pass(Handle &h) {
  h.out.need((size_t)h.n * sizeof(double4));
  k_p2p<<<grid_for(h.nleaves, WARPS), WARPS * 32, 0, h.stream>>>(
      h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(), h.p2p_off.as<int>(),
      h.p2p_ent.as<u32>(), h.src.as<double4>(), h.out.as<double4>(), h.prm.images ? h.prm.cycle : 0.0);
  h.launches++;
  FMM_LAUNCH();
}

void direct_sum(Handle &h, double4 *targets, double4 *out, long nt) {
  dim3 grid(grid_for(nt, DT), grid_for(h.n, DCHUNK));
  k_direct<<<grid, DT, 0, h.stream>>>(targets, nt, h.src.as<double4>(), h.n, out);
  h.launches++;
  FMM_LAUNCH();
}

}  // namespace fmm
