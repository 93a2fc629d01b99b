// Upward and downward passes in FP64: P2M at the leaves, M2M bottom-up one
// level per launch, L2L top-down one level per launch, L2P at the leaves
// (3d/kernel.h:187-323; traversal order 3d/traverse_eager.h:127-190, which
// the level-synchronous launches respect: a cell's children are complete
// before its M2M, and its parent's local is final before its L2L).
//
// Mapping: one warp per cell.  Harmonic columns are built by lane = order m
// into shared memory; the translations then give each lane whole output
// coefficients (j,k), accumulated in a warp-private shared buffer.
#include "fmm.cuh"
#include "harmonics.cuh"

namespace fmm {

namespace {

constexpr int WARPS = 4;

// Y(deg, o) for any sign of o from the m>=0 table.
__device__ __forceinline__ double2 ylook(const double2 *Y, int n, int o) {
  return o >= 0 ? Y[tri(n) + o] : cconj(Y[tri(n) - o]);
}

__device__ __forceinline__ int sgn(int n) { return (n & 1) ? -1 : 1; }

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
__global__ void __launch_bounds__(WARPS * 32) k_m2m(int c0, int c1, const int *child, const int *nchild,
                                                    const double4 *xr, double2 *M, int P) {
  extern __shared__ double2 sh[];
  const int nt = tri(P);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = c0 + blockIdx.x * WARPS + wid;
  if (c >= c1) return;
  const int nk = nchild[c];
  if (nk == 0) return;
  double2 *acc = sh + wid * 3 * nt, *Y = acc + nt, *Mc = Y + nt;
  for (int k = lane; k < nt; k += 32) acc[k] = make_double2(0, 0);
  const double4 X = xr[c];
  for (int q = child[c]; q < child[c] + nk; q++) {
    const double4 K = xr[q];
    const Sph g = sph_of(X.x - K.x, X.y - K.y, X.z - K.z);
    __syncwarp();
    if (lane < P)
      regular_column(lane, P, g.r, g, g.e, [&](int n, double2 v, double2) { Y[tri(n) + lane] = v; });
    for (int k = lane; k < nt; k += 32) Mc[k] = M[(long)q * nt + k];
    __syncwarp();
    for (int o = lane; o < nt; o += 32) {
      int j = 0;
      while (tri(j + 1) <= o) j++;
      const int k = o - tri(j);
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
      acc[o].x += s.x;
      acc[o].y += s.y;
    }
  }
  __syncwarp();
  for (int k = lane; k < nt; k += 32) M[(long)c * nt + k] = acc[k];
}

// L2L (3d/kernel.h:262-291), one warp per child at one level: the child
// pulls its parent's local expansion.
__global__ void __launch_bounds__(WARPS * 32) k_l2l(int c0, int c1, const int *parent, const double4 *xr,
                                                    double2 *L, int P) {
  extern __shared__ double2 sh[];
  const int nt = tri(P);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = c0 + blockIdx.x * WARPS + wid;
  if (c >= c1) return;
  const int pa = parent[c];
  double2 *Y = sh + wid * 2 * nt, *Lp = Y + nt;
  const double4 X = xr[c], Q = xr[pa];
  const Sph g = sph_of(X.x - Q.x, X.y - Q.y, X.z - Q.z);
  if (lane < P)
    regular_column(lane, P, g.r, g, g.e, [&](int n, double2 v, double2) { Y[tri(n) + lane] = v; });
  for (int k = lane; k < nt; k += 32) Lp[k] = L[(long)pa * nt + k];
  __syncwarp();
  for (int o = lane; o < nt; o += 32) {
    int j = 0;
    while (tri(j + 1) <= o) j++;
    const int k = o - tri(j);
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
    double2 &d = L[(long)c * nt + o];
    d.x += s.x;
    d.y += s.y;
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
      s0 += w2 * re * n;
      s1 += w2 * red;
      s2 += w2 * rei * m;
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

void expansions_set_attributes() {
  double rc[2 * EXAFMM_MAX_P + 4];
  rc[0] = 0;
  for (int k = 1; k < 2 * EXAFMM_MAX_P + 4; k++) rc[k] = 1.0 / k;
  FMM_CUDA(cudaMemcpyToSymbol(c_recip, rc, sizeof(rc)));
  cudaFuncSetAttribute(k_p2m, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_m2m, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_l2l, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_l2p, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

void upward_pass(Handle &h) {
  cudaStream_t s = h.stream;
  const int P = h.prm.P, nt = tri(P);
  h.M.need((size_t)h.ncells * nt * sizeof(double2));
  h.L.need((size_t)h.ncells * nt * sizeof(double2));
  k_p2m<<<grid_for(h.nleaves, WARPS), WARPS * 32, WARPS * nt * sizeof(double2), s>>>(
      h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(), h.c_xr.as<double4>(),
      h.src.as<double4>(), h.M.as<double2>(), P);
  h.launches++;
  FMM_LAUNCH();
  for (int l = h.depth - 1; l >= 0; l--) {
    const int c0 = h.level_base[l], c1 = h.level_base[l + 1];
    if (c1 <= c0) continue;
    k_m2m<<<grid_for(c1 - c0, WARPS), WARPS * 32, WARPS * 3 * nt * sizeof(double2), s>>>(
        c0, c1, h.c_child.as<int>(), h.c_nchild.as<int>(), h.c_xr.as<double4>(), h.M.as<double2>(), P);
    h.launches++;
    FMM_LAUNCH();
  }
}

void downward_pass(Handle &h) {
  cudaStream_t s = h.stream;
  const int P = h.prm.P, nt = tri(P);
  for (int l = 1; l <= h.depth; l++) {
    const int c0 = h.level_base[l], c1 = h.level_base[l + 1];
    if (c1 <= c0) continue;
    k_l2l<<<grid_for(c1 - c0, WARPS), WARPS * 32, WARPS * 2 * nt * sizeof(double2), s>>>(
        c0, c1, h.c_parent.as<int>(), h.c_xr.as<double4>(), h.L.as<double2>(), P);
    h.launches++;
    FMM_LAUNCH();
  }
  k_l2p<<<grid_for(h.nleaves, WARPS), WARPS * 32, WARPS * nt * sizeof(double2), s>>>(
      h.leaves.as<int>(), h.nleaves, h.c_begin.as<int>(), h.c_count.as<int>(), h.c_xr.as<double4>(),
      h.src.as<double4>(), h.L.as<double2>(), h.out.as<double4>(), P);
  h.launches++;
  FMM_LAUNCH();
}

}  // namespace fmm
