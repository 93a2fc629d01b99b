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

// P2M (3d/kernel.h:187-202): M[n][m] += q * Y_n^m(rho, alpha, -beta).
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
  for (int b = begin[c]; b < begin[c] + count[c]; b++) {
    const double4 B = src[b];
    const Sph g = sph_of(B.x - C.x, B.y - C.y, B.z - C.z);
    if (lane < P) {
      regular_column(lane, P, g.r, g, cconj(g.e), [&](int n, double2 Y, double2) {
        double2 &a = acc[tri(n) + lane];
        a.x += B.w * Y.x;
        a.y += B.w * Y.y;
      });
    }
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
  for (int b = begin[c]; b < begin[c] + count[c]; b++) {
    const double4 B = src[b];
    const Sph g = sph_of(B.x - C.x, B.y - C.y, B.z - C.z);
    double pot = 0, s0 = 0, s1 = 0, s2 = 0;
    if (lane < P) {
      const int m = lane;
      const double w2 = m == 0 ? 1.0 : 2.0;
      regular_column(m, P, g.r, g, g.e, [&](int n, double2 Y, double2 dY) {
        const double2 l = Lc[tri(n) + m];
        const double re = l.x * Y.x - l.y * Y.y;        // Re(L Y)
        const double red = l.x * dY.x - l.y * dY.y;     // Re(L dY)
        const double rei = -(l.x * Y.y + l.y * Y.x);    // Re(L Y i)
        pot += w2 * re;
        if (g.r != 0) s0 += w2 * re / g.r * n;
        s1 += w2 * red;
        s2 += w2 * rei * m;
      });
    }
    for (int o = 16; o > 0; o >>= 1) {
      pot += __shfl_xor_sync(0xffffffffu, pot, o);
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
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
