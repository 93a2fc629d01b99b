// M2L in FP64 (3d/kernel.h:233-260; periodic shift 3dp/kernel.h:200).
//
//   L_j^k += sum_{n,m} A_n^m s(j,k,m) Z_{j+n}^{m-k}(Xi - Xj - iX*cycle)
// with A_n^m = M_n^m (m >= 0) or conj(M_n^{-m}) (m < 0), and the sign
// s = (-1)^j for m < 0, (-1)^(j+m) for 0 <= m <= k, (-1)^(j+k) for m > k.
// The reference forms the irregular harmonics only up to degree P-1 (evalLocal
// loops n < P; the rest of its 4P^2 table stays zero), so only n <= P-1-j
// contributes -- the triangular truncation is kept here by bounding n.
//
// Target-centric: one warp owns one target cell and walks its M2L list; per
// source the lanes build the irregular columns (lane = m) in shared memory,
// then each lane accumulates whole output coefficients.  L is stored, not
// added: M2L is the first writer of the local expansions.
#include "fmm.cuh"
#include "harmonics.cuh"

namespace fmm {

namespace {

constexpr int WARPS = 4;
constexpr int IMG_SHIFT = 26;
constexpr u32 IDX_MASK = (1u << IMG_SHIFT) - 1;

// ekey == nullptr: every entry, L stored.  Otherwise only the entries the
// grouped path left out (ekey < 0), added to L.
__global__ void __launch_bounds__(WARPS * 32) k_m2l(int ncells, const int *off, const u32 *ent, const double4 *xr,
                                                    const double2 *M, double2 *L, int P, double cycle,
                                                    const int *ekey) {
  extern __shared__ double2 sh[];
  const int nt = tri(P);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * WARPS + wid;
  if (c >= ncells) return;
  double2 *acc = sh + wid * 3 * nt, *Z = acc + nt, *A = Z + nt;
  for (int k = lane; k < nt; k += 32) acc[k] = make_double2(0, 0);
  const double4 X = xr[c];
  for (int e = off[c]; e < off[c + 1]; e++) {
    if (ekey && ekey[e] >= 0) continue;
    const u32 en = ent[e];
    const int src = (int)(en & IDX_MASK), img = (int)(en >> IMG_SHIFT);
    const double4 Y = xr[src];
    const double dx = X.x - Y.x - (img % 3 - 1) * cycle;
    const double dy = X.y - Y.y - ((img / 3) % 3 - 1) * cycle;
    const double dz = X.z - Y.z - (img / 9 - 1) * cycle;
    const Sph g = sph_of(dx, dy, dz);
    __syncwarp();
    if (lane < P) irregular_column(lane, P, g.r, g, [&](int n, double2 v) { Z[tri(n) + lane] = v; });
    for (int k = lane; k < nt; k += 32) A[k] = M[(long)src * nt + k];
    __syncwarp();
    for (int o = lane; o < nt; o += 32) {
      int j = 0;
      while (tri(j + 1) <= o) j++;
      const int k = o - tri(j);
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
      acc[o].x += sx;
      acc[o].y += sy;
    }
  }
  __syncwarp();
  for (int k = lane; k < nt; k += 32) {
    if (ekey) {
      L[(long)c * nt + k].x += acc[k].x;
      L[(long)c * nt + k].y += acc[k].y;
    } else {
      L[(long)c * nt + k] = acc[k];
    }
  }
}

}  // namespace

bool m2l_grouped_available(int P);
void m2l_grouped_pass(Handle &h);

static void launch_direct_form(Handle &h, const int *ekey) {
  const int P = h.prm.P, nt = tri(P);
  k_m2l<<<grid_for(h.ncells, WARPS), WARPS * 32, WARPS * 3 * nt * sizeof(double2), h.stream>>>(
      h.ncells, h.m2l_off.as<int>(), h.m2l_ent.as<u32>(), h.c_xr.as<double4>(), h.M.as<double2>(),
      h.L.as<double2>(), P, h.prm.images ? h.prm.cycle : 0.0, ekey);
  h.launches++;
  FMM_LAUNCH();
}

void m2l_residual(Handle &h, const int *ekey) { launch_direct_form(h, ekey); }

void m2l_pass(Handle &h) {
  if (h.prm.dim == 2) return m2l_pass_2d(h);
  h.L.need((size_t)h.ncells * tri(h.prm.P) * sizeof(double2));
  if (!h.force_direct_m2l && m2l_grouped_available(h.prm.P)) {
    m2l_grouped_pass(h);
  } else {
    order_m2l_lists(h);  // the direct form sums each target's entries in list order
    launch_direct_form(h, nullptr);
  }
}

void m2l_set_attributes() {
  cudaFuncSetAttribute(k_m2l, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

}  // namespace fmm
