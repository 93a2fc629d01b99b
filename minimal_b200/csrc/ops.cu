// Single-operator entry points: the reference's kernel functions P2P, P2M,
// M2M, M2L, L2L and L2P (3d/kernel.h:122-323; the 3dp periodic shift of P2P
// and M2L, 3dp/kernel.h:133,200) on cells the caller describes, one call per
// operator, as the reference's kernel test and its operator chain call them
// (3d/kernel.cxx:4-91, test/test_kernel.h:6-94).  The passes of an
// evaluation never use these entry points: they run the tree-wide kernels.
//
// P2M and L2P run the FP64 pass kernels on a one-cell tree.  M2M, L2L and M2L
// take any offsets (the pass kernels use the octree's fixed child offsets and
// grouped operators), so they have kernels of their own here: one CTA builds
// the offset's harmonics in shared memory (one thread per order m) and every
// thread forms output coefficients with the shared translation formulas.
// Everything is FP64; results accumulate into the caller's outputs, as the
// reference's += does.
#include <algorithm>

#include "fmm.cuh"
#include "harmonics.cuh"
#include "translations.cuh"

namespace fmm {

void op_p2m(const int *mini, const double4 *xr, const double4 *src, double2 *M, int P, cudaStream_t s);
void op_l2p(const int *mini, const double4 *xr, const double4 *src, const double2 *L, double4 *out, int P,
            cudaStream_t s);

namespace {

constexpr int OT = 256;  // threads of the translation kernels

__device__ __forceinline__ void jk_of(int o, int &j, int &k) {
  j = order_of(o);
  k = o - tri(j);
}

// Regular harmonics Y_n^m (n < P, m >= 0) of offset d into Ysh.
__device__ void regular_table(int P, double dx, double dy, double dz, double2 *Ysh) {
  const Sph g = sph_of(dx, dy, dz);
  if ((int)threadIdx.x < P)
    regular_column(threadIdx.x, P, g.r, g, g.e, [&](int n, double2 Y, double2) { Ysh[tri(n) + threadIdx.x] = Y; });
}

// M2M (3d/kernel.h:204-231): Mp += the children's multipoles shifted to the
// parent, offset parent - child.  Kind 0.  L2L (3d/kernel.h:262-291): each
// child's L += the parent's local shifted to it, offset child - parent.
// Kind 1.
__global__ void __launch_bounds__(OT) k_op_shift(int kind, int P, double4 parent, const double4 *kids, int nkid,
                                                 const double2 *in, double2 *out) {
  extern __shared__ double2 sh[];
  const int nt = tri(P);
  double2 *Ysh = sh, *Ash = sh + nt;
  double2 acc[(EXAFMM_MAX_P * (EXAFMM_MAX_P + 1) / 2 + OT - 1) / OT];
  for (int q = 0; q < (int)(sizeof(acc) / sizeof(acc[0])); q++) acc[q] = make_double2(0, 0);
  if (kind == 1)
    for (int o = threadIdx.x; o < nt; o += OT) Ash[o] = in[o];
  for (int c = 0; c < nkid; c++) {
    __syncthreads();
    const double4 K = kids[c];
    if (kind == 0) {
      regular_table(P, parent.x - K.x, parent.y - K.y, parent.z - K.z, Ysh);
      for (int o = threadIdx.x; o < nt; o += OT) Ash[o] = in[(long)c * nt + o];
    } else {
      regular_table(P, K.x - parent.x, K.y - parent.y, K.z - parent.z, Ysh);
    }
    __syncthreads();
    for (int o = threadIdx.x, q = 0; o < nt; o += OT, q++) {
      int j, k;
      jk_of(o, j, k);
      if (kind == 0) {
        const double2 v = m2m_coeff(j, k, Ash, Ysh);
        acc[q].x += v.x;
        acc[q].y += v.y;
      } else {
        const double2 v = l2l_coeff(j, k, P, Ash, Ysh);
        out[(long)c * nt + o].x += v.x;
        out[(long)c * nt + o].y += v.y;
      }
    }
  }
  if (kind == 0)
    for (int o = threadIdx.x, q = 0; o < nt; o += OT, q++) {
      out[o].x += acc[q].x;
      out[o].y += acc[q].y;
    }
}

// M2L (3d/kernel.h:233-260; 3dp/kernel.h:198-200): L += the source's
// multipole translated to the target, offset target - source - shift.
__global__ void __launch_bounds__(OT) k_op_m2l(int P, double4 tgt, double4 srcc, double3 shift, const double2 *M,
                                               double2 *L) {
  extern __shared__ double2 sh[];
  const int nt = tri(P);
  double2 *Zsh = sh, *Msh = sh + nt;
  const Sph g = sph_of(tgt.x - srcc.x - shift.x, tgt.y - srcc.y - shift.y, tgt.z - srcc.z - shift.z);
  if ((int)threadIdx.x < P)
    irregular_column(threadIdx.x, P, g.r, g, [&](int n, double2 z) { Zsh[tri(n) + threadIdx.x] = z; });
  for (int o = threadIdx.x; o < nt; o += OT) Msh[o] = M[o];
  __syncthreads();
  for (int o = threadIdx.x; o < nt; o += OT) {
    int j, k;
    jk_of(o, j, k);
    const double2 v = m2l_coeff(j, k, P, Msh, Zsh);
    L[o].x += v.x;
    L[o].y += v.y;
  }
}

// P2P (3d/kernel.h:122-150; 3dp/kernel.h:133): one thread per target, the
// sources in shared-memory tiles, the reference's pair arithmetic
// (dX = Xi - Xj - shift, zero distance skipped).  Records in place.
constexpr int PT = 256;
__global__ void __launch_bounds__(PT) k_op_p2p(double *t8, long nt, const double *s8, long ns, double3 shift) {
  __shared__ double4 tile[PT];
  const long i = (long)blockIdx.x * PT + threadIdx.x;
  double tx = 0, ty = 0, tz = 0;
  if (i < nt) {
    tx = t8[8 * i];
    ty = t8[8 * i + 1];
    tz = t8[8 * i + 2];
  }
  double pot = 0, ax = 0, ay = 0, az = 0;
  for (long b = 0; b < ns; b += PT) {
    __syncthreads();
    if (b + threadIdx.x < ns) {
      const double *r = s8 + 8 * (b + threadIdx.x);
      tile[threadIdx.x] = make_double4(r[0], r[1], r[2], r[3]);
    }
    __syncthreads();
    const int m = (int)min((long)PT, ns - b);
    for (int k = 0; k < m; k++) {
      const double4 S = tile[k];
      const double dx = tx - S.x - shift.x, dy = ty - S.y - shift.y, dz = tz - S.z - shift.z;
      const double R2 = dx * dx + dy * dy + dz * dz;
      if (R2 != 0) {
        const double i2 = 1.0 / R2, iR = S.w * sqrt(i2), f = i2 * iR;
        pot += iR;
        ax += dx * f;
        ay += dy * f;
        az += dz * f;
      }
    }
  }
  if (i < nt) {
    t8[8 * i + 4] += pot;
    t8[8 * i + 5] -= ax;
    t8[8 * i + 6] -= ay;
    t8[8 * i + 7] -= az;
  }
}

// Body records -> (x,y,z,q) and (p,F) of the one-cell tree; back after L2P.
__global__ void k_op_pack(const double *r8, long n, double4 *xq, double4 *pf) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *r = r8 + 8 * i;
  xq[i] = make_double4(r[0], r[1], r[2], r[3]);
  if (pf) pf[i] = make_double4(r[4], r[5], r[6], r[7]);
}

__global__ void k_op_unpack(const double4 *pf, long n, double *r8) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double *r = r8 + 8 * i;
  r[4] = pf[i].x;
  r[5] = pf[i].y;
  r[6] = pf[i].z;
  r[7] = pf[i].w;
}

__global__ void k_op_add(const double2 *a, double2 *b, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    b[i].x += a[i].x;
    b[i].y += a[i].y;
  }
}

// Device copies of the call's arrays: a host array is staged in `scratch`
// (and copied back for outputs); a device array is used in place.
struct Staging {
  Handle &h;
  int where;
  size_t used = 0;
  struct Back {
    void *host;
    void *dev;
    size_t bytes;
  };
  std::vector<Back> back;
  Staging(Handle &h_, int w) : h(h_), where(w) {}
  static size_t round(size_t b) { return (b + 255) / 256 * 256; }
  char *take(size_t bytes) {
    if (used + round(bytes) > h.op_scratch.bytes) throw Error{EXAFMM_ERR_STATE, "operator scratch too small"};
    char *d = h.op_scratch.as<char>() + used;
    used += round(bytes);
    return d;
  }
  template <class T>
  T *in(const void *p, size_t bytes, bool output) {
    if (where == EXAFMM_DEVICE) return (T *)p;
    char *d = take(bytes);
    if (bytes) FMM_CUDA(cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, h.stream));
    if (output) back.push_back({(void *)p, d, bytes});
    return (T *)d;
  }
  template <class T>
  T *tmp(size_t bytes) {
    return (T *)take(bytes);
  }
  void finish() {
    for (const Back &b : back)
      if (b.bytes) FMM_CUDA(cudaMemcpyAsync(b.host, b.dev, b.bytes, cudaMemcpyDeviceToHost, h.stream));
    FMM_CUDA(cudaStreamSynchronize(h.stream));
  }
};

void need_scratch(Handle &h, size_t bytes) {
  h.op_scratch.need(bytes + 16 * 256);
}

void check_where(int where) {
  if (where != EXAFMM_HOST && where != EXAFMM_DEVICE) throw Error{EXAFMM_ERR_ARG, "where must be HOST or DEVICE"};
}

double4 cell_of(const double *c4, int where, Handle &h) {
  double v[4];
  if (where == EXAFMM_DEVICE) FMM_CUDA(cudaMemcpy(v, c4, sizeof(v), cudaMemcpyDeviceToHost));
  else for (int d = 0; d < 4; d++) v[d] = c4[d];
  (void)h;
  return make_double4(v[0], v[1], v[2], v[3]);
}

double3 shift_of(const double *s3, int where) {
  if (!s3) return make_double3(0, 0, 0);
  double v[3];
  if (where == EXAFMM_DEVICE) FMM_CUDA(cudaMemcpy(v, s3, sizeof(v), cudaMemcpyDeviceToHost));
  else for (int d = 0; d < 3; d++) v[d] = s3[d];
  return make_double3(v[0], v[1], v[2]);
}

size_t shift_smem(int P) { return 2 * (size_t)tri(P) * sizeof(double2); }

}  // namespace

void ops_set_attributes() {
  cudaFuncSetAttribute(k_op_shift, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shift_smem(EXAFMM_MAX_P));
  cudaFuncSetAttribute(k_op_m2l, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shift_smem(EXAFMM_MAX_P));
}

void op_p2p_call(Handle &h, double *t8, long nt, const double *s8, long ns, const double *shift3, int where) {
  check_where(where);
  if (!t8 || !s8 || nt < 0 || ns < 0) throw Error{EXAFMM_ERR_ARG, "p2p: need target and source records"};
  if (nt == 0 || ns == 0) return;
  const double3 sh = shift_of(shift3, where);
  need_scratch(h, (size_t)(nt + ns) * 64);
  Staging st(h, where);
  double *dt = st.in<double>(t8, nt * 64, true);
  const double *ds = st.in<double>(s8, ns * 64, false);
  k_op_p2p<<<grid_for(nt, PT), PT, 0, h.stream>>>(dt, nt, ds, ns, sh);
  h.launches++;
  FMM_LAUNCH();
  st.finish();
}

void op_p2m_call(Handle &h, const double *cell4, const double *b8, long nb, double *M, int where) {
  check_where(where);
  if (!cell4 || !M || (nb > 0 && !b8) || nb < 0) throw Error{EXAFMM_ERR_ARG, "p2m: need a cell, bodies and M"};
  const int P = h.prm.P, nt = tri(P);
  if (nb >= (1ll << 31)) throw Error{EXAFMM_ERR_ARG, "p2m: at most 2^31 - 1 bodies per cell"};
  need_scratch(h, 64 + 32 + (size_t)nb * (64 + 32) + 2 * (size_t)nt * 16);
  Staging st(h, where);
  const double4 C = cell_of(cell4, where, h);
  int *mini = st.tmp<int>(3 * sizeof(int));
  const int mh[3] = {0, 0, (int)nb};
  FMM_CUDA(cudaMemcpyAsync(mini, mh, sizeof(mh), cudaMemcpyHostToDevice, h.stream));
  double4 *xr = st.tmp<double4>(sizeof(double4));
  FMM_CUDA(cudaMemcpyAsync(xr, &C, sizeof(C), cudaMemcpyHostToDevice, h.stream));
  double2 *Mout = st.in<double2>(M, (size_t)nt * 16, true);
  if (nb == 0) {
    st.finish();
    return;
  }
  const double *db = st.in<double>(b8, (size_t)nb * 64, false);
  double4 *xq = st.tmp<double4>((size_t)nb * sizeof(double4));
  double2 *Mn = st.tmp<double2>((size_t)nt * 16);
  k_op_pack<<<grid_for(nb, 256), 256, 0, h.stream>>>(db, nb, xq, nullptr);
  op_p2m(mini, xr, xq, Mn, P, h.stream);  // writes the cell's P2M
  k_op_add<<<grid_for(nt, 256), 256, 0, h.stream>>>(Mn, Mout, nt);
  h.launches += 3;
  FMM_LAUNCH();
  st.finish();
}

void op_l2p_call(Handle &h, const double *cell4, const double *L, double *b8, long nb, int where) {
  check_where(where);
  if (!cell4 || !L || (nb > 0 && !b8) || nb < 0) throw Error{EXAFMM_ERR_ARG, "l2p: need a cell, L and bodies"};
  const int P = h.prm.P, nt = tri(P);
  if (nb >= (1ll << 31)) throw Error{EXAFMM_ERR_ARG, "l2p: at most 2^31 - 1 bodies per cell"};
  if (nb == 0) return;
  need_scratch(h, 64 + 32 + (size_t)nb * (64 + 64) + (size_t)nt * 16);
  Staging st(h, where);
  const double4 C = cell_of(cell4, where, h);
  int *mini = st.tmp<int>(3 * sizeof(int));
  const int mh[3] = {0, 0, (int)nb};
  FMM_CUDA(cudaMemcpyAsync(mini, mh, sizeof(mh), cudaMemcpyHostToDevice, h.stream));
  double4 *xr = st.tmp<double4>(sizeof(double4));
  FMM_CUDA(cudaMemcpyAsync(xr, &C, sizeof(C), cudaMemcpyHostToDevice, h.stream));
  const double2 *dL = st.in<double2>(L, (size_t)nt * 16, false);
  double *db = st.in<double>(b8, (size_t)nb * 64, true);
  double4 *xq = st.tmp<double4>((size_t)nb * sizeof(double4));
  double4 *pf = st.tmp<double4>((size_t)nb * sizeof(double4));
  k_op_pack<<<grid_for(nb, 256), 256, 0, h.stream>>>(db, nb, xq, pf);
  op_l2p(mini, xr, xq, dL, pf, P, h.stream);  // adds into p, F
  k_op_unpack<<<grid_for(nb, 256), 256, 0, h.stream>>>(pf, nb, db);
  h.launches += 3;
  FMM_LAUNCH();
  st.finish();
}

void op_shift_call(Handle &h, int kind, const double *parent4, const double *in, int nkid, const double *kids4,
                   double *out, int where) {
  check_where(where);
  const char *name = kind == 0 ? "m2m" : "l2l";
  if (!parent4 || !in || !out || nkid < 0 || (nkid > 0 && !kids4))
    throw Error{EXAFMM_ERR_ARG, std::string(name) + ": need the parent, the children and the expansions"};
  if (nkid == 0) return;
  const int P = h.prm.P, nt = tri(P);
  need_scratch(h, (size_t)nkid * 32 + (size_t)(nkid + 1) * nt * 16);
  Staging st(h, where);
  const double4 Pc = cell_of(parent4, where, h);
  const double4 *dk = st.in<double4>(kids4, (size_t)nkid * 32, false);
  // M2M: in = the children's M, out = the parent's M; L2L: in = the parent's
  // L, out = the children's L
  const size_t in_n = kind == 0 ? (size_t)nkid * nt : nt, out_n = kind == 0 ? nt : (size_t)nkid * nt;
  const double2 *din = st.in<double2>(in, in_n * 16, false);
  double2 *dout = st.in<double2>(out, out_n * 16, true);
  k_op_shift<<<1, OT, shift_smem(P), h.stream>>>(kind, P, Pc, dk, nkid, din, dout);
  h.launches++;
  FMM_LAUNCH();
  st.finish();
}

void op_m2l_call(Handle &h, const double *t4, double *L, const double *s4, const double *M, const double *shift3,
                 int where) {
  check_where(where);
  if (!t4 || !L || !s4 || !M) throw Error{EXAFMM_ERR_ARG, "m2l: need the target, L, the source and M"};
  const int P = h.prm.P, nt = tri(P);
  need_scratch(h, 2 * (size_t)nt * 16);
  Staging st(h, where);
  const double4 T = cell_of(t4, where, h), S = cell_of(s4, where, h);
  const double3 sh = shift_of(shift3, where);
  const double2 *dM = st.in<double2>(M, (size_t)nt * 16, false);
  double2 *dL = st.in<double2>(L, (size_t)nt * 16, true);
  k_op_m2l<<<1, OT, shift_smem(P), h.stream>>>(P, T, S, sh, dM, dL);
  h.launches++;
  FMM_LAUNCH();
  st.finish();
}

}  // namespace fmm
