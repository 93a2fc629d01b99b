// GPU octree build, bit-exact against the reference's recursive build
// (3d/build_tree.h:24-96, identical in 3dp/).
//
// The reference splits a cell by comparing each body with a centre that is
// produced by rounded FP64 additions, Xchild = X +/- R0/2^(level+1)
// (:116-126), leaf when NBODY <= ncrit (:81), children in octant order, bodies
// stably partitioned (:91-114).  Here:
//   1. bounds: min/max reduction, then X0, R0 exactly as getBounds (:7-21);
//   2. keys: per body, the octant digit of every level, each computed against
//      the centre of the body's own cell at that level by the same rounded
//      recurrence (__dadd_rn, no FMA contraction) -> a 3-bit-per-level key;
//   3. a stable LSD radix sort of (key, input index) on the key bits;
//   4. cells straight from the sorted keys: body i starts the cell of level l
//      that contains it iff the level-l key prefix changes at i and the parent
//      run holds more than ncrit bodies; run lengths come from binary searches
//      on the sorted keys.  Counting those cells per body and scanning gives
//      every cell its depth-first pre-order rank (cells sorted by first body,
//      then level) without any recursion;
//   5. a stable sort of the pre-order table by level gives the BFS layout the
//      level-synchronous passes use (children stay contiguous), and the
//      reference's own cell numbering (children appended as one block per
//      parent in pre-order) follows from a scan of child counts;
//   6. bodies inside each leaf are put back into input order (the reference's
//      stable partition never reorders bodies of one leaf).
// The key holds 3 bits per level for the first `key_levels` levels; if a cell
// at that depth still needs splitting the build is repeated with all 21.
//
// Batches of independent systems build one forest: every system gets its own
// bounds and root geometry, the system index sits above the octant digits in
// the sort key (so it is the level-0 prefix), each system's root always exists,
// and nothing else changes -- every system's cells and body order come out as
// if it were built alone, one after the other.
#include <cmath>

#include "fmm.cuh"

namespace fmm {

namespace {

constexpr int TB = 256;

__device__ __forceinline__ double dmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double dmax(double a, double b) { return fmax(a, b); }

__global__ void k_bounds_partial(const double4 *in, long n, double *part) {
  double lo[3] = {in[0].x, in[0].y, in[0].z}, hi[3] = {lo[0], lo[1], lo[2]};
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double4 b = in[i];
    lo[0] = dmin(b.x, lo[0]); lo[1] = dmin(b.y, lo[1]); lo[2] = dmin(b.z, lo[2]);
    hi[0] = dmax(b.x, hi[0]); hi[1] = dmax(b.y, hi[1]); hi[2] = dmax(b.z, hi[2]);
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int d = 0; d < 3; d++) {
      lo[d] = dmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = dmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  __shared__ double s[TB / 32][6];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int d = 0; d < 3; d++) { s[w][d] = lo[d]; s[w][3 + d] = hi[d]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < TB / 32; k++)
      for (int d = 0; d < 3; d++) { s[0][d] = dmin(s[0][d], s[k][d]); s[0][3 + d] = dmax(s[0][3 + d], s[k][3 + d]); }
    for (int d = 0; d < 6; d++) part[blockIdx.x * 6 + d] = s[0][d];
  }
}

// Min/max of the block's threads into thread 0 (exact operations: the
// reduction order cannot change the result).
__device__ void block_minmax(double lo[3], double hi[3]) {
  __shared__ double s[TB / 32][6];
  for (int o = 16; o > 0; o >>= 1)
    for (int d = 0; d < 3; d++) {
      lo[d] = dmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = dmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int d = 0; d < 3; d++) { s[w][d] = lo[d]; s[w][3 + d] = hi[d]; }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 1; k < TB / 32; k++)
      for (int d = 0; d < 3; d++) { lo[d] = dmin(s[k][d], lo[d]); hi[d] = dmax(s[k][3 + d], hi[d]); }
}

// getBounds (3d/build_tree.h:7-21): centre = (max+min)/2, R0 = largest
// half-extent about that centre, times 1.00001.
__global__ void k_bounds_final(const double *part, int nb, RootGeom *g) {
  double lo[3] = {part[0], part[1], part[2]}, hi[3] = {part[3], part[4], part[5]};
  for (int k = threadIdx.x; k < nb; k += blockDim.x)
    for (int d = 0; d < 3; d++) { lo[d] = dmin(part[6 * k + d], lo[d]); hi[d] = dmax(part[6 * k + 3 + d], hi[d]); }
  block_minmax(lo, hi);
  if (threadIdx.x != 0) return;
  double R0 = 0;
  for (int d = 0; d < 3; d++) {
    g->X0[d] = __ddiv_rn(__dadd_rn(hi[d], lo[d]), 2.0);
    R0 = dmax(__dadd_rn(g->X0[d], -lo[d]), R0);
    R0 = dmax(__dadd_rn(hi[d], -g->X0[d]), R0);
  }
  g->R0 = __dmul_rn(R0, 1.00001);
}

// Bounds of every system of a batch: one block per system, then the same
// getBounds arithmetic as k_bounds_final.
__global__ void k_bounds_systems(const double4 *in, const long long *off, RootGeom *geom) {
  const long b0 = off[blockIdx.x], b1 = off[blockIdx.x + 1];
  double lo[3] = {in[b0].x, in[b0].y, in[b0].z}, hi[3] = {lo[0], lo[1], lo[2]};
  for (long i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
    const double4 b = in[i];
    lo[0] = dmin(b.x, lo[0]); lo[1] = dmin(b.y, lo[1]); lo[2] = dmin(b.z, lo[2]);
    hi[0] = dmax(b.x, hi[0]); hi[1] = dmax(b.y, hi[1]); hi[2] = dmax(b.z, hi[2]);
  }
  block_minmax(lo, hi);
  if (threadIdx.x != 0) return;
  RootGeom *g = geom + blockIdx.x;
  double R0 = 0;
  for (int d = 0; d < 3; d++) {
    g->X0[d] = __ddiv_rn(__dadd_rn(hi[d], lo[d]), 2.0);
    R0 = dmax(__dadd_rn(g->X0[d], -lo[d]), R0);
    R0 = dmax(__dadd_rn(hi[d], -g->X0[d]), R0);
  }
  g->R0 = __dmul_rn(R0, 1.00001);
}

// System of body i: the last s with off[s] <= i (off: nsys+1 offsets).
__device__ __forceinline__ int system_of(const long long *off, int nsys, long i) {
  int lo = 0, hi = nsys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Octant digits of each body, level by level, against the exact centres of
// its system's cells; the system index above them.
__global__ void k_keys(const double4 *in, long n, const RootGeom *geom, const long long *sys_off, int nsys, int D,
                       u64 *keys, u32 *vals) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 b = in[i];
  const int sys = nsys > 1 ? system_of(sys_off, nsys, i) : 0;
  const RootGeom *g = geom + sys;
  double cx = g->X0[0], cy = g->X0[1], cz = g->X0[2];
  const double R0 = g->R0;
  u64 key = (u64)sys;
  double r = R0;
  for (int l = 0; l < D; l++) {
    const int ox = b.x > cx, oy = b.y > cy, oz = b.z > cz;
    key = (key << 3) | (u64)(ox | (oy << 1) | (oz << 2));
    r = __dmul_rn(r, 0.5);  // R0 / 2^(l+1): halving is the correctly rounded quotient
    cx = __dadd_rn(cx, ox ? r : -r);
    cy = __dadd_rn(cy, oy ? r : -r);
    cz = __dadd_rn(cz, oz ? r : -r);
  }
  keys[i] = key;
  vals[i] = (u32)i;
}

// Level-l prefix of a key: the system index and the first l octant digits.
__device__ __forceinline__ u64 prefix_of(u64 key, int D, int l) { return key >> (3 * (D - l)); }

// First index in [lo, hi) whose level-l prefix exceeds p (keys sorted, and
// keys[lo] has a prefix <= p): a galloping search up from lo, then a binary
// search in the last step -- runs near the leaves are short, so this takes
// about twice the log of the run length instead of the log of the range.
__device__ long upper_run(const u64 *keys, long lo, long hi, int D, int l, u64 p) {
  long a = lo, step = 1;
  while (a + step < hi && prefix_of(keys[a + step], D, l) <= p) {
    a += step;
    step <<= 1;
  }
  long L = a + 1, H = a + step < hi ? a + step : hi;  // the answer is in [L, H]
  while (L < H) {
    const long mid = (L + H) >> 1;
    if (prefix_of(keys[mid], D, l) > p) H = mid; else L = mid + 1;
  }
  return L;
}
// First index in [lo, hi) whose level-l prefix is >= p (keys[hi], when it
// exists, has a prefix >= p): galloping down from hi.
__device__ long lower_run(const u64 *keys, long lo, long hi, int D, int l, u64 p) {
  long b = hi, step = 1;
  while (b - step >= lo && prefix_of(keys[b - step], D, l) >= p) {
    b -= step;
    step <<= 1;
  }
  long L = b - step < lo ? lo : b - step + 1, H = b;  // the answer is in [L, H]
  while (L < H) {
    const long mid = (L + H) >> 1;
    if (prefix_of(keys[mid], D, l) >= p) H = mid; else L = mid + 1;
  }
  return L;
}

// Shallowest level whose key prefix at i differs from i-1 (D+1: same key).
__device__ __forceinline__ int first_level(const u64 *keys, long i, int D) {
  if (i == 0) return 0;
  const u64 x = keys[i] ^ keys[i - 1];
  if (x == 0) return D + 1;
  const int h = 63 - __clzll((long long)x);
  if (h >= 3 * D) return 0;  // another system: its root starts here
  return D - h / 3;
}

// Shallowest level whose key prefixes of x and y differ (D+1: none).
__device__ __forceinline__ int diff_level(u64 x, u64 y, int D) {
  const u64 d = x ^ y;
  if (d == 0) return D + 1;
  const int h = 63 - __clzll((long long)d);
  if (h >= 3 * D) return 0;  // another system
  return D - h / 3;
}

// Bodies from i on (i included) in i's level-l run, counted up to cap.
__device__ long run_ahead(const u64 *keys, long i, long n, int D, int l, u64 p, long cap) {
  const long last = i + cap < n ? i + cap : n;
  if (last == i + cap && prefix_of(keys[last - 1], D, l) == p) return cap;
  long L = i + 1, H = last;  // the run ends in [L, H]
  while (L < H) {
    const long mid = (L + H) >> 1;
    if (prefix_of(keys[mid], D, l) > p) H = mid; else L = mid + 1;
  }
  return L - i;
}

// Number of cells whose first body is sorted position i (a chain of nested
// first-children), plus the depth overflow check.  A run that starts at i
// holds more than ncrit bodies iff body i + ncrit shares its prefix, so the
// chain length follows from one comparison of keys; the parent test counts
// at most ncrit + 1 bodies on either side of i.
__global__ void k_chain(const u64 *keys, long n, int D, int ncrit, int *lfirst, int *chain, DevCounters *ctr) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int lf = first_level(keys, i, D);
  lfirst[i] = lf;
  int len = 0;
  if (lf <= D) {
    const u64 key = keys[i];
    bool parent_splits = true;  // a system's root is always a cell
    if (lf > 0) {
      const u64 pp = prefix_of(key, D, lf - 1);
      const long R = run_ahead(keys, i, n, D, lf - 1, pp, (long)ncrit + 1);
      const long need = (long)ncrit + 1 - R;  // parent bodies wanted before i
      parent_splits = need <= 0 || (i - need >= 0 && prefix_of(keys[i - need], D, lf - 1) == pp);
    }
    if (parent_splits) {
      // levels lf, lf+1, ... while the run from i exceeds ncrit, then the leaf
      int last = i + ncrit < n ? diff_level(key, keys[i + ncrit], D) : lf;
      if (last < lf) last = lf;
      if (last > D) {
        ctr->overflow = 1;
        last = D;
      }
      len = last - lf + 1;
    }
  }
  chain[i] = len;
}

struct PreTables {
  int *begin, *count, *level, *parent, *nchild;
  double4 *xr;
};

// The body that starts each cell (pre-order rank -> sorted body position).
__global__ void k_cell_owner(long n, const int *chain, const int *prebase, int *owner) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int len = chain[i];
  for (int k = 0; k < len; k++) owner[prebase[i] + k] = (int)i;
}

// One thread per cell (pre-order rank p): the k-th cell of the chain that
// starts at body i = owner[p] is at level lfirst[i] + k.
__global__ void k_cells(const u64 *keys, long n, long C, int D, const int *lfirst, const int *owner,
                        const int *prebase, const RootGeom *g, PreTables t, DevCounters *ctr) {
  __shared__ int lc[EXAFMM_MAX_LEVEL + 2];  // cells per level made by this block
  if (threadIdx.x < EXAFMM_MAX_LEVEL + 2) lc[threadIdx.x] = 0;
  __syncthreads();
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < C) {
    const long i = owner[p];
    const int k = (int)(p - prebase[i]), lf = lfirst[i], l = lf + k;
    const u64 key = keys[i];
    const RootGeom *gs = g + (long)(key >> (3 * D));  // the body's system
    double cx = gs->X0[0], cy = gs->X0[1], cz = gs->X0[2];
    double r = gs->R0;  // R0 / 2^l, halved exactly level by level
    for (int q = 0; q < l; q++) {  // centre of the level-l cell holding body i
      const int o = (int)((key >> (3 * (D - 1 - q))) & 7);
      r = __dmul_rn(r, 0.5);
      cx = __dadd_rn(cx, (o & 1) ? r : -r);
      cy = __dadd_rn(cy, (o & 2) ? r : -r);
      cz = __dadd_rn(cz, (o & 4) ? r : -r);
    }
    int parent = (int)p - 1;  // the chain's previous cell
    if (k == 0) {
      parent = -1;
      if (lf > 0) {
        const long b0 = lower_run(keys, 0, i, D, lf - 1, prefix_of(key, D, lf - 1));
        parent = prebase[b0] + (lf - 1 - lfirst[b0]);
      }
    }
    const long e = upper_run(keys, i, n, D, l, prefix_of(key, D, l));
    t.begin[p] = (int)i;
    t.count[p] = (int)(e - i);
    t.level[p] = l;
    t.parent[p] = parent;
    t.xr[p] = make_double4(cx, cy, cz, r);
    atomicAdd_block(&lc[l], 1);
    if (parent >= 0) atomicAdd(&t.nchild[parent], 1);
  }
  __syncthreads();
  if (threadIdx.x < EXAFMM_MAX_LEVEL + 2 && lc[threadIdx.x]) atomicAdd(&ctr->level_count[threadIdx.x], lc[threadIdx.x]);
}

__global__ void k_level_keys(const int *level, long c, u64 *k, u32 *v) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c) return;
  k[i] = (u64)level[i];
  v[i] = (u32)i;
}

__global__ void k_invert(const u32 *pre_of_bfs, long c, int *bfs_of_pre) {
  const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b < c) bfs_of_pre[pre_of_bfs[b]] = (int)b;
}

struct BfsCells {
  int *begin, *count, *child, *nchild, *parent, *level, *pre;
  double4 *xr;
};

__global__ void k_gather_cells(const u32 *pre_of_bfs, const int *bfs_of_pre, long c, PreTables t, BfsCells o,
                               int *is_leaf) {
  const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= c) return;
  const int p = (int)pre_of_bfs[b];
  o.begin[b] = t.begin[p];
  o.count[b] = t.count[p];
  o.level[b] = t.level[p];
  o.xr[b] = t.xr[p];
  o.parent[b] = t.parent[p] >= 0 ? bfs_of_pre[t.parent[p]] : -1;
  const int nc = t.nchild[p];
  o.nchild[b] = nc;
  o.child[b] = nc ? bfs_of_pre[p + 1] : -1;
  o.pre[b] = p;
  is_leaf[b] = nc == 0;
}

// Reference cell number: 1 + (children allocated by parents earlier in
// pre-order) + rank among siblings (3d/build_tree.h:69-84).
__global__ void k_ref_index(BfsCells o, long c, const int *blockstart_pre, int *ref) {
  const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= c) return;
  const int par = o.parent[b];
  ref[b] = par < 0 ? 0 : 1 + blockstart_pre[o.pre[par]] + (int)(b - o.child[par]);
}

__global__ void k_compact_leaves(const int *is_leaf, const int *pos, long c, int *leaves) {
  const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b < c && is_leaf[b]) leaves[pos[b]] = (int)b;
}

// Bodies of one leaf back into input order (warp per leaf, rank sort).
// Bodies of each leaf back to input order (a body's slot is the rank of its
// input index among the leaf's), gathered into src.  With srcf (3D mixed
// form) also the FP32 copy of each body as an offset from its leaf centre
// (FP64 subtraction, one rounding) and the body's leaf, as k_make_srcf makes
// them: one pass over the bodies instead of three.
__global__ void k_leaf_order(const int *leaves, int nleaves, const int *begin, const int *count, const double4 *xr,
                             const u32 *vals, const double4 *in, int *perm, double4 *src, float4 *srcf,
                             int *body_leaf) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nleaves) return;
  const int c = leaves[w], b0 = begin[c], nb = count[c];
  const double4 C = xr[c];
  for (int a = lane; a < nb; a += 32) {
    const u32 v = vals[b0 + a];
    int r = 0;
    for (int k = 0; k < nb; k++) r += vals[b0 + k] < v;
    const int b = b0 + r;
    perm[b] = (int)v;
    const double4 B = in[v];
    src[b] = B;
    if (srcf) {
      srcf[b] = make_float4((float)(B.x - C.x), (float)(B.y - C.y), (float)(B.z - C.z), (float)B.w);
      body_leaf[b] = w;
    }
  }
}


__global__ void k_zero_counters(DevCounters *c) {
  const int t = threadIdx.x;
  int *w = (int *)c;
  for (int k = t; k < (int)(sizeof(DevCounters) / sizeof(int)); k += blockDim.x) w[k] = 0;
}

}  // namespace

void build_tree(Handle &h) {
  const long n = h.n;
  cudaStream_t s = h.stream;
  h.srcf_ready = false;  // set again once the new tree's FP32 sources are made
  const int nsys = h.nsys;
  h.geom.need((size_t)nsys * sizeof(RootGeom));
  h.counters.need(sizeof(DevCounters));
  DevCounters *ctr = h.counters.as<DevCounters>();
  RootGeom *g = h.geom.as<RootGeom>();
  const long long *sys_off = nsys > 1 ? h.sys_off.as<long long>() : nullptr;

  // 1. bounds
  if (nsys > 1) {
    k_bounds_systems<<<nsys, TB, 0, s>>>(h.in.as<double4>(), sys_off, g);
    h.launches++;
  } else {
    const int nbp = (int)std::min<long>(4 * 148, (n + TB - 1) / TB);
    h.hist.need((size_t)nbp * 6 * sizeof(double));
    k_bounds_partial<<<nbp, TB, 0, s>>>(h.in.as<double4>(), n, h.hist.as<double>());
    k_bounds_final<<<1, TB, 0, s>>>(h.hist.as<double>(), nbp, g);
    h.launches += 2;
  }
  FMM_LAUNCH();

  // the system index takes the key bits above the octant digits
  int sys_bits = 0;
  while ((1ll << sys_bits) < nsys) sys_bits++;
  const int max_levels = std::min(EXAFMM_MAX_LEVEL, (64 - sys_bits) / 3);
  int D = h.key_levels;
  if (D <= 0) {
    long nmax = n;
    if (nsys > 1) {
      nmax = 0;
      for (int q = 0; q < nsys; q++) nmax = std::max<long>(nmax, (long)(h.sys_off_host[q + 1] - h.sys_off_host[q]));
    }
    double ratio = (double)nmax / (double)(h.prm.ncrit > 0 ? h.prm.ncrit : 1);
    D = (int)std::ceil(std::log(std::max(ratio, 1.0)) / std::log(8.0)) + 3;
    D = std::min(std::max(D, 2), max_levels);
  }
  D = std::min(D, max_levels);
  for (h.keys[0].need(n * 8), h.keys[1].need(n * 8), h.vals[0].need(n * 4), h.vals[1].need(n * 4);;) {
    k_zero_counters<<<1, 256, 0, s>>>(ctr);
    u64 *k = h.keys[0].as<u64>(), *k2 = h.keys[1].as<u64>();
    u32 *v = h.vals[0].as<u32>(), *v2 = h.vals[1].as<u32>();
    k_keys<<<grid_for(n, TB), TB, 0, s>>>(h.in.as<double4>(), n, g, sys_off, nsys, D, k, v);
    h.launches += 2;
    FMM_LAUNCH();
    radix_sort_pairs(h, k, v, k2, v2, n, 0, 3 * D + sys_bits);
    h.lfirst.need(n * 4);
    h.chain.need(n * 4);
    h.prebase.need((n + 1) * 4);
    k_chain<<<grid_for(n, TB), TB, 0, s>>>(k, n, D, h.prm.ncrit, h.lfirst.as<int>(), h.chain.as<int>(), ctr);
    h.launches++;
    FMM_LAUNCH();
    scan_exclusive_int(h, h.chain.as<int>(), h.prebase.as<int>(), n, &ctr->ncells);
    FMM_CUDA(cudaMemcpyAsync(&h.hc, ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
    FMM_CUDA(cudaStreamSynchronize(s));
    if (h.hc.overflow) {
      if (D == max_levels)
        throw Error{EXAFMM_ERR_DEPTH, "more than ncrit bodies share a cell at the deepest level (" +
                                          std::to_string(max_levels) + "): coincident bodies?"};
      D = max_levels;
      continue;
    }
    const long C = h.hc.ncells;
    h.ncells = (int)C;
    h.key_levels = D;
    // pre-order tables (reuse the idle sort buffers' siblings)
    h.pre_tmp.need(C * (6 * sizeof(int) + sizeof(double4)) + 256);
    PreTables t;
    t.xr = h.pre_tmp.as<double4>();
    t.begin = (int *)(t.xr + C);
    t.count = t.begin + C;
    t.level = t.count + C;
    t.parent = t.level + C;
    t.nchild = t.parent + C;
    int *owner = t.nchild + C;
    FMM_CUDA(cudaMemsetAsync(t.nchild, 0, C * sizeof(int), s));
    k_cell_owner<<<grid_for(n, TB), TB, 0, s>>>(n, h.chain.as<int>(), h.prebase.as<int>(), owner);
    k_cells<<<grid_for(C, TB), TB, 0, s>>>(k, n, C, D, h.lfirst.as<int>(), owner, h.prebase.as<int>(), g, t, ctr);
    h.launches += 2;
    FMM_LAUNCH();

    // 5. BFS order = stable sort of pre-order cells by level
    const long Cp = (C + 3) & ~3L;  // every table starts 16-byte aligned (vector loads in the scans)
    h.ctmp.need(Cp * (2 * sizeof(u64) + 2 * sizeof(u32) + 4 * sizeof(int)) + 256);
    u64 *lk = h.ctmp.as<u64>(), *lk2 = lk + Cp;
    u32 *lv = (u32 *)(lk2 + Cp), *lv2 = lv + Cp;
    int *bfs_of_pre = (int *)(lv2 + Cp), *is_leaf = bfs_of_pre + Cp, *blockstart = is_leaf + Cp,
        *leafpos = blockstart + Cp;
    k_level_keys<<<grid_for(C, TB), TB, 0, s>>>(t.level, C, lk, lv);
    h.launches++;
    FMM_LAUNCH();
    radix_sort_pairs(h, lk, lv, lk2, lv2, C, 0, 5);
    k_invert<<<grid_for(C, TB), TB, 0, s>>>(lv, C, bfs_of_pre);
    h.launches++;
    h.c_begin.need(C * 4); h.c_count.need(C * 4); h.c_child.need(C * 4); h.c_nchild.need(C * 4);
    h.c_parent.need(C * 4); h.c_level.need(C * 4); h.c_pre.need(C * 4); h.c_ref.need(C * 4);
    h.c_xr.need(C * sizeof(double4));
    BfsCells o{h.c_begin.as<int>(), h.c_count.as<int>(), h.c_child.as<int>(), h.c_nchild.as<int>(),
               h.c_parent.as<int>(), h.c_level.as<int>(), h.c_pre.as<int>(), h.c_xr.as<double4>()};
    k_gather_cells<<<grid_for(C, TB), TB, 0, s>>>(lv, bfs_of_pre, C, t, o, is_leaf);
    h.launches++;
    FMM_LAUNCH();
    // reference numbering
    scan_exclusive_int(h, t.nchild, blockstart, C, nullptr);
    k_ref_index<<<grid_for(C, TB), TB, 0, s>>>(o, C, blockstart, h.c_ref.as<int>());
    h.launches++;
    // leaves
    scan_exclusive_int(h, is_leaf, leafpos, C, &ctr->nleaves);
    h.leaves.need(C * 4);
    k_compact_leaves<<<grid_for(C, TB), TB, 0, s>>>(is_leaf, leafpos, C, h.leaves.as<int>());
    h.launches++;
    FMM_LAUNCH();
    FMM_CUDA(cudaMemcpyAsync(&h.hc, ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
    FMM_CUDA(cudaStreamSynchronize(s));
    h.nleaves = h.hc.nleaves;
    h.depth = 0;
    h.level_base[0] = 0;
    for (int l = 0; l <= EXAFMM_MAX_LEVEL; l++) {
      h.level_base[l + 1] = h.level_base[l] + h.hc.level_count[l];
      if (h.hc.level_count[l]) h.depth = l;
    }
    // 6. bodies of each leaf back to input order and gathered (the mixed
    // form's FP32 sources with them)
    h.perm.need(n * 4);
    h.src.need(n * sizeof(double4));
    const bool srcf = h.prm.precision == EXAFMM_MIXED && h.prm.dim == 3;
    if (srcf) {
      h.srcf.need((size_t)n * sizeof(float4));
      h.body_leaf.need((size_t)n * sizeof(int));
    }
    k_leaf_order<<<grid_for((long)h.nleaves * 32, TB), TB, 0, s>>>(
        h.leaves.as<int>(), h.nleaves, o.begin, o.count, o.xr, v, h.in.as<double4>(), h.perm.as<int>(),
        h.src.as<double4>(), srcf ? h.srcf.as<float4>() : nullptr, srcf ? h.body_leaf.as<int>() : nullptr);
    h.launches++;
    FMM_LAUNCH();
    h.srcf_ready = srcf;
    break;
  }
  // 2D bodies lie at z = 0: the octree is the quadtree (the z digit is the
  // same for every body of a level); its cells go to the plane z = 0
  if (h.prm.dim == 2) flatten_tree_2d(h);
}

}  // namespace fmm
