// GPU interaction-list builder: the reference's dual-tree traversal
// (3d/traverse_eager.h:147-165, recorded as lists by 3d/traverse_lazy.h:27-44;
// periodic shifts 3dp/traverse_lazy.h:39-58 and the 27-image loop
// 3dp/traverse_lazy.h:128-134)
// run breadth first over a frontier of (target, source, image) cell pairs.
//
// Each step applies the reference's branch rules to every pair of the
// frontier with the same rounded FP64 arithmetic (no FMA):
//   |Xi - Xj - iX*cycle|^2 * theta^2 > (Ri + Rj)^2  -> M2L entry
//   else both leaves                                 -> P2P entry
//   else Cj leaf or (Ri >= Rj and Ci not a leaf)     -> (children of Ci, Cj)
//   else                                             -> (Ci, children of Cj)
// Emission uses one warp scan and one atomic per list per warp.  The entries are then bucketed per
// target cell (CSR) and each target's entries are ordered as the recursion
// would have recorded them: image-loop order first (x outermost), then the
// source's depth-first pre-order rank (a depth-first walk meets the sources
// of one target in pre-order, because a target-side split never reorders
// them).  The result equals getList's per-cell lists entry for entry.
#include "group_key.cuh"

namespace fmm {

namespace {

constexpr int TB = 256;
constexpr int WALK_PAIRS = 2;  // frontier pairs per thread per walk iteration
constexpr int IMG_SHIFT = 26;             // entry = src | img << 26
constexpr u32 IDX_MASK = (1u << IMG_SHIFT) - 1;

struct CellView {
  const double4 *xr;
  const int *child, *nchild;
};

__device__ __forceinline__ void img3(int img, int &x, int &y, int &z) {
  x = img % 3 - 1;
  y = (img / 3) % 3 - 1;
  z = img / 9 - 1;
}

// Level difference of two cells from their radii (R0 / 2^level, exactly):
// the difference of the FP64 exponent fields when both are normal numbers,
// else of ilogb.
__device__ __forceinline__ int radius_level_diff(double rb, double ra) {
  const int eb = (__double2hiint(rb) >> 20) & 0x7ff, ea = (__double2hiint(ra) >> 20) & 0x7ff;
  if (eb != 0 && ea != 0 && eb != 0x7ff && ea != 0x7ff) return eb - ea;
  return ilogb(rb) - ilogb(ra);
}

// One step of the walk.  Each thread takes WP frontier pairs per iteration
// (the block's CHUNK = TB * WP consecutive pairs, pair r of thread t at
// r * TB + t), so one block scan and one atomic per list reserve the output
// ranges of CHUNK pairs; a thread's entries of one list are consecutive.
// PERIODIC false: every pair is of image 13 (no shift), so the shift terms,
// zero, are left out: x - 0 is x in every rounding.
template <int WP, bool PERIODIC>
__global__ void __launch_bounds__(TB) k_walk(CellView cv, const int2 *fin, const unsigned long long *nin_p,
                                            int2 *fout, unsigned long long *nout, unsigned long long *nnext,
                                            u64 fcap, int2 *m2l, unsigned long long *nm2l, u64 mcap, int2 *p2p,
                                            unsigned long long *np2p, u64 pcap, double theta, double cycle,
                                            int depth, int *overflow, int *m2l_key, int *occ, int *gflag,
                                            int *nres) {
  constexpr int NW = TB / 32, CHUNK = TB * WP;
  static_assert(CHUNK < 4096, "per-block M2L and P2P counts are packed in 12-bit fields");
  __shared__ int s_tot[NW], s_totk[NW];    // every warp's packed list counts and frontier count
  __shared__ unsigned long long s_base[3];  // the block's M2L, P2P and frontier ranges
  __shared__ int s_res;                     // M2L entries without a group key
  if (threadIdx.x == 0) s_res = 0;
  int res = 0;
  // the producer counts appends past its capacity (to size the retry); only
  // the stored entries may be read
  const u64 nin = min((u64)*nin_p, fcap);
  // the counter the step after next appends to: nothing reads it any more
  if (blockIdx.x == 0 && threadIdx.x == 0) *nnext = 0;
  const u64 stride = (u64)gridDim.x * CHUNK;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  // every thread of a block iterates the same number of times (block-wide appends)
  for (u64 base = (u64)blockIdx.x * CHUNK; base < nin; base += stride) {
    int2 pr[WP];
#pragma unroll
    for (int r = 0; r < WP; r++) {
      const u64 idx = base + (u64)r * TB + threadIdx.x;
      pr[r] = idx < nin ? fin[idx] : make_int2(0, -1);  // y = -1: no pair
    }
    int kind[WP], nk[WP], first[WP], key[WP];  // kind: -1 none, 0 m2l, 1 p2p, 2 split i, 3 split j
    int nm = 0, np = 0, nf = 0;
#pragma unroll
    for (int r = 0; r < WP; r++) {
      kind[r] = -1;
      nk[r] = 0;
      first[r] = 0;
      key[r] = -1;
      if (pr[r].y < 0) continue;
      const int i = pr[r].x & (int)IDX_MASK, img = PERIODIC ? (int)((u32)pr[r].x >> IMG_SHIFT) : 13, j = pr[r].y;
      const double4 a = cv.xr[i], b = cv.xr[j];
      double dx = __dadd_rn(a.x, -b.x), dy = __dadd_rn(a.y, -b.y), dz = __dadd_rn(a.z, -b.z);
      if (PERIODIC) {
        int ix, iy, iz;
        img3(img, ix, iy, iz);
        dx = __dadd_rn(dx, -__dmul_rn((double)ix, cycle));
        dy = __dadd_rn(dy, -__dmul_rn((double)iy, cycle));
        dz = __dadd_rn(dz, -__dmul_rn((double)iz, cycle));
      }
      const double nrm = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      const double R2 = __dmul_rn(__dmul_rn(nrm, theta), theta);
      const double rs = __dadd_rn(a.w, b.w);
      const int ci = cv.nchild[i], cj = cv.nchild[j];
      if (R2 > __dmul_rn(rs, rs)) {
        kind[r] = 0;
        // the group key of the grouped M2L (radii are R0 / 2^level exactly,
        // so their exponents give the level difference)
        const int dl = radius_level_diff(b.w, a.w);
        if (img == 13) key[r] = m2l_group_key(a, b, dl);
        else key[r] = m2l_image_key(a, b, dl, img, cv.xr[0].w, cycle, depth);
        if (key[r] >= 0) m2l_mark_key(key[r], i, occ, gflag);
        else res++;
        nm++;
      } else if (ci == 0 && cj == 0) {
        kind[r] = 1;
        np++;
      } else if (cj == 0 || (a.w >= b.w && ci != 0)) {
        kind[r] = 2;
        nk[r] = ci;
        first[r] = cv.child[i];
      } else {
        kind[r] = 3;
        nk[r] = cj;
        first[r] = cv.child[j];
      }
      nf += nk[r];
    }
    // warp scans for the three appends: M2L count in bits 0-11 and P2P in
    // 12-23 of one word (at most CHUNK each per block), frontier pairs in a
    // second
    const int mine = nm | (np << 12);
    int incl = mine, inck = nf;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o), tk = __shfl_up_sync(0xffffffffu, inck, o);
      if (lane >= o) {
        incl += t;
        inck += tk;
      }
    }
    __syncthreads();  // the previous iteration's block ranges are consumed
    if (lane == 31) {
      s_tot[wid] = incl;
      s_totk[wid] = inck;
    }
    __syncthreads();
    if (threadIdx.x < 3) {  // threads 0, 1, 2 reserve the block's M2L, P2P and frontier ranges
      int tot = 0;
      for (int w = 0; w < NW; w++) tot += threadIdx.x == 2 ? s_totk[w] : s_tot[w];
      const unsigned n = threadIdx.x == 0 ? (tot & 4095) : threadIdx.x == 1 ? ((tot >> 12) & 4095) : tot;
      unsigned long long *ctr = threadIdx.x == 0 ? nm2l : threadIdx.x == 1 ? np2p : nout;
      s_base[threadIdx.x] = n ? atomicAdd(ctr, (unsigned long long)n) : 0ull;
    }
    __syncthreads();
    int wpre = 0, wprek = 0;  // earlier warps of the block
    for (int w = 0; w < wid; w++) {
      wpre += s_tot[w];
      wprek += s_totk[w];
    }
    const int excl = wpre + incl - mine;
    unsigned long long sm = s_base[0] + (excl & 4095), sp = s_base[1] + ((excl >> 12) & 4095),
                       sf = s_base[2] + (wprek + inck - nf);
#pragma unroll
    for (int r = 0; r < WP; r++) {
      if (kind[r] == 0) {
        if (sm < mcap) {
          m2l[sm] = pr[r];
          m2l_key[sm] = key[r];
        } else {
          *overflow = 1;
        }
        sm++;
      } else if (kind[r] == 1) {
        if (sp < pcap) p2p[sp] = pr[r]; else *overflow = 1;
        sp++;
      } else if (nk[r] > 0) {
        const int img = (int)((u32)pr[r].x >> IMG_SHIFT);
        for (int c = 0; c < nk[r]; c++) {
          if (sf + c < fcap) {
            fout[sf + c] = kind[r] == 2 ? make_int2((first[r] + c) | (img << IMG_SHIFT), pr[r].y)
                                        : make_int2(pr[r].x, first[r] + c);
          } else {
            *overflow = 1;
          }
        }
        sf += nk[r];
      }
    }
  }
  if (res) atomicAdd_block(&s_res, res);
  __syncthreads();
  if (threadIdx.x == 0 && s_res) atomicAdd(nres, s_res);
}

// Root pairs of the walk: (root, root) of every system of a batch (the roots
// are the first nsys cells), or the 27 image pairs of a periodic system.
__global__ void k_seed(int2 *f, unsigned long long *n, int images, int nsys, int dim) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (images == 0) {
    if (t < nsys) f[t] = make_int2(t | (13 << IMG_SHIFT), t);
    if (t == 0) *n = (unsigned long long)nsys;
  } else if (dim == 2) {
    // the 2dp image loop: x outer, y inner, in the plane (z = 0: img 9..17)
    if (t < 9) {
      const int x = t / 3 - 1, y = t % 3 - 1;
      f[t] = make_int2(0 | (((x + 1) + 3 * (y + 1) + 9) << IMG_SHIFT), 0);
    }
    if (t == 0) *n = 9;
  } else if (t < 27) {
    // image loop order of the reference: x outermost, z innermost; img is
    // periodic1D = (x+1) + 3(y+1) + 9(z+1)
    const int x = t / 9 - 1, y = (t / 3) % 3 - 1, z = t % 3 - 1;
    const int img = (x + 1) + 3 * (y + 1) + 9 * (z + 1);
    f[t] = make_int2(0 | (img << IMG_SHIFT), 0);
    if (t == 0) *n = 27;
  }
}

// Entries of one target often arrive together (a split emits the children
// of one cell side by side): lanes with the same target add once.
__global__ void k_count_tgt(const int2 *e, const unsigned long long *n_p, u64 cap, int *cnt) {
  const u64 n = min((u64)*n_p, cap);
  for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (u64)gridDim.x * blockDim.x) {
    const int t = e[k].x & (int)IDX_MASK;
    const unsigned peers = __match_any_sync(__activemask(), t);
    if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&cnt[t], __popc(peers));
  }
}

__global__ void k_bucket(const int2 *e, const unsigned long long *n_p, u64 cap, const int *off, int *fill,
                         u32 *ent) {
  const u64 n = min((u64)*n_p, cap);
  const int lane = threadIdx.x & 31;
  for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (u64)gridDim.x * blockDim.x) {
    const int2 v = e[k];
    const int t = v.x & (int)IDX_MASK;
    const u32 img = (u32)v.x >> IMG_SHIFT;
    const unsigned act = __activemask();
    const unsigned peers = __match_any_sync(act, t);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&fill[t], __popc(peers));
    base = __shfl_sync(act, base, leader);
    const int pos = off[t] + base + __popc(peers & ((1u << lane) - 1));
    ent[pos] = (u32)v.y | (img << IMG_SHIFT);
  }
}

// Recording order of the reference inside one target's list.
__device__ __forceinline__ u64 order_key(u32 e, const int *pre) {
  const u32 img = e >> IMG_SHIFT;
  const u32 x = img % 3, y = (img / 3) % 3, z = img / 9;  // (x+1),(y+1),(z+1)
  const u64 loop = x * 9 + y * 3 + z;                     // x outermost
  return (loop << 32) | (u64)(u32)pre[e & IDX_MASK];
}

// One warp per target: rank sort of the target's entries by order_key, keys
// staged in shared memory (segments longer than SEG_SMEM rank from global).
constexpr int SEG_WARPS = 4;
constexpr int SEG_SMEM = 512;

__global__ void __launch_bounds__(SEG_WARPS * 32) k_order_segments(const int *off, int ncells, const u32 *in,
                                                                  u32 *out, const int *pre) {
  __shared__ u64 keys[SEG_WARPS][SEG_SMEM];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * SEG_WARPS + wid;
  if (w >= ncells) return;
  const int b = off[w], m = off[w + 1] - b;
  if (m <= SEG_SMEM) {
    for (int a = lane; a < m; a += 32) keys[wid][a] = order_key(in[b + a], pre);
    __syncwarp();
    for (int a = lane; a < m; a += 32) {
      const u64 key = keys[wid][a];
      int r = 0;
      for (int k = 0; k < m; k++) r += keys[wid][k] < key;
      out[b + r] = in[b + a];
    }
  } else {
    for (int a = lane; a < m; a += 32) {
      const u32 e = in[b + a];
      const u64 key = order_key(e, pre);
      int r = 0;
      for (int k = 0; k < m; k++) r += order_key(in[b + k], pre) < key;
      out[b + r] = e;
    }
  }
}

// The same order as a 32-bit key, (loop << 27) | pre, for trees of fewer
// than 2^27 cells (the common case): rank sort with the keys read four at a
// time and two entries ranked per pass, half the shared memory of the
// 64-bit version (so more warps per SM).
__device__ __forceinline__ u32 order_key32(u32 e, const int *pre) {
  const u32 img = e >> IMG_SHIFT;
  const u32 x = img % 3, y = (img / 3) % 3, z = img / 9;
  return ((x * 9 + y * 3 + z) << 27) | (u32)pre[e & IDX_MASK];
}

constexpr int SEG32_SMEM = 512;  // keys per warp held in shared memory

__global__ void __launch_bounds__(SEG_WARPS * 32) k_order_segments32(const int *off, int ncells, const u32 *in,
                                                                    u32 *out, const int *pre) {
  __shared__ __align__(16) u32 keys[SEG_WARPS][SEG32_SMEM];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * SEG_WARPS + wid;
  if (w >= ncells) return;
  const int b = off[w], m = off[w + 1] - b;
  if (m > SEG32_SMEM) {  // long segments: rank from global memory
    for (int a = lane; a < m; a += 32) {
      const u32 e = in[b + a], key = order_key32(e, pre);
      int r = 0;
      for (int k = 0; k < m; k++) r += order_key32(in[b + k], pre) < key;
      out[b + r] = e;
    }
    return;
  }
  const int m4 = (m + 3) & ~3;  // padded with keys that rank below none
  for (int a = lane; a < m4; a += 32) keys[wid][a] = a < m ? order_key32(in[b + a], pre) : 0xFFFFFFFFu;
  __syncwarp();
  const uint4 *k4 = (const uint4 *)keys[wid];
  for (int a = lane; a < m; a += 64) {
    const bool two = a + 32 < m;
    const u32 key0 = keys[wid][a], key1 = two ? keys[wid][a + 32] : 0u;
    int r0 = 0, r1 = 0;
    for (int k = 0; k < m4 / 4; k++) {
      const uint4 q = k4[k];
      r0 += (q.x < key0) + (q.y < key0) + (q.z < key0) + (q.w < key0);
      r1 += (q.x < key1) + (q.y < key1) + (q.z < key1) + (q.w < key1);
    }
    out[b + r0] = in[b + a];
    if (two) out[b + r1] = in[b + a + 32];
  }
}

// Blocks of one wave of the walk: as many as are resident on the GPU at once.
int walk_blocks(Handle &h, bool periodic) {
  if (h.nsm == 0) FMM_CUDA(cudaDeviceGetAttribute(&h.nsm, cudaDevAttrMultiProcessorCount, h.prm.device));
  int occ = 1;
  FMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &occ, periodic ? k_walk<WALK_PAIRS, true> : k_walk<WALK_PAIRS, false>, TB, 0));
  return h.nsm * std::max(occ, 1);
}

}  // namespace

// CSR by target from the raw (target, source) pairs.  With `order` the
// entries of each target are put in the reference's recording order;
// without it they stay in arrival order (not deterministic) until
// order_m2l_lists() runs.
static void bucket(Handle &h, const int2 *raw, unsigned long long *n_dev, int64_t n, Buf &off_b, Buf &ent_b,
                   bool order) {
  cudaStream_t s = h.stream;
  const int C = h.ncells;
  off_b.need((size_t)(C + 1) * 4);
  ent_b.need((size_t)(n > 0 ? n : 1) * 4 * 2);
  h.fill.need((size_t)(C + 1) * 4);
  int *cnt = h.fill.as<int>();
  FMM_CUDA(cudaMemsetAsync(cnt, 0, (size_t)(C + 1) * 4, s));
  const int g = 148 * 8;
  k_count_tgt<<<g, TB, 0, s>>>(raw, n_dev, (u64)n, cnt);
  scan_exclusive_int(h, cnt, off_b.as<int>(), C + 1, nullptr);
  FMM_CUDA(cudaMemsetAsync(cnt, 0, (size_t)(C + 1) * 4, s));
  u32 *tmp = ent_b.as<u32>() + (n > 0 ? n : 1);
  k_bucket<<<g, TB, 0, s>>>(raw, n_dev, (u64)n, off_b.as<int>(), cnt, order ? tmp : ent_b.as<u32>());
  h.launches += 2;
  if (order) {
    if (C < (1 << 27))
      k_order_segments32<<<grid_for(C, SEG_WARPS), SEG_WARPS * 32, 0, s>>>(off_b.as<int>(), C, tmp,
                                                                          ent_b.as<u32>(), h.c_pre.as<int>());
    else
      k_order_segments<<<grid_for(C, SEG_WARPS), SEG_WARPS * 32, 0, s>>>(off_b.as<int>(), C, tmp, ent_b.as<u32>(),
                                                                        h.c_pre.as<int>());
    h.launches++;
  }
  FMM_LAUNCH();
}

// The M2L lists as CSR by target in the reference's order, built from the
// walk's raw entries when first needed.
void order_m2l_lists(Handle &h) {
  if (h.m2l_ordered) return;
  bucket(h, h.m2l_raw.as<int2>(), &h.counters.as<DevCounters>()->n_m2l, h.n_m2l, h.m2l_off, h.m2l_ent, true);
  h.m2l_ordered = true;
}

void build_lists(Handle &h) {
  cudaStream_t s = h.stream;
  h.g_plan.valid = false;  // new lists: the M2L grouping is redone
  DevCounters *ctr = h.counters.as<DevCounters>();
  const int C = h.ncells;
  // capacities: kept between calls, never below a size estimate for this tree
  h.frontier_cap = std::max<size_t>(h.frontier_cap, (size_t)C * 256 + 4096);
  h.m2l_cap = std::max<size_t>(h.m2l_cap, (size_t)C * 200 + 1024);
  h.p2p_cap = std::max<size_t>(h.p2p_cap, (size_t)h.nleaves * 90 + 1024);
  const int images = h.prm.images;
  const long ks = key_space(images, h.depth);
  h.g_occ.need((size_t)ks * sizeof(int) * 2 + 64);  // key occupancy, then its scan
  h.g_cnt.need((size_t)C * sizeof(int) * 2 + 64);           // targets with grouped entries, then tile slots
  int *occ = h.g_occ.as<int>(), *gflag = h.g_cnt.as<int>();
  for (int attempt = 0;; attempt++) {
    h.frontier[0].need(h.frontier_cap * sizeof(int2));
    h.frontier[1].need(h.frontier_cap * sizeof(int2));
    h.m2l_raw.need(h.m2l_cap * sizeof(int2));
    h.p2p_raw.need(h.p2p_cap * sizeof(int2));
    FMM_CUDA(cudaMemsetAsync(&ctr->n_m2l, 0, sizeof(unsigned long long) * 5, s));  // list and frontier counts
    FMM_CUDA(cudaMemsetAsync(&ctr->list_overflow, 0, sizeof(int), s));
    FMM_CUDA(cudaMemsetAsync(&ctr->walk_resid, 0, sizeof(int), s));
    // group keys of the M2L entries, and the keys and targets that occur
    h.m2l_key.need(h.m2l_cap * sizeof(int));
    FMM_CUDA(cudaMemsetAsync(occ, 0, (size_t)ks * sizeof(int), s));
    FMM_CUDA(cudaMemsetAsync(gflag, 0, (size_t)C * sizeof(int), s));
    k_seed<<<grid_for(std::max(h.nsys, 32), 256), 256, 0, s>>>(h.frontier[0].as<int2>(), &ctr->frontier[0], images,
                                                                h.nsys, h.prm.dim == 2 ? 2 : 3);
    h.launches++;
    CellView cv{h.c_xr.as<double4>(), h.c_child.as<int>(), h.c_nchild.as<int>()};
    const int steps = 2 * h.depth + 3;
    const int walk_grid = walk_blocks(h, images != 0);
    auto walk = images != 0 ? k_walk<WALK_PAIRS, true> : k_walk<WALK_PAIRS, false>;
    // frontier counters rotate over three words: step st reads word st % 3,
    // appends to (st + 1) % 3 (zeroed by step st - 1, or above) and zeroes
    // (st + 2) % 3
    for (int st = 0; st < steps; st++) {
      const int a = st & 1, b = a ^ 1;
      walk<<<walk_grid, TB, 0, s>>>(cv, h.frontier[a].as<int2>(), &ctr->frontier[st % 3], h.frontier[b].as<int2>(),
                                    &ctr->frontier[(st + 1) % 3], &ctr->frontier[(st + 2) % 3], h.frontier_cap,
                                    h.m2l_raw.as<int2>(), &ctr->n_m2l, h.m2l_cap, h.p2p_raw.as<int2>(), &ctr->n_p2p,
                                    h.p2p_cap, h.prm.theta, images ? h.prm.cycle : 0.0, h.depth, &ctr->list_overflow,
                                    h.m2l_key.as<int>(), occ, gflag, &ctr->walk_resid);
      h.launches++;
      FMM_LAUNCH();
    }
    FMM_CUDA(cudaMemcpyAsync(&h.hc, ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
    FMM_CUDA(cudaStreamSynchronize(s));
    if (h.hc.list_overflow) {
      // a dropped frontier pair also hides its descendants' entries: grow
      // everything and walk again
      if (attempt >= 4) throw Error{EXAFMM_ERR_CAPACITY, "interaction list buffers kept overflowing"};
      h.m2l_cap = std::max<size_t>(2 * h.m2l_cap, (size_t)(h.hc.n_m2l * 5 / 4 + 1024));
      h.p2p_cap = std::max<size_t>(2 * h.p2p_cap, (size_t)(h.hc.n_p2p * 5 / 4 + 1024));
      h.frontier_cap *= 4;
      continue;
    }
    if (h.hc.frontier[steps % 3] != 0)
      throw Error{EXAFMM_ERR_STATE, "dual-tree walk did not finish in 2*depth+3 steps"};
    break;
  }
  h.n_m2l = (int64_t)h.hc.n_m2l;
  h.n_p2p = (int64_t)h.hc.n_p2p;
  // The grouped M2L reads the raw entries in any order, so the M2L lists
  // become per-target CSR in the reference's order only when something reads
  // that order: an export, the direct-form kernel, or residual entries.  The
  // P2P lists are ordered always: their order is the near field's summation
  // order, which keeps results reproducible.
  h.m2l_ordered = false;
  if (h.force_direct_m2l || h.prm.dim == 2) order_m2l_lists(h);
  bucket(h, h.p2p_raw.as<int2>(), &ctr->n_p2p, h.n_p2p, h.p2p_off, h.p2p_ent, true);
}

// Lists in the reference's cell numbering (host arrays, CSR over ref index).
void export_lists(Handle &h, int *m2l_off, int *m2l_src, int *m2l_img, int *p2p_off, int *p2p_src, int *p2p_img) {
  order_m2l_lists(h);
  // the ordering runs on the handle's (non-blocking) stream: the plain
  // copies below must wait for it
  FMM_CUDA(cudaStreamSynchronize(h.stream));
  const int C = h.ncells;
  std::vector<int> ref(C), moff(C + 1), poff(C + 1);
  std::vector<u32> ment(h.n_m2l > 0 ? h.n_m2l : 1), pent(h.n_p2p > 0 ? h.n_p2p : 1);
  FMM_CUDA(cudaMemcpy(ref.data(), h.c_ref.p, C * 4, cudaMemcpyDeviceToHost));
  FMM_CUDA(cudaMemcpy(moff.data(), h.m2l_off.p, (C + 1) * 4, cudaMemcpyDeviceToHost));
  FMM_CUDA(cudaMemcpy(poff.data(), h.p2p_off.p, (C + 1) * 4, cudaMemcpyDeviceToHost));
  if (h.n_m2l) FMM_CUDA(cudaMemcpy(ment.data(), h.m2l_ent.p, h.n_m2l * 4, cudaMemcpyDeviceToHost));
  if (h.n_p2p) FMM_CUDA(cudaMemcpy(pent.data(), h.p2p_ent.p, h.n_p2p * 4, cudaMemcpyDeviceToHost));
  std::vector<int> bfs_of_ref(C);
  for (int b = 0; b < C; b++) bfs_of_ref[ref[b]] = b;
  // image index of the reference's variant: 3D periodic1D, or in 2D
  // (ix+1) + 3 (iy+1), the 3D index of an in-plane image minus 9
  const int img0 = h.prm.dim == 2 ? 9 : 0;
  int a = 0, q = 0;
  for (int r = 0; r < C; r++) {
    const int b = bfs_of_ref[r];
    m2l_off[r] = a;
    p2p_off[r] = q;
    for (int k = moff[b]; k < moff[b + 1]; k++, a++) {
      m2l_src[a] = ref[ment[k] & IDX_MASK];
      m2l_img[a] = (int)(ment[k] >> IMG_SHIFT) - img0;
    }
    for (int k = poff[b]; k < poff[b + 1]; k++, q++) {
      p2p_src[q] = ref[pent[k] & IDX_MASK];
      p2p_img[q] = (int)(pent[k] >> IMG_SHIFT) - img0;
    }
  }
  m2l_off[C] = a;
  p2p_off[C] = q;
}

}  // namespace fmm
