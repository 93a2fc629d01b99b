// Grouped M2L: the translation as dense contractions of precomputed operators
// (3d/kernel.h:233-260 is the per-pair operator being grouped).
//
// Scaling makes one operator serve every level.  With M~_n = M_n / R_s^n,
// L~_j = L_j * R_t^(j+1), r_f the radius of the finer of target and source,
// and v = (X_t - X_s) / r_f (an exact integer vector: level-l centres sit at
// X0 + odd * R0/2^l), the truncated M2L becomes
//   L~_j^k = sum_{n,m} s(j,k,m) rho^n 2^(d'(j+1)) Z_{j+n}^{m-k}(v) A~_n^m,
// rho = 2^max(0, lt-ls), d' = max(0, ls-lt): the operator depends only on the
// group key (lt - ls, v).  Realified (2x2 real blocks per complex input
// with conj(M) folded in), it is a 2NT x 2NT real matrix, zero for j+n >= P.
//
// Pipeline per evaluation:
//   keys       the walk's key of every M2L entry, or k_gkeys (ordered
//              lists; mixed-form periodic entries, where image entries with
//              a tiny fractional offset become ghost-source entries with
//              free-space keys); periodic image entries carry the image and
//              level in their key; far-out offsets or level gaps beyond the
//              key range stay "residual" and are done by the direct-form
//              kernel; occupancy of the key space;
//   scan       group ids of the occupied keys;
//   k_gops     the realified operator of every group not yet cached (FP64;
//              k_gops16: FP16 hi/lo images for the tensor core);
//   tiles      targets with grouped entries sorted by (level, child rank) and
//              cut into tiles (32 targets for DMMA, 128 for tcgen05); the
//              (tile, group) pairs that hold entries are marked, scanned into
//              segment ids and filled with the source cell of every tile slot;
//   k_gemm64   one CTA (8 warps) per tile: for each group of the tile, the
//              operator and the 32 gathered scaled multipoles are copied into
//              shared memory with cp.async (two stages: the next group's
//              copies run under this group's contraction), accumulated with
//              FP64 DMMA (mma.m8n8k4) in registers; then the warps' pieces
//              are reduced, unscaled and stored in L;
//   k_m2l_tc   the mixed form's contraction on tcgen05 (below).
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "fmm.cuh"
#include "harmonics.cuh"
#include "group_key.cuh"
#include "m2l_group.h"
#include "tc.cuh"
#include "translations.cuh"

namespace fmm {

void m2l_residual(Handle &h, const int *ekey);  // m2l.cu

namespace {

constexpr int TB = 256;
constexpr int IMG_SHIFT = 26;
constexpr u32 IDX_MASK = (1u << IMG_SHIFT) - 1;
// Row stride (doubles) of the FP64 contraction's staged multipoles: target
// rows of KP values, padded to 4 mod 16 so that the DMMA B-fragment reads
// (8 rows x 4 consecutive k per instruction) take the minimum two wavefronts.
__host__ __device__ constexpr int gp_kpad(int KP) { return KP + 4; }  // KP is a multiple of 16
static_assert(GP_WARPS * 32 == GP_TILE * 8, "k_gemm64 copies each staged row with 8 threads");
constexpr int TC_TILE = 128;    // targets per tile on the tensor core (MMA M)
constexpr int TC_EPI_WARPS = 4; // warps 0-3: epilogue (warp w owns TMEM lanes 32w..32w+31)
constexpr int TC_LOAD_WARP = 4; // first of the producer warps
constexpr int TC_LOAD_WARPS = 4;
constexpr int TC_MMA_WARP = TC_LOAD_WARP + TC_LOAD_WARPS;  // MMA issuer, TMEM owner
constexpr int TC_THREADS = 32 * (TC_MMA_WARP + 1);
constexpr int TC_MAX_STAGES = 4;  // pipeline stages (groups in flight), as many as shared memory holds
// Groups accumulated in FP32 in tensor memory before the partial sum is
// folded into the compensated running sum.  The tensor core's FP32
// accumulation truncates toward zero, so with same-signed contributions (all
// charges positive) its error is a bias that grows with the MMAs per window:
// measured on 200,000 Plummer bodies at P = 12, the local expansions' mean
// relative error was -1.6e-6 over 16 groups, -4.1e-7 over two and -2.9e-7
// over one (potential error 2.7x, 1.22x and 1.15x FP64's).  Defaults, from
// measurements at 1M uniform bodies: P <= 10 (two accumulators in tensor
// memory) two groups, 3.45 ms per evaluation at P = 10 against 3.39 with 16;
// P = 11, 12 (one accumulator and the running sum in tensor memory) one
// group, 4.59 ms at P = 12 against 4.53; larger P (windows added to L in
// global memory, where every window costs a read-modify-write) four.  A
// wider window, set with exafmm_b200_set_tile, trades accuracy for time.
int default_flush(int P) { return P <= 10 ? 2 : (P <= 12 ? 1 : 4); }
// Limit of every wait of the tensor-core kernel (the drain of copies and MMAs
// already in flight gets twice as long): a wait that runs out flags
// EXAFMM_ERR_TIMEOUT instead of hanging the GPU.
constexpr long TC_WAIT_NS = 2000000000L;
// group keys read back with the counts (more take a second read)
constexpr int OP_KEYS_HOST = 8192;

// Group key of every M2L entry of the ordered CSR lists (expanded to pairs);
// marks the keys that occur and the targets that have grouped entries.  (The
// walk does the same for its raw entries.)
// With `gscan` (mixed form, periodic): an image entry that has a ghost takes
// the ghost's free-space key, and its source becomes the ghost's multipole
// row, ncells + ghost index.
__global__ void k_gkeys(long n, int2 *pairs, const double4 *xr, const int *level, int *ekey, int *occ,
                        int *gflag, int *nres, double cycle, int depth, const int *gscan, int ncells) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int key = -1;
  if (e < n) {
    const int2 pr = pairs[e];
    const int t = pr.x & (int)IDX_MASK, img = (int)((u32)pr.x >> IMG_SHIFT), s = pr.y;
    if (img == 13) {
      key = m2l_group_key(xr[t], xr[s], level[t] - level[s]);
    } else {
      long gslot = -1;
      double3 shift;
      if (gscan) key = m2l_ghost_key(xr[t], xr[s], level[t] - level[s], img, s, xr[0].w, cycle, depth, &gslot, &shift);
      if (key >= 0) pairs[e] = make_int2(pr.x, ncells + gscan[gslot]);
      else key = m2l_image_key(xr[t], xr[s], level[t] - level[s], img, xr[0].w, cycle, depth);
    }
    if (key >= 0) m2l_mark_key(key, t, occ, gflag);
    ekey[e] = key;
  }
  const int nr = __syncthreads_count(e < n && key < 0);  // one atomic per block
  if (threadIdx.x == 0 && nr) atomicAdd(nres, nr);
}

// Ghost slots used by the image entries (see m2l_ghost_key).
__global__ void k_ghost_mark(long n, const int2 *pairs, const double4 *xr, const int *level, double cycle, int depth,
                             int *gmark) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int2 pr = pairs[e];
  const int t = pr.x & (int)IDX_MASK, img = (int)((u32)pr.x >> IMG_SHIFT), s = pr.y;
  if (img == 13) return;
  long gslot = -1;
  double3 shift;
  if (m2l_ghost_key(xr[t], xr[s], level[t] - level[s], img, s, xr[0].w, cycle, depth, &gslot, &shift) >= 0 &&
      gmark[gslot] == 0)
    gmark[gslot] = 1;
}

// The slot of every ghost, in slot order.
__global__ void k_ghost_list(long nslots, const int *gmark, const int *gscan, int *gslots) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nslots && gmark[i]) gslots[gscan[i]] = (int)i;
}

// CSR lists expanded to (target | img << 26, source) pairs in list order.
__global__ void k_csr_pairs(int ncells, const int *off, const u32 *ent, int2 *pairs) {
  const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (c >= ncells) return;
  for (int e = off[c] + lane; e < off[c + 1]; e += 32) {
    const u32 en = ent[e];
    pairs[e] = make_int2(c | (int)((en >> IMG_SHIFT) << IMG_SHIFT), (int)(en & IDX_MASK));
  }
}

__global__ void k_key_of_gid(long nkeys, const int *occ, const int *gidx, int *key_of) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nkeys && occ[k]) key_of[gidx[k]] = (int)k;
}

struct PlanDev {
  int P, NT, KP, nrb, wsize, maxrank, maxp;
  const int *woff, *jmin, *pieces, *prank;
};

// Geometry an operator key needs: the root radius and the period (image
// keys), the tree depth (image key slots).
struct KeyGeom {
  const double4 *xr;  // xr[0].w: root radius
  double cycle;
  int depth;
};

// Irregular harmonics of the group's offset (an integer vector, or for an
// image key its exact fractional offset) into shared memory (threads m < P
// build column m); returns the level difference.
__device__ int group_harmonics(int key, int P, double2 *Zsh, KeyGeom kg) {
  double vx, vy, vz;
  const int dl = m2l_key_offset(key, key < KEY_SPACE ? 1.0 : kg.xr[0].w, kg.cycle, kg.depth, vx, vy, vz);
  if (threadIdx.x < P) {
    const Sph sg = sph_of(vx, vy, vz);
    const int m = threadIdx.x;
    irregular_column(m, P, sg.r, sg, [&](int n, double2 z) { Zsh[tri(n) + m] = z; });
  }
  __syncthreads();
  return dl;
}

// Entry (row, col) of the realified, scaled operator (zero outside 2NT x 2NT
// and outside the truncation j + n < P).
__device__ double op_value(int row, int col, int P, int NT, int dl, const double2 *Zsh) {
  if (row >= 2 * NT || col >= 2 * NT) return 0.0;
  const int o = row >> 1, cr = row & 1;
  int j = 0;
  while (tri(j + 1) <= o) j++;
  const int kk = o - tri(j);
  const int ci = col >> 1, cc = col & 1;
  int n = 0;
  while (tri(n + 1) <= ci) n++;
  const int mu = ci - tri(n);
  if (j + n > P - 1) return 0.0;
  const int d = j + n;
  const double rho = dl > 0 ? (double)(1 << dl) : 1.0;  // source coarser: R_s / r_f
  const int dp = dl < 0 ? -dl : 0;                        // source finer: R_t / r_f = 2^dp
  const double f = pow(rho, (double)n) * pow(2.0, (double)(dp * (j + 1))) * ((j & 1) ? -1.0 : 1.0);
  // T(m) = sigma(kk, m) * f * Z_d^{m - kk}
  auto T = [&](int m) {
    const int e = m < 0 ? 0 : (m <= kk ? m : kk);
    const int om = m - kk;
    double2 z = Zsh[tri(d) + (om < 0 ? -om : om)];
    if (om < 0) z.y = -z.y;
    const double s = ((e & 1) ? -1.0 : 1.0) * f;
    return make_double2(s * z.x, s * z.y);
  };
  const double2 tp = T(mu);
  const double2 tm = mu > 0 ? T(-mu) : make_double2(0, 0);
  if (cr == 0 && cc == 0) return tp.x + tm.x;
  if (cr == 0 && cc == 1) return -(tp.y - tm.y);
  if (cr == 1 && cc == 0) return tp.y + tm.y;
  return tp.x - tm.x;
}

// One CTA per group: the realified, scaled operator in row-block layout.
__global__ void k_gops(const int *keys, const int *slots, PlanDev pd, double *ops, KeyGeom kg) {
  extern __shared__ double2 Zsh[];  // NT irregular harmonics of v
  const int dl = group_harmonics(keys[blockIdx.x], pd.P, Zsh, kg);
  double *W = ops + (size_t)slots[blockIdx.x] * pd.wsize;
  for (int i = threadIdx.x; i < pd.wsize; i += blockDim.x) {
    int rb = 0;
    while (pd.woff[rb + 1] <= i) rb++;
    const int li = i - pd.woff[rb];
    W[i] = op_value(rb * 8 + (li & 7), li >> 3, pd.P, pd.NT, dl, Zsh);
  }
}

// Tensor-core layout of the operators.  Output rows (N) are cut into blocks
// of 64, one MMA N per block; a block whose smallest output order is j only
// reads inputs of order n < P - j (the operator is zero beyond), so it keeps
// 16 * ksteps input columns.  Each block is stored K-major with the 128-byte
// swizzle: atoms of 64 input columns, each atom `rows` x 128 bytes.  The
// multipole tile (A) is 128 rows x atomsA atoms, hi and lo parts.
//
// The operator image (hi and lo parts, 2 * bimg bytes, one bulk copy) holds
// the blocks one after the other.  A block's region holds its hi atoms and
// its lo atoms: all hi atoms then all lo atoms, or -- a "paired" block --
// each hi atom followed by its lo atom, so that the hi and lo rows form one
// B operand of 2 * rows rows: one MMA then makes hi*hi and hi*lo together
// (A read once), into 2 * rows accumulator columns (the products of the hi
// rows, then those of the lo rows, added by the epilogue), and the lo*hi
// MMA adds into the second half.  Block b's accumulator columns start at
// dcol[b].  A "narrow" block (after the first, fewer than four K steps, so
// less than one 64-column atom: the high output orders need only the low
// input orders) is stored in the 32-byte swizzle instead: per K step the
// block's rows x 32 bytes, the two 16-byte chunks of a row swapped where the
// row's bit 2 is set -- no padding to 128-byte rows to copy.
struct TcPlan {
  int nb;                            // output row blocks
  int rows[4], ksteps[4];            // rows, K steps of 16
  int boff[4];                       // byte offset of the block's region in the image
  int astride[4], lodelta[4];        // bytes from one hi atom to the next; from a hi atom to its lo atom
  int pair[4];                       // paired block
  int narrow[4];                     // block in the 32-byte swizzle (one rows x 32-byte slab per K step)
  int dcol[4];                       // first accumulator column
  int accw;                          // accumulator columns
  int bimg;                          // half the bytes of the operator image
  int atomsA;                        // 64-column atoms of the multipole tile
  int abytes;                        // bytes of one (hi or lo) multipole tile
};

constexpr int tc_tri(int n) { return n * (n + 1) / 2; }

// pair_first: block 0 is paired (the orders whose accumulators leave room)
constexpr TcPlan make_tc_plan(int P, int KP, bool pair_first) {
  TcPlan t{};
  t.nb = (KP + 63) / 64;
  int off = 0, col = 0;
  for (int b = 0; b < t.nb; b++) {
    t.rows[b] = KP - 64 * b < 64 ? KP - 64 * b : 64;
    int j = 0;
    while (tc_tri(j + 1) <= 32 * b) j++;  // order of the block's first output
    const int kreal = 2 * tc_tri(P - j);
    const int k16 = (kreal + 15) / 16 * 16;
    t.ksteps[b] = (k16 < KP ? k16 : KP) / 16;
    const int natoms = (t.ksteps[b] + 3) / 4, ab = t.rows[b] * 128;
    t.pair[b] = pair_first && b == 0;
    t.narrow[b] = b > 0 && t.ksteps[b] < 4;
    t.boff[b] = off;
    if (t.narrow[b]) {
      t.astride[b] = t.rows[b] * 32;  // bytes per K step
      t.lodelta[b] = t.ksteps[b] * t.rows[b] * 32;
      off += 2 * t.ksteps[b] * t.rows[b] * 32;
    } else {
      t.astride[b] = t.pair[b] ? 2 * ab : ab;
      t.lodelta[b] = t.pair[b] ? ab : natoms * ab;
      off += 2 * natoms * ab;
    }
    t.dcol[b] = col;
    col += (t.pair[b] ? 2 : 1) * t.rows[b];
  }
  t.accw = col;
  t.bimg = off / 2;
  t.atomsA = (KP + 63) / 64;
  t.abytes = TC_TILE * 128 * t.atomsA;
  return t;
}

// Orders whose block 0 is paired: P = 8 and 10, where two accumulators of
// the wider block 0 and an FP32 running sum fit in TMEM.
constexpr bool tc_pair_first(int P) { return P == 8 || P == 10; }

constexpr size_t TC_SMEM_MAX = 227 * 1024;  // opt-in shared memory per CTA on sm_100

constexpr int tc_kp(int P) { return (P * (P + 1) + 15) / 16 * 16; }
constexpr size_t tc_stage_bytes(const TcPlan &t) { return 2 * (size_t)t.abytes + 2 * (size_t)t.bimg; }
// + 1024 to align the stages to the swizzle atom, + 256 for the barriers and the TMEM slot
constexpr size_t TC_SMEM_EXTRA = 1024 + 256;
// as many stages as fit, at most TC_MAX_STAGES
constexpr int tc_stages(const TcPlan &t) {
  int n = 1;
  while (n < TC_MAX_STAGES && (n + 1) * tc_stage_bytes(t) + TC_SMEM_EXTRA <= TC_SMEM_MAX) n++;
  return n;
}
constexpr size_t tc_smem(const TcPlan &t) { return tc_stages(t) * tc_stage_bytes(t) + TC_SMEM_EXTRA; }

// Tensor-memory layout of the accumulators (columns; 128 lanes = targets):
// nacc accumulators of KP columns `stride` apart, used in turn, one per
// window (the tensor core fills one while the epilogue folds another; with
// one, the tensor core waits for each fold).  fold = 1: the double-FP32
// running sum at columns [hi, hi + KP) and [lo, lo + KP); fold = 2: an FP32
// running sum at [hi, hi + KP) (round-to-nearest adds); fold = 0: windows are
// added to L in global memory.  ncols is the allocation (a power of two).
struct TcAcc {
  int nacc, fold;
  uint32_t stride, hi, lo, ncols;
};
constexpr int TC_MAX_ACC = 3;

// columns of one TMEM accumulator: a power of two >= KP (and >= 32)
constexpr uint32_t tc_half_cols(int KP) {
  uint32_t c = 32;
  while (c < (uint32_t)KP) c <<= 1;
  return c;
}

// Two accumulators and the running sum where they fit (KP up to 128: P <=
// 10), else one accumulator and the running sum (3 x KP rounded to 32
// columns within 512: P = 11, 12), else windows added to L in global memory.
constexpr TcAcc tc_acc_layout(int KP) {
  const uint32_t hc = tc_half_cols(KP), k32 = ((uint32_t)KP + 31u) / 32u * 32u;
  if (4 * hc <= 512) return TcAcc{2, 1, hc, 2 * hc, 3 * hc, 4 * hc};
  if (3 * k32 <= 512) return TcAcc{1, 1, 0, k32, 2 * k32, 512};
  return TcAcc{2, 0, hc, 0, 0, 2 * hc};
}

// Orders compiled with their plan: three accumulators, so that a fold has
// two windows' time before the tensor core needs its accumulator again --
// with the double-FP32 running sum where five fit (KP <= 64), else (KP <=
// 128) with an FP32 running sum.  The window sums carry the tensor core's
// truncating FP32 accumulation, which the short window bounds; the running
// sum's round-to-nearest adds are unbiased, ~sqrt(windows) * 2^-24 relative
// (about 6e-7 over the ~95 windows of a tile at P = 10, far below the
// expansion's error).  Otherwise the layout above.
constexpr TcAcc tc_acc_fixed(int KP, const TcPlan &t) {
  if (t.pair[0]) {  // two accumulators of the paired width (64-column steps) and an FP32 running sum
    const uint32_t st = ((uint32_t)t.accw + 63u) / 64u * 64u;
    if (2 * st + (uint32_t)KP <= 512) return TcAcc{2, 3, st, 2 * st, 0, 512};
  }
  const uint32_t hc = tc_half_cols(KP);
  if (5 * hc <= 512) return TcAcc{3, 1, hc, 3 * hc, 4 * hc, 5 * hc <= 256 ? 256u : 512u};
  if (4 * hc <= 512) return TcAcc{3, 2, hc, 3 * hc, 0, 512};
  return tc_acc_layout(KP);
}

// The orders compiled with their plan as constants (6, 8, 10 and 12, the
// switch in contract()): the MMA issue loop and the producers' copy loop
// unroll with immediate offsets, so the issuing thread and the producers
// spend fewer instructions per segment.  Other orders take the plan at run
// time.
template <int PT>
struct TcFixed {
  static constexpr int KP = tc_kp(PT);
  static constexpr TcPlan plan = make_tc_plan(PT, KP, tc_pair_first(PT));
  static constexpr int nstage = tc_stages(plan);
  static constexpr TcAcc acc = tc_acc_fixed(KP, plan);
};

// One CTA per group: the operator split into FP16 hi + lo parts, written as
// the byte image the MMA reads from shared memory (hi image, then lo image).
__global__ void k_gops16(const int *keys, const int *slots, int P, TcPlan pl, __half *ops16, KeyGeom kg) {
  extern __shared__ double2 Zsh[];
  const int NT = tri(P);
  const int dl = group_harmonics(keys[blockIdx.x], P, Zsh, kg);
  const int nh = pl.bimg / 2;  // halves per image
  __half *Wh = ops16 + (size_t)slots[blockIdx.x] * 2 * nh;  // the whole image (hi and lo parts)
  for (int e = threadIdx.x; e < nh; e += blockDim.x) {
    const int byte = 2 * e;
    // `byte` enumerates the hi values block by block, atom by atom; its hi
    // and lo values go to their places in the block's region
    auto hsize = [&](int q) {  // bytes of block q's hi part
      return pl.narrow[q] ? pl.ksteps[q] * pl.rows[q] * 32 : (pl.ksteps[q] + 3) / 4 * pl.rows[q] * 128;
    };
    int b = 0, lb = 0;  // block, and its first byte in this enumeration
    while (b + 1 < pl.nb && lb + hsize(b) <= byte) {
      lb += hsize(b);
      b++;
    }
    const int rem = byte - lb;
    int rb, k, ph;  // output row in the block, input column, the hi value's byte in the image
    if (pl.narrow[b]) {  // undo the 32-byte swizzle
      const int ts = rem / (pl.rows[b] * 32), w = rem - ts * (pl.rows[b] * 32);
      rb = w >> 5;
      k = ts * 16 + ((((w >> 4) & 1) ^ ((rb >> 2) & 1)) << 3) + ((w >> 1) & 7);
      ph = pl.boff[b] + rem;
    } else {  // undo the 128-byte swizzle
      const int ab = pl.rows[b] * 128, a = rem / ab, r2 = rem - a * ab;
      const int chunk = (r2 >> 4) & 7, q = (r2 >> 1) & 7;
      rb = r2 >> 7;
      k = a * 64 + ((chunk ^ (rb & 7)) << 3) + q;
      ph = pl.boff[b] + a * pl.astride[b] + r2;
    }
    const double w = k < 16 * pl.ksteps[b] ? op_value(64 * b + rb, k, P, NT, dl, Zsh) : 0.0;
    const __half hi = __double2half(w);
    Wh[ph / 2] = hi;
    Wh[(ph + pl.lodelta[b]) / 2] = __double2half(w - (double)__half2float(hi));
  }
}

// Scaled multipoles split into FP16 hi + lo rows (KP values per cell each).
// Scaled, realified multipole entry k of cell c: M[c][n,m] / R_c^n, k = 2*(tri(n)+m)+{0,1}.
__device__ __forceinline__ double mscaled(int c, int k, int NT, const double4 *xr, const double2 *M) {
  if (k >= 2 * NT) return 0.0;
  const int ci = k >> 1;
  int n = 0;
  while (tri(n + 1) <= ci) n++;
  const double inv = 1.0 / xr[c].w;
  double s = 1;
  for (int q = 0; q < n; q++) s *= inv;
  const double2 m = M[(long)c * NT + ci];
  return (k & 1 ? m.y : m.x) * s;
}

// Scaled, realified multipoles: Mt[c][k] (FP64 form).
__global__ void k_mscale(int ncells, int P, int KP, const double4 *xr, const double2 *M, double *Mt) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)ncells * KP) return;
  const int c = (int)(i / KP), k = (int)(i - (long)c * KP);
  Mt[i] = mscaled(c, k, tri(P), xr, M);
}

// Degree n of coefficient index ci (tri(n) <= ci < tri(n + 1)) and 1 / R^n.
__device__ __forceinline__ double mscale_factor(int ci, double R) {
  int n = (int)((sqrtf(8.0f * ci + 1.0f) - 1.0f) * 0.5f);
  while (tri(n) > ci) n--;
  while (tri(n + 1) <= ci) n++;
  const double inv = 1.0 / R;
  double s = 1, b = inv;  // inv^n
  for (int e = n; e; e >>= 1, b *= b)
    if (e & 1) s *= b;
  return s;
}

// Power-of-two exponent E of the FP16 split: the largest scaled multipole
// times 2^E lies in [2^14, 2^15), so every source's leading coefficients are
// normal FP16 numbers with an 11-bit lo part below them, whatever the scale
// of the charges (charges of 1/N put a leaf's monopole below FP16's smallest
// normal number), and nothing reaches FP16's largest (65504).
__device__ __forceinline__ int m16_exponent(unsigned long long bits) {
  const double mx = __longlong_as_double((long long)bits);
  if (!(mx > 0.0) || !isfinite(mx)) return 0;
  const int e = 14 - ilogb(mx);
  return e < -500 ? -500 : (e > 500 ? 500 : e);
}

// Largest |real or imaginary part| of the scaled multipoles M_n / R^n over
// the cells that can be M2L sources (every level but the roots'), into
// *mx as double bits (non-negative doubles order like their bit patterns).
__global__ void k_m16_max(int ncells, int P, const double4 *xr, const int *level, const double2 *M,
                          unsigned long long *mx) {
  const int NT = tri(P);
  double v = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < (long)ncells * NT;
       i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i / NT), ci = (int)(i - (long)c * NT);
    if (level[c] == 0) continue;
    const double2 m = M[i];
    const double s = mscale_factor(ci, xr[c].w);
    v = fmax(v, fmax(fabs(m.x), fabs(m.y)) * s);
  }
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __shared__ double wmax[TB / 32];
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = fmax(v, wmax[w]);
    if (v > 0.0) atomicMax(mx, (unsigned long long)__double_as_longlong(v));
  }
}

// Mixed form: the scaled multipoles, times 2^E (m16_exponent), split into
// FP16 hi and lo parts (M16[c][0..KP) hi, M16[c][KP..2KP) lo), written
// directly; one thread per coefficient (n, m) writes its real and imaginary
// parts.
__global__ void k_mscale16(int ncells, int P, int KP, const double4 *xr, const double2 *M,
                           const unsigned long long *mx, __half2 *M16) {
  const int half_kp = KP / 2;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)ncells * half_kp) return;
  const long c = i / half_kp;
  const int ci = (int)(i - c * half_kp), NT = tri(P);
  double2 v = make_double2(0, 0);
  if (ci < NT) {
    const double s = scalbn(mscale_factor(ci, xr[c].w), m16_exponent(*mx));
    const double2 m = M[c * NT + ci];
    v = make_double2(m.x * s, m.y * s);
  }
  const __half hx = __double2half(v.x), hy = __double2half(v.y);
  __half2 *row = M16 + c * KP;  // KP half2 = 2 KP halves: hi then lo
  row[ci] = __halves2half2(hx, hy);
  row[half_kp + ci] = __halves2half2(__double2half(v.x - (double)__half2float(hx)),
                                     __double2half(v.y - (double)__half2float(hy)));
}

// Harmonics of the ghost shifts: the shift of image img at finer level lf is
// f m, f = rint(s) - s with s the image's offset in cell units and m the
// level's cell radius R0 / 2^lf, the same for every ghost of (img, lf).  A
// warp per (img, lf), lane m < P generating column m: Y[(ic * nlev + lf) * NT].
__global__ void __launch_bounds__(32) k_ghost_harm(int nlev, const double4 *xr, int P, double cycle, double2 *Y) {
  const int key = blockIdx.x, ic = key / nlev, lf = key % nlev, lane = threadIdx.x;
  const int NT = tri(P);
  const int img = ic < 13 ? ic : ic + 1;
  const double R0 = xr[0].w, m = scalbn(R0, -lf);
  const int ix = img % 3 - 1, iy = (img / 3) % 3 - 1, iz = img / 9 - 1;
  const double sx = image_shift_units(ix, lf, R0, cycle), sy = image_shift_units(iy, lf, R0, cycle),
               sz = image_shift_units(iz, lf, R0, cycle);
  const Sph sg = sph_of((rint(sx) - sx) * m, (rint(sy) - sy) * m, (rint(sz) - sz) * m);
  double2 *row = Y + (size_t)key * NT;
  if (lane < P) regular_column(lane, P, sg.r, sg, sg.e, [&](int n, double2 y, double2) { row[tri(n) + lane] = y; });
}

// A warp per ghost (GH_WARPS per block): the source's multipole moved by the
// M2M shift f r onto the ghost centre (3d/kernel.h:204-231 for one child,
// offset ghost - source = f r, with the shift's harmonics from
// k_ghost_harm), scaled like k_mscale16 (1 / R^n, times 2^E) and split into
// the ghost's FP16 hi / lo row, M16[ncells + g].
constexpr int GH_WARPS = 8;
__global__ void __launch_bounds__(GH_WARPS * 32) k_ghost16(int nghost, const int *gslots, const double4 *xr,
                                                           const double2 *M, const double2 *Yh, int nlev, int P,
                                                           int KP, const unsigned long long *mx, int ncells,
                                                           __half2 *M16) {
  extern __shared__ double2 gsh[];  // per warp: the source multipole
  const int NT = tri(P), wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = blockIdx.x * GH_WARPS + wp;
  if (g >= nghost) return;  // warp-uniform; the kernel has no block barrier
  double2 *Msh = gsh + (size_t)wp * NT;
  const int slot = gslots[g];
  const int s = slot / GHOST_SLOTS, ic = (slot % GHOST_SLOTS) / 4, dlf = slot % 4;
  const double4 Y = xr[s];
  const double R0 = xr[0].w, m = scalbn(Y.w, -dlf);
  const int lf = ilogb(R0) - ilogb(m);
  const double2 *Ysh = Yh + (size_t)(ic * nlev + lf) * NT;
  for (int k = lane; k < NT; k += 32) Msh[k] = M[(long)s * NT + k];
  __syncwarp();
  const double E = scalbn(1.0, m16_exponent(*mx));
  const int half_kp = KP / 2;
  __half2 *row = M16 + (long)(ncells + g) * KP;
  for (int ci = lane; ci < half_kp; ci += 32) {
    double2 v = make_double2(0, 0);
    if (ci < NT) {
      const int j = order_of(ci), k = ci - tri(j);
      const double2 mm = m2m_coeff(j, k, Msh, Ysh);
      const double sc = mscale_factor(ci, Y.w) * E;
      v = make_double2(mm.x * sc, mm.y * sc);
    }
    const __half hx = __double2half(v.x), hy = __double2half(v.y);
    row[ci] = __halves2half2(hx, hy);
    row[half_kp + ci] = __halves2half2(__double2half(v.x - (double)__half2float(hx)),
                                       __double2half(v.y - (double)__half2float(hy)));
  }
}

__global__ void k_tkeys(int ncells, const int *gflag, const int *level, const int *parent, const int *child,
                        u64 *keys, u32 *vals, int *counts) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const bool f = c < ncells && gflag[c];
  if (c < ncells) {
    const int pa = parent[c];
    const int cls = pa < 0 ? 0 : c - child[pa];
    keys[c] = f ? (u64)(level[c] * 8 + cls) : 255ull;
    vals[c] = (u32)c;
  }
  const int nf = __syncthreads_count(f);
  if (threadIdx.x == 0 && nf) atomicAdd(&counts[1], nf);
}

__global__ void k_tiles(int ntiles, int tile_n, int nflag, const u32 *sorted, int *tile_tgt, int *tslot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntiles * tile_n) return;
  if (i < nflag) {
    const int c = (int)sorted[i];
    tile_tgt[i] = c;
    tslot[c] = i;
  } else {
    tile_tgt[i] = -1;
  }
}

// (tile, group) segments without sorting: mark every (tile, group) pair
// that holds a grouped entry, scan the marks into segment ids (tiles in
// order, groups in order within a tile), then write each entry's source into
// its segment's slot.  A target has at most one entry per group, so every
// (segment, slot) is written once.
__global__ void k_gmark(long n, const int2 *pairs, const int *ekey, const int *gidx, const int *tslot, int tile_n,
                        int ngroups, int *mark) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || ekey[e] < 0) return;
  const int t = pairs[e].x & (int)IDX_MASK;
  mark[(long)(tslot[t] / tile_n) * ngroups + gidx[ekey[e]]] = 1;
}

__global__ void k_gfill(long n, const int2 *pairs, const int *ekey, const int *gidx, const int *tslot, int tile_n,
                        int ngroups, const int *segid, int *tg_src) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || ekey[e] < 0) return;
  const int2 pr = pairs[e];
  const int ts = tslot[pr.x & (int)IDX_MASK];
  const int sg = segid[(long)(ts / tile_n) * ngroups + gidx[ekey[e]]];
  tg_src[(long)sg * tile_n + ts % tile_n] = pr.y;
}

// Every marked (tile, group): its segment's operator slot in the cache.
__global__ void k_seg_gid(long nmark, int ngroups, const int *mark, const int *segid, const int *slot_of_gid,
                          int *tg_gid) {
  const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < nmark && mark[r]) tg_gid[segid[r]] = slot_of_gid[(int)(r % ngroups)];
}

// The rows of the segments that exist (count on the device) set to -1.
__global__ void k_fill_rows(int *tg_src, const int *nseg, int tile_n) {
  const long n = (long)*nseg * tile_n;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) tg_src[i] = -1;
}

// First segment of every tile (the exclusive scan at the tile's first
// group), and the end.
__global__ void k_tg_off(int ntiles, int ngroups, const int *segid, const int *nseg, int *tg_off) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < ntiles) tg_off[t] = segid[(long)t * ngroups];
  if (t == ntiles) tg_off[t] = *nseg;
}



__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Largest tile t < ntiles with tg_off[t] <= s (the tile holding segment s,
// for s below the segment count).
__device__ __forceinline__ int tile_at(const int *tg_off, int ntiles, int s) {
  int lo = 0, hi = ntiles - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tg_off[mid] <= s) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// First segment of CTA c of G when nseg segments are cut into equal ranges.
__device__ __forceinline__ int range_start(int nseg, int c, int G) { return (int)((long long)nseg * c / G); }

// MAXP: the plan's pieces per warp (pd.maxp); at GP_MAXP_SMALL the
// accumulators leave registers for two CTAs per SM.
template <int MAXP>
__global__ void __launch_bounds__(GP_WARPS * 32, MAXP == GP_MAXP_SMALL ? 2 : 1)
    k_gemm64(const int *tile_tgt, const int *tg_off, const int *tg_gid, const int *tg_src, const double *ops,
             const double *Mt, const double4 *xr, double2 *L, PlanDev pd, int nstage, int ntiles, double2 *part) {
  extern __shared__ __align__(16) double smd[];  // nstage x (operator, gathered multipoles); then the reduction
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int pc[MAXP], wo[MAXP];
#pragma unroll
  for (int p = 0; p < MAXP; p++) {
    pc[p] = pd.pieces[warp * MAXP + p];
    wo[p] = pc[p] >= 0 ? pd.woff[pc[p] & 255] : 0;
  }
  double acc[MAXP][4][2];
  const int KP = pd.KP;
  const int KPAD = gp_kpad(KP);
  const size_t sstride = (size_t)pd.wsize + (size_t)GP_TILE * KPAD;  // doubles per stage (even: 16-byte rows)
  const int ar = lane >> 2, ak = lane & 3;
  // group g's operator and its 32 gathered multipoles into stage b, as
  // asynchronous copies (absent targets: zeros).  The multipoles stay in
  // rows (target-major, X[col][k]): each source row, KP contiguous doubles,
  // is copied in 16-byte chunks by 8 threads (thread t: row t / 8, chunks
  // t % 8, t % 8 + 8, ...), one index load per row.
  const int xcol = tid >> 3, xpart = tid & 7;
  auto issue = [&](int g, int b) {
    double *Wd = smd + (size_t)b * sstride, *Xd = Wd + pd.wsize;
    const double *Wg = ops + (size_t)tg_gid[g] * pd.wsize;
    for (int i = tid; i < pd.wsize / 2; i += blockDim.x) tc::cp_async16(Wd + 2 * i, Wg + 2 * i, 16u);
    const int s = tg_src[(long)g * GP_TILE + xcol];
    const double *src = Mt + (long)(s >= 0 ? s : 0) * KP;
    double *dst = Xd + xcol * KPAD;
    for (int c = xpart; c < KP / 2; c += 8) tc::cp_async16(dst + 2 * c, src + 2 * c, s >= 0 ? 16u : 0u);
    tc::cp_async_commit();
  };
  // this CTA's segments [r0, r1): with `part`, an equal range of all the
  // segments (tiles cut by a range boundary are written to `part` and added
  // by k_m2l_join, as in k_m2l_tc); else tile blockIdx.x
  int r0, r1, tfirst;
  if (part) {
    const int nseg = tg_off[ntiles];
    r0 = range_start(nseg, blockIdx.x, gridDim.x);
    r1 = range_start(nseg, blockIdx.x + 1, gridDim.x);
    tfirst = r1 > r0 ? tile_at(tg_off, ntiles, r0) : ntiles;
  } else {
    tfirst = blockIdx.x;
    r0 = tg_off[tfirst];
    r1 = tg_off[tfirst + 1];
  }
  for (int tile = tfirst; tile < ntiles; tile++) {
  const int g0 = max(r0, tg_off[tile]), g1 = min(r1, tg_off[tile + 1]);
  if (g0 >= r1) break;
  if (g1 <= g0) continue;  // no segments: L stays zero
#pragma unroll
  for (int p = 0; p < MAXP; p++)
#pragma unroll
    for (int cb = 0; cb < 4; cb++) acc[p][cb][0] = acc[p][cb][1] = 0;
  if (nstage == 2) issue(g0, 0);
  for (int g = g0; g < g1; g++) {
    // two stages: the next group's copies run while this one is contracted
    const int b = nstage == 2 ? (g - g0) & 1 : 0;
    if (nstage != 2) {
      issue(g, 0);
      tc::cp_async_wait_all();
    } else if (g + 1 < g1) {
      issue(g + 1, b ^ 1);
      tc::cp_async_wait_1();
    } else {
      tc::cp_async_wait_all();
    }
    __syncthreads();
    const double *Wsm = smd + (size_t)b * sstride, *Xsm = Wsm + pd.wsize;
#pragma unroll
    for (int p = 0; p < MAXP; p++) {
      if (pc[p] < 0) continue;
      const int k0 = (pc[p] >> 8) & 4095, k1 = pc[p] >> 20;
      const double *Wb = Wsm + wo[p];
      for (int k = k0; k < k1; k += 4) {
        const double a = Wb[(k + ak) * 8 + ar];
        const double *xb = Xsm + ar * KPAD + k + ak;
#pragma unroll
        for (int cb = 0; cb < 4; cb++) dmma(acc[p][cb][0], acc[p][cb][1], a, xb[cb * 8 * KPAD]);
      }
    }
    __syncthreads();  // stage b is free for group g + 2
  }
  // reduce the pieces into Y[row][col] (rank 0 stores, higher ranks add)
  double *Y = smd;
  __syncthreads();
  for (int rank = 0; rank <= pd.maxrank; rank++) {
#pragma unroll
    for (int p = 0; p < MAXP; p++) {
      if (pc[p] < 0 || pd.prank[warp * MAXP + p] != rank) continue;
      const int rb = pc[p] & 255;
#pragma unroll
      for (int cb = 0; cb < 4; cb++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          double &y = Y[(rb * 8 + ar) * GP_TILE + cb * 8 + ak * 2 + h];
          y = rank == 0 ? acc[p][cb][h] : y + acc[p][cb][h];
        }
    }
    __syncthreads();
  }
  // unscale (L = L~ / R_t^(j+1)) and store, or write the part
  const bool whole = tg_off[tile] >= r0 && tg_off[tile + 1] <= r1;
  double2 *slot = whole ? nullptr : part + (size_t)(2 * blockIdx.x + (tile == tfirst ? 0 : 1)) * GP_TILE * pd.NT;
  for (int i = tid; i < GP_TILE * pd.NT; i += blockDim.x) {
    const int col = i / pd.NT, o = i - col * pd.NT;
    const int t = tile_tgt[tile * GP_TILE + col];
    if (t < 0) continue;
    int j = 0;
    while (tri(j + 1) <= o) j++;
    const double inv = 1.0 / xr[t].w;
    double s = inv;
    for (int q = 0; q < j; q++) s *= inv;
    const double2 v = make_double2(Y[(2 * o) * GP_TILE + col] * s, Y[(2 * o + 1) * GP_TILE + col] * s);
    if (whole) L[(long)t * pd.NT + o] = v;
    else slot[i] = v;
  }
  __syncthreads();  // the next tile's copies reuse the reduction's shared memory
  }
}

// Mixed form on the tensor core: one CTA per tile of 128 targets, warp
// specialised.  For every group of the tile the operator (B: N = output rows
// in blocks of 64, K-truncated per block) and the 128 gathered scaled
// multipoles (A: 128 targets x KP inputs), both as FP16 hi + lo parts in the
// 128-byte swizzled K-major layout, are staged in shared memory, and one
// thread issues the three products hi*hi + hi*lo + lo*hi per K step of 16
// (tcgen05.mma kind::f16), accumulating in FP32 in tensor memory.
//   producer warps: per group, wait for its stage to be free, then one bulk
//     copy (operator) and 16-byte cp.async copies of the gathered multipole
//     rows land on the stage's barriers; two stages;
//   MMA warp: waits for the stage, issues the MMAs, commits the stage back;
//     two TMEM accumulators alternate every `flush_every` groups;
//   epilogue warps: fold each finished accumulator into a double-FP32
//     running sum in TMEM (or into L when TMEM has no room) while the tensor
//     core fills the other, so no FP32 sum runs over more than `flush_every`
//     groups; finally store L in FP64.
// Every mbarrier wait is bounded; a role that times out flags the error and
// stops, the others time out in turn, in-flight copies and MMAs are drained
// (bounded) and TMEM is freed.
// Accumulator epilogues.  Row = target t of this thread (TMEM lane).
// tc_fold adds the FP32 accumulator into a double-FP32 running sum (hi, lo)
// kept in TMEM beside it: Knuth's TwoSum per element, error terms summed in
// lo, so the running sum carries ~48 bits.
__device__ __forceinline__ void tc_fold(uint32_t acc, uint32_t hi, uint32_t lo, int cb, int ce) {
  for (int c0 = cb; c0 < ce; c0 += 16) {
    uint32_t a[16], h[16], l[16];
    tc::ld_32x32b_x16_async(acc + (uint32_t)c0, a);
    tc::ld_32x32b_x16_async(hi + (uint32_t)c0, h);
    tc::ld_32x32b_x16_async(lo + (uint32_t)c0, l);
    tc::wait_ld();
#pragma unroll
    for (int k = 0; k < 16; k++) {
      const float x = __uint_as_float(a[k]), s0 = __uint_as_float(h[k]);
      const float sum = s0 + x, bp = sum - s0;
      const float e = (s0 - (sum - bp)) + (x - bp);
      h[k] = __float_as_uint(sum);
      l[k] = __float_as_uint(__uint_as_float(l[k]) + e);
    }
    tc::st_32x32b_x16(hi + (uint32_t)c0, h);
    tc::st_32x32b_x16(lo + (uint32_t)c0, l);
  }
  tc::wait_st();
}

// tc_fold with an FP32 running sum (round-to-nearest adds, no error term).
__device__ __forceinline__ void tc_fold32(uint32_t acc, uint32_t hi, int cb, int ce) {
  for (int c0 = cb; c0 < ce; c0 += 16) {
    uint32_t a[16], h[16];
    tc::ld_32x32b_x16_async(acc + (uint32_t)c0, a);
    tc::ld_32x32b_x16_async(hi + (uint32_t)c0, h);
    tc::wait_ld();
#pragma unroll
    for (int k = 0; k < 16; k++) h[k] = __float_as_uint(__uint_as_float(h[k]) + __uint_as_float(a[k]));
    tc::st_32x32b_x16(hi + (uint32_t)c0, h);
  }
  tc::wait_st();
}

// tc_fold32 for a plan with paired blocks: output column c of block b is
// the sum of accumulator columns dcol[b] + w and, paired, dcol[b] + rows[b]
// + w (w = c - 64 b).
__device__ __forceinline__ void tc_fold_paired(uint32_t acc, uint32_t sum, const TcPlan &pl, int KP) {
  for (int c0 = 0; c0 < KP; c0 += 16) {
    const int b = c0 >> 6, w = c0 - 64 * b;
    const uint32_t big = acc + (uint32_t)(pl.dcol[b] + w);
    uint32_t a[16], m[16], h[16];
    tc::ld_32x32b_x16_async(big, a);
    if (pl.pair[b]) tc::ld_32x32b_x16_async(big + (uint32_t)pl.rows[b], m);
    tc::ld_32x32b_x16_async(sum + (uint32_t)c0, h);
    tc::wait_ld();
    if (!pl.pair[b])
#pragma unroll
      for (int k = 0; k < 16; k++) m[k] = 0u;
#pragma unroll
    for (int k = 0; k < 16; k++)
      h[k] = __float_as_uint(__uint_as_float(h[k]) + (__uint_as_float(a[k]) + __uint_as_float(m[k])));
    tc::st_32x32b_x16(sum + (uint32_t)c0, h);
  }
  tc::wait_st();
}

__device__ __forceinline__ void tc_zero(uint32_t cols, int cb, int ce) {
  const uint32_t z[16] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int c0 = cb; c0 < ce; c0 += 16) tc::st_32x32b_x16(cols + (uint32_t)c0, z);
  tc::wait_st();
}

// Stores the running sum as the FP64 local expansion, unscaled
// (L = L~ / R_t^(j+1), and the split's 2^E removed: us = 2^-E).  The tile is
// the only grouped writer of its targets.
__device__ __forceinline__ void tc_store(uint32_t hi, uint32_t lo, bool has_lo, int t, double inv, double us, int cb,
                                         int ce, int NT, double2 *L) {
  int j = 0;
  double sj = inv * us;  // us * inv^(j+1)
  for (int c0 = cb; c0 < ce; c0 += 16) {
    uint32_t h[16], l[16];
    tc::ld_32x32b_x16_async(hi + (uint32_t)c0, h);
    if (has_lo) tc::ld_32x32b_x16_async(lo + (uint32_t)c0, l);
    tc::wait_ld();
    if (t < 0) continue;
    if (!has_lo)
#pragma unroll
      for (int k = 0; k < 16; k++) l[k] = 0u;
    for (int k = 0; k < 16; k += 2) {
      const int o = (c0 + k) >> 1;
      if (o >= NT) break;
      while (tri(j + 1) <= o) {
        j++;
        sj *= inv;
      }
      const double re = (double)__uint_as_float(h[k]) + (double)__uint_as_float(l[k]);
      const double im = (double)__uint_as_float(h[k + 1]) + (double)__uint_as_float(l[k + 1]);
      L[(long)t * NT + o] = make_double2(re * sj, im * sj);
    }
  }
}

// Without room in TMEM for the running sum (KP > 128): the accumulator is
// added into the FP64 L in global memory, eight independent
// read-modify-writes at a time.
__device__ __forceinline__ void tc_flush_global(uint32_t acc, int t, double inv, double us, int cb, int ce, int NT,
                                                double2 *L) {
  int j = 0;
  double sj = inv * us;
  for (int c0 = cb; c0 < ce; c0 += 16) {
    float v[16];
    tc::ld_32x32b_x16(acc + (uint32_t)c0, v);
    if (t < 0) continue;
    double2 cur[8];
    double sc[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int o = (c0 >> 1) + k;
      sc[k] = 0;
      if (o < NT) {
        while (tri(j + 1) <= o) {
          j++;
          sj *= inv;
        }
        sc[k] = sj;
        cur[k] = L[(long)t * NT + o];
      }
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int o = (c0 >> 1) + k;
      if (o < NT)
        L[(long)t * NT + o] =
            make_double2(cur[k].x + (double)v[2 * k] * sc[k], cur[k].y + (double)v[2 * k + 1] * sc[k]);
    }
  }
}

// PT > 0: the order PT with its plan and stage count as compile-time
// constants (the run-time arguments are then ignored); PT = 0: any order.
// Work split of the orders compiled with their plan and a running sum in
// TMEM ("balanced"): one CTA per SM, each taking an equal contiguous range of
// the (tile, group) segments -- the tiles hold 182 to 325 segments at 1M
// uniform bodies, and with two tiles per SM the SM that drew the longest
// ones set the kernel's time (720 us against 557 us of average SM work).  A
// CTA stores the tiles that lie wholly in its range; of a tile cut by a
// range boundary it writes its partial sums to `part` (slot 0: its first
// tile, 1: its last), which k_m2l_join adds in CTA order (deterministic).
// Otherwise one CTA per tile.
template <int PT>
__global__ void __launch_bounds__(TC_THREADS, 1) k_m2l_tc(const int *tile_tgt, const int *tg_off, const int *tg_gid,
                                                          const int *tg_src, const unsigned char *ops,
                                                          const __half *M16, const double4 *xr, double2 *L, int P_,
                                                          int KP_, TcPlan pl_,
                                                          int nstage_, TcAcc ta_, int flush_every,
                                                          const unsigned long long *m16_max, int *err, long wait_ns,
                                                          long stall_ns, int ntiles, double2 *part) {
  constexpr bool FIX = PT > 0;
  constexpr bool BAL = FIX && TcFixed<PT>::acc.fold != 0;
  const int P = FIX ? PT : P_, KP = FIX ? TcFixed<PT>::KP : KP_, nstage = FIX ? TcFixed<PT>::nstage : nstage_;
  const TcPlan pl = FIX ? TcFixed<PT>::plan : pl_;
  const TcAcc ta = FIX ? TcFixed<PT>::acc : ta_;
  extern __shared__ __align__(1024) unsigned char smraw[];
  unsigned char *base = smraw + ((1024u - (tc::smem_u32(smraw) & 1023u)) & 1023u);  // swizzle atoms: 1024-aligned
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t abytes = (uint32_t)pl.abytes, bimg = (uint32_t)pl.bimg;
  const uint32_t stage_bytes = 2 * abytes + 2 * bimg;  // A hi, A lo, B hi, B lo
  uint64_t *full = (uint64_t *)(base + (size_t)nstage * stage_bytes);  // [stage] multipoles landed (producer warps)
  uint64_t *bful = full + TC_MAX_STAGES;                               // [stage] operator landed (bulk copy bytes)
  uint64_t *empty = bful + TC_MAX_STAGES;                              // [stage] MMAs reading the stage finished
  uint64_t *accf = empty + TC_MAX_STAGES;                              // [acc] accumulator window complete
  uint64_t *acce = accf + TC_MAX_ACC;                                  // [acc] accumulator folded, reusable
  uint64_t *stall = acce + TC_MAX_ACC;  // nothing arrives here (the stall test hook waits on it)
  uint32_t *tslot = (uint32_t *)(stall + 1);
  volatile int *abort = (volatile int *)(tslot + 1);  // a role gave up: the others stop waiting
  const uint32_t ncols = ta.ncols;
  const int fold = ta.fold;
  // window w uses accumulator a = w % nacc for the u-th time, u = w / nacc
  // (both kept as counters): its barriers complete once per use
  if (warp == TC_MMA_WARP) tc::alloc(tslot, ncols);
  if (tid == 0) {
    for (int b = 0; b < TC_MAX_STAGES; b++) {
      tc::mbar_init(&full[b], TC_LOAD_WARPS * 32);
      tc::mbar_init(&bful[b], 1);
      tc::mbar_init(&empty[b], 1);
    }
    for (int b = 0; b < TC_MAX_ACC; b++) {
      tc::mbar_init(&accf[b], 1);
      tc::mbar_init(&acce[b], TC_EPI_WARPS);
    }
    tc::mbar_init(stall, 1);
    *abort = 0;
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tslot;
  // this CTA's segments [g0, g1) and the first tile they touch
  int g0, g1, tfirst;
  if (BAL) {
    const int nseg = tg_off[ntiles];
    g0 = range_start(nseg, blockIdx.x, gridDim.x);
    g1 = range_start(nseg, blockIdx.x + 1, gridDim.x);
    tfirst = g1 > g0 ? tile_at(tg_off, ntiles, g0) : 0;
  } else {
    tfirst = blockIdx.x;
    g0 = tg_off[tfirst];
    g1 = tg_off[tfirst + 1];
  }
  const int n = g1 - g0;
  auto parity = [&](int k) { return (uint32_t)(k / nstage) & 1u; };

  if (warp < TC_EPI_WARPS) {
    // ---- epilogue: warp w owns TMEM lanes 32w.. = targets 32w..; per tile
    // of the range, its windows (as the MMA issuer closes them: every
    // flush_every groups and at the tile's last group in the range)
    const double us = scalbn(1.0, -m16_exponent(*m16_max));
    const int NT = tri(P);
    const uint32_t lanes = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t sum_hi = lanes + ta.hi, sum_lo = lanes + ta.lo;
    bool ok = true;
    int a = 0, u = 0;  // accumulator of the next window, and its use count
    for (int tt = tfirst; ok && n > 0 && tt < ntiles; tt++) {
      const int ts = max(g0, tg_off[tt]), te = min(g1, tg_off[tt + 1]);
      if (ts >= g1) break;
      if (te <= ts) continue;  // a tile without segments
      const int t = tile_tgt[tt * TC_TILE + tid];
      const double inv = t >= 0 ? 1.0 / xr[t].w : 0.0;
      if (fold) tc_zero(sum_hi, 0, KP);
      if (fold == 1) tc_zero(sum_lo, 0, KP);
      const int nwin = (te - ts + flush_every - 1) / flush_every;
      for (int w = 0; w < nwin; w++) {
        ok = __all_sync(0xffffffffu, tc::mbar_wait(&accf[a], (uint32_t)u & 1u, wait_ns, abort));
        if (!ok) break;
        tc::fence_after();
        const uint32_t acc = lanes + (uint32_t)a * ta.stride;
        if (fold == 1) tc_fold(acc, sum_hi, sum_lo, 0, KP);
        else if (fold == 2) tc_fold32(acc, sum_hi, 0, KP);
        else if (fold == 3) tc_fold_paired(acc, sum_hi, pl, KP);
        else tc_flush_global(acc, t, inv, us, 0, KP, NT, L);
        tc::fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&acce[a]);
        if (++a == ta.nacc) {
          a = 0;
          u++;
        }
      }
      if (!ok || !fold) continue;
      if (tg_off[tt] >= g0 && tg_off[tt + 1] <= g1) {
        tc_store(sum_hi, sum_lo, fold == 1, t, inv, us, 0, KP, NT, L);
      } else {  // a part of a tile cut by a range boundary
        double2 *slot = part + (size_t)(2 * blockIdx.x + (tt == tfirst ? 0 : 1)) * TC_TILE * NT;
        tc_store(sum_hi, sum_lo, fold == 1, t >= 0 ? tid : -1, inv, us, 0, KP, NT, slot);
      }
    }
    if (!ok) {
      *abort = 1;
      if (lane == 0) atomicExch(err, 1);
    }
  } else if (warp < TC_LOAD_WARP + TC_LOAD_WARPS) {
    // ---- producers: warp pw copies target rows 32pw..32pw+31 of the tile
    // with cp.async into the swizzled layout.  Lane l takes rows
    // 32pw + (l >> 1) and 32pw + 16 + (l >> 1), and of each source row (the
    // multipole's hi then lo halves, 4 KP contiguous bytes in global memory)
    // the 16-byte chunks of parity l & 1: the two lanes of a pair copy the
    // two halves of every 32-byte sector in the same instruction, so each
    // sector is requested from L2 once (one lane per row requested every
    // sector twice, and the L1-to-L2 request path was the kernel's limit).
    // Absent targets are zero-filled.  Producer thread 0 also starts the
    // operator's bulk copy.  Each thread's copies arrive on the stage's
    // barrier by themselves (cp.async.mbarrier.arrive), so the producers run
    // up to `nstage` groups ahead of the MMAs.  The next group's source rows
    // and operator slot are loaded one group ahead.
    const int pw = warp - TC_LOAD_WARP, par = lane & 1;
    const int ra = 32 * pw + (lane >> 1), rb = ra + 16;
    const int half = KP / 8;  // 16-byte chunks of one half (hi or lo) of a source row; even
    auto src_of = [&](int k) {
      const int *row = tg_src + (long)(g0 + k) * TC_TILE;
      return k < n ? make_int2(row[ra], row[rb]) : make_int2(-1, -1);
    };
    const bool bulk = pw == 0 && lane == 0;  // the thread that starts the operator's bulk copy
    auto gid_of = [&](int k) { return bulk && k < n ? tg_gid[g0 + k] : 0; };
    auto issue = [&](int st, int2 s2, int gid) {
      unsigned char *S = base + (size_t)st * stage_bytes;
      if (bulk) {
        tc::mbar_arrive_expect_tx(&bful[st], 2 * bimg);
        tc::bulk_g2s(S + 2 * abytes, ops + (size_t)gid * 2 * bimg, 2 * bimg, &bful[st]);
      }
      // chunk c = c0 + par with c0 even: half is even, so c0 alone decides
      // the half (hl) and the atom, and the lane's parity only sets bit 4 of
      // the in-row offset (folded into the row's swizzle q)
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int r = j ? rb : ra, s = j ? s2.y : s2.x;
        const __half *src = M16 + (size_t)(s < 0 ? 0 : s) * 2 * KP + par * 8;
        const uint32_t nb = s >= 0 ? 16u : 0u, q = ((uint32_t)par << 4) ^ ((uint32_t)(r & 7) << 4);
        unsigned char *R = S + r * 128;
#pragma unroll
        for (int c0 = 0; c0 < 2 * half; c0 += 2) {
          const int hl = c0 >= half, cc0 = c0 - hl * half;
          const uint32_t off = hl * abytes + (cc0 >> 3) * (TC_TILE * 128) + ((((uint32_t)cc0 & 7) << 4) ^ q);
          tc::cp_async16(R + off, src + c0 * 8, nb);
        }
      }
      tc::cp_async_commit();
    };
    bool ok = true;
    int last = -1, lst = 0;
    int2 s_next = src_of(0);
    int gid_next = gid_of(0);
    // stage st of round rnd = k / nstage (counters, no divisions)
    for (int k = 0, st = 0, rnd = 0; k < n; k++) {
      if (rnd > 0) {  // the stage is free once the MMAs of group k - nstage are done
        ok = __all_sync(0xffffffffu, tc::mbar_wait(&empty[st], (uint32_t)(rnd - 1) & 1u, wait_ns, abort));
        if (!ok) break;
      }
      issue(st, s_next, gid_next);
      tc::cp_async_arrive(&full[st]);  // arrives when this thread's copies have landed
      last = k;
      lst = st;
      s_next = src_of(k + 1);
      gid_next = gid_of(k + 1);
      if (++st == nstage) {
        st = 0;
        rnd++;
      }
    }
    if (!ok) {
      *abort = 1;
      if (lane == 0) atomicExch(err, 1);
    }
    // drain this thread's copies; the operator's bulk copy completes by
    // itself (bounded wait, no abort: the copy must land before exit)
    tc::cp_async_wait_all();
    if (pw == 0 && lane == 0 && last >= 0) tc::mbar_wait(&bful[lst], parity(last), 2 * wait_ns);
  } else if (warp == TC_MMA_WARP) {
    // ---- MMA issuer (one thread): per group and output block, K steps of
    // hi*hi + hi*lo + lo*hi into the window's accumulator
    if (lane == 0) {
      int rows[4], ksteps[4];
      uint32_t boff[4], idesc[4], idesc2[4];
#pragma unroll
      for (int b = 0; b < 4; b++) {
        rows[b] = b < pl.nb ? pl.rows[b] : 0;
        ksteps[b] = b < pl.nb ? pl.ksteps[b] : 0;
        boff[b] = b < pl.nb ? (uint32_t)pl.boff[b] : 0u;
        idesc[b] = tc::idesc_f16_f32(TC_TILE, rows[b] > 0 ? rows[b] : 16);
        idesc2[b] = tc::idesc_f16_f32(TC_TILE, rows[b] > 0 ? 2 * rows[b] : 16);  // paired: hi and lo rows
      }
      // test hook: a wait on a barrier that nothing arrives at, as if the
      // tensor core's inputs never came; it runs out after stall_ns
      bool ok = stall_ns <= 0 || tc::mbar_wait(stall, 0u, stall_ns, abort);
      int last = -1, lst = 0;
      // end of the current tile's segments in the range (a window closes
      // there too)
      int tcur = tfirst, tend = BAL ? min(g1, tg_off[tfirst + 1]) : g1;
      // stage st of round rnd = k / nstage; the window has kf groups so far
      // and uses accumulator a for the u-th time (counters, no divisions)
      for (int k = 0, st = 0, rnd = 0, kf = 0, a = 0, u = 0; ok && k < n; k++) {
        if (BAL && g0 + k >= tend) {  // next tile (skipping tiles without segments)
          do tcur++;
          while (tg_off[tcur + 1] <= g0 + k);
          tend = min(g1, tg_off[tcur + 1]);
        }
        const bool close = kf == flush_every - 1 || g0 + k + 1 == tend;
        const uint32_t ph = (uint32_t)rnd & 1u;
        ok = tc::mbar_wait(&full[st], ph, wait_ns, abort) && tc::mbar_wait(&bful[st], ph, wait_ns, abort);
        // a new window reuses accumulator a once the epilogue has folded
        // its previous use
        if (ok && kf == 0 && u > 0) ok = tc::mbar_wait(&acce[a], (uint32_t)(u - 1) & 1u, wait_ns, abort);
        if (!ok) break;
        tc::fence_after();
        const uint32_t sA = tc::smem_u32(base + (size_t)st * stage_bytes), sB = sA + 2 * abytes;
        const uint64_t dA = tc::smem_desc_sw128(sA), dB = tc::smem_desc_sw128(sB), dB32 = tc::smem_desc_sw32(sB);
        const uint64_t lo_a = abytes >> 4;  // descriptor start fields count 16 bytes
        const bool fresh = kf == 0;
        const uint32_t acc = tmem + (uint32_t)a * ta.stride;
        // per K step: hi*hi, then hi*lo with the same A, then lo*hi (issuing
        // the small products first lowered the truncation bias by a third
        // but cost 15% of the M2L time: consecutive MMAs on one A are faster)
#pragma unroll
        for (int b = 0; b < 4; b++) {
          if (b >= pl.nb) break;
#pragma unroll
          for (int ks = 0; ks < ksteps[b]; ks++) {
            const uint64_t ao = ((uint64_t)(ks >> 2) * (TC_TILE * 128) + (uint64_t)(ks & 3) * 32) >> 4;
            const uint64_t bo =
                pl.narrow[b] ? ((uint64_t)boff[b] + (uint64_t)ks * pl.astride[b]) >> 4
                             : ((uint64_t)boff[b] + (uint64_t)(ks >> 2) * pl.astride[b] + (uint64_t)(ks & 3) * 32) >> 4;
            const uint64_t lo_b = (uint64_t)pl.lodelta[b] >> 4;
            const uint32_t d = acc + (uint32_t)pl.dcol[b];
            if (pl.narrow[b]) {
              tc::mma_f16(d, dA + ao, dB32 + bo, idesc[b], (!fresh || ks > 0) ? 1u : 0u);
              tc::mma_f16(d, dA + ao, dB32 + lo_b + bo, idesc[b], 1u);
              tc::mma_f16(d, dA + lo_a + ao, dB32 + bo, idesc[b], 1u);
            } else if (pl.pair[b]) {  // hi*hi and hi*lo in one MMA (columns [0, rows) and [rows, 2 rows)), then lo*hi
              tc::mma_f16(d, dA + ao, dB + bo, idesc2[b], (!fresh || ks > 0) ? 1u : 0u);
              tc::mma_f16(d + (uint32_t)rows[b], dA + lo_a + ao, dB + bo, idesc[b], 1u);
            } else {
              tc::mma_f16(d, dA + ao, dB + bo, idesc[b], (!fresh || ks > 0) ? 1u : 0u);
              tc::mma_f16(d, dA + ao, dB + lo_b + bo, idesc[b], 1u);
              tc::mma_f16(d, dA + lo_a + ao, dB + bo, idesc[b], 1u);
            }
          }
        }
        tc::commit(&empty[st]);
        if (close) tc::commit(&accf[a]);
        last = k;
        lst = st;
        if (++st == nstage) {
          st = 0;
          rnd++;
        }
        if (close) {
          kf = 0;
          if (++a == ta.nacc) {
            a = 0;
            u++;
          }
        } else {
          kf++;
        }
      }
      if (!ok) {
        *abort = 1;
        atomicExch(err, 1);
      }
      // drain: the MMAs already issued complete by themselves (no abort)
      if (last >= 0) tc::mbar_wait(&empty[lst], parity(last), 2 * wait_ns);
    }
    __syncwarp();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (warp == TC_MMA_WARP) tc::dealloc(tmem, ncols);
}

// Tiles cut by the balanced ranges of k_m2l_tc / k_gemm64 (tiles of tile_n
// targets): L of the tile's targets is the sum of the CTAs' parts, added in
// CTA order.  One CTA per tile; threads run over (target row, coefficient)
// with the coefficient fastest, so the parts and L are read and written
// contiguously.
constexpr int JOIN_T = 256;
__global__ void __launch_bounds__(JOIN_T) k_m2l_join(const int *tile_tgt, const int *tg_off, int ntiles, int G,
                                                     const double2 *part, int NT, int tile_n, double2 *L) {
  const int t = blockIdx.x, nseg = tg_off[ntiles];
  const int a = tg_off[t], b = tg_off[t + 1];
  if (b <= a) return;
  // the CTA whose range holds segment s
  auto cta_of = [&](int s) {
    int c = (int)((long long)s * G / nseg);
    while (c + 1 < G && range_start(nseg, c + 1, G) <= s) c++;
    while (c > 0 && range_start(nseg, c, G) > s) c--;
    return c;
  };
  const int c0 = cta_of(a), c1 = cta_of(b - 1);
  if (c0 == c1) return;  // the tile lies in one range: stored by its CTA
  // the tile is the first tile (slot 0) of every CTA after c0, whose ranges
  // start inside it; for c0 it is the last (slot 1) unless c0's range
  // starts at the tile
  const int slot0 = range_start(nseg, c0, G) < a ? 1 : 0;
  for (int e = threadIdx.x; e < tile_n * NT; e += JOIN_T) {
    const int row = e / NT, o = e - row * NT, tgt = tile_tgt[t * tile_n + row];
    if (tgt < 0) continue;
    double2 sum = make_double2(0, 0);
    for (int c = c0; c <= c1; c++) {
      const int slot = c == c0 ? slot0 : 0;
      const double2 v = part[(size_t)(2 * c + slot) * tile_n * NT + e];
      sum.x += v.x;
      sum.y += v.y;
    }
    L[(long)tgt * NT + o] = sum;
  }
}

struct PlanCache {
  GroupPlan host;
  int *dev = nullptr;
};

PlanCache &plan_cache(int P) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, PlanCache> cache;
  int dev = 0;
  FMM_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_pair(dev, P);
  auto it = cache.find(key);
  if (it == cache.end()) {
    PlanCache pc;
    pc.host = make_group_plan(P);
    if (pc.host.P == P) {
      const GroupPlan &g = pc.host;
      std::vector<int> buf;
      buf.insert(buf.end(), g.woff.begin(), g.woff.end());
      buf.insert(buf.end(), g.jmin.begin(), g.jmin.end());
      buf.insert(buf.end(), g.pieces.begin(), g.pieces.end());
      buf.insert(buf.end(), g.prank.begin(), g.prank.end());
      FMM_CUDA(cudaMalloc(&pc.dev, buf.size() * sizeof(int)));
      FMM_CUDA(cudaMemcpy(pc.dev, buf.data(), buf.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    it = cache.emplace(key, pc).first;
  }
  return it->second;
}

PlanDev plan_dev(const PlanCache &pc) {
  const GroupPlan &g = pc.host;
  PlanDev d;
  d.P = g.P; d.NT = g.NT; d.KP = g.KP; d.nrb = g.nrb; d.wsize = g.wsize; d.maxrank = g.maxrank; d.maxp = g.maxp;
  d.woff = pc.dev;
  d.jmin = d.woff + g.nrb + 1;
  d.pieces = d.jmin + g.nrb;
  d.prank = d.pieces + GP_WARPS * g.maxp;
  return d;
}

size_t gemm64_smem(const GroupPlan &g, int nstage = 1) {
  const size_t stage = (size_t)g.wsize + (size_t)GP_TILE * gp_kpad(g.KP);
  const size_t red = (size_t)g.nrb * 8 * GP_TILE;
  return std::max(nstage * stage, red) * sizeof(double);
}

bool tc_available(int P) {
  const int KP = tc_kp(P);
  return KP <= 256 && tc_smem(make_tc_plan(P, KP, tc_pair_first(P))) <= TC_SMEM_MAX;
}

}  // namespace

int m2l_flush_interval(const Handle &h) { return h.tile_m2l_flush > 0 ? h.tile_m2l_flush : default_flush(h.prm.P); }

bool m2l_grouped_available(int P) {
  PlanCache &pc = plan_cache(P);
  return pc.host.P == P && gemm64_smem(pc.host) <= 200 * 1024;
}

void m2l_grouped_set_attributes() {
  cudaFuncSetAttribute(k_gemm64<GP_MAXP_SMALL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX);
  cudaFuncSetAttribute(k_gemm64<GP_MAXP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX);
  cudaFuncSetAttribute(k_m2l_tc<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX);
  cudaFuncSetAttribute(k_m2l_tc<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX);
  cudaFuncSetAttribute(k_m2l_tc<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX);
  cudaFuncSetAttribute(k_m2l_tc<10>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX);
  cudaFuncSetAttribute(k_m2l_tc<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX);
}

// Grouped M2L of the whole tree: L stored for every cell (zero where no
// M2L entry), residual entries added by the direct-form kernel.  FP64 form:
// DMMA over tiles of 32 targets; mixed form: tcgen05 split-FP16 over tiles of
// 128 targets (orders whose operator does not fit fall back to DMMA).
// The contraction over the grouping held in the handle (tiles, segment
// tables, operator slots) with this evaluation's scaled multipoles.
void contract(Handle &h, bool tcore, const TcPlan &tp, int KP16, const GroupPlan &gp, const PlanDev &pd) {
  cudaStream_t s = h.stream;
  const int P = h.prm.P, ntiles = h.g_ntiles, tile_n = tcore ? TC_TILE : GP_TILE;
  const long nseg = h.g_nseg;
  int *tg_src = h.g_tg.as<int>(), *tg_gid = tg_src + (size_t)nseg * tile_n, *tg_off = tg_gid + nseg;
  DevCounters *ctr = h.counters.as<DevCounters>();
  if (tcore) {
    FMM_CUDA(cudaMemsetAsync(&ctr->tc_error, 0, sizeof(int), s));
    // the orders compiled with their plan as constants; those with a running
    // sum in TMEM take balanced segment ranges, one CTA per SM
    const bool fixed = P == 6 || P == 8 || P == 10 || P == 12;
    const bool bal = fixed && tc_acc_fixed(KP16, tp).fold != 0;
    if (bal && h.nsm == 0) FMM_CUDA(cudaDeviceGetAttribute(&h.nsm, cudaDevAttrMultiProcessorCount, h.prm.device));
    const int G = bal ? std::min(ntiles, h.nsm) : ntiles, NT = tri(P);
    if (bal) h.g_part.need((size_t)G * 2 * TC_TILE * NT * sizeof(double2));
    double2 *part = bal ? h.g_part.as<double2>() : nullptr;
    auto launch = [&](auto kern) {
      kern<<<G, TC_THREADS, tc_smem(tp), s>>>(h.g_tile.as<int>(), tg_off, tg_gid, tg_src, h.g_ops.as<unsigned char>(),
                                              h.g_m16.as<__half>(), h.c_xr.as<double4>(), h.L.as<double2>(), P, KP16,
                                              tp, tc_stages(tp), tc_acc_layout(KP16), m2l_flush_interval(h),
                                              &ctr->m16_max, &ctr->tc_error, TC_WAIT_NS, h.tc_stall_ns, ntiles, part);
    };
    switch (P) {
      case 6: launch(k_m2l_tc<6>); break;
      case 8: launch(k_m2l_tc<8>); break;
      case 10: launch(k_m2l_tc<10>); break;
      case 12: launch(k_m2l_tc<12>); break;
      default: launch(k_m2l_tc<0>);
    }
    if (bal) {
      k_m2l_join<<<ntiles, JOIN_T, 0, s>>>(h.g_tile.as<int>(), tg_off, ntiles, G, part, NT, TC_TILE,
                                          h.L.as<double2>());
      h.launches++;
    }
    h.tc_stall_ns = 0;  // the test hook stalls one launch
    FMM_CUDA(cudaMemcpyAsync(h.flags_host, &ctr->tc_error, sizeof(int), cudaMemcpyDeviceToHost, s));
    h.g_used_tc = true;
  } else {
    // two pipeline stages where they fit in shared memory (P <= 12), else
    // one.  P <= 11: equal segment ranges over as many CTAs as fit on the GPU
    // at once (at 1M uniform bodies 7.82 -> 7.29 ms per evaluation at P = 8,
    // 9.03 -> 8.47 at P = 10, 9.69 -> 9.35 at P = 11); above, one CTA per
    // tile (P = 12, two one-stage CTAs per SM: 9.69 against 9.78 ms with the
    // ranges)
    auto kern = gp.maxp == GP_MAXP_SMALL ? k_gemm64<GP_MAXP_SMALL> : k_gemm64<GP_MAXP>;
    int nst = gemm64_smem(gp, 2) <= TC_SMEM_MAX ? 2 : 1;
    if (nst == 2) {  // one stage where that doubles the CTAs per SM (P = 12: 1 -> 2 CTAs)
      int occ1 = 0, occ2 = 0;
      FMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, kern, GP_WARPS * 32, gemm64_smem(gp, 1)));
      FMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, kern, GP_WARPS * 32, gemm64_smem(gp, 2)));
      if (occ1 >= 2 * occ2) nst = 1;
    }
    const size_t smem = gemm64_smem(gp, nst);
    const bool bal = P <= 11;
    int G = ntiles;
    const int NT = tri(P);
    double2 *part = nullptr;
    if (bal) {
      int occ = 1;
      FMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, GP_WARPS * 32, smem));
      if (h.nsm == 0) FMM_CUDA(cudaDeviceGetAttribute(&h.nsm, cudaDevAttrMultiProcessorCount, h.prm.device));
      G = std::max(1, std::min(ntiles, h.nsm * std::max(occ, 1)));
      h.g_part.need((size_t)G * 2 * GP_TILE * NT * sizeof(double2));
      part = h.g_part.as<double2>();
    }
    kern<<<G, GP_WARPS * 32, smem, s>>>(h.g_tile.as<int>(), tg_off, tg_gid, tg_src, h.g_ops.as<double>(),
                                        h.g_mt.as<double>(), h.c_xr.as<double4>(), h.L.as<double2>(), pd, nst, ntiles,
                                        part);
    if (bal) {
      k_m2l_join<<<ntiles, JOIN_T, 0, s>>>(h.g_tile.as<int>(), tg_off, ntiles, G, part, NT, GP_TILE,
                                          h.L.as<double2>());
      h.launches++;
    }
  }
  h.launches++;
}

void m2l_grouped_pass(Handle &h) {
  cudaStream_t s = h.stream;
  const int P = h.prm.P, NT = tri(P), C = h.ncells;
  PlanCache &pc = plan_cache(P);
  const GroupPlan &gp = pc.host;
  const PlanDev pd = plan_dev(pc);
  const bool tcore = h.prm.precision == EXAFMM_MIXED && tc_available(P);
  const int KP16 = tc_kp(P);
  const TcPlan tp = make_tc_plan(P, KP16, tc_pair_first(P));
  const int tile_n = tcore ? TC_TILE : GP_TILE;
  const long nent = h.n_m2l;
  h.L.need((size_t)C * NT * sizeof(double2));
  FMM_CUDA(cudaMemsetAsync(h.L.p, 0, (size_t)C * NT * sizeof(double2), s));
  h.g_used_tc = false;
  if (nent == 0) return;

  // scaled multipoles: FP64 (DMMA) or FP16 hi/lo (tensor core)
  if (tcore) {
    h.g_m16.need((size_t)C * 2 * KP16 * sizeof(__half));
    u64 *m16_max = &h.counters.as<DevCounters>()->m16_max;
    FMM_CUDA(cudaMemsetAsync(m16_max, 0, sizeof(u64), s));
    k_m16_max<<<std::min<long>(grid_for((long)C * NT, TB), 148 * 8), TB, 0, s>>>(
        C, P, h.c_xr.as<double4>(), h.c_level.as<int>(), h.M.as<double2>(), m16_max);
    k_mscale16<<<grid_for((long)C * (KP16 / 2), TB), TB, 0, s>>>(C, P, KP16, h.c_xr.as<double4>(),
                                                                 h.M.as<double2>(), m16_max, h.g_m16.as<__half2>());
    h.launches++;
  } else {
    h.g_mt.need((size_t)C * gp.KP * sizeof(double));
    k_mscale<<<grid_for((long)C * gp.KP, TB), TB, 0, s>>>(C, P, gp.KP, h.c_xr.as<double4>(), h.M.as<double2>(),
                                                          h.g_mt.as<double>());
  }
  // ghost sources (mixed form, periodic): their rows after the cells' in
  // M16, from this evaluation's multipoles
  const double cyc = h.prm.images ? h.prm.cycle : 0.0;
  auto ghost_rows = [&]() {
    if (h.g_nghost <= 0) return;
    const size_t row = (size_t)2 * KP16 * sizeof(__half);
    if (h.g_m16.bytes < (size_t)(C + h.g_nghost) * row) {  // grown: the cell rows again
      h.g_m16.need((size_t)(C + h.g_nghost) * row);
      k_mscale16<<<grid_for((long)C * (KP16 / 2), TB), TB, 0, s>>>(C, P, KP16, h.c_xr.as<double4>(),
                                                                   h.M.as<double2>(),
                                                                   &h.counters.as<DevCounters>()->m16_max,
                                                                   h.g_m16.as<__half2>());
      h.launches++;
    }
    const long nsl = (long)C * GHOST_SLOTS;
    // the shifts' harmonics, per (image, finer level): levels up to the
    // deepest cell's, whose ghosts sit at most 3 levels below a source
    const int nlev = h.depth + 4;
    h.g_gharm.need((size_t)26 * nlev * NT * sizeof(double2));
    k_ghost_harm<<<26 * nlev, 32, 0, s>>>(nlev, h.c_xr.as<double4>(), P, cyc, h.g_gharm.as<double2>());
    k_ghost16<<<(h.g_nghost + GH_WARPS - 1) / GH_WARPS, GH_WARPS * 32, GH_WARPS * NT * sizeof(double2), s>>>(
        h.g_nghost, h.g_gmark.as<int>() + 2 * nsl, h.c_xr.as<double4>(), h.M.as<double2>(), h.g_gharm.as<double2>(),
        nlev, P, KP16, &h.counters.as<DevCounters>()->m16_max, C, h.g_m16.as<__half2>());
    h.launches += 2;
    FMM_LAUNCH();
  };
  // same lists, P and form as the last grouping: contract directly
  if (h.g_plan.valid && h.g_plan.P == P && h.g_plan.tcore == tcore && h.g_plan.ordered == h.m2l_ordered) {
    ghost_rows();
    if (h.g_ngroups > 0) contract(h, tcore, tp, KP16, gp, pd);
    h.launches++;
    FMM_LAUNCH();
    if (h.g_plan.nres > 0) m2l_residual(h, h.m2l_ordered ? h.g_ekey.as<int>() : h.m2l_key.as<int>());
    return;
  }
  // the entries and their group keys: the walk's raw pairs with the keys
  // (and key / target occupancy) it produced, or the ordered CSR lists
  // expanded (then the entry index is the CSR position the residual kernel
  // reads) with their keys computed here
  const int2 *pairs = h.m2l_raw.as<int2>();
  const int *ekey = h.m2l_key.as<int>();
  const long ks = key_space(h.prm.images, h.depth);
  int *occ = h.g_occ.as<int>(), *gidx = occ + ks;  // sized by build_lists
  int *gflag = h.g_cnt.as<int>(), *tslot = gflag + C;
  DevCounters *ctr = h.counters.as<DevCounters>();
  int *counts = ctr->gcounts;
  FMM_CUDA(cudaMemsetAsync(counts, 0, 4 * sizeof(int), s));
  // keys computed here: for the ordered lists, and for the mixed form's
  // periodic entries (ghost sources change their keys)
  const bool ghosts = tcore && h.prm.images > 0;
  const bool rekey = h.m2l_ordered || ghosts;
  if (rekey) {
    // the grouping's own copy of the pairs (k_gkeys points ghost entries at
    // ghost rows; the lists themselves stay as the walk made them)
    h.g_pairs.need(nent * sizeof(int2));
    if (h.m2l_ordered)
      k_csr_pairs<<<grid_for((long)C * 32, TB), TB, 0, s>>>(C, h.m2l_off.as<int>(), h.m2l_ent.as<u32>(),
                                                            h.g_pairs.as<int2>());
    else
      FMM_CUDA(cudaMemcpyAsync(h.g_pairs.p, h.m2l_raw.p, nent * sizeof(int2), cudaMemcpyDeviceToDevice, s));
    pairs = h.g_pairs.as<int2>();
    h.g_ekey.need(nent * sizeof(int));
    FMM_CUDA(cudaMemsetAsync(occ, 0, (size_t)ks * sizeof(int), s));
    FMM_CUDA(cudaMemsetAsync(gflag, 0, (size_t)C * sizeof(int), s));
    // ghosts: image entries with a tiny fractional offset use free-space
    // keys (mixed form only: the FP64 form keeps the reference's offsets)
    const int *gscan = nullptr;
    FMM_CUDA(cudaMemsetAsync(&ctr->nghost, 0, sizeof(int), s));
    if (ghosts) {
      const long nsl = (long)C * GHOST_SLOTS;
      h.g_gmark.need((size_t)nsl * 3 * sizeof(int) + 64);
      int *gmark = h.g_gmark.as<int>(), *gsc = gmark + nsl, *gslots = gsc + nsl;
      FMM_CUDA(cudaMemsetAsync(gmark, 0, (size_t)nsl * sizeof(int), s));
      k_ghost_mark<<<grid_for(nent, TB), TB, 0, s>>>(nent, h.g_pairs.as<int2>(), h.c_xr.as<double4>(),
                                                     h.c_level.as<int>(), cyc, h.depth, gmark);
      scan_exclusive_int(h, gmark, gsc, nsl, &ctr->nghost);
      k_ghost_list<<<grid_for(nsl, TB), TB, 0, s>>>(nsl, gmark, gsc, gslots);
      gscan = gsc;
      h.launches += 2;
    }
    k_gkeys<<<grid_for(nent, TB), TB, 0, s>>>(nent, h.g_pairs.as<int2>(), h.c_xr.as<double4>(), h.c_level.as<int>(),
                                              h.g_ekey.as<int>(), occ, gflag, &counts[0], cyc, h.depth, gscan, C);
    ekey = h.g_ekey.as<int>();
    h.launches += 2;
  }
  // dense group ids, the key of each, the flagged targets in tile order;
  // then one read of the counts and of the keys (for the operator cache)
  scan_exclusive_int(h, occ, gidx, ks, &counts[2]);
  const long keys_cap = std::max<long>(OP_KEYS_HOST, std::min<long>(ks, nent));
  h.g_keyof.need((size_t)keys_cap * sizeof(int));
  k_key_of_gid<<<grid_for(ks, TB), TB, 0, s>>>(ks, occ, gidx, h.g_keyof.as<int>());
  h.g_tk.need((size_t)C * 2 * (sizeof(u64) + sizeof(u32)) + 64);
  u64 *tk = h.g_tk.as<u64>(), *tk2 = tk + C;
  u32 *tv = (u32 *)(tk2 + C), *tv2 = tv + C;
  k_tkeys<<<grid_for(C, TB), TB, 0, s>>>(C, gflag, h.c_level.as<int>(), h.c_parent.as<int>(), h.c_child.as<int>(),
                                         tk, tv, counts);
  if (!h.keys_host) FMM_CUDA(cudaMallocHost((void **)&h.keys_host, OP_KEYS_HOST * sizeof(int)));
  FMM_CUDA(cudaMemcpyAsync(&h.hc, ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
  FMM_CUDA(cudaMemcpyAsync(h.keys_host, h.g_keyof.p, OP_KEYS_HOST * sizeof(int), cudaMemcpyDeviceToHost, s));
  double4 root{};
  FMM_CUDA(cudaMemcpyAsync(&root, h.c_xr.p, sizeof(double4), cudaMemcpyDeviceToHost, s));
  FMM_CUDA(cudaStreamSynchronize(s));
  const int nres = rekey ? h.hc.gcounts[0] : h.hc.walk_resid;
  const int nflag = h.hc.gcounts[1], ngroups = h.hc.gcounts[2];
  h.g_nghost = rekey ? h.hc.nghost : 0;
  h.launches += 4;
  if (nres > 0 && !h.m2l_ordered) {  // residual entries are summed in list order: order, then start over
    order_m2l_lists(h);
    m2l_grouped_pass(h);
    return;
  }
  h.g_ngroups = ngroups;
  if (ngroups > 0) {
    // operators: cached per handle by group key (they depend only on the key
    // and P); only keys not seen before are built
    const int layout = tcore ? 1 : 0;
    // image keys also depend on the period, the root radius and the depth
    const bool img_geom_changed = h.prm.images > 0 && (h.op_cycle != cyc || h.op_R0 != root.w || h.op_depth != h.depth);
    if (h.op_P != P || h.op_layout != layout || img_geom_changed) {
      h.op_slot.clear();
      h.op_P = P;
      h.op_layout = layout;
    }
    if (h.prm.images > 0) {
      h.op_cycle = cyc;
      h.op_R0 = root.w;
      h.op_depth = h.depth;
    }
    const size_t op_bytes = tcore ? (size_t)2 * tp.bimg : (size_t)gp.wsize * sizeof(double);
    std::vector<int> &key_of = h.op_host_keys;
    key_of.assign(h.keys_host, h.keys_host + std::min(ngroups, OP_KEYS_HOST));
    if (ngroups > OP_KEYS_HOST) {  // more keys than the first read carried
      key_of.resize(ngroups);
      FMM_CUDA(cudaMemcpy(key_of.data() + OP_KEYS_HOST, h.g_keyof.as<int>() + OP_KEYS_HOST,
                          (size_t)(ngroups - OP_KEYS_HOST) * sizeof(int), cudaMemcpyDeviceToHost));
    }
    std::vector<int> &slot_of = h.op_host_slots, &new_keys = h.op_host_new_keys, &new_slots = h.op_host_new_slots;
    slot_of.resize(ngroups);
    new_keys.clear();
    new_slots.clear();
    for (int g = 0; g < ngroups; g++) {
      auto it = h.op_slot.find(key_of[g]);
      if (it == h.op_slot.end()) {
        const int sl = (int)h.op_slot.size();
        it = h.op_slot.emplace(key_of[g], sl).first;
        new_keys.push_back(key_of[g]);
        new_slots.push_back(sl);
      }
      slot_of[g] = it->second;
    }
    const size_t nslots = h.op_slot.size();
    if (nslots * op_bytes > h.g_ops.bytes) {  // grow, keeping the operators built so far
      Buf grown;
      grown.need(std::max(nslots, (size_t)64) * op_bytes * 2);
      if (h.g_ops.p && nslots > new_keys.size())
        FMM_CUDA(cudaMemcpyAsync(grown.p, h.g_ops.p, (nslots - new_keys.size()) * op_bytes, cudaMemcpyDeviceToDevice,
                                 s));
      FMM_CUDA(cudaStreamSynchronize(s));
      h.g_ops.release();
      h.g_ops = grown;
    }
    h.g_slot.need((size_t)(ngroups + 2 * new_keys.size() + 2) * sizeof(int));
    int *d_slot_of = h.g_slot.as<int>(), *d_new_keys = d_slot_of + ngroups,
        *d_new_slots = d_new_keys + new_keys.size();
    FMM_CUDA(cudaMemcpyAsync(d_slot_of, slot_of.data(), (size_t)ngroups * sizeof(int), cudaMemcpyHostToDevice, s));
    if (!new_keys.empty()) {
      FMM_CUDA(cudaMemcpyAsync(d_new_keys, new_keys.data(), new_keys.size() * sizeof(int), cudaMemcpyHostToDevice, s));
      FMM_CUDA(cudaMemcpyAsync(d_new_slots, new_slots.data(), new_slots.size() * sizeof(int), cudaMemcpyHostToDevice,
                               s));
      const KeyGeom kg{h.c_xr.as<double4>(), cyc, h.depth};
      if (tcore)
        k_gops16<<<(int)new_keys.size(), 256, NT * sizeof(double2), s>>>(d_new_keys, d_new_slots, P, tp,
                                                                          h.g_ops.as<__half>(), kg);
      else
        k_gops<<<(int)new_keys.size(), 128, NT * sizeof(double2), s>>>(d_new_keys, d_new_slots, pd,
                                                                        h.g_ops.as<double>(), kg);
      h.launches++;
    }
    // tiles of targets
    const int ntiles = (nflag + tile_n - 1) / tile_n;
    radix_sort_pairs(h, tk, tv, tk2, tv2, C, 0, 8);
    h.g_tile.need((size_t)ntiles * tile_n * sizeof(int) + 64);
    k_tiles<<<grid_for((long)ntiles * tile_n, TB), TB, 0, s>>>(ntiles, tile_n, nflag, tv, h.g_tile.as<int>(), tslot);
    // (tile, group) segments
    const long nmark = (long)ntiles * ngroups;
    h.g_seg.need((size_t)(nmark + 1) * sizeof(int) * 2);
    int *mark = h.g_seg.as<int>(), *segid = mark + nmark + 1;
    FMM_CUDA(cudaMemsetAsync(mark, 0, (size_t)nmark * sizeof(int), s));
    k_gmark<<<grid_for(nent, TB), TB, 0, s>>>(nent, pairs, ekey, gidx, tslot, tile_n, ngroups, mark);
    scan_exclusive_int(h, mark, segid, nmark, &counts[3]);
    // segment tables sized for every (tile, group) pair when that is small
    // (no read of the segment count), else read the count
    long nseg = nmark;
    if ((size_t)nmark * (tile_n + 1) * sizeof(int) > ((size_t)1 << 30)) {
      FMM_CUDA(cudaMemcpyAsync(&h.hc, ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
      FMM_CUDA(cudaStreamSynchronize(s));
      nseg = h.hc.gcounts[3];
    }
    h.g_tg.need(((size_t)nseg * (tile_n + 1) + ntiles + 2) * sizeof(int));
    // tg_src first: its rows of tile_n slots stay 16-byte aligned
    int *tg_src = h.g_tg.as<int>(), *tg_gid = tg_src + (size_t)nseg * tile_n, *tg_off = tg_gid + nseg;
    k_fill_rows<<<148 * 4, TB, 0, s>>>(tg_src, &counts[3], tile_n);  // absent targets: -1
    k_gfill<<<grid_for(nent, TB), TB, 0, s>>>(nent, pairs, ekey, gidx, tslot, tile_n, ngroups, segid, tg_src);
    k_seg_gid<<<grid_for(nmark, TB), TB, 0, s>>>(nmark, ngroups, mark, segid, d_slot_of, tg_gid);
    k_tg_off<<<grid_for(ntiles + 1, TB), TB, 0, s>>>(ntiles, ngroups, segid, &counts[3], tg_off);
    h.g_ntiles = ntiles;
    h.g_nseg = nseg;  // an upper bound unless it was read
    ghost_rows();
    contract(h, tcore, tp, KP16, gp, pd);
    h.launches += 10;
    FMM_LAUNCH();
  }
  h.g_plan.valid = true;
  h.g_plan.tcore = tcore;
  h.g_plan.ordered = h.m2l_ordered;
  h.g_plan.P = P;
  h.g_plan.nres = nres;
  if (nres > 0) m2l_residual(h, ekey);
}

}  // namespace fmm
