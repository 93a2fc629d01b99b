// Device-wide primitives used by the tree and list builders: an exclusive
// scan of int arrays and a stable LSD radix sort of (u64 key, u32 value)
// pairs.  Both are plain three-kernel designs sized for B200 (1024-thread scan
// tiles, 2048-key sort tiles with warp-match ranking); all traffic is
// coalesced except the radix scatter, which writes runs per digit.
#include "fmm.cuh"

namespace fmm {

namespace {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr long SCAN_SMALL_TILES = 64;  // single-launch scan up to 64 tiles (256K ints)
constexpr long SCAN_TWO_TILES = 4096;  // two-launch scan up to 4096 tiles (16M ints)

__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of SCAN_TILE ints; writes per-block totals.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile(const int *in, int *out, long n, int *block_tot) {
  __shared__ int warp_sum[SCAN_THREADS / 32];
  const long base = (long)blockIdx.x * SCAN_TILE + (long)threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  int s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = warp_incl_scan(s);
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = warp_sum[lane];
    int wi = warp_incl_scan(w);
    warp_sum[lane] = wi - w;
    if (lane == 31 && block_tot) block_tot[blockIdx.x] = wi;
  }
  __syncthreads();
  int run = warp_sum[warp] + incl - s;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

__global__ void k_scan_add(int *out, long n, const int *block_off) {
  const long i = (long)blockIdx.x * SCAN_TILE + threadIdx.x;
  const int add = block_off[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    long j = i + (long)k * SCAN_THREADS;
    if (j < n) out[j] += add;
  }
}

__global__ void k_copy_int(int *dst, const int *src) { *dst = *src; }

// Per-tile sums (first launch of the two-launch scan).
__global__ void __launch_bounds__(SCAN_THREADS) k_tile_sums(const int *in, long n, int *sums) {
  __shared__ int warp_sum[SCAN_THREADS / 32];
  const long base = (long)blockIdx.x * SCAN_TILE + (long)threadIdx.x * SCAN_ITEMS;
  int v = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) v += base + k < n ? in[base + k] : 0;
  v = warp_incl_scan(v);
  if ((threadIdx.x & 31) == 31) warp_sum[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int t = warp_incl_scan(warp_sum[threadIdx.x]);
    if (threadIdx.x == 31) sums[blockIdx.x] = t;
  }
}

// Second launch: block b adds up the sums of the tiles before it (at most a
// few thousand ints), then scans its tile; the last block writes the total.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles2(const int *in, int *out, long n, const int *sums,
                                                             int *total_dev) {
  __shared__ int warp_sum[SCAN_THREADS / 32];
  __shared__ int s_prefix;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int pre = 0;
  for (int i = threadIdx.x; i < (int)blockIdx.x; i += SCAN_THREADS) pre += sums[i];
  pre = warp_incl_scan(pre);
  if (lane == 31) warp_sum[warp] = pre;
  __syncthreads();
  if (warp == 0) {
    const int t = warp_incl_scan(warp_sum[lane]);
    if (lane == 31) s_prefix = t;
  }
  __syncthreads();
  const int prefix = s_prefix;
  __syncthreads();
  const long base = (long)blockIdx.x * SCAN_TILE + (long)threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    v[k] = base + k < n ? in[base + k] : 0;
    sum += v[k];
  }
  const int incl = warp_incl_scan(sum);
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int w = warp_sum[lane];
    const int wi = warp_incl_scan(w);
    warp_sum[lane] = wi - w;
    if (lane == 31 && total_dev && blockIdx.x == gridDim.x - 1) *total_dev = prefix + wi;
  }
  __syncthreads();
  int run = prefix + warp_sum[warp] + incl - sum;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

// Exclusive scan of a short array (a few tiles) in one launch: block b
// first sums all input before its tile (every block reads at most a few
// hundred KB), then scans its tile as k_scan_tile does; the last block also
// writes the total.  Input and output must not overlap.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_small(const int *in, int *out, long n, int *total_dev) {
  __shared__ int warp_sum[SCAN_THREADS / 32];
  __shared__ int s_prefix;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long lim = (long)blockIdx.x * SCAN_TILE;  // a multiple of 4: int4 loads
  int pre = 0;
  for (long i = threadIdx.x; 4 * i < lim; i += SCAN_THREADS) {
    const int4 v = ((const int4 *)in)[i];
    pre += (v.x + v.y) + (v.z + v.w);
  }
  pre = warp_incl_scan(pre);
  if (lane == 31) warp_sum[warp] = pre;
  __syncthreads();
  if (warp == 0) {
    const int t = warp_incl_scan(warp_sum[lane]);
    if (lane == 31) s_prefix = t;
  }
  __syncthreads();
  const int prefix = s_prefix;
  __syncthreads();  // warp_sum is reused below
  const long base = lim + (long)threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    v[k] = base + k < n ? in[base + k] : 0;
    sum += v[k];
  }
  const int incl = warp_incl_scan(sum);
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int w = warp_sum[lane];
    const int wi = warp_incl_scan(w);
    warp_sum[lane] = wi - w;
    if (lane == 31 && total_dev && blockIdx.x == gridDim.x - 1) *total_dev = prefix + wi;
  }
  __syncthreads();
  int run = prefix + warp_sum[warp] + incl - sum;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}



void scan_rec(Handle &h, const int *in, int *out, long n, int *total_dev, int *work) {
  const long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  int *tot = work;
  k_scan_tile<<<(unsigned)nb, SCAN_THREADS, 0, h.stream>>>(in, out, n, tot);
  h.launches++;
  FMM_LAUNCH();
  if (nb == 1) {
    if (total_dev) {
      k_copy_int<<<1, 1, 0, h.stream>>>(total_dev, tot);
      h.launches++;
    }
    return;
  }
  int *tot_scan = work + nb;
  scan_rec(h, tot, tot_scan, nb, total_dev, work + 2 * nb);
  k_scan_add<<<(unsigned)nb, SCAN_THREADS, 0, h.stream>>>(out, n, tot_scan);
  h.launches++;
  FMM_LAUNCH();
}

// ---------------------------------------------------------------- radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_BINS = 256;

__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const u64 *keys, long n, int shift, u64 mask, int *hist,
                                                       int ntiles) {
  __shared__ int hs[RS_BINS];
  hs[threadIdx.x] = 0;
  __syncthreads();
  const long base = (long)blockIdx.x * RS_TILE;
#pragma unroll
  for (int k = 0; k < RS_ITEMS; k++) {
    long i = base + k * RS_THREADS + threadIdx.x;
    if (i < n) atomicAdd(&hs[(keys[i] >> shift) & mask], 1);
  }
  __syncthreads();
  hist[(long)threadIdx.x * ntiles + blockIdx.x] = hs[threadIdx.x];
}

// Block d: exclusive scan of digit d's counts over the tiles, into
// offs[d * ntiles + tile], and the digit's total into dtot[d].
__global__ void __launch_bounds__(RS_THREADS) k_rs_digit_scan(const int *hist, int *offs, int *dtot, int ntiles) {
  __shared__ int warp_sum[RS_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int *h = hist + (long)blockIdx.x * ntiles;
  int *o = offs + (long)blockIdx.x * ntiles;
  int carry = 0;
  for (int base = 0; base < ntiles; base += RS_THREADS) {
    const int i = base + threadIdx.x;
    const int v = i < ntiles ? h[i] : 0;
    const int incl = warp_incl_scan(v);
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    int wpre = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < RS_THREADS / 32; w++) {
      const int ws = warp_sum[w];
      wpre += w < warp ? ws : 0;
      tot += ws;
    }
    if (i < ntiles) o[i] = carry + wpre + incl - v;
    carry += tot;
    __syncthreads();  // warp_sum is rewritten by the next chunk
  }
  if (threadIdx.x == 0) dtot[blockIdx.x] = carry;
}

// Stable scatter of one tile.  Warp w ranks its contiguous 256 items
// (8 rounds of 32 lanes, per-warp digit counters bumped by the leader of
// each group of equal digits), the counts of the 8 warps are combined into
// tile-local digit offsets, the items are sorted by digit inside the tile in
// shared memory, and then written out in order: items of one digit are
// contiguous in the output, so the stores coalesce.
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const u64 *kin, const u32 *vin, u64 *kout, u32 *vout,
                                                          long n, int shift, u64 mask, const int *offs,
                                                          const int *dtot, int ntiles) {
  constexpr int NW = RS_THREADS / 32, PER = RS_TILE / NW;  // 256 items per warp
  static_assert(RS_BINS == RS_THREADS, "one thread per digit scans the digit totals");
  __shared__ int wcnt[NW][RS_BINS + 1];                     // per-warp digit counts, then offsets
  __shared__ int loff[RS_BINS + 1];                         // tile-local digit offsets
  __shared__ int dbase[RS_BINS];                            // first output slot of each digit
  __shared__ int dsum[NW];
  __shared__ u64 sk[RS_TILE];
  __shared__ u32 sv[RS_TILE];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int k = t; k < NW * (RS_BINS + 1); k += RS_THREADS) (&wcnt[0][0])[k] = 0;
  {  // exclusive scan of the digit totals
    const int c = dtot[t];
    const int incl = warp_incl_scan(c);
    if (lane == 31) dsum[warp] = incl;
    __syncthreads();
    int wpre = 0;
#pragma unroll
    for (int w = 0; w < NW; w++) wpre += w < warp ? dsum[w] : 0;
    dbase[t] = wpre + incl - c;
  }
  __syncthreads();
  const long tile0 = (long)blockIdx.x * RS_TILE;
  const int valid = (int)(n - tile0 < RS_TILE ? n - tile0 : RS_TILE);
  u64 key[RS_ITEMS];
  u32 val[RS_ITEMS];
  int dig[RS_ITEMS], pos[RS_ITEMS];
#pragma unroll
  for (int r = 0; r < RS_ITEMS; r++) {
    const int j = warp * PER + r * 32 + lane;
    const bool ok = j < valid;
    key[r] = ok ? kin[tile0 + j] : 0;
    val[r] = ok ? vin[tile0 + j] : 0;
    dig[r] = ok ? (int)((key[r] >> shift) & mask) : RS_BINS;  // padding sorts last
  }
#pragma unroll
  for (int r = 0; r < RS_ITEMS; r++) {
    const unsigned peers = __match_any_sync(0xffffffffu, dig[r]);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) {
      base = wcnt[warp][dig[r]];
      wcnt[warp][dig[r]] = base + __popc(peers);
    }
    pos[r] = __shfl_sync(0xffffffffu, base, leader) + __popc(peers & ((1u << lane) - 1u));
    __syncwarp();
  }
  __syncthreads();
  // per digit: offsets of the warps' runs, and the digit's total
  for (int d = t; d <= RS_BINS; d += RS_THREADS) {
    int run = 0;
#pragma unroll
    for (int w = 0; w < NW; w++) {
      const int c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
    loff[d] = run;
  }
  __syncthreads();
  // exclusive scan of the digit totals (thread 0 of each warp scans a slice)
  if (t < 32) {
    constexpr int SL = (RS_BINS + 1 + 31) / 32;
    int tot = 0;
    for (int k = 0; k < SL; k++) tot += lane * SL + k <= RS_BINS ? loff[lane * SL + k] : 0;
    int incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    int run = incl - tot;
    for (int k = 0; k < SL; k++) {
      const int d = lane * SL + k;
      if (d <= RS_BINS) {
        const int c = loff[d];
        loff[d] = run;
        run += c;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ITEMS; r++) {
    const int lp = loff[dig[r]] + wcnt[warp][dig[r]] + pos[r];
    sk[lp] = key[r];
    sv[lp] = val[r];
  }
  __syncthreads();
  for (int j = t; j < valid; j += RS_THREADS) {
    const u64 k = sk[j];
    const int d = (int)((k >> shift) & mask);
    const long o = (long)dbase[d] + offs[(long)d * ntiles + blockIdx.x] + (j - loff[d]);
    kout[o] = k;
    vout[o] = sv[j];
  }
}

}  // namespace

void scan_exclusive_int(Handle &h, const int *in, int *out, long n, int *total_dev) {
  if (n <= 0) return;
  const long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (nb <= SCAN_SMALL_TILES && ((uintptr_t)in & 15) == 0) {  // short: one launch
    k_scan_small<<<(unsigned)nb, SCAN_THREADS, 0, h.stream>>>(in, out, n, total_dev);
    h.launches++;
    FMM_LAUNCH();
    return;
  }
  if (nb <= SCAN_TWO_TILES) {  // tile sums, then every tile adds the sums before it
    h.scan_tmp.need(nb * sizeof(int));
    k_tile_sums<<<(unsigned)nb, SCAN_THREADS, 0, h.stream>>>(in, n, h.scan_tmp.as<int>());
    k_scan_tiles2<<<(unsigned)nb, SCAN_THREADS, 0, h.stream>>>(in, out, n, h.scan_tmp.as<int>(), total_dev);
    h.launches += 2;
    FMM_LAUNCH();
    return;
  }
  long need = 0, m = n;
  while (true) {
    long nb = (m + SCAN_TILE - 1) / SCAN_TILE;
    need += 2 * nb + 2;
    if (nb == 1) break;
    m = nb;
  }
  h.scan_tmp.need(need * sizeof(int));
  scan_rec(h, in, out, n, total_dev, h.scan_tmp.as<int>());
}

// Sorts bits [lo_bit, hi_bit) of the keys, stable, 8 bits per pass.  On
// return k/v point at the sorted data (the buffers may have been swapped).
void radix_sort_pairs(Handle &h, u64 *&k, u32 *&v, u64 *&k2, u32 *&v2, long n, int lo_bit, int hi_bit) {
  if (n <= 1 || hi_bit <= lo_bit) return;
  const int ntiles = (int)((n + RS_TILE - 1) / RS_TILE);
  h.hist.need(((size_t)2 * RS_BINS * ntiles + RS_BINS) * sizeof(int));
  int *hist = h.hist.as<int>();
  int *offs = hist + (long)RS_BINS * ntiles;
  int *dtot = offs + (long)RS_BINS * ntiles;
  for (int shift = lo_bit; shift < hi_bit; shift += 8) {
    const int bits = hi_bit - shift < 8 ? hi_bit - shift : 8;
    const u64 mask = (1ull << bits) - 1;
    k_rs_hist<<<ntiles, RS_THREADS, 0, h.stream>>>(k, n, shift, mask, hist, ntiles);
    // per digit over the tiles; the scatter adds the scanned digit totals
    k_rs_digit_scan<<<RS_BINS, RS_THREADS, 0, h.stream>>>(hist, offs, dtot, ntiles);
    h.launches += 2;
    FMM_LAUNCH();
    k_rs_scatter<<<ntiles, RS_THREADS, 0, h.stream>>>(k, v, k2, v2, n, shift, mask, offs, dtot, ntiles);
    h.launches++;
    FMM_LAUNCH();
    u64 *tk = k; k = k2; k2 = tk;
    u32 *tv = v; v = v2; v2 = tv;
  }
}

}  // namespace fmm
