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

// Stable scatter: items are ranked in (round, warp, lane) order, which is
// their input order inside the tile.
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const u64 *kin, const u32 *vin, u64 *kout, u32 *vout,
                                                          long n, int shift, u64 mask, const int *offs,
                                                          int ntiles) {
  __shared__ int run[RS_BINS];
  __shared__ int wcnt[RS_THREADS / 32][RS_BINS];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  run[t] = offs[(long)t * ntiles + blockIdx.x];
  const long tile0 = (long)blockIdx.x * RS_TILE;
  for (int k = 0; k < RS_ITEMS; k++) {
    const long i = tile0 + (long)k * RS_THREADS + t;
    const bool valid = i < n;
    const u64 key = valid ? kin[i] : 0;
    const u32 val = valid ? vin[i] : 0;
    const int d = valid ? (int)((key >> shift) & mask) : RS_BINS;
#pragma unroll
    for (int w = 0; w < RS_THREADS / 32; w++) wcnt[w][t] = 0;
    __syncthreads();
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    int r = run[t];
#pragma unroll
    for (int w = 0; w < RS_THREADS / 32; w++) {
      int c = wcnt[w][t];
      wcnt[w][t] = r;
      r += c;
    }
    run[t] = r;
    __syncthreads();
    if (valid) {
      const int pos = wcnt[warp][d] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
  }
}

}  // namespace

void scan_exclusive_int(Handle &h, const int *in, int *out, long n, int *total_dev) {
  if (n <= 0) return;
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
  h.hist.need((size_t)2 * RS_BINS * ntiles * sizeof(int));
  int *hist = h.hist.as<int>();
  int *offs = hist + (long)RS_BINS * ntiles;
  for (int shift = lo_bit; shift < hi_bit; shift += 8) {
    const int bits = hi_bit - shift < 8 ? hi_bit - shift : 8;
    const u64 mask = (1ull << bits) - 1;
    k_rs_hist<<<ntiles, RS_THREADS, 0, h.stream>>>(k, n, shift, mask, hist, ntiles);
    h.launches++;
    FMM_LAUNCH();
    scan_exclusive_int(h, hist, offs, (long)RS_BINS * ntiles, nullptr);
    k_rs_scatter<<<ntiles, RS_THREADS, 0, h.stream>>>(k, v, k2, v2, n, shift, mask, offs, ntiles);
    h.launches++;
    FMM_LAUNCH();
    u64 *tk = k; k = k2; k2 = tk;
    u32 *tv = v; v = v2; v2 = tv;
  }
}

}  // namespace fmm
