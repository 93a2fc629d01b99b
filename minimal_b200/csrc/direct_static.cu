// Direct summation for callers that cannot allocate device memory.
//
// exafmm_b200_direct() works on a handle, and a handle allocates: its bodies,
// its tree, and the staging arrays that direct() packs the targets into.
// Some callers are not allowed to do that -- a code that reserves all of HBM
// in its own pool at start-up, or a real-time loop that must never enter the
// CUDA allocator while it runs.  exafmm_b200_direct_static() serves them: the
// caller passes its own device arrays of sources and targets, and the only
// memory beyond those is the fixed array g_direct_scratch below, which lives
// in the library image and is created when the library is loaded onto a GPU.
//
// Limits and sharing rules:
//  - at most EXAFMM_DIRECT_STATIC_MAX_TARGETS targets per call (the scratch
//    holds two 32-byte records per target: 4 MiB in total per GPU, held by
//    every GPU that loads the library until the process exits);
//  - every call uses the same scratch array, and a call leaves its contents
//    behind; each call re-initialises the part it uses before reading it;
//  - calls run asynchronously on the caller's stream, which must belong to
//    the current device (a stream of another device is rejected); two calls
//    that overlap on the GPU (different streams, or different host threads)
//    race on the scratch and must be serialised by the caller;
//  - the first call on each device looks up the device address of the
//    scratch array (cudaGetSymbolAddress); make that first call before any
//    stream capture.  The address is kept for the life of the process: after
//    cudaDeviceReset() on a device, this entry point must not be called on
//    that device again;
//  - any number of sources (the source chunks are looped over in the kernel).
#include <algorithm>
#include <mutex>

#include "fmm.cuh"

namespace {

constexpr int MAXT = EXAFMM_DIRECT_STATIC_MAX_TARGETS;
constexpr int NDEV = 64;
constexpr int DT = 256;
constexpr int DCHUNK = 8192;

// [0, MAXT): packed target x,y,z,q; [MAXT, 2*MAXT): accumulated p,Fx,Fy,Fz.
static __device__ __align__(256) double4 g_direct_scratch[2 * MAXT];

std::mutex g_mu;
void *g_scratch_addr[NDEV] = {nullptr};

__global__ void k_ds_pack(const double *targets8, long nt, double4 *xq, double4 *pf) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  const double *r = targets8 + 8 * i;
  xq[i] = make_double4(r[0], r[1], r[2], r[3]);
  pf[i] = make_double4(r[4], r[5], r[6], r[7]);  // accumulate onto the caller's p, F
}

// Block (x, y) sums source chunks y, y + gridDim.y, ... of DCHUNK sources
// onto its DT targets.
__global__ void __launch_bounds__(DT) k_ds_sum(const double4 *xq, long nt, const double *src8, long ns,
                                               double4 *pf) {
  __shared__ double4 tile[DT];
  const long i = (long)blockIdx.x * DT + threadIdx.x;
  const double4 T = i < nt ? xq[i] : make_double4(0, 0, 0, 0);
  double p = 0, ax = 0, ay = 0, az = 0;
  for (long s0 = (long)blockIdx.y * DCHUNK; s0 < ns; s0 += (long)gridDim.y * DCHUNK) {
    const long s1 = min(ns, s0 + DCHUNK);
    for (long b = s0; b < s1; b += DT) {
      __syncthreads();
      if (b + threadIdx.x < s1) {
        const double *r = src8 + 8 * (b + threadIdx.x);
        tile[threadIdx.x] = make_double4(r[0], r[1], r[2], r[3]);
      }
      __syncthreads();
      const int m = (int)min((long)DT, s1 - b);
      for (int k = 0; k < m; k++) {
        const double4 s = tile[k];
        const double dx = T.x - s.x, dy = T.y - s.y, dz = T.z - s.z;
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double ir = r2 > 0 ? rsqrt(r2) : 0.0;  // zero distance skipped (3d/kernel.h:135)
        const double qir = s.w * ir, qir3 = qir * ir * ir;
        p += qir;
        ax += dx * qir3;
        ay += dy * qir3;
        az += dz * qir3;
      }
    }
  }
  if (i < nt) {
    atomicAdd(&pf[i].x, p);
    atomicAdd(&pf[i].y, -ax);
    atomicAdd(&pf[i].z, -ay);
    atomicAdd(&pf[i].w, -az);
  }
}

__global__ void k_ds_unpack(const double4 *pf, long nt, double *targets8) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  double *r = targets8 + 8 * i;
  r[4] = pf[i].x;
  r[5] = pf[i].y;
  r[6] = pf[i].z;
  r[7] = pf[i].w;
}

}  // namespace

extern thread_local std::string exafmm_b200_static_err;

extern "C" int exafmm_b200_direct_static(const double *sources8, int64_t ns, double *targets8, int64_t nt,
                                         void *stream) {
  if (!sources8 || !targets8 || ns <= 0 || nt <= 0) {
    exafmm_b200_static_err = "direct_static: need device arrays of sources and targets, ns > 0 and nt > 0";
    return EXAFMM_ERR_ARG;
  }
  if (nt > MAXT) {
    exafmm_b200_static_err = "direct_static: " + std::to_string(nt) + " targets exceed the fixed scratch of " +
                             std::to_string(MAXT) + "; split the targets into calls of at most that many";
    return EXAFMM_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NDEV) {
    cudaGetLastError();
    exafmm_b200_static_err = "direct_static: no current CUDA device";
    return EXAFMM_ERR_NOGPU;
  }
  void *base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
      // host code sees only a stand-in for the __device__ array: ask for its
      // address on this device once, with this device current
      cudaError_t e = cudaGetSymbolAddress(&g_scratch_addr[dev], g_direct_scratch);
      if (e != cudaSuccess) {
        cudaGetLastError();
        g_scratch_addr[dev] = nullptr;
        exafmm_b200_static_err = std::string("direct_static: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
        return EXAFMM_ERR_CUDA;
      }
    }
    base = g_scratch_addr[dev];
  }
  double4 *xq = (double4 *)base, *pf = xq + MAXT;
  cudaStream_t s = (cudaStream_t)stream;
  if (s) {  // the scratch address is this device's: the stream must be too
    int sdev = -1;
    if (cudaStreamGetDevice(s, &sdev) != cudaSuccess || sdev != dev) {
      cudaGetLastError();
      exafmm_b200_static_err = "direct_static: the stream does not belong to the current device";
      return EXAFMM_ERR_ARG;
    }
  }
  const unsigned gt = (unsigned)((nt + DT - 1) / DT);
  k_ds_pack<<<gt, DT, 0, s>>>(targets8, nt, xq, pf);
  const long nchunk = (ns + DCHUNK - 1) / DCHUNK;
  dim3 grid(gt, (unsigned)std::min<long>(nchunk, 1024));
  k_ds_sum<<<grid, DT, 0, s>>>(xq, nt, sources8, ns, pf);
  k_ds_unpack<<<gt, DT, 0, s>>>(pf, nt, targets8);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    exafmm_b200_static_err = std::string("direct_static: launch failed: ") + cudaGetErrorString(e);
    return EXAFMM_ERR_CUDA;
  }
  exafmm_b200_static_err.clear();  // as the handle calls do on success
  return EXAFMM_OK;
}
