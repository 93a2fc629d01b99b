// FMA-pipe peak of the current device, for roofline denominators: the device
// has no published FP64/FP32 vector figure in the pool's measured peaks.
// Independent FMA chains (8 per thread) keep the pipe full; one launch of
// 148 x 8 blocks x 256 threads, timed with CUDA events.
#include <algorithm>

#include "fmm.cuh"

namespace fmm {
namespace {

template <class T>
__global__ void __launch_bounds__(256) k_fma(T *out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = (T)(threadIdx.x + k);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = x[k] * a + b;
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == (T)12345.678) out[0] = s;  // keeps the chains live
}

// Packed FP32x2 chains (fma.rn.f32x2: two FP32 FMAs per instruction, the
// form the FP32 near field uses); 8 chains of two lanes each per thread.
__global__ void __launch_bounds__(256) k_fma_f32x2(float *out, int iters, float a, float b) {
  unsigned long long x[8], av, bv;
  asm("mov.b64 %0, {%1, %1};" : "=l"(av) : "f"(a));
  asm("mov.b64 %0, {%1, %1};" : "=l"(bv) : "f"(b));
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const float lo = (float)(threadIdx.x + k), hi = lo + 0.5f;
    asm("mov.b64 %0, {%1, %2};" : "=l"(x[k]) : "f"(lo), "f"(hi));
  }
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[k]) : "l"(av), "l"(bv));
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x[k]));
    s += lo + hi;
  }
  if (s == 12345.678f) out[0] = s;  // keeps the chains live
}

template <class T>
double run(int iters) {
  T *d = nullptr;
  FMM_CUDA(cudaMalloc(&d, sizeof(T)));
  int dev = 0, sms = 0;
  FMM_CUDA(cudaGetDevice(&dev));
  FMM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 8, threads = 256;
  cudaEvent_t a, b;
  FMM_CUDA(cudaEventCreate(&a));
  FMM_CUDA(cudaEventCreate(&b));
  k_fma<T><<<blocks, threads>>>(d, iters / 8, (T)0.999999, (T)1e-7);  // warm-up
  FMM_CUDA(cudaEventRecord(a));
  k_fma<T><<<blocks, threads>>>(d, iters, (T)0.999999, (T)1e-7);
  FMM_CUDA(cudaEventRecord(b));
  FMM_CUDA(cudaEventSynchronize(b));
  float ms = 0;
  FMM_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d);
  const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
  return flops / (ms * 1e-3) / 1e12;
}

double run_f32x2(int iters) {
  float *d = nullptr;
  FMM_CUDA(cudaMalloc(&d, sizeof(float)));
  int dev = 0, sms = 0;
  FMM_CUDA(cudaGetDevice(&dev));
  FMM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 8, threads = 256;
  cudaEvent_t a, b;
  FMM_CUDA(cudaEventCreate(&a));
  FMM_CUDA(cudaEventCreate(&b));
  k_fma_f32x2<<<blocks, threads>>>(d, iters / 8, 0.999999f, 1e-7f);  // warm-up
  FMM_CUDA(cudaEventRecord(a));
  k_fma_f32x2<<<blocks, threads>>>(d, iters, 0.999999f, 1e-7f);
  FMM_CUDA(cudaEventRecord(b));
  FMM_CUDA(cudaEventSynchronize(b));
  float ms = 0;
  FMM_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d);
  const double flops = 2.0 * 2.0 * 8.0 * (double)iters * blocks * threads;  // 2 lanes per FMA
  return flops / (ms * 1e-3) / 1e12;
}

}  // namespace

// kind 0 (EXAFMM_FP64): scalar FP64 chains.  kind 1 (EXAFMM_MIXED): FP32,
// the larger of scalar and packed FP32x2 chains (a roofline against the
// smaller would overstate a kernel that issues packed instructions).
// kind 2: scalar FP32 chains only; kind 3: packed FP32x2 chains only.
double fma_peak_tflops(int kind) {
  switch (kind) {
    case 0: return run<double>(4096);
    case 2: return run<float>(8192);
    case 3: return run_f32x2(8192);
    default: return std::max(run<float>(8192), run_f32x2(8192));
  }
}

}  // namespace fmm
