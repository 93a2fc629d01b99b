// FMA-pipe peak of the current device, for roofline denominators: the device
// has no published FP64/FP32 vector figure in the pool's measured peaks.
// Independent FMA chains (8 per thread) keep the pipe full; one launch of
// 148 x 8 blocks x 256 threads, timed with CUDA events.
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

}  // namespace

double fma_peak_tflops(int precision) { return precision == EXAFMM_FP64 ? run<double>(4096) : run<float>(8192); }

}  // namespace fmm
