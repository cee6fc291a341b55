// Arithmetic peaks of this GPU, measured: FP64 and FP32 fused multiply-add
// throughput.  The FP64-bound stage kernels (Navier-Stokes at high order,
// the FP64 Euler stage) report their pipe utilisation against this number
// rather than a datasheet figure.
//
// Method: every thread of a full grid (8 CTAs of 256 threads per SM) runs 8
// independent FMA chains for `iters` iterations; throughput = 2 flops x
// chains x iters x threads / elapsed (CUDA events around the launch, best of
// `reps` launches after one warm-up).  The chains depend on launch
// arguments, so nothing is folded at compile time, and a never-taken store
// keeps the results live.
#include <cuda_runtime.h>

#include "dgmx_internal.hpp"

namespace {

template <class T>
__global__ void __launch_bounds__(256) fma_chains(T *sink, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) x[c] = T(threadIdx.x) * T(1e-3) + T(c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = fma(x[c], a, b);
  }
  T s = T(0);
#pragma unroll
  for (int c = 0; c < 8; ++c) s += x[c];
  if (s == T(-1.2345e-7)) sink[0] = s;
}

template <class T>
cudaError_t measure(int device, int reps, double *tflops) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return e;
  int nsm = 0;
  if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return e;
  T *sink = nullptr;
  if ((e = cudaMalloc(&sink, 16)) != cudaSuccess) return e;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 256, blocks = nsm * 8, iters = 16384;
  float best = 0.0f;
  for (int r = 0; r <= reps && e == cudaSuccess; ++r) {
    cudaEventRecord(e0);
    fma_chains<T><<<blocks, threads>>>(sink, iters, T(0.999999), T(1e-7));
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    float ms = 0.0f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && (best == 0.0f || ms < best)) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (e != cudaSuccess) return e;
  *tflops = 2.0 * 8 * (double)iters * threads * blocks / (best * 1e-3) / 1e12;
  return cudaSuccess;
}

}  // namespace

extern "C" dgmx_status dgmx_measure_fma_peak(int device, int fp64, int reps, double *tflops) {
  if (!tflops || reps < 1) return DGMX_ERR_ARGUMENT;
  const cudaError_t e = fp64 ? measure<double>(device, reps, tflops) : measure<float>(device, reps, tflops);
  return e == cudaSuccess ? DGMX_OK : DGMX_ERR_CUDA;
}
