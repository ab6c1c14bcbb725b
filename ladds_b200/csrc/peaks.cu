// peaks.cu -- measures the FP64 and FP32 FMA-pipe throughput of the device.
//
// The roofline of the propagation kernel is the FP64 (or, in split precision,
// mixed FP64/FP32) arithmetic pipe, for which no measured peak is supplied by
// the pool.  This diagnostic runs long chains of independent FMAs (8 per
// thread, a grid of 8 CTAs per SM) and reports FLOP/s (2 per FMA), timed with
// CUDA events on its own stream.  Not part of the LADDS interface.
#include <cuda_runtime.h>

#include <cstdint>

template <typename T>
__global__ void __launch_bounds__(256) k_fma_chain(T *out, int iters, T a, T b) {
  T r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = (T)(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = r[k] * a + b;
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += r[k];
  if (s == (T)12345.678) out[0] = s;  // keeps the chains alive
}

template <typename T>
static int measure(int device, double *tflops) {
  if (cudaSetDevice(device) != cudaSuccess) return 2;
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return 2;
  T *out = nullptr;
  if (cudaMalloc(&out, sizeof(T)) != cudaSuccess) return 7;
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = p.multiProcessorCount * 8, threads = 256, iters = 4096;
  k_fma_chain<T><<<blocks, threads, 0, st>>>(out, 256, (T)0.999999, (T)1e-7);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0, st);
    k_fma_chain<T><<<blocks, threads, 0, st>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  const int rc = cudaGetLastError() == cudaSuccess ? 0 : 2;
  *tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (best * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  cudaFree(out);
  return rc;
}

extern "C" int ladds_measure_fma_tflops(int device, double *fp64, double *fp32) {
  if (!fp64 || !fp32) return 1;
  int rc = measure<double>(device, fp64);
  if (!rc) rc = measure<float>(device, fp32);
  return rc;
}
