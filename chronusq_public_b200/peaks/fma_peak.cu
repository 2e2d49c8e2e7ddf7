// FP64 / FP32 FMA throughput microbenchmark (CUDA cores).  The direct J/K
// build is bound by FP64 (and, on the mixed path, FP32) FMA issue, so its
// roofline denominators are measured here on the running GPU.
#include <cuda_runtime.h>

template <typename T>
__global__ void fma_loop(T* out, int iters, T a, T b) {
  T x0 = threadIdx.x * T(1e-3), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
  T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
      x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
    }
  }
  T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == T(-12345.678)) out[0] = s;  // keeps the chains alive
}

extern "C" double cqf_fma_peak_tflops(int fp64, int iters) {
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  void* out = nullptr;
  cudaMalloc(&out, 16);
  const int threads = 256, blocks = nsm * 8;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(e0);
    if (fp64)
      fma_loop<double><<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
    else
      fma_loop<float><<<blocks, threads>>>((float*)out, iters, 0.999999f, 1e-7f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
  return flops / (best * 1e-3) / 1e12;
}
