// FP64 FMA throughput of the current GPU: the roofline denominator of the
// FP64 predictor (the measured peak files carry HBM and bf16 figures only).
// Benchmark support, built as its own library (libexa_fp64_probe.so) and
// loaded by the benchmark alone; the product library does not contain it.
#include <cuda_runtime.h>

namespace {

// 8 independent DFMA chains per thread; the result is written so the chains
// stay live.  2 FLOP per FMA.
__global__ void k_fp64_fma(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-7, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
  double x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

}  // namespace

extern "C" {

/* TFLOP/s of dependent-chain DFMA over all SMs (8 CTAs of 256 threads per
 * SM); returns the cudaError_t of the run (0 = success). */
int exa_probe_fp64_fma_tflops(double* tflops) {
  if (!tflops) return (int)cudaErrorInvalidValue;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, blocks = sms * 8, iters = 2048;
  double* out = nullptr;
  cudaError_t e = cudaMalloc(&out, sizeof(double) * blocks * threads);
  if (e != cudaSuccess) return (int)e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_fp64_fma<<<blocks, threads>>>(out, 64, 0.999999, 1e-9);  // warm-up
  cudaEventRecord(a);
  k_fp64_fma<<<blocks, threads>>>(out, iters, 0.999999, 1e-9);
  cudaEventRecord(b);
  e = cudaEventSynchronize(b);
  float ms = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (e != cudaSuccess) return (int)e;
  const double flop = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flop / (ms * 1e-3) / 1e12;
  return 0;
}

}  // extern "C"
