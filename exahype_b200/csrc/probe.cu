// Device capability probes used as roofline denominators by the benchmark:
// FP64 FMA throughput (no FP64 figure is shipped with the measured peaks)
// and a plain DRAM copy bandwidth.
#include "exa_device.cuh"

namespace exa {

// 8 independent DFMA chains per thread; the result is written so the chains
// are live.  2 FLOP per FMA.
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

// FP64 tensor-core (DMMA, mma.sync m8n8k4 f64) throughput: 4 independent
// accumulator fragments per warp, operands held in registers.
__global__ void k_dmma(double* out, int iters, double a0, double b0) {
  double a = a0 + threadIdx.x * 1e-9, b = b0 - threadIdx.x * 1e-9;
  double c[4][2];
#pragma unroll
  for (int k = 0; k < 4; k++) c[k][0] = c[k][1] = 0.0;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int r = 0; r < 8; r++)
#pragma unroll
      for (int k = 0; k < 4; k++)
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(c[k][0]), "+d"(c[k][1])
                     : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 4; k++) s += c[k][0] + c[k][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_copy(const double4* __restrict__ in, double4* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = in[i];
}

// sum (a-b)^2, sum b^2, max |a-b|, max |b| over n doubles (block partials
// combined with atomics on the bit patterns of non-negative doubles)
__global__ void k_diff_norms(const double* a, const double* b, size_t n, double* sums,
                             unsigned long long* maxes) {
  double s0 = 0, s1 = 0, m0 = 0, m1 = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double d = a[i] - b[i];
    s0 += d * d;
    s1 += b[i] * b[i];
    m0 = fmax(m0, fabs(d));
    m1 = fmax(m1, fabs(b[i]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
    m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&sums[0], s0);
    atomicAdd(&sums[1], s1);
    atomicMax(&maxes[0], (unsigned long long)__double_as_longlong(m0));
    atomicMax(&maxes[1], (unsigned long long)__double_as_longlong(m1));
  }
}

}  // namespace exa

using namespace exa;

extern "C" {

exa_status_t exa_measure_fp64_peak(double* tflops) {
  if (!tflops) return set_error(EXA_EINVAL, "NULL tflops");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, blocks = sms * 8, iters = 2048;
  double* out = nullptr;
  cudaError_t e = cudaMalloc(&out, sizeof(double) * blocks * threads);
  if (e != cudaSuccess) return cuda_status(e, "probe alloc");
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_fp64_fma<<<blocks, threads>>>(out, 64, 0.999999, 1e-9);  // warm-up
  cudaEventRecord(a);
  k_fp64_fma<<<blocks, threads>>>(out, iters, 0.999999, 1e-9);
  cudaEventRecord(b);
  count_launch(2);
  e = cudaEventSynchronize(b);
  float ms = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (e != cudaSuccess) return cuda_status(e, "probe fp64");
  const double flop = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flop / (ms * 1e-3) / 1e12;
  return EXA_OK;
}

exa_status_t exa_measure_fp64_tensor_peak(double* tflops) {
  if (!tflops) return set_error(EXA_EINVAL, "NULL tflops");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, blocks = sms * 4, iters = 1024;
  double* out = nullptr;
  cudaError_t e = cudaMalloc(&out, sizeof(double) * blocks * threads);
  if (e != cudaSuccess) return cuda_status(e, "probe alloc");
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_dmma<<<blocks, threads>>>(out, 16, 1e-3, 1e-3);  // warm-up
  cudaEventRecord(a);
  k_dmma<<<blocks, threads>>>(out, iters, 1e-3, 1e-3);
  cudaEventRecord(b);
  count_launch(2);
  e = cudaEventSynchronize(b);
  float ms = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (e != cudaSuccess) return cuda_status(e, "probe dmma");
  const double warps = (double)blocks * threads / 32;
  const double flop = 2.0 * 8 * 8 * 4 * 8 * 4 * (double)iters * warps;
  *tflops = flop / (ms * 1e-3) / 1e12;
  return EXA_OK;
}

exa_status_t exa_measure_copy_bandwidth(size_t bytes, double* gbs) {
  if (!gbs || bytes < 1024) return set_error(EXA_EINVAL, "bad argument");
  const size_t n = bytes / sizeof(double4);
  double4 *in = nullptr, *out = nullptr;
  cudaError_t e = cudaMalloc(&in, n * sizeof(double4));
  if (e == cudaSuccess) e = cudaMalloc(&out, n * sizeof(double4));
  if (e != cudaSuccess) {
    cudaFree(in);
    return cuda_status(e, "probe alloc");
  }
  cudaMemset(in, 0, n * sizeof(double4));
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_copy<<<sms * 4, 512>>>(in, out, n);
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(a);
    k_copy<<<sms * 4, 512>>>(in, out, n);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best) best = ms;
  }
  count_launch(6);
  e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(in);
  cudaFree(out);
  if (e != cudaSuccess) return cuda_status(e, "probe copy");
  *gbs = 2.0 * n * sizeof(double4) / (best * 1e-3) / 1e9;
  return EXA_OK;
}

exa_status_t exa_diff_norms(const double* a, const double* b, size_t n, double* out, void* stream) {
  if (!a || !b || !out) return set_error(EXA_EINVAL, "NULL argument");
  cudaStream_t st = as_stream(stream);
  double* buf = nullptr;
  cudaError_t e = cudaMallocAsync(&buf, 4 * sizeof(double), st);
  if (e != cudaSuccess) return cuda_status(e, "diff norms alloc");
  e = cudaMemsetAsync(buf, 0, 4 * sizeof(double), st);
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess && n > 0) {
    k_diff_norms<<<sms * 4, 256, 0, st>>>(a, b, n, buf, (unsigned long long*)(buf + 2));
    count_launch();
    e = cudaGetLastError();
  }
  double h[4] = {0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, buf, sizeof(h), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(buf, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "diff norms");
  out[0] = h[1] > 0 ? sqrt(h[0] / h[1]) : sqrt(h[0]);  // relative L2
  out[1] = h[3] > 0 ? h[2] / h[3] : h[2];              // relative Linf
  out[2] = sqrt(h[0]);
  out[3] = h[2];
  return EXA_OK;
}

}  // extern "C"
