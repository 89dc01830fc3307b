// Device error norms of one array against another (used by the
// mixed-precision accuracy report and the parity checks of the grid).
#include "exa_device.cuh"

namespace exa {

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
