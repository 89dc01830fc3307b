// AMR transfer operators between a coarse cell (or face) and a descendant
// `level_delta` levels down (3:1 refinement per level): the reference's
// volume/faceUnknowns{Prolongation,Restriction}
// (kernels/aderdg/generic/c/{2d,3d}/amrRoutines.cpph) for batches of items
// resident on the GPU.
//
// A single level is a tensor-product operator; it is applied as k
// one-dimensional passes (sum factorisation: B terms per output instead of
// B^k), in shared memory, one CTA per item:
//   prolongation  out[m] = sum_n in[n] prod_d P[s_d][n_d][m_d]
//   restriction   out[m] = sum_n in[n] prod_d w[n_d] P[s_d][m_d][n_d] / (3 w[m_d])
// with P the fine-grid projector (P[s][n][m] = phi_n((s + x_m) / 3)) and w
// the Gauss-Legendre weights.  Levels are applied from the most significant
// base-3 digit of the descendant index (prolongation) or the least
// significant one (restriction), as the reference does; restriction adds
// the result to the coarse array (the reference accumulates the children).
#include "exa_device.cuh"

#define EXA_TABLE_QUAL static const
#include "dg_tables.h"

namespace exa {

static __constant__ double c_fgp[kMaxOrder + 1][3][10][10];

constexpr int kAmrNT = 128;

// one direction d: out[..m_d..][v] = sum_p op[m_d][p] in[..p..][v], op the
// B x B operator of this level and direction staged in shared memory (a
// per-thread constant-memory lookup with a thread-dependent index would be
// serialised); NV > 0 fixes the variable count at compile time
template <int K, int B, int NV>
__device__ __forceinline__ void amr_pass(double* out, const double* in, int nvar_rt, int d, const double* op) {
  const int nvar = NV > 0 ? NV : nvar_rt;
  int stride = nvar;
  for (int e = 0; e < d; e++) stride *= B;
  int total = nvar;
  for (int e = 0; e < K; e++) total *= B;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int md = (i / stride) % B;
    const int base = i - md * stride;
    const double* row = op + md * B;
    double acc = 0.0;
#pragma unroll
    for (int p = 0; p < B; p++) acc += row[p] * in[base + p * stride];
    out[i] = acc;
  }
}

template <int K, int B, int NV>
__global__ void __launch_bounds__(kAmrNT, 12) k_amr(int order, int nvar_rt, int restrict_op, double* dst,
                                                const double* src, const long* src_item, int level_delta,
                                                const int* index) {
  extern __shared__ double sm[];
  __shared__ double sop[3][B * B];  // this level's operator per direction, [m][p]
  const int nvar = NV > 0 ? NV : nvar_rt;
  int total = nvar;
  for (int e = 0; e < K; e++) total *= B;
  double* a = sm;
  double* b = sm + total;
  const long item = blockIdx.x;
  const long s_item = src_item ? src_item[item] : item;
  const double* in = src + s_item * total;
  for (int i = threadIdx.x; i < total; i += blockDim.x) a[i] = in[i];
  int cur[3] = {0, 0, 0};
  for (int d = 0; d < K; d++) cur[d] = index[item * 3 + d];
  const double* w = c_dg[order].w;
  for (int l = 1; l <= level_delta; l++) {
    int sub[3];
    if (restrict_op) {
      for (int d = 0; d < K; d++) {
        sub[d] = cur[d] % 3;
        cur[d] /= 3;
      }
    } else {
      int sig = 1;
      for (int e = 0; e < level_delta - l; e++) sig *= 3;
      for (int d = 0; d < K; d++) {
        sub[d] = cur[d] / sig;
        cur[d] %= sig;
      }
    }
    __syncthreads();  // the previous level's passes are done with sop
    for (int t = threadIdx.x; t < K * B * B; t += blockDim.x) {
      const int d = t / (B * B), md = (t / B) % B, p = t % B;
      sop[d][md * B + p] = restrict_op ? w[p] * c_fgp[order][sub[d]][md][p] / (3.0 * w[md])
                                       : c_fgp[order][sub[d]][p][md];
    }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < K; d++) {
      amr_pass<K, B, NV>(b, a, nvar, d, sop[d]);
      __syncthreads();
      double* t = a;
      a = b;
      b = t;
    }
  }
  double* out = dst + item * total;
  for (int i = threadIdx.x; i < total; i += blockDim.x) out[i] = restrict_op ? out[i] + a[i] : a[i];
}

template <int K>
static exa_status_t launch_amr_k(int order, int nvar, int restrict_op, long count, double* dst, const double* src,
                                 const long* src_item, int level_delta, const int* index, cudaStream_t st) {
  long total = nvar;
  for (int e = 0; e < K; e++) total *= order + 1;
  const size_t smem = 2 * total * sizeof(double);
#define EXA_AMR(BB)                                                                              \
  case BB - 1: {                                                                                 \
    if (nvar == kV)                                                                              \
      k_amr<K, BB, kV><<<(unsigned)count, kAmrNT, smem, st>>>(order, nvar, restrict_op, dst, src, \
                                                              src_item, level_delta, index);     \
    else                                                                                         \
      k_amr<K, BB, 0><<<(unsigned)count, kAmrNT, smem, st>>>(order, nvar, restrict_op, dst, src,  \
                                                             src_item, level_delta, index);      \
    break;                                                                                       \
  }
  switch (order) {
    EXA_AMR(2) EXA_AMR(3) EXA_AMR(4) EXA_AMR(5) EXA_AMR(6) EXA_AMR(7)
    default: return set_error(EXA_EINVAL, "AMR transfers: order must be in 1..6");
  }
#undef EXA_AMR
  count_launch();
  return cuda_status(cudaGetLastError(), "k_amr");
}

static exa_status_t launch_amr(int k, int order, int nvar, int restrict_op, long count, double* dst,
                               const double* src, const long* src_item, int level_delta, const int* index,
                               void* stream) {
  if (exa_status_t s = ensure_tables()) return s;
  if (!dst || !src || !index || count < 0) return set_error(EXA_EINVAL, "bad AMR arguments");
  if (nvar < 1 || nvar > 64) return set_error(EXA_EINVAL, "nvar must be in 1..64");
  if (level_delta < 1 || level_delta > 12) return set_error(EXA_EINVAL, "level_delta must be in 1..12");
  if (count == 0) return EXA_OK;
  if (count > 0x7fffffffL) return set_error(EXA_EINVAL, "too many items");
  long total = nvar;
  for (int e = 0; e < k; e++) total *= order + 1;
  if (2 * total * (long)sizeof(double) > 200 * 1024) return set_error(EXA_EINVAL, "item too large");
  cudaStream_t st = as_stream(stream);
  switch (k) {
    case 1: return launch_amr_k<1>(order, nvar, restrict_op, count, dst, src, src_item, level_delta, index, st);
    case 2: return launch_amr_k<2>(order, nvar, restrict_op, count, dst, src, src_item, level_delta, index, st);
    case 3: return launch_amr_k<3>(order, nvar, restrict_op, count, dst, src, src_item, level_delta, index, st);
  }
  return set_error(EXA_EINVAL, "k (node dimensions) must be 1, 2 or 3");
}

exa_status_t upload_tables_amr() {
  size_t bytes = 0;
  const void* h = host_dg_tables(&bytes);
  cudaError_t e = cudaMemcpyToSymbol(c_dg, h, bytes);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_fgp, exa_fgp, sizeof(exa_fgp));
  return cuda_status(e, "upload tables (amr)");
}

}  // namespace exa

using namespace exa;

extern "C" {

exa_status_t exa_aderdg_amr_prolongation(int k, int order, int nvar, long count, double* fine,
                                         const double* coarse, const long* coarse_item, int level_delta,
                                         const int* index, void* stream) {
  return launch_amr(k, order, nvar, 0, count, fine, coarse, coarse_item, level_delta, index, stream);
}

exa_status_t exa_aderdg_amr_restriction(int k, int order, int nvar, long count, double* coarse,
                                        const double* fine, int level_delta, const int* index, void* stream) {
  return launch_amr(k, order, nvar, 1, count, coarse, fine, nullptr, level_delta, index, stream);
}

}  // extern "C"
