// Fused ADER-DG space-time predictor + volume integral (FP64 path).
//
// Computes, per cell, what the reference does in
//   spaceTimePredictorNonlinear  (kernels/aderdg/generic/c/3d/
//                                 spaceTimePredictorNonlinear.cpph:523-577)
//   volumeIntegralNonlinear      (kernels/aderdg/generic/c/3d/
//                                 volumeIntegralNonlinear.cpph:26-125)
// and the 2D counterparts (c/2d/...).
//
// Design (B = N+1 nodes per direction, V = 5):
//  * one thread per spatial node, one cell per CTA in 3D (B^3 nodes padded
//    to whole warps), several cells per CTA in 2D;
//  * the thread keeps its node's space-time iterate q[t][m] (B*V doubles)
//    and the Picard accumulators in registers; only the flux of the current
//    time slice goes through shared memory, where the directional
//    derivative reads whole lines of it;
//  * the Picard update is rewritten as
//      q_new[t] = c0[t] * luh - dt * sum_n tA[t][n] * G[n]
//      G[n]     = sum_d (1/dx_d) * sum_p deriv[s_d][p] * F_d[n](s_d -> p)
//    with deriv = Kxi^T / w and tA = iK1 * diag(w), algebraically identical
//    to the reference's rhs / iK1 form (spaceTimePredictorNonlinear.cpph:
//    117-296) up to rounding;
//  * convergence: the same squared-increment criterion < 1e-14 and the same
//    maximum of 2(N+1) iterations (:82, :298-306), decided per cell;
//  * after convergence: time averages, face extrapolation and the volume
//    integral from shared memory; outputs are lduh, lQhbnd, lFhbnd.
#include "exa_device.cuh"
#include "aderdg_predictor_body.cuh"
#include "aderdg_predictor_fp64_lines_body.cuh"
#include "aderdg_predictor_fp64_prog_body.cuh"

namespace exa {

template <int DIM, int N, int NPAR, bool PLANAR, int FULL>
__global__ void __launch_bounds__(PredShape<DIM, N, NPAR>::NT) k_predictor(PredArgs a) {
  extern __shared__ double smem[];
  predictor_block<DIM, N, NPAR, PLANAR, FULL>(a, blockIdx.x, smem);
}

// ------------------------------------------------------------ dispatch
template <int DIM, int N, int NPAR, bool PLANAR, int FULL>
static exa_status_t launch_t(const PredArgs& a, cudaStream_t st) {
  using S = PredShape<DIM, N, NPAR>;
  auto kern = k_predictor<DIM, N, NPAR, PLANAR, FULL>;
  const size_t smem = sizeof(double) * S::SM_DOUBLES;
  static bool attr_done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_done[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "predictor attribute");
    attr_done[dev & 63] = true;
  }
  const long nblocks = (a.ncells + S::CPB - 1) / S::CPB;
  if (nblocks <= 0) return EXA_OK;
  if (nblocks > 0x7fffffffL) return set_error(EXA_EINVAL, "too many cells");
  kern<<<(unsigned)nblocks, S::NT, smem, st>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_predictor launch");
}

template <int DIM, int N, bool PLANAR>
__global__ void __launch_bounds__(Fp64LineShape<DIM, N>::NT) k_predictor_lines(PredArgs a) {
  extern __shared__ double smem[];
  predictor_fp64_lines_block<DIM, N, PLANAR>(a, blockIdx.x, smem);
}

template <int DIM, int N, bool PLANAR>
static exa_status_t launch_lines_fp64(const PredArgs& a, cudaStream_t st) {
  using S = Fp64LineShape<DIM, N>;
  auto kern = k_predictor_lines<DIM, N, PLANAR>;
  const size_t smem = sizeof(double) * S::SM_DOUBLES;
  static bool attr_done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_done[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "predictor (lines) attribute");
    attr_done[dev & 63] = true;
  }
  const long nblocks = (a.ncells + S::CPB - 1) / S::CPB;
  if (nblocks <= 0) return EXA_OK;
  if (nblocks > 0x7fffffffL) return set_error(EXA_EINVAL, "too many cells");
  kern<<<(unsigned)nblocks, S::NT, smem, st>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_predictor_lines launch");
}

// progressive line-owner variant (aderdg_predictor_fp64_prog_body.cuh): 3D,
// one cell per CTA, 60 KB of shared memory, bounded for 3 CTAs per SM
template <int DIM, int N, bool PLANAR>
__global__ void __launch_bounds__(Fp64ProgShape<DIM, N>::NT, 3) k_predictor_prog(PredArgs a) {
  extern __shared__ double smem[];
  predictor_fp64_prog_block<DIM, N, PLANAR>(a, blockIdx.x, smem);
}

template <int DIM, int N, bool PLANAR>
static exa_status_t launch_prog_fp64(const PredArgs& a, cudaStream_t st) {
  using S = Fp64ProgShape<DIM, N>;
  auto kern = k_predictor_prog<DIM, N, PLANAR>;
  const size_t smem = sizeof(double) * S::SM_DOUBLES;
  static bool attr_done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_done[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return cuda_status(e, "predictor (progressive) attribute");
    attr_done[dev & 63] = true;
  }
  if (a.ncells <= 0) return EXA_OK;
  const long blocks = (a.ncells + S::CPB - 1) / S::CPB;
  if (blocks > 0x7fffffffL) return set_error(EXA_EINVAL, "too many cells");
  kern<<<(unsigned)blocks, S::NT, smem, st>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_predictor_prog launch");
}

template <int DIM, int N>
static exa_status_t launch_dn(const exa_aderdg_desc_t& d, const PredArgs& a, int full,
                              cudaStream_t st) {
  const bool planar = d.pde == EXA_PDE_EULER_PLANAR;
  // knob 3: 1 = node-gather, 2 = line-owner contraction, 3 = the
  // progressive line-owner form (FP64, not for the reference-temporaries
  // mode); default: progressive for order 4 (3D Euler: 3 CTAs per SM, it
  // measured 6.5 % faster than the line-owner kernel at 81^3; 2D: 7 % in
  // the ensemble's order-4 launches), line-owner for the other orders >= 4,
  // where it measured faster in 2D and 3D (for orders 2-3 the cell has more
  // line tasks than threads and node-gather wins)
  const int variant = tune_get(kTuneFp64Variant, 0);
  if constexpr (N == 4)
    if (d.npar == 0 && !full && (variant == 3 || variant == 0) && !(DIM == 3 && planar)) {
      if constexpr (DIM == 2)
        if (planar) return launch_prog_fp64<DIM, N, true>(a, st);
      return launch_prog_fp64<DIM, N, false>(a, st);
    }
  if (d.npar == 0 && !full && (variant >= 2 || (variant == 0 && N >= 4))) {
    if (DIM == 3 && planar) return set_error(EXA_EINVAL, "planar Euler is a 2D PDE");
    return planar ? launch_lines_fp64<DIM, N, true>(a, st) : launch_lines_fp64<DIM, N, false>(a, st);
  }
  if (d.npar == 0) {
    if (DIM == 2 && planar)
      return full ? launch_t<DIM, N, 0, true, 1>(a, st) : launch_t<DIM, N, 0, true, 0>(a, st);
    if (DIM == 3 && planar) return set_error(EXA_EINVAL, "planar Euler is a 2D PDE");
    return full ? launch_t<DIM, N, 0, false, 1>(a, st) : launch_t<DIM, N, 0, false, 0>(a, st);
  }
  if (d.npar == 1 && N == 3 && full) {
    if (DIM == 2 && planar) return launch_t<DIM, N, 1, true, 1>(a, st);
    if (DIM == 3 && !planar) return launch_t<DIM, N, 1, false, 1>(a, st);
  }
  return set_error(EXA_EINVAL, "nPar=1 is supported for order 3 drop-in calls only");
}

exa_status_t launch_predictor(const exa_aderdg_desc_t& d, const PredArgs& a, int full,
                              cudaStream_t st) {
  if (!full && d.precision == EXA_PREC_MIXED) return launch_predictor_mixed(d, a, st);
  if (d.dim == 3) {
    switch (d.order) {
      case 2: return launch_dn<3, 2>(d, a, full, st);
      case 3: return launch_dn<3, 3>(d, a, full, st);
      case 4: return launch_dn<3, 4>(d, a, full, st);
      case 5: return launch_dn<3, 5>(d, a, full, st);
    }
  } else if (d.dim == 2) {
    switch (d.order) {
      case 2: return launch_dn<2, 2>(d, a, full, st);
      case 3: return launch_dn<2, 3>(d, a, full, st);
      case 4: return launch_dn<2, 4>(d, a, full, st);
      case 5: return launch_dn<2, 5>(d, a, full, st);
    }
  }
  return set_error(EXA_EINVAL, "unsupported dim/order for the predictor (dim 2|3, order 2..5)");
}

exa_status_t upload_tables_predictor() {
  size_t bytes = 0;
  const void* h = host_dg_tables(&bytes);
  return cuda_status(cudaMemcpyToSymbol(c_dg, h, bytes), "upload tables (predictor)");
}

}  // namespace exa
