// Mixed-precision ADER-DG space-time predictor + volume integral.
//
// Same operator as k_predictor (aderdg_predictor.cu) and the reference's
// spaceTimePredictorNonlinear + volumeIntegralNonlinear; only the
// arithmetic of the Picard contractions changes:
//  * the base state luh and its flux F0 = F(luh) stay FP64, and the
//    derivative of F0 is computed once per cell in FP64;
//  * the Picard iterate is carried as the FP32 deviation dq = q - luh (an
//    O(dt) quantity: FP32 rounding is ~1e-7 of the deviation, ~1e-9 of the
//    state);
//  * the flux is evaluated in FP64 from luh + dq; only its deviation
//    dF = F(q) - F0 is rounded to FP32, exchanged through shared memory (half
//    the bytes of the FP64 path) and contracted with the derivative and the
//    time matrix in FP32 with FP32 accumulation (twice the FMA rate);
//  * the FP64 part of every iterate is fixed (luh and D.F0 do not change
//    between Picard iterations), so the new deviation dq = base - dt acc and
//    its squared increment are formed in FP32 from an FP64-derived base;
//  * the time averages, face extrapolation and volume integral are FP64, as
//    are the Riemann solves, surface integral, update and dt (k_corrector);
//  * time slices are software-pipelined: the FP64 flux of slice n+1 is
//    computed between the same barriers as the FP32 derivative of slice n.
#include "exa_device.cuh"
#include "aderdg_predictor_mixed_body.cuh"
#include "aderdg_predictor_lines_body.cuh"
#include "aderdg_predictor_tc_body.cuh"
#include "aderdg_predictor_mixed_prog_body.cuh"

namespace exa {

template <int DIM, int N, bool PLANAR, int MINB>
__global__ void __launch_bounds__(MixShape<DIM, N>::NT, MINB) k_predictor_mixed(PredArgs a) {
  extern __shared__ double smem[];
  predictor_mixed_block<DIM, N, PLANAR>(a, blockIdx.x, smem);
}

template <int DIM, int N, bool PLANAR, int MINB>
static exa_status_t launch_mixed_t(const PredArgs& a, cudaStream_t st) {
  using S = MixShape<DIM, N>;
  auto kern = k_predictor_mixed<DIM, N, PLANAR, MINB>;
  const size_t smem = sizeof(double) * S::SM_DOUBLES;
  static bool attr_done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_done[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "mixed predictor attribute");
    attr_done[dev & 63] = true;
  }
  const long nblocks = (a.ncells + S::CPB - 1) / S::CPB;
  if (nblocks <= 0) return EXA_OK;
  kern<<<(unsigned)nblocks, S::NT, smem, st>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_predictor_mixed launch");
}

template <int DIM, int N, bool PLANAR, int MINB>
__global__ void __launch_bounds__(LineShape<DIM, N>::NT, MINB) k_predictor_mixed_lines(PredArgs a) {
  extern __shared__ double smem[];
  predictor_mixed_lines_block<DIM, N, PLANAR>(a, blockIdx.x, smem);
}

template <int DIM, int N, bool PLANAR, int MINB>
static exa_status_t launch_lines_t(const PredArgs& a, cudaStream_t st) {
  using S = LineShape<DIM, N>;
  auto kern = k_predictor_mixed_lines<DIM, N, PLANAR, MINB>;
  const size_t smem = sizeof(double) * S::SM_DOUBLES;
  static bool attr_done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_done[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "mixed predictor (lines) attribute");
    attr_done[dev & 63] = true;
  }
  const long nblocks = (a.ncells + S::CPB - 1) / S::CPB;
  if (nblocks <= 0) return EXA_OK;
  kern<<<(unsigned)nblocks, S::NT, smem, st>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_predictor_mixed_lines launch");
}

// progressive line-owner variant, 3D (aderdg_predictor_mixed_prog_body.cuh):
// 44 KB of shared memory, bounded for 4 CTAs per SM
template <int DIM, int N, bool PLANAR, int MINB>
__global__ void __launch_bounds__(MixProgShape<DIM, N>::NT, MINB) k_predictor_mixed_prog(PredArgs a) {
  extern __shared__ double smem[];
  predictor_mixed_prog_block<DIM, N, PLANAR>(a, blockIdx.x, smem);
}

template <int DIM, int N, int MINB, bool PLANAR = false>
static exa_status_t launch_mixed_prog(const PredArgs& a, cudaStream_t st) {
  using S = MixProgShape<DIM, N>;
  auto kern = k_predictor_mixed_prog<DIM, N, PLANAR, MINB>;
  const size_t smem = sizeof(double) * S::SM_DOUBLES;
  static bool attr_done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_done[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return cuda_status(e, "mixed predictor (progressive) attribute");
    attr_done[dev & 63] = true;
  }
  if (a.ncells <= 0) return EXA_OK;
  const long blocks = (a.ncells + S::CPB - 1) / S::CPB;
  if (blocks > 0x7fffffffL) return set_error(EXA_EINVAL, "too many cells");
  kern<<<(unsigned)blocks, S::NT, smem, st>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_predictor_mixed_prog launch");
}

// tensor-core variant, 3D order 4 (aderdg_predictor_tc_body.cuh): 128
// threads, 3 CTAs per SM
template <bool PLANAR>
__global__ void __launch_bounds__(TcShape::NT, 3) k_predictor_mixed_tc(PredArgs a) {
  extern __shared__ double smem[];
  predictor_mixed_tc_block<PLANAR>(a, blockIdx.x, smem);
}

static exa_status_t launch_predictor_mixed_tc(const PredArgs& a, cudaStream_t st) {
  auto kern = k_predictor_mixed_tc<false>;
  const size_t smem = sizeof(double) * TcShape::SM_DOUBLES;
  static bool attr_done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_done[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "mixed predictor (tensor cores) attribute");
    attr_done[dev & 63] = true;
  }
  if (a.ncells <= 0) return EXA_OK;
  kern<<<(unsigned)a.ncells, TcShape::NT, smem, st>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_predictor_mixed_tc launch");
}

// line-owner variant (aderdg_predictor_lines_body.cuh)
static exa_status_t launch_predictor_mixed_lines(const exa_aderdg_desc_t& d, const PredArgs& a,
                                                 cudaStream_t st) {
  const bool planar = d.pde == EXA_PDE_EULER_PLANAR;
  if (d.dim == 3 && !planar) {
    switch (d.order) {
      case 2: return launch_lines_t<3, 2, false, 1>(a, st);
      case 3: return launch_lines_t<3, 3, false, 1>(a, st);
      case 4: {
        const int occ = tune_get(kTuneMixedOccupancy, 0);
        if (occ == 1) return launch_lines_t<3, 4, false, 1>(a, st);
        if (occ >= 4) return launch_lines_t<3, 4, false, 4>(a, st);
        return launch_lines_t<3, 4, false, 3>(a, st);
      }
      case 5: return launch_lines_t<3, 5, false, 1>(a, st);
    }
  } else if (d.dim == 2) {
    switch (d.order) {
      case 2: return planar ? launch_lines_t<2, 2, true, 1>(a, st) : launch_lines_t<2, 2, false, 1>(a, st);
      case 3: return planar ? launch_lines_t<2, 3, true, 1>(a, st) : launch_lines_t<2, 3, false, 1>(a, st);
      case 4: return planar ? launch_lines_t<2, 4, true, 1>(a, st) : launch_lines_t<2, 4, false, 1>(a, st);
      case 5: return planar ? launch_lines_t<2, 5, true, 1>(a, st) : launch_lines_t<2, 5, false, 1>(a, st);
    }
  }
  return set_error(EXA_EINVAL, "unsupported dim/order for the mixed predictor");
}

exa_status_t launch_predictor_mixed(const exa_aderdg_desc_t& d, const PredArgs& a, cudaStream_t st) {
  // knob 2: 1 = node-gather contraction, 2 = line-owner contraction,
  // 3 = line-owner on tensor cores, 4 = progressive line-owner; default:
  // progressive for 3D order 4 Euler and 2D order 5, line-owner for the
  // other orders >= 4
  // (measured faster in 2D and 3D), node-gather for orders 2-3
  const int variant = tune_get(kTuneMixedVariant, 0);
  if (d.npar == 0 && variant == 3 && d.dim == 3 && d.order == 4 && d.pde == EXA_PDE_EULER)
    return launch_predictor_mixed_tc(a, st);
  // knob 2 = 4, and the default for 3D order 4 Euler: the progressive
  // line-owner form (4 CTAs per SM; measured 9 % faster per step than the
  // line-owner kernel at 81^3, bit-identical results)
  if (d.npar == 0 && (variant == 4 || variant == 0) && d.dim == 3 && d.order == 4 && d.pde == EXA_PDE_EULER) {
    // knob 0 for this form: 5 = 96 registers (5 CTAs/SM), else 128 (4 CTAs/SM)
    if (tune_get(kTuneMixedOccupancy, 0) == 5) return launch_mixed_prog<3, 4, 5>(a, st);
    return launch_mixed_prog<3, 4, 4>(a, st);
  }
  // and for 2D order 5 (two cells per CTA, 128 registers: 4 CTAs per SM
  // instead of 3; 8 % faster in the ensemble's order-5 launches)
  if (d.npar == 0 && (variant == 4 || variant == 0) && d.dim == 2 && d.order == 5) {
    if (d.pde == EXA_PDE_EULER_PLANAR) return launch_mixed_prog<2, 5, 4, true>(a, st);
    return launch_mixed_prog<2, 5, 4, false>(a, st);
  }
  if (d.npar == 0 && (variant >= 2 || (variant == 0 && d.order >= 4)))
    return launch_predictor_mixed_lines(d, a, st);
  if (d.npar != 0) return set_error(EXA_EINVAL, "mixed precision: npar must be 0");
  const bool planar = d.pde == EXA_PDE_EULER_PLANAR;
  // knob: minimum resident CTAs per SM for 3D N=4 (register cap 255 / 170 / 128)
  const int occ = tune_get(kTuneMixedOccupancy, 0);
  if (d.dim == 3 && !planar) {
    switch (d.order) {
      case 2: return launch_mixed_t<3, 2, false, 1>(a, st);
      case 3: return launch_mixed_t<3, 3, false, 1>(a, st);
      case 4:
        // default 3 CTAs/SM (168 registers, no spills): measured fastest
        if (occ >= 4) return launch_mixed_t<3, 4, false, 4>(a, st);
        if (occ == 1) return launch_mixed_t<3, 4, false, 1>(a, st);
        return launch_mixed_t<3, 4, false, 3>(a, st);
      case 5: return launch_mixed_t<3, 5, false, 1>(a, st);
    }
  } else if (d.dim == 2) {
    switch (d.order) {
      case 2: return planar ? launch_mixed_t<2, 2, true, 1>(a, st) : launch_mixed_t<2, 2, false, 1>(a, st);
      case 3: return planar ? launch_mixed_t<2, 3, true, 1>(a, st) : launch_mixed_t<2, 3, false, 1>(a, st);
      case 4: return planar ? launch_mixed_t<2, 4, true, 1>(a, st) : launch_mixed_t<2, 4, false, 1>(a, st);
      case 5: return planar ? launch_mixed_t<2, 5, true, 1>(a, st) : launch_mixed_t<2, 5, false, 1>(a, st);
    }
  }
  return set_error(EXA_EINVAL, "unsupported dim/order for the mixed predictor");
}

exa_status_t upload_tables_predictor_mixed() {
  size_t bytes = 0;
  const void* h = host_dg_tables(&bytes);
  cudaError_t e = cudaMemcpyToSymbol(c_dg, h, bytes);
  if (e == cudaSuccess) {
    const void* hf = host_dg_tables_f(&bytes);
    e = cudaMemcpyToSymbol(c_dgf, hf, bytes);
  }
  return cuda_status(e, "upload tables (mixed predictor)");
}

}  // namespace exa
