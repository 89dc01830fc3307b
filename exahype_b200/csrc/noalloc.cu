// Allocation-free variant of the per-cell space-time predictor drop-in.
//
// exa_aderdg_spaceTimePredictor stages the cell through a device workspace
// that the library allocates with cudaMalloc on first use (and re-allocates
// when a larger order arrives).  Some callers cannot let that happen:
//  * many host threads calling the per-cell kernels concurrently, as
//    ExaHyPE's TBB workers do (mappings/Prediction.cpp:152): cudaMalloc and
//    cudaFree take a device-wide lock and cudaFree synchronises the device,
//    stalling every other worker's work;
//  * processes whose device memory is already handed out by a pool
//    allocator, where a late cudaMalloc fails with out-of-memory.
// exa_aderdg_spaceTimePredictor_noalloc therefore stages through a
// file-scope __device__ array of fixed size that every GPU holds from the
// moment the library is loaded until the process exits.  Its copies are
// synchronous on the default stream, like the drop-in's.
#include <mutex>

#include "exa_device.cuh"

namespace exa {

// 64 Ki doubles (512 KiB): one cell of any supported order (2..5), 2D or 3D,
// with up to one parameter needs at most ~44 Ki doubles.
constexpr size_t kNoAllocScratchDoubles = 65536;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

struct NoAllocDevice {
  std::mutex mu;       // serialises the calls of this process on one device
  double* ptr = nullptr;
};
static NoAllocDevice g_noalloc[256];

}  // namespace exa

using namespace exa;

extern "C" {

exa_status_t exa_aderdg_spaceTimePredictor_noalloc(
    const exa_aderdg_desc_t* desc, double* lQhbnd, double* lFhbnd,
    double** tempSpaceTimeUnknowns, double** tempSpaceTimeFluxUnknowns, double* tempUnknowns,
    double* tempFluxUnknowns, double* tempStateSizedVectors, const double* luh, const double* dx,
    double dt, double* pointForceSources, int* picardIterations) {
  (void)tempStateSizedVectors;
  (void)pointForceSources;
  // the drop-in's own descriptor checks (dim, order, nvar, npar, pde, dx)
  if (exa_status_t s = check_aderdg_desc(desc)) return s;
  if (!lQhbnd || !lFhbnd || !luh || !tempUnknowns || !tempFluxUnknowns)
    return set_error(EXA_EINVAL, "NULL buffer");
  exa_aderdg_desc_t d = *desc;
  if (dx)
    for (int i = 0; i < d.dim; i++) d.dx[i] = dx[i];
  for (int i = 0; i < d.dim; i++)
    if (!(d.dx[i] > 0.0)) return set_error(EXA_EINVAL, "dx must be positive");

  const int B = d.order + 1, D = d.nvar + d.npar, V = d.nvar;
  int nn = 1, nf = 1;
  for (int i = 0; i < d.dim; i++) nn *= B;
  for (int i = 0; i < d.dim - 1; i++) nf *= B;
  const size_t n_luh = (size_t)nn * D, n_lqi = (size_t)nn * B * D;
  const size_t n_lfi = (size_t)nn * B * (d.dim + 1) * V, n_qhi = (size_t)nn * D;
  const size_t n_fhi = (size_t)nn * (d.dim + 1) * V, n_lduh = (size_t)nn * V;
  const size_t n_qb = (size_t)2 * d.dim * nf * D, n_fb = (size_t)2 * d.dim * nf * V;
  const size_t need = n_luh + n_lqi + n_lfi + n_qhi + n_fhi + n_lduh + n_qb + n_fb + 1;
  if (need > kNoAllocScratchDoubles)
    return set_error(EXA_EINVAL, "cell needs more than the 65536-double static scratch");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
  NoAllocDevice& nd = g_noalloc[dev & 255];
  std::lock_guard<std::mutex> lk(nd.mu);
  if (!nd.ptr) {
    // one-time set-up on this device: the device address of the scratch
    // array (its host-side name is not a device address) and the operator
    // tables in constant memory
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(noalloc scratch)");
    if (exa_status_t s = ensure_tables()) return s;
    nd.ptr = p;
  }
  double* w = nd.ptr;
  double *wl = w, *wqi = wl + n_luh, *wfi = wqi + n_lqi, *wqhi = wfi + n_lfi, *wfhi = wqhi + n_qhi,
         *wdu = wfhi + n_fhi, *wqb = wdu + n_lduh, *wfb = wqb + n_qb;
  int* wit = (int*)(wfb + n_fb);

  // The kernel writes every element of every output it produces, so the
  // contents left by the previous call need no clearing.
  e = cudaMemcpy(wl, luh, n_luh * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_status(e, "copy luh");
  PredArgs a{};
  a.ncells = 1;
  a.luh = wl;
  a.dt = dt;
  a.dt_dev = nullptr;
  for (int i = 0; i < 3; i++) a.idx[i] = i < d.dim ? 1.0 / d.dx[i] : 0.0;
  a.lduh = wdu;
  a.lQhbnd = wqb;
  a.lFhbnd = wfb;
  a.iters = wit;
  a.stats = nullptr;
  a.lQi = wqi;
  a.lFi = wfi;
  a.lQhi = wqhi;
  a.lFhi = wfhi;
  a.precision = EXA_PREC_FP64;
  if (exa_status_t s = launch_predictor(d, a, 1, 0)) return s;
  e = cudaMemcpy(lQhbnd, wqb, n_qb * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(lFhbnd, wfb, n_fb * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(tempUnknowns, wqhi, n_qhi * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(tempFluxUnknowns, wfhi, n_fhi * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && tempSpaceTimeUnknowns && tempSpaceTimeUnknowns[0])
    e = cudaMemcpy(tempSpaceTimeUnknowns[0], wqi, n_lqi * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && tempSpaceTimeFluxUnknowns && tempSpaceTimeFluxUnknowns[0])
    e = cudaMemcpy(tempSpaceTimeFluxUnknowns[0], wfi, n_lfi * sizeof(double), cudaMemcpyDeviceToHost);
  int it = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&it, wit, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e, "copy predictor outputs");
  if (picardIterations) *picardIterations = it;
  return EXA_OK;
}

}  // extern "C"
