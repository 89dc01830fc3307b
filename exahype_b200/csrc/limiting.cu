// Cell-status and bookkeeping kernels of the limiting ADER-DG grid (the
// a-posteriori subcell limiter of exahype/solvers/LimitingADERDGSolver.cpp on
// a uniform 2D or 3D grid, periodic or with outflow / reflecting walls).  Per step, after the unlimited DG candidate:
//   k_lim_admissible   physical admissibility of the candidate (positive
//                      density and pressure at every node), folded into the
//                      DMP verdict (LimitingADERDGSolver.cpp:839-876,
//                      1028-1048)
//   k_lim_base_status  Troubled for cells that fail; cells that were
//                      Troubled stay so for steps-till-cured more steps, then
//                      become NeighbourOfTroubled1 (determineLimiterStatus-
//                      AfterSolutionUpdate, :933-991)
//   k_lim_spread       one face-neighbour hop of status spreading: a cell
//                      takes max(own, neighbour - 1) (ADERDGSolver.cpp
//                      mergeWithLimiterStatus :2482-2500)
//   k_lim_lists        the cells that need a subcell patch (status >=
//                      NeighbourOfTroubled3) and the cells the FV solver
//                      updates (status >= NeighbourOfTroubled2)
//   k_lim_local /      the new cell-local extrema and their merge with the
//   k_lim_merge        face neighbours' (mergeSolutionMinMaxOnFace,
//                      LimitingADERDGSolver.cpp:1792-1853)
// Status values follow ADERDGCellDescription::LimiterStatus: Ok 0,
// NeighbourOfTroubled4 1, ..3 2, ..2 3, ..1 4, Troubled 5.
#include <float.h>

#include "exa_device.cuh"

namespace exa {

constexpr int kLimTroubled = 5, kLimNT1 = 4, kLimNT2 = 3, kLimNT3 = 2;

__global__ void k_lim_admissible(int npc, long ncells, int planar, const double* luh, int* ok) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;  // node
  if (i >= ncells * npc) return;
  const double* q = luh + i * kV;
  const double rho = q[0];
  const double j2 = planar ? q[1] * q[1] + q[2] * q[2] : q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  const double p = (kGamma - 1.0) * (q[4] - 0.5 * j2 / rho);
  if (!(rho > 0.0 && p > 0.0 && isfinite(p))) ok[i / npc] = 0;
}

__global__ void k_lim_base_status(long ncells, const int* ok, int* status, int* cure, int steps_till_cured) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  int base = 0;
  if (!ok[c]) {
    cure[c] = steps_till_cured + 1;
    base = kLimTroubled;
  } else if (status[c] == kLimTroubled) {
    const int left = cure[c] - 1;
    if (left <= 0) {
      base = kLimNT1;
      cure[c] = steps_till_cured;
    } else {
      base = kLimTroubled;
      cure[c] = left;
    }
  }
  status[c] = base;
}

// grid of n.x x n.y x n.z cells (n.z = 1 in 2D), x fastest; bc[d] = 0
// periodic, else the domain ends in direction d
struct LimGrid {
  int nx, ny, nz, dim;
  int bc[3];
  __host__ __device__ __forceinline__ long cells() const { return (long)nx * ny * nz; }
  // the neighbour across face f = 2 d + (0 lower, 1 upper), -1 outside
  __device__ __forceinline__ long nb(long c, int f) const {
    int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((long)nx * ny));
    const int d = f >> 1;
    const bool up = f & 1;
    int* p = d == 0 ? &x : (d == 1 ? &y : &z);
    const int n = d == 0 ? nx : (d == 1 ? ny : nz);
    if (up ? *p + 1 == n : *p == 0) {
      if (bc[d] != 0) return -1;
      *p = up ? 0 : n - 1;
    } else {
      *p += up ? 1 : -1;
    }
    return ((long)z * ny + y) * nx + x;
  }
};

__global__ void k_lim_spread(LimGrid G, const int* in, int* out) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.cells()) return;
  int nb = 0;
  for (int f = 0; f < 2 * G.dim; f++) {
    const long o = G.nb(c, f);
    if (o >= 0) nb = max(nb, in[o]);
  }
  out[c] = max(in[c], nb - 1);
}

// counts[0]: cells with a subcell patch, counts[1]: FV-updated cells,
// counts[2]: Troubled cells
__global__ void k_lim_lists(long ncells, const int* status, int* list_patch, int* list_fv, int* counts) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const int s = status[c];
  if (s >= kLimNT3) list_patch[atomicAdd(counts + 0, 1)] = (int)c;
  if (s >= kLimNT2) list_fv[atomicAdd(counts + 1, 1)] = (int)c;
  if (s == kLimTroubled) atomicAdd(counts + 2, 1);
}

// face block 0 of the per-cell extrema -> loc [cell][min | max][nobs]
__global__ void k_lim_local(long ncells, int nf, int nobs, const double* bmin, const double* bmax, double* loc) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncells * nobs) return;
  const long c = k / nobs;
  const int v = (int)(k % nobs);
  loc[(c * 2 + 0) * nobs + v] = bmin[c * nf * nobs + v];
  loc[(c * 2 + 1) * nobs + v] = bmax[c * nf * nobs + v];
}

// face f of a cell: extrema of the cell and of its neighbour across f; one
// thread per (cell, observable)
__global__ void k_lim_merge(LimGrid G, int nobs, const double* loc, double* bmin, double* bmax) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= G.cells() * nobs) return;
  const int v = (int)(k % nobs);
  const long c = k / nobs;
  const int nf = 2 * G.dim;
  const double mo = loc[(c * 2) * nobs + v], xo = loc[(c * 2 + 1) * nobs + v];
  for (int f = 0; f < nf; f++) {
    const long nb0 = G.nb(c, f);
    const long nb = nb0 >= 0 ? nb0 : c;  // a domain-boundary face keeps the cell's own extrema
    const double mn = loc[(nb * 2) * nobs + v], xn = loc[(nb * 2 + 1) * nobs + v];
    bmin[(c * nf + f) * nobs + v] = mn < mo ? mn : mo;
    bmax[(c * nf + f) * nobs + v] = xo < xn ? xn : xo;
  }
}

// NaN / Inf in the final state of the FV-updated cells
__global__ void k_lim_finite(int npc, const double* luh, const int* list, const int* count, int* nan_flag) {
  const long total = (long)*count * npc * kV;
  for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long)gridDim.x * blockDim.x) {
    const long cell = list[k / (npc * kV)];
    if (!isfinite(luh[cell * npc * kV + k % (npc * kV)])) atomicOr(nan_flag, 1);
  }
}

static unsigned blocks(long n, int nt) { return (unsigned)((n + nt - 1) / nt); }

static LimGrid lim_grid(int dim, const int* n, const int* bc) {
  LimGrid G;
  G.nx = n[0];
  G.ny = n[1];
  G.nz = dim == 3 ? n[2] : 1;
  G.dim = dim;
  for (int d = 0; d < 3; d++) G.bc[d] = bc && d < dim ? bc[d] : 0;
  return G;
}

exa_status_t limiting_status(int dim, const int* ncell, const int* bc, int npc, int planar, int admissibility,
                             int steps_till_cured, const double* luh, int* ok, int* status, int* status_tmp,
                             int* cure, int* list_patch, int* list_fv, int* counts, cudaStream_t st) {
  const LimGrid G = lim_grid(dim, ncell, bc);
  const long n = (long)G.nx * G.ny * G.nz;
  if (admissibility) k_lim_admissible<<<blocks(n * npc, 256), 256, 0, st>>>(npc, n, planar, luh, ok);
  k_lim_base_status<<<blocks(n, 256), 256, 0, st>>>(n, ok, status, cure, steps_till_cured);
  // four hops: Troubled (5) reaches NeighbourOfTroubled4 (1)
  for (int h = 0; h < 4; h++) {
    k_lim_spread<<<blocks(n, 256), 256, 0, st>>>(G, (h & 1) ? status_tmp : status, (h & 1) ? status : status_tmp);
  }
  cudaError_t e = cudaMemsetAsync(counts, 0, 3 * sizeof(int), st);
  if (e != cudaSuccess) return cuda_status(e, "limiter counters");
  k_lim_lists<<<blocks(n, 256), 256, 0, st>>>(n, status, list_patch, list_fv, counts);
  count_launch(6 + (admissibility ? 1 : 0));
  return cuda_status(cudaGetLastError(), "limiter status kernels");
}

exa_status_t limiting_merge_bounds(int dim, const int* ncell, const int* bc, int nobs, double* bmin, double* bmax,
                                   double* loc, cudaStream_t st) {
  const LimGrid G = lim_grid(dim, ncell, bc);
  const long n = (long)G.nx * G.ny * G.nz;
  k_lim_local<<<blocks(n * nobs, 256), 256, 0, st>>>(n, 2 * dim, nobs, bmin, bmax, loc);
  k_lim_merge<<<blocks(n * nobs, 256), 256, 0, st>>>(G, nobs, loc, bmin, bmax);
  count_launch(2);
  return cuda_status(cudaGetLastError(), "limiter bound merge");
}

exa_status_t limiting_check_finite(int npc, const double* luh, const int* list, const int* count, int* nan_flag,
                                   cudaStream_t st) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_lim_finite<<<(unsigned)(2 * sms), 256, 0, st>>>(npc, luh, list, count, nan_flag);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_lim_finite");
}

}  // namespace exa
