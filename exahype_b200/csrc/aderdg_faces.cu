// ADER-DG face and cell-local kernels:
//  * k_corrector: fused Rusanov Riemann solve on the 2*dim faces of a cell,
//    surface integral, solution update and the next step's CFL time step
//    (per-cell min + one atomic min per cell into a device slot), on a
//    uniform periodic grid;
//  * batched drop-ins with the reference's semantics: Riemann on a face
//    list (in place), surface integral, volume integral, solution update,
//    stable time step;
//  * the nodal initial condition.
// Reference: kernels/aderdg/generic/c/{2d,3d}/{riemannSolverNonlinear,
// surfaceIntegralNonlinear,volumeIntegralNonlinear,solutionUpdate,
// stableTimeStepSize}.cpph and exahype/solvers/ADERDGSolver.cpp:2744-2826
// (face pairing: left cell face 2d+1, right cell face 2d).
#include <float.h>

#include "exa_device.cuh"
#include "aderdg_corrector_body.cuh"

namespace exa {

template <int DIM, int N, bool PLANAR>
__global__ void __launch_bounds__(CellShape<DIM, N>::NT) k_corrector(CorrArgs a) {
  extern __shared__ double smem[];
  corrector_block<DIM, N, PLANAR>(a, blockIdx.x, smem);
}

exa_status_t launch_corrector(int dim, int order, int pde, const CorrArgs& a, cudaStream_t st) {
  const bool planar = pde == EXA_PDE_EULER_PLANAR;
#define EXA_CORR(D_, N_, P_)                                                                 \
  do {                                                                                       \
    using S = CellShape<D_, N_>;                                                             \
    auto kern = k_corrector<D_, N_, P_>;                                                     \
    const size_t sm = sizeof(double) *                                                       \
        (S::CPB * (4 * S::NFACE * S::NF * S::V + S::NFACE * 2 * S::V + S::NFACE) + S::NT / 32 + 1); \
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
    if (e != cudaSuccess) return cuda_status(e, "corrector attribute");                      \
    const long nb = (a.ncells + S::CPB - 1) / S::CPB;                                        \
    if (nb <= 0) return EXA_OK;                                                              \
    kern<<<(unsigned)nb, S::NT, sm, st>>>(a);                                                \
    count_launch();                                                                          \
    return cuda_status(cudaGetLastError(), "k_corrector launch");                           \
  } while (0)
  if (dim == 3 && !planar) {
    switch (order) {
      case 2: EXA_CORR(3, 2, false);
      case 3: EXA_CORR(3, 3, false);
      case 4: EXA_CORR(3, 4, false);
      case 5: EXA_CORR(3, 5, false);
    }
  } else if (dim == 2) {
    if (planar) {
      switch (order) {
        case 2: EXA_CORR(2, 2, true);
        case 3: EXA_CORR(2, 3, true);
        case 4: EXA_CORR(2, 4, true);
        case 5: EXA_CORR(2, 5, true);
      }
    } else {
      switch (order) {
        case 2: EXA_CORR(2, 2, false);
        case 3: EXA_CORR(2, 3, false);
        case 4: EXA_CORR(2, 4, false);
        case 5: EXA_CORR(2, 5, false);
      }
    }
  }
#undef EXA_CORR
  return set_error(EXA_EINVAL, "unsupported dim/order/pde for the corrector");
}

// ------------------------------------------------------ batched drop-ins
// One thread per node, generic over runtime sizes (these are the simple
// reference-semantics kernels; the fused grid path above is the fast one).
struct NodeArgs {
  long ncells;
  int dim, B, D, V;
  int order;
  double dx[3];
  double dt;
  double factor;
  int planar;
};

__device__ __forceinline__ void node_coords(int s, int B, int dim, int* sd) {
  sd[0] = s % B;
  sd[1] = (s / B) % B;
  sd[2] = dim == 3 ? s / (B * B) : 0;
}

__global__ void k_solution_update(NodeArgs a, double* luh, const double* lduh) {
  const int nn = a.dim == 3 ? a.B * a.B * a.B : a.B * a.B;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= a.ncells * nn) return;
  const long c = gid / nn;
  const int s = (int)(gid % nn);
  int sd[3];
  node_coords(s, a.B, a.dim, sd);
  const DGConst& T = c_dg[a.order];
  double W = 1.0;
  for (int e = a.dim - 1; e >= 0; e--) W *= T.w[sd[e]];
  const double us = a.dt / W;
  for (int m = 0; m < a.V; m++)
    luh[(c * nn + s) * a.D + m] += lduh[(c * nn + s) * a.V + m] * us;
}

__global__ void k_surface_integral(NodeArgs a, double* lduh, const double* lF) {
  const int nn = a.dim == 3 ? a.B * a.B * a.B : a.B * a.B;
  const int nf = a.dim == 3 ? a.B * a.B : a.B;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= a.ncells * nn) return;
  const long c = gid / nn;
  const int s = (int)(gid % nn);
  int sd[3];
  node_coords(s, a.B, a.dim, sd);
  const DGConst& T = c_dg[a.order];
  const double* F = lF + c * 2 * a.dim * nf * a.V;
  for (int d = 0; d < a.dim; d++) {
    double wprod = 1.0;
    for (int e = a.dim - 1; e >= 0; e--)
      if (e != d) wprod *= T.w[sd[e]];
    const double us = wprod / a.dx[d];
    int j;
    if (a.dim == 3) j = d == 0 ? sd[2] * a.B + sd[1] : (d == 1 ? sd[2] * a.B + sd[0] : sd[1] * a.B + sd[0]);
    else j = d == 0 ? sd[1] : sd[0];
    for (int m = 0; m < a.V; m++)
      lduh[(c * nn + s) * a.V + m] -=
          (F[((2 * d + 1) * nf + j) * a.V + m] * T.fr[sd[d]] - F[((2 * d) * nf + j) * a.V + m] * T.fl[sd[d]]) * us;
  }
}

// lFhi in the reference's block layouts (x [z][y][x], y [z][x][y], z [y][x][z])
__global__ void k_volume_integral(NodeArgs a, double* lduh, const double* lFhi) {
  const int B = a.B;
  const int nn = a.dim == 3 ? B * B * B : B * B;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= a.ncells * nn) return;
  const long c = gid / nn;
  const int s = (int)(gid % nn);
  int sd[3];
  node_coords(s, B, a.dim, sd);
  const DGConst& T = c_dg[a.order];
  const double* F = lFhi + c * (a.dim + 1) * nn * a.V;
  double out[5] = {0, 0, 0, 0, 0};
  for (int d = 0; d < a.dim; d++) {
    double wprod = 1.0;
    for (int e = a.dim - 1; e >= 0; e--)
      if (e != d) wprod *= T.w[sd[e]];
    const double us = wprod / a.dx[d];
    for (int p = 0; p < B; p++) {
      int pos;
      if (a.dim == 3) {
        if (d == 0) pos = (sd[2] * B + sd[1]) * B + p;
        else if (d == 1) pos = (sd[2] * B + sd[0]) * B + p;
        else pos = (sd[1] * B + sd[0]) * B + p;
      } else {
        pos = d == 0 ? sd[1] * B + p : sd[0] * B + p;
      }
      const double k = T.kxi[sd[d]][p];
      for (int m = 0; m < a.V; m++) out[m] += k * F[(d * nn + pos) * a.V + m] * us;
    }
  }
  // source block (volumeIntegralNonlinear.cpph:104-122); zero for Euler
  double W = 1.0;
  for (int e = a.dim - 1; e >= 0; e--) W *= T.w[sd[e]];
  for (int m = 0; m < a.V; m++) out[m] += W * F[(a.dim * nn + s) * a.V + m];
  for (int m = 0; m < a.V; m++) lduh[(c * nn + s) * a.V + m] = out[m];
}

// per-cell stable dt; one warp per cell
__global__ void k_stable_dt(NodeArgs a, const double* luh, double* dt_cell,
                            unsigned long long* dt_min) {
  const int nn = a.dim == 3 ? a.B * a.B * a.B : a.B * a.B;
  const long c = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= a.ncells) return;
  double dt = DBL_MAX;
  for (int s = lane; s < nn; s += 32) {
    const double* q = luh + (c * nn + s) * a.D;
    double den = 0.0;
    for (int d = 0; d < a.dim; d++)
      den += (a.planar ? euler_max_eig<true>(q, d) : euler_max_eig<false>(q, d)) / a.dx[d];
    dt = fmin(dt, a.factor / den);
  }
  for (int o = 16; o > 0; o >>= 1) dt = fmin(dt, __shfl_xor_sync(0xffffffffu, dt, o));
  if (lane == 0) {
    if (dt_cell) dt_cell[c] = dt;
    if (dt_min) atomic_min_pos_double(dt_min, dt);
  }
}

// global minimum only: grid-stride over all nodes (consecutive threads read
// consecutive nodes), one atomic per CTA
__global__ void k_stable_dt_min(NodeArgs a, const double* luh, unsigned long long* dt_min) {
  __shared__ double wmin[8];
  const int nn = a.dim == 3 ? a.B * a.B * a.B : a.B * a.B;
  const long total = a.ncells * nn;
  double dt = DBL_MAX;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const double* q = luh + i * a.D;
    double den = 0.0;
    for (int d = 0; d < a.dim; d++)
      den += (a.planar ? euler_max_eig<true>(q, d) : euler_max_eig<false>(q, d)) / a.dx[d];
    dt = fmin(dt, a.factor / den);
  }
  for (int o = 16; o > 0; o >>= 1) dt = fmin(dt, __shfl_xor_sync(0xffffffffu, dt, o));
  if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = dt;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) dt = fmin(dt, wmin[w]);
    atomic_min_pos_double(dt_min, dt);
  }
}

// Rusanov on a face list; one warp per face, in place on lFhbnd
__global__ void k_riemann_faces(NodeArgs a, long nfaces, const int* left, const int* right,
                                const int* dir, const double* lQhbnd, double* lFhbnd) {
  const int B = a.B, nf = a.dim == 3 ? B * B : B;
  const long fidx = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (fidx >= nfaces) return;
  const int d = dir[fidx];
  const DGConst& T = c_dg[a.order];
  const long cl = left[fidx], cr = right[fidx];
  const double* QL = lQhbnd + (cl * 2 * a.dim + 2 * d + 1) * nf * a.D;
  const double* QR = lQhbnd + (cr * 2 * a.dim + 2 * d) * nf * a.D;
  double* FL = lFhbnd + (cl * 2 * a.dim + 2 * d + 1) * nf * a.V;
  double* FR = lFhbnd + (cr * 2 * a.dim + 2 * d) * nf * a.V;
  double avL[5] = {0, 0, 0, 0, 0}, avR[5] = {0, 0, 0, 0, 0};
  if (lane == 0) {
    for (int j = 0; j < nf; j++) {
      const double w = a.dim == 3 ? T.w[j / B] * T.w[j % B] : T.w[j];
      for (int m = 0; m < a.V; m++) {
        avL[m] += w * QL[j * a.D + m];
        avR[m] += w * QR[j * a.D + m];
      }
    }
  }
  for (int m = 0; m < 5; m++) {
    avL[m] = __shfl_sync(0xffffffffu, avL[m], 0);
    avR[m] = __shfl_sync(0xffffffffu, avR[m], 0);
  }
  const double smax = a.planar ? fmax(euler_max_eig<true>(avL, d), euler_max_eig<true>(avR, d))
                               : fmax(euler_max_eig<false>(avL, d), euler_max_eig<false>(avR, d));
  for (int k = lane; k < nf * a.V; k += 32) {
    const int j = k / a.V, m = k % a.V;
    const double f = 0.5 * (FR[k] + FL[k]) - 0.5 * smax * (QR[j * a.D + m] - QL[j * a.D + m]);
    FL[k] = f;
    FR[k] = f;
  }
}

static NodeArgs node_args(const exa_aderdg_desc_t& d, long ncells) {
  NodeArgs a;
  a.ncells = ncells;
  a.dim = d.dim;
  a.B = d.order + 1;
  a.V = d.nvar;
  a.D = d.nvar + d.npar;
  a.order = d.order;
  for (int i = 0; i < 3; i++) a.dx[i] = d.dx[i];
  a.dt = 0;
  a.factor = 0;
  a.planar = d.pde == EXA_PDE_EULER_PLANAR;
  return a;
}

static exa_status_t check_desc(const exa_aderdg_desc_t& d) {
  if ((d.dim != 2 && d.dim != 3) || d.order < 1 || d.order > kMaxOrder || d.nvar != kV ||
      d.npar < 0 || d.npar > 8)
    return set_error(EXA_EINVAL, "unsupported descriptor");
  return EXA_OK;
}

static unsigned grid_for(long work, int bs) { return (unsigned)((work + bs - 1) / bs); }

exa_status_t launch_solution_update(const exa_aderdg_desc_t& d, long ncells, double* luh,
                                    const double* lduh, double dt, cudaStream_t st) {
  if (exa_status_t s = check_desc(d)) return s;
  NodeArgs a = node_args(d, ncells);
  a.dt = dt;
  const long work = ncells * (d.dim == 3 ? a.B * a.B * a.B : a.B * a.B);
  if (work == 0) return EXA_OK;
  k_solution_update<<<grid_for(work, 256), 256, 0, st>>>(a, luh, lduh);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_solution_update");
}

exa_status_t launch_surface_integral(const exa_aderdg_desc_t& d, long ncells, double* lduh,
                                     const double* lFhbnd, cudaStream_t st) {
  if (exa_status_t s = check_desc(d)) return s;
  NodeArgs a = node_args(d, ncells);
  const long work = ncells * (d.dim == 3 ? a.B * a.B * a.B : a.B * a.B);
  if (work == 0) return EXA_OK;
  k_surface_integral<<<grid_for(work, 256), 256, 0, st>>>(a, lduh, lFhbnd);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_surface_integral");
}

exa_status_t launch_volume_integral(const exa_aderdg_desc_t& d, long ncells, double* lduh,
                                    const double* lFhi, cudaStream_t st) {
  if (exa_status_t s = check_desc(d)) return s;
  NodeArgs a = node_args(d, ncells);
  const long work = ncells * (d.dim == 3 ? a.B * a.B * a.B : a.B * a.B);
  if (work == 0) return EXA_OK;
  k_volume_integral<<<grid_for(work, 256), 256, 0, st>>>(a, lduh, lFhi);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_volume_integral");
}

exa_status_t launch_stable_dt(const exa_aderdg_desc_t& d, long ncells, const double* luh,
                              double factor, double* dt_cell, unsigned long long* dt_min,
                              cudaStream_t st) {
  if (exa_status_t s = check_desc(d)) return s;
  NodeArgs a = node_args(d, ncells);
  a.factor = factor;
  if (ncells == 0) return EXA_OK;
  if (!dt_cell && dt_min) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long nodes = ncells * (d.dim == 3 ? a.B * a.B * a.B : a.B * a.B);
    const long blocks = (nodes + 255) / 256;
    k_stable_dt_min<<<(unsigned)(blocks < 8L * sms ? blocks : 8L * sms), 256, 0, st>>>(a, luh, dt_min);
    count_launch();
    return cuda_status(cudaGetLastError(), "k_stable_dt_min");
  }
  k_stable_dt<<<grid_for(ncells * 32, 256), 256, 0, st>>>(a, luh, dt_cell, dt_min);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_stable_dt");
}

exa_status_t launch_riemann_faces(const exa_aderdg_desc_t& d, long nfaces, const int* left,
                                  const int* right, const int* dir, const double* lQhbnd,
                                  double* lFhbnd, cudaStream_t st) {
  if (exa_status_t s = check_desc(d)) return s;
  NodeArgs a = node_args(d, 0);
  if (nfaces == 0) return EXA_OK;
  k_riemann_faces<<<grid_for(nfaces * 32, 256), 256, 0, st>>>(a, nfaces, left, right, dir,
                                                              lQhbnd, lFhbnd);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_riemann_faces");
}

// ------------------------------------------------------ initial condition
__device__ __forceinline__ double noise_u01(unsigned long long seed, unsigned long long idx) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (idx + 1ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

struct ICArgs {
  long ncells;
  long cell_offset;
  int dim, B, order, kind;
  int n[3];
  double dx[3];
  double param, noise;
  unsigned long long seed;
};

__global__ void k_grid_ic(ICArgs a, double* luh) {
  const int nn = a.dim == 3 ? a.B * a.B * a.B : a.B * a.B;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= a.ncells * nn) return;
  const long c = gid / nn + a.cell_offset;  // index in the whole domain
  const int s = (int)(gid % nn);
  const int cx = (int)(c % a.n[0]), cy = (int)((c / a.n[0]) % a.n[1]);
  const unsigned long long node = (unsigned long long)c * nn + s;
  const int ix = s % a.B, iy = (s / a.B) % a.B;
  const double* nodes = c_dg[a.order].nodes;
  const double x = (cx + nodes[ix]) * a.dx[0];
  const double y = (cy + nodes[iy]) * a.dx[1];
  const double nz = a.noise != 0.0 ? a.noise * (2.0 * noise_u01(a.seed, node) - 1.0) : 0.0;
  const double pi = 3.14159265358979323846;
  double rho, u, v, p;
  if (a.kind == 0) {
    const double eps = a.param, R = 0.1;
    const double xb = (x - 0.5) / R, yb = (y - 0.5) / R;
    const double r2 = xb * xb + yb * yb;
    const double e = exp(0.5 * (1.0 - r2));
    u = 1.0 - eps / (2 * pi) * yb * e;
    v = 1.0 + eps / (2 * pi) * xb * e;
    const double Tm = 1.0 - (kGamma - 1) * eps * eps / (8 * kGamma * pi * pi) * e * e;
    rho = pow(Tm, 1.0 / (kGamma - 1));
    p = rho * Tm;
  } else {
    rho = 1.0 + a.param * sin(2 * pi * (x + y));
    u = 1.0;
    v = 1.0;
    p = 1.0;
  }
  const double r = rho * (1.0 + nz);
  double* Q = luh + gid * 5;
  Q[0] = r;
  Q[1] = r * u;
  Q[2] = r * v;
  Q[3] = 0.0;
  Q[4] = p / (kGamma - 1) + 0.5 * r * (u * u + v * v);
}

exa_status_t launch_grid_ic(int dim, int order, const int* n, const double* dx, double* luh,
                            int kind, double param, uint64_t seed, double noise,
                            cudaStream_t st, long cell_offset, int n_last_global) {
  ICArgs a;
  a.cell_offset = cell_offset;
  a.dim = dim;
  a.order = order;
  a.B = order + 1;
  a.kind = kind;
  a.ncells = 1;
  for (int i = 0; i < 3; i++) {
    a.n[i] = i < dim ? n[i] : 1;
    a.dx[i] = dx[i];
    a.ncells *= a.n[i];
  }
  // coordinates come from the whole-domain index: the last dimension spans
  // n_last_global cells there
  if (n_last_global > 0) a.n[dim - 1] = n_last_global;
  a.param = param;
  a.noise = noise;
  a.seed = seed;
  const long work = a.ncells * (dim == 3 ? a.B * a.B * a.B : a.B * a.B);
  k_grid_ic<<<grid_for(work, 256), 256, 0, st>>>(a, luh);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_grid_ic");
}

exa_status_t upload_tables_faces() {
  size_t bytes = 0;
  const void* h = host_dg_tables(&bytes);
  return cuda_status(cudaMemcpyToSymbol(c_dg, h, bytes), "upload tables (faces)");
}

}  // namespace exa
