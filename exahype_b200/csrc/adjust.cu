// Solution adjustment: the reference's solutionAdjustment kernel
// (kernels/aderdg/generic/c/3d/solutionAdjustment.cpph:17-52, 2D
// c/2d/solutionAdjustment.cpph) calls the solver's adjustPointSolution hook
// at every Gauss-Legendre node of a cell, x = center + dx (xi - 1/2), with
// the node's weight, t and dt.  The hooks here are built-in device forms
// (exa_adjust_t); one thread per node.
#include "exa_device.cuh"

namespace exa {

struct AdjArgs {
  long ncells;
  int dim, order, B;
  double dx[3];
  const double* centers;  // [ncells][dim], or nullptr: grid cell (i + 1/2) dx
  int n[3];               // grid extents (centers == nullptr)
  double t, dt;           // or, with time_dev: t = *time_dev + *dt_dev
  const double* time_dev;
  const double* dt_dev;
  exa_adjust_t hook;
};

// the built-in adjustPointSolution forms (Q = 5 Euler variables, gamma 1.4)
__device__ __forceinline__ void adjust_point(const exa_adjust_t& h, int dim, const double* x, double t, double dt,
                                             double* Q) {
  const double pi = 3.14159265358979323846;
  if (h.kind == EXA_ADJUST_SINE_WAVE) {
    const double rho = 1.0 + h.param[0] * sin(2 * pi * (x[0] + x[1]));
    const double u = 1.0, v = 1.0, p = 1.0;
    Q[0] = rho;
    Q[1] = rho * u;
    Q[2] = rho * v;
    Q[3] = 0.0;
    Q[4] = p / (kGamma - 1) + 0.5 * rho * (u * u + v * v);
  } else if (h.kind == EXA_ADJUST_ISENTROPIC_VORTEX) {
    const double eps = h.param[0], R = 0.1;
    const double xb = (x[0] - 0.5) / R, yb = (x[1] - 0.5) / R;
    const double r2 = xb * xb + yb * yb;
    const double e = exp(0.5 * (1.0 - r2));
    const double u = 1.0 - eps / (2 * pi) * yb * e;
    const double v = 1.0 + eps / (2 * pi) * xb * e;
    const double Tm = 1.0 - (kGamma - 1) * eps * eps / (8 * kGamma * pi * pi) * e * e;
    const double rho = pow(Tm, 1.0 / (kGamma - 1));
    const double p = rho * Tm;
    Q[0] = rho;
    Q[1] = rho * u;
    Q[2] = rho * v;
    Q[3] = 0.0;
    Q[4] = p / (kGamma - 1) + 0.5 * rho * (u * u + v * v);
  } else if (h.kind == EXA_ADJUST_HEAT_SOURCE) {
    double r2 = 0.0;
    for (int d = 0; d < dim; d++) r2 += (x[d] - h.param[3 + d]) * (x[d] - h.param[3 + d]);
    Q[4] += dt * h.param[0] * exp(-r2 / (h.param[1] * h.param[1])) * (1.0 + sin(2 * pi * h.param[2] * t));
  }
}

__global__ void k_adjust(AdjArgs a, double* luh) {
  const int B = a.B;
  const int nn = a.dim == 3 ? B * B * B : B * B;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= a.ncells * nn) return;
  const long c = gid / nn;
  const int s = (int)(gid % nn);
  const DGConst& T = c_dg[a.order];
  double ctr[3];
  if (a.centers) {
    for (int d = 0; d < a.dim; d++) ctr[d] = a.centers[c * a.dim + d];
  } else {
    const int ci[3] = {(int)(c % a.n[0]), (int)((c / a.n[0]) % a.n[1]), (int)(c / ((long)a.n[0] * a.n[1]))};
    for (int d = 0; d < a.dim; d++) ctr[d] = (ci[d] + 0.5) * a.dx[d];
  }
  // node s = ((i B + j) B + k) in 3D (i slowest, as the reference's loops),
  // (i B + j) in 2D; the fastest index runs along x
  double x[3];
  if (a.dim == 3) {
    const int k = s % B, j = (s / B) % B, i = s / (B * B);
    x[2] = ctr[2] + a.dx[2] * (T.nodes[i] - 0.5);
    x[1] = ctr[1] + a.dx[1] * (T.nodes[j] - 0.5);
    x[0] = ctr[0] + a.dx[0] * (T.nodes[k] - 0.5);
  } else {
    const int j = s % B, i = s / B;
    x[0] = ctr[0] + a.dx[0] * (T.nodes[j] - 0.5);
    x[1] = ctr[1] + a.dx[1] * (T.nodes[i] - 0.5);
    x[2] = 0.0;
  }
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;
  const double t = a.time_dev ? *a.time_dev + dt : a.t;
  adjust_point(a.hook, a.dim, x, t, dt, luh + gid * kV);
}

static exa_status_t check_hook(const exa_adjust_t* h) {
  if (!h) return set_error(EXA_EINVAL, "NULL adjustment hook");
  if (h->kind < EXA_ADJUST_NONE || h->kind > EXA_ADJUST_HEAT_SOURCE) return set_error(EXA_EINVAL, "unknown hook");
  if (h->when != EXA_ADJUST_AT_START && h->when != EXA_ADJUST_ALWAYS)
    return set_error(EXA_EINVAL, "adjustment: when must be EXA_ADJUST_AT_START or EXA_ADJUST_ALWAYS");
  if (h->kind == EXA_ADJUST_HEAT_SOURCE && !(h->param[1] > 0.0))
    return set_error(EXA_EINVAL, "heat source: width must be positive");
  return EXA_OK;
}

static exa_status_t launch_adjust(const AdjArgs& a, double* luh, cudaStream_t st) {
  const long work = a.ncells * (a.dim == 3 ? (long)a.B * a.B * a.B : (long)a.B * a.B);
  if (work == 0) return EXA_OK;
  k_adjust<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(a, luh);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_adjust");
}

exa_status_t grid_adjust(int dim, int order, const int* n, const double* dx, long ncells, double* luh,
                         const double* time_dev, const double* dt_dev, const exa_adjust_t& hook, cudaStream_t st) {
  AdjArgs a{};
  a.ncells = ncells;
  a.dim = dim;
  a.order = order;
  a.B = order + 1;
  for (int d = 0; d < 3; d++) {
    a.dx[d] = d < dim ? dx[d] : 1.0;
    a.n[d] = d < dim ? n[d] : 1;
  }
  a.time_dev = time_dev;
  a.dt_dev = dt_dev;
  a.hook = hook;
  return launch_adjust(a, luh, st);
}

exa_status_t check_adjust_hook(const exa_adjust_t* h) { return check_hook(h); }

// this file's copy of the DG constants (every translation unit has its own)
exa_status_t upload_tables_adjust() {
  size_t bytes = 0;
  const void* h = host_dg_tables(&bytes);
  return cuda_status(cudaMemcpyToSymbol(c_dg, h, bytes), "upload tables (adjust)");
}

}  // namespace exa

using namespace exa;

extern "C" {

exa_status_t exa_aderdg_solution_adjustment(const exa_aderdg_desc_t* desc, long ncells, double* luh,
                                            const double* centers, double t, double dt,
                                            const exa_adjust_t* hook, void* stream) {
  if (!desc) return set_error(EXA_EINVAL, "NULL descriptor");
  if (desc->dim != 2 && desc->dim != 3) return set_error(EXA_EINVAL, "dim must be 2 or 3");
  if (desc->order < 1 || desc->order > kMaxOrder) return set_error(EXA_EINVAL, "unsupported order");
  if (desc->nvar != kV || desc->npar != 0) return set_error(EXA_EINVAL, "adjustment: nvar 5, npar 0");
  if (exa_status_t s = check_hook(hook)) return s;
  if (ncells < 0 || !luh || !centers) return set_error(EXA_EINVAL, "bad argument");
  if (exa_status_t s = ensure_tables()) return s;
  // useAdjustSolution of the demonstrators: the start of the run only
  if (hook->kind == EXA_ADJUST_NONE || (hook->when == EXA_ADJUST_AT_START && t != 0.0)) return EXA_OK;
  AdjArgs a{};
  a.ncells = ncells;
  a.dim = desc->dim;
  a.order = desc->order;
  a.B = desc->order + 1;
  for (int d = 0; d < 3; d++) a.dx[d] = d < desc->dim ? desc->dx[d] : 1.0;
  a.centers = centers;
  a.t = t;
  a.dt = dt;
  a.hook = *hook;
  return launch_adjust(a, luh, as_stream(stream));
}

}  // extern "C"
