// Uniform periodic ADER-DG grid on one GPU: the device-side replacement for
// the Peano spacetree + ADERDGSolver bookkeeping of the reference.
//
// One time step (reference non-fused order, exahype/runners/Runner.cpp:
// 1125-1160):
//   k_predictor   spaceTimePredictor + volumeIntegral, dt read on the device
//   k_corrector   Riemann on all faces + surfaceIntegral + solutionUpdate,
//                 and the next dt (min over nodes, atomic min over cells)
//   k_commit      one thread: time += dt, log dt, dt <- next, reset slot
// Nothing returns to the host inside a step, so a step is a fixed sequence
// of launches that a CUDA graph replays.
#include <cstring>
#include <new>
#include <float.h>

#include "exa_device.cuh"

namespace exa {
double host_pnpm(int order);

struct GridDev {
  double dt;                     // dt of the current step
  unsigned long long dt_next;    // atomic-min slot (bit pattern)
  double time;
  unsigned long long step;
  unsigned long long stats[2];   // sum of Picard iterations, non-converged cells
  int nan_flag;
  // debug scan (exa_aderdg_grid_set_debug): the first array seen holding a
  // non-finite value (1 lduh, 2 lQhbnd, 3 lFhbnd after the predictor; 4 luh
  // after the update), the step and the element index
  int nan_where;
  unsigned long long nan_step;
  unsigned long long nan_index;
};

__global__ void k_debug_reset(GridDev* g) {
  g->nan_where = 0;
  g->nan_step = ~0ULL;  // not yet recorded
  g->nan_index = ~0ULL;
}

// Debug scan of one array for non-finite values; the first array of the
// first step to hold one is recorded (later scans leave it), with the
// smallest such element index of that array.
__global__ void k_scan_nonfinite(const double* a, long n, int where, GridDev* g) {
  const long stride = (long)gridDim.x * blockDim.x;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (isfinite(a[i])) continue;
    const int prev = atomicCAS(&g->nan_where, 0, where);
    if (prev == 0) {
      atomicExch(&g->nan_step, g->step);
      g->nan_flag = 1;
    }
    // the index only from the recording scan (the step's other threads may
    // still see the step unrecorded; a later step sees it recorded)
    const unsigned long long ns = atomicAdd(&g->nan_step, 0ULL);
    if (prev == 0 || (prev == where && (ns == ~0ULL || ns == g->step)))
      atomicMin(&g->nan_index, (unsigned long long)i);
  }
}

__global__ void k_commit(GridDev* g, double* dt_log, int log_cap, int fixed, double dt_fixed) {
  const double dt = g->dt;
  g->time += dt;
  dt_log[g->step % (unsigned long long)log_cap] = dt;
  g->step += 1;
  if (fixed) {
    g->dt = dt_fixed;
  } else {
    g->dt = __longlong_as_double((long long)g->dt_next);
    g->dt_next = 0x7FF0000000000000ULL;  // +inf
  }
}

__global__ void k_prime(GridDev* g) {
  g->dt = __longlong_as_double((long long)g->dt_next);
  g->dt_next = 0x7FF0000000000000ULL;
}

// Slab boundary faces -> send buffers.  The lowest layer's lower face of the
// last dimension (face 2(dim-1)) goes to the slab below, the highest layer's
// upper face (face 2(dim-1)+1) to the slab above; both as
// [layer cell][Q | F][face node][var].  One thread per double of a face.
__global__ void k_halo_pack(long layer, long ncells, int fv, int nfv, int fdim, const double* qb,
                            const double* fb, double* send_lo, double* send_hi) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= 2 * layer * nfv) return;
  const bool hi = gid >= layer * nfv;
  const long k = hi ? gid - layer * nfv : gid;
  const long lc = k / nfv;
  const int r = (int)(k % nfv);
  const long cell = hi ? ncells - layer + lc : lc;
  const long src = cell * fv + (long)(2 * fdim + (hi ? 1 : 0)) * nfv + r;
  double* dst = (hi ? send_hi : send_lo) + lc * 2 * nfv;
  dst[r] = qb[src];
  dst[nfv + r] = fb[src];
}

}  // namespace exa

using namespace exa;

struct exa_aderdg_grid {
  exa_aderdg_grid_config_t cfg;
  exa_aderdg_desc_t desc;
  int device = 0;
  long ncells = 0;
  cudaStream_t st = nullptr;
  double* luh = nullptr;
  double* lduh = nullptr;
  double* qb = nullptr;
  double* fb = nullptr;
  GridDev* gd = nullptr;
  double* dt_log = nullptr;
  // slab decomposition (exa_aderdg_grid_set_halo): send / receive buffers
  double* halo = nullptr;  // send_lo | send_hi | recv_lo | recv_hi
  long layer = 0;          // cells in one layer of the last dimension
  size_t halo_count = 0;   // doubles per buffer
  int bc[3] = {0, 0, 0};   // EXA_BC_* per dimension
  int log_cap = 4096;
  double dt_factor = 0;
  bool primed = false;
  bool use_graph = false;
  bool debug = false;  // scan each phase's outputs for non-finite values
  cudaGraphExec_t graph = nullptr;
  // optional per-phase CUDA-event timing (predictor / corrector+commit)
  bool profile = false;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  double ms_pred = 0, ms_corr = 0;
  unsigned long long prof_steps = 0;
  uint64_t graph_launches = 3;  // kernels in one captured step
  // solution adjustment after every update (exa_aderdg_grid_set_adjustment)
  bool adj_on = false;
  exa_adjust_t adj{};
  // a-posteriori subcell limiter (exa_aderdg_grid_set_limiter)
  bool lim_on = false;
  exa_limiter_config_t lim_cfg{};
  int lim_ghost = 0;
  void* lim_block = nullptr;    // one allocation, carved below
  double* lim_prev = nullptr;   // luh before the step
  double* lim_patch = nullptr;  // subcell patches [cell][(S + 2g)^2][V]
  double* lim_bmin = nullptr;   // [cell][4 faces][nobs]
  double* lim_bmax = nullptr;
  double* lim_loc = nullptr;    // [cell][min | max][nobs]
  int* lim_ok = nullptr;        // DMP and admissibility verdict per cell
  int* lim_status = nullptr;
  int* lim_status_tmp = nullptr;
  int* lim_cure = nullptr;
  int* lim_list_patch = nullptr;
  int* lim_list_fv = nullptr;
  int* lim_counts = nullptr;    // patches, FV cells, Troubled cells
};

static size_t grid_sizes(const exa_aderdg_grid_config_t* c, long* ncells, size_t* n_luh,
                         size_t* n_face) {
  long nc = 1;
  for (int i = 0; i < c->dim; i++) nc *= c->n[i];
  const int B = c->order + 1;
  size_t nn = 1, nf = 1;
  for (int i = 0; i < c->dim; i++) nn *= B;
  for (int i = 0; i < c->dim - 1; i++) nf *= B;
  *ncells = nc;
  *n_luh = nc * nn * kV;
  *n_face = nc * 2 * c->dim * nf * kV;
  return sizeof(double) * (2 * *n_luh + 2 * *n_face) + sizeof(GridDev) + 4096 * sizeof(double);
}

static exa_status_t grid_prime(exa_aderdg_grid* g) {
  if (g->cfg.dt_policy == 2) {
    GridDev h{};
    h.dt = g->cfg.dt_fixed;
    h.dt_next = 0x7FF0000000000000ULL;
    // keep time/step/stats: only overwrite dt fields
    cudaError_t e = cudaMemcpyAsync(&g->gd->dt, &h.dt, sizeof(double), cudaMemcpyHostToDevice, g->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
    if (e != cudaSuccess) return cuda_status(e, "prime fixed dt");
    g->primed = true;
    return EXA_OK;
  }
  const unsigned long long inf = 0x7FF0000000000000ULL;
  cudaError_t e = cudaMemcpyAsync(&g->gd->dt_next, &inf, 8, cudaMemcpyHostToDevice, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  if (e != cudaSuccess) return cuda_status(e, "prime dt slot");
  if (exa_status_t s = launch_stable_dt(g->desc, g->ncells, g->luh, g->dt_factor, nullptr,
                                        &g->gd->dt_next, g->st))
    return s;
  k_prime<<<1, 1, 0, g->st>>>(g->gd);
  count_launch();
  if (exa_status_t s = cuda_status(cudaGetLastError(), "k_prime")) return s;
  g->primed = true;
  return EXA_OK;
}

static exa_status_t grid_predict(exa_aderdg_grid* g) {
  PredArgs a{};
  a.ncells = g->ncells;
  a.luh = g->luh;
  a.dt = 0.0;
  a.dt_dev = &g->gd->dt;
  for (int i = 0; i < 3; i++) a.idx[i] = i < g->cfg.dim ? 1.0 / g->desc.dx[i] : 0.0;
  a.lduh = g->lduh;
  a.lQhbnd = g->qb;
  a.lFhbnd = g->fb;
  a.iters = nullptr;
  a.stats = g->gd->stats;
  a.precision = g->cfg.precision;
  if (exa_status_t s = launch_predictor(g->desc, a, 0, g->st)) return s;
  if (g->halo) {
    const int B = g->cfg.order + 1;
    const int nfv = (g->cfg.dim == 3 ? B * B : B) * kV;
    const long work = 2 * g->layer * nfv;
    k_halo_pack<<<(unsigned)((work + 255) / 256), 256, 0, g->st>>>(
        g->layer, g->ncells, 2 * g->cfg.dim * nfv, nfv, g->cfg.dim - 1, g->qb, g->fb, g->halo,
        g->halo + g->halo_count);
    count_launch();
    if (exa_status_t s = cuda_status(cudaGetLastError(), "k_halo_pack")) return s;
  }
  return EXA_OK;
}

static exa_status_t grid_correct(exa_aderdg_grid* g) {
  CorrArgs c{};
  c.ncells = g->ncells;
  for (int i = 0; i < 3; i++) {
    c.n[i] = i < g->cfg.dim ? g->cfg.n[i] : 1;
    c.dx[i] = g->desc.dx[i];
  }
  c.dt_dev = &g->gd->dt;
  c.luh = g->luh;
  c.lduh = g->lduh;
  c.lQhbnd = g->qb;
  c.lFhbnd = g->fb;
  // with the limiter the candidate may be unusable in troubled cells: the
  // next dt and the NaN check come after the limiting
  c.dt_next = (g->cfg.dt_policy == 2 || g->lim_on || g->adj_on) ? nullptr : &g->gd->dt_next;
  c.dt_factor = g->dt_factor;
  c.nan_flag = g->lim_on ? nullptr : &g->gd->nan_flag;
  if (g->halo) {
    c.halo_lo = g->halo + 2 * g->halo_count;
    c.halo_hi = g->halo + 3 * g->halo_count;
  }
  for (int i = 0; i < 3; i++) {
    c.bc[i] = i < g->cfg.dim ? g->bc[i] : 0;
    c.bc_any |= c.bc[i] != 0;
  }
  return launch_corrector(g->cfg.dim, g->cfg.order, g->cfg.pde, c, g->st);
}

// The limiting part of a step (LimitingADERDGSolver: updateLimiterStatus-
// AndMinAndMaxAfterSolutionUpdate, then the local recomputation of the
// cells whose dominant solver is the FV solver), after the DG candidate:
//   DMP (bounds merged from the previous step) + admissibility -> status;
//   subcell patches of the previous solution for every cell with status >=
//   NeighbourOfTroubled3; one FV step on the patches of the cells with status
//   >= NeighbourOfTroubled2, projected back onto their DG polynomials;
//   new extrema (FV patch for those cells, nodes / Lobatto points / subcells
//   of the candidate for the others) merged over faces; the next dt from the
//   final state.
static exa_status_t grid_limit(exa_aderdg_grid* g) {
  const exa_limiter_config_t& L = g->lim_cfg;
  const int dim = g->cfg.dim, order = g->cfg.order, nobs = L.nobs;
  const int S = 2 * order + 1, npc = dim == 3 ? (order + 1) * (order + 1) * (order + 1) : (order + 1) * (order + 1);
  const int planar = g->cfg.pde == EXA_PDE_EULER_PLANAR;
  if (exa_status_t s = limiter_launch(kLimDmp, dim, order, kV, nobs, 0, g->ncells, g->luh, nullptr, g->lim_bmin,
                                      g->lim_bmax, g->lim_ok, L.relaxation, L.difference_scaling, g->st, nullptr,
                                      nullptr))
    return s;
  if (exa_status_t s = limiting_status(dim, g->cfg.n, g->bc, npc, planar, L.check_admissibility,
                                       L.steps_till_cured, g->luh, g->lim_ok, g->lim_status, g->lim_status_tmp,
                                       g->lim_cure, g->lim_list_patch, g->lim_list_fv, g->lim_counts, g->st))
    return s;
  if (exa_status_t s = limiter_launch(kLimToFv, dim, order, kV, 0, g->lim_ghost, g->ncells, g->lim_prev,
                                      g->lim_patch, nullptr, nullptr, nullptr, 0, 0, g->st, g->lim_list_patch,
                                      g->lim_counts + 0))
    return s;
  if (dim == 2) {
    if (exa_status_t s = fv_subcell_step(L.scheme, planar, S, g->lim_ghost, g->cfg.n[0], g->cfg.n[1],
                                         g->desc.dx[0] / S, g->desc.dx[1] / S, g->lim_patch, g->lim_list_fv,
                                         g->lim_counts + 1, g->ncells, &g->gd->dt, g->st, g->bc))
      return s;
  } else {
    const double h[3] = {g->desc.dx[0] / S, g->desc.dx[1] / S, g->desc.dx[2] / S};
    if (exa_status_t s = fv3_subcell_step(L.scheme, S, g->lim_ghost, g->cfg.n, h, g->lim_patch, g->lim_list_fv,
                                          g->lim_counts + 1, g->ncells, &g->gd->dt, g->st, g->bc))
      return s;
  }
  if (exa_status_t s = limiter_launch(kLimToDg, dim, order, kV, 0, g->lim_ghost, g->ncells, g->lim_patch, g->luh,
                                      nullptr, nullptr, nullptr, 0, 0, g->st, g->lim_list_fv, g->lim_counts + 1))
    return s;
  if (exa_status_t s = limiter_launch(kLimFvMinMax, dim, order, kV, nobs, g->lim_ghost, g->ncells, g->lim_patch,
                                      nullptr, g->lim_bmin, g->lim_bmax, nullptr, 0, 0, g->st, g->lim_list_fv,
                                      g->lim_counts + 1))
    return s;
  if (exa_status_t s = limiting_merge_bounds(dim, g->cfg.n, g->bc, nobs, g->lim_bmin, g->lim_bmax, g->lim_loc, g->st))
    return s;
  if (exa_status_t s = limiting_check_finite(npc, g->luh, g->lim_list_fv, g->lim_counts + 1, &g->gd->nan_flag, g->st))
    return s;
  if (g->cfg.dt_policy != 2)
    return launch_stable_dt(g->desc, g->ncells, g->luh, g->dt_factor, nullptr, &g->gd->dt_next, g->st);
  return EXA_OK;
}

// extrema of the current state merged over faces (the bounds of the first
// DMP check), all cells Ok
static exa_status_t grid_limiter_reset(exa_aderdg_grid* g) {
  const int nobs = g->lim_cfg.nobs;
  cudaError_t e = cudaMemsetAsync(g->lim_status, 0, g->ncells * sizeof(int), g->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->lim_cure, 0, g->ncells * sizeof(int), g->st);
  if (e != cudaSuccess) return cuda_status(e, "limiter reset");
  if (exa_status_t s = limiter_launch(kLimMinMax, g->cfg.dim, g->cfg.order, kV, nobs, 0, g->ncells, g->luh, nullptr,
                                      g->lim_bmin, g->lim_bmax, nullptr, 0, 0, g->st, nullptr, nullptr))
    return s;
  if (exa_status_t s = limiting_merge_bounds(g->cfg.dim, g->cfg.n, g->bc, nobs, g->lim_bmin, g->lim_bmax, g->lim_loc, g->st))
    return s;
  return cuda_status(cudaStreamSynchronize(g->st), "limiter reset");
}

// debug scans: after the predictor (after = 0) its three output arrays,
// after the update (after = 1) the state
static exa_status_t grid_scan(exa_aderdg_grid* g, int after) {
  long nc;
  size_t n_luh, n_face;
  grid_sizes(&g->cfg, &nc, &n_luh, &n_face);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned grid = (unsigned)(4 * sms);
  if (after == 0) {
    k_scan_nonfinite<<<grid, 256, 0, g->st>>>(g->lduh, (long)n_luh, 1, g->gd);
    k_scan_nonfinite<<<grid, 256, 0, g->st>>>(g->qb, (long)n_face, 2, g->gd);
    k_scan_nonfinite<<<grid, 256, 0, g->st>>>(g->fb, (long)n_face, 3, g->gd);
    count_launch(3);
  } else {
    k_scan_nonfinite<<<grid, 256, 0, g->st>>>(g->luh, (long)n_luh, 4, g->gd);
    count_launch();
  }
  return cuda_status(cudaGetLastError(), "k_scan_nonfinite");
}

static exa_status_t grid_commit(exa_aderdg_grid* g) {
  k_commit<<<1, 1, 0, g->st>>>(g->gd, g->dt_log, g->log_cap, g->cfg.dt_policy == 2, g->cfg.dt_fixed);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_commit");
}

static exa_status_t grid_launch_step(exa_aderdg_grid* g) {
  if (g->profile) cudaEventRecord(g->ev[0], g->st);
  if (g->lim_on) {
    long nc;
    size_t n_luh, n_face;
    grid_sizes(&g->cfg, &nc, &n_luh, &n_face);
    cudaError_t e = cudaMemcpyAsync(g->lim_prev, g->luh, n_luh * sizeof(double), cudaMemcpyDeviceToDevice, g->st);
    if (e != cudaSuccess) return cuda_status(e, "limiter: keep previous solution");
  }
  if (exa_status_t s = grid_predict(g)) return s;
  if (g->debug)
    if (exa_status_t s = grid_scan(g, 0)) return s;
  if (g->profile) cudaEventRecord(g->ev[1], g->st);
  if (exa_status_t s = grid_correct(g)) return s;
  if (g->lim_on)
    if (exa_status_t s = grid_limit(g)) return s;
  if (g->adj_on) {
    // ADERDGSolver::updateSolution (:2158-2170): the hook after the update
    // at t + dt; the next dt from the adjusted state
    if (exa_status_t s = grid_adjust(g->cfg.dim, g->cfg.order, g->cfg.n, g->desc.dx, g->ncells, g->luh,
                                     &g->gd->time, &g->gd->dt, g->adj, g->st))
      return s;
    if (g->cfg.dt_policy != 2)
      if (exa_status_t s = launch_stable_dt(g->desc, g->ncells, g->luh, g->dt_factor, nullptr, &g->gd->dt_next, g->st))
        return s;
  }
  if (g->debug)
    if (exa_status_t s = grid_scan(g, 1)) return s;
  if (exa_status_t s = grid_commit(g)) return s;
  if (g->profile) {
    cudaEventRecord(g->ev[2], g->st);
    cudaError_t e = cudaEventSynchronize(g->ev[2]);
    if (e != cudaSuccess) return cuda_status(e, "profile sync");
    float a1 = 0, a2 = 0;
    cudaEventElapsedTime(&a1, g->ev[0], g->ev[1]);
    cudaEventElapsedTime(&a2, g->ev[1], g->ev[2]);
    g->ms_pred += a1;
    g->ms_corr += a2;
    g->prof_steps++;
  }
  return EXA_OK;
}

extern "C" {

size_t exa_aderdg_grid_footprint(const exa_aderdg_grid_config_t* cfg) {
  if (!cfg) return 0;
  long nc;
  size_t a, b;
  return grid_sizes(cfg, &nc, &a, &b);
}

exa_status_t exa_aderdg_grid_create(const exa_aderdg_grid_config_t* cfg, exa_aderdg_grid** out) {
  if (!cfg || !out) return set_error(EXA_EINVAL, "NULL argument");
  if (cfg->dim != 2 && cfg->dim != 3) return set_error(EXA_EINVAL, "dim must be 2 or 3");
  if (cfg->order < 2 || cfg->order > 5) return set_error(EXA_EINVAL, "order must be in 2..5");
  for (int i = 0; i < cfg->dim; i++)
    if (cfg->n[i] < 1 || !(cfg->length[i] > 0)) return set_error(EXA_EINVAL, "bad grid size");
  if (cfg->dt_policy < 0 || cfg->dt_policy > 2) return set_error(EXA_EINVAL, "bad dt_policy");
  if (cfg->dt_policy == 2 && !(cfg->dt_fixed > 0)) return set_error(EXA_EINVAL, "dt_fixed must be > 0");
  if (!(cfg->cfl > 0)) return set_error(EXA_EINVAL, "cfl must be > 0");
  if (cfg->precision != EXA_PREC_FP64 && cfg->precision != EXA_PREC_MIXED)
    return set_error(EXA_EINVAL, "bad precision");
  exa_aderdg_grid* g = new (std::nothrow) exa_aderdg_grid;
  if (!g) return set_error(EXA_ENOMEM, "host allocation");
  g->cfg = *cfg;
  g->desc.dim = cfg->dim;
  g->desc.order = cfg->order;
  g->desc.nvar = kV;
  g->desc.npar = 0;
  g->desc.pde = cfg->pde;
  g->desc.precision = cfg->precision;
  for (int i = 0; i < 3; i++) g->desc.dx[i] = i < cfg->dim ? cfg->length[i] / cfg->n[i] : 1.0;
  g->dt_factor = cfg->dt_policy == 0 ? cfg->cfl * host_pnpm(cfg->order)
                                     : cfg->cfl / (2 * cfg->order + 1);
  cudaGetDevice(&g->device);
  exa_status_t s = ensure_tables();
  size_t n_luh, n_face;
  grid_sizes(cfg, &g->ncells, &n_luh, &n_face);
  cudaError_t e = cudaSuccess;
  if (!s) e = cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking);
  if (!s && e == cudaSuccess) e = cudaMalloc(&g->luh, n_luh * sizeof(double));
  if (!s && e == cudaSuccess) e = cudaMalloc(&g->lduh, n_luh * sizeof(double));
  if (!s && e == cudaSuccess) e = cudaMalloc(&g->qb, n_face * sizeof(double));
  if (!s && e == cudaSuccess) e = cudaMalloc(&g->fb, n_face * sizeof(double));
  if (!s && e == cudaSuccess) e = cudaMalloc(&g->gd, sizeof(GridDev));
  if (!s && e == cudaSuccess) e = cudaMalloc(&g->dt_log, g->log_cap * sizeof(double));
  if (!s && e == cudaSuccess) e = cudaMemsetAsync(g->gd, 0, sizeof(GridDev), g->st);
  if (!s && e == cudaSuccess) e = cudaMemsetAsync(g->luh, 0, n_luh * sizeof(double), g->st);
  if (!s && e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  if (!s && e != cudaSuccess) s = cuda_status(e, "grid allocation");
  if (s) {
    exa_aderdg_grid_destroy(g);
    return s;
  }
  *out = g;
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_destroy(exa_aderdg_grid* g) {
  if (!g) return EXA_OK;
  if (g->st) cudaStreamSynchronize(g->st);
  if (g->graph) cudaGraphExecDestroy(g->graph);
  for (int i = 0; i < 3; i++)
    if (g->ev[i]) cudaEventDestroy(g->ev[i]);
  cudaFree(g->luh);
  cudaFree(g->lduh);
  cudaFree(g->qb);
  cudaFree(g->fb);
  cudaFree(g->gd);
  cudaFree(g->dt_log);
  cudaFree(g->halo);
  cudaFree(g->lim_block);
  if (g->st) cudaStreamDestroy(g->st);
  delete g;
  return EXA_OK;
}

long exa_aderdg_grid_ncells(const exa_aderdg_grid* g) { return g ? g->ncells : 0; }

exa_status_t exa_aderdg_grid_init(exa_aderdg_grid* g, int kind, double param, uint64_t seed,
                                  double noise_amp) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (kind < 0 || kind > 1) return set_error(EXA_EINVAL, "unknown initial condition");
  if (exa_status_t s = launch_grid_ic(g->cfg.dim, g->cfg.order, g->cfg.n, g->desc.dx, g->luh, kind,
                                      param, seed, noise_amp, g->st))
    return s;
  g->primed = false;
  if (g->lim_on)
    if (exa_status_t s = grid_limiter_reset(g)) return s;
  return cuda_status(cudaStreamSynchronize(g->st), "grid init");
}

exa_status_t exa_aderdg_grid_set_state(exa_aderdg_grid* g, const double* host_luh) {
  if (!g || !host_luh) return set_error(EXA_EINVAL, "NULL argument");
  long nc;
  size_t n_luh, n_face;
  grid_sizes(&g->cfg, &nc, &n_luh, &n_face);
  cudaError_t e = cudaMemcpyAsync(g->luh, host_luh, n_luh * sizeof(double), cudaMemcpyHostToDevice, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  g->primed = false;
  if (e == cudaSuccess && g->lim_on)
    if (exa_status_t s = grid_limiter_reset(g)) return s;
  return cuda_status(e, "grid set_state");
}

exa_status_t exa_aderdg_grid_get_state(exa_aderdg_grid* g, double* host_luh) {
  if (!g || !host_luh) return set_error(EXA_EINVAL, "NULL argument");
  long nc;
  size_t n_luh, n_face;
  grid_sizes(&g->cfg, &nc, &n_luh, &n_face);
  cudaError_t e = cudaMemcpyAsync(host_luh, g->luh, n_luh * sizeof(double), cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  return cuda_status(e, "grid get_state");
}

exa_status_t exa_aderdg_grid_use_graph(exa_aderdg_grid* g, int enable) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  g->use_graph = enable != 0;
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_set_debug(exa_aderdg_grid* g, int enable) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (g->graph) {  // the captured step has no scans (or has them)
    cudaGraphExecDestroy(g->graph);
    g->graph = nullptr;
  }
  g->debug = enable != 0;
  // a fresh record
  k_debug_reset<<<1, 1, 0, g->st>>>(g->gd);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_debug_reset");
}

exa_status_t exa_aderdg_grid_debug_status(exa_aderdg_grid* g, int* where, uint64_t* step, uint64_t* index) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  GridDev h{};
  cudaError_t e = cudaMemcpyAsync(&h, g->gd, sizeof(GridDev), cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  if (e != cudaSuccess) return cuda_status(e, "grid debug status");
  if (where) *where = h.nan_where;
  if (step) *step = h.nan_where ? h.nan_step : 0;
  if (index) *index = h.nan_where ? h.nan_index : 0;
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_profile(exa_aderdg_grid* g, int enable) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (enable && !g->ev[0])
    for (int i = 0; i < 3; i++) {
      cudaError_t e = cudaEventCreate(&g->ev[i]);
      if (e != cudaSuccess) return cuda_status(e, "profile events");
    }
  g->profile = enable != 0;
  if (g->profile) g->use_graph = false;
  g->ms_pred = g->ms_corr = 0;
  g->prof_steps = 0;
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_phase_times(exa_aderdg_grid* g, double* ms_predictor,
                                         double* ms_corrector, uint64_t* steps) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (ms_predictor) *ms_predictor = g->ms_pred;
  if (ms_corrector) *ms_corrector = g->ms_corr;
  if (steps) *steps = g->prof_steps;
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_stream(exa_aderdg_grid* g, void** stream) {
  if (!g || !stream) return set_error(EXA_EINVAL, "NULL argument");
  *stream = g->st;
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_device_state(exa_aderdg_grid* g, double** luh_dev) {
  if (!g || !luh_dev) return set_error(EXA_EINVAL, "NULL argument");
  *luh_dev = g->luh;
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_step(exa_aderdg_grid* g, int nsteps, double* dt_host) {
  if (!g || nsteps < 0) return set_error(EXA_EINVAL, "bad argument");
  if (g->halo)
    return set_error(EXA_EINVAL, "a grid with slab halos advances through exa_aderdg_grid_phase");
  if (dt_host && nsteps > g->log_cap) return set_error(EXA_EINVAL, "too many steps for the dt log");
  if (!g->primed)
    if (exa_status_t s = grid_prime(g)) return s;
  unsigned long long step0 = 0;
  if (dt_host) {
    cudaError_t e = cudaMemcpyAsync(&step0, &g->gd->step, 8, cudaMemcpyDeviceToHost, g->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
    if (e != cudaSuccess) return cuda_status(e, "read step");
  }
  if (g->use_graph && !g->graph && nsteps > 0) {
    cudaGraph_t graph;
    cudaError_t e = cudaStreamBeginCapture(g->st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_status(e, "begin capture");
    const uint64_t l0 = exa_launch_count();
    exa_status_t s = grid_launch_step(g);
    g->graph_launches = exa_launch_count() - l0;
    e = cudaStreamEndCapture(g->st, &graph);
    if (s) return s;
    if (e != cudaSuccess) return cuda_status(e, "end capture");
    e = cudaGraphInstantiate(&g->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_status(e, "graph instantiate");
  }
  for (int i = 0; i < nsteps; i++) {
    if (g->use_graph) {
      cudaError_t e = cudaGraphLaunch(g->graph, g->st);
      if (e != cudaSuccess) return cuda_status(e, "graph launch");
      count_launch(g->graph_launches);
    } else if (exa_status_t s = grid_launch_step(g)) {
      return s;
    }
  }
  if (dt_host && nsteps > 0) {
    // copy the dt log entries of these steps (ring buffer)
    for (int i = 0; i < nsteps; i++) {
      const unsigned long long k = (step0 + i) % (unsigned long long)g->log_cap;
      cudaError_t e = cudaMemcpyAsync(dt_host + i, g->dt_log + k, sizeof(double), cudaMemcpyDeviceToHost, g->st);
      if (e != cudaSuccess) return cuda_status(e, "read dt log");
    }
    cudaError_t e = cudaStreamSynchronize(g->st);
    if (e != cudaSuccess) return cuda_status(e, "step sync");
  }
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_status(exa_aderdg_grid* g, double* time, uint64_t* picard_iters_sum,
                                    uint64_t* nonconverged, int* nan_flag) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  GridDev h;
  cudaError_t e = cudaMemcpyAsync(&h, g->gd, sizeof(GridDev), cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  if (e != cudaSuccess) return cuda_status(e, "grid status");
  if (time) *time = h.time;
  if (picard_iters_sum) *picard_iters_sum = h.stats[0];
  if (nonconverged) *nonconverged = h.stats[1];
  if (nan_flag) *nan_flag = h.nan_flag;
  if (h.nan_flag) return EXA_ENAN;
  if (h.stats[1]) return EXA_ENONCONV;
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_init_slab(exa_aderdg_grid* g, int kind, double param, uint64_t seed,
                                       double noise_amp, int rank, int nranks) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (kind < 0 || kind > 1) return set_error(EXA_EINVAL, "unknown initial condition");
  if (nranks < 1 || rank < 0 || rank >= nranks) return set_error(EXA_EINVAL, "bad slab rank");
  const int last = g->cfg.n[g->cfg.dim - 1];
  if (exa_status_t s = launch_grid_ic(g->cfg.dim, g->cfg.order, g->cfg.n, g->desc.dx, g->luh, kind,
                                      param, seed, noise_amp, g->st, (long)rank * g->ncells,
                                      last * nranks))
    return s;
  g->primed = false;
  return cuda_status(cudaStreamSynchronize(g->st), "grid init");
}

exa_status_t exa_aderdg_grid_set_boundary(exa_aderdg_grid* g, const int* bc) {
  if (!g || !bc) return set_error(EXA_EINVAL, "NULL argument");
  for (int i = 0; i < g->cfg.dim; i++)
    if (bc[i] < EXA_BC_PERIODIC || bc[i] > EXA_BC_REFLECT) return set_error(EXA_EINVAL, "unknown boundary rule");
  if (g->halo && bc[g->cfg.dim - 1] != EXA_BC_PERIODIC)
    return set_error(EXA_EINVAL, "slab halos need a periodic last dimension");
  for (int i = 0; i < 3; i++) g->bc[i] = i < g->cfg.dim ? bc[i] : 0;
  if (g->graph) {  // the captured step holds the old arguments
    cudaGraphExecDestroy(g->graph);
    g->graph = nullptr;
  }
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_set_adjustment(exa_aderdg_grid* g, const exa_adjust_t* hook) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (hook)
    if (exa_status_t s = check_adjust_hook(hook)) return s;
  const bool on = hook && hook->kind != EXA_ADJUST_NONE && hook->when == EXA_ADJUST_ALWAYS;
  if (on && g->lim_on) return set_error(EXA_EINVAL, "adjustment: not with the limiter");
  if (on && g->halo) return set_error(EXA_EINVAL, "adjustment: not with slab halos");
  if (g->graph) {  // the captured step changes
    cudaGraphExecDestroy(g->graph);
    g->graph = nullptr;
  }
  g->adj_on = on;
  g->adj = on ? *hook : exa_adjust_t{};
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_set_limiter(exa_aderdg_grid* g, const exa_limiter_config_t* cfg) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (g->graph) {  // the captured step changes
    cudaGraphExecDestroy(g->graph);
    g->graph = nullptr;
  }
  if (!cfg) {
    cudaStreamSynchronize(g->st);
    cudaFree(g->lim_block);
    g->lim_block = nullptr;
    g->lim_on = false;
    return EXA_OK;
  }
  if (g->halo) return set_error(EXA_EINVAL, "limiter: not with slab halos");
  if (g->adj_on) return set_error(EXA_EINVAL, "limiter: not with a solution adjustment");
  if (g->cfg.dim == 3) {
    // one CTA stages a subcell patch with its ghosts (fv3d.cu)
    const int S = 2 * g->cfg.order + 1, gw = cfg->scheme == 0 ? 1 : 2;
    if (fv3_smem(S, gw, cfg->scheme) > 200 * 1024)
      return set_error(EXA_EINVAL, "limiter: 3D subcell patch too large (MUSCL-Hancock needs order <= 5)");
  }
  if (cfg->scheme != 0 && cfg->scheme != 1) return set_error(EXA_EINVAL, "limiter: scheme must be 0 or 1");
  if (cfg->nobs < 1 || cfg->nobs > kV) return set_error(EXA_EINVAL, "limiter: nobs must be in 1..5");
  if (!(cfg->relaxation >= 0) || !(cfg->difference_scaling >= 0))
    return set_error(EXA_EINVAL, "limiter: DMP parameters must not be negative");
  if (cfg->steps_till_cured < 0) return set_error(EXA_EINVAL, "limiter: steps_till_cured must not be negative");
  cudaStreamSynchronize(g->st);
  cudaFree(g->lim_block);
  g->lim_block = nullptr;
  g->lim_on = false;
  g->lim_cfg = *cfg;
  g->lim_ghost = cfg->scheme == 0 ? 1 : 2;
  const long n = g->ncells;
  const int B = g->cfg.order + 1, SG = 2 * g->cfg.order + 1 + 2 * g->lim_ghost;
  const size_t npc = g->cfg.dim == 3 ? (size_t)B * B * B : (size_t)B * B;
  const size_t spc = g->cfg.dim == 3 ? (size_t)SG * SG * SG : (size_t)SG * SG;
  const size_t d_prev = (size_t)n * npc * kV, d_patch = (size_t)n * spc * kV;
  const size_t d_b = (size_t)n * 2 * g->cfg.dim * cfg->nobs, d_loc = (size_t)n * 2 * cfg->nobs;
  const size_t doubles = d_prev + d_patch + 2 * d_b + d_loc;
  const size_t ints = 6 * (size_t)n + 4;
  cudaError_t e = cudaMalloc(&g->lim_block, doubles * sizeof(double) + ints * sizeof(int));
  if (e != cudaSuccess) return cuda_status(e, "limiter allocation");
  double* p = static_cast<double*>(g->lim_block);
  g->lim_prev = p;
  p += d_prev;
  g->lim_patch = p;
  p += d_patch;
  g->lim_bmin = p;
  p += d_b;
  g->lim_bmax = p;
  p += d_b;
  g->lim_loc = p;
  p += d_loc;
  int* q = reinterpret_cast<int*>(p);
  g->lim_ok = q;
  g->lim_status = q + n;
  g->lim_status_tmp = q + 2 * n;
  g->lim_cure = q + 3 * n;
  g->lim_list_patch = q + 4 * n;
  g->lim_list_fv = q + 5 * n;
  g->lim_counts = q + 6 * n;
  e = cudaMemsetAsync(g->lim_patch, 0, d_patch * sizeof(double), g->st);
  if (e != cudaSuccess) return cuda_status(e, "limiter allocation");
  g->lim_on = true;
  return grid_limiter_reset(g);
}

exa_status_t exa_aderdg_grid_limiter_status(exa_aderdg_grid* g, int* host_status, int* counts) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (!g->lim_on) return set_error(EXA_EINVAL, "limiter not enabled");
  cudaError_t e = cudaSuccess;
  if (host_status)
    e = cudaMemcpyAsync(host_status, g->lim_status, g->ncells * sizeof(int), cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess && counts) e = cudaMemcpyAsync(counts, g->lim_counts, 3 * sizeof(int), cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  return cuda_status(e, "limiter status");
}

exa_status_t exa_aderdg_grid_limiter_bounds(exa_aderdg_grid* g, double* host_min, double* host_max) {
  if (!g || !host_min || !host_max) return set_error(EXA_EINVAL, "NULL argument");
  if (!g->lim_on) return set_error(EXA_EINVAL, "limiter not enabled");
  const size_t bytes = (size_t)g->ncells * 2 * g->cfg.dim * g->lim_cfg.nobs * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(host_min, g->lim_bmin, bytes, cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(host_max, g->lim_bmax, bytes, cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  return cuda_status(e, "limiter bounds");
}

exa_status_t exa_aderdg_grid_set_halo(exa_aderdg_grid* g, int enable) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (enable && g->bc[g->cfg.dim - 1] != EXA_BC_PERIODIC)
    return set_error(EXA_EINVAL, "slab halos need a periodic last dimension");
  if (enable && g->adj_on) return set_error(EXA_EINVAL, "slab halos: not with a solution adjustment");
  if (g->graph) {
    cudaGraphExecDestroy(g->graph);
    g->graph = nullptr;
  }
  if (!enable) {
    cudaStreamSynchronize(g->st);
    cudaFree(g->halo);
    g->halo = nullptr;
    g->halo_count = 0;
    return EXA_OK;
  }
  if (g->halo) return EXA_OK;
  const int B = g->cfg.order + 1;
  const size_t nfv = (size_t)(g->cfg.dim == 3 ? B * B : B) * kV;
  g->layer = g->ncells / g->cfg.n[g->cfg.dim - 1];
  g->halo_count = (size_t)g->layer * 2 * nfv;
  cudaError_t e = cudaMalloc(&g->halo, 4 * g->halo_count * sizeof(double));
  if (e == cudaSuccess) e = cudaMemsetAsync(g->halo, 0, 4 * g->halo_count * sizeof(double), g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  if (e != cudaSuccess) {
    cudaFree(g->halo);
    g->halo = nullptr;
    g->halo_count = 0;
    return cuda_status(e, "halo buffers");
  }
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_halo_buffers(exa_aderdg_grid* g, double** send_lo, double** send_hi,
                                          double** recv_lo, double** recv_hi, size_t* count) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (!g->halo) return set_error(EXA_EINVAL, "grid has no slab halos");
  if (send_lo) *send_lo = g->halo;
  if (send_hi) *send_hi = g->halo + g->halo_count;
  if (recv_lo) *recv_lo = g->halo + 2 * g->halo_count;
  if (recv_hi) *recv_hi = g->halo + 3 * g->halo_count;
  if (count) *count = g->halo_count;
  return EXA_OK;
}

exa_status_t exa_aderdg_grid_dt_slot(exa_aderdg_grid* g, uint64_t** slot) {
  if (!g || !slot) return set_error(EXA_EINVAL, "NULL argument");
  *slot = (uint64_t*)&g->gd->dt_next;
  return EXA_OK;
}

}  // extern "C"

namespace exa {
bool grid_fixed_dt(const exa_aderdg_grid* g) { return g->cfg.dt_policy == 2; }
}  // namespace exa

extern "C" {

exa_status_t exa_aderdg_grid_phase(exa_aderdg_grid* g, int phase) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  switch (phase) {
    case EXA_PHASE_PRIME_LOCAL: {
      if (g->cfg.dt_policy == 2) return set_error(EXA_EINVAL, "fixed dt needs no priming");
      const unsigned long long inf = 0x7FF0000000000000ULL;
      cudaError_t e = cudaMemcpyAsync(&g->gd->dt_next, &inf, 8, cudaMemcpyHostToDevice, g->st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
      if (e != cudaSuccess) return cuda_status(e, "prime dt slot");
      return launch_stable_dt(g->desc, g->ncells, g->luh, g->dt_factor, nullptr, &g->gd->dt_next, g->st);
    }
    case EXA_PHASE_PRIME_COMMIT:
      if (g->cfg.dt_policy == 2) return grid_prime(g);
      k_prime<<<1, 1, 0, g->st>>>(g->gd);
      count_launch();
      if (exa_status_t s = cuda_status(cudaGetLastError(), "k_prime")) return s;
      g->primed = true;
      return EXA_OK;
    case EXA_PHASE_PREDICT: {
      if (!g->primed) return set_error(EXA_EINVAL, "grid dt not primed");
      if (g->profile) cudaEventRecord(g->ev[0], g->st);
      exa_status_t s = grid_predict(g);
      if (g->profile) cudaEventRecord(g->ev[1], g->st);
      return s;
    }
    case EXA_PHASE_CORRECT:
      if (!g->primed) return set_error(EXA_EINVAL, "grid dt not primed");
      return grid_correct(g);
    case EXA_PHASE_COMMIT: {
      if (!g->primed) return set_error(EXA_EINVAL, "grid dt not primed");
      if (exa_status_t s = grid_commit(g)) return s;
      if (g->profile) {
        // predictor, then everything after it (exchange wait, corrector, commit)
        cudaEventRecord(g->ev[2], g->st);
        cudaError_t e = cudaEventSynchronize(g->ev[2]);
        if (e != cudaSuccess) return cuda_status(e, "profile sync");
        float a1 = 0, a2 = 0;
        cudaEventElapsedTime(&a1, g->ev[0], g->ev[1]);
        cudaEventElapsedTime(&a2, g->ev[1], g->ev[2]);
        g->ms_pred += a1;
        g->ms_corr += a2;
        g->prof_steps++;
      }
      return EXA_OK;
    }
  }
  return set_error(EXA_EINVAL, "unknown phase");
}

}  // extern "C"
