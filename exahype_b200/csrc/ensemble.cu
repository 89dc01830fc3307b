// Ensemble of independent 2D ADER-DG solves stepped by one persistent
// launch per step.
//
// Each solve is a uniform periodic 2D grid with its own order (2..5), size,
// time-step size and step budget (the per-solve state the reference keeps in
// its solver object, ADERDGSolver.cpp:557-585).  One cooperative kernel per
// step runs, for every active solve:
//   phase 1  predictor + volume integral on every cell block   (work items)
//   phase 2  Riemann + surface integral + update + next dt      (work items)
//   phase 3  per-solve commit: time, dt <- next dt, step budget
// separated by grid-wide barriers.  CTAs pull work items (one block of
// cells of one solve) from an atomic counter, so solves of different order
// and size share the machine without per-solve launches; the step is a
// single graph node once captured.  Device memory for all solves comes from
// one arena allocated at creation (admission by footprint, no allocation on
// the step path).
#include <cooperative_groups.h>

#include <algorithm>
#include <mutex>
#include <new>
#include <vector>
#include <float.h>

#include "exa_device.cuh"
#include "aderdg_predictor_body.cuh"
#include "aderdg_predictor_mixed_body.cuh"
#include "aderdg_predictor_lines_body.cuh"
#include "aderdg_predictor_fp64_lines_body.cuh"
#include "aderdg_predictor_fp64_prog_body.cuh"
#include "aderdg_predictor_mixed_prog_body.cuh"
#include "aderdg_corrector_body.cuh"

namespace cg = cooperative_groups;

namespace exa {
double host_pnpm(int order);

struct SolveDev {
  int order, pde, dt_policy, active;  // active: 1 while steps remain
  int n[2];
  double dx[2];
  long ncells;
  double* luh;
  double* lduh;
  double* qb;
  double* fb;
  double dt_factor, dt_fixed;
  // time-step state
  double dt;
  unsigned long long dt_next;
  double time;
  unsigned long long steps_done;
  long long steps_left;  // < 0: unlimited
  unsigned long long stats[2];
  int nan_flag;
  int pad;
};

struct WorkItem {
  int solve;
  int block;
};

struct EnsArgs {
  SolveDev* solves;
  int nsolves;
  const WorkItem* items;
  int nitems;
  int grab;            // work items taken per atomic
  unsigned int* ctr;   // [2] phase counters, reset by phase 3
  int precision;
  int lines_mask;      // bit N set: order N's predictor uses the line-owner contraction
};

constexpr int kEnsNT = 128;

constexpr int cmax(int a, int b) { return a > b ? a : b; }
// default: orders whose predictor runs the line-owner contraction (as the
// stand-alone kernels do by default: measured faster from order 4 on); the
// autotuner may choose per order (exa_ensemble_tune_contraction)
constexpr int kEnsLinesDefault = (1 << 4) | (1 << 5);
// shared memory (doubles) the largest 2D order needs in either phase and
// either contraction
template <int N>
constexpr int ens_smem_n() {
  return cmax(cmax(cmax(Fp64LineShape<2, N>::SM_DOUBLES, PredShape<2, N, 0>::SM_DOUBLES),
                   cmax(LineShape<2, N>::SM_DOUBLES, MixShape<2, N>::SM_DOUBLES)),
              CorrShapeSmem<2, N>::value);
}
constexpr int kEnsSmemDoubles = cmax(cmax(ens_smem_n<2>(), ens_smem_n<3>()), cmax(ens_smem_n<4>(), ens_smem_n<5>()));

__device__ __forceinline__ PredArgs pred_args(const SolveDev& sv, int precision) {
  PredArgs a{};
  a.ncells = sv.ncells;
  a.luh = sv.luh;
  a.dt = 0.0;
  a.dt_dev = &sv.dt;
  a.idx[0] = 1.0 / sv.dx[0];
  a.idx[1] = 1.0 / sv.dx[1];
  a.idx[2] = 0.0;
  a.lduh = sv.lduh;
  a.lQhbnd = sv.qb;
  a.lFhbnd = sv.fb;
  a.iters = nullptr;
  a.stats = const_cast<unsigned long long*>(sv.stats);
  a.precision = precision;
  return a;
}

__device__ __forceinline__ CorrArgs corr_args(SolveDev& sv) {
  CorrArgs c{};
  c.ncells = sv.ncells;
  c.n[0] = sv.n[0];
  c.n[1] = sv.n[1];
  c.n[2] = 1;
  c.dx[0] = sv.dx[0];
  c.dx[1] = sv.dx[1];
  c.dx[2] = 1.0;
  c.dt_dev = &sv.dt;
  c.luh = sv.luh;
  c.lduh = sv.lduh;
  c.lQhbnd = sv.qb;
  c.lFhbnd = sv.fb;
  c.dt_next = sv.dt_policy == 2 ? nullptr : &sv.dt_next;
  c.dt_factor = sv.dt_factor;
  c.nan_flag = &sv.nan_flag;
  return c;
}

// One non-inlined function per (phase, order, precision, pde form): each
// keeps the register allocation of the stand-alone kernel instead of
// sharing one allocation across every path of the persistent kernel.
template <int N, bool PLANAR, int PREC, bool LINES>
__device__ __noinline__ void ens_pred(const SolveDev* sv, int block, double* smem, int precision) {
  const PredArgs a = pred_args(*sv, precision);
  if constexpr (LINES) {
    // (compile-time branches: each instantiation holds only its own body)
    // mixed order 5: the progressive form (128 registers instead of 168,
    // four CTAs per SM: 10.0 -> 9.2 ms per step of 24 order-5 solves); at
    // order 4 the two measured the same and the line-owner form stays
    if constexpr (PREC != 0) {
      if constexpr (N == 5) predictor_mixed_prog_block<2, N, PLANAR>(a, block, smem);
      else predictor_mixed_lines_block<2, N, PLANAR>(a, block, smem);
    }
    // FP64 order 4: the progressive form (three CTAs per SM in the
    // per-order launch, 7 % faster); order 5 keeps the line-owner form,
    // which its registers suit better (measured 10.9 ms per step of a
    // 512k-cell ensemble against 11.3 ms progressive)
    else if constexpr (N == 4) predictor_fp64_prog_block<2, N, PLANAR>(a, block, smem);
    else predictor_fp64_lines_block<2, N, PLANAR>(a, block, smem);
  } else {
    if (PREC) predictor_mixed_block<2, N, PLANAR>(a, block, smem);
    else predictor_block<2, N, 0, PLANAR, 0>(a, block, smem);
  }
}

template <int N, bool PLANAR>
__device__ __noinline__ void ens_corr(SolveDev* sv, int block, double* smem) {
  const CorrArgs c = corr_args(*sv);
  corrector_block<2, N, PLANAR>(c, block, smem);
}

template <int N, int PREC>
__device__ __forceinline__ void run_pred_n(const SolveDev& sv, int block, double* smem, int precision, bool lines) {
  const bool planar = sv.pde == EXA_PDE_EULER_PLANAR;
  if (lines) {
    if (planar) ens_pred<N, true, PREC, true>(&sv, block, smem, precision);
    else ens_pred<N, false, PREC, true>(&sv, block, smem, precision);
  } else {
    if (planar) ens_pred<N, true, PREC, false>(&sv, block, smem, precision);
    else ens_pred<N, false, PREC, false>(&sv, block, smem, precision);
  }
}

template <int PREC>
__device__ __forceinline__ void run_pred(const SolveDev& sv, int block, double* smem, int precision,
                                         int lines_mask) {
  const bool lines = (lines_mask >> sv.order) & 1;
  switch (sv.order) {
    case 2: run_pred_n<2, PREC>(sv, block, smem, precision, lines); break;
    case 3: run_pred_n<3, PREC>(sv, block, smem, precision, lines); break;
    case 4: run_pred_n<4, PREC>(sv, block, smem, precision, lines); break;
    case 5: run_pred_n<5, PREC>(sv, block, smem, precision, lines); break;
  }
}

__device__ __forceinline__ void run_corr(SolveDev& sv, int block, double* smem) {
  const bool planar = sv.pde == EXA_PDE_EULER_PLANAR;
  switch (sv.order) {
    case 2: planar ? ens_corr<2, true>(&sv, block, smem) : ens_corr<2, false>(&sv, block, smem); break;
    case 3: planar ? ens_corr<3, true>(&sv, block, smem) : ens_corr<3, false>(&sv, block, smem); break;
    case 4: planar ? ens_corr<4, true>(&sv, block, smem) : ens_corr<4, false>(&sv, block, smem); break;
    case 5: planar ? ens_corr<5, true>(&sv, block, smem) : ens_corr<5, false>(&sv, block, smem); break;
  }
}

// end of a step for one solve: time, step count, next dt, step budget
__device__ __forceinline__ void ens_commit(SolveDev& sv) {
  if (!sv.active) return;
  if (sv.nan_flag) {
    // this step produced a non-finite state: the solve stops here (not
    // counted as a step) and is reported failed; the others go on
    sv.active = 0;
    return;
  }
  sv.time += sv.dt;
  sv.steps_done += 1;
  if (sv.dt_policy == 2) {
    sv.dt = sv.dt_fixed;
  } else {
    sv.dt = __longlong_as_double((long long)sv.dt_next);
    sv.dt_next = 0x7FF0000000000000ULL;
  }
  if (sv.steps_left > 0) {
    sv.steps_left -= 1;
    if (sv.steps_left == 0) sv.active = 0;
  }
}

// Per-order launch mode: one CTA per work item of one order (the items of
// an order are contiguous from `first`), each launch with that order's own
// shared memory and occupancy; then a commit launch over the solves.
// CTA blockIdx.x of an order's launch -> (solve, block of that solve): the
// order's segments a.items[first .. first + nseg) hold each solve's first
// block in the order's block numbering (ascending)
__device__ __forceinline__ WorkItem ens_segment_item(const EnsArgs& a, int first, int nseg) {
  const int b = blockIdx.x;
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.items[first + mid].block <= b) lo = mid;
    else hi = mid - 1;
  }
  const WorkItem seg = a.items[first + lo];
  return WorkItem{seg.solve, b - seg.block};
}

// order 4 in FP64 with the line-owner contraction (the progressive form)
// is bounded to three CTAs per SM; 0 leaves the others unconstrained
template <int N, int PREC, bool LINES>
constexpr int ens_pred_minb() { return (N == 4 && PREC == 0 && LINES) ? 3 : 0; }

template <int N, int PREC, bool LINES>
__global__ void __launch_bounds__(kEnsNT, ens_pred_minb<N, PREC, LINES>()) k_ens_pred_order(EnsArgs a, int first, int nseg) {
  extern __shared__ double smem[];
  const WorkItem it = ens_segment_item(a, first, nseg);
  const SolveDev& sv = a.solves[it.solve];
  if (!sv.active) return;  // uniform across the CTA
  if (sv.pde == EXA_PDE_EULER_PLANAR) ens_pred<N, true, PREC, LINES>(&sv, it.block, smem, a.precision);
  else ens_pred<N, false, PREC, LINES>(&sv, it.block, smem, a.precision);
}

template <int N>
__global__ void __launch_bounds__(kEnsNT) k_ens_corr_order(EnsArgs a, int first, int nseg) {
  extern __shared__ double smem[];
  const WorkItem it = ens_segment_item(a, first, nseg);
  SolveDev& sv = a.solves[it.solve];
  if (!sv.active) return;
  if (sv.pde == EXA_PDE_EULER_PLANAR) ens_corr<N, true>(&sv, it.block, smem);
  else ens_corr<N, false>(&sv, it.block, smem);
}

__global__ void k_ens_commit(EnsArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < a.nsolves) ens_commit(a.solves[s]);
}

template <int N, int PREC, bool LINES>
constexpr int ens_pred_smem() {
  return LINES ? (PREC ? (N == 5 ? MixProgShape<2, N>::SM_DOUBLES : LineShape<2, N>::SM_DOUBLES)
                        : (N == 4 ? Fp64ProgShape<2, N>::SM_DOUBLES : Fp64LineShape<2, N>::SM_DOUBLES))
               : (PREC ? MixShape<2, N>::SM_DOUBLES : PredShape<2, N, 0>::SM_DOUBLES);
}

template <int PREC>
__global__ void __launch_bounds__(kEnsNT) k_ensemble_step(EnsArgs a) {
  cg::grid_group grid = cg::this_grid();
  extern __shared__ double smem[];
  __shared__ int s_item;
  for (int phase = 0; phase < 2; phase++) {
    for (;;) {
      if (threadIdx.x == 0) s_item = (int)atomicAdd(&a.ctr[phase], (unsigned)a.grab);
      __syncthreads();
      const int w0 = s_item;
      __syncthreads();
      if (w0 >= a.nitems) break;
      const int w1 = min(w0 + a.grab, a.nitems);
      for (int w = w0; w < w1; w++) {
        const WorkItem it = a.items[w];
        SolveDev& sv = a.solves[it.solve];
        if (!sv.active) continue;  // uniform across the CTA
        if (phase == 0) run_pred<PREC>(sv, it.block, smem, a.precision, a.lines_mask);
        else run_corr(sv, it.block, smem);
        __syncthreads();  // smem reuse by the next item
      }
    }
    grid.sync();
  }
  // phase 3: commit every active solve
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  for (int s = gtid; s < a.nsolves; s += gridDim.x * blockDim.x) ens_commit(a.solves[s]);
  if (gtid == 0) {
    a.ctr[0] = 0;
    a.ctr[1] = 0;
  }
}

// first dt of a newly added solve: the reduced value (or the fixed dt)
__global__ void k_solve_prime(SolveDev* sv) {
  sv->dt = sv->dt_policy == 2 ? sv->dt_fixed : __longlong_as_double((long long)sv->dt_next);
  sv->dt_next = 0x7FF0000000000000ULL;
}

exa_status_t upload_tables_ensemble() {
  size_t bytes = 0;
  const void* h = host_dg_tables(&bytes);
  cudaError_t e = cudaMemcpyToSymbol(c_dg, h, bytes);
  if (e == cudaSuccess) {
    const void* hf = host_dg_tables_f(&bytes);
    e = cudaMemcpyToSymbol(c_dgf, hf, bytes);
  }
  return cuda_status(e, "upload tables (ensemble)");
}

}  // namespace exa

using namespace exa;

// ------------------------------------------------------------------ host
struct ArenaBlock {
  size_t off, size;
};

struct exa_ensemble {
  int device = 0;
  int precision = 0;
  int max_solves = 0;
  cudaStream_t st = nullptr;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  std::vector<ArenaBlock> free_list;  // sorted by offset
  std::vector<SolveDev> host;         // mirror of the device descriptors
  std::vector<size_t> alloc_off, alloc_size;
  std::vector<char> used;
  SolveDev* d_solves = nullptr;
  WorkItem* d_items = nullptr;
  int items_cap = 0, nitems = 0;
  unsigned int* d_ctr = nullptr;
  bool dirty = true;  // solve set changed: rebuild items, re-capture
  bool use_graph = false;
  cudaGraphExec_t graph = nullptr;
  // tuning (exa_ensemble_tune): CTAs per SM, items per grab, order policy
  int ctas_per_sm = 0, grab = 1, order_policy = 0;
  int lines_mask = kEnsLinesDefault;  // per order: line-owner (bit set) or node-gather contraction
  // launch mode (exa_ensemble_set_launch_mode): 0 one persistent cooperative
  // launch per step; 1 per-order launches (items of an order contiguous)
  int mode = 0;
  // per-order launches: the orders' predictor + corrector pairs run on one
  // stream each (forked from st, joined before the commit), so one order's
  // launch tail overlaps the others' work
  cudaStream_t ost[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t fork_ev = nullptr;
  cudaEvent_t join_ev[4] = {nullptr, nullptr, nullptr, nullptr};
  int order_first[6] = {0, 0, 0, 0, 0, 0}, order_count[6] = {0, 0, 0, 0, 0, 0};  // segments per order
  long order_blocks[6] = {0, 0, 0, 0, 0, 0};  // blocks of cells per order (per-order launches)
  bool order_attrs = false;
  int grid = 0;
  std::mutex mu;
};

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

static exa_status_t solve_sizes(const exa_solve_config_t* c, long* ncells, size_t* n_luh, size_t* n_face) {
  if (!c) return set_error(EXA_EINVAL, "NULL solve config");
  if (c->order < 2 || c->order > 5) return set_error(EXA_EINVAL, "order must be in 2..5");
  if (c->n[0] < 1 || c->n[1] < 1 || !(c->length[0] > 0) || !(c->length[1] > 0))
    return set_error(EXA_EINVAL, "bad grid size");
  if (c->pde != EXA_PDE_EULER && c->pde != EXA_PDE_EULER_PLANAR) return set_error(EXA_EINVAL, "pde");
  if (c->dt_policy < 0 || c->dt_policy > 2 || (c->dt_policy == 2 && !(c->dt_fixed > 0)) || !(c->cfl > 0))
    return set_error(EXA_EINVAL, "bad dt policy");
  if (c->ic_kind < 0 || c->ic_kind > 1) return set_error(EXA_EINVAL, "unknown initial condition");
  const int B = c->order + 1;
  *ncells = (long)c->n[0] * c->n[1];
  *n_luh = (size_t)*ncells * B * B * kV;
  *n_face = (size_t)*ncells * 4 * B * kV;
  return EXA_OK;
}

static size_t solve_footprint(long, size_t n_luh, size_t n_face) {
  return align256(n_luh * 8) * 2 + align256(n_face * 8) * 2;
}

static bool arena_alloc(exa_ensemble* e, size_t bytes, size_t* off) {
  for (size_t i = 0; i < e->free_list.size(); i++) {
    ArenaBlock& b = e->free_list[i];
    if (b.size >= bytes) {
      *off = b.off;
      b.off += bytes;
      b.size -= bytes;
      if (b.size == 0) e->free_list.erase(e->free_list.begin() + i);
      return true;
    }
  }
  return false;
}

static void arena_free(exa_ensemble* e, size_t off, size_t bytes) {
  ArenaBlock nb{off, bytes};
  auto it = std::lower_bound(e->free_list.begin(), e->free_list.end(), nb,
                             [](const ArenaBlock& a, const ArenaBlock& b) { return a.off < b.off; });
  it = e->free_list.insert(it, nb);
  // coalesce with neighbours
  size_t i = it - e->free_list.begin();
  if (i + 1 < e->free_list.size() && e->free_list[i].off + e->free_list[i].size == e->free_list[i + 1].off) {
    e->free_list[i].size += e->free_list[i + 1].size;
    e->free_list.erase(e->free_list.begin() + i + 1);
  }
  if (i > 0 && e->free_list[i - 1].off + e->free_list[i - 1].size == e->free_list[i].off) {
    e->free_list[i - 1].size += e->free_list[i].size;
    e->free_list.erase(e->free_list.begin() + i);
  }
}

static int cells_per_block(int order) {
  const int B = order + 1, npc = B * B;
  int g = 1;
  if (npc <= 32) {
    while (g < npc) g <<= 1;
  } else {
    g = (npc + 31) / 32 * 32;
  }
  return kEnsNT / g > 0 ? kEnsNT / g : 1;
}

static exa_status_t upload_items(exa_ensemble* e, const std::vector<WorkItem>& items) {
  if ((int)items.size() > e->items_cap) {
    if (e->d_items) cudaFree(e->d_items);
    e->d_items = nullptr;
    e->items_cap = std::max<int>((int)items.size(), 1024);
    cudaError_t err = cudaMalloc(&e->d_items, sizeof(WorkItem) * e->items_cap);
    if (err != cudaSuccess) {
      e->items_cap = 0;
      return cuda_status(err, "ensemble work items");
    }
  }
  e->nitems = (int)items.size();
  if (e->nitems) {
    // stream-ordered after the launches that read the previous list; a copy
    // from pageable memory is staged before the call returns
    cudaError_t err = cudaMemcpyAsync(e->d_items, items.data(), sizeof(WorkItem) * e->nitems,
                                      cudaMemcpyHostToDevice, e->st);
    if (err != cudaSuccess) return cuda_status(err, "upload work items");
  }
  return EXA_OK;
}

static exa_status_t rebuild_items(exa_ensemble* e) {
  std::vector<WorkItem> items;
  for (int n = 0; n < 6; n++) e->order_first[n] = e->order_count[n] = e->order_blocks[n] = 0;
  if (e->mode == 1) {
    // per-order launches: per order, one segment per active solve holding
    // the order's running block count at its first block (block field);
    // CTA b of the order's launch finds its segment by binary search.  Work
    // on the host is per solve, not per block.
    std::vector<WorkItem> per[6];
    for (int s = 0; s < e->max_solves; s++) {
      if (!e->used[s] || !e->host[s].active) continue;
      const int n = e->host[s].order;
      const long nb = (e->host[s].ncells + cells_per_block(n) - 1) / cells_per_block(n);
      per[n].push_back(WorkItem{s, (int)e->order_blocks[n]});
      e->order_blocks[n] += nb;
    }
    for (int n = 5; n >= 2; n--) {
      e->order_first[n] = (int)items.size();
      e->order_count[n] = (int)per[n].size();
      items.insert(items.end(), per[n].begin(), per[n].end());
    }
  } else {
    // persistent launch: one work item per block of cells of each active
    // solve; costly orders first (longest-processing-time order) unless the
    // policy interleaves
    for (int s = 0; s < e->max_solves; s++) {
      if (!e->used[s] || !e->host[s].active) continue;
      const long nb = (e->host[s].ncells + cells_per_block(e->host[s].order) - 1) / cells_per_block(e->host[s].order);
      for (long b = 0; b < nb; b++) items.push_back(WorkItem{s, (int)b});
    }
    if (e->order_policy == 0) {
      std::stable_sort(items.begin(), items.end(), [&](const WorkItem& a, const WorkItem& b) {
        return e->host[a.solve].order > e->host[b.solve].order;
      });
    }
  }
  if (exa_status_t st = upload_items(e, items)) return st;
  if (e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  e->dirty = false;
  return EXA_OK;
}

template <int N, int PREC>
static cudaError_t set_order_attrs() {
  cudaError_t e = cudaFuncSetAttribute(k_ens_pred_order<N, PREC, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(double) * ens_pred_smem<N, PREC, true>()));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_ens_pred_order<N, PREC, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(double) * ens_pred_smem<N, PREC, false>()));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_ens_corr_order<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(double) * CorrShapeSmem<2, N>::value));
  return e;
}

template <int N, int PREC>
static void launch_pred_order(const EnsArgs& a, const exa_ensemble* e, cudaStream_t st) {
  const long blocks = e->order_blocks[N];
  if (blocks == 0) return;
  if ((e->lines_mask >> N) & 1)
    k_ens_pred_order<N, PREC, true><<<(unsigned)blocks, kEnsNT, sizeof(double) * ens_pred_smem<N, PREC, true>(), st>>>(
        a, e->order_first[N], e->order_count[N]);
  else
    k_ens_pred_order<N, PREC, false><<<(unsigned)blocks, kEnsNT, sizeof(double) * ens_pred_smem<N, PREC, false>(),
                                       st>>>(a, e->order_first[N], e->order_count[N]);
  count_launch();
}

template <int N>
static void launch_corr_order(const EnsArgs& a, const exa_ensemble* e, cudaStream_t st) {
  const long blocks = e->order_blocks[N];
  if (blocks == 0) return;
  k_ens_corr_order<N><<<(unsigned)blocks, kEnsNT, sizeof(double) * CorrShapeSmem<2, N>::value, st>>>(
      a, e->order_first[N], e->order_count[N]);
  count_launch();
}

template <int PREC>
static exa_status_t launch_step_orders(exa_ensemble* e, const EnsArgs& a) {
  if (!e->order_attrs) {
    cudaError_t err = set_order_attrs<2, PREC>();
    if (err == cudaSuccess) err = set_order_attrs<3, PREC>();
    if (err == cudaSuccess) err = set_order_attrs<4, PREC>();
    if (err == cudaSuccess) err = set_order_attrs<5, PREC>();
    if (err != cudaSuccess) return cuda_status(err, "ensemble per-order attributes");
    e->order_attrs = true;
  }
  // one branch per order present (the solves of different orders share
  // nothing until the commit), costly orders issued first
  cudaError_t err = cudaEventRecord(e->fork_ev, e->st);
  for (int n = 5; n >= 2 && err == cudaSuccess; n--) {
    if (e->order_blocks[n] == 0) continue;
    cudaStream_t os = e->ost[n - 2];
    err = cudaStreamWaitEvent(os, e->fork_ev, 0);
    if (err != cudaSuccess) break;
    switch (n) {
      case 5: launch_pred_order<5, PREC>(a, e, os); launch_corr_order<5>(a, e, os); break;
      case 4: launch_pred_order<4, PREC>(a, e, os); launch_corr_order<4>(a, e, os); break;
      case 3: launch_pred_order<3, PREC>(a, e, os); launch_corr_order<3>(a, e, os); break;
      default: launch_pred_order<2, PREC>(a, e, os); launch_corr_order<2>(a, e, os); break;
    }
    err = cudaEventRecord(e->join_ev[n - 2], os);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(e->st, e->join_ev[n - 2], 0);
  }
  if (err != cudaSuccess) return cuda_status(err, "ensemble per-order branches");
  k_ens_commit<<<(a.nsolves + 127) / 128, 128, 0, e->st>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "ensemble per-order launches");
}

static exa_status_t launch_step(exa_ensemble* e) {
  EnsArgs a;
  a.solves = e->d_solves;
  a.nsolves = e->max_solves;
  a.items = e->d_items;
  a.nitems = e->nitems;
  a.grab = e->grab;
  a.ctr = e->d_ctr;
  a.precision = e->precision;
  a.lines_mask = e->lines_mask;
  if (e->mode == 1)
    return e->precision == EXA_PREC_MIXED ? launch_step_orders<1>(e, a) : launch_step_orders<0>(e, a);
  void* args[] = {&a};
  const size_t smem = sizeof(double) * kEnsSmemDoubles;
  cudaError_t err;
  if (e->precision == EXA_PREC_MIXED)
    err = cudaLaunchCooperativeKernel((void*)k_ensemble_step<1>, e->grid, kEnsNT, args, smem, e->st);
  else
    err = cudaLaunchCooperativeKernel((void*)k_ensemble_step<0>, e->grid, kEnsNT, args, smem, e->st);
  count_launch();
  return cuda_status(err, "k_ensemble_step launch");
}

static exa_status_t configure_grid(exa_ensemble* e) {
  const size_t smem = sizeof(double) * kEnsSmemDoubles;
  const void* k = e->precision == EXA_PREC_MIXED ? (const void*)k_ensemble_step<1> : (const void*)k_ensemble_step<0>;
  cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return cuda_status(err, "ensemble attribute");
  int per_sm = 0, sms = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kEnsNT, smem);
  if (err != cudaSuccess) return cuda_status(err, "ensemble occupancy");
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  if (per_sm < 1) return set_error(EXA_ECUDA, "ensemble kernel cannot be resident");
  const int want = e->ctas_per_sm > 0 ? std::min(e->ctas_per_sm, per_sm) : per_sm;
  e->grid = want * sms;
  if (e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  return EXA_OK;
}

namespace exa {
bool ens_arena_alloc(exa_ensemble* e, size_t bytes, char** ptr, size_t* off) {
  std::lock_guard<std::mutex> lk(e->mu);
  if (!arena_alloc(e, align256(bytes), off)) return false;
  *ptr = e->arena + *off;
  return true;
}
void ens_arena_free(exa_ensemble* e, size_t off, size_t bytes) {
  std::lock_guard<std::mutex> lk(e->mu);
  arena_free(e, off, align256(bytes));
}
cudaStream_t ens_stream(exa_ensemble* e) { return e->st; }
// The kernels skip an inactive solve without touching its state, faces or
// arena range, so a finished solve's memory can go back to the arena while
// a step is in flight; its record is zeroed after that step, in stream order.
exa_status_t ens_remove_finished(exa_ensemble* e, int slot) {
  std::lock_guard<std::mutex> lk(e->mu);
  if (slot < 0 || slot >= e->max_solves || !e->used[slot]) return set_error(EXA_ENOTFOUND, "slot not in use");
  const cudaError_t err = cudaMemsetAsync(e->d_solves + slot, 0, sizeof(SolveDev), e->st);
  if (err != cudaSuccess) return cuda_status(err, "ensemble remove");
  arena_free(e, e->alloc_off[slot], e->alloc_size[slot]);
  e->used[slot] = 0;
  e->host[slot] = SolveDev{};
  e->dirty = true;
  return EXA_OK;
}
}  // namespace exa

extern "C" {

size_t exa_ensemble_footprint(const exa_solve_config_t* cfg) {
  long nc;
  size_t a, b;
  if (solve_sizes(cfg, &nc, &a, &b)) return 0;
  return solve_footprint(nc, a, b);
}

exa_status_t exa_ensemble_create(int precision, int max_solves, size_t arena_bytes, exa_ensemble** out) {
  if (!out || max_solves < 1 || max_solves > (1 << 20) || arena_bytes < 4096)
    return set_error(EXA_EINVAL, "bad ensemble arguments");
  if (precision != EXA_PREC_FP64 && precision != EXA_PREC_MIXED) return set_error(EXA_EINVAL, "precision");
  exa_ensemble* e = new (std::nothrow) exa_ensemble;
  if (!e) return set_error(EXA_ENOMEM, "host allocation");
  e->precision = precision;
  e->max_solves = max_solves;
  e->arena_bytes = arena_bytes;
  cudaGetDevice(&e->device);
  e->host.assign(max_solves, SolveDev{});
  e->alloc_off.assign(max_solves, 0);
  e->alloc_size.assign(max_solves, 0);
  e->used.assign(max_solves, 0);
  exa_status_t s = ensure_tables();
  cudaError_t err = cudaSuccess;
  if (!s) err = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking);
  for (int k = 0; k < 4 && !s && err == cudaSuccess; k++) {
    err = cudaStreamCreateWithFlags(&e->ost[k], cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->join_ev[k], cudaEventDisableTiming);
  }
  if (!s && err == cudaSuccess) err = cudaEventCreateWithFlags(&e->fork_ev, cudaEventDisableTiming);
  if (!s && err == cudaSuccess) err = cudaMalloc(&e->arena, arena_bytes);
  if (!s && err == cudaSuccess) err = cudaMalloc(&e->d_solves, sizeof(SolveDev) * max_solves);
  if (!s && err == cudaSuccess) err = cudaMalloc(&e->d_ctr, 2 * sizeof(unsigned int));
  if (!s && err == cudaSuccess) err = cudaMemsetAsync(e->d_ctr, 0, 2 * sizeof(unsigned int), e->st);
  if (!s && err == cudaSuccess) err = cudaMemsetAsync(e->d_solves, 0, sizeof(SolveDev) * max_solves, e->st);
  if (!s && err == cudaSuccess) err = cudaStreamSynchronize(e->st);
  if (!s && err != cudaSuccess) s = cuda_status(err, "ensemble allocation");
  if (!s) s = configure_grid(e);
  if (s) {
    exa_ensemble_destroy(e);
    return s;
  }
  e->free_list.push_back(ArenaBlock{0, arena_bytes});
  *out = e;
  return EXA_OK;
}

exa_status_t exa_ensemble_destroy(exa_ensemble* e) {
  if (!e) return EXA_OK;
  if (e->st) cudaStreamSynchronize(e->st);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  cudaFree(e->arena);
  cudaFree(e->d_solves);
  cudaFree(e->d_items);
  cudaFree(e->d_ctr);
  if (e->st) cudaStreamDestroy(e->st);
  for (int k = 0; k < 4; k++) {
    if (e->ost[k]) cudaStreamDestroy(e->ost[k]);
    if (e->join_ev[k]) cudaEventDestroy(e->join_ev[k]);
  }
  if (e->fork_ev) cudaEventDestroy(e->fork_ev);
  delete e;
  return EXA_OK;
}

exa_status_t exa_ensemble_add(exa_ensemble* e, const exa_solve_config_t* c, long long steps, int* slot) {
  if (!e || !slot) return set_error(EXA_EINVAL, "NULL argument");
  long nc;
  size_t n_luh, n_face;
  if (exa_status_t s = solve_sizes(c, &nc, &n_luh, &n_face)) return s;
  std::lock_guard<std::mutex> lk(e->mu);
  int sl = -1;
  for (int i = 0; i < e->max_solves; i++)
    if (!e->used[i]) { sl = i; break; }
  if (sl < 0) return set_error(EXA_EBUSY, "no free solve slot");
  const size_t bytes = solve_footprint(nc, n_luh, n_face);
  size_t off = 0;
  if (!arena_alloc(e, bytes, &off)) return set_error(EXA_EBUSY, "not enough free device memory in the arena");
  SolveDev& sv = e->host[sl];
  sv = SolveDev{};
  sv.order = c->order;
  sv.pde = c->pde;
  sv.dt_policy = c->dt_policy;
  sv.active = steps != 0;
  sv.n[0] = c->n[0];
  sv.n[1] = c->n[1];
  sv.dx[0] = c->length[0] / c->n[0];
  sv.dx[1] = c->length[1] / c->n[1];
  sv.ncells = nc;
  char* base = e->arena + off;
  sv.luh = (double*)base;
  sv.lduh = (double*)(base + align256(n_luh * 8));
  sv.qb = (double*)(base + 2 * align256(n_luh * 8));
  sv.fb = (double*)(base + 2 * align256(n_luh * 8) + align256(n_face * 8));
  sv.dt_factor = c->dt_policy == 0 ? c->cfl * host_pnpm(c->order) : c->cfl / (2 * c->order + 1);
  sv.dt_fixed = c->dt_fixed;
  sv.dt_next = 0x7FF0000000000000ULL;
  sv.steps_left = steps;
  e->used[sl] = 1;
  e->alloc_off[sl] = off;
  e->alloc_size[sl] = bytes;
  // initial condition and first dt on the device
  double dx3[3] = {sv.dx[0], sv.dx[1], 1.0};
  int n3[3] = {sv.n[0], sv.n[1], 1};
  exa_status_t s = launch_grid_ic(2, c->order, n3, dx3, sv.luh, c->ic_kind, c->ic_param, c->seed, c->noise, e->st);
  cudaError_t err = cudaSuccess;
  if (!s) err = cudaMemcpyAsync(e->d_solves + sl, &sv, sizeof(SolveDev), cudaMemcpyHostToDevice, e->st);
  if (!s && err == cudaSuccess && c->dt_policy != 2) {
    exa_aderdg_desc_t d{2, c->order, kV, 0, c->pde, e->precision, {sv.dx[0], sv.dx[1], 1.0}};
    s = launch_stable_dt(d, nc, sv.luh, sv.dt_factor, nullptr, &e->d_solves[sl].dt_next, e->st);
  }
  if (!s && err == cudaSuccess) {
    k_solve_prime<<<1, 1, 0, e->st>>>(e->d_solves + sl);
    count_launch();
    err = cudaGetLastError();
  }
  if (!s && err != cudaSuccess) s = cuda_status(err, "ensemble add");
  if (s) {
    e->used[sl] = 0;
    arena_free(e, off, bytes);
    return s;
  }
  e->dirty = true;
  *slot = sl;
  return EXA_OK;
}

exa_status_t exa_ensemble_remove(exa_ensemble* e, int slot) {
  if (!e || slot < 0 || slot >= e->max_solves) return set_error(EXA_EINVAL, "bad slot");
  std::lock_guard<std::mutex> lk(e->mu);
  if (!e->used[slot]) return set_error(EXA_ENOTFOUND, "slot not in use");
  cudaStreamSynchronize(e->st);
  SolveDev z{};
  cudaError_t err = cudaMemcpy(e->d_solves + slot, &z, sizeof(SolveDev), cudaMemcpyHostToDevice);
  if (err != cudaSuccess) return cuda_status(err, "ensemble remove");
  arena_free(e, e->alloc_off[slot], e->alloc_size[slot]);
  e->used[slot] = 0;
  e->host[slot] = z;
  e->dirty = true;
  return EXA_OK;
}

exa_status_t exa_ensemble_step(exa_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return set_error(EXA_EINVAL, "bad argument");
  std::lock_guard<std::mutex> lk(e->mu);
  if (e->dirty)
    if (exa_status_t s = rebuild_items(e)) return s;
  if (e->nitems == 0) return EXA_OK;
  if (e->use_graph && !e->graph) {
    cudaGraph_t g;
    cudaError_t err = cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) return cuda_status(err, "ensemble capture");
    exa_status_t s = launch_step(e);
    err = cudaStreamEndCapture(e->st, &g);
    if (s) return s;
    if (err != cudaSuccess) return cuda_status(err, "ensemble end capture");
    err = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) return cuda_status(err, "ensemble graph instantiate");
  }
  for (int i = 0; i < nsteps; i++) {
    if (e->use_graph) {
      cudaError_t err = cudaGraphLaunch(e->graph, e->st);
      count_launch();
      if (err != cudaSuccess) return cuda_status(err, "ensemble graph launch");
    } else if (exa_status_t s = launch_step(e)) {
      return s;
    }
  }
  return EXA_OK;
}

exa_status_t exa_ensemble_use_graph(exa_ensemble* e, int enable) {
  if (!e) return set_error(EXA_EINVAL, "NULL ensemble");
  std::lock_guard<std::mutex> lk(e->mu);
  e->use_graph = enable != 0;
  return EXA_OK;
}

exa_status_t exa_ensemble_tune(exa_ensemble* e, int ctas_per_sm, int grab, int order_policy) {
  if (!e || grab < 1 || grab > 64 || ctas_per_sm < 0 || order_policy < 0 || order_policy > 1)
    return set_error(EXA_EINVAL, "bad tuning");
  std::lock_guard<std::mutex> lk(e->mu);
  cudaStreamSynchronize(e->st);
  e->ctas_per_sm = ctas_per_sm;
  e->grab = grab;
  e->order_policy = order_policy;
  e->dirty = true;
  return configure_grid(e);
}

exa_status_t exa_ensemble_tune_contraction(exa_ensemble* e, int lines_mask) {
  if (!e || (lines_mask & ~0x3C)) return set_error(EXA_EINVAL, "contraction mask: bits 2..5 (orders) only");
  std::lock_guard<std::mutex> lk(e->mu);
  cudaStreamSynchronize(e->st);
  e->lines_mask = lines_mask;
  e->dirty = true;  // the step graph holds the kernel arguments
  return EXA_OK;
}

exa_status_t exa_ensemble_set_launch_mode(exa_ensemble* e, int mode) {
  if (!e || mode < 0 || mode > 1) return set_error(EXA_EINVAL, "launch mode: 0 persistent, 1 per order");
  std::lock_guard<std::mutex> lk(e->mu);
  cudaStreamSynchronize(e->st);
  e->mode = mode;
  e->dirty = true;  // item order and the step graph
  return EXA_OK;
}

exa_status_t exa_ensemble_synchronize(exa_ensemble* e) {
  if (!e) return set_error(EXA_EINVAL, "NULL ensemble");
  return cuda_status(cudaStreamSynchronize(e->st), "ensemble sync");
}

exa_status_t exa_ensemble_stream(exa_ensemble* e, void** stream) {
  if (!e || !stream) return set_error(EXA_EINVAL, "NULL argument");
  *stream = e->st;
  return EXA_OK;
}

exa_status_t exa_ensemble_get_state(exa_ensemble* e, int slot, double* host_luh) {
  if (!e || !host_luh || slot < 0 || slot >= e->max_solves) return set_error(EXA_EINVAL, "bad argument");
  if (!e->used[slot]) return set_error(EXA_ENOTFOUND, "slot not in use");
  const SolveDev& sv = e->host[slot];
  const int B = sv.order + 1;
  cudaError_t err = cudaMemcpyAsync(host_luh, sv.luh, sizeof(double) * sv.ncells * B * B * kV,
                                    cudaMemcpyDeviceToHost, e->st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->st);
  return cuda_status(err, "ensemble get_state");
}

exa_status_t exa_ensemble_checkpoint(exa_ensemble* e, int slot, double* host_luh, exa_solve_checkpoint_t* ck) {
  if (!e || !host_luh || !ck || slot < 0 || slot >= e->max_solves) return set_error(EXA_EINVAL, "bad argument");
  std::lock_guard<std::mutex> lk(e->mu);
  if (!e->used[slot]) return set_error(EXA_ENOTFOUND, "slot not in use");
  const SolveDev& hs = e->host[slot];
  const int B = hs.order + 1;
  SolveDev d{};
  cudaError_t err = cudaMemcpyAsync(host_luh, hs.luh, sizeof(double) * hs.ncells * B * B * kV,
                                    cudaMemcpyDeviceToHost, e->st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(&d, e->d_solves + slot, sizeof(SolveDev), cudaMemcpyDeviceToHost, e->st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->st);
  if (err != cudaSuccess) return cuda_status(err, "ensemble checkpoint");
  *ck = exa_solve_checkpoint_t{};
  ck->time = d.time;
  ck->dt = d.dt;
  ck->dt_next_bits = d.dt_next;
  ck->steps_done = d.steps_done;
  ck->steps_left = d.steps_left;
  ck->picard = d.stats[0];
  ck->nonconverged = d.stats[1];
  ck->active = d.active;
  ck->nan_flag = d.nan_flag;
  return EXA_OK;
}

exa_status_t exa_ensemble_restore(exa_ensemble* e, const exa_solve_config_t* c, const double* host_luh,
                                  const exa_solve_checkpoint_t* ck, int* slot) {
  if (!e || !c || !host_luh || !ck || !slot) return set_error(EXA_EINVAL, "NULL argument");
  long nc;
  size_t n_luh, n_face;
  if (exa_status_t s = solve_sizes(c, &nc, &n_luh, &n_face)) return s;
  std::lock_guard<std::mutex> lk(e->mu);
  int sl = -1;
  for (int i = 0; i < e->max_solves; i++)
    if (!e->used[i]) { sl = i; break; }
  if (sl < 0) return set_error(EXA_EBUSY, "no free solve slot");
  const size_t bytes = solve_footprint(nc, n_luh, n_face);
  size_t off = 0;
  if (!arena_alloc(e, bytes, &off)) return set_error(EXA_EBUSY, "not enough free device memory in the arena");
  SolveDev& sv = e->host[sl];
  sv = SolveDev{};
  sv.order = c->order;
  sv.pde = c->pde;
  sv.dt_policy = c->dt_policy;
  sv.n[0] = c->n[0];
  sv.n[1] = c->n[1];
  sv.dx[0] = c->length[0] / c->n[0];
  sv.dx[1] = c->length[1] / c->n[1];
  sv.ncells = nc;
  char* base = e->arena + off;
  sv.luh = (double*)base;
  sv.lduh = (double*)(base + align256(n_luh * 8));
  sv.qb = (double*)(base + 2 * align256(n_luh * 8));
  sv.fb = (double*)(base + 2 * align256(n_luh * 8) + align256(n_face * 8));
  sv.dt_factor = c->dt_policy == 0 ? c->cfl * host_pnpm(c->order) : c->cfl / (2 * c->order + 1);
  sv.dt_fixed = c->dt_fixed;
  // the time-step state exactly as checkpointed: the solve continues with
  // the dt its last corrector reduced, bit for bit as if never removed
  sv.active = ck->active;
  sv.dt = ck->dt;
  sv.dt_next = ck->dt_next_bits;
  sv.time = ck->time;
  sv.steps_done = ck->steps_done;
  sv.steps_left = ck->steps_left;
  sv.stats[0] = ck->picard;
  sv.stats[1] = ck->nonconverged;
  sv.nan_flag = ck->nan_flag;
  e->used[sl] = 1;
  e->alloc_off[sl] = off;
  e->alloc_size[sl] = bytes;
  cudaError_t err = cudaMemcpyAsync(sv.luh, host_luh, n_luh * 8, cudaMemcpyHostToDevice, e->st);
  if (err == cudaSuccess) err = cudaMemcpyAsync(e->d_solves + sl, &sv, sizeof(SolveDev), cudaMemcpyHostToDevice, e->st);
  // the host copy must not be reused before the upload has read it
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->st);
  if (err != cudaSuccess) {
    e->used[sl] = 0;
    arena_free(e, off, bytes);
    sv = SolveDev{};
    return cuda_status(err, "ensemble restore");
  }
  e->dirty = true;
  *slot = sl;
  return EXA_OK;
}

exa_status_t exa_ensemble_device_state(exa_ensemble* e, int slot, double** luh_dev) {
  if (!e || !luh_dev || slot < 0 || slot >= e->max_solves) return set_error(EXA_EINVAL, "bad argument");
  if (!e->used[slot]) return set_error(EXA_ENOTFOUND, "slot not in use");
  *luh_dev = e->host[slot].luh;
  return EXA_OK;
}

/* Reads every slot's state: time, steps done, remaining-active flag, Picard
 * iteration sum, NaN flag (arrays of max_solves entries, each nullable). */
exa_status_t exa_ensemble_status(exa_ensemble* e, double* time, uint64_t* steps_done, int* active,
                                 uint64_t* picard, int* nan_flag) {
  if (!e) return set_error(EXA_EINVAL, "NULL ensemble");
  std::vector<SolveDev> h(e->max_solves);
  cudaError_t err = cudaMemcpyAsync(h.data(), e->d_solves, sizeof(SolveDev) * e->max_solves,
                                    cudaMemcpyDeviceToHost, e->st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->st);
  if (err != cudaSuccess) return cuda_status(err, "ensemble status");
  bool any_nan = false;
  for (int i = 0; i < e->max_solves; i++) {
    const bool u = e->used[i];
    if (time) time[i] = u ? h[i].time : 0.0;
    if (steps_done) steps_done[i] = u ? h[i].steps_done : 0;
    if (active) active[i] = u ? h[i].active : 0;
    if (picard) picard[i] = u ? h[i].stats[0] : 0;
    if (nan_flag) nan_flag[i] = u ? h[i].nan_flag : 0;
    any_nan = any_nan || (u && h[i].nan_flag);
    if (u && e->host[i].active && !h[i].active) {
      e->host[i].active = 0;  // finished: its work items are dropped at the next rebuild
      e->dirty = true;
    }
  }
  return any_nan ? EXA_ENAN : EXA_OK;
}

long exa_ensemble_active_cells(exa_ensemble* e) {
  if (!e) return 0;
  long n = 0;
  for (int i = 0; i < e->max_solves; i++)
    if (e->used[i] && e->host[i].active) n += e->host[i].ncells;
  return n;
}

exa_status_t exa_ensemble_info(exa_ensemble* e, int* grid_ctas, int* nitems, size_t* arena_free_bytes) {
  if (!e) return set_error(EXA_EINVAL, "NULL ensemble");
  if (grid_ctas) *grid_ctas = e->grid;
  if (nitems) *nitems = e->nitems;
  if (arena_free_bytes) {
    size_t f = 0;
    for (auto& b : e->free_list) f += b.size;
    *arena_free_bytes = f;
  }
  return EXA_OK;
}

}  // extern "C"
