// Internal host-side declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/exa_kernels.h"

namespace exa {

// Process-wide tuning knobs (set through exa_tune_set, read by launchers).
enum TuneKey {
  kTuneMixedOccupancy = 0,
  kTuneFp64Occupancy = 1,
  kTuneMixedVariant = 2,
  kTuneFp64Variant = 3,
  kTuneLimiterCellsPerCta = 4,
  kTuneFvGodunov = 5,
  kTuneCount = 8
};
int tune_get(int key, int dflt);

// Records a CUDA error (message retrievable by exa_last_error_string) and
// maps it to EXA_ECUDA.
exa_status_t cuda_status(cudaError_t e, const char* where);
exa_status_t set_error(exa_status_t s, const char* msg);
void count_launch(uint64_t n = 1);
// Makes sure the constant-memory tables of every translation unit are
// uploaded on the current device.
exa_status_t ensure_tables();
// Whether a grid steps with a fixed dt (no dt reduction between slabs).
bool grid_fixed_dt(const exa_aderdg_grid* g);

// Descriptor checks of the per-cell ADER-DG drop-ins (dim, order, nvar,
// npar, pde, dx), without the table upload.
exa_status_t check_aderdg_desc(const exa_aderdg_desc_t* d);

// Arguments of the fused predictor kernel (one struct so the launch
// wrappers stay small).
struct PredArgs {
  long ncells;
  const double* luh;
  double dt;
  const double* dt_dev;
  double idx[3];     // 1/dx
  double* lduh;
  double* lQhbnd;
  double* lFhbnd;
  int* iters;
  unsigned long long* stats;
  // full (reference temporaries) outputs, mode 1 only
  double* lQi;
  double* lFi;
  double* lQhi;
  double* lFhi;
  // mixed-precision error feedback (unused in FP64 mode)
  int precision;
};

exa_status_t launch_predictor(const exa_aderdg_desc_t& d, const PredArgs& a, int full,
                              cudaStream_t st);
exa_status_t launch_predictor_mixed(const exa_aderdg_desc_t& d, const PredArgs& a, cudaStream_t st);

// fused Riemann + surface integral + update + next-dt on a uniform periodic grid
struct CorrArgs {
  long ncells;
  int n[3];
  double dx[3];
  const double* dt_dev;     // dt of this step
  double* luh;
  const double* lduh;
  const double* lQhbnd;
  const double* lFhbnd;
  unsigned long long* dt_next;  // atomic-min slot for the next dt (nullable)
  double dt_factor;             // CFL*PNPM[N] or CFL/(2N+1)
  int* nan_flag;
  // Slab decomposition along the last dimension: when set, the neighbours
  // across the lower / upper end of that dimension are not the periodic
  // wrap-around cells but face data received from the adjacent slabs,
  // [layer cell][Q | F][face nodes][var] (layer cell = index within the
  // boundary layer).  NULL = periodic.
  const double* halo_lo;
  const double* halo_hi;
  // boundary rule per dimension (EXA_BC_*; 0 = periodic) and whether any
  // dimension is not periodic (uniform over the CTA: guards a barrier)
  int bc[3];
  int bc_any;
};
exa_status_t launch_corrector(int dim, int order, int pde, const CorrArgs& a, cudaStream_t st);

// per-cell stable dt (+ optional global min via atomic slot)
exa_status_t launch_stable_dt(const exa_aderdg_desc_t& d, long ncells, const double* luh,
                              double factor, double* dt_cell, unsigned long long* dt_min_bits,
                              cudaStream_t st);
exa_status_t launch_volume_integral(const exa_aderdg_desc_t& d, long ncells, double* lduh,
                                    const double* lFhi, cudaStream_t st);
exa_status_t launch_surface_integral(const exa_aderdg_desc_t& d, long ncells, double* lduh,
                                     const double* lFhbnd, cudaStream_t st);
exa_status_t launch_solution_update(const exa_aderdg_desc_t& d, long ncells, double* luh,
                                    const double* lduh, double dt, cudaStream_t st);
exa_status_t launch_riemann_faces(const exa_aderdg_desc_t& d, long nfaces, const int* left,
                                  const int* right, const int* dir, const double* lQhbnd,
                                  double* lFhbnd, cudaStream_t st);
// cell_offset / n_last_global place a slab of the last dimension inside a
// larger domain (global cell index = local + cell_offset); 0 / n[dim-1] for
// a whole domain.
exa_status_t launch_grid_ic(int dim, int order, const int* n, const double* dx, double* luh,
                            int kind, double param, uint64_t seed, double noise,
                            cudaStream_t st, long cell_offset = 0, int n_last_global = 0);

// Device-resident single periodic patch; slots = 3 x 64-bit scalars
// ([0] dt, [1] time, [2] next dt), time must start at 0 (caller zeroes it).
exa_status_t fv_patch_prime_async(const exa_fv_desc_t& d, const double* luh, unsigned long long* slots,
                                  cudaStream_t st);
exa_status_t fv_patch_step_async(int scheme, const exa_fv_desc_t& d, const double* luh, double* luh_new,
                                 unsigned long long* slots, cudaStream_t st);
exa_status_t launch_fv_ic(const exa_fv_desc_t& d, double* luh, double amp, uint64_t seed, double noise,
                          cudaStream_t st);
// arena of an ensemble, shared with the serving engine
bool ens_arena_alloc(exa_ensemble* e, size_t bytes, char** ptr, size_t* off);
void ens_arena_free(exa_ensemble* e, size_t off, size_t bytes);
cudaStream_t ens_stream(exa_ensemble* e);
// exa_ensemble_remove of a finished solve (inactive on the device): the slot
// is cleared in stream order and its memory returned without a host wait
exa_status_t ens_remove_finished(exa_ensemble* e, int slot);

exa_status_t launch_rusanov_one(int pde, int d, const double* qL, const double* qR, double* out);

// table uploads, one per translation unit holding kernels
exa_status_t upload_tables_predictor();
exa_status_t upload_tables_predictor_mixed();
exa_status_t upload_tables_ensemble();
exa_status_t upload_tables_faces();
exa_status_t upload_tables_fv();
exa_status_t upload_tables_amr();
exa_status_t upload_tables_limiter();
exa_status_t upload_tables_adjust();

// FV step (scheme 0 Godunov, 1 MUSCL-Hancock) on the subcell patches
// lim[cell] (P subcells + g ghost layers per direction, 5 variables) of the
// cells list[0 .. *count) of a periodic npx x npy grid: face ghosts from the
// neighbour cells' patches, then the update in place with *dt_dev (fv.cu);
// the 3D counterpart on an n[0] x n[1] x n[2] grid (fv3d.cu)
// bc[d] (nullable: periodic) = EXA_BC_*: at a domain boundary the ghosts
// come from the patch's own boundary layers (the reference's
// boundaryLayerExtraction / ghostLayerFillingAtBoundary, commons.cpph:
// 100-340), with the normal momentum negated for reflecting walls
exa_status_t fv_subcell_step(int scheme, int planar, int P, int g, int npx, int npy, double hx, double hy,
                             double* lim, const int* list, const int* count, long maxcells, const double* dt_dev,
                             cudaStream_t st, const int* bc = nullptr);
exa_status_t fv3_subcell_step(int scheme, int P, int g, const int* n, const double* h, double* lim, const int* list,
                              const int* count, long maxcells, const double* dt_dev, cudaStream_t st,
                              const int* bc = nullptr);

// 3D finite volumes (fv3d.cu): one CTA per patch of P^3 cells + g ghost
// layers, [z][y][x][D]; h = cell sizes; dt read from dt_dev when non-null;
// optional patch selection list[0 .. *count) (then npatches bounds it)
exa_status_t fv3_update(int scheme, int P, int g, int D, const double* h, long npatches, double* luh_new,
                        const double* luh, double dt, const double* dt_dev, double* max_dt, const int* list,
                        const int* count, cudaStream_t st);
exa_status_t fv3_stable_dt(int P, int g, int D, const double* h, long npatches, const double* luh, double* dt_patch,
                           cudaStream_t st);
exa_status_t fv3_periodic_ghosts(int P, int g, int D, long npatches, double* luh, cudaStream_t st);
size_t fv3_smem(int P, int g, int scheme);

// limiting-grid bookkeeping (limiting.cu): status from the DMP /
// admissibility verdicts with spreading and the cell lists; the merge of
// the per-cell extrema over faces; a finiteness check of listed cells
// solution adjustment on a uniform grid (adjust.cu): the hook at every node
// of every cell, cell centers (i + 1/2) dx, t = *time_dev + *dt_dev
exa_status_t grid_adjust(int dim, int order, const int* n, const double* dx, long ncells, double* luh,
                         const double* time_dev, const double* dt_dev, const exa_adjust_t& hook, cudaStream_t st);
exa_status_t check_adjust_hook(const exa_adjust_t* h);
exa_status_t limiting_status(int dim, const int* ncell, const int* bc, int npc, int planar, int admissibility,
                             int steps_till_cured, const double* luh, int* ok, int* status, int* status_tmp,
                             int* cure, int* list_patch, int* list_fv, int* counts, cudaStream_t st);
exa_status_t limiting_merge_bounds(int dim, const int* ncell, const int* bc, int nobs, double* bmin, double* bmax,
                                   double* loc, cudaStream_t st);
exa_status_t limiting_check_finite(int npc, const double* luh, const int* list, const int* count, int* nan_flag,
                                   cudaStream_t st);

// limiter kernels (limiter.cu) on all cells, or on cells list[0 .. *count)
// when list / count (device) are given
enum LimiterOp { kLimToFv = 0, kLimToDg = 1, kLimMinMax = 2, kLimDmp = 3, kLimFvMinMax = 4 };
exa_status_t limiter_launch(int op, int dim, int order, int nvar, int nobs, int ghost, long ncells, const double* in,
                            double* out, double* mn, double* mx, int* ok, double relax, double scaling,
                            cudaStream_t st, const int* list, const int* count);
// host copy of the derived tables (same bytes as the device constants)
const void* host_dg_tables(size_t* bytes);
const void* host_dg_tables_f(size_t* bytes);  // FP32 copies (DGConstF)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// One live periodic FV patch of the serving batch (fv.cu): the state
// alternates between buf[0] and buf[1]; slots: [0] dt of the current step,
// [1] simulated time, [2] next dt (atomic min), [3] index of the buffer that
// holds the state.  Patches of one launch are listed by their first tile
// (tile0, ascending); tiles_x tiles per tile row.
struct FVServePatch {
  double* buf[2];
  unsigned long long* slots;
  int P, g, tiles_x, tile0;
  double hx, hy;
};
// tiles of a patch of `patch` cells per side for the scheme's tile kernel
int fv_serve_tiles(int scheme, int patch, int* tiles_x);
// one step of every listed patch (device table of np entries, ntiles tiles
// in all) and the per-patch commit, on stream st
exa_status_t fv_serve_step_async(int scheme, bool planar, const FVServePatch* table, int np, int ntiles,
                                 cudaStream_t st);

}  // namespace exa
