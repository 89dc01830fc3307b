/*
 * exahype_b200 -- C ABI of the B200 (sm_100a) ADER-DG / finite-volume
 * cell-update library (libexahype_b200.so).
 *
 * The entry points mirror the generic C++ kernels of ExaHyPE
 * (ExaHyPE/kernels/aderdg/generic/Kernels.h:86-175,
 * kernels/finitevolumes/{godunov,musclhancock,riemannsolvers,commons}/c/)
 * and the solver methods that call them (the toolkit-generated
 * Abstract<Solver>, Toolkit/src/eu/exahype/solvers/templates/
 * AbstractGenericADERDGSolverHeader.template:166-177 and
 * AbstractGenericFiniteVolumesSolverHeader.template:52-63).
 *
 * Conventions
 *  - All data are FP64 in the reference's row-major per-cell layouts
 *    (ExaHyPE/kernels/KernelUtils.h:243-320), slowest index first:
 *      luh    [z][y][x][nVar+nPar]          (2D: [y][x][...])
 *      lduh   [z][y][x][nVar]
 *      lQhbnd [2*dim][B][B][nVar+nPar], lFhbnd [2*dim][B][B][nVar]
 *      lFhi   (dim+1) blocks: x [z][y][x], y [z][x][y], z [y][x][z], source
 *    with B = order+1.  Batched entry points take `ncells` cells stored
 *    back to back (cell stride = size of one cell's array).
 *  - The PDE is compiled in: compressible Euler, nVar = 5, gamma = 1.4.
 *    PDE callbacks of the reference (flux, eigenvalues) cannot cross to
 *    the device, so the PDE is selected by enum.
 *  - Every function returns an exa_status_t; nothing aborts.  Device
 *    entry points are asynchronous on `stream` (a cudaStream_t passed as
 *    void*, NULL = legacy default stream) and never allocate.
 *  - Kernels are reentrant; concurrent calls on different streams need
 *    distinct output buffers, as in the reference (TBB workers with
 *    distinct temporaries, mappings/Prediction.cpp:152).
 */
#ifndef EXA_KERNELS_H
#define EXA_KERNELS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status */
typedef int exa_status_t;
#define EXA_OK          0
#define EXA_EINVAL      1  /* unsupported dimension/order/size or NULL pointer */
#define EXA_ENONCONV    2  /* Picard iteration hit 2(N+1) iterations in >= 1 cell */
#define EXA_ENAN        3  /* a NaN/Inf was produced */
#define EXA_ETIMEDOUT   4  /* a bounded device-side wait gave up */
#define EXA_ECUDA       5  /* CUDA runtime error (see exa_last_error_string) */
#define EXA_ENOMEM      6  /* device or host allocation failed */
#define EXA_EBUSY       7  /* admission refused: not enough free slots/memory */
#define EXA_ENOTFOUND   8  /* unknown handle / request id */

const char* exa_status_string(exa_status_t s);
const char* exa_last_error_string(void);

typedef enum {
  EXA_PDE_EULER = 0,        /* pressure from all three momenta */
  EXA_PDE_EULER_PLANAR = 1  /* 2D "2.5D" form of the reference's kernel tests */
} exa_pde_t;

typedef enum {
  EXA_PREC_FP64 = 0,  /* plain path: every operation in FP64 */
  EXA_PREC_MIXED = 1  /* Picard contractions in reduced precision; update,
                         face fluxes and dt stay FP64 */
} exa_precision_t;

/* Describes one ADER-DG solver instance (the compile-time constants of the
 * generated Abstract<Solver>: NumberOfVariables/Parameters, Order,
 * AbstractGenericADERDGSolverHeader.template:31-34). */
typedef struct {
  int dim;        /* 2 or 3 */
  int order;      /* N; supported 2..5 (3 also with nPar = 1) */
  int nvar;       /* must be 5 */
  int npar;       /* 0, or 1 for the drop-in per-cell calls */
  int pde;        /* exa_pde_t */
  int precision;  /* exa_precision_t */
  double dx[3];   /* cell size per dimension */
} exa_aderdg_desc_t;

/* ---------------------------------------------- device/runtime helpers */
int exa_device_count(void);
exa_status_t exa_set_device(int device);
exa_status_t exa_device_alloc(size_t bytes, void** ptr);
exa_status_t exa_device_free(void* ptr);
exa_status_t exa_host_alloc_pinned(size_t bytes, void** ptr);
exa_status_t exa_host_free_pinned(void* ptr);
exa_status_t exa_memcpy_h2d(void* dst, const void* src, size_t bytes, void* stream);
exa_status_t exa_memcpy_d2h(void* dst, const void* src, size_t bytes, void* stream);
exa_status_t exa_memset_device(void* dst, int value, size_t bytes, void* stream);
exa_status_t exa_stream_create(void** stream);
exa_status_t exa_stream_destroy(void* stream);
exa_status_t exa_stream_synchronize(void* stream);
exa_status_t exa_device_synchronize(void);
/* CUDA-event timer on a stream */
exa_status_t exa_timer_create(void** timer);
exa_status_t exa_timer_destroy(void* timer);
exa_status_t exa_timer_start(void* timer, void* stream);
exa_status_t exa_timer_stop(void* timer, void* stream);
exa_status_t exa_timer_elapsed_ms(void* timer, float* ms);
/* number of kernels this library has launched in this process */
uint64_t exa_launch_count(void);
/* Diagnostic: capacity in doubles of the device workspace that the per-cell
 * drop-ins below allocate on first use on `device` (0 = not allocated).  No
 * counterpart in the reference. */
exa_status_t exa_dropin_workspace_doubles(int device, size_t* doubles);
/* Tuning knobs chosen by the autotuner (exahype_b200/autotune.py) or the
 * user; process-wide.  Keys: 0 = register budget of the 3D order-4 mixed
 * predictor as minimum resident CTAs per SM (node-gather and line-owner
 * forms: 1 unconstrained, 3 168 registers (the default), 4 128 registers;
 * progressive form: 5 96 registers, otherwise 128), 1 = the FP64 predictor's
 * (0: unconstrained; non-zero: cap for 3 CTAs/SM), 2 = contraction of the
 * mixed predictor (1: node-gather, 2: line-owner, 3: line-owner on tensor
 * cores (3xTF32, 3D order 4), 4: progressive line-owner (3D order 4 Euler,
 * 2D order 5); 0: progressive for 3D order 4 Euler and 2D order 5,
 * line-owner for the other orders >= 4, node-gather otherwise), 3 = the same
 * for the FP64 predictor (1: node-gather, 2: line-owner, 3: progressive
 * line-owner, order 4 (3D: Euler); 0: progressive for order 4 (3D: Euler),
 * line-owner for the other orders >= 4, node-gather otherwise), 4 = cells per CTA of the limiter kernels (0: automatic),
 * 5 = the fused 2D Godunov step (one patch, the patch grid; 1: 32 x 8 tile
 * kernel; otherwise the sweep kernel, warps walking up strips of rows).  exa_tune_get
 * returns -1 for keys never set. */
exa_status_t exa_tune_set(int key, int value);
int exa_tune_get(int key);
/* Error norms of device array a against reference b (n doubles): out[0]
 * relative L2 ||a-b||/||b||, out[1] relative Linf max|a-b|/max|b|,
 * out[2] ||a-b||, out[3] max|a-b|.  Synchronous on stream. */
exa_status_t exa_diff_norms(const double* a, const double* b, size_t n, double* out, void* stream);

/* ---------------------------------- ADER-DG: per-cell drop-ins (host) --
 * Same argument lists and semantics as the generated solver methods; the
 * buffers are HOST pointers for one cell.  Each call copies to the device,
 * runs the batched kernel on one cell and copies back (synchronous).  They
 * exist for semantic equivalence with the reference; throughput callers use
 * the batched device entry points below. */

/* Abstract<Solver>::spaceTimePredictor
 * (AbstractGenericADERDGSolverImplementation.template:50-124) ->
 * kernels::aderdg::generic::c::spaceTimePredictorNonlinear
 * (kernels/aderdg/generic/c/3d/spaceTimePredictorNonlinear.cpph:523-577).
 * Writes lQhbnd, lFhbnd, tempUnknowns (lQhi) and tempFluxUnknowns (lFhi);
 * if non-NULL also tempSpaceTimeUnknowns[0] (lQi) and
 * tempSpaceTimeFluxUnknowns[0] (lFi).  tempStateSizedVectors and
 * pointForceSources are ignored (no point sources in this PDE). */
exa_status_t exa_aderdg_spaceTimePredictor(
    const exa_aderdg_desc_t* desc, double* lQhbnd, double* lFhbnd,
    double** tempSpaceTimeUnknowns, double** tempSpaceTimeFluxUnknowns,
    double* tempUnknowns, double* tempFluxUnknowns,
    double* tempStateSizedVectors, const double* luh, const double* dx,
    double dt, double* pointForceSources, int* picardIterations);

/* Allocation-free variant of exa_aderdg_spaceTimePredictor (same arguments,
 * same checks, same results).  It has no counterpart in the reference: it
 * exists for callers that must not trigger a device allocation -- many host
 * threads calling per-cell kernels at once, as the reference's TBB workers
 * do (cudaMalloc/cudaFree take a device-wide lock and cudaFree synchronises
 * the device, stalling every other worker), or processes whose device memory
 * is already handed out by a pool allocator (a late cudaMalloc fails there).
 * The cell is staged through a file-scope device array of 65536 doubles
 * (512 KiB) that every GPU holds from library load to process exit; every
 * supported cell (order 2..5, 2D/3D, nPar <= 1) fits, larger requests get
 * EXA_EINVAL.  The first call on a device performs a one-time set-up (looks
 * up the array's device address, uploads the operator tables).  All calls
 * on a device share the one
 * array and keep the last call's contents; calls of this process are
 * serialised by a lock, any other overlap on the GPU races.  Like the
 * drop-in it copies synchronously on the default stream. */
exa_status_t exa_aderdg_spaceTimePredictor_noalloc(
    const exa_aderdg_desc_t* desc, double* lQhbnd, double* lFhbnd,
    double** tempSpaceTimeUnknowns, double** tempSpaceTimeFluxUnknowns,
    double* tempUnknowns, double* tempFluxUnknowns,
    double* tempStateSizedVectors, const double* luh, const double* dx,
    double dt, double* pointForceSources, int* picardIterations);

/* Abstract<Solver>::volumeIntegral -> volumeIntegralNonlinear
 * (kernels/aderdg/generic/c/3d/volumeIntegralNonlinear.cpph:26-125) */
exa_status_t exa_aderdg_volumeIntegral(const exa_aderdg_desc_t* desc,
                                       double* lduh, const double* lFhi,
                                       const double* dx);

/* Abstract<Solver>::surfaceIntegral -> surfaceIntegralNonlinear
 * (kernels/aderdg/generic/c/3d/surfaceIntegralNonlinear.cpph:21-85) */
exa_status_t exa_aderdg_surfaceIntegral(const exa_aderdg_desc_t* desc,
                                        double* lduh, const double* lFhbnd,
                                        const double* dx);

/* Abstract<Solver>::riemannSolver -> riemannSolverNonlinear<false>
 * (kernels/aderdg/generic/c/3d/riemannSolverNonlinear.cpph:37-120).
 * Rusanov flux; overwrites FL and FR in place with the numerical flux. */
exa_status_t exa_aderdg_riemannSolver(
    const exa_aderdg_desc_t* desc, double* FL, double* FR, const double* QL,
    const double* QR, double* tempFaceUnknownsArray,
    double** tempStateSizedVectors, double** tempStateSizedSquareMatrices,
    double dt, int normalNonZeroIndex, int isBoundaryFace);

/* Abstract<Solver>::solutionUpdate -> solutionUpdate
 * (kernels/aderdg/generic/c/3d/solutionUpdate.cpph:23-47) */
exa_status_t exa_aderdg_solutionUpdate(const exa_aderdg_desc_t* desc,
                                       double* luh, const double* lduh,
                                       double dt);

/* Abstract<Solver>::stableTimeStepSize -> stableTimeStepSize
 * (kernels/aderdg/generic/c/3d/stableTimeStepSize.cpph:21-61), CFL 0.9 */
exa_status_t exa_aderdg_stableTimeStepSize(const exa_aderdg_desc_t* desc,
                                           const double* luh,
                                           double* tempEigenvalues,
                                           const double* dx, double* dt_out);

/* ------------------------------ ADER-DG: batched device entry points --
 * Device pointers, `ncells` cells back to back, asynchronous on stream. */

/* spaceTimePredictor + volumeIntegral for every cell, fused
 * (ADERDGSolver::performPredictionAndVolumeIntegral, ADERDGSolver.cpp:
 * 1818-1946).  dt is read from *dt_dev when dt_dev != NULL, else `dt`.
 * picard_iters (nullable) receives the iterations per cell; stats
 * (nullable, 2 x uint64 on the device) accumulates {sum of iterations,
 * cells that did not converge}. */
exa_status_t exa_aderdg_predictor_vi(const exa_aderdg_desc_t* desc, long ncells,
                                     const double* luh, double dt,
                                     const double* dt_dev, double* lduh,
                                     double* lQhbnd, double* lFhbnd,
                                     int* picard_iters, uint64_t* stats,
                                     void* stream);

/* Same as above but also writes the reference's temporaries per cell:
 * lQi [z][y][x][t][nData], lFi [t][z][y][x][dim+1][nVar], lQhi, lFhi. */
exa_status_t exa_aderdg_predictor_full(const exa_aderdg_desc_t* desc, long ncells,
                                       const double* luh, double dt,
                                       double* lQi, double* lFi, double* lQhi,
                                       double* lFhi, double* lduh, double* lQhbnd,
                                       double* lFhbnd, int* picard_iters,
                                       void* stream);

/* volumeIntegralNonlinear for every cell (lFhi in reference layout). */
exa_status_t exa_aderdg_volume_integral(const exa_aderdg_desc_t* desc, long ncells,
                                        double* lduh, const double* lFhi,
                                        void* stream);

/* surfaceIntegralNonlinear for every cell. */
exa_status_t exa_aderdg_surface_integral(const exa_aderdg_desc_t* desc, long ncells,
                                         double* lduh, const double* lFhbnd,
                                         void* stream);

/* solutionUpdate for every cell. */
exa_status_t exa_aderdg_solution_update(const exa_aderdg_desc_t* desc, long ncells,
                                        double* luh, const double* lduh,
                                        double dt, void* stream);

/* Riemann solver on an explicit list of faces (ADERDGSolver::
 * solveRiemannProblemAtInterface, ADERDGSolver.cpp:2744-2826): face k joins
 * the face 2*dir+1 of cell left[k] and the face 2*dir of cell right[k];
 * both lFhbnd face blocks are overwritten with the Rusanov flux. */
exa_status_t exa_aderdg_riemann_faces(const exa_aderdg_desc_t* desc, long nfaces,
                                      const int* left, const int* right,
                                      const int* dir, const double* lQhbnd,
                                      double* lFhbnd, void* stream);

/* stableTimeStepSize for every cell; dt_cell (nullable) per cell, dt_min
 * (nullable, one double) receives the minimum over all cells (the global
 * min-reduction of TimeStepSizeComputation.cpp:83-109,204). */
exa_status_t exa_aderdg_stable_dt(const exa_aderdg_desc_t* desc, long ncells,
                                  const double* luh, double* dt_cell,
                                  double* dt_min, void* stream);

/* ------------------------------------ ADER-DG: uniform periodic grid --
 * The Peano spacetree is replaced by a uniform periodic cell array on one
 * GPU.  A step is dt -> predictor+VI -> Riemann -> SI -> update in the
 * reference's non-fused order (Runner.cpp:1125-1160); on the device the
 * Riemann solve, surface integral, update and the next step's dt
 * reduction are one fused kernel. */
typedef struct exa_aderdg_grid exa_aderdg_grid;

typedef struct {
  int dim, order;
  int n[3];            /* cells per dimension */
  double length[3];    /* domain extent; dx = length/n */
  int pde, precision;
  int dt_policy;       /* 0: CFL*PNPM[N] (reference), 1: CFL/(2N+1), 2: fixed */
  double cfl;          /* 0.9 in the reference's generated solvers */
  double dt_fixed;
} exa_aderdg_grid_config_t;

exa_status_t exa_aderdg_grid_create(const exa_aderdg_grid_config_t* cfg,
                                    exa_aderdg_grid** out);
exa_status_t exa_aderdg_grid_destroy(exa_aderdg_grid* g);
/* bytes of device memory a grid with this config needs */
size_t exa_aderdg_grid_footprint(const exa_aderdg_grid_config_t* cfg);
/* nodal initial condition on the device: kind 0 isentropic vortex
 * (param = strength), kind 1 density sine wave (param = amplitude); both
 * with seeded uniform density noise of relative amplitude noise_amp. */
exa_status_t exa_aderdg_grid_init(exa_aderdg_grid* g, int kind, double param,
                                  uint64_t seed, double noise_amp);
exa_status_t exa_aderdg_grid_set_state(exa_aderdg_grid* g, const double* host_luh);
exa_status_t exa_aderdg_grid_get_state(exa_aderdg_grid* g, double* host_luh);
/* advance nsteps; dt_host (nullable) receives nsteps dt values (forces a
 * device->host read at the end).  NaN and Picard non-convergence are
 * reported through exa_aderdg_grid_status (EXA_ENAN / EXA_ENONCONV). */
exa_status_t exa_aderdg_grid_step(exa_aderdg_grid* g, int nsteps, double* dt_host);
/* capture one step pair in a CUDA graph and replay it for later steps */
exa_status_t exa_aderdg_grid_use_graph(exa_aderdg_grid* g, int enable);
/* Boundary conditions per dimension (both ends), replacing the periodic
 * wrap.  The reference applies the user's boundaryValues hook at every face
 * node of a domain-boundary face (aderdg/generic/c/3d/boundaryConditions.cpph:
 * 24-85) and solves the Riemann problem between the cell's face data and the
 * returned outside state, the outside taken as the left state on faces 2d
 * and as the right state on faces 2d+1 (ADERDGSolver.cpp:2854-2925
 * applyBoundaryConditions).  PDE hooks cannot cross to the device, so the
 * outside state is one of these built-in rules:
 *   EXA_BC_OUTFLOW: QOut = QIn, FOut = FIn (the EulerFV demonstrator's rule,
 *     Demonstrators/EulerFV/MyEulerSolver.cpp:87-98);
 *   EXA_BC_REFLECT: QOut = QIn with the normal momentum negated, FOut = the
 *     normal flux of QOut (slip wall). */
enum { EXA_BC_PERIODIC = 0, EXA_BC_OUTFLOW = 1, EXA_BC_REFLECT = 2 };
exa_status_t exa_aderdg_grid_set_boundary(exa_aderdg_grid* g, const int* bc);
/* Solution adjustment (kernels/aderdg/generic/c/{2d,3d}/solutionAdjustment.
 * cpph: the solver's adjustPointSolution hook called at every Gauss-Legendre
 * node x = center + dx (xi - 1/2) of a cell with the node's weight, t and
 * dt; ADERDGSolver.cpp:2072-2092 applies it for the initial conditions at
 * t = 0 and :2158-2170 after every solutionUpdate at t + dt, whenever the
 * solver's useAdjustSolution says so).  PDE hooks cannot cross to the
 * device, so the hook is one of these built-in forms:
 *   EXA_ADJUST_SINE_WAVE: Q := (rho = 1 + a sin(2 pi (x0 + x1)), u = v = 1,
 *     w = 0, p = 1), param[0] = a (the 2D sine-wave benchmark state);
 *   EXA_ADJUST_ISENTROPIC_VORTEX: Q := the isentropic vortex of strength
 *     eps = param[0] around (1/2, 1/2), radius 0.1, on the flow (1, 1)
 *     (the 3D benchmark state, extruded in z);
 *   EXA_ADJUST_HEAT_SOURCE: time-dependent forcing, E += dt A exp(-|x -
 *     xc|^2 / s^2) (1 + sin(2 pi f t)), param = {A, s, f, xc0, xc1, xc2}.
 * when = EXA_ADJUST_AT_START applies the hook only at t == 0 (the
 * demonstrators' useAdjustSolution), EXA_ADJUST_ALWAYS at every call. */
enum { EXA_ADJUST_NONE = 0, EXA_ADJUST_SINE_WAVE = 1, EXA_ADJUST_ISENTROPIC_VORTEX = 2,
       EXA_ADJUST_HEAT_SOURCE = 3 };
enum { EXA_ADJUST_AT_START = 0, EXA_ADJUST_ALWAYS = 1 };
typedef struct {
  int kind;        /* EXA_ADJUST_* */
  int when;        /* EXA_ADJUST_AT_START or EXA_ADJUST_ALWAYS */
  double param[6];
} exa_adjust_t;
/* kernels::aderdg::generic::c::solutionAdjustment (Kernels.h:129-131, 347)
 * for one cell, HOST pointers: luh [B^dim][5], center[dim], dx[dim]. */
exa_status_t exa_aderdg_solutionAdjustment(int dim, int order, double* luh, const double* center,
                                           const double* dx, double t, double dt, const exa_adjust_t* hook);
/* batched, device-resident: luh [ncells][B^dim][5], centers [ncells][dim]
 * (device), cell size desc->dx */
exa_status_t exa_aderdg_solution_adjustment(const exa_aderdg_desc_t* desc, long ncells, double* luh,
                                            const double* centers, double t, double dt,
                                            const exa_adjust_t* hook, void* stream);
/* The grid applies the hook after every step's update at the new time
 * t + dt with that dt (ADERDGSolver::updateSolution :2158-2170; cell centers
 * (i + 1/2) dx), before the next dt is taken from the adjusted state; NULL
 * (or kind EXA_ADJUST_NONE) turns it off.  EXA_ADJUST_AT_START hooks never
 * fire during stepping (t > 0); exa_aderdg_grid_init sets the initial
 * state. */
exa_status_t exa_aderdg_grid_set_adjustment(exa_aderdg_grid* g, const exa_adjust_t* hook);
exa_status_t exa_aderdg_grid_stream(exa_aderdg_grid* g, void** stream);
/* Debug scan: with enable, every step scans the predictor's outputs (lduh,
 * lQhbnd, lFhbnd) and, after the update, the state for non-finite values
 * (one extra pass over each array).  exa_aderdg_grid_debug_status reports
 * where the first one was seen since the scan was enabled: where = 0 none,
 * 1 lduh, 2 lQhbnd, 3 lFhbnd, 4 luh; the step (counted from grid creation)
 * and the smallest element index of that array.  A NaN seeded into the
 * state shows up in the predictor's outputs of its cell (where = 1). */
exa_status_t exa_aderdg_grid_set_debug(exa_aderdg_grid* g, int enable);
exa_status_t exa_aderdg_grid_debug_status(exa_aderdg_grid* g, int* where, uint64_t* step, uint64_t* index);
/* per-phase CUDA-event timing of every step (disables graph replay):
 * predictor (k_predictor) and corrector (k_corrector + k_commit) */
exa_status_t exa_aderdg_grid_profile(exa_aderdg_grid* g, int enable);
exa_status_t exa_aderdg_grid_phase_times(exa_aderdg_grid* g, double* ms_predictor,
                                         double* ms_corrector, uint64_t* steps);
exa_status_t exa_aderdg_grid_device_state(exa_aderdg_grid* g, double** luh_dev);
/* time, accumulated Picard iterations, non-converged cell count, NaN flag.
 * Returns EXA_ENAN once a step produced a non-finite state (the reference's
 * validateNoNansInADERDGSolver, ADERDGSolver.cpp:1746), else EXA_ENONCONV
 * once any cell's Picard loop stopped at 2(N+1) iterations without meeting
 * its tolerance (the reference only warns, spaceTimePredictorNonlinear.cpph:
 * 308-315: the step's result is kept), else EXA_OK; the outputs are written
 * in every case. */
exa_status_t exa_aderdg_grid_status(exa_aderdg_grid* g, double* time,
                                    uint64_t* picard_iters_sum,
                                    uint64_t* nonconverged, int* nan_flag);
long exa_aderdg_grid_ncells(const exa_aderdg_grid* g);

/* ---- AMR transfer operators ----
 * volume/faceUnknownsProlongation and ...Restriction
 * (kernels/aderdg/generic/c/{2d,3d}/amrRoutines.cpph, declared in
 * kernels/aderdg/generic/Kernels.h:169-205) for `count` items on the device:
 * item i moves nodal data of k node dimensions (k = dim for cell volumes
 * luh, dim-1 for face arrays lQhbnd / lFhbnd), [node][var] with nvar values
 * per node, between a coarse cell (face) and its descendant level_delta
 * levels down (3:1 refinement per level); index[3 i + d] in
 * [0, 3^level_delta) is the descendant's position along direction d (the
 * reference's subcellIndex / subfaceIndex).
 * prolongation: fine[i] = P(coarse[coarse_item ? coarse_item[i] : i]);
 * restriction:  coarse[i] += R(fine[i]) (the reference adds each child's
 * contribution into the parent; outputs of different items must not
 * alias).  Orders 1..6; arrays of B^k nvar doubles per item, back to back. */
exa_status_t exa_aderdg_amr_prolongation(int k, int order, int nvar, long count, double* fine,
                                         const double* coarse, const long* coarse_item, int level_delta,
                                         const int* index, void* stream);
exa_status_t exa_aderdg_amr_restriction(int k, int order, int nvar, long count, double* coarse,
                                        const double* fine, int level_delta, const int* index, void* stream);

/* ---- A-posteriori subcell limiter ----
 * kernels/limiter/generic/c/Limiter.cpp (declared in
 * kernels/limiter/generic/Limiter.h:41-130) for `ncells` cells on the
 * device.  Per cell: luh [z][y][x][nvar] with B = order+1 points per
 * direction; lim [z][y][x][nvar] with S + 2 g points per direction, S =
 * 2 order + 1 subcells and g = ghost_layer_width (the FV solver's ghost
 * layer, 1 Godunov / 2 MUSCL-Hancock); the projections touch only the
 * interior of lim.  Observables are the first nobs variables (the default
 * mapDiscreteMaximumPrincipleObservables of the generated solvers,
 * AbstractGenericADERDGSolverHeader.template:159-163); obs_min / obs_max
 * hold [2 dim][nobs] per cell (ADERDGCellDescription solutionMin /
 * solutionMax).  Orders 1..6, nvar 1..64. */

/* projectOnFVLimiterSpace (Limiter.cpp:23-64): lim interior = subcell
 * means of the DG polynomial (uh2lim of LimiterProjectionMatrices.cpp). */
exa_status_t exa_limiter_project_on_fv(int dim, int order, int nvar, int ghost_layer_width, long ncells,
                                       const double* luh, double* lim, void* stream);
/* projectOnDGSpace (Limiter.cpp:67-110): conservative least-squares
 * reconstruction of the nodal values from the subcell means (lim2uh). */
exa_status_t exa_limiter_project_on_dg(int dim, int order, int nvar, int ghost_layer_width, long ncells,
                                       const double* lim, double* luh, void* stream);
/* findCellLocalMinAndMax (Limiter.cpp:212-251): extrema of the observables
 * over the nodes, the Gauss-Lobatto points and the subcell means, written
 * to every face block (LimitingADERDGSolver::determineSolverMinAndMax,
 * LimitingADERDGSolver.cpp:1080-1116). */
exa_status_t exa_limiter_local_min_max(int dim, int order, int nvar, int nobs, long ncells, const double* luh,
                                       double* obs_min, double* obs_max, void* stream);
/* findCellLocalLimiterMinAndMax (Limiter.cpp:170-207) over the interior of
 * lim, written to every face block (determineLimiterMinAndMax,
 * LimitingADERDGSolver.cpp:1118-1150). */
exa_status_t exa_limiter_fv_min_max(int dim, int order, int nvar, int nobs, int ghost_layer_width, long ncells,
                                    const double* lim, double* obs_min, double* obs_max, void* stream);
/* discreteMaximumPrincipleAndMinAndMaxSearch (Limiter.cpp:113-167): on
 * entry obs_min/obs_max hold the bounds merged from the neighbours per
 * face; dmp_ok[cell] = 1 if every observable of the new solution stays
 * within [min - d, max + d], d = max(relaxation, difference_scaling (max -
 * min)); face block 0 receives the new cell extrema, face block 1 the
 * merged bounds (as in the reference).  nobs >= 1. */
exa_status_t exa_limiter_dmp(int dim, int order, int nvar, int nobs, long ncells, const double* luh,
                             double relaxation, double difference_scaling, double* obs_min, double* obs_max,
                             int* dmp_ok, void* stream);

/* ---- Limiting ADER-DG on the uniform grid ----
 * exahype::solvers::LimitingADERDGSolver (exahype/solvers/
 * LimitingADERDGSolver.cpp) on an exa_aderdg_grid (2D or 3D): each step the
 * unlimited DG candidate is checked by the DMP (bounds: the cell's and its
 * face neighbours' extrema of the previous step) and, if enabled, by
 * physical admissibility (positive density and pressure at every node);
 * failing cells become Troubled, their status spreads over four face hops
 * (NeighbourOfTroubled1..4), the cells Troubled .. NeighbourOfTroubled2
 * recompute the step with the FV scheme on 2N+1 subcells per direction
 * started from the previous solution (ghost subcells from the neighbour
 * cells' projected previous solutions, NeighbourOfTroubled3 included) and
 * project the result back (LimitingADERDGSolver::recomputeSolution,
 * :1378-1441); the next bounds and the next dt come from the final state.
 * With exa_aderdg_grid_set_boundary's rules, a domain-boundary face adds no
 * neighbour status (mergeWithBoundaryOrEmptyCellMetadata sets the facewise
 * status 0) and keeps the cell's own extrema, and a subcell patch's ghost
 * layers there mirror its boundary layers, ghost k <- interior g - 1 - k
 * from the face, the normal momentum negated for EXA_BC_REFLECT
 * (FiniteVolumesSolver::mergeWithBoundaryData, finitevolumes/commons/c/
 * commons.cpph:175-340).
 * Parameters as in the reference's solver specification. */
typedef struct {
  int scheme;                /* subcell FV scheme: 0 Godunov, 1 MUSCL-Hancock */
  int nobs;                  /* dmp-observables: the first nobs variables, 1..5 */
  double relaxation;         /* dmp-relaxation-parameter (delta_0) */
  double difference_scaling; /* dmp-difference-scaling (epsilon) */
  int steps_till_cured;      /* steps-till-cured */
  int check_admissibility;   /* 1: density and pressure > 0 at every node */
} exa_limiter_config_t;

/* Enables (cfg != NULL) or disables the limiter of a grid.  Needs no slab
 * halos (3D MUSCL-Hancock subcells: order <= 5);
 * allocates the limiter state (previous solution, one subcell patch per
 * cell, bounds, statuses) and sets every cell Ok with bounds from the
 * current state (also after init/set_state). */
exa_status_t exa_aderdg_grid_set_limiter(exa_aderdg_grid* g, const exa_limiter_config_t* cfg);
/* status per cell (nullable host array of ncells ints, LimiterStatus values
 * Ok 0 .. Troubled 5) and counts[3] (nullable): cells with a subcell patch,
 * FV-updated cells, Troubled cells, of the last step */
exa_status_t exa_aderdg_grid_limiter_status(exa_aderdg_grid* g, int* host_status, int* counts);
/* the DMP bounds for the next step, [cell][2 dim faces][nobs] each */
exa_status_t exa_aderdg_grid_limiter_bounds(exa_aderdg_grid* g, double* host_min, double* host_max);

/* Per-cell drop-ins with the reference's argument lists (HOST pointers,
 * synchronous; the limiter kernels take the dimension from the build, here
 * it is an argument). */
exa_status_t exa_limiter_projectOnFVLimiterSpace(int dim, const double* luh, int numberOfVariables,
                                                 int basisSize, int ghostLayerWidth, double* lim);
exa_status_t exa_limiter_projectOnDGSpace(int dim, const double* lim, int numberOfVariables, int basisSize,
                                          int ghostLayerWidth, double* luh);
exa_status_t exa_limiter_findCellLocalMinAndMax(int dim, const double* luh, int numberOfVariables,
                                                int basisSize, int numberOfObservables,
                                                double* localMinPerObservable, double* localMaxPerObservable);
exa_status_t exa_limiter_discreteMaximumPrincipleAndMinAndMaxSearch(
    int dim, const double* luh, int numberOfVariables, int basisSize, int numberOfObservables,
    double relaxationParameter, double differenceScaling, double* boundaryMinPerObservable,
    double* boundaryMaxPerObservable, int* discreteMaximumPrincipleSatisfied);

/* ---- Slab decomposition of one grid over several GPUs ----
 * The reference distributes its spacetree over MPI ranks inside Peano: per
 * remote face, ADERDGSolver::sendDataToNeighbour (exahype/solvers/
 * ADERDGSolver.cpp:3379) sends that face's lQhbnd and lFhbnd, and the
 * receiving rank's mergeWithNeighbourData (:3451) solves the Riemann problem
 * with the received data (:3521, solveRiemannProblemAtInterface :3539), so
 * both ranks solve every boundary face.  Here a periodic grid is
 * cut into slabs along its last dimension (z in 3D, y in 2D), one slab per
 * GPU; each slab is an exa_aderdg_grid of the slab's size with halos on.
 * Per step the host (any transport: NCCL, a peer copy, a local copy)
 *   1. exa_aderdg_grid_phase(PREDICT): predictor; the slab's boundary faces
 *      are packed into send_lo (lower end) and send_hi (upper end);
 *   2. moves send_hi of slab r into recv_lo of slab r+1 and send_lo of slab
 *      r into recv_hi of slab r-1 (periodic in r);
 *   3. exa_aderdg_grid_phase(CORRECT): Riemann / surface integral / update,
 *      faces across the slab ends taken from recv_lo / recv_hi; the slab's
 *      minimum next dt lands in the dt slot (uint64 bit pattern of a
 *      positive double, so an unsigned or signed integer MIN reduction over
 *      slabs gives the global minimum);
 *   4. reduces the dt slot with MIN over slabs, then phase(COMMIT).
 * Before the first step: phase(PRIME_LOCAL), MIN reduction of the slot,
 * phase(PRIME_COMMIT).  All phases are stream-ordered on the grid's stream.
 * The result equals the undivided periodic grid's bit for bit (both sides of
 * a slab-boundary face solve the same Riemann problem from the same data). */
enum {
  EXA_PHASE_PREDICT = 0,
  EXA_PHASE_CORRECT = 1,
  EXA_PHASE_COMMIT = 2,
  EXA_PHASE_PRIME_LOCAL = 3,
  EXA_PHASE_PRIME_COMMIT = 4
};
exa_status_t exa_aderdg_grid_set_halo(exa_aderdg_grid* g, int enable);
/* device buffers of `count` doubles each, [layer cell][Q | F][face node][var] */
exa_status_t exa_aderdg_grid_halo_buffers(exa_aderdg_grid* g, double** send_lo, double** send_hi,
                                          double** recv_lo, double** recv_hi, size_t* count);
exa_status_t exa_aderdg_grid_dt_slot(exa_aderdg_grid* g, uint64_t** slot);
exa_status_t exa_aderdg_grid_phase(exa_aderdg_grid* g, int phase);
/* initial condition of slab `rank` of `nranks` (coordinates and noise of
 * the whole domain; the grid's n and length are the slab's) */
exa_status_t exa_aderdg_grid_init_slab(exa_aderdg_grid* g, int kind, double param, uint64_t seed,
                                       double noise_amp, int rank, int nranks);

/* Slab transport over NCCL inside the library (replaces the reference's MPI
 * face exchange, ADERDGSolver::sendDataToNeighbour / mergeWithNeighbourData,
 * ADERDGSolver.cpp:3379 and :3451, and the global dt minimum of
 * TimeStepSizeComputation.cpp:83-109).  One communicator per process (rank
 * r holds slab r of nranks along the last dimension, on the current device):
 * rank 0 makes the 128-byte id with exa_nccl_unique_id, every rank passes
 * it to exa_slab_comm_create.  exa_aderdg_grid_slab_step enqueues nsteps
 * whole steps on the grid's stream (predict, NCCL send/recv of the two
 * boundary face layers, correct, NCCL MIN all-reduce of the dt slot,
 * commit) and waits for them; if they have not finished after timeout_s
 * seconds per step (<= 0: 60 s) the communicator is aborted and
 * EXA_ETIMEDOUT returned.  With nranks == 1 the face layers are copied on
 * the stream.  NCCL is opened at run time (libnccl.so.2); without it these
 * calls return EXA_ECUDA with the reason. */
typedef struct exa_slab_comm exa_slab_comm;
exa_status_t exa_nccl_unique_id(void* id128);
exa_status_t exa_slab_comm_create(const void* id128, int nranks, int rank, exa_slab_comm** out);
exa_status_t exa_slab_comm_destroy(exa_slab_comm* c);
exa_status_t exa_aderdg_grid_slab_prime(exa_aderdg_grid* g, exa_slab_comm* c, double timeout_s);
exa_status_t exa_aderdg_grid_slab_step(exa_aderdg_grid* g, exa_slab_comm* c, int nsteps, double timeout_s);

/* ------------------------------------ ADER-DG: ensemble of 2D solves --
 * Many independent uniform periodic 2D grids (each its own order 2..5, size,
 * dt and step budget -- the per-solver state of ADERDGSolver.cpp:557-585)
 * advanced together by ONE cooperative persistent kernel per step: CTAs take
 * work items (a block of cells of one solve) from an atomic counter through
 * the predictor phase, a grid-wide barrier, the corrector phase, a barrier,
 * and a per-solve commit.  Device memory comes from an arena allocated at
 * creation; adding a solve fails with EXA_EBUSY when its footprint does not
 * fit (admission by footprint). */
typedef struct exa_ensemble exa_ensemble;

typedef struct {
  int order;          /* 2..5 */
  int n[2];           /* cells */
  double length[2];   /* domain extent */
  int pde;            /* exa_pde_t */
  int dt_policy;      /* as exa_aderdg_grid_config_t */
  double cfl, dt_fixed;
  int ic_kind;        /* 0 isentropic vortex, 1 density sine wave */
  double ic_param;    /* vortex strength / sine amplitude */
  uint64_t seed;
  double noise;       /* relative density noise amplitude */
} exa_solve_config_t;

size_t exa_ensemble_footprint(const exa_solve_config_t* cfg);
exa_status_t exa_ensemble_create(int precision, int max_solves, size_t arena_bytes,
                                 exa_ensemble** out);
exa_status_t exa_ensemble_destroy(exa_ensemble* e);
/* steps: step budget (< 0 unlimited); the solve stops after it */
exa_status_t exa_ensemble_add(exa_ensemble* e, const exa_solve_config_t* cfg, long long steps,
                              int* slot);
exa_status_t exa_ensemble_remove(exa_ensemble* e, int slot);
exa_status_t exa_ensemble_step(exa_ensemble* e, int nsteps);
exa_status_t exa_ensemble_use_graph(exa_ensemble* e, int enable);
/* schedule knobs: persistent CTAs per SM (0 = max resident), work items per
 * atomic grab, work order (0 = costly orders first, 1 = solve order) */
exa_status_t exa_ensemble_tune(exa_ensemble* e, int ctas_per_sm, int grab, int order_policy);
/* contraction of each order's predictor inside the persistent launch: bit N
 * of lines_mask set = line-owner contraction, clear = node-gather (default:
 * orders 4 and 5 line-owner); results agree to rounding */
exa_status_t exa_ensemble_tune_contraction(exa_ensemble* e, int lines_mask);
/* launch form of a step: 0 (default) one persistent cooperative launch
 * (work items taken from an atomic counter, grid barriers between the
 * phases); 1 one launch per order and phase (each with that order's own
 * shared memory and occupancy) and a commit launch, the same arithmetic */
exa_status_t exa_ensemble_set_launch_mode(exa_ensemble* e, int mode);
exa_status_t exa_ensemble_synchronize(exa_ensemble* e);
exa_status_t exa_ensemble_stream(exa_ensemble* e, void** stream);
exa_status_t exa_ensemble_get_state(exa_ensemble* e, int slot, double* host_luh);
/* Checkpoint of one solve: its state (host_luh, as exa_ensemble_get_state)
 * and its time-step scalars.  exa_ensemble_restore adds a solve of the same
 * configuration from a checkpoint (EXA_EBUSY when it does not fit now); it
 * then continues bit for bit as the checkpointed solve would have. */
typedef struct {
  double time;            /* simulated time */
  double dt;              /* dt of the next step */
  uint64_t dt_next_bits;  /* the next-dt reduction slot (bit pattern) */
  uint64_t steps_done;
  int64_t steps_left;     /* < 0: unlimited */
  uint64_t picard, nonconverged;
  int active, nan_flag;
} exa_solve_checkpoint_t;
exa_status_t exa_ensemble_checkpoint(exa_ensemble* e, int slot, double* host_luh, exa_solve_checkpoint_t* ck);
exa_status_t exa_ensemble_restore(exa_ensemble* e, const exa_solve_config_t* cfg, const double* host_luh,
                                  const exa_solve_checkpoint_t* ck, int* slot);
exa_status_t exa_ensemble_device_state(exa_ensemble* e, int slot, double** luh_dev);
exa_status_t exa_ensemble_status(exa_ensemble* e, double* time, uint64_t* steps_done, int* active,
                                 uint64_t* picard, int* nan_flag);
long exa_ensemble_active_cells(exa_ensemble* e);
exa_status_t exa_ensemble_info(exa_ensemble* e, int* grid_ctas, int* nitems,
                               size_t* arena_free_bytes);

/* -------------------------------------------------------- serving --
 * Continuous batching of solve requests: admission by device-memory
 * footprint (EXA_EBUSY when a request does not fit now), state resident on
 * the device until the result is collected, every tick advances every
 * active request (ADER-DG requests one step, in the ensemble's launches; FV
 * patches up to exa_server_set_fv_steps steps, on a second stream that
 * overlaps them). */
typedef struct exa_server exa_server;

#define EXA_REQ_ADERDG 0
#define EXA_REQ_FV 1

typedef struct {
  int kind;               /* EXA_REQ_ADERDG or EXA_REQ_FV */
  exa_solve_config_t dg;  /* ADER-DG solve; for FV: pde, ic_param, seed, noise */
  int fv_scheme;          /* 0 Godunov, 1 MUSCL-Hancock */
  int fv_patch;           /* cells per side */
  double fv_length;       /* domain extent */
  long long steps;        /* step budget (>= 1) */
} exa_request_t;

size_t exa_server_footprint(const exa_request_t* r);
exa_status_t exa_server_create(size_t hbm_budget, int max_requests, int precision, exa_server** out);
exa_status_t exa_server_destroy(exa_server* s);
exa_status_t exa_server_submit(exa_server* s, const exa_request_t* r, uint64_t* id);
exa_status_t exa_server_tick(exa_server* s, int* ncompleted);
exa_status_t exa_server_completed(exa_server* s, uint64_t* ids, int cap, int* n);
size_t exa_server_result_size(exa_server* s, uint64_t id);
/* copies the final state (ADER-DG: [cell][y][x][var]; FV: the patch incl.
 * ghosts, [y][x][var]) and releases the request's device memory */
exa_status_t exa_server_result(exa_server* s, uint64_t id, double* host_out, double* sim_time,
                               long long* steps_done);
exa_status_t exa_server_info(exa_server* s, int* live_requests, long* active_dg_cells,
                             size_t* arena_free_bytes);
/* how the ADER-DG requests of a tick are launched: the ensemble's launch
 * form (exa_ensemble_set_launch_mode) and whether a tick's launches replay
 * a CUDA graph (re-captured whenever the set of requests changes; default
 * 1 and 1: one launch per order and phase, graph replay) */
exa_status_t exa_server_tune(exa_server* s, int launch_mode, int use_graph);
/* FV requests advance `steps` steps per tick (default 3), on the FV
 * stream that overlaps the ADER-DG launch, whose step is the longer one.  A
 * request never takes more steps than its budget, and its result is the
 * same whatever the setting. */
exa_status_t exa_server_set_fv_steps(exa_server* s, int steps);
/* device pointer of a live request's current state (ADER-DG: the solve's
 * luh; FV: the patch buffer that holds the state), for zero-copy inspection
 * between ticks */
exa_status_t exa_server_device_state(exa_server* s, uint64_t id, double** luh_dev);
/* Eviction: a running request's state and time-step scalars move to host
 * memory and its device memory returns to the arena; ticks skip it until
 * exa_server_restore re-admits it (EXA_EBUSY while it does not fit), after
 * which it continues bit for bit as if never evicted.  exa_server_evicted
 * reports the state. */
exa_status_t exa_server_evict(exa_server* s, uint64_t id);
exa_status_t exa_server_restore(exa_server* s, uint64_t id);
exa_status_t exa_server_evicted(exa_server* s, uint64_t id, int* evicted);
/* Preemption in exa_server_run: when the oldest waiting request has waited
 * longer than wait_s and does not fit, running requests that have been
 * resident for at least wait_s are evicted, largest footprint first, until
 * it fits; evicted requests are restored, before new admissions, as soon as
 * they fit.  wait_s <= 0 (the default): no preemption. */
exa_status_t exa_server_set_eviction(exa_server* s, double wait_s);
/* How exa_server_run hands out finished results: 1 (the default) each
 * finished state is copied into pinned staging memory on its own stream
 * while the next tick runs, and handed out (copied into results[i], device
 * memory released) once that copy has completed; 0 each is copied
 * synchronously right after its tick, the GPU idle meanwhile.  Results are
 * the same either way. */
exa_status_t exa_server_set_result_mode(exa_server* s, int mode);
/* capacity of that pinned staging ring in bytes (default 256 MiB, at least
 * 4096; allocated at the first run that needs it and grown to the largest
 * single result); results wait for older ones to be handed out while the
 * ring is full.  Call between runs. */
exa_status_t exa_server_set_staging(exa_server* s, size_t bytes);
/* host seconds of the last exa_server_run: [0] launching ticks, [1] waiting
 * for them, [2] handing out results, [3] arrivals, admission and eviction */
exa_status_t exa_server_loop_times(exa_server* s, double* seconds4);

/* One request of a stream run by exa_server_run (times in seconds after the
 * start of the run). */
typedef struct {
  double arrival_s;      /* in: when the request arrives */
  double admitted_s;     /* out: when it was admitted (-1: never) */
  double completed_s;    /* out: when its result was on the host (-1: not completed) */
  double sim_time;       /* out: simulated time reached */
  long long steps_done;  /* out */
  int status;            /* out: EXA_OK; EXA_ENAN for a solve that produced a non-finite state
                            (stopped there, its state returned, the others unaffected); -1 not completed */
  int evictions;         /* out: how often it was evicted to host memory (exa_server_set_eviction) */
} exa_request_record_t;

/* The serving loop, from this host thread: requests arrive at their
 * arrival_s; arrived requests are admitted first-fit in arrival order as
 * memory and slots free up; every tick advances every admitted request
 * (continuous batching, exa_server_tick); finished results are copied
 * out (into results[i] when results and results[i] are non-NULL) and their
 * memory freed.  Returns when every request has completed or after
 * time_limit_s seconds (<= 0: no limit); ticks (nullable) receives the tick
 * count.  No counterpart in the reference (its requests are whole runs of
 * the executable); the solves are the reference's step as in the ensemble. */
exa_status_t exa_server_run(exa_server* s, const exa_request_t* reqs, exa_request_record_t* rec, int n,
                            double time_limit_s, double* const* results, uint64_t* ticks);

/* ------------------------------------------------ finite volumes (2D) --
 * One patch of patch x patch cells with `ghost` ghost layers, layout
 * [y][x][nData] over (patch+2*ghost)^2 cells (reference FV solvers,
 * PatchSize / GhostLayerWidth, AbstractGenericFiniteVolumesSolverHeader.
 * template:30-34).  Batched over `npatches` patches back to back. */
typedef struct {
  int dim;      /* 2, or 3 (EXA_PDE_EULER; a patch with its ghosts in 200 KB: patch <= 15 Godunov, <= 11 MUSCL-Hancock) */
  int patch;    /* PatchSize */
  int ghost;    /* 1 for Godunov, 2 for MUSCL-Hancock */
  int nvar, npar, pde;
  double dx[3]; /* patch extent (cell size = dx/patch) */
} exa_fv_desc_t;

/* godunov::c::solutionUpdate (kernels/finitevolumes/godunov/c/2d/
 * godunov.cpph:33-120; 3D: godunov/c/3d/godunov.cpph:35-143, with
 * musclhancock/c/3d/musclhancock.cpph:50-311 and commons.cpph:410-455 for
 * the two below): luh_new (a copy of luh on entry) is advanced in
 * place; max_dt (nullable, device, one double per patch) receives the
 * admissible dt.  Rusanov faces (riemannsolvers/c/rusanov.cpph:24-83). */
exa_status_t exa_fv_godunov_update(const exa_fv_desc_t* desc, long npatches,
                                   double* luh_new, const double* luh,
                                   double dt, double* max_dt, void* stream);
/* musclhancock::c::solutionUpdate (kernels/finitevolumes/musclhancock/c/
 * 2d/musclhancock.cpph:50-240), CFL 0.99 for max_dt. */
exa_status_t exa_fv_musclhancock_update(const exa_fv_desc_t* desc, long npatches,
                                        double* luh_new, const double* luh,
                                        double dt, double* max_dt, void* stream);
/* commons::c::stableTimeStepSize (commons/c/commons.cpph:26-67), per patch */
exa_status_t exa_fv_stable_dt(const exa_fv_desc_t* desc, long npatches,
                              const double* luh, double* dt_patch, void* stream);
/* fills the ghost layers of every patch periodically from itself */
exa_status_t exa_fv_periodic_ghosts(const exa_fv_desc_t* desc, long npatches,
                                    double* luh, void* stream);
/* ---- Device-resident periodic FV domain ----
 * One periodic 2D patch of patch x patch cells (plus the scheme's ghost
 * width: 1 Godunov, 2 MUSCL-Hancock) over [0,length)^2, stepped on the
 * device with the reference's per-step semantics: dt = the
 * commons::stableTimeStepSize rule (commons.cpph:26-67) on the current
 * state, then godunov/musclhancock::solutionUpdate (godunov.cpph:33-120,
 * musclhancock.cpph:50-240) with periodic ghost values.  Two launches per
 * step: a fused update that loads tiles straight from the periodic interior
 * and also reduces the next dt, and a one-thread commit.  State layout
 * [y][x][var] with ghosts; ghost cells of a stepped state are not
 * meaningful.  Initial condition: rho = 1 + amp sin(2 pi (x+y)), u = v = 1,
 * p = 1, with seeded relative density noise. */
typedef struct exa_fv_grid exa_fv_grid;
exa_status_t exa_fv_grid_create(int scheme, int patch, double length, int pde, exa_fv_grid** out);
exa_status_t exa_fv_grid_destroy(exa_fv_grid* g);
size_t exa_fv_grid_state_size(const exa_fv_grid* g);
exa_status_t exa_fv_grid_init(exa_fv_grid* g, double amp, uint64_t seed, double noise);
exa_status_t exa_fv_grid_set_state(exa_fv_grid* g, const double* host);
exa_status_t exa_fv_grid_get_state(exa_fv_grid* g, double* host);
exa_status_t exa_fv_grid_step(exa_fv_grid* g, int nsteps);
/* simulated time and the dt the next step will take */
exa_status_t exa_fv_grid_status(exa_fv_grid* g, double* time, double* dt_next);
exa_status_t exa_fv_grid_stream(exa_fv_grid* g, void** stream);
exa_status_t exa_fv_grid_device_state(exa_fv_grid* g, double** luh_dev);

/* ---- Device-resident grid of FV patches (the reference's FV layout) ----
 * npx x npy patches (periodic, or with exa_fv_patchgrid_set_boundary's
 * rules) of patch x patch subcells (+ ghost layers: 1
 * Godunov, 2 MUSCL-Hancock) over [0,length)^2, stored back to back (x
 * fastest) like the batched FV entry points.  One step: face ghost layers
 * copied from the neighbouring patches' boundary layers (ghostLayerFilling,
 * kernels/finitevolumes/commons/c/commons.cpph:337-405, per face as in
 * FiniteVolumesSolver::mergeNeighbours, FiniteVolumesSolver.cpp:659-686),
 * dt = the CFL rule minimised over every patch, then each patch's
 * godunov/musclhancock::solutionUpdate with that dt (the reference's
 * in-place semantics: luh_new = luh, then updated).  The patches do not
 * reproduce one big patch exactly: MUSCL-Hancock does not half-step-evolve
 * ghost cells, so faces between patches see unevolved neighbour states, as
 * in the reference.  Initial condition as exa_fv_grid_init, on the whole
 * domain. */
typedef struct exa_fv_patchgrid exa_fv_patchgrid;
exa_status_t exa_fv_patchgrid_create(int scheme, int patch, int npx, int npy, double length, int pde,
                                     exa_fv_patchgrid** out);
exa_status_t exa_fv_patchgrid_destroy(exa_fv_patchgrid* g);
size_t exa_fv_patchgrid_state_size(const exa_fv_patchgrid* g);
exa_status_t exa_fv_patchgrid_init(exa_fv_patchgrid* g, double amp, uint64_t seed, double noise);
exa_status_t exa_fv_patchgrid_set_state(exa_fv_patchgrid* g, const double* host);
exa_status_t exa_fv_patchgrid_get_state(exa_fv_patchgrid* g, double* host);
exa_status_t exa_fv_patchgrid_step(exa_fv_patchgrid* g, int nsteps);
/* simulated time and the dt of the last step */
exa_status_t exa_fv_patchgrid_status(exa_fv_patchgrid* g, double* time, double* last_dt);
exa_status_t exa_fv_patchgrid_stream(exa_fv_patchgrid* g, void** stream);
/* Boundary rule per dimension (bc[2], EXA_BC_*) in place of the periodic
 * wrap: a domain-boundary patch fills that face's ghost layers from its own
 * boundary layers as FiniteVolumesSolver::mergeWithBoundaryData does
 * (FiniteVolumesSolver.cpp:689-727: boundaryLayerExtraction,
 * boundaryConditions with the mirrored index K = g - 1 - k through the
 * boundaryValues hook, ghostLayerFillingAtBoundary; commons.cpph:99-340):
 * ghost k from the face <- interior layer k from the face; EXA_BC_OUTFLOW
 * copies (the EulerFV demonstrator's boundaryValues), EXA_BC_REFLECT also
 * negates the normal momentum. */
exa_status_t exa_fv_patchgrid_set_boundary(exa_fv_patchgrid* g, const int* bc);

/* rusanov (riemannsolvers/c/rusanov.cpph:24-83), host drop-in, returns s_max */
exa_status_t exa_fv_rusanov(int dim, int nvar, int npar, int pde, double* fL,
                            double* fR, const double* qL, const double* qR,
                            int normalNonZero, double* s_max);

#ifdef __cplusplus
}
#endif
#endif /* EXA_KERNELS_H */
