/*
 * CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64 restatement of ExaHyPE's generic kernels for the
 * ADER-DG / finite-volume cell-update path, used by the test suite, the
 * smoke check and the CPU-baseline leg of the benchmark as the checker for
 * the CUDA library.  It is never linked into, loaded by or called from the
 * product library (libexahype_b200.so).
 *
 * Parity is pinned two ways: against the reference's golden vectors
 * (exahype/tests/kernels/testdata/generic_euler_testdata.cpp, extracted to
 * tests/golden/) and against the reference's own generic kernels compiled
 * from its sources into oracle/_ref (oracle/Makefile).
 *
 * All arrays use the reference's row-major layouts (ExaHyPE/kernels/
 * KernelUtils.h:243-320 idx2..idx6), slowest index first:
 *   luh     [z][y][x][nData]            (2D: [y][x][nData])
 *   lQi     [z][y][x][t][nData]
 *   lFi     [t][z][y][x][dim+1][nVar]
 *   lQhi    [z][y][x][nData]
 *   lFhi    (dim+1) blocks of B^dim*nVar: x [z][y][x], y [z][x][y],
 *           z [y][x][z], source [z][y][x]
 *   lQhbnd  [2*dim][B][B][nData],  lFhbnd [2*dim][B][B][nVar]
 *   lduh    [z][y][x][nVar]
 */
#ifndef EXA_ORACLE_H
#define EXA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* PDE selector: 0 = compressible Euler with all three momenta in the
 * pressure (ExaHyPE/exahype/tests/kernels/c/GenericEulerKernelTest3D.cpp:26-82,
 * Demonstrators/EulerFV/MyEulerSolver.cpp:58-98); 1 = the "2.5D" planar
 * variant whose pressure only uses the in-plane momenta
 * (GenericEulerKernelTest2D.cpp:28-79). */
void orc_euler_flux(int dim, int planar, const double* Q, double* F);
void orc_euler_eigenvalues(int planar, const double* Q, int d, double* lambda);

/* ---- ADER-DG, one cell, reference argument semantics ---- */
int orc_stp_nonlinear(int dim, int order, int nvar, int npar, int planar,
                      double* lQhbnd, double* lFhbnd,
                      double* lQi, double* lQi_old, double* rhs, double* lFi,
                      double* lQhi, double* lFhi,
                      const double* luh, const double* dx, double dt);
void orc_volume_integral(int dim, int order, int nvar, int use_source,
                         double* lduh, const double* lFhi, const double* dx);
void orc_surface_integral(int dim, int order, int nvar,
                          double* lduh, const double* lFhbnd, const double* dx);
void orc_riemann(int dim, int order, int nvar, int npar, int planar,
                 double* FL, double* FR, const double* QL, const double* QR,
                 int direction);
void orc_solution_update(int dim, int order, int nvar, int npar,
                         double* luh, const double* lduh, double dt);
double orc_stable_dt(int dim, int order, int nvar, int npar, int planar,
                     const double* luh, const double* dx, double cfl);

/* ---- ADER-DG uniform periodic grid (n[0] x n[1] (x n[2]) cells) ---- */
/* dt_policy: 0 = reference PNPM rule, 1 = CFL/(2N+1), 2 = fixed dt_fixed */
double orc_aderdg_grid_dt(int dim, int order, int planar, const int* n,
                          const double* dx, const double* luh, int dt_policy,
                          double cfl);
/* One full step in the reference's non-fused order.  luh is updated in
 * place; iters (optional, one int per cell) receives Picard iterations.
 * Returns the dt used. */
double orc_aderdg_grid_step(int dim, int order, int planar, const int* n,
                            const double* dx, double* luh, int dt_policy,
                            double cfl, double dt_fixed, int* iters,
                            int nthreads);
/* Slab of a periodic grid cut along its last dimension (n = the slab's
 * cells).  predict: predictor + volume integral of every cell into lduh,
 * face data into qb/fb ([cell][2 dim][face nodes][var]), and the slab's
 * boundary faces packed as [layer cell][Q | F][face nodes][var]: face
 * 2(dim-1) of the lowest layer into send_lo, face 2(dim-1)+1 of the highest
 * into send_hi.  correct: Riemann on every face (faces across the slab ends
 * against recv_lo / recv_hi, the adjacent slabs' packed faces), surface
 * integral and update of luh.  Same per-face arithmetic as
 * orc_aderdg_grid_step, so slabs reproduce the undivided grid exactly. */
void orc_aderdg_slab_predict(int dim, int order, int planar, const int* n,
                             const double* dx, const double* luh, double dt,
                             double* lduh, double* qb, double* fb,
                             double* send_lo, double* send_hi);
void orc_aderdg_slab_correct(int dim, int order, int planar, const int* n,
                             const double* dx, double* luh, double* lduh,
                             double* qb, double* fb, const double* recv_lo,
                             const double* recv_hi, double dt);
/* As orc_aderdg_grid_step with a boundary rule per dimension (NULL or 0 =
 * periodic, 1 = outflow, 2 = reflecting wall; see orc_boundary_values). */
double orc_aderdg_grid_step_bc(int dim, int order, int planar, const int* n,
                               const double* dx, double* luh, int dt_policy,
                               double cfl, double dt_fixed, int* iters,
                               int nthreads, const int* bc);
/* CPU-baseline sample: one step's per-cell work on ncells independent
 * cells (each its own periodic neighbour). */
void orc_aderdg_sample_step(int dim, int order, int planar, long ncells,
                            const double* dx, double* luh, double dt,
                            int nthreads);
/* Nodal initial condition on the grid: isentropic vortex / sine wave with
 * seeded density noise.  kind: 0 = isentropic vortex (u=v=1 background,
 * strength eps), 1 = density sine rho=1+amp*sin(2 pi (x+y)), u=v=1, p=1. */
void orc_aderdg_grid_ic(int dim, int order, const int* n, const double* dx,
                        double* luh, int kind, double param,
                        unsigned long long seed, double noise_amp);

/* ---- finite volumes, 2D patch (reference godunov / musclhancock) ---- */
/* PDE callbacks of orc_rusanov_pde: F is [dim][nvar], lam is [nvar] */
typedef void (*orc_flux_fn)(void* ctx, const double* q, double* F);
typedef void (*orc_eig_fn)(void* ctx, const double* q, int d, double* lam);
double orc_rusanov_pde(int dim, int nvar, orc_flux_fn flux, orc_eig_fn eig, void* ctx,
                       double* fL, double* fR, const double* qL, const double* qR, int d);
double orc_rusanov(int dim, int nvar, int npar, int planar, double* fL,
                   double* fR, const double* qL, const double* qR, int d);
double orc_fv_godunov_2d(int patch, int ghost, int nvar, int npar, int planar,
                         double* luh_new, const double* luh, const double* dx,
                         double dt);
double orc_fv_musclhancock_2d(int patch, int ghost, int nvar, int npar,
                              int planar, double* luh_new, const double* luh,
                              const double* dx, double dt);
double orc_fv_stable_dt_2d(int patch, int ghost, int nvar, int npar,
                           int planar, const double* luh, const double* dx,
                           double cfl);
void orc_fv_periodic_ghosts_2d(int patch, int ghost, int ndata, double* luh);
/* scheme: 0 godunov (ghost 1), 1 musclhancock (ghost 2).  Fills the
 * periodic ghosts, takes dt from the stable-dt rule (CFL 0.9) unless
 * dt_fixed > 0, updates luh in place; returns dt. */
double orc_fv_patch_step_2d(int scheme, int patch, int planar, double* luh,
                            const double* dx, double dt_fixed,
                            double* max_admissible_dt);

/* AMR transfer between a coarse cell (or face) and its fine descendant
 * `level_delta` levels down (3:1 per level), for k-dimensional nodal arrays
 * [node][var] (k = dim for cell volumes, dim-1 for faces); index[d] in
 * [0, 3^level_delta) = the descendant's position in direction d.
 * Prolongation overwrites `fine`; restriction ADDS the fine contribution
 * to `coarse` (the reference accumulates the 3^(k level_delta) children).
 * volume/faceUnknownsProlongation / ...Restriction, amrRoutines.cpph. */
void orc_amr_prolongation(int k, int order, int nvar, double* fine, const double* coarse,
                          int level_delta, const int* index);
void orc_amr_restriction(int k, int order, int nvar, double* coarse, const double* fine,
                         int level_delta, const int* index);
/* 3D counterparts on one patch of P^3 cells + g ghost layers ([z][y][x][D],
 * D = nvar + npar), the 3D Euler PDE (godunov/c/3d/godunov.cpph:35-143,
 * musclhancock/c/3d/musclhancock.cpph:50-311, commons.cpph:410-455). */
double orc_fv_godunov_3d(int patch, int ghost, int nvar, int npar, double* luh_new, const double* luh,
                         const double* dx, double dt);
double orc_fv_musclhancock_3d(int patch, int ghost, int nvar, int npar, double* luh_new, const double* luh,
                              const double* dx, double dt);
double orc_fv_stable_dt_3d(int patch, int ghost, int nvar, int npar, const double* luh, const double* dx,
                           double cfl);
void orc_fv_periodic_ghosts_3d(int patch, int ghost, int ndata, double* luh);
/* one step of a periodic npx x npy grid of FV patches (dx = patch extent) */
double orc_fv_patchgrid_step_2d(int scheme, int P, int npx, int npy, int planar,
                                double* luh, const double* dx);
/* the same with a boundary rule per dimension (bc[2], nullable: periodic):
 * domain-boundary faces filled by orc_fv_boundary_ghosts */
double orc_fv_patchgrid_step_2d_bc(int scheme, int P, int npx, int npy, int planar, double* luh, const double* dx,
                                   const int* bc);

/* A-posteriori subcell limiter, kernels/limiter/generic/c/Limiter.cpp, for
 * one cell of order N (B = N+1 nodes, S = 2N+1 subcells per direction):
 *   luh  [z][y][x][nvar] (B^dim points),
 *   lim  [z][y][x][nvar] ((S+2g)^dim points, g = ghost layer width; the
 *        projections read / write the interior only).
 * Observables are the first nobs variables (the generated solvers' default
 * mapDiscreteMaximumPrincipleObservables,
 * AbstractGenericADERDGSolverHeader.template:159-163).  Min/max arrays are
 * [2 dim][nobs] per cell (face-major, as ADERDGCellDescription's
 * solutionMin/solutionMax). */
void orc_limiter_project_on_fv(int dim, int order, int nvar, int ghost, const double* luh,
                               double* lim);
void orc_limiter_project_on_dg(int dim, int order, int nvar, int ghost, const double* lim,
                               double* luh);
/* findCellLocalMinAndMax (nodes, Gauss-Lobatto points, subcell means) into
 * face 0, copied to every face (LimitingADERDGSolver::determineSolverMinAndMax) */
void orc_limiter_local_min_max(int dim, int order, int nvar, int nobs, const double* luh,
                               double* obs_min, double* obs_max);
/* findCellLocalLimiterMinAndMax, copied to every face
 * (LimitingADERDGSolver::determineLimiterMinAndMax) */
void orc_limiter_fv_min_max(int dim, int order, int nvar, int nobs, int ghost,
                            const double* lim, double* obs_min, double* obs_max);
/* discreteMaximumPrincipleAndMinAndMaxSearch; returns 1 if satisfied */
int orc_limiter_dmp(int dim, int order, int nvar, int nobs, const double* luh, double relaxation,
                    double difference_scaling, double* obs_min, double* obs_max);

/* One step of the limiting ADER-DG grid (2D or 3D, n[0] x n[1]
 * (x n[2]) cells, order N, 5 variables), a restatement of
 * LimitingADERDGSolver's step on a uniform mesh: DG candidate with dt; DMP
 * against bmin/bmax ([cell][2 dim][nobs], updated in place to the next
 * step's bounds) and, if `admissibility`, positive density and pressure at
 * every node; statuses (status / cure per cell, in/out; Ok 0 .. Troubled 5)
 * with four hops of spreading; subcell FV recomputation (scheme 0 Godunov,
 * 1 MUSCL-Hancock) from the previous solution for status >= 3, ghost
 * subcells from the neighbours' projected previous solutions (status >= 2);
 * counts (nullable) = {cells with a patch, FV cells, Troubled cells}.
 * bc (nullable: periodic) = boundary rule per dimension (0 periodic,
 * 1 outflow, 2 reflecting wall) for the DG faces, the status spreading, the
 * bounds merge and the subcell ghost layers.
 * Returns the next dt (orc_aderdg_grid_dt with dt_policy / cfl on the final
 * state). */
double orc_limiting_grid_step(int dim, int order, const int* n, const double* dx, int planar, double* luh,
                              int* status, int* cure, double* bmin, double* bmax, int scheme, int nobs,
                              double relaxation, double difference_scaling, int steps_till_cured, int admissibility,
                              double dt, int dt_policy, double cfl, int* counts, const int* bc);
/* Ghost layers of one FV patch ([S]^dim x 5 values, S = P + 2 g, (z) y x
 * order) at a domain-boundary face 2 d + side: FiniteVolumesSolver::
 * mergeWithBoundaryData (FiniteVolumesSolver.cpp:689-727) extracts the g
 * layers next to the face (boundaryLayerExtraction), maps ghost k to the
 * extracted layer K = g - 1 - k through boundaryValues (boundaryConditions,
 * finitevolumes/commons/c/commons.cpph:175-265 and 726-875) and stores them
 * (ghostLayerFillingAtBoundary), so the ghost k layers from the face mirror
 * the interior k layers from the face (3D lower y and z faces: every ghost
 * layer repeats the layer next to the face, as the reference's extraction
 * there reads the first interior layer for every k).  rule 1 copies
 * (outflow), rule 2 negates the normal momentum (reflecting wall). */
void orc_fv_boundary_ghosts(int dim, int P, int g, double* luh, int face, int rule);
/* bounds of the first DMP check: local extrema merged over faces */
void orc_limiting_initial_bounds(int dim, int order, const int* n, const double* luh, int nobs, double* bmin,
                                 double* bmax, const int* bc);

/* solutionAdjustment of one cell with a built-in adjustPointSolution form
 * (kind 1 sine wave, 2 isentropic vortex, 3 heat source; when 0: only at
 * t == 0, 1: always), as exa_adjust_t of the device library. */
void orc_solution_adjustment(int dim, int order, double* luh, const double* center, const double* dx, double t,
                             double dt, int kind, int when, const double* param);

/* counter-based noise shared with the device IC kernel */
double orc_noise_u01(unsigned long long seed, unsigned long long idx);

#ifdef __cplusplus
}
#endif
#endif
