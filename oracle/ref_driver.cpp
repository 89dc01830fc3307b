/*
 * Harness around the reference's own generic kernels -- TEST
 * INFRASTRUCTURE ONLY.  Built by `make -C oracle ref` from the reference
 * sources in place (nothing is copied into this repository) into
 * oracle/_ref/libexa_ref{2d,3d}.so; used to pin the C oracle and as the
 * timed CPU baseline ("kind": "reference").
 *
 * The solver type below plays the role the reference's unit tests give the
 * test class itself (exahype/tests/kernels/c/GenericEulerKernelTest3D.cpp:
 * 26-132): it supplies the PDE callbacks and the compile-time constants the
 * kernel templates read.  The grid driver reproduces the non-fused step
 * order of exahype/runners/Runner.cpp:1125-1160 on a uniform periodic grid.
 */
#include <vector>
#include <set>
#include <thread>
#include <pthread.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "kernels/aderdg/generic/Kernels.h"
#include "kernels/finitevolumes/riemannsolvers/c/riemannsolvers.h"
#include "kernels/finitevolumes/commons/c/commons.h"
#include "kernels/finitevolumes/godunov/c/godunov.h"
#include "kernels/finitevolumes/musclhancock/c/musclhancock.h"
#include "kernels/GaussLegendreQuadrature.h"
#include "kernels/DGMatrices.h"
#include "kernels/GaussLobattoQuadrature.h"
#include "kernels/LimiterProjectionMatrices.h"
#include "kernels/limiter/generic/Limiter.h"
#include "exahype/solvers/ADERDGSolver.h"
#include "adjust_hooks.h"

namespace {

struct TablesInit {
  TablesInit() {
    std::set<int> orders;
    for (int i = 0; i < 10; i++) orders.insert(i);
    kernels::initGaussLegendreNodesAndWeights(orders);
    kernels::initDGMatrices(orders);
    kernels::initGaussLobattoNodesAndWeights(orders);
    kernels::initLimiterProjectionMatrices(orders);
  }
};
TablesInit tables_init;

constexpr double GAMMA_ = 1.4;

/* Euler PDE.  3D: all momenta in the pressure; 2D: the kernel tests'
 * planar form (GenericEulerKernelTest2D.cpp:28-79). */
inline double pressure(const double* Q, double irho) {
#if DIMENSIONS == 3
  return (GAMMA_ - 1) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) * irho);
#else
  return (GAMMA_ - 1) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) * irho);
#endif
}

template <int ORDER, int NPAR, int PATCH = 8, int GHOST = 1>
struct Euler {
  static constexpr int NumberOfVariables = 5;
  static constexpr int NumberOfParameters = NPAR;
  static constexpr int Order = ORDER;
  static constexpr int PatchSize = PATCH;
  static constexpr int GhostLayerWidth = GHOST;
  static constexpr double CFL = 0.9;

  void flux(const double* const Q, double** F) {
    const double irho = 1.0 / Q[0];
    const double p = pressure(Q, irho);
    for (int d = 0; d < DIMENSIONS; d++) {
      double* f = F[d];
      f[0] = Q[d + 1];
      f[1] = irho * Q[d + 1] * Q[1];
      f[2] = irho * Q[d + 1] * Q[2];
      f[3] = irho * Q[d + 1] * Q[3];
      f[d + 1] += p;
      f[4] = irho * Q[d + 1] * (Q[4] + p);
    }
  }
  void eigenvalues(const double* const Q, const int d, double* lambda) {
    const double irho = 1.0 / Q[0];
    const double p = pressure(Q, irho);
    const double un = Q[d + 1] * irho;
    const double c = std::sqrt(GAMMA_ * p * irho);
    lambda[0] = un - c; lambda[1] = un; lambda[2] = un; lambda[3] = un; lambda[4] = un + c;
  }
  void fusedSource(const double* const, const double* const, double* S) {
    for (int i = 0; i < 5; i++) S[i] = 0.0;
  }
  void algebraicSource(const double* const, double* S) {
    for (int i = 0; i < 5; i++) S[i] = 0.0;
  }
  void nonConservativeProduct(const double* const, const double* const, double* B) {
    for (int i = 0; i < 5; i++) B[i] = 0.0;
  }
  void coefficientMatrix(const double* const, const int, double* Bn) {
    for (int i = 0; i < 25; i++) Bn[i] = 0.0;
  }
  void pointSource(const double* const, const double* const, const double, const double, double*, int) {}
  /* ADER-DG boundary hook (ADERDGSolver::boundaryValues, called per face
   * node by boundaryConditions.cpph): rule 1 copies the inside state and
   * flux (outflow), rule 2 negates the normal momentum and takes the normal
   * flux of that reflected state (slip wall) */
  void boundaryValues(const double* const, const double, const double, const int, const int normalNonZero,
                      const double* const fluxIn, const double* const stateIn, double* fluxOut,
                      double* stateOut) {
    for (int m = 0; m < 5; m++) {
      stateOut[m] = stateIn[m];
      fluxOut[m] = fluxIn[m];
    }
    if (rule == 2) {
      stateOut[normalNonZero + 1] = -stateOut[normalNonZero + 1];
      double F2[3][5];
      double* F[3] = {F2[0], F2[1], F2[2]};
      flux(stateOut, F);
      for (int m = 0; m < 5; m++) fluxOut[m] = F2[normalNonZero][m];
    }
  }
  /* adjustPointSolution: one of the built-in forms of adjust_hooks.h */
  int adj_kind = 0;
  const double* adj_param = nullptr;
  void adjustPointSolution(const double* const x, const double, const double t, const double dt, double* Q) {
    orc_adjust_point(adj_kind, DIMENSIONS, adj_param, x, t, dt, Q);
  }
  /* FV boundary hook (FiniteVolumesSolver::boundaryValues): rule 1 copies
   * the inside state (EulerFV's outflow), rule 2 also negates the normal
   * momentum (slip wall) */
  int rule = 1;
  void boundaryValues(const double* const, const double, const double, const int, const int normalNonZero,
                      const double* const stateIn, double* stateOut) {
    for (int m = 0; m < 5; m++) stateOut[m] = stateIn[m];
    if (rule == 2) stateOut[normalNonZero + 1] = -stateOut[normalNonZero + 1];
  }
  double riemannSolver(double* fL, double* fR, const double* qL, const double* qR, int d) {
    return kernels::finitevolumes::riemannsolvers::c::rusanov<false, true>(*this, fL, fR, qL, qR, d);
  }
};

typedef tarch::la::Vector<DIMENSIONS, double> Vec;

Vec vec(const double* dx) {
#if DIMENSIONS == 3
  return Vec(dx[0], dx[1], dx[2]);
#else
  return Vec(dx[0], dx[1]);
#endif
}

constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

template <int N, int P>
struct DG {
  typedef Euler<N, P> S;
  static constexpr int B = N + 1, V = 5, D = V + P;
  static constexpr int NN = ipow(B, DIMENSIONS);
  static constexpr int NF = ipow(B, DIMENSIONS - 1);

  struct Temps {
    std::vector<double> st, stf, qhi, fhi;
    double* stp[4];
    double* stfp[2];
    Temps() : st(4 * NN * B * D), stf(2 * NN * B * (DIMENSIONS + 1) * V), qhi(NN * D),
              fhi(NN * (DIMENSIONS + 1) * V) {
      for (int i = 0; i < 4; i++) stp[i] = st.data() + i * NN * B * D;
      for (int i = 0; i < 2; i++) stfp[i] = stf.data() + i * NN * B * (DIMENSIONS + 1) * V;
    }
  };

  static void stp(const double* luh, double* lQi, double* lQhi, double* lFhi, double* qb,
                  double* fb, const double* dx, double dt, Temps& t) {
    S s;
    double tmpvec[5];
    kernels::aderdg::generic::c::spaceTimePredictorNonlinear<false, true, false, S>(
        s, qb, fb, t.stp, t.stfp, t.qhi.data(), t.fhi.data(), tmpvec, luh, vec(dx), dt);
    if (lQi) std::memcpy(lQi, t.stp[0], sizeof(double) * NN * B * D);
    if (lQhi) std::memcpy(lQhi, t.qhi.data(), sizeof(double) * NN * D);
    if (lFhi) std::memcpy(lFhi, t.fhi.data(), sizeof(double) * NN * (DIMENSIONS + 1) * V);
  }
  static void vi(double* lduh, const double* lFhi, const double* dx) {
    kernels::aderdg::generic::c::volumeIntegralNonlinear<false, true, V, B>(lduh, lFhi, vec(dx));
  }
  static void si(double* lduh, const double* lFhbnd, const double* dx) {
    kernels::aderdg::generic::c::surfaceIntegralNonlinear<V, B>(lduh, lFhbnd, vec(dx));
  }
  static void riemann(double* FL, double* FR, const double* QL, const double* QR, int d) {
    S s;
    kernels::aderdg::generic::c::riemannSolverNonlinear<false, S>(s, FL, FR, QL, QR, nullptr,
                                                                   nullptr, nullptr, 0.0, d);
  }
  static void update(double* luh, const double* lduh, double dt) {
    S s;
    kernels::aderdg::generic::c::solutionUpdate<S>(s, luh, lduh, dt);
  }
  static double dt(const double* luh, const double* dx) {
    S s;
    double lam[5];
    return kernels::aderdg::generic::c::stableTimeStepSize<S>(s, luh, lam, vec(dx));
  }
  /* one step on a uniform grid (reference non-fused order); periodic in
   * every dimension d with bc == nullptr or bc[d] == 0, else the faces on
   * the two domain ends of d go through the reference's boundaryConditions
   * kernel with rule bc[d] and the Riemann solve of
   * ADERDGSolver::applyBoundaryConditions (ADERDGSolver.cpp:2854-2925:
   * outside state on the left for faces 2d, on the right for faces 2d+1) */
  static double grid_step(const int* n, const double* dx, double* luh, int policy,
                          double dt_fixed, int nthreads, const int* bc = nullptr) {
    static_assert(P == 0, "grid step without parameters");
    const long nc = DIMENSIONS == 3 ? (long)n[0] * n[1] * n[2] : (long)n[0] * n[1];
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    double dtv = dt_fixed;
    if (policy != 2) {
      double m = DBL_MAX;
#pragma omp parallel for reduction(min : m)
      for (long c = 0; c < nc; c++) {
        double d = dt(luh + c * NN * D, dx);
        if (policy == 1) d = d / kernels_pnpm() / (2 * N + 1);
        m = d < m ? d : m;
      }
      dtv = m;
    }
    // the solver's per-cell arrays (lduh, lQhbnd, lFhbnd) persist between
    // steps as the reference's cell descriptions do; every kernel writes
    // its outputs in full (volumeIntegral and the extrapolation zero them)
    static std::vector<double> lduh, qb, fb;
    lduh.resize(nc * NN * V);
    qb.resize(nc * 2 * DIMENSIONS * NF * D);
    fb.resize(nc * 2 * DIMENSIONS * NF * V);
#pragma omp parallel
    {
      Temps t;
#pragma omp for schedule(dynamic, 16)
      for (long c = 0; c < nc; c++) {
        stp(luh + c * NN * D, nullptr, nullptr, nullptr, qb.data() + c * 2 * DIMENSIONS * NF * D,
            fb.data() + c * 2 * DIMENSIONS * NF * V, dx, dtv, t);
        vi(lduh.data() + c * NN * V, t.fhi.data(), dx);
      }
    }
    for (int d = 0; d < DIMENSIONS; d++) {
      const int rule = bc ? bc[d] : 0;
#pragma omp parallel for
      for (long c = 0; c < nc; c++) {
        int r[3] = {(int)(c % n[0]), (int)((c / n[0]) % n[1]),
                    DIMENSIONS == 3 ? (int)(c / ((long)n[0] * n[1])) : 0};
        if (rule) {
          const int j0 = r[d];
          if (j0 == 0) boundary_face(c, 2 * d, d, rule, dx, dtv, qb.data(), fb.data());
          if (j0 + 1 == n[d]) {
            boundary_face(c, 2 * d + 1, d, rule, dx, dtv, qb.data(), fb.data());
            continue;
          }
        }
        r[d] = (r[d] + 1) % n[d];
        long cr = DIMENSIONS == 3 ? ((long)r[2] * n[1] + r[1]) * n[0] + r[0]
                                  : (long)r[1] * n[0] + r[0];
        riemann(fb.data() + (c * 2 * DIMENSIONS + 2 * d + 1) * NF * V,
                fb.data() + (cr * 2 * DIMENSIONS + 2 * d) * NF * V,
                qb.data() + (c * 2 * DIMENSIONS + 2 * d + 1) * NF * D,
                qb.data() + (cr * 2 * DIMENSIONS + 2 * d) * NF * D, d);
      }
    }
#pragma omp parallel for
    for (long c = 0; c < nc; c++) {
      si(lduh.data() + c * NN * V, fb.data() + c * 2 * DIMENSIONS * NF * V, dx);
      update(luh + c * NN * D, lduh.data() + c * NN * V, dtv);
    }
    return dtv;
  }
  /* the domain-boundary face `face` of cell c: outside state from the
   * reference's boundaryConditions kernel, then the Riemann solve with the
   * outside state on the side applyBoundaryConditions puts it */
  static void boundary_face(long c, int face, int d, int rule, const double* dx, double dtv,
                            const double* qb, double* fb) {
    S s;
    s.rule = rule;
    double qo[NF * D], fo[NF * V];
    double* FIn = fb + (c * 2 * DIMENSIONS + face) * NF * V;
    const double* QIn = qb + (c * 2 * DIMENSIONS + face) * NF * D;
    kernels::aderdg::generic::c::boundaryConditions<S>(s, fo, qo, FIn, QIn, Vec(0.5), vec(dx), 0.0, dtv,
                                                       face, d);
    if (face % 2 == 0) riemann(fo, FIn, qo, QIn, d);
    else riemann(FIn, fo, QIn, qo, d);
  }
  /* per-cell work of one step on ncells independent cells (each its own
   * periodic neighbour): the CPU-baseline sample */
  static void sample_step(long nc, const double* dx, double* luh, double dtv, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel
    {
      Temps t;
      std::vector<double> lduh(NN * V), qb(2 * DIMENSIONS * NF * D), fb(2 * DIMENSIONS * NF * V);
#pragma omp for schedule(dynamic, 16)
      for (long c = 0; c < nc; c++) {
        double* u = luh + c * NN * D;
        stp(u, nullptr, nullptr, nullptr, qb.data(), fb.data(), dx, dtv, t);
        vi(lduh.data(), t.fhi.data(), dx);
        for (int d = 0; d < DIMENSIONS; d++)
          riemann(fb.data() + (2 * d + 1) * NF * V, fb.data() + (2 * d) * NF * V,
                  qb.data() + (2 * d + 1) * NF * D, qb.data() + (2 * d) * NF * D, d);
        si(lduh.data(), fb.data(), dx);
        update(u, lduh.data(), dtv);
      }
    }
  }
  static double kernels_pnpm() {
    static const double pnpm[10] = {1.0, 0.33, 0.17, 0.1, 0.069, 0.045, 0.038, 0.03, 0.02, 0.015};
    return pnpm[N];
  }
};

#define EXA_ORDERS(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7)

}  // namespace

/* Runs f() on a thread with a 1 GiB stack: the reference keeps its FV work
 * arrays on the stack (musclhancock/c/2d/musclhancock.cpph:75,102-105), a
 * 256^2 MUSCL-Hancock patch needs ~25 MB of them. */
template <typename F>
static void on_big_stack(F f) {
  struct Run {
    static void* go(void* p) {
      (*static_cast<F*>(p))();
      return nullptr;
    }
  };
  pthread_attr_t a;
  pthread_attr_init(&a);
  pthread_attr_setstacksize(&a, (size_t)1 << 30);
  pthread_t th;
  if (pthread_create(&th, &a, &Run::go, &f) == 0) pthread_join(th, nullptr);
  pthread_attr_destroy(&a);
}

/* The mock PDE of the reference's Rusanov unit test (exahype/tests/kernels/
 * finitevolumes/riemannsolvers/c/RusanovTest.cpp:33-60, RusanovTest.h:37-38):
 * 4 variables, 3 parameters, zero flux, every eigenvalue 1. */
struct ZeroFluxZeroNCP {
  static constexpr int NumberOfVariables = 4;
  static constexpr int NumberOfParameters = 3;
  void flux(const double* const, double**) {}
  void eigenvalues(const double* const, const int, double* lambda) {
    for (int i = 0; i < NumberOfVariables; i++) lambda[i] = 1.0;
  }
  void nonConservativeProduct(const double* const, const double* const, double*) {}
};

#if DIMENSIONS == 2
/* One step of a single periodic FV patch with the reference's godunov
 * (scheme 0, ghost 1) or musclhancock (scheme 1, ghost 2) kernel; the
 * patch size is a template constant of the reference, so a fixed set is
 * instantiated.  Runs on a thread with a 1 GiB stack because the
 * reference keeps its MUSCL work arrays on the stack
 * (musclhancock/c/2d/musclhancock.cpph:75,102-105). */
template <int PS, int G>
static double fv_step_t(int scheme, double* luh, const double* dx, double dt_fixed,
                        double* adm) {
  typedef Euler<0, 0, PS, G> S;
  const int SZ = PS + 2 * G;
  S s;
  /* periodic ghosts */
  for (int j = 0; j < SZ; j++)
    for (int k = 0; k < SZ; k++) {
      if (j >= G && j < G + PS && k >= G && k < G + PS) continue;
      int sj = G + ((j - G) % PS + PS) % PS, sk = G + ((k - G) % PS + PS) % PS;
      std::memcpy(luh + ((long)j * SZ + k) * 5, luh + ((long)sj * SZ + sk) * 5, 5 * sizeof(double));
    }
  double lam[5];
  double dt = dt_fixed > 0 ? dt_fixed
                           : kernels::finitevolumes::commons::c::stableTimeStepSize<S>(s, luh, lam, vec(dx));
  std::vector<double> old(luh, luh + (long)SZ * SZ * 5);
  double a;
  if (scheme == 0)
    a = kernels::finitevolumes::godunov::c::solutionUpdate<false, false, true, S>(
        s, luh, old.data(), nullptr, nullptr, vec(dx), dt);
  else
    a = kernels::finitevolumes::musclhancock::c::solutionUpdate<false, false, true, S>(
        s, luh, old.data(), nullptr, nullptr, vec(dx), dt);
  if (adm) *adm = a;
  return dt;
}

#endif

#if DIMENSIONS == 3
/* 3D counterpart of fv_step_t (godunov/c/3d, musclhancock/c/3d) on one
 * periodic patch; the MUSCL work arrays of the reference live on the stack
 * (musclhancock/c/3d/musclhancock.cpph:74-118), small patches only. */
template <int PS, int G>
static double fv_step3_t(int scheme, double* luh, const double* dx, double dt_fixed, double* adm) {
  typedef Euler<0, 0, PS, G> S;
  const int SZ = PS + 2 * G;
  S s;
  for (int i = 0; i < SZ; i++)
    for (int j = 0; j < SZ; j++)
      for (int k = 0; k < SZ; k++) {
        const int si = G + ((i - G) % PS + PS) % PS, sj = G + ((j - G) % PS + PS) % PS,
                  sk = G + ((k - G) % PS + PS) % PS;
        if (si == i && sj == j && sk == k) continue;
        std::memcpy(luh + (((long)i * SZ + j) * SZ + k) * 5, luh + (((long)si * SZ + sj) * SZ + sk) * 5,
                    5 * sizeof(double));
      }
  double lam[5];
  double dt = dt_fixed > 0 ? dt_fixed
                           : kernels::finitevolumes::commons::c::stableTimeStepSize<S>(s, luh, lam, vec(dx));
  std::vector<double> old(luh, luh + (long)SZ * SZ * SZ * 5);
  double a;
  if (scheme == 0)
    a = kernels::finitevolumes::godunov::c::solutionUpdate<false, false, true, S>(
        s, luh, old.data(), nullptr, nullptr, vec(dx), dt);
  else
    a = kernels::finitevolumes::musclhancock::c::solutionUpdate<false, false, true, S>(
        s, luh, old.data(), nullptr, nullptr, vec(dx), dt);
  if (adm) *adm = a;
  return dt;
}
#endif

/* The reference's ghost filling of one FV patch at a domain-boundary face
 * (FiniteVolumesSolver::mergeWithBoundaryData, FiniteVolumesSolver.cpp:
 * 689-727): boundaryLayerExtraction, boundaryConditions and
 * ghostLayerFillingAtBoundary of finitevolumes/commons/c/commons.cpph for
 * face 2 d + side, with the boundary rule of Euler::boundaryValues. */
template <int PS, int G>
static void fv_boundary_t(double* luh, int face, int rule) {
  typedef Euler<0, 0, PS, G> S;
  namespace FC = kernels::finitevolumes::commons::c;
  S s;
  s.rule = rule;
  const int d = face >> 1;
  tarch::la::Vector<DIMENSIONS, int> pos(0);
  pos[d] = (face & 1) ? 1 : -1;
  long bnd = G * 5;
  for (int i = 1; i < DIMENSIONS; i++) bnd *= PS;
  std::vector<double> in(bnd), out(bnd);
  FC::boundaryLayerExtraction<S>(s, in.data(), luh, pos);
  FC::boundaryConditions<S>(s, out.data(), in.data(), Vec(0.5), Vec(1.0), 0.0, 0.0, face, d);
  FC::ghostLayerFillingAtBoundary<S>(s, luh, out.data(), pos);
}

extern "C" {

/* The reference's solutionAdjustment kernel (c/{2d,3d}/solutionAdjustment.
 * cpph) on one cell of order 2..5 with a built-in hook of adjust_hooks.h */
int ref_solution_adjustment(int order, double* luh, const double* center, const double* dx, double t, double dt,
                            int kind, const double* param) {
#define ACASE(N)                                                                  \
  case N: {                                                                       \
    Euler<N, 0> s;                                                                \
    s.adj_kind = kind;                                                            \
    s.adj_param = param;                                                          \
    kernels::aderdg::generic::c::solutionAdjustment(s, luh, vec(center), vec(dx), t, dt); \
    return 0;                                                                     \
  }
  switch (order) { ACASE(2) ACASE(3) ACASE(4) ACASE(5) }
#undef ACASE
  return -1;
}

/* patch 3, 5, 7, 9 or 11 subcells (limiter patches of orders 1..5) with
 * ghost 1 or 2; returns -1 for other sizes */
int ref_fv_boundary(int patch, int ghost, double* luh, int face, int rule) {
#define BCASE(P)                                                   \
  case P:                                                          \
    if (ghost == 1) fv_boundary_t<P, 1>(luh, face, rule);          \
    else fv_boundary_t<P, 2>(luh, face, rule);                     \
    return 0;
  if (ghost != 1 && ghost != 2) return -1;
  switch (patch) { BCASE(3) BCASE(5) BCASE(7) BCASE(9) BCASE(11) }
#undef BCASE
  return -1;
}

int ref_stp(int order, int npar, const double* luh, double* lQi, double* lQhi, double* lFhi,
            double* qb, double* fb, const double* dx, double dt) {
  if (npar == 1 && order == 3) {
    DG<3, 1>::Temps t;
    DG<3, 1>::stp(luh, lQi, lQhi, lFhi, qb, fb, dx, dt, t);
    return 0;
  }
  if (npar != 0) return -1;
#define CASE(N) case N: { DG<N, 0>::Temps t; DG<N, 0>::stp(luh, lQi, lQhi, lFhi, qb, fb, dx, dt, t); return 0; }
  switch (order) { EXA_ORDERS(CASE) }
#undef CASE
  return -1;
}

int ref_volume_integral(int order, double* lduh, const double* lFhi, const double* dx) {
#define CASE(N) case N: DG<N, 0>::vi(lduh, lFhi, dx); return 0;
  switch (order) { EXA_ORDERS(CASE) }
#undef CASE
  return -1;
}

int ref_surface_integral(int order, double* lduh, const double* lFhbnd, const double* dx) {
#define CASE(N) case N: DG<N, 0>::si(lduh, lFhbnd, dx); return 0;
  switch (order) { EXA_ORDERS(CASE) }
#undef CASE
  return -1;
}

int ref_riemann(int order, int npar, double* FL, double* FR, const double* QL, const double* QR,
                int d) {
  if (npar == 1 && order == 3) { DG<3, 1>::riemann(FL, FR, QL, QR, d); return 0; }
  if (npar != 0) return -1;
#define CASE(N) case N: DG<N, 0>::riemann(FL, FR, QL, QR, d); return 0;
  switch (order) { EXA_ORDERS(CASE) }
#undef CASE
  return -1;
}

int ref_solution_update(int order, int npar, double* luh, const double* lduh, double dt) {
  if (npar == 1 && order == 3) { DG<3, 1>::update(luh, lduh, dt); return 0; }
  if (npar != 0) return -1;
#define CASE(N) case N: DG<N, 0>::update(luh, lduh, dt); return 0;
  switch (order) { EXA_ORDERS(CASE) }
#undef CASE
  return -1;
}

double ref_stable_dt(int order, int npar, const double* luh, const double* dx) {
  if (npar == 1 && order == 3) return DG<3, 1>::dt(luh, dx);
  if (npar != 0) return -1;
#define CASE(N) case N: return DG<N, 0>::dt(luh, dx);
  switch (order) { EXA_ORDERS(CASE) }
#undef CASE
  return -1;
}

double ref_grid_step(int order, const int* n, const double* dx, double* luh, int policy,
                     double dt_fixed, int nthreads) {
#define CASE(N) case N: return DG<N, 0>::grid_step(n, dx, luh, policy, dt_fixed, nthreads);
  switch (order) { EXA_ORDERS(CASE) }
#undef CASE
  return -1;
}

/* As ref_grid_step with a boundary rule per dimension (0 periodic, 1 outflow,
 * 2 reflecting wall) */
double ref_grid_step_bc(int order, const int* n, const double* dx, double* luh, int policy,
                        double dt_fixed, int nthreads, const int* bc) {
#define CASE(N) case N: return DG<N, 0>::grid_step(n, dx, luh, policy, dt_fixed, nthreads, bc);
  switch (order) { EXA_ORDERS(CASE) }
#undef CASE
  return -1;
}

/* The reference's rusanov on the unit test's mock PDE (useNCP = false,
 * useFlux = true, as RusanovTest.cpp:81-88 calls it); returns s_max */
double ref_rusanov_mock(double* fL, double* fR, const double* qL, const double* qR, int d) {
  ZeroFluxZeroNCP s;
  return kernels::finitevolumes::riemannsolvers::c::rusanov<false, true, ZeroFluxZeroNCP>(s, fL, fR, qL, qR,
                                                                                          d);
}

int ref_sample_step(int order, long ncells, const double* dx, double* luh, double dt,
                    int nthreads) {
#define CASE(N) case N: DG<N, 0>::sample_step(ncells, dx, luh, dt, nthreads); return 0;
  switch (order) { EXA_ORDERS(CASE) }
#undef CASE
  return -1;
}

#if DIMENSIONS == 2
double ref_fv_step(int scheme, int patch, double* luh, const double* dx, double dt_fixed,
                   double* adm) {
  double r = -1;
  on_big_stack([&]() {
#define PCASE(P)                                                        \
  case P:                                                               \
    r = scheme == 0 ? fv_step_t<P, 1>(0, luh, dx, dt_fixed, adm)        \
                    : fv_step_t<P, 2>(1, luh, dx, dt_fixed, adm);       \
    break;
    switch (patch) { PCASE(4) PCASE(5) PCASE(8) PCASE(16) PCASE(32) PCASE(64) PCASE(128) PCASE(256) }
#undef PCASE
  });
  return r;
}
#endif

#if DIMENSIONS == 3
/* one step of a periodic 3D patch (patch 4, 5, 7 or 9) with the reference's
 * 3D godunov (scheme 0, ghost 1) or musclhancock (scheme 1, ghost 2) */
double ref_fv_step(int scheme, int patch, double* luh, const double* dx, double dt_fixed, double* adm) {
  double r = -1;
  on_big_stack([&]() {
#define PCASE(P)                                                          \
  case P:                                                                 \
    r = scheme == 0 ? fv_step3_t<P, 1>(0, luh, dx, dt_fixed, adm)         \
                    : fv_step3_t<P, 2>(1, luh, dx, dt_fixed, adm);        \
    break;
    switch (patch) { PCASE(4) PCASE(5) PCASE(7) PCASE(9) }
#undef PCASE
  });
  return r;
}
#endif

/* AMR transfer operators of the reference (amrRoutines.cpph), nVar = 5,
 * nPar = 0, from level 0 to level `level_delta`.  what: 0 volume
 * prolongation (out_q = luhFine), 1 volume restriction (out_q += ...),
 * 2 face prolongation (out_q/out_f = lQhbnd/lFhbnd of the fine face),
 * 3 face restriction (accumulates). */
int ref_amr(int what, int order, double* out_q, double* out_f, const double* in_q, const double* in_f,
            int level_delta, const int* index) {
  tarch::la::Vector<DIMENSIONS, int> vi;
  tarch::la::Vector<DIMENSIONS - 1, int> fi;
  for (int d = 0; d < DIMENSIONS; d++) vi[d] = index[d];
  for (int d = 0; d < DIMENSIONS - 1; d++) fi[d] = index[d];
  namespace K = kernels::aderdg::generic::c;
#define CASE(N)                                                                                     \
  case N:                                                                                           \
    if (what == 0) K::volumeUnknownsProlongation<5, 0, N + 1>(out_q, in_q, 0, level_delta, vi);     \
    else if (what == 1) K::volumeUnknownsRestriction<5, 0, N + 1>(out_q, in_q, 0, level_delta, vi); \
    else if (what == 2) K::faceUnknownsProlongation<5, 0, N + 1>(out_q, out_f, in_q, in_f, 0, level_delta, fi); \
    else K::faceUnknownsRestriction<5, 0, N + 1>(out_q, out_f, in_q, in_f, 0, level_delta, fi);    \
    return 0;
  switch (order) { EXA_ORDERS(CASE) }
#undef CASE
  return -1;
}

/* The reference's a-posteriori limiter kernels (kernels/limiter/generic/c/
 * Limiter.cpp) for one cell, driven through the solver stand-in of
 * ref_shim/exahype/solvers/ADERDGSolver.h.  what: 0 projectOnFVLimiterSpace
 * (in = luh, out = lim), 1 projectOnDGSpace (in = lim, out = luh),
 * 2 findCellLocalMinAndMax (in = luh), 3 findCellLocalLimiterMinAndMax
 * (in = lim), 4 discreteMaximumPrincipleAndMinAndMaxSearch (in = luh;
 * obs_min/obs_max are the [2 dim][nobs] in/out blocks; returns 1 if the
 * DMP holds). */
int ref_limiter(int what, int order, int nvar, int nobs, int ghost, const double* in, double* out,
                double* obs_min, double* obs_max, double relaxation, double difference_scaling) {
  namespace L = kernels::limiter::generic::c;
  const exahype::solvers::ADERDGSolver solver(nvar, order + 1, nobs);
  switch (what) {
    case 0: L::projectOnFVLimiterSpace(in, nvar, order + 1, ghost, out); return 0;
    case 1: L::projectOnDGSpace(in, nvar, order + 1, ghost, out); return 0;
    case 2: L::findCellLocalMinAndMax(in, &solver, obs_min, obs_max); return 0;
    case 3: L::findCellLocalLimiterMinAndMax(in, &solver, ghost, obs_min, obs_max); return 0;
    case 4:
      return L::discreteMaximumPrincipleAndMinAndMaxSearch(in, &solver, relaxation, difference_scaling,
                                                            obs_min, obs_max) ? 1 : 0;
  }
  return -1;
}

/* The limiter projection tables as the reference builds them at start-up
 * (LimiterProjectionMatrices.cpp:40-140) and its Gauss-Lobatto nodes:
 * uh2lim [B][S], uh2lob [B][B], lim2uh [S][B], lob [B]. */
int ref_limiter_tables(int order, double* uh2lim, double* uh2lob, double* lim2uh, double* lob) {
  const int B = order + 1, S = 2 * order + 1;
  for (int i = 0; i < B * S; i++) uh2lim[i] = kernels::uh2lim[order][i];
  for (int i = 0; i < B * B; i++) uh2lob[i] = kernels::uh2lob[order][i];
  for (int i = 0; i < S * B; i++) lim2uh[i] = kernels::lim2uh[order][i];
  for (int i = 0; i < B; i++) lob[i] = kernels::gaussLobattoNodes[order][i];
  return 0;
}

}  // extern "C"
