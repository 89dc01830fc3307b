// C++ adaptor over the C ABI (exa_kernels.h) with the template names and
// argument lists of ExaHyPE's generic kernels, so code written against
//   kernels::aderdg::generic::c::*            (ExaHyPE/kernels/aderdg/generic/Kernels.h:86-175)
//   kernels::finitevolumes::riemannsolvers::c::rusanov (riemannsolvers/c/riemannsolvers.h:30-32)
// can switch by namespace to exahype_b200::kernels::...  The SolverType
// supplies NumberOfVariables, NumberOfParameters and Order exactly as for the
// reference templates; the PDE is the library's compiled-in Euler functor
// (a solver may define `static constexpr int ExaPde = EXA_PDE_EULER_PLANAR`
// to select the planar 2D form).  Dimension is a template argument because
// the reference's DIMENSIONS macro is not available to a library header; the
// dx argument may be any type with operator[] (tarch::la::Vector included).
//
// Errors: the reference kernels return void and abort on misuse; these
// wrappers throw exahype_b200::Error carrying the exa_status_t.
#pragma once
#include <stdexcept>
#include <string>

#include "exa_kernels.h"

namespace exahype_b200 {

struct Error : std::runtime_error {
  exa_status_t status;
  Error(exa_status_t s, const char* where)
      : std::runtime_error(std::string(where) + ": " + exa_status_string(s) + " (" +
                           exa_last_error_string() + ")"),
        status(s) {}
};

inline void check(exa_status_t s, const char* where) {
  if (s != EXA_OK) throw Error(s, where);
}

namespace detail {
template <typename T, typename = int>
struct PdeOf { static constexpr int value = EXA_PDE_EULER; };
template <typename T>
struct PdeOf<T, decltype((void)T::ExaPde, 0)> { static constexpr int value = T::ExaPde; };

template <int Order_, int NumberOfVariables_>
struct PlainSolver {
  static constexpr int Order = Order_;
  static constexpr int NumberOfVariables = NumberOfVariables_;
  static constexpr int NumberOfParameters = 0;
};

template <int DIM, typename SolverType, typename Vec>
exa_aderdg_desc_t desc(const Vec& dx) {
  exa_aderdg_desc_t d;
  d.dim = DIM;
  d.order = SolverType::Order;
  d.nvar = SolverType::NumberOfVariables;
  d.npar = SolverType::NumberOfParameters;
  d.pde = PdeOf<SolverType>::value;
  d.precision = EXA_PREC_FP64;
  for (int i = 0; i < 3; i++) d.dx[i] = i < DIM ? static_cast<double>(dx[i]) : 1.0;
  return d;
}
}  // namespace detail

namespace kernels {
namespace aderdg {
namespace generic {
namespace c {

// spaceTimePredictorNonlinear<useSource, useFlux, useNCP, SolverType>
// (kernels/aderdg/generic/c/3d/spaceTimePredictorNonlinear.cpph:523-577)
template <int DIM, bool useSource, bool useFlux, bool useNCP, typename SolverType, typename Vec>
void spaceTimePredictorNonlinear(SolverType&, double* lQhbnd, double* lFhbnd,
                                 double** tempSpaceTimeUnknowns,
                                 double** tempSpaceTimeFluxUnknowns, double* tempUnknowns,
                                 double* tempFluxUnknowns, double* tempStateSizedVector,
                                 const double* const luh, const Vec& dx, const double dt) {
  static_assert(useFlux, "the compiled-in Euler PDE has a conservative flux");
  const exa_aderdg_desc_t d = detail::desc<DIM, SolverType>(dx);
  check(exa_aderdg_spaceTimePredictor(&d, lQhbnd, lFhbnd, tempSpaceTimeUnknowns,
                                      tempSpaceTimeFluxUnknowns, tempUnknowns, tempFluxUnknowns,
                                      tempStateSizedVector, luh, d.dx, dt, nullptr, nullptr),
        "spaceTimePredictorNonlinear");
}

// volumeIntegralNonlinear<useSourceOrNCP, useFlux, numberOfVariables, basisSize>
// (c/3d/volumeIntegralNonlinear.cpph:26-125); the source block of lFhi is
// added (it is zero for the Euler PDE), as with useSourceOrNCP = true.
template <int DIM, bool useSourceOrNCP, bool useFlux, int numberOfVariables, int basisSize,
          typename Vec>
void volumeIntegralNonlinear(double* lduh, const double* const lFhi, const Vec& dx) {
  typedef detail::PlainSolver<basisSize - 1, numberOfVariables> S;
  const exa_aderdg_desc_t d = detail::desc<DIM, S>(dx);
  check(exa_aderdg_volumeIntegral(&d, lduh, lFhi, d.dx), "volumeIntegralNonlinear");
}

// surfaceIntegralNonlinear<numberOfVariables, basisSize> (c/3d/surfaceIntegralNonlinear.cpph:21-85)
template <int DIM, int numberOfVariables, int basisSize, typename Vec>
void surfaceIntegralNonlinear(double* lduh, const double* const lFbnd, const Vec& dx) {
  typedef detail::PlainSolver<basisSize - 1, numberOfVariables> S;
  const exa_aderdg_desc_t d = detail::desc<DIM, S>(dx);
  check(exa_aderdg_surfaceIntegral(&d, lduh, lFbnd, d.dx), "surfaceIntegralNonlinear");
}

// riemannSolverNonlinear<useNCP, SolverType> (c/3d/riemannSolverNonlinear.cpph:37-120)
template <int DIM, bool useNCP, typename SolverType>
void riemannSolverNonlinear(SolverType&, double* FL, double* FR, const double* const QL,
                            const double* const QR, double* tempFaceUnknownsArray,
                            double** tempStateSizedVectors, double** tempStateSizedSquareMatrices,
                            const double dt, const int normalNonZero) {
  static_assert(!useNCP, "the compiled-in Euler PDE has no non-conservative product");
  const double one[3] = {1.0, 1.0, 1.0};
  const exa_aderdg_desc_t d = detail::desc<DIM, SolverType>(one);
  check(exa_aderdg_riemannSolver(&d, FL, FR, QL, QR, tempFaceUnknownsArray, tempStateSizedVectors,
                                 tempStateSizedSquareMatrices, dt, normalNonZero, 0),
        "riemannSolverNonlinear");
}

// solutionUpdate<SolverType> (c/3d/solutionUpdate.cpph:23-47)
template <int DIM, typename SolverType>
void solutionUpdate(SolverType&, double* luh, const double* const lduh, const double dt) {
  const double one[3] = {1.0, 1.0, 1.0};
  const exa_aderdg_desc_t d = detail::desc<DIM, SolverType>(one);
  check(exa_aderdg_solutionUpdate(&d, luh, lduh, dt), "solutionUpdate");
}

// stableTimeStepSize<SolverType> (c/3d/stableTimeStepSize.cpph:21-61), CFL 0.9
template <int DIM, typename SolverType, typename Vec>
double stableTimeStepSize(SolverType&, const double* const luh, double* tempEigenvalues,
                          const Vec& dx) {
  const exa_aderdg_desc_t d = detail::desc<DIM, SolverType>(dx);
  double dt = 0.0;
  check(exa_aderdg_stableTimeStepSize(&d, luh, tempEigenvalues, d.dx, &dt), "stableTimeStepSize");
  return dt;
}

}  // namespace c
}  // namespace generic
}  // namespace aderdg

namespace finitevolumes {
namespace riemannsolvers {
namespace c {
// rusanov<useNCP, useFlux, SolverType> (riemannsolvers/c/rusanov.cpph:24-83)
template <int DIM, bool useNCP, bool useFlux, typename SolverType>
double rusanov(SolverType&, double* fnL, double* fnR, const double* qL, const double* qR,
               int normalNonZero) {
  static_assert(useFlux && !useNCP, "compiled-in Euler PDE");
  double smax = 0.0;
  check(exa_fv_rusanov(DIM, SolverType::NumberOfVariables, SolverType::NumberOfParameters,
                       detail::PdeOf<SolverType>::value, fnL, fnR, qL, qR, normalNonZero, &smax),
        "rusanov");
  return smax;
}
}  // namespace c
}  // namespace riemannsolvers
}  // namespace finitevolumes
}  // namespace kernels
}  // namespace exahype_b200
