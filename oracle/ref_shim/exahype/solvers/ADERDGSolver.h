#pragma once
// Project-written stand-in for the solver object that the reference's
// limiter kernels query (kernels/limiter/generic/c/Limiter.cpp takes a
// `const exahype::solvers::ADERDGSolver*`): only the four accessors those
// kernels call.  The observables map is the generated solvers' default
// (copy the first numberOfObservables values of Q).
#include <algorithm>

namespace exahype {
namespace solvers {

class ADERDGSolver {
 public:
  ADERDGSolver(int numberOfVariables, int nodesPerCoordinateAxis, int dmpObservables)
      : _nvar(numberOfVariables), _basis(nodesPerCoordinateAxis), _nobs(dmpObservables) {}
  int getNumberOfVariables() const { return _nvar; }
  int getNodesPerCoordinateAxis() const { return _basis; }
  int getDMPObservables() const { return _nobs; }
  void mapDiscreteMaximumPrincipleObservables(double* observables, const int numberOfObservables,
                                              const double* const Q) const {
    if (numberOfObservables > 0) std::copy_n(Q, numberOfObservables, observables);
  }

 private:
  int _nvar, _basis, _nobs;
};

}  // namespace solvers
}  // namespace exahype
