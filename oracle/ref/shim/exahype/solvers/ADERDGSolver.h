// Stand-in for the solver base class that the reference limiter kernels
// (kernels/limiter/generic/c/Limiter.cpp) query: DMP observable count, basis
// size, variable count and the observable map. The oracle's PDE classes
// derive from it.
#pragma once
namespace exahype { namespace solvers {
class ADERDGSolver {
 public:
  virtual ~ADERDGSolver() {}
  virtual int getDMPObservables() const = 0;
  virtual int getNodesPerCoordinateAxis() const = 0;
  virtual int getNumberOfVariables() const = 0;
  virtual void mapDiscreteMaximumPrincipleObservables(double* observables, const int numberOfObservables,
                                                      const double* const Q) const = 0;
};
}}
