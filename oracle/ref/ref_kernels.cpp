// Oracle-only wrapper: exposes the reference's own generic C++ kernels
// (ExaHyPE/kernels/...) behind plain C entry points so that the test suite and
// the CPU baseline can call them. This file is test infrastructure; it is
// compiled once per dimension (-DDIMENSIONS=2/3) against the unmodified
// reference sources by oracle/ref/Makefile and never ships with the product.
//
// The PDE classes below restate the PDEs the reference uses for this path:
//   * EulerDemo  -- Demonstrators/EulerADERDG/MyEulerSolver_ADERDG.cpp:102-160
//                   (5 variables, gamma 1.4, 3 momentum components in 2D too)
//   * EulerTest  -- exahype/tests/kernels/c/GenericEulerKernelTest{2D,3D}.cpp:28-77
//                   ("2.5D" Euler in 2D, one material parameter)
//   * EulerSourceNCP -- EulerTest with useSource = useNCP = true: an algebraic
//                   source of this repository's choosing and the kernel tests'
//                   non-zero non-conservative product mock
//                   (GenericEulerKernelTest3D.cpp:84-110 with
//                   _setNcpAndMatrixBToZero false)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <set>
#include <algorithm>

// g++ 13 no longer provides std::abs<double> as a function template that
// std::transform can take; riemannSolverNonlinear.cpph:70-71 relies on it.
namespace std {
template <typename T> inline T abs(T x) { return x < 0 ? -x : x; }
}

#include "kernels/aderdg/generic/Kernels.h"
#include "kernels/GaussLegendreQuadrature.h"
#include "kernels/GaussLobattoQuadrature.h"
#include "kernels/DGMatrices.h"
#include "kernels/DGBasisFunctions.h"
#include "kernels/LimiterProjectionMatrices.h"
#include "kernels/limiter/generic/Limiter.h"
#include "kernels/finitevolumes/riemannsolvers/c/riemannsolvers.h"
#include "kernels/finitevolumes/musclhancock/c/musclhancock.h"
#include "kernels/finitevolumes/commons/c/commons.h"
#include "exahype/solvers/ADERDGSolver.h"

#if DIMENSIONS == 2
#define REFNAME(x) ref2d_##x
#else
#define REFNAME(x) ref3d_##x
#endif

namespace {

// Base for both PDEs: counts flux calls so the driver can report how many
// Picard sweeps the reference predictor ran (b^(d+1) flux calls per sweep).
template <int N_, int nPar_>
struct PDEBase : public exahype::solvers::ADERDGSolver {
  static constexpr int NumberOfVariables = 5;
  static constexpr int NumberOfParameters = nPar_;
  static constexpr int Order = N_;
  static constexpr double CFL = 0.9;
  static constexpr int PatchSize = 2 * N_ + 1;
  static constexpr int GhostLayerWidth = 2;
  static constexpr bool kSourceNCP = false;  // instantiate the kernels with useSource = useNCP = true
  long fluxCalls = 0;
  int getDMPObservables() const override { return NumberOfVariables; }
  int getNodesPerCoordinateAxis() const override { return N_ + 1; }
  int getNumberOfVariables() const override { return NumberOfVariables; }
  void mapDiscreteMaximumPrincipleObservables(double* obs, const int n, const double* const Q) const override {
    for (int i = 0; i < NumberOfVariables; ++i) obs[i] = Q[i];
  }
  void algebraicSource(const double* const, double* S) { for (int i = 0; i < 5; i++) S[i] = 0.0; }
  void nonConservativeProduct(const double* const, const double* const, double* B) { for (int i = 0; i < 5; i++) B[i] = 0.0; }
  void adjustPointSolution(const double* const, const double, const double, double*) {}
  bool isPhysicallyAdmissible(const double* const, const double* const obsMin, const double* const,
                              const int, const tarch::la::Vector<DIMENSIONS, double>&,
                              const tarch::la::Vector<DIMENSIONS, double>&, const double, const double) const {
    if (obsMin[0] <= 0.0) return false;
    if (obsMin[4] <= 0.0) return false;
    return true;
  }
};

// Euler as in the demonstrator (pressure from all three momentum components).
template <int N_>
struct EulerDemo : public PDEBase<N_, 0> {
  void flux(const double* const Q, double** F) {
    this->fluxCalls++;
    const double GAMMA = 1.4;
    const double irho = 1. / Q[0];
    const double jj = Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3];
    const double p = (GAMMA - 1) * (Q[4] - 0.5 * irho * jj);
    for (int d = 0; d < DIMENSIONS; d++) {
      F[d][0] = Q[1 + d];
      for (int a = 0; a < 3; a++) F[d][1 + a] = irho * (Q[1 + d] * Q[1 + a]) + (d == a ? p : 0.0);
      F[d][4] = (irho * (Q[4] + p)) * Q[1 + d];
    }
  }
  void eigenvalues(const double* const Q, const int d, double* lambda) {
    const double GAMMA = 1.4;
    const double irho = 1. / Q[0];
    const double jj = Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3];
    const double p = (GAMMA - 1) * (Q[4] - 0.5 * irho * jj);
    const double u_n = Q[d + 1] * irho;
    const double c = std::sqrt(GAMMA * p * irho);
    lambda[0] = u_n - c;
    lambda[1] = u_n;
    lambda[2] = u_n;
    lambda[3] = u_n;
    lambda[4] = u_n + c;
  }
  // boundaryValues of the ADER-DG and the FV solver, the kind set per call
  // through boundary_kind: 0 outflow (the inside state and flux copied), 1
  // the demonstrator's reflective walls (MyEulerSolver_ADERDG.cpp:63-87: the
  // normal momentum negated and that state's normal flux; the FV solver's
  // MyEulerSolver_FV.cpp:47-62: the normal momentum negated), restated
  static thread_local int boundary_kind;
  void boundaryValues(const double* const, const double, const double, const int, const int normalNonZero,
                      const double* const fluxIn, const double* const stateIn, double* fluxOut, double* stateOut) {
    std::copy_n(stateIn, 5, stateOut);
    if (boundary_kind == 1) {
      stateOut[1 + normalNonZero] = -stateOut[1 + normalNonZero];
      double F0[3][5] = {};
      double* F[3] = {F0[0], F0[1], F0[2]};
      flux(stateOut, F);
      std::copy_n(F[normalNonZero], 5, fluxOut);
    } else {
      std::copy_n(fluxIn, 5, fluxOut);
    }
  }
  void boundaryValues(const double* const, const double, const double, const int, const int normalNonZero,
                      const double* const stateIn, double* stateOut) {
    std::copy_n(stateIn, 5, stateOut);
    if (boundary_kind == 1) stateOut[1 + normalNonZero] = -stateOut[1 + normalNonZero];
  }
  double riemannSolver(double* fL, double* fR, const double* qL, const double* qR, int normalNonZero) {
    return kernels::finitevolumes::riemannsolvers::c::rusanov<false, true, EulerDemo<N_>>(*this, fL, fR, qL, qR, normalNonZero);
  }
};

template <int N_>
thread_local int EulerDemo<N_>::boundary_kind = 0;

// The kernel-test mock PDE (2.5D in 2D; one material parameter).
template <int N_>
struct EulerTest : public PDEBase<N_, 1> {
  void flux(const double* const Q, double** F) {
    this->fluxCalls++;
    const double GAMMA = 1.4;
    const double irho = 1.0 / Q[0];
#if DIMENSIONS == 2
    const double p = (GAMMA - 1) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) * irho);
#else
    const double p = (GAMMA - 1) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) * irho);
#endif
    for (int d = 0; d < DIMENSIONS; d++) {
      double* f = F[d];
      f[0] = Q[1 + d];
      for (int a = 0; a < 3; a++) f[1 + a] = irho * Q[1 + d] * Q[1 + a] + (d == a ? p : 0.0);
      f[4] = irho * Q[1 + d] * (Q[4] + p);
    }
  }
  void eigenvalues(const double* const Q, const int d, double* lambda) {
    const double GAMMA = 1.4;
    double irho = 1.0 / Q[0];
#if DIMENSIONS == 2
    double p = (GAMMA - 1) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) * irho);
#else
    double p = (GAMMA - 1) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) * irho);
#endif
    double u_n = Q[d + 1] * irho;
    double c = std::sqrt(GAMMA * p * irho);
    lambda[0] = u_n - c;
    lambda[1] = u_n;
    lambda[2] = u_n;
    lambda[3] = u_n;
    lambda[4] = u_n + c;
  }
  void boundaryValues(const double* const, const double, const double, const int, const int,
                      const double* const fluxIn, const double* const stateIn, double* fluxOut, double* stateOut) {
    std::copy_n(stateIn, 6, stateOut);
    std::copy_n(fluxIn, 5, fluxOut);
  }
  // GenericEulerKernelTest{2D,3D}.cpp: the zero system matrix of the mock
  void coefficientMatrix(const double* const, const int, double* Bn) { std::fill_n(Bn, 25, 0.0); }
};

template <int N_>
struct EulerSourceNCP : public EulerTest<N_> {
  static constexpr bool kSourceNCP = true;
  void algebraicSource(const double* const Q, double* S) {
    S[0] = 0.0;
    S[1] = -0.5 * Q[1];
    S[2] = -0.5 * Q[2];
    S[3] = -0.5 * Q[3];
    S[4] = 0.1 * Q[0];
  }
  void nonConservativeProduct(const double* const Q, const double* const gradQ, double* BgradQ) {
    BgradQ[0] = Q[0];
    BgradQ[1] = Q[3];
    BgradQ[2] = 3.0;
    BgradQ[3] = gradQ[0];
    BgradQ[4] = 0.7;
  }
};

// The kernel tests' linear elastic-wave PDE (exahype/tests/kernels/c/
// ElasticityKernelTest2D.cpp:31-235: 9 variables, parameters lambda, mu, rho),
// restated for the linear kernels; the z parts are the ones written out
// (commented) beside the x and y parts there.
template <int N_>
struct Elastic {
  static constexpr int NumberOfVariables = 9;
  static constexpr int NumberOfParameters = 3;
  static constexpr int Order = N_;
  static constexpr double CFL = 0.9;
  void flux(const double* const, double** F) {
    for (int d = 0; d < DIMENSIONS; d++) std::fill_n(F[d], 9, 0.0);
  }
  void algebraicSource(const double* const, double* S) { std::fill_n(S, 9, 0.0); }
  // boundaryValues (this repository's; the kernel tests define none): kind 0
  // copies the inside state (outflow), kind 1 a rigid wall (the three
  // velocities negated); set per call through boundary_kind
  static thread_local int boundary_kind;
  // pointSource (UserSolverInterface.h:75; this repository's mock, the
  // kernel tests define none): a Ricker wavelet of peak frequency f0 and delay
  // t0, amplitude amp, on the three normal stresses, at x0 whatever x; the
  // parameters x0[3], t0, f0, amp are set per call through point_source
  static thread_local double point_source[6];
  void pointSource(const double* const, const double t, const double, double* forceVector, double* x0) {
    const double r = 3.14159265358979323846 * point_source[4] * (t - point_source[3]);
    const double a = r * r;
    const double w = point_source[5] * ((1.0 - 2.0 * a) * std::exp(-a));
    for (int v = 0; v < 9; v++) forceVector[v] = v < 3 ? w : 0.0;
    for (int d = 0; d < DIMENSIONS; d++) x0[d] = point_source[d];
  }
  void boundaryValues(const double* const, const double, const double, const int, const int,
                      const double* const fluxIn, const double* const stateIn, double* fluxOut, double* stateOut) {
    std::copy_n(stateIn, 12, stateOut);
    std::copy_n(fluxIn, 9, fluxOut);
    if (boundary_kind == 1)
      for (int v = 6; v < 9; v++) stateOut[v] = -stateOut[v];
  }
  void eigenvalues(const double* const Q, const int, double* lambda) {
    std::fill_n(lambda, 9, 0.0);
    const double lam = Q[9], mu = Q[10], rho0 = Q[11];
    const double cp = std::sqrt((lam + 2 * mu) / rho0);
    const double cs = std::sqrt(mu / rho0);
    lambda[0] = -cp;
    lambda[1] = -cs;
    lambda[2] = -cs;
    lambda[3] = 0.0;
    lambda[4] = 0.0;
    lambda[5] = 0.0;
    lambda[6] = +cs;
    lambda[7] = +cs;
    lambda[8] = +cp;
  }
  void nonConservativeProduct(const double* const Q, const double* const gradQ, double* BgradQ) {
    std::fill_n(BgradQ, 9 * DIMENSIONS, 0.0);
    const double lam = Q[9], mu = Q[10], irho = 1.0 / Q[11];
    const double* gx = gradQ;
    const double* gy = gradQ + 9;
    double* bx = BgradQ;
    double* by = BgradQ + 9;
    bx[0] = -(lam + 2 * mu) * gx[6];
    bx[1] = -lam * gx[6];
    bx[2] = -lam * gx[6];
    bx[3] = -mu * gx[7];
    bx[4] = 0.0;
    bx[5] = -mu * gx[8];
    bx[6] = -irho * gx[0];
    bx[7] = -irho * gx[3];
    bx[8] = -irho * gx[5];
    by[0] = -lam * gy[7];
    by[1] = -(lam + 2 * mu) * gy[7];
    by[2] = -lam * gy[7];
    by[3] = -mu * gy[6];
    by[4] = -mu * gy[8];
    by[5] = 0.0;
    by[6] = -irho * gy[3];
    by[7] = -irho * gy[1];
    by[8] = -irho * gy[4];
#if DIMENSIONS == 3
    const double* gz = gradQ + 18;
    double* bz = BgradQ + 18;
    bz[0] = -lam * gz[8];
    bz[1] = -lam * gz[8];
    bz[2] = -(lam + 2 * mu) * gz[8];
    bz[3] = 0.0;
    bz[4] = -mu * gz[7];
    bz[5] = -mu * gz[6];
    bz[6] = -irho * gz[5];
    bz[7] = -irho * gz[4];
    bz[8] = -irho * gz[2];
#endif
  }
  void coefficientMatrix(const double* const Q, const int normalNonZero, double* Bn) {
    std::fill_n(Bn, 81, 0.0);
    const double lam = Q[9], mu = Q[10], irho = 1.0 / Q[11];
#define B(r, c) Bn[(r - 1) * 9 + (c - 1)]
    switch (normalNonZero) {
      case 0:
        B(7, 1) = -(lam + 2 * mu); B(7, 2) = -lam; B(7, 3) = -lam; B(8, 4) = -mu; B(9, 6) = -mu;
        B(1, 7) = -irho; B(4, 8) = -irho; B(6, 9) = -irho;
        break;
      case 1:
        B(8, 1) = -lam; B(8, 2) = -(lam + 2 * mu); B(8, 3) = -lam; B(7, 4) = -mu; B(9, 5) = -mu;
        B(4, 7) = -irho; B(2, 8) = -irho; B(5, 9) = -irho;
        break;
      default:
        B(9, 1) = -lam; B(9, 2) = -lam; B(9, 3) = -(lam + 2 * mu); B(8, 5) = -mu; B(7, 6) = -mu;
        B(6, 7) = -irho; B(5, 8) = -irho; B(3, 9) = -irho;
        break;
    }
#undef B
  }
};

template <int N_>
thread_local int Elastic<N_>::boundary_kind = 0;
template <int N_>
thread_local double Elastic<N_>::point_source[6] = {0, 0, 0, 0, 0, 0};

template <int D> using Vec = tarch::la::Vector<D, double>;

Vec<DIMENSIONS> vec(const double* a) {
  Vec<DIMENSIONS> v;
  for (int d = 0; d < DIMENSIONS; d++) v[d] = a[d];
  return v;
}

constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

// ---- per-cell kernel drivers ------------------------------------------------
template <class S>
int predictor(const double* luh, const double* dxa, double dt, double* lQhbnd, double* lFhbnd, double* lduh,
              double* lQi_out, double* lFi_out, double* lQhi_out, double* lFhi_out) {
  constexpr int b = S::Order + 1;
  constexpr int nV = S::NumberOfVariables, nD = nV + S::NumberOfParameters;
  constexpr int st = ipow(b, DIMENSIONS + 1);
  constexpr int sp = ipow(b, DIMENSIONS);
  static thread_local double lQi[st * nD], rhs[st * nD], lFi[st * (DIMENSIONS + 1) * nV], gradQ[st * DIMENSIONS * nV];
  static thread_local double lQhi[sp * nD], lFhi[sp * (DIMENSIONS + 1) * nV];
  double* stu[2] = {lQi, rhs};
  double* stf[2] = {lFi, gradQ};
  std::fill_n(lFi, st * (DIMENSIONS + 1) * nV, 0.0);
  S s;
  constexpr bool SN = S::kSourceNCP;
  kernels::aderdg::generic::c::spaceTimePredictorNonlinear<SN, true, SN, false, S>(
      s, lQhbnd, lFhbnd, stu, stf, lQhi, lFhi, luh, vec(dxa), dt);
  if (lduh) kernels::aderdg::generic::c::volumeIntegralNonlinear<SN, true, false, nV, b>(lduh, lFi, lFhi, vec(dxa));
  if (lQi_out) std::copy_n(lQi, st * nD, lQi_out);
  if (lFi_out) std::copy_n(lFi, st * (DIMENSIONS + 1) * nV, lFi_out);
  if (lQhi_out) std::copy_n(lQhi, sp * nD, lQhi_out);
  if (lFhi_out) std::copy_n(lFhi, sp * (DIMENSIONS + 1) * nV, lFhi_out);
  return (int)(s.fluxCalls / st);
}

template <class S>
void riemann(double* FL, double* FR, const double* QL, const double* QR, double dt, int dir) {
  S s;
  kernels::aderdg::generic::c::riemannSolverNonlinear<S::kSourceNCP, S>(s, FL, FR, QL, QR, dt, dir);
}

// ADERDGSolver::applyBoundaryConditions (exahype/solvers/ADERDGSolver.cpp:2893-2962)
template <class S>
void boundary_face(double* FIn, const double* QIn, const double* centre, const double* size, double t, double dt,
                   int faceIndex) {
  constexpr int b = S::Order + 1;
  constexpr int nV = S::NumberOfVariables, nD = nV + S::NumberOfParameters;
  constexpr int nf = ipow(b, DIMENSIONS - 1);
  double QOut[nf * nD], FOut[nf * nV];
  S s;
  const int dir = (faceIndex - faceIndex % 2) / 2;
  kernels::aderdg::generic::c::boundaryConditions<S>(s, FOut, QOut, FIn, QIn, vec(centre), vec(size), t, dt,
                                                      faceIndex, dir);
  if (faceIndex % 2 == 0)
    kernels::aderdg::generic::c::riemannSolverNonlinear<S::kSourceNCP, S>(s, FOut, FIn, QOut, QIn, dt, dir);
  else
    kernels::aderdg::generic::c::riemannSolverNonlinear<S::kSourceNCP, S>(s, FIn, FOut, QIn, QOut, dt, dir);
}

template <class S>
void surface(double* lduh, const double* lFhbnd, const double* dxa) {
  kernels::aderdg::generic::c::surfaceIntegralNonlinear<S::NumberOfVariables, S::Order + 1>(lduh, lFhbnd, vec(dxa));
}

template <class S>
void update(double* luh, const double* lduh, double dt) {
  S s;
  kernels::aderdg::generic::c::solutionUpdate<S>(s, luh, lduh, dt);
}

template <class S>
double stable_dt(const double* luh, const double* dxa) {
  S s;
  return kernels::aderdg::generic::c::stableTimeStepSize<S>(s, luh, vec(dxa));
}

// ---- linear kernels ----------------------------------------------------------
// spaceTimePredictorLinear<usePointSource=false, useSource=false,
// useFlux=false, useNCP=true> + volumeIntegralLinear (Toolkit/src/eu/exahype/
// solvers/templates/AbstractGenericADERDGSolverImplementation.template:53-54,85-86)
template <class S>
void lin_predictor(const double* luh, const double* dxa, double dt, double* lQhbnd, double* lFhbnd, double* lduh,
                   double* lQhi_out, double* lFhi_out) {
  constexpr int b = S::Order + 1;
  constexpr int nV = S::NumberOfVariables, nD = nV + S::NumberOfParameters;
  constexpr int sp = ipow(b, DIMENSIONS);
  constexpr int st = sp * b;
  static thread_local double lQi[(st + sp) * nD], lFi[st * (2 * DIMENSIONS + 1) * nV], gradQ[st * DIMENSIONS * nV];
  static thread_local double lQh[sp * nD], lFh[sp * (DIMENSIONS + 1) * nV];
  double* stu[2] = {lQi, nullptr};
  double* stf[2] = {lFi, gradQ};
  S s;
  kernels::aderdg::generic::c::spaceTimePredictorLinear<false, false, false, true, S>(
      s, lQhbnd, lFhbnd, stu, stf, lQh, lFh, luh, vec(dxa), dt, nullptr);
  if (lduh) kernels::aderdg::generic::c::volumeIntegralLinear<false, false, nV, b>(lduh, lFh, vec(dxa));
  if (lQhi_out) std::copy_n(lQh, sp * nD, lQhi_out);
  if (lFhi_out) std::copy_n(lFh, sp * DIMENSIONS * nV, lFhi_out);
}
// pointSource (kernels/aderdg/generic/c/{2d,3d}/pointSource.cpph) for the
// cell with the given centre and widths, into PSi [b+1][b^d][nV]
template <class S>
void point_source(const double* ps, double t, double dt, const double* centre, const double* dxa, double* PSi) {
  S s;
  std::copy_n(ps, 6, S::point_source);
  kernels::aderdg::generic::c::pointSource<S>(s, t, dt, vec(centre), vec(dxa), S::NumberOfVariables,
                                              S::NumberOfParameters, S::Order + 1, PSi);
}
// the same predictor with usePointSource = true, the source of the cell at
// centre evaluated from t over [t, t + dt] (ADERDGSolver.cpp:1929-1960: the
// glue's pointSource, then spaceTimePredictor with its forces)
template <class S>
void lin_predictor_ps(const double* ps, const double* centre, double t, const double* luh, const double* dxa,
                      double dt, double* lQhbnd, double* lFhbnd, double* lduh, double* lQhi_out, double* lFhi_out) {
  constexpr int b = S::Order + 1;
  constexpr int nV = S::NumberOfVariables, nD = nV + S::NumberOfParameters;
  constexpr int sp = ipow(b, DIMENSIONS);
  constexpr int st = sp * b;
  static thread_local double lQi[(st + sp) * nD], lFi[st * (2 * DIMENSIONS + 1) * nV], gradQ[st * DIMENSIONS * nV];
  static thread_local double lQh[sp * nD], lFh[sp * (DIMENSIONS + 1) * nV], PSi[(b + 1) * sp * nV];
  double* stu[2] = {lQi, nullptr};
  double* stf[2] = {lFi, gradQ};
  point_source<S>(ps, t, dt, centre, dxa, PSi);
  S s;
  kernels::aderdg::generic::c::spaceTimePredictorLinear<true, false, false, true, S>(
      s, lQhbnd, lFhbnd, stu, stf, lQh, lFh, luh, vec(dxa), dt, PSi);
  if (lduh) kernels::aderdg::generic::c::volumeIntegralLinear<false, false, nV, b>(lduh, lFh, vec(dxa));
  if (lQhi_out) std::copy_n(lQh, sp * nD, lQhi_out);
  if (lFhi_out) std::copy_n(lFh, sp * DIMENSIONS * nV, lFhi_out);
}
template <class S>
void lin_riemann(double* FL, double* FR, const double* QL, const double* QR, double dt, int dir) {
  S s;
  kernels::aderdg::generic::c::riemannSolverLinear<true, S>(s, FL, FR, QL, QR, dt, dir);
}
// ADERDGSolver::applyBoundaryConditions (exahype/solvers/ADERDGSolver.cpp:2893-2962)
// for a linear solver: boundaryConditions, then riemannSolverLinear
template <class S>
void lin_boundary_face(double* FIn, const double* QIn, int faceIndex, int kind) {
  constexpr int b = S::Order + 1;
  constexpr int nV = S::NumberOfVariables, nD = nV + S::NumberOfParameters;
  constexpr int nf = ipow(b, DIMENSIONS - 1);
  double QOut[nf * nD], FOut[nf * nV];
  S s;
  S::boundary_kind = kind;
  const int dir = (faceIndex - faceIndex % 2) / 2;
  Vec<DIMENSIONS> c(0.5), h(0.1);
  kernels::aderdg::generic::c::boundaryConditions<S>(s, FOut, QOut, FIn, QIn, c, h, 0.0, 0.0, faceIndex, dir);
  if (faceIndex % 2 == 0)
    kernels::aderdg::generic::c::riemannSolverLinear<true, S>(s, FOut, FIn, QOut, QIn, 0.0, dir);
  else
    kernels::aderdg::generic::c::riemannSolverLinear<true, S>(s, FIn, FOut, QIn, QOut, 0.0, dir);
}
template <class S>
void lin_surface(double* lduh, const double* lFhbnd, const double* dxa) {
  kernels::aderdg::generic::c::surfaceIntegralLinear<S::NumberOfVariables, S::Order + 1>(lduh, lFhbnd, vec(dxa));
}
template <class S>
void lin_volume(double* lduh, const double* lFhi, const double* dxa) {
  kernels::aderdg::generic::c::volumeIntegralLinear<false, false, S::NumberOfVariables, S::Order + 1>(lduh, lFhi,
                                                                                                    vec(dxa));
}

// ---- limiter and FV kernels (Euler demonstrator PDE) ------------------------
template <class S>
void project_fv(const double* luh, double* lim) {
  kernels::limiter::generic::c::projectOnFVLimiterSpace(luh, 5, S::Order + 1, S::GhostLayerWidth, lim);
}
template <class S>
void project_dg(const double* lim, double* luh) {
  kernels::limiter::generic::c::projectOnDGSpace(lim, 5, S::Order + 1, S::GhostLayerWidth, luh);
}
template <class S>
void local_minmax(const double* luh, double* mn, double* mx) {
  S s;
  kernels::limiter::generic::c::findCellLocalMinAndMax(luh, &s, mn, mx);
}
template <class S>
void limiter_minmax(const double* lim, double* mn, double* mx) {
  S s;
  kernels::limiter::generic::c::findCellLocalLimiterMinAndMax(lim, &s, S::GhostLayerWidth, mn, mx);
}
template <class S>
int dmp(const double* luh, double relax, double scale, double* mn, double* mx) {
  S s;
  return kernels::limiter::generic::c::discreteMaximumPrincipleAndMinAndMaxSearch(luh, &s, relax, scale, mn, mx);
}
template <class S>
double muscl(double* lnew, const double* lold, const double* dxa, double dt) {
  S s;
  return kernels::finitevolumes::musclhancock::c::solutionUpdate<false, false, true, S>(s, lnew, lold, vec(dxa), dt);
}
template <class S>
void fv_ghost(double* lim, const double* nb, int face) {
  S s;
  tarch::la::Vector<DIMENSIONS, int> pos(0);
  pos[face / 2] = (face % 2) ? 1 : -1;
  kernels::finitevolumes::commons::c::ghostLayerFilling<S>(s, lim, nb, pos);
}
template <class S>
void fv_boundary(double* lim, int face) {
  S s;
  constexpr int P = S::PatchSize, g = S::GhostLayerWidth;
  double in[ipow(P, DIMENSIONS - 1) * g * 5], out[ipow(P, DIMENSIONS - 1) * g * 5];
  tarch::la::Vector<DIMENSIONS, int> pos(0);
  pos[face / 2] = (face % 2) ? 1 : -1;
  Vec<DIMENSIONS> c(0.5), h(0.1);
  kernels::finitevolumes::commons::c::boundaryLayerExtraction<S>(s, in, lim, pos);
  kernels::finitevolumes::commons::c::boundaryConditions<S>(s, out, in, c, h, 0.0, 0.0, face, face / 2);
  kernels::finitevolumes::commons::c::ghostLayerFillingAtBoundary<S>(s, lim, out, pos);
}

// ---- AMR transfer operators (amrRoutines.cpph) and the plotter's projection --
template <int nV, int nP, int b>
void amr_call(int op, double* a, double* bb, const double* c, const double* d, int levelDelta, const int* index) {
  tarch::la::Vector<DIMENSIONS, int> cell;
  tarch::la::Vector<DIMENSIONS - 1, int> face;
  for (int k = 0; k < DIMENSIONS; k++) cell[k] = index[k];
  for (int k = 0; k < DIMENSIONS - 1; k++) face[k] = index[k];
  namespace K = kernels::aderdg::generic::c;
  switch (op) {
    case 0: K::volumeUnknownsProlongation<nV, nP, b>(a, c, 0, levelDelta, cell); break;
    case 1: K::volumeUnknownsRestriction<nV, nP, b>(a, c, 0, levelDelta, cell); break;
    case 2: K::faceUnknownsProlongation<nV, nP, b>(a, bb, c, d, 0, levelDelta, face); break;
    default: K::faceUnknownsRestriction<nV, nP, b>(a, bb, c, d, 0, levelDelta, face); break;
  }
}

// ADERDG2CartesianVTK::plotVertexData (exahype/plotters/VTK/ADERDG2CartesianVTK.cpp):
// the solution at the (N+1)^d equidistant vertices of a cell, x fastest
void plot_vertices(int N, int nvar, const double* u, double* out) {
  const int b = N + 1, nz = DIMENSIONS == 3 ? b : 1;
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < b; iy++)
      for (int ix = 0; ix < b; ix++)
        for (int v = 0; v < nvar; v++) {
          double acc = 0.0;
          for (int gz = 0; gz < nz; gz++)
            for (int gy = 0; gy < b; gy++)
              for (int gx = 0; gx < b; gx++) {
                const int g = (gz * b + gy) * b + gx;
                acc += kernels::equidistantGridProjector1d[N][gy][iy] * kernels::equidistantGridProjector1d[N][gx][ix] *
#if DIMENSIONS == 3
                       kernels::equidistantGridProjector1d[N][gz][iz] *
#endif
                       u[g * nvar + v];
              }
          out[((iz * b + iy) * b + ix) * nvar + v] = acc;
        }
}

}  // namespace

#define DISPATCH_ELASTIC(N, call)                                        \
  do {                                                                  \
    switch (N) {                                                        \
      case 3: { typedef Elastic<3> S; call; } break;                    \
      case 4: { typedef Elastic<4> S; call; } break;                    \
      case 5: { typedef Elastic<5> S; call; } break;                    \
      default: std::fprintf(stderr, "ref: order %d not built\n", N);   \
    }                                                                   \
  } while (0)

// linear kernels: the elastic-wave PDE, or (pde 1) the Euler mock
#define DISPATCH_LIN(pde, N, call)                                       \
  do {                                                                  \
    if (pde == 2 || pde == 4) {                                         \
      DISPATCH_ELASTIC(N, call);                                        \
    } else {                                                            \
      switch (N) {                                                      \
        case 3: { typedef EulerTest<3> S; call; } break;                \
        case 5: { typedef EulerTest<5> S; call; } break;                \
        default: std::fprintf(stderr, "ref: order %d not built\n", N); \
      }                                                                 \
    }                                                                   \
  } while (0)

#define DISPATCH(pde, N, call)                                              \
  do {                                                                      \
    if (pde == 0) {                                                         \
      switch (N) {                                                          \
        case 3: { typedef EulerDemo<3> S; call; } break;                    \
        case 4: { typedef EulerDemo<4> S; call; } break;                    \
        case 5: { typedef EulerDemo<5> S; call; } break;                    \
        case 7: { typedef EulerDemo<7> S; call; } break;                    \
        default: std::fprintf(stderr, "ref: order %d not built\n", N);     \
      }                                                                     \
    } else if (pde == 3) {                                                  \
      switch (N) {                                                          \
        case 3: { typedef EulerSourceNCP<3> S; call; } break;               \
        case 5: { typedef EulerSourceNCP<5> S; call; } break;               \
        default: std::fprintf(stderr, "ref: order %d not built\n", N);     \
      }                                                                     \
    } else {                                                                \
      switch (N) {                                                          \
        case 3: { typedef EulerTest<3> S; call; } break;                    \
        case 5: { typedef EulerTest<5> S; call; } break;                    \
        default: std::fprintf(stderr, "ref: order %d not built\n", N);     \
      }                                                                     \
    }                                                                       \
  } while (0)

// limiter / FV kernels exist for the demonstrator PDE only
#define DISPATCH_EULER(N, call)                                          \
  do {                                                                  \
    switch (N) {                                                        \
      case 3: { typedef EulerDemo<3> S; call; } break;                  \
      case 4: { typedef EulerDemo<4> S; call; } break;                  \
      case 5: { typedef EulerDemo<5> S; call; } break;                  \
      case 7: { typedef EulerDemo<7> S; call; } break;                  \
      default: std::fprintf(stderr, "ref: order %d not built\n", N);   \
    }                                                                   \
  } while (0)

extern "C" {

void REFNAME(init)() {
  static bool done = false;
  if (done) return;
  std::set<int> orders;
  kernels::initGaussLegendreNodesAndWeights(orders);
  kernels::initGaussLobattoNodesAndWeights(orders);
  kernels::initDGMatrices(orders);
  kernels::initLimiterProjectionMatrices(orders);
  kernels::initBasisFunctions(orders);
  done = true;
}

// Copies one of the reference's operator tables for order N into out.
// Returns the number of doubles written, or -1 for an unknown name.
int REFNAME(table)(const char* name, int N, double* out) {
  REFNAME(init)();
  const int b = N + 1, bl = 2 * N + 1;
  int k = 0;
  if (!std::strcmp(name, "weights")) { for (int i = 0; i < b; i++) out[k++] = kernels::gaussLegendreWeights[N][i]; }
  else if (!std::strcmp(name, "nodes")) { for (int i = 0; i < b; i++) out[k++] = kernels::gaussLegendreNodes[N][i]; }
  else if (!std::strcmp(name, "lobatto_nodes")) { for (int i = 0; i < b; i++) out[k++] = kernels::gaussLobattoNodes[N][i]; }
  else if (!std::strcmp(name, "lobatto_weights")) { for (int i = 0; i < b; i++) out[k++] = kernels::gaussLobattoWeights[N][i]; }
  else if (!std::strcmp(name, "FLCoeff")) { for (int i = 0; i < b; i++) out[k++] = kernels::FLCoeff[N][i]; }
  else if (!std::strcmp(name, "FRCoeff")) { for (int i = 0; i < b; i++) out[k++] = kernels::FRCoeff[N][i]; }
  else if (!std::strcmp(name, "FCoeff")) { for (int s = 0; s < 2; s++) for (int i = 0; i < b; i++) out[k++] = kernels::FCoeff[N][s][i]; }
  else if (!std::strcmp(name, "Kxi")) { for (int i = 0; i < b; i++) for (int j = 0; j < b; j++) out[k++] = kernels::Kxi[N][i][j]; }
  else if (!std::strcmp(name, "iK1")) { for (int i = 0; i < b; i++) for (int j = 0; j < b; j++) out[k++] = kernels::iK1[N][i][j]; }
  else if (!std::strcmp(name, "dudx")) { for (int i = 0; i < b; i++) for (int j = 0; j < b; j++) out[k++] = kernels::dudx[N][i][j]; }
  else if (!std::strcmp(name, "uh2lim")) { for (int i = 0; i < b * bl; i++) out[k++] = kernels::uh2lim[N][i]; }
  else if (!std::strcmp(name, "lim2uh")) { for (int i = 0; i < b * bl; i++) out[k++] = kernels::lim2uh[N][i]; }
  else if (!std::strcmp(name, "uh2lob")) { for (int i = 0; i < b * b; i++) out[k++] = kernels::uh2lob[N][i]; }
  else if (!std::strcmp(name, "fineGridProjector1d")) {
    for (int j = 0; j < 3; j++) for (int n = 0; n < b; n++) for (int m = 0; m < b; m++) out[k++] = kernels::fineGridProjector1d[N][j][n][m];
  } else if (!std::strcmp(name, "equidistantGridProjector1d")) {
    for (int n = 0; n < b; n++) for (int i = 0; i < b; i++) out[k++] = kernels::equidistantGridProjector1d[N][n][i];
  }
  else return -1;
  return k;
}

int REFNAME(predictor)(int pde, int N, const double* luh, const double* dx, double dt, double* lQhbnd,
                       double* lFhbnd, double* lduh, double* lQi, double* lFi, double* lQhi, double* lFhi) {
  REFNAME(init)();
  int it = -1;
  DISPATCH(pde, N, it = predictor<S>(luh, dx, dt, lQhbnd, lFhbnd, lduh, lQi, lFi, lQhi, lFhi));
  return it;
}

void REFNAME(riemann)(int pde, int N, double* FL, double* FR, const double* QL, const double* QR, double dt,
                      int dir) {
  REFNAME(init)();
  DISPATCH(pde, N, riemann<S>(FL, FR, QL, QR, dt, dir));
}

void REFNAME(boundary_face)(int pde, int N, double* FIn, const double* QIn, const double* centre,
                            const double* size, double t, double dt, int faceIndex) {
  REFNAME(init)();
  DISPATCH(pde, N, boundary_face<S>(FIn, QIn, centre, size, t, dt, faceIndex));
}

void REFNAME(surface_integral)(int pde, int N, double* lduh, const double* lFhbnd, const double* dx) {
  REFNAME(init)();
  DISPATCH(pde, N, surface<S>(lduh, lFhbnd, dx));
}

void REFNAME(solution_update)(int pde, int N, double* luh, const double* lduh, double dt) {
  REFNAME(init)();
  if (pde == 2 || pde == 4) DISPATCH_ELASTIC(N, update<S>(luh, lduh, dt));
  else DISPATCH(pde, N, update<S>(luh, lduh, dt));
}

void REFNAME(project_fv)(int N, const double* luh, double* lim) { REFNAME(init)(); DISPATCH_EULER(N, project_fv<S>(luh, lim)); }
void REFNAME(project_dg)(int N, const double* lim, double* luh) { REFNAME(init)(); DISPATCH_EULER(N, project_dg<S>(lim, luh)); }
void REFNAME(local_minmax)(int N, const double* luh, double* mn, double* mx) {
  REFNAME(init)();
  DISPATCH_EULER(N, local_minmax<S>(luh, mn, mx));
}
void REFNAME(limiter_minmax)(int N, const double* lim, double* mn, double* mx) {
  REFNAME(init)();
  DISPATCH_EULER(N, limiter_minmax<S>(lim, mn, mx));
}
int REFNAME(dmp)(int N, const double* luh, double relax, double scale, double* mn, double* mx) {
  REFNAME(init)();
  int r = -1;
  DISPATCH_EULER(N, r = dmp<S>(luh, relax, scale, mn, mx));
  return r;
}
double REFNAME(musclhancock)(int N, double* lnew, const double* lold, const double* dx, double dt) {
  REFNAME(init)();
  double r = 0;
  DISPATCH_EULER(N, r = muscl<S>(lnew, lold, dx, dt));
  return r;
}
void REFNAME(fv_ghost)(int N, double* lim, const double* nb, int face) { DISPATCH_EULER(N, fv_ghost<S>(lim, nb, face)); }
void REFNAME(fv_boundary)(int N, double* lim, int face) { DISPATCH_EULER(N, fv_boundary<S>(lim, face)); }
// the demonstrator's Euler PDE with the boundary kind of the domain face
// (0 outflow, 1 reflective): FV ghost layers, DG boundary face
void REFNAME(fv_boundary_kind)(int N, double* lim, int face, int kind) {
  DISPATCH_EULER(N, { S::boundary_kind = kind; fv_boundary<S>(lim, face); S::boundary_kind = 0; });
}
void REFNAME(boundary_face_kind)(int N, double* FIn, const double* QIn, int faceIndex, int kind) {
  REFNAME(init)();
  const double c[3] = {0.5, 0.5, 0.5}, h[3] = {0.1, 0.1, 0.1};
  DISPATCH_EULER(N, { S::boundary_kind = kind; boundary_face<S>(FIn, QIn, c, h, 0.0, 0.0, faceIndex); S::boundary_kind = 0; });
}

double REFNAME(stable_dt)(int pde, int N, const double* luh, const double* dx) {
  REFNAME(init)();
  double r = -1;
  if (pde == 2 || pde == 4) DISPATCH_ELASTIC(N, r = stable_dt<S>(luh, dx));
  else DISPATCH(pde, N, r = stable_dt<S>(luh, dx));
  return r;
}

// op: 0 volume prolongation (a = fine, c = coarse), 1 volume restriction
// (a = coarse += , c = fine), 2 face prolongation (a, bb = fine state, flux;
// c, d = coarse), 3 face restriction (a, bb = coarse +=; c, d = fine);
// (nv, np) = variables, parameters
int REFNAME(amr)(int op, int nv, int np, int N, double* a, double* bb, const double* c, const double* d,
                 int levelDelta, const int* index) {
  REFNAME(init)();
#define AMR_N(NV, NP)                                                                           \
  if (nv == NV && np == NP) {                                                                   \
    switch (N) {                                                                                \
      case 3: amr_call<NV, NP, 4>(op, a, bb, c, d, levelDelta, index); return 0;                \
      case 4: amr_call<NV, NP, 5>(op, a, bb, c, d, levelDelta, index); return 0;                \
      case 5: amr_call<NV, NP, 6>(op, a, bb, c, d, levelDelta, index); return 0;                \
      default: return -1;                                                                       \
    }                                                                                           \
  }
  AMR_N(5, 0)
  AMR_N(5, 1)
  AMR_N(9, 3)
  AMR_N(1, 1)
#undef AMR_N
  return -1;
}

void REFNAME(plot_vertices)(int N, int nvar, const double* u, double* out) {
  REFNAME(init)();
  plot_vertices(N, nvar, u, out);
}

void REFNAME(lin_predictor)(int pde, int N, const double* luh, const double* dx, double dt, double* lQhbnd,
                            double* lFhbnd, double* lduh, double* lQhi, double* lFhi) {
  REFNAME(init)();
  DISPATCH_ELASTIC(N, lin_predictor<S>(luh, dx, dt, lQhbnd, lFhbnd, lduh, lQhi, lFhi));
  (void)pde;
}
void REFNAME(lin_riemann)(int pde, int N, double* FL, double* FR, const double* QL, const double* QR, double dt,
                          int dir) {
  REFNAME(init)();
  DISPATCH_LIN(pde, N, lin_riemann<S>(FL, FR, QL, QR, dt, dir));
}
void REFNAME(lin_boundary_face)(int pde, int N, double* FIn, const double* QIn, int faceIndex, int kind) {
  REFNAME(init)();
  if (pde != 2 && pde != 4) return;
  DISPATCH_ELASTIC(N, lin_boundary_face<S>(FIn, QIn, faceIndex, kind));
}
void REFNAME(point_source)(int N, const double* ps, double t, double dt, const double* centre, const double* dx,
                           double* PSi) {
  REFNAME(init)();
  DISPATCH_ELASTIC(N, point_source<S>(ps, t, dt, centre, dx, PSi));
}
void REFNAME(lin_predictor_ps)(int N, const double* ps, const double* centre, double t, const double* luh,
                               const double* dx, double dt, double* lQhbnd, double* lFhbnd, double* lduh,
                               double* lQhi, double* lFhi) {
  REFNAME(init)();
  DISPATCH_ELASTIC(N, lin_predictor_ps<S>(ps, centre, t, luh, dx, dt, lQhbnd, lFhbnd, lduh, lQhi, lFhi));
}
void REFNAME(lin_surface_integral)(int pde, int N, double* lduh, const double* lFhbnd, const double* dx) {
  REFNAME(init)();
  DISPATCH_LIN(pde, N, lin_surface<S>(lduh, lFhbnd, dx));
}
void REFNAME(lin_volume_integral)(int pde, int N, double* lduh, const double* lFhi, const double* dx) {
  REFNAME(init)();
  DISPATCH_LIN(pde, N, lin_volume<S>(lduh, lFhi, dx));
}

}  // extern "C"
