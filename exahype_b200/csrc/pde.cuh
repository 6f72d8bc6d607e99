// User-PDE hooks as __device__ functors. A PDE type provides what the
// reference's UserSolverInterface (exahype/solvers/UserSolverInterface.h:42-203)
// asks of a nonlinear conservative solver:
//   nVar, nPar                      -- NumberOfVariables / NumberOfParameters
//   flux<DIM>(Q, F[DIM][nVar])      -- flux(Q, F)
//   eigenvalues(Q, d, lambda)       -- eigenvalues(Q, normalNonZero, lambda)
//   boundaryValues(...)             -- boundaryValues(x,t,dt,faceIndex,normal,FIn,QIn,FOut,QOut)
//   fvBoundaryValues(...)           -- the FV solver's boundaryValues(x,t,dt,faceIndex,normal,QIn,QOut)
//   isPhysicallyAdmissible(min,max) -- isPhysicallyAdmissible(...)
//   observables(Q, obs)             -- mapDiscreteMaximumPrincipleObservables(...)
// New PDEs are added by writing such a struct and instantiating the kernel
// templates for it (see capi.cu).
#pragma once
#include <cuda_runtime.h>

namespace exa {

// Boundary-condition kinds handed to boundaryValues.
enum BoundaryKind : int { kOutflow = 0, kReflective = 1 };

// Compressible Euler, 5 conserved variables (rho, j[3], E), gamma = 1.4, as in
// Demonstrators/EulerADERDG/MyEulerSolver_ADERDG.cpp:102-160. The pressure uses
// all three momentum components in 2D too.
struct EulerPDE {
  static constexpr int nVar = 5;
  static constexpr int nPar = 0;
  static constexpr int nObs = 5;

  __host__ __device__ static double pressure(const double* Q, double irho) {
    const double GAMMA = 1.4;
    const double jj = Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3];
    return (GAMMA - 1) * (Q[4] - 0.5 * irho * jj);
  }

  template <int DIM>
  __device__ static void flux(const double* Q, double (*F)[nVar]) {
    const double irho = 1. / Q[0];
    const double p = pressure(Q, irho);
    const double e = irho * (Q[4] + p);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      F[d][0] = Q[1 + d];
#pragma unroll
      for (int a = 0; a < 3; a++) F[d][1 + a] = irho * (Q[1 + d] * Q[1 + a]) + (d == a ? p : 0.0);
      F[d][4] = e * Q[1 + d];
    }
  }

  __device__ static void eigenvalues(const double* Q, int d, double* lambda) {
    const double irho = 1. / Q[0];
    const double p = pressure(Q, irho);
    const double u_n = Q[d + 1] * irho;
    const double c = sqrt(1.4 * p * irho);
    lambda[0] = u_n - c;
    lambda[1] = u_n;
    lambda[2] = u_n;
    lambda[3] = u_n;
    lambda[4] = u_n + c;
  }

  // max_v |lambda_v(Q, d)| evaluated with IEEE round-to-nearest operations and
  // no contraction, so that the time-step size matches the reference bit for bit.
  __device__ static double max_abs_eigenvalue_exact(const double* Q, int d) {
    const double irho = __ddiv_rn(1.0, Q[0]);
    const double jj = __dadd_rn(__dadd_rn(__dmul_rn(Q[1], Q[1]), __dmul_rn(Q[2], Q[2])), __dmul_rn(Q[3], Q[3]));
    const double p = __dmul_rn(1.4 - 1, __dsub_rn(Q[4], __dmul_rn(__dmul_rn(0.5, irho), jj)));
    const double u_n = __dmul_rn(Q[d + 1], irho);
    const double c = __dsqrt_rn(__dmul_rn(__dmul_rn(1.4, p), irho));
    const double l0 = fabs(__dsub_rn(u_n, c)), l1 = fabs(u_n), l4 = fabs(__dadd_rn(u_n, c));
    // std::max(|lambda_v|, running max) over v = 0..4, starting from 0.0
    double m = 0.0;
    m = (l0 < m) ? m : l0;
    m = (l1 < m) ? m : l1;
    m = (l1 < m) ? m : l1;
    m = (l1 < m) ? m : l1;
    m = (l4 < m) ? m : l4;
    return m;
  }

  // kOutflow: QOut = QIn, FOut = FIn. kReflective: the demonstrator's
  // MyEulerSolver_ADERDG.cpp:67-88 (mirror the normal momentum, recompute F).
  template <int DIM>
  __device__ static void boundaryValues(int kind, int normal, const double* FIn, const double* QIn, double* FOut,
                                        double* QOut) {
    for (int v = 0; v < nVar + nPar; v++) QOut[v] = QIn[v];
    if (kind == kReflective) {
      QOut[1 + normal] = -QOut[1 + normal];
      double F[DIM][nVar];
      flux<DIM>(QOut, F);
      for (int v = 0; v < nVar; v++) FOut[v] = F[normal][v];
    } else {
      for (int v = 0; v < nVar; v++) FOut[v] = FIn[v];
    }
  }

  __device__ static void fvBoundaryValues(int kind, int normal, const double* QIn, double* QOut) {
    for (int v = 0; v < nVar + nPar; v++) QOut[v] = QIn[v];
    if (kind == kReflective) QOut[1 + normal] = -QOut[1 + normal];
  }

  // MyEulerSolver_ADERDG.cpp:137-145: the observables are the conserved variables.
  __device__ static void observables(const double* Q, double* obs) {
    for (int v = 0; v < nObs; v++) obs[v] = Q[v];
  }
  // MyEulerSolver_ADERDG.cpp:147-160: density and energy must stay positive.
  __device__ static bool isPhysicallyAdmissible(const double* obsMin, const double* /*obsMax*/) {
    if (obsMin[0] <= 0.0) return false;
    if (obsMin[4] <= 0.0) return false;
    return true;
  }
};

// The mock PDE of the reference kernel tests (exahype/tests/kernels/c/
// GenericEulerKernelTest2D.cpp:28-77, ...3D.cpp:26-77): Euler with one material
// parameter; in 2D the pressure only sees the x and y momentum ("2.5D").
// It exists so the reference's golden vectors can be replayed on the GPU.
struct EulerTestPDE {
  static constexpr int nVar = 5;
  static constexpr int nPar = 1;
  static constexpr int nObs = 5;

  template <int DIM>
  __host__ __device__ static double pressure(const double* Q, double irho) {
    const double GAMMA = 1.4;
    if (DIM == 2) return (GAMMA - 1) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) * irho);
    return (GAMMA - 1) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) * irho);
  }

  template <int DIM>
  __device__ static void flux(const double* Q, double (*F)[nVar]) {
    const double irho = 1.0 / Q[0];
    const double p = pressure<DIM>(Q, irho);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      F[d][0] = Q[1 + d];
#pragma unroll
      for (int a = 0; a < 3; a++) F[d][1 + a] = irho * Q[1 + d] * Q[1 + a] + (d == a ? p : 0.0);
      F[d][4] = irho * Q[1 + d] * (Q[4] + p);
    }
  }

  template <int DIM>
  __device__ static void eigenvalues_dim(const double* Q, int d, double* lambda) {
    const double irho = 1.0 / Q[0];
    const double p = pressure<DIM>(Q, irho);
    const double u_n = Q[d + 1] * irho;
    const double c = sqrt(1.4 * p * irho);
    lambda[0] = u_n - c;
    lambda[1] = u_n;
    lambda[2] = u_n;
    lambda[3] = u_n;
    lambda[4] = u_n + c;
  }
  // the face kernels call eigenvalues(Q, d, lambda); the 2.5D pressure needs the
  // dimension, which the kernels pass through eigenvalues_dim.
  template <int DIM>
  __device__ static double max_abs_eigenvalue_exact(const double* Q, int d) {
    const double irho = __ddiv_rn(1.0, Q[0]);
    double jj = __dadd_rn(__dmul_rn(Q[1], Q[1]), __dmul_rn(Q[2], Q[2]));
    if (DIM == 3) jj = __dadd_rn(jj, __dmul_rn(Q[3], Q[3]));
    const double p = __dmul_rn(1.4 - 1, __dsub_rn(Q[4], __dmul_rn(__dmul_rn(0.5, jj), irho)));
    const double u_n = __dmul_rn(Q[d + 1], irho);
    const double c = __dsqrt_rn(__dmul_rn(__dmul_rn(1.4, p), irho));
    const double l0 = fabs(__dsub_rn(u_n, c)), l1 = fabs(u_n), l4 = fabs(__dadd_rn(u_n, c));
    double m = 0.0;
    m = (l0 < m) ? m : l0;
    m = (l1 < m) ? m : l1;
    m = (l4 < m) ? m : l4;
    return m;
  }
  template <int DIM>
  __device__ static void boundaryValues(int, int, const double* FIn, const double* QIn, double* FOut, double* QOut) {
    for (int v = 0; v < nVar + nPar; v++) QOut[v] = QIn[v];
    for (int v = 0; v < nVar; v++) FOut[v] = FIn[v];
  }
  __device__ static void fvBoundaryValues(int, int, const double* QIn, double* QOut) {
    for (int v = 0; v < nVar + nPar; v++) QOut[v] = QIn[v];
  }
  __device__ static void observables(const double* Q, double* obs) {
    for (int v = 0; v < nObs; v++) obs[v] = Q[v];
  }
  __device__ static bool isPhysicallyAdmissible(const double* obsMin, const double*) {
    if (obsMin[0] <= 0.0) return false;
    if (obsMin[4] <= 0.0) return false;
    return true;
  }
};

// Uniform access for the kernels: eigenvalues and the exact max-eigenvalue
// for either PDE, given the dimension.
template <class PDE, int DIM>
struct Hooks {
  __device__ static void eigenvalues(const double* Q, int d, double* l) { PDE::eigenvalues(Q, d, l); }
  __device__ static double max_abs_eig_exact(const double* Q, int d) { return PDE::max_abs_eigenvalue_exact(Q, d); }
};
template <int DIM>
struct Hooks<EulerTestPDE, DIM> {
  __device__ static void eigenvalues(const double* Q, int d, double* l) { EulerTestPDE::eigenvalues_dim<DIM>(Q, d, l); }
  __device__ static double max_abs_eig_exact(const double* Q, int d) {
    return EulerTestPDE::max_abs_eigenvalue_exact<DIM>(Q, d);
  }
};

}  // namespace exa
