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
//   kSource, kNCP                   -- the generated glue's useSource / useNCP
// and, where kSource / kNCP are set,
//   algebraicSource(Q, S[nVar])                     -- algebraicSource(Q, S)
//   ncp<DIM>(Q, gradQ[DIM][nVar], BgradQ[nVar])     -- nonConservativeProduct(Q, gradQ, BgradQ)
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
  static constexpr bool kLinear = false;  // nonlinear kernels (Picard predictor, Rusanov on fluxes)
  static constexpr bool kSource = false, kNCP = false;

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
  static constexpr bool kLinear = false;
  static constexpr bool kSource = false, kNCP = false;

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

// The kernel-test mock with an algebraic source and a non-conservative
// product switched on (useSource = useNCP = true): the source is this
// library's choice (momentum damping, an energy source proportional to the
// density), the product is the tests' non-zero mock
// (exahype/tests/kernels/c/GenericEulerKernelTest3D.cpp:84-110, 2D :80-103,
// with _setNcpAndMatrixBToZero false). It exercises the predictor's source
// branch (3d/spaceTimePredictorNonlinear.cpph:238-276), the time-averaged
// source of the volume integral and the Riemann solver's fluctuations
// (3d/riemannSolverNonlinear.cpph:92-110).
struct EulerSourceNCPPDE : EulerTestPDE {
  static constexpr bool kSource = true, kNCP = true;
  __device__ static void algebraicSource(const double* Q, double* S) {
    S[0] = 0.0;
    S[1] = -0.5 * Q[1];
    S[2] = -0.5 * Q[2];
    S[3] = -0.5 * Q[3];
    S[4] = 0.1 * Q[0];
  }
  template <int DIM>
  __device__ static void ncp(const double* Q, const double (*G)[nVar], double* B) {
    B[0] = Q[0];
    B[1] = Q[3];
    B[2] = 3.0;
    B[3] = G[0][0];
    B[4] = 0.7;
  }
};

// Linear elastic waves in velocity-stress form, the PDE of the reference's
// linear kernel tests (exahype/tests/kernels/c/ElasticityKernelTest2D.cpp:
// 31-235): variables sxx syy szz sxy syz sxz u v w, material parameters
// lambda mu rho. A linear PDE supplies what the reference's linear kernels
// ask of the user solver instead of a flux:
//   ncp<DIM>(Q, gradQ[DIM][nVar], BgradQ[DIM][nVar]) -- nonConservativeProduct
//                                                       (BgradQ a DIM x nVar tensor)
//   ncp_dir(Q, d, gradQ_d, BgradQ_d)                  -- its direction-d part
//   coefficient_matrix(Q, d, Bn[nVar][nVar])          -- coefficientMatrix
//   eigenvalues(Q, d, lambda)                         -- eigenvalues
// with (BgradQ_d)_k = sum_l Bn_d[l][k] (gradQ_d)_l, and
//   ncp_uses(d, v)  which gradient components ncp reads (no counterpart in
//                   the reference, which computes them all). The z-direction parts are
// the ones written out (commented) beside the x and y parts in the test.
struct ElasticPDE {
  static constexpr int nVar = 9;
  static constexpr int nPar = 3;
  static constexpr int nObs = 9;
  static constexpr bool kLinear = true;
  static constexpr bool kSource = false, kNCP = false;  // (its product enters the linear kernels directly)
  static constexpr bool kPointSource = false;           // the generated glue's usePointSource

  // boundaryValues (this library's; the reference's kernel tests define
  // none for this PDE): kOutflow copies the inside state, kReflective is a
  // rigid wall, the inside state with the three velocities negated; the
  // material parameters are copied
  template <int DIM>
  __device__ static void boundaryValues(int kind, int /*normal*/, const double* FIn, const double* QIn, double* FOut,
                                        double* QOut) {
    for (int v = 0; v < nVar + nPar; v++) QOut[v] = QIn[v];
    if (kind == kReflective)
      for (int v = 6; v < 9; v++) QOut[v] = -QOut[v];
    for (int v = 0; v < nVar; v++) FOut[v] = FIn[v];
  }

  // the product of one direction: B_d = B_d(Q) gradQ_d (a linear PDE's
  // product separates by direction)
  __device__ static void ncp_dir(const double* Q, int d, const double* G, double* B) {
    const double lam = Q[9], mu = Q[10], irho = 1.0 / Q[11];
    const double lm2 = lam + 2 * mu;
    if (d == 0) {
      B[0] = -lm2 * G[6];
      B[1] = -lam * G[6];
      B[2] = -lam * G[6];
      B[3] = -mu * G[7];
      B[4] = 0.0;
      B[5] = -mu * G[8];
      B[6] = -irho * G[0];
      B[7] = -irho * G[3];
      B[8] = -irho * G[5];
    } else if (d == 1) {
      B[0] = -lam * G[7];
      B[1] = -lm2 * G[7];
      B[2] = -lam * G[7];
      B[3] = -mu * G[6];
      B[4] = -mu * G[8];
      B[5] = 0.0;
      B[6] = -irho * G[3];
      B[7] = -irho * G[1];
      B[8] = -irho * G[4];
    } else {
      B[0] = -lam * G[8];
      B[1] = -lam * G[8];
      B[2] = -lm2 * G[8];
      B[3] = 0.0;
      B[4] = -mu * G[7];
      B[5] = -mu * G[6];
      B[6] = -irho * G[5];
      B[7] = -irho * G[4];
      B[8] = -irho * G[2];
    }
  }

  template <int DIM>
  __device__ static void ncp(const double* Q, const double (*G)[nVar], double (*B)[nVar]) {
#pragma unroll
    for (int d = 0; d < DIM; d++) ncp_dir(Q, d, G[d], B[d]);
  }

  // which gradient components ncp reads: direction d, variable v (the
  // predictor computes only these; the others would not change its result)
  __host__ __device__ static constexpr bool ncp_uses(int d, int v) {
    return d == 0 ? (v == 0 || v == 3 || v == 5 || v >= 6)
         : d == 1 ? (v == 1 || v == 3 || v == 4 || v >= 6)
                  : (v == 2 || v == 4 || v == 5 || v >= 6);
  }

  // Bn row-major [l][k], all other entries zero
  __device__ static void coefficient_matrix(const double* Q, int d, double* Bn) {
    for (int i = 0; i < nVar * nVar; i++) Bn[i] = 0.0;
    const double lam = Q[9], mu = Q[10], irho = 1.0 / Q[11];
    const double lm2 = lam + 2 * mu;
    if (d == 0) {
      Bn[6 * 9 + 0] = -lm2; Bn[6 * 9 + 1] = -lam; Bn[6 * 9 + 2] = -lam; Bn[7 * 9 + 3] = -mu; Bn[8 * 9 + 5] = -mu;
      Bn[0 * 9 + 6] = -irho; Bn[3 * 9 + 7] = -irho; Bn[5 * 9 + 8] = -irho;
    } else if (d == 1) {
      Bn[7 * 9 + 0] = -lam; Bn[7 * 9 + 1] = -lm2; Bn[7 * 9 + 2] = -lam; Bn[6 * 9 + 3] = -mu; Bn[8 * 9 + 4] = -mu;
      Bn[3 * 9 + 6] = -irho; Bn[1 * 9 + 7] = -irho; Bn[4 * 9 + 8] = -irho;
    } else {
      Bn[8 * 9 + 0] = -lam; Bn[8 * 9 + 1] = -lam; Bn[8 * 9 + 2] = -lm2; Bn[7 * 9 + 4] = -mu; Bn[6 * 9 + 5] = -mu;
      Bn[5 * 9 + 6] = -irho; Bn[4 * 9 + 7] = -irho; Bn[2 * 9 + 8] = -irho;
    }
  }

  __device__ static void eigenvalues(const double* Q, int /*d*/, double* lambda) {
    const double lam = Q[9], mu = Q[10], rho = Q[11];
    const double cp = sqrt((lam + 2 * mu) / rho);
    const double cs = sqrt(mu / rho);
    lambda[0] = -cp;
    lambda[1] = -cs;
    lambda[2] = -cs;
    lambda[3] = 0.0;
    lambda[4] = 0.0;
    lambda[5] = 0.0;
    lambda[6] = cs;
    lambda[7] = cs;
    lambda[8] = cp;
  }

  // max_v |lambda_v| with round-to-nearest operations (max(cp, cs) is exact
  // in any order), so that the time step matches the reference bit for bit
  __device__ static double max_abs_eigenvalue_exact(const double* Q, int /*d*/) {
    const double lam = Q[9], mu = Q[10], rho = Q[11];
    const double cp = __dsqrt_rn(__ddiv_rn(__dadd_rn(lam, __dmul_rn(2.0, mu)), rho));
    const double cs = __dsqrt_rn(__ddiv_rn(mu, rho));
    return (cp < cs) ? cs : cp;
  }
};

// ElasticPDE with a point source (usePointSource = true): the source of this
// library's point-source mock (the reference's kernel tests define none), a
// Ricker wavelet of peak frequency f0 and delay t0, amplitude amp, on the
// three normal stresses, located at x0 whatever the node position x
// (UserSolverInterface::pointSource(x, t, dt, forceVector, x0),
// exahype/solvers/UserSolverInterface.h:75). ps = {x0[3], t0, f0, amp} comes
// from the solver. sourcePosition gives x0 without a node: the kernels skip
// the cells whose closed box does not hold it.
struct ElasticPointSourcePDE : ElasticPDE {
  static constexpr bool kPointSource = true;
  __device__ static void pointSource(const double* /*x*/, double t, double /*dt*/, double* force, double* x0,
                                     const double* ps) {
    const double r = (3.14159265358979323846 * ps[4]) * (t - ps[3]);
    const double a = r * r;
    const double w = ps[5] * ((1.0 - 2.0 * a) * exp(-a));
#pragma unroll
    for (int v = 0; v < nVar; v++) force[v] = v < 3 ? w : 0.0;
    sourcePosition(ps, x0);
  }
  __device__ static void sourcePosition(const double* ps, double* x0) {
    for (int d = 0; d < 3; d++) x0[d] = ps[d];
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
template <int DIM>
struct Hooks<EulerSourceNCPPDE, DIM> : Hooks<EulerTestPDE, DIM> {};

}  // namespace exa
