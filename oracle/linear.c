/*
 * ORACLE -- test infrastructure only (see oracle.h). Plain-C restatement of
 * the reference's generic LINEAR ADER-DG kernels for one cell / one face, in
 * the reference's loop nesting and operation order (compiled with
 * -ffp-contract=off). Citations are to ExaHyPE/kernels/aderdg/generic/c/
 * {2d,3d}/ unless stated.
 *
 *   spaceTimePredictorLinear  2d/spaceTimePredictorLinear.cpph:35-409,
 *                             3d/spaceTimePredictorLinear.cpph:34-446
 *                             (Cauchy-Kovalevski procedure; useSource and
 *                             the 2D flux branch off, the non-conservative
 *                             product on, usePointSource for pde 4)
 *   pointSource               2d/pointSource.cpph:30-127,
 *                             3d/pointSource.cpph:28-143
 *   volumeIntegralLinear      2d/volumeIntegralLinear.cpph:26-50,
 *                             3d/volumeIntegralLinear.cpph:20-52
 *   surfaceIntegralLinear     2d/surfaceIntegralLinear.cpph:24-66,
 *                             3d/surfaceIntegralLinear.cpph:24-91
 *   riemannSolverLinear       2d/riemannSolverLinear.cpph:23-126,
 *                             3d/riemannSolverLinear.cpph:20-136
 *   boundaryConditions        2d/boundaryConditions.cpph:24-72,
 *                             3d/boundaryConditions.cpph:24-85, then
 *                             riemannSolverLinear (boundary faces)
 *
 * Dimension-generic form as in oracle.c: a 2D cell is a 3D cell with one
 * z-layer of unit weight. Every 2D product of the reference either has no
 * z factor or starts with it, so the 2D results are bit-identical.
 *
 * PDE hooks (pde 2, linear elastic waves; variables sxx syy szz sxy syz sxz
 * u v w, parameters lambda mu rho) restate the reference's kernel-test PDE
 * exahype/tests/kernels/c/ElasticityKernelTest2D.cpp:31-235 (flux-free:
 * nonConservativeProduct, eigenvalues, coefficientMatrix); the z-direction
 * parts are the ones written out (commented) beside the x and y parts there.
 * pde 1 (the generic Euler kernel-test mock) has the zero coefficient matrix
 * of exahype/tests/kernels/c/GenericEulerKernelTest3D.cpp:108-130.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define LMAXB 10

typedef struct {
  int d, N, b, nz, nV, nD, P, F;
  const double *w, *FL, *FR, *dudx;
  double wz[LMAXB];
} lgeo;

static lgeo lmk(const orc_solver* s) {
  lgeo g;
  g.d = s->dim;
  g.N = s->order;
  g.b = s->order + 1;
  g.nz = s->dim == 3 ? g.b : 1;
  g.nV = orc_nvar(s);
  g.nD = g.nV + orc_npar(s);
  g.P = g.nz * g.b * g.b;
  g.F = s->dim == 3 ? g.b * g.b : g.b;
  g.w = orc_table("weights", g.N);
  g.FL = orc_table("FLCoeff", g.N);
  g.FR = orc_table("FRCoeff", g.N);
  g.dudx = orc_table("dudx", g.N);
  for (int i = 0; i < LMAXB; i++) g.wz[i] = (s->dim == 3 && i < g.b) ? g.w[i] : 1.0;
  return g;
}
#define LPT(g, z, y, x) (((z) * (g).b + (y)) * (g).b + (x))

/* ---- PDE hooks of the linear kernels ------------------------------------ */

/* nonConservativeProduct: BgradQ[d][nV] from Q[nD] and gradQ[d][nV]
 * (ElasticityKernelTest2D.cpp:131-188). */
void orc_ncp(const orc_solver* s, const double* Q, const double* gradQ, double* BgradQ) {
  const int nV = orc_nvar(s);
  for (int i = 0; i < nV * s->dim; i++) BgradQ[i] = 0.0;
  if (!ORC_ELASTIC(s)) return;
  const double lam = Q[9], mu = Q[10], irho = 1.0 / Q[11];
  const double* gx = gradQ;
  const double* gy = gradQ + nV;
  double* bx = BgradQ;
  double* by = BgradQ + nV;
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
  if (s->dim == 3) {
    const double* gz = gradQ + 2 * nV;
    double* bz = BgradQ + 2 * nV;
    bz[0] = -lam * gz[8];
    bz[1] = -lam * gz[8];
    bz[2] = -(lam + 2 * mu) * gz[8];
    bz[3] = 0.0;
    bz[4] = -mu * gz[7];
    bz[5] = -mu * gz[6];
    bz[6] = -irho * gz[5];
    bz[7] = -irho * gz[4];
    bz[8] = -irho * gz[2];
  }
}

/* coefficientMatrix: Bn[nV][nV] (row-major) for the normal d
 * (ElasticityKernelTest2D.cpp:190-235). */
void orc_coefficient_matrix(const orc_solver* s, const double* Q, int d, double* Bn) {
  const int nV = orc_nvar(s);
  for (int i = 0; i < nV * nV; i++) Bn[i] = 0.0;
  if (!ORC_ELASTIC(s)) return;
  const double lam = Q[9], mu = Q[10], irho = 1.0 / Q[11];
#define B(r, c) Bn[(r - 1) * nV + (c - 1)]
  if (d == 0) {
    B(7, 1) = -(lam + 2 * mu);
    B(7, 2) = -lam;
    B(7, 3) = -lam;
    B(8, 4) = -mu;
    B(9, 6) = -mu;
    B(1, 7) = -irho;
    B(4, 8) = -irho;
    B(6, 9) = -irho;
  } else if (d == 1) {
    B(8, 1) = -lam;
    B(8, 2) = -(lam + 2 * mu);
    B(8, 3) = -lam;
    B(7, 4) = -mu;
    B(9, 5) = -mu;
    B(4, 7) = -irho;
    B(2, 8) = -irho;
    B(5, 9) = -irho;
  } else {
    B(9, 1) = -lam;
    B(9, 2) = -lam;
    B(9, 3) = -(lam + 2 * mu);
    B(8, 5) = -mu;
    B(7, 6) = -mu;
    B(6, 7) = -irho;
    B(5, 8) = -irho;
    B(3, 9) = -irho;
  }
#undef B
}

/* ---- spaceTimePredictorLinear (+ volumeIntegralLinear when lduh != 0) ----
 * lQhi [b^d][nD] and lFhi [d][b^d][nV] (the reference's tempUnknowns and
 * tempFluxUnknowns) are optional outputs. */
void orc_lin_predictor(const orc_solver* s, const double* luh, const double* dx, double dt, double* lQhbnd,
                       double* lFhbnd, double* lduh, double* lQhi_out, double* lFhi_out) {
  orc_lin_predictor_ps(s, luh, dx, dt, 0, lQhbnd, lFhbnd, lduh, lQhi_out, lFhi_out);
}

void orc_lin_predictor_ps(const orc_solver* s, const double* luh, const double* dx, double dt, const double* PSi,
                          double* lQhbnd, double* lFhbnd, double* lduh, double* lQhi_out, double* lFhi_out) {
  const lgeo g = lmk(s);
  const int b = g.b, nV = g.nV, nD = g.nD, d = g.d, P = g.P, F = g.F, nz = g.nz;
  double* lQi = (double*)calloc((size_t)(b + 1) * P * nD, sizeof(double)); /* [i][p][nD] */
  double* lFi = (double*)calloc((size_t)b * P * d * nV, sizeof(double));   /* [i][p][d][nV] */
  double* gradQ = (double*)calloc((size_t)P * d * nV, sizeof(double));      /* [p][d][nV] */
  double* lQh = (double*)calloc((size_t)P * nD, sizeof(double));
  double* lFh = (double*)calloc((size_t)d * P * nV, sizeof(double));        /* [d][p][nV] */
#define QI(i, p, v) lQi[((size_t)(i) * P + (p)) * nD + (v)]
#define FI(i, p, m, v) lFi[(((size_t)(i) * P + (p)) * d + (m)) * nV + (v)]
#define GQ(p, m, v) gradQ[((p) * d + (m)) * nV + (v)]
  /* zeroth time derivative = initial condition (2d:60-68, 3d:58-67) */
  for (int p = 0; p < P; p++)
    for (int v = 0; v < nD; v++) QI(0, p, v) = luh[p * nD + v];
#define PS(n, p, v) PSi[((size_t)(n) * P + (p)) * nV + (v)]
  if (PSi) {
    /* the time integral of the source into derivative 0 (2d:73-84, 3d:77-90),
     * its value at t into derivative 1 (2d:88-94, 3d:93-101) */
    for (int p = 0; p < P; p++)
      for (int v = 0; v < nV; v++) {
        double sum = 0.0;
        for (int n = 1; n < b + 1; n++) sum = sum + g.w[n - 1] * PS(n, p, v);
        QI(0, p, v) += dt * sum;
      }
    for (int p = 0; p < P; p++)
      for (int v = 0; v < nV; v++) QI(1, p, v) += PS(0, p, v);
  }
  /* Cauchy-Kovalevski (2d:126-232, 3d:123-227) */
  for (int i = 0; i < b; i++) {
    memset(gradQ, 0, sizeof(double) * P * d * nV);
    for (int z = 0; z < nz; z++) /* x derivative */
      for (int y = 0; y < b; y++)
        for (int l = 0; l < b; l++)
          for (int m = 0; m < nV; m++)
            for (int n = 0; n < b; n++)
              GQ(LPT(g, z, y, l), 0, m) += 1.0 / dx[0] * QI(i, LPT(g, z, y, n), m) * g.dudx[l * b + n];
    for (int z = 0; z < nz; z++) /* y derivative */
      for (int x = 0; x < b; x++)
        for (int l = 0; l < b; l++)
          for (int m = 0; m < nV; m++)
            for (int n = 0; n < b; n++)
              GQ(LPT(g, z, l, x), 1, m) += 1.0 / dx[1] * QI(i, LPT(g, z, n, x), m) * g.dudx[l * b + n];
    if (d == 3) /* z derivative */
      for (int y = 0; y < b; y++)
        for (int x = 0; x < b; x++)
          for (int l = 0; l < b; l++)
            for (int m = 0; m < nV; m++)
              for (int n = 0; n < b; n++)
                GQ(LPT(g, l, y, x), 2, m) += 1.0 / dx[2] * QI(i, LPT(g, n, y, x), m) * g.dudx[l * b + n];
    for (int p = 0; p < P; p++) orc_ncp(s, &QI(i, p, 0), &GQ(p, 0, 0), &FI(i, p, 0, 0));
    for (int p = 0; p < P; p++) {
      for (int m = 0; m < d; m++)
        for (int v = 0; v < nV; v++) QI(i + 1, p, v) -= FI(i, p, m, v);
      for (int v = nV; v < nD; v++) QI(i + 1, p, v) = QI(i, p, v);
    }
  }
  /* time averages (2d:246-268, 3d:238-262 and 2d:271-300, 3d:264-292) */
  for (int p = 0; p < P; p++)
    for (int v = 0; v < nD; v++) lQh[p * nD + v] = QI(0, p, v);
  double dtavFac = 0.5 * dt;
  for (int i = 1; i < b; i++) {
    for (int p = 0; p < P; p++)
      for (int v = 0; v < nV; v++) lQh[p * nD + v] += dtavFac * QI(i, p, v);
    dtavFac *= dt / (i + 2);
  }
  for (int m = 0; m < d; m++)
    for (int p = 0; p < P; p++)
      for (int v = 0; v < nV; v++) lFh[((size_t)m * P + p) * nV + v] = FI(0, p, m, v);
  dtavFac = 0.5 * dt;
  for (int i = 1; i < b; i++) {
    for (int m = 0; m < d; m++)
      for (int p = 0; p < P; p++)
        for (int v = 0; v < nV; v++) lFh[((size_t)m * P + p) * nV + v] += dtavFac * FI(i, p, m, v);
    dtavFac *= dt / (i + 2);
  }
  if (PSi) /* the time integral of the source, split over the directions (2d:310-324, 3d:294-308) */
    for (int m = 0; m < d; m++)
      for (int p = 0; p < P; p++)
        for (int v = 0; v < nV; v++) {
          double sum = 0.0;
          for (int n = 1; n < b + 1; n++) sum = sum + g.w[n - 1] * PS(n, p, v);
          lFh[((size_t)m * P + p) * nV + v] += sum / d;
        }
#undef PS
  /* boundary extrapolation (2d:318-405, 3d:308-440) */
  memset(lQhbnd, 0, sizeof(double) * 2 * d * F * nD);
  memset(lFhbnd, 0, sizeof(double) * 2 * d * F * nV);
  for (int dir = 0; dir < d; dir++)
    for (int fn = 0; fn < F; fn++) {
      int a = fn / b, c = fn % b;
      if (d == 2) { a = 0; c = fn; }
      /* face nodes: x-face (z,y), y-face (z,x), z-face (y,x) */
      for (int v = 0; v < nD; v++)
        for (int l = 0; l < b; l++) {
          const int p = dir == 0 ? LPT(g, a, c, l) : dir == 1 ? LPT(g, a, l, c) : LPT(g, l, a, c);
          lQhbnd[((2 * dir) * F + fn) * nD + v] += lQh[p * nD + v] * g.FL[l];
          lQhbnd[((2 * dir + 1) * F + fn) * nD + v] += lQh[p * nD + v] * g.FR[l];
        }
      for (int v = 0; v < nV; v++)
        for (int l = 0; l < b; l++) {
          const int p = dir == 0 ? LPT(g, a, c, l) : dir == 1 ? LPT(g, a, l, c) : LPT(g, l, a, c);
          lFhbnd[((2 * dir) * F + fn) * nV + v] += lFh[((size_t)dir * P + p) * nV + v] * g.FL[l];
          lFhbnd[((2 * dir + 1) * F + fn) * nV + v] += lFh[((size_t)dir * P + p) * nV + v] * g.FR[l];
        }
    }
  if (lduh) orc_lin_volume_integral(s, lduh, lFh, dx);
  if (lQhi_out) memcpy(lQhi_out, lQh, sizeof(double) * P * nD);
  if (lFhi_out) memcpy(lFhi_out, lFh, sizeof(double) * d * P * nV);
#undef QI
#undef FI
#undef GQ
  free(lQi);
  free(lFi);
  free(gradQ);
  free(lQh);
  free(lFh);
}

/* volumeIntegralLinear: lduh = -w_node sum_d lFhi[d] (lFhi [d][b^d][nV]) */
void orc_lin_volume_integral(const orc_solver* s, double* lduh, const double* lFhi, const double* dx) {
  const lgeo g = lmk(s);
  (void)dx;
  const int b = g.b, nV = g.nV, P = g.P;
  memset(lduh, 0, sizeof(double) * P * nV);
  for (int z = 0; z < g.nz; z++)
    for (int y = 0; y < b; y++)
      for (int x = 0; x < b; x++) {
        const double weight = g.wz[z] * g.w[y] * g.w[x];
        const int p = LPT(g, z, y, x);
        for (int l = 0; l < nV; l++)
          for (int m = 0; m < g.d; m++) lduh[p * nV + l] -= weight * lFhi[((size_t)m * P + p) * nV + l];
      }
}

/* surfaceIntegralLinear: the fluctuations of both faces of a direction are
 * added, each with its own extrapolation coefficient (weight / dx). */
void orc_lin_surface_integral(const orc_solver* s, double* lduh, const double* lFhbnd, const double* dx) {
  const lgeo g = lmk(s);
  const int b = g.b, nV = g.nV, F = g.F;
#define FB(face, fn, v) lFhbnd[((face) * F + (fn)) * nV + (v)]
  for (int z = 0; z < g.nz; z++) /* x faces */
    for (int y = 0; y < b; y++) {
      const double us = (g.wz[z] * g.w[y]) / dx[0];
      const int fn = z * b + y;
      for (int x = 0; x < b; x++)
        for (int v = 0; v < nV; v++)
          lduh[LPT(g, z, y, x) * nV + v] -= (FB(1, fn, v) * g.FR[x] + FB(0, fn, v) * g.FL[x]) * us;
    }
  for (int z = 0; z < g.nz; z++) /* y faces */
    for (int y = 0; y < b; y++)
      for (int x = 0; x < b; x++) {
        const double us = (g.wz[z] * g.w[x]) / dx[1];
        const int fn = z * b + x;
        for (int v = 0; v < nV; v++)
          lduh[LPT(g, z, y, x) * nV + v] -= (FB(3, fn, v) * g.FR[y] + FB(2, fn, v) * g.FL[y]) * us;
      }
  if (g.d == 3) /* z faces */
    for (int z = 0; z < b; z++)
      for (int y = 0; y < b; y++)
        for (int x = 0; x < b; x++) {
          const double us = (g.w[y] * g.w[x]) / dx[2];
          const int fn = y * b + x;
          for (int v = 0; v < nV; v++)
            lduh[LPT(g, z, y, x) * nV + v] -= (FB(5, fn, v) * g.FR[z] + FB(4, fn, v) * g.FL[z]) * us;
        }
#undef FB
}

/* riemannSolverLinear: Rusanov with scalar dissipation on the fluctuation
 * form, FL = (Bn - smax I)^T dQ, FR = (Bn + smax I)^T dQ, dQ = (QR - QL)/2,
 * Bn evaluated once in the mean of the face-averaged states. FL and FR are
 * outputs only. */
void orc_lin_riemann(const orc_solver* s, double* FL, double* FR, const double* QL, const double* QR, int dir) {
  const lgeo g = lmk(s);
  const int b = g.b, nV = g.nV, nD = g.nD, F = g.F;
  double QavL[16] = {0}, QavR[16] = {0}, Qav[16];
  for (int fn = 0; fn < F; fn++) {
    int a = fn / b, c = fn % b;
    if (g.d == 2) { a = 0; c = fn; }
    const double weight = g.wz[a] * g.w[c];
    for (int k = 0; k < nD; k++) {
      QavL[k] += weight * QL[fn * nD + k];
      QavR[k] += weight * QR[fn * nD + k];
    }
  }
  double LL[16], LR[16];
  orc_eigenvalues(s, QavL, dir, LL);
  orc_eigenvalues(s, QavR, dir, LR);
  double smL = fabs(LL[0]), smR = fabs(LR[0]);
  for (int k = 1; k < nV; k++) { /* std::max_element over |lambda| */
    if (smL < fabs(LL[k])) smL = fabs(LL[k]);
    if (smR < fabs(LR[k])) smR = fabs(LR[k]);
  }
  const double smax = (smL < smR) ? smR : smL;
  for (int k = 0; k < nD; k++) Qav[k] = 0.5 * (QavL[k] + QavR[k]);
  double Bn[16 * 16], Bm[16 * 16], Bp[16 * 16];
  orc_coefficient_matrix(s, Qav, dir, Bn);
  for (int i = 0; i < nV * nV; i++) Bm[i] = Bp[i] = Bn[i];
  for (int i = 0; i < nV; i++) {
    Bm[i * nV + i] -= smax;
    Bp[i * nV + i] += smax;
  }
  for (int fn = 0; fn < F; fn++) {
    double dq[16];
    for (int k = 0; k < nD; k++) dq[k] = 0.5 * (QR[fn * nD + k] - QL[fn * nD + k]);
    for (int j = 0; j < nV; j++) {
      double fl = 0.0, fr = 0.0;
      for (int k = 0; k < nV; k++) {
        fl += Bm[k * nV + j] * dq[k];
        fr += Bp[k * nV + j] * dq[k];
      }
      FL[fn * nV + j] = fl;
      FR[fn * nV + j] = fr;
    }
  }
}

/* Boundary faces of a linear solver: ADERDGSolver::applyBoundaryConditions
 * (exahype/solvers/ADERDGSolver.cpp:2893-2962) with the generic
 * boundaryConditions kernel (3d/boundaryConditions.cpph:24-85) -- the user's
 * boundaryValues at every face node -- followed by riemannSolverLinear with
 * the outside state on the outer side (FOut, FIn, QOut, QIn for an even
 * face, FIn, FOut, QIn, QOut for an odd one); only the cell's own
 * fluctuation is kept. boundaryValues of the elastic-wave PDE (this
 * repository's, the reference's kernel tests define none): kind 0 copies
 * the inside state (outflow), kind 1 a rigid wall, the inside state with
 * the three velocities negated; parameters are copied. */
void orc_lin_boundary_face(const orc_solver* s, double* FIn, const double* QIn, int faceIndex, int kind) {
  const lgeo g = lmk(s);
  const int dir = (faceIndex - faceIndex % 2) / 2;
  double QOut[100 * 12], FOut[100 * 9];
  memcpy(QOut, QIn, sizeof(double) * g.F * g.nD);
  memcpy(FOut, FIn, sizeof(double) * g.F * g.nV);
  if (kind == 1 && ORC_ELASTIC(s))
    for (int fn = 0; fn < g.F; fn++)
      for (int v = 6; v < 9; v++) QOut[fn * g.nD + v] = -QOut[fn * g.nD + v];
  if (faceIndex % 2 == 0)
    orc_lin_riemann(s, FOut, FIn, QOut, QIn, dir);
  else
    orc_lin_riemann(s, FIn, FOut, QIn, QOut, dir);
}

/* ---- point sources -------------------------------------------------------
 * The point-source mock of pde 4 (this repository's; the reference's kernel
 * tests define none): a Ricker wavelet of peak frequency f0 and delay t0,
 * amplitude amp, on the three normal stresses, located at x0 whatever the
 * node position x (UserSolverInterface::pointSource(x, t, dt, forceVector,
 * x0), exahype/solvers/UserSolverInterface.h:75). */
static void elastic_point_source(const orc_solver* s, const double* x, double t, double dt, double* force,
                                 double* x0) {
  (void)x;
  (void)dt;
  const double r = 3.14159265358979323846 * s->ps[4] * (t - s->ps[3]);
  const double a = r * r;
  const double w = s->ps[5] * ((1.0 - 2.0 * a) * exp(-a));
  for (int v = 0; v < 9; v++) force[v] = v < 3 ? w : 0.0;
  for (int d = 0; d < 3; d++) x0[d] = s->ps[d];
}

/* Lagrange basis polynomial i of the Gauss-Legendre nodes of order N at xi
 * (the reference's basisFunctions[N][i], DGBasisFunctions.h:53, as the
 * product over the other nodes) */
static double lagrange(const double* nodes, int b, int i, double xi) {
  double r = 1.0;
  for (int m = 0; m < b; m++)
    if (m != i) r *= (xi - nodes[m]) / (nodes[i] - nodes[m]);
  return r;
}

void orc_point_source(const orc_solver* s, double t, double dt, const double* centre, const double* dx, double* PSi) {
  const lgeo g = lmk(s);
  const int b = g.b, nV = g.nV, P = g.P, d = g.d;
  const double* nodes = orc_table("nodes", g.N);
  for (int n = 0; n < b + 1; n++) {
    const double tn = n == 0 ? t : dt * nodes[n - 1] + t;
    for (int p = 0; p < P; p++) {
      /* node (z, y, x) of the cell; 2D: (y, x) */
      const int ix = p % b, iy = (p / b) % b, iz = d == 3 ? p / (b * b) : 0;
      double x[3] = {0, 0, 0}, x0[3] = {0, 0, 0}, xr[3] = {0, 0, 0};
      if (d == 3) x[2] = centre[2] + dx[2] * (nodes[iz] - 0.5);
      x[1] = centre[1] + dx[1] * (nodes[iy] - 0.5);
      x[0] = centre[0] + dx[0] * (nodes[ix] - 0.5);
      double* out = PSi + ((size_t)n * P + p) * nV;
      elastic_point_source(s, x, tn, dt, out, x0);
      int inside = 1;
      for (int e = 0; e < d; e++) {
        const double off = centre[e] - dx[e] / 2.;
        xr[e] = x0[e] - off;
        xr[e] /= dx[e];
        inside = inside && xr[e] >= 0. && xr[e] <= 1.0;
      }
      for (int v = 0; v < nV; v++) {
        if (!inside) {
          out[v] = 0.0;
          continue;
        }
        double value;
        if (d == 3) {
          value = lagrange(nodes, b, iz, xr[2]) * lagrange(nodes, b, iy, xr[1]) * lagrange(nodes, b, ix, xr[0]) * out[v];
          value /= ((g.w[iz]) * dx[2] * (g.w[iy]) * dx[1] * (g.w[ix]) * dx[0]);
        } else {
          value = lagrange(nodes, b, iy, xr[1]) * lagrange(nodes, b, ix, xr[0]) * out[v];
          value /= ((g.w[iy]) * dx[1] * (g.w[ix]) * dx[0]);
        }
        out[v] = value;
      }
    }
  }
}
