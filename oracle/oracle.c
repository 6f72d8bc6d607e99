/*
 * ORACLE -- test infrastructure only (see oracle.h). Plain-C restatement of
 * the reference's generic nonlinear ADER-DG kernels for one cell / one face,
 * with the reference's loop nesting and operation order (compile with
 * -ffp-contract=off so no FMA is formed). Citations are to the reference
 * tree, ExaHyPE/kernels/aderdg/generic/c/{2d,3d}/ unless stated.
 *
 * Dimension-generic form: a 2D cell is a 3D cell with one z-layer whose
 * quadrature weight is 1.0. Every product in the reference starts with the
 * outermost (z-like) factor, so multiplying by the unit weight is exact and
 * the 2D results are bit-identical to the reference's 2D kernels.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../exahype_b200/csrc/dg_tables.h"

#define MAXB 10

const double* orc_table(const char* name, int N) {
#define T(nm) if (!strcmp(name, #nm)) return exa_tab_##nm + exa_tab_##nm##_off[N];
  T(nodes) T(weights) T(lobatto_nodes) T(lobatto_weights) T(FLCoeff) T(FRCoeff) T(FCoeff) T(Kxi) T(iK1)
  T(dudx) T(uh2lim) T(lim2uh) T(uh2lob) T(fineGridProjector1d) T(equidistantGridProjector1d)
#undef T
  return 0;
}

int orc_nvar(const orc_solver* s) { return ORC_ELASTIC(s) ? 9 : 5; }
int orc_npar(const orc_solver* s) { return (s->pde == 1 || s->pde == 3) ? 1 : ORC_ELASTIC(s) ? 3 : 0; }

/* pde 3: the kernel-test mock with an algebraic source and its
 * non-conservative product switched on (useSource = useNCP = true) */
static int use_source(const orc_solver* s) { return s->pde == 3; }
static int use_ncp(const orc_solver* s) { return s->pde == 3; }

/* algebraicSource (UserSolverInterface.h:92) of pde 3: momentum damping and
 * an energy source proportional to the density; zero for the other PDEs */
void orc_source(const orc_solver* s, const double* Q, double* S) {
  for (int v = 0; v < 5; v++) S[v] = 0.0;
  if (s->pde != 3) return;
  S[1] = -0.5 * Q[1];
  S[2] = -0.5 * Q[2];
  S[3] = -0.5 * Q[3];
  S[4] = 0.1 * Q[0];
}

/* nonConservativeProduct (UserSolverInterface.h:116) of the nonlinear
 * kernels: BgradQ[nV] from Q and gradQ[dim][nV]. pde 3: the non-zero mock of
 * exahype/tests/kernels/c/GenericEulerKernelTest2D.cpp:80-103 and
 * GenericEulerKernelTest3D.cpp:84-110 (_setNcpAndMatrixBToZero false). */
void orc_ncp_nonlinear(const orc_solver* s, const double* Q, const double* gradQ, double* BgradQ) {
  for (int v = 0; v < 5; v++) BgradQ[v] = 0.0;
  if (s->pde != 3) return;
  BgradQ[0] = Q[0];
  BgradQ[1] = Q[3];
  BgradQ[2] = 3.0;
  BgradQ[3] = gradQ[0];
  BgradQ[4] = 0.7;
}

/* ---- PDE hooks ----------------------------------------------------------
 * pde 0: Demonstrators/EulerADERDG/MyEulerSolver_ADERDG.cpp:102-135
 *        p = (gamma-1)(E - 0.5 irho |j|^2), |j|^2 over all three components.
 * pde 1: exahype/tests/kernels/c/GenericEulerKernelTest2D.cpp:28-77 (2.5D)
 *        and GenericEulerKernelTest3D.cpp:26-77. */
static double pressure(const orc_solver* s, const double* Q, double irho) {
  const double GAMMA = 1.4;
  if (s->pde == 0) {
    const double jj = Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3];
    return (GAMMA - 1) * (Q[4] - 0.5 * irho * jj);
  }
  if (s->dim == 2) return (GAMMA - 1) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) * irho);
  return (GAMMA - 1) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) * irho);
}

void orc_flux(const orc_solver* s, const double* Q, double* F) {
  const double irho = 1.0 / Q[0];
  const double p = pressure(s, Q, irho);
  for (int d = 0; d < s->dim; d++) {
    double* f = F + 5 * d;
    f[0] = Q[1 + d];
    for (int a = 0; a < 3; a++) {
      if (s->pde == 0)
        f[1 + a] = irho * (Q[1 + d] * Q[1 + a]) + (d == a ? p : 0.0);
      else
        f[1 + a] = irho * Q[1 + d] * Q[1 + a] + (d == a ? p : 0.0);
    }
    if (s->pde == 0)
      f[4] = (irho * (Q[4] + p)) * Q[1 + d];
    else
      f[4] = irho * Q[1 + d] * (Q[4] + p);
  }
}

void orc_eigenvalues(const orc_solver* s, const double* Q, int d, double* lambda) {
  if (ORC_ELASTIC(s)) { /* elastic waves: ElasticityKernelTest2D.cpp:99-125 */
    const double lam = Q[9], mu = Q[10], rho0 = Q[11];
    const double cp = sqrt((lam + 2 * mu) / rho0);
    const double cs = sqrt(mu / rho0);
    lambda[0] = -cp;
    lambda[1] = -cs;
    lambda[2] = -cs;
    lambda[3] = 0.0;
    lambda[4] = 0.0;
    lambda[5] = 0.0;
    lambda[6] = +cs;
    lambda[7] = +cs;
    lambda[8] = +cp;
    return;
  }
  const double GAMMA = 1.4;
  const double irho = 1.0 / Q[0];
  const double p = pressure(s, Q, irho);
  const double u_n = Q[d + 1] * irho;
  const double c = sqrt(GAMMA * p * irho);
  lambda[0] = u_n - c;
  lambda[1] = u_n;
  lambda[2] = u_n;
  lambda[3] = u_n;
  lambda[4] = u_n + c;
}

static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */

/* ---- geometry helpers --------------------------------------------------- */
typedef struct {
  int d, N, b, nz, nV, nD, P, F;
  const double *w, *FL, *FR, *Kxi, *iK1, *dudx;
  double wz[MAXB]; /* z-weights: w in 3D, {1.0} in 2D */
} geo;

static geo mkgeo(const orc_solver* s) {
  geo g;
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
  g.Kxi = orc_table("Kxi", g.N);
  g.iK1 = orc_table("iK1", g.N);
  g.dudx = orc_table("dudx", g.N);
  for (int i = 0; i < MAXB; i++) g.wz[i] = (s->dim == 3 && i < g.b) ? g.w[i] : 1.0;
  return g;
}
#define PT(g, z, y, x) (((z) * (g).b + (y)) * (g).b + (x))

/* ---- predictor -----------------------------------------------------------
 * aderPicardLoopNonlinear: 3d/spaceTimePredictorNonlinear.cpph:42-329,
 * 2d/spaceTimePredictorNonlinear.cpph:41-284 (useFlux only). */
static int picard(const orc_solver* s, const geo* g, const double* luh, const double* dx, double dt, double* lQi,
                  double* lFi, double* rhs) {
  const int b = g->b, nV = g->nV, nD = g->nD, d = g->d, nz = g->nz;
  const int dd1 = d + 1;
  double invDx[3];
  for (int i = 0; i < d; i++) invDx[i] = 1.0 / dx[i];
#define LQI(z, y, x, t, v) lQi[((PT(*g, z, y, x)) * b + (t)) * nD + (v)]
#define LFI(t, z, y, x, k, v) lFi[(((t) * g->P + PT(*g, z, y, x)) * dd1 + (k)) * nV + (v)]
#define RHS(t, z, y, x, v) rhs[((t) * g->P + PT(*g, z, y, x)) * nV + (v)]
#define LUH(z, y, x, v) luh[(PT(*g, z, y, x)) * nD + (v)]
  /* trivial initial guess :66-82 */
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < b; y++)
      for (int x = 0; x < b; x++)
        for (int t = 0; t < b; t++)
          for (int v = 0; v < nD; v++) LQI(z, y, x, t, v) = LUH(z, y, x, v);
  const int maxIter = 2 * (g->N + 1); /* :85 */
  int iter;
  for (iter = 0; iter < maxIter; iter++) {
    for (int t = 0; t < b; t++) {
      /* fluxes :96-122 */
      for (int z = 0; z < nz; z++)
        for (int y = 0; y < b; y++)
          for (int x = 0; x < b; x++) {
            double F[3 * 5];
            orc_flux(s, &LQI(z, y, x, t, 0), F);
            for (int k = 0; k < d; k++)
              for (int v = 0; v < nV; v++) LFI(t, z, y, x, k, v) = F[k * 5 + v];
          }
      /* rhs0 = w_xyz FLCoeff[t] luh :124-141 */
      for (int z = 0; z < nz; z++)
        for (int y = 0; y < b; y++)
          for (int x = 0; x < b; x++) {
            const double weight = g->wz[z] * g->w[y] * g->w[x];
            for (int v = 0; v < nV; v++) RHS(t, z, y, x, v) = weight * g->FL[t] * LUH(z, y, x, v);
          }
      /* x derivative :151-178 */
      for (int z = 0; z < nz; z++)
        for (int y = 0; y < b; y++) {
          const double weight = g->w[t] * g->wz[z] * g->w[y];
          const double us = weight * dt * invDx[0];
          for (int l = 0; l < b; l++)
            for (int v = 0; v < nV; v++)
              for (int n = 0; n < b; n++) RHS(t, z, y, l, v) -= us * LFI(t, z, y, n, 0, v) * g->Kxi[n * b + l];
        }
      /* y derivative :180-207 */
      for (int z = 0; z < nz; z++)
        for (int x = 0; x < b; x++) {
          const double weight = g->w[t] * g->wz[z] * g->w[x];
          const double us = weight * dt * invDx[1];
          for (int l = 0; l < b; l++)
            for (int v = 0; v < nV; v++)
              for (int n = 0; n < b; n++) RHS(t, z, l, x, v) -= us * LFI(t, z, n, x, 1, v) * g->Kxi[n * b + l];
        }
      /* z derivative :209-236 */
      if (d == 3)
        for (int y = 0; y < b; y++)
          for (int x = 0; x < b; x++) {
            const double weight = g->w[t] * g->w[y] * g->w[x];
            const double us = weight * dt * invDx[2];
            for (int l = 0; l < b; l++)
              for (int v = 0; v < nV; v++)
                for (int n = 0; n < b; n++) RHS(t, l, y, x, v) -= us * LFI(t, n, y, x, 2, v) * g->Kxi[n * b + l];
          }
      /* gradients of lQi for the non-conservative product (:171-174,
       * :199-202, :228-231; 2d :145-148, :169-172), then the algebraic
       * source minus the product, stored in the source block of lFi and
       * added to rhs with w_t w_xyz dt (:238-276; 2d :180-211) */
      if (use_source(s) || use_ncp(s))
        for (int z = 0; z < nz; z++)
          for (int y = 0; y < b; y++)
            for (int x = 0; x < b; x++) {
              double gq[3 * 5];
              for (int i = 0; i < 3 * 5; i++) gq[i] = 0.0;
              if (use_ncp(s))
                for (int v = 0; v < nV; v++)
                  for (int n = 0; n < b; n++) {
                    gq[0 * 5 + v] += 1.0 * invDx[0] * LQI(z, y, n, t, v) * g->dudx[x * b + n];
                    gq[1 * 5 + v] += 1.0 * invDx[1] * LQI(z, n, x, t, v) * g->dudx[y * b + n];
                    if (d == 3) gq[2 * 5 + v] += 1.0 * invDx[2] * LQI(n, y, x, t, v) * g->dudx[z * b + n];
                  }
              const double weight =
                  d == 3 ? g->w[t] * g->w[z] * g->w[y] * g->w[x] : g->w[t] * g->w[y] * g->w[x];
              const double us = weight * dt;
              double S[5], ncp[5];
              orc_source(s, &LQI(z, y, x, t, 0), S);
              if (use_ncp(s)) {
                orc_ncp_nonlinear(s, &LQI(z, y, x, t, 0), gq, ncp);
                for (int v = 0; v < nV; v++) S[v] -= ncp[v];
              }
              for (int v = 0; v < nV; v++) {
                LFI(t, z, y, x, d, v) = S[v];
                RHS(t, z, y, x, v) += us * S[v];
              }
            }
    }
    /* discrete time integral and residual :280-311 */
    double sq_res = 0.0;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < b; y++)
        for (int x = 0; x < b; x++) {
          const double weight = g->wz[z] * g->w[y] * g->w[x];
          const double iweight = 1.0 / weight;
          for (int l = 0; l < b; l++)
            for (int v = 0; v < nV; v++) {
              double qn = 0;
              for (int n = 0; n < b; n++) qn += iweight * RHS(n, z, y, x, v) * g->iK1[l * b + n];
              const double diff = qn - LQI(z, y, x, l, v);
              sq_res += diff * diff;
              LQI(z, y, x, l, v) = qn;
            }
        }
    /* exit condition :315-318 */
    if (sq_res < 1e-7 * 1e-7) {
      iter++;
      break;
    }
  }
  return iter < maxIter ? iter : maxIter;
}

/* aderPredictorNonlinear 3d:337-409 / 2d:292-347 and aderExtrapolatorNonlinear
 * 3d:411-528 / 2d:349-422. lFhi_d is stored with coordinate d fastest before
 * the variable: x:(z,y,x) y:(z,x,y) z:(y,x,z); face nodes for direction d run
 * over the other coordinates in (z,y,x) order. */
static void time_average_extrapolate(const geo* g, const double* lQi, const double* lFi, double* lQhi, double* lFhi,
                                     double* lQhbnd, double* lFhbnd, int source_block) {
  const int b = g->b, nV = g->nV, nD = g->nD, d = g->d, nz = g->nz, dd1 = d + 1;
  const int P = g->P, F = g->F;
  memset(lQhi, 0, sizeof(double) * P * nD);
  memset(lFhi, 0, sizeof(double) * P * nV * dd1);
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < b; y++)
      for (int x = 0; x < b; x++) {
        const int fx = (z * b + y) * b + x, fy = (z * b + x) * b + y, fz = (y * b + x) * nz + z;
        for (int v = 0; v < nV; v++)
          for (int m = 0; m < b; m++) {
            lFhi[0 * P * nV + fx * nV + v] += lFi[((m * P + PT(*g, z, y, x)) * dd1 + 0) * nV + v] * g->w[m];
            lFhi[1 * P * nV + fy * nV + v] += lFi[((m * P + PT(*g, z, y, x)) * dd1 + 1) * nV + v] * g->w[m];
            if (d == 3)
              lFhi[2 * P * nV + fz * nV + v] += lFi[((m * P + PT(*g, z, y, x)) * dd1 + 2) * nV + v] * g->w[m];
            /* lShi, the time-averaged source (3d :391-396, 2d :328-332) */
            if (source_block)
              lFhi[d * P * nV + PT(*g, z, y, x) * nV + v] += lFi[((m * P + PT(*g, z, y, x)) * dd1 + d) * nV + v] * g->w[m];
          }
        for (int v = 0; v < nD; v++)
          for (int m = 0; m < b; m++)
            lQhi[PT(*g, z, y, x) * nD + v] += lQi[(PT(*g, z, y, x) * b + m) * nD + v] * g->w[m];
      }
  memset(lQhbnd, 0, sizeof(double) * 2 * d * F * nD);
  memset(lFhbnd, 0, sizeof(double) * 2 * d * F * nV);
  for (int dir = 0; dir < d; dir++) {
    const double* Fh = lFhi + dir * P * nV;
    for (int fn = 0; fn < F; fn++) {
      /* fn enumerates the face nodes (a,c) = other coordinates in (z,y,x) order */
      for (int v = 0; v < nV; v++)
        for (int l = 0; l < b; l++) {
          lFhbnd[((2 * dir) * F + fn) * nV + v] += Fh[(fn * b + l) * nV + v] * g->FL[l];
          lFhbnd[((2 * dir + 1) * F + fn) * nV + v] += Fh[(fn * b + l) * nV + v] * g->FR[l];
        }
      int a = fn / b, c = fn % b; /* 3D: a,c = outer,inner free coordinate */
      if (d == 2) { a = 0; c = fn; }
      for (int v = 0; v < nD; v++)
        for (int l = 0; l < b; l++) {
          int p;
          if (dir == 0) p = PT(*g, a, c, l);           /* x-face node (z,y) */
          else if (dir == 1) p = PT(*g, a, l, c);      /* y-face node (z,x) */
          else p = PT(*g, l, a, c);                    /* z-face node (y,x) */
          lQhbnd[((2 * dir) * F + fn) * nD + v] += lQhi[p * nD + v] * g->FL[l];
          lQhbnd[((2 * dir + 1) * F + fn) * nD + v] += lQhi[p * nD + v] * g->FR[l];
        }
    }
  }
}

/* volumeIntegralNonlinear, noTimeAveraging=false: 3d/volumeIntegralNonlinear.cpph:135-225,
 * 2d/volumeIntegralNonlinear.cpph:115-173 */
void orc_volume_integral(const orc_solver* s, double* lduh, const double* lFhi, const double* dx) {
  geo g = mkgeo(s);
  const int b = g.b, nV = g.nV, P = g.P;
  double invDx[3];
  for (int i = 0; i < g.d; i++) invDx[i] = 1.0 / dx[i];
  memset(lduh, 0, sizeof(double) * P * nV);
  for (int dir = 0; dir < g.d; dir++) {
    const double* Fh = lFhi + dir * P * nV;
    for (int fn = 0; fn < g.F; fn++) {
      int a = fn / b, c = fn % b;
      if (g.d == 2) { a = 0; c = fn; }
      const double weight = (g.d == 3 ? g.w[a] : 1.0) * g.w[c];
      const double us = weight * invDx[dir];
      for (int k = 0; k < b; k++) {
        int p;
        if (dir == 0) p = PT(g, a, c, k);
        else if (dir == 1) p = PT(g, a, k, c);
        else p = PT(g, k, a, c);
        for (int v = 0; v < nV; v++)
          for (int m = 0; m < b; m++) lduh[p * nV + v] += g.Kxi[k * b + m] * Fh[(fn * b + m) * nV + v] * us;
      }
    }
  }
  /* useSourceOrNCP: lduh += w_xyz lShi (3d :206-224, 2d :158-172) */
  if (use_source(s) || use_ncp(s))
    for (int z = 0; z < g.nz; z++)
      for (int y = 0; y < b; y++)
        for (int x = 0; x < b; x++) {
          const double weight = g.d == 3 ? g.w[z] * g.w[y] * g.w[x] : g.w[y] * g.w[x];
          for (int v = 0; v < nV; v++) lduh[PT(g, z, y, x) * nV + v] += weight * lFhi[(g.d * P + PT(g, z, y, x)) * nV + v];
        }
}

int orc_predictor(const orc_solver* s, const double* luh, const double* dx, double dt, double* lQhbnd,
                  double* lFhbnd, double* lduh, double* lQi_out, double* lFi_out, double* lQhi_out,
                  double* lFhi_out) {
  geo g = mkgeo(s);
  const int st = g.P * g.b;
  double* lQi = (double*)malloc(sizeof(double) * st * g.nD);
  double* lFi = (double*)calloc((size_t)st * (g.d + 1) * g.nV, sizeof(double));
  double* rhs = (double*)malloc(sizeof(double) * st * g.nV);
  double* lQhi = (double*)malloc(sizeof(double) * g.P * g.nD);
  double* lFhi = (double*)malloc(sizeof(double) * g.P * g.nV * (g.d + 1));
  const int it = picard(s, &g, luh, dx, dt, lQi, lFi, rhs);
  time_average_extrapolate(&g, lQi, lFi, lQhi, lFhi, lQhbnd, lFhbnd, use_source(s) || use_ncp(s));
  if (lduh) orc_volume_integral(s, lduh, lFhi, dx);
  if (lQi_out) memcpy(lQi_out, lQi, sizeof(double) * st * g.nD);
  if (lFi_out) memcpy(lFi_out, lFi, sizeof(double) * st * (g.d + 1) * g.nV);
  if (lQhi_out) memcpy(lQhi_out, lQhi, sizeof(double) * g.P * g.nD);
  if (lFhi_out) memcpy(lFhi_out, lFhi, sizeof(double) * g.P * g.nV * (g.d + 1));
  free(lQi);
  free(lFi);
  free(rhs);
  free(lQhi);
  free(lFhi);
  return it;
}

/* riemannSolverNonlinear<useNCP>: 3d/riemannSolverNonlinear.cpph:37-117,
 * 2d/riemannSolverNonlinear.cpph:37-111 */
void orc_riemann(const orc_solver* s, double* FL, double* FR, const double* QL, const double* QR, int dir) {
  geo g = mkgeo(s);
  const int b = g.b, nV = g.nV, nD = g.nD;
  double QavL[8] = {0}, QavR[8] = {0};
  for (int fn = 0; fn < g.F; fn++) {
    int a = fn / b, c = fn % b;
    if (g.d == 2) { a = 0; c = fn; }
    const double weight = (g.d == 3 ? g.w[a] : 1.0) * g.w[c];
    for (int k = 0; k < nD; k++) {
      QavL[k] += weight * QL[fn * nD + k];
      QavR[k] += weight * QR[fn * nD + k];
    }
  }
  double LL[5], LR[5];
  orc_eigenvalues(s, QavL, dir, LL);
  orc_eigenvalues(s, QavR, dir, LR);
  double smL = fabs(LL[0]), smR = fabs(LR[0]);
  for (int k = 1; k < nV; k++) {
    if (smL < fabs(LL[k])) smL = fabs(LL[k]); /* std::max_element */
    if (smR < fabs(LR[k])) smR = fabs(LR[k]);
  }
  const double smax = dmax(smL, smR);
  double gradQ[3 * 5] = {0}, Qavg[8] = {0}, ncp[5] = {0};
  for (int fn = 0; fn < g.F; fn++) {
    if (use_ncp(s)) { /* useNCP (3d :92-100, 2d :86-93): one-sided jump along the normal */
      for (int l = 0; l < nV; l++) {
        gradQ[dir * 5 + l] = QR[fn * nD + l] - QL[fn * nD + l];
        Qavg[l] = 0.5 * (QR[fn * nD + l] + QL[fn * nD + l]);
      }
      orc_ncp_nonlinear(s, Qavg, gradQ, ncp);
    }
    for (int k = 0; k < nV; k++) {
      FL[fn * nV + k] = 0.5 * (FR[fn * nV + k] + FL[fn * nV + k]) - 0.5 * smax * (QR[fn * nD + k] - QL[fn * nD + k]);
      if (use_ncp(s)) {
        FR[fn * nV + k] = FL[fn * nV + k] - 0.5 * ncp[k];
        FL[fn * nV + k] = FL[fn * nV + k] + 0.5 * ncp[k];
      } else {
        FR[fn * nV + k] = FL[fn * nV + k];
      }
    }
  }
}

/* ADERDGSolver::applyBoundaryConditions (exahype/solvers/ADERDGSolver.cpp:2893-2962)
 * with boundaryConditions 3d/boundaryConditions.cpph:24-85. The PDEs here
 * use outflow values (QOut = QIn, FOut = FIn). */
void orc_boundary_face(const orc_solver* s, double* FIn, const double* QIn, const double* centre,
                       const double* size, double t, double dt, int faceIndex) {
  geo g = mkgeo(s);
  (void)centre; (void)size; (void)t; (void)dt;
  const int dir = (faceIndex - faceIndex % 2) / 2;
  double QOut[100 * 6], FOut[100 * 5];
  memcpy(QOut, QIn, sizeof(double) * g.F * g.nD);
  memcpy(FOut, FIn, sizeof(double) * g.F * g.nV);
  if (faceIndex % 2 == 0)
    orc_riemann(s, FOut, FIn, QOut, QIn, dir);
  else
    orc_riemann(s, FIn, FOut, QIn, QOut, dir);
}

/* Reflective walls: the boundaryValues of the reference's Euler demonstrator
 * (Demonstrators/EulerADERDG/MyEulerSolver_ADERDG.cpp:82-87) -- the inside
 * state with its normal momentum negated and that state's normal flux --
 * then the Rusanov flux as in orc_boundary_face. Euler only. */
void orc_boundary_face_reflective(const orc_solver* s, double* FIn, const double* QIn, int faceIndex) {
  geo g = mkgeo(s);
  const int dir = (faceIndex - faceIndex % 2) / 2;
  double QOut[100 * 6], FOut[100 * 5], F[3 * 5];
  for (int fn = 0; fn < g.F; fn++) {
    for (int v = 0; v < g.nD; v++) QOut[fn * g.nD + v] = QIn[fn * g.nD + v];
    QOut[fn * g.nD + 1 + dir] = -QOut[fn * g.nD + 1 + dir];
    orc_flux(s, QOut + fn * g.nD, F);
    for (int v = 0; v < g.nV; v++) FOut[fn * g.nV + v] = F[5 * dir + v];
  }
  if (faceIndex % 2 == 0)
    orc_riemann(s, FOut, FIn, QOut, QIn, dir);
  else
    orc_riemann(s, FIn, FOut, QIn, QOut, dir);
}

/* surfaceIntegralNonlinear: 3d/surfaceIntegralNonlinear.cpph:21-90, 2d:26-67 */
void orc_surface_integral(const orc_solver* s, double* lduh, const double* lFhbnd, const double* dx) {
  geo g = mkgeo(s);
  const int b = g.b, nV = g.nV, F = g.F;
  double invDx[3];
  for (int i = 0; i < g.d; i++) invDx[i] = 1.0 / dx[i];
#define FB(face, fn, v) lFhbnd[((face) * F + (fn)) * nV + (v)]
  /* x faces */
  for (int z = 0; z < g.nz; z++)
    for (int y = 0; y < b; y++) {
      const double us = (g.wz[z] * g.w[y]) * invDx[0];
      const int fn = z * b + y;
      for (int x = 0; x < b; x++)
        for (int v = 0; v < nV; v++)
          lduh[PT(g, z, y, x) * nV + v] -= (FB(1, fn, v) * g.FR[x] - FB(0, fn, v) * g.FL[x]) * us;
    }
  /* y faces */
  for (int z = 0; z < g.nz; z++)
    for (int y = 0; y < b; y++)
      for (int x = 0; x < b; x++) {
        const double us = (g.wz[z] * g.w[x]) * invDx[1];
        const int fn = z * b + x;
        for (int v = 0; v < nV; v++)
          lduh[PT(g, z, y, x) * nV + v] -= (FB(3, fn, v) * g.FR[y] - FB(2, fn, v) * g.FL[y]) * us;
      }
  /* z faces */
  if (g.d == 3)
    for (int z = 0; z < g.nz; z++)
      for (int y = 0; y < b; y++)
        for (int x = 0; x < b; x++) {
          const double us = (g.w[y] * g.w[x]) * invDx[2];
          const int fn = y * b + x;
          for (int v = 0; v < nV; v++)
            lduh[PT(g, z, y, x) * nV + v] -= (FB(5, fn, v) * g.FR[z] - FB(4, fn, v) * g.FL[z]) * us;
        }
#undef FB
}

/* solutionUpdate: 3d/solutionUpdate.cpph:23-47, 2d:23-45 */
void orc_solution_update(const orc_solver* s, double* luh, const double* lduh, double dt) {
  geo g = mkgeo(s);
  for (int z = 0; z < g.nz; z++)
    for (int y = 0; y < g.b; y++)
      for (int x = 0; x < g.b; x++) {
        const double weight = g.wz[z] * g.w[y] * g.w[x];
        const double us = dt / weight;
        const int p = PT(g, z, y, x);
        for (int v = 0; v < g.nV; v++) luh[p * g.nD + v] += lduh[p * g.nV + v] * us;
      }
}

/* stableTimeStepSize: 3d/stableTimeStepSize.cpph:21-63, 2d:13-58; CFL 0.9 from
 * Toolkit/.../AbstractGenericADERDGSolverHeader.template:35 */
double orc_stable_dt(const orc_solver* s, const double* luh, const double* dx) {
  static const double PNPM[10] = {1.0, 0.33, 0.17, 0.1, 0.069, 0.045, 0.038, 0.03, 0.02, 0.015};
  const double cfl = 0.9;
  geo g = mkgeo(s);
  double invDx[3];
  for (int i = 0; i < g.d; i++) invDx[i] = 1.0 / dx[i];
  double dt = DBL_MAX;
  for (int p = 0; p < g.P; p++) {
    double den = 0.0;
    for (int d = 0; d < g.d; d++) {
      double lam[16];
      orc_eigenvalues(s, luh + p * g.nD, d, lam);
      double me = 0.0;
      for (int k = 0; k < g.nV; k++) me = dmax(fabs(lam[k]), me);
      den += me * invDx[d];
    }
    dt = dmin(dt, cfl * PNPM[g.N] / den);
  }
  return dt;
}
