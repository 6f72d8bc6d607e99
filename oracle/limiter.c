/*
 * ORACLE -- test infrastructure only (see oracle.h). Plain-C restatement of
 * the reference's a-posteriori subcell limiter kernels and the FV
 * MUSCL-Hancock update, Euler PDE (nD = nV = 5):
 *   kernels/limiter/generic/c/Limiter.cpp                 (projections, DMP, min/max)
 *   kernels/finitevolumes/musclhancock/c/{2d,3d}/musclhancock.cpph
 *   kernels/finitevolumes/riemannsolvers/c/rusanov.cpph
 *   kernels/finitevolumes/commons/c/commons.cpph          (ghost layers, FV boundary)
 * FV patches carry g = 2 ghost layers: lim[(z)][y][x][nV] with E = 2N+1+2g
 * cells per axis. The ghost corners are never written by halo exchange and
 * stay zero, as in the reference's zero-initialised patch storage.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
void orc_fv_boundary_fill_kind(const orc_solver* s, double* lim, int face, int kind);

#define GW 2 /* ghost layer width (GenericFiniteVolumesMUSCLHancockInC.java:12) */

static int E_of(const orc_solver* s) { return 2 * s->order + 1 + 2 * GW; }
int orc_fv_patch_size(const orc_solver* s) {
  const int E = E_of(s);
  return (s->dim == 3 ? E * E * E : E * E) * orc_nvar(s);
}

static double dmax(double a, double b) { return (a < b) ? b : a; }
static double dmin(double a, double b) { return (b < a) ? b : a; }

/* projectOnFVLimiterSpace, Limiter.cpp:23-66 (interior cells only) */
void orc_project_fv(const orc_solver* s, const double* luh, double* lim) {
  const int b = s->order + 1, B = 2 * s->order + 1, nV = orc_nvar(s), E = E_of(s);
  const int b3 = s->dim == 3 ? b : 1, B3 = s->dim == 3 ? B : 1, g3 = s->dim == 3 ? GW : 0, E3 = s->dim == 3 ? E : 1;
  const double* C = orc_table("uh2lim", s->order); /* [k][i] */
  for (int z = g3; z < B3 + g3; z++)
    for (int y = GW; y < B + GW; y++)
      for (int x = GW; x < B + GW; x++)
        for (int v = 0; v < nV; v++) {
          double acc = 0;
          for (int iz = 0; iz < b3; iz++)
            for (int iy = 0; iy < b; iy++)
              for (int ix = 0; ix < b; ix++) {
                double t = luh[((iz * b + iy) * b + ix) * nV + v];
                if (s->dim == 3) t *= C[iz * B + (z - g3)];
                acc += t * C[iy * B + (y - GW)] * C[ix * B + (x - GW)];
              }
          lim[((z * E + y) * E + x) * nV + v] = acc;
        }
  (void)E3;
}

/* projectOnDGSpace, Limiter.cpp:69-112 */
void orc_project_dg(const orc_solver* s, const double* lim, double* luh) {
  const int b = s->order + 1, B = 2 * s->order + 1, nV = orc_nvar(s), E = E_of(s);
  const int b3 = s->dim == 3 ? b : 1, B3 = s->dim == 3 ? B : 1, g3 = s->dim == 3 ? GW : 0;
  const double* C = orc_table("lim2uh", s->order); /* [i][j] */
  for (int z = 0; z < b3; z++)
    for (int y = 0; y < b; y++)
      for (int x = 0; x < b; x++)
        for (int v = 0; v < nV; v++) {
          double acc = 0;
          for (int iz = g3; iz < B3 + g3; iz++)
            for (int iy = GW; iy < B + GW; iy++)
              for (int ix = GW; ix < B + GW; ix++) {
                double t = lim[((iz * E + iy) * E + ix) * nV + v];
                if (s->dim == 3) t *= C[(iz - g3) * b + z];
                acc += t * C[(iy - GW) * b + y] * C[(ix - GW) * b + x];
              }
          luh[((z * b + y) * b + x) * nV + v] = acc;
        }
}

/* findCellLocalMinAndMax + compareWithADERDGSolutionAtGaussLobattoNodes +
 * compareWithADERDGSolutionAtFVSubcellCenters, Limiter.cpp:210-368; the
 * observables of Euler are the conserved variables (MyEulerSolver_ADERDG.cpp:137-145). */
void orc_local_minmax(const orc_solver* s, const double* luh, double* mn, double* mx) {
  const int b = s->order + 1, B = 2 * s->order + 1, nV = orc_nvar(s);
  const int b3 = s->dim == 3 ? b : 1, B3 = s->dim == 3 ? B : 1;
  for (int v = 0; v < nV; v++) {
    mn[v] = DBL_MAX;
    mx[v] = -DBL_MAX;
  }
  for (int p = 0; p < b3 * b * b; p++)
    for (int v = 0; v < nV; v++) {
      mn[v] = dmin(mn[v], luh[p * nV + v]);
      mx[v] = dmax(mx[v], luh[p * nV + v]);
    }
  const double* L = orc_table("uh2lob", s->order); /* [j][i] */
  for (int z = 0; z < b3; z++)
    for (int y = 0; y < b; y++)
      for (int x = 0; x < b; x++)
        for (int v = 0; v < nV; v++) {
          double acc = 0.0;
          for (int iz = 0; iz < b3; iz++)
            for (int iy = 0; iy < b; iy++)
              for (int ix = 0; ix < b; ix++) {
                double t = luh[((iz * b + iy) * b + ix) * nV + v];
                if (s->dim == 3) t *= L[iz * b + z];
                acc += t * L[iy * b + y] * L[ix * b + x];
              }
          mn[v] = dmin(mn[v], acc);
          mx[v] = dmax(mx[v], acc);
        }
  const double* C = orc_table("uh2lim", s->order);
  for (int z = 0; z < B3; z++)
    for (int y = 0; y < B; y++)
      for (int x = 0; x < B; x++)
        for (int v = 0; v < nV; v++) {
          double acc = 0.0;
          for (int iz = 0; iz < b3; iz++)
            for (int iy = 0; iy < b; iy++)
              for (int ix = 0; ix < b; ix++) {
                double t = luh[((iz * b + iy) * b + ix) * nV + v];
                if (s->dim == 3) t *= C[iz * B + z];
                acc += t * C[iy * B + y] * C[ix * B + x];
              }
          mn[v] = dmin(mn[v], acc);
          mx[v] = dmax(mx[v], acc);
        }
}

/* findCellLocalLimiterMinAndMax, Limiter.cpp:167-205 (interior subcells) */
void orc_limiter_minmax(const orc_solver* s, const double* lim, double* mn, double* mx) {
  const int B = 2 * s->order + 1, nV = orc_nvar(s), E = E_of(s);
  const int B3 = s->dim == 3 ? B : 1, g3 = s->dim == 3 ? GW : 0;
  for (int v = 0; v < nV; v++) {
    mn[v] = DBL_MAX;
    mx[v] = -DBL_MAX;
  }
  for (int z = g3; z < B3 + g3; z++)
    for (int y = GW; y < B + GW; y++)
      for (int x = GW; x < B + GW; x++)
        for (int v = 0; v < nV; v++) {
          const double q = lim[((z * E + y) * E + x) * nV + v];
          mn[v] = dmin(mn[v], q);
          mx[v] = dmax(mx[v], q);
        }
}

/* discreteMaximumPrincipleAndMinAndMaxSearch, Limiter.cpp:114-165: returns 1
 * if the DMP holds; block 0 <- new local min/max, block 1 <- boundary min/max */
int orc_dmp(const orc_solver* s, const double* luh, double relax, double scale, double* minB, double* maxB) {
  const int nO = orc_nvar(s), D2 = 2 * s->dim;
  double lmin[8], lmax[8];
  orc_local_minmax(s, luh, lmin, lmax);
  int ok = 1;
  for (int v = 0; v < nO; v++) {
    double bmin = minB[v], bmax = maxB[v];
    for (int i = 1; i < D2; i++) bmin = dmin(bmin, minB[i * nO + v]);
    for (int i = 1; i < D2; i++) bmax = dmax(bmax, maxB[i * nO + v]);
    double sd = (bmax - bmin) * scale;
    sd = dmax(sd, relax);
    if ((lmin[v] < (bmin - sd)) || (lmax[v] > (bmax + sd))) ok = 0;
    minB[v] = lmin[v];
    maxB[v] = lmax[v];
    minB[v + nO] = bmin;
    maxB[v + nO] = bmax;
  }
  return ok;
}

/* Euler isPhysicallyAdmissible (MyEulerSolver_ADERDG.cpp:147-160) */
int orc_admissible(const orc_solver* s, const double* obsMin) {
  (void)s;
  if (obsMin[0] <= 0.0) return 0;
  if (obsMin[4] <= 0.0) return 0;
  return 1;
}

/* FV Rusanov, riemannsolvers/c/rusanov.cpph:24-83 (2D) / :98-156 (3D) */
static double fv_rusanov(const orc_solver* s, double* fnL, double* fnR, const double* qL, const double* qR, int d) {
  const int nV = 5;
  double sL[5], sR[5];
  orc_eigenvalues(s, qL, d, sL);
  orc_eigenvalues(s, qR, d, sR);
  double smax = -1.0;
  for (int i = 0; i < nV; i++) smax = dmax(fabs(sL[i]), smax);
  for (int i = 0; i < nV; i++) smax = dmax(fabs(sR[i]), smax);
  double FL[15], FR[15];
  orc_flux(s, qL, FL);
  orc_flux(s, qR, FR);
  for (int i = 0; i < nV; i++) {
    fnL[i] = 0.5 * smax * (qL[i] - qR[i]);
    fnL[i] += 0.5 * (FL[d * 5 + i] + FR[d * 5 + i]);
    fnR[i] = fnL[i];
  }
  return smax;
}

static double minmod(double a, double b) { /* musclhancock.cpph:29-38 */
  if (a * b < 0.0) return 0.0;
  if (fabs(a) < fabs(b)) return a;
  return b;
}

/* musclhancock::c::solutionUpdate (2d/musclhancock.cpph:50-276,
 * 3d/musclhancock.cpph) without source/NCP: lnew must hold a copy of lold
 * (ghosts included). Returns the admissible FV step (diagnostic only). */
double orc_musclhancock(const orc_solver* s, double* lnew, const double* lold, const double* dx, double dt) {
  const int d3 = s->dim == 3;
  const int B = 2 * s->order + 1, E = E_of(s), nV = 5, pB = GW, pE = GW + B;
  const int zlo = d3 ? pB - 1 : 0, zhi = d3 ? pE + 1 : 1; /* z range incl. the first ghost ring */
  const double cflFactor = 0.99; /* musclhancock.h:27 */
  double cs[3], ics[3], icsdt[3];
  for (int d = 0; d < s->dim; d++) {
    cs[d] = dx[d] / B;
    ics[d] = 1. / cs[d];
    icsdt[d] = dt * ics[d];
  }
  const int nc = (d3 ? E : 1) * E * E;
#define ID(z, y, x) ((((z) * E + (y)) * E + (x)) * nV)
  double* slope = (double*)calloc((size_t)nc * 3 * nV, sizeof(double));
  double* w = (double*)calloc((size_t)nc * 6 * nV, sizeof(double)); /* wL/wR per direction */
#define SL(z, y, x, d, v) slope[((((z) * E + (y)) * E + (x)) * 3 + (d)) * nV + (v)]
#define WL(z, y, x, d, v) w[((((z) * E + (y)) * E + (x)) * 6 + 2 * (d)) * nV + (v)]
#define WR(z, y, x, d, v) w[((((z) * E + (y)) * E + (x)) * 6 + 2 * (d) + 1) * nV + (v)]
  /* slopes, incl. the first ghost ring (:80-99) */
  for (int z = zlo; z < zhi; z++)
    for (int y = pB - 1; y < pE + 1; y++)
      for (int x = pB - 1; x < pE + 1; x++)
        for (int v = 0; v < nV; v++) {
          const double* u = lold;
          SL(z, y, x, 0, v) = minmod(u[ID(z, y, x + 1) + v] - u[ID(z, y, x) + v], u[ID(z, y, x) + v] - u[ID(z, y, x - 1) + v]) * ics[0];
          SL(z, y, x, 1, v) = minmod(u[ID(z, y + 1, x) + v] - u[ID(z, y, x) + v], u[ID(z, y, x) + v] - u[ID(z, y - 1, x) + v]) * ics[1];
          if (d3)
            SL(z, y, x, 2, v) = minmod(u[ID(z + 1, y, x) + v] - u[ID(z, y, x) + v], u[ID(z, y, x) + v] - u[ID(z - 1, y, x) + v]) * ics[2];
        }
  /* boundary extrapolation (:108-127) */
  for (int z = zlo; z < zhi; z++)
    for (int y = pB - 1; y < pE + 1; y++)
      for (int x = pB - 1; x < pE + 1; x++)
        for (int d = 0; d < s->dim; d++)
          for (int v = 0; v < nV; v++) {
            const double u = lold[ID(z, y, x) + v];
            WL(z, y, x, d, v) = u - 0.5 * cs[d] * SL(z, y, x, d, v);
            WR(z, y, x, d, v) = u + 0.5 * cs[d] * SL(z, y, x, d, v);
          }
  /* half-step evolution with flux differences (:138-194); ghost-ring corners
   * of the reference's skip test are never read by the edge loops below */
  for (int z = zlo; z < zhi; z++)
    for (int y = pB - 1; y < pE + 1; y++)
      for (int x = pB - 1; x < pE + 1; x++) {
        double Qt[5] = {0, 0, 0, 0, 0};
        double F[15];
        for (int d = 0; d < s->dim; d++) {
          double wl[5], wr[5];
          for (int v = 0; v < nV; v++) {
            wl[v] = WL(z, y, x, d, v);
            wr[v] = WR(z, y, x, d, v);
          }
          orc_flux(s, wl, F);
          for (int v = 0; v < nV; v++) Qt[v] += F[d * 5 + v] * ics[d];
          orc_flux(s, wr, F);
          for (int v = 0; v < nV; v++) Qt[v] -= F[d * 5 + v] * ics[d];
        }
        for (int d = 0; d < s->dim; d++)
          for (int v = 0; v < nV; v++) {
            WL(z, y, x, d, v) += 0.5 * dt * Qt[v];
            WR(z, y, x, d, v) += 0.5 * dt * Qt[v];
          }
      }
  /* Riemann problems on the subcell faces (:197-238) */
  double dtmax = DBL_MAX;
  double fL[5], fR[5], ql[5], qr[5];
  const int zi0 = d3 ? pB : 0, zi1 = d3 ? pE : 1;
  for (int z = zi0; z < zi1; z++)
    for (int y = pB; y < pE; y++)
      for (int x = pB - 1; x < pE; x++) {
        for (int v = 0; v < nV; v++) {
          ql[v] = WR(z, y, x, 0, v);
          qr[v] = WL(z, y, x + 1, 0, v);
        }
        const double sm = fv_rusanov(s, fL, fR, ql, qr, 0);
        dtmax = dmin(dtmax, cflFactor / s->dim * cs[0] / sm);
        for (int v = 0; v < nV; v++) {
          lnew[ID(z, y, x) + v] -= icsdt[0] * fL[v];
          lnew[ID(z, y, x + 1) + v] += icsdt[0] * fR[v];
        }
      }
  for (int z = zi0; z < zi1; z++)
    for (int y = pB - 1; y < pE; y++)
      for (int x = pB; x < pE; x++) {
        for (int v = 0; v < nV; v++) {
          ql[v] = WR(z, y, x, 1, v);
          qr[v] = WL(z, y + 1, x, 1, v);
        }
        const double sm = fv_rusanov(s, fL, fR, ql, qr, 1);
        dtmax = dmin(dtmax, cflFactor / s->dim * cs[1] / sm);
        for (int v = 0; v < nV; v++) {
          lnew[ID(z, y, x) + v] -= icsdt[1] * fL[v];
          lnew[ID(z, y + 1, x) + v] += icsdt[1] * fR[v];
        }
      }
  if (d3)
    for (int z = pB - 1; z < pE; z++)
      for (int y = pB; y < pE; y++)
        for (int x = pB; x < pE; x++) {
          for (int v = 0; v < nV; v++) {
            ql[v] = WR(z, y, x, 2, v);
            qr[v] = WL(z + 1, y, x, 2, v);
          }
          const double sm = fv_rusanov(s, fL, fR, ql, qr, 2);
          dtmax = dmin(dtmax, cflFactor / s->dim * cs[2] / sm);
          for (int v = 0; v < nV; v++) {
            lnew[ID(z, y, x) + v] -= icsdt[2] * fL[v];
            lnew[ID(z + 1, y, x) + v] += icsdt[2] * fR[v];
          }
        }
  free(slope);
  free(w);
  return dtmax;
#undef ID
#undef SL
#undef WL
#undef WR
}

/* ghostLayerFilling (commons.cpph:336-401 2D, :873-981 3D): fill the g ghost
 * layers of `lim` on side `face` (0:-x 1:+x 2:-y 3:+y 4:-z 5:+z) from the
 * neighbour patch `nb` across that face. */
void orc_fv_ghost_fill(const orc_solver* s, double* lim, const double* nb, int face) {
  const int B = 2 * s->order + 1, E = E_of(s), nV = orc_nvar(s), pB = GW, pE = GW + B;
  const int d = face / 2, side = face % 2;
  const int d3 = s->dim == 3;
  const int z0 = d3 ? pB : 0, z1 = d3 ? pE : 1;
  for (int a = (d == 2 ? pB : z0); a < (d == 2 ? pE : z1); a++) /* outer transverse coordinate */
    for (int c = pB; c < pE; c++)
      for (int k = 0; k < GW; k++) {
        /* ghost index along d and the neighbour's source index */
        const int gi = side ? pE + k : k;
        const int si = side ? pB + k : pE - GW + k;
        int dz, dy, dx, sz, sy, sx;
        if (d == 0) { dz = a; dy = c; dx = gi; sz = a; sy = c; sx = si; }
        else if (d == 1) { dz = a; dy = gi; dx = c; sz = a; sy = si; sx = c; }
        else { dz = gi; dy = a; dx = c; sz = si; sy = a; sx = c; }
        memcpy(lim + ((dz * E + dy) * E + dx) * nV, nb + ((sz * E + sy) * E + sx) * nV, sizeof(double) * nV);
      }
}

/* FV boundary face: boundaryLayerExtraction + boundaryConditions (the inside
 * state of the mirrored layer through the FV solver's boundaryValues) +
 * ghostLayerFillingAtBoundary (commons.cpph:98-334, FiniteVolumesSolver.cpp:
 * 805-842). kind 0 outflow: stateOut = stateIn; kind 1 reflective, the
 * EulerADERDG demonstrator's MyEulerSolver_FV.cpp:47-62: the normal momentum
 * negated. */
void orc_fv_boundary_fill(const orc_solver* s, double* lim, int face) { orc_fv_boundary_fill_kind(s, lim, face, 0); }

void orc_fv_boundary_fill_kind(const orc_solver* s, double* lim, int face, int kind) {
  const int B = 2 * s->order + 1, E = E_of(s), nV = orc_nvar(s), pB = GW, pE = GW + B;
  const int d = face / 2, side = face % 2;
  const int d3 = s->dim == 3;
  const int z0 = d3 ? pB : 0, z1 = d3 ? pE : 1;
  for (int a = (d == 2 ? pB : z0); a < (d == 2 ? pE : z1); a++)
    for (int c = pB; c < pE; c++)
      for (int k = 0; k < GW; k++) {
        const int K = GW - k - 1;
        /* left face: ghost k <- interior layer pB+K; right face: ghost pE+k <- interior pE-GW+K.
         * 3D y- and z-left faces: the reference's boundaryLayerExtraction
         * (commons.cpph:551-562, :581-592) copies the first interior layer
         * pB into both boundary layers, so both ghosts come from pB. */
        const int gi = side ? pE + k : k;
        const int si = side ? pE - GW + K : (d3 && d >= 1 ? pB : pB + K);
        int dz, dy, dx, sz, sy, sx;
        if (d == 0) { dz = a; dy = c; dx = gi; sz = a; sy = c; sx = si; }
        else if (d == 1) { dz = a; dy = gi; dx = c; sz = a; sy = si; sx = c; }
        else { dz = gi; dy = a; dx = c; sz = si; sy = a; sx = c; }
        double* out = lim + ((dz * E + dy) * E + dx) * nV;
        memcpy(out, lim + ((sz * E + sy) * E + sx) * nV, sizeof(double) * nV);
        if (kind == 1) out[1 + d] = -out[1 + d];
      }
}
