/*
 * ORACLE -- test infrastructure only (see oracle.h). Plain-C restatement of
 * the reference's AMR transfer operators between a cell (or face) and its
 * descendants levelDelta levels finer, ExaHyPE/kernels/aderdg/generic/c/
 * {2d,3d}/amrRoutines.cpph, and of the equidistant-grid projection the
 * plotters use (exahype/tests/kernels/c/GenericEulerKernelTest.cpp:67-121,
 * kernels::equidistantGridProjector1d), in the reference's loop nesting and
 * operation order (compiled with -ffp-contract=off):
 *
 *   faceUnknownsProlongation    3d:42-134,  2d:41-135
 *   faceUnknownsRestriction     3d:169-246, 2d:168-255
 *   volumeUnknownsProlongation  3d:307-369, 2d:282-355
 *   volumeUnknownsRestriction   3d:404-466, 2d:386-452
 *
 * A subcell (subface) index holds one base-3 digit per level, the most
 * significant digit for the level next to the coarse cell; prolongation
 * applies the single-level operators from the coarse level down,
 * restriction from the fine level up and adds the result to the coarse data.
 * P = fineGridProjector1d[N][third][n][m] = phi_n((third + x_m) / 3).
 * Data are [node][var] with the first index (x, or the inner face
 * coordinate) fastest; nvar counts every value per node (parameters
 * included).
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define AMAXB 10

static const double* proj(int N, int third) { return orc_table("fineGridProjector1d", N) + third * (N + 1) * (N + 1); }

/* single level, volume, 2D / 3D (amrRoutines.cpph singleLevelVolumeUnknowns*) */
static void vol_prolong1(int dim, int N, int nvar, double* fine, const double* coarse, const int* s) {
  const int b = N + 1;
  const double *P0 = proj(N, s[0]), *P1 = proj(N, s[1]), *P2 = dim == 3 ? proj(N, s[2]) : 0;
  if (dim == 2) {
    for (int m2 = 0; m2 < b; ++m2)
      for (int m1 = 0; m1 < b; ++m1)
        for (int iv = 0; iv < nvar; iv++)
          for (int n2 = 0; n2 < b; ++n2)
            for (int n1 = 0; n1 < b; ++n1)
              fine[(m2 * b + m1) * nvar + iv] += coarse[(n2 * b + n1) * nvar + iv] * P0[n1 * b + m1] * P1[n2 * b + m2];
    return;
  }
  for (int m3 = 0; m3 < b; ++m3)
    for (int m2 = 0; m2 < b; ++m2)
      for (int m1 = 0; m1 < b; ++m1)
        for (int iv = 0; iv < nvar; iv++)
          for (int n3 = 0; n3 < b; ++n3)
            for (int n2 = 0; n2 < b; ++n2)
              for (int n1 = 0; n1 < b; ++n1)
                fine[((m3 * b + m2) * b + m1) * nvar + iv] += coarse[((n3 * b + n2) * b + n1) * nvar + iv] *
                                                              P0[n1 * b + m1] * P1[n2 * b + m2] * P2[n3 * b + m3];
}

static void vol_restrict1(int dim, int N, int nvar, double* coarse, const double* fine, const int* s) {
  const int b = N + 1;
  const double* w = orc_table("weights", N);
  const double *P0 = proj(N, s[0]), *P1 = proj(N, s[1]), *P2 = dim == 3 ? proj(N, s[2]) : 0;
  if (dim == 2) {
    for (int m2 = 0; m2 < b; ++m2)
      for (int m1 = 0; m1 < b; ++m1)
        for (int iv = 0; iv < nvar; iv++)
          for (int n2 = 0; n2 < b; ++n2)
            for (int n1 = 0; n1 < b; ++n1)
              coarse[(m2 * b + m1) * nvar + iv] += w[n1] * w[n2] * P0[m1 * b + n1] * P1[m2 * b + n2] *
                                                   fine[(n2 * b + n1) * nvar + iv] / w[m1] / w[m2] / 9.0;
    return;
  }
  for (int m3 = 0; m3 < b; ++m3)
    for (int m2 = 0; m2 < b; ++m2)
      for (int m1 = 0; m1 < b; ++m1)
        for (int iv = 0; iv < nvar; iv++)
          for (int n3 = 0; n3 < b; ++n3)
            for (int n2 = 0; n2 < b; ++n2)
              for (int n1 = 0; n1 < b; ++n1)
                coarse[((m3 * b + m2) * b + m1) * nvar + iv] +=
                    w[n1] * w[n2] * w[n3] * P0[m1 * b + n1] * P1[m2 * b + n2] * P2[m3 * b + n3] *
                    fine[((n3 * b + n2) * b + n1) * nvar + iv] / w[m1] / w[m2] / w[m3] / 27.0;
}

/* single level, face (one dimension lower than the cell) */
static void face_prolong1(int dim, int N, int nvar, double* fine, const double* coarse, const int* s) {
  const int b = N + 1;
  const double *P0 = proj(N, s[0]), *P1 = dim == 3 ? proj(N, s[1]) : 0;
  if (dim == 2) {
    for (int m1 = 0; m1 < b; ++m1)
      for (int iv = 0; iv < nvar; ++iv)
        for (int n1 = 0; n1 < b; ++n1) fine[m1 * nvar + iv] += coarse[n1 * nvar + iv] * P0[n1 * b + m1];
    return;
  }
  for (int m2 = 0; m2 < b; ++m2)
    for (int m1 = 0; m1 < b; ++m1)
      for (int iv = 0; iv < nvar; ++iv)
        for (int n2 = 0; n2 < b; ++n2)
          for (int n1 = 0; n1 < b; ++n1)
            fine[(m2 * b + m1) * nvar + iv] += coarse[(n2 * b + n1) * nvar + iv] * P0[n1 * b + m1] * P1[n2 * b + m2];
}

static void face_restrict1(int dim, int N, int nvar, double* coarse, const double* fine, const int* s) {
  const int b = N + 1;
  const double* w = orc_table("weights", N);
  const double *P0 = proj(N, s[0]), *P1 = dim == 3 ? proj(N, s[1]) : 0;
  if (dim == 2) {
    for (int m1 = 0; m1 < b; ++m1)
      for (int iv = 0; iv < nvar; ++iv)
        for (int n1 = 0; n1 < b; ++n1)
          coarse[m1 * nvar + iv] += w[n1] * P0[m1 * b + n1] * fine[n1 * nvar + iv] / w[m1] / 3.0;
    return;
  }
  for (int m2 = 0; m2 < b; ++m2)
    for (int m1 = 0; m1 < b; ++m1)
      for (int iv = 0; iv < nvar; ++iv)
        for (int n2 = 0; n2 < b; ++n2)
          for (int n1 = 0; n1 < b; ++n1)
            coarse[(m2 * b + m1) * nvar + iv] +=
                w[n1] * w[n2] * P0[m1 * b + n1] * P1[m2 * b + n2] * fine[(n2 * b + n1) * nvar + iv] / w[m1] / w[m2] / 9.0;
}

static int ipow3(int e) {
  int r = 1;
  while (e-- > 0) r *= 3;
  return r;
}

typedef void (*level_op)(int, int, int, double*, const double*, const int*);

/* prolongation: digits from the most significant (3^(levelDelta-1)) down;
 * the buffers alternate so that the last level is written to `fine` */
static void prolong(level_op op, int dim, int N, int nvar, int nidx, int size, double* fine, const double* coarse,
                    int levelDelta, const int* index) {
  double* tmp = (double*)calloc(size, sizeof(double));
  double* cur = (levelDelta % 2 == 0) ? tmp : fine;
  const double* prev = coarse;
  int rest[3] = {0, 0, 0}, digit[3] = {0, 0, 0};
  for (int k = 0; k < nidx; k++) rest[k] = index[k];
  for (int l = 1; l <= levelDelta; l++) {
    const int sig = ipow3(levelDelta - l);
    for (int k = 0; k < nidx; k++) {
      digit[k] = (rest[k] - rest[k] % sig) / sig;
      rest[k] = rest[k] % sig;
    }
    memset(cur, 0, sizeof(double) * size);
    op(dim, N, nvar, cur, prev, digit);
    prev = cur;
    cur = (cur == tmp) ? fine : tmp;
  }
  free(tmp);
}

/* restriction: digits from the least significant up, result added to coarse */
static void restrict_(level_op op, int dim, int N, int nvar, int nidx, int size, double* coarse, const double* fine,
                      int levelDelta, const int* index) {
  double* t1 = (double*)calloc(size, sizeof(double));
  double* t2 = (double*)calloc(size, sizeof(double));
  double* cur = t1;
  const double* prev = fine;
  int rest[3] = {0, 0, 0}, digit[3] = {0, 0, 0};
  for (int k = 0; k < nidx; k++) rest[k] = index[k];
  for (int l = 1; l <= levelDelta; l++) {
    for (int k = 0; k < nidx; k++) {
      digit[k] = rest[k] % 3;
      rest[k] = (rest[k] - digit[k]) / 3;
    }
    memset(cur, 0, sizeof(double) * size);
    op(dim, N, nvar, cur, prev, digit);
    prev = cur;
    cur = (cur == t1) ? t2 : t1;
  }
  for (int i = 0; i < size; i++) coarse[i] += prev[i];
  free(t1);
  free(t2);
}

static int cell_size(int dim, int N, int nvar) { return (dim == 3 ? (N + 1) * (N + 1) * (N + 1) : (N + 1) * (N + 1)) * nvar; }
static int face_size(int dim, int N, int nvar) { return (dim == 3 ? (N + 1) * (N + 1) : (N + 1)) * nvar; }

void orc_volume_prolongation(int dim, int N, int nvar, double* luhFine, const double* luhCoarse, int levelDelta,
                             const int* subcellIndex) {
  if (levelDelta < 1) return;
  prolong(vol_prolong1, dim, N, nvar, dim, cell_size(dim, N, nvar), luhFine, luhCoarse, levelDelta, subcellIndex);
}
void orc_volume_restriction(int dim, int N, int nvar, double* luhCoarse, const double* luhFine, int levelDelta,
                            const int* subcellIndex) {
  if (levelDelta < 1) return;
  restrict_(vol_restrict1, dim, N, nvar, dim, cell_size(dim, N, nvar), luhCoarse, luhFine, levelDelta, subcellIndex);
}
/* faces: the state slab (nvar values per node) and the flux slab (nflux) */
void orc_face_prolongation(int dim, int N, int nvar, int nflux, double* lQhbndFine, double* lFhbndFine,
                           const double* lQhbndCoarse, const double* lFhbndCoarse, int levelDelta,
                           const int* subfaceIndex) {
  if (levelDelta < 1) return;
  prolong(face_prolong1, dim, N, nvar, dim - 1, face_size(dim, N, nvar), lQhbndFine, lQhbndCoarse, levelDelta,
          subfaceIndex);
  prolong(face_prolong1, dim, N, nflux, dim - 1, face_size(dim, N, nflux), lFhbndFine, lFhbndCoarse, levelDelta,
          subfaceIndex);
}
void orc_face_restriction(int dim, int N, int nvar, int nflux, double* lQhbndCoarse, double* lFhbndCoarse,
                          const double* lQhbndFine, const double* lFhbndFine, int levelDelta, const int* subfaceIndex) {
  if (levelDelta < 1) return;
  restrict_(face_restrict1, dim, N, nvar, dim - 1, face_size(dim, N, nvar), lQhbndCoarse, lQhbndFine, levelDelta,
            subfaceIndex);
  restrict_(face_restrict1, dim, N, nflux, dim - 1, face_size(dim, N, nflux), lFhbndCoarse, lFhbndFine, levelDelta,
            subfaceIndex);
}

/* values of one cell at the (N+1)^d equidistant points i/N of each axis
 * (the vertices ADERDG2CartesianVTK::plotVertexData writes,
 * exahype/plotters/VTK/ADERDG2CartesianVTK.cpp), out[point][var] with x
 * fastest: sum over Gauss nodes of E[ii_y][i_y] E[ii_x][i_x] (E[ii_z][i_z])
 * u[node][var], E = equidistantGridProjector1d[N] */
void orc_equidistant_projection(int dim, int N, int nvar, const double* luh, double* out) {
  const int b = N + 1, nz = dim == 3 ? b : 1;
  const double* E = orc_table("equidistantGridProjector1d", N);
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < b; iy++)
      for (int ix = 0; ix < b; ix++)
        for (int v = 0; v < nvar; v++) {
          double value = 0.0;
          for (int gz = 0; gz < nz; gz++)
            for (int gy = 0; gy < b; gy++)
              for (int gx = 0; gx < b; gx++) {
                const double e = dim == 3 ? E[gy * b + iy] * E[gx * b + ix] * E[gz * b + iz] : E[gy * b + iy] * E[gx * b + ix];
                value += e * luh[((gz * b + gy) * b + gx) * nvar + v];
              }
          out[((iz * b + iy) * b + ix) * nvar + v] = value;
        }
}
