/*
 * ORACLE -- test infrastructure only. A plain-C restatement of ExaHyPE's
 * generic nonlinear ADER-DG kernels, limiter kernels and FV MUSCL-Hancock
 * update, plus a uniform-mesh harness that sequences them the way the
 * reference solver does. It is the checker for the CUDA path: only the test
 * suite, the smoke check and the bench's CPU-baseline leg may call it.
 *
 * Parity pins: tests/golden/ (the reference's own kernel-test vectors) and the
 * reference kernels themselves compiled from source into oracle/_ref/.
 */
#ifndef EXA_ORACLE_H
#define EXA_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* PDE ids: 0 = Euler as in the EulerADERDG demonstrator (outflow boundary),
 *          1 = the "2.5D" Euler mock of the reference kernel tests (nPar = 1),
 *          2 = linear elastic waves of the reference kernel tests (nVar = 9,
 *              nPar = 3: lambda, mu, rho; linear kernels only),
 *          3 = pde 1 with an algebraic source and the kernel tests' non-zero
 *              non-conservative product (useSource = useNCP = true),
 *          4 = pde 2 with a point source (usePointSource = true): ps holds
 *              its position x0[3], delay t0, peak frequency f0, amplitude. */
typedef struct {
  int dim;   /* 2 or 3 */
  int order; /* N, basis size N+1 */
  int pde;
  double ps[6];
} orc_solver;

/* the elastic-wave PDEs (2, 4) */
#define ORC_ELASTIC(s) ((s)->pde == 2 || (s)->pde == 4)

int orc_nvar(const orc_solver* s);
int orc_npar(const orc_solver* s);

/* spaceTimePredictorNonlinear (+ volumeIntegralNonlinear when lduh != 0).
 * Optional temporaries in the reference layouts (may be 0):
 *   lQi[z][y][x][t][nD], lFi[t][z][y][x][d+1][nV], lQhi[z][y][x][nD],
 *   lFhi[d+1][..][nV] (per-direction transposed blocks).
 * Returns the number of Picard sweeps executed. */
int orc_predictor(const orc_solver* s, const double* luh, const double* dx, double dt, double* lQhbnd,
                  double* lFhbnd, double* lduh, double* lQi, double* lFi, double* lQhi, double* lFhi);
void orc_volume_integral(const orc_solver* s, double* lduh, const double* lFhi, const double* dx);
void orc_riemann(const orc_solver* s, double* FL, double* FR, const double* QL, const double* QR, int dir);
void orc_boundary_face(const orc_solver* s, double* FIn, const double* QIn, const double* centre,
                       const double* size, double t, double dt, int faceIndex);
void orc_boundary_face_reflective(const orc_solver* s, double* FIn, const double* QIn, int faceIndex);
void orc_surface_integral(const orc_solver* s, double* lduh, const double* lFhbnd, const double* dx);
void orc_solution_update(const orc_solver* s, double* luh, const double* lduh, double dt);
double orc_stable_dt(const orc_solver* s, const double* luh, const double* dx);

/* PDE hooks */
void orc_flux(const orc_solver* s, const double* Q, double* F /* [dim][nV] */);
void orc_eigenvalues(const orc_solver* s, const double* Q, int d, double* lambda);
void orc_ncp(const orc_solver* s, const double* Q, const double* gradQ /* [dim][nV] */, double* BgradQ);
void orc_source(const orc_solver* s, const double* Q, double* S /* [nV] */);
void orc_ncp_nonlinear(const orc_solver* s, const double* Q, const double* gradQ /* [dim][nV] */,
                       double* BgradQ /* [nV] */);
void orc_coefficient_matrix(const orc_solver* s, const double* Q, int d, double* Bn /* [nV][nV] */);

/* Linear kernels (linear.c): spaceTimePredictorLinear (Cauchy-Kovalevski,
 * non-conservative product) + volumeIntegralLinear when lduh != 0; lQhi
 * [b^d][nD] and lFhi [d][b^d][nV] optional. */
void orc_lin_predictor(const orc_solver* s, const double* luh, const double* dx, double dt, double* lQhbnd,
                       double* lFhbnd, double* lduh, double* lQhi, double* lFhi);
/* the same with point sources (usePointSource = true): PSi [b+1][b^d][nV]
 * from orc_point_source (NULL: none) */
void orc_lin_predictor_ps(const orc_solver* s, const double* luh, const double* dx, double dt, const double* PSi,
                          double* lQhbnd, double* lFhbnd, double* lduh, double* lQhi, double* lFhi);
/* pointSource (2d/pointSource.cpph:30-127, 3d/pointSource.cpph:28-143): the
 * PDE's point source at every (time slot, node) of the cell with the given
 * centre and widths, projected onto the cell's basis; PSi [b+1][b^d][nV] */
void orc_point_source(const orc_solver* s, double t, double dt, const double* centre, const double* dx, double* PSi);
void orc_lin_volume_integral(const orc_solver* s, double* lduh, const double* lFhi, const double* dx);
void orc_lin_surface_integral(const orc_solver* s, double* lduh, const double* lFhbnd, const double* dx);
void orc_lin_riemann(const orc_solver* s, double* FL, double* FR, const double* QL, const double* QR, int dir);
/* boundary face of a linear solver: boundaryValues (kind 0 outflow, 1 rigid
 * wall) + riemannSolverLinear, the cell's own fluctuation into FIn */
void orc_lin_boundary_face(const orc_solver* s, double* FIn, const double* QIn, int faceIndex, int kind);

/* AMR transfer operators (amr.c) between a cell / face and its descendant
 * levelDelta levels finer; subcell / subface indices per axis in
 * 0 .. 3^levelDelta - 1; nvar values per node (parameters included), nflux
 * per flux node. Restrictions add to the coarse data. */
void orc_volume_prolongation(int dim, int N, int nvar, double* luhFine, const double* luhCoarse, int levelDelta,
                             const int* subcellIndex);
void orc_volume_restriction(int dim, int N, int nvar, double* luhCoarse, const double* luhFine, int levelDelta,
                            const int* subcellIndex);
void orc_face_prolongation(int dim, int N, int nvar, int nflux, double* lQhbndFine, double* lFhbndFine,
                           const double* lQhbndCoarse, const double* lFhbndCoarse, int levelDelta,
                           const int* subfaceIndex);
void orc_face_restriction(int dim, int N, int nvar, int nflux, double* lQhbndCoarse, double* lFhbndCoarse,
                          const double* lQhbndFine, const double* lFhbndFine, int levelDelta, const int* subfaceIndex);
/* one cell's values at the (N+1)^d equidistant points (plotters) */
void orc_equidistant_projection(int dim, int N, int nvar, const double* luh, double* out);

/* table access (generated dg_tables.h) */
const double* orc_table(const char* name, int order);

#ifdef __cplusplus
}
#endif
#endif
