/*
 * exahype_b200 -- C ABI of the B200 ADER-DG hot path.
 *
 * Two layers:
 *  1. Kernel entry points that replace, batched over many cells or faces, the
 *     calls the reference's generated solver glue makes into its generic
 *     kernels (Toolkit/src/eu/exahype/solvers/templates/
 *     AbstractGenericADERDGSolverImplementation.template:46-149, virtuals in
 *     ExaHyPE/exahype/solvers/ADERDGSolver.h:961-1085). Buffers are device
 *     pointers in the reference's per-cell layouts (kernels/KernelUtils.h),
 *     cells stored back to back; calls are ordered on `stream` and never
 *     allocate.
 *  2. A uniform-mesh solver (exa_mesh_*) that owns device-resident state and
 *     sequences the kernels the way the reference's non-fused time step does
 *     (exahype/runners/Runner.cpp:1116-1162).
 *
 * Layouts (N = order, b = N+1, d = dimension, nV = variables, nD = nV + parameters):
 *   luh    [cell][b^d][nD]            lduh   [cell][b^d][nV]
 *   lQhbnd [cell][2d][b^(d-1)][nD]    lFhbnd [cell][2d][b^(d-1)][nV]
 * Face index 0:-x 1:+x 2:-y 3:+y 4:-z 5:+z.
 *
 * Every function returns EXA_OK (0) or a negative EXA_ERR_* code; the text of
 * the last error of the calling thread is available from exa_last_error().
 */
#ifndef EXAHYPE_B200_H
#define EXAHYPE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EXA_OK 0
#define EXA_ERR_ARG (-1)         /* bad argument (null pointer, size, unsupported order/dimension) */
#define EXA_ERR_UNSUPPORTED (-2) /* this build has no kernels for the requested combination */
#define EXA_ERR_CUDA (-3)        /* a CUDA call failed; see exa_last_error() */
#define EXA_ERR_NOMEM (-4)       /* device allocation failed (mesh creation only) */
#define EXA_ERR_STATE (-5)       /* call out of order (e.g. step before init) */

/* PDE identifiers. */
#define EXA_PDE_EULER 0      /* compressible Euler, 5 variables (EulerADERDG demonstrator) */
#define EXA_PDE_EULER_TEST 1 /* the reference kernel tests' mock Euler with one parameter */
#define EXA_PDE_ELASTIC 2    /* linear elastic waves, 9 variables + 3 parameters (lambda, mu, rho); linear kernels */
/* EXA_PDE_EULER_TEST with useSource = useNCP = true: an algebraic source
 * (momentum damping, an energy source proportional to the density) and the
 * kernel tests' non-zero non-conservative product mock
 * (exahype/tests/kernels/c/GenericEulerKernelTest3D.cpp:84-110); orders 3
 * and 5. The predictor's source branch runs in the node-form kernel (the
 * line form has none), the Riemann and boundary kernels add the product's
 * fluctuations, the volume integral the time-averaged source. */
#define EXA_PDE_EULER_SOURCE_NCP 3
/* EXA_PDE_ELASTIC with a point source (usePointSource = true): a Ricker
 * wavelet on the three normal stresses at a fixed position, parameters set
 * by exa_solver_set_point_source; orders 3 and 5. Its predictor is
 * exa_space_time_predictor_linear_point_source; meshes evaluate the source
 * themselves. */
#define EXA_PDE_ELASTIC_POINT_SOURCE 4

/* Boundary kinds for exa_boundary_conditions / exa_mesh_create. */
#define EXA_BC_PERIODIC (-1)
#define EXA_BC_OUTFLOW 0
#define EXA_BC_REFLECTIVE 1

typedef struct exa_solver exa_solver;
typedef struct exa_mesh exa_mesh;

const char* exa_last_error(void);
const char* exa_version(void);

/* Kernel set for one (dimension, order, PDE): ADERDGSolver's constructor
 * arguments (exahype/solvers/ADERDGSolver.cpp:~430). */
int exa_solver_create(int dim, int order, int pde, exa_solver** out);
int exa_solver_destroy(exa_solver* s);
/* sizes in doubles: [0] unknowns per cell (b^d nV), [1] data per cell (b^d nD),
 * [2] data per face (b^(d-1) nD), [3] fluxes per face (b^(d-1) nV)
 * (ADERDGSolver::get{UnknownsPerCell,DataPerCell,BndFaceSize,BndFluxSize}). */
int exa_solver_sizes(const exa_solver* s, int* sizes4);

/* Predictor variants: how a cell's nodes and variables are spread over
 * threads and how many blocks per SM the register budget targets. The
 * autotuner (no counterpart in the reference, whose generic kernels have one
 * shape per order) times every variant on `ncells` synthetic cells of this
 * solver's order and keeps the fastest; variant_ms[EXA_PREDICTOR_VARIANTS]
 * (optional) receives the per-variant milliseconds. It allocates and frees
 * its own device buffers and synchronises the device. */
#define EXA_PREDICTOR_VARIANTS 9  /* size of variant_ms; 4 and 5 (mixed) are not timed (-1) */
/* Variant 8 keeps the Picard iterate of the line-form predictor in the SM's
 * tensor memory (solvers of order up to 5 with five state variables; other
 * shapes run variant 6 under this number). */
/* Variants beyond the autotuned ones (exa_solver_set_variant only): the
 * mixed-precision predictor. Its first Picard sweep is the FP64 sweep; every
 * later sweep forms the flux increment F(q^k) - F(q^(k-1)) in FP64 and runs
 * the stiffness contractions and the iK1 fold of that increment in FP32,
 * adding the FP32 update to the FP64 iterate (no counterpart in the
 * reference, whose predictor is FP64 throughout). Results differ from the
 * FP64 predictor at the level of FP32 rounding of the later updates. */
#define EXA_PREDICTOR_MIXED 4    /* mixed line form, 1 block per SM */
#define EXA_PREDICTOR_MIXED_2 5  /* mixed line form, 2 blocks per SM where they fit */
int exa_solver_autotune(exa_solver* s, int ncells, double* variant_ms, int* chosen);
int exa_solver_set_variant(exa_solver* s, int variant);
/* The point source of EXA_PDE_ELASTIC_POINT_SOURCE (the user's pointSource,
 * exahype/solvers/UserSolverInterface.h:75, of this library's point-source
 * PDE): force amplitude * (1 - 2 a) exp(-a), a = (pi f0 (t - t0))^2, on the
 * normal stresses, located at x0[dim]. Defaults: x0 = (0.5, 0.5, 0.5),
 * t0 = 0.1, f0 = 8, amplitude 1. EXA_ERR_UNSUPPORTED for other PDEs. */
int exa_solver_set_point_source(exa_solver* s, const double* x0, double t0, double f0, double amplitude);
int exa_solver_get_variant(const exa_solver* s, int* variant);

/* spaceTimePredictor (Kernels.h:85-95) + volumeIntegral (Kernels.h:104-106)
 * for ncells cells: reads luh, writes lQhbnd, lFhbnd and, when lduh is not
 * NULL, the volume integral lduh. dt_dev: device pointer to the predictor
 * step size. dx: host array of d cell widths. iterations_dev (optional):
 * per-cell Picard sweep counts. cell_list (optional, device): indices of the
 * cells to process (ncells entries); NULL processes cells 0..ncells-1. */
int exa_space_time_predictor_nonlinear(const exa_solver* s, const double* luh, double* lQhbnd, double* lFhbnd,
                                       double* lduh, const double* dt_dev, const double* dx, int ncells,
                                       const int* cell_list, int* iterations_dev, void* stream);
/* As above, also writing the reference's temporaries per cell (golden-vector
 * replay): lQi [b^d][b][nD], lFi [b][b^d][d+1][nV] (flux slots only; the
 * source slot is left untouched), lQhi [b^d][nD], lFhi [d+1][b^d][nV]. */
int exa_space_time_predictor_nonlinear_temps(const exa_solver* s, const double* luh, double* lQhbnd,
                                             double* lFhbnd, double* lduh, const double* dt_dev, const double* dx,
                                             int ncells, int* iterations_dev, double* lQi, double* lFi,
                                             double* lQhi, double* lFhi, void* stream);
/* riemannSolver (Kernels.h:136-142) for nfaces interior faces: face f joins
 * cell face_left[f] (its face 2*dir+1) and face_right[f] (its face 2*dir),
 * dir = face_dir[f]; the Rusanov flux is written to both cells' lFhbnd slots
 * (ADERDGSolver::solveRiemannProblemAtInterface, ADERDGSolver.cpp:2789-2866). */
int exa_riemann_solver_nonlinear(const exa_solver* s, const double* lQhbnd, double* lFhbnd, const int* face_left,
                                 const int* face_right, const int* face_dir, int nfaces, void* stream);
/* Linear kernels, for solvers of a linear PDE (EXA_PDE_ELASTIC[_POINT_SOURCE]; the reference's
 * generated glue calls them when the solver is linear,
 * AbstractGenericADERDGSolverImplementation.template:53-54,85-86,101-149).
 * The nonlinear entry points above reject a linear solver and vice versa;
 * exa_corrector applies the linear surface integral for a linear solver.
 *
 * spaceTimePredictorLinear (Kernels.h, c/{2d,3d}/spaceTimePredictorLinear.cpph;
 * Cauchy-Kovalevski with the PDE's non-conservative product) and, when lduh
 * is not NULL, volumeIntegralLinear; arguments as for the nonlinear
 * predictor. */
int exa_space_time_predictor_linear(const exa_solver* s, const double* luh, double* lQhbnd, double* lFhbnd,
                                    double* lduh, const double* dt_dev, const double* dx, int ncells,
                                    const int* cell_list, void* stream);
/* As above, also writing the time averages per cell (golden-vector replay):
 * lQhi [b^d][nD] and lFhi [d][b^d][nV] (the reference's tempUnknowns and
 * tempFluxUnknowns). */
int exa_space_time_predictor_linear_temps(const exa_solver* s, const double* luh, double* lQhbnd, double* lFhbnd,
                                          double* lduh, const double* dt_dev, const double* dx, int ncells,
                                          double* lQhi, double* lFhi, void* stream);
/* The linear predictor of a point-source PDE (spaceTimePredictorLinear
 * <usePointSource = true>, after the glue's pointSource(t, dt, centre, dx,
 * forces) of each cell, ADERDGSolver.cpp:1929-1960 and
 * c/{2d,3d}/pointSource.cpph): *t_dev is the time stamp of the solution the
 * predictor starts from, centres[3 * cell + d] (device) the cells' centres;
 * a cell whose closed box does not hold the source is predicted without it.
 * lQhi / lFhi: optional time averages as for _temps (both or neither). The
 * two entry points above reject a point-source PDE. */
int exa_space_time_predictor_linear_point_source(const exa_solver* s, const double* luh, double* lQhbnd,
                                                 double* lFhbnd, double* lduh, const double* t_dev,
                                                 const double* dt_dev, const double* dx, const double* centres,
                                                 int ncells, const int* cell_list, double* lQhi, double* lFhi,
                                                 void* stream);
/* riemannSolverLinear (c/{2d,3d}/riemannSolverLinear.cpph) for nfaces
 * interior faces, face arrays as for exa_riemann_solver_nonlinear: the
 * fluctuations (Bn -/+ smax I)^T (QR - QL)/2 are written to the left / right
 * cell's lFhbnd slot (the extrapolated fluxes there are not read). */
int exa_riemann_solver_linear(const exa_solver* s, const double* lQhbnd, double* lFhbnd, const int* face_left,
                              const int* face_right, const int* face_dir, int nfaces, void* stream);
/* volumeIntegralLinear (c/{2d,3d}/volumeIntegralLinear.cpph) on its own:
 * lduh = -w sum_d lFhi[d], lFhi per cell [d][b^d][nV]. */
int exa_volume_integral_linear(const exa_solver* s, double* lduh, const double* lFhi, int ncells, void* stream);
/* AMR transfer operators (kernels/aderdg/generic/c/{2d,3d}/amrRoutines.cpph,
 * Kernels.h:159-201), batched: transfer k moves data between fine cell (or
 * face slot) fine[k] and its ancestor coarse[k], level_delta[k] levels
 * coarser (1..12); the subcell index holds one base-3 digit per level per axis
 * (0 .. 3^level_delta - 1), 3 ints per transfer for cells, 2 for faces (2D:
 * the first is used). Face slots index lQhbnd/lFhbnd as cell * 2d + face.
 * Prolongations overwrite the fine data; restrictions ADD the restricted
 * data to the coarse data (atomically, so descendants of one ancestor may
 * share a call; their sum order is not fixed). Transfers with an invalid
 * level_delta or index are skipped. All arrays are device arrays. */
int exa_volume_unknowns_prolongation(const exa_solver* s, double* luh_fine, const double* luh_coarse, int n,
                                     const int* fine_cell, const int* coarse_cell, const int* level_delta,
                                     const int* subcell_index, void* stream);
int exa_volume_unknowns_restriction(const exa_solver* s, double* luh_coarse, const double* luh_fine, int n,
                                    const int* fine_cell, const int* coarse_cell, const int* level_delta,
                                    const int* subcell_index, void* stream);
int exa_face_unknowns_prolongation(const exa_solver* s, double* lQhbnd_fine, double* lFhbnd_fine,
                                   const double* lQhbnd_coarse, const double* lFhbnd_coarse, int n,
                                   const int* fine_slot, const int* coarse_slot, const int* level_delta,
                                   const int* subface_index, void* stream);
int exa_face_unknowns_restriction(const exa_solver* s, double* lQhbnd_coarse, double* lFhbnd_coarse,
                                  const double* lQhbnd_fine, const double* lFhbnd_fine, int n, const int* fine_slot,
                                  const int* coarse_slot, const int* level_delta, const int* subface_index,
                                  void* stream);
/* The solution of ncells cells at their (N+1)^d equidistant vertices
 * (x fastest), vertices [cell][b^d][nD]: what the plotter
 * ADERDG2CartesianVTK::plotVertexData evaluates with
 * equidistantGridProjector1d (exahype/plotters/VTK/ADERDG2CartesianVTK.cpp). */
int exa_plot_vertices(const exa_solver* s, const double* luh, double* vertices, int ncells, void* stream);
/* boundaryConditions + riemannSolver on boundary faces (ADERDGSolver::
 * applyBoundaryConditions, ADERDGSolver.cpp:2893-2962): face f is face
 * bface[f] of cell bcell[f]; kind is EXA_BC_OUTFLOW or EXA_BC_REFLECTIVE. */
int exa_boundary_conditions(const exa_solver* s, const double* lQhbnd, double* lFhbnd, const int* bcell,
                            const int* bface, int nb, int kind, void* stream);
/* surfaceIntegral (Kernels.h:110-112) + solutionUpdate (Kernels.h:97-98) +
 * stableTimeStepSize (Kernels.h:155-157) for ncells cells, fused: luh is
 * advanced by *dt_dev and the minimum admissible step over the cells is
 * min-combined into *dt_min_dev (initialise it with exa_reset_min). With
 * update == 0 only the time step of the current luh is computed. */
int exa_corrector(const exa_solver* s, double* luh, const double* lduh, const double* lFhbnd, const double* dt_dev,
                  double* dt_min_dev, const double* dx, int ncells, const int* cell_list, int update, void* stream);
/* *dev = DBL_MAX, ordered on stream. */
int exa_reset_min(double* dev, void* stream);

/* ---- uniform-mesh solver ------------------------------------------------ */
/* cells[d]: cells per axis; offset/size[d]: domain; bc[2d]: per domain face
 * EXA_BC_PERIODIC / EXA_BC_OUTFLOW / EXA_BC_REFLECTIVE (periodic must be set
 * on both faces of an axis). Allocates all device state. */
int exa_mesh_create(const exa_solver* s, const int* cells, const double* offset, const double* size, const int* bc,
                    exa_mesh** out);
/* A statically refined periodic mesh: the coarse grid of exa_mesh_create with
 * the box of coarse cells box_lo[d] <= c[d] < box_hi[d] refined once (3^d
 * fine cells each; at least one coarse cell must surround the box). Global
 * time stepping; the same exa_mesh_* calls step and write it (not
 * exa_mesh_init_fused). Solution order: the unrefined coarse cells
 * (x fastest over the coarse grid, refined ones skipped), then the fine cells
 * (x fastest over the box's fine grid). Replaces the spacetree's hanging-face
 * handling for this layout: after every predictor the refined cells that
 * face coarse cells (ancestors) receive the restriction of their fine
 * children's face data (ADERDGSolver::restrictToTopMostParent,
 * exahype/solvers/ADERDGSolver.cpp:2465-2515) and the virtual fine cells
 * across the box's faces (descendants) the prolongation of their coarse
 * parent's (prolongateFaceDataToDescendant, :2334-2382); Riemann problems
 * pair coarse cells with ancestors and fine cells with descendants
 * (solveRiemannProblemAtInterface, :2789). */
int exa_mesh_create_refined(const exa_solver* s, const int* cells, const double* offset, const double* size,
                            const int* box_lo, const int* box_hi, exa_mesh** out);
/* The same with nboxes nested refined boxes (1..8) and optional domain
 * boundaries bc[2d] (NULL: periodic; EXA_BC_PERIODIC on both faces of an
 * axis, or EXA_BC_OUTFLOW / EXA_BC_REFLECTIVE per face, those for nonlinear
 * PDEs only): box k (box_lo/box_hi
 * [3k .. 3k+2]) is given in the cell coordinates of level k (level 0 the
 * coarse grid, level k+1 the box k refined once, whose coordinates run over
 * the whole domain at that level: 3^(k+1) cells[d]) and must lie inside
 * level k's region with at least one level-k cell around it. Solution order:
 * the unrefined cells of level 0, then of level 1, ..., each x fastest over
 * its region. exa_mesh_create_refined is the case nboxes = 1. */
int exa_mesh_create_nested(const exa_solver* s, const int* cells, const double* offset, const double* size,
                           const int* bc, int nboxes, const int* box_lo, const int* box_hi, exa_mesh** out);
/* The general form: box k refines the positions box_lo <= p < box_hi
 * ([3k .. 3k+2]) of level box_level[k] (0..7; level-l coordinates span the
 * whole domain, 3^l cells[d] per axis). Several boxes may refine one level
 * (overlapping or touching boxes refine their union); the region of level
 * l >= 1 is the union of the level-(l-1) boxes refined once, and every box
 * must lie inside its level's region with one cell of margin. Solution
 * order: level by level, the cells of each level x fastest over the
 * level's bounding rectangle. exa_mesh_create_nested is the case
 * box_level[k] = k. */
int exa_mesh_create_boxes(const exa_solver* s, const int* cells, const double* offset, const double* size,
                          const int* bc, int nboxes, const int* box_level, const int* box_lo, const int* box_hi,
                          exa_mesh** out);
/* Static AMR between steps: replaces the refinement of a mesh made by
 * exa_mesh_create_boxes (nboxes may be 0: the coarse grid alone) by the
 * given boxes. A cell of the new mesh that was a cell keeps its data, one
 * inside a coarser old cell gets that cell's prolongation, one covering
 * finer old cells the sum of their restrictions (prolongateVolumeData /
 * restrictVolumeData, exahype/solvers/ADERDGSolver.cpp:1437-1470,1694-1735).
 * The time stamp and step count are kept; the admissible step is recomputed
 * from the new solution and the predictor runs on every cell. The handle
 * stays valid; the mesh's stream (exa_mesh_stream) and cell count change.
 * Not for meshes in fused time stepping. Synchronises the old stream. */
int exa_mesh_regrid(exa_mesh* m, int nboxes, const int* box_level, const int* box_lo, const int* box_hi);
int exa_mesh_destroy(exa_mesh* m);
int exa_mesh_num_cells(const exa_mesh* m, int* ncells);
/* host <-> device solution, luh layout above, cells in x-fastest order */
int exa_mesh_set_solution(exa_mesh* m, const double* luh_host);
int exa_mesh_get_solution(exa_mesh* m, double* luh_host);
/* Asynchronous solution copy ordered on the mesh stream: to_device != 0 copies
 * host -> device, else device -> host. nbytes must equal the solution size;
 * use page-locked host memory for overlap. */
int exa_mesh_copy_solution(exa_mesh* m, void* host, size_t nbytes, int to_device);
/* Sets t = t0, computes the first admissible step from the current solution
 * and runs the first predictor (Runner::runAsMaster, Runner.cpp:681-700). */
int exa_mesh_init(exa_mesh* m, double t0);
/* Fused time stepping (the reference's fuse-algorithmic-steps option,
 * exahype/runners/Runner.cpp:1053-1114, with global time steps): instead of
 * exa_mesh_init. Every later step runs the predictor right after the update
 * with an estimated step size, so no global reduction separates the two;
 * when the stable step of the updated solution turns out smaller than the
 * estimate, the estimate is replaced by weight * stable and the predictor is
 * rerun (TimeStepSizeComputation.cpp:167-204, ADERDGSolver.cpp:559-613);
 * weight in (0, 1] is the reference's fuse-algorithmic-steps-factor.
 * exa_mesh_state then reports the corrector time stamp and step size. */
int exa_mesh_init_fused(exa_mesh* m, double t0, double weight);
/* fused time stepping: the predictor step size estimate and the number of
 * predictor reruns so far */
int exa_mesh_fused_state(exa_mesh* m, double* predictor_dt, long long* reruns);
/* nsteps time steps with host input and output streamed around them: step
 * k first takes its solution from host_in + (k % nin) * nbytes, then steps,
 * then leaves its result at host_out + (k % nout) * nbytes. The copies run on
 * two streams of their own through device staging buffers, so the upload of
 * step k+1 and the download of step k-1 overlap the compute of step k (use
 * pinned host memory). Returns after enqueuing; the mesh stream completes
 * after the last download (exa_mesh_synchronize). No counterpart in the
 * reference: host<->device streaming for servers and end-to-end runs. */
int exa_mesh_step_io(exa_mesh* m, const void* host_in, int nin, void* host_out, int nout, size_t nbytes,
                     int nsteps);
/* nsteps non-fused time steps (Riemann, corrector + dt, predictor) without
 * host synchronisation. */
int exa_mesh_step(exa_mesh* m, int nsteps);
/* Steps while t < t_end and dt > 0 (Runner.cpp:708-709; no clamp of the last
 * step), at most max_steps; returns the steps taken in *steps. */
int exa_mesh_run_until(exa_mesh* m, double t_end, int max_steps, int* steps);
/* current time, current (predictor) step size, steps taken, and the total
 * number of Picard sweeps executed by the predictor so far */
int exa_mesh_state(exa_mesh* m, double* t, double* dt, long long* steps, long long* picard_sweeps);
int exa_mesh_synchronize(exa_mesh* m);
/* validateNoNansInADERDGSolver (exahype/solvers/ADERDGSolver.cpp:1778-1829)
 * as a status instead of assertions: *nonfinite_cells = the number of cells
 * with a non-finite value in their solution, update, or extrapolated state
 * or flux face data. Synchronises the mesh's stream. */
int exa_mesh_validate(exa_mesh* m, long long* nonfinite_cells);
/* Writes the mesh's current solution as a legacy VTK unstructured grid (text,
 * or binary when binary != 0): every cell a patch of (N+1)^d vertices with
 * N^d pixels / voxels, vertex data "Q" (all nD values, from
 * exa_plot_vertices) and "time" -- the layout of the reference's
 * ADERDG2CartesianVTK vertex plotter. Synchronises the mesh's stream. */
int exa_mesh_write_vtk(exa_mesh* m, const char* path, int binary);
/* The same layout with the points at every cell's Gauss-Legendre nodes and
 * the nodal values as they are (no projection) -- the reference's
 * ADERDG2LegendreVTK vertex plotter
 * (exahype/plotters/VTK/ADERDG2LegendreVTK.cpp:280-380). */
int exa_mesh_write_vtk_legendre(exa_mesh* m, const char* path, int binary);
/* Moves the mesh's work to a new stream of stream priority `level` (0: the
 * default, least urgent; each level up is more urgent, capped at the device's
 * range): where several streams' kernels wait for SMs, the higher priority's
 * go first. Synchronises the mesh's stream; call it between steps. */
int exa_mesh_set_priority(exa_mesh* m, int level);
/* the CUDA stream (cudaStream_t) all of the mesh's work is ordered on */
int exa_mesh_stream(exa_mesh* m, void** stream);
/* Per-phase device timing with CUDA events recorded on the mesh stream around
 * every phase of every step (0 disables). exa_mesh_phase_times returns the
 * accumulated milliseconds and launch counts of phases
 * 0 predictor+volume, 1 Riemann (interior + boundary), 2 corrector+dt,
 * 3 bookkeeping, since the last reset (synchronises the stream). */
int exa_mesh_set_profiling(exa_mesh* m, int on);
int exa_mesh_phase_times(exa_mesh* m, double* ms4, long long* launches4, int reset);

/* ---- limiter kernels (batched, stream-ordered, EXA_PDE_EULER) ------------- */
/* FV patches: lim[cell][(2N+5)^d][5] (2N+1 subcells plus 2 ghost layers per
 * side, (z,y,x) order). cell_list (optional, device): the cells to process. */
/* projectOnFVLimiterSpace (kernels/limiter/generic/Limiter.h:48,
 * Limiter.cpp:23-66): interior subcells of lim from luh. */
int exa_project_on_fv_limiter_space(const exa_solver* s, const double* luh, double* lim, int ncells,
                                    const int* cell_list, void* stream);
/* projectOnDGSpace (Limiter.h:58, Limiter.cpp:69-112): luh from the interior
 * subcells of lim. */
int exa_project_on_dg_space(const exa_solver* s, const double* lim, double* luh, int ncells, const int* cell_list,
                            void* stream);
/* FiniteVolumesSolver::updateSolution's kernel call (FiniteVolumesSolver.cpp:662-715;
 * musclhancock::c::solutionUpdate, musclhancock.h:38-41, generated glue
 * AbstractGenericFiniteVolumesSolverInCImplementation.template:48-51): for every
 * listed cell lim_old <- lim (ghost layers included; the caller has filled
 * them), then lim <- the MUSCL-Hancock update of lim_old by *dt_dev, and, when
 * luh is not NULL, luh <- projectOnDGSpace(lim). 3D patches need device
 * scratch of at least exa_fv_musclhancock_scratch_bytes(s, ncells) bytes (less
 * runs with fewer blocks; less than one block's share is an error); 2D needs
 * none (scratch may be NULL). */
int exa_fv_musclhancock_scratch_bytes(const exa_solver* s, int ncells, size_t* bytes);
int exa_fv_musclhancock_update(const exa_solver* s, double* lim, double* lim_old, double* luh, const double* dt_dev,
                               const double* dx, int ncells, const int* cell_list, void* scratch, size_t scratch_bytes,
                               void* stream);
/* The same update without any device allocation and without caller scratch
 * (no counterpart in the reference, whose kernels take their scratch from the
 * caller's per-thread temporaries, TemporaryVariables.cpp:68-111). For callers
 * that cannot hand out device memory: code inside a framework traversal that
 * owns no device allocator, or a host thread that must not call cudaMalloc or
 * cudaFree because they can synchronise the device. The scratch is a 32 MiB
 * array inside the library; a call runs as many blocks as fit in it (3D N=3:
 * 151, N=5: 47, N=7: 20; 2D needs none), and an order whose one-block share
 * exceeds it is rejected with EXA_ERR_UNSUPPORTED. Nothing in it has to start
 * at zero. All calls share the array: calls that overlap in time (on
 * different streams or threads) race on it and must be serialised. The first
 * call on a device (and the first after a reset of that device) looks the
 * array up and sets kernel attributes; make it before any stream capture
 * begins. */
int exa_fv_musclhancock_update_noalloc(const exa_solver* s, double* lim, double* lim_old, double* luh,
                                       const double* dt_dev, const double* dx, int ncells, const int* cell_list,
                                       void* stream);

/* ---- uniform mesh with the a-posteriori subcell limiter ------------------- */
/* The LimitingADERDGSolver (exahype/solvers/LimitingADERDGSolver.h:82-1508)
 * over the uniform mesh: every cell carries a limiter status, DMP min/max
 * blocks per face and, while its status is > 0, an FV patch of (2N+1)^d
 * subcells with 2 ghost layers (MUSCL-Hancock, minmod, Rusanov;
 * GenericFiniteVolumesMUSCLHancockInC). Euler PDE only (EXA_PDE_EULER);
 * boundary faces periodic, outflow or reflective (the EulerADERDG
 * demonstrator's walls: normal momentum negated in the DG boundaryValues,
 * MyEulerSolver_ADERDG.cpp:63-87, and in the FV solver's, MyEulerSolver_FV.cpp:47-62).
 *   helper_layers h: activeFV status A = h+1, troubled status T = 2h+1
 *     (LimitingADERDGSolver.h:452-458 and the generated solver's constructor);
 *   cure_steps: iterationsToCureTroubledCell (:452-458), the specification
 *     file's steps-till-cured (EulerADERDG.exahype:62 uses 10);
 *   relax / scale: DMPRelaxationParameter (delta0) and DMPDifferenceScaling
 *     (epsilon) of the discrete maximum principle, 1e-4 / 1e-3 by default.
 * The step follows the reference's non-fused limiting sequence
 * (mergeNeighboursBasedOnLimiterStatus :1146, updateSolution :873,
 * determineLimiterStatusAfterSolutionUpdate :304, then on an irregular limiter
 * domain change limiter status spreading, reinitialiseSolversLocally :1006 and
 * recomputeSolutionLocally :1029, and the prediction of every cell with
 * status < T) without host synchronisation. */
typedef struct exa_lmesh exa_lmesh;
int exa_lmesh_create(const exa_solver* s, const int* cells, const double* offset, const double* size, const int* bc,
                     int helper_layers, int cure_steps, double relax, double scale, exa_lmesh** out);
int exa_lmesh_destroy(exa_lmesh* m);
/* host <-> device DG solution (layout and cell order of exa_mesh) */
int exa_lmesh_set_solution(exa_lmesh* m, const double* luh_host);
int exa_lmesh_get_solution(exa_lmesh* m, double* luh_host);
/* exa_mesh_write_vtk's layout for a limiting mesh (the DG solution, which
 * the limiter keeps current in limited cells too) plus the vertex data
 * "Limiter-Status" (each vertex its cell's status) -- the reference's
 * LimitingADERDG2CartesianVTK vertex plotter
 * (exahype/plotters/VTK/LimitingADERDG2CartesianVTK.cpp:251-300). */
int exa_lmesh_write_vtk(exa_lmesh* lm, const char* path, int binary);
/* Optional FV initial condition at the subcell centres, [cell][(2N+1)^d][5]
 * (the FV solver's adjustSolution at t = 0); limiter patches allocated at
 * initialisation start from it instead of from the DG projection. */
int exa_lmesh_set_fv_initial(exa_lmesh* m, const double* fv_host);
/* Initial limiter status from the physical admissibility of the initial data,
 * status spreading, first admissible step and first predictor
 * (LimitingADERDGSolver::setInitialConditions :849, Runner.cpp:681-700). */
int exa_lmesh_init(exa_lmesh* m, double t0);
int exa_lmesh_step(exa_lmesh* m, int nsteps);
int exa_lmesh_run_until(exa_lmesh* m, double t_end, int max_steps, int* steps);
/* time, current step size, steps, Picard sweeps, steps with an irregular
 * limiter domain change (local recomputation) */
int exa_lmesh_state(exa_lmesh* m, double* t, double* dt, long long* steps, long long* picard_sweeps,
                    long long* irregular_steps);
/* limiter status per cell (0 DG, 1..h helper, A..T-1 FV-active, T troubled) */
int exa_lmesh_get_status(exa_lmesh* m, int* status_host);
/* FV patches [cell][E^d][5], E = 2N+5 (ghost layers included; cells whose
 * patch is not allocated hold stale values) and per-cell allocation flags */
int exa_lmesh_get_limiter(exa_lmesh* m, double* lim_host, int* allocated_host);
int exa_lmesh_synchronize(exa_lmesh* m);
int exa_lmesh_set_priority(exa_lmesh* m, int level);  /* as exa_mesh_set_priority */
int exa_lmesh_stream(exa_lmesh* m, void** stream);

/* ---- batched ragged ensemble (no counterpart in the reference) ------------ */
/* Many independent uniform-mesh solves (any mix of dimension, order, size and
 * boundary kinds, each with its own global time step as one exa_mesh would
 * have) advanced together: instances of one (dim, order, pde) share device
 * arrays, so each phase of a step is one launch per order, and the whole step
 * is replayed as one CUDA graph. Every instance computes exactly what an
 * exa_mesh of the same problem computes (same predictor variant), whatever
 * else is in the batch.
 * exa_batch_add copies the initial solution (exa_mesh layout) and returns an
 * instance id; adds and removes take effect at the next exa_batch_commit or
 * exa_batch_step (new instances get exa_mesh_init's first step size and
 * predictor, t = 0). The first instance of an order runs the predictor
 * autotuner for that order unless exa_batch_set_variant set its variant
 * before. The batch's stream has the highest stream
 * priority, so its kernels go ahead of other streams' when both wait for SMs. */
typedef struct exa_batch exa_batch;
int exa_batch_create(exa_batch** out);
int exa_batch_destroy(exa_batch* b);
int exa_batch_add(exa_batch* b, int dim, int order, int pde, const int* cells, const double* size, const int* bc,
                  const double* luh_host, int* id);
int exa_batch_remove(exa_batch* b, int id);
int exa_batch_commit(exa_batch* b);
/* nsteps steps of every live instance (one graph launch per step unless
 * exa_batch_set_graph(b, 0)); no host synchronisation */
int exa_batch_step(exa_batch* b, int nsteps);
int exa_batch_set_graph(exa_batch* b, int on);
int exa_batch_set_variant(exa_batch* b, int dim, int order, int pde, int variant);
int exa_batch_get_variant(const exa_batch* b, int dim, int order, int pde, int* variant);
int exa_batch_state(exa_batch* b, int id, double* t, double* dt, long long* steps);
int exa_batch_get_solution(exa_batch* b, int id, double* luh_host);
/* device bytes an instance of that shape adds, and the batch's current total
 * (for admission by memory budget) */
int exa_batch_instance_bytes(int dim, int order, int pde, const int* cells, size_t* bytes);
int exa_batch_device_bytes(const exa_batch* b, size_t* bytes);
int exa_batch_sweeps(exa_batch* b, long long* picard_sweeps);
int exa_batch_synchronize(exa_batch* b);
int exa_batch_stream(exa_batch* b, void** stream);

/* Measurement helper (no counterpart in the reference): sustained FP64 FMA
 * throughput of the current GPU in TFLOP/s, from independent DFMA chains on
 * every SM timed with CUDA events -- the FP64 roofline of the predictor. */
int exa_fp64_peak_probe(double* tflops);
/* Measurement helper (no counterpart in the reference): FP64 tensor-core
 * throughput in TFLOP/s, from independent mma.sync m8n8k4 f64 accumulator
 * chains on every SM. On B200 it equals the DFMA figure: the two share one
 * FP64 pipe, so tensor-core tiles cannot raise the predictor's FP64 ceiling. */
int exa_fp64_mma_peak_probe(double* tflops);

#ifdef __cplusplus
}
#endif
#endif
