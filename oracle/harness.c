/*
 * ORACLE harness -- test infrastructure only. A uniform Cartesian mesh driven
 * by the reference's non-fused, globally time-stepped ADER-DG step
 * (exahype/runners/Runner.cpp:681-709, 1116-1162):
 *   init:   dt = min over cells of stableTimeStepSize(u0); predictor(u0, dt)
 *   step:   1. riemannSolver on every interior face, boundaryConditions +
 *              riemannSolver on every boundary face   (mappings/Merging.cpp)
 *           2. per cell: surfaceIntegral, solutionUpdate(dt), new admissible
 *              step from the updated solution           (mappings/SolutionUpdate.cpp)
 *           3. t += dt; dt = min over cells              (ADERDGSolver.cpp:560-592)
 *           4. per cell: predictor + volume integral with the new dt
 *                                                        (mappings/Prediction.cpp)
 *   loop:   while t < t_end && dt > 0 (no clamp of the last step).
 *
 * Fused time stepping (the reference's fuse-algorithmic-steps option,
 * global time stepping, one rank), hrn_init_fused / hrn_step_fused:
 *   init:   s0 = min stable step of u0; corrector and predictor step s0,
 *           predictor stamp t0 + s0 (TimeStepSizeComputation::endIteration ->
 *           ADERDGSolver::updateTimeStepSizesFused, ADERDGSolver.cpp:594-613);
 *           predictor(u0, s0)
 *   step:   Riemann / boundary; per cell corrector with the corrector step,
 *           then at once the predictor with the predictor step (fusedTimeStep,
 *           ADERDGSolver.cpp:1853-1878); s = min stable step of the updated
 *           solution; used = predictor step (s if 0); if used > s the
 *           predictor step becomes w s and the next estimate w s, else the next
 *           estimate is min(s, (used + w s) / 2)
 *           (TimeStepSizeComputation.cpp:167-204); startNewTimeStep
 *           (ADERDGSolver.cpp:559-592): corrector stamp = predictor stamp,
 *           corrector step = predictor step, predictor stamp += predictor
 *           step, predictor step = next estimate; if the step was too large
 *           the predictor is rerun with the new predictor step
 *           (Runner.cpp:1103-1109, mappings/Prediction.cpp)
 *   loop:   while corrector stamp < t_end && corrector step > 0
 *           (Solver::getMinSolverTimeStampOfAllSolvers: the corrector stamp).
 * The per-cell / per-face kernels come from a backend table, so the same
 * sequencing drives both the C restatement and the reference kernels.
 * Cells run in parallel on `nthreads` POSIX threads.
 *
 * This file is #included by the translation unit that defines the backend.
 */
#include <float.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  void* ctx;
  int dim, order, nvar, ndata;
  int (*predictor)(void* ctx, const double* luh, const double* dx, double dt, double* lQhbnd, double* lFhbnd,
                   double* lduh);
  void (*riemann)(void* ctx, double* FL, double* FR, const double* QL, const double* QR, int dir);
  void (*boundary_face)(void* ctx, double* FIn, const double* QIn, int faceIndex);
  void (*surface_integral)(void* ctx, double* lduh, const double* lFhbnd, const double* dx);
  void (*solution_update)(void* ctx, double* luh, const double* lduh, double dt);
  double (*stable_dt)(void* ctx, const double* luh, const double* dx);
  /* optional: a boundary face that needs the boundary kind of its domain
   * face (0 outflow, 1 reflective); used instead of boundary_face when set */
  void (*boundary_face_kind)(void* ctx, double* FIn, const double* QIn, int faceIndex, int kind);
  /* optional: a predictor that needs the cell's centre and the time stamp of
   * the solution it starts from (point sources); used instead of predictor
   * when set */
  int (*predictor_at)(void* ctx, const double* luh, const double* dx, const double* centre, double t, double dt,
                      double* lQhbnd, double* lFhbnd, double* lduh);
} hrn_backend;

typedef struct {
  hrn_backend k;
  int dim, cells[3], ncells, P, F, nthreads;
  double dx[3];
  int bc[6]; /* -1 periodic, 0 outflow, 1 reflective */
  double *luh, *lduh, *lQhbnd, *lFhbnd;
  int *fl, *fr, *fd, nfaces, *bcell, *bface, nb;
  int* iters;
  double t, dt;     /* corrector time stamp and step size */
  double pdt;       /* step size of the next predictor call */
  double pt;        /* time stamp of the solution the next predictor call starts from */
  long steps, sweeps;
  /* fused time stepping */
  int fused;
  double w, tp, next;  /* rerun weight, predictor time stamp, next-step estimate */
  long reruns;
} hrn_mesh;

static int hrn_cid(const hrn_mesh* m, int i, int j, int k) { return (k * m->cells[1] + j) * m->cells[0] + i; }

static hrn_mesh* hrn_create(const hrn_backend* k, const int* cells, const double* size, const int* bc, int nthreads) {
  hrn_mesh* m = (hrn_mesh*)calloc(1, sizeof(hrn_mesh));
  m->k = *k;
  m->dim = k->dim;
  m->nthreads = nthreads < 1 ? 1 : nthreads;
  int b = k->order + 1;
  m->P = m->dim == 3 ? b * b * b : b * b;
  m->F = m->dim == 3 ? b * b : b;
  m->ncells = 1;
  for (int d = 0; d < 3; d++) {
    m->cells[d] = d < m->dim ? cells[d] : 1;
    m->dx[d] = d < m->dim ? size[d] / cells[d] : 1.0;
    m->ncells *= m->cells[d];
  }
  for (int f = 0; f < 2 * m->dim; f++) m->bc[f] = bc[f];
  const size_t n = m->ncells;
  m->luh = (double*)calloc(n * m->P * k->ndata, sizeof(double));
  m->lduh = (double*)calloc(n * m->P * k->nvar, sizeof(double));
  m->lQhbnd = (double*)calloc(n * 2 * m->dim * m->F * k->ndata, sizeof(double));
  m->lFhbnd = (double*)calloc(n * 2 * m->dim * m->F * k->nvar, sizeof(double));
  m->iters = (int*)calloc(n, sizeof(int));
  /* face lists in the order the GPU mesh builds them */
  m->fl = (int*)malloc(sizeof(int) * n * 3);
  m->fr = (int*)malloc(sizeof(int) * n * 3);
  m->fd = (int*)malloc(sizeof(int) * n * 3);
  m->bcell = (int*)malloc(sizeof(int) * n * 6);
  m->bface = (int*)malloc(sizeof(int) * n * 6);
  for (int kk = 0; kk < m->cells[2]; kk++)
    for (int j = 0; j < m->cells[1]; j++)
      for (int i = 0; i < m->cells[0]; i++) {
        const int c = hrn_cid(m, i, j, kk);
        int ijk[3] = {i, j, kk};
        for (int d = 0; d < m->dim; d++) {
          int nb[3] = {i, j, kk};
          nb[d] = ijk[d] + 1;
          if (nb[d] < m->cells[d] || m->bc[2 * d + 1] == -1) {
            if (nb[d] >= m->cells[d]) nb[d] = 0;
            m->fl[m->nfaces] = c;
            m->fr[m->nfaces] = hrn_cid(m, nb[0], nb[1], nb[2]);
            m->fd[m->nfaces] = d;
            m->nfaces++;
          } else {
            m->bcell[m->nb] = c;
            m->bface[m->nb] = 2 * d + 1;
            m->nb++;
          }
          if (ijk[d] == 0 && m->bc[2 * d] != -1) {
            m->bcell[m->nb] = c;
            m->bface[m->nb] = 2 * d;
            m->nb++;
          }
        }
      }
  return m;
}

static void hrn_destroy(hrn_mesh* m) {
  if (!m) return;
  free(m->luh); free(m->lduh); free(m->lQhbnd); free(m->lFhbnd); free(m->iters);
  free(m->fl); free(m->fr); free(m->fd); free(m->bcell); free(m->bface);
  free(m);
}

/* ---- parallel loops over cells / faces ---- */
typedef struct {
  hrn_mesh* m;
  int phase, lo, hi;
  double dtmin;
} hrn_job;

static void hrn_run_range(hrn_job* j) {
  hrn_mesh* m = j->m;
  const hrn_backend* k = &m->k;
  const int P = m->P, F = m->F, nV = k->nvar, nD = k->ndata, D2 = 2 * m->dim;
  j->dtmin = DBL_MAX;
  for (int i = j->lo; i < j->hi; i++) {
    if (j->phase == 0 && k->predictor_at) { /* predictor + volume integral at the cell's centre */
      const int ijk[3] = {i % m->cells[0], (i / m->cells[0]) % m->cells[1], i / (m->cells[0] * m->cells[1])};
      double centre[3];
      for (int d = 0; d < 3; d++) centre[d] = ijk[d] * m->dx[d] + 0.5 * m->dx[d];
      m->iters[i] = k->predictor_at(k->ctx, m->luh + (size_t)i * P * nD, m->dx, centre, m->pt, m->pdt,
                                    m->lQhbnd + (size_t)i * D2 * F * nD, m->lFhbnd + (size_t)i * D2 * F * nV,
                                    m->lduh + (size_t)i * P * nV);
    } else if (j->phase == 0) { /* predictor + volume integral */
      m->iters[i] = k->predictor(k->ctx, m->luh + (size_t)i * P * nD, m->dx, m->pdt, m->lQhbnd + (size_t)i * D2 * F * nD,
                                 m->lFhbnd + (size_t)i * D2 * F * nV, m->lduh + (size_t)i * P * nV);
    } else if (j->phase == 1) { /* interior face */
      const int cl = m->fl[i], cr = m->fr[i], d = m->fd[i];
      k->riemann(k->ctx, m->lFhbnd + ((size_t)cl * D2 + 2 * d + 1) * F * nV, m->lFhbnd + ((size_t)cr * D2 + 2 * d) * F * nV,
                 m->lQhbnd + ((size_t)cl * D2 + 2 * d + 1) * F * nD, m->lQhbnd + ((size_t)cr * D2 + 2 * d) * F * nD, d);
    } else if (j->phase == 2) { /* boundary face */
      const int c = m->bcell[i], f = m->bface[i];
      if (k->boundary_face_kind)
        k->boundary_face_kind(k->ctx, m->lFhbnd + ((size_t)c * D2 + f) * F * nV,
                              m->lQhbnd + ((size_t)c * D2 + f) * F * nD, f, m->bc[f]);
      else
        k->boundary_face(k->ctx, m->lFhbnd + ((size_t)c * D2 + f) * F * nV, m->lQhbnd + ((size_t)c * D2 + f) * F * nD, f);
    } else if (j->phase == 3) { /* corrector + admissible step */
      double* u = m->luh + (size_t)i * P * nD;
      double* du = m->lduh + (size_t)i * P * nV;
      k->surface_integral(k->ctx, du, m->lFhbnd + (size_t)i * D2 * F * nV, m->dx);
      k->solution_update(k->ctx, u, du, m->dt);
      const double d = k->stable_dt(k->ctx, u, m->dx);
      j->dtmin = (d < j->dtmin) ? d : j->dtmin;
    } else { /* admissible step only */
      const double d = k->stable_dt(k->ctx, m->luh + (size_t)i * P * nD, m->dx);
      j->dtmin = (d < j->dtmin) ? d : j->dtmin;
    }
  }
}

static void* hrn_thread(void* a) {
  hrn_run_range((hrn_job*)a);
  return 0;
}

/* runs `phase` over [0, n); returns the min of the per-item step sizes */
static double hrn_parallel(hrn_mesh* m, int phase, int n) {
  const int T = m->nthreads < n ? m->nthreads : (n > 0 ? n : 1);
  hrn_job jobs[256];
  pthread_t th[256];
  const int nt = T > 256 ? 256 : T;
  for (int t = 0; t < nt; t++) {
    jobs[t].m = m;
    jobs[t].phase = phase;
    jobs[t].lo = (int)((long)n * t / nt);
    jobs[t].hi = (int)((long)n * (t + 1) / nt);
  }
  if (nt == 1) {
    hrn_run_range(&jobs[0]);
  } else {
    for (int t = 1; t < nt; t++) pthread_create(&th[t], 0, hrn_thread, &jobs[t]);
    hrn_run_range(&jobs[0]);
    for (int t = 1; t < nt; t++) pthread_join(th[t], 0);
  }
  double r = DBL_MAX;
  for (int t = 0; t < nt; t++) r = (jobs[t].dtmin < r) ? jobs[t].dtmin : r;
  return r;
}

static void hrn_predict(hrn_mesh* m) {
  hrn_parallel(m, 0, m->ncells);
  for (int i = 0; i < m->ncells; i++) m->sweeps += m->iters[i];
}

static void hrn_init(hrn_mesh* m, double t0) {
  m->t = t0;
  m->steps = 0;
  m->sweeps = 0;
  m->fused = 0;
  m->dt = hrn_parallel(m, 4, m->ncells);
  m->pdt = m->dt;
  m->pt = t0;
  hrn_predict(m);
}

static void hrn_init_fused(hrn_mesh* m, double t0, double w) {
  m->t = t0;
  m->steps = 0;
  m->sweeps = 0;
  m->fused = 1;
  m->w = w;
  m->reruns = 0;
  const double s0 = hrn_parallel(m, 4, m->ncells);
  m->dt = s0;
  m->pdt = s0;
  m->tp = t0 + s0;
  m->next = DBL_MAX;
  m->pt = t0;
  hrn_predict(m);
}

static void hrn_step_fused(hrn_mesh* m) {
  hrn_parallel(m, 1, m->nfaces);
  hrn_parallel(m, 2, m->nb);
  const double s = hrn_parallel(m, 3, m->ncells); /* corrector with m->dt */
  m->pt = m->tp;                                  /* the updated solution's stamp */
  hrn_predict(m);                                 /* predictor with m->pdt */
  double next = DBL_MAX;
  next = (s < next) ? s : next; /* updateMinNextPredictorTimeStepSize */
  const double used = (m->pdt == 0.0) ? s : m->pdt;
  const int unstable = used > s;
  if (unstable) {
    const double ws = m->w * s;
    next = (ws < next) ? ws : next;
    m->pdt = ws;
  } else {
    const double avg = 0.5 * (used + m->w * s);
    next = (avg < next) ? avg : next;
  }
  /* startNewTimeStep */
  m->t = m->tp;
  m->dt = m->pdt;
  m->tp = m->tp + m->pdt;
  m->pdt = next;
  m->steps++;
  if (unstable) {
    m->reruns++;
    m->pt = m->t;
    hrn_predict(m);
  }
}

static void hrn_step(hrn_mesh* m, int n) {
  if (m->fused) {
    for (int s = 0; s < n; s++) hrn_step_fused(m);
    return;
  }
  for (int s = 0; s < n; s++) {
    hrn_parallel(m, 1, m->nfaces);
    hrn_parallel(m, 2, m->nb);
    const double dtn = hrn_parallel(m, 3, m->ncells);
    m->t += m->dt;
    m->dt = dtn;
    m->pdt = dtn;
    m->pt = m->t;
    m->steps++;
    hrn_predict(m);
  }
}

static int hrn_run_until(hrn_mesh* m, double t_end, int max_steps) {
  int n = 0;
  while (n < max_steps && m->t < t_end && m->dt > 0.0) {
    hrn_step(m, 1);
    n++;
  }
  return n;
}
