/*
 * ORACLE harness, limiting ADER-DG -- test infrastructure only. A uniform
 * mesh with the reference's a-posteriori subcell limiter sequencing
 * (exahype/solvers/LimitingADERDGSolver.cpp, mappings/{Merging,SolutionUpdate,
 * LimiterStatusSpreading,LocalRecomputation,Prediction}.cpp,
 * runners/Runner.cpp:866-946,1116-1162), globally time stepped, non-fused:
 *
 * merge (per face, current statuses s1,s2; A = activeFV = h+1, T = troubled = 2h+1):
 *   both < A: DG Riemann; both >= A: FV ghost layers; mixed: both
 *   (mergeNeighboursBasedOnLimiterStatus, :1560-1628); DMP min/max of the two
 *   face blocks (mergeSolutionMinMaxOnFace, :1654-1690); facewise statuses
 *   max(0, max(min(s1,T),min(s2,T)) - 1) (ADERDGSolver.cpp:2544-2560).
 *   Boundary faces: DG boundary if s < A, FV boundary otherwise (outflow or
 *   reflective, per domain face).
 * update (per cell, LimitingADERDGSolver::updateSolution :843-908):
 *   s == 0: DG corrector; 0 < s < A: DG corrector, FV copy = projection;
 *   s >= A: MUSCL-Hancock on the FV patch, DG solution = its projection.
 *   New admissible step from the DG solution; DMP (+ admissibility) on it
 *   (:910-1067); FV cells overwrite all min/max blocks with FV-subcell values;
 *   status machine determineLimiterStatusAfterSolutionUpdate (:956-994).
 * irregular change (a cell with s < A became troubled): status spreading (T
 *   sweeps of the facewise merge, :392-405), reinitialiseSolversLocally
 *   (rollback of cells with s > 0, :1329-1360), local recomputation (FV ghost
 *   exchange only, recomputeSolutionLocally :1396-1436) and a new admissible
 *   step from all cells.
 * predictor for cells with s < T (mappings/Prediction.cpp:176-178).
 *
 * The FV re-update of the local recomputation uses the step size of the step
 * being redone. The solver clock follows the reference's bookkeeping: on an
 * irregular step LocalRecomputation::endIteration runs startNewTimeStep() and
 * reconstructStandardTimeSteppingData() a second time
 * (mappings/LocalRecomputation.cpp:193-207 after SolutionUpdate.cpp:308-322),
 * so the corrector time stamp advances by the step size found after the update
 * once more and the next step uses the size found after the recomputation.
 * This file is #included after harness.c.
 */

typedef struct {
  void (*project_fv)(void* ctx, const double* luh, double* lim);
  void (*project_dg)(void* ctx, const double* lim, double* luh);
  void (*limiter_minmax)(void* ctx, const double* lim, double* mn, double* mx);
  void (*local_minmax)(void* ctx, const double* luh, double* mn, double* mx);
  int (*dmp)(void* ctx, const double* luh, double relax, double scale, double* minB, double* maxB);
  int (*admissible)(void* ctx, const double* obsMin);
  void (*fv_update)(void* ctx, double* lnew, const double* lold, const double* dx, double dt);
  void (*fv_ghost)(void* ctx, double* lim, const double* nb, int face);
  void (*fv_boundary)(void* ctx, double* lim, int face);
  int fv_size; /* doubles per FV patch incl. ghosts */
  /* optional: an FV boundary face that needs the boundary kind of its domain
   * face (0 outflow, 1 reflective); used instead of fv_boundary when set */
  void (*fv_boundary_kind)(void* ctx, double* lim, int face, int kind);
} lhrn_backend;

typedef struct {
  hrn_mesh* m;
  lhrn_backend L;
  int h, A, T, cure_steps;
  double relax, scale;
  int *s, *s_prev, *cure, *fs, *has_lim;
  double *minB, *maxB, *lim, *lim_prev, *luh_prev;
  long irregular_steps, troubled_cell_steps;
  int last_change; /* 0 regular, 1 irregular */
  double* fv_ic; /* optional FV initial condition [cell][B^d][nV] at subcell centres */
} lhrn;

static lhrn* lhrn_create(const hrn_backend* k, const lhrn_backend* L, const int* cells, const double* size,
                         const int* bc, int nthreads, int helper_layers, int cure_steps, double relax, double scale) {
  lhrn* r = (lhrn*)calloc(1, sizeof(lhrn));
  r->m = hrn_create(k, cells, size, bc, nthreads);
  r->L = *L;
  r->h = helper_layers;
  r->A = helper_layers + 1;
  r->T = 2 * helper_layers + 1;
  r->cure_steps = cure_steps;
  r->relax = relax;
  r->scale = scale;
  const int n = r->m->ncells, D2 = 2 * r->m->dim, nO = k->nvar;
  r->s = (int*)calloc(n, sizeof(int));
  r->s_prev = (int*)calloc(n, sizeof(int));
  r->cure = (int*)calloc(n, sizeof(int));
  r->fs = (int*)calloc((size_t)n * D2, sizeof(int));
  r->has_lim = (int*)calloc(n, sizeof(int));
  r->minB = (double*)calloc((size_t)n * D2 * nO, sizeof(double));
  r->maxB = (double*)calloc((size_t)n * D2 * nO, sizeof(double));
  r->lim = (double*)calloc((size_t)n * L->fv_size, sizeof(double));
  r->lim_prev = (double*)calloc((size_t)n * L->fv_size, sizeof(double));
  r->luh_prev = (double*)calloc((size_t)n * r->m->P * k->ndata, sizeof(double));
  return r;
}

static void lhrn_destroy(lhrn* r) {
  if (!r) return;
  hrn_destroy(r->m);
  free(r->s); free(r->s_prev); free(r->cure); free(r->fs); free(r->has_lim);
  free(r->minB); free(r->maxB); free(r->lim); free(r->lim_prev); free(r->luh_prev);
  free(r->fv_ic);
  free(r);
}

#define LH_LUH(r, c) ((r)->m->luh + (size_t)(c) * (r)->m->P * (r)->m->k.ndata)
#define LH_LUHP(r, c) ((r)->luh_prev + (size_t)(c) * (r)->m->P * (r)->m->k.ndata)
#define LH_LIM(r, c) ((r)->lim + (size_t)(c) * (r)->L.fv_size)
#define LH_LIMP(r, c) ((r)->lim_prev + (size_t)(c) * (r)->L.fv_size)

static int lh_imin(int a, int b) { return a < b ? a : b; }
static int lh_imax(int a, int b) { return a > b ? a : b; }

/* allocate (zeroed) an FV patch; the reference allocates lazily on s > 0 */
static void lh_alloc(lhrn* r, int c) {
  if (!r->has_lim[c]) {
    memset(LH_LIM(r, c), 0, sizeof(double) * r->L.fv_size);
    memset(LH_LIMP(r, c), 0, sizeof(double) * r->L.fv_size);
    r->has_lim[c] = 1;
  }
}
static void lh_swap_lim(lhrn* r, int c) {
  double* a = LH_LIM(r, c);
  double* b = LH_LIMP(r, c);
  for (int i = 0; i < r->L.fv_size; i++) {
    const double t = a[i];
    a[i] = b[i];
    b[i] = t;
  }
}
static void lh_swap_luh(lhrn* r, int c) {
  double* a = LH_LUH(r, c);
  double* b = LH_LUHP(r, c);
  for (int i = 0; i < r->m->P * r->m->k.ndata; i++) {
    const double t = a[i];
    a[i] = b[i];
    b[i] = t;
  }
}

/* min/max of the DG solution into all 2d blocks (determineSolverMinAndMax, :1101-1130) */
static void lh_solver_minmax(lhrn* r, int c) {
  const int nO = r->m->k.nvar, D2 = 2 * r->m->dim;
  double* mn = r->minB + (size_t)c * D2 * nO;
  double* mx = r->maxB + (size_t)c * D2 * nO;
  r->L.local_minmax(r->m->k.ctx, LH_LUH(r, c), mn, mx);
  for (int i = 1; i < D2; i++) {
    memcpy(mn + i * nO, mn, sizeof(double) * nO);
    memcpy(mx + i * nO, mx, sizeof(double) * nO);
  }
}
static void lh_limiter_minmax(lhrn* r, int c) { /* determineLimiterMinAndMax, :1132-1159 */
  const int nO = r->m->k.nvar, D2 = 2 * r->m->dim;
  double* mn = r->minB + (size_t)c * D2 * nO;
  double* mx = r->maxB + (size_t)c * D2 * nO;
  r->L.limiter_minmax(r->m->k.ctx, LH_LIM(r, c), mn, mx);
  for (int i = 1; i < D2; i++) {
    memcpy(mn + i * nO, mn, sizeof(double) * nO);
    memcpy(mx + i * nO, mx, sizeof(double) * nO);
  }
}

static void lh_spread_once(lhrn* r) { /* one LimiterStatusSpreading iteration */
  hrn_mesh* m = r->m;
  const int D2 = 2 * m->dim;
  memset(r->fs, 0, sizeof(int) * (size_t)m->ncells * D2);
  for (int f = 0; f < m->nfaces; f++) {
    const int c1 = m->fl[f], c2 = m->fr[f], d = m->fd[f];
    const int v = lh_imax(0, lh_imax(lh_imin(r->s[c1], r->T), lh_imin(r->s[c2], r->T)) - 1);
    r->fs[c1 * D2 + 2 * d + 1] = v;
    r->fs[c2 * D2 + 2 * d] = v;
  }
  for (int c = 0; c < m->ncells; c++) {
    if (r->s[c] < r->T) {
      int mx = 0;
      for (int i = 0; i < D2; i++) mx = lh_imax(mx, r->fs[c * D2 + i]);
      r->s[c] = mx;
    } else {
      r->s[c] = r->T;
      r->cure[c] = r->cure_steps + 1;
    }
    if (r->s[c] > 0) lh_alloc(r, c);
  }
  memset(r->fs, 0, sizeof(int) * (size_t)m->ncells * D2);
}

static void lh_predict(lhrn* r) {
  hrn_mesh* m = r->m;
  const hrn_backend* k = &m->k;
  const int P = m->P, F = m->F, nV = k->nvar, nD = k->ndata, D2 = 2 * m->dim;
  for (int c = 0; c < m->ncells; c++) {
    if (r->s[c] >= r->T) {
      m->iters[c] = 0;
      continue;
    }
    m->iters[c] = k->predictor(k->ctx, LH_LUH(r, c), m->dx, m->dt, m->lQhbnd + (size_t)c * D2 * F * nD,
                               m->lFhbnd + (size_t)c * D2 * F * nV, m->lduh + (size_t)c * P * nV);
    m->sweeps += m->iters[c];
  }
}

/* initial conditions already in m->luh */
static void lhrn_init(lhrn* r, double t0) {
  hrn_mesh* m = r->m;
  m->t = t0;
  m->steps = 0;
  m->sweeps = 0;
  for (int c = 0; c < m->ncells; c++) {
    r->s[c] = 0;
    r->cure[c] = 0;
    r->has_lim[c] = 0;
    lh_solver_minmax(r, c); /* updateLimiterStatusAndMinAndMaxAfterSetInitialConditions, :1069-1083 */
    const int nO = m->k.nvar, D2 = 2 * m->dim;
    if (!r->L.admissible(m->k.ctx, r->minB + (size_t)c * D2 * nO)) {
      r->cure[c] = r->cure_steps + 1;
      r->s[c] = r->T;
    }
  }
  int any = 0;
  for (int c = 0; c < m->ncells; c++) any |= r->s[c] > 0;
  if (any) {
    for (int it = 0; it < r->T; it++) lh_spread_once(r);
    /* limiter patches start from the FV solver's own initial condition at the
     * subcell centres (LimitingADERDGSolver::setInitialConditions, :745-770),
     * or from the projection of the DG solution when none is given */
    const int dim = m->dim, B = 2 * m->k.order + 1, E = B + 4, nV = m->k.nvar;
    const int Bd = dim == 3 ? B * B * B : B * B;
    for (int c = 0; c < m->ncells; c++)
      if (r->s[c] > 0) {
        lh_alloc(r, c);
        if (r->fv_ic) {
          double* l = LH_LIM(r, c);
          for (int q = 0; q < Bd; q++) {
            const int x = q % B, y = (q / B) % B, z = dim == 3 ? q / (B * B) : 0;
            const int zz = dim == 3 ? z + 2 : 0;
            memcpy(l + ((zz * E + y + 2) * E + x + 2) * nV, r->fv_ic + ((size_t)c * Bd + q) * nV, sizeof(double) * nV);
          }
        } else {
          r->L.project_fv(m->k.ctx, LH_LUH(r, c), LH_LIM(r, c));
        }
      }
  }
  double dt = DBL_MAX;
  for (int c = 0; c < m->ncells; c++) {
    const double d = m->k.stable_dt(m->k.ctx, LH_LUH(r, c), m->dx);
    dt = (d < dt) ? d : dt;
  }
  m->dt = dt;
  lh_predict(r);
}

/* FV ghost exchange / boundary for one face pair or boundary face */
static void lh_fv_face(lhrn* r, int c1, int c2, int d) {
  if (!r->has_lim[c1] || !r->has_lim[c2]) return;
  r->L.fv_ghost(r->m->k.ctx, LH_LIM(r, c1), LH_LIM(r, c2), 2 * d + 1);
  r->L.fv_ghost(r->m->k.ctx, LH_LIM(r, c2), LH_LIM(r, c1), 2 * d);
}

static void lh_merge(lhrn* r, int recompute) {
  hrn_mesh* m = r->m;
  const hrn_backend* k = &m->k;
  const int F = m->F, nV = k->nvar, nD = k->ndata, D2 = 2 * m->dim, nO = k->nvar;
  for (int f = 0; f < m->nfaces; f++) {
    const int c1 = m->fl[f], c2 = m->fr[f], d = m->fd[f];
    const int s1 = r->s[c1], s2 = r->s[c2];
    const int dg = !recompute && (s1 < r->A || s2 < r->A);
    const int fv = s1 >= r->A || s2 >= r->A;
    if (fv) lh_fv_face(r, c1, c2, d);
    if (dg)
      k->riemann(k->ctx, m->lFhbnd + ((size_t)c1 * D2 + 2 * d + 1) * F * nV,
                 m->lFhbnd + ((size_t)c2 * D2 + 2 * d) * F * nV, m->lQhbnd + ((size_t)c1 * D2 + 2 * d + 1) * F * nD,
                 m->lQhbnd + ((size_t)c2 * D2 + 2 * d) * F * nD, d);
    if (!recompute) {
      double* mn1 = r->minB + ((size_t)c1 * D2 + 2 * d + 1) * nO;
      double* mn2 = r->minB + ((size_t)c2 * D2 + 2 * d) * nO;
      double* mx1 = r->maxB + ((size_t)c1 * D2 + 2 * d + 1) * nO;
      double* mx2 = r->maxB + ((size_t)c2 * D2 + 2 * d) * nO;
      for (int i = 0; i < nO; i++) {
        const double mn = (mn2[i] < mn1[i]) ? mn2[i] : mn1[i];
        const double mx = (mx1[i] < mx2[i]) ? mx2[i] : mx1[i];
        mn1[i] = mn2[i] = mn;
        mx1[i] = mx2[i] = mx;
      }
      const int v = lh_imax(0, lh_imax(lh_imin(s1, r->T), lh_imin(s2, r->T)) - 1);
      r->fs[c1 * D2 + 2 * d + 1] = v;
      r->fs[c2 * D2 + 2 * d] = v;
    }
  }
  for (int f = 0; f < m->nb; f++) {
    const int c = m->bcell[f], face = m->bface[f];
    if (r->s[c] < r->A) {
      if (!recompute) {
        double* FIn = m->lFhbnd + ((size_t)c * D2 + face) * F * nV;
        const double* QIn = m->lQhbnd + ((size_t)c * D2 + face) * F * nD;
        if (k->boundary_face_kind)
          k->boundary_face_kind(k->ctx, FIn, QIn, face, m->bc[face]);
        else
          k->boundary_face(k->ctx, FIn, QIn, face);
      }
    } else if (r->has_lim[c]) {
      if (r->L.fv_boundary_kind)
        r->L.fv_boundary_kind(k->ctx, LH_LIM(r, c), face, m->bc[face]);
      else
        r->L.fv_boundary(k->ctx, LH_LIM(r, c), face);
    }
  }
}

static void lh_fv_step(lhrn* r, int c, double dt) {
  lh_alloc(r, c);
  memcpy(LH_LIMP(r, c), LH_LIM(r, c), sizeof(double) * r->L.fv_size);
  r->L.fv_update(r->m->k.ctx, LH_LIM(r, c), LH_LIMP(r, c), r->m->dx, dt);
  r->L.project_dg(r->m->k.ctx, LH_LIM(r, c), LH_LUH(r, c));
}

static void lhrn_step(lhrn* r) {
  hrn_mesh* m = r->m;
  const hrn_backend* k = &m->k;
  const int P = m->P, F = m->F, nV = k->nvar, nD = k->ndata, D2 = 2 * m->dim, nO = k->nvar;
  const double dt = m->dt;
  lh_merge(r, 0);
  double dtn = DBL_MAX;
  int irregular = 0;
  for (int c = 0; c < m->ncells; c++) {
    const int s = r->s[c];
    r->s_prev[c] = s;
    double* u = LH_LUH(r, c);
    if (s < r->A) {
      memcpy(LH_LUHP(r, c), u, sizeof(double) * P * nD);
      double* du = m->lduh + (size_t)c * P * nV;
      k->surface_integral(k->ctx, du, m->lFhbnd + (size_t)c * D2 * F * nV, m->dx);
      k->solution_update(k->ctx, u, du, dt);
      if (s > 0) {
        lh_alloc(r, c);
        lh_swap_lim(r, c);
        r->L.project_fv(k->ctx, u, LH_LIM(r, c));
      }
    } else {
      lh_fv_step(r, c, dt);
    }
    if (s == 0) r->has_lim[c] = 0; /* ensureNoUnrequiredLimiterPatchIsAllocatedOnComputeCell */
    const double d = k->stable_dt(k->ctx, u, m->dx);
    dtn = (d < dtn) ? d : dtn;
    double* mn = r->minB + (size_t)c * D2 * nO;
    double* mx = r->maxB + (size_t)c * D2 * nO;
    const int valid = r->L.dmp(k->ctx, u, r->relax, r->scale, mn, mx) && r->L.admissible(k->ctx, mn);
    if (s >= r->A) lh_limiter_minmax(r, c);
    if (!valid) {
      r->cure[c] = r->cure_steps + 1;
      if (!(s > r->A)) irregular = 1;
      r->s[c] = r->T;
    } else if (r->s_prev[c] >= r->T) {
      r->s[c] = r->T;
      r->cure[c] -= 1;
      if (r->cure[c] == 0) {
        r->s[c] = r->T - 1;
        r->cure[c] = r->cure_steps + 1;
      }
    } else {
      int mxs = 0;
      for (int i = 0; i < D2; i++) mxs = lh_imax(mxs, r->fs[c * D2 + i]);
      r->s[c] = mxs;
    }
    /* allocateLimiterPatchAfterSolutionUpdate, :939-954 */
    if (r->s[c] > 0 && !r->has_lim[c]) {
      lh_alloc(r, c);
      if (r->s[c] < r->A) r->L.project_fv(k->ctx, u, LH_LIM(r, c));
    }
    for (int i = 0; i < D2; i++) r->fs[c * D2 + i] = 0;
  }
  for (int c = 0; c < m->ncells; c++) r->troubled_cell_steps += r->s[c] >= r->T;
  r->last_change = irregular;
  const double dt_after_update = dtn;
  if (irregular) {
    r->irregular_steps++;
    for (int it = 0; it < r->T; it++) lh_spread_once(r);
    /* reinitialiseSolversLocally, :1329-1360 */
    for (int c = 0; c < m->ncells; c++) {
      if (r->s[c] > 0) {
        lh_alloc(r, c);
        if (r->s_prev[c] >= r->A) {
          lh_swap_lim(r, c);
          r->L.project_dg(k->ctx, LH_LIM(r, c), LH_LUH(r, c));
        } else {
          lh_swap_luh(r, c);
          r->L.project_fv(k->ctx, LH_LUH(r, c), LH_LIM(r, c));
        }
        if (r->s[c] >= r->T) r->cure[c] = r->cure_steps + 1;
      } else {
        r->has_lim[c] = 0;
      }
    }
    /* local recomputation: FV ghost layers only, then recomputeSolutionLocally */
    lh_merge(r, 1);
    dtn = DBL_MAX;
    for (int c = 0; c < m->ncells; c++) {
      if (r->s[c] > 0) {
        if (r->s[c] >= r->A) {
          lh_fv_step(r, c, dt);
        } else if (r->s_prev[c] < r->A) {
          lh_swap_luh(r, c);
          r->L.project_fv(k->ctx, LH_LUH(r, c), LH_LIM(r, c));
        } else {
          lh_swap_lim(r, c);
          r->L.project_dg(k->ctx, LH_LIM(r, c), LH_LUH(r, c));
        }
      }
      const double d = k->stable_dt(k->ctx, LH_LUH(r, c), m->dx);
      dtn = (d < dtn) ? d : dtn;
    }
  }
  m->t += dt;
  if (irregular) m->t += dt_after_update;
  m->dt = dtn;
  m->steps++;
  lh_predict(r);
}

static int lhrn_run_until(lhrn* r, double t_end, int max_steps) {
  int n = 0;
  while (n < max_steps && r->m->t < t_end && r->m->dt > 0.0) {
    lhrn_step(r);
    n++;
  }
  return n;
}
