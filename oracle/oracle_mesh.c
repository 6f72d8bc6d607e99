/* ORACLE -- test infrastructure only: the uniform-mesh harness (harness.c)
 * over the C restatement of the kernels (oracle.c). */
#include "oracle.h"
#include "harness.c"
#include "limiting_harness.c"

static int be_pred(void* c, const double* luh, const double* dx, double dt, double* qb, double* fb, double* du) {
  return orc_predictor((const orc_solver*)c, luh, dx, dt, qb, fb, du, 0, 0, 0, 0);
}
static void be_riem(void* c, double* FL, double* FR, const double* QL, const double* QR, int d) {
  orc_riemann((const orc_solver*)c, FL, FR, QL, QR, d);
}
static void be_bnd(void* c, double* FIn, const double* QIn, int f) {
  const double z[3] = {0, 0, 0};
  orc_boundary_face((const orc_solver*)c, FIn, QIn, z, z, 0.0, 0.0, f);
}
/* Euler (pde 0): outflow, or the demonstrator's reflective walls */
static void be_bnd_kind(void* c, double* FIn, const double* QIn, int f, int kind) {
  if (kind == 1)
    orc_boundary_face_reflective((const orc_solver*)c, FIn, QIn, f);
  else
    be_bnd(c, FIn, QIn, f);
}
static void be_surf(void* c, double* du, const double* fb, const double* dx) { orc_surface_integral((const orc_solver*)c, du, fb, dx); }
static void be_upd(void* c, double* u, const double* du, double dt) { orc_solution_update((const orc_solver*)c, u, du, dt); }
static double be_dt(void* c, const double* u, const double* dx) { return orc_stable_dt((const orc_solver*)c, u, dx); }

/* linear PDEs (pde 2, 4): Cauchy-Kovalevski predictor, linear Riemann solver,
 * surface integral and boundary faces (outflow, rigid wall) */
static int be_lpred(void* c, const double* luh, const double* dx, double dt, double* qb, double* fb, double* du) {
  orc_lin_predictor((const orc_solver*)c, luh, dx, dt, qb, fb, du, 0, 0);
  return 0;
}
static void be_lriem(void* c, double* FL, double* FR, const double* QL, const double* QR, int d) {
  orc_lin_riemann((const orc_solver*)c, FL, FR, QL, QR, d);
}
static void be_lsurf(void* c, double* du, const double* fb, const double* dx) {
  orc_lin_surface_integral((const orc_solver*)c, du, fb, dx);
}
static void be_lbnd(void* c, double* FIn, const double* QIn, int f, int kind) {
  orc_lin_boundary_face((const orc_solver*)c, FIn, QIn, f, kind);
}
/* point sources (pde 4): pointSource at the cell's centre, then the linear
 * predictor with usePointSource */
static int be_lpred_ps(void* c, const double* luh, const double* dx, const double* centre, double t, double dt,
                       double* qb, double* fb, double* du) {
  const orc_solver* s = (const orc_solver*)c;
  const int b = s->order + 1, P = s->dim == 3 ? b * b * b : b * b;
  double* PSi = (double*)malloc(sizeof(double) * (b + 1) * P * orc_nvar(s));
  orc_point_source(s, t, dt, centre, dx, PSi);
  orc_lin_predictor_ps(s, luh, dx, dt, PSi, qb, fb, du, 0, 0);
  free(PSi);
  return 0;
}

typedef struct {
  orc_solver s;
  hrn_mesh* m;
} orc_mesh;

void* orc_mesh_create(int dim, int order, int pde, const int* cells, const double* size, const int* bc, int nthreads) {
  orc_mesh* om = (orc_mesh*)calloc(1, sizeof(orc_mesh));
  om->s.dim = dim;
  om->s.order = order;
  om->s.pde = pde;
  hrn_backend k = {&om->s, dim, order, orc_nvar(&om->s), orc_nvar(&om->s) + orc_npar(&om->s),
                   be_pred, be_riem, be_bnd, be_surf, be_upd, be_dt};
  if (pde == 0) k.boundary_face_kind = be_bnd_kind;
  if (ORC_ELASTIC(&om->s)) {
    k.predictor = be_lpred;
    k.riemann = be_lriem;
    k.surface_integral = be_lsurf;
    k.boundary_face_kind = be_lbnd;
    if (pde == 4) k.predictor_at = be_lpred_ps;
  }
  om->m = hrn_create(&k, cells, size, bc, nthreads);
  return om;
}
/* the point source of pde 4: x0[3], t0, f0, amplitude */
void orc_mesh_set_point_source(void* h, const double* ps) {
  for (int i = 0; i < 6; i++) ((orc_mesh*)h)->s.ps[i] = ps[i];
}
void orc_mesh_destroy(void* h) { orc_mesh* om = (orc_mesh*)h; hrn_destroy(om->m); free(om); }
static size_t nsol(hrn_mesh* m) { return (size_t)m->ncells * m->P * m->k.ndata; }
void orc_mesh_set_solution(void* h, const double* u) { hrn_mesh* m = ((orc_mesh*)h)->m; memcpy(m->luh, u, nsol(m) * 8); }
void orc_mesh_get_solution(void* h, double* u) { hrn_mesh* m = ((orc_mesh*)h)->m; memcpy(u, m->luh, nsol(m) * 8); }
void orc_mesh_init(void* h, double t0) { hrn_init(((orc_mesh*)h)->m, t0); }
/* fused time stepping with rerun weight w (hrn_init_fused in harness.c) */
void orc_mesh_init_fused(void* h, double t0, double w) { hrn_init_fused(((orc_mesh*)h)->m, t0, w); }
double orc_mesh_predictor_dt(void* h) { return ((orc_mesh*)h)->m->pdt; }
long orc_mesh_reruns(void* h) { return ((orc_mesh*)h)->m->reruns; }
void orc_mesh_step(void* h, int n) { hrn_step(((orc_mesh*)h)->m, n); }
int orc_mesh_run_until(void* h, double t_end, int max_steps) { return hrn_run_until(((orc_mesh*)h)->m, t_end, max_steps); }
double orc_mesh_time(void* h) { return ((orc_mesh*)h)->m->t; }
double orc_mesh_dt(void* h) { return ((orc_mesh*)h)->m->dt; }
long orc_mesh_steps(void* h) { return ((orc_mesh*)h)->m->steps; }
long orc_mesh_sweeps(void* h) { return ((orc_mesh*)h)->m->sweeps; }

/* ---- limiting mesh over the C restatement ---- */
void orc_project_fv(const orc_solver* s, const double* luh, double* lim);
void orc_project_dg(const orc_solver* s, const double* lim, double* luh);
void orc_local_minmax(const orc_solver* s, const double* luh, double* mn, double* mx);
void orc_limiter_minmax(const orc_solver* s, const double* lim, double* mn, double* mx);
int orc_dmp(const orc_solver* s, const double* luh, double relax, double scale, double* minB, double* maxB);
int orc_admissible(const orc_solver* s, const double* obsMin);
double orc_musclhancock(const orc_solver* s, double* lnew, const double* lold, const double* dx, double dt);
void orc_fv_ghost_fill(const orc_solver* s, double* lim, const double* nb, int face);
void orc_fv_boundary_fill(const orc_solver* s, double* lim, int face);
int orc_fv_patch_size(const orc_solver* s);

static void lb_pfv(void* c, const double* u, double* l) { orc_project_fv((const orc_solver*)c, u, l); }
static void lb_pdg(void* c, const double* l, double* u) { orc_project_dg((const orc_solver*)c, l, u); }
static void lb_lmm(void* c, const double* l, double* a, double* b) { orc_limiter_minmax((const orc_solver*)c, l, a, b); }
static void lb_smm(void* c, const double* u, double* a, double* b) { orc_local_minmax((const orc_solver*)c, u, a, b); }
static int lb_dmp(void* c, const double* u, double r, double sc, double* a, double* b) { return orc_dmp((const orc_solver*)c, u, r, sc, a, b); }
static int lb_adm(void* c, const double* m) { return orc_admissible((const orc_solver*)c, m); }
static void lb_fvu(void* c, double* ln, const double* lo, const double* dx, double dt) { orc_musclhancock((const orc_solver*)c, ln, lo, dx, dt); }
static void lb_fvg(void* c, double* l, const double* nb, int f) { orc_fv_ghost_fill((const orc_solver*)c, l, nb, f); }
static void lb_fvb(void* c, double* l, int f) { orc_fv_boundary_fill((const orc_solver*)c, l, f); }
void orc_fv_boundary_fill_kind(const orc_solver* s, double* lim, int face, int kind);
static void lb_fvb_kind(void* c, double* l, int f, int kind) { orc_fv_boundary_fill_kind((const orc_solver*)c, l, f, kind); }

typedef struct {
  orc_solver s;
  lhrn* r;
} orc_lmesh;

void* orc_lmesh_create(int dim, int order, const int* cells, const double* size, const int* bc, int nthreads,
                       int helper_layers, int cure_steps, double relax, double scale) {
  orc_lmesh* om = (orc_lmesh*)calloc(1, sizeof(orc_lmesh));
  om->s.dim = dim;
  om->s.order = order;
  om->s.pde = 0;
  hrn_backend k = {&om->s, dim, order, 5, 5, be_pred, be_riem, be_bnd, be_surf, be_upd, be_dt};
  k.boundary_face_kind = be_bnd_kind;
  lhrn_backend L = {lb_pfv, lb_pdg, lb_lmm, lb_smm, lb_dmp, lb_adm, lb_fvu, lb_fvg, lb_fvb, orc_fv_patch_size(&om->s)};
  L.fv_boundary_kind = lb_fvb_kind;
  om->r = lhrn_create(&k, &L, cells, size, bc, nthreads, helper_layers, cure_steps, relax, scale);
  return om;
}
void orc_lmesh_destroy(void* h) { orc_lmesh* om = (orc_lmesh*)h; lhrn_destroy(om->r); free(om); }
void orc_lmesh_set_solution(void* h, const double* u) { hrn_mesh* m = ((orc_lmesh*)h)->r->m; memcpy(m->luh, u, nsol(m) * 8); }
void orc_lmesh_get_solution(void* h, double* u) { hrn_mesh* m = ((orc_lmesh*)h)->r->m; memcpy(u, m->luh, nsol(m) * 8); }
void orc_lmesh_init(void* h, double t0) { lhrn_init(((orc_lmesh*)h)->r, t0); }
/* FV initial condition for cells that are limited at t0: [cell][(2N+1)^d][nV] */
void orc_lmesh_set_fv_initial(void* h, const double* v) {
  lhrn* r = ((orc_lmesh*)h)->r;
  const int B = 2 * r->m->k.order + 1, Bd = r->m->dim == 3 ? B * B * B : B * B;
  const size_t n = (size_t)r->m->ncells * Bd * r->m->k.nvar;
  free(r->fv_ic);
  r->fv_ic = (double*)malloc(sizeof(double) * n);
  memcpy(r->fv_ic, v, sizeof(double) * n);
}
void orc_lmesh_step(void* h, int n) { for (int i = 0; i < n; i++) lhrn_step(((orc_lmesh*)h)->r); }
int orc_lmesh_run_until(void* h, double t_end, int max_steps) { return lhrn_run_until(((orc_lmesh*)h)->r, t_end, max_steps); }
double orc_lmesh_time(void* h) { return ((orc_lmesh*)h)->r->m->t; }
double orc_lmesh_dt(void* h) { return ((orc_lmesh*)h)->r->m->dt; }
long orc_lmesh_steps(void* h) { return ((orc_lmesh*)h)->r->m->steps; }
long orc_lmesh_sweeps(void* h) { return ((orc_lmesh*)h)->r->m->sweeps; }
void orc_lmesh_status(void* h, int* s) { lhrn* r = ((orc_lmesh*)h)->r; memcpy(s, r->s, sizeof(int) * r->m->ncells); }
long orc_lmesh_irregular_steps(void* h) { return ((orc_lmesh*)h)->r->irregular_steps; }
/* FV patches [cell][E^d][nV] (ghost layers included) and allocation flags */
void orc_lmesh_limiter(void* h, double* lim, int* allocated) {
  lhrn* r = ((orc_lmesh*)h)->r;
  if (lim) memcpy(lim, r->lim, sizeof(double) * (size_t)r->m->ncells * r->L.fv_size);
  if (allocated) memcpy(allocated, r->has_lim, sizeof(int) * r->m->ncells);
}
