// Oracle-only: the uniform-mesh harness (oracle/harness.c) driving the
// reference's own kernels (ref_kernels.cpp). This is the CPU baseline path:
// the reference's generic kernels, parallel across cells on POSIX threads.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>

extern "C" {
#include "../harness.c"
#include "../limiting_harness.c"
}

#if DIMENSIONS == 2
#define REFNAME(x) ref2d_##x
#else
#define REFNAME(x) ref3d_##x
#endif

extern "C" {
int REFNAME(predictor)(int pde, int N, const double* luh, const double* dx, double dt, double* lQhbnd, double* lFhbnd,
                       double* lduh, double* lQi, double* lFi, double* lQhi, double* lFhi);
void REFNAME(riemann)(int pde, int N, double* FL, double* FR, const double* QL, const double* QR, double dt, int dir);
void REFNAME(boundary_face)(int pde, int N, double* FIn, const double* QIn, const double* centre, const double* size,
                            double t, double dt, int faceIndex);
void REFNAME(surface_integral)(int pde, int N, double* lduh, const double* lFhbnd, const double* dx);
void REFNAME(solution_update)(int pde, int N, double* luh, const double* lduh, double dt);
double REFNAME(stable_dt)(int pde, int N, const double* luh, const double* dx);
void REFNAME(lin_predictor)(int pde, int N, const double* luh, const double* dx, double dt, double* lQhbnd,
                            double* lFhbnd, double* lduh, double* lQhi, double* lFhi);
void REFNAME(lin_riemann)(int pde, int N, double* FL, double* FR, const double* QL, const double* QR, double dt,
                          int dir);
void REFNAME(lin_surface_integral)(int pde, int N, double* lduh, const double* lFhbnd, const double* dx);
void REFNAME(lin_boundary_face)(int pde, int N, double* FIn, const double* QIn, int faceIndex, int kind);
void REFNAME(boundary_face_kind)(int N, double* FIn, const double* QIn, int faceIndex, int kind);
void REFNAME(fv_boundary_kind)(int N, double* lim, int face, int kind);
void REFNAME(lin_predictor_ps)(int N, const double* ps, const double* centre, double t, const double* luh,
                               const double* dx, double dt, double* lQhbnd, double* lFhbnd, double* lduh,
                               double* lQhi, double* lFhi);
void REFNAME(init)();
void REFNAME(project_fv)(int N, const double* luh, double* lim);
void REFNAME(project_dg)(int N, const double* lim, double* luh);
void REFNAME(local_minmax)(int N, const double* luh, double* mn, double* mx);
void REFNAME(limiter_minmax)(int N, const double* lim, double* mn, double* mx);
int REFNAME(dmp)(int N, const double* luh, double relax, double scale, double* mn, double* mx);
double REFNAME(musclhancock)(int N, double* lnew, const double* lold, const double* dx, double dt);
void REFNAME(fv_ghost)(int N, double* lim, const double* nb, int face);
void REFNAME(fv_boundary)(int N, double* lim, int face);
}

namespace {
struct Ctx { int pde, N; double ps[6]; };
int be_pred(void* c, const double* luh, const double* dx, double dt, double* qb, double* fb, double* du) {
  Ctx* x = (Ctx*)c;
  return REFNAME(predictor)(x->pde, x->N, luh, dx, dt, qb, fb, du, nullptr, nullptr, nullptr, nullptr);
}
void be_riem(void* c, double* FL, double* FR, const double* QL, const double* QR, int d) {
  Ctx* x = (Ctx*)c;
  REFNAME(riemann)(x->pde, x->N, FL, FR, QL, QR, 0.0, d);
}
void be_bnd(void* c, double* FIn, const double* QIn, int f) {
  Ctx* x = (Ctx*)c;
  const double z[3] = {0, 0, 0};
  REFNAME(boundary_face)(x->pde, x->N, FIn, QIn, z, z, 0.0, 0.0, f);
}
// the demonstrator's Euler PDE (pde 0): outflow or reflective walls
void be_bnd_kind(void* c, double* FIn, const double* QIn, int f, int kind) {
  REFNAME(boundary_face_kind)(((Ctx*)c)->N, FIn, QIn, f, kind);
}
void be_surf(void* c, double* du, const double* fb, const double* dx) { Ctx* x = (Ctx*)c; REFNAME(surface_integral)(x->pde, x->N, du, fb, dx); }
void be_upd(void* c, double* u, const double* du, double dt) { Ctx* x = (Ctx*)c; REFNAME(solution_update)(x->pde, x->N, u, du, dt); }
double be_dt(void* c, const double* u, const double* dx) { Ctx* x = (Ctx*)c; return REFNAME(stable_dt)(x->pde, x->N, u, dx); }
// linear PDE (elastic waves): Cauchy-Kovalevski predictor, linear Riemann
// solver, surface integral and boundary faces; with point sources (pde 4)
// the predictor of each cell runs after its pointSource
int be_lpred(void* c, const double* luh, const double* dx, double dt, double* qb, double* fb, double* du) {
  Ctx* x = (Ctx*)c;
  REFNAME(lin_predictor)(x->pde, x->N, luh, dx, dt, qb, fb, du, nullptr, nullptr);
  return 0;
}
void be_lriem(void* c, double* FL, double* FR, const double* QL, const double* QR, int d) {
  Ctx* x = (Ctx*)c;
  REFNAME(lin_riemann)(x->pde, x->N, FL, FR, QL, QR, 0.0, d);
}
void be_lsurf(void* c, double* du, const double* fb, const double* dx) {
  Ctx* x = (Ctx*)c;
  REFNAME(lin_surface_integral)(x->pde, x->N, du, fb, dx);
}
void be_lbnd(void* c, double* FIn, const double* QIn, int f, int kind) {
  Ctx* x = (Ctx*)c;
  REFNAME(lin_boundary_face)(x->pde, x->N, FIn, QIn, f, kind);
}
int be_lpred_ps(void* c, const double* luh, const double* dx, const double* centre, double t, double dt, double* qb,
                double* fb, double* du) {
  Ctx* x = (Ctx*)c;
  REFNAME(lin_predictor_ps)(x->N, x->ps, centre, t, luh, dx, dt, qb, fb, du, nullptr, nullptr);
  return 0;
}
struct RefMesh { Ctx c; hrn_mesh* m; };
size_t nsol(hrn_mesh* m) { return (size_t)m->ncells * m->P * m->k.ndata; }
}

extern "C" {
void* REFNAME(mesh_create)(int order, int pde, const int* cells, const double* size, const int* bc, int nthreads) {
  REFNAME(init)();
  RefMesh* r = new RefMesh();
  r->c.pde = pde;
  r->c.N = order;
  hrn_backend k = {&r->c, DIMENSIONS, order, 5, 5 + (pde == 1 || pde == 3 ? 1 : 0), be_pred, be_riem, be_bnd, be_surf, be_upd, be_dt};
  if (pde == 0) k.boundary_face_kind = be_bnd_kind;
  if (pde == 2 || pde == 4) {
    k.nvar = 9;
    k.ndata = 12;
    k.predictor = be_lpred;
    k.riemann = be_lriem;
    k.surface_integral = be_lsurf;
    k.boundary_face_kind = be_lbnd;
    if (pde == 4) k.predictor_at = be_lpred_ps;
  }
  r->m = hrn_create(&k, cells, size, bc, nthreads);
  return r;
}
void REFNAME(mesh_set_point_source)(void* h, const double* ps) { std::copy_n(ps, 6, ((RefMesh*)h)->c.ps); }
void REFNAME(mesh_destroy)(void* h) { RefMesh* r = (RefMesh*)h; hrn_destroy(r->m); delete r; }
void REFNAME(mesh_set_solution)(void* h, const double* u) { hrn_mesh* m = ((RefMesh*)h)->m; memcpy(m->luh, u, nsol(m) * 8); }
void REFNAME(mesh_get_solution)(void* h, double* u) { hrn_mesh* m = ((RefMesh*)h)->m; memcpy(u, m->luh, nsol(m) * 8); }
void REFNAME(mesh_init)(void* h, double t0) { hrn_init(((RefMesh*)h)->m, t0); }
void REFNAME(mesh_init_fused)(void* h, double t0, double w) { hrn_init_fused(((RefMesh*)h)->m, t0, w); }
double REFNAME(mesh_predictor_dt)(void* h) { return ((RefMesh*)h)->m->pdt; }
long REFNAME(mesh_reruns)(void* h) { return ((RefMesh*)h)->m->reruns; }
void REFNAME(mesh_step)(void* h, int n) { hrn_step(((RefMesh*)h)->m, n); }
int REFNAME(mesh_run_until)(void* h, double t_end, int max_steps) { return hrn_run_until(((RefMesh*)h)->m, t_end, max_steps); }
double REFNAME(mesh_time)(void* h) { return ((RefMesh*)h)->m->t; }
double REFNAME(mesh_dt)(void* h) { return ((RefMesh*)h)->m->dt; }
long REFNAME(mesh_steps)(void* h) { return ((RefMesh*)h)->m->steps; }
long REFNAME(mesh_sweeps)(void* h) { return ((RefMesh*)h)->m->sweeps; }
}

namespace {
void lb_pfv(void* c, const double* u, double* l) { REFNAME(project_fv)(((Ctx*)c)->N, u, l); }
void lb_pdg(void* c, const double* l, double* u) { REFNAME(project_dg)(((Ctx*)c)->N, l, u); }
void lb_lmm(void* c, const double* l, double* a, double* b) { REFNAME(limiter_minmax)(((Ctx*)c)->N, l, a, b); }
void lb_smm(void* c, const double* u, double* a, double* b) { REFNAME(local_minmax)(((Ctx*)c)->N, u, a, b); }
int lb_dmp(void* c, const double* u, double r, double sc, double* a, double* b) { return REFNAME(dmp)(((Ctx*)c)->N, u, r, sc, a, b); }
int lb_adm(void* c, const double* m) { return !(m[0] <= 0.0) && !(m[4] <= 0.0); }
void lb_fvu(void* c, double* ln, const double* lo, const double* dx, double dt) { REFNAME(musclhancock)(((Ctx*)c)->N, ln, lo, dx, dt); }
void lb_fvg(void* c, double* l, const double* nb, int f) { REFNAME(fv_ghost)(((Ctx*)c)->N, l, nb, f); }
void lb_fvb(void* c, double* l, int f) { REFNAME(fv_boundary)(((Ctx*)c)->N, l, f); }
void lb_fvb_kind(void* c, double* l, int f, int kind) { REFNAME(fv_boundary_kind)(((Ctx*)c)->N, l, f, kind); }
struct RefLMesh { Ctx c; lhrn* r; };
}

extern "C" {
void* REFNAME(lmesh_create)(int order, const int* cells, const double* size, const int* bc, int nthreads,
                            int helper_layers, int cure_steps, double relax, double scale) {
  REFNAME(init)();
  RefLMesh* r = new RefLMesh();
  r->c.pde = 0;
  r->c.N = order;
  const int B = 2 * order + 1, E = B + 4;
  const int fv = (DIMENSIONS == 3 ? E * E * E : E * E) * 5;
  hrn_backend k = {&r->c, DIMENSIONS, order, 5, 5, be_pred, be_riem, be_bnd, be_surf, be_upd, be_dt};
  k.boundary_face_kind = be_bnd_kind;
  lhrn_backend L = {lb_pfv, lb_pdg, lb_lmm, lb_smm, lb_dmp, lb_adm, lb_fvu, lb_fvg, lb_fvb, fv};
  L.fv_boundary_kind = lb_fvb_kind;
  r->r = lhrn_create(&k, &L, cells, size, bc, nthreads, helper_layers, cure_steps, relax, scale);
  return r;
}
void REFNAME(lmesh_destroy)(void* h) { RefLMesh* r = (RefLMesh*)h; lhrn_destroy(r->r); delete r; }
void REFNAME(lmesh_set_solution)(void* h, const double* u) { hrn_mesh* m = ((RefLMesh*)h)->r->m; memcpy(m->luh, u, nsol(m) * 8); }
void REFNAME(lmesh_get_solution)(void* h, double* u) { hrn_mesh* m = ((RefLMesh*)h)->r->m; memcpy(u, m->luh, nsol(m) * 8); }
void REFNAME(lmesh_set_fv_initial)(void* h, const double* v) {
  lhrn* r = ((RefLMesh*)h)->r;
  const int B = 2 * r->m->k.order + 1, Bd = r->m->dim == 3 ? B * B * B : B * B;
  const size_t n = (size_t)r->m->ncells * Bd * 5;
  free(r->fv_ic);
  r->fv_ic = (double*)malloc(sizeof(double) * n);
  memcpy(r->fv_ic, v, sizeof(double) * n);
}
void REFNAME(lmesh_init)(void* h, double t0) { lhrn_init(((RefLMesh*)h)->r, t0); }
void REFNAME(lmesh_step)(void* h, int n) { for (int i = 0; i < n; i++) lhrn_step(((RefLMesh*)h)->r); }
int REFNAME(lmesh_run_until)(void* h, double t_end, int max_steps) { return lhrn_run_until(((RefLMesh*)h)->r, t_end, max_steps); }
double REFNAME(lmesh_time)(void* h) { return ((RefLMesh*)h)->r->m->t; }
double REFNAME(lmesh_dt)(void* h) { return ((RefLMesh*)h)->r->m->dt; }
long REFNAME(lmesh_steps)(void* h) { return ((RefLMesh*)h)->r->m->steps; }
long REFNAME(lmesh_sweeps)(void* h) { return ((RefLMesh*)h)->r->m->sweeps; }
void REFNAME(lmesh_status)(void* h, int* s) { lhrn* r = ((RefLMesh*)h)->r; memcpy(s, r->s, sizeof(int) * r->m->ncells); }
long REFNAME(lmesh_irregular_steps)(void* h) { return ((RefLMesh*)h)->r->irregular_steps; }
void REFNAME(lmesh_limiter)(void* h, double* lim, int* allocated) {
  lhrn* r = ((RefLMesh*)h)->r;
  if (lim) memcpy(lim, r->lim, sizeof(double) * (size_t)r->m->ncells * r->L.fv_size);
  if (allocated) memcpy(allocated, r->has_lim, sizeof(int) * r->m->ncells);
}
}
