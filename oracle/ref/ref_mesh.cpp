// Oracle-only: the uniform-mesh harness (oracle/harness.c) driving the
// reference's own kernels (ref_kernels.cpp). This is the CPU baseline path:
// the reference's generic kernels, parallel across cells on POSIX threads.
#include <cstdio>
#include <cstdlib>
#include <cstring>

extern "C" {
#include "../harness.c"
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
void REFNAME(init)();
}

namespace {
struct Ctx { int pde, N; };
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
void be_surf(void* c, double* du, const double* fb, const double* dx) { Ctx* x = (Ctx*)c; REFNAME(surface_integral)(x->pde, x->N, du, fb, dx); }
void be_upd(void* c, double* u, const double* du, double dt) { Ctx* x = (Ctx*)c; REFNAME(solution_update)(x->pde, x->N, u, du, dt); }
double be_dt(void* c, const double* u, const double* dx) { Ctx* x = (Ctx*)c; return REFNAME(stable_dt)(x->pde, x->N, u, dx); }
struct RefMesh { Ctx c; hrn_mesh* m; };
size_t nsol(hrn_mesh* m) { return (size_t)m->ncells * m->P * m->k.ndata; }
}

extern "C" {
void* REFNAME(mesh_create)(int order, int pde, const int* cells, const double* size, const int* bc, int nthreads) {
  REFNAME(init)();
  RefMesh* r = new RefMesh();
  r->c.pde = pde;
  r->c.N = order;
  hrn_backend k = {&r->c, DIMENSIONS, order, 5, 5 + (pde == 1 ? 1 : 0), be_pred, be_riem, be_bnd, be_surf, be_upd, be_dt};
  r->m = hrn_create(&k, cells, size, bc, nthreads);
  return r;
}
void REFNAME(mesh_destroy)(void* h) { RefMesh* r = (RefMesh*)h; hrn_destroy(r->m); delete r; }
void REFNAME(mesh_set_solution)(void* h, const double* u) { hrn_mesh* m = ((RefMesh*)h)->m; memcpy(m->luh, u, nsol(m) * 8); }
void REFNAME(mesh_get_solution)(void* h, double* u) { hrn_mesh* m = ((RefMesh*)h)->m; memcpy(u, m->luh, nsol(m) * 8); }
void REFNAME(mesh_init)(void* h, double t0) { hrn_init(((RefMesh*)h)->m, t0); }
void REFNAME(mesh_step)(void* h, int n) { hrn_step(((RefMesh*)h)->m, n); }
int REFNAME(mesh_run_until)(void* h, double t_end, int max_steps) { return hrn_run_until(((RefMesh*)h)->m, t_end, max_steps); }
double REFNAME(mesh_time)(void* h) { return ((RefMesh*)h)->m->t; }
double REFNAME(mesh_dt)(void* h) { return ((RefMesh*)h)->m->dt; }
long REFNAME(mesh_steps)(void* h) { return ((RefMesh*)h)->m->steps; }
long REFNAME(mesh_sweeps)(void* h) { return ((RefMesh*)h)->m->sweeps; }
}
