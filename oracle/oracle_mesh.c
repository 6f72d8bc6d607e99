/* ORACLE -- test infrastructure only: the uniform-mesh harness (harness.c)
 * over the C restatement of the kernels (oracle.c). */
#include "oracle.h"
#include "harness.c"

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
static void be_surf(void* c, double* du, const double* fb, const double* dx) { orc_surface_integral((const orc_solver*)c, du, fb, dx); }
static void be_upd(void* c, double* u, const double* du, double dt) { orc_solution_update((const orc_solver*)c, u, du, dt); }
static double be_dt(void* c, const double* u, const double* dx) { return orc_stable_dt((const orc_solver*)c, u, dx); }

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
  om->m = hrn_create(&k, cells, size, bc, nthreads);
  return om;
}
void orc_mesh_destroy(void* h) { orc_mesh* om = (orc_mesh*)h; hrn_destroy(om->m); free(om); }
static size_t nsol(hrn_mesh* m) { return (size_t)m->ncells * m->P * m->k.ndata; }
void orc_mesh_set_solution(void* h, const double* u) { hrn_mesh* m = ((orc_mesh*)h)->m; memcpy(m->luh, u, nsol(m) * 8); }
void orc_mesh_get_solution(void* h, double* u) { hrn_mesh* m = ((orc_mesh*)h)->m; memcpy(u, m->luh, nsol(m) * 8); }
void orc_mesh_init(void* h, double t0) { hrn_init(((orc_mesh*)h)->m, t0); }
void orc_mesh_step(void* h, int n) { hrn_step(((orc_mesh*)h)->m, n); }
int orc_mesh_run_until(void* h, double t_end, int max_steps) { return hrn_run_until(((orc_mesh*)h)->m, t_end, max_steps); }
double orc_mesh_time(void* h) { return ((orc_mesh*)h)->m->t; }
double orc_mesh_dt(void* h) { return ((orc_mesh*)h)->m->dt; }
long orc_mesh_steps(void* h) { return ((orc_mesh*)h)->m->steps; }
long orc_mesh_sweeps(void* h) { return ((orc_mesh*)h)->m->sweeps; }
