// Linear ADER-DG kernels for PDEs given by a non-conservative product
// (PDE::kLinear, e.g. ElasticPDE):
//   ck_predictor_kernel    spaceTimePredictorLinear (2d/spaceTimePredictorLinear.cpph:35-409,
//                          3d/spaceTimePredictorLinear.cpph:34-446) + volumeIntegralLinear
//                          (3d/volumeIntegralLinear.cpph:20-52); for a PDE with a point
//                          source also pointSource (3d/pointSource.cpph:28-143)
//   riemann_linear_kernel  riemannSolverLinear (3d/riemannSolverLinear.cpph:20-136)
//   boundary_linear_kernel boundaryConditions + riemannSolverLinear on boundary faces
//   volume_linear_kernel   volumeIntegralLinear on its own (kernel-level entry point)
// The surface integral is the corrector's linear form (aderdg.cuh).
//
// The predictor is the Cauchy-Kovalevski procedure: time derivative i+1 of
// the solution is -sum_d B_d(Q_i) grad_d Q_i, evaluated b times; the time
// averages over [0, dt] weight derivative i by dt^i / (i+1)!. Per derivative
// level the cell's state sits in shared memory; the gradients are 1-D line
// contractions with dudx (one thread per (direction, line, variable)), the
// non-conservative product and both time averages are per node (one thread
// per node, accumulators in registers). No iteration and no convergence test.
#pragma once
#include "aderdg.cuh"

namespace exa {

// Order of the gradient items, from a shared-memory bank model (64-bit
// accesses, 16 bank pairs per half-warp) of the gradient phase's strided line
// accesses: for 3D with 6 or 5 nodes per axis consecutive threads take
// consecutive lines of one component, elsewhere consecutive components of
// one line. Odd node strides keep the per-node phase conflict-free.
constexpr bool ck_line_major(int dim, int b) { return dim == 3 ? b >= 5 : (b == 6 || b == 4); }

// the (direction, variable) gradient components the PDE's ncp reads
template <class PDE, int DIM>
struct GradPairs {
  int d[DIM * PDE::nVar], v[DIM * PDE::nVar], n;
  constexpr GradPairs() : d(), v(), n(0) {
    for (int dd = 0; dd < DIM; dd++)
      for (int vv = 0; vv < PDE::nVar; vv++)
        if (PDE::ncp_uses(dd, vv)) {
          d[n] = dd;
          v[n] = vv;
          n++;
        }
  }
};

template <int DIM, int N, class PDE>
struct CKCfg : Shape<DIM, N, PDE> {
  using S = Shape<DIM, N, PDE>;
  static constexpr int CPB = cells_per_block<S::P>();
  static constexpr int THREADS = CPB * S::P;
  static constexpr int LINES = S::P / S::b;          // lines per direction
  static constexpr int QS = S::nD | 1;          // node stride of the state
  static constexpr int GS = (DIM * S::nV) | 1;  // node stride of the gradients [d][nV]
  static constexpr bool LMAJ = ck_line_major(DIM, S::b);
  static constexpr int SQ = S::P * QS, SG = S::P * GS;
  static constexpr size_t SMEM = sizeof(double) * (size_t)CPB * (SQ + SG);
  static constexpr int NPAIRS = GradPairs<PDE, DIM>().n;
  static constexpr int GITEMS = CPB * NPAIRS * LINES;  // gradient line items per block
  static constexpr int IPT = (GITEMS + THREADS - 1) / THREADS;
  static_assert(S::P < 1024 && S::nV <= 16 && CPB <= 16, "packed item descriptors");
};

// node of line L along direction d at position n; L enumerates the other
// coordinates in (z, y, x) order (face-node order of the reference)
template <int DIM, int b>
__device__ __forceinline__ int line_node(int d, int L, int n) {
  const int a0 = L / b, a1 = L % b;
  if (DIM == 2) return d == 0 ? L * b + n : n * b + L;
  return d == 0 ? (a0 * b + a1) * b + n : d == 1 ? (a0 * b + n) * b + a1 : (n * b + a0) * b + a1;
}

// Lagrange basis polynomial i of the Gauss-Legendre nodes of order N at xi
// (the reference's basisFunctions[N][i], kernels/DGBasisFunctions.h:53), as
// the product over the other nodes
template <int N>
__device__ double lagrange_at(int i, double xi) {
  const OrderTables& T = c_tab[N];
  double r = 1.0;
#pragma unroll
  for (int m = 0; m < N + 1; m++)
    if (m != i) r = __dmul_rn(r, __ddiv_rn(__dsub_rn(xi, T.x[m]), __dsub_rn(T.x[i], T.x[m])));
  return r;
}

// Whether the point source of PDE::sourcePosition lies in the closed cell of
// centre c and widths h, tested on the reference coordinates as pointSource
// tests them
template <int DIM, class PDE>
__device__ bool point_source_in_cell(const Geometry& geo, const double* c, const double* h) {
  double x0[3];
  PDE::sourcePosition(geo.ps, x0);
  bool in = true;
#pragma unroll
  for (int e = 0; e < DIM; e++) {
    const double xr = __ddiv_rn(__dsub_rn(x0[e], __dsub_rn(c[e], __ddiv_rn(h[e], 2.0))), h[e]);
    in = in && xr >= 0.0 && xr <= 1.0;
  }
  return in;
}

// pointSource (2d/pointSource.cpph:30-127, 3d/pointSource.cpph:28-143) at
// node p of the cell of centre c and widths h, time slot n (0: t; n >= 1:
// Gauss-Legendre time node n - 1 of [t, t + dt]): the PDE's source at the
// node's position, projected onto the node's basis function at the source's
// reference coordinates and divided by the node's quadrature weight and the
// cell's widths; zero where the source lies outside the closed cell. The
// reference's operations in its order, rounded one by one.
template <int DIM, int N, class PDE>
__device__ void node_point_source(const Geometry& geo, const double* c, const double* h, int p, double t, double dt,
                                  int n, double* out) {
  constexpr int b = N + 1;
  const OrderTables& T = c_tab[N];
  const int ix = p % b, iy = (p / b) % b, iz = DIM == 3 ? p / (b * b) : 0;
  const double tn = n == 0 ? t : __dadd_rn(__dmul_rn(dt, T.x[n - 1]), t);
  double x[3] = {0.0, 0.0, 0.0}, x0[3];
  x[0] = __dadd_rn(c[0], __dmul_rn(h[0], __dsub_rn(T.x[ix], 0.5)));
  x[1] = __dadd_rn(c[1], __dmul_rn(h[1], __dsub_rn(T.x[iy], 0.5)));
  if (DIM == 3) x[2] = __dadd_rn(c[2], __dmul_rn(h[2], __dsub_rn(T.x[iz], 0.5)));
  PDE::pointSource(x, tn, dt, out, x0, geo.ps);
  double xr[3] = {0.0, 0.0, 0.0};
  bool in = true;
#pragma unroll
  for (int e = 0; e < DIM; e++) {
    xr[e] = __ddiv_rn(__dsub_rn(x0[e], __dsub_rn(c[e], __ddiv_rn(h[e], 2.0))), h[e]);
    in = in && xr[e] >= 0.0 && xr[e] <= 1.0;
  }
  double phi, den;
  if (DIM == 3) {
    phi = __dmul_rn(__dmul_rn(lagrange_at<N>(iz, xr[2]), lagrange_at<N>(iy, xr[1])), lagrange_at<N>(ix, xr[0]));
    den = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(T.w[iz], h[2]), T.w[iy]), h[1]), T.w[ix]), h[0]);
  } else {
    phi = __dmul_rn(lagrange_at<N>(iy, xr[1]), lagrange_at<N>(ix, xr[0]));
    den = __dmul_rn(__dmul_rn(__dmul_rn(T.w[iy], h[1]), T.w[ix]), h[0]);
  }
#pragma unroll
  for (int v = 0; v < PDE::nVar; v++) out[v] = in ? __ddiv_rn(__dmul_rn(phi, out[v]), den) : 0.0;
}

// sum over the time slots n = 1..b of w[n-1] * pointSource (the time
// integral the predictor adds, 3d/spaceTimePredictorLinear.cpph:77-90 and
// :294-308)
template <int DIM, int N, class PDE>
__device__ void node_point_source_sum(const Geometry& geo, const double* c, const double* h, int p, double t,
                                      double dt, double* sum) {
  const OrderTables& T = c_tab[N];
#pragma unroll
  for (int v = 0; v < PDE::nVar; v++) sum[v] = 0.0;
  for (int n = 1; n < N + 2; n++) {
    double val[PDE::nVar];
    node_point_source<DIM, N, PDE>(geo, c, h, p, t, dt, n, val);
#pragma unroll
    for (int v = 0; v < PDE::nVar; v++) sum[v] = __dadd_rn(sum[v], __dmul_rn(T.w[n - 1], val[v]));
  }
}

// NREG: register cap per thread, regs_for_blocks<THREADS, blocks per SM>()
template <int DIM, int N, class PDE, int NREG>
__global__ void __launch_bounds__(CKCfg<DIM, N, PDE>::THREADS) __maxnreg__(NREG)
    ck_predictor_kernel(const double* __restrict__ luh, double* __restrict__ lQhbnd, double* __restrict__ lFhbnd,
                        double* __restrict__ lduh, const double* __restrict__ dt_ptr, Geometry geo, int ncells,
                        const int* __restrict__ cell_list, const int* __restrict__ count,
                        double* __restrict__ lQhi_out, double* __restrict__ lFhi_out) {
  using C = CKCfg<DIM, N, PDE>;
  constexpr int b = C::b, P = C::P, nV = C::nV, nD = C::nD, LINES = C::LINES, QS = C::QS, GS = C::GS;
  constexpr int F = C::F;
  extern __shared__ double smem[];
  const OrderTables& T = c_tab[N];
  const int lc = threadIdx.x / P;
  const int p = threadIdx.x - lc * P;
  const int slot = blockIdx.x * C::CPB + lc;
  const int nact = count ? min(*count, ncells) : ncells;
  if ((int)blockIdx.x * C::CPB >= nact) return;  // whole block, before its first barrier
  const bool active = slot < nact;
  const int cell = active ? (cell_list ? cell_list[slot] : slot) : 0;
  double* sQ = smem + lc * C::SQ;
  double* sG = smem + C::CPB * C::SQ + lc * C::SG;
  const int inst = cell_instance(geo, cell);
  const double dt = dt_ptr[inst];
  __shared__ double s_idx[C::CPB][3];
  __shared__ int s_cell[C::CPB];
  if (p == 0) {
    s_cell[lc] = active ? cell : -1;
#pragma unroll
    for (int d = 0; d < 3; d++) s_idx[lc][d] = d < DIM ? 1.0 / cell_width(geo, inst, d) : 0.0;
  }
  // point sources: this cell's centre, widths and time stamp, and whether
  // the source lies in it (the same for all threads of the cell)
  constexpr bool PS = PDE::kPointSource;
  double pc[3] = {0.0, 0.0, 0.0}, ph[3] = {1.0, 1.0, 1.0}, pt = 0.0;
  bool src = false;
  if constexpr (PS) {
    if (active && geo.centre) {
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        pc[d] = geo.centre[3 * (size_t)cell + d];
        ph[d] = cell_width(geo, inst, d);
      }
      pt = *geo.time;
      src = point_source_in_cell<DIM, PDE>(geo, pc, ph);
    }
  }
  // level 0: the solution (parameters included); inactive slots get unit
  // parameters so that their arithmetic stays finite. A point source adds dt
  // times its time integral (3d/spaceTimePredictorLinear.cpph:77-90).
  double qh[nV];
  {
    double psw[nV];
#pragma unroll
    for (int v = 0; v < nV; v++) psw[v] = 0.0;
    if constexpr (PS)
      if (src) node_point_source_sum<DIM, N, PDE>(geo, pc, ph, p, pt, dt, psw);
#pragma unroll
    for (int v = 0; v < nD; v++) {
      double q = active ? __ldg(luh + ((size_t)cell * P + p) * nD + v) : (v < nV ? 0.0 : 1.0);
      if (v < nV && PS && src) q = __dadd_rn(q, __dmul_rn(dt, psw[v]));
      sQ[p * QS + v] = q;
      if (v < nV) qh[v] = q;
    }
  }
  double fh[DIM][nV];
  double fac_i = 0.0, fac_n = 0.5 * dt;  // weights of levels i and i+1 in the time averages
  // the block's gradient items, packed once: first node of the line (10
  // bits), direction (2), variable (4), cell of the block (4); item k of
  // thread t is s_desc[k][t], -1: none
  __shared__ int s_desc[C::IPT][C::THREADS];
  // the (direction, variable) pairs, copied with compile-time indices (a
  // runtime index into the constexpr table would build a copy of it in every
  // thread's local memory)
  __shared__ int s_pair[C::NPAIRS];
  if (threadIdx.x == 0) {
    constexpr GradPairs<PDE, DIM> GP;
#pragma unroll
    for (int i = 0; i < C::NPAIRS; i++) s_pair[i] = GP.d[i] | GP.v[i] << 4;
  }
  __syncthreads();
  for (int k = 0; k < C::IPT; k++) {
    const int it = threadIdx.x + k * C::THREADS;
    int dsc = -1;
    if (it < C::GITEMS) {
      const int L = C::LMAJ ? it % LINES : (it / C::NPAIRS) % LINES;
      const int pr = C::LMAJ ? (it / LINES) % C::NPAIRS : it % C::NPAIRS;
      const int c = it / (C::NPAIRS * LINES);
      const int d = s_pair[pr] & 15, v = s_pair[pr] >> 4;
      dsc = line_node<DIM, b>(d, L, 0) | d << 10 | v << 12 | c << 16;
    }
    s_desc[k][threadIdx.x] = dsc;
  }
  for (int i = 0; i < b; i++) {
    __syncthreads();  // level i complete in sQ; previous per-node phase done with sG
    // spatial gradients of level i, one line per item, into sG[node][d][v]
    // (the components ncp reads)
#pragma unroll 1
    for (int k = 0; k < C::IPT; k++) {
      const int dsc = s_desc[k][threadIdx.x];
      if (dsc < 0) continue;
      const int node0 = dsc & 1023, d = (dsc >> 10) & 3, v = (dsc >> 12) & 15, c = dsc >> 16;
      if (s_cell[c] < 0) continue;
      const int step = d == 0 ? 1 : d == 1 ? b : b * b;  // node stride along the line
      const double* q = smem + c * C::SQ + node0 * QS + v;
      double* g = smem + C::CPB * C::SQ + c * C::SG + node0 * GS + d * nV + v;
      const double idx = s_idx[c][d];
      double f[b];
#pragma unroll
      for (int n = 0; n < b; n++) f[n] = idx * q[n * step * QS];
#pragma unroll
      for (int l = 0; l < b; l++) {
        double s = 0.0;
#pragma unroll
        for (int n = 0; n < b; n++) s = fma(f[n], T.dudx[l * b + n], s);
        g[l * step * GS] = s;
      }
    }
    __syncthreads();
    // per node: non-conservative product one direction at a time (few
    // registers live), time averages, next level
    {
      // level 1 starts from the point source's value at t (:93-101)
      double qn[nV];
#pragma unroll
      for (int v = 0; v < nV; v++) qn[v] = 0.0;
      if constexpr (PS)
        if (src && i == 0) node_point_source<DIM, N, PDE>(geo, pc, ph, p, pt, dt, 0, qn);
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        double B[nV];
        PDE::ncp_dir(sQ + p * QS, d, sG + p * GS + d * nV, B);
#pragma unroll
        for (int v = 0; v < nV; v++) {
          fh[d][v] = i == 0 ? B[v] : fma(fac_i, B[v], fh[d][v]);
          qn[v] -= B[v];
        }
      }
      if (i + 1 < b) {
#pragma unroll
        for (int v = 0; v < nV; v++) {
          qh[v] = fma(fac_n, qn[v], qh[v]);
          sQ[p * QS + v] = qn[v];  // own node only; parameters stay
        }
      }
      fac_i = fac_n;
      fac_n = fac_n * (dt / (i + 3));
    }
  }
  if constexpr (PS) {
    if (src) {  // the time integral of the source, split over the directions (:294-308)
      double psw[nV];
      node_point_source_sum<DIM, N, PDE>(geo, pc, ph, p, pt, dt, psw);
#pragma unroll
      for (int d = 0; d < DIM; d++)
#pragma unroll
        for (int v = 0; v < nV; v++) fh[d][v] = __dadd_rn(fh[d][v], __ddiv_rn(psw[v], (double)DIM));
    }
  }
  __syncthreads();
  // stage the time averages for the extrapolation: lQhi in sQ, lFhi in sG
#pragma unroll
  for (int v = 0; v < nV; v++) sQ[p * QS + v] = qh[v];
#pragma unroll
  for (int d = 0; d < DIM; d++)
#pragma unroll
    for (int v = 0; v < nV; v++) sG[p * GS + d * nV + v] = fh[d][v];
  if (active) {
    if (lQhi_out)
      for (int v = 0; v < nD; v++) lQhi_out[((size_t)cell * P + p) * nD + v] = sQ[p * QS + v];
    if (lFhi_out)  // from the staged copy: indexing fh here would put it in local memory
      for (int d = 0; d < DIM; d++)
        for (int v = 0; v < nV; v++) lFhi_out[(((size_t)cell * DIM + d) * P + p) * nV + v] = sG[p * GS + d * nV + v];
  }
  __syncthreads();
  // boundary extrapolation: states (parameters included) and normal fluxes
  constexpr int QITEMS = C::CPB * DIM * LINES * nD;
  for (int it = threadIdx.x; it < QITEMS; it += C::THREADS) {
    const int v = it % nD;
    const int L = (it / nD) % LINES;
    const int d = (it / (nD * LINES)) % DIM;
    const int c = it / (nD * LINES * DIM);
    const int cc = s_cell[c];
    if (cc < 0) continue;
    const double* q = smem + c * C::SQ;
    double sl = 0.0, sr = 0.0;
#pragma unroll
    for (int l = 0; l < b; l++) {
      const double x = q[line_node<DIM, b>(d, L, l) * QS + v];
      sl += x * T.FL[l];
      sr += x * T.FR[l];
    }
    lQhbnd[(((size_t)cc * 2 * DIM + 2 * d) * F + L) * nD + v] = sl;
    lQhbnd[(((size_t)cc * 2 * DIM + 2 * d + 1) * F + L) * nD + v] = sr;
  }
  constexpr int FITEMS = C::CPB * DIM * LINES * nV;
  for (int it = threadIdx.x; it < FITEMS; it += C::THREADS) {
    const int v = it % nV;
    const int L = (it / nV) % LINES;
    const int d = (it / (nV * LINES)) % DIM;
    const int c = it / (nV * LINES * DIM);
    const int cc = s_cell[c];
    if (cc < 0) continue;
    const double* g = smem + C::CPB * C::SQ + c * C::SG;
    double sl = 0.0, sr = 0.0;
#pragma unroll
    for (int l = 0; l < b; l++) {
      const double x = g[line_node<DIM, b>(d, L, l) * GS + d * nV + v];
      sl += x * T.FL[l];
      sr += x * T.FR[l];
    }
    lFhbnd[(((size_t)cc * 2 * DIM + 2 * d) * F + L) * nV + v] = sl;
    lFhbnd[(((size_t)cc * 2 * DIM + 2 * d + 1) * F + L) * nV + v] = sr;
  }
  if (!lduh) return;
  // volumeIntegralLinear from the staged lFhi, staged in turn in the cell's
  // state buffer and written by consecutive threads to consecutive addresses
  // (a thread's own nV values would leave every store instruction a partial
  // write of 32 sectors)
  __syncthreads();
  if (active) {
    const int x = p % b, y = (p / b) % b, z = DIM == 3 ? p / (b * b) : 0;
    const double w = (DIM == 3 ? T.w[z] * T.w[y] : T.w[y]) * T.w[x];
#pragma unroll
    for (int v = 0; v < nV; v++) {
      double du = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; d++) du -= w * sG[p * GS + d * nV + v];
      sQ[p * nV + v] = du;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < C::CPB * P * nV; i += C::THREADS) {
    const int c = i / (P * nV), e = i - c * (P * nV);
    const int cc = s_cell[c];
    if (cc >= 0) lduh[(size_t)cc * P * nV + e] = smem[c * C::SQ + e];
  }
}

// The linear Riemann solve of one face by one warp: face averages of both
// sides (parameters included), smax from both averages' eigenvalues, Bn from
// the PDE's coefficient_matrix in their mean (shared memory, sBw), then per
// face node FL = (Bn - smax I)^T dQ and FR = (Bn + smax I)^T dQ with
// dQ = (QR - QL) / 2 (staged in sDQw). FL or FR may be NULL (not written).
template <int DIM, int N, class PDE>
__device__ __forceinline__ void linear_face_flux(const double* QL, const double* QR, double* FL, double* FR, int dir,
                                                 int lane, double* sBw, double* sDQw) {
  using S = Shape<DIM, N, PDE>;
  constexpr int F = S::F, nV = S::nV, nD = S::nD;
  // this lane's state differences are loaded before the face averages, so
  // that all of the face's loads are in flight together
  constexpr int E = F * nV, EPL = (E + 31) / 32;
  double dq[EPL];
#pragma unroll
  for (int i = 0; i < EPL; i++) {
    const int e = lane + 32 * i, fn = e / nV, k = e - fn * nV;
    dq[i] = e < E ? 0.5 * (QR[fn * nD + k] - QL[fn * nD + k]) : 0.0;
  }
  double aL[nD], aR[nD];
  face_average<DIM, N, PDE>(QL, lane, aL);
  face_average<DIM, N, PDE>(QR, lane, aR);
  const double smax = face_smax<DIM, PDE>(aL, aR, dir);
  if (lane == 0) {
    double av[nD];
#pragma unroll
    for (int k = 0; k < nD; k++) av[k] = 0.5 * (aL[k] + aR[k]);
    PDE::coefficient_matrix(av, dir, sBw);
  }
#pragma unroll
  for (int i = 0; i < EPL; i++) {
    const int e = lane + 32 * i;
    if (e < E) sDQw[e] = dq[i];
  }
  __syncwarp();
  for (int e = lane; e < F * nV; e += 32) {
    const int fn = e / nV, j = e - fn * nV;
    const double* d = sDQw + fn * nV;
    double fl = 0.0, fr = 0.0;
#pragma unroll
    for (int k = 0; k < nV; k++) {
      const double bkj = sBw[k * nV + j];
      fl = fma(k == j ? bkj - smax : bkj, d[k], fl);
      fr = fma(k == j ? bkj + smax : bkj, d[k], fr);
    }
    if (FL) FL[e] = fl;
    if (FR) FR[e] = fr;
  }
}

// riemannSolverLinear on interior faces, one warp per face. FL goes to the
// left cell's face 2 dir + 1, FR to the right cell's face 2 dir; the
// extrapolated fluxes there are not read.
template <int DIM, int N, class PDE>
__global__ void __launch_bounds__(128) riemann_linear_kernel(const double* __restrict__ lQhbnd,
                                                             double* __restrict__ lFhbnd,
                                                             const int* __restrict__ face_left,
                                                             const int* __restrict__ face_right,
                                                             const int* __restrict__ face_dir, int nfaces,
                                                             const int* __restrict__ gate = nullptr) {
  using S = Shape<DIM, N, PDE>;
  constexpr int F = S::F, nV = S::nV, nD = S::nD;
  __shared__ double sB[4][nV * nV];
  __shared__ double sDQ[4][F * nV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int f = blockIdx.x * (blockDim.x >> 5) + w;
  if (gate && !*gate) return;
  if (f >= nfaces) return;
  const int cl = face_left[f], cr = face_right[f], dir = face_dir[f];
  const double* QL = lQhbnd + ((size_t)cl * 2 * DIM + 2 * dir + 1) * F * nD;
  const double* QR = lQhbnd + ((size_t)cr * 2 * DIM + 2 * dir) * F * nD;
  double* FL = lFhbnd + ((size_t)cl * 2 * DIM + 2 * dir + 1) * F * nV;
  double* FR = lFhbnd + ((size_t)cr * 2 * DIM + 2 * dir) * F * nV;
  linear_face_flux<DIM, N, PDE>(QL, QR, FL, FR, dir, lane, sB[w], sDQ[w]);
}

// Boundary faces of a linear solver: ADERDGSolver::applyBoundaryConditions
// (exahype/solvers/ADERDGSolver.cpp:2893-2962) -- the PDE's boundaryValues
// at every face node (boundaryConditions, 3d/boundaryConditions.cpph:24-85),
// staged in shared memory, then riemannSolverLinear with the outside state on
// the outer side (QOut, QIn for an even face, QIn, QOut for an odd one); only
// the cell's own fluctuation is written. One warp per boundary face.
template <int DIM, int N, class PDE>
__global__ void __launch_bounds__(128) boundary_linear_kernel(const double* __restrict__ lQhbnd,
                                                              double* __restrict__ lFhbnd,
                                                              const int* __restrict__ bcell,
                                                              const int* __restrict__ bface, int nb, int kind,
                                                              const int* __restrict__ gate = nullptr) {
  using S = Shape<DIM, N, PDE>;
  constexpr int F = S::F, nV = S::nV, nD = S::nD;
  __shared__ double sB[4][nV * nV];
  __shared__ double sDQ[4][F * nV];
  __shared__ double sQO[4][F * nD];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int f = blockIdx.x * (blockDim.x >> 5) + w;
  if (f >= nb || (gate && !*gate)) return;
  const int c = bcell[f], face = bface[f], dir = face >> 1;
  const double* QIn = lQhbnd + ((size_t)c * 2 * DIM + face) * F * nD;
  double* FIn = lFhbnd + ((size_t)c * 2 * DIM + face) * F * nV;
  for (int fn = lane; fn < F; fn += 32) {
    double fo[nV];
    PDE::template boundaryValues<DIM>(kind, dir, FIn + fn * nV, QIn + fn * nD, fo, sQO[w] + fn * nD);
  }
  __syncwarp();
  if ((face & 1) == 0)
    linear_face_flux<DIM, N, PDE>(sQO[w], QIn, nullptr, FIn, dir, lane, sB[w], sDQ[w]);
  else
    linear_face_flux<DIM, N, PDE>(QIn, sQO[w], FIn, nullptr, dir, lane, sB[w], sDQ[w]);
}

// volumeIntegralLinear alone: lduh = -w_node sum_d lFhi[d], lFhi per cell [d][b^d][nV]
template <int DIM, int N, class PDE>
__global__ void volume_linear_kernel(double* __restrict__ lduh, const double* __restrict__ lFhi, int ncells) {
  using S = Shape<DIM, N, PDE>;
  constexpr int b = S::b, P = S::P, nV = S::nV;
  const OrderTables& T = c_tab[N];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)ncells * P) return;
  const int cell = (int)(i / P), p = (int)(i - (long long)cell * P);
  const int x = p % b, y = (p / b) % b, z = DIM == 3 ? p / (b * b) : 0;
  const double w = (DIM == 3 ? T.w[z] * T.w[y] : T.w[y]) * T.w[x];
#pragma unroll
  for (int v = 0; v < nV; v++) {
    double du = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) du -= w * lFhi[(((size_t)cell * DIM + d) * P + p) * nV + v];
    lduh[((size_t)cell * P + p) * nV + v] = du;
  }
}

}  // namespace exa
