// ADER-DG cell and face kernels (FP64), one template per (DIM, N, PDE).
//
// Layouts in HBM are the reference's per-cell layouts (kernels/KernelUtils.h
// idx helpers, last index fastest), cells stored back to back:
//   luh    [cell][z][y][x][nD]          lduh   [cell][z][y][x][nV]
//   lQhbnd [cell][2*DIM][face node][nD] lFhbnd [cell][2*DIM][face node][nV]
// Face order 0:-x 1:+x 2:-y 3:+y 4:-z 5:+z; face nodes run over the two other
// coordinates in (z,y,x) order (kernels/aderdg/generic/Kernels.h:69-74).
#pragma once
#include "common.cuh"
#include "pde.cuh"

namespace exa {

template <int DIM, int N, class PDE>
struct Shape {
  static constexpr int b = N + 1;
  static constexpr int P = ipow(b, DIM);      // nodes per cell
  static constexpr int F = ipow(b, DIM - 1);  // nodes per face
  static constexpr int nV = PDE::nVar;
  static constexpr int nP = PDE::nPar;
  static constexpr int nD = nV + nP;
  static constexpr int maxIter = 2 * (N + 1);  // spaceTimePredictorNonlinear.cpph:85
};

// Cells per block for the one-thread-per-node cell kernels.
template <int P>
constexpr int cells_per_block() { return P >= 256 ? 1 : 256 / P; }
constexpr int pow2ceil(int v) { return v <= 1 ? 1 : 2 * pow2ceil((v + 1) / 2); }

// Cell widths of one mesh, or of a batch of independent instances: with
// inst != NULL cell c belongs to instance inst[c], whose widths are
// inst_dx[3 inst + d] and whose step size is dt[inst[c]] (the kernels' dt
// pointer then points at the per-instance array).
struct Geometry {
  double dx[3];
  const int* inst;
  const double* inst_dx;
  // point sources (PDE::kPointSource): cell centres [cell][3], the time
  // stamp of the solution the predictor starts from (one for all cells), the
  // source's parameters; no centres: no source
  const double* centre;
  const double* time;
  double ps[6];
};
__device__ __forceinline__ int cell_instance(const Geometry& g, int cell) { return g.inst ? g.inst[cell] : 0; }
__device__ __forceinline__ double cell_width(const Geometry& g, int inst, int d) {
  return g.inst ? g.inst_dx[3 * inst + d] : g.dx[d];
}

// ---------------------------------------------------------------------------
// Space-time predictor: the discrete Picard iteration of
// aderPicardLoopNonlinear (3d/spaceTimePredictorNonlinear.cpph:42-329) with
// the time averaging (:337-409), the boundary extrapolation (:411-528) and
// volumeIntegralNonlinear (3d/volumeIntegralNonlinear.cpph:135-225) fused into
// one kernel.
//
// Work split: VSPLIT threads own one spatial node of one cell, each a slice of
// the nV conserved variables. Per Picard sweep the time slices are processed
// one at a time: the slice's fluxes go to shared memory, every thread forms
// its (node, variables) rhs from the three derivative contractions and folds
// it into its registers through iK1. Resident in shared memory per cell: the
// space-time iterate lQi [P][b][nD] and one flux slice [DIM][P][nV].
// MINB is the number of blocks per SM the register budget is sized for.
template <int DIM, int N, class PDE, int VSPLIT = 1, int MINB = 1>
struct PredictorCfg : Shape<DIM, N, PDE> {
  using S = Shape<DIM, N, PDE>;
  static constexpr int CPB = cells_per_block<S::P>();
  static constexpr int TPC = CPB * S::P;                     // threads per variable slice
  static constexpr int THREADS = VSPLIT * TPC;
  static constexpr int MIN_BLOCKS = MINB;
  static constexpr int NVT = (S::nV + VSPLIT - 1) / VSPLIT;  // variables per thread
  static constexpr int SF = DIM * S::P * S::nV;             // one flux slice per cell
  static constexpr int SR = VSPLIT * S::P + 1;              // residual partials + the cell's sum
  static constexpr int SK = S::b * S::b;                    // Kxi copy (per block)
  // lQi node stride: odd (no bank conflicts across nodes) when that still fits
  static constexpr int QS = sizeof(double) * (CPB * (S::P * (S::b * S::nD + 1) + SF + SR) + SK) <= 227 * 1024
                                ? S::b * S::nD + 1 : S::b * S::nD;
  static constexpr int SQ = S::P * QS;                      // lQi per cell
  static constexpr size_t SMEM = sizeof(double) * (size_t)(CPB * (SQ + SF + SR) + SK);
};

struct PredictorTemps {  // optional reference-layout temporaries (golden replay)
  double *lQi, *lFi, *lQhi, *lFhi;
};

// The source term of a PDE with an algebraic source and/or a
// non-conservative product at space-time node (x, y, z; t) of a cell whose
// iterate lQi sits in shared memory (node stride QS): S = algebraicSource(Q)
// - B(Q) gradQ, the gradients contracted from the iterate's lines with dudx
// and 1/dx (3d/spaceTimePredictorNonlinear.cpph:171-174, 199-202, 228-231,
// 238-276; 2d :145-148, 169-172, 180-211).
template <int DIM, int N, class PDE>
__device__ __forceinline__ void node_source(const double* sQ, int QS, int t, int x, int y, int z, double invDx0,
                                            double invDx1, double invDx2, double* S) {
  using Sh = Shape<DIM, N, PDE>;
  constexpr int b = Sh::b, nV = Sh::nV, nD = Sh::nD;
  const OrderTables& T = c_tab[N];
  const int p = (z * b + y) * b + x;
  double Q[nD];
#pragma unroll
  for (int v = 0; v < nD; v++) Q[v] = sQ[p * QS + t * nD + v];
  if constexpr (PDE::kSource) {
    PDE::algebraicSource(Q, S);
  } else {
#pragma unroll
    for (int v = 0; v < nV; v++) S[v] = 0.0;
  }
  if constexpr (PDE::kNCP) {
    double G[DIM][nV];
#pragma unroll
    for (int v = 0; v < nV; v++) {
      double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
      for (int n = 0; n < b; n++) {
        gx += invDx0 * sQ[((z * b + y) * b + n) * QS + t * nD + v] * T.dudx[x * b + n];
        gy += invDx1 * sQ[((z * b + n) * b + x) * QS + t * nD + v] * T.dudx[y * b + n];
        if (DIM == 3) gz += invDx2 * sQ[((n * b + y) * b + x) * QS + t * nD + v] * T.dudx[z * b + n];
      }
      G[0][v] = gx;
      G[1][v] = gy;
      if (DIM == 3) G[DIM - 1][v] = gz;
    }
    double B[nV];
    PDE::template ncp<DIM>(Q, G, B);
#pragma unroll
    for (int v = 0; v < nV; v++) S[v] -= B[v];
  }
}

template <int DIM, int N, class PDE, bool TEMPS, int VSPLIT, int MINB>
__global__ void __launch_bounds__(PredictorCfg<DIM, N, PDE, VSPLIT, MINB>::THREADS, MINB)
    predictor_kernel(const double* __restrict__ luh, double* __restrict__ lQhbnd, double* __restrict__ lFhbnd,
                     double* __restrict__ lduh, int* __restrict__ iters, const double* __restrict__ dt_ptr,
                     Geometry geo, int ncells, const int* __restrict__ cell_list, PredictorTemps tmp,
                     const int* __restrict__ count) {
  using C = PredictorCfg<DIM, N, PDE, VSPLIT, MINB>;
  constexpr int b = C::b, P = C::P, F = C::F, nV = C::nV, nD = C::nD, NVT = C::NVT, QS = C::QS;
  constexpr bool SRC = PDE::kSource || PDE::kNCP;  // useSource || useNCP
  static_assert(!SRC || VSPLIT == 1, "the source term is formed per node by one thread");
  extern __shared__ double smem[];
  const OrderTables& T = c_tab[N];

  // a device-side count that leaves this block without cells: the whole
  // block returns before its first barrier (a gated launch costs little)
  if (count && (int)blockIdx.x * C::CPB >= min(*count, ncells)) return;
  const int part_id = threadIdx.x / C::TPC;  // which variable slice
  const int r = threadIdx.x - part_id * C::TPC;
  const int lc = r / P;
  const int p = r - lc * P;
  const int v0 = part_id * NVT;
  const bool lead = part_id == 0;  // evaluates fluxes and owns the parameters
  const int slot = blockIdx.x * C::CPB + lc;
  const bool active = slot < (count ? min(*count, ncells) : ncells);  // count: optional device-side list length
  const int cell = active ? (cell_list ? cell_list[slot] : slot) : 0;

  double* sQ = smem + lc * C::SQ;
  double* sF = smem + C::CPB * C::SQ + lc * C::SF;
  double* sR = smem + C::CPB * (C::SQ + C::SF) + lc * C::SR;
  double* sK = smem + C::CPB * (C::SQ + C::SF + C::SR);
  for (int i = threadIdx.x; i < C::SK; i += blockDim.x) sK[i] = T.Kxi[i];

  const int x = p % b, y = (p / b) % b, z = DIM == 3 ? p / (b * b) : 0;
  const double wx = T.w[x], wy = T.w[y], wz = DIM == 3 ? T.w[z] : 1.0;
  const double wpt = wz * wy * wx;  // reference order (w_z w_y) w_x
  const double iw = 1.0 / wpt;
  const int inst = cell_instance(geo, cell);
  const double dt = dt_ptr[inst];
  const double invDx0 = 1.0 / cell_width(geo, inst, 0), invDx1 = 1.0 / cell_width(geo, inst, 1);
  const double invDx2 = DIM == 3 ? 1.0 / cell_width(geo, inst, 2) : 0.0;

  // own variables of luh (for the rhs0 term); the lead thread also seeds the
  // whole trivial initial guess lQi(:,t) = luh (:66-82)
  double lu[NVT];
  {
    const double* src = luh + ((size_t)cell * P + p) * nD;
#pragma unroll
    for (int j = 0; j < NVT; j++) lu[j] = (active && v0 + j < nV) ? __ldg(src + v0 + j) : 0.0;
    if (lead) {
      double q[nD];
#pragma unroll
      for (int v = 0; v < nD; v++) q[v] = active ? __ldg(src + v) : 0.0;
#pragma unroll
      for (int t = 0; t < b; t++)
#pragma unroll
        for (int v = 0; v < nD; v++) sQ[p * QS + t * nD + v] = q[v];
    }
  }

  double fh[DIM][nV];  // lead threads: time-averaged fluxes of the last sweep
  double sh[SRC ? nV : 1];  // and the time-averaged source (lShi)
  bool done = !active;
  int it_done = 0;
  for (int iter = 0; iter < C::maxIter; iter++) {
    double qn[b][NVT];
#pragma unroll
    for (int l = 0; l < b; l++)
#pragma unroll
      for (int j = 0; j < NVT; j++) qn[l][j] = 0.0;

    for (int t = 0; t < b; t++) {
      __syncthreads();  // previous slice's readers are done with sF (and lQi is seeded)
      if (!done && lead) {
        double Q[nD];
#pragma unroll
        for (int v = 0; v < nD; v++) Q[v] = sQ[p * QS + t * nD + v];
        double Fl[DIM][nV];
        PDE::template flux<DIM>(Q, Fl);
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int v = 0; v < nV; v++) sF[(d * P + p) * nV + v] = Fl[d][v];
      }
      __syncthreads();
      if (!done) {
        // derivative contractions (:151-236); the quadrature factor of each
        // direction is applied once per node instead of once per term
        double ax[NVT], ay[NVT], az[NVT];
#pragma unroll
        for (int j = 0; j < NVT; j++) ax[j] = ay[j] = az[j] = 0.0;
        {
          const double* Fx = sF + (0 * P + (z * b + y) * b) * nV + v0;
#pragma unroll
          for (int n = 0; n < b; n++) {
            const double k = sK[n * b + x];
#pragma unroll
            for (int j = 0; j < NVT; j++)
              if (v0 + j < nV) ax[j] = fma(Fx[n * nV + j], k, ax[j]);
          }
        }
        {
          const double* Fy = sF + (1 * P + z * b * b + x) * nV + v0;
#pragma unroll
          for (int n = 0; n < b; n++) {
            const double k = sK[n * b + y];
#pragma unroll
            for (int j = 0; j < NVT; j++)
              if (v0 + j < nV) ay[j] = fma(Fy[n * b * nV + j], k, ay[j]);
          }
        }
        if (DIM == 3) {
          const double* Fz = sF + (2 * P + y * b + x) * nV + v0;
#pragma unroll
          for (int n = 0; n < b; n++) {
            const double k = sK[n * b + z];
#pragma unroll
            for (int j = 0; j < NVT; j++)
              if (v0 + j < nV) az[j] = fma(Fz[n * b * b * nV + j], k, az[j]);
          }
        }
        const double usx = (T.w[t] * wz) * wy * dt * invDx0;
        const double usy = (T.w[t] * wz) * wx * dt * invDx1;
        const double usz = DIM == 3 ? (T.w[t] * wy) * wx * dt * invDx2 : 0.0;
        const double r0 = wpt * T.FL[t];
        // source and non-conservative product, weighted w_t w_xyz dt (:238-276)
        double src[SRC ? nV : 1];
        if constexpr (SRC) {
          node_source<DIM, N, PDE>(sQ, QS, t, x, y, z, invDx0, invDx1, invDx2, src);
          const double uss = (DIM == 3 ? ((T.w[t] * wz) * wy) * wx : (T.w[t] * wy) * wx) * dt;
#pragma unroll
          for (int v = 0; v < nV; v++) src[v] *= uss;
        }
        // discrete time integral (:280-311): lQi_new[l] += iw rhs[t] iK1[l][t]
#pragma unroll
        for (int j = 0; j < NVT; j++) {
          double rhs = r0 * lu[j] - usx * ax[j] - usy * ay[j];
          if (DIM == 3) rhs -= usz * az[j];
          if constexpr (SRC) rhs += src[j];
          const double ir = iw * rhs;
#pragma unroll
          for (int l = 0; l < b; l++) qn[l][j] = fma(ir, T.iK1[l * b + t], qn[l][j]);
        }
      }
    }
    // residual (:282-311): partial sums per (node, slice), reduced per cell by a warp
    double part = 0.0;
    if (!done) {
#pragma unroll
      for (int l = 0; l < b; l++)
#pragma unroll
        for (int j = 0; j < NVT; j++)
          if (v0 + j < nV) {
            const double dq = qn[l][j] - sQ[p * QS + l * nD + v0 + j];
            part = fma(dq, dq, part);
          }
    }
    sR[part_id * P + p] = part;
    __syncthreads();
    {
      constexpr int kFullWarps = C::THREADS / 32;
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      if (warp < kFullWarps) {
        for (int c = warp; c < C::CPB; c += kFullWarps) {
          double* rr = smem + C::CPB * (C::SQ + C::SF) + c * C::SR;
          double acc = 0.0;
          for (int i = lane; i < VSPLIT * P; i += 32) acc += rr[i];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
          if (lane == 0) rr[VSPLIT * P] = acc;
        }
      }
    }
    __syncthreads();
    const double sq_res = sR[VSPLIT * P];
    if (!done) {
      it_done = iter + 1;
      const bool conv = sq_res < 1e-7 * 1e-7;  // exit condition (:315-318)
      if (conv || iter + 1 == C::maxIter) {
        // lFhi is the time average of the fluxes this sweep evaluated, i.e. of
        // the iterate before the update (:337-409): the lead thread re-evaluates
        // them from its node's old lQi row before the row is overwritten.
        if (lead) {
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int v = 0; v < nV; v++) fh[d][v] = 0.0;
          if constexpr (SRC) {
#pragma unroll
            for (int v = 0; v < nV; v++) sh[v] = 0.0;
          }
          for (int t = 0; t < b; t++) {
            double Q[nD];
#pragma unroll
            for (int v = 0; v < nD; v++) Q[v] = sQ[p * QS + t * nD + v];
            double Fl[DIM][nV];
            PDE::template flux<DIM>(Q, Fl);
#pragma unroll
            for (int d = 0; d < DIM; d++)
#pragma unroll
              for (int v = 0; v < nV; v++) fh[d][v] += Fl[d][v] * T.w[t];
            double St[SRC ? nV : 1];
            if constexpr (SRC) {  // lShi (:391-396), from the same iterate
              node_source<DIM, N, PDE>(sQ, QS, t, x, y, z, invDx0, invDx1, invDx2, St);
#pragma unroll
              for (int v = 0; v < nV; v++) sh[v] += St[v] * T.w[t];
            }
            if (TEMPS) {
              double* dst = tmp.lFi + (((size_t)cell * b + t) * P + p) * (DIM + 1) * nV;
#pragma unroll
              for (int d = 0; d < DIM; d++)
#pragma unroll
                for (int v = 0; v < nV; v++) dst[d * nV + v] = Fl[d][v];
              if constexpr (SRC) {
#pragma unroll
                for (int v = 0; v < nV; v++) dst[DIM * nV + v] = St[v];
              }
            }
          }
        }
        done = true;
      }
    }
    // the lead thread of a node may still read the old row above; every
    // thread overwrites its own variables only after the barrier
    __syncthreads();
    if (it_done == iter + 1) {
#pragma unroll
      for (int l = 0; l < b; l++)
#pragma unroll
        for (int j = 0; j < NVT; j++)
          if (v0 + j < nV) sQ[p * QS + l * nD + v0 + j] = qn[l][j];
    }
    if (!__syncthreads_or(!done)) break;
  }
  if (iters && active && lead && p == 0) iters[cell] = it_done;

  // time averages (:337-409). lQhi from the final lQi (lead threads).
  double qh[nD];
  if (lead) {
#pragma unroll
    for (int v = 0; v < nD; v++) {
      double s = 0.0;
#pragma unroll
      for (int m = 0; m < b; m++) s += sQ[p * QS + m * nD + v] * T.w[m];
      qh[v] = s;
    }
  }
  if (TEMPS && active && lead) {
    double* dq = tmp.lQi + ((size_t)cell * P + p) * b * nD;
    for (int i = 0; i < b * nD; i++) dq[i] = sQ[p * QS + i];
    for (int v = 0; v < nD; v++) tmp.lQhi[((size_t)cell * P + p) * nD + v] = qh[v];
    // reference lFhi blocks: x (z,y,x), y (z,x,y), z (y,x,z), then the source block
    double* fhd = tmp.lFhi + (size_t)cell * (DIM + 1) * P * nV;
    const int py = DIM == 3 ? (z * b + x) * b + y : x * b + y;
    const int pz = (y * b + x) * b + z;
    for (int v = 0; v < nV; v++) {
      fhd[(0 * P + p) * nV + v] = fh[0][v];
      fhd[(1 * P + py) * nV + v] = fh[1][v];
      if (DIM == 3) fhd[(2 * P + pz) * nV + v] = fh[DIM - 1][v];
      fhd[(DIM * P + p) * nV + v] = SRC ? sh[SRC ? v : 0] : 0.0;
    }
  }
  __syncthreads();  // everyone has read its lQi row
  double* sQh = sQ;  // lQhi [P][nD] reuses the lQi buffer
  if (lead) {
#pragma unroll
    for (int v = 0; v < nD; v++) sQh[p * nD + v] = qh[v];
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int v = 0; v < nV; v++) sF[(d * P + p) * nV + v] = fh[d][v];
  }
  __syncthreads();
  if (!active) return;

  // volume integral at this node, own variables (3d/volumeIntegralNonlinear.cpph:135-225)
  if (lduh) {
    double* dst = lduh + ((size_t)cell * P + p) * nV;
    const double usx = (wz * wy) * invDx0, usy = (wz * wx) * invDx1, usz = (wy * wx) * invDx2;
#pragma unroll
    for (int j = 0; j < NVT; j++) {
      const int v = v0 + j;
      if (v >= nV) break;
      double sx = 0.0, sy = 0.0, sz = 0.0;
      const double* Fx = sF + (0 * P + (z * b + y) * b) * nV + v;
      const double* Fy = sF + (1 * P + z * b * b + x) * nV + v;
#pragma unroll
      for (int m = 0; m < b; m++) {
        sx = fma(sK[x * b + m], Fx[m * nV], sx);
        sy = fma(sK[y * b + m], Fy[m * b * nV], sy);
      }
      double du = sx * usx + sy * usy;
      if (DIM == 3) {
        const double* Fz = sF + (2 * P + y * b + x) * nV + v;
#pragma unroll
        for (int m = 0; m < b; m++) sz = fma(sK[z * b + m], Fz[m * b * b * nV], sz);
        du += sz * usz;
      }
      if constexpr (SRC) du += wpt * sh[v];  // useSourceOrNCP: + w_xyz lShi (3d :206-224, 2d :158-172)
      dst[v] = du;
    }
  }

  // boundary extrapolation (3d/spaceTimePredictorNonlinear.cpph:411-528)
  for (int k = part_id * P + p; k < DIM * F; k += VSPLIT * P) {
    const int dir = k / F, fn = k - dir * F;
    const int a = DIM == 3 ? fn / b : 0, c = DIM == 3 ? fn % b : fn;
    // node index of position l along dir on this face line
    const int base = dir == 0 ? (a * b + c) * b : dir == 1 ? a * b * b + c : a * b + c;
    const int stride = dir == 0 ? 1 : dir == 1 ? b : b * b;
    double* qL = lQhbnd + (((size_t)cell * 2 * DIM + 2 * dir) * F + fn) * nD;
    double* qR = lQhbnd + (((size_t)cell * 2 * DIM + 2 * dir + 1) * F + fn) * nD;
    double* fL = lFhbnd + (((size_t)cell * 2 * DIM + 2 * dir) * F + fn) * nV;
    double* fR = lFhbnd + (((size_t)cell * 2 * DIM + 2 * dir + 1) * F + fn) * nV;
#pragma unroll
    for (int v = 0; v < nV; v++) {
      double sl = 0.0, sr = 0.0;
#pragma unroll
      for (int l = 0; l < b; l++) {
        const double f = sF[(dir * P + base + l * stride) * nV + v];
        sl += f * T.FL[l];
        sr += f * T.FR[l];
      }
      fL[v] = sl;
      fR[v] = sr;
    }
#pragma unroll
    for (int v = 0; v < nD; v++) {
      double sl = 0.0, sr = 0.0;
#pragma unroll
      for (int l = 0; l < b; l++) {
        const double q = sQh[(base + l * stride) * nD + v];
        sl += q * T.FL[l];
        sr += q * T.FR[l];
      }
      qL[v] = sl;
      qR[v] = sr;
    }
  }
}

// ---------------------------------------------------------------------------
// Rusanov flux on interior faces: riemannSolverNonlinear<useNCP>
// (3d/riemannSolverNonlinear.cpph:37-117). One warp per face: weighted face
// averages of both states by warp-shuffle reduction, one smax per face from
// the averaged states, then F = (FL+FR)/2 - smax (QR-QL)/2 written to both
// sides (with a non-conservative product, plus / minus half its value). The face joins cell `left` (its face 2*dir+1) and cell `right` (its
// face 2*dir).
template <int DIM, int N, class PDE>
__device__ __forceinline__ void face_average(const double* Q, int lane, double* avg) {
  using S = Shape<DIM, N, PDE>;
  const OrderTables& T = c_tab[N];
#pragma unroll
  for (int k = 0; k < S::nD; k++) avg[k] = 0.0;
  for (int fn = lane; fn < S::F; fn += 32) {
    const double wf = DIM == 3 ? T.w[fn / S::b] * T.w[fn % S::b] : T.w[fn];
#pragma unroll
    for (int k = 0; k < S::nD; k++) avg[k] += wf * Q[fn * S::nD + k];
  }
#pragma unroll
  for (int k = 0; k < S::nD; k++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) avg[k] += __shfl_xor_sync(0xffffffffu, avg[k], o);
}

template <int DIM, class PDE>
__device__ __forceinline__ double face_smax(const double* aL, const double* aR, int dir) {
  double LL[PDE::nVar], LR[PDE::nVar];
  Hooks<PDE, DIM>::eigenvalues(aL, dir, LL);
  Hooks<PDE, DIM>::eigenvalues(aR, dir, LR);
  double sL = fabs(LL[0]), sR = fabs(LR[0]);
#pragma unroll
  for (int k = 1; k < PDE::nVar; k++) {
    if (sL < fabs(LL[k])) sL = fabs(LL[k]);
    if (sR < fabs(LR[k])) sR = fabs(LR[k]);
  }
  return (sL < sR) ? sR : sL;
}

// Component k of the non-conservative product at one face node of a PDE
// with kNCP: B(Qavg) gradQ with Qavg = (QL + QR) / 2 and gradQ zero but for
// the normal direction's row QR - QL (riemannSolverNonlinear.cpph 3d :92-100,
// 2d :86-93).
template <int DIM, class PDE>
__device__ __forceinline__ double face_ncp(const double* QL, const double* QR, int dir, int k) {
  constexpr int nV = PDE::nVar, nD = PDE::nVar + PDE::nPar;
  double Qavg[nD], G[DIM][nV], B[nV];
#pragma unroll
  for (int l = 0; l < nD; l++) Qavg[l] = l < nV ? 0.5 * (QR[l] + QL[l]) : 0.0;
#pragma unroll
  for (int d = 0; d < DIM; d++)
#pragma unroll
    for (int l = 0; l < nV; l++) G[d][l] = d == dir ? QR[l] - QL[l] : 0.0;
  PDE::template ncp<DIM>(Qavg, G, B);
  return B[k];
}

template <int DIM, int N, class PDE>
__global__ void __launch_bounds__(128) riemann_kernel(const double* __restrict__ lQhbnd, double* __restrict__ lFhbnd,
                                                      const int* __restrict__ face_left,
                                                      const int* __restrict__ face_right,
                                                      const int* __restrict__ face_dir, int nfaces,
                                                      const int* __restrict__ gate = nullptr) {
  using S = Shape<DIM, N, PDE>;
  constexpr int F = S::F, nV = S::nV, nD = S::nD;
  const int lane = threadIdx.x & 31;
  const int f = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (gate && !*gate) return;  // gate (optional, device): 0 skips the launch's work
  if (f >= nfaces) return;
  const int cl = face_left[f], cr = face_right[f], dir = face_dir[f];
  const double* QL = lQhbnd + ((size_t)cl * 2 * DIM + 2 * dir + 1) * F * nD;
  const double* QR = lQhbnd + ((size_t)cr * 2 * DIM + 2 * dir) * F * nD;
  double* FL = lFhbnd + ((size_t)cl * 2 * DIM + 2 * dir + 1) * F * nV;
  double* FR = lFhbnd + ((size_t)cr * 2 * DIM + 2 * dir) * F * nV;
  // this lane's flux and state differences are loaded before the face
  // averages, so that all of the face's loads are in flight together
  constexpr int E = F * nV, EPL = (E + 31) / 32;
  double fl[EPL], fr[EPL], dq[EPL];
#pragma unroll
  for (int i = 0; i < EPL; i++) {
    const int e = lane + 32 * i, fn = e / nV, k = e - fn * nV;
    const bool in = e < E;
    fl[i] = in ? FL[e] : 0.0;
    fr[i] = in ? FR[e] : 0.0;
    dq[i] = in ? QR[fn * nD + k] - QL[fn * nD + k] : 0.0;
  }
  double aL[nD], aR[nD];
  face_average<DIM, N, PDE>(QL, lane, aL);
  face_average<DIM, N, PDE>(QR, lane, aR);
  const double smax = face_smax<DIM, PDE>(aL, aR, dir);
#pragma unroll
  for (int i = 0; i < EPL; i++) {
    const int e = lane + 32 * i;
    if (e < E) {
      const double r = 0.5 * (fr[i] + fl[i]) - 0.5 * smax * dq[i];
      if constexpr (PDE::kNCP) {
        // useNCP (:92-110): the product of the node's mean state and its jump
        // along the normal splits into fluctuations, + on the left, - on the right
        const int fn = e / nV, k = e - fn * nV;
        const double half = 0.5 * face_ncp<DIM, PDE>(QL + fn * nD, QR + fn * nD, dir, k);
        FL[e] = r + half;
        FR[e] = r - half;
      } else {
        FL[e] = r;
        FR[e] = r;
      }
    }
  }
}

// Boundary faces: ADERDGSolver::applyBoundaryConditions
// (exahype/solvers/ADERDGSolver.cpp:2893-2962) -- user boundaryValues at every
// face node, then the Rusanov flux with the outside state on the outer side
// (argument order by faceIndex parity). Only the cell's own flux is kept.
template <int DIM, int N, class PDE>
__global__ void __launch_bounds__(128) boundary_kernel(const double* __restrict__ lQhbnd, double* __restrict__ lFhbnd,
                                                       const int* __restrict__ bcell, const int* __restrict__ bface,
                                                       int nb, int kind, const int* __restrict__ gate = nullptr) {
  using S = Shape<DIM, N, PDE>;
  constexpr int F = S::F, nV = S::nV, nD = S::nD;
  const int lane = threadIdx.x & 31;
  const int f = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (f >= nb || (gate && !*gate)) return;
  const int c = bcell[f], face = bface[f], dir = face >> 1;
  const double* QIn = lQhbnd + ((size_t)c * 2 * DIM + face) * F * nD;
  double* FIn = lFhbnd + ((size_t)c * 2 * DIM + face) * F * nV;
  const OrderTables& T = c_tab[N];
  double aIn[nD], aOut[nD];
#pragma unroll
  for (int k = 0; k < nD; k++) aIn[k] = aOut[k] = 0.0;
  for (int fn = lane; fn < F; fn += 32) {
    const double wf = DIM == 3 ? T.w[fn / S::b] * T.w[fn % S::b] : T.w[fn];
    double qo[nD], fo[nV];
    PDE::template boundaryValues<DIM>(kind, dir, FIn + fn * nV, QIn + fn * nD, fo, qo);
#pragma unroll
    for (int k = 0; k < nD; k++) {
      aIn[k] += wf * QIn[fn * nD + k];
      aOut[k] += wf * qo[k];
    }
  }
#pragma unroll
  for (int k = 0; k < nD; k++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      aIn[k] += __shfl_xor_sync(0xffffffffu, aIn[k], o);
      aOut[k] += __shfl_xor_sync(0xffffffffu, aOut[k], o);
    }
  // riemannSolver(FOut, FIn, QOut, QIn) for even faces, (FIn, FOut, QIn, QOut) for odd
  const bool even = (face & 1) == 0;
  const double smax = even ? face_smax<DIM, PDE>(aOut, aIn, dir) : face_smax<DIM, PDE>(aIn, aOut, dir);
  __syncwarp();
  for (int fn = lane; fn < F; fn += 32) {
    double qo[nD], fo[nV];
    PDE::template boundaryValues<DIM>(kind, dir, FIn + fn * nV, QIn + fn * nD, fo, qo);
#pragma unroll
    for (int k = 0; k < nV; k++) {
      const double fi = FIn[fn * nV + k], qi = QIn[fn * nD + k];
      double r = even ? 0.5 * (fi + fo[k]) - 0.5 * smax * (qi - qo[k])
                      : 0.5 * (fo[k] + fi) - 0.5 * smax * (qo[k] - qi);
      if constexpr (PDE::kNCP) {  // the cell is the right side of an even face, the left of an odd one
        if (even)
          r -= 0.5 * face_ncp<DIM, PDE>(qo, QIn + fn * nD, dir, k);
        else
          r += 0.5 * face_ncp<DIM, PDE>(QIn + fn * nD, qo, dir, k);
      }
      FIn[fn * nV + k] = r;
    }
  }
}

// ---------------------------------------------------------------------------
// surfaceIntegral + solutionUpdate at node p of one cell (du: the cell's
// lduh at the node, NULL for no update; Fb: the cell's lFhbnd; q: the node's
// state, updated in place; invDx: 1/dx per direction, rounded to nearest).
// Returns the denominator of the node's admissible step 0.9 PNPM / den,
// den = sum_d maxAbsEigenvalue_d(q) / dx_d.
template <int DIM, int N, class PDE>
__device__ __forceinline__ double corrector_node(double* q, const double* __restrict__ du_in,
                                                 const double* __restrict__ Fb, int p, const Geometry& geo, int inst,
                                                 const double* __restrict__ dt_ptr, double invDx0, double invDx1,
                                                 double invDx2) {
  using S = Shape<DIM, N, PDE>;
  constexpr int b = S::b, F = S::F, nV = S::nV;
  const OrderTables& T = c_tab[N];
  const int x = p % b, y = (p / b) % b, z = DIM == 3 ? p / (b * b) : 0;
  const double wx = T.w[x], wy = T.w[y], wz = DIM == 3 ? T.w[z] : 1.0;
  if (du_in) {
    double du[nV];
#pragma unroll
    for (int v = 0; v < nV; v++) du[v] = du_in[v];
    // nonlinear: surfaceIntegralNonlinear, flux difference times w / dx;
    // linear (surfaceIntegralLinear, 3d/surfaceIntegralLinear.cpph:24-91):
    // the two faces' fluctuations are added, scaled by w divided by dx
    constexpr bool LIN = PDE::kLinear;
    {
      const double us = LIN ? (wz * wy) / cell_width(geo, inst, 0) : (wz * wy) * invDx0;
      const int fn = DIM == 3 ? z * b + y : y;
#pragma unroll
      for (int v = 0; v < nV; v++)
        du[v] -= (LIN ? Fb[(1 * F + fn) * nV + v] * T.FR[x] + Fb[(0 * F + fn) * nV + v] * T.FL[x]
                      : Fb[(1 * F + fn) * nV + v] * T.FR[x] - Fb[(0 * F + fn) * nV + v] * T.FL[x]) * us;
    }
    {
      const double us = LIN ? (wz * wx) / cell_width(geo, inst, 1) : (wz * wx) * invDx1;
      const int fn = DIM == 3 ? z * b + x : x;
#pragma unroll
      for (int v = 0; v < nV; v++)
        du[v] -= (LIN ? Fb[(3 * F + fn) * nV + v] * T.FR[y] + Fb[(2 * F + fn) * nV + v] * T.FL[y]
                      : Fb[(3 * F + fn) * nV + v] * T.FR[y] - Fb[(2 * F + fn) * nV + v] * T.FL[y]) * us;
    }
    if (DIM == 3) {
      const double us = LIN ? (wy * wx) / cell_width(geo, inst, 2) : (wy * wx) * invDx2;
      const int fn = y * b + x;
#pragma unroll
      for (int v = 0; v < nV; v++)
        du[v] -= (LIN ? Fb[(5 * F + fn) * nV + v] * T.FR[z] + Fb[(4 * F + fn) * nV + v] * T.FL[z]
                      : Fb[(5 * F + fn) * nV + v] * T.FR[z] - Fb[(4 * F + fn) * nV + v] * T.FL[z]) * us;
    }
    const double us = dt_ptr[inst] / (wz * wy * wx);
#pragma unroll
    for (int v = 0; v < nV; v++) q[v] += du[v] * us;
  }
  double den = 0.0;
  den = __dadd_rn(den, __dmul_rn(Hooks<PDE, DIM>::max_abs_eig_exact(q, 0), invDx0));
  den = __dadd_rn(den, __dmul_rn(Hooks<PDE, DIM>::max_abs_eig_exact(q, 1), invDx1));
  if (DIM == 3) den = __dadd_rn(den, __dmul_rn(Hooks<PDE, DIM>::max_abs_eig_exact(q, 2), invDx2));
  return den;
}

// Corrector: surfaceIntegralNonlinear (3d/surfaceIntegralNonlinear.cpph:21-90)
// or, for a linear PDE, surfaceIntegralLinear,
// solutionUpdate (3d/solutionUpdate.cpph:23-47) and stableTimeStepSize
// (3d/stableTimeStepSize.cpph:21-63) fused, one thread per node. The new
// admissible step is min-reduced over the whole launch into *dt_out; the
// time-step arithmetic uses explicit round-to-nearest operations so that it
// reproduces the reference's unfused evaluation bit for bit.
//
// The block's cells' luh, lduh and lFhbnd are staged in shared memory by
// coalesced loads (all issued before the first shared store) and luh is
// written back the same way: per-node accesses of nD consecutive doubles
// would make every load and store instruction touch 32 sectors.
template <int DIM, int N, class PDE>
struct CorrectorCfg : Shape<DIM, N, PDE> {
  using S = Shape<DIM, N, PDE>;
  static constexpr int CPB = cells_per_block<S::P>();
  // whole warps: the block min-reduction shuffles across full warps
  static constexpr int THREADS = (CPB * S::P + 31) / 32 * 32;
  // per cell in shared memory: state (node stride QS, odd against bank
  // conflicts), update (stride nV), face fluxes
  static constexpr int QS = S::nD | 1;
  static constexpr int OU = 0, ODU = S::P * QS, OFB = ODU + S::P * S::nV;
  static constexpr int SC = OFB + 2 * DIM * S::F * S::nV;
  static constexpr size_t SMEM = sizeof(double) * (size_t)CPB * SC;
  static_assert(SMEM <= 227 * 1024, "corrector staging exceeds shared memory");
};

template <int DIM, int N, class PDE>
__global__ void __launch_bounds__(CorrectorCfg<DIM, N, PDE>::THREADS)
    corrector_kernel(double* __restrict__ luh, const double* __restrict__ lduh, const double* __restrict__ lFhbnd,
                     const double* __restrict__ dt_ptr, double* __restrict__ dt_out, Geometry geo, int ncells,
                     const int* __restrict__ cell_list, int do_update, const int* __restrict__ count) {
  using C = CorrectorCfg<DIM, N, PDE>;
  constexpr int P = C::P, F = C::F, nV = C::nV, nD = C::nD, QS = C::QS, SC = C::SC;
  constexpr int SU = P * nD, SDU = P * nV, SFB = 2 * DIM * F * nV;  // per-cell global extents
  extern __shared__ double smem[];
  __shared__ double red[32];
  __shared__ int s_cell[C::CPB];
  const int lc = threadIdx.x / P;
  const int p = threadIdx.x - lc * P;
  const int slot = blockIdx.x * C::CPB + lc;
  const int nact = count ? min(*count, ncells) : ncells;  // count: optional device-side list length
  if ((int)blockIdx.x * C::CPB >= nact) return;           // whole block, before its first barrier
  // padding threads only join the reduction
  const bool active = lc < C::CPB && slot < nact;
  if (threadIdx.x < C::CPB) {
    const int s = blockIdx.x * C::CPB + threadIdx.x;
    s_cell[threadIdx.x] = s < nact ? (cell_list ? cell_list[s] : s) : -1;
  }
  __syncthreads();
  {
    // loads of the three arrays into registers, then the shared stores
    constexpr int KU = (C::CPB * SU + C::THREADS - 1) / C::THREADS;
    constexpr int KD = (C::CPB * SDU + C::THREADS - 1) / C::THREADS;
    constexpr int KF = (C::CPB * SFB + C::THREADS - 1) / C::THREADS;
    double vu[KU], vd[KD], vf[KF];
#pragma unroll
    for (int k = 0; k < KU; k++) {
      const int i = threadIdx.x + k * C::THREADS, c = i / SU, e = i - c * SU;
      vu[k] = (c < C::CPB && s_cell[c] >= 0) ? luh[(size_t)s_cell[c] * SU + e] : 0.0;
    }
    if (do_update) {
#pragma unroll
      for (int k = 0; k < KD; k++) {
        const int i = threadIdx.x + k * C::THREADS, c = i / SDU, e = i - c * SDU;
        vd[k] = (c < C::CPB && s_cell[c] >= 0) ? lduh[(size_t)s_cell[c] * SDU + e] : 0.0;
      }
#pragma unroll
      for (int k = 0; k < KF; k++) {
        const int i = threadIdx.x + k * C::THREADS, c = i / SFB, e = i - c * SFB;
        vf[k] = (c < C::CPB && s_cell[c] >= 0) ? lFhbnd[(size_t)s_cell[c] * SFB + e] : 0.0;
      }
    }
#pragma unroll
    for (int k = 0; k < KU; k++) {
      const int i = threadIdx.x + k * C::THREADS, c = i / SU, e = i - c * SU;
      if (c < C::CPB) smem[c * SC + C::OU + (e / nD) * QS + e % nD] = vu[k];
    }
    if (do_update) {
#pragma unroll
      for (int k = 0; k < KD; k++) {
        const int i = threadIdx.x + k * C::THREADS, c = i / SDU, e = i - c * SDU;
        if (c < C::CPB) smem[c * SC + C::ODU + e] = vd[k];
      }
#pragma unroll
      for (int k = 0; k < KF; k++) {
        const int i = threadIdx.x + k * C::THREADS, c = i / SFB, e = i - c * SFB;
        if (c < C::CPB) smem[c * SC + C::OFB + e] = vf[k];
      }
    }
  }
  __syncthreads();
  double dtmin = __longlong_as_double(0x7fefffffffffffffll);  // DBL_MAX
  int inst = 0;
  if (active) {
    inst = cell_instance(geo, s_cell[lc]);
    double* st = smem + lc * SC;
    double q[nD];
#pragma unroll
    for (int v = 0; v < nD; v++) q[v] = st[C::OU + p * QS + v];
    const double invDx0 = __ddiv_rn(1.0, cell_width(geo, inst, 0)), invDx1 = __ddiv_rn(1.0, cell_width(geo, inst, 1));
    const double invDx2 = DIM == 3 ? __ddiv_rn(1.0, cell_width(geo, inst, 2)) : 0.0;
    const double den = corrector_node<DIM, N, PDE>(q, do_update ? st + C::ODU + p * nV : nullptr, st + C::OFB, p,
                                                   geo, inst, dt_ptr, invDx0, invDx1, invDx2);
    // dt = std::min(dt, candidate) from DBL_MAX, as the reference: a NaN or
    // infinite candidate (a node with negative pressure, a zero denominator)
    // never replaces the running minimum, here nor in the reductions below
    const double cand = __ddiv_rn(__dmul_rn(0.9, pnpm(N)), den);
    dtmin = (cand < dtmin) ? cand : dtmin;
    if (do_update)
#pragma unroll
      for (int v = 0; v < nV; v++) st[C::OU + p * QS + v] = q[v];
  }
  if (do_update) {  // the updated state, written back coalesced
    __syncthreads();
#pragma unroll
    for (int k = 0; k < (C::CPB * SU + C::THREADS - 1) / C::THREADS; k++) {
      const int i = threadIdx.x + k * C::THREADS, c = i / SU, e = i - c * SU;
      if (c < C::CPB && s_cell[c] >= 0) luh[(size_t)s_cell[c] * SU + e] = smem[c * SC + C::OU + (e / nD) * QS + e % nD];
    }
  }
  // A batch block may hold cells of two instances (instances are contiguous
  // cell ranges): then every thread min-combines into its own instance.
  __shared__ int s_inst[2];
  if (geo.inst) {
    if (threadIdx.x == 0) s_inst[0] = INT_MAX, s_inst[1] = INT_MIN;
    __syncthreads();
    if (active) {
      atomicMin(&s_inst[0], inst);
      atomicMax(&s_inst[1], inst);
    }
    __syncthreads();
    if (s_inst[0] != s_inst[1] && s_inst[0] != INT_MAX) {
      if (active && dt_out) atomic_min_pos_double(dt_out + inst, dtmin);
      return;
    }
    inst = s_inst[0] == INT_MAX ? 0 : s_inst[0];
  }
  // block min, then one atomic per block
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double other = __shfl_xor_sync(0xffffffffu, dtmin, o);
    dtmin = (other < dtmin) ? other : dtmin;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dtmin;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = (blockDim.x + 31) >> 5;
    double m = threadIdx.x < nw ? red[threadIdx.x] : __longlong_as_double(0x7fefffffffffffffll);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_xor_sync(0xffffffffu, m, o);
      m = (other < m) ? other : m;
    }
    if (threadIdx.x == 0 && dt_out) atomic_min_pos_double(dt_out + inst, m);
  }
}

// Sets *a = DBL_MAX (start of a min-reduction) and optionally advances the
// time-stepping scalars on the device so that no host round trip is needed
// between steps.
__global__ void reset_min_kernel(double* a) { *a = __longlong_as_double(0x7fefffffffffffffll); }

}  // namespace exa
