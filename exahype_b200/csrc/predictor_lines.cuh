// Space-time predictor, "line" form.
//
// Same algorithm and outputs as predictor_kernel (aderdg.cuh): the Picard
// iteration of aderPicardLoopNonlinear (3d/spaceTimePredictorNonlinear.cpph:
// 42-329), time averaging (:337-409), extrapolation (:411-528) and
// volumeIntegralNonlinear (3d/volumeIntegralNonlinear.cpph:135-225).
//
// The derivative contractions are organised around 1-D lines instead of
// nodes, which is what bounds the node form (every derivative term reloads a
// flux value from shared memory). Per time slice:
//   A  one thread per node evaluates the flux and stores it line-major,
//      sF[d][n][L][v]: d direction, n position along d, L the line (the other
//      two coordinates, in (z,y,x) order or swapped, per direction), v the
//      variable;
//   B  one thread per (d, L, v) loads its line once, forms all b outputs
//      sum_n F[n] Kxi[n][l] with the stiffness entries as compile-time-indexed
//      constant-bank operands, scales by the line's quadrature factor and
//      writes them back in place;
//   C  one thread per node adds its three directional contributions to the
//      rhs and folds the rhs into its Picard accumulators through iK1.
// Shared memory per cell: lQi [P][b][nD], one line-major slice, residuals.
//
// TM (five state variables, at most 60 columns per thread): the Picard
// iterate lQi lives in tensor memory instead (tmem.cuh: each thread owns one
// TMEM lane, 60 columns of it), so that its reads and writes (phase A, the
// residual, the update, the time average) leave the shared-memory pipe,
// which bounds this kernel. The tensor-memory instructions are
// warp-collective, so the block is rounded up to whole warps (3D N=5, 216
// nodes: 224 threads; 2D N=5, seven cells of 36: 256); the threads without
// a node take part in those instructions and in the phase-B items only.
// With several cells per block a warp can hold nodes of cells in different
// states (iterating, converged), so there every tensor-memory instruction is
// issued under block-uniform control only, and per-cell work is selected by
// the data (a converged cell stores its unchanged iterate back).
#pragma once
#include "aderdg.cuh"
#include "tmem.cuh"

namespace exa {

// Stride of one n-slab of the line-major flux slice, chosen per (b, DIM) with
// a shared-memory bank model (64-bit accesses, 16 bank pairs per half-warp)
// over the three access patterns of a slice; the fallback is odd.
constexpr int line_slab(int b, int dim, int lines5) {
  return dim == 3 ? (b == 6 ? 190 : b == 4 ? 84 : b == 8 ? 322 : b == 5 ? 137 : lines5 + 1)
                  : (b == 6 ? 30 : b == 4 ? 20 : b == 8 ? 42 : b == 5 ? 25 : lines5 + 1);
}
// 3D, b = 6, five variables: a stride and line order per direction. Phases A
// and C access the slab node by node (the thread's node fixes n and the line
// in every direction); with one common stride the x direction's 16-lane
// groups hit the same bank pair up to three times (63 wavefronts per
// direction triple and 216 nodes against 42 conflict-free). Strides 181 / 190
// / 180 with the x direction's line index in (y, z) order give 50, phase B
// staying conflict-free (its items are consecutive along the lines).
constexpr int line_slab_dir(int b, int dim, int nv, int d, int fallback) {
  return (dim == 3 && b == 6 && nv == 5) ? (d == 0 ? 181 : d == 1 ? 190 : 180) : fallback;
}
constexpr bool line_swap_dir(int b, int dim, int nv, int d) { return dim == 3 && b == 6 && nv == 5 && d == 0; }

// MIXED: the mixed-precision form (see predictor_lines_kernel) keeps each
// node's last FP32 update in shared memory, SD doubles per cell.
// TS: time slices per phase (each phase of a Picard sweep handles TS slices
// between two barriers; TS slice buffers per cell).
template <int DIM, int N, class PDE, int MINB, bool MIXED = false, int TS = 1, bool TM = false>
struct LinesCfg : Shape<DIM, N, PDE> {
  using S = Shape<DIM, N, PDE>;
  static constexpr int CPB = cells_per_block<S::P>();
  static constexpr int THREADS = TM ? (CPB * S::P + 31) / 32 * 32 : CPB * S::P;
  static constexpr int LINES = S::P / S::b;  // lines per direction = face nodes
  static constexpr int SR = S::P + 1;
  static constexpr int SD = MIXED ? (S::P * S::b * S::nV + 1) / 2 : 0;
  static constexpr int SLAB0 = S::nV == 5 ? line_slab(S::b, DIM, LINES * 5) : LINES * S::nV + 1;
  static constexpr int SS0 = line_slab_dir(S::b, DIM, S::nV, 0, SLAB0);
  static constexpr int SS1 = line_slab_dir(S::b, DIM, S::nV, 1, SLAB0);
  static constexpr int SS2 = line_slab_dir(S::b, DIM, S::nV, 2, SLAB0);
  static constexpr int SFJ0 = S::b * (SS0 + SS1 + (DIM == 3 ? SS2 : 0));
  // padded strides (bank-conflict-free) where they fit in 227 KB, packed otherwise
  static constexpr bool kPad =
      sizeof(double) * (size_t)(CPB * (S::P * (S::b * S::nD + 1) + TS * SFJ0 + SR + SD)) <= 227 * 1024;
  static constexpr int QS = kPad ? S::b * S::nD + 1 : S::b * S::nD;  // lQi node stride
  // TM: 32-bit columns per thread and per CTA (the warps of a lane quadrant
  // take consecutive column ranges)
  static constexpr int TCOL = 64;
  static constexpr int TCOLS = TCOL * ((THREADS / 32 + 3) / 4);
  static_assert(!TM || (!MIXED && S::nD == 5 && S::nV == 5 && 2 * S::b * S::nD <= TCOL && THREADS <= 256),
                "tensor-memory iterate: five doubles per node and slice, at most 256 threads");
  // lQi region (TM: none; the region later holds the time-averaged state and
  // the staged volume integral of every node)
  static constexpr int SQ = TM ? S::P * (S::nD > S::nV ? S::nD : S::nV) : S::P * QS;
  // per direction d: stride along the line, first element, line order
  static constexpr __host__ __device__ int sstride(int d) {
    return kPad ? (d == 0 ? SS0 : d == 1 ? SS1 : SS2) : LINES * S::nV;
  }
  static constexpr __host__ __device__ int sbase(int d) {
    return S::b * (d > 0 ? sstride(0) : 0) + S::b * (d > 1 ? sstride(1) : 0);
  }
  static constexpr __host__ __device__ bool sswap(int d) { return kPad && line_swap_dir(S::b, DIM, S::nV, d); }
  static constexpr int SFJ = sbase(DIM - 1) + S::b * sstride(DIM - 1);  // one slice
  static constexpr int SF = TS * SFJ;
  static constexpr size_t SMEM = sizeof(double) * (size_t)(CPB * (SQ + SF + SR + SD));
  static constexpr int ITEMS = CPB * DIM * LINES * S::nV;  // phase-B work items per block
  static constexpr int IPT = (ITEMS + THREADS - 1) / THREADS;  // items per thread
};

// node p = (z, y, x) -> position n along direction d and line index L (the
// face-node order of the direction's faces: the other two coordinates, the
// slower one first)
template <int DIM, int b>
__device__ __forceinline__ void node_line(int d, int z, int y, int x, int& n, int& L) {
  if (d == 0) { n = x; L = z * b + y; }
  else if (d == 1) { n = y; L = z * b + x; }
  else { n = z; L = y * b + x; }
}
// a line's face-node index <-> its index in the slab (the same, or its two
// coordinates swapped; the map is its own inverse)
template <int b>
__device__ __forceinline__ int line_swapped(bool swap, int L) { return swap ? (L % b) * b + L / b : L; }

// MIXED: the first sweep is the FP64 sweep above; every later sweep k works
// on increments. Its flux increment dF = F(q^k) - F(q^k - d^k) (d^k the
// node's last update, kept in FP32) is formed in FP64 and stored in FP32; the
// line contractions of dF run in FP32 (half the shared-memory bytes, FP32
// arithmetic); the iK1 fold accumulates in FP64 and the update d^(k+1) is
// added to the FP64 iterate. The rhs0 term
// cancels in the difference, so FP32 only ever carries the increments, whose
// rounding (relative 6e-8 of the update) is far below the stop test's scale.
// The stop test and the outputs are as in the FP64 form.
template <int DIM, int N, class PDE, bool TEMPS, int MINB, bool MIXED = false, int TS = 1, bool TM = false>
__global__ void __launch_bounds__(LinesCfg<DIM, N, PDE, MINB, MIXED, TS, TM>::THREADS, MINB)
    predictor_lines_kernel(const double* __restrict__ luh, double* __restrict__ lQhbnd, double* __restrict__ lFhbnd,
                           double* __restrict__ lduh, int* __restrict__ iters, const double* __restrict__ dt_ptr,
                           Geometry geo, int ncells, const int* __restrict__ cell_list, PredictorTemps tmp,
                           const int* __restrict__ count) {
  using C = LinesCfg<DIM, N, PDE, MINB, MIXED, TS, TM>;
  static_assert(!MIXED || TS == 1, "the mixed form works one slice at a time");
  static_assert(!TM || !TEMPS, "the tensor-memory form writes no temporaries");
  constexpr int b = C::b, P = C::P, nV = C::nV, nD = C::nD, LINES = C::LINES, QS = C::QS;
  extern __shared__ double smem[];
  const OrderTables& T = c_tab[N];

  // a device-side count that leaves this block without cells: the whole
  // block returns before its first barrier (a gated launch costs little)
  if (count && (int)blockIdx.x * C::CPB >= min(*count, ncells)) return;
  const int lc = TM ? min((int)threadIdx.x / P, C::CPB - 1) : threadIdx.x / P;
  const int p = threadIdx.x - lc * P;
  const bool nd_ok = !TM || p < P;  // TM: the threads past the last node hold none
  constexpr bool kTMany = TM && C::CPB > 1;  // tensor memory, several cells per block
  // TM: the CTA's tensor memory (warp 0 allocates it here and frees it after
  // the last read of the iterate)
  const int warp = threadIdx.x >> 5;
  constexpr bool tm = TM;
  __shared__ uint32_t s_tbase;
  uint32_t taddr = 0;
  if constexpr (TM) {
    if (warp == 0) tmem::alloc(&s_tbase, C::TCOLS);
    tmem::fence_before_sync();
    __syncthreads();
    tmem::fence_after_sync();
    taddr = s_tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(C::TCOL * (warp >> 2));
  }
  const int slot = blockIdx.x * C::CPB + lc;
  const bool active = slot < (count ? min(*count, ncells) : ncells);  // count: optional device-side list length
  const int cell = active ? (cell_list ? cell_list[slot] : slot) : 0;
  double* sQ = smem + lc * C::SQ;
  double* sQn = sQ + p * QS;  // this node's iterate (not TM)
  double* sF = smem + C::CPB * C::SQ + lc * C::SF;
  double* sR = smem + C::CPB * (C::SQ + C::SF) + lc * C::SR;
  double* sFall = smem + C::CPB * C::SQ;
  // FP32 views (mixed sweeps): the slices at the same offsets in float units
  // (a cell's float slice is its double slice's first half), the updates
  float* sF32 = reinterpret_cast<float*>(sF);
  float* sFall32 = reinterpret_cast<float*>(sFall);
  float* sD = reinterpret_cast<float*>(smem + C::CPB * (C::SQ + C::SF + C::SR) + lc * C::SD);

  // quadrature weights in shared memory: phase-B threads index them by line,
  // which would serialise on the constant cache
  __shared__ double s_w[b];
  if (threadIdx.x < b) s_w[threadIdx.x] = T.w[threadIdx.x];
  const int x = p % b, y = (p / b) % b, z = DIM == 3 ? p / (b * b) : 0;
  const double wx = T.w[x], wy = T.w[y], wz = DIM == 3 ? T.w[z] : 1.0;
  const double wpt = wz * wy * wx;
  const double iw = 1.0 / wpt;
  const int inst = cell_instance(geo, cell);
  const double dt = dt_ptr[inst];
  const double invDx0 = 1.0 / cell_width(geo, inst, 0), invDx1 = 1.0 / cell_width(geo, inst, 1);
  const double invDx2 = DIM == 3 ? 1.0 / cell_width(geo, inst, 2) : 0.0;
  // step size and inverse widths of every cell of the block (phase-B items
  // and the epilogue work on other cells of the block than their thread's)
  __shared__ double s_dt[C::CPB], s_idx[C::CPB][3];
  if (p == 0) {
    s_dt[lc] = dt;
    s_idx[lc][0] = invDx0;
    s_idx[lc][1] = invDx1;
    s_idx[lc][2] = invDx2;
  }
  // this node's slot in each direction's part of a slice (+ v)
  int sa[DIM];
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    int n, L;
    node_line<DIM, b>(d, z, y, x, n, L);
    sa[d] = C::sbase(d) + n * C::sstride(d) + line_swapped<b>(C::sswap(d), L) * nV;
  }

  // slice t of this node's iterate: load (nD values), store (the nV variables
  // the iteration updates; the parameters keep their initial values)
  auto q_ld = [&](int t, double* Q) {
    if (tm) {
      uint32_t r[10];
      tmem::ld10(taddr + 10u * t, r);
      tmem::wait_ld(r);
      tmem::unpack5(r, Q);
    } else {
#pragma unroll
      for (int v = 0; v < nD; v++) Q[v] = sQn[t * nD + v];
    }
  };
  auto q_st = [&](int t, const double* Q) {
    if (tm) {
      uint32_t r[10];
      tmem::pack5(Q, r);
      tmem::st10(taddr + 10u * t, r);
    } else {
#pragma unroll
      for (int v = 0; v < nV; v++) sQn[t * nD + v] = Q[v];
    }
  };

  double lu[nV];
  {
    const double* src = luh + ((size_t)cell * P + p) * nD;
    double q[nD];
#pragma unroll
    for (int v = 0; v < nD; v++) q[v] = active && nd_ok ? __ldg(src + v) : 0.0;
#pragma unroll
    for (int v = 0; v < nV; v++) lu[v] = q[v];
#pragma unroll
    for (int t = 0; t < b; t++) {
      if (tm) {
        q_st(t, q);  // nD == nV
      } else {
#pragma unroll
        for (int v = 0; v < nD; v++) sQn[t * nD + v] = q[v];
      }
    }
    if (tm) tmem::wait_st();
  }

  // Which cells of the block still iterate; phase B skips converged cells.
  __shared__ int s_done[C::CPB];
  if (p == 0) s_done[lc] = !active;
  __syncthreads();  // s_w
  // this thread's phase-B items (direction, line, variable): slice offset,
  // cell, and the line's quadrature factor w_a w_c dt / dx_d (times w_t later)
  // (their slab offsets are recomputed where used: kept in registers next to
  // these factors they spill)
  double it_us[C::IPT];
#pragma unroll
  for (int k = 0; k < C::IPT; k++) {
    const int it = threadIdx.x + k * C::THREADS;
    it_us[k] = 0.0;
    if (it < C::ITEMS) {
      const int L = (it / nV) % LINES;  // slab order; the factor is symmetric in the two coordinates
      const int d = (it / (nV * LINES)) % DIM;
      const int c = it / (nV * LINES * DIM);
      const int a0 = L / b, a1 = L % b;
      it_us[k] = (DIM == 3 ? s_w[a0] : 1.0) * s_w[a1] * s_dt[c] * s_idx[c][d];
    }
  }

  bool done = !active;
  int it_done = 0;
  for (int iter = 0; iter < C::maxIter; iter++) {
    const bool low = MIXED && iter > 0;  // an FP32 increment sweep
    double qn[b][nV];  // the new iterate (FP64 sweep) or the update (increment sweep)
#pragma unroll
    for (int l = 0; l < b; l++)
#pragma unroll
      for (int v = 0; v < nV; v++) qn[l][v] = 0.0;

    // The first sweep starts from the trivial guess lQi(:,t) = luh for every
    // t, so its fluxes and their contractions are the same in every time
    // slice: phases A and B run once (slice 0, without the w_t factor) and
    // phase C of every slice reads that one result, scaled by w_t (no
    // barrier is needed between those phase-C passes: nothing writes sF).
    const bool first = iter == 0;
    for (int t0 = 0; t0 < b; t0 += TS) {
      const bool reuse = first && t0 > 0;  // block-uniform
      // phase C of the previous slices is done with sF (at t0 = 0 the
      // prologue's or the residual's barriers already ordered that)
      if (!reuse && t0 > 0) __syncthreads();
      // A: fluxes of slices t0 .. t0+TS-1, line-major, slice j in buffer j
      if (reuse) {
      } else if (!done && low) {  // flux increments in FP64, stored as FP32
        const int t = t0;
        double Q[nD], Qp[nD];
#pragma unroll
        for (int v = 0; v < nD; v++) Q[v] = Qp[v] = sQn[t * nD + v];
#pragma unroll
        for (int v = 0; v < nV; v++) Qp[v] -= (double)sD[(p * b + t) * nV + v];
        double Fl[DIM][nV], Fp[DIM][nV];
        PDE::template flux<DIM>(Q, Fl);
        PDE::template flux<DIM>(Qp, Fp);
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int v = 0; v < nV; v++)
            sF32[sa[d] + v] = (float)(Fl[d][v] - Fp[d][v]);
      } else if (kTMany || !done) {
#pragma unroll
        for (int j = 0; j < TS; j++) {
          const int t = t0 + j;
          if (t < b && !(first && j > 0)) {
            double Q[nD];
            q_ld(t, Q);  // kTMany: by every thread, the conditions are block-uniform
            if (!nd_ok || done) continue;
            double Fl[DIM][nV];
            PDE::template flux<DIM>(Q, Fl);
#pragma unroll
            for (int d = 0; d < DIM; d++)
#pragma unroll
              for (int v = 0; v < nV; v++) sF[j * C::SFJ + sa[d] + v] = Fl[d][v];
          }
        }
      }
      if (!reuse) __syncthreads();
      // B: line contractions, in place
#pragma unroll
      for (int k = 0; k < C::IPT; k++) {
        const int it = threadIdx.x + k * C::THREADS;
        if (reuse || it >= C::ITEMS) continue;
        const int ic = it / (nV * LINES * DIM);
        if (s_done[ic]) continue;
        const int id = (it / (nV * LINES)) % DIM;
        const int is = C::sstride(id);
        const int io = ic * C::SF + C::sbase(id) + it % (nV * LINES);
        if (low) {
          const int t = t0;
          float* base = sFall32 + io + ic * C::SF;
          float f[b];
#pragma unroll
          for (int n = 0; n < b; n++) f[n] = base[n * is];
          const float us = (float)(T.w[t] * it_us[k]);
#pragma unroll
          for (int l = 0; l < b; l++) {
            float s = 0.0f;
#pragma unroll
            for (int n = 0; n < b; n++) s = fmaf(f[n], T.Kxi_f[n * b + l], s);
            base[l * is] = us * s;
          }
          continue;
        }
#pragma unroll
        for (int j = 0; j < TS; j++) {
          const int t = t0 + j;
          if (t >= b || (first && j > 0)) break;
          double* base = sFall + io + j * C::SFJ;
          double f[b];
#pragma unroll
          for (int n = 0; n < b; n++) f[n] = base[n * is];
          const double us = first ? it_us[k] : T.w[t] * it_us[k];
          if constexpr (b % 2 == 0) {  // even and odd parts (OrderTables::KxiP/KxiQ)
            constexpr int h = b / 2;
            double fp[h], fm[h];
#pragma unroll
            for (int n = 0; n < h; n++) {
              fp[n] = f[n] + f[b - 1 - n];
              fm[n] = f[n] - f[b - 1 - n];
            }
#pragma unroll
            for (int l = 0; l < h; l++) {
              double A = 0.0, Bq = 0.0;
#pragma unroll
              for (int n = 0; n < h; n++) {
                A = fma(fp[n], T.KxiP[n * h + l], A);
                Bq = fma(fm[n], T.KxiQ[n * h + l], Bq);
              }
              base[l * is] = us * (Bq + A);
              base[(b - 1 - l) * is] = us * (Bq - A);
            }
          } else {
#pragma unroll
            for (int l = 0; l < b; l++) {
              double s = 0.0;
#pragma unroll
              for (int n = 0; n < b; n++) s = fma(f[n], T.Kxi[n * b + l], s);
              base[l * is] = us * s;
            }
          }
        }
      }
      if (!reuse) __syncthreads();
      // C: rhs at this node, folded into the Picard accumulators
      if (!nd_ok) {
      } else if (!done && low) {  // increment: the rhs0 term cancels
        const int t = t0;
#pragma unroll
        for (int v = 0; v < nV; v++) {
          double rhs = 0.0;
#pragma unroll
          for (int d = 0; d < DIM; d++) rhs -= (double)sF32[sa[d] + v];
          const double ir = iw * rhs;
#pragma unroll
          for (int l = 0; l < b; l++) qn[l][v] = fma(ir, T.iK1[l * b + t], qn[l][v]);
        }
      } else if (!done && first) {  // slices t0 .. t0+TS-1 from the one contraction of F(luh)
#pragma unroll
        for (int j = 0; j < TS; j++) {
          const int t = t0 + j;
          if (t < b) {
            const double r0 = wpt * T.FL[t], wt = T.w[t];
#pragma unroll
            for (int v = 0; v < nV; v++) {
              double sv = 0.0;
#pragma unroll
              for (int d = 0; d < DIM; d++) sv += sF[sa[d] + v];
              const double ir = iw * (r0 * lu[v] - wt * sv);
#pragma unroll
              for (int l = 0; l < b; l++) qn[l][v] = fma(ir, T.iK1[l * b + t], qn[l][v]);
            }
          }
        }
      } else if (!done) {
#pragma unroll
        for (int j = 0; j < TS; j++) {
          const int t = t0 + j;
          if (t < b) {
            const double r0 = wpt * T.FL[t];
#pragma unroll
            for (int v = 0; v < nV; v++) {
              double rhs = r0 * lu[v];
#pragma unroll
              for (int d = 0; d < DIM; d++) rhs -= sF[j * C::SFJ + sa[d] + v];
              const double ir = iw * rhs;
#pragma unroll
              for (int l = 0; l < b; l++) qn[l][v] = fma(ir, T.iK1[l * b + t], qn[l][v]);
            }
          }
        }
      }
    }
    // residual, reduced per cell by one warp
    double part = 0.0;
    if (kTMany || !done) {
#pragma unroll
      for (int l = 0; l < b; l++) {
        double qo[nD];
        if (!low) q_ld(l, qo);
        if (kTMany && done) continue;
#pragma unroll
        for (int v = 0; v < nV; v++) {
          const double dq = low ? qn[l][v] : qn[l][v] - qo[v];
          part = fma(dq, dq, part);
          if (MIXED) sD[(p * b + l) * nV + v] = (float)dq;  // own node only: no barrier needed
        }
      }
    }
    double sq_res;
    if constexpr (TM && C::CPB == 1) {
      // whole warps, one cell: each warp sums its lanes (the threads without
      // a node add zero), one barrier, every thread adds the warp sums in
      // the same order
      constexpr int NW = C::THREADS / 32;
      double acc = nd_ok ? part : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if ((threadIdx.x & 31) == 0) sR[warp] = acc;
      __syncthreads();
      sq_res = 0.0;
#pragma unroll
      for (int w = 0; w < NW; w++) sq_res += sR[w];
    } else {
      if (nd_ok) sR[p] = part;
      __syncthreads();
      {
        constexpr int kFullWarps = C::THREADS / 32;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (warp < kFullWarps) {
          for (int c = warp; c < C::CPB; c += kFullWarps) {
            double* rr = smem + C::CPB * (C::SQ + C::SF) + c * C::SR;
            double acc = 0.0;
            for (int i = lane; i < P; i += 32) acc += rr[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) rr[P] = acc;
          }
        }
      }
      __syncthreads();
      sq_res = sR[P];
    }
    if constexpr (kTMany) {
      // every thread: each slice's old iterate is read and the new one (a
      // finished cell: the old one) written back; a cell that converges now
      // takes the time average of its old fluxes
      const bool conv = !done && (sq_res < 1e-7 * 1e-7 || iter + 1 == C::maxIter);
      if (!done) it_done = iter + 1;
      double fh[DIM][nV];
#pragma unroll
      for (int d = 0; d < DIM; d++)
#pragma unroll
        for (int v = 0; v < nV; v++) fh[d][v] = 0.0;
#pragma unroll
      for (int t = 0; t < b; t++) {
        double Q[nD], W[nD];
        q_ld(t, Q);
#pragma unroll
        for (int v = 0; v < nD; v++) W[v] = done ? Q[v] : qn[t][v];
        q_st(t, W);
        if (conv && nd_ok) {
          double Fl[DIM][nV];
          PDE::template flux<DIM>(Q, Fl);
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int v = 0; v < nV; v++) fh[d][v] += Fl[d][v] * T.w[t];
        }
      }
      if (conv && nd_ok)
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int v = 0; v < nV; v++) sF[sa[d] + v] = fh[d][v];
      if (conv) done = true;
      tmem::wait_st();
    } else if (!done) {
      it_done = iter + 1;
      if (sq_res < 1e-7 * 1e-7 || iter + 1 == C::maxIter) {
        // time-averaged fluxes of this sweep = of the iterate before the
        // update; kept in this node's slots of the cell's slice buffer (which
        // no phase touches again once the cell is done), not in registers
        // that would stay live across the sweeps. Each slice of the new
        // iterate replaces the old one as soon as its flux is taken, so the
        // accumulators, the fluxes and the whole new iterate are never live
        // together (they would spill).
        double fh[DIM][nV];
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int v = 0; v < nV; v++) fh[d][v] = 0.0;
#pragma unroll
        for (int t = 0; t < b; t++) {
          double Q[nD];
          q_ld(t, Q);
          if (low) {
#pragma unroll
            for (int v = 0; v < nV; v++) sQn[t * nD + v] += qn[t][v];
          } else {
            q_st(t, qn[t]);
          }
          if (!nd_ok) continue;
          double Fl[DIM][nV];
          PDE::template flux<DIM>(Q, Fl);
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int v = 0; v < nV; v++) fh[d][v] += Fl[d][v] * T.w[t];
          if (TEMPS) {
            double* dst = tmp.lFi + (((size_t)cell * b + t) * P + p) * (DIM + 1) * nV;
#pragma unroll
            for (int d = 0; d < DIM; d++)
#pragma unroll
              for (int v = 0; v < nV; v++) dst[d * nV + v] = Fl[d][v];
          }
        }
        if (nd_ok)
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int v = 0; v < nV; v++) sF[sa[d] + v] = fh[d][v];
        done = true;
      } else {
#pragma unroll
        for (int l = 0; l < b; l++) {
          if (low) {
#pragma unroll
            for (int v = 0; v < nV; v++) sQn[l * nD + v] += qn[l][v];
          } else {
            q_st(l, qn[l]);
          }
        }
      }
      if (tm) tmem::wait_st();  // the next sweep (or the time average) reads them
    }
    if (p == 0) s_done[lc] = done;
    if constexpr (C::CPB == 1) {  // one cell: every thread read the same sum
      if (done) break;
    } else if (!__syncthreads_or(!done)) {
      break;
    }
  }
  if (iters && active && p == 0) iters[cell] = it_done;

  // time average of lQi (lQhi)
  double qh[nD];
#pragma unroll
  for (int v = 0; v < nD; v++) qh[v] = 0.0;
#pragma unroll
  for (int m = 0; m < b; m++) {
    double Q[nD];
    q_ld(m, Q);
#pragma unroll
    for (int v = 0; v < nD; v++) qh[v] += Q[v] * T.w[m];
  }
  if (TEMPS && active) {
    double* dq = tmp.lQi + ((size_t)cell * P + p) * b * nD;
    for (int i = 0; i < b * nD; i++) dq[i] = sQn[i];
    for (int v = 0; v < nD; v++) tmp.lQhi[((size_t)cell * P + p) * nD + v] = qh[v];
    double* fhd = tmp.lFhi + (size_t)cell * (DIM + 1) * P * nV;
    const int py = DIM == 3 ? (z * b + x) * b + y : x * b + y;
    const int pz = (y * b + x) * b + z;
    for (int v = 0; v < nV; v++) {
      fhd[(0 * P + p) * nV + v] = sF[sa[0] + v];
      fhd[(1 * P + py) * nV + v] = sF[sa[1] + v];
      if (DIM == 3) fhd[(2 * P + pz) * nV + v] = sF[sa[DIM - 1] + v];
      fhd[(DIM * P + p) * nV + v] = 0.0;
    }
  }
  if constexpr (TM) tmem::fence_before_sync();
  __syncthreads();
  if constexpr (TM) {  // every warp has read its iterate (each load waited)
    tmem::fence_after_sync();
    if (warp == 0) tmem::dealloc(s_tbase, C::TCOLS);
  }
  double* sQh = sQ;  // lQhi [P][nD]
#pragma unroll
  for (int v = 0; v < nD; v++)
    if (nd_ok) sQh[p * nD + v] = qh[v];
  if (p == 0) s_done[lc] = !active;
  __syncthreads();

  // extrapolated fluxes and the volume-integral line contractions
  // (transposed stiffness, quadrature factor w_a w_c / dx), in place
  for (int it = threadIdx.x; it < C::ITEMS; it += C::THREADS) {
    const int v = it % nV;
    const int Ls = (it / nV) % LINES;  // slab order
    const int d = (it / (nV * LINES)) % DIM;
    const int c = it / (nV * LINES * DIM);
    if (s_done[c]) continue;
    const int slot_c = blockIdx.x * C::CPB + c;
    const int cell_c = cell_list ? cell_list[slot_c] : slot_c;
    const int is = C::sstride(d);
    const int L = line_swapped<b>(C::sswap(d), Ls);  // face-node order
    double* base = sFall + c * C::SF + C::sbase(d) + Ls * nV + v;
    double f[b];
#pragma unroll
    for (int n = 0; n < b; n++) f[n] = base[n * is];
    double sl = 0.0, sr = 0.0;
#pragma unroll
    for (int l = 0; l < b; l++) {
      sl += f[l] * T.FL[l];
      sr += f[l] * T.FR[l];
    }
    lFhbnd[(((size_t)cell_c * 2 * DIM + 2 * d) * LINES + L) * nV + v] = sl;
    lFhbnd[(((size_t)cell_c * 2 * DIM + 2 * d + 1) * LINES + L) * nV + v] = sr;
    const int a0 = L / b, a1 = L % b;
    const double us = (DIM == 3 ? s_w[a0] : 1.0) * s_w[a1] * s_idx[c][d];
#pragma unroll
    for (int k = 0; k < b; k++) {
      double s = 0.0;
#pragma unroll
      for (int m = 0; m < b; m++) s = fma(T.Kxi[k * b + m], f[m], s);
      base[k * is] = s * us;
    }
  }
  // extrapolated states from lQhi lines
  constexpr int QITEMS = C::CPB * DIM * LINES * nD;
  for (int it = threadIdx.x; it < QITEMS; it += C::THREADS) {
    const int v = it % nD;
    const int L = (it / nD) % LINES;
    const int d = (it / (nD * LINES)) % DIM;
    const int c = it / (nD * LINES * DIM);
    if (s_done[c]) continue;
    const int slot_c = blockIdx.x * C::CPB + c;
    const int cell_c = cell_list ? cell_list[slot_c] : slot_c;
    const double* qh_c = smem + c * C::SQ;
    const int a0 = L / b, a1 = L % b;
    const int base = d == 0 ? (a0 * b + a1) * b : d == 1 ? a0 * b * b + a1 : a0 * b + a1;
    const int stride = d == 0 ? 1 : d == 1 ? b : b * b;
    const int bs = DIM == 3 ? base : (d == 0 ? a1 * b : a1);
    double sl = 0.0, sr = 0.0;
#pragma unroll
    for (int l = 0; l < b; l++) {
      const double q = qh_c[(bs + l * stride) * nD + v];
      sl += q * T.FL[l];
      sr += q * T.FR[l];
    }
    lQhbnd[(((size_t)cell_c * 2 * DIM + 2 * d) * LINES + L) * nD + v] = sl;
    lQhbnd[(((size_t)cell_c * 2 * DIM + 2 * d + 1) * LINES + L) * nD + v] = sr;
  }
  __syncthreads();
  if (!lduh) return;
  // the volume integral at this node, staged in the cell's lQi buffer (free
  // now) and written by consecutive threads to consecutive addresses: a
  // node's own nV doubles per thread would make every store instruction a
  // partial write of 32 sectors
  if (active && nd_ok) {
#pragma unroll
    for (int v = 0; v < nV; v++) {
      double du = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; d++) du += sF[sa[d] + v];
      sQ[p * nV + v] = du;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < C::CPB * P * nV; i += C::THREADS) {
    const int c = i / (P * nV), e = i - c * (P * nV);
    if (s_done[c]) continue;
    const int slot_c = blockIdx.x * C::CPB + c;
    const int cell_c = cell_list ? cell_list[slot_c] : slot_c;
    lduh[(size_t)cell_c * P * nV + e] = smem[c * C::SQ + e];
  }
}

}  // namespace exa
