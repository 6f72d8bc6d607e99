// A-posteriori subcell limiter on the GPU: DG <-> FV projections, DMP and
// admissibility, MUSCL-Hancock FV update of limited cells, FV halo exchange
// and the limiter status machine, for the Euler PDE (nV = 5, no parameters).
//
// Reference semantics (cited per kernel): kernels/limiter/generic/c/Limiter.cpp,
// kernels/finitevolumes/musclhancock/c/{2d,3d}/musclhancock.cpph,
// kernels/finitevolumes/commons/c/commons.cpph and the sequencing of
// exahype/solvers/LimitingADERDGSolver.cpp.
//
// FV patches: lim[cell][(z)][y][x][nV], E = 2N+1+2g cells per axis, g = 2 ghost
// layers; the ghost corners stay zero (never written by the halo exchange).
// Per-cell status data: s (limiter status), s_prev, cure counter, facewise
// statuses fs[2d], has_lim (patch allocated), DMP blocks minB/maxB[2d][nV].
#pragma once
#include <type_traits>

#include "aderdg.cuh"

namespace exa {

constexpr int kGW = 2;  // ghost layer width (GenericFiniteVolumesMUSCLHancockInC.java:12)

template <int DIM, int N>
struct LimShape {
  static constexpr int b = N + 1;
  static constexpr int B = 2 * N + 1;
  static constexpr int E = B + 2 * kGW;
  static constexpr int P = ipow(b, DIM);
  static constexpr int PB = ipow(B, DIM);   // subcells
  static constexpr int PE = ipow(E, DIM);   // patch cells incl. ghosts
  static constexpr int nV = 5;
  static constexpr int LS = PE * nV;        // doubles per patch
};

struct LimParams {
  int A, T, cure_steps;  // activeFV = h+1, troubled = 2h+1, steps-till-cured
  double relax, scale;   // DMP delta0 and epsilon
};

// patch index of interior subcell (z,y,x) (0-based in [0,B))
template <int DIM, int N>
__device__ __forceinline__ int lim_index(int z, int y, int x) {
  using L = LimShape<DIM, N>;
  return DIM == 3 ? (((z + kGW) * L::E + y + kGW) * L::E + x + kGW) : ((y + kGW) * L::E + x + kGW);
}

// ---------------------------------------------------------------------------
// The threads that process one cell: a whole block, or one warp of a block
// that holds several cells (small 2D cells, where block-wide barriers would
// dominate the little work per cell).
struct BlockGroup {
  __device__ static int tid() { return threadIdx.x; }
  __device__ static int size() { return blockDim.x; }
  __device__ static int index() { return 0; }
  __device__ static void sync() { __syncthreads(); }
};
struct WarpGroup {
  __device__ static int tid() { return threadIdx.x & 31; }
  __device__ static int size() { return 32; }
  __device__ static int index() { return threadIdx.x >> 5; }
  __device__ static void sync() { __syncwarp(); }
};

// Copies src[0..n) to dst[0..n), eight loads per thread in flight before the
// stores (dst may be shared memory).
template <class G>
__device__ __forceinline__ void copy_group(double* __restrict__ dst, const double* __restrict__ src, int n) {
  constexpr int K = 8;
  for (int i0 = G::tid(); i0 < n; i0 += K * G::size()) {
    double x[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int i = i0 + k * G::size();
      if (i < n) x[k] = src[i];
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int i = i0 + k * G::size();
      if (i < n) dst[i] = x[k];
    }
  }
}

// Exchanges the contents of a[0..n) and b[0..n) (the reference swaps a
// patch's solution and previous-solution pointers; here both live in dense
// per-cell arrays). Each thread issues the loads of eight elements of both
// arrays before any store, so that a group of one warp waits on a few
// memory round trips, not one per 32 elements.
template <class G>
__device__ __forceinline__ void swap_group(double* __restrict__ a, double* __restrict__ b, int n) {
  constexpr int K = 8;
  for (int i0 = G::tid(); i0 < n; i0 += K * G::size()) {
    double x[K], y[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int i = i0 + k * G::size();
      if (i < n) {
        x[k] = a[i];
        y[k] = b[i];
      }
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int i = i0 + k * G::size();
      if (i < n) {
        a[i] = y[k];
        b[i] = x[k];
      }
    }
  }
}

// Separable tensor-product maps for one cell, executed by one thread group.
// out[o1..][v] = sum_in src[in..][v] prod_d M[in_d][o_d], M row-major [IN][OUT].
// Summation is per axis (x, then y, then z) rather than the reference's single
// triple loop; the difference is at round-off level.
template <int DIM, int IN, int OUT, class G = BlockGroup, class Src, class Dst>
__device__ void tensor_map(Src src, Dst dst, const double* M, double* tmp) {
  constexpr int nV = 5;
  if constexpr (DIM == 2 && std::is_same<G, WarpGroup>::value) {
    // one warp: a lane per (row, column) pair with the 5 variables unrolled,
    // so that the index arithmetic is paid once per pair and dst sees a
    // compile-time variable; every output is the same fma chain, in the same
    // order, as in the generic form below
    for (int i = G::tid(); i < IN * OUT; i += 32) {
      const int xo = i % OUT, y = i / OUT;
      double s[nV];
#pragma unroll
      for (int v = 0; v < nV; v++) s[v] = 0.0;
#pragma unroll
      for (int x = 0; x < IN; x++) {
        const double m = M[x * OUT + xo];
#pragma unroll
        for (int v = 0; v < nV; v++) s[v] += src(0, y, x, v) * m;
      }
#pragma unroll
      for (int v = 0; v < nV; v++) tmp[i * nV + v] = s[v];
    }
    G::sync();
    for (int i = G::tid(); i < OUT * OUT; i += 32) {
      const int xo = i % OUT, yo = i / OUT;
      double s[nV];
#pragma unroll
      for (int v = 0; v < nV; v++) s[v] = 0.0;
#pragma unroll
      for (int y = 0; y < IN; y++) {
        const double m = M[y * OUT + yo];
#pragma unroll
        for (int v = 0; v < nV; v++) s[v] += tmp[(y * OUT + xo) * nV + v] * m;
      }
#pragma unroll
      for (int v = 0; v < nV; v++) dst(0, yo, xo, v, s[v]);
    }
  } else if (DIM == 2) {
    // t[y][xo][v] = sum_x src(y,x,v) M[x][xo]
    for (int i = G::tid(); i < IN * OUT * nV; i += G::size()) {
      const int v = i % nV, xo = (i / nV) % OUT, y = i / (nV * OUT);
      double s = 0.0;
#pragma unroll
      for (int x = 0; x < IN; x++) s += src(0, y, x, v) * M[x * OUT + xo];
      tmp[i] = s;
    }
    G::sync();
    for (int i = G::tid(); i < OUT * OUT * nV; i += G::size()) {
      const int v = i % nV, xo = (i / nV) % OUT, yo = i / (nV * OUT);
      double s = 0.0;
#pragma unroll
      for (int y = 0; y < IN; y++) s += tmp[(y * OUT + xo) * nV + v] * M[y * OUT + yo];
      dst(0, yo, xo, v, s);
    }
  } else {
    double* t1 = tmp;                      // [z][y][xo]
    double* t2 = tmp + IN * IN * OUT * nV;  // [z][yo][xo]
    for (int i = G::tid(); i < IN * IN * OUT * nV; i += G::size()) {
      const int v = i % nV, xo = (i / nV) % OUT, y = (i / (nV * OUT)) % IN, z = i / (nV * OUT * IN);
      double s = 0.0;
#pragma unroll
      for (int x = 0; x < IN; x++) s += src(z, y, x, v) * M[x * OUT + xo];
      t1[i] = s;
    }
    G::sync();
    for (int i = G::tid(); i < IN * OUT * OUT * nV; i += G::size()) {
      const int v = i % nV, xo = (i / nV) % OUT, yo = (i / (nV * OUT)) % OUT, z = i / (nV * OUT * OUT);
      double s = 0.0;
#pragma unroll
      for (int y = 0; y < IN; y++) s += t1[((z * IN + y) * OUT + xo) * nV + v] * M[y * OUT + yo];
      t2[i] = s;
    }
    G::sync();
    for (int i = G::tid(); i < OUT * OUT * OUT * nV; i += G::size()) {
      const int v = i % nV, xo = (i / nV) % OUT, yo = (i / (nV * OUT)) % OUT, zo = i / (nV * OUT * OUT);
      double s = 0.0;
#pragma unroll
      for (int z = 0; z < IN; z++) s += t2[((z * OUT + yo) * OUT + xo) * nV + v] * M[z * OUT + zo];
      dst(zo, yo, xo, v, s);
    }
  }
  G::sync();
}

template <int DIM, int IN, int OUT>
constexpr int tensor_tmp() {
  return DIM == 2 ? IN * OUT * 5 : (IN * IN * OUT + IN * OUT * OUT) * 5;
}

// projectOnFVLimiterSpace (Limiter.cpp:23-66): DG nodes -> interior subcells
template <int DIM, int N, class G = BlockGroup>
__device__ void project_fv_block(const double* luh, double* lim, double* tmp, const double* uh2lim = nullptr) {
  using L = LimShape<DIM, N>;
  tensor_map<DIM, L::b, L::B, G>(
      [&](int z, int y, int x, int v) { return luh[(((DIM == 3 ? z * L::b : 0) + y) * L::b + x) * L::nV + v]; },
      [&](int z, int y, int x, int v, double s) { lim[lim_index<DIM, N>(z, y, x) * L::nV + v] = s; },
      uh2lim ? uh2lim : g_lim_tab[N].uh2lim, tmp);
}
// projectOnDGSpace (Limiter.cpp:69-112): interior subcells -> DG nodes
template <int DIM, int N, class G = BlockGroup>
__device__ void project_dg_block(const double* lim, double* luh, double* tmp) {
  using L = LimShape<DIM, N>;
  tensor_map<DIM, L::B, L::b, G>(
      [&](int z, int y, int x, int v) { return lim[lim_index<DIM, N>(z, y, x) * L::nV + v]; },
      [&](int z, int y, int x, int v, double s) { luh[(((DIM == 3 ? z * L::b : 0) + y) * L::b + x) * L::nV + v] = s; },
      g_lim_tab[N].lim2uh, tmp);
}

// block-wide min/max of 5 variables: each thread passes its partial values
__device__ __forceinline__ void block_minmax5(double* mn, double* mx, double* red /*[2*5*32]*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int v = 0; v < 5; v++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double a = __shfl_xor_sync(0xffffffffu, mn[v], o);
      const double c = __shfl_xor_sync(0xffffffffu, mx[v], o);
      mn[v] = (a < mn[v]) ? a : mn[v];
      mx[v] = (mx[v] < c) ? c : mx[v];
    }
    if (lane == 0) {
      red[v * 32 + warp] = mn[v];
      red[160 + v * 32 + warp] = mx[v];
    }
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int v = 0; v < 5; v++) {
      double a = lane < nw ? red[v * 32 + lane] : __longlong_as_double(0x7fefffffffffffffll);
      double c = lane < nw ? red[160 + v * 32 + lane] : -__longlong_as_double(0x7fefffffffffffffll);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double a2 = __shfl_xor_sync(0xffffffffu, a, o);
        const double c2 = __shfl_xor_sync(0xffffffffu, c, o);
        a = (a2 < a) ? a2 : a;
        c = (c < c2) ? c2 : c;
      }
      if (lane == 0) {
        red[v * 32] = a;
        red[160 + v * 32] = c;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int v = 0; v < 5; v++) {
    mn[v] = red[v * 32];
    mx[v] = red[160 + v * 32];
  }
  __syncthreads();
}

// the same for one warp: shuffles only, every lane ends with the result
__device__ __forceinline__ void warp_minmax5(double* mn, double* mx) {
#pragma unroll
  for (int v = 0; v < 5; v++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double a = __shfl_xor_sync(0xffffffffu, mn[v], o);
      const double c = __shfl_xor_sync(0xffffffffu, mx[v], o);
      mn[v] = (a < mn[v]) ? a : mn[v];
      mx[v] = (mx[v] < c) ? c : mx[v];
    }
}

template <class G>
struct GroupReduce {  // a whole block: through shared memory
  __device__ static void minmax5(double* mn, double* mx, double* red) { block_minmax5(mn, mx, red); }
};
template <>
struct GroupReduce<WarpGroup> {  // one warp: shuffles
  __device__ static void minmax5(double* mn, double* mx, double*) { warp_minmax5(mn, mx); }
};

// ---------------------------------------------------------------------------
// Face merge (mergeSolutionMinMaxOnFace :1654-1690, mergeNeighboursLimiterStatus
// ADERDGSolver.cpp:2544-2595): one thread per interior face. minmax == 0 only
// recomputes the facewise statuses (limiter status spreading).
template <int DIM>
__global__ void lim_merge_faces_kernel(const int* __restrict__ fl, const int* __restrict__ fr,
                                       const int* __restrict__ fd, int nfaces, const int* __restrict__ s,
                                       double* __restrict__ minB, double* __restrict__ maxB, int* __restrict__ fs,
                                       int T, int minmax, const int* __restrict__ gate) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nfaces || (gate && !*gate)) return;
  constexpr int D2 = 2 * DIM;
  const int c1 = fl[f], c2 = fr[f], d = fd[f];
  const int f1 = 2 * d + 1, f2 = 2 * d;
  const int s1 = s[c1], s2 = s[c2];
  const int v = max(0, max(min(s1, T), min(s2, T)) - 1);
  fs[c1 * D2 + f1] = v;
  fs[c2 * D2 + f2] = v;
  if (minmax) {
    double* mn1 = minB + ((size_t)c1 * D2 + f1) * 5;
    double* mn2 = minB + ((size_t)c2 * D2 + f2) * 5;
    double* mx1 = maxB + ((size_t)c1 * D2 + f1) * 5;
    double* mx2 = maxB + ((size_t)c2 * D2 + f2) * 5;
    // all twenty loads before the first store (the four blocks lie in one
    // array each, so the compiler could not move a load above a store)
    double a1[5], a2[5], b1[5], b2[5];
#pragma unroll
    for (int i = 0; i < 5; i++) {
      a1[i] = mn1[i];
      a2[i] = mn2[i];
      b1[i] = mx1[i];
      b2[i] = mx2[i];
    }
#pragma unroll
    for (int i = 0; i < 5; i++) {
      const double mn = (a2[i] < a1[i]) ? a2[i] : a1[i];
      const double mx = (b1[i] < b2[i]) ? b2[i] : b1[i];
      mn1[i] = mn2[i] = mn;
      mx1[i] = mx2[i] = mx;
    }
  }
}

// FV halo exchange (ghostLayerFilling, commons.cpph:336-401 / :873-981) on
// interior faces where either side is FV-active, and the outflow FV boundary
// (boundaryLayerExtraction + boundaryConditions + ghostLayerFillingAtBoundary,
// commons.cpph:98-334) on boundary faces of FV-active cells. One warp per face.
template <int DIM, int N>
__global__ void __launch_bounds__(128) lim_fv_halo_kernel(const int* __restrict__ fl, const int* __restrict__ fr,
                                                          const int* __restrict__ fd, int nfaces,
                                                          const int* __restrict__ bcell, const int* __restrict__ bface,
                                                          int nb, int nb_out, const int* __restrict__ s,
                                                          const int* __restrict__ has_lim, double* __restrict__ lim,
                                                          int A, const int* __restrict__ gate) {
  using L = LimShape<DIM, N>;
  constexpr int E = L::E, B = L::B, nV = L::nV;
  const int lane = threadIdx.x & 31;
  const int f = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (f >= nfaces + nb || (gate && !*gate)) return;
  constexpr int TR = DIM == 3 ? B * B : B;  // transverse subcells of a face
  constexpr int WORK = TR * kGW * nV;
  auto cell_at = [&](int d, int a, int c, int k) {  // (a, c) transverse, k along d
    int z, y, x;
    if (d == 0) { z = a; y = c; x = k; }
    else if (d == 1) { z = a; y = k; x = c; }
    else { z = k; y = a; x = c; }
    return DIM == 3 ? (z * E + y) * E + x : y * E + x;
  };
  const int zr = DIM == 3 ? kGW : 0;
  if (f < nfaces) {
    const int c1 = fl[f], c2 = fr[f], d = fd[f];
    if (!(s[c1] >= A || s[c2] >= A) || !has_lim[c1] || !has_lim[c2]) return;
    double* l1 = lim + (size_t)c1 * L::LS;
    double* l2 = lim + (size_t)c2 * L::LS;
    for (int i = lane; i < WORK; i += 32) {
      const int v = i % nV, k = (i / nV) % kGW, t = i / (nV * kGW);
      const int a = DIM == 3 ? t / B + kGW : (d == 2 ? 0 : zr), c = (DIM == 3 ? t % B : t) + kGW;
      const int aa = DIM == 3 ? a : 0;
      // c1's +d ghosts from c2's first layers; c2's -d ghosts from c1's last layers
      l1[cell_at(d, aa, c, B + kGW + k) * nV + v] = l2[cell_at(d, aa, c, kGW + k) * nV + v];
      l2[cell_at(d, aa, c, k) * nV + v] = l1[cell_at(d, aa, c, B + k) * nV + v];
    }
  } else {
    // boundary faces: the first nb_out outflow, the others rigid walls
    const int bf = f - nfaces, c = bcell[bf], face = bface[bf], d = face >> 1, side = face & 1;
    const bool wall = bf >= nb_out;
    if (!(s[c] >= A) || !has_lim[c]) return;
    double* l = lim + (size_t)c * L::LS;
    for (int i = lane; i < WORK; i += 32) {
      const int v = i % nV, k = (i / nV) % kGW, t = i / (nV * kGW);
      const int a = DIM == 3 ? t / B + kGW : 0, cc = (DIM == 3 ? t % B : t) + kGW;
      // the mirrored layer is the inside state; at 3D y- and z-left faces the
      // reference's boundaryLayerExtraction (commons.cpph:551-562, :581-592)
      // takes the first interior layer for both ghost layers
      const int K = kGW - k - 1;
      const int gi = side ? B + kGW + k : k;
      const int si = side ? B + K : kGW + ((DIM == 3 && d >= 1) ? 0 : K);
      // PDE::fvBoundaryValues: outflow copies it, the wall negates the normal momentum
      const double q = l[cell_at(d, a, cc, si) * nV + v];
      l[cell_at(d, a, cc, gi) * nV + v] = (wall && v == 1 + d) ? -q : q;
    }
  }
}

// ---------------------------------------------------------------------------
// MUSCL-Hancock (2d/musclhancock.cpph:50-276, 3d/musclhancock.cpph) on the
// cells of `list` (length *count when count is given, else nlist; list NULL:
// cells 0..n-1), then projectOnDGSpace of the result into luh (unless NULL). Before the
// update lim_prev <- lim (FiniteVolumesSolver::updateSolution,
// FiniteVolumesSolver.cpp:662-715). Work arrays (evolved boundary states and
// edge fluxes) live in shared memory when they fit, else in a per-block slice
// of global scratch.
template <int DIM, int N>
struct MusclCfg {
  using L = LimShape<DIM, N>;
  static constexpr int R = L::B + 2;  // interior + first ghost ring per axis
  static constexpr int NR = ipow(R, DIM);
  static constexpr int W = NR * DIM * 2 * L::nV;                          // evolved wL/wR
  static constexpr int NE = (L::B + 1) * ipow(L::B, DIM - 1);             // edges per direction
  static constexpr int FX = DIM * NE * L::nV;                             // edge fluxes
  static constexpr int TMP = tensor_tmp<DIM, L::B, L::b>();
  static constexpr int SCR = W + FX;
  static constexpr bool kShared = sizeof(double) * (SCR + TMP + 320) <= 200 * 1024;
  static constexpr size_t SMEM = sizeof(double) * ((kShared ? SCR : 0) + TMP + 320);
  static constexpr int THREADS = 256;
};

__device__ __forceinline__ double minmod_dev(double a, double b) {  // musclhancock.cpph:29-38
  if (a * b < 0.0) return 0.0;
  if (fabs(a) < fabs(b)) return a;
  return b;
}

template <int DIM, class PDE>
__device__ __forceinline__ void dir_flux(const double* q, int d, double* f) {
  double F[DIM][5];
  PDE::template flux<DIM>(q, F);
#pragma unroll
  for (int v = 0; v < 5; v++) f[v] = F[d][v];
}

template <int DIM, int N, class PDE>
__global__ void __launch_bounds__(256) lim_muscl_kernel(const int* __restrict__ list, const int* __restrict__ count,
                                                       int nlist, double* __restrict__ lim, double* __restrict__ lim_prev,
                                                       double* __restrict__ luh, Geometry geo,
                                                       const double* __restrict__ dt_ptr, double* __restrict__ gscratch,
                                                       const int* __restrict__ gate) {
  using L = LimShape<DIM, N>;
  using C = MusclCfg<DIM, N>;
  constexpr int E = L::E, B = L::B, nV = L::nV, R = C::R;
  if (gate && !*gate) return;
  extern __shared__ double smem[];
  double* tmp = smem;
  double* scr = C::kShared ? smem + C::TMP + 320 : gscratch + (size_t)blockIdx.x * C::SCR;
  double* W = scr;
  double* FX = scr + C::W;
  const double dt = *dt_ptr;
  double cs[3], ics[3], icsdt[3];
  for (int d = 0; d < DIM; d++) {
    cs[d] = geo.dx[d] / B;
    ics[d] = 1. / cs[d];
    icsdt[d] = dt * ics[d];
  }
  const int n = count ? *count : nlist;
  for (int li = blockIdx.x; li < n; li += gridDim.x) {
    const int cell = list ? list[li] : li;
    double* l = lim + (size_t)cell * L::LS;
    double* lp = lim_prev + (size_t)cell * L::LS;
    for (int i = threadIdx.x; i < L::LS; i += blockDim.x) lp[i] = l[i];
    __syncthreads();
    auto U = [&](int z, int y, int x, int v) {
      return lp[((DIM == 3 ? z * E : 0) + y) * E * nV + x * nV + v];
    };
    // slopes, extrapolation and half-step evolution on interior + first ghost ring
    for (int q = threadIdx.x; q < C::NR; q += blockDim.x) {
      const int x = q % R + kGW - 1, y = (q / R) % R + kGW - 1, z = DIM == 3 ? q / (R * R) + kGW - 1 : 0;
      double wl[DIM][5], wr[DIM][5];
#pragma unroll
      for (int v = 0; v < nV; v++) {
        const double u = U(z, y, x, v);
        const double sx = minmod_dev(U(z, y, x + 1, v) - u, u - U(z, y, x - 1, v)) * ics[0];
        wl[0][v] = u - 0.5 * cs[0] * sx;
        wr[0][v] = u + 0.5 * cs[0] * sx;
        const double sy = minmod_dev(U(z, y + 1, x, v) - u, u - U(z, y - 1, x, v)) * ics[1];
        wl[1][v] = u - 0.5 * cs[1] * sy;
        wr[1][v] = u + 0.5 * cs[1] * sy;
        if (DIM == 3) {
          const double sz = minmod_dev(U(z + 1, y, x, v) - u, u - U(z - 1, y, x, v)) * ics[DIM - 1];
          wl[DIM - 1][v] = u - 0.5 * cs[DIM - 1] * sz;
          wr[DIM - 1][v] = u + 0.5 * cs[DIM - 1] * sz;
        }
      }
      double Qt[5] = {0, 0, 0, 0, 0};
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        double f[5];
        dir_flux<DIM, PDE>(wl[d], d, f);
#pragma unroll
        for (int v = 0; v < nV; v++) Qt[v] += f[v] * ics[d];
        dir_flux<DIM, PDE>(wr[d], d, f);
#pragma unroll
        for (int v = 0; v < nV; v++) Qt[v] -= f[v] * ics[d];
      }
#pragma unroll
      for (int d = 0; d < DIM; d++)
#pragma unroll
        for (int v = 0; v < nV; v++) {
          W[((q * DIM + d) * 2 + 0) * nV + v] = wl[d][v] + 0.5 * dt * Qt[v];
          W[((q * DIM + d) * 2 + 1) * nV + v] = wr[d][v] + 0.5 * dt * Qt[v];
        }
    }
    __syncthreads();
    // Rusanov flux on every subcell edge (rusanov.cpph): edge e of direction d
    // joins positions k and k+1 along d, k in [-1, B) relative to the interior
    for (int i = threadIdx.x; i < DIM * C::NE; i += blockDim.x) {
      const int d = i / C::NE, e = i % C::NE;
      const int k = e % (B + 1) - 1, t = e / (B + 1);
      const int a = DIM == 3 ? t / B : 0, c = DIM == 3 ? t % B : t;  // transverse interior coordinates
      int pl[3], pr[3];  // (z,y,x) ring coordinates (ring index 0 = first ghost layer)
      if (d == 0) { pl[0] = a + 1; pl[1] = c + 1; pl[2] = k + 1; }
      else if (d == 1) { pl[0] = a + 1; pl[1] = k + 1; pl[2] = c + 1; }
      else { pl[0] = k + 1; pl[1] = a + 1; pl[2] = c + 1; }
      pr[0] = pl[0]; pr[1] = pl[1]; pr[2] = pl[2];
      pr[2 - d] += 1;
      if (DIM == 2) { pl[0] = 0; pr[0] = 0; }
      const int qL = ((DIM == 3 ? pl[0] * R : 0) + pl[1]) * R + pl[2];
      const int qR = ((DIM == 3 ? pr[0] * R : 0) + pr[1]) * R + pr[2];
      const double* ql = W + ((qL * DIM + d) * 2 + 1) * nV;  // wR of the left subcell
      const double* qr = W + ((qR * DIM + d) * 2 + 0) * nV;  // wL of the right subcell
      double lL[5], lR[5];
      Hooks<PDE, DIM>::eigenvalues(ql, d, lL);
      Hooks<PDE, DIM>::eigenvalues(qr, d, lR);
      double smax = -1.0;
#pragma unroll
      for (int v = 0; v < nV; v++) smax = (fabs(lL[v]) < smax) ? smax : fabs(lL[v]);
#pragma unroll
      for (int v = 0; v < nV; v++) smax = (fabs(lR[v]) < smax) ? smax : fabs(lR[v]);
      double fLq[5], fRq[5];
      dir_flux<DIM, PDE>(ql, d, fLq);
      dir_flux<DIM, PDE>(qr, d, fRq);
#pragma unroll
      for (int v = 0; v < nV; v++) {
        double fn = 0.5 * smax * (ql[v] - qr[v]);
        fn += 0.5 * (fLq[v] + fRq[v]);
        FX[i * nV + v] = fn;
      }
    }
    __syncthreads();
    // update of the interior subcells in the reference's accumulation order:
    // +left x edge, -right x edge, then y, then z
    for (int i = threadIdx.x; i < L::PB * nV; i += blockDim.x) {
      const int v = i % nV, sc = i / nV;
      const int x = sc % B, y = (sc / B) % B, z = DIM == 3 ? sc / (B * B) : 0;
      double u = U(z + (DIM == 3 ? kGW : 0), y + kGW, x + kGW, v);
      // edge index within direction d: (transverse t, k) with k = position + 1 for the left edge
      {
        const int t = DIM == 3 ? z * B + y : y;
        u += icsdt[0] * FX[((0 * C::NE) + t * (B + 1) + x) * nV + v];
        u -= icsdt[0] * FX[((0 * C::NE) + t * (B + 1) + x + 1) * nV + v];
      }
      {
        const int t = DIM == 3 ? z * B + x : x;
        u += icsdt[1] * FX[((1 * C::NE) + t * (B + 1) + y) * nV + v];
        u -= icsdt[1] * FX[((1 * C::NE) + t * (B + 1) + y + 1) * nV + v];
      }
      if (DIM == 3) {
        const int t = y * B + x;
        u += icsdt[DIM - 1] * FX[(((DIM - 1) * C::NE) + t * (B + 1) + z) * nV + v];
        u -= icsdt[DIM - 1] * FX[(((DIM - 1) * C::NE) + t * (B + 1) + z + 1) * nV + v];
      }
      l[lim_index<DIM, N>(z, y, x) * nV + v] = u;
    }
    // the reference's edge loops also touch the first ghost layer on every
    // face (one edge each); the ghost corners stay untouched
    for (int i = threadIdx.x; i < DIM * 2 * ipow(B, DIM - 1) * nV; i += blockDim.x) {
      const int v = i % nV, t = (i / nV) % ipow(B, DIM - 1), side = (i / (nV * ipow(B, DIM - 1))) % 2;
      const int d = i / (nV * ipow(B, DIM - 1) * 2);
      const int a = DIM == 3 ? t / B + kGW : 0, c = (DIM == 3 ? t % B : t) + kGW;
      const int k = side ? B + kGW : kGW - 1;
      int z, y, x;
      if (d == 0) { z = a; y = c; x = k; }
      else if (d == 1) { z = a; y = k; x = c; }
      else { z = k; y = a; x = c; }
      const int idx = ((DIM == 3 ? z * E : 0) + y) * E + x;
      const double f = FX[((d * C::NE) + t * (B + 1) + (side ? B : 0)) * nV + v];
      if (side)
        l[idx * nV + v] += icsdt[d] * f;
      else
        l[idx * nV + v] -= icsdt[d] * f;
    }
    __syncthreads();
    if (luh) project_dg_block<DIM, N>(l, luh + (size_t)cell * L::P * nV, tmp);
  }
}

// ---------------------------------------------------------------------------
// Status bookkeeping kernels, one block per cell.

template <int DIM, int N>
struct PostCfg {
  using L = LimShape<DIM, N>;
  static constexpr int TMP = tensor_tmp<DIM, L::b, L::B>() > tensor_tmp<DIM, L::b, L::b>()
                                 ? tensor_tmp<DIM, L::b, L::B>() : tensor_tmp<DIM, L::b, L::b>();
  static constexpr int THREADS = 128;
  static constexpr size_t SMEM = sizeof(double) * (TMP + 320);
  // the post-update kernel of 2D meshes runs one warp per cell, 4 per block
  static constexpr bool kWarp = DIM == 2;
  using Group = typename std::conditional<kWarp, WarpGroup, BlockGroup>::type;
  static constexpr int CELLS = kWarp ? THREADS / 32 : 1;
  // per cell: tensor-map scratch, reduction slots, the staged DG solution and
  // the two projection tables
  static constexpr int STAGE = L::P * L::nV + L::b * L::b + L::b * L::B;
  static constexpr int PER = TMP + 320 + STAGE;
  static constexpr size_t POST_SMEM = sizeof(double) * CELLS * PER;
};

// Min/max of the observables (the conserved variables) over the
// Gauss-Legendre nodes, the Gauss-Lobatto nodes and the subcell centres of one
// cell (findCellLocalMinAndMax + compareWithADERDGSolutionAtGaussLobattoNodes +
// compareWithADERDGSolutionAtFVSubcellCenters, Limiter.cpp:210-368). Block-wide;
// every thread ends with the cell's values in mn/mx.
template <int DIM, int N, class G = BlockGroup>
__device__ void local_minmax_block(const double* u, double* mn, double* mx, double* tmp, double* red,
                                   const double* uh2lob, const double* uh2lim) {
  using L = LimShape<DIM, N>;
  constexpr int nV = L::nV;
#pragma unroll
  for (int v = 0; v < 5; v++) {
    mn[v] = __longlong_as_double(0x7fefffffffffffffll);
    mx[v] = -mn[v];
  }
  for (int p = G::tid(); p < L::P; p += G::size()) {
#pragma unroll
    for (int v = 0; v < 5; v++) {
      const double q = u[p * nV + v];
      mn[v] = (q < mn[v]) ? q : mn[v];
      mx[v] = (mx[v] < q) ? q : mx[v];
    }
  }
  // the projected values are folded into the running min/max as they are
  // produced; the variable is selected with compile-time indices so that
  // mn/mx stay in registers
  auto fold = [&](int, int, int, int v, double val) {
#pragma unroll
    for (int w = 0; w < 5; w++)
      if (w == v) {
        mn[w] = (val < mn[w]) ? val : mn[w];
        mx[w] = (mx[w] < val) ? val : mx[w];
      }
  };
  auto src = [&](int z, int y, int x, int v) { return u[(((DIM == 3 ? z * L::b : 0) + y) * L::b + x) * nV + v]; };
  tensor_map<DIM, L::b, L::b, G>(src, fold, uh2lob, tmp);
  tensor_map<DIM, L::b, L::B, G>(src, fold, uh2lim, tmp);
  GroupReduce<G>::minmax5(mn, mx, red);
}

// Initial limiter status (updateLimiterStatusAndMinAndMaxAfterSetInitialConditions,
// LimitingADERDGSolver.cpp:1069-1083, determineSolverMinAndMax :1101-1130): the
// local min/max of the initial DG solution into every face block; a cell whose
// values are not physically admissible starts troubled. One block per cell.
template <int DIM, int N, class PDE>
__global__ void __launch_bounds__(128) lim_init_kernel(int ncells, const double* __restrict__ luh, int* __restrict__ s,
                                                       int* __restrict__ s_prev, int* __restrict__ cure,
                                                       int* __restrict__ fs, int* __restrict__ has_lim,
                                                       double* __restrict__ minB, double* __restrict__ maxB,
                                                       LimParams prm) {
  using L = LimShape<DIM, N>;
  using C = PostCfg<DIM, N>;
  constexpr int D2 = 2 * DIM;
  extern __shared__ double smem[];
  const int cell = blockIdx.x;
  if (cell >= ncells) return;
  double mn[5], mx[5];
  local_minmax_block<DIM, N>(luh + (size_t)cell * L::P * L::nV, mn, mx, smem, smem + C::TMP, g_lim_tab[N].uh2lob,
                             g_lim_tab[N].uh2lim);
  if (threadIdx.x == 0) {
    double* mnB = minB + (size_t)cell * D2 * 5;
    double* mxB = maxB + (size_t)cell * D2 * 5;
    for (int i = 0; i < D2; i++)
      for (int v = 0; v < 5; v++) {
        mnB[i * 5 + v] = mn[v];
        mxB[i * 5 + v] = mx[v];
      }
    const bool ok = PDE::isPhysicallyAdmissible(mnB, mxB);
    s[cell] = ok ? 0 : prm.T;
    s_prev[cell] = 0;
    cure[cell] = ok ? 0 : prm.cure_steps + 1;
    has_lim[cell] = 0;
    for (int i = 0; i < D2; i++) fs[cell * D2 + i] = 0;
  }
}

// Limiter patches of the cells with s > 0 after the initial status spreading
// start from the FV solver's own initial condition at the subcell centres
// (fv_ic[cell][B^d][nV], LimitingADERDGSolver::setInitialConditions :745-770),
// or, without one, from the projection of the DG solution. One block per cell.
template <int DIM, int N>
__global__ void __launch_bounds__(128) lim_seed_kernel(int ncells, const int* __restrict__ s,
                                                       const double* __restrict__ luh, const double* __restrict__ fv_ic,
                                                       double* __restrict__ lim) {
  using L = LimShape<DIM, N>;
  extern __shared__ double tmp[];
  const int cell = blockIdx.x;
  if (cell >= ncells || s[cell] <= 0) return;
  double* l = lim + (size_t)cell * L::LS;
  if (fv_ic) {
    const double* src = fv_ic + (size_t)cell * L::PB * L::nV;
    for (int i = threadIdx.x; i < L::PB * L::nV; i += blockDim.x) {
      const int v = i % L::nV, q = i / L::nV;
      const int x = q % L::B, y = (q / L::B) % L::B, z = DIM == 3 ? q / (L::B * L::B) : 0;
      l[lim_index<DIM, N>(z, y, x) * L::nV + v] = src[i];
    }
  } else {
    project_fv_block<DIM, N>(luh + (size_t)cell * L::P * L::nV, l, tmp);
  }
}

// After the cell updates of a step (LimitingADERDGSolver::updateSolution
// :843-908 for 0 < s < A, updateLimiterStatusAndMinAndMaxAfterSolutionUpdate
// :910-937, determineLimiterStatusAfterSolutionUpdate :956-994,
// allocateLimiterPatchAfterSolutionUpdate :939-954): per cell
//   - 0 < s < A: FV copy swapped with its previous and refreshed by projection;
//     s == 0: patch released
//   - admissible step (exact arithmetic) -> *dt_min
//   - DMP over GL, Gauss-Lobatto and subcell values, admissibility, the
//     FV-subcell min/max for FV-active cells, the status machine
//   - an irregular change (a cell with s <= A became troubled) sets *irregular.
// run (optional): the kernel does nothing when it holds 0.
// G: one block per cell (BlockGroup) or one warp per cell, 4 cells per block
// (WarpGroup; 2D).
template <int DIM, int N, class PDE, class G = BlockGroup>
__global__ void __launch_bounds__(128) lim_post_update_kernel(
    int ncells, double* __restrict__ luh, int* __restrict__ s, int* __restrict__ s_prev, int* __restrict__ cure,
    int* __restrict__ fs, int* __restrict__ has_lim, double* __restrict__ minB, double* __restrict__ maxB,
    double* __restrict__ lim, double* __restrict__ lim_prev, Geometry geo, LimParams prm,
    double* __restrict__ dt_min, int* __restrict__ irregular, const int* __restrict__ run = nullptr) {
  using L = LimShape<DIM, N>;
  using C = PostCfg<DIM, N>;
  if (run && !*run) return;
  constexpr int nV = L::nV, D2 = 2 * DIM;
  extern __shared__ double smem[];
  double* tmp = smem + G::index() * C::PER;
  double* red = tmp + C::TMP;
  double* su = red + 320;                  // the cell's DG solution after the update
  double* slob = su + L::P * L::nV;        // uh2lob
  double* slim = slob + L::b * L::b;       // uh2lim
  __shared__ int s_flags_all[4][4];
  int* s_flags = s_flags_all[G::index()];
  const int cell = blockIdx.x * (blockDim.x / G::size()) + G::index();
  if (cell >= ncells) return;
  const int st = s[cell];  // status before the update
  double* u = luh + (size_t)cell * L::P * nV;
  double* l = lim + (size_t)cell * L::LS;
  double* lp = lim_prev + (size_t)cell * L::LS;
  if (G::tid() == 0) {
    s_prev[cell] = st;
    s_flags[0] = has_lim[cell];
  }
  // one warp per cell: the cell's face min/max blocks, facewise statuses and
  // cure counter are loaded now, one value per lane, so that the status
  // machine at the end waits on no global load
  constexpr bool kWarp = std::is_same<G, WarpGroup>::value;
  double pmn = 0.0, pmx = 0.0;
  int pfs = 0, pcure = 0;
  if constexpr (kWarp) {
    const int j = G::tid();
    if (j < D2 * 5) {
      pmn = minB[(size_t)cell * D2 * 5 + j];
      pmx = maxB[(size_t)cell * D2 * 5 + j];
    }
    if (j < D2) pfs = fs[cell * D2 + j];
    if (j == 0) pcure = cure[cell];
  }
  G::sync();
  if (st > 0 && st < prm.A) {
    if (!s_flags[0])
      for (int i = G::tid(); i < L::LS; i += G::size()) l[i] = lp[i] = 0.0;
    G::sync();
    swap_group<G>(l, lp, L::LS);
    G::sync();
    project_fv_block<DIM, N, G>(u, l, tmp, g_lim_tab[N].uh2lim);
    if (G::tid() == 0) has_lim[cell] = 1;
  }
  if (st == 0 && G::tid() == 0) has_lim[cell] = 0;  // ensureNoUnrequiredLimiterPatchIsAllocatedOnComputeCell
  // admissible step of the new solution
  const double invDx0 = __ddiv_rn(1.0, geo.dx[0]), invDx1 = __ddiv_rn(1.0, geo.dx[1]);
  const double invDx2 = DIM == 3 ? __ddiv_rn(1.0, geo.dx[2]) : 0.0;
  // stage the (final) DG solution and the projection tables of this order
  copy_group<G>(su, u, L::P * nV);
  copy_group<G>(slob, g_lim_tab[N].uh2lob, L::b * L::b);
  copy_group<G>(slim, g_lim_tab[N].uh2lim, L::b * L::B);
  G::sync();
  double dtm = __longlong_as_double(0x7fefffffffffffffll);
  for (int p = G::tid(); p < L::P; p += G::size()) {
    const double* q = su + p * nV;
    double den = 0.0;
    den = __dadd_rn(den, __dmul_rn(Hooks<PDE, DIM>::max_abs_eig_exact(q, 0), invDx0));
    den = __dadd_rn(den, __dmul_rn(Hooks<PDE, DIM>::max_abs_eig_exact(q, 1), invDx1));
    if (DIM == 3) den = __dadd_rn(den, __dmul_rn(Hooks<PDE, DIM>::max_abs_eig_exact(q, 2), invDx2));
    const double d = __ddiv_rn(__dmul_rn(0.9, pnpm(N)), den);
    dtm = (d < dtm) ? d : dtm;
  }
  {  // block min of the step
    double m = dtm;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double x = __shfl_xor_sync(0xffffffffu, m, o);
      m = (x < m) ? x : m;
    }
    if ((threadIdx.x & 31) == 0) atomic_min_pos_double(dt_min, m);
  }
  double mn[5], mx[5];
  local_minmax_block<DIM, N, G>(su, mn, mx, tmp, red, slob, slim);
  // FV-subcell min/max of FV-active cells (findCellLocalLimiterMinAndMax, :167-205)
  double fmn[5], fmx[5];
  if (st >= prm.A) {
#pragma unroll
    for (int v = 0; v < 5; v++) {
      fmn[v] = __longlong_as_double(0x7fefffffffffffffll);
      fmx[v] = -fmn[v];
    }
#pragma unroll 4
    for (int i = G::tid(); i < L::PB; i += G::size()) {
      const int x = i % L::B, y = (i / L::B) % L::B, z = DIM == 3 ? i / (L::B * L::B) : 0;
      const double* q = l + lim_index<DIM, N>(z, y, x) * nV;
#pragma unroll
      for (int v = 0; v < 5; v++) {
        fmn[v] = (q[v] < fmn[v]) ? q[v] : fmn[v];
        fmx[v] = (fmx[v] < q[v]) ? q[v] : fmx[v];
      }
    }
    GroupReduce<G>::minmax5(fmn, fmx, red);
  }
  if constexpr (kWarp) {
    // the same as the block form below, lane v < 5 taking variable v
    const int lane = G::tid(), v = lane % 5;
    double mnv = mn[0], mxv = mx[0], fmnv = 0.0, fmxv = 0.0;
#pragma unroll
    for (int w = 1; w < 5; w++)
      if (w == v) {
        mnv = mn[w];
        mxv = mx[w];
      }
    if (st >= prm.A) {
      fmnv = fmn[0];
      fmxv = fmx[0];
#pragma unroll
      for (int w = 1; w < 5; w++)
        if (w == v) {
          fmnv = fmn[w];
          fmxv = fmx[w];
        }
    }
    // discreteMaximumPrincipleAndMinAndMaxSearch (Limiter.cpp:114-165)
    double bmin = __shfl_sync(0xffffffffu, pmn, v), bmax = __shfl_sync(0xffffffffu, pmx, v);
#pragma unroll
    for (int i = 1; i < D2; i++) {
      const double a = __shfl_sync(0xffffffffu, pmn, i * 5 + v), c = __shfl_sync(0xffffffffu, pmx, i * 5 + v);
      bmin = (a < bmin) ? a : bmin;
      bmax = (bmax < c) ? c : bmax;
    }
    double sd = (bmax - bmin) * prm.scale;
    sd = (sd < prm.relax) ? prm.relax : sd;
    const bool okv = !((mnv < (bmin - sd)) || (mxv > (bmax + sd)));
    bool ok = __all_sync(0xffffffffu, lane >= 5 || okv);
    if (ok) ok = PDE::isPhysicallyAdmissible(mn, mx);  // on the new local min/max
    double* mnB = minB + (size_t)cell * D2 * 5;
    double* mxB = maxB + (size_t)cell * D2 * 5;
    if (st >= prm.A) {
      if (lane < D2 * 5) {
        mnB[lane] = fmnv;
        mxB[lane] = fmxv;
      }
    } else if (lane < 5) {
      mnB[v] = mnv;
      mxB[v] = mxv;
      mnB[v + 5] = bmin;
      mxB[v + 5] = bmax;
    }
    int fm = 0;
#pragma unroll
    for (int i = 0; i < D2; i++) fm = max(fm, __shfl_sync(0xffffffffu, pfs, i));
    if (lane < D2) fs[cell * D2 + lane] = 0;
    if (lane == 0) {
      int ns;
      if (!ok) {
        cure[cell] = prm.cure_steps + 1;
        if (!(st > prm.A)) atomicOr(irregular, 1);
        ns = prm.T;
      } else if (st >= prm.T) {
        ns = prm.T;
        int c = pcure - 1;
        if (c == 0) {
          ns = prm.T - 1;
          c = prm.cure_steps + 1;
        }
        cure[cell] = c;
      } else {
        ns = fm;
      }
      s[cell] = ns;
      const int had = (st == 0) ? 0 : (st < prm.A ? 1 : s_flags[0]);
      s_flags[1] = ns;
      s_flags[2] = (ns > 0 && !had);
      if (s_flags[2]) has_lim[cell] = 1;
    }
  } else if (G::tid() == 0) {
    double* mnB = minB + (size_t)cell * D2 * 5;
    double* mxB = maxB + (size_t)cell * D2 * 5;
    // discreteMaximumPrincipleAndMinAndMaxSearch (Limiter.cpp:114-165)
    bool ok = true;
    for (int v = 0; v < 5; v++) {
      double bmin = mnB[v], bmax = mxB[v];
      for (int i = 1; i < D2; i++) bmin = (mnB[i * 5 + v] < bmin) ? mnB[i * 5 + v] : bmin;
      for (int i = 1; i < D2; i++) bmax = (bmax < mxB[i * 5 + v]) ? mxB[i * 5 + v] : bmax;
      double sd = (bmax - bmin) * prm.scale;
      sd = (sd < prm.relax) ? prm.relax : sd;
      if ((mn[v] < (bmin - sd)) || (mx[v] > (bmax + sd))) ok = false;
      mnB[v] = mn[v];
      mxB[v] = mx[v];
      mnB[v + 5] = bmin;
      mxB[v + 5] = bmax;
    }
    if (ok) ok = PDE::isPhysicallyAdmissible(mnB, mxB);  // on the new local min/max
    if (st >= prm.A)
      for (int i = 0; i < D2; i++)
        for (int v = 0; v < 5; v++) {
          mnB[i * 5 + v] = fmn[v];
          mxB[i * 5 + v] = fmx[v];
        }
    int ns;
    if (!ok) {
      cure[cell] = prm.cure_steps + 1;
      if (!(st > prm.A)) atomicOr(irregular, 1);
      ns = prm.T;
    } else if (st >= prm.T) {
      ns = prm.T;
      cure[cell] -= 1;
      if (cure[cell] == 0) {
        ns = prm.T - 1;
        cure[cell] = prm.cure_steps + 1;
      }
    } else {
      ns = 0;
      for (int i = 0; i < D2; i++) ns = max(ns, fs[cell * D2 + i]);
    }
    s[cell] = ns;
    for (int i = 0; i < D2; i++) fs[cell * D2 + i] = 0;
    const int had = (st == 0) ? 0 : (st < prm.A ? 1 : has_lim[cell]);
    s_flags[1] = ns;
    s_flags[2] = (ns > 0 && !had);
    if (s_flags[2]) has_lim[cell] = 1;
  }
  G::sync();
  if (s_flags[2]) {  // newly allocated patch: zeroed; projection for helper cells
    for (int i = G::tid(); i < L::LS; i += G::size()) l[i] = lp[i] = 0.0;
    G::sync();
    if (s_flags[1] < prm.A) project_fv_block<DIM, N, G>(su, l, tmp, slim);
  }
}

// One limiter status spreading sweep, cell part (updateLimiterStatusDuringLimiterStatusSpreading,
// :392-405); one warp per cell (the status by lane 0, a newly required patch
// zeroed by the whole warp). The face part is lim_merge_faces_kernel(minmax = 0).
template <int DIM, int N>
__global__ void lim_spread_cells_kernel(int ncells, int* __restrict__ s, int* __restrict__ cure,
                                        int* __restrict__ fs, int* __restrict__ has_lim, double* __restrict__ lim,
                                        double* __restrict__ lim_prev, LimParams prm, const int* __restrict__ gate) {
  using L = LimShape<DIM, N>;
  constexpr int D2 = 2 * DIM;
  const int c = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (c >= ncells || (gate && !*gate)) return;
  int alloc = 0;
  if (lane == 0) {
    // every load first (one memory round trip), then the status machine
    const int sc = s[c], hl = has_lim[c];
    int fsc[D2];
#pragma unroll
    for (int i = 0; i < D2; i++) fsc[i] = fs[c * D2 + i];
    int ns;
    if (sc < prm.T) {
      ns = 0;
#pragma unroll
      for (int i = 0; i < D2; i++) ns = max(ns, fsc[i]);
    } else {
      ns = prm.T;
      cure[c] = prm.cure_steps + 1;
    }
    s[c] = ns;
#pragma unroll
    for (int i = 0; i < D2; i++) fs[c * D2 + i] = 0;
    alloc = ns > 0 && !hl;
    if (alloc) has_lim[c] = 1;
  }
  if (__shfl_sync(0xffffffffu, alloc, 0)) {
    double* l = lim + (size_t)c * L::LS;
    double* lp = lim_prev + (size_t)c * L::LS;
    for (int i = lane; i < L::LS; i += 32) l[i] = lp[i] = 0.0;
  }
}

// scratch of one cell's projections (either direction)
template <int DIM, int N>
constexpr int proj_tmp() {
  using L = LimShape<DIM, N>;
  return tensor_tmp<DIM, L::b, L::B>() > tensor_tmp<DIM, L::B, L::b>() ? tensor_tmp<DIM, L::b, L::B>()
                                                                         : tensor_tmp<DIM, L::B, L::b>();
}

// reinitialiseSolversLocally (:1329-1360). G: one block per cell, or one
// warp per cell with blockDim.x / 32 cells per block (2D).
template <int DIM, int N, class G = BlockGroup>
__global__ void __launch_bounds__(128) lim_reinit_kernel(int ncells, double* __restrict__ luh,
                                                         double* __restrict__ luh_prev, const int* __restrict__ s,
                                                         const int* __restrict__ s_prev, int* __restrict__ cure,
                                                         int* __restrict__ has_lim, double* __restrict__ lim,
                                                         double* __restrict__ lim_prev, LimParams prm,
                                                         const int* __restrict__ gate) {
  using L = LimShape<DIM, N>;
  extern __shared__ double smem[];
  double* tmp = smem + G::index() * proj_tmp<DIM, N>();
  const int c = blockIdx.x * (blockDim.x / G::size()) + G::index();
  if (c >= ncells || !*gate) return;
  const int st = s[c];
  if (st <= 0) {
    if (G::tid() == 0) has_lim[c] = 0;
    return;
  }
  double* u = luh + (size_t)c * L::P * L::nV;
  double* up = luh_prev + (size_t)c * L::P * L::nV;
  double* l = lim + (size_t)c * L::LS;
  double* lp = lim_prev + (size_t)c * L::LS;
  if (s_prev[c] >= prm.A) {
    swap_group<G>(l, lp, L::LS);
    G::sync();
    project_dg_block<DIM, N, G>(l, u, tmp);
  } else {
    swap_group<G>(u, up, L::P * L::nV);
    G::sync();
    project_fv_block<DIM, N, G>(u, l, tmp);
  }
  if (G::tid() == 0 && st >= prm.T) cure[c] = prm.cure_steps + 1;
}

// recomputeSolutionLocally (:1396-1436) for cells with 0 < s < A, then the
// admissible step of every cell (the FV-active cells were re-updated by
// lim_muscl_kernel just before). G as for lim_reinit_kernel.
template <int DIM, int N, class PDE, class G = BlockGroup>
__global__ void __launch_bounds__(128) lim_recompute_kernel(int ncells, double* __restrict__ luh,
                                                            double* __restrict__ luh_prev, const int* __restrict__ s,
                                                            const int* __restrict__ s_prev, double* __restrict__ lim,
                                                            double* __restrict__ lim_prev, Geometry geo, LimParams prm,
                                                            double* __restrict__ dt_min, const int* __restrict__ gate) {
  using L = LimShape<DIM, N>;
  extern __shared__ double smem[];
  double* tmp = smem + G::index() * proj_tmp<DIM, N>();
  const int c = blockIdx.x * (blockDim.x / G::size()) + G::index();
  if (c >= ncells || !*gate) return;
  const int st = s[c];
  double* u = luh + (size_t)c * L::P * L::nV;
  if (st > 0 && st < prm.A) {
    double* l = lim + (size_t)c * L::LS;
    if (s_prev[c] < prm.A) {
      double* up = luh_prev + (size_t)c * L::P * L::nV;
      swap_group<G>(u, up, L::P * L::nV);
      G::sync();
      project_fv_block<DIM, N, G>(u, l, tmp);
    } else {
      double* lp = lim_prev + (size_t)c * L::LS;
      swap_group<G>(l, lp, L::LS);
      G::sync();
      project_dg_block<DIM, N, G>(l, u, tmp);
    }
  }
  G::sync();
  const double invDx0 = __ddiv_rn(1.0, geo.dx[0]), invDx1 = __ddiv_rn(1.0, geo.dx[1]);
  const double invDx2 = DIM == 3 ? __ddiv_rn(1.0, geo.dx[2]) : 0.0;
  double dtm = __longlong_as_double(0x7fefffffffffffffll);
  for (int p = G::tid(); p < L::P; p += G::size()) {
    const double* q = u + p * L::nV;
    double den = 0.0;
    den = __dadd_rn(den, __dmul_rn(Hooks<PDE, DIM>::max_abs_eig_exact(q, 0), invDx0));
    den = __dadd_rn(den, __dmul_rn(Hooks<PDE, DIM>::max_abs_eig_exact(q, 1), invDx1));
    if (DIM == 3) den = __dadd_rn(den, __dmul_rn(Hooks<PDE, DIM>::max_abs_eig_exact(q, 2), invDx2));
    const double d = __ddiv_rn(__dmul_rn(0.9, pnpm(N)), den);
    dtm = (d < dtm) ? d : dtm;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_xor_sync(0xffffffffu, dtm, o);
    dtm = (x < dtm) ? x : dtm;
  }
  // warps without a node hold DBL_MAX: no atomic
  if ((threadIdx.x & 31) == 0 && (threadIdx.x & ~31) % G::size() < L::P) atomic_min_pos_double(dt_min, dtm);
}

// Batched projections for the kernel-level entry points: one block per listed
// cell (list NULL: cells 0..n-1). to_fv: luh -> interior subcells of lim,
// else interior subcells of lim -> luh.
template <int DIM, int N>
__global__ void __launch_bounds__(128) lim_project_kernel(const int* __restrict__ list, int n,
                                                          double* __restrict__ luh, double* __restrict__ lim,
                                                          int to_fv) {
  using L = LimShape<DIM, N>;
  extern __shared__ double tmp[];
  if ((int)blockIdx.x >= n) return;
  const int c = list ? list[blockIdx.x] : (int)blockIdx.x;
  double* u = luh + (size_t)c * L::P * L::nV;
  double* l = lim + (size_t)c * L::LS;
  if (to_fv)
    project_fv_block<DIM, N>(u, l, tmp);
  else
    project_dg_block<DIM, N>(l, u, tmp);
}

// Compacts the cells whose status satisfies lo <= s < hi into list/count
// (order is irrelevant: every cell is computed independently).
__global__ void lim_select_kernel(int ncells, const int* __restrict__ s, int lo, int hi, int* __restrict__ list,
                                  int* __restrict__ count, const int* __restrict__ gate) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (gate && !*gate) return;
  if (c < ncells && s[c] >= lo && s[c] < hi) list[atomicAdd(count, 1)] = c;
}
// Two such lists from one pass: lo1 <= s < hi1 and lo2 <= s < hi2.
__global__ void lim_select2_kernel(int ncells, const int* __restrict__ s, int lo1, int hi1, int* __restrict__ list1,
                                   int* __restrict__ count1, int lo2, int hi2, int* __restrict__ list2,
                                   int* __restrict__ count2, const int* __restrict__ gate) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (gate && !*gate) return;
  if (c >= ncells) return;
  const int sc = s[c];
  if (sc >= lo1 && sc < hi1) list1[atomicAdd(count1, 1)] = c;
  if (sc >= lo2 && sc < hi2) list2[atomicAdd(count2, 1)] = c;
}

}  // namespace exa
