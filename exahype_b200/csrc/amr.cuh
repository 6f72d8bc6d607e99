// AMR transfer operators and the plotters' vertex projection on the GPU.
//
//   amr_volume_kernel  volumeUnknownsProlongation / volumeUnknownsRestriction
//                      (kernels/aderdg/generic/c/{2d,3d}/amrRoutines.cpph)
//   amr_face_kernel    faceUnknownsProlongation / faceUnknownsRestriction
//   plot_vertex_kernel the (N+1)^d equidistant vertex values that
//                      ADERDG2CartesianVTK::plotVertexData writes
//                      (exahype/plotters/VTK/ADERDG2CartesianVTK.cpp)
//
// One block per transfer (a fine cell or face and its coarse ancestor,
// levelDelta levels apart, the subcell index holding one base-3 digit per
// level). Per level the tensor-product operator is applied one axis at a
// time in shared memory (the reference sums the full product per output; the
// sums differ in rounding order only): prolongation with
// P[third][n][m] = phi_n((third + x_m)/3) from the coarse level down,
// restriction with w_n P[third][m][n] / (3 w_m) per axis from the fine level
// up. Restrictions add into the coarse data with atomicAdd, so any number of
// descendants can be restricted into one ancestor in one launch (the sum order
// is not fixed).
#pragma once
#include "aderdg.cuh"

namespace exa {

// Operator tables in constant memory, packed over the orders 1..9 (offset of
// order N: sum over lower orders of (N'+1)^2, times 3 for the thirds):
// fineGridProjector1d [third][n][m], the restriction factors
// w_n P[third][m][n] / (3 w_m) as [third][m][n], equidistantGridProjector1d
// [n][i]. A block reads one matrix with block-uniform addresses, so the
// coefficients come from the constant cache by broadcast.
constexpr int amr_off(int N) { return N <= 1 ? 0 : amr_off(N - 1) + N * N; }
constexpr int kAmrSq = amr_off(kMaxOrder + 1);  // sum of (N+1)^2 over N = 1..9
__constant__ double c_amr_fine[3 * kAmrSq];
__constant__ double c_amr_restr[3 * kAmrSq];
__constant__ double c_amr_equi[kAmrSq];

// applies a 1-D operator along axis AX (0 = fastest) of a tensor with NAX
// axes of length b and NV values per node, one thread per line:
// out[.., m, ..] = sum_n M[m][n] in[.., n, ..], M given as a pointer and
// row/column strides (compile-time indices: the coefficients are read
// with uniform addresses); all threads of the block take part
template <int b, int NAX, int AX, int NV, int RS, int CS>
__device__ __forceinline__ void apply_axis(const double* in, double* out, const double* M) {
  constexpr int total = NV * ipow(b, NAX), stride = NV * ipow(b, AX), lines = total / b;
  for (int it = threadIdx.x; it < lines; it += blockDim.x) {
    const int lo = it % stride, hi = it / stride;
    const int base = hi * stride * b + lo;
    double x[b];
#pragma unroll
    for (int n = 0; n < b; n++) x[n] = in[base + n * stride];
#pragma unroll
    for (int m = 0; m < b; m++) {
      double s = 0.0;
#pragma unroll
      for (int n = 0; n < b; n++) s = fma(M[m * RS + n * CS], x[n], s);
      out[base + m * stride] = s;
    }
  }
}

// the operator of each axis in turn (axis k uses mats[k]), ping-ponging
// between the two buffers; returns the buffer holding the result
template <int b, int NAX, int NV, int RS, int CS>
__device__ __forceinline__ double* apply_axes(double* cur, double* nxt, const double* const* mats) {
  __syncthreads();
  apply_axis<b, NAX, 0, NV, RS, CS>(cur, nxt, mats[0]);
  if (NAX == 1) return nxt;
  __syncthreads();
  apply_axis<b, NAX, 1, NV, RS, CS>(nxt, cur, mats[1]);
  if (NAX == 2) return cur;
  __syncthreads();
  apply_axis<b, NAX, 2, NV, RS, CS>(cur, nxt, mats[2]);
  return nxt;
}

// one axis of a single-level transfer: the digit picks the third; each case
// has a compile-time table address, so the coefficients are constant-bank
// operands (prolongation P[n][m], restriction R[m][n])
template <int N, int NAX, int AX, int NV, bool R>
__device__ __forceinline__ void transfer_axis(const double* in, double* out, int digit) {
  constexpr int b = N + 1, base = 3 * amr_off(N), RS = R ? b : 1, CS = R ? 1 : b;
  const double* tab = R ? c_amr_restr : c_amr_fine;
  if (digit == 0)
    apply_axis<b, NAX, AX, NV, RS, CS>(in, out, tab + base);
  else if (digit == 1)
    apply_axis<b, NAX, AX, NV, RS, CS>(in, out, tab + base + b * b);
  else
    apply_axis<b, NAX, AX, NV, RS, CS>(in, out, tab + base + 2 * b * b);
}

template <int N, int NAX, int NV, bool R>
__device__ __forceinline__ double* transfer_level(double* cur, double* nxt, const int* digit) {
  __syncthreads();
  transfer_axis<N, NAX, 0, NV, R>(cur, nxt, digit[0]);
  if (NAX == 1) return nxt;
  __syncthreads();
  transfer_axis<N, NAX, 1, NV, R>(nxt, cur, digit[1]);
  if (NAX == 2) return cur;
  __syncthreads();
  transfer_axis<N, NAX, 2, NV, R>(cur, nxt, digit[2]);
  return nxt;
}

// levelDelta in 1..kMaxLevelDelta and every index digit-string in
// [0, 3^levelDelta): transfers that break this are skipped (no table read
// outside the three thirds)
constexpr int kMaxLevelDelta = 12;
__device__ __forceinline__ bool valid_index(int ld, const int* index, int nax) {
  if (ld < 1 || ld > kMaxLevelDelta) return false;
  int lim = 1;
  for (int l = 0; l < ld; l++) lim *= 3;
  for (int k = 0; k < nax; k++)
    if (index[k] < 0 || index[k] >= lim) return false;
  return true;
}

// one transfer of `nax`-dimensional nodal data (nv values per node) between
// levels: restrict == false prolongates src (coarse) into dst (fine),
// restrict == true restricts src (fine) and adds it to dst (coarse)
template <int N, int NAX, int NV>
__device__ void amr_transfer(const double* __restrict__ src, double* __restrict__ dst, int levelDelta,
                             const int* index, bool restrict_, double* bufA, double* bufB) {
  constexpr int b = N + 1;
  constexpr int size = NV * ipow(b, NAX);
  for (int e = threadIdx.x; e < size; e += blockDim.x) bufA[e] = src[e];
  int rest[3] = {index[0], index[1], index[2]};
  int sig = 1;
  for (int l = 1; l < levelDelta; l++) sig *= 3;
  double* cur = bufA;
  double* nxt = bufB;
  for (int l = 0; l < levelDelta; l++) {
    int digit[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < NAX; k++) {
      if (!restrict_) {  // most significant digit first
        digit[k] = rest[k] / sig;
        rest[k] = rest[k] % sig;
      } else {  // least significant digit first
        digit[k] = rest[k] % 3;
        rest[k] = rest[k] / 3;
      }
    }
    sig = sig > 1 ? sig / 3 : 1;
    double* res = restrict_ ? transfer_level<N, NAX, NV, true>(cur, nxt, digit)
                            : transfer_level<N, NAX, NV, false>(cur, nxt, digit);
    nxt = res == cur ? nxt : cur;
    cur = res;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < size; e += blockDim.x) {
    if (restrict_)
      atomicAdd(dst + e, cur[e]);
    else
      dst[e] = cur[e];
  }
  __syncthreads();  // the buffers may be reused by the caller
}

// op 0: prolongation, 1: restriction. item k: fine cell fine[k], coarse cell
// coarse[k], levelDelta[k], subcell index idx[3k .. 3k+2]
template <int DIM, int N, int ND>
__global__ void __launch_bounds__(256) amr_volume_kernel(double* __restrict__ luh_a, const double* __restrict__ luh_b,
                                                         int n, const int* __restrict__ fine,
                                                         const int* __restrict__ coarse,
                                                         const int* __restrict__ level_delta,
                                                         const int* __restrict__ idx, int op) {
  constexpr int P = ipow(N + 1, DIM);
  __shared__ double bufA[P * ND], bufB[P * ND];
  const int k = blockIdx.x;
  if (k >= n) return;
  const int ld = level_delta[k];
  const int index[3] = {idx[3 * k], idx[3 * k + 1], DIM == 3 ? idx[3 * k + 2] : 0};
  if (!valid_index(ld, index, DIM)) return;
  if (op == 0)  // luh_a: fine (written), luh_b: coarse
    amr_transfer<N, DIM, ND>(luh_b + (size_t)coarse[k] * P * ND, luh_a + (size_t)fine[k] * P * ND, ld, index, false,
                             bufA, bufB);
  else  // luh_a: coarse (added to), luh_b: fine
    amr_transfer<N, DIM, ND>(luh_b + (size_t)fine[k] * P * ND, luh_a + (size_t)coarse[k] * P * ND, ld, index, true,
                             bufA, bufB);
}

// faces: item k moves face slot fine[k] <-> coarse[k] (slot = cell * 2 DIM +
// face) of the state array (ND per node) and the flux array (NV per node)
template <int DIM, int N, int ND, int NV>
__global__ void __launch_bounds__(256) amr_face_kernel(double* __restrict__ q_a, double* __restrict__ f_a,
                                                       const double* __restrict__ q_b, const double* __restrict__ f_b,
                                                       int n, const int* __restrict__ fine,
                                                       const int* __restrict__ coarse,
                                                       const int* __restrict__ level_delta,
                                                       const int* __restrict__ idx, int op) {
  constexpr int F = ipow(N + 1, DIM - 1);
  __shared__ double bufA[F * ND], bufB[F * ND];
  const int k = blockIdx.x;
  if (k >= n) return;
  const int ld = level_delta[k];
  const int index[3] = {idx[2 * k], DIM == 3 ? idx[2 * k + 1] : 0, 0};
  if (!valid_index(ld, index, DIM - 1)) return;
  const bool r = op != 0;
  const size_t from = r ? fine[k] : coarse[k], to = r ? coarse[k] : fine[k];
  amr_transfer<N, DIM - 1, ND>(q_b + from * F * ND, q_a + to * F * ND, ld, index, r, bufA, bufB);
  amr_transfer<N, DIM - 1, NV>(f_b + from * F * NV, f_a + to * F * NV, ld, index, r, bufA, bufB);
}

// the solution of every cell at its (N+1)^d equidistant vertices (x fastest),
// one block per cell
template <int DIM, int N, int ND>
__global__ void __launch_bounds__(256) plot_vertex_kernel(const double* __restrict__ luh, double* __restrict__ out,
                                                          int ncells) {
  constexpr int b = N + 1, P = ipow(b, DIM);
  __shared__ double bufA[P * ND], bufB[P * ND];
  const int c = blockIdx.x;
  if (c >= ncells) return;
  for (int e = threadIdx.x; e < P * ND; e += blockDim.x) bufA[e] = luh[(size_t)c * P * ND + e];
  const double* E = c_amr_equi + amr_off(N);  // E[n][i]: out[i] = sum_n E[n][i] in[n]
  const double* mats[3] = {E, E, E};
  double* cur = apply_axes<b, DIM, ND, 1, b>(bufA, bufB, mats);
  __syncthreads();
  for (int e = threadIdx.x; e < P * ND; e += blockDim.x) out[(size_t)c * P * ND + e] = cur[e];
}

}  // namespace exa
