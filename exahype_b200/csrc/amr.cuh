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

// per order: fineGridProjector1d [third][n][m], the restriction factors
// w_n P[third][m][n] / (3 w_m) as [third][m][n], and
// equidistantGridProjector1d [n][i]
struct AmrTables {
  double fine[3 * kMaxB * kMaxB];
  double restr[3 * kMaxB * kMaxB];
  double equi[kMaxB * kMaxB];
};
__device__ AmrTables g_amr_tab[kMaxOrder + 1];

// applies a 1-D operator along axis AX (0 = fastest) of a tensor with NAX
// axes of length b and NV values per node: out[.., m, ..] =
// sum_n op(m, n) in[.., n, ..]; all threads of the block take part
template <int b, int NAX, int AX, int NV, class Op>
__device__ __forceinline__ void apply_axis(const double* in, double* out, Op op) {
  constexpr int total = NV * ipow(b, NAX), stride = NV * ipow(b, AX);
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int m = (e / stride) % b;
    const int base = e - m * stride;
    double s = 0.0;
#pragma unroll
    for (int n = 0; n < b; n++) s = fma(op(m, n), in[base + n * stride], s);
    out[e] = s;
  }
}

// the operator of each axis in turn (axis k uses ops(k)), ping-ponging
// between the two buffers; returns the buffer holding the result
template <int b, int NAX, int NV, class Ops>
__device__ __forceinline__ double* apply_axes(double* cur, double* nxt, Ops ops) {
  __syncthreads();
  apply_axis<b, NAX, 0, NV>(cur, nxt, ops(0));
  if (NAX == 1) return nxt;
  __syncthreads();
  apply_axis<b, NAX, 1, NV>(nxt, cur, ops(1));
  if (NAX == 2) return cur;
  __syncthreads();
  apply_axis<b, NAX, 2, NV>(cur, nxt, ops(2));
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
  const AmrTables& A = g_amr_tab[N];
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
    const double* tab = restrict_ ? A.restr : A.fine;
    double* res = apply_axes<b, NAX, NV>(cur, nxt, [&](int ax) {
      const double* M = tab + digit[ax] * b * b;
      const bool r = restrict_;
      return [M, r](int m, int n) { return r ? M[m * b + n] : M[n * b + m]; };
    });
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
  const AmrTables& A = g_amr_tab[N];
  for (int e = threadIdx.x; e < P * ND; e += blockDim.x) bufA[e] = luh[(size_t)c * P * ND + e];
  const double* E = A.equi;
  double* cur = apply_axes<b, DIM, ND>(bufA, bufB, [E](int) { return [E](int i, int n) { return E[n * b + i]; }; });
  __syncthreads();
  for (int e = threadIdx.x; e < P * ND; e += blockDim.x) out[(size_t)c * P * ND + e] = cur[e];
}

}  // namespace exa
