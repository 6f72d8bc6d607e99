// Shared device-side definitions: operator tables in constant memory,
// compile-time basis sizes and small helpers.
#pragma once
#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

#include "dg_tables.h"

namespace exa {

constexpr int kMaxOrder = 9;
constexpr int kMaxB = kMaxOrder + 1;

// One order's 1-D operators, in constant memory. Layouts follow the reference
// (kernels/DGMatrices.h:47-80): Kxi[k][l], iK1[l][n], dudx[l][n] row-major
// (dudx: derivative of basis function n at node l, used by the linear
// predictor's spatial gradients).
struct OrderTables {
  double w[kMaxB], x[kMaxB], FL[kMaxB], FR[kMaxB];
  double Kxi[kMaxB * kMaxB], iK1[kMaxB * kMaxB], dudx[kMaxB * kMaxB];
  double lobatto[kMaxB];
  // FP32 copy of Kxi for the mixed-precision Picard sweeps
  float Kxi_f[kMaxB * kMaxB];
  // even b: Kxi is centro-antisymmetric (Kxi[b-1-n][b-1-l] = -Kxi[n][l], the
  // Gauss-Legendre nodes being symmetric), so a line contraction
  // out_l = sum_n f_n Kxi[n][l] splits into the even and odd parts of f:
  // with h = b/2, fp_n = f_n + f_(b-1-n), fm_n = f_n - f_(b-1-n) (n < h),
  // A_l = sum_n fp_n KxiP[n][l], B_l = sum_n fm_n KxiQ[n][l] (l < h):
  // out_l = B_l + A_l, out_(b-1-l) = B_l - A_l, where
  // KxiP[n][l] = (Kxi[n][l] + Kxi[b-1-n][l]) / 2, KxiQ the difference / 2
  double KxiP[(kMaxB / 2) * (kMaxB / 2)], KxiQ[(kMaxB / 2) * (kMaxB / 2)];
};

// Limiter projections of one order, in global memory (they are read by
// whole blocks through shared-memory staging, and the constant bank is kept
// for the predictor's operands).
struct LimiterTables {
  double uh2lim[kMaxB * (2 * kMaxOrder + 1)];  // [k][i]: DG basis k -> subcell i
  double lim2uh[(2 * kMaxOrder + 1) * kMaxB];  // [i][j]: subcell i -> DG basis j
  double uh2lob[kMaxB * kMaxB];                // [j][i]: DG basis j at Lobatto node i
};

// Filled by upload_tables() (capi.cu) when the first solver is created on a
// device. The library is one translation unit, so this is the only definition.
__constant__ OrderTables c_tab[kMaxOrder + 1];
__device__ LimiterTables g_lim_tab[kMaxOrder + 1];

constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

// register cap per thread that lets BLOCKS blocks of THREADS threads be
// resident on one SM: the warps are spread over the 4 sub-partitions, each
// with 16 K registers, allocated in multiples of 8 per thread
template <int THREADS, int BLOCKS>
constexpr int regs_for_blocks() {
  return (16384 / (((BLOCKS * ((THREADS + 31) / 32)) + 3) / 4 * 32)) / 8 * 8 > 255
             ? 255
             : (16384 / (((BLOCKS * ((THREADS + 31) / 32)) + 3) / 4 * 32)) / 8 * 8;
}

// Minimum-stability constants of stableTimeStepSize (kernels/aderdg/generic/c/3d/stableTimeStepSize.cpph:33-34).
__host__ __device__ constexpr double pnpm(int N) {
  return N == 0 ? 1.0 : N == 1 ? 0.33 : N == 2 ? 0.17 : N == 3 ? 0.1 : N == 4 ? 0.069 : N == 5 ? 0.045
       : N == 6 ? 0.038 : N == 7 ? 0.03 : N == 8 ? 0.02 : 0.015;
}

// positive doubles order like their bit patterns: a min-reduction over
// time-step sizes can use an integer atomicMin on the bits.
__device__ __forceinline__ void atomic_min_pos_double(double* addr, double v) {
  atomicMin(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

}  // namespace exa
