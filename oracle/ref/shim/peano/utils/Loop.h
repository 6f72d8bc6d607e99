// Stand-in for Peano's d-dimensional loop, written for the oracle build:
// dfor(i, n) visits every integer vector i with 0 <= i[d] < n, i[0] fastest;
// dLinearisedWithoutLookup(i, n) is sum_d i[d] n^d.
#pragma once
#include "tarch/Assertions.h"
#include "tarch/la/Vector.h"
namespace peano { namespace utils {
template <int D> inline bool dforNext(tarch::la::Vector<D, int>& i, int n) {
  for (int d = 0; d < D; d++) {
    if (++i[d] < n) return true;
    i[d] = 0;
  }
  return false;
}
template <int D> inline int dLinearisedWithoutLookup(const tarch::la::Vector<D, int>& i, int n) {
  int r = 0;
  for (int d = D - 1; d >= 0; d--) r = r * n + i[d];
  return r;
}
}}
#define dfor(i, n)                                                                   \
  for (tarch::la::Vector<DIMENSIONS, int> i(0), i##_end(0); !i##_end[0];            \
       i##_end[0] = !peano::utils::dforNext(i, n))
