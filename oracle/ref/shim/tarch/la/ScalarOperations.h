// stand-in for tarch/la/ScalarOperations.h: tolerance compares used in asserts
#pragma once
#include <cmath>
namespace tarch { namespace la {
inline bool equals(double a, double b, double tol = 1e-14) { return std::fabs(a - b) <= tol; }
inline bool greater(double a, double b, double tol = 1e-14) { return a - b > tol; }
inline bool greaterEquals(double a, double b, double tol = 1e-14) { return a - b >= -tol; }
inline bool smaller(double a, double b, double tol = 1e-14) { return b - a > tol; }
}}
