// Minimal stand-in for Peano's tarch::la::Vector, written for the oracle build
// of the reference kernels. Only what the generic ADER-DG / limiter / FV
// kernels touch: element access, a few constructors and scalar arithmetic.
// It carries no numerics of its own beyond plain IEEE + and *.
#pragma once
#include <cmath>
namespace tarch { namespace la {
template <int N, typename T> struct Vector {
  T v[N];
  Vector() { for (int i = 0; i < N; i++) v[i] = T(); }
  explicit Vector(const T& a) { for (int i = 0; i < N; i++) v[i] = a; }
  Vector(const T& a, const T& b) { v[0] = a; if (N > 1) v[1] = b; }
  Vector(const T& a, const T& b, const T& c) { v[0] = a; if (N > 1) v[1] = b; if (N > 2) v[2] = c; }
  T& operator[](int i) { return v[i]; }
  const T& operator[](int i) const { return v[i]; }
  T& operator()(int i) { return v[i]; }
  const T& operator()(int i) const { return v[i]; }
  int size() const { return N; }
  T* data() { return v; }
  const T* data() const { return v; }
};
template <int N, typename T> Vector<N, T> operator+(const Vector<N, T>& a, const Vector<N, T>& b) {
  Vector<N, T> r; for (int i = 0; i < N; i++) r[i] = a[i] + b[i]; return r; }
template <int N, typename T> Vector<N, T> operator-(const Vector<N, T>& a, const Vector<N, T>& b) {
  Vector<N, T> r; for (int i = 0; i < N; i++) r[i] = a[i] - b[i]; return r; }
template <int N, typename T> Vector<N, T> operator*(const T& s, const Vector<N, T>& a) {
  Vector<N, T> r; for (int i = 0; i < N; i++) r[i] = s * a[i]; return r; }
template <int N, typename T> Vector<N, T> operator*(const Vector<N, T>& a, const T& s) {
  Vector<N, T> r; for (int i = 0; i < N; i++) r[i] = a[i] * s; return r; }
template <int N, typename T> Vector<N, T> operator/(const Vector<N, T>& a, const T& s) {
  Vector<N, T> r; for (int i = 0; i < N; i++) r[i] = a[i] / s; return r; }
template <int N, typename T> T volume(const Vector<N, T>& a) { T r = 1; for (int i = 0; i < N; i++) r *= a[i]; return r; }
inline int aPowI(int i, int a) { int r = 1; for (int k = 0; k < i; k++) r *= a; return r; }
}}
