// flopcount.hpp -- FP64 operation counter for the oracle.
//
// TEST INFRASTRUCTURE ONLY (measurement of the oracle, never shipped).
// Force-included (g++ -include) ahead of the oracle's C sources compiled as
// C++, it replaces every `double` of the oracle by `fdouble`, a double that
// counts its own arithmetic: each +, -, *, / and each sqrt/exp/pow/cos call on
// an fdouble adds one to the counters below.  Comparisons, fabs, copysign
// and conversions are not counted (no FP64 arithmetic in the sense of an
// operation count).  The oracle restates the reference's serial algorithm
// (primitives recomputed by every operator call, as the reference's
// procedure pointers do), so the count is the reference algorithm's own
// FP64 work per cell-update.  Built and run by oracle/Makefile's `flopcount`
// target; its output is the oracle's figure that bench.py reports.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

struct FlopCounts {
  unsigned long long add, mul, div, sqrt, transcendental;
};
extern FlopCounts g_flops;

struct fdouble {
  double v;
  fdouble() = default;
  fdouble(double x) : v(x) {}
  explicit operator int() const { return (int)v; }
  explicit operator long() const { return (long)v; }
  explicit operator unsigned long() const { return (unsigned long)v; }
  explicit operator float() const { return (float)v; }
  explicit operator bool() const { return v != 0.0; }

  friend fdouble operator+(fdouble a, fdouble b) { g_flops.add++; return fdouble(a.v + b.v); }
  friend fdouble operator-(fdouble a, fdouble b) { g_flops.add++; return fdouble(a.v - b.v); }
  friend fdouble operator*(fdouble a, fdouble b) { g_flops.mul++; return fdouble(a.v * b.v); }
  friend fdouble operator/(fdouble a, fdouble b) { g_flops.div++; return fdouble(a.v / b.v); }
  friend fdouble operator-(fdouble a) { return fdouble(-a.v); }
  friend fdouble operator+(fdouble a) { return a; }
  fdouble& operator+=(fdouble b) { g_flops.add++; v += b.v; return *this; }
  fdouble& operator-=(fdouble b) { g_flops.add++; v -= b.v; return *this; }
  fdouble& operator*=(fdouble b) { g_flops.mul++; v *= b.v; return *this; }
  fdouble& operator/=(fdouble b) { g_flops.div++; v /= b.v; return *this; }
  friend bool operator<(fdouble a, fdouble b) { return a.v < b.v; }
  friend bool operator<=(fdouble a, fdouble b) { return a.v <= b.v; }
  friend bool operator>(fdouble a, fdouble b) { return a.v > b.v; }
  friend bool operator>=(fdouble a, fdouble b) { return a.v >= b.v; }
  friend bool operator==(fdouble a, fdouble b) { return a.v == b.v; }
  friend bool operator!=(fdouble a, fdouble b) { return a.v != b.v; }
};

inline fdouble sqrt(fdouble a) { g_flops.sqrt++; return fdouble(std::sqrt(a.v)); }
inline fdouble exp(fdouble a) { g_flops.transcendental++; return fdouble(std::exp(a.v)); }
inline fdouble cos(fdouble a) { g_flops.transcendental++; return fdouble(std::cos(a.v)); }
inline fdouble sin(fdouble a) { g_flops.transcendental++; return fdouble(std::sin(a.v)); }
inline fdouble log(fdouble a) { g_flops.transcendental++; return fdouble(std::log(a.v)); }
inline fdouble tanh(fdouble a) { g_flops.transcendental++; return fdouble(std::tanh(a.v)); }
inline fdouble pow(fdouble a, fdouble b) {
  g_flops.transcendental++;
  return fdouble(std::pow(a.v, b.v));
}
inline fdouble fabs(fdouble a) { return fdouble(std::fabs(a.v)); }
inline fdouble copysign(fdouble a, fdouble b) { return fdouble(std::copysign(a.v, b.v)); }
inline fdouble fmax(fdouble a, fdouble b) { return fdouble(std::fmax(a.v, b.v)); }
inline fdouble fmin(fdouble a, fdouble b) { return fdouble(std::fmin(a.v, b.v)); }
inline fdouble floor(fdouble a) { return fdouble(std::floor(a.v)); }
inline bool isfinite(fdouble a) { return std::isfinite(a.v); }
inline bool isnan(fdouble a) { return std::isnan(a.v); }

#define double fdouble
#define restrict __restrict
