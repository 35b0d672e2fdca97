// flop_count.h -- a counting scalar type for the oracle (test infrastructure).
//
// Cnt behaves like double and tallies every floating-point operation it
// takes part in.  The oracle's numeric kernels are templates over the scalar
// type; instantiated with Cnt they give the algorithmic operation count of
// one synthesis or one SVD solve of the reference's algorithm, which the
// benchmark multiplies by the event counts the device reports.
#pragma once
#include <math.h>

struct FlopTally {
  long long add = 0, mul = 0, div = 0, sqrt_ = 0, exp_ = 0, trig = 0, special = 0, cmp = 0;
};

extern thread_local FlopTally g_tally;

struct Cnt {
  double v;
  Cnt() : v(0) {}
  Cnt(double x) : v(x) {}
  explicit operator int() const { return (int)v; }
  friend Cnt operator+(Cnt a, Cnt b) { g_tally.add++; return Cnt(a.v + b.v); }
  friend Cnt operator-(Cnt a, Cnt b) { g_tally.add++; return Cnt(a.v - b.v); }
  friend Cnt operator*(Cnt a, Cnt b) { g_tally.mul++; return Cnt(a.v * b.v); }
  friend Cnt operator/(Cnt a, Cnt b) { g_tally.div++; return Cnt(a.v / b.v); }
  friend Cnt operator-(Cnt a) { return Cnt(-a.v); }
  Cnt &operator+=(Cnt b) { g_tally.add++; v += b.v; return *this; }
  Cnt &operator-=(Cnt b) { g_tally.add++; v -= b.v; return *this; }
  Cnt &operator*=(Cnt b) { g_tally.mul++; v *= b.v; return *this; }
  Cnt &operator/=(Cnt b) { g_tally.div++; v /= b.v; return *this; }
  friend bool operator<(Cnt a, Cnt b) { g_tally.cmp++; return a.v < b.v; }
  friend bool operator>(Cnt a, Cnt b) { g_tally.cmp++; return a.v > b.v; }
  friend bool operator<=(Cnt a, Cnt b) { g_tally.cmp++; return a.v <= b.v; }
  friend bool operator>=(Cnt a, Cnt b) { g_tally.cmp++; return a.v >= b.v; }
  friend bool operator==(Cnt a, Cnt b) { g_tally.cmp++; return a.v == b.v; }
  friend bool operator!=(Cnt a, Cnt b) { g_tally.cmp++; return a.v != b.v; }
  friend Cnt fabs(Cnt a) { return Cnt(::fabs(a.v)); }
  friend Cnt copysign(Cnt a, Cnt b) { return Cnt(::copysign(a.v, b.v)); }
  friend Cnt round(Cnt a) { return Cnt(::round(a.v)); }
  friend Cnt sqrt(Cnt a) { g_tally.sqrt_++; return Cnt(::sqrt(a.v)); }
  friend Cnt exp(Cnt a) { g_tally.exp_++; return Cnt(::exp(a.v)); }
  friend Cnt log(Cnt a) { g_tally.exp_++; return Cnt(::log(a.v)); }
  friend Cnt sin(Cnt a) { g_tally.trig++; return Cnt(::sin(a.v)); }
  friend Cnt cos(Cnt a) { g_tally.trig++; return Cnt(::cos(a.v)); }
  friend Cnt erfc(Cnt a) { g_tally.special++; return Cnt(::erfc(a.v)); }
};
