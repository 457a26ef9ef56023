// Reverse-mode differentiation for the adjoint of the solve stage: a scalar that records each
// operation, with the partial derivatives of its result, on the calling thread's tape, and a sweep
// that carries adjoints back from the results to the inputs.
//
// Used the same way in device code (the reverse kernels, bearing_gpu.cu) and in host code (the
// reverse of the host side of the step, world.cpp): a piece of the step is replayed from its
// recorded inputs with `TV` scalars (each input a leaf), the adjoints of its results are seeded,
// sweep() runs, and the leaves' adjoints are read.  The values a TV carries are computed with the
// very operations, in the very order, of plain double code, so a replay takes every branch the
// recorded step took: the derivative is the one of the step's own active set (which points
// pushed, which branch of each clamp, how many Newton rounds).
//
// Where a function has no derivative the replay takes one side's:
//   sqrt at 0: 0 (the lever of a point on the friction anchor, a body not turning);
//   |x| at 0: 0;  atan2 at (0, 0): 0;  a comparison or a min / max: the branch the values took.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define BGAD_HD __host__ __device__ __forceinline__
#else
#define BGAD_HD inline
#endif

namespace bgad {

// One thread's tape: node k has up to two parents (pa, pb; -1 for none) and the partial
// derivatives of its value with respect to each (da, db).  A node with no parents is a leaf.
struct Tape {
  int32_t n;
  int32_t cap;
  int32_t* pa;
  int32_t* pb;
  double* da;
  double* db;
  double* adj;
  int32_t overflow;   // a node did not fit: the replay's adjoints are not to be used
  int32_t peak;       // the most nodes any replay on this tape has recorded
};

// The calling thread's tape (defined once, where the tapes are set up: device and host side).
#ifdef __CUDA_ARCH__
__device__ Tape* thread_tape();
#else
Tape* thread_tape();
#endif

BGAD_HD int32_t node(int32_t a, double da, int32_t b, double db) {
  Tape* t = thread_tape();
  if (t->n >= t->cap) {
    t->overflow = 1;
    return -1;
  }
  const int32_t k = t->n++;
  t->pa[k] = a;
  t->da[k] = da;
  t->pb[k] = b;
  t->db[k] = db;
  return k;
}

// A recorded value: v, and its node on the tape (-1: a constant).
struct TV {
  double v;
  int32_t i;
  BGAD_HD TV() : v(0), i(-1) {}
  BGAD_HD TV(double x) : v(x), i(-1) {}   // NOLINT: constants mix freely with recorded values
  BGAD_HD TV(double x, int32_t k) : v(x), i(k) {}
};

// A leaf: an input whose adjoint the sweep leaves behind.
BGAD_HD TV leaf(double x) { return TV(x, node(-1, 0.0, -1, 0.0)); }

BGAD_HD TV unary(double r, const TV& a, double d) { return a.i < 0 ? TV(r) : TV(r, node(a.i, d, -1, 0.0)); }
BGAD_HD TV binary(double r, const TV& a, double da, const TV& b, double db) {
  if (a.i < 0 && b.i < 0) return TV(r);
  return TV(r, node(a.i, da, b.i, db));
}

BGAD_HD TV operator+(const TV& a, const TV& b) { return binary(a.v + b.v, a, 1.0, b, 1.0); }
BGAD_HD TV operator-(const TV& a, const TV& b) { return binary(a.v - b.v, a, 1.0, b, -1.0); }
BGAD_HD TV operator*(const TV& a, const TV& b) { return binary(a.v * b.v, a, b.v, b, a.v); }
BGAD_HD TV operator/(const TV& a, const TV& b) {
  const double r = a.v / b.v;
  return binary(r, a, 1.0 / b.v, b, -r / b.v);
}
BGAD_HD TV operator-(const TV& a) { return unary(-a.v, a, -1.0); }
BGAD_HD TV& operator+=(TV& a, const TV& b) { return a = a + b; }
BGAD_HD TV& operator-=(TV& a, const TV& b) { return a = a - b; }
BGAD_HD TV& operator*=(TV& a, const TV& b) { return a = a * b; }
BGAD_HD TV& operator/=(TV& a, const TV& b) { return a = a / b; }

BGAD_HD bool operator<(const TV& a, const TV& b) { return a.v < b.v; }
BGAD_HD bool operator>(const TV& a, const TV& b) { return a.v > b.v; }
BGAD_HD bool operator<=(const TV& a, const TV& b) { return a.v <= b.v; }
BGAD_HD bool operator>=(const TV& a, const TV& b) { return a.v >= b.v; }
BGAD_HD bool operator==(const TV& a, const TV& b) { return a.v == b.v; }
BGAD_HD bool operator!=(const TV& a, const TV& b) { return a.v != b.v; }

BGAD_HD TV sqrt(const TV& a) {
  const double r = ::sqrt(a.v);
  return unary(r, a, r > 0 ? 0.5 / r : 0.0);
}
BGAD_HD TV fabs(const TV& a) { return unary(a.v < 0 ? -a.v : a.v, a, a.v < 0 ? -1.0 : a.v > 0 ? 1.0 : 0.0); }

// The value of a scalar, recorded or plain.
BGAD_HD double val(const TV& a) { return a.v; }
BGAD_HD double val(double a) { return a; }

// Clears the tape for a new replay (an overflow stays flagged until the caller reads it).
BGAD_HD void reset(Tape* t) {
  if (t->n > t->peak) t->peak = t->n;
  t->n = 0;
}

// Adds g to the adjoint of x's node (nothing for a constant).
BGAD_HD void seed(Tape* t, const TV& x, double g) {
  if (x.i >= 0) t->adj[x.i] += g;
}

// The adjoint a node has after the sweep (0 for a constant).
BGAD_HD double adjoint(const Tape* t, const TV& x) { return x.i >= 0 ? t->adj[x.i] : 0.0; }

// Zeroes every adjoint of the recorded nodes; then seed(), then sweep().
BGAD_HD void clear_adjoints(Tape* t) {
  for (int32_t k = 0; k < t->n; k++) t->adj[k] = 0;
}

BGAD_HD void sweep(Tape* t) {
  for (int32_t k = t->n - 1; k >= 0; k--) {
    const double g = t->adj[k];
    if (g == 0) continue;
    if (t->pa[k] >= 0) t->adj[t->pa[k]] += t->da[k] * g;
    if (t->pb[k] >= 0) t->adj[t->pb[k]] += t->db[k] * g;
  }
}

}  // namespace bgad
