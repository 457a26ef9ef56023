// The solve stage on the device: every phase of src/world.js:962-1032 as device functions over
// the layout in layout.cuh, written once for a "team" of threads.  GridTeam is every thread of
// a persistent cooperative grid working on one world: grid-wide barriers between phases,
// and within each row pass a dataflow over per-body counters instead of a barrier per colour (see
// flow_pass).  BlockTeam is one CTA working on one world of a batch, colour by colour with block
// barriers.  Within a colour no two rows share a body the solve moves (src/graph.js:1-33), so a
// colour's rows run in any order with the same bits; across colours only each body's own order
// of rows matters, which is what the counters keep.
//
// Arithmetic follows the reference's operation order exactly (built with -fmad=false), so each
// value is the one the reference's FP64 JavaScript computes.  Functions cite what they follow:
//   src/contact.js  inertias 1302-1310, inverseAt 1493-1508, lockedInverse 1520-1549,
//                   prepareRows 1346-1445, core 1199-1219, lever 1565-1581, turning/along
//                   1728-1737, warmRows 1616-1663, pushes 1672-1724, solveRows 1805-2090,
//                   writeBack 2101-2104, restitution 2229-2251, slipped/turned 1122-1182
//   src/world.js    start snapshot 964-974, _accelerate 1495-1530, _move 1533-1563,
//                   tumble 2739-2763, untwist 2777-2805, advance 2820-2828, angular 2831-2834
//   src/core/math.js rotate 211-219, axesOf 222-227, quatMultiply 230-238, atan/atan2 138-200
#pragma once

#include <math.h>
#include <stdint.h>

#include "layout.cuh"

namespace bg {

constexpr double COMPLIANCE = 9.5367431640625e-7;   // 2^-20, src/forest.js:67
constexpr double SPIN_DISC = 2.0 / 3.0;             // src/contact.js:146
constexpr double WORLD_SPIN = 3.141592653589793;    // src/world.js:171
constexpr double ROUNDED = 1.0 / 17592186044416.0;  // 2^-44, src/world.js:2812

// Loads: ldi for columns no thread writes during the stage (read-only path), ldm for
// everything the stage writes (at L2, so a value written by another SM is seen after a barrier).
template <class T>
__device__ __forceinline__ T ldi(const T* p) { return __ldg(p); }
template <class T>
__device__ __forceinline__ T ldm(const T* p) { return __ldcg(p); }
template <class T>
__device__ __forceinline__ void stm(T* p, T v) { __stcg(p, v); }

__device__ __forceinline__ double js_max(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a > b) return a;
  if (b > a) return b;
  if (a == 0 && b == 0) return signbit(a) ? b : a;
  return a;
}

// rotate: src/core/math.js:211-219.
__device__ __forceinline__ void rotate(const double* q, double x, double y, double z, bool inverse, double* out) {
  const double s = inverse ? -1.0 : 1.0;
  const double ux = q[0] * s, uy = q[1] * s, uz = q[2] * s, w = q[3];
  const double tx = 2 * (uy * z - uz * y), ty = 2 * (uz * x - ux * z), tz = 2 * (ux * y - uy * x);
  out[0] = x + w * tx + (uy * tz - uz * ty);
  out[1] = y + w * ty + (uz * tx - ux * tz);
  out[2] = z + w * tz + (ux * ty - uy * tx);
}

// axesOf: src/core/math.js:222-227.
__device__ __forceinline__ void axes_of(const double* q, double* ax) {
  const double x = q[0], y = q[1], z = q[2], w = q[3];
  ax[0] = 1 - 2 * (y * y + z * z); ax[1] = 2 * (x * y + z * w); ax[2] = 2 * (x * z - y * w);
  ax[3] = 2 * (x * y - z * w); ax[4] = 1 - 2 * (x * x + z * z); ax[5] = 2 * (y * z + x * w);
  ax[6] = 2 * (x * z + y * w); ax[7] = 2 * (y * z - x * w); ax[8] = 1 - 2 * (x * x + y * y);
}

// The reference's own arctangent (src/core/math.js:127-200, fdlibm's method and constants as it
// states them), so slipped() turns angles to the same bits.
__host__ __device__ __forceinline__ double ref_atan(double x) {
  const double ATAN_HI[4] = {4.63647609000806093515e-01, 7.85398163397448278999e-01,
                             9.82793723247329054082e-01, 1.57079632679489655800e+00};
  const double ATAN_LO[4] = {2.26987774529616870924e-17, 3.06161699786838301793e-17,
                             1.39033110312309984516e-17, 6.12323399573676603587e-17};
  const double AT0 = 3.33333333333329318027e-01, AT1 = -1.99999999998764832476e-01,
               AT2 = 1.42857142725034663711e-01, AT3 = -1.11111104054623557880e-01,
               AT4 = 9.09088713343650656196e-02, AT5 = -7.69187620504482999495e-02,
               AT6 = 6.66107313738753120669e-02, AT7 = -5.83357013379057348645e-02,
               AT8 = 4.97687799461593236017e-02, AT9 = -3.65315727442169155270e-02,
               AT10 = 1.62858201153657823623e-02;
  if (x != x) return x;
  const double ax = fabs(x);
  if (ax >= 7.378697629483821e+19) return x > 0 ? ATAN_HI[3] + ATAN_LO[3] : -ATAN_HI[3] - ATAN_LO[3];
  int id;
  double t;
  if (ax < 0.4375) {
    if (ax < 7.450580596923828e-09) return x;
    id = -1; t = x;
  } else if (ax < 0.6875) {
    id = 0; t = (2 * ax - 1) / (2 + ax);
  } else if (ax < 1.1875) {
    id = 1; t = (ax - 1) / (ax + 1);
  } else if (ax < 2.4375) {
    id = 2; t = (ax - 1.5) / (1 + 1.5 * ax);
  } else {
    id = 3; t = -1 / ax;
  }
  const double z = t * t, w = z * z;
  const double s1 = z * (AT0 + w * (AT2 + w * (AT4 + w * (AT6 + w * (AT8 + w * AT10)))));
  const double s2 = w * (AT1 + w * (AT3 + w * (AT5 + w * (AT7 + w * AT9))));
  if (id < 0) return t - t * (s1 + s2);
  const double r = ATAN_HI[id] - ((t * (s1 + s2) - ATAN_LO[id]) - t);
  return x < 0 ? -r : r;
}

__host__ __device__ __forceinline__ double ref_atan2(double y, double x) {
  const double PI_ = 3.1415926535897931160e+00, PI_LO = 1.2246467991473531772e-16;
  const double PI_O_2 = 1.5707963267948965580e+00, PI_O_4 = 7.8539816339744827900e-01;
  if (x != x || y != y) return x + y;
  if (x == 1) return ref_atan(y);
  const bool ny = y < 0 || (y == 0 && signbit(y)), nx = x < 0 || (x == 0 && signbit(x));
  int m = (ny ? 1 : 0) | (nx ? 2 : 0);
  if (y == 0) return m < 2 ? y : m == 2 ? PI_ : -PI_;
  if (x == 0) return y < 0 ? -PI_O_2 : PI_O_2;
  const double ax = fabs(x), ay = fabs(y);
  if (isinf(ax)) {
    if (isinf(ay)) {
      const double r[4] = {PI_O_4, -PI_O_4, 3 * PI_O_4, -3 * PI_O_4};
      return r[m];
    }
    const double r[4] = {0.0, -0.0, PI_, -PI_};
    return r[m];
  }
  if (isinf(ay)) return y < 0 ? -PI_O_2 : PI_O_2;
  double z;
  if (ay > ax * 1.152921504606847e+18) {
    z = PI_O_2 + 0.5 * PI_LO;
    m &= 1;
  } else if (x < 0 && ay < ax * 8.673617379884035e-19) {
    z = 0;
  } else {
    z = ref_atan(ay / ax);
  }
  switch (m) {
    case 0: return z;
    case 1: return -z;
    case 2: return PI_ - (z - PI_LO);
    default: return (z - PI_LO) - PI_;
  }
}

// ---- barriers ----

// A grid-wide barrier whose wait is bounded: past `budget` polls it records status 1 and every
// block leaves the stage at its next barrier, so the kernel always ends.  The arrival count only
// grows (the host zeroes it before each launch): a block arriving as the k-th of all arrivals is in
// barrier k / blocks and waits for the count to reach the end of that barrier, so no block has to
// reset anything for the next one.
__device__ __forceinline__ bool grid_barrier(const StageParams& p) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int G = gridDim.x;
    __threadfence();
    const unsigned int old = atomicAdd(p.bar_count, 1u);
    const unsigned int target = (old / G + 1u) * G;
    long long it = 0;
    for (;;) {
      unsigned int seen;
      asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(p.bar_count) : "memory");
      if (seen >= target) break;
      if (++it > p.budget) {
        atomicExch(p.status, 1);
        break;
      }
    }
    __threadfence();
    if (*(volatile int32_t*)p.status != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

struct GridTeam {
  static constexpr bool kGrid = true;
  int rank, size;
  bool lead;   // the block that runs the stage's serial parts
  __device__ GridTeam() : rank(blockIdx.x * blockDim.x + threadIdx.x), size(gridDim.x * blockDim.x), lead(blockIdx.x == 0) {}
  __device__ bool sync(const StageParams& p) const { return grid_barrier(p); }
  __device__ int lane_in_lead() const { return threadIdx.x; }
  // Items from..to-1 spread over every block, each block a contiguous share, so a colour's rows
  // reach every SM however few there are.
  template <class F>
  __device__ void each(int from, int to, F f) const {
    const int n = to - from;
    if (n <= 0) return;
    const int per = (n + static_cast<int>(gridDim.x) - 1) / static_cast<int>(gridDim.x);
    const int lo = from + static_cast<int>(blockIdx.x) * per;
    const int hi = min(to, lo + per);
    for (int m = lo + static_cast<int>(threadIdx.x); m < hi; m += blockDim.x) f(m);
  }
};

// ---- the grid's dataflow passes ----
//
// A pass over every solved row with no barrier between colours: a row waits only until the rows
// before it (in solve order) on each body it moves are done, which is all that colour order
// guarantees and all the reference's order depends on (src/graph.js:1-33).  Each body's counter
// counts its rows done in the stage; row m of pass `pass` on body X may start when it reaches
// pass * deg[X] + rank, and moves it on by one when its writes are out (release / acquire).
// Work goes to warps as runs of rows in solve order, each warp taking its runs in ascending
// order, so the earliest waiting row always has every predecessor done or running: no cycle.
// Every wait is bounded by the step's budget; past it the status word is set and all waits end.

// Both bodies' counters are read together with relaxed loads and a single acq_rel fence follows
// once both are far enough (the PTX memory model's fence-based acquire pattern); a row's writes are
// published the same way, one fence and then relaxed stores (the release pattern).  Two ld.acquire
// in a row would cost two trips to L2 on every row's critical path; this costs one.
__device__ __forceinline__ unsigned int load_relaxed(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void store_relaxed(unsigned int* p, unsigned int v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// The count body x must reach before row m of `pass` may move it (0: no wait; a static body, or
// the body's first row of the first pass).
__device__ __forceinline__ unsigned int flow_target(const StageParams& p, int x, int rank, int pass) {
  return rank < 0 ? 0u : static_cast<unsigned int>(pass) * static_cast<unsigned int>(ldi(p.B.deg + x)) +
                             static_cast<unsigned int>(rank);
}

__device__ __forceinline__ void flow_signal(const StageParams& p, int a, int ra, unsigned int ta, int b, int rb,
                                            unsigned int tb) {
  fence_acq_rel();
  if (ra >= 0) store_relaxed(p.B.done + a, ta + 1u);
  if (rb >= 0) store_relaxed(p.B.done + b, tb + 1u);
}

template <class F>
__device__ __forceinline__ void flow_pass(const StageParams& p, int pass, F row) {
  const int lane = static_cast<int>(threadIdx.x) & 31;
  const int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int warps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
  for (int c = warp; c < p.nchunks; c += warps) {
    const int2 run = p.chunks[c];
    if (lane < run.y) {
      const int m = run.x + lane;
      const int a = ldi(p.R.a + m), b = ldi(p.R.b + m);
      const int ra = ldi(p.R.rank_a + m), rb = ldi(p.R.rank_b + m);
      const unsigned int ta = flow_target(p, a, ra, pass), tb = flow_target(p, b, rb, pass);
      // The row's rest runs inside the wait, so each lane goes on the moment its own bodies are
      // ready rather than when the whole run's are; a lane still waiting sleeps between polls,
      // which lets the warp run the lanes that are ready.
      row(m, [&](auto&& finish) {
        long long it = 0;
        for (;;) {
          const unsigned int va = ta == 0 ? 0u : load_relaxed(p.B.done + a);
          const unsigned int vb = tb == 0 ? 0u : load_relaxed(p.B.done + b);
          if (va >= ta && vb >= tb) {
            fence_acq_rel();
            finish();
            flow_signal(p, a, ra, ta, b, rb, tb);
            return true;
          }
          if (++it > p.budget || ((it & 255) == 0 && *(volatile int32_t*)p.status != 0)) {
            atomicExch(p.status, 1);
            return false;
          }
          __nanosleep(200);
        }
      });
    }
    __syncwarp();
  }
}

struct BlockTeam {
  static constexpr bool kGrid = false;
  int rank, size;
  bool lead;
  __device__ BlockTeam() : rank(threadIdx.x), size(blockDim.x), lead(true) {}
  __device__ bool sync(const StageParams&) const { __syncthreads(); return true; }
  __device__ int lane_in_lead() const { return threadIdx.x; }
  template <class F>
  __device__ void each(int from, int to, F f) const {
    for (int m = from + static_cast<int>(threadIdx.x); m < to; m += blockDim.x) f(m);
  }
};

// ---- bodies ----

__device__ __forceinline__ uint32_t shape_of(uint32_t f) { return (f >> F_SHAPE_SHIFT) & 3u; }

// lockedInverse: src/contact.js:1520-1549.
__device__ void locked_inverse(const double* ax, const double* I, int lock, double* out) {
  const int SYM[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
  const double i0 = I[0], i1 = I[1], i2 = I[2];
  const double x0 = ax[0], x1 = ax[1], x2 = ax[2];
  const double y0 = ax[3], y1 = ax[4], y2 = ax[5];
  const double z0 = ax[6], z1 = ax[7], z2 = ax[8];
  double M6[6];
  M6[0] = x0 * x0 * i0 + y0 * y0 * i1 + z0 * z0 * i2;
  M6[1] = x0 * x1 * i0 + y0 * y1 * i1 + z0 * z1 * i2;
  M6[2] = x0 * x2 * i0 + y0 * y2 * i1 + z0 * z2 * i2;
  M6[3] = x1 * x1 * i0 + y1 * y1 * i1 + z1 * z1 * i2;
  M6[4] = x1 * x2 * i0 + y1 * y2 * i1 + z1 * z2 * i2;
  M6[5] = x2 * x2 * i0 + y2 * y2 * i1 + z2 * z2 * i2;
  for (int k = 0; k < 6; k++) out[k] = 0;
  int first = -1, second = -1;
  for (int k = 0; k < 3; k++) {
    if (lock >> k & 1) continue;
    if (first < 0) first = k; else second = k;
  }
  if (first < 0) return;
  const int ff = SYM[4 * first];
  if (second < 0) {
    if (M6[ff] > 0) out[ff] = 1 / M6[ff];
    return;
  }
  const int ss = SYM[4 * second], fs = SYM[3 * first + second];
  const double det = M6[ff] * M6[ss] - M6[fs] * M6[fs];
  if (!(det > 0)) return;
  out[ff] = M6[ss] / det; out[ss] = M6[ff] / det; out[fs] = -M6[fs] / det;
}

// inertias (contact.js:1302-1310) and the start snapshot (world.js:968-973) for awake body s.
__device__ void body_begin(const StageParams& p, int s, bool touching) {
  const BodiesDev& B = p.B;
  const uint32_t f = ldi(B.fl + s);
  double q[4];
  for (int k = 0; k < 4; k++) q[k] = ldm(B.pq + 8 * s + 4 + k);
  if (touching) {
    double out[6];
    if (f & F_FROZEN) {
      for (int k = 0; k < 6; k++) out[k] = 0;
    } else if ((f & F_TYPE) != 0) {
      for (int k = 0; k < 6; k++) out[k] = 0;
    } else {
      double ax[9];
      axes_of(q, ax);
      const int lock = static_cast<int>((f >> F_LOCK_SHIFT) & 7u);
      if (lock != 0) {
        double I[3];
        for (int k = 0; k < 3; k++) I[k] = ldi(B.pr + 12 * s + k);
        locked_inverse(ax, I, lock, out);
      } else {
        const double i0 = ldi(B.pr + 12 * s + 3), i1 = ldi(B.pr + 12 * s + 4), i2 = ldi(B.pr + 12 * s + 5);
        const double x0 = ax[0], x1 = ax[1], x2 = ax[2];
        const double y0 = ax[3], y1 = ax[4], y2 = ax[5];
        const double z0 = ax[6], z1 = ax[7], z2 = ax[8];
        out[0] = x0 * x0 * i0 + y0 * y0 * i1 + z0 * z0 * i2;
        out[1] = x0 * x1 * i0 + y0 * y1 * i1 + z0 * z1 * i2;
        out[2] = x0 * x2 * i0 + y0 * y2 * i1 + z0 * z2 * i2;
        out[3] = x1 * x1 * i0 + y1 * y1 * i1 + z1 * z1 * i2;
        out[4] = x1 * x2 * i0 + y1 * y2 * i1 + z1 * z2 * i2;
        out[5] = x2 * x2 * i0 + y2 * y2 * i1 + z2 * z2 * i2;
      }
    }
    for (int k = 0; k < 6; k++) stm(B.mi + 8 * s + 1 + k, out[k]);
  }
  for (int k = 0; k < 3; k++) stm(B.st + 4 * s + k, ldm(B.pq + 8 * s + k));
  for (int k = 0; k < 4; k++) stm(B.sq + 4 * s + k, q[k]);
}

// _accelerate for body s: src/world.js:1495-1530.
__device__ void accelerate_body(const StageParams& p, int s, double h, const double* gravity) {
  const BodiesDev& B = p.B;
  const uint32_t f = ldi(B.fl + s);
  if ((f & F_TYPE) != 0 || (f & F_FROZEN)) return;
  const double gx = gravity[0] * h, gy = gravity[1] * h, gz = gravity[2] * h;
  const double most = WORLD_SPIN / (h * p.substeps);
  double* vw = B.vw + 8 * s;
  double v0 = ldm(vw), v1 = ldm(vw + 1), v2 = ldm(vw + 2), w0 = ldm(vw + 3), w1 = ldm(vw + 4), w2 = ldm(vw + 5);
  const double g = ldi(B.pr + 12 * s + 11);
  v0 += gx * g; v1 += gy * g; v2 += gz * g;
  const double damping = ldi(B.pr + 12 * s + 9), angularDamping = ldi(B.pr + 12 * s + 10);
  if (damping != 0) {
    const double k = 1 / (1 + h * damping);
    v0 *= k; v1 *= k; v2 *= k;
  }
  if (angularDamping != 0) {
    const double k = 1 / (1 + h * angularDamping);
    w0 *= k; w1 *= k; w2 *= k;
  }
  if (shape_of(f) != 1u || (f & F_FRAMED)) {
    const double w2s = w0 * w0 + w1 * w1 + w2 * w2;
    if (w2s > most * most) {
      const double k = most / sqrt(w2s);
      w0 *= k; w1 *= k; w2 *= k;
    }
  }
  stm(vw, v0); stm(vw + 1, v1); stm(vw + 2, v2); stm(vw + 3, w0); stm(vw + 4, w1); stm(vw + 5, w2);
}

// advance: src/world.js:2820-2828.
__device__ __forceinline__ void advance(const double* q, double wx, double wy, double wz, double h, double* out) {
  const double x = q[0], y = q[1], z = q[2], w = q[3];
  const double nx = x + h * (wx * w + wy * z - wz * y);
  const double ny = y + h * (wy * w + wz * x - wx * z);
  const double nz = z + h * (wz * w + wx * y - wy * x);
  const double nw = w - h * (wx * x + wy * y + wz * z);
  const double l = 1 / sqrt(nx * nx + ny * ny + nz * nz + nw * nw);
  out[0] = nx * l; out[1] = ny * l; out[2] = nz * l; out[3] = nw * l;
}

// angular: src/world.js:2831-2834.
__device__ __forceinline__ void angular_of(const double* q, const double* inv, double lx, double ly, double lz, double* v3) {
  rotate(q, lx, ly, lz, true, v3);
  rotate(q, v3[0] * inv[0], v3[1] * inv[1], v3[2] * inv[2], false, v3);
}

// untwist: src/world.js:2777-2805.
__device__ void untwist(double* q, const double* inv, double lx, double ly, double lz, double most) {
  double Bv[3];
  rotate(q, lx, ly, lz, true, Bv);
  const double bx = Bv[0], by = Bv[1], bz = Bv[2], ll = bx * bx + by * by + bz * bz;
  double x = bx, y = by, z = bz;
  for (int round = 0; round < 2; round++) {
    const double gx = x * inv[0], gy = y * inv[1], gz = z * inv[2];
    const double over = x * gx + y * gy + z * gz - most;
    if (!(over > 0)) break;
    const double k = (gx * x + gy * y + gz * z) / ll, tx = gx - k * x, ty = gy - k * y, tz = gz - k * z;
    const double tt = tx * tx + ty * ty + tz * tz;
    if (!(tt > 0)) break;
    const double a = 0.5 * over / tt;
    x -= a * tx; y -= a * ty; z -= a * tz;
    const double back = sqrt(ll / (x * x + y * y + z * z));
    x *= back; y *= back; z *= back;
  }
  const double cx = y * bz - z * by, cy = z * bx - x * bz, cz = x * by - y * bx;
  const double cw = ll + x * bx + y * by + z * bz;
  const double l = sqrt(cx * cx + cy * cy + cz * cz + cw * cw);
  if (!(l > 0)) return;
  const double T4[4] = {cx / l, cy / l, cz / l, cw / l};
  const double ax = q[0], ay = q[1], az = q[2], aw = q[3];
  const double Q0 = aw * T4[0] + ax * T4[3] + ay * T4[2] - az * T4[1];
  const double Q1 = aw * T4[1] + ay * T4[3] + az * T4[0] - ax * T4[2];
  const double Q2 = aw * T4[2] + az * T4[3] + ax * T4[1] - ay * T4[0];
  const double Q3 = aw * T4[3] - ax * T4[0] - ay * T4[1] - az * T4[2];
  const double n = 1 / sqrt(Q0 * Q0 + Q1 * Q1 + Q2 * Q2 + Q3 * Q3);
  q[0] = Q0 * n; q[1] = Q1 * n; q[2] = Q2 * n; q[3] = Q3 * n;
}

// _move for body s (src/world.js:1533-1563), tumble (2739-2763) for a lopsided dynamic body.
__device__ void move_body(const StageParams& p, int s, double h) {
  const BodiesDev& B = p.B;
  const uint32_t f = ldi(B.fl + s);
  if (f & F_FROZEN) return;
  double* pq = B.pq + 8 * s;
  double* vw = B.vw + 8 * s;
  const double v0 = ldm(vw), v1 = ldm(vw + 1), v2 = ldm(vw + 2);
  double w[3] = {ldm(vw + 3), ldm(vw + 4), ldm(vw + 5)};
  double p0 = ldm(pq), p1 = ldm(pq + 1), p2 = ldm(pq + 2);
  p0 += v0 * h; p1 += v1 * h; p2 += v2 * h;
  stm(pq, p0); stm(pq + 1, p1); stm(pq + 2, p2);
  const bool turning = w[0] != 0 || w[1] != 0 || w[2] != 0;
  if (!turning) return;
  double q[4] = {ldm(pq + 4), ldm(pq + 5), ldm(pq + 6), ldm(pq + 7)};
  const double* pr = B.pr + 12 * s;
  const double I[3] = {ldi(pr), ldi(pr + 1), ldi(pr + 2)};
  if ((f & F_TYPE) == 0 && ((f >> F_LOCK_SHIFT) & 7u) == 0 && !(f & F_JOINTED) && (I[0] != I[1] || I[1] != I[2])) {
    const double inv[3] = {ldi(pr + 3), ldi(pr + 4), ldi(pr + 5)};
    double* tc = B.tc + 4 * s;
    double left[3] = {ldm(tc), ldm(tc + 1), ldm(tc + 2)};
    double ceiling = ldm(tc + 3);
    double v3[3], q4[4];
    rotate(q, w[0], w[1], w[2], true, v3);
    rotate(q, v3[0] * I[0], v3[1] * I[1], v3[2] * I[2], false, v3);
    const double lx = v3[0], ly = v3[1], lz = v3[2];
    if (w[0] != left[0] || w[1] != left[1] || w[2] != left[2]) ceiling = w[0] * lx + w[1] * ly + w[2] * lz;
    const double most = ceiling;
    advance(q, w[0], w[1], w[2], h * 0.25, q4);
    angular_of(q4, inv, lx, ly, lz, v3);
    advance(q, v3[0], v3[1], v3[2], h * 0.5, q);
    angular_of(q, inv, lx, ly, lz, v3);
    if (v3[0] * lx + v3[1] * ly + v3[2] * lz > most * (1 + ROUNDED)) {
      untwist(q, inv, lx, ly, lz, most);
      angular_of(q, inv, lx, ly, lz, v3);
    }
    stm(vw + 3, v3[0]); stm(vw + 4, v3[1]); stm(vw + 5, v3[2]);
    stm(tc, v3[0]); stm(tc + 1, v3[1]); stm(tc + 2, v3[2]); stm(tc + 3, ceiling);
  } else {
    advance(q, w[0], w[1], w[2], h * 0.5, q);
  }
  stm(pq + 4, q[0]); stm(pq + 5, q[1]); stm(pq + 6, q[2]); stm(pq + 7, q[3]);
}

// ---- rows ----

struct BodyLoad {
  double im;
  double I[6];
};

__device__ __forceinline__ void load_mass(const BodiesDev& B, int s, BodyLoad& o) {
  const double* mi = B.mi + 8 * s;
  o.im = ldm(mi);
  for (int k = 0; k < 6; k++) o.I[k] = ldm(mi + 1 + k);
}

// along / turning: src/contact.js:1728-1737.
__device__ __forceinline__ double along(const double* I, double x, double y, double z) {
  return I[0] * x * x + I[3] * y * y + I[5] * z * z + 2 * (I[1] * x * y + I[2] * x * z + I[4] * y * z);
}
__device__ __forceinline__ double turning(const double* Ia, const double* Ib, double x, double y, double z) {
  const double k = along(Ia, x, y, z) + along(Ib, x, y, z);
  return k > 0 ? 1 / k : 0;
}

// lever: src/contact.js:1565-1581.
__device__ __forceinline__ double lever(double* jac, const BodyLoad& A, const BodyLoad& Bb, double rax, double ray,
                                        double raz, double rbx, double rby, double rbz, double dx, double dy, double dz) {
  const double* Ia = A.I;
  const double* Ib = Bb.I;
  const double cax = ray * dz - raz * dy, cay = raz * dx - rax * dz, caz = rax * dy - ray * dx;
  const double cbx = rby * dz - rbz * dy, cby = rbz * dx - rbx * dz, cbz = rbx * dy - rby * dx;
  const double iax = Ia[0] * cax + Ia[1] * cay + Ia[2] * caz;
  const double iay = Ia[1] * cax + Ia[3] * cay + Ia[4] * caz;
  const double iaz = Ia[2] * cax + Ia[4] * cay + Ia[5] * caz;
  const double ibx = Ib[0] * cbx + Ib[1] * cby + Ib[2] * cbz;
  const double iby = Ib[1] * cbx + Ib[3] * cby + Ib[4] * cbz;
  const double ibz = Ib[2] * cbx + Ib[4] * cby + Ib[5] * cbz;
  jac[0] = cax; jac[1] = cay; jac[2] = caz;
  jac[3] = cbx; jac[4] = cby; jac[5] = cbz;
  jac[6] = iax; jac[7] = iay; jac[8] = iaz;
  jac[9] = ibx; jac[10] = iby; jac[11] = ibz;
  const double k = A.im + Bb.im + cax * iax + cay * iay + caz * iaz + cbx * ibx + cby * iby + cbz * ibz;
  return k > 0 ? 1 / k : 0;
}

// core: src/contact.js:1199-1219 (whole bodies).
__device__ __forceinline__ void core(uint32_t shape, const double* q, const double* dims, double x, double y, double z,
                                     double* out, double* v3) {
  if (shape == 1u) {
    out[0] = 0; out[1] = 0; out[2] = 0;
    v3[0] = 0; v3[1] = 0; v3[2] = 0;
    return;
  }
  rotate(q, x, y, z, true, v3);
  if (shape != 2u) {
    out[0] = v3[0]; out[1] = v3[1]; out[2] = v3[2];
    v3[0] = x; v3[1] = y; v3[2] = z;
    return;
  }
  const double half = (dims[1] - 2 * dims[0]) * 0.5;
  out[0] = 0; out[1] = v3[1] < -half ? -half : v3[1] > half ? half : v3[1]; out[2] = 0;
  rotate(q, 0, out[1], 0, false, v3);
}

// prepareRows for row m: src/contact.js:1346-1445.
__device__ void prepare_row(const StageParams& p, int m) {
  const RowsDev& R = p.R;
  const BodiesDev& B = p.B;
  const int64_t cap = R.cap;
  const int a = ldi(R.a + m), b = ldi(R.b + m);
  BodyLoad A, Bb;
  load_mass(B, a, A);
  load_mass(B, b, Bb);
  const double ima = A.im, imb = Bb.im;
  const double nx = ldi(R.n + m), ny = ldi(R.n + cap + m), nz = ldi(R.n + 2 * cap + m);
  const double t1x = ldi(R.t1 + m), t1y = ldi(R.t1 + cap + m), t1z = ldi(R.t1 + 2 * cap + m);
  const double t2x = ldi(R.t2 + m), t2y = ldi(R.t2 + cap + m), t2z = ldi(R.t2 + 2 * cap + m);
  const int count = ldi(R.points + m);
  if (count <= 2) {
    stm(R.rm1 + m, turning(A.I, Bb.I, t1x, t1y, t1z));
    stm(R.rm2 + m, turning(A.I, Bb.I, t2x, t2y, t2z));
  }
  stm(R.sm + m, turning(A.I, Bb.I, nx, ny, nz));
  const double tol = ldi(R.tolerance + m);
  double pa[3], pb[3], qa[4], qb[4], va[3], wa[3], vb[3], wb[3], da[3], db[3];
  for (int k = 0; k < 3; k++) {
    pa[k] = ldm(B.pq + 8 * a + k); pb[k] = ldm(B.pq + 8 * b + k);
    va[k] = ldm(B.vw + 8 * a + k); wa[k] = ldm(B.vw + 8 * a + 3 + k);
    vb[k] = ldm(B.vw + 8 * b + k); wb[k] = ldm(B.vw + 8 * b + 3 + k);
    da[k] = ldi(B.pr + 12 * a + 6 + k); db[k] = ldi(B.pr + 12 * b + 6 + k);
  }
  for (int k = 0; k < 4; k++) { qa[k] = ldm(B.pq + 8 * a + 4 + k); qb[k] = ldm(B.pq + 8 * b + 4 + k); }
  const uint32_t sa = shape_of(ldi(B.fl + a)), sb = shape_of(ldi(B.fl + b));
  double weight = 0, ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0;
  double ex = 0, ey = 0, ez = 0, fx = 0, fy = 0, fz = 0;
  double jacs[P][J];
  double ras[P][3];
#pragma unroll
  for (int k = 0; k < P; k++) {
    if (k >= count) break;
    const double px = ldi(R.point + (k * 3) * cap + m), py = ldi(R.point + (k * 3 + 1) * cap + m),
                 pz = ldi(R.point + (k * 3 + 2) * cap + m);
    const double rax = px - pa[0], ray = py - pa[1], raz = pz - pa[2];
    const double rbx = px + ldi(R.shift + (k * 3) * cap + m) - pb[0], rby = py + ldi(R.shift + (k * 3 + 1) * cap + m) - pb[1],
                 rbz = pz + ldi(R.shift + (k * 3 + 2) * cap + m) - pb[2];
    ras[k][0] = rax; ras[k][1] = ray; ras[k][2] = raz;
    double la[3], lb[3], ca[3], cb[3];
    core(sa, qa, da, rax, ray, raz, la, ca);
    core(sb, qb, db, rbx, rby, rbz, lb, cb);
    for (int c = 0; c < 3; c++) {
      stm(R.la + (k * 3 + c) * cap + m, la[c]);
      stm(R.lb + (k * 3 + c) * cap + m, lb[c]);
    }
    const double sep = ldi(R.separation + k * cap + m);
    stm(R.adjusted + k * cap + m, sep - ((cb[0] - ca[0]) * nx + (cb[1] - ca[1]) * ny + (cb[2] - ca[2]) * nz));
    const double nm = lever(jacs[k], A, Bb, rax, ray, raz, rbx, rby, rbz, nx, ny, nz);
    stm(R.normalMass + k * cap + m, nm);
    for (int c = 0; c < J; c++) stm(R.jac + (k * J + c) * cap + m, jacs[k][c]);
    stm(R.maxni + k * cap + m, 0.0);
    const double s = sep / tol, near = s <= 1 ? 1 : s >= 2 ? 0 : 2 - s;
    weight += near;
    ax += near * rax; ay += near * ray; az += near * raz; bx += near * rbx; by += near * rby; bz += near * rbz;
    ex += rax; ey += ray; ez += raz; fx += rbx; fy += rby; fz += rbz;
    const double dvx = vb[0] + wb[1] * rbz - wb[2] * rby - va[0] - wa[1] * raz + wa[2] * ray;
    const double dvy = vb[1] + wb[2] * rbx - wb[0] * rbz - va[1] - wa[2] * rax + wa[0] * raz;
    const double dvz = vb[2] + wb[0] * rby - wb[1] * rbx - va[2] - wa[0] * ray + wa[1] * rax;
    stm(R.relvel + k * cap + m, dvx * nx + dvy * ny + dvz * nz);
  }
  if (count >= 2) {
    const double s = ima + imb;
#pragma unroll
    for (int k = 0; k < P; k++) {
      if (k >= count) break;
#pragma unroll
      for (int l = 0; l <= k; l++) {
        const double* jk = jacs[k];
        const double* jl = jacs[l];
        const double e = s + jk[0] * jl[6] + jk[1] * jl[7] + jk[2] * jl[8] + jk[3] * jl[9] + jk[4] * jl[10] + jk[5] * jl[11];
        stm(R.K + (P * k + l) * cap + m, e);
        stm(R.K + (P * l + k) * cap + m, e);
      }
    }
  }
  if (weight == 0) { weight = count; ax = ex; ay = ey; az = ez; bx = fx; by = fy; bz = fz; }
  ax /= weight; ay /= weight; az /= weight; bx /= weight; by /= weight; bz /= weight;
  stm(R.anchorA + m, ax); stm(R.anchorA + cap + m, ay); stm(R.anchorA + 2 * cap + m, az);
  stm(R.anchorB + m, bx); stm(R.anchorB + cap + m, by); stm(R.anchorB + 2 * cap + m, bz);
#pragma unroll
  for (int k = 0; k < P; k++) {
    if (k >= count) break;
    double dx = ras[k][0] - ax, dy = ras[k][1] - ay, dz = ras[k][2] - az;
    const double alongN = dx * nx + dy * ny + dz * nz;
    dx -= alongN * nx; dy -= alongN * ny; dz -= alongN * nz;
    stm(R.lever + k * cap + m, sqrt(dx * dx + dy * dy + dz * dz));
  }
  double fj[FJ];
  lever(fj, A, Bb, ax, ay, az, bx, by, bz, t1x, t1y, t1z);
  lever(fj + 12, A, Bb, ax, ay, az, bx, by, bz, t2x, t2y, t2z);
  for (int c = 0; c < FJ; c++) stm(R.fjac + c * cap + m, fj[c]);
  const double k11 = ima + imb + fj[0] * fj[6] + fj[1] * fj[7] + fj[2] * fj[8] + fj[3] * fj[9] + fj[4] * fj[10] + fj[5] * fj[11];
  const double k22 = ima + imb + fj[12] * fj[18] + fj[13] * fj[19] + fj[14] * fj[20] + fj[15] * fj[21] + fj[16] * fj[22]
    + fj[17] * fj[23];
  const double k12 = fj[12] * fj[6] + fj[13] * fj[7] + fj[14] * fj[8] + fj[15] * fj[9] + fj[16] * fj[10] + fj[17] * fj[11];
  const double det = k11 * k22 - k12 * k12;
  if (det > 0) {
    stm(R.tm + m, k22 / det); stm(R.tm + cap + m, -k12 / det); stm(R.tm + 2 * cap + m, k11 / det);
  } else {
    stm(R.tm + m, 0.0); stm(R.tm + cap + m, 0.0); stm(R.tm + 2 * cap + m, 0.0);
  }
}

__device__ __forceinline__ void write_back(const BodiesDev& B, double im, int s, double vx, double vy, double vz,
                                           double wx, double wy, double wz) {
  if (im == 0) return;
  double* vw = B.vw + 8 * s;
  stm(vw, vx); stm(vw + 1, vy); stm(vw + 2, vz); stm(vw + 3, wx); stm(vw + 4, wy); stm(vw + 5, wz);
}

// A row's gate: gate(finish) runs `finish` (the row once its bodies are ready) and says whether it
// ran.  OpenGate runs it at once (a CTA's colour-by-colour passes); the grid's waits for its bodies.
struct OpenGate {
  template <class F>
  __device__ __forceinline__ bool operator()(F&& finish) const {
    finish();
    return true;
  }
};

// warmRows for row m: src/contact.js:1616-1663, for a row of N points.  Every array index below
// is known at compile time, so nothing goes to local memory.
template <int N, class Gate>
__device__ __forceinline__ void warm_row_n(const StageParams& p, int m, Gate gate) {
  const RowsDev& R = p.R;
  const BodiesDev& B = p.B;
  const int64_t cap = R.cap;
  const int a = ldi(R.a + m), b = ldi(R.b + m);
  // every load first: the row's own columns, then its two bodies
  const double nx = ldi(R.n + m), ny = ldi(R.n + cap + m), nz = ldi(R.n + 2 * cap + m);
  const double t1x = ldi(R.t1 + m), t1y = ldi(R.t1 + cap + m), t1z = ldi(R.t1 + 2 * cap + m);
  const double t2x = ldi(R.t2 + m), t2y = ldi(R.t2 + cap + m), t2z = ldi(R.t2 + 2 * cap + m);
  double ln[N], ia[N][3], ib[N][3];
#pragma unroll
  for (int k = 0; k < N; k++) {
    ln[k] = ldm(R.ni + k * cap + m);
    const double* jac = R.jac + (k * J) * cap + m;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      ia[k][c] = ldm(jac + (6 + c) * cap);
      ib[k][c] = ldm(jac + (9 + c) * cap);
    }
  }
  double fa[6], fb[6];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    fa[c] = ldm(R.fjac + (6 + c) * cap + m);
    fa[3 + c] = ldm(R.fjac + (18 + c) * cap + m);
    fb[c] = ldm(R.fjac + (9 + c) * cap + m);
    fb[3 + c] = ldm(R.fjac + (21 + c) * cap + m);
  }
  const double l1 = ldm(R.ti1 + m), l2 = ldm(R.ti2 + m);
  const double r1 = ldm(R.ri1 + m), r2 = ldm(R.ri2 + m), sp = ldm(R.si + m);
  BodyLoad A, Bb;   // the bodies' masses: fixed for the whole stage
  load_mass(B, a, A);
  load_mass(B, b, Bb);
  gate([&]() {
    const double ima = A.im, imb = Bb.im;
    const double* va = B.vw + 8 * a;
    const double* vb = B.vw + 8 * b;
    double vax = ldm(va), vay = ldm(va + 1), vaz = ldm(va + 2), wax = ldm(va + 3), way = ldm(va + 4), waz = ldm(va + 5);
    double vbx = ldm(vb), vby = ldm(vb + 1), vbz = ldm(vb + 2), wbx = ldm(vb + 3), wby = ldm(vb + 4), wbz = ldm(vb + 5);
#pragma unroll
    for (int k = 0; k < N; k++) {
      const double l = ln[k];
      const double px = nx * l, py = ny * l, pz = nz * l;
      vax -= ima * px; vay -= ima * py; vaz -= ima * pz;
      vbx += imb * px; vby += imb * py; vbz += imb * pz;
      wax -= ia[k][0] * l; way -= ia[k][1] * l; waz -= ia[k][2] * l;
      wbx += ib[k][0] * l; wby += ib[k][1] * l; wbz += ib[k][2] * l;
    }
    {
      const double px = t1x * l1 + t2x * l2, py = t1y * l1 + t2y * l2, pz = t1z * l1 + t2z * l2;
      vax -= ima * px; vay -= ima * py; vaz -= ima * pz;
      vbx += imb * px; vby += imb * py; vbz += imb * pz;
      wax -= fa[0] * l1 + fa[3] * l2; way -= fa[1] * l1 + fa[4] * l2; waz -= fa[2] * l1 + fa[5] * l2;
      wbx += fb[0] * l1 + fb[3] * l2; wby += fb[1] * l1 + fb[4] * l2; wbz += fb[2] * l1 + fb[5] * l2;
    }
    {
      const double* Ia = A.I;
      const double* Ib = Bb.I;
      const double lx = t1x * r1 + t2x * r2 + nx * sp, ly = t1y * r1 + t2y * r2 + ny * sp, lz = t1z * r1 + t2z * r2 + nz * sp;
      wax -= Ia[0] * lx + Ia[1] * ly + Ia[2] * lz;
      way -= Ia[1] * lx + Ia[3] * ly + Ia[4] * lz;
      waz -= Ia[2] * lx + Ia[4] * ly + Ia[5] * lz;
      wbx += Ib[0] * lx + Ib[1] * ly + Ib[2] * lz;
      wby += Ib[1] * lx + Ib[3] * ly + Ib[4] * lz;
      wbz += Ib[2] * lx + Ib[4] * ly + Ib[5] * lz;
    }
    write_back(B, ima, a, vax, vay, vaz, wax, way, waz);
    write_back(B, imb, b, vbx, vby, vbz, wbx, wby, wbz);
  });
}

template <class Gate>
__device__ __forceinline__ void warm_row(const StageParams& p, int m, Gate gate) {
  switch (ldi(p.R.points + m)) {
    case 1: warm_row_n<1>(p, m, gate); break;
    case 2: warm_row_n<2>(p, m, gate); break;
    case 3: warm_row_n<3>(p, m, gate); break;
    default: warm_row_n<4>(p, m, gate); break;
  }
}

// pushes: src/contact.js:1672-1724.  The set of every point, which a resting manifold takes on
// nearly every pass, has its own instance per point count with every index a compile-time constant
// (the reference's own written-out set-15 path for four points is exactly these operations); any
// other set takes the reference's loops, over index lists in local memory.  One unrolled instance
// per point count rather than one per set keeps the row solver's code small.
__host__ __device__ constexpr int set_size(int set, int n) {
  return n == 0 ? 0 : ((set & 1) + set_size(set >> 1, n - 1));
}
// The r-th point of SET (the reference's IN[r]).
__host__ __device__ constexpr int set_point(int set, int r, int k = 0) {
  return (set & 1) ? (r == 0 ? k : set_point(set >> 1, r - 1, k + 1)) : set_point(set >> 1, r, k + 1);
}

template <int N, int SET>
__device__ __forceinline__ void solve_set(const double (&K)[N][N], const double (&give)[N], const double (&wanted)[N],
                                          double (&solved)[N]) {
  constexpr int n = set_size(SET, N);
#pragma unroll
  for (int k = 0; k < N; k++) solved[k] = 0;
  if (n == 0) return;
  double AS[n > 0 ? n : 1][n > 0 ? n : 1], RS[n > 0 ? n : 1], XS[n > 0 ? n : 1];
#pragma unroll
  for (int r = 0; r < n; r++) {
#pragma unroll
    for (int s = 0; s < n; s++) AS[r][s] = K[set_point(SET, r)][set_point(SET, s)];
    AS[r][r] *= 1 + give[set_point(SET, r)];
    RS[r] = wanted[set_point(SET, r)];
  }
#pragma unroll
  for (int col = 0; col < n; col++) {
    const double pivot = AS[col][col];
#pragma unroll
    for (int r = col + 1; r < n; r++) {
      const double f = AS[r][col] / pivot;
#pragma unroll
      for (int s = col + 1; s < n; s++) AS[r][s] -= f * AS[col][s];
      RS[r] -= f * RS[col];
    }
  }
#pragma unroll
  for (int r = n - 1; r >= 0; r--) {
    double x = RS[r];
#pragma unroll
    for (int s = r + 1; s < n; s++) x -= AS[r][s] * XS[s];
    XS[r] = x / AS[r][r];
    solved[set_point(SET, r)] = XS[r];
  }
}

// Any subset, by the reference's own loops (src/contact.js:1700-1723): index lists and a small
// matrix in local memory, the same operations in the same order.
template <int N>
__device__ __forceinline__ void pushes_any(const double (&K)[N][N], int set, const double (&give)[N],
                                           const double (&wanted)[N], double (&solved)[N]) {
  double Kl[N * N], gl[N], wl[N], sl[N];
#pragma unroll
  for (int k = 0; k < N; k++) {
    gl[k] = give[k]; wl[k] = wanted[k]; sl[k] = 0;
#pragma unroll
    for (int l = 0; l < N; l++) Kl[k * N + l] = K[k][l];
  }
  int in[N];
  int n = 0;
#pragma unroll 1
  for (int k = 0; k < N; k++)
    if (set >> k & 1) in[n++] = k;
  double AS[N * N], RS[N], XS[N];
#pragma unroll 1
  for (int r = 0; r < n; r++) {
    const int kr = in[r];
#pragma unroll 1
    for (int s = 0; s < n; s++) AS[r * N + s] = Kl[kr * N + in[s]];
    AS[r * N + r] *= 1 + gl[kr];
    RS[r] = wl[kr];
  }
#pragma unroll 1
  for (int col = 0; col < n; col++) {
    const double pivot = AS[col * N + col];
#pragma unroll 1
    for (int r = col + 1; r < n; r++) {
      const double f = AS[r * N + col] / pivot;
#pragma unroll 1
      for (int s = col + 1; s < n; s++) AS[r * N + s] -= f * AS[col * N + s];
      RS[r] -= f * RS[col];
    }
  }
#pragma unroll 1
  for (int r = n - 1; r >= 0; r--) {
    double x = RS[r];
#pragma unroll 1
    for (int s = r + 1; s < n; s++) x -= AS[r * N + s] * XS[s];
    XS[r] = x / AS[r * N + r];
    sl[in[r]] = XS[r];
  }
#pragma unroll
  for (int k = 0; k < N; k++) solved[k] = sl[k];
}

template <int N>
__device__ __forceinline__ void pushes_n(const double (&K)[N][N], int set, const double (&give)[N],
                                         const double (&wanted)[N], double (&solved)[N]) {
  if (set == (1 << N) - 1) solve_set<N, (1 << N) - 1>(K, give, wanted, solved);
  else pushes_any<N>(K, set, give, wanted, solved);
}

// solveRows for row m, one pass, a row of N points: src/contact.js:1805-2090.  The row's own
// columns are read first, then what no row of the pass can change: its bodies' masses (fixed for
// the stage) and, where the separations are worked out, their poses (moves happen between passes),
// with the separations and soft targets they give.  The rest (its bodies' velocities, the
// arithmetic, every store at the end) is handed to `gate`, which runs it once the rows before it
// on its bodies are done (the grid) or at once (a CTA).  So once its bodies are ready, the row
// costs one trip to memory (their two velocity records) and its velocity arithmetic.
//
// BIAS: the biased solve (the substep's first pass) or relax; KNOWN: the separations the last relax
// pass left in `now` still hold (src/contact.js:1802-1803, 1852), or they are worked out from the
// bodies' drift.  Each pass kind is its own instance, carrying only the values it uses.
template <int N, bool BIAS, bool KNOWN, class Gate>
__device__ void solve_row_n(const StageParams& p, int m, double h, Gate gate) {
  constexpr bool bias = BIAS, known = KNOWN;
  const RowsDev& R = p.R;
  const BodiesDev& B = p.B;
  const int64_t cap = R.cap;
  const Soft soft = p.soft;
  const double inv = 1 / h;
  const double springy = soft.impulseScale / soft.massScale + COMPLIANCE;
  // ---- the row's own columns ----
  const int a = ldi(R.a + m), b = ldi(R.b + m);
  const double nx = ldi(R.n + m), ny = ldi(R.n + cap + m), nz = ldi(R.n + 2 * cap + m);
  const double maxBias = ldi(R.tolerance + m) * inv;
  double sep[N];
  double la[N][3], lb[N][3];
  if (known) {
#pragma unroll
    for (int k = 0; k < N; k++) sep[k] = ldm(R.now + k * cap + m);
  } else {
#pragma unroll
    for (int k = 0; k < N; k++) {
      sep[k] = ldm(R.adjusted + k * cap + m);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        la[k][c] = ldm(R.la + (k * 3 + c) * cap + m);
        lb[k][c] = ldm(R.lb + (k * 3 + c) * cap + m);
      }
    }
  }
  double ni[N], jn[N][6], jw[N][6], mx[N], nmass[N], lev[N];
#pragma unroll
  for (int k = 0; k < N; k++) {
    ni[k] = ldm(R.ni + k * cap + m);
    mx[k] = ldm(R.maxni + k * cap + m);
    nmass[k] = ldm(R.normalMass + k * cap + m);
    lev[k] = ldm(R.lever + k * cap + m);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      jn[k][c] = ldm(R.jac + (k * J + c) * cap + m);
      jw[k][c] = ldm(R.jac + (k * J + 6 + c) * cap + m);
    }
  }
  double Kb[N][N];
  if (N >= 2) {
#pragma unroll
    for (int k = 0; k < N; k++)
#pragma unroll
      for (int l = 0; l < N; l++) Kb[k][l] = ldm(R.K + (P * k + l) * cap + m);
  }
  const double mu = ldi(R.friction + m), patch = ldi(R.patch + m);
  const double t1x = ldi(R.t1 + m), t1y = ldi(R.t1 + cap + m), t1z = ldi(R.t1 + 2 * cap + m);
  const double t2x = ldi(R.t2 + m), t2y = ldi(R.t2 + cap + m), t2z = ldi(R.t2 + 2 * cap + m);
  double fj[FJ];
#pragma unroll
  for (int c = 0; c < FJ; c++) fj[c] = ldm(R.fjac + c * cap + m);
  const double s1 = ldm(R.drift1 + m), s2 = ldm(R.drift2 + m);
  const double tm0 = ldm(R.tm + m), tm1 = ldm(R.tm + cap + m), tm2 = ldm(R.tm + 2 * cap + m);
  const double o1 = ldm(R.ti1 + m), o2 = ldm(R.ti2 + m);
  double r1 = 0, r2 = 0, rm1 = 0, rm2 = 0;
  if (N <= 2) {
    r1 = ldm(R.ri1 + m); r2 = ldm(R.ri2 + m);
    rm1 = ldm(R.rm1 + m); rm2 = ldm(R.rm2 + m);
  }
  const double s0 = ldm(R.si + m), smass = ldm(R.sm + m);
  // ---- what the pass cannot change: the bodies' masses (fixed for the stage) and, where the
  // separations are worked out, their poses (moves happen between passes) ----
  BodyLoad A, Bb;
  load_mass(B, a, A);
  load_mass(B, b, Bb);
  double dn = 0, nax = 0, nay = 0, naz = 0, nbx = 0, nby = 0, nbz = 0;
  if (!known) {
    const double* pqa = B.pq + 8 * a;
    const double* pqb = B.pq + 8 * b;
    const double* sta = B.st + 4 * a;
    const double* stb = B.st + 4 * b;
    const double dx = (ldm(pqb) - ldm(stb)) - (ldm(pqa) - ldm(sta));
    const double dy = (ldm(pqb + 1) - ldm(stb + 1)) - (ldm(pqa + 1) - ldm(sta + 1));
    const double dz = (ldm(pqb + 2) - ldm(stb + 2)) - (ldm(pqa + 2) - ldm(sta + 2));
    dn = dx * nx + dy * ny + dz * nz;
    double qa[4], qb[4], v3[3];
#pragma unroll
    for (int k = 0; k < 4; k++) { qa[k] = ldm(pqa + 4 + k); qb[k] = ldm(pqb + 4 + k); }
    rotate(qa, nx, ny, nz, true, v3);
    nax = v3[0]; nay = v3[1]; naz = v3[2];
    rotate(qb, nx, ny, nz, true, v3);
    nbx = v3[0]; nby = v3[1]; nbz = v3[2];
  }
  // ---- the arithmetic, in the reference's order ----
  double target[N], massScale[N], impulseScale[N], give[N], nowv[N];
  double least = INFINITY;
#pragma unroll
  for (int k = 0; k < N; k++) {
    double s;
    if (known) {
      s = sep[k];
    } else {
      s = dn + (lb[k][0] * nbx + lb[k][1] * nby + lb[k][2] * nbz) - (la[k][0] * nax + la[k][1] * nay + la[k][2] * naz)
        + sep[k];
    }
    nowv[k] = s;
    if (s < least) least = s;
    if (s > 0) {
      target[k] = s * inv; massScale[k] = 1; impulseScale[k] = 0; give[k] = COMPLIANCE;
    } else if (bias) {
      target[k] = js_max(soft.biasRate * s, -maxBias);
      massScale[k] = soft.massScale; impulseScale[k] = soft.impulseScale; give[k] = springy;
    } else {
      target[k] = 0; massScale[k] = 1; impulseScale[k] = 0; give[k] = COMPLIANCE;
    }
  }
  // ---- the rows before this one on its bodies ----
  gate([&]() {
    // ---- its bodies' velocities, the only thing the rows before it change ----
    const double* va = B.vw + 8 * a;
    const double* vb = B.vw + 8 * b;
    double vax = ldm(va), vay = ldm(va + 1), vaz = ldm(va + 2), wax = ldm(va + 3), way = ldm(va + 4), waz = ldm(va + 5);
    double vbx = ldm(vb), vby = ldm(vb + 1), vbz = ldm(vb + 2), wbx = ldm(vb + 3), wby = ldm(vb + 4), wbz = ldm(vb + 5);
    const double ima = A.im, imb = Bb.im;
    double closingNow[N], solved[N];
    if (N == 1 || !(Kb[0][0] > 0)) {
#pragma unroll
      for (int k = 0; k < N; k++) {
        const double* jac = jn[k];
        const double vn = (vbx - vax) * nx + (vby - vay) * ny + (vbz - vaz) * nz
          + wbx * jac[3] + wby * jac[4] + wbz * jac[5] - wax * jac[0] - way * jac[1] - waz * jac[2];
        const double old = ni[k];
        double next = old - nmass[k] * massScale[k] * (vn + target[k]) - impulseScale[k] * old;
        if (next < 0) next = 0;
        closingNow[k] = vn; solved[k] = next;
      }
    } else {
#pragma unroll
      for (int k = 0; k < N; k++) {
        const double* jac = jn[k];
        closingNow[k] = (vbx - vax) * nx + (vby - vay) * ny + (vbz - vaz) * nz
          + wbx * jac[3] + wby * jac[4] + wbz * jac[5] - wax * jac[0] - way * jac[1] - waz * jac[2];
      }
      double wanted[N];
      int set = 0;
#pragma unroll
      for (int k = 0; k < N; k++) {
        double r = -closingNow[k] - target[k];
#pragma unroll
        for (int l = 0; l < N; l++) r += Kb[k][l] * ni[l];
        wanted[k] = r;
        if (r > 0) set |= 1 << k;
      }
      for (int round = 0;; round++) {
        pushes_n<N>(Kb, set, give, wanted, solved);
        int flip = -1;
#pragma unroll
        for (int k = 0; k < N; k++) {
          if (flip < 0) {
            if (set >> k & 1) {
              if (solved[k] < 0) flip = k;
            } else {
              double r = -wanted[k];
#pragma unroll
              for (int l = 0; l < N; l++) r += Kb[k][l] * solved[l];
              if (r < 0) flip = k;
            }
          }
        }
        if (flip < 0 || round == 1 << N) break;
        set ^= 1 << flip;
      }
    }
    double rv[N];
    bool rvset[N];
#pragma unroll
    for (int k = 0; k < N; k++) {
      const double old = ni[k], next = solved[k] > 0 ? solved[k] : 0;
      const double d = next - old;
      ni[k] = next;
      rvset[k] = d > 0 && mx[k] == 0;
      rv[k] = closingNow[k];
      if (d > mx[k]) mx[k] = d;
      const double px = nx * d, py = ny * d, pz = nz * d;
      vax -= ima * px; vay -= ima * py; vaz -= ima * pz;
      vbx += imb * px; vby += imb * py; vbz += imb * pz;
      wax -= jw[k][0] * d; way -= jw[k][1] * d; waz -= jw[k][2] * d;
      wbx += jw[k][3] * d; wby += jw[k][4] * d; wbz += jw[k][5] * d;
    }
    double pressed = 0, twisted = 0;
#pragma unroll
    for (int k = 0; k < N; k++) {
      pressed += ni[k];
      twisted += lev[k] * ni[k];
    }
    double n1f, n2f;
    uint8_t sliding;
    {
      const double* g = fj + 12;
      const double dvx = vbx - vax, dvy = vby - vay, dvz = vbz - vaz;
      double v1 = dvx * t1x + dvy * t1y + dvz * t1z + wbx * fj[3] + wby * fj[4] + wbz * fj[5] - wax * fj[0] - way * fj[1] - waz * fj[2];
      double v2 = dvx * t2x + dvy * t2y + dvz * t2z + wbx * g[3] + wby * g[4] + wbz * g[5] - wax * g[0] - way * g[1] - waz * g[2];
      if (bias && (s1 != 0 || s2 != 0)) {
        double b1 = soft.biasRate * s1, b2 = soft.biasRate * s2;
        const double bb = b1 * b1 + b2 * b2;
        if (bb > maxBias * maxBias) {
          const double scale = maxBias / sqrt(bb);
          b1 *= scale; b2 *= scale;
        }
        v1 += b1; v2 += b2;
      }
      double n1 = o1 - (tm0 * v1 + tm1 * v2), n2 = o2 - (tm1 * v1 + tm2 * v2);
      const double limit = mu * pressed, l2 = n1 * n1 + n2 * n2;
      if (l2 > limit * limit) {
        const double ma = tm0, mb = tm1, mc = tm2;
        double al = 0, x = n1, y = n2, ll = l2;
        while (limit > 0) {
          const double ab = al * mb, d = (1 + al * ma) * (1 + al * mc) - ab * ab;
          const double px = ma * x + mb * y, py = mb * x + mc * y;
          const double wx = ((1 + al * mc) * px - ab * py) / d, wy = ((1 + al * ma) * py - ab * px) / d;
          const double lw = x * wx + y * wy;
          if (!(lw > 0)) break;
          const double next = al + (sqrt(ll) / limit - 1) * ll / lw;
          if (!(next > al)) break;
          al = next;
          const double ab2 = al * mb, d2 = (1 + al * ma) * (1 + al * mc) - ab2 * ab2;
          x = ((1 + al * mc) * n1 - ab2 * n2) / d2; y = ((1 + al * ma) * n2 - ab2 * n1) / d2;
          ll = x * x + y * y;
          if (!(ll > limit * limit)) break;
        }
        const double scale = limit / sqrt(ll);
        n1 = x * scale; n2 = y * scale;
        sliding = 1;
      } else {
        sliding = 0;
      }
      n1f = n1; n2f = n2;
      const double d1 = n1 - o1, d2 = n2 - o2;
      const double px = t1x * d1 + t2x * d2, py = t1y * d1 + t2y * d2, pz = t1z * d1 + t2z * d2;
      vax -= ima * px; vay -= ima * py; vaz -= ima * pz;
      vbx += imb * px; vby += imb * py; vbz += imb * pz;
      wax -= fj[6] * d1 + g[6] * d2; way -= fj[7] * d1 + g[7] * d2; waz -= fj[8] * d1 + g[8] * d2;
      wbx += fj[9] * d1 + g[9] * d2; wby += fj[10] * d1 + g[10] * d2; wbz += fj[11] * d1 + g[11] * d2;
    }
    const double* Ia = A.I;
    const double* Ib = Bb.I;
    double r1f = 0, r2f = 0;
    if (N <= 2) {
      const double most = patch * pressed;
      const double ux = wbx - wax, uy = wby - way, uz = wbz - waz;
      double n1 = r1 - rm1 * (ux * t1x + uy * t1y + uz * t1z);
      double n2 = r2 - rm2 * (ux * t2x + uy * t2y + uz * t2z);
      const double l2 = n1 * n1 + n2 * n2;
      if (l2 > most * most) {
        const double scale = most / sqrt(l2);
        n1 *= scale; n2 *= scale;
      }
      r1f = n1; r2f = n2;
      const double d1 = n1 - r1, d2 = n2 - r2;
      const double lx = t1x * d1 + t2x * d2, ly = t1y * d1 + t2y * d2, lz = t1z * d1 + t2z * d2;
      wax -= Ia[0] * lx + Ia[1] * ly + Ia[2] * lz;
      way -= Ia[1] * lx + Ia[3] * ly + Ia[4] * lz;
      waz -= Ia[2] * lx + Ia[4] * ly + Ia[5] * lz;
      wbx += Ib[0] * lx + Ib[1] * ly + Ib[2] * lz;
      wby += Ib[1] * lx + Ib[3] * ly + Ib[4] * lz;
      wbz += Ib[2] * lx + Ib[4] * ly + Ib[5] * lz;
    }
    double s1f;
    {
      const double limit = N == 1 ? SPIN_DISC * mu * patch * pressed : mu * twisted;
      double sv = s0 - smass * ((wbx - wax) * nx + (wby - way) * ny + (wbz - waz) * nz);
      if (sv > limit) sv = limit; else if (sv < -limit) sv = -limit;
      s1f = sv;
      const double ds = sv - s0, lx = nx * ds, ly = ny * ds, lz = nz * ds;
      wax -= Ia[0] * lx + Ia[1] * ly + Ia[2] * lz;
      way -= Ia[1] * lx + Ia[3] * ly + Ia[4] * lz;
      waz -= Ia[2] * lx + Ia[4] * ly + Ia[5] * lz;
      wbx += Ib[0] * lx + Ib[1] * ly + Ib[2] * lz;
      wby += Ib[1] * lx + Ib[3] * ly + Ib[4] * lz;
      wbz += Ib[2] * lx + Ib[4] * ly + Ib[5] * lz;
    }
    // ---- every store, last: the bodies first, which the rows after this one wait for ----
    write_back(B, ima, a, vax, vay, vaz, wax, way, waz);
    write_back(B, imb, b, vbx, vby, vbz, wbx, wby, wbz);
#pragma unroll
    for (int k = 0; k < N; k++) {
      if (!known && !bias) stm(R.now + k * cap + m, nowv[k]);
      stm(R.ni + k * cap + m, ni[k]);
      if (rvset[k]) stm(R.relvel + k * cap + m, rv[k]);
      stm(R.maxni + k * cap + m, mx[k]);
    }
    stm(R.gap + m, least);
    stm(R.sliding + m, sliding);
    stm(R.ti1 + m, n1f); stm(R.ti2 + m, n2f);
    if (N <= 2) { stm(R.ri1 + m, r1f); stm(R.ri2 + m, r2f); }
    stm(R.si + m, s1f);
  });
}

template <bool BIAS, bool KNOWN, class Gate>
__device__ __forceinline__ void solve_row(const StageParams& p, int m, double h, Gate gate) {
  switch (ldi(p.R.points + m)) {
    case 1: solve_row_n<1, BIAS, KNOWN>(p, m, h, gate); break;
    case 2: solve_row_n<2, BIAS, KNOWN>(p, m, h, gate); break;
    case 3: solve_row_n<3, BIAS, KNOWN>(p, m, h, gate); break;
    default: solve_row_n<4, BIAS, KNOWN>(p, m, h, gate); break;
  }
}

// The substep's biased pass: the first substep works the separations out, later ones take the
// relax pass's (src/contact.js:1802-1803).
template <class Gate>
__device__ __forceinline__ void solve_biased(const StageParams& p, int m, double h, int sub, Gate gate) {
  if (sub > 0) solve_row<true, true>(p, m, h, gate);
  else solve_row<true, false>(p, m, h, gate);
}

// Whether any of six doubles differs in its bits from what is stored at q.
__device__ __forceinline__ bool changed6(const double* v, const double* q) {
  bool any = false;
  for (int c = 0; c < 6; c++)
    any |= __double_as_longlong(v[c]) != __double_as_longlong(ldm(q + c));
  return any;
}

// Whether row m has a point restitution() works on: src/contact.js:2233-2241.  What it reads
// (relativeVelocity, maxNormalImpulse) restitution() never changes, so this holds throughout.
__device__ __forceinline__ bool bouncy(const StageParams& p, int m, int solved_end, double gravity) {
  const RowsDev& R = p.R;
  const int64_t cap = R.cap;
  const double e = ldi(R.restitution + m);
  if (e == 0 || m >= solved_end) return false;
  const double threshold = sqrt(2 * gravity * ldi(R.tolerance + m));
  const int count = ldi(R.points + m);
  for (int k = 0; k < count; k++) {
    if (ldm(R.relvel + k * cap + m) > -threshold || ldm(R.maxni + k * cap + m) == 0) continue;
    return true;
  }
  return false;
}

// restitution for row m: src/contact.js:2234-2250 (closing 2216-2220, push 1743-1749).
//
// push() also writes a body with inverse mass 0 (a static or kinematic one): v -= 0 * px, which
// leaves its bits alone unless px is not finite (0 * inf is NaN) or a -0 component meets a -0
// product.  Rows of one round share such bodies, so the rounds (EXACT false) leave them unwritten
// and instead raise *redo where push() would have changed one: restitution_stage then redoes the
// world's restitution one row at a time in found order (EXACT true), writing every body as push()
// does.  Until a push would change such a body, both ways give the same bits (each dynamic body
// sees its pushes in found order either way).
template <bool EXACT>
__device__ void bounce_row(const StageParams& p, int m, double gravity, int* redo) {
  const RowsDev& R = p.R;
  const BodiesDev& B = p.B;
  const int64_t cap = R.cap;
  const double e = ldi(R.restitution + m);
  const double threshold = sqrt(2 * gravity * ldi(R.tolerance + m));
  const int a = ldi(R.a + m), b = ldi(R.b + m);
  const double nx = ldi(R.n + m), ny = ldi(R.n + cap + m), nz = ldi(R.n + 2 * cap + m);
  const double ima = ldm(B.mi + 8 * a), imb = ldm(B.mi + 8 * b);
  double* pa = B.vw + 8 * a;
  double* pb = B.vw + 8 * b;
  double va[6], vb[6];
  for (int c = 0; c < 6; c++) { va[c] = ldm(pa + c); vb[c] = ldm(pb + c); }
  const int count = ldi(R.points + m);
  for (int k = 0; k < count; k++) {
    const double rv = ldm(R.relvel + k * cap + m);
    if (rv > -threshold || ldm(R.maxni + k * cap + m) == 0) continue;
    const double* jac = R.jac + (k * J) * cap + m;
    const double vn = (vb[0] - va[0]) * nx + (vb[1] - va[1]) * ny + (vb[2] - va[2]) * nz
      + vb[3] * ldm(jac + 3 * cap) + vb[4] * ldm(jac + 4 * cap) + vb[5] * ldm(jac + 5 * cap)
      - va[3] * ldm(jac) - va[4] * ldm(jac + cap) - va[5] * ldm(jac + 2 * cap);
    const double old = ldm(R.ni + k * cap + m);
    double next = old - ldm(R.normalMass + k * cap + m) * (vn + e * rv);
    if (next < 0) next = 0;
    const double d = next - old;
    stm(R.ni + k * cap + m, next);
    const double px = nx * d, py = ny * d, pz = nz * d;
    va[0] -= ima * px; va[1] -= ima * py; va[2] -= ima * pz;
    vb[0] += imb * px; vb[1] += imb * py; vb[2] += imb * pz;
    va[3] -= ldm(jac + 6 * cap) * d; va[4] -= ldm(jac + 7 * cap) * d; va[5] -= ldm(jac + 8 * cap) * d;
    vb[3] += ldm(jac + 9 * cap) * d; vb[4] += ldm(jac + 10 * cap) * d; vb[5] += ldm(jac + 11 * cap) * d;
  }
  if (EXACT) {
    for (int c = 0; c < 6; c++) stm(pa + c, va[c]);
    for (int c = 0; c < 6; c++) stm(pb + c, vb[c]);
    return;
  }
  if (ima != 0) for (int c = 0; c < 6; c++) stm(pa + c, va[c]);
  else if (changed6(va, pa)) *redo = 1;
  if (imb != 0) for (int c = 0; c < 6; c++) stm(pb + c, vb[c]);
  else if (changed6(vb, pb)) *redo = 1;
}

// turned: src/contact.js:1168-1182.
__device__ void turned(const BodiesDev& B, int s, double* T) {
  double q[4], q0[4];
  for (int k = 0; k < 4; k++) { q[k] = ldm(B.pq + 8 * s + 4 + k); q0[k] = ldm(B.sq + 4 * s + k); }
  const double ax = q[0], ay = q[1], az = q[2], aw = q[3];
  const double bx = -q0[0], by = -q0[1], bz = -q0[2], bw = q0[3];
  double ux = aw * bx + ax * bw + ay * bz - az * by;
  double uy = aw * by + ay * bw + az * bx - ax * bz;
  double uz = aw * bz + az * bw + ax * by - ay * bx;
  double uw = aw * bw - ax * bx - ay * by - az * bz;
  if (uw < 0) { ux = -ux; uy = -uy; uz = -uz; uw = -uw; }
  const double sine = sqrt(ux * ux + uy * uy + uz * uz);
  const double k = sine == 0 ? 0 : 2 * ref_atan2(sine, uw) / sine;
  for (int c = 0; c < 3; c++) T[c] = ldm(B.pq + 8 * s + c) - ldm(B.st + 4 * s + c);
  T[3] = ux * k; T[4] = uy * k; T[5] = uz * k;
}

// slipped for row m: src/contact.js:1122-1153.
__device__ void slipped_row(const StageParams& p, int m) {
  const RowsDev& R = p.R;
  const BodiesDev& B = p.B;
  const int64_t cap = R.cap;
  const int a = ldi(R.a + m), b = ldi(R.b + m);
  const int count = ldi(R.points + m);
  double pressed = 0;
  bool impact = false;
  for (int k = 0; k < count; k++) {
    pressed += ldm(R.ni + k * cap + m);
    if (ldi(R.shift + (k * 3) * cap + m) != 0 || ldi(R.shift + (k * 3 + 1) * cap + m) != 0 ||
        ldi(R.shift + (k * 3 + 2) * cap + m) != 0)
      impact = true;
  }
  if (ldm(R.sliding + m) != 0 || pressed == 0 || impact) {
    stm(R.drift1 + m, 0.0); stm(R.drift2 + m, 0.0);
    return;
  }
  double T[6];
  double dx = 0, dy = 0, dz = 0;
  if (ldi(B.fl + b) & F_AWAKE) {
    turned(B, b, T);
    const double rx = ldm(R.anchorB + m), ry = ldm(R.anchorB + cap + m), rz = ldm(R.anchorB + 2 * cap + m);
    dx = T[0] + T[4] * rz - T[5] * ry;
    dy = T[1] + T[5] * rx - T[3] * rz;
    dz = T[2] + T[3] * ry - T[4] * rx;
  }
  if (ldi(B.fl + a) & F_AWAKE) {
    turned(B, a, T);
    const double rx = ldm(R.anchorA + m), ry = ldm(R.anchorA + cap + m), rz = ldm(R.anchorA + 2 * cap + m);
    dx -= T[0] + T[4] * rz - T[5] * ry;
    dy -= T[1] + T[5] * rx - T[3] * rz;
    dz -= T[2] + T[3] * ry - T[4] * rx;
  }
  const double t1x = ldi(R.t1 + m), t1y = ldi(R.t1 + cap + m), t1z = ldi(R.t1 + 2 * cap + m);
  const double t2x = ldi(R.t2 + m), t2y = ldi(R.t2 + cap + m), t2z = ldi(R.t2 + 2 * cap + m);
  stm(R.drift1 + m, ldm(R.drift1 + m) + (dx * t1x + dy * t1y + dz * t1z));
  stm(R.drift2 + m, ldm(R.drift2 + m) + (dx * t2x + dy * t2y + dz * t2z));
}

// ---- the stage ----

// restitution over one world's rows in found order, run by the lead block: the bouncy rows are
// listed in found order, then taken in rounds, each round every listed row whose dynamic bodies
// no earlier listed row still waits on; so each body sees its rows' pushes in found order.
template <class Team>
__device__ bool restitution_stage(const StageParams& p, const WorldDesc& w, const Team& t, double gravity) {
  const RowsDev& R = p.R;
  const BodiesDev& B = p.B;
  const int nrows = w.nrows;
  const int solved_end = w.row0 + w.solved;
  // 1. The bouncy rows, in found order: each block counts its share, then writes it in order.
  __shared__ int s_scan[1024];
  __shared__ int s_base;
  __shared__ int s_own_count;
  // Per-block counts: in global memory for a grid team, which spans blocks; a block team's own.
  int* counts = Team::kGrid ? p.block_counts : &s_own_count;
  const int nblocks = (t.size + static_cast<int>(blockDim.x) - 1) / static_cast<int>(blockDim.x);
  const int bid = t.rank / static_cast<int>(blockDim.x);
  const int per = (nrows + nblocks - 1) / nblocks;
  const int from = bid * per, to = min(nrows, from + per);
  int mine = 0;
  for (int f = from + static_cast<int>(threadIdx.x); f < to; f += blockDim.x) {
    if (bouncy(p, ldi(R.row + w.row0 + f), solved_end, gravity)) mine++;
  }
  // block sum
  s_scan[threadIdx.x] = mine;
  __syncthreads();
  for (int off = 1; off < static_cast<int>(blockDim.x); off <<= 1) {
    const int v = threadIdx.x >= static_cast<unsigned>(off) ? s_scan[threadIdx.x - off] : 0;
    __syncthreads();
    s_scan[threadIdx.x] += v;
    __syncthreads();
  }
  if (threadIdx.x == blockDim.x - 1) counts[bid] = s_scan[threadIdx.x];
  if (!t.sync(p)) return false;
  if (threadIdx.x == 0) {
    int base = 0;
    for (int k = 0; k < bid; k++) base += Team::kGrid ? ldm(counts + k) : counts[k];
    s_base = base;
  }
  __syncthreads();
  // write this block's bouncy rows in order, a chunk of blockDim at a time
  int written = s_base;
  for (int f0 = from; f0 < to; f0 += blockDim.x) {
    const int f = f0 + static_cast<int>(threadIdx.x);
    const bool on = f < to && bouncy(p, ldi(R.row + w.row0 + f), solved_end, gravity);
    s_scan[threadIdx.x] = on ? 1 : 0;
    __syncthreads();
    for (int off = 1; off < static_cast<int>(blockDim.x); off <<= 1) {
      const int v = threadIdx.x >= static_cast<unsigned>(off) ? s_scan[threadIdx.x - off] : 0;
      __syncthreads();
      s_scan[threadIdx.x] += v;
      __syncthreads();
    }
    if (on) stm(R.active + w.row0 + written + s_scan[threadIdx.x] - 1, ldi(R.row + w.row0 + f));
    written += s_scan[blockDim.x - 1];
    __syncthreads();
  }
  if (!t.sync(p)) return false;
  // 2. The rounds, by the lead block alone.
  if (t.lead) {
    __shared__ int s_total;
    if (threadIdx.x == 0) {
      int total = 0;
      for (int k = 0; k < nblocks; k++) total += Team::kGrid ? ldm(counts + k) : counts[k];
      s_total = total;
    }
    __shared__ int s_redo;
    if (threadIdx.x == 0) s_redo = 0;
    __syncthreads();
    int n = s_total;
    int32_t* list = R.active + w.row0;
    int32_t* next = R.pending + w.row0;
    // What a redo starts from: each listed row's two bodies' velocities and its normal impulses as
    // restitution begins, kept in the row's la and now columns (read only by the substeps' passes,
    // which are over).
    const int64_t cap = R.cap;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int m = ldm(list + i);
      const int a = ldi(R.a + m), b = ldi(R.b + m);
      for (int c = 0; c < 6; c++) {
        stm(R.la + c * cap + m, ldm(B.vw + 8 * a + c));
        stm(R.la + (6 + c) * cap + m, ldm(B.vw + 8 * b + c));
      }
      for (int k = 0; k < P; k++) stm(R.now + k * cap + m, ldm(R.ni + k * cap + m));
    }
    __syncthreads();
    int guard = 0;
    while (n > 0 && guard++ < nrows + 1) {
      // every pending row bids for its dynamic bodies with its place in the list
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int m = ldm(list + i);
        const int a = ldi(R.a + m), b = ldi(R.b + m);
        if (ldm(B.mi + 8 * a) != 0) atomicMin(B.head + a, i);
        if (ldm(B.mi + 8 * b) != 0) atomicMin(B.head + b, i);
      }
      __syncthreads();
      __threadfence_block();
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int m = ldm(list + i);
        const int a = ldi(R.a + m), b = ldi(R.b + m);
        const bool ra = ldm(B.mi + 8 * a) == 0 || ldm(B.head + a) == i;
        const bool rb = ldm(B.mi + 8 * b) == 0 || ldm(B.head + b) == i;
        if (ra && rb) bounce_row<false>(p, m, gravity, &s_redo);
      }
      __syncthreads();
      // the rows not taken, in order, become the next list; the bids are cleared
      __shared__ int s_kept;
      if (threadIdx.x == 0) s_kept = 0;
      __syncthreads();
      for (int i0 = 0; i0 < n; i0 += blockDim.x) {
        const int i = i0 + static_cast<int>(threadIdx.x);
        int keep = 0, m = 0;
        if (i < n) {
          m = ldm(list + i);
          const int a = ldi(R.a + m), b = ldi(R.b + m);
          const bool ra = ldm(B.mi + 8 * a) == 0 || ldm(B.head + a) == i;
          const bool rb = ldm(B.mi + 8 * b) == 0 || ldm(B.head + b) == i;
          keep = (ra && rb) ? 0 : 1;
        }
        s_scan[threadIdx.x] = keep;
        __syncthreads();
        for (int off = 1; off < static_cast<int>(blockDim.x); off <<= 1) {
          const int v = threadIdx.x >= static_cast<unsigned>(off) ? s_scan[threadIdx.x - off] : 0;
          __syncthreads();
          s_scan[threadIdx.x] += v;
          __syncthreads();
        }
        if (keep) stm(next + s_kept + s_scan[threadIdx.x] - 1, m);
        __syncthreads();
        if (threadIdx.x == 0) s_kept += s_scan[blockDim.x - 1];
        __syncthreads();
      }
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int m = ldm(list + i);
        const int a = ldi(R.a + m), b = ldi(R.b + m);
        atomicExch(B.head + a, 0x7fffffff);
        atomicExch(B.head + b, 0x7fffffff);
      }
      __syncthreads();
      n = s_kept;
      int32_t* tmp = list;
      list = next;
      next = tmp;
      __syncthreads();
    }
    // A push would have changed a body of inverse mass 0: back to the snapshot, then the
    // reference's own order, one row after another, on one thread.
    if (s_redo && threadIdx.x == 0) {
      for (int f = 0; f < nrows; f++) {
        const int m = ldi(R.row + w.row0 + f);
        if (!bouncy(p, m, solved_end, gravity)) continue;
        const int a = ldi(R.a + m), b = ldi(R.b + m);
        for (int c = 0; c < 6; c++) {
          stm(B.vw + 8 * a + c, ldm(R.la + c * cap + m));
          stm(B.vw + 8 * b + c, ldm(R.la + (6 + c) * cap + m));
        }
        for (int k = 0; k < P; k++) stm(R.ni + k * cap + m, ldm(R.now + k * cap + m));
      }
      for (int f = 0; f < nrows; f++) {
        const int m = ldi(R.row + w.row0 + f);
        if (bouncy(p, m, solved_end, gravity)) bounce_row<true>(p, m, gravity, nullptr);
      }
    }
    __syncthreads();
  }
  return t.sync(p);
}

// The whole solve stage for world w, by team t.  Returns false if a barrier gave up.
template <class Team>
__device__ bool solve_stage(const StageParams& p, const WorldDesc& w, const Team& t) {
  const bool touching = w.nrows > 0;
  const int substeps = p.substeps;
  const double h = p.dt / substeps;
  const int* starts = w.starts;
  const int r0 = w.row0;
  t.each(0, w.nawake, [&](int i) { body_begin(p, ldi(p.B.awake_list + w.awake0 + i), touching); });
  if (!t.sync(p)) return false;
  if (touching) {
    t.each(0, w.solved, [&](int m) { prepare_row(p, r0 + m); });
    if (!t.sync(p)) return false;
  }
  int pass = 0;   // row passes so far: the dataflow counters' epoch
  for (int sub = 0; sub < substeps; sub++) {
    t.each(0, w.nawake, [&](int i) { accelerate_body(p, ldi(p.B.awake_list + w.awake0 + i), h, w.gravity); });
    if (!t.sync(p)) return false;
    if (touching) {
      if constexpr (Team::kGrid) {
        // warm and solve flow into each other: a solve row waits for its bodies' warm rows
        flow_pass(p, pass++, [&](int m, auto gate) { warm_row(p, m, gate); });
        if (sub > 0) flow_pass(p, pass++, [&](int m, auto gate) { solve_row<true, true>(p, m, h, gate); });
        else flow_pass(p, pass++, [&](int m, auto gate) { solve_row<true, false>(p, m, h, gate); });
        if (!t.sync(p)) return false;
      } else {
        for (int k = 0; k < NCOLOURS; k++) {
          if (starts[k + 1] <= starts[k]) continue;
          t.each(starts[k], starts[k + 1], [&](int m) { warm_row(p, r0 + m, OpenGate()); });
          if (!t.sync(p)) return false;
        }
        if (starts[OVERFLOW_RUN + 1] > starts[OVERFLOW_RUN]) {
          if (t.rank == 0)
            for (int m = starts[OVERFLOW_RUN]; m < starts[OVERFLOW_RUN + 1]; m++) warm_row(p, r0 + m, OpenGate());
          if (!t.sync(p)) return false;
        }
        for (int k = 0; k < NCOLOURS; k++) {
          if (starts[k + 1] <= starts[k]) continue;
          t.each(starts[k], starts[k + 1], [&](int m) { solve_biased(p, r0 + m, h, sub, OpenGate()); });
          if (!t.sync(p)) return false;
        }
        if (starts[OVERFLOW_RUN + 1] > starts[OVERFLOW_RUN]) {
          if (t.rank == 0)
            for (int m = starts[OVERFLOW_RUN]; m < starts[OVERFLOW_RUN + 1]; m++) solve_biased(p, r0 + m, h, sub, OpenGate());
          if (!t.sync(p)) return false;
        }
      }
    }
    t.each(0, w.nawake, [&](int i) { move_body(p, ldi(p.B.awake_list + w.awake0 + i), h); });
    if (!t.sync(p)) return false;
    if (touching) {
      if constexpr (Team::kGrid) {
        flow_pass(p, pass++, [&](int m, auto gate) { solve_row<false, false>(p, m, h, gate); });
        if (!t.sync(p)) return false;
      } else {
        for (int k = 0; k < NCOLOURS; k++) {
          if (starts[k + 1] <= starts[k]) continue;
          t.each(starts[k], starts[k + 1], [&](int m) { solve_row<false, false>(p, r0 + m, h, OpenGate()); });
          if (!t.sync(p)) return false;
        }
        if (starts[OVERFLOW_RUN + 1] > starts[OVERFLOW_RUN]) {
          if (t.rank == 0)
            for (int m = starts[OVERFLOW_RUN]; m < starts[OVERFLOW_RUN + 1]; m++) solve_row<false, false>(p, r0 + m, h, OpenGate());
          if (!t.sync(p)) return false;
        }
      }
    }
  }
  if (touching) {
    const double* g = w.gravity;
    const double gravity = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    if (!restitution_stage(p, w, t, gravity)) return false;
    t.each(0, w.solved, [&](int m) { slipped_row(p, r0 + m); });
  }
  return true;
}

// Every world of a batch on the persistent grid, as one stage: the body passes over all worlds'
// awake bodies at once (each with its own world's gravity), the row passes as one flow over all
// worlds' runs (worlds share no body, so their rows never wait on each other), and restitution
// and the drift update world by world, one block a world, since both keep each world's found
// order.  The same operations as solve_stage on each world, in each body's same order.
// A flow pass over a batch's runs (each row's turn exactly as in flow_pass).
template <class F>
__device__ __forceinline__ void batch_flow_pass(const StageParams& p, int pass, F row) {
  const int lane = static_cast<int>(threadIdx.x) & 31;
  const int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int warps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
  for (int c = warp; c < p.nbruns; c += warps) {
    const int2 run = p.bruns[c];
    if (lane < run.y) {
      const int m = ldi(p.brun_rows + run.x + lane);
      const int a = ldi(p.R.a + m), b = ldi(p.R.b + m);
      const int ra = ldi(p.R.rank_a + m), rb = ldi(p.R.rank_b + m);
      const unsigned int ta = flow_target(p, a, ra, pass), tb = flow_target(p, b, rb, pass);
      row(m, [&](auto&& finish) {
        long long it = 0;
        for (;;) {
          const unsigned int va = ta == 0 ? 0u : load_relaxed(p.B.done + a);
          const unsigned int vb = tb == 0 ? 0u : load_relaxed(p.B.done + b);
          if (va >= ta && vb >= tb) {
            fence_acq_rel();
            finish();
            flow_signal(p, a, ra, ta, b, rb, tb);
            return true;
          }
          if (++it > p.budget || ((it & 255) == 0 && *(volatile int32_t*)p.status != 0)) {
            atomicExch(p.status, 1);
            return false;
          }
          __nanosleep(200);
        }
      });
    }
    __syncwarp();
  }
}

__device__ bool batch_stage(const StageParams& p) {
  GridTeam t;
  const int substeps = p.substeps;
  const double h = p.dt / substeps;
  const int lane = static_cast<int>(threadIdx.x) & 31;
  const int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int warps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
  // every solved row once: the runs list holds exactly the solved rows of every world
  auto each_row = [&](auto f) {
    for (int c = warp; c < p.nbruns; c += warps) {
      const int2 run = p.bruns[c];
      if (lane < run.y) f(ldi(p.brun_rows + run.x + lane));
    }
  };
  auto world_of_body = [&](int x) -> const WorldDesc& { return p.worlds[ldi(p.body_world + x)]; };
  t.each(0, p.nawake_total, [&](int i) {
    const int x = ldi(p.B.awake_list + i);
    body_begin(p, x, world_of_body(x).nrows > 0);
  });
  if (!t.sync(p)) return false;
  each_row([&](int m) { prepare_row(p, m); });
  if (!t.sync(p)) return false;
  int pass = 0;
  for (int sub = 0; sub < substeps; sub++) {
    t.each(0, p.nawake_total, [&](int i) {
      const int x = ldi(p.B.awake_list + i);
      accelerate_body(p, x, h, world_of_body(x).gravity);
    });
    if (!t.sync(p)) return false;
    batch_flow_pass(p, pass++, [&](int m, auto gate) { warm_row(p, m, gate); });
    if (sub > 0) batch_flow_pass(p, pass++, [&](int m, auto gate) { solve_row<true, true>(p, m, h, gate); });
    else batch_flow_pass(p, pass++, [&](int m, auto gate) { solve_row<true, false>(p, m, h, gate); });
    if (!t.sync(p)) return false;
    t.each(0, p.nawake_total, [&](int i) { move_body(p, ldi(p.B.awake_list + i), h); });
    if (!t.sync(p)) return false;
    batch_flow_pass(p, pass++, [&](int m, auto gate) { solve_row<false, false>(p, m, h, gate); });
    if (!t.sync(p)) return false;
  }
  BlockTeam bt;
  for (int wi = blockIdx.x; wi < p.nworlds; wi += gridDim.x) {
    const WorldDesc w = p.worlds[wi];
    if (w.nrows > 0) {
      const double* g = w.gravity;
      const double gravity = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
      if (!restitution_stage(p, w, bt, gravity)) return false;
      bt.each(0, w.solved, [&](int m) { slipped_row(p, w.row0 + m); });
    }
    __syncthreads();
  }
  return true;
}

}  // namespace bg
