// ORACLE - test infrastructure only.  A line-by-line CPU restatement of Bearing's contact
// solve stage, used by tests/ and by bench.py's CPU-baseline leg as the checker and the timed
// CPU baseline.  The product path (libbearing_gpu.so) never links or calls anything here.
//
// Parity unpinned: the reference is JavaScript and no JS engine exists in this environment, so
// no output of the reference itself can be produced here, and the reference's tests hold no
// stored numeric vectors.  This restatement is checked against the reference's behavioural
// tests and published measurements (tests/test_oracle_behaviour.py), and the CUDA path is
// pinned against it bit for bit (tests/test_gpu_parity.py).
//
// Every function follows the reference's operation order exactly, in IEEE FP64, compiled
// with -ffp-contract=off and no fast-math, so each + - * / sqrt rounds as JavaScript's does.
// Citations are to the reference's files:
//   src/contact.js   inertias 1302-1310, inverseAt 1493-1508, lockedInverse 1520-1549,
//                    prepareRows 1346-1445, core 1199-1219, lever 1565-1581,
//                    turning/along 1728-1737, makeSoft 1591-1597, warmRows 1616-1663,
//                    pushes 1672-1724, solveRows 1805-2090, writeBack 2101-2104,
//                    restitution 2229-2251, closing 2216-2220, push 1743-1749,
//                    slipped 1122-1153, turned 1168-1182, JOBS/LEAST 2113-2146
//   src/world.js     step 962-1032, _accelerate 1495-1530, _move 1533-1563,
//                    tumble 2739-2763, untwist 2777-2805, advance 2820-2828, angular 2831-2834
//   src/core/math.js rotate 211-219, axesOf 222-227, quatMultiply 230-238, atan 138-161,
//                    atan2 173-200
//   src/core/jobs.js run 344-381, claim 425-440 (the thread split of the timed baseline)
//   src/forest.js:67 COMPLIANCE
//
// The stage is written once for any scalar T (StageT): double for the checker and the CPU
// baseline, dual numbers (dual.hpp) for the derivative checker of the adjoint, which also restates
// the host side's per-row work that feeds the stage (src/contact.js emit 889-921, basis 1283-1292,
// carry 999-1036, keep 1091-1115) and differentiates the narrowphase through its templated form.

#include "../include/bearing_gpu.h"
#include "../include/bearing_world.h"
#include "../bearing_b200/host/collide_impl.hpp"
#include "dual.hpp"

#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <functional>
#include <limits>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

namespace {

constexpr int P = 4;
constexpr int J = 12;
constexpr int FJ = 24;
constexpr int COLOURS = 32;
constexpr int OVERFLOW_ = 32;
constexpr int RESTING = 33;
constexpr double COMPLIANCE = 9.5367431640625e-7;   // 2^-20, src/forest.js:67
constexpr double SPIN = 2.0 / 3.0;                  // src/contact.js:146
constexpr double WORLD_SPIN = 3.141592653589793;    // Math.PI, src/world.js:171
constexpr double STIFFNESS = 1.0 / 8.0;             // src/world.js:115
constexpr double DAMPING_RATIO = 10;                // src/world.js:118
constexpr double ROUNDED = 1.0 / 17592186044416.0;  // 2^-44, src/world.js:2812
constexpr double PI = 3.141592653589793;
constexpr double INF = std::numeric_limits<double>::infinity();

// ---- src/core/math.js ----

// The scalar type of a template's other arguments, not deduced from this one (a 0 passed for it
// converts to T).
template <class T>
struct same_as {
  using type = T;
};

// rotate(q, o, x, y, z, inverse, out): math.js:211-219.
template <class T>
inline void rotate(const T* q, typename same_as<T>::type x, typename same_as<T>::type y, typename same_as<T>::type z,
                   bool inverse, T* out) {
  const double s = inverse ? -1 : 1;
  const T ux = q[0] * s, uy = q[1] * s, uz = q[2] * s, w = q[3];
  const T tx = 2 * (uy * z - uz * y), ty = 2 * (uz * x - ux * z), tz = 2 * (ux * y - uy * x);
  out[0] = x + w * tx + (uy * tz - uz * ty);
  out[1] = y + w * ty + (uz * tx - ux * tz);
  out[2] = z + w * tz + (ux * ty - uy * tx);
}

// axesOf: math.js:222-227.
template <class T>
inline void axesOf(const T* q, T* ax) {
  const T x = q[0], y = q[1], z = q[2], w = q[3];
  ax[0] = 1 - 2 * (y * y + z * z); ax[1] = 2 * (x * y + z * w); ax[2] = 2 * (x * z - y * w);
  ax[3] = 2 * (x * y - z * w); ax[4] = 1 - 2 * (x * x + z * z); ax[5] = 2 * (y * z + x * w);
  ax[6] = 2 * (x * z + y * w); ax[7] = 2 * (y * z - x * w); ax[8] = 1 - 2 * (x * x + y * y);
}

// quatMultiply: math.js:230-238.
template <class T>
inline void quatMultiply(const T* a, const T* b, T* out) {
  const T ax = a[0], ay = a[1], az = a[2], aw = a[3];
  const T bx = b[0], by = b[1], bz = b[2], bw = b[3];
  out[0] = aw * bx + ax * bw + ay * bz - az * by;
  out[1] = aw * by + ay * bw + az * bx - ax * bz;
  out[2] = aw * bz + az * bw + ax * by - ay * bx;
  out[3] = aw * bw - ax * bx - ay * by - az * bz;
}

// fdlibm's arctangent as math.js:127-161 states it (its constants are fdlibm's).
const double ATAN_HI[4] = {4.63647609000806093515e-01, 7.85398163397448278999e-01,
                           9.82793723247329054082e-01, 1.57079632679489655800e+00};
const double ATAN_LO[4] = {2.26987774529616870924e-17, 3.06161699786838301793e-17,
                           1.39033110312309984516e-17, 6.12323399573676603587e-17};
constexpr double AT0 = 3.33333333333329318027e-01, AT1 = -1.99999999998764832476e-01,
                 AT2 = 1.42857142725034663711e-01, AT3 = -1.11111104054623557880e-01,
                 AT4 = 9.09088713343650656196e-02, AT5 = -7.69187620504482999495e-02,
                 AT6 = 6.66107313738753120669e-02, AT7 = -5.83357013379057348645e-02,
                 AT8 = 4.97687799461593236017e-02, AT9 = -3.65315727442169155270e-02,
                 AT10 = 1.62858201153657823623e-02;
constexpr double M_PI_ = 3.1415926535897931160e+00, PI_LO = 1.2246467991473531772e-16;
constexpr double PI_O_2 = 1.5707963267948965580e+00, PI_O_4 = 7.8539816339744827900e-01;
constexpr double TWO_66 = 7.378697629483821e+19, TWO_M27 = 7.450580596923828e-09;
constexpr double TWO_60 = 1.152921504606847e+18, TWO_M60 = 8.673617379884035e-19;

double js_atan(double x) {
  if (x != x) return x;
  const double ax = std::fabs(x);
  if (ax >= TWO_66) return x > 0 ? ATAN_HI[3] + ATAN_LO[3] : -ATAN_HI[3] - ATAN_LO[3];
  int id;
  double t;
  if (ax < 0.4375) {
    if (ax < TWO_M27) return x;
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

inline bool negative(double v) { return v < 0 || (v == 0 && std::signbit(v)); }

// atan2: math.js:173-200.
double js_atan2(double y, double x) {
  if (x != x || y != y) return x + y;
  if (x == 1) return js_atan(y);
  int m = (negative(y) ? 1 : 0) | (negative(x) ? 2 : 0);
  if (y == 0) return m < 2 ? y : m == 2 ? M_PI_ : -M_PI_;
  if (x == 0) return y < 0 ? -PI_O_2 : PI_O_2;
  const double ax = std::fabs(x), ay = std::fabs(y);
  if (ax == INF) {
    if (ay == INF) {
      const double r[4] = {PI_O_4, -PI_O_4, 3 * PI_O_4, -3 * PI_O_4};
      return r[m];
    }
    const double r[4] = {0.0, -0.0, M_PI_, -M_PI_};
    return r[m];
  }
  if (ay == INF) return y < 0 ? -PI_O_2 : PI_O_2;
  double z;
  if (ay > ax * TWO_60) {
    z = PI_O_2 + 0.5 * PI_LO;
    m &= 1;
  } else if (x < 0 && ay < ax * TWO_M60) {
    z = 0;
  } else {
    z = js_atan(ay / ax);
  }
  switch (m) {
    case 0: return z;
    case 1: return -z;
    case 2: return M_PI_ - (z - PI_LO);
    default: return (z - PI_LO) - M_PI_;
  }
}

inline double val(double x) { return x; }
using std::fabs;
using std::sqrt;

// Math.max for two numbers: NaN wins, and +0 beats -0.
template <class T>
inline T js_max(const T& a, const T& b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a > b) return a;
  if (b > a) return b;
  if (a == 0 && b == 0) return std::signbit(val(a)) ? b : a;
  return a;
}

// atan2 for any scalar: the value is js_atan2's; a scalar carrying derivatives gets them from
// d atan2(y, x) = (x dy - y dx) / (x^2 + y^2) (0 at the origin), through its own atan2_lift.
inline double atan2T(double y, double x) { return js_atan2(y, x); }
inline dual::D atan2T(const dual::D& y, const dual::D& x) { return dual::atan2_lift(js_atan2(y.v, x.v), y, x); }

// ---- the thread split of src/core/jobs.js (run 344-381, claim 425-440) ----

class Pool {
 public:
  explicit Pool(int workers) : workers_(workers) {
    for (int i = 0; i < workers_; i++) threads_.emplace_back([this] { loop(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      shutdown_ = true;
      epoch_++;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }
  int workers() const { return workers_; }

  // Jobs.run: below `least` items, inline; else cut into (workers+1)*4 chunks claimed by a
  // cursor, every thread the caller included taking chunks until none is left.
  void run(int from, int to, int least, const std::function<void(int, int)>& job) {
    const int n = to - from;
    if (workers_ == 0 || n < least) {
      job(from, to);
      return;
    }
    const int chunks = (workers_ + 1) * 4;
    const int chunk = (n + chunks - 1) / chunks;
    uint64_t epoch;
    {
      std::lock_guard<std::mutex> g(mu_);
      job_ = &job;
      from_ = from;
      count_ = n;
      chunk_ = chunk;
      completed_.store(0);
      epoch = ++epoch_;
      // The cursor carries the dispatch's epoch (src/core/jobs.js:80-83): a worker still holding
      // an earlier dispatch's arguments can never claim a chunk of this one.
      cursor_.store(epoch << 32);
    }
    cv_.notify_all();
    claim();
    while (completed_.load(std::memory_order_acquire) < n) std::this_thread::yield();
    std::lock_guard<std::mutex> g(mu_);
    job_ = nullptr;
  }

 private:
  void claim() {
    const std::function<void(int, int)>* job;
    int from, count, chunk;
    uint64_t epoch;
    {
      std::lock_guard<std::mutex> g(mu_);
      job = job_;
      from = from_;
      count = count_;
      chunk = chunk_;
      epoch = epoch_;
    }
    if (job == nullptr) return;
    for (;;) {
      uint64_t cursor = cursor_.load();
      if ((cursor >> 32) != epoch) return;
      const int index = static_cast<int>(cursor & 0xffffffffu);
      const int start = index * chunk;
      if (start >= count) return;
      if (!cursor_.compare_exchange_weak(cursor, cursor + 1)) continue;
      const int end = start + chunk < count ? start + chunk : count;
      (*job)(from + start, from + end);
      completed_.fetch_add(end - start, std::memory_order_release);
    }
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return epoch_ != seen; });
        seen = epoch_;
        if (shutdown_) return;
      }
      claim();
    }
  }
  int workers_;
  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable cv_;
  uint64_t epoch_ = 0;
  bool shutdown_ = false;
  const std::function<void(int, int)>* job_ = nullptr;
  int from_ = 0, count_ = 0, chunk_ = 1;
  std::atomic<uint64_t> cursor_{0};
  std::atomic<int> completed_{0};
};

// LEAST: src/contact.js:2146 (warm 16, solve 4, prepare 2).
constexpr int LEAST_WARM = 16, LEAST_SOLVE = 4, LEAST_PREPARE = 2;

struct Soft {
  double biasRate = 0, massScale = 1, impulseScale = 0;
};

// makeSoft: contact.js:1591-1597.
Soft makeSoft(double hertz, double zeta, double h) {
  Soft out;
  const double omega = 2 * PI * hertz;
  const double a1 = 2 * zeta + h * omega, a2 = h * omega * a1, a3 = 1 / (1 + a2);
  out.biasRate = omega / a1;
  out.massScale = a2 * a3;
  out.impulseScale = a3;
  return out;
}

// The columns the solve stage reads and writes, with scalar T for every number that depends on the
// state (T for the stage itself, dual numbers for the derivative checker) and T for the
// bodies' and rows' fixed properties (masses, inertias, sizes, dampings, tolerances, patches).
template <class T>
struct BodiesT {
  int32_t capacity, awake_count;
  const int32_t* awake_list;
  const uint8_t* awake;
  T *position, *rotation, *velocity, *angular, *tumbled, *ceiling, *start, *start_q, *inv_i;
  const double *inv_mass, *inertia, *inv_inertia, *dims, *damping, *angular_damping, *gravity_scale;
  const uint8_t *type, *shape, *frozen, *framed, *lock;
  const int32_t* joint_head;
};

template <class T>
struct RowsT {
  int32_t count, solved;
  int32_t starts[BG_STARTS];
  const int32_t *row, *a, *b;
  const uint8_t* points;
  T *normal, *t1, *t2, *friction, *restitution;
  const double *tolerance, *patch;
  T *separation, *point;
  const double* shift;
  T *normal_impulse, *tangent_impulse1, *tangent_impulse2, *roll_impulse1, *roll_impulse2, *spin_impulse;
  T *drift1, *drift2, *gap, *max_normal_impulse, *relative_velocity;
  uint8_t* sliding;
  T *anchor_a, *anchor_b;
};

BodiesT<double> bodies_of(const bg_bodies& B) {
  BodiesT<double> o;
  o.capacity = B.capacity; o.awake_count = B.awake_count; o.awake_list = B.awake_list; o.awake = B.awake;
  o.position = B.position; o.rotation = B.rotation; o.velocity = B.velocity; o.angular = B.angular;
  o.tumbled = B.tumbled; o.ceiling = B.ceiling; o.start = B.start; o.start_q = B.start_q; o.inv_i = B.inv_i;
  o.inv_mass = B.inv_mass; o.inertia = B.inertia; o.inv_inertia = B.inv_inertia; o.dims = B.dims;
  o.damping = B.damping; o.angular_damping = B.angular_damping; o.gravity_scale = B.gravity_scale;
  o.type = B.type; o.shape = B.shape; o.frozen = B.frozen; o.framed = B.framed; o.lock = B.lock;
  o.joint_head = B.joint_head;
  return o;
}

RowsT<double> rows_of(const bg_rows& R) {
  RowsT<double> o;
  o.count = R.count; o.solved = R.solved;
  for (int k = 0; k < BG_STARTS; k++) o.starts[k] = R.starts[k];
  o.row = R.row; o.a = R.a; o.b = R.b; o.points = R.points;
  o.normal = const_cast<double*>(R.normal); o.t1 = const_cast<double*>(R.t1); o.t2 = const_cast<double*>(R.t2);
  o.friction = const_cast<double*>(R.friction); o.restitution = const_cast<double*>(R.restitution);
  o.tolerance = R.tolerance; o.patch = R.patch;
  o.separation = const_cast<double*>(R.separation); o.point = const_cast<double*>(R.point); o.shift = R.shift;
  o.normal_impulse = R.normal_impulse; o.tangent_impulse1 = R.tangent_impulse1; o.tangent_impulse2 = R.tangent_impulse2;
  o.roll_impulse1 = R.roll_impulse1; o.roll_impulse2 = R.roll_impulse2; o.spin_impulse = R.spin_impulse;
  o.drift1 = R.drift1; o.drift2 = R.drift2; o.gap = R.gap; o.max_normal_impulse = R.max_normal_impulse;
  o.relative_velocity = R.relative_velocity; o.sliding = R.sliding; o.anchor_a = R.anchor_a; o.anchor_b = R.anchor_b;
  return o;
}

// The solve stage over one world's views.
template <class T>
class Stage {
 public:
  Stage(const BodiesT<T>& B, const RowsT<T>& C, Pool* pool) : B_(B), C_(C), pool_(pool) {
    const size_t m = static_cast<size_t>(C.count > 0 ? C.count : 1), p = m * P;
    la_.assign(3 * p, 0); lb_.assign(3 * p, 0); ra_.assign(3 * p, 0); rb_.assign(3 * p, 0);
    adjusted_.assign(p, 0); now_.assign(p, 0); normalMass_.assign(p, 0); jac_.assign(J * p, 0);
    block_.assign(P * p, 0); lever_.assign(p, 0);
    fjac_.assign(FJ * m, 0); tangentMass_.assign(3 * m, 0); rollMass1_.assign(m, 0);
    rollMass2_.assign(m, 0); spinMass_.assign(m, 0); anchorA_.assign(3 * m, 0); anchorB_.assign(3 * m, 0);
  }

  void run(const bg_step& step) {
    const int touching = C_.count;
    const int substeps = step.substeps;
    const double h = step.dt / substeps;
    if (touching > 0) inertias();
    // world.js:968-973: where each awake body starts.
    for (int i = 0; i < B_.awake_count; i++) {
      const int s = B_.awake_list[i];
      for (int k = 0; k < 3; k++) B_.start[3 * s + k] = B_.position[3 * s + k];
      for (int k = 0; k < 4; k++) B_.start_q[4 * s + k] = B_.rotation[4 * s + k];
    }
    if (touching > 0) {
      par(0, C_.solved, LEAST_PREPARE, [&](int f, int t) { prepareRows(f, t); });
      soft_ = makeSoft(STIFFNESS / h, DAMPING_RATIO, h);
    }
    for (int sub = 0; sub < substeps; sub++) {
      accelerate(h, step);
      if (touching > 0) warmStart();
      if (touching > 0) solve(h, true, sub > 0);
      move(h);
      if (touching > 0) solve(h, false, false);
    }
    if (touching > 0) {
      const double* g = step.gravity;
      restitution(std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]));
      // store()'s slipped() half, contact.js:1071-1074: each solved row in found order.
      for (int f = 0; f < C_.count; f++) {
        const int m = C_.row[f];
        if (m >= C_.solved) continue;
        slipped(m);
      }
    }
    if (C_.anchor_a != nullptr)
      std::copy(anchorA_.begin(), anchorA_.begin() + 3 * static_cast<size_t>(C_.count), C_.anchor_a);
    if (C_.anchor_b != nullptr)
      std::copy(anchorB_.begin(), anchorB_.begin() + 3 * static_cast<size_t>(C_.count), C_.anchor_b);
  }

 private:
  template <class F>
  void par(int from, int to, int least, F&& f) {
    if (to <= from) return;
    if (pool_ == nullptr) {
      f(from, to);
      return;
    }
    std::function<void(int, int)> job = f;
    pool_->run(from, to, least, job);
  }

  // inertias: contact.js:1302-1310; inverseAt 1493-1508; lockedInverse 1520-1549.
  void inertias() {
    for (int i = 0; i < B_.awake_count; i++) {
      const int s = B_.awake_list[i];
      T* out = B_.inv_i + 6 * s;
      if (B_.frozen[s] != 0) {
        for (int k = 0; k < 6; k++) out[k] = 0;
        continue;
      }
      T ax[9];
      axesOf(B_.rotation + 4 * s, ax);
      inverseAt(s, ax, out);
    }
  }
  void inverseAt(int s, const T* ax, T* out) {
    if (B_.type[s] != BG_DYNAMIC) {
      for (int k = 0; k < 6; k++) out[k] = 0;
      return;
    }
    if (B_.lock[s] != 0) {
      lockedInverse(ax, B_.inertia + 3 * s, B_.lock[s], out);
      return;
    }
    const double* inv = B_.inv_inertia + 3 * s;
    const T i0 = inv[0], i1 = inv[1], i2 = inv[2];
    const T x0 = ax[0], x1 = ax[1], x2 = ax[2];
    const T y0 = ax[3], y1 = ax[4], y2 = ax[5];
    const T z0 = ax[6], z1 = ax[7], z2 = ax[8];
    out[0] = x0 * x0 * i0 + y0 * y0 * i1 + z0 * z0 * i2;
    out[1] = x0 * x1 * i0 + y0 * y1 * i1 + z0 * z1 * i2;
    out[2] = x0 * x2 * i0 + y0 * y2 * i1 + z0 * z2 * i2;
    out[3] = x1 * x1 * i0 + y1 * y1 * i1 + z1 * z1 * i2;
    out[4] = x1 * x2 * i0 + y1 * y2 * i1 + z1 * z2 * i2;
    out[5] = x2 * x2 * i0 + y2 * y2 * i1 + z2 * z2 * i2;
  }
  static void lockedInverse(const T* ax, const double* I, int lock, T* out) {
    static const int SYM[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    const T i0 = I[0], i1 = I[1], i2 = I[2];
    const T x0 = ax[0], x1 = ax[1], x2 = ax[2];
    const T y0 = ax[3], y1 = ax[4], y2 = ax[5];
    const T z0 = ax[6], z1 = ax[7], z2 = ax[8];
    T M6[6];
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
    const T det = M6[ff] * M6[ss] - M6[fs] * M6[fs];
    if (!(det > 0)) return;
    out[ff] = M6[ss] / det; out[ss] = M6[ff] / det; out[fs] = -M6[fs] / det;
  }

  // core(): contact.js:1199-1219 (whole bodies only; parts are not on this path).
  void core(int s, T x, T y, T z, T* out, T* v3) const {
    const int shape = B_.shape[s];
    const T* q = B_.rotation + 4 * s;
    if (shape == BG_SPHERE) {
      out[0] = 0; out[1] = 0; out[2] = 0;
      v3[0] = 0; v3[1] = 0; v3[2] = 0;
      return;
    }
    rotate(q, x, y, z, true, v3);
    if (shape != BG_CAPSULE) {
      out[0] = v3[0]; out[1] = v3[1]; out[2] = v3[2];
      v3[0] = x; v3[1] = y; v3[2] = z;
      return;
    }
    const double* d = B_.dims + 3 * s;
    const T half = (d[1] - 2 * d[0]) * 0.5;
    out[0] = 0; out[1] = v3[1] < -half ? -half : v3[1] > half ? half : v3[1]; out[2] = 0;
    rotate(q, 0, out[1], 0, false, v3);
  }

  // lever(): contact.js:1565-1581.
  T lever(T* jac, int a, int b, double ima, double imb, T rax, T ray, T raz,
               T rbx, T rby, T rbz, T dx, T dy, T dz) const {
    const T* invI = B_.inv_i;
    const T cax = ray * dz - raz * dy, cay = raz * dx - rax * dz, caz = rax * dy - ray * dx;
    const T cbx = rby * dz - rbz * dy, cby = rbz * dx - rbx * dz, cbz = rbx * dy - rby * dx;
    const int oa = a * 6, ob = b * 6;
    const T iax = invI[oa] * cax + invI[oa + 1] * cay + invI[oa + 2] * caz;
    const T iay = invI[oa + 1] * cax + invI[oa + 3] * cay + invI[oa + 4] * caz;
    const T iaz = invI[oa + 2] * cax + invI[oa + 4] * cay + invI[oa + 5] * caz;
    const T ibx = invI[ob] * cbx + invI[ob + 1] * cby + invI[ob + 2] * cbz;
    const T iby = invI[ob + 1] * cbx + invI[ob + 3] * cby + invI[ob + 4] * cbz;
    const T ibz = invI[ob + 2] * cbx + invI[ob + 4] * cby + invI[ob + 5] * cbz;
    jac[0] = cax; jac[1] = cay; jac[2] = caz;
    jac[3] = cbx; jac[4] = cby; jac[5] = cbz;
    jac[6] = iax; jac[7] = iay; jac[8] = iaz;
    jac[9] = ibx; jac[10] = iby; jac[11] = ibz;
    const T k = ima + imb + cax * iax + cay * iay + caz * iaz + cbx * ibx + cby * iby + cbz * ibz;
    return k > 0 ? 1 / k : 0;
  }

  // along / turning: contact.js:1728-1737.
  static T along(const T* invI, T x, T y, T z) {
    return invI[0] * x * x + invI[3] * y * y + invI[5] * z * z
      + 2 * (invI[1] * x * y + invI[2] * x * z + invI[4] * y * z);
  }
  T turning(int a, int b, T x, T y, T z) const {
    const T k = along(B_.inv_i + a * 6, x, y, z) + along(B_.inv_i + b * 6, x, y, z);
    return k > 0 ? 1 / k : 0;
  }

  // prepareRows: contact.js:1346-1445.
  void prepareRows(int from, int to) {
    const T* p = B_.position;
    const T* v = B_.velocity;
    const T* w = B_.angular;
    for (int m = from; m < to; m++) {
      const int a = C_.a[m], b = C_.b[m], a3 = a * 3, b3 = b * 3;
      const double ima = B_.inv_mass[a], imb = B_.inv_mass[b];
      const int m3 = 3 * m;
      const T nx = C_.normal[m3], ny = C_.normal[m3 + 1], nz = C_.normal[m3 + 2];
      const T* T1 = C_.t1 + m3;
      const T* T2 = C_.t2 + m3;
      const int count = C_.points[m];
      if (count <= 2) {
        rollMass1_[m] = turning(a, b, T1[0], T1[1], T1[2]);
        rollMass2_[m] = turning(a, b, T2[0], T2[1], T2[2]);
      }
      spinMass_[m] = turning(a, b, nx, ny, nz);
      const double tol = C_.tolerance[m];
      T weight = 0, ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0;
      T ex = 0, ey = 0, ez = 0, fx = 0, fy = 0, fz = 0;
      for (int k = 0; k < count; k++) {
        const int i = m * P + k, i3 = 3 * i;
        const T px = C_.point[i3], py = C_.point[i3 + 1], pz = C_.point[i3 + 2];
        const T rax = px - p[a3], ray = py - p[a3 + 1], raz = pz - p[a3 + 2];
        const T rbx = px + C_.shift[i3] - p[b3], rby = py + C_.shift[i3 + 1] - p[b3 + 1],
                     rbz = pz + C_.shift[i3 + 2] - p[b3 + 2];
        ra_[i3] = rax; ra_[i3 + 1] = ray; ra_[i3 + 2] = raz;
        rb_[i3] = rbx; rb_[i3 + 1] = rby; rb_[i3 + 2] = rbz;
        T va[3], vb[3];
        core(a, rax, ray, raz, &la_[i3], va);
        core(b, rbx, rby, rbz, &lb_[i3], vb);
        adjusted_[i] = C_.separation[i] - ((vb[0] - va[0]) * nx + (vb[1] - va[1]) * ny + (vb[2] - va[2]) * nz);
        normalMass_[i] = lever(&jac_[J * i], a, b, ima, imb, rax, ray, raz, rbx, rby, rbz, nx, ny, nz);
        C_.max_normal_impulse[i] = 0;
        const T s = C_.separation[i] / tol, near = s <= 1 ? 1 : s >= 2 ? 0 : 2 - s;
        weight += near;
        ax += near * rax; ay += near * ray; az += near * raz; bx += near * rbx; by += near * rby; bz += near * rbz;
        ex += rax; ey += ray; ez += raz; fx += rbx; fy += rby; fz += rbz;
        const T dvx = v[b3] + w[b3 + 1] * rbz - w[b3 + 2] * rby - v[a3] - w[a3 + 1] * raz + w[a3 + 2] * ray;
        const T dvy = v[b3 + 1] + w[b3 + 2] * rbx - w[b3] * rbz - v[a3 + 1] - w[a3 + 2] * rax + w[a3] * raz;
        const T dvz = v[b3 + 2] + w[b3] * rby - w[b3 + 1] * rbx - v[a3 + 2] - w[a3] * ray + w[a3 + 1] * rax;
        C_.relative_velocity[i] = dvx * nx + dvy * ny + dvz * nz;
      }
      const int n = count;
      if (n >= 2) {
        const double s = ima + imb;
        T* K = &block_[m * P * P];
        for (int k = 0; k < n; k++) {
          const T* jk = &jac_[J * (m * P + k)];
          for (int l = 0; l <= k; l++) {
            const T* jl = &jac_[J * (m * P + l)];
            const T e = s + jk[0] * jl[6] + jk[1] * jl[7] + jk[2] * jl[8]
              + jk[3] * jl[9] + jk[4] * jl[10] + jk[5] * jl[11];
            K[P * k + l] = e; K[P * l + k] = e;
          }
        }
      }
      if (weight == 0) { weight = count; ax = ex; ay = ey; az = ez; bx = fx; by = fy; bz = fz; }
      ax /= weight; ay /= weight; az /= weight; bx /= weight; by /= weight; bz /= weight;
      anchorA_[m3] = ax; anchorA_[m3 + 1] = ay; anchorA_[m3 + 2] = az;
      anchorB_[m3] = bx; anchorB_[m3 + 1] = by; anchorB_[m3 + 2] = bz;
      for (int k = 0; k < count; k++) {
        const int i3 = 3 * (m * P + k);
        T dx = ra_[i3] - ax, dy = ra_[i3 + 1] - ay, dz = ra_[i3 + 2] - az;
        const T alongN = dx * nx + dy * ny + dz * nz;
        dx -= alongN * nx; dy -= alongN * ny; dz -= alongN * nz;
        lever_[m * P + k] = sqrt(dx * dx + dy * dy + dz * dz);
      }
      T* jac = &fjac_[FJ * m];
      lever(jac, a, b, ima, imb, ax, ay, az, bx, by, bz, T1[0], T1[1], T1[2]);
      lever(jac + 12, a, b, ima, imb, ax, ay, az, bx, by, bz, T2[0], T2[1], T2[2]);
      const T k11 = ima + imb + jac[0] * jac[6] + jac[1] * jac[7] + jac[2] * jac[8]
        + jac[3] * jac[9] + jac[4] * jac[10] + jac[5] * jac[11];
      const T k22 = ima + imb + jac[12] * jac[18] + jac[13] * jac[19] + jac[14] * jac[20]
        + jac[15] * jac[21] + jac[16] * jac[22] + jac[17] * jac[23];
      const T k12 = jac[12] * jac[6] + jac[13] * jac[7] + jac[14] * jac[8]
        + jac[15] * jac[9] + jac[16] * jac[10] + jac[17] * jac[11];
      const T det = k11 * k22 - k12 * k12;
      if (det > 0) {
        tangentMass_[m3] = k22 / det; tangentMass_[m3 + 1] = -k12 / det; tangentMass_[m3 + 2] = k11 / det;
      } else {
        tangentMass_[m3] = 0; tangentMass_[m3 + 1] = 0; tangentMass_[m3 + 2] = 0;
      }
    }
  }

  // writeBack: contact.js:2101-2104.
  void writeBack(double im, int s3, T vx, T vy, T vz, T wx, T wy, T wz) {
    if (im == 0) return;
    T* v = B_.velocity;
    T* w = B_.angular;
    v[s3] = vx; v[s3 + 1] = vy; v[s3 + 2] = vz; w[s3] = wx; w[s3 + 1] = wy; w[s3 + 2] = wz;
  }

  // warmStart: contact.js:1604-1613; warmRows 1616-1663.
  void warmStart() {
    if (pool_ == nullptr) {
      warmRows(0, C_.solved);
      return;
    }
    for (int k = 0; k < COLOURS; k++)
      if (C_.starts[k + 1] > C_.starts[k])
        par(C_.starts[k], C_.starts[k + 1], LEAST_WARM, [&](int f, int t) { warmRows(f, t); });
    warmRows(C_.starts[OVERFLOW_], C_.starts[OVERFLOW_ + 1]);
  }
  void warmRows(int from, int to) {
    const T* v = B_.velocity;
    const T* w = B_.angular;
    const T* invI = B_.inv_i;
    for (int m = from; m < to; m++) {
      const int a = C_.a[m], b = C_.b[m], a3 = a * 3, b3 = b * 3, m3 = 3 * m;
      const double ima = B_.inv_mass[a], imb = B_.inv_mass[b];
      const T nx = C_.normal[m3], ny = C_.normal[m3 + 1], nz = C_.normal[m3 + 2];
      const T t1x = C_.t1[m3], t1y = C_.t1[m3 + 1], t1z = C_.t1[m3 + 2];
      const T t2x = C_.t2[m3], t2y = C_.t2[m3 + 1], t2z = C_.t2[m3 + 2];
      T vax = v[a3], vay = v[a3 + 1], vaz = v[a3 + 2], wax = w[a3], way = w[a3 + 1], waz = w[a3 + 2];
      T vbx = v[b3], vby = v[b3 + 1], vbz = v[b3 + 2], wbx = w[b3], wby = w[b3 + 1], wbz = w[b3 + 2];
      for (int k = 0; k < C_.points[m]; k++) {
        const int i = m * P + k;
        const T* jac = &jac_[J * i];
        const T ln = C_.normal_impulse[i];
        const T px = nx * ln, py = ny * ln, pz = nz * ln;
        vax -= ima * px; vay -= ima * py; vaz -= ima * pz;
        vbx += imb * px; vby += imb * py; vbz += imb * pz;
        wax -= jac[6] * ln; way -= jac[7] * ln; waz -= jac[8] * ln;
        wbx += jac[9] * ln; wby += jac[10] * ln; wbz += jac[11] * ln;
      }
      {
        const T* fj = &fjac_[FJ * m];
        const T l1 = C_.tangent_impulse1[m], l2 = C_.tangent_impulse2[m];
        const T px = t1x * l1 + t2x * l2, py = t1y * l1 + t2y * l2, pz = t1z * l1 + t2z * l2;
        vax -= ima * px; vay -= ima * py; vaz -= ima * pz;
        vbx += imb * px; vby += imb * py; vbz += imb * pz;
        wax -= fj[6] * l1 + fj[18] * l2; way -= fj[7] * l1 + fj[19] * l2; waz -= fj[8] * l1 + fj[20] * l2;
        wbx += fj[9] * l1 + fj[21] * l2; wby += fj[10] * l1 + fj[22] * l2; wbz += fj[11] * l1 + fj[23] * l2;
      }
      {
        const T r1 = C_.roll_impulse1[m], r2 = C_.roll_impulse2[m], sp = C_.spin_impulse[m];
        const int oa = a * 6, ob = b * 6;
        const T lx = t1x * r1 + t2x * r2 + nx * sp, ly = t1y * r1 + t2y * r2 + ny * sp,
                     lz = t1z * r1 + t2z * r2 + nz * sp;
        wax -= invI[oa] * lx + invI[oa + 1] * ly + invI[oa + 2] * lz;
        way -= invI[oa + 1] * lx + invI[oa + 3] * ly + invI[oa + 4] * lz;
        waz -= invI[oa + 2] * lx + invI[oa + 4] * ly + invI[oa + 5] * lz;
        wbx += invI[ob] * lx + invI[ob + 1] * ly + invI[ob + 2] * lz;
        wby += invI[ob + 1] * lx + invI[ob + 3] * ly + invI[ob + 4] * lz;
        wbz += invI[ob + 2] * lx + invI[ob + 4] * ly + invI[ob + 5] * lz;
      }
      writeBack(ima, a3, vax, vay, vaz, wax, way, waz);
      writeBack(imb, b3, vbx, vby, vbz, wbx, wby, wbz);
    }
  }

  // pushes: contact.js:1672-1724.
  static void pushes(const T* K, int count, int set, const T* give, const T* wanted,
                     T* solved) {
    if (set == 15) {
      const T g0 = 1 + give[0], g1 = 1 + give[1], g2 = 1 + give[2], g3 = 1 + give[3];
      T a00 = K[0] * g0, a01 = K[1], a02 = K[2], a03 = K[3];
      T a10 = K[4], a11 = K[5] * g1, a12 = K[6], a13 = K[7];
      T a20 = K[8], a21 = K[9], a22 = K[10] * g2, a23 = K[11];
      T a30 = K[12], a31 = K[13], a32 = K[14], a33 = K[15] * g3;
      T r0 = wanted[0], r1 = wanted[1], r2 = wanted[2], r3 = wanted[3], f;
      f = a10 / a00; a11 -= f * a01; a12 -= f * a02; a13 -= f * a03; r1 -= f * r0;
      f = a20 / a00; a21 -= f * a01; a22 -= f * a02; a23 -= f * a03; r2 -= f * r0;
      f = a30 / a00; a31 -= f * a01; a32 -= f * a02; a33 -= f * a03; r3 -= f * r0;
      f = a21 / a11; a22 -= f * a12; a23 -= f * a13; r2 -= f * r1;
      f = a31 / a11; a32 -= f * a12; a33 -= f * a13; r3 -= f * r1;
      f = a32 / a22; a33 -= f * a23; r3 -= f * r2;
      const T x3 = r3 / a33;
      const T x2 = (r2 - a23 * x3) / a22;
      const T x1 = (r1 - a12 * x2 - a13 * x3) / a11;
      const T x0 = (r0 - a01 * x1 - a02 * x2 - a03 * x3) / a00;
      solved[0] = x0; solved[1] = x1; solved[2] = x2; solved[3] = x3;
      (void)a20; (void)a30;
      return;
    }
    T AS[P * P], RS[P], XS[P];
    int IN[P];
    int n = 0;
    for (int k = 0; k < count; k++) {
      solved[k] = 0;
      if (set >> k & 1) IN[n++] = k;
    }
    for (int r = 0; r < n; r++) {
      const int kr = IN[r];
      for (int s = 0; s < n; s++) AS[r * P + s] = K[P * kr + IN[s]];
      AS[r * P + r] *= 1 + give[kr];
      RS[r] = wanted[kr];
    }
    for (int col = 0; col < n; col++) {
      const T pivot = AS[col * P + col];
      for (int r = col + 1; r < n; r++) {
        const T f = AS[r * P + col] / pivot;
        for (int s = col + 1; s < n; s++) AS[r * P + s] -= f * AS[col * P + s];
        RS[r] -= f * RS[col];
      }
    }
    for (int r = n - 1; r >= 0; r--) {
      T x = RS[r];
      for (int s = r + 1; s < n; s++) x -= AS[r * P + s] * XS[s];
      XS[r] = x / AS[r * P + r];
      solved[IN[r]] = XS[r];
    }
  }

  // solve: contact.js:1782-1796.
  void solve(double h, bool bias, bool known) {
    if (pool_ == nullptr) {
      solveRows(h, bias, known, 0, C_.solved);
      return;
    }
    for (int k = 0; k < COLOURS; k++)
      if (C_.starts[k + 1] > C_.starts[k])
        par(C_.starts[k], C_.starts[k + 1], LEAST_SOLVE, [&](int f, int t) { solveRows(h, bias, known, f, t); });
    solveRows(h, bias, known, C_.starts[OVERFLOW_], C_.starts[OVERFLOW_ + 1]);
  }

  // solveRows: contact.js:1805-2090.
  void solveRows(double h, bool bias, bool known, int from, int to) {
    T* v = B_.velocity;
    T* w = B_.angular;
    const T* invI = B_.inv_i;
    const T* p = B_.position;
    const T* start = B_.start;
    const T* q = B_.rotation;
    const double inv = 1 / h;
    const Soft soft = soft_;
    const double springy = soft.impulseScale / soft.massScale + COMPLIANCE;
    T target[P], massScale[P], impulseScale[P], give[P], closingNow[P], wanted[P], solved[P];
    for (int m = from; m < to; m++) {
      const int a = C_.a[m], b = C_.b[m], a3 = a * 3, b3 = b * 3, m3 = 3 * m;
      const T nx = C_.normal[m3], ny = C_.normal[m3 + 1], nz = C_.normal[m3 + 2];
      const T dx = (p[b3] - start[b3]) - (p[a3] - start[a3]);
      const T dy = (p[b3 + 1] - start[b3 + 1]) - (p[a3 + 1] - start[a3 + 1]);
      const T dz = (p[b3 + 2] - start[b3 + 2]) - (p[a3 + 2] - start[a3 + 2]);
      const T maxBias = C_.tolerance[m] * inv;
      const int count = C_.points[m];
      T dn = 0, nax = 0, nay = 0, naz = 0, nbx = 0, nby = 0, nbz = 0;
      if (!known) {
        T v3[3];
        dn = dx * nx + dy * ny + dz * nz;
        rotate(q + a * 4, nx, ny, nz, true, v3);
        nax = v3[0]; nay = v3[1]; naz = v3[2];
        rotate(q + b * 4, nx, ny, nz, true, v3);
        nbx = v3[0]; nby = v3[1]; nbz = v3[2];
      }
      T least = INF;
      for (int k = 0; k < count; k++) {
        const int i = m * P + k, i3 = 3 * i;
        T s;
        if (known) {
          s = now_[i];
        } else {
          s = dn + (lb_[i3] * nbx + lb_[i3 + 1] * nby + lb_[i3 + 2] * nbz)
            - (la_[i3] * nax + la_[i3 + 1] * nay + la_[i3 + 2] * naz) + adjusted_[i];
          if (!bias) now_[i] = s;
        }
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
      C_.gap[m] = least;
      const double ima = B_.inv_mass[a], imb = B_.inv_mass[b];
      const T* K = &block_[m * P * P];
      T vax = v[a3], vay = v[a3 + 1], vaz = v[a3 + 2], wax = w[a3], way = w[a3 + 1], waz = w[a3 + 2];
      T vbx = v[b3], vby = v[b3 + 1], vbz = v[b3 + 2], wbx = w[b3], wby = w[b3 + 1], wbz = w[b3 + 2];
      if (count == 1 || !(K[0] > 0)) {
        for (int k = 0; k < count; k++) {
          const int i = m * P + k;
          const T* jac = &jac_[J * i];
          const T vn = (vbx - vax) * nx + (vby - vay) * ny + (vbz - vaz) * nz
            + wbx * jac[3] + wby * jac[4] + wbz * jac[5] - wax * jac[0] - way * jac[1] - waz * jac[2];
          const T old = C_.normal_impulse[i];
          T next = old - normalMass_[i] * massScale[k] * (vn + target[k]) - impulseScale[k] * old;
          if (next < 0) next = 0;
          closingNow[k] = vn; solved[k] = next;
        }
      } else {
        for (int k = 0; k < count; k++) {
          const T* jac = &jac_[J * (m * P + k)];
          closingNow[k] = (vbx - vax) * nx + (vby - vay) * ny + (vbz - vaz) * nz
            + wbx * jac[3] + wby * jac[4] + wbz * jac[5] - wax * jac[0] - way * jac[1] - waz * jac[2];
        }
        int set = 0;
        for (int k = 0; k < count; k++) {
          T r = -closingNow[k] - target[k];
          for (int l = 0; l < count; l++) r += K[P * k + l] * C_.normal_impulse[m * P + l];
          wanted[k] = r;
          if (r > 0) set |= 1 << k;
        }
        for (int round = 0;; round++) {
          pushes(K, count, set, give, wanted, solved);
          int flip = -1;
          for (int k = 0; k < count && flip < 0; k++) {
            if (set >> k & 1) {
              if (solved[k] < 0) flip = k;
            } else {
              T r = -wanted[k];
              for (int l = 0; l < count; l++) r += K[P * k + l] * solved[l];
              if (r < 0) flip = k;
            }
          }
          if (flip < 0 || round == 1 << count) break;
          set ^= 1 << flip;
        }
      }
      for (int k = 0; k < count; k++) {
        const int i = m * P + k;
        const T* jac = &jac_[J * i];
        const T old = C_.normal_impulse[i], next = solved[k] > 0 ? solved[k] : 0;
        const T d = next - old;
        C_.normal_impulse[i] = next;
        if (d > 0 && C_.max_normal_impulse[i] == 0) C_.relative_velocity[i] = closingNow[k];
        if (d > C_.max_normal_impulse[i]) C_.max_normal_impulse[i] = d;
        const T px = nx * d, py = ny * d, pz = nz * d;
        vax -= ima * px; vay -= ima * py; vaz -= ima * pz;
        vbx += imb * px; vby += imb * py; vbz += imb * pz;
        wax -= jac[6] * d; way -= jac[7] * d; waz -= jac[8] * d;
        wbx += jac[9] * d; wby += jac[10] * d; wbz += jac[11] * d;
      }
      const T mu = C_.friction[m];
      const int oa = a * 6, ob = b * 6;
      const T t1x = C_.t1[m3], t1y = C_.t1[m3 + 1], t1z = C_.t1[m3 + 2];
      const T t2x = C_.t2[m3], t2y = C_.t2[m3 + 1], t2z = C_.t2[m3 + 2];
      T pressed = 0, twisted = 0;
      for (int k = 0; k < count; k++) {
        const int i = m * P + k;
        pressed += C_.normal_impulse[i];
        twisted += lever_[i] * C_.normal_impulse[i];
      }
      {
        const T* fj = &fjac_[FJ * m];
        const T* g = fj + 12;
        const T dvx = vbx - vax, dvy = vby - vay, dvz = vbz - vaz;
        T v1 = dvx * t1x + dvy * t1y + dvz * t1z
          + wbx * fj[3] + wby * fj[4] + wbz * fj[5] - wax * fj[0] - way * fj[1] - waz * fj[2];
        T v2 = dvx * t2x + dvy * t2y + dvz * t2z
          + wbx * g[3] + wby * g[4] + wbz * g[5] - wax * g[0] - way * g[1] - waz * g[2];
        const T s1 = C_.drift1[m], s2 = C_.drift2[m];
        if (bias && (s1 != 0 || s2 != 0)) {
          T b1 = soft.biasRate * s1, b2 = soft.biasRate * s2;
          const T bb = b1 * b1 + b2 * b2;
          if (bb > maxBias * maxBias) {
            const T scale = maxBias / sqrt(bb);
            b1 *= scale; b2 *= scale;
          }
          v1 += b1; v2 += b2;
        }
        const T* tm = &tangentMass_[m3];
        const T o1 = C_.tangent_impulse1[m], o2 = C_.tangent_impulse2[m];
        T n1 = o1 - (tm[0] * v1 + tm[1] * v2), n2 = o2 - (tm[1] * v1 + tm[2] * v2);
        const T limit = mu * pressed, l2 = n1 * n1 + n2 * n2;
        if (l2 > limit * limit) {
          const T ma = tm[0], mb = tm[1], mc = tm[2];
          T al = 0, x = n1, y = n2, ll = l2;
          while (limit > 0) {
            const T ab = al * mb, d = (1 + al * ma) * (1 + al * mc) - ab * ab;
            const T px = ma * x + mb * y, py = mb * x + mc * y;
            const T wx = ((1 + al * mc) * px - ab * py) / d, wy = ((1 + al * ma) * py - ab * px) / d;
            const T lw = x * wx + y * wy;
            if (!(lw > 0)) break;
            const T next = al + (sqrt(ll) / limit - 1) * ll / lw;
            if (!(next > al)) break;
            al = next;
            const T ab2 = al * mb, d2 = (1 + al * ma) * (1 + al * mc) - ab2 * ab2;
            x = ((1 + al * mc) * n1 - ab2 * n2) / d2; y = ((1 + al * ma) * n2 - ab2 * n1) / d2;
            ll = x * x + y * y;
            if (!(ll > limit * limit)) break;
          }
          const T scale = limit / sqrt(ll);
          n1 = x * scale; n2 = y * scale;
          C_.sliding[m] = 1;
        } else {
          C_.sliding[m] = 0;
        }
        C_.tangent_impulse1[m] = n1; C_.tangent_impulse2[m] = n2;
        const T d1 = n1 - o1, d2 = n2 - o2;
        const T px = t1x * d1 + t2x * d2, py = t1y * d1 + t2y * d2, pz = t1z * d1 + t2z * d2;
        vax -= ima * px; vay -= ima * py; vaz -= ima * pz;
        vbx += imb * px; vby += imb * py; vbz += imb * pz;
        wax -= fj[6] * d1 + g[6] * d2; way -= fj[7] * d1 + g[7] * d2; waz -= fj[8] * d1 + g[8] * d2;
        wbx += fj[9] * d1 + g[9] * d2; wby += fj[10] * d1 + g[10] * d2; wbz += fj[11] * d1 + g[11] * d2;
      }
      if (count <= 2) {
        const T most = C_.patch[m] * pressed;
        const T ux = wbx - wax, uy = wby - way, uz = wbz - waz;
        const T r1 = C_.roll_impulse1[m], r2 = C_.roll_impulse2[m];
        T n1 = r1 - rollMass1_[m] * (ux * t1x + uy * t1y + uz * t1z);
        T n2 = r2 - rollMass2_[m] * (ux * t2x + uy * t2y + uz * t2z);
        const T l2 = n1 * n1 + n2 * n2;
        if (l2 > most * most) {
          const T scale = most / sqrt(l2);
          n1 *= scale; n2 *= scale;
        }
        C_.roll_impulse1[m] = n1; C_.roll_impulse2[m] = n2;
        const T d1 = n1 - r1, d2 = n2 - r2;
        const T lx = t1x * d1 + t2x * d2, ly = t1y * d1 + t2y * d2, lz = t1z * d1 + t2z * d2;
        wax -= invI[oa] * lx + invI[oa + 1] * ly + invI[oa + 2] * lz;
        way -= invI[oa + 1] * lx + invI[oa + 3] * ly + invI[oa + 4] * lz;
        waz -= invI[oa + 2] * lx + invI[oa + 4] * ly + invI[oa + 5] * lz;
        wbx += invI[ob] * lx + invI[ob + 1] * ly + invI[ob + 2] * lz;
        wby += invI[ob + 1] * lx + invI[ob + 3] * ly + invI[ob + 4] * lz;
        wbz += invI[ob + 2] * lx + invI[ob + 4] * ly + invI[ob + 5] * lz;
      }
      {
        const T limit = count == 1 ? SPIN * mu * C_.patch[m] * pressed : mu * twisted;
        const T s0 = C_.spin_impulse[m];
        T s1 = s0 - spinMass_[m] * ((wbx - wax) * nx + (wby - way) * ny + (wbz - waz) * nz);
        if (s1 > limit) s1 = limit; else if (s1 < -limit) s1 = -limit;
        C_.spin_impulse[m] = s1;
        const T ds = s1 - s0, lx = nx * ds, ly = ny * ds, lz = nz * ds;
        wax -= invI[oa] * lx + invI[oa + 1] * ly + invI[oa + 2] * lz;
        way -= invI[oa + 1] * lx + invI[oa + 3] * ly + invI[oa + 4] * lz;
        waz -= invI[oa + 2] * lx + invI[oa + 4] * ly + invI[oa + 5] * lz;
        wbx += invI[ob] * lx + invI[ob + 1] * ly + invI[ob + 2] * lz;
        wby += invI[ob + 1] * lx + invI[ob + 3] * ly + invI[ob + 4] * lz;
        wbz += invI[ob + 2] * lx + invI[ob + 4] * ly + invI[ob + 5] * lz;
      }
      writeBack(ima, a3, vax, vay, vaz, wax, way, waz);
      writeBack(imb, b3, vbx, vby, vbz, wbx, wby, wbz);
    }
  }

  // _accelerate: world.js:1495-1530.
  void accelerate(double h, const bg_step& step) {
    T* v = B_.velocity;
    T* w = B_.angular;
    const double gx = step.gravity[0] * h, gy = step.gravity[1] * h, gz = step.gravity[2] * h;
    const double most = WORLD_SPIN / (h * step.substeps);
    for (int i = 0; i < B_.awake_count; i++) {
      const int s = B_.awake_list[i];
      if (B_.type[s] != BG_DYNAMIC || B_.frozen[s] != 0) continue;
      const int s3 = s * 3;
      const double g = B_.gravity_scale[s];
      v[s3] += gx * g; v[s3 + 1] += gy * g; v[s3 + 2] += gz * g;
      if (B_.damping[s] != 0) {
        const T k = 1 / (1 + h * B_.damping[s]);
        v[s3] *= k; v[s3 + 1] *= k; v[s3 + 2] *= k;
      }
      if (B_.angular_damping[s] != 0) {
        const T k = 1 / (1 + h * B_.angular_damping[s]);
        w[s3] *= k; w[s3 + 1] *= k; w[s3 + 2] *= k;
      }
      if (B_.shape[s] != BG_SPHERE || B_.framed[s] == 1) {
        const T w2 = w[s3] * w[s3] + w[s3 + 1] * w[s3 + 1] + w[s3 + 2] * w[s3 + 2];
        if (w2 > most * most) {
          const T k = most / sqrt(w2);
          w[s3] *= k; w[s3 + 1] *= k; w[s3 + 2] *= k;
        }
      }
    }
  }

  // advance: world.js:2820-2828.
  static void advance(const T* q, T wx, T wy, T wz, double h, T* out) {
    const T x = q[0], y = q[1], z = q[2], w = q[3];
    const T nx = x + h * (wx * w + wy * z - wz * y);
    const T ny = y + h * (wy * w + wz * x - wx * z);
    const T nz = z + h * (wz * w + wx * y - wy * x);
    const T nw = w - h * (wx * x + wy * y + wz * z);
    const T l = 1 / sqrt(nx * nx + ny * ny + nz * nz + nw * nw);
    out[0] = nx * l; out[1] = ny * l; out[2] = nz * l; out[3] = nw * l;
  }

  // angular: world.js:2831-2834.
  static void angular(const T* q, const double* inv, T lx, T ly, T lz, T* v3) {
    rotate(q, lx, ly, lz, true, v3);
    rotate(q, v3[0] * inv[0], v3[1] * inv[1], v3[2] * inv[2], false, v3);
  }

  // untwist: world.js:2777-2805.
  static void untwist(T* q, const double* inv, T lx, T ly, T lz, T most) {
    T B[3];
    rotate(q, lx, ly, lz, true, B);
    const T bx = B[0], by = B[1], bz = B[2], ll = bx * bx + by * by + bz * bz;
    T x = bx, y = by, z = bz;
    for (int round = 0; round < 2; round++) {
      const T gx = x * inv[0], gy = y * inv[1], gz = z * inv[2];
      const T over = x * gx + y * gy + z * gz - most;
      if (!(over > 0)) break;
      const T k = (gx * x + gy * y + gz * z) / ll, tx = gx - k * x, ty = gy - k * y, tz = gz - k * z;
      const T tt = tx * tx + ty * ty + tz * tz;
      if (!(tt > 0)) break;
      const T a = 0.5 * over / tt;
      x -= a * tx; y -= a * ty; z -= a * tz;
      const T back = sqrt(ll / (x * x + y * y + z * z));
      x *= back; y *= back; z *= back;
    }
    const T cx = y * bz - z * by, cy = z * bx - x * bz, cz = x * by - y * bx;
    const T cw = ll + x * bx + y * by + z * bz;
    const T l = sqrt(cx * cx + cy * cy + cz * cz + cw * cw);
    if (!(l > 0)) return;
    const T T4[4] = {cx / l, cy / l, cz / l, cw / l};
    T Q4[4];
    quatMultiply(q, T4, Q4);
    const T n = 1 / sqrt(Q4[0] * Q4[0] + Q4[1] * Q4[1] + Q4[2] * Q4[2] + Q4[3] * Q4[3]);
    q[0] = Q4[0] * n; q[1] = Q4[1] * n; q[2] = Q4[2] * n; q[3] = Q4[3] * n;
  }

  // tumble: world.js:2739-2763.
  void tumble(int s, double dt) {
    T* q = B_.rotation + 4 * s;
    const double* I = B_.inertia + 3 * s;
    const double* inv = B_.inv_inertia + 3 * s;
    T* w = B_.angular + 3 * s;
    T* left = B_.tumbled + 3 * s;
    T v3[3], q4[4];
    rotate(q, w[0], w[1], w[2], true, v3);
    rotate(q, v3[0] * I[0], v3[1] * I[1], v3[2] * I[2], false, v3);
    const T lx = v3[0], ly = v3[1], lz = v3[2];
    if (w[0] != left[0] || w[1] != left[1] || w[2] != left[2]) {
      B_.ceiling[s] = w[0] * lx + w[1] * ly + w[2] * lz;
    }
    const T most = B_.ceiling[s];
    advance(q, w[0], w[1], w[2], dt * 0.25, q4);
    angular(q4, inv, lx, ly, lz, v3);
    advance(q, v3[0], v3[1], v3[2], dt * 0.5, q);
    angular(q, inv, lx, ly, lz, v3);
    if (v3[0] * lx + v3[1] * ly + v3[2] * lz > most * (1 + ROUNDED)) {
      untwist(q, inv, lx, ly, lz, most);
      angular(q, inv, lx, ly, lz, v3);
    }
    w[0] = v3[0]; w[1] = v3[1]; w[2] = v3[2];
    left[0] = v3[0]; left[1] = v3[1]; left[2] = v3[2];
  }

  // _move: world.js:1533-1563.
  void move(double h) {
    T* p = B_.position;
    T* q = B_.rotation;
    const T* v = B_.velocity;
    const T* w = B_.angular;
    const double* I = B_.inertia;
    const double half = h * 0.5;
    for (int i = 0; i < B_.awake_count; i++) {
      const int s = B_.awake_list[i], s3 = s * 3, s4 = s * 4;
      if (B_.frozen[s] != 0) continue;
      p[s3] += v[s3] * h; p[s3 + 1] += v[s3 + 1] * h; p[s3 + 2] += v[s3 + 2] * h;
      const T wx = w[s3], wy = w[s3 + 1], wz = w[s3 + 2];
      const bool turningNow = wx != 0 || wy != 0 || wz != 0;
      if (turningNow && B_.type[s] == BG_DYNAMIC && B_.lock[s] == 0 && B_.joint_head[s] == 0
          && (I[s3] != I[s3 + 1] || I[s3 + 1] != I[s3 + 2])) {
        tumble(s, h);
      } else if (turningNow) {
        advance(q + s4, wx, wy, wz, half, q + s4);
      }
    }
  }

  // restitution: contact.js:2229-2251 (closing 2216-2220, push 1743-1749).
  void restitution(double gravity) {
    T* v = B_.velocity;
    T* w = B_.angular;
    for (int f = 0; f < C_.count; f++) {
      const int m = C_.row[f];
      const T e = C_.restitution[m];
      if (e == 0 || m >= C_.solved) continue;
      const double threshold = std::sqrt(2 * gravity * C_.tolerance[m]);
      const int a = C_.a[m], b = C_.b[m], a3 = a * 3, b3 = b * 3, m3 = 3 * m;
      const T nx = C_.normal[m3], ny = C_.normal[m3 + 1], nz = C_.normal[m3 + 2];
      const double ima = B_.inv_mass[a], imb = B_.inv_mass[b];
      for (int k = 0; k < C_.points[m]; k++) {
        const int i = m * P + k;
        if (C_.relative_velocity[i] > -threshold || C_.max_normal_impulse[i] == 0) continue;
        const T* jac = &jac_[J * i];
        const T vn = (v[b3] - v[a3]) * nx + (v[b3 + 1] - v[a3 + 1]) * ny + (v[b3 + 2] - v[a3 + 2]) * nz
          + w[b3] * jac[3] + w[b3 + 1] * jac[4] + w[b3 + 2] * jac[5]
          - w[a3] * jac[0] - w[a3 + 1] * jac[1] - w[a3 + 2] * jac[2];
        const T old = C_.normal_impulse[i];
        T next = old - normalMass_[i] * (vn + e * C_.relative_velocity[i]);
        if (next < 0) next = 0;
        const T d = next - old;
        C_.normal_impulse[i] = next;
        const T px = nx * d, py = ny * d, pz = nz * d;
        v[a3] -= ima * px; v[a3 + 1] -= ima * py; v[a3 + 2] -= ima * pz;
        v[b3] += imb * px; v[b3 + 1] += imb * py; v[b3 + 2] += imb * pz;
        w[a3] -= jac[6] * d; w[a3 + 1] -= jac[7] * d; w[a3 + 2] -= jac[8] * d;
        w[b3] += jac[9] * d; w[b3 + 1] += jac[10] * d; w[b3 + 2] += jac[11] * d;
      }
    }
  }

  // turned: contact.js:1168-1182.
  void turned(int s, T* out) const {
    const int s3 = s * 3, s4 = s * 4;
    const T* q = B_.rotation + s4;
    const T* q0 = B_.start_q + s4;
    const T ax = q[0], ay = q[1], az = q[2], aw = q[3];
    const T bx = -q0[0], by = -q0[1], bz = -q0[2], bw = q0[3];
    T ux = aw * bx + ax * bw + ay * bz - az * by;
    T uy = aw * by + ay * bw + az * bx - ax * bz;
    T uz = aw * bz + az * bw + ax * by - ay * bx;
    T uw = aw * bw - ax * bx - ay * by - az * bz;
    if (uw < 0) { ux = -ux; uy = -uy; uz = -uz; uw = -uw; }
    const T sine = sqrt(ux * ux + uy * uy + uz * uz);
    const T k = sine == 0 ? 0 : 2 * atan2T(sine, uw) / sine;
    out[0] = B_.position[s3] - B_.start[s3];
    out[1] = B_.position[s3 + 1] - B_.start[s3 + 1];
    out[2] = B_.position[s3 + 2] - B_.start[s3 + 2];
    out[3] = ux * k; out[4] = uy * k; out[5] = uz * k;
  }

  // slipped: contact.js:1122-1153.
  void slipped(int m) {
    const int a = C_.a[m], b = C_.b[m], m3 = 3 * m;
    T pressed = 0;
    bool impact = false;
    for (int k = 0; k < C_.points[m]; k++) {
      const int i = m * P + k, i3 = 3 * i;
      pressed += C_.normal_impulse[i];
      if (C_.shift[i3] != 0 || C_.shift[i3 + 1] != 0 || C_.shift[i3 + 2] != 0) impact = true;
    }
    if (C_.sliding[m] != 0 || pressed == 0 || impact) {
      C_.drift1[m] = 0; C_.drift2[m] = 0;
      return;
    }
    T turn[12];
    T dx = 0, dy = 0, dz = 0;
    if (B_.awake[b] != 0) {
      turned(b, turn);
      const T rx = anchorB_[m3], ry = anchorB_[m3 + 1], rz = anchorB_[m3 + 2];
      dx = turn[0] + turn[4] * rz - turn[5] * ry;
      dy = turn[1] + turn[5] * rx - turn[3] * rz;
      dz = turn[2] + turn[3] * ry - turn[4] * rx;
    }
    if (B_.awake[a] != 0) {
      turned(a, turn + 6);
      const T rx = anchorA_[m3], ry = anchorA_[m3 + 1], rz = anchorA_[m3 + 2];
      dx -= turn[6] + turn[10] * rz - turn[11] * ry;
      dy -= turn[7] + turn[11] * rx - turn[9] * rz;
      dz -= turn[8] + turn[9] * ry - turn[10] * rx;
    }
    C_.drift1[m] += dx * C_.t1[m3] + dy * C_.t1[m3 + 1] + dz * C_.t1[m3 + 2];
    C_.drift2[m] += dx * C_.t2[m3] + dy * C_.t2[m3 + 1] + dz * C_.t2[m3 + 2];
  }

  const BodiesT<T>& B_;
  const RowsT<T>& C_;
  Pool* pool_;
  Soft soft_;
  std::vector<T> la_, lb_, ra_, rb_, adjusted_, now_, normalMass_, jac_, block_, lever_;
  std::vector<T> fjac_, tangentMass_, rollMass1_, rollMass2_, spinMass_, anchorA_, anchorB_;
};

Pool* g_pool = nullptr;
int g_pool_workers = -1;

}  // namespace

extern "C" {

// The reference's CPU solve stage over one world, with `workers` worker threads beside the
// calling one (0: single-threaded, as a World with workers 0).  Returns 0.
int32_t oracle_solve_step(const bg_bodies* bodies, const bg_rows* rows, const bg_step* step, int32_t workers) {
  Pool* pool = nullptr;
  if (workers > 0) {
    if (g_pool_workers != workers) {
      delete g_pool;
      g_pool = new Pool(workers);
      g_pool_workers = workers;
    }
    pool = g_pool;
  }
  const BodiesT<double> B = bodies_of(*bodies);
  const RowsT<double> R = rows_of(*rows);
  Stage<double> stage(B, R, pool);
  stage.run(*step);
  return 0;
}

// The same with bw_solver's signature (bearing_world.h): `user` is the worker count.
int32_t oracle_solver(void* user, const bg_bodies* bodies, const bg_rows* rows, const bg_step* step) {
  return oracle_solve_step(bodies, rows, step, static_cast<int32_t>(reinterpret_cast<intptr_t>(user)));
}

// fdlibm atan2 as the reference states it (src/core/math.js:173-200), for tests.
double oracle_atan2(double y, double x) { return js_atan2(y, x); }

void oracle_release_threads(void) {
  delete g_pool;
  g_pool = nullptr;
  g_pool_workers = -1;
}

}  // extern "C"

// ---- the derivative checker: one world's steps in dual numbers ----
//
// The host side of each step (bounds, pairs, colours, the pairs' memory) runs in double in the
// product's host library, which decides what is discrete: which pairs meet, the rows' order and
// colours, which remembered points carry.  For each row this restates in dual numbers what depends
// on the bodies' state and on the materials: the narrowphase (collideT), emit's mixing of friction
// and restitution, basis and carry; then the whole solve stage (StageT), then keep into a dual
// copy of each pair's memory.  The step's real parts go back into the host's columns, so the host
// world goes on exactly as if the double stage had run.

namespace {

using dual::D;

struct DualMemory {
  int points = 0;
  uint32_t pid[P] = {0, 0, 0, 0};
  D ni[P];
  D friction[3], twist[3], slip[3];
};

struct DualWorld {
  int n = 0;
  std::vector<D> position, rotation, velocity, angular, tumbled, ceiling, start, start_q, inv_i, friction, restitution;
  std::map<uint64_t, DualMemory> memory;
};

uint64_t pair_key(int a, int b) { return (static_cast<uint64_t>(static_cast<uint32_t>(a)) << 32) | static_cast<uint32_t>(b); }

// Math.max (as emit() mixes restitution), for dual numbers.
D mix_max(const D& a, const D& b) { return js_max(a, b); }

// basis: src/contact.js:1283-1292.
void basis_dual(const D* n, D* t1, D* t2) {
  const D nx = n[0], ny = n[1], nz = n[2];
  const D ax = fabs(nx), ay = fabs(ny), az = fabs(nz);
  D tx, ty, tz;
  if (ax <= ay && ax <= az) { tx = 0; ty = nz; tz = -ny; } else if (ay <= az) { tx = -nz; ty = 0; tz = nx; } else { tx = ny; ty = -nx; tz = 0; }
  const D l = 1 / sqrt(tx * tx + ty * ty + tz * tz);
  tx *= l; ty *= l; tz *= l;
  t1[0] = tx; t1[1] = ty; t1[2] = tz;
  t2[0] = ny * tz - nz * ty; t2[1] = nz * tx - nx * tz; t2[2] = nx * ty - ny * tx;
}

}  // namespace

extern "C" {

// A dual copy of a world's bodies as `B` holds them (zero derivatives), and of each body's
// friction and restitution (World._friction / _restitution, which emit() mixes).
void* oracle_dual_create(const bg_bodies* B, const double* friction, const double* restitution) {
  DualWorld* w = new DualWorld();
  const int n = B->capacity;
  w->n = n;
  auto take = [](std::vector<D>& dst, const double* src, size_t k) {
    dst.assign(k, D());
    for (size_t i = 0; i < k; i++) dst[i] = D(src[i]);
  };
  const size_t s = static_cast<size_t>(n);
  take(w->position, B->position, 3 * s); take(w->rotation, B->rotation, 4 * s);
  take(w->velocity, B->velocity, 3 * s); take(w->angular, B->angular, 3 * s);
  take(w->tumbled, B->tumbled, 3 * s); take(w->ceiling, B->ceiling, s);
  take(w->start, B->start, 3 * s); take(w->start_q, B->start_q, 4 * s); take(w->inv_i, B->inv_i, 6 * s);
  take(w->friction, friction, s); take(w->restitution, restitution, s);
  return w;
}

void oracle_dual_destroy(void* h) { delete static_cast<DualWorld*>(h); }

int32_t oracle_dual_tangents(void) { return dual::K; }

// Direction `tangent` (0..K-1) is: what = 0, body slot's velocity component; what = 1, every
// body's friction; what = 2, every body's restitution.
int32_t oracle_dual_seed(void* h, int32_t what, int32_t slot, int32_t component, int32_t tangent) {
  DualWorld* w = static_cast<DualWorld*>(h);
  if (tangent < 0 || tangent >= dual::K) return BG_EINVAL;
  if (what == 0) {
    if (slot < 0 || slot >= w->n || component < 0 || component > 2) return BG_EINVAL;
    w->velocity[3 * static_cast<size_t>(slot) + static_cast<size_t>(component)].d[tangent] = 1;
  } else if (what == 1) {
    for (D& f : w->friction) f.d[tangent] = 1;
  } else if (what == 2) {
    for (D& e : w->restitution) e.d[tangent] = 1;
  } else {
    return BG_EINVAL;
  }
  return BG_OK;
}

// One step in dual numbers, after the host's bw_begin_step: B and R are the host's views of the
// solve stage's input, `mem` its bw_row_memory.  Writes the step's real parts into the stage's
// output columns of B and R.  Returns 0, or -1 where the dual recomputation of a row's manifold
// does not reproduce the host's (a different count, id or value: the two would not be the same
// program), -2 where carried memory is missing.
int32_t oracle_dual_step(void* h, const bg_bodies* B, const bg_rows* R, const bg_step* S, const bw_row_memory* mem) {
  DualWorld* w = static_cast<DualWorld*>(h);
  const int n = w->n, count = R->count;
  if (B->capacity != n) return BG_EINVAL;
  const size_t c = static_cast<size_t>(count > 0 ? count : 1);
  // Every column starts as the host's (entries past a row's point count keep whatever bits they
  // hold there); what depends on the state is then recomputed below.
  auto from = [count](const double* src, size_t per) {
    std::vector<D> out(per * static_cast<size_t>(count > 0 ? count : 1));
    for (size_t i = 0; i < per * static_cast<size_t>(count); i++) out[i] = D(src[i]);
    return out;
  };
  std::vector<D> normal = from(R->normal, 3), t1 = from(R->t1, 3), t2 = from(R->t2, 3), friction = from(R->friction, 1),
                 restitution = from(R->restitution, 1), separation = from(R->separation, P), point = from(R->point, 3 * P);
  std::vector<D> ni = from(R->normal_impulse, P), ti1 = from(R->tangent_impulse1, 1), ti2 = from(R->tangent_impulse2, 1),
                 ri1 = from(R->roll_impulse1, 1), ri2 = from(R->roll_impulse2, 1), si = from(R->spin_impulse, 1),
                 drift1 = from(R->drift1, 1), drift2 = from(R->drift2, 1), gap = from(R->gap, 1),
                 maxni = from(R->max_normal_impulse, P), relvel = from(R->relative_velocity, P),
                 anchor_a = from(R->anchor_a, 3), anchor_b = from(R->anchor_b, 3);
  std::vector<double> shift(R->shift, R->shift + 3 * P * static_cast<size_t>(count));
  shift.resize(3 * P * c, 0.0);
  std::vector<uint8_t> sliding(R->sliding, R->sliding + count);
  sliding.resize(c, 0);
  // 1. each row's manifold, materials and carried memory
  for (int m = 0; m < count; m++) {
    const int a = R->a[m], b = R->b[m];
    bearing::ShapeT<D> sh[2];
    for (int e = 0; e < 2; e++) {
      const int s = e == 0 ? a : b;
      const double* d = B->dims + 3 * s;
      bearing::ShapeT<D>& x = sh[e];
      if (B->shape[s] == BG_BOX) {
        x.kind = bearing::K_BOX;
        x.half[0] = d[0] * 0.5; x.half[1] = d[1] * 0.5; x.half[2] = d[2] * 0.5;
      } else if (B->shape[s] == BG_SPHERE) {
        x.kind = bearing::K_SPHERE;
        x.half[0] = d[0];
      } else {
        x.kind = bearing::K_CAPSULE;
        x.half[0] = d[0];
        x.half[1] = (d[1] - 2 * d[0]) * 0.5;
      }
      for (int k = 0; k < 3; k++) x.center[k] = w->position[3 * s + k];
      const double scale = B->type[s] == BG_DYNAMIC ? B->gravity_scale[s] : 0;
      for (int k = 0; k < 3; k++) x.weight[k] = S->gravity[k] * scale;
      axesOf(&w->rotation[4 * static_cast<size_t>(s)], x.axes);
    }
    bearing::ManifoldT<D> mf;
    bearing::collideT<D>(sh[0], sh[1], mem->margin[m], R->tolerance[m], mf);
    if (mf.count != R->points[m]) return -1;
    for (int k = 0; k < mf.count; k++) {
      if (mf.ids[k] != mem->pid[P * m + k] || mf.separations[k].v != R->separation[P * m + k]) return -1;
      for (int q = 0; q < 3; q++)
        if (mf.points[3 * k + q].v != R->point[12 * m + 3 * k + q]) return -1;
    }
    for (int q = 0; q < 3; q++) {
      if (mf.normal[q].v != R->normal[3 * m + q]) return -1;
      normal[3 * m + q] = mf.normal[q];
    }
    // emit: src/contact.js:901-921
    friction[m] = sqrt(w->friction[a] * w->friction[b]);
    restitution[m] = mix_max(w->restitution[a], w->restitution[b]);
    ri1[m] = 0; ri2[m] = 0; si[m] = 0; ti1[m] = 0; ti2[m] = 0; drift1[m] = 0; drift2[m] = 0;
    for (int k = 0; k < mf.count; k++) {
      separation[P * m + k] = mf.separations[k];
      for (int q = 0; q < 3; q++) point[12 * m + 3 * k + q] = mf.points[3 * k + q];
      ni[P * m + k] = 0;
    }
    basis_dual(&normal[3 * m], &t1[3 * m], &t2[3 * m]);
    // carry: src/contact.js:999-1036
    const int remembered = mem->remembered[m];
    if (remembered == 0) continue;
    auto it = w->memory.find(pair_key(a, b));
    if (it == w->memory.end() || it->second.points != remembered) return -2;
    const DualMemory& from = it->second;
    for (int j = 0; j < remembered; j++)
      if (from.pid[j] != mem->memory_pid[P * m + j]) return -2;
    const D* T1 = &t1[3 * m];
    const D* T2 = &t2[3 * m];
    const D* N = &normal[3 * m];
    const int pts = R->points[m];
    if (pts <= 2) {
      ri1[m] = from.twist[0] * T1[0] + from.twist[1] * T1[1] + from.twist[2] * T1[2];
      ri2[m] = from.twist[0] * T2[0] + from.twist[1] * T2[1] + from.twist[2] * T2[2];
    }
    si[m] = from.twist[0] * N[0] + from.twist[1] * N[1] + from.twist[2] * N[2];
    ti1[m] = from.friction[0] * T1[0] + from.friction[1] * T1[1] + from.friction[2] * T1[2];
    ti2[m] = from.friction[0] * T2[0] + from.friction[1] * T2[1] + from.friction[2] * T2[2];
    bool same = false;
    for (int k = 0; k < pts; k++) {
      const uint32_t id = mem->pid[P * m + k];
      for (int j = 0; j < remembered; j++) {
        if (from.pid[j] != id) continue;
        ni[P * m + k] = from.ni[j];
        same = true;
        break;
      }
    }
    if (same) {
      drift1[m] = from.slip[0] * T1[0] + from.slip[1] * T1[1] + from.slip[2] * T1[2];
      drift2[m] = from.slip[0] * T2[0] + from.slip[1] * T2[1] + from.slip[2] * T2[2];
    }
  }
  // The host's rows must carry the same (real) values: it ran the same code in double.
  for (int m = 0; m < count; m++) {
    for (int k = 0; k < R->points[m]; k++)
      if (ni[P * m + k].v != R->normal_impulse[P * m + k]) return -1;
    if (ti1[m].v != R->tangent_impulse1[m] || ti2[m].v != R->tangent_impulse2[m] || si[m].v != R->spin_impulse[m] ||
        drift1[m].v != R->drift1[m] || drift2[m].v != R->drift2[m] || friction[m].v != R->friction[m] ||
        restitution[m].v != R->restitution[m])
      return -1;
    for (int q = 0; q < 3; q++)
      if (t1[3 * m + q].v != R->t1[3 * m + q] || t2[3 * m + q].v != R->t2[3 * m + q]) return -1;
  }
  // 2. the solve stage
  BodiesT<D> DB;
  DB.capacity = n; DB.awake_count = B->awake_count; DB.awake_list = B->awake_list; DB.awake = B->awake;
  DB.position = w->position.data(); DB.rotation = w->rotation.data(); DB.velocity = w->velocity.data();
  DB.angular = w->angular.data(); DB.tumbled = w->tumbled.data(); DB.ceiling = w->ceiling.data();
  DB.start = w->start.data(); DB.start_q = w->start_q.data(); DB.inv_i = w->inv_i.data();
  DB.inv_mass = B->inv_mass; DB.inertia = B->inertia; DB.inv_inertia = B->inv_inertia; DB.dims = B->dims;
  DB.damping = B->damping; DB.angular_damping = B->angular_damping; DB.gravity_scale = B->gravity_scale;
  DB.type = B->type; DB.shape = B->shape; DB.frozen = B->frozen; DB.framed = B->framed; DB.lock = B->lock;
  DB.joint_head = B->joint_head;
  RowsT<D> DR;
  DR.count = count; DR.solved = R->solved;
  for (int k = 0; k < BG_STARTS; k++) DR.starts[k] = R->starts[k];
  DR.row = R->row; DR.a = R->a; DR.b = R->b; DR.points = R->points;
  DR.normal = normal.data(); DR.t1 = t1.data(); DR.t2 = t2.data(); DR.friction = friction.data();
  DR.restitution = restitution.data(); DR.tolerance = R->tolerance; DR.patch = R->patch;
  DR.separation = separation.data(); DR.point = point.data(); DR.shift = shift.data();
  DR.normal_impulse = ni.data(); DR.tangent_impulse1 = ti1.data(); DR.tangent_impulse2 = ti2.data();
  DR.roll_impulse1 = ri1.data(); DR.roll_impulse2 = ri2.data(); DR.spin_impulse = si.data();
  DR.drift1 = drift1.data(); DR.drift2 = drift2.data(); DR.gap = gap.data(); DR.max_normal_impulse = maxni.data();
  DR.relative_velocity = relvel.data(); DR.sliding = sliding.data(); DR.anchor_a = anchor_a.data();
  DR.anchor_b = anchor_b.data();
  {
    Stage<D> stage(DB, DR, nullptr);
    stage.run(*S);
  }
  // 3. keep: src/contact.js:1091-1115, each solved row into its pair's memory
  for (int m = 0; m < R->solved; m++) {
    DualMemory& to = w->memory[pair_key(R->a[m], R->b[m])];
    const int pts = R->points[m];
    to.points = pts;
    const D* T1 = &t1[3 * m];
    const D* T2 = &t2[3 * m];
    const D* N = &normal[3 * m];
    for (int q = 0; q < 3; q++) {
      to.twist[q] = T1[q] * ri1[m] + T2[q] * ri2[m] + N[q] * si[m];
      to.friction[q] = T1[q] * ti1[m] + T2[q] * ti2[m];
      to.slip[q] = T1[q] * drift1[m] + T2[q] * drift2[m];
    }
    for (int k = 0; k < pts; k++) {
      to.pid[k] = mem->pid[P * m + k];
      to.ni[k] = ni[P * m + k];
    }
  }
  // 4. the real parts into the host's output columns
  auto put = [](double* dst, const std::vector<D>& src, size_t k) {
    if (dst != nullptr)
      for (size_t i = 0; i < k; i++) dst[i] = src[i].v;
  };
  const size_t s = static_cast<size_t>(n), r = static_cast<size_t>(count);
  put(B->position, w->position, 3 * s); put(B->rotation, w->rotation, 4 * s); put(B->velocity, w->velocity, 3 * s);
  put(B->angular, w->angular, 3 * s); put(B->tumbled, w->tumbled, 3 * s); put(B->ceiling, w->ceiling, s);
  put(B->start, w->start, 3 * s); put(B->start_q, w->start_q, 4 * s); put(B->inv_i, w->inv_i, 6 * s);
  put(R->normal_impulse, ni, P * r); put(R->tangent_impulse1, ti1, r); put(R->tangent_impulse2, ti2, r);
  put(R->roll_impulse1, ri1, r); put(R->roll_impulse2, ri2, r); put(R->spin_impulse, si, r);
  put(R->drift1, drift1, r); put(R->drift2, drift2, r); put(R->gap, gap, r);
  put(R->max_normal_impulse, maxni, P * r); put(R->relative_velocity, relvel, P * r);
  put(R->anchor_a, anchor_a, 3 * r); put(R->anchor_b, anchor_b, 3 * r);
  for (size_t i = 0; i < r; i++) R->sliding[i] = sliding[i];
  return BG_OK;
}

// Body slot's position (3) and rotation (4) values, and their derivatives (7 x K, row-major).
int32_t oracle_dual_pose(const void* h, int32_t slot, double* value, double* tangents) {
  const DualWorld* w = static_cast<const DualWorld*>(h);
  if (slot < 0 || slot >= w->n) return BG_EINVAL;
  for (int k = 0; k < 7; k++) {
    const D& x = k < 3 ? w->position[3 * static_cast<size_t>(slot) + static_cast<size_t>(k)]
                       : w->rotation[4 * static_cast<size_t>(slot) + static_cast<size_t>(k - 3)];
    value[k] = x.v;
    for (int t = 0; t < dual::K; t++) tangents[dual::K * k + t] = x.d[t];
  }
  return BG_OK;
}

// One solve stage in dual numbers along one direction: `B`, `R` and `S` are its input as
// oracle_solve_step takes it; `dB` and `dR` give, in the same layout, the input's tangent (the
// columns the stage reads: bodies' position, rotation, velocity, angular, tumbled, ceiling; rows'
// normal, t1, t2, friction, restitution, separation, point, and the impulses and drift carried
// in), and receive the tangent of everything the stage writes.  The real parts go into B and R as
// oracle_solve_step leaves them.  Used to check the adjoint by dot products: for any seed y and
// direction x, y . (J x) here equals (J^T y) . x from the reverse sweep.
int32_t oracle_stage_jvp(const bg_bodies* B, const bg_rows* R, const bg_step* S, const bg_bodies* dB, const bg_rows* dR) {
  const size_t n = static_cast<size_t>(B->capacity), c = static_cast<size_t>(R->count);
  auto lift = [](const double* v, const double* d, size_t k) {
    std::vector<D> out(k > 0 ? k : 1);
    for (size_t i = 0; i < k; i++) {
      out[i] = D(v[i]);
      out[i].d[0] = d != nullptr ? d[i] : 0.0;
    }
    return out;
  };
  std::vector<D> position = lift(B->position, dB->position, 3 * n), rotation = lift(B->rotation, dB->rotation, 4 * n),
                 velocity = lift(B->velocity, dB->velocity, 3 * n), angular = lift(B->angular, dB->angular, 3 * n),
                 tumbled = lift(B->tumbled, dB->tumbled, 3 * n), ceiling = lift(B->ceiling, dB->ceiling, n),
                 start = lift(B->start, nullptr, 3 * n), start_q = lift(B->start_q, nullptr, 4 * n),
                 inv_i = lift(B->inv_i, nullptr, 6 * n);
  std::vector<D> normal = lift(R->normal, dR->normal, 3 * c), t1 = lift(R->t1, dR->t1, 3 * c),
                 t2 = lift(R->t2, dR->t2, 3 * c), friction = lift(R->friction, dR->friction, c),
                 restitution = lift(R->restitution, dR->restitution, c),
                 separation = lift(R->separation, dR->separation, P * c), point = lift(R->point, dR->point, 3 * P * c),
                 ni = lift(R->normal_impulse, dR->normal_impulse, P * c),
                 ti1 = lift(R->tangent_impulse1, dR->tangent_impulse1, c),
                 ti2 = lift(R->tangent_impulse2, dR->tangent_impulse2, c),
                 ri1 = lift(R->roll_impulse1, dR->roll_impulse1, c), ri2 = lift(R->roll_impulse2, dR->roll_impulse2, c),
                 si = lift(R->spin_impulse, dR->spin_impulse, c), drift1 = lift(R->drift1, dR->drift1, c),
                 drift2 = lift(R->drift2, dR->drift2, c), gap = lift(R->gap, nullptr, c),
                 maxni = lift(R->max_normal_impulse, nullptr, P * c), relvel = lift(R->relative_velocity, nullptr, P * c),
                 anchor_a = lift(R->anchor_a, nullptr, 3 * c), anchor_b = lift(R->anchor_b, nullptr, 3 * c);
  BodiesT<D> DB;
  DB.capacity = B->capacity; DB.awake_count = B->awake_count; DB.awake_list = B->awake_list; DB.awake = B->awake;
  DB.position = position.data(); DB.rotation = rotation.data(); DB.velocity = velocity.data();
  DB.angular = angular.data(); DB.tumbled = tumbled.data(); DB.ceiling = ceiling.data();
  DB.start = start.data(); DB.start_q = start_q.data(); DB.inv_i = inv_i.data();
  DB.inv_mass = B->inv_mass; DB.inertia = B->inertia; DB.inv_inertia = B->inv_inertia; DB.dims = B->dims;
  DB.damping = B->damping; DB.angular_damping = B->angular_damping; DB.gravity_scale = B->gravity_scale;
  DB.type = B->type; DB.shape = B->shape; DB.frozen = B->frozen; DB.framed = B->framed; DB.lock = B->lock;
  DB.joint_head = B->joint_head;
  RowsT<D> DR;
  DR.count = R->count; DR.solved = R->solved;
  for (int k = 0; k < BG_STARTS; k++) DR.starts[k] = R->starts[k];
  DR.row = R->row; DR.a = R->a; DR.b = R->b; DR.points = R->points;
  DR.normal = normal.data(); DR.t1 = t1.data(); DR.t2 = t2.data(); DR.friction = friction.data();
  DR.restitution = restitution.data(); DR.tolerance = R->tolerance; DR.patch = R->patch;
  DR.separation = separation.data(); DR.point = point.data(); DR.shift = R->shift;
  DR.normal_impulse = ni.data(); DR.tangent_impulse1 = ti1.data(); DR.tangent_impulse2 = ti2.data();
  DR.roll_impulse1 = ri1.data(); DR.roll_impulse2 = ri2.data(); DR.spin_impulse = si.data();
  DR.drift1 = drift1.data(); DR.drift2 = drift2.data(); DR.gap = gap.data(); DR.max_normal_impulse = maxni.data();
  DR.relative_velocity = relvel.data(); DR.sliding = R->sliding; DR.anchor_a = anchor_a.data();
  DR.anchor_b = anchor_b.data();
  {
    Stage<D> stage(DB, DR, nullptr);
    stage.run(*S);
  }
  auto drop = [](double* v, double* d, const std::vector<D>& src, size_t k) {
    for (size_t i = 0; i < k; i++) {
      if (v != nullptr) v[i] = src[i].v;
      if (d != nullptr) d[i] = src[i].d[0];
    }
  };
  drop(B->position, dB->position, position, 3 * n); drop(B->rotation, dB->rotation, rotation, 4 * n);
  drop(B->velocity, dB->velocity, velocity, 3 * n); drop(B->angular, dB->angular, angular, 3 * n);
  drop(B->tumbled, dB->tumbled, tumbled, 3 * n); drop(B->ceiling, dB->ceiling, ceiling, n);
  drop(B->start, dB->start, start, 3 * n); drop(B->start_q, dB->start_q, start_q, 4 * n);
  drop(B->inv_i, dB->inv_i, inv_i, 6 * n);
  drop(R->normal_impulse, dR->normal_impulse, ni, P * c); drop(R->tangent_impulse1, dR->tangent_impulse1, ti1, c);
  drop(R->tangent_impulse2, dR->tangent_impulse2, ti2, c); drop(R->roll_impulse1, dR->roll_impulse1, ri1, c);
  drop(R->roll_impulse2, dR->roll_impulse2, ri2, c); drop(R->spin_impulse, dR->spin_impulse, si, c);
  drop(R->drift1, dR->drift1, drift1, c); drop(R->drift2, dR->drift2, drift2, c); drop(R->gap, dR->gap, gap, c);
  drop(R->max_normal_impulse, dR->max_normal_impulse, maxni, P * c);
  drop(R->relative_velocity, dR->relative_velocity, relvel, P * c);
  drop(R->anchor_a, dR->anchor_a, anchor_a, 3 * c); drop(R->anchor_b, dR->anchor_b, anchor_b, 3 * c);
  return BG_OK;
}

}  // extern "C"
