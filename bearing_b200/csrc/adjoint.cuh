// The adjoint of the solve stage: gradients of a loss on a step's results with respect to the
// step's inputs, for batches of small worlds (one warp a world).
//
// Forward: the world's solve stage runs again from the step's input, colour by colour, and each
// pass leaves behind what its rows and bodies read before they ran (their velocities, impulses and
// poses: the "records").  Reverse: the passes run backwards (restitution, then each substep's
// relax, move, solve, warm start and accelerate, last substep first, then prepare and the start
// snapshot), colour by colour in reverse, and each row or body is replayed from its record with
// recording scalars (tape.hpp): the replay takes the very branches the forward pass took (the set
// of points the block LCP pushed, how many Newton rounds the friction cone took, which clamps
// held, whether a body tumbled), its results are seeded with the adjoints gathered so far, and the
// sweep gives the adjoints of what it read.  Rows of one colour share no body the solve moves
// (src/graph.js:1-33), so a colour's replays write disjoint adjoints and run in parallel; the
// overflow run replays one row at a time in reverse order.
//
// Each function restates the reference's arithmetic for any scalar T, citing what it follows:
//   src/contact.js  inertias 1302-1310, inverseAt 1493-1508, prepareRows 1346-1445, core
//                   1199-1219, lever 1565-1581, turning/along 1728-1737, warmRows 1616-1663,
//                   pushes 1672-1724, solveRows 1805-2090, writeBack 2101-2104, restitution
//                   2229-2251 (closing 2216-2220, push 1743-1749), slipped/turned 1122-1182
//   src/world.js    start snapshot 964-974, _accelerate 1495-1530, _move 1533-1563,
//                   tumble 2739-2763, untwist 2777-2805, advance 2820-2828, angular 2831-2834
//   src/core/math.js rotate 211-219, axesOf 222-227, quatMultiply 230-238
// With T = double and no contraction (-fmad=false), the forward pass gives the reference's bits.
//
// Scope: dynamic and static bodies (boxes, spheres, capsules) with no locks, no freezing and no
// joints; bg_backward refuses other worlds with BG_EUNSUPPORTED.
#pragma once

#include <math.h>
#include <stdint.h>

#include "stage.cuh"
#include "tape.hpp"

namespace bgadj {

#ifdef __CUDACC__
#define AHD __host__ __device__
#else
#define AHD
#endif

using bgad::TV;

constexpr int P = 4;
constexpr double COMPLIANCE = 9.5367431640625e-7;   // 2^-20, src/forest.js:67
constexpr double SPIN_DISC = 2.0 / 3.0;             // src/contact.js:146
constexpr double WORLD_SPIN = 3.141592653589793;    // src/world.js:171
constexpr double ROUNDED = 1.0 / 17592186044416.0;  // 2^-44, src/world.js:2812

// What prepare() leaves per row (doubles), and where.
constexpr int PR_RA = 0, PR_RB = 12, PR_LA = 24, PR_LB = 36, PR_ADJ = 48, PR_NM = 52, PR_JAC = 56, PR_K = 104,
              PR_LEV = 120, PR_FJ = 124, PR_TM = 148, PR_RM1 = 151, PR_RM2 = 152, PR_SM = 153, PR_ANA = 154,
              PR_ANB = 157, PREP = 160;
// A row's state a pass reads and writes: ni[4], ti1, ti2, ri1, ri2, si, maxni[4], relvel[4],
// now[4], gap, sliding (as 0 / 1).
constexpr int RS_NI = 0, RS_TI1 = 4, RS_TI2 = 5, RS_RI1 = 6, RS_RI2 = 7, RS_SI = 8, RS_MAXNI = 9, RS_RELVEL = 13,
              RS_NOW = 17, RS_GAP = 21, RS_SLID = 22, RSTATE = 23;
// A row's record before a pass: its state, then its bodies' velocities (v a, w a, v b, w b).
constexpr int REC_ROW = RSTATE + 12;
// A body's record in a substep: v, w before accelerate; p, q, v, w, tumbled, ceiling before move.
constexpr int RB_ACC = 0, RB_P = 6, RB_Q = 9, RB_V = 13, RB_W = 16, RB_TUM = 19, RB_CEIL = 22, REC_BODY = 23;
// A bouncy row's record before restitution: v a, w a, v b, w b, ni[4].
constexpr int REC_REST = 16;

using bgad::val;

// atan2 with the reference's own arctangent for the value (src/core/math.js:173-200), and its
// derivative (x dy - y dx) / (x^2 + y^2), 0 at the origin.
AHD inline double atan2_(double y, double x) { return bg::ref_atan2(y, x); }
AHD inline TV atan2_(const TV& y, const TV& x) {
  const double r = bg::ref_atan2(y.v, x.v), den = x.v * x.v + y.v * y.v;
  return bgad::binary(r, y, den > 0 ? x.v / den : 0.0, x, den > 0 ? -y.v / den : 0.0);
}

// Math.max with JavaScript's NaN and signed-zero rules.
template <class T>
AHD T jsmax(const T& a, const T& b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a > b) return a;
  if (b > a) return b;
  if (a == 0 && b == 0) return signbit(val(a)) ? b : a;
  return a;
}

// rotate: src/core/math.js:211-219.
template <class T>
AHD void rotate(const T* q, T x, T y, T z, bool inverse, T* out) {
  const double s = inverse ? -1 : 1;
  const T ux = q[0] * s, uy = q[1] * s, uz = q[2] * s, w = q[3];
  const T tx = 2 * (uy * z - uz * y), ty = 2 * (uz * x - ux * z), tz = 2 * (ux * y - uy * x);
  out[0] = x + w * tx + (uy * tz - uz * ty);
  out[1] = y + w * ty + (uz * tx - ux * tz);
  out[2] = z + w * tz + (ux * ty - uy * tx);
}

// axesOf: src/core/math.js:222-227.
template <class T>
AHD void axes_of(const T* q, T* ax) {
  const T x = q[0], y = q[1], z = q[2], w = q[3];
  ax[0] = 1 - 2 * (y * y + z * z); ax[1] = 2 * (x * y + z * w); ax[2] = 2 * (x * z - y * w);
  ax[3] = 2 * (x * y - z * w); ax[4] = 1 - 2 * (x * x + z * z); ax[5] = 2 * (y * z + x * w);
  ax[6] = 2 * (x * z + y * w); ax[7] = 2 * (y * z - x * w); ax[8] = 1 - 2 * (x * x + y * y);
}

// quatMultiply: src/core/math.js:230-238.
template <class T>
AHD void quat_mul(const T* a, const T* b, T* out) {
  const T ax = a[0], ay = a[1], az = a[2], aw = a[3];
  const T bx = b[0], by = b[1], bz = b[2], bw = b[3];
  out[0] = aw * bx + ax * bw + ay * bz - az * by;
  out[1] = aw * by + ay * bw + az * bx - ax * bz;
  out[2] = aw * bz + az * bw + ax * by - ay * bx;
  out[3] = aw * bw - ax * bx - ay * by - az * bz;
}

// ---- bodies ----

// inverseAt for a dynamic, unlocked body: R diag(1/I) R^T as six entries (src/contact.js:1493-1508).
template <class T>
AHD void inverse_inertia(const T* q, const double* inv, T* out) {
  T ax[9];
  axes_of(q, ax);
  const double i0 = inv[0], i1 = inv[1], i2 = inv[2];
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

// What a body's substep reads besides its state (src/world.js:1495-1563).
struct BodyConst {
  bool dynamic, sphere_unframed, lopsided;
  double gravity_scale, damping, angular_damping;
  double inertia[3], inv_inertia[3];
};

// _accelerate for one awake body: src/world.js:1495-1530.
template <class T>
AHD void accelerate(const BodyConst& b, const double* g, double h, int substeps, T* v, T* w) {
  if (!b.dynamic) return;
  const double gx = g[0] * h, gy = g[1] * h, gz = g[2] * h;
  const double most = WORLD_SPIN / (h * substeps);
  const double s = b.gravity_scale;
  v[0] += gx * s; v[1] += gy * s; v[2] += gz * s;
  if (b.damping != 0) {
    const double k = 1 / (1 + h * b.damping);
    v[0] *= k; v[1] *= k; v[2] *= k;
  }
  if (b.angular_damping != 0) {
    const double k = 1 / (1 + h * b.angular_damping);
    w[0] *= k; w[1] *= k; w[2] *= k;
  }
  if (!b.sphere_unframed) {
    const T w2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    if (w2 > most * most) {
      const T k = most / sqrt(w2);
      w[0] *= k; w[1] *= k; w[2] *= k;
    }
  }
}

// advance: src/world.js:2820-2828.
template <class T>
AHD void advance(const T* q, T wx, T wy, T wz, double h, T* out) {
  const T x = q[0], y = q[1], z = q[2], w = q[3];
  const T nx = x + h * (wx * w + wy * z - wz * y);
  const T ny = y + h * (wy * w + wz * x - wx * z);
  const T nz = z + h * (wz * w + wx * y - wy * x);
  const T nw = w - h * (wx * x + wy * y + wz * z);
  const T l = 1 / sqrt(nx * nx + ny * ny + nz * nz + nw * nw);
  out[0] = nx * l; out[1] = ny * l; out[2] = nz * l; out[3] = nw * l;
}

// angular: src/world.js:2831-2834.
template <class T>
AHD void angular_of(const T* q, const double* inv, T lx, T ly, T lz, T* out) {
  T v3[3];
  rotate(q, lx, ly, lz, true, v3);
  rotate(q, v3[0] * inv[0], v3[1] * inv[1], v3[2] * inv[2], false, out);
}

// untwist: src/world.js:2777-2805.
template <class T>
AHD void untwist(T* q, const double* inv, T lx, T ly, T lz, T most) {
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
  quat_mul(q, T4, Q4);
  const T n = 1 / sqrt(Q4[0] * Q4[0] + Q4[1] * Q4[1] + Q4[2] * Q4[2] + Q4[3] * Q4[3]);
  q[0] = Q4[0] * n; q[1] = Q4[1] * n; q[2] = Q4[2] * n; q[3] = Q4[3] * n;
}

// _move for one awake body (src/world.js:1533-1563), tumble() for a lopsided one (2739-2763).
template <class T>
AHD void move(const BodyConst& b, double h, T* p, T* q, const T* v, T* w, T* left, T* ceiling) {
  p[0] += v[0] * h; p[1] += v[1] * h; p[2] += v[2] * h;
  const T wx = w[0], wy = w[1], wz = w[2];
  const bool turning = wx != 0 || wy != 0 || wz != 0;
  if (turning && b.dynamic && b.lopsided) {
    const double* I = b.inertia;
    const double* inv = b.inv_inertia;
    T v3[3], q4[4];
    rotate(q, w[0], w[1], w[2], true, v3);
    rotate(q, v3[0] * I[0], v3[1] * I[1], v3[2] * I[2], false, v3);
    const T lx = v3[0], ly = v3[1], lz = v3[2];
    if (w[0] != left[0] || w[1] != left[1] || w[2] != left[2]) ceiling[0] = w[0] * lx + w[1] * ly + w[2] * lz;
    const T most = ceiling[0];
    advance(q, w[0], w[1], w[2], h * 0.25, q4);
    angular_of(q4, inv, lx, ly, lz, v3);
    advance(q, v3[0], v3[1], v3[2], h * 0.5, q);
    angular_of(q, inv, lx, ly, lz, v3);
    if (v3[0] * lx + v3[1] * ly + v3[2] * lz > most * (1 + ROUNDED)) {
      untwist(q, inv, lx, ly, lz, most);
      angular_of(q, inv, lx, ly, lz, v3);
    }
    w[0] = v3[0]; w[1] = v3[1]; w[2] = v3[2];
    left[0] = v3[0]; left[1] = v3[1]; left[2] = v3[2];
  } else if (turning) {
    advance(q, wx, wy, wz, h * 0.5, q);
  }
}

// ---- rows ----

// Everything a row reads or writes, as pointers: into the world's columns for the forward pass, or
// into a replay's own arrays of leaves.
template <class T>
struct RowIO {
  T *va, *wa, *vb, *wb;                    // the bodies' velocities
  const T *pa, *pb, *qa, *qb, *sa, *sb;    // poses and where the step started them
  const T *ia, *ib;                        // world inverse inertias (6 each)
  double ima, imb;
  T* st;                                   // the row's state (RS_*)
  T* pr;                                   // what prepare() left (PR_*)
  const T *normal, *t1, *t2, *friction, *restitution, *separation, *point;
  T *drift1, *drift2;
  double tolerance, patch;
  const double* shift;
  int count;
  int shape_a, shape_b;
  double dims_a[3], dims_b[3];
};

// core(): src/contact.js:1199-1219, whole bodies.
template <class T>
AHD void core(int shape, const double* dims, const T* q, T x, T y, T z, T* out, T* v3) {
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
  const double half = (dims[1] - 2 * dims[0]) * 0.5;
  out[0] = 0; out[1] = v3[1] < -half ? T(-half) : v3[1] > half ? T(half) : v3[1]; out[2] = 0;
  rotate(q, T(0), out[1], T(0), false, v3);
}

// lever(): src/contact.js:1565-1581.
template <class T>
AHD T lever(T* jac, const T* ia, const T* ib, double ima, double imb, T rax, T ray, T raz, T rbx, T rby, T rbz,
            T dx, T dy, T dz) {
  const T cax = ray * dz - raz * dy, cay = raz * dx - rax * dz, caz = rax * dy - ray * dx;
  const T cbx = rby * dz - rbz * dy, cby = rbz * dx - rbx * dz, cbz = rbx * dy - rby * dx;
  const T iax = ia[0] * cax + ia[1] * cay + ia[2] * caz;
  const T iay = ia[1] * cax + ia[3] * cay + ia[4] * caz;
  const T iaz = ia[2] * cax + ia[4] * cay + ia[5] * caz;
  const T ibx = ib[0] * cbx + ib[1] * cby + ib[2] * cbz;
  const T iby = ib[1] * cbx + ib[3] * cby + ib[4] * cbz;
  const T ibz = ib[2] * cbx + ib[4] * cby + ib[5] * cbz;
  jac[0] = cax; jac[1] = cay; jac[2] = caz;
  jac[3] = cbx; jac[4] = cby; jac[5] = cbz;
  jac[6] = iax; jac[7] = iay; jac[8] = iaz;
  jac[9] = ibx; jac[10] = iby; jac[11] = ibz;
  const T k = ima + imb + cax * iax + cay * iay + caz * iaz + cbx * ibx + cby * iby + cbz * ibz;
  return k > 0 ? 1 / k : T(0);
}

// along / turning: src/contact.js:1728-1737.
template <class T>
AHD T along(const T* I, T x, T y, T z) {
  return I[0] * x * x + I[3] * y * y + I[5] * z * z + 2 * (I[1] * x * y + I[2] * x * z + I[4] * y * z);
}
template <class T>
AHD T turning(const T* ia, const T* ib, T x, T y, T z) {
  const T k = along(ia, x, y, z) + along(ib, x, y, z);
  return k > 0 ? 1 / k : T(0);
}

// prepareRows for one row: src/contact.js:1346-1445.  Writes pr[] and the state's relvel and
// maxni.
template <class T>
AHD void prepare_row(const RowIO<T>& r) {
  T* pr = r.pr;
  T* st = r.st;
  const T nx = r.normal[0], ny = r.normal[1], nz = r.normal[2];
  const T* T1 = r.t1;
  const T* T2 = r.t2;
  const int count = r.count;
  if (count <= 2) {
    pr[PR_RM1] = turning(r.ia, r.ib, T1[0], T1[1], T1[2]);
    pr[PR_RM2] = turning(r.ia, r.ib, T2[0], T2[1], T2[2]);
  }
  pr[PR_SM] = turning(r.ia, r.ib, nx, ny, nz);
  const double tol = r.tolerance;
  T weight = 0, ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0;
  T ex = 0, ey = 0, ez = 0, fx = 0, fy = 0, fz = 0;
  for (int k = 0; k < count; k++) {
    const int i3 = 3 * k;
    const T px = r.point[i3], py = r.point[i3 + 1], pz = r.point[i3 + 2];
    const T rax = px - r.pa[0], ray = py - r.pa[1], raz = pz - r.pa[2];
    const T rbx = px + r.shift[i3] - r.pb[0], rby = py + r.shift[i3 + 1] - r.pb[1], rbz = pz + r.shift[i3 + 2] - r.pb[2];
    pr[PR_RA + i3] = rax; pr[PR_RA + i3 + 1] = ray; pr[PR_RA + i3 + 2] = raz;
    pr[PR_RB + i3] = rbx; pr[PR_RB + i3 + 1] = rby; pr[PR_RB + i3 + 2] = rbz;
    T va[3], vb[3];
    core(r.shape_a, r.dims_a, r.qa, rax, ray, raz, &pr[PR_LA + i3], va);
    core(r.shape_b, r.dims_b, r.qb, rbx, rby, rbz, &pr[PR_LB + i3], vb);
    pr[PR_ADJ + k] = r.separation[k] - ((vb[0] - va[0]) * nx + (vb[1] - va[1]) * ny + (vb[2] - va[2]) * nz);
    pr[PR_NM + k] = lever(&pr[PR_JAC + 12 * k], r.ia, r.ib, r.ima, r.imb, rax, ray, raz, rbx, rby, rbz, nx, ny, nz);
    st[RS_MAXNI + k] = 0;
    const T s = r.separation[k] / tol;
    const T near = s <= 1 ? T(1) : s >= 2 ? T(0) : 2 - s;
    weight += near;
    ax += near * rax; ay += near * ray; az += near * raz; bx += near * rbx; by += near * rby; bz += near * rbz;
    ex += rax; ey += ray; ez += raz; fx += rbx; fy += rby; fz += rbz;
    const T* va_ = r.va;
    const T* wa_ = r.wa;
    const T* vb_ = r.vb;
    const T* wb_ = r.wb;
    const T dvx = vb_[0] + wb_[1] * rbz - wb_[2] * rby - va_[0] - wa_[1] * raz + wa_[2] * ray;
    const T dvy = vb_[1] + wb_[2] * rbx - wb_[0] * rbz - va_[1] - wa_[2] * rax + wa_[0] * raz;
    const T dvz = vb_[2] + wb_[0] * rby - wb_[1] * rbx - va_[2] - wa_[0] * ray + wa_[1] * rax;
    st[RS_RELVEL + k] = dvx * nx + dvy * ny + dvz * nz;
  }
  if (count >= 2) {
    const double s = r.ima + r.imb;
    T* K = &pr[PR_K];
    for (int k = 0; k < count; k++) {
      const T* jk = &pr[PR_JAC + 12 * k];
      for (int l = 0; l <= k; l++) {
        const T* jl = &pr[PR_JAC + 12 * l];
        const T e = s + jk[0] * jl[6] + jk[1] * jl[7] + jk[2] * jl[8] + jk[3] * jl[9] + jk[4] * jl[10] + jk[5] * jl[11];
        K[P * k + l] = e; K[P * l + k] = e;
      }
    }
  }
  if (weight == 0) { weight = count; ax = ex; ay = ey; az = ez; bx = fx; by = fy; bz = fz; }
  ax /= weight; ay /= weight; az /= weight; bx /= weight; by /= weight; bz /= weight;
  pr[PR_ANA] = ax; pr[PR_ANA + 1] = ay; pr[PR_ANA + 2] = az;
  pr[PR_ANB] = bx; pr[PR_ANB + 1] = by; pr[PR_ANB + 2] = bz;
  for (int k = 0; k < count; k++) {
    const int i3 = 3 * k;
    T dx = pr[PR_RA + i3] - ax, dy = pr[PR_RA + i3 + 1] - ay, dz = pr[PR_RA + i3 + 2] - az;
    const T alongN = dx * nx + dy * ny + dz * nz;
    dx -= alongN * nx; dy -= alongN * ny; dz -= alongN * nz;
    pr[PR_LEV + k] = sqrt(dx * dx + dy * dy + dz * dz);
  }
  T* fj = &pr[PR_FJ];
  lever(fj, r.ia, r.ib, r.ima, r.imb, ax, ay, az, bx, by, bz, T1[0], T1[1], T1[2]);
  lever(fj + 12, r.ia, r.ib, r.ima, r.imb, ax, ay, az, bx, by, bz, T2[0], T2[1], T2[2]);
  const T k11 = r.ima + r.imb + fj[0] * fj[6] + fj[1] * fj[7] + fj[2] * fj[8] + fj[3] * fj[9] + fj[4] * fj[10] + fj[5] * fj[11];
  const T k22 = r.ima + r.imb + fj[12] * fj[18] + fj[13] * fj[19] + fj[14] * fj[20] + fj[15] * fj[21] + fj[16] * fj[22] +
                fj[17] * fj[23];
  const T k12 = fj[12] * fj[6] + fj[13] * fj[7] + fj[14] * fj[8] + fj[15] * fj[9] + fj[16] * fj[10] + fj[17] * fj[11];
  const T det = k11 * k22 - k12 * k12;
  if (det > 0) {
    pr[PR_TM] = k22 / det; pr[PR_TM + 1] = -k12 / det; pr[PR_TM + 2] = k11 / det;
  } else {
    pr[PR_TM] = 0; pr[PR_TM + 1] = 0; pr[PR_TM + 2] = 0;
  }
}

// writeBack: src/contact.js:2101-2104 (a body with inverse mass 0 is not written).
template <class T>
AHD void write_back(double im, T* v, T* w, const T* vl, const T* wl) {
  if (im == 0) return;
  for (int c = 0; c < 3; c++) { v[c] = vl[c]; w[c] = wl[c]; }
}

// warmRows for one row: src/contact.js:1616-1663.
template <class T>
AHD void warm_row(const RowIO<T>& r) {
  const T* st = r.st;
  const T* pr = r.pr;
  const T nx = r.normal[0], ny = r.normal[1], nz = r.normal[2];
  const T t1x = r.t1[0], t1y = r.t1[1], t1z = r.t1[2];
  const T t2x = r.t2[0], t2y = r.t2[1], t2z = r.t2[2];
  const double ima = r.ima, imb = r.imb;
  T va[3] = {r.va[0], r.va[1], r.va[2]}, wa[3] = {r.wa[0], r.wa[1], r.wa[2]};
  T vb[3] = {r.vb[0], r.vb[1], r.vb[2]}, wb[3] = {r.wb[0], r.wb[1], r.wb[2]};
  for (int k = 0; k < r.count; k++) {
    const T* jac = &pr[PR_JAC + 12 * k];
    const T ln = st[RS_NI + k];
    const T px = nx * ln, py = ny * ln, pz = nz * ln;
    va[0] -= ima * px; va[1] -= ima * py; va[2] -= ima * pz;
    vb[0] += imb * px; vb[1] += imb * py; vb[2] += imb * pz;
    wa[0] -= jac[6] * ln; wa[1] -= jac[7] * ln; wa[2] -= jac[8] * ln;
    wb[0] += jac[9] * ln; wb[1] += jac[10] * ln; wb[2] += jac[11] * ln;
  }
  {
    const T* fj = &pr[PR_FJ];
    const T l1 = st[RS_TI1], l2 = st[RS_TI2];
    const T px = t1x * l1 + t2x * l2, py = t1y * l1 + t2y * l2, pz = t1z * l1 + t2z * l2;
    va[0] -= ima * px; va[1] -= ima * py; va[2] -= ima * pz;
    vb[0] += imb * px; vb[1] += imb * py; vb[2] += imb * pz;
    wa[0] -= fj[6] * l1 + fj[18] * l2; wa[1] -= fj[7] * l1 + fj[19] * l2; wa[2] -= fj[8] * l1 + fj[20] * l2;
    wb[0] += fj[9] * l1 + fj[21] * l2; wb[1] += fj[10] * l1 + fj[22] * l2; wb[2] += fj[11] * l1 + fj[23] * l2;
  }
  {
    const T r1 = st[RS_RI1], r2 = st[RS_RI2], sp = st[RS_SI];
    const T* ia = r.ia;
    const T* ib = r.ib;
    const T lx = t1x * r1 + t2x * r2 + nx * sp, ly = t1y * r1 + t2y * r2 + ny * sp, lz = t1z * r1 + t2z * r2 + nz * sp;
    wa[0] -= ia[0] * lx + ia[1] * ly + ia[2] * lz;
    wa[1] -= ia[1] * lx + ia[3] * ly + ia[4] * lz;
    wa[2] -= ia[2] * lx + ia[4] * ly + ia[5] * lz;
    wb[0] += ib[0] * lx + ib[1] * ly + ib[2] * lz;
    wb[1] += ib[1] * lx + ib[3] * ly + ib[4] * lz;
    wb[2] += ib[2] * lx + ib[4] * ly + ib[5] * lz;
  }
  write_back(ima, r.va, r.wa, va, wa);
  write_back(imb, r.vb, r.wb, vb, wb);
}

// pushes: src/contact.js:1672-1724, the block's equations on the points in `set`.
template <class T>
AHD void pushes(const T* K, int count, int set, const double* give, const T* wanted, T* solved) {
  T AS[P * P], RS[P], XS[P];
  int IN[P];
  int n = 0;
  for (int k = 0; k < count; k++) {
    solved[k] = 0;
    if (set >> k & 1) IN[n++] = k;
  }
  if (set == 15) {
    const double g0 = 1 + give[0], g1 = 1 + give[1], g2 = 1 + give[2], g3 = 1 + give[3];
    T a00 = K[0] * g0, a01 = K[1], a02 = K[2], a03 = K[3];
    T a11 = K[5] * g1, a12 = K[6], a13 = K[7];
    T a21 = K[9], a22 = K[10] * g2, a23 = K[11];
    T a31 = K[13], a32 = K[14], a33 = K[15] * g3;
    const T a10 = K[4], a20 = K[8], a30 = K[12];
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
    return;
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

// The soft-contact constants for the substep (makeSoft, src/contact.js:1591-1597).
struct SoftK {
  double biasRate, massScale, impulseScale;
};

// The friction cone's projection (src/contact.js:2015-2033): (n1, n2) outside the ellipse of the
// inverse tangent mass (ma mb; mb mc) scaled to `limit`, brought onto it by Newton's method on the
// multiplier al, in place.
template <class T>
AHD void cone(const T& limit, const T& ma, const T& mb, const T& mc, T& n1, T& n2) {
  T al = 0, x = n1, y = n2, ll = n1 * n1 + n2 * n2;
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
}

// solveRows for one row: src/contact.js:1805-2090.  bias: a solving pass (else relaxing);
// known: the separations the last relaxing pass left in now[] still hold.
template <class T>
AHD void solve_row(const RowIO<T>& r, double h, bool bias, bool known, const SoftK& soft) {
  T* st = r.st;
  const T* pr = r.pr;
  const double inv = 1 / h;
  const double springy = soft.impulseScale / soft.massScale + COMPLIANCE;
  const T nx = r.normal[0], ny = r.normal[1], nz = r.normal[2];
  const double maxBias = r.tolerance * inv;
  const int count = r.count;
  T target[P], closingNow[P], wanted[P], solved[P];
  double massScale[P], impulseScale[P], give[P];
  T dn = 0, nax = 0, nay = 0, naz = 0, nbx = 0, nby = 0, nbz = 0;
  if (!known) {
    const T dx = (r.pb[0] - r.sb[0]) - (r.pa[0] - r.sa[0]);
    const T dy = (r.pb[1] - r.sb[1]) - (r.pa[1] - r.sa[1]);
    const T dz = (r.pb[2] - r.sb[2]) - (r.pa[2] - r.sa[2]);
    T v3[3];
    dn = dx * nx + dy * ny + dz * nz;
    rotate(r.qa, nx, ny, nz, true, v3);
    nax = v3[0]; nay = v3[1]; naz = v3[2];
    rotate(r.qb, nx, ny, nz, true, v3);
    nbx = v3[0]; nby = v3[1]; nbz = v3[2];
  }
  T least = INFINITY;
  for (int k = 0; k < count; k++) {
    const int i3 = 3 * k;
    T s;
    if (known) {
      s = st[RS_NOW + k];
    } else {
      s = dn + (pr[PR_LB + i3] * nbx + pr[PR_LB + i3 + 1] * nby + pr[PR_LB + i3 + 2] * nbz) -
          (pr[PR_LA + i3] * nax + pr[PR_LA + i3 + 1] * nay + pr[PR_LA + i3 + 2] * naz) + pr[PR_ADJ + k];
      if (!bias) st[RS_NOW + k] = s;
    }
    if (s < least) least = s;
    if (s > 0) {
      target[k] = s * inv; massScale[k] = 1; impulseScale[k] = 0; give[k] = COMPLIANCE;
    } else if (bias) {
      target[k] = jsmax(soft.biasRate * s, T(-maxBias));
      massScale[k] = soft.massScale; impulseScale[k] = soft.impulseScale; give[k] = springy;
    } else {
      target[k] = 0; massScale[k] = 1; impulseScale[k] = 0; give[k] = COMPLIANCE;
    }
  }
  st[RS_GAP] = least;
  const double ima = r.ima, imb = r.imb;
  const T* K = &pr[PR_K];
  T vax = r.va[0], vay = r.va[1], vaz = r.va[2], wax = r.wa[0], way = r.wa[1], waz = r.wa[2];
  T vbx = r.vb[0], vby = r.vb[1], vbz = r.vb[2], wbx = r.wb[0], wby = r.wb[1], wbz = r.wb[2];
  if (count == 1 || !(K[0] > 0)) {
    for (int k = 0; k < count; k++) {
      const T* jac = &pr[PR_JAC + 12 * k];
      const T vn = (vbx - vax) * nx + (vby - vay) * ny + (vbz - vaz) * nz + wbx * jac[3] + wby * jac[4] + wbz * jac[5] -
                   wax * jac[0] - way * jac[1] - waz * jac[2];
      const T old = st[RS_NI + k];
      T next = old - pr[PR_NM + k] * massScale[k] * (vn + target[k]) - impulseScale[k] * old;
      if (next < 0) next = 0;
      closingNow[k] = vn; solved[k] = next;
    }
  } else {
    for (int k = 0; k < count; k++) {
      const T* jac = &pr[PR_JAC + 12 * k];
      closingNow[k] = (vbx - vax) * nx + (vby - vay) * ny + (vbz - vaz) * nz + wbx * jac[3] + wby * jac[4] +
                      wbz * jac[5] - wax * jac[0] - way * jac[1] - waz * jac[2];
    }
    int set = 0;
    for (int k = 0; k < count; k++) {
      T rr = -closingNow[k] - target[k];
      for (int l = 0; l < count; l++) rr += K[P * k + l] * st[RS_NI + l];
      wanted[k] = rr;
      if (rr > 0) set |= 1 << k;
    }
    for (int round = 0;; round++) {
      pushes(K, count, set, give, wanted, solved);
      int flip = -1;
      for (int k = 0; k < count && flip < 0; k++) {
        if (set >> k & 1) {
          if (solved[k] < 0) flip = k;
        } else {
          T rr = -wanted[k];
          for (int l = 0; l < count; l++) rr += K[P * k + l] * solved[l];
          if (rr < 0) flip = k;
        }
      }
      if (flip < 0 || round == 1 << count) break;
      set ^= 1 << flip;
    }
  }
  for (int k = 0; k < count; k++) {
    const T* jac = &pr[PR_JAC + 12 * k];
    const T old = st[RS_NI + k], next = solved[k] > 0 ? solved[k] : T(0);
    const T d = next - old;
    st[RS_NI + k] = next;
    if (d > 0 && st[RS_MAXNI + k] == 0) st[RS_RELVEL + k] = closingNow[k];
    if (d > st[RS_MAXNI + k]) st[RS_MAXNI + k] = d;
    const T px = nx * d, py = ny * d, pz = nz * d;
    vax -= ima * px; vay -= ima * py; vaz -= ima * pz;
    vbx += imb * px; vby += imb * py; vbz += imb * pz;
    wax -= jac[6] * d; way -= jac[7] * d; waz -= jac[8] * d;
    wbx += jac[9] * d; wby += jac[10] * d; wbz += jac[11] * d;
  }
  const T mu = r.friction[0];
  const T t1x = r.t1[0], t1y = r.t1[1], t1z = r.t1[2];
  const T t2x = r.t2[0], t2y = r.t2[1], t2z = r.t2[2];
  T pressed = 0, twisted = 0;
  for (int k = 0; k < count; k++) {
    pressed += st[RS_NI + k];
    twisted += pr[PR_LEV + k] * st[RS_NI + k];
  }
  {
    const T* fj = &pr[PR_FJ];
    const T* g = fj + 12;
    const T dvx = vbx - vax, dvy = vby - vay, dvz = vbz - vaz;
    T v1 = dvx * t1x + dvy * t1y + dvz * t1z + wbx * fj[3] + wby * fj[4] + wbz * fj[5] - wax * fj[0] - way * fj[1] -
           waz * fj[2];
    T v2 = dvx * t2x + dvy * t2y + dvz * t2z + wbx * g[3] + wby * g[4] + wbz * g[5] - wax * g[0] - way * g[1] - waz * g[2];
    const T s1 = r.drift1[0], s2 = r.drift2[0];
    if (bias && (s1 != 0 || s2 != 0)) {
      T b1 = soft.biasRate * s1, b2 = soft.biasRate * s2;
      const T bb = b1 * b1 + b2 * b2;
      if (bb > maxBias * maxBias) {
        const T scale = maxBias / sqrt(bb);
        b1 *= scale; b2 *= scale;
      }
      v1 += b1; v2 += b2;
    }
    const T* tm = &pr[PR_TM];
    const T o1 = st[RS_TI1], o2 = st[RS_TI2];
    T n1 = o1 - (tm[0] * v1 + tm[1] * v2), n2 = o2 - (tm[1] * v1 + tm[2] * v2);
    const T limit = mu * pressed, l2 = n1 * n1 + n2 * n2;
    if (l2 > limit * limit) {
      cone(limit, tm[0], tm[1], tm[2], n1, n2);
      st[RS_SLID] = 1;
    } else {
      st[RS_SLID] = 0;
    }
    st[RS_TI1] = n1; st[RS_TI2] = n2;
    const T d1 = n1 - o1, d2 = n2 - o2;
    const T px = t1x * d1 + t2x * d2, py = t1y * d1 + t2y * d2, pz = t1z * d1 + t2z * d2;
    vax -= ima * px; vay -= ima * py; vaz -= ima * pz;
    vbx += imb * px; vby += imb * py; vbz += imb * pz;
    wax -= fj[6] * d1 + g[6] * d2; way -= fj[7] * d1 + g[7] * d2; waz -= fj[8] * d1 + g[8] * d2;
    wbx += fj[9] * d1 + g[9] * d2; wby += fj[10] * d1 + g[10] * d2; wbz += fj[11] * d1 + g[11] * d2;
  }
  const T* ia = r.ia;
  const T* ib = r.ib;
  if (count <= 2) {
    const T most = r.patch * pressed;
    const T ux = wbx - wax, uy = wby - way, uz = wbz - waz;
    const T r1 = st[RS_RI1], r2 = st[RS_RI2];
    T n1 = r1 - pr[PR_RM1] * (ux * t1x + uy * t1y + uz * t1z);
    T n2 = r2 - pr[PR_RM2] * (ux * t2x + uy * t2y + uz * t2z);
    const T l2 = n1 * n1 + n2 * n2;
    if (l2 > most * most) {
      const T scale = most / sqrt(l2);
      n1 *= scale; n2 *= scale;
    }
    st[RS_RI1] = n1; st[RS_RI2] = n2;
    const T d1 = n1 - r1, d2 = n2 - r2;
    const T lx = t1x * d1 + t2x * d2, ly = t1y * d1 + t2y * d2, lz = t1z * d1 + t2z * d2;
    wax -= ia[0] * lx + ia[1] * ly + ia[2] * lz;
    way -= ia[1] * lx + ia[3] * ly + ia[4] * lz;
    waz -= ia[2] * lx + ia[4] * ly + ia[5] * lz;
    wbx += ib[0] * lx + ib[1] * ly + ib[2] * lz;
    wby += ib[1] * lx + ib[3] * ly + ib[4] * lz;
    wbz += ib[2] * lx + ib[4] * ly + ib[5] * lz;
  }
  {
    const T limit = count == 1 ? SPIN_DISC * mu * r.patch * pressed : mu * twisted;
    const T s0 = st[RS_SI];
    T s1 = s0 - pr[PR_SM] * ((wbx - wax) * nx + (wby - way) * ny + (wbz - waz) * nz);
    if (s1 > limit) s1 = limit; else if (s1 < -limit) s1 = -limit;
    st[RS_SI] = s1;
    const T ds = s1 - s0, lx = nx * ds, ly = ny * ds, lz = nz * ds;
    wax -= ia[0] * lx + ia[1] * ly + ia[2] * lz;
    way -= ia[1] * lx + ia[3] * ly + ia[4] * lz;
    waz -= ia[2] * lx + ia[4] * ly + ia[5] * lz;
    wbx += ib[0] * lx + ib[1] * ly + ib[2] * lz;
    wby += ib[1] * lx + ib[3] * ly + ib[4] * lz;
    wbz += ib[2] * lx + ib[4] * ly + ib[5] * lz;
  }
  const T va[3] = {vax, vay, vaz}, wa[3] = {wax, way, waz}, vb[3] = {vbx, vby, vbz}, wb[3] = {wbx, wby, wbz};
  write_back(ima, r.va, r.wa, va, wa);
  write_back(imb, r.vb, r.wb, vb, wb);
}

// Whether row r has a point restitution() works on: src/contact.js:2233-2241.
template <class T>
AHD bool bouncy(const RowIO<T>& r, double gravity) {
  if (r.restitution[0] == 0) return false;
  const double threshold = sqrt(2 * gravity * r.tolerance);
  for (int k = 0; k < r.count; k++)
    if (!(r.st[RS_RELVEL + k] > -threshold || r.st[RS_MAXNI + k] == 0)) return true;
  return false;
}

// restitution for one row: src/contact.js:2234-2250 (closing 2216-2220, push 1743-1749).  Every
// body is written as push() writes it, a body of inverse mass 0 included (v - 0 * px).
template <class T>
AHD void bounce_row(const RowIO<T>& r, double gravity) {
  T* st = r.st;
  const T* pr = r.pr;
  const T e = r.restitution[0];
  const double threshold = sqrt(2 * gravity * r.tolerance);
  const T nx = r.normal[0], ny = r.normal[1], nz = r.normal[2];
  const double ima = r.ima, imb = r.imb;
  for (int k = 0; k < r.count; k++) {
    const T rv = st[RS_RELVEL + k];
    if (rv > -threshold || st[RS_MAXNI + k] == 0) continue;
    const T* jac = &pr[PR_JAC + 12 * k];
    const T vn = (r.vb[0] - r.va[0]) * nx + (r.vb[1] - r.va[1]) * ny + (r.vb[2] - r.va[2]) * nz + r.wb[0] * jac[3] +
                 r.wb[1] * jac[4] + r.wb[2] * jac[5] - r.wa[0] * jac[0] - r.wa[1] * jac[1] - r.wa[2] * jac[2];
    const T old = st[RS_NI + k];
    T next = old - pr[PR_NM + k] * (vn + e * rv);
    if (next < 0) next = 0;
    const T d = next - old;
    st[RS_NI + k] = next;
    const T px = nx * d, py = ny * d, pz = nz * d;
    r.va[0] -= ima * px; r.va[1] -= ima * py; r.va[2] -= ima * pz;
    r.vb[0] += imb * px; r.vb[1] += imb * py; r.vb[2] += imb * pz;
    r.wa[0] -= jac[6] * d; r.wa[1] -= jac[7] * d; r.wa[2] -= jac[8] * d;
    r.wb[0] += jac[9] * d; r.wb[1] += jac[10] * d; r.wb[2] += jac[11] * d;
  }
}

// turned: src/contact.js:1168-1182.
template <class T>
AHD void turned(const T* p, const T* start, const T* q, const T* q0, T* out) {
  const T ax = q[0], ay = q[1], az = q[2], aw = q[3];
  const T bx = -q0[0], by = -q0[1], bz = -q0[2], bw = q0[3];
  T ux = aw * bx + ax * bw + ay * bz - az * by;
  T uy = aw * by + ay * bw + az * bx - ax * bz;
  T uz = aw * bz + az * bw + ax * by - ay * bx;
  T uw = aw * bw - ax * bx - ay * by - az * bz;
  if (uw < 0) { ux = -ux; uy = -uy; uz = -uz; uw = -uw; }
  const T sine = sqrt(ux * ux + uy * uy + uz * uz);
  const T k = sine == 0 ? T(0) : 2 * atan2_(sine, uw) / sine;
  out[0] = p[0] - start[0]; out[1] = p[1] - start[1]; out[2] = p[2] - start[2];
  out[3] = ux * k; out[4] = uy * k; out[5] = uz * k;
}

// slipped for one row: src/contact.js:1122-1153.  The poses are the step's last; qa0 / qb0 the
// start rotations.  awake_a / awake_b: whether each body moved in the step.
template <class T>
AHD void slipped_row(const RowIO<T>& r, const T* qa0, const T* qb0, bool awake_a, bool awake_b) {
  T pressed = 0;
  bool impact = false;
  for (int k = 0; k < r.count; k++) {
    pressed += r.st[RS_NI + k];
    if (r.shift[3 * k] != 0 || r.shift[3 * k + 1] != 0 || r.shift[3 * k + 2] != 0) impact = true;
  }
  if (r.st[RS_SLID] != 0 || pressed == 0 || impact) {
    r.drift1[0] = 0; r.drift2[0] = 0;
    return;
  }
  T turn[6];
  T dx = 0, dy = 0, dz = 0;
  if (awake_b) {
    turned(r.pb, r.sb, r.qb, qb0, turn);
    const T rx = r.pr[PR_ANB], ry = r.pr[PR_ANB + 1], rz = r.pr[PR_ANB + 2];
    dx = turn[0] + turn[4] * rz - turn[5] * ry;
    dy = turn[1] + turn[5] * rx - turn[3] * rz;
    dz = turn[2] + turn[3] * ry - turn[4] * rx;
  }
  if (awake_a) {
    turned(r.pa, r.sa, r.qa, qa0, turn);
    const T rx = r.pr[PR_ANA], ry = r.pr[PR_ANA + 1], rz = r.pr[PR_ANA + 2];
    dx -= turn[0] + turn[4] * rz - turn[5] * ry;
    dy -= turn[1] + turn[5] * rx - turn[3] * rz;
    dz -= turn[2] + turn[3] * ry - turn[4] * rx;
  }
  r.drift1[0] += dx * r.t1[0] + dy * r.t1[1] + dz * r.t1[2];
  r.drift2[0] += dx * r.t2[0] + dy * r.t2[1] + dz * r.t2[2];
}

// ---- one world's step: forward with records, then the reverse sweep ----

// One world of a batch: where its slots, awake entries and rows start (rows' a, b and row[] are
// local to it).
struct AdjWorld {
  int32_t body0, nbodies, awake0, nawake, row0, nrows, solved;
  int32_t starts[BG_STARTS];
  double gravity[3];
};

// Every array the adjoint kernel reads or writes, in the caller's layout (bearing_gpu.h) where
// the caller gave it, per row or per slot otherwise.
struct AdjParams {
  // the step's input (read only)
  const double *in_p, *in_q, *in_v, *in_w, *in_tum, *in_ceil;
  const double *inv_mass, *inertia, *inv_inertia, *dims, *damping, *ang_damping, *grav_scale;
  const uint8_t *type, *shape, *framed, *awake;
  const int32_t* awake_list;
  const int32_t *row, *a, *b;
  const uint8_t* points;
  const double *normal, *t1, *t2, *friction, *restitution, *tolerance, *patch, *separation, *point, *shift;
  const double *in_ni, *in_ti1, *in_ti2, *in_ri1, *in_ri2, *in_si, *in_drift1, *in_drift2, *in_maxni, *in_relvel,
      *in_gap;
  // the forward pass's state
  double *p, *q, *v, *w, *tum, *ceil, *start, *startq, *invI;
  double *st, *pr, *drift1, *drift2;
  // records
  double *rec_row, *rec_body, *rec_rest;
  int64_t rows_total, bodies_total;
  // the adjoints of the step's results for each row's impulses (4, 1, 1, 1, 1, 1 per row)
  const double *seed_ni, *seed_ti1, *seed_ti2, *seed_ri1, *seed_ri2, *seed_si;
  // adjoints: bp .. bceil and bdrift seeded with those of the step's results, left holding those
  // of its inputs
  double *bp, *bq, *bv, *bw, *btum, *bceil, *bstart, *bstartq, *binvI;
  double *bst, *bpr, *bdrift1, *bdrift2, *bnormal, *bt1, *bt2, *bfriction, *brestitution, *bseparation, *bpoint;
  // the step
  double dt;
  int32_t substeps;
  SoftK soft;
  const AdjWorld* worlds;
  int32_t nworlds;
  int32_t* status;   // set to 1 where a replay did not fit its tape
};

AHD inline BodyConst body_const(const AdjParams& A, int s) {
  BodyConst b;
  b.dynamic = A.type[s] == BG_DYNAMIC;
  b.sphere_unframed = A.shape[s] == BG_SPHERE && A.framed[s] != 1;
  const double* I = A.inertia + 3 * s;
  b.lopsided = I[0] != I[1] || I[1] != I[2];
  b.gravity_scale = A.grav_scale[s];
  b.damping = A.damping[s];
  b.angular_damping = A.ang_damping[s];
  for (int k = 0; k < 3; k++) { b.inertia[k] = I[k]; b.inv_inertia[k] = A.inv_inertia[3 * s + k]; }
  return b;
}

// Row m (global) of world W as the forward pass sees it: pointers into the working columns.
AHD inline RowIO<double> row_io(const AdjParams& A, const AdjWorld& W, int m) {
  RowIO<double> r;
  const int a = W.body0 + A.a[m], b = W.body0 + A.b[m];
  r.va = A.v + 3 * a; r.wa = A.w + 3 * a; r.vb = A.v + 3 * b; r.wb = A.w + 3 * b;
  r.pa = A.p + 3 * a; r.pb = A.p + 3 * b; r.qa = A.q + 4 * a; r.qb = A.q + 4 * b;
  r.sa = A.start + 3 * a; r.sb = A.start + 3 * b;
  r.ia = A.invI + 6 * a; r.ib = A.invI + 6 * b;
  r.ima = A.inv_mass[a]; r.imb = A.inv_mass[b];
  r.st = A.st + RSTATE * static_cast<int64_t>(m);
  r.pr = A.pr + PREP * static_cast<int64_t>(m);
  r.normal = A.normal + 3 * m; r.t1 = A.t1 + 3 * m; r.t2 = A.t2 + 3 * m;
  r.friction = A.friction + m; r.restitution = A.restitution + m;
  r.separation = A.separation + 4 * m; r.point = A.point + 12 * m;
  r.drift1 = A.drift1 + m; r.drift2 = A.drift2 + m;
  r.tolerance = A.tolerance[m]; r.patch = A.patch[m]; r.shift = A.shift + 12 * m;
  r.count = A.points[m];
  r.shape_a = A.shape[a]; r.shape_b = A.shape[b];
  for (int k = 0; k < 3; k++) { r.dims_a[k] = A.dims[3 * a + k]; r.dims_b[k] = A.dims[3 * b + k]; }
  return r;
}

// A row's replay: every value it reads as a leaf on the calling thread's tape.
struct RowLeaves {
  TV va[3], wa[3], vb[3], wb[3], pa[3], pb[3], qa[4], qb[4], sa[3], sb[3], qa0[4], qb0[4], ia[6], ib[6];
  TV st[RSTATE], pr[PREP];
  TV normal[3], t1[3], t2[3], friction, restitution, separation[P], point[3 * P], drift1, drift2;
};

AHD inline void leaves(TV* dst, const double* src, int n) {
  for (int k = 0; k < n; k++) dst[k] = bgad::leaf(src[k]);
}

AHD inline RowIO<TV> leaf_io(RowLeaves& L, const RowIO<double>& r) {
  RowIO<TV> o;
  o.va = L.va; o.wa = L.wa; o.vb = L.vb; o.wb = L.wb; o.pa = L.pa; o.pb = L.pb; o.qa = L.qa; o.qb = L.qb;
  o.sa = L.sa; o.sb = L.sb; o.ia = L.ia; o.ib = L.ib; o.ima = r.ima; o.imb = r.imb; o.st = L.st; o.pr = L.pr;
  o.normal = L.normal; o.t1 = L.t1; o.t2 = L.t2; o.friction = &L.friction; o.restitution = &L.restitution;
  o.separation = L.separation; o.point = L.point; o.drift1 = &L.drift1; o.drift2 = &L.drift2;
  o.tolerance = r.tolerance; o.patch = r.patch; o.shift = r.shift; o.count = r.count;
  o.shape_a = r.shape_a; o.shape_b = r.shape_b;
  for (int k = 0; k < 3; k++) { o.dims_a[k] = r.dims_a[k]; o.dims_b[k] = r.dims_b[k]; }
  return o;
}

AHD inline void add_adjoints(double* dst, const bgad::Tape* t, const TV* src, int n) {
  for (int k = 0; k < n; k++) dst[k] += bgad::adjoint(t, src[k]);
}
AHD inline void set_adjoints(double* dst, const bgad::Tape* t, const TV* src, int n) {
  for (int k = 0; k < n; k++) dst[k] = bgad::adjoint(t, src[k]);
}

// The passes of a substep, in order.
enum Pass { WARM = 0, SOLVE = 1, RELAX = 2 };

template <class Lane>
AHD void run_pass(const AdjParams& A, const AdjWorld& W, const Lane& lane, int pass, int sub, double h) {
  const int kind = pass % 3;
  const int64_t base = static_cast<int64_t>(pass) * A.rows_total;
  auto one = [&](int m) {
    const RowIO<double> r = row_io(A, W, m);
    double* rec = A.rec_row + (base + m) * REC_ROW;
    for (int k = 0; k < RSTATE; k++) rec[k] = r.st[k];
    for (int c = 0; c < 3; c++) {
      rec[RSTATE + c] = r.va[c]; rec[RSTATE + 3 + c] = r.wa[c];
      rec[RSTATE + 6 + c] = r.vb[c]; rec[RSTATE + 9 + c] = r.wb[c];
    }
    if (kind == WARM) warm_row(r);
    else solve_row(r, h, kind == SOLVE, kind == SOLVE && sub > 0, A.soft);
  };
  for (int k = 0; k < bg::NCOLOURS; k++) {
    for (int m = W.starts[k] + lane.id; m < W.starts[k + 1]; m += lane.n) one(W.row0 + m);
    lane.sync();
  }
  if (lane.id == 0)
    for (int m = W.starts[bg::OVERFLOW_RUN]; m < W.starts[bg::OVERFLOW_RUN + 1]; m++) one(W.row0 + m);
  lane.sync();
}

// The world's solve stage from its input, leaving the records the reverse sweep replays from.
template <class Lane>
AHD void forward(const AdjParams& A, const AdjWorld& W, const Lane& lane) {
  const double h = A.dt / A.substeps;
  const bool touching = W.nrows > 0;
  for (int s = W.body0 + lane.id; s < W.body0 + W.nbodies; s += lane.n) {
    for (int k = 0; k < 3; k++) {
      A.p[3 * s + k] = A.in_p[3 * s + k]; A.v[3 * s + k] = A.in_v[3 * s + k]; A.w[3 * s + k] = A.in_w[3 * s + k];
      A.tum[3 * s + k] = A.in_tum[3 * s + k]; A.start[3 * s + k] = A.in_p[3 * s + k];
    }
    for (int k = 0; k < 4; k++) { A.q[4 * s + k] = A.in_q[4 * s + k]; A.startq[4 * s + k] = A.in_q[4 * s + k]; }
    for (int k = 0; k < 6; k++) A.invI[6 * s + k] = 0;
    A.ceil[s] = A.in_ceil[s];
  }
  for (int m = W.row0 + lane.id; m < W.row0 + W.nrows; m += lane.n) {
    double* st = A.st + RSTATE * static_cast<int64_t>(m);
    for (int k = 0; k < P; k++) {
      st[RS_NI + k] = A.in_ni[4 * m + k]; st[RS_MAXNI + k] = A.in_maxni[4 * m + k];
      st[RS_RELVEL + k] = A.in_relvel[4 * m + k]; st[RS_NOW + k] = 0;
    }
    st[RS_TI1] = A.in_ti1[m]; st[RS_TI2] = A.in_ti2[m]; st[RS_RI1] = A.in_ri1[m]; st[RS_RI2] = A.in_ri2[m];
    st[RS_SI] = A.in_si[m]; st[RS_GAP] = A.in_gap[m]; st[RS_SLID] = 0;
    A.drift1[m] = A.in_drift1[m]; A.drift2[m] = A.in_drift2[m];
  }
  lane.sync();
  // inertias and the start snapshot: src/contact.js:1302-1310, src/world.js:964-974
  for (int i = W.awake0 + lane.id; i < W.awake0 + W.nawake; i += lane.n) {
    const int s = W.body0 + A.awake_list[i];
    if (touching && A.type[s] == BG_DYNAMIC) inverse_inertia(A.q + 4 * s, A.inv_inertia + 3 * s, A.invI + 6 * s);
  }
  lane.sync();
  if (touching) {
    for (int m = lane.id; m < W.solved; m += lane.n) prepare_row(row_io(A, W, W.row0 + m));
    lane.sync();
  }
  for (int sub = 0; sub < A.substeps; sub++) {
    for (int i = W.awake0 + lane.id; i < W.awake0 + W.nawake; i += lane.n) {
      const int s = W.body0 + A.awake_list[i];
      double* rec = A.rec_body + (static_cast<int64_t>(sub) * A.bodies_total + s) * REC_BODY;
      for (int k = 0; k < 3; k++) { rec[RB_ACC + k] = A.v[3 * s + k]; rec[RB_ACC + 3 + k] = A.w[3 * s + k]; }
      accelerate(body_const(A, s), W.gravity, h, A.substeps, A.v + 3 * s, A.w + 3 * s);
    }
    lane.sync();
    if (touching) {
      run_pass(A, W, lane, 3 * sub + WARM, sub, h);
      run_pass(A, W, lane, 3 * sub + SOLVE, sub, h);
    }
    for (int i = W.awake0 + lane.id; i < W.awake0 + W.nawake; i += lane.n) {
      const int s = W.body0 + A.awake_list[i];
      double* rec = A.rec_body + (static_cast<int64_t>(sub) * A.bodies_total + s) * REC_BODY;
      for (int k = 0; k < 3; k++) {
        rec[RB_P + k] = A.p[3 * s + k]; rec[RB_V + k] = A.v[3 * s + k]; rec[RB_W + k] = A.w[3 * s + k];
        rec[RB_TUM + k] = A.tum[3 * s + k];
      }
      for (int k = 0; k < 4; k++) rec[RB_Q + k] = A.q[4 * s + k];
      rec[RB_CEIL] = A.ceil[s];
      move(body_const(A, s), h, A.p + 3 * s, A.q + 4 * s, A.v + 3 * s, A.w + 3 * s, A.tum + 3 * s, A.ceil + s);
    }
    lane.sync();
    if (touching) run_pass(A, W, lane, 3 * sub + RELAX, sub, h);
  }
  if (!touching) return;
  const double* g = W.gravity;
  const double gravity = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  if (lane.id == 0) {
    for (int f = 0; f < W.nrows; f++) {
      const int m = W.row0 + A.row[W.row0 + f];
      if (m >= W.row0 + W.solved) continue;
      const RowIO<double> r = row_io(A, W, m);
      if (!bouncy(r, gravity)) continue;
      double* rec = A.rec_rest + static_cast<int64_t>(m) * REC_REST;
      for (int c = 0; c < 3; c++) { rec[c] = r.va[c]; rec[3 + c] = r.wa[c]; rec[6 + c] = r.vb[c]; rec[9 + c] = r.wb[c]; }
      for (int k = 0; k < P; k++) rec[12 + k] = r.st[RS_NI + k];
      bounce_row(r, gravity);
    }
  }
  lane.sync();
  for (int m = lane.id; m < W.solved; m += lane.n) {
    const RowIO<double> r = row_io(A, W, W.row0 + m);
    const int a = W.body0 + A.a[W.row0 + m], b = W.body0 + A.b[W.row0 + m];
    slipped_row(r, A.startq + 4 * a, A.startq + 4 * b, A.awake[a] != 0, A.awake[b] != 0);
  }
  lane.sync();
}

// A body whose adjoints the sweep carries: one that moves (the others' values are constants).
AHD inline bool moving(const AdjParams& A, int s) { return A.type[s] == BG_DYNAMIC && A.inv_mass[s] != 0; }

// ---- the row passes' reverse, by hand ----
//
// The warm start and the solve / relax row are the bulk of the replays (three a row a substep), so
// their vector-Jacobian products are written out instead of recorded: each runs the row forward in
// double from its record, keeping what the reverse needs, then carries the adjoints back through
// the same steps in reverse order, with the branches the forward took (the block's active set, the
// clamps that held, whether the cone projected).  Only the cone's Newton rounds, a short loop whose
// length varies, are replayed on the thread's tape.  The derivatives are those the recorded replay
// gives (the same functions of the same branches), to rounding.

// b += M^T g for the symmetric 3x3 M stored xx xy xz yy yz zz, with M's adjoints: for w -= M l
// (sign -1) or w += M l (sign 1), given w's adjoint g, returns l's adjoint contribution in bl and
// adds to M's adjoint bm.
AHD inline void sym_apply_vjp(const double* M, const double* l, const double* g, double sign, double* bl, double* bm) {
  bl[0] += sign * (M[0] * g[0] + M[1] * g[1] + M[2] * g[2]);
  bl[1] += sign * (M[1] * g[0] + M[3] * g[1] + M[4] * g[2]);
  bl[2] += sign * (M[2] * g[0] + M[4] * g[1] + M[5] * g[2]);
  if (bm == nullptr) return;
  bm[0] += sign * g[0] * l[0];
  bm[1] += sign * (g[0] * l[1] + g[1] * l[0]);
  bm[2] += sign * (g[0] * l[2] + g[2] * l[0]);
  bm[3] += sign * g[1] * l[1];
  bm[4] += sign * (g[1] * l[2] + g[2] * l[1]);
  bm[5] += sign * g[2] * l[2];
}

AHD inline double dot3(const double* x, const double* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; }

// rotate(q, v, inverse)'s reverse (src/core/math.js:211-219): adds q's and v's adjoints, given the
// result's (g).  u = s q.xyz, t = 2 u x v, out = v + w t + u x t.
AHD inline void rotate_vjp(const double* q, const double* v, bool inverse, const double* g, double* bq, double* bv) {
  const double s = inverse ? -1 : 1;
  const double u[3] = {q[0] * s, q[1] * s, q[2] * s}, w = q[3];
  const double t[3] = {2 * (u[1] * v[2] - u[2] * v[1]), 2 * (u[2] * v[0] - u[0] * v[2]), 2 * (u[0] * v[1] - u[1] * v[0])};
  // out = v + w t + u x t
  double bt[3] = {w * g[0] + (g[1] * u[2] - g[2] * u[1]), w * g[1] + (g[2] * u[0] - g[0] * u[2]),
                  w * g[2] + (g[0] * u[1] - g[1] * u[0])};   // w g + g x u
  double bu[3] = {t[1] * g[2] - t[2] * g[1], t[2] * g[0] - t[0] * g[2], t[0] * g[1] - t[1] * g[0]};   // t x g
  const double bw = dot3(g, t);
  // t = 2 u x v
  bu[0] += 2 * (v[1] * bt[2] - v[2] * bt[1]); bu[1] += 2 * (v[2] * bt[0] - v[0] * bt[2]);
  bu[2] += 2 * (v[0] * bt[1] - v[1] * bt[0]);
  if (bv != nullptr) {
    bv[0] += g[0] + 2 * (bt[1] * u[2] - bt[2] * u[1]);
    bv[1] += g[1] + 2 * (bt[2] * u[0] - bt[0] * u[2]);
    bv[2] += g[2] + 2 * (bt[0] * u[1] - bt[1] * u[0]);
  }
  bq[0] += s * bu[0]; bq[1] += s * bu[1]; bq[2] += s * bu[2]; bq[3] += bw;
}

// Which argument Math.max (jsmax) returns: true for the first.
AHD inline bool jsmax_first(double a, double b) {
  if (a != a) return true;
  if (b != b) return false;
  if (a > b) return true;
  if (b > a) return false;
  if (a == 0 && b == 0) return !signbit(a);
  return true;
}

// The adjoints one row replay leaves: its bodies' velocities (v a, w a, v b, w b), its state, and
// additions to its prepared terms, its basis and materials, drift, poses and inertias.
struct RowBar {
  double v[12];                  // v a, w a, v b, w b
  double st[RSTATE];
  double pr[PREP];
  double n[3], t1[3], t2[3], mu, d1, d2;
  double pa[3], pb[3], qa[4], qb[4], sa[3], sb[3], ia[6], ib[6];
};

AHD inline void zero(double* x, int n) {
  for (int k = 0; k < n; k++) x[k] = 0;
}

// warmRows' reverse (src/contact.js:1616-1663).  The row moves its bodies by its impulses and
// leaves its state as it was: velocities' adjoints pass through, and the impulses, levers, basis
// and inertias gather theirs.  o: the row's record (state, velocities); b: in, the adjoints of the
// row's results (v, st); out, those of its input, plus the additions.
AHD inline void warm_row_vjp(const RowIO<double>& r, RowBar& b) {
  const double* st = r.st;
  const double* pr = r.pr;
  const double* n = r.normal;
  const double* t1 = r.t1;
  const double* t2 = r.t2;
  const double* ga = b.v + 3;   // w a's adjoint
  const double* gb = b.v + 9;   // w b's adjoint
  const double bP[3] = {-r.ima * b.v[0] + r.imb * b.v[6], -r.ima * b.v[1] + r.imb * b.v[7],
                        -r.ima * b.v[2] + r.imb * b.v[8]};
  for (int k = 0; k < r.count; k++) {
    const double* jac = &pr[PR_JAC + 12 * k];
    double* bj = &b.pr[PR_JAC + 12 * k];
    const double ln = st[RS_NI + k];
    for (int c = 0; c < 3; c++) {
      b.n[c] += bP[c] * ln;
      bj[6 + c] -= ga[c] * ln;
      bj[9 + c] += gb[c] * ln;
    }
    b.st[RS_NI + k] += dot3(bP, n) - dot3(ga, jac + 6) + dot3(gb, jac + 9);
  }
  {
    const double* fj = &pr[PR_FJ];
    double* bf = &b.pr[PR_FJ];
    const double l1 = st[RS_TI1], l2 = st[RS_TI2];
    for (int c = 0; c < 3; c++) {
      b.t1[c] += bP[c] * l1;
      b.t2[c] += bP[c] * l2;
      bf[6 + c] -= ga[c] * l1; bf[18 + c] -= ga[c] * l2;
      bf[9 + c] += gb[c] * l1; bf[21 + c] += gb[c] * l2;
    }
    b.st[RS_TI1] += dot3(bP, t1) - dot3(ga, fj + 6) + dot3(gb, fj + 9);
    b.st[RS_TI2] += dot3(bP, t2) - dot3(ga, fj + 18) + dot3(gb, fj + 21);
  }
  {
    const double r1 = st[RS_RI1], r2 = st[RS_RI2], sp = st[RS_SI];
    const double L[3] = {t1[0] * r1 + t2[0] * r2 + n[0] * sp, t1[1] * r1 + t2[1] * r2 + n[1] * sp,
                         t1[2] * r1 + t2[2] * r2 + n[2] * sp};
    double bL[3] = {0, 0, 0};
    sym_apply_vjp(r.ia, L, ga, -1, bL, b.ia);
    sym_apply_vjp(r.ib, L, gb, 1, bL, b.ib);
    for (int c = 0; c < 3; c++) {
      b.t1[c] += bL[c] * r1;
      b.t2[c] += bL[c] * r2;
      b.n[c] += bL[c] * sp;
    }
    b.st[RS_RI1] += dot3(bL, t1);
    b.st[RS_RI2] += dot3(bL, t2);
    b.st[RS_SI] += dot3(bL, n);
  }
}

// solveRows' reverse for one row (src/contact.js:1805-2090): the forward in double from the row's
// record (r: its state and velocities before the pass, poses, prepared terms), then the reverse,
// block by block from the last: twist, rolling, friction, the normal impulses (the block LCP on
// its final active set, or the per-point update), the targets and the separations.  b: in, the
// adjoints of the row's results; out, those of its input, plus the additions.  Returns false if
// the cone's replay did not fit the tape.
AHD inline bool solve_row_vjp(const RowIO<double>& r, double h, bool bias, bool known, const SoftK& soft, RowBar& b) {
  const double* st = r.st;
  const double* pr = r.pr;
  const double* n = r.normal;
  const double* t1 = r.t1;
  const double* t2 = r.t2;
  const double inv = 1 / h;
  const double springy = soft.impulseScale / soft.massScale + COMPLIANCE;
  const double maxBias = r.tolerance * inv;
  const int count = r.count;
  const double ima = r.ima, imb = r.imb;
  // ---- forward, keeping what the reverse reads ----
  double dx3[3] = {0, 0, 0}, na[3] = {0, 0, 0}, nb[3] = {0, 0, 0};
  double sep[P], target[P], ms[P], is[P], give[P];
  bool tfirst[P];   // the bias clamp returned its first argument
  if (!known) {
    for (int c = 0; c < 3; c++) dx3[c] = (r.pb[c] - r.sb[c]) - (r.pa[c] - r.sa[c]);
    const double dn = dx3[0] * n[0] + dx3[1] * n[1] + dx3[2] * n[2];
    rotate(r.qa, n[0], n[1], n[2], true, na);
    rotate(r.qb, n[0], n[1], n[2], true, nb);
    for (int k = 0; k < count; k++) {
      const int i3 = 3 * k;
      sep[k] = dn + (pr[PR_LB + i3] * nb[0] + pr[PR_LB + i3 + 1] * nb[1] + pr[PR_LB + i3 + 2] * nb[2]) -
               (pr[PR_LA + i3] * na[0] + pr[PR_LA + i3 + 1] * na[1] + pr[PR_LA + i3 + 2] * na[2]) + pr[PR_ADJ + k];
    }
  } else {
    for (int k = 0; k < count; k++) sep[k] = st[RS_NOW + k];
  }
  int least_k = -1;
  {
    double least = INFINITY;
    for (int k = 0; k < count; k++)
      if (sep[k] < least) { least = sep[k]; least_k = k; }
  }
  for (int k = 0; k < count; k++) {
    const double sv = sep[k];
    tfirst[k] = false;
    if (sv > 0) {
      target[k] = sv * inv; ms[k] = 1; is[k] = 0; give[k] = COMPLIANCE;
    } else if (bias) {
      tfirst[k] = jsmax_first(soft.biasRate * sv, -maxBias);
      target[k] = jsmax(soft.biasRate * sv, -maxBias);
      ms[k] = soft.massScale; is[k] = soft.impulseScale; give[k] = springy;
    } else {
      target[k] = 0; ms[k] = 1; is[k] = 0; give[k] = COMPLIANCE;
    }
  }
  const double* K = &pr[PR_K];
  double V[12];
  for (int c = 0; c < 3; c++) { V[c] = r.va[c]; V[3 + c] = r.wa[c]; V[6 + c] = r.vb[c]; V[9 + c] = r.wb[c]; }
  const double V0c[12] = {V[0], V[1], V[2], V[3], V[4], V[5], V[6], V[7], V[8], V[9], V[10], V[11]};
  double closing[P], solved[P], nraw[P];
  const bool block = !(count == 1 || !(K[0] > 0));
  int set = 0;
  double wanted[P];
  for (int k = 0; k < count; k++) {
    const double* jac = &pr[PR_JAC + 12 * k];
    closing[k] = (V[6] - V[0]) * n[0] + (V[7] - V[1]) * n[1] + (V[8] - V[2]) * n[2] + V[9] * jac[3] +
                 V[10] * jac[4] + V[11] * jac[5] - V[3] * jac[0] - V[4] * jac[1] - V[5] * jac[2];
  }
  if (!block) {
    for (int k = 0; k < count; k++) {
      const double old = st[RS_NI + k];
      nraw[k] = old - pr[PR_NM + k] * ms[k] * (closing[k] + target[k]) - is[k] * old;
      solved[k] = nraw[k] < 0 ? 0 : nraw[k];
    }
  } else {
    for (int k = 0; k < count; k++) {
      double rr = -closing[k] - target[k];
      for (int l = 0; l < count; l++) rr += K[P * k + l] * st[RS_NI + l];
      wanted[k] = rr;
      if (rr > 0) set |= 1 << k;
    }
    for (int round = 0;; round++) {
      pushes(K, count, set, give, wanted, solved);
      int flip = -1;
      for (int k = 0; k < count && flip < 0; k++) {
        if (set >> k & 1) {
          if (solved[k] < 0) flip = k;
        } else {
          double rr = -wanted[k];
          for (int l = 0; l < count; l++) rr += K[P * k + l] * solved[l];
          if (rr < 0) flip = k;
        }
      }
      if (flip < 0 || round == 1 << count) break;
      set ^= 1 << flip;
    }
  }
  double next[P], d[P];
  bool rvset[P], mxset[P];
  double pressed = 0, twisted = 0;
  for (int k = 0; k < count; k++) {
    const double* jac = &pr[PR_JAC + 12 * k];
    next[k] = solved[k] > 0 ? solved[k] : 0;
    d[k] = next[k] - st[RS_NI + k];
    rvset[k] = d[k] > 0 && st[RS_MAXNI + k] == 0;
    mxset[k] = d[k] > st[RS_MAXNI + k];
    for (int c = 0; c < 3; c++) {
      V[c] -= ima * (n[c] * d[k]);
      V[6 + c] += imb * (n[c] * d[k]);
      V[3 + c] -= jac[6 + c] * d[k];
      V[9 + c] += jac[9 + c] * d[k];
    }
  }
  for (int k = 0; k < count; k++) {
    pressed += next[k];
    twisted += pr[PR_LEV + k] * next[k];
  }
  // friction
  const double V1[12] = {V[0], V[1], V[2], V[3], V[4], V[5], V[6], V[7], V[8], V[9], V[10], V[11]};
  const double* fj = &pr[PR_FJ];
  const double* gj = fj + 12;
  const double* tm = &pr[PR_TM];
  const double mu = r.friction[0];
  const double dv[3] = {V[6] - V[0], V[7] - V[1], V[8] - V[2]};
  double v1 = dot3(dv, t1) + V[9] * fj[3] + V[10] * fj[4] + V[11] * fj[5] - V[3] * fj[0] - V[4] * fj[1] - V[5] * fj[2];
  double v2 = dot3(dv, t2) + V[9] * gj[3] + V[10] * gj[4] + V[11] * gj[5] - V[3] * gj[0] - V[4] * gj[1] - V[5] * gj[2];
  const double s1d = r.drift1[0], s2d = r.drift2[0];
  const bool drifts = bias && (s1d != 0 || s2d != 0);
  double b1r = 0, b2r = 0, bsc = 1, bq = 0;
  bool bscaled = false;
  if (drifts) {
    b1r = soft.biasRate * s1d; b2r = soft.biasRate * s2d;
    const double bb = b1r * b1r + b2r * b2r;
    double b1 = b1r, b2 = b2r;
    if (bb > maxBias * maxBias) {
      bscaled = true;
      bq = sqrt(bb);
      bsc = maxBias / bq;
      b1 *= bsc; b2 *= bsc;
    }
    v1 += b1; v2 += b2;
  }
  const double o1 = st[RS_TI1], o2 = st[RS_TI2];
  const double n1 = o1 - (tm[0] * v1 + tm[1] * v2), n2 = o2 - (tm[1] * v1 + tm[2] * v2);
  const double limit = mu * pressed, l2 = n1 * n1 + n2 * n2;
  const bool projected = l2 > limit * limit;
  double n1f = n1, n2f = n2;
  if (projected) cone(limit, tm[0], tm[1], tm[2], n1f, n2f);
  const double dd1 = n1f - o1, dd2 = n2f - o2;
  {
    const double px = t1[0] * dd1 + t2[0] * dd2, py = t1[1] * dd1 + t2[1] * dd2, pz = t1[2] * dd1 + t2[2] * dd2;
    V[0] -= ima * px; V[1] -= ima * py; V[2] -= ima * pz;
    V[6] += imb * px; V[7] += imb * py; V[8] += imb * pz;
    for (int c = 0; c < 3; c++) {
      V[3 + c] -= fj[6 + c] * dd1 + gj[6 + c] * dd2;
      V[9 + c] += fj[9 + c] * dd1 + gj[9 + c] * dd2;
    }
  }
  // rolling
  const bool rolls = count <= 2;
  double most = 0, u[3] = {0, 0, 0}, p1 = 0, p2 = 0, n1r0 = 0, n2r0 = 0, rq = 0, rsc = 1, dr1 = 0, dr2 = 0;
  bool rscaled = false;
  double Lr[3] = {0, 0, 0};
  if (rolls) {
    most = r.patch * pressed;
    for (int c = 0; c < 3; c++) u[c] = V[9 + c] - V[3 + c];
    p1 = dot3(u, t1); p2 = dot3(u, t2);
    n1r0 = st[RS_RI1] - pr[PR_RM1] * p1;
    n2r0 = st[RS_RI2] - pr[PR_RM2] * p2;
    const double l2r = n1r0 * n1r0 + n2r0 * n2r0;
    double n1r = n1r0, n2r = n2r0;
    if (l2r > most * most) {
      rscaled = true;
      rq = sqrt(l2r);
      rsc = most / rq;
      n1r *= rsc; n2r *= rsc;
    }
    dr1 = n1r - st[RS_RI1]; dr2 = n2r - st[RS_RI2];
    for (int c = 0; c < 3; c++) Lr[c] = t1[c] * dr1 + t2[c] * dr2;
    double wa[3] = {V[3], V[4], V[5]}, wb[3] = {V[9], V[10], V[11]};
    const double* ia = r.ia;
    const double* ib = r.ib;
    wa[0] -= ia[0] * Lr[0] + ia[1] * Lr[1] + ia[2] * Lr[2];
    wa[1] -= ia[1] * Lr[0] + ia[3] * Lr[1] + ia[4] * Lr[2];
    wa[2] -= ia[2] * Lr[0] + ia[4] * Lr[1] + ia[5] * Lr[2];
    wb[0] += ib[0] * Lr[0] + ib[1] * Lr[1] + ib[2] * Lr[2];
    wb[1] += ib[1] * Lr[0] + ib[3] * Lr[1] + ib[4] * Lr[2];
    wb[2] += ib[2] * Lr[0] + ib[4] * Lr[1] + ib[5] * Lr[2];
    for (int c = 0; c < 3; c++) { V[3 + c] = wa[c]; V[9 + c] = wb[c]; }
  }
  // twist
  const double limit_s = count == 1 ? SPIN_DISC * mu * r.patch * pressed : mu * twisted;
  const double s0 = st[RS_SI];
  const double us = (V[9] - V[3]) * n[0] + (V[10] - V[4]) * n[1] + (V[11] - V[5]) * n[2];
  const double svr = s0 - pr[PR_SM] * us;
  const int sclamp = svr > limit_s ? 1 : svr < -limit_s ? -1 : 0;
  const double sv = sclamp == 1 ? limit_s : sclamp == -1 ? -limit_s : svr;
  const double ds = sv - s0;
  const double Ls[3] = {n[0] * ds, n[1] * ds, n[2] * ds};
  const double V3[12] = {V[0], V[1], V[2], V[3], V[4], V[5], V[6], V[7], V[8], V[9], V[10], V[11]};

  // ---- reverse ----
  const double b_gap = b.st[RS_GAP];   // gap is the least separation; its input is overwritten
  double* g = b.v;   // the adjoint of the velocities, from the row's results back to its input
  double b_pressed = 0, b_twisted = 0, b_mu = 0;
  // twist: w a -= Ia Ls, w b += Ib Ls; si = sv
  {
    double bL[3] = {0, 0, 0};
    sym_apply_vjp(r.ia, Ls, g + 3, -1, bL, b.ia);
    sym_apply_vjp(r.ib, Ls, g + 9, 1, bL, b.ib);
    const double b_ds = dot3(bL, n);
    for (int c = 0; c < 3; c++) b.n[c] += bL[c] * ds;
    const double b_sv = b.st[RS_SI] + b_ds;
    double b_s0 = -b_ds, b_svr = 0, b_limit = 0;
    if (sclamp == 1) b_limit = b_sv;
    else if (sclamp == -1) b_limit = -b_sv;
    else b_svr = b_sv;
    b_s0 += b_svr;
    b.pr[PR_SM] += -b_svr * us;
    const double b_us = -b_svr * pr[PR_SM];
    for (int c = 0; c < 3; c++) {
      g[9 + c] += b_us * n[c];
      g[3 + c] -= b_us * n[c];
      b.n[c] += b_us * (V3[9 + c] - V3[3 + c]);
    }
    if (count == 1) {
      b_mu += b_limit * SPIN_DISC * r.patch * pressed;
      b_pressed += b_limit * SPIN_DISC * mu * r.patch;
    } else {
      b_mu += b_limit * twisted;
      b_twisted += b_limit * mu;
    }
    b.st[RS_SI] = b_s0;
  }
  // rolling
  if (rolls) {
    double bL[3] = {0, 0, 0};
    sym_apply_vjp(r.ia, Lr, g + 3, -1, bL, b.ia);
    sym_apply_vjp(r.ib, Lr, g + 9, 1, bL, b.ib);
    for (int c = 0; c < 3; c++) { b.t1[c] += bL[c] * dr1; b.t2[c] += bL[c] * dr2; }
    const double b_dr1 = dot3(bL, t1), b_dr2 = dot3(bL, t2);
    const double b_n1r = b.st[RS_RI1] + b_dr1, b_n2r = b.st[RS_RI2] + b_dr2;
    double b_r1 = -b_dr1, b_r2 = -b_dr2;
    double b_n1r0 = b_n1r, b_n2r0 = b_n2r;
    if (rscaled) {
      b_n1r0 = b_n1r * rsc; b_n2r0 = b_n2r * rsc;
      const double b_sc = b_n1r * n1r0 + b_n2r * n2r0;
      const double b_most = b_sc / rq;
      const double b_q = -b_sc * most / (rq * rq);
      const double b_l2r = b_q * 0.5 / rq;
      b_n1r0 += 2 * n1r0 * b_l2r; b_n2r0 += 2 * n2r0 * b_l2r;
      b_pressed += b_most * r.patch;
    }
    b_r1 += b_n1r0; b_r2 += b_n2r0;
    b.pr[PR_RM1] += -b_n1r0 * p1; b.pr[PR_RM2] += -b_n2r0 * p2;
    const double b_p1 = -b_n1r0 * pr[PR_RM1], b_p2 = -b_n2r0 * pr[PR_RM2];
    for (int c = 0; c < 3; c++) {
      const double bu = b_p1 * t1[c] + b_p2 * t2[c];
      b.t1[c] += b_p1 * u[c]; b.t2[c] += b_p2 * u[c];
      g[9 + c] += bu; g[3 + c] -= bu;
    }
    b.st[RS_RI1] = b_r1; b.st[RS_RI2] = b_r2;
  }
  // friction
  {
    const double bP[3] = {-ima * g[0] + imb * g[6], -ima * g[1] + imb * g[7], -ima * g[2] + imb * g[8]};
    double* bf = &b.pr[PR_FJ];
    double* bg = bf + 12;
    double b_dd1 = dot3(bP, t1), b_dd2 = dot3(bP, t2);
    for (int c = 0; c < 3; c++) {
      b.t1[c] += bP[c] * dd1; b.t2[c] += bP[c] * dd2;
      b_dd1 += -g[3 + c] * fj[6 + c] + g[9 + c] * fj[9 + c];
      b_dd2 += -g[3 + c] * gj[6 + c] + g[9 + c] * gj[9 + c];
      bf[6 + c] -= g[3 + c] * dd1; bg[6 + c] -= g[3 + c] * dd2;
      bf[9 + c] += g[9 + c] * dd1; bg[9 + c] += g[9 + c] * dd2;
    }
    const double b_n1f = b.st[RS_TI1] + b_dd1, b_n2f = b.st[RS_TI2] + b_dd2;
    double b_o1 = -b_dd1, b_o2 = -b_dd2;
    double b_n1 = b_n1f, b_n2 = b_n2f, b_limit = 0, btm[3] = {0, 0, 0};
    if (projected) {
      // the cone's rounds, replayed on the tape
      bgad::Tape* t = bgad::thread_tape();
      bgad::reset(t);
      const TV ln1 = bgad::leaf(n1), ln2 = bgad::leaf(n2), llim = bgad::leaf(limit);
      const TV lma = bgad::leaf(tm[0]), lmb = bgad::leaf(tm[1]), lmc = bgad::leaf(tm[2]);
      TV x = ln1, y = ln2;
      cone(llim, lma, lmb, lmc, x, y);
      if (t->overflow) return false;
      bgad::clear_adjoints(t);
      bgad::seed(t, x, b_n1f);
      bgad::seed(t, y, b_n2f);
      bgad::sweep(t);
      b_n1 = bgad::adjoint(t, ln1); b_n2 = bgad::adjoint(t, ln2); b_limit = bgad::adjoint(t, llim);
      btm[0] = bgad::adjoint(t, lma); btm[1] = bgad::adjoint(t, lmb); btm[2] = bgad::adjoint(t, lmc);
    }
    b_mu += b_limit * pressed;
    b_pressed += b_limit * mu;
    // n1 = o1 - (tm0 v1 + tm1 v2), n2 = o2 - (tm1 v1 + tm2 v2)
    b_o1 += b_n1; b_o2 += b_n2;
    btm[0] += -b_n1 * v1; btm[1] += -b_n1 * v2 - b_n2 * v1; btm[2] += -b_n2 * v2;
    const double b_v1 = -b_n1 * tm[0] - b_n2 * tm[1], b_v2 = -b_n1 * tm[1] - b_n2 * tm[2];
    double* bt = &b.pr[PR_TM];
    bt[0] += btm[0]; bt[1] += btm[1]; bt[2] += btm[2];
    if (drifts) {
      double b_b1r = b_v1, b_b2r = b_v2;
      if (bscaled) {
        b_b1r = b_v1 * bsc; b_b2r = b_v2 * bsc;
        const double b_sc = b_v1 * b1r + b_v2 * b2r;
        const double b_q = -b_sc * maxBias / (bq * bq);
        const double b_bb = b_q * 0.5 / bq;
        b_b1r += 2 * b1r * b_bb; b_b2r += 2 * b2r * b_bb;
      }
      b.d1 += soft.biasRate * b_b1r;
      b.d2 += soft.biasRate * b_b2r;
    }
    // v1 = dv . t1 + wb . fj[3..5] - wa . fj[0..2]; v2 the same with t2 and g
    const double dv1[3] = {V1[6] - V1[0], V1[7] - V1[1], V1[8] - V1[2]};
    for (int c = 0; c < 3; c++) {
      const double bdv = b_v1 * t1[c] + b_v2 * t2[c];
      b.t1[c] += b_v1 * dv1[c]; b.t2[c] += b_v2 * dv1[c];
      g[6 + c] += bdv; g[c] -= bdv;
      g[9 + c] += b_v1 * fj[3 + c] + b_v2 * gj[3 + c];
      g[3 + c] -= b_v1 * fj[c] + b_v2 * gj[c];
      bf[3 + c] += b_v1 * V1[9 + c]; bg[3 + c] += b_v2 * V1[9 + c];
      bf[c] -= b_v1 * V1[3 + c]; bg[c] -= b_v2 * V1[3 + c];
    }
    b.st[RS_TI1] = b_o1; b.st[RS_TI2] = b_o2;
  }
  b.mu += b_mu;
  // the normal impulses
  double b_next[P], b_closing[P], b_target[P], b_old[P];
  for (int k = 0; k < count; k++) {
    b_next[k] = b.st[RS_NI + k] + b_pressed + pr[PR_LEV + k] * b_twisted;
    b.pr[PR_LEV + k] += b_twisted * next[k];
    b_closing[k] = 0; b_target[k] = 0; b_old[k] = 0;
  }
  {
    const double bP[3] = {-ima * g[0] + imb * g[6], -ima * g[1] + imb * g[7], -ima * g[2] + imb * g[8]};
    for (int k = 0; k < count; k++) {
      const double* jac = &pr[PR_JAC + 12 * k];
      double* bj = &b.pr[PR_JAC + 12 * k];
      double b_d = dot3(bP, n) - dot3(g + 3, jac + 6) + dot3(g + 9, jac + 9);
      for (int c = 0; c < 3; c++) {
        b.n[c] += bP[c] * d[k];
        bj[6 + c] -= g[3 + c] * d[k];
        bj[9 + c] += g[9 + c] * d[k];
      }
      if (mxset[k]) { b_d += b.st[RS_MAXNI + k]; b.st[RS_MAXNI + k] = 0; }
      if (rvset[k]) { b_closing[k] += b.st[RS_RELVEL + k]; b.st[RS_RELVEL + k] = 0; }
      b_next[k] += b_d;
      b_old[k] -= b_d;
    }
  }
  double b_solved[P];
  for (int k = 0; k < count; k++) b_solved[k] = solved[k] > 0 ? b_next[k] : 0;
  if (!block) {
    for (int k = 0; k < count; k++) {
      const double b_raw = nraw[k] < 0 ? 0 : b_solved[k];
      b_old[k] += b_raw * (1 - is[k]);
      b.pr[PR_NM + k] += -b_raw * ms[k] * (closing[k] + target[k]);
      const double c = -b_raw * pr[PR_NM + k] * ms[k];
      b_closing[k] += c;
      b_target[k] += c;
    }
  } else {
    // solved = A^-1 wanted on the final set S (A = K_SS, its diagonal times 1 + give): A is
    // symmetric, so wanted's adjoint is A^-1 times solved's (the same solve), and A's is minus
    // the outer product of the two
    double bw[P];
    pushes(K, count, set, give, b_solved, bw);
    double* bK = &b.pr[PR_K];
    for (int k = 0; k < count; k++) {
      if (!(set >> k & 1)) continue;
      for (int l = 0; l < count; l++) {
        if (!(set >> l & 1)) continue;
        const double scale = k == l ? 1 + give[k] : 1.0;
        bK[P * k + l] += -bw[k] * solved[l] * scale;
      }
      // wanted_k = -closing_k - target_k + sum_l K_kl old_l
      b_closing[k] -= bw[k];
      b_target[k] -= bw[k];
      for (int l = 0; l < count; l++) {
        bK[P * k + l] += bw[k] * st[RS_NI + l];
        b_old[l] += bw[k] * K[P * k + l];
      }
    }
  }
  for (int k = 0; k < count; k++) b.st[RS_NI + k] = b_old[k];
  // closing_k = (vb - va) . n + wb . jac[3..5] - wa . jac[0..2], at the pass's start
  for (int k = 0; k < count; k++) {
    const double* jac = &pr[PR_JAC + 12 * k];
    double* bj = &b.pr[PR_JAC + 12 * k];
    const double bc = b_closing[k];
    for (int c = 0; c < 3; c++) {
      g[6 + c] += bc * n[c]; g[c] -= bc * n[c];
      b.n[c] += bc * (V0c[6 + c] - V0c[c]);
      g[9 + c] += bc * jac[3 + c]; bj[3 + c] += bc * V0c[9 + c];
      g[3 + c] -= bc * jac[c]; bj[c] -= bc * V0c[3 + c];
    }
  }
  // targets and separations
  double b_sep[P];
  for (int k = 0; k < count; k++) {
    b_sep[k] = 0;
    if (sep[k] > 0) b_sep[k] = b_target[k] * inv;
    else if (bias && tfirst[k]) b_sep[k] = b_target[k] * soft.biasRate;
  }
  if (least_k >= 0) b_sep[least_k] += b_gap;
  b.st[RS_GAP] = 0;
  b.st[RS_SLID] = 0;
  if (known) {
    for (int k = 0; k < count; k++) b.st[RS_NOW + k] += b_sep[k];
  } else {
    for (int k = 0; k < count; k++)
      if (!bias) { b_sep[k] += b.st[RS_NOW + k]; b.st[RS_NOW + k] = 0; }
    double b_dn = 0, b_na[3] = {0, 0, 0}, b_nb[3] = {0, 0, 0};
    for (int k = 0; k < count; k++) {
      const int i3 = 3 * k;
      b_dn += b_sep[k];
      for (int c = 0; c < 3; c++) {
        b.pr[PR_LB + i3 + c] += b_sep[k] * nb[c];
        b_nb[c] += b_sep[k] * pr[PR_LB + i3 + c];
        b.pr[PR_LA + i3 + c] -= b_sep[k] * na[c];
        b_na[c] -= b_sep[k] * pr[PR_LA + i3 + c];
      }
      b.pr[PR_ADJ + k] += b_sep[k];
    }
    for (int c = 0; c < 3; c++) {
      const double bd = b_dn * n[c];
      b.n[c] += b_dn * dx3[c];
      b.pb[c] += bd; b.sb[c] -= bd; b.pa[c] -= bd; b.sa[c] += bd;
    }
    rotate_vjp(r.qa, n, true, b_na, b.qa, b.n);
    rotate_vjp(r.qb, n, true, b_nb, b.qb, b.n);
  }
  return true;
}

// Replays row m of a pass (kind WARM / SOLVE / RELAX, substep sub) from its record.  The poses it
// reads (relax, and the first substep's solve) are those after the substep's move: the next
// substep's record before its move, or the step's last.
template <class Lane>
AHD void replay_pass_row(const AdjParams& A, const AdjWorld& W, int m, int pass, int sub, double h) {
  const int kind = pass % 3;
  RowIO<double> r = row_io(A, W, m);
  const int a = W.body0 + A.a[m], b = W.body0 + A.b[m];
  const double* rec = A.rec_row + (static_cast<int64_t>(pass) * A.rows_total + m) * REC_ROW;
  // the row's input as the record holds it: its state and its bodies' velocities before the pass
  double st[RSTATE], va[3], wa[3], vb[3], wb[3];
  for (int k = 0; k < RSTATE; k++) st[k] = rec[k];
  for (int c = 0; c < 3; c++) {
    va[c] = rec[RSTATE + c]; wa[c] = rec[RSTATE + 3 + c]; vb[c] = rec[RSTATE + 6 + c]; wb[c] = rec[RSTATE + 9 + c];
  }
  r.st = st; r.va = va; r.wa = wa; r.vb = vb; r.wb = wb;
  double drift1 = A.in_drift1[m], drift2 = A.in_drift2[m];   // the step's input: only slipped() moves them
  r.drift1 = &drift1; r.drift2 = &drift2;
  const bool reads_pose = kind == RELAX || (kind == SOLVE && sub == 0);
  // during relax(sub): after move(sub); during solve(0): before move(0)
  const int at = kind == RELAX ? sub + 1 : sub;
  if (at < A.substeps) {
    const double* ra = A.rec_body + (static_cast<int64_t>(at) * A.bodies_total + a) * REC_BODY;
    const double* rb = A.rec_body + (static_cast<int64_t>(at) * A.bodies_total + b) * REC_BODY;
    r.pa = A.awake[a] ? ra + RB_P : A.p + 3 * a; r.qa = A.awake[a] ? ra + RB_Q : A.q + 4 * a;
    r.pb = A.awake[b] ? rb + RB_P : A.p + 3 * b; r.qb = A.awake[b] ? rb + RB_Q : A.q + 4 * b;
  } else {
    r.pa = A.p + 3 * a; r.qa = A.q + 4 * a; r.pb = A.p + 3 * b; r.qb = A.q + 4 * b;
  }
  const bool ma = moving(A, a), mb = moving(A, b);
  RowBar B;
  zero(B.v, 12); zero(B.pr, PREP); zero(B.n, 3); zero(B.t1, 3); zero(B.t2, 3); B.mu = 0; B.d1 = 0; B.d2 = 0;
  zero(B.pa, 3); zero(B.pb, 3); zero(B.qa, 4); zero(B.qb, 4); zero(B.sa, 3); zero(B.sb, 3); zero(B.ia, 6); zero(B.ib, 6);
  for (int c = 0; c < 3; c++) {
    if (ma) { B.v[c] = A.bv[3 * a + c]; B.v[3 + c] = A.bw[3 * a + c]; }
    if (mb) { B.v[6 + c] = A.bv[3 * b + c]; B.v[9 + c] = A.bw[3 * b + c]; }
  }
  double* bst = A.bst + RSTATE * static_cast<int64_t>(m);
  for (int k = 0; k < RSTATE; k++) B.st[k] = bst[k];
  if (kind == WARM) {
    warm_row_vjp(r, B);
  } else if (!solve_row_vjp(r, h, kind == SOLVE, kind == SOLVE && sub > 0, A.soft, B)) {
    *A.status = 1;
    return;
  }
  // results: the adjoints of the state and velocities it read replace those of what it wrote;
  // everything else it read adds to its adjoint
  for (int k = 0; k < RSTATE; k++) bst[k] = B.st[k];
  for (int c = 0; c < 3; c++) {
    if (ma) { A.bv[3 * a + c] = B.v[c]; A.bw[3 * a + c] = B.v[3 + c]; }
    if (mb) { A.bv[3 * b + c] = B.v[6 + c]; A.bw[3 * b + c] = B.v[9 + c]; }
  }
  if (reads_pose) {
    if (ma) {
      for (int c = 0; c < 3; c++) { A.bp[3 * a + c] += B.pa[c]; A.bstart[3 * a + c] += B.sa[c]; }
      for (int c = 0; c < 4; c++) A.bq[4 * a + c] += B.qa[c];
    }
    if (mb) {
      for (int c = 0; c < 3; c++) { A.bp[3 * b + c] += B.pb[c]; A.bstart[3 * b + c] += B.sb[c]; }
      for (int c = 0; c < 4; c++) A.bq[4 * b + c] += B.qb[c];
    }
  }
  if (ma) for (int c = 0; c < 6; c++) A.binvI[6 * a + c] += B.ia[c];
  if (mb) for (int c = 0; c < 6; c++) A.binvI[6 * b + c] += B.ib[c];
  // the prepared terms the pass read, and only those (the rest of B.pr is 0)
  double* bpr = A.bpr + PREP * static_cast<int64_t>(m);
  auto flush = [&](int from, int to) {
    for (int k = from; k < to; k++) bpr[k] += B.pr[k];
  };
  const int count = r.count;
  if (kind == WARM) {
    for (int k = 0; k < count; k++) flush(PR_JAC + 12 * k + 6, PR_JAC + 12 * k + 12);
    flush(PR_FJ + 6, PR_FJ + 12);
    flush(PR_FJ + 18, PR_FJ + 24);
  } else {
    if (reads_pose) {
      flush(PR_LA, PR_LA + 3 * count);
      flush(PR_LB, PR_LB + 3 * count);
      flush(PR_ADJ, PR_ADJ + count);
    }
    flush(PR_NM, PR_NM + count);
    flush(PR_JAC, PR_JAC + 12 * count);
    for (int k = 0; k < count; k++) flush(PR_K + P * k, PR_K + P * k + count);
    flush(PR_LEV, PR_LEV + count);
    flush(PR_FJ, PR_TM + 3);   // FJ (24) then TM (3)
    if (count <= 2) flush(PR_RM1, PR_RM2 + 1);
    flush(PR_SM, PR_SM + 1);
  }
  for (int c = 0; c < 3; c++) {
    A.bnormal[3 * m + c] += B.n[c]; A.bt1[3 * m + c] += B.t1[c]; A.bt2[3 * m + c] += B.t2[c];
  }
  A.bfriction[m] += B.mu;
  A.bdrift1[m] += B.d1;
  A.bdrift2[m] += B.d2;
}

template <class Lane>
AHD void reverse_pass(const AdjParams& A, const AdjWorld& W, const Lane& lane, int pass, int sub, double h) {
  if (lane.id == 0)
    for (int m = W.starts[bg::OVERFLOW_RUN + 1] - 1; m >= W.starts[bg::OVERFLOW_RUN]; m--)
      replay_pass_row<Lane>(A, W, W.row0 + m, pass, sub, h);
  lane.sync();
  for (int k = bg::NCOLOURS - 1; k >= 0; k--) {
    for (int m = W.starts[k] + lane.id; m < W.starts[k + 1]; m += lane.n) replay_pass_row<Lane>(A, W, W.row0 + m, pass, sub, h);
    lane.sync();
  }
}

// The reverse sweep of the world's step, after forward(): turns the adjoints of the step's results
// (seeded in bp .. bceil and bdrift, and the impulses' from seed_*) into those of its input.
template <class Lane>
AHD void reverse(const AdjParams& A, const AdjWorld& W, const Lane& lane) {
  const double h = A.dt / A.substeps;
  const bool touching = W.nrows > 0;
  for (int s = W.body0 + lane.id; s < W.body0 + W.nbodies; s += lane.n) {
    for (int k = 0; k < 3; k++) A.bstart[3 * s + k] = 0;
    for (int k = 0; k < 4; k++) A.bstartq[4 * s + k] = 0;
    for (int k = 0; k < 6; k++) A.binvI[6 * s + k] = 0;
    if (moving(A, s)) continue;
    // A body that does not move (static, kinematic) is a constant of the step: no adjoints.
    for (int k = 0; k < 3; k++) {
      A.bp[3 * s + k] = 0; A.bv[3 * s + k] = 0; A.bw[3 * s + k] = 0; A.btum[3 * s + k] = 0;
    }
    for (int k = 0; k < 4; k++) A.bq[4 * s + k] = 0;
    A.bceil[s] = 0;
  }
  for (int m = W.row0 + lane.id; m < W.row0 + W.nrows; m += lane.n) {
    double* bst = A.bst + RSTATE * static_cast<int64_t>(m);
    for (int k = 0; k < P; k++) bst[RS_NI + k] = A.seed_ni[4 * m + k];
    bst[RS_TI1] = A.seed_ti1[m]; bst[RS_TI2] = A.seed_ti2[m]; bst[RS_RI1] = A.seed_ri1[m];
    bst[RS_RI2] = A.seed_ri2[m]; bst[RS_SI] = A.seed_si[m];
    for (int k = RS_MAXNI; k < RSTATE; k++) bst[k] = 0;
    double* bpr = A.bpr + PREP * static_cast<int64_t>(m);
    for (int k = 0; k < PREP; k++) bpr[k] = 0;
    for (int k = 0; k < 3; k++) { A.bnormal[3 * m + k] = 0; A.bt1[3 * m + k] = 0; A.bt2[3 * m + k] = 0; }
    for (int k = 0; k < P; k++) A.bseparation[4 * m + k] = 0;
    for (int k = 0; k < 12; k++) A.bpoint[12 * m + k] = 0;
    A.bfriction[m] = 0;
    A.brestitution[m] = 0;
  }
  lane.sync();
  if (touching) {
    // slipped (src/contact.js:1122-1153), colour by colour: a colour's rows share no moving body
    auto slip = [&](int m) {
      bgad::Tape* t = bgad::thread_tape();
      bgad::reset(t);
      const RowIO<double> r = row_io(A, W, m);
      const int a = W.body0 + A.a[m], b = W.body0 + A.b[m];
      RowLeaves L;
      for (int k = 0; k < RSTATE; k++) L.st[k] = TV(r.st[k]);
      leaves(L.pa, r.pa, 3); leaves(L.pb, r.pb, 3); leaves(L.qa, r.qa, 4); leaves(L.qb, r.qb, 4);
      leaves(L.sa, r.sa, 3); leaves(L.sb, r.sb, 3);
      leaves(L.qa0, A.startq + 4 * a, 4); leaves(L.qb0, A.startq + 4 * b, 4);
      for (int k = 0; k < PREP; k++) L.pr[k] = TV(r.pr[k]);
      leaves(L.pr + PR_ANA, r.pr + PR_ANA, 6);
      leaves(L.t1, r.t1, 3); leaves(L.t2, r.t2, 3);
      L.drift1 = bgad::leaf(A.in_drift1[m]); L.drift2 = bgad::leaf(A.in_drift2[m]);
      const TV in_d1 = L.drift1, in_d2 = L.drift2;   // slipped() overwrites them in L
      const RowIO<TV> o = leaf_io(L, r);
      slipped_row(o, L.qa0, L.qb0, A.awake[a] != 0, A.awake[b] != 0);
      if (t->overflow) {
        *A.status = 1;
        return;
      }
      bgad::clear_adjoints(t);
      bgad::seed(t, L.drift1, A.bdrift1[m]);
      bgad::seed(t, L.drift2, A.bdrift2[m]);
      bgad::sweep(t);
      A.bdrift1[m] = bgad::adjoint(t, in_d1);
      A.bdrift2[m] = bgad::adjoint(t, in_d2);
      if (moving(A, a)) {
        add_adjoints(A.bp + 3 * a, t, L.pa, 3); add_adjoints(A.bq + 4 * a, t, L.qa, 4);
        add_adjoints(A.bstart + 3 * a, t, L.sa, 3); add_adjoints(A.bstartq + 4 * a, t, L.qa0, 4);
      }
      if (moving(A, b)) {
        add_adjoints(A.bp + 3 * b, t, L.pb, 3); add_adjoints(A.bq + 4 * b, t, L.qb, 4);
        add_adjoints(A.bstart + 3 * b, t, L.sb, 3); add_adjoints(A.bstartq + 4 * b, t, L.qb0, 4);
      }
      add_adjoints(A.bpr + PREP * static_cast<int64_t>(m) + PR_ANA, t, L.pr + PR_ANA, 6);
      add_adjoints(A.bt1 + 3 * m, t, L.t1, 3);
      add_adjoints(A.bt2 + 3 * m, t, L.t2, 3);
    };
    for (int k = 0; k < bg::NCOLOURS; k++) {
      for (int m = W.starts[k] + lane.id; m < W.starts[k + 1]; m += lane.n) slip(W.row0 + m);
      lane.sync();
    }
    if (lane.id == 0)
      for (int m = W.starts[bg::OVERFLOW_RUN]; m < W.starts[bg::OVERFLOW_RUN + 1]; m++) slip(W.row0 + m);
    lane.sync();
    // restitution (src/contact.js:2229-2251), in reverse found order, one thread
    const double* g = W.gravity;
    const double gravity = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    if (lane.id == 0) {
      for (int f = W.nrows - 1; f >= 0; f--) {
        const int m = W.row0 + A.row[W.row0 + f];
        if (m >= W.row0 + W.solved) continue;
        const RowIO<double> r = row_io(A, W, m);
        if (!bouncy(r, gravity)) continue;
        bgad::Tape* t = bgad::thread_tape();
        bgad::reset(t);
        const int a = W.body0 + A.a[m], b = W.body0 + A.b[m];
        const double* rec = A.rec_rest + static_cast<int64_t>(m) * REC_REST;
        RowLeaves L;
        for (int k = 0; k < RSTATE; k++) L.st[k] = TV(r.st[k]);
        leaves(L.st + RS_NI, rec + 12, P);
        leaves(L.st + RS_RELVEL, r.st + RS_RELVEL, P);
        leaves(L.va, rec, 3); leaves(L.wa, rec + 3, 3); leaves(L.vb, rec + 6, 3); leaves(L.wb, rec + 9, 3);
        leaves(L.pr, r.pr, PREP);
        leaves(L.normal, r.normal, 3);
        L.restitution = bgad::leaf(r.restitution[0]);
        TV in_v[12], in_ni[P];   // bounce_row() overwrites these in L
        for (int c = 0; c < 3; c++) { in_v[c] = L.va[c]; in_v[3 + c] = L.wa[c]; in_v[6 + c] = L.vb[c]; in_v[9 + c] = L.wb[c]; }
        for (int k = 0; k < P; k++) in_ni[k] = L.st[RS_NI + k];
        const RowIO<TV> o = leaf_io(L, r);
        bounce_row(o, gravity);
        if (t->overflow) {
          *A.status = 1;
          break;
        }
        bgad::clear_adjoints(t);
        const bool ma = moving(A, a), mb = moving(A, b);
        for (int c = 0; c < 3; c++) {
          if (ma) { bgad::seed(t, L.va[c], A.bv[3 * a + c]); bgad::seed(t, L.wa[c], A.bw[3 * a + c]); }
          if (mb) { bgad::seed(t, L.vb[c], A.bv[3 * b + c]); bgad::seed(t, L.wb[c], A.bw[3 * b + c]); }
        }
        double* bst = A.bst + RSTATE * static_cast<int64_t>(m);
        for (int k = 0; k < P; k++) bgad::seed(t, L.st[RS_NI + k], bst[RS_NI + k]);
        bgad::sweep(t);
        if (ma) { set_adjoints(A.bv + 3 * a, t, in_v, 3); set_adjoints(A.bw + 3 * a, t, in_v + 3, 3); }
        if (mb) { set_adjoints(A.bv + 3 * b, t, in_v + 6, 3); set_adjoints(A.bw + 3 * b, t, in_v + 9, 3); }
        set_adjoints(bst + RS_NI, t, in_ni, P);
        add_adjoints(bst + RS_RELVEL, t, L.st + RS_RELVEL, P);
        add_adjoints(A.bpr + PREP * static_cast<int64_t>(m), t, L.pr, PREP);
        add_adjoints(A.bnormal + 3 * m, t, L.normal, 3);
        A.brestitution[m] += bgad::adjoint(t, L.restitution);
      }
    }
    lane.sync();
  }
  for (int sub = A.substeps - 1; sub >= 0; sub--) {
    if (touching) reverse_pass(A, W, lane, 3 * sub + RELAX, sub, h);
    // move (src/world.js:1533-1563)
    for (int i = W.awake0 + lane.id; i < W.awake0 + W.nawake; i += lane.n) {
      const int s = W.body0 + A.awake_list[i];
      if (!moving(A, s)) continue;
      bgad::Tape* t = bgad::thread_tape();
      bgad::reset(t);
      const double* rec = A.rec_body + (static_cast<int64_t>(sub) * A.bodies_total + s) * REC_BODY;
      TV p[3], q[4], v[3], w[3], tum[3], ceil;
      leaves(p, rec + RB_P, 3); leaves(q, rec + RB_Q, 4); leaves(v, rec + RB_V, 3); leaves(w, rec + RB_W, 3);
      leaves(tum, rec + RB_TUM, 3);
      ceil = bgad::leaf(rec[RB_CEIL]);
      TV p1[3] = {p[0], p[1], p[2]}, q1[4] = {q[0], q[1], q[2], q[3]}, w1[3] = {w[0], w[1], w[2]};
      TV tum1[3] = {tum[0], tum[1], tum[2]}, ceil1 = ceil;
      move(body_const(A, s), h, p1, q1, v, w1, tum1, &ceil1);
      if (t->overflow) {
        *A.status = 1;
        continue;
      }
      bgad::clear_adjoints(t);
      for (int k = 0; k < 3; k++) {
        bgad::seed(t, p1[k], A.bp[3 * s + k]); bgad::seed(t, v[k], A.bv[3 * s + k]);
        bgad::seed(t, w1[k], A.bw[3 * s + k]); bgad::seed(t, tum1[k], A.btum[3 * s + k]);
      }
      for (int k = 0; k < 4; k++) bgad::seed(t, q1[k], A.bq[4 * s + k]);
      bgad::seed(t, ceil1, A.bceil[s]);
      bgad::sweep(t);
      set_adjoints(A.bp + 3 * s, t, p, 3); set_adjoints(A.bq + 4 * s, t, q, 4); set_adjoints(A.bv + 3 * s, t, v, 3);
      set_adjoints(A.bw + 3 * s, t, w, 3); set_adjoints(A.btum + 3 * s, t, tum, 3);
      A.bceil[s] = bgad::adjoint(t, ceil);
    }
    lane.sync();
    if (touching) {
      reverse_pass(A, W, lane, 3 * sub + SOLVE, sub, h);
      reverse_pass(A, W, lane, 3 * sub + WARM, sub, h);
    }
    // accelerate (src/world.js:1495-1530), its reverse written out: gravity adds a constant, the
    // dampings scale, and the spin limit scales w onto the sphere of radius `most` when it holds
    for (int i = W.awake0 + lane.id; i < W.awake0 + W.nawake; i += lane.n) {
      const int s = W.body0 + A.awake_list[i];
      if (!moving(A, s)) continue;
      const BodyConst bc = body_const(A, s);
      if (!bc.dynamic) continue;
      const double* rec = A.rec_body + (static_cast<int64_t>(sub) * A.bodies_total + s) * REC_BODY;
      const double most = WORLD_SPIN / (h * A.substeps);
      const double kv = bc.damping != 0 ? 1 / (1 + h * bc.damping) : 1.0;
      const double kw = bc.angular_damping != 0 ? 1 / (1 + h * bc.angular_damping) : 1.0;
      double w1[3];
      for (int k = 0; k < 3; k++) w1[k] = bc.angular_damping != 0 ? rec[RB_ACC + 3 + k] * kw : rec[RB_ACC + 3 + k];
      double* bw = A.bw + 3 * s;
      if (!bc.sphere_unframed) {
        const double w2 = w1[0] * w1[0] + w1[1] * w1[1] + w1[2] * w1[2];
        if (w2 > most * most) {
          const double q = sqrt(w2), c = most / q;
          const double b_c = bw[0] * w1[0] + bw[1] * w1[1] + bw[2] * w1[2];
          const double b_w2 = -b_c * most / (q * q) * 0.5 / q;
          for (int k = 0; k < 3; k++) bw[k] = c * bw[k] + 2 * w1[k] * b_w2;
        }
      }
      for (int k = 0; k < 3; k++) {
        if (bc.angular_damping != 0) bw[k] *= kw;
        if (bc.damping != 0) A.bv[3 * s + k] *= kv;
      }
    }
    lane.sync();
  }
  if (touching) {
    // prepare (src/contact.js:1346-1445), colour by colour, from the step's input
    auto prep = [&](int m) {
      bgad::Tape* t = bgad::thread_tape();
      bgad::reset(t);
      const RowIO<double> r = row_io(A, W, m);
      const int a = W.body0 + A.a[m], b = W.body0 + A.b[m];
      RowLeaves L;
      for (int k = 0; k < RSTATE; k++) L.st[k] = TV(0.0);
      leaves(L.pa, A.in_p + 3 * a, 3); leaves(L.pb, A.in_p + 3 * b, 3);
      leaves(L.qa, A.in_q + 4 * a, 4); leaves(L.qb, A.in_q + 4 * b, 4);
      leaves(L.va, A.in_v + 3 * a, 3); leaves(L.wa, A.in_w + 3 * a, 3);
      leaves(L.vb, A.in_v + 3 * b, 3); leaves(L.wb, A.in_w + 3 * b, 3);
      leaves(L.ia, r.ia, 6); leaves(L.ib, r.ib, 6);
      leaves(L.normal, r.normal, 3); leaves(L.t1, r.t1, 3); leaves(L.t2, r.t2, 3);
      leaves(L.separation, r.separation, P); leaves(L.point, r.point, 3 * P);
      const RowIO<TV> o = leaf_io(L, r);   // it writes only pr and st, which it does not read
      prepare_row(o);
      if (t->overflow) {
        *A.status = 1;
        return;
      }
      bgad::clear_adjoints(t);
      const double* bpr = A.bpr + PREP * static_cast<int64_t>(m);
      for (int k = 0; k < PREP; k++) bgad::seed(t, L.pr[k], bpr[k]);
      const double* bst = A.bst + RSTATE * static_cast<int64_t>(m);
      for (int k = 0; k < P; k++) bgad::seed(t, L.st[RS_RELVEL + k], bst[RS_RELVEL + k]);
      bgad::sweep(t);
      if (moving(A, a)) {
        add_adjoints(A.bp + 3 * a, t, L.pa, 3); add_adjoints(A.bq + 4 * a, t, L.qa, 4);
        add_adjoints(A.bv + 3 * a, t, L.va, 3); add_adjoints(A.bw + 3 * a, t, L.wa, 3);
        add_adjoints(A.binvI + 6 * a, t, L.ia, 6);
      }
      if (moving(A, b)) {
        add_adjoints(A.bp + 3 * b, t, L.pb, 3); add_adjoints(A.bq + 4 * b, t, L.qb, 4);
        add_adjoints(A.bv + 3 * b, t, L.vb, 3); add_adjoints(A.bw + 3 * b, t, L.wb, 3);
        add_adjoints(A.binvI + 6 * b, t, L.ib, 6);
      }
      add_adjoints(A.bnormal + 3 * m, t, L.normal, 3);
      add_adjoints(A.bt1 + 3 * m, t, L.t1, 3);
      add_adjoints(A.bt2 + 3 * m, t, L.t2, 3);
      add_adjoints(A.bseparation + 4 * m, t, L.separation, P);
      add_adjoints(A.bpoint + 12 * m, t, L.point, 3 * P);
    };
    for (int k = 0; k < bg::NCOLOURS; k++) {
      for (int m = W.starts[k] + lane.id; m < W.starts[k + 1]; m += lane.n) prep(W.row0 + m);
      lane.sync();
    }
    if (lane.id == 0)
      for (int m = W.starts[bg::OVERFLOW_RUN]; m < W.starts[bg::OVERFLOW_RUN + 1]; m++) prep(W.row0 + m);
    lane.sync();
  }
  // the start snapshot and inertias (src/world.js:964-974, src/contact.js:1302-1310)
  for (int i = W.awake0 + lane.id; i < W.awake0 + W.nawake; i += lane.n) {
    const int s = W.body0 + A.awake_list[i];
    if (!moving(A, s)) continue;
    for (int k = 0; k < 3; k++) A.bp[3 * s + k] += A.bstart[3 * s + k];
    for (int k = 0; k < 4; k++) A.bq[4 * s + k] += A.bstartq[4 * s + k];
    if (!touching) continue;
    bgad::Tape* t = bgad::thread_tape();
    bgad::reset(t);
    TV q[4], out[6];
    leaves(q, A.in_q + 4 * s, 4);
    inverse_inertia(q, A.inv_inertia + 3 * s, out);
    bgad::clear_adjoints(t);
    for (int k = 0; k < 6; k++) bgad::seed(t, out[k], A.binvI[6 * s + k]);
    bgad::sweep(t);
    add_adjoints(A.bq + 4 * s, t, q, 4);
  }
  lane.sync();
}

}  // namespace bgadj
