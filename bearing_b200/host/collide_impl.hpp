// Sphere, capsule and box contacts, in the reference narrowphase's operation order
// (src/collide.js), for any scalar type T: double for the step itself, a recording scalar for the
// adjoint's replay (the derivative of each contact's points, normal and separations with respect
// to the two bodies' poses), dual numbers for the tests' checker.  Each function cites the lines it
// follows.  The reference keeps its scratch in module variables; here they live in one NarrowT
// object per call, so calls on different threads never share them.
//
// A T needs + - * /, comparisons, sqrt and fabs found by argument-dependent lookup, and val(x),
// its plain value (signbit reads it).  Integer results (ids, feature numbers, counts) and every
// branch follow the values, so all instantiations find the same contacts.
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>

#include "collide.hpp"

// The same source serves the host side of the step (g++) and the device narrowphase (nvcc, one
// thread a pair): every function is callable from both.
#if defined(__CUDACC__)
#define NW_HD __host__ __device__
#else
#define NW_HD
#endif

namespace bearing {
namespace narrow_detail {

using std::fabs;
using std::sqrt;
NW_HD inline double val(double x) { return x; }
// The sign bit of x (Math.max / Math.min tell +0 from -0 by it).
NW_HD inline bool sign_bit(double x) {
#if defined(__CUDA_ARCH__)
  return __double_as_longlong(x) < 0;
#else
  return std::signbit(x);
#endif
}

constexpr double INF = std::numeric_limits<double>::infinity();
constexpr double PARALLEL = 7.450580596923828e-9;   // 2^-27, src/collide.js:686

// The reference's small tables, as functions (device code reads no host arrays).
// CORNER_P, CORNER_Q: src/collide.js:703.
NW_HD inline int corner_p(int v) { return v == 1 || v == 2 ? 1 : -1; }
NW_HD inline int corner_q(int v) { return v >= 2 ? 1 : -1; }
// EDGE_FROM, EDGE_TO: src/collide.js:791 (edges along x: corners 2i, 2i+1; along y: 0 1 4 5 to
// +2; along z: 0 1 2 3 to +4).
NW_HD inline int edge_from(int i) { return i < 4 ? 2 * i : i < 8 ? (i - 4) + ((i - 4) >= 2 ? 2 : 0) : i - 8; }
NW_HD inline int edge_to(int i) { return edge_from(i) + (i < 4 ? 1 : i < 8 ? 2 : 4); }
// EDGE_PLANE {3, 0, 2, 1}, PLANE_EDGE {1, 3, 2, 0}: src/collide.js:869.
NW_HD inline int edge_plane(int e) { return e == 0 ? 3 : e == 1 ? 0 : e == 2 ? 2 : 1; }
NW_HD inline int plane_edge(int k) { return k == 0 ? 1 : k == 1 ? 3 : k == 2 ? 2 : 0; }

// SWAPPED[f]: src/collide.js:870-877, entry by entry: a corner v of the incident face and the
// crossing of its two reference planes trade places, an edge-plane crossing is renumbered from
// the other box's side, and every other feature keeps its number.
NW_HD inline int swapped_feature(int f) {
  if (f < 4) return 20 + 4 * (corner_p(f) > 0 ? 0 : 1) + (corner_q(f) > 0 ? 2 : 3);
  if (f < 20) return 4 + 4 * plane_edge((f - 4) % 4) + edge_plane((f - 4) / 4);
  for (int v = 0; v < 4; v++)
    if (f == 20 + 4 * (corner_p(v) > 0 ? 0 : 1) + (corner_q(v) > 0 ? 2 : 3)) return v;
  return f;
}

template <class T>
struct NarrowT {
  using Shape = ShapeT<T>;
  using Manifold = ManifoldT<T>;
  // sgn, clamp01: src/collide.js:246-247.
  NW_HD static T sgn(const T& x) { return x < 0 ? T(-1) : T(1); }
  NW_HD static T clamp01(const T& x) { return x < 0 ? T(0) : x > 1 ? T(1) : x; }
  // Math.max / Math.min with JavaScript's NaN and signed-zero rules.
  NW_HD static T jmax(const T& a, const T& b) {
    if (a != a) return a;
    if (b != b) return b;
    if (a > b) return a;
    if (b > a) return b;
    if (a == 0 && b == 0) return sign_bit(val(a)) ? b : a;
    return a;
  }
  NW_HD static T jmin(const T& a, const T& b) {
    if (a != a) return a;
    if (b != b) return b;
    if (a < b) return a;
    if (b < a) return b;
    if (a == 0 && b == 0) return sign_bit(val(a)) ? a : b;
    return a;
  }

  const Shape* shapeA = nullptr;
  const Shape* shapeB = nullptr;
  T unit[3] = {0, 0, 0};
  T segS = 0, segT = 0;
  T segA[6], segB[6], local[6], edge[6], world[3];
  T polyA[24], polyB[24];
  int featA[8], featB[8], lineA[8], lineB[8];
  T kept[24], keptSep[8];
  uint32_t keptId[8];
  T cosines[9];
  T cornerA[24], cornerB[24];
  int FOUR[4];
  T FOOT[3];

  // normalize: src/collide.js:257-264.
  NW_HD T normalize(T x, T y, T z) {
    const T m = jmax(jmax(fabs(x), fabs(y)), fabs(z));
    if (m == 0) return 0;
    const T sx = x / m, sy = y / m, sz = z / m;
    const T l = sqrt(sx * sx + sy * sy + sz * sz);
    unit[0] = sx / l; unit[1] = sy / l; unit[2] = sz / l;
    return l * m;
  }
  // perpendicular: src/collide.js:272-277.
  NW_HD void perpendicular(T vx, T vy, T vz) {
    const T ax = fabs(vx), ay = fabs(vy), az = fabs(vz);
    if (ax <= ay && ax <= az) normalize(0, vz, -vy);
    else if (ay <= az) normalize(-vz, 0, vx);
    else normalize(vy, -vx, 0);
  }
  NW_HD static void setNormal(Manifold& out, T x, T y, T z) {
    out.normal[0] = x; out.normal[1] = y; out.normal[2] = z;
  }
  NW_HD static void addPoint(Manifold& out, T x, T y, T z, T separation, uint32_t id) {
    const int k = out.count++;
    out.points[3 * k] = x; out.points[3 * k + 1] = y; out.points[3 * k + 2] = z;
    out.separations[k] = separation;
    out.ids[k] = id;
  }
  // balls: src/collide.js:296-306.
  NW_HD bool balls(T ax, T ay, T az, T ra, T bx, T by, T bz, T rb,
             T fx, T fy, T fz, T margin, Manifold& out, uint32_t id) {
    const T dist = normalize(bx - ax, by - ay, bz - az);
    const T separation = dist - ra - rb;
    if (separation > margin) return false;
    const T nx = dist > 0 ? unit[0] : fx, ny = dist > 0 ? unit[1] : fy, nz = dist > 0 ? unit[2] : fz;
    setNormal(out, nx, ny, nz);
    const T t = ra + separation * 0.5;
    addPoint(out, ax + nx * t, ay + ny * t, az + nz * t, separation, id);
    return true;
  }
  // segment: src/collide.js:309-313.
  NW_HD static void segment(const Shape& c, T* out) {
    const T h = c.half[1];
    const T* y = c.axes;
    out[0] = c.center[0] - y[3] * h; out[1] = c.center[1] - y[4] * h; out[2] = c.center[2] - y[5] * h;
    out[3] = c.center[0] + y[3] * h; out[4] = c.center[1] + y[4] * h; out[5] = c.center[2] + y[5] * h;
  }
  // nearestOnSegment: src/collide.js:316-321.
  NW_HD static T nearestOnSegment(const T* s, T x, T y, T z) {
    const T dx = s[3] - s[0], dy = s[4] - s[1], dz = s[5] - s[2];
    const T dd = dx * dx + dy * dy + dz * dz;
    if (dd == 0) return 0;
    return clamp01(((x - s[0]) * dx + (y - s[1]) * dy + (z - s[2]) * dz) / dd);
  }
  // closestSegments: src/collide.js:332-349.
  NW_HD void closestSegments(const T* p, const T* q) {
    const T d1x = p[3] - p[0], d1y = p[4] - p[1], d1z = p[5] - p[2];
    const T d2x = q[3] - q[0], d2y = q[4] - q[1], d2z = q[5] - q[2];
    const T rx = p[0] - q[0], ry = p[1] - q[1], rz = p[2] - q[2];
    const T a = d1x * d1x + d1y * d1y + d1z * d1z;
    const T e = d2x * d2x + d2y * d2y + d2z * d2z;
    const T f = d2x * rx + d2y * ry + d2z * rz;
    if (a == 0 && e == 0) { segS = 0; segT = 0; return; }
    if (a == 0) { segS = 0; segT = clamp01(f / e); return; }
    const T c = d1x * rx + d1y * ry + d1z * rz;
    if (e == 0) { segT = 0; segS = clamp01(-c / a); return; }
    const T b = d1x * d2x + d1y * d2y + d1z * d2z;
    const T denom = a * e - b * b;
    T s = denom != 0 ? clamp01((b * f - c * e) / denom) : 0;
    T t = (b * s + f) / e;
    if (t < 0) { t = 0; s = clamp01(-c / a); } else if (t > 1) { t = 1; s = clamp01((b - c) / a); }
    segS = s; segT = t;
  }

  // sphereSphere: src/collide.js:353-357.
  NW_HD void sphereSphere(const Shape& a, const Shape& b, T margin, Manifold& out) {
    balls(a.center[0], a.center[1], a.center[2], a.half[0], b.center[0], b.center[1], b.center[2], b.half[0],
          0, 1, 0, margin, out, 0);
  }
  // sphereCapsule: src/collide.js:361-369.
  NW_HD void sphereCapsule(const Shape& a, const Shape& b, T margin, Manifold& out) {
    const T* c = a.center;
    segment(b, segB);
    const T t = nearestOnSegment(segB, c[0], c[1], c[2]);
    const T qx = segB[0] + (segB[3] - segB[0]) * t, qy = segB[1] + (segB[4] - segB[1]) * t,
                 qz = segB[2] + (segB[5] - segB[2]) * t;
    perpendicular(b.axes[3], b.axes[4], b.axes[5]);
    balls(c[0], c[1], c[2], a.half[0], qx, qy, qz, b.half[0], unit[0], unit[1], unit[2], margin, out, 0);
  }
  // sphereBox: src/collide.js:371-403.
  NW_HD void sphereBox(const Shape& a, const Shape& b, T margin, Manifold& out) {
    const T* ax = b.axes;
    const T* h = b.half;
    const T r = a.half[0];
    const T dx = a.center[0] - b.center[0], dy = a.center[1] - b.center[1], dz = a.center[2] - b.center[2];
    const T lx = dx * ax[0] + dy * ax[1] + dz * ax[2];
    const T ly = dx * ax[3] + dy * ax[4] + dz * ax[5];
    const T lz = dx * ax[6] + dy * ax[7] + dz * ax[8];
    const bool inside = fabs(lx) <= h[0] && fabs(ly) <= h[1] && fabs(lz) <= h[2];
    if (!inside) {
      const T qx = jmax(-h[0], jmin(h[0], lx));
      const T qy = jmax(-h[1], jmin(h[1], ly));
      const T qz = jmax(-h[2], jmin(h[2], lz));
      const T wx = b.center[0] + ax[0] * qx + ax[3] * qy + ax[6] * qz;
      const T wy = b.center[1] + ax[1] * qx + ax[4] * qy + ax[7] * qz;
      const T wz = b.center[2] + ax[2] * qx + ax[5] * qy + ax[8] * qz;
      balls(a.center[0], a.center[1], a.center[2], r, wx, wy, wz, 0, 0, 1, 0, margin, out, 0);
      return;
    }
    int axis = 0;
    T depth = h[0] - fabs(lx);
    if (h[1] - fabs(ly) < depth) { axis = 1; depth = h[1] - fabs(ly); }
    if (h[2] - fabs(lz) < depth) { axis = 2; depth = h[2] - fabs(lz); }
    const T l = axis == 0 ? lx : axis == 1 ? ly : lz;
    const T s = -sgn(l);
    const T nx = ax[3 * axis] * s, ny = ax[3 * axis + 1] * s, nz = ax[3 * axis + 2] * s;
    setNormal(out, nx, ny, nz);
    const T separation = -(depth + r);
    const T t = r + separation * 0.5;
    addPoint(out, a.center[0] + nx * t, a.center[1] + ny * t, a.center[2] + nz * t, separation, 0);
  }

  // capsuleCapsule: src/collide.js:424-482.
  NW_HD void capsuleCapsule(const Shape& a, const Shape& b, T margin, T tolerance, Manifold& out) {
    segment(a, segA);
    segment(b, segB);
    closestSegments(segA, segB);
    const T s = segS, t = segT;
    const T pax = segA[0] + (segA[3] - segA[0]) * s, pay = segA[1] + (segA[4] - segA[1]) * s,
                 paz = segA[2] + (segA[5] - segA[2]) * s;
    const T pbx = segB[0] + (segB[3] - segB[0]) * t, pby = segB[1] + (segB[4] - segB[1]) * t,
                 pbz = segB[2] + (segB[5] - segB[2]) * t;
    const T ra = a.half[0], rb = b.half[0];
    const T* ya = a.axes;
    const T* yb = b.axes;
    if (normalize(ya[4] * yb[5] - ya[5] * yb[4], ya[5] * yb[3] - ya[3] * yb[5], ya[3] * yb[4] - ya[4] * yb[3]) == 0) {
      perpendicular(ya[3], ya[4], ya[5]);
    }
    const T fx = unit[0], fy = unit[1], fz = unit[2];
    if (!balls(pax, pay, paz, ra, pbx, pby, pbz, rb, fx, fy, fz, margin, out, 0)) return;
    const T closest = out.separations[0];
    const T cx = out.points[0], cy = out.points[1], cz = out.points[2];
    out.count = 0;
    const T h = a.half[1];
    if (h > 0 && b.half[1] > 0) {
      const T k0 = (segB[0] - a.center[0]) * ya[3] + (segB[1] - a.center[1]) * ya[4] + (segB[2] - a.center[2]) * ya[5];
      const T k1 = (segB[3] - segB[0]) * ya[3] + (segB[4] - segB[1]) * ya[4] + (segB[5] - segB[2]) * ya[5];
      T u0 = 0, u1 = 1;
      if (k1 != 0) {
        const T ua = (-h - k0) / k1, ub = (h - k0) / k1;
        u0 = jmax(0, jmin(ua, ub));
        u1 = jmin(1, jmax(ua, ub));
      } else if (k0 < -h || k0 > h) {
        u1 = -1;
      }
      if (u1 > u0) {
        const T* n = out.normal;
        T deepest = INF;
        for (int e = 0; e < 2; e++) {
          const T u = e == 0 ? u0 : u1;
          const T bx = segB[0] + (segB[3] - segB[0]) * u, by = segB[1] + (segB[4] - segB[1]) * u,
                       bz = segB[2] + (segB[5] - segB[2]) * u;
          const T alongA = jmax(-h, jmin(h, k0 + k1 * u));
          const T ax = a.center[0] + ya[3] * alongA, ay = a.center[1] + ya[4] * alongA,
                       az = a.center[2] + ya[5] * alongA;
          const T gx = bx - ax, gy = by - ay, gz = bz - az;
          const T normalGap = gx * n[0] + gy * n[1] + gz * n[2];
          const T separation = normalGap - ra - rb;
          if (separation > margin) continue;
          if (gx * gx + gy * gy + gz * gz - normalGap * normalGap > tolerance * tolerance) continue;
          deepest = jmin(deepest, separation);
          const T m = ra + separation * 0.5;
          addPoint(out, ax + n[0] * m, ay + n[1] * m, az + n[2] * m, separation, static_cast<uint32_t>(1 + e));
        }
        if (out.count > 0 && closest < deepest) addPoint(out, cx, cy, cz, closest, 0);
        if (out.count > 0) return;
      }
    }
    addPoint(out, cx, cy, cz, closest, 0);
  }

  // toWorld: src/collide.js:552-557.
  NW_HD void toWorld(const Shape& b, T x, T y, T z) {
    const T* ax = b.axes;
    world[0] = b.center[0] + ax[0] * x + ax[3] * y + ax[6] * z;
    world[1] = b.center[1] + ax[1] * x + ax[4] * y + ax[7] * z;
    world[2] = b.center[2] + ax[2] * x + ax[5] * y + ax[8] * z;
  }
  // segmentHitsBox: src/collide.js:560-575.
  NW_HD static bool segmentHitsBox(const T* s, const T* h) {
    T t0 = 0, t1 = 1;
    for (int i = 0; i < 3; i++) {
      const T p = s[i], d = s[3 + i] - s[i];
      if (d == 0) {
        if (p < -h[i] || p > h[i]) return false;
        continue;
      }
      T ta = (-h[i] - p) / d, tb = (h[i] - p) / d;
      if (ta > tb) { const T x = ta; ta = tb; tb = x; }
      if (ta > t0) t0 = ta;
      if (tb < t1) t1 = tb;
      if (t0 > t1) return false;
    }
    return true;
  }
  // clipToFace: src/collide.js:583-615.
  NW_HD bool clipToFace(const Shape& b, int axis, T facing, T r, T margin, Manifold& out, uint32_t idBase) {
    const T* h = b.half;
    const int j = (axis + 1) % 3, k = (axis + 2) % 3;
    T u0 = 0, u1 = 1;
    for (int pass = 0; pass < 2; pass++) {
      const int c = pass == 0 ? j : k;
      const T p = local[c], d = local[3 + c] - local[c];
      if (d == 0) {
        if (p < -h[c] || p > h[c]) return false;
        continue;
      }
      T ta = (-h[c] - p) / d, tb = (h[c] - p) / d;
      if (ta > tb) { const T x = ta; ta = tb; tb = x; }
      if (ta > u0) u0 = ta;
      if (tb < u1) u1 = tb;
    }
    if (u0 > u1) return false;
    const T* ax = b.axes;
    setNormal(out, -facing * ax[3 * axis], -facing * ax[3 * axis + 1], -facing * ax[3 * axis + 2]);
    const int face = 2 * axis + (facing > 0 ? 1 : 0);
    for (int e = 0; e < (u1 > u0 ? 2 : 1); e++) {
      const T u = e == 0 ? u0 : u1;
      const T px = local[0] + (local[3] - local[0]) * u, py = local[1] + (local[4] - local[1]) * u,
                   pz = local[2] + (local[5] - local[2]) * u;
      const T above = facing * (axis == 0 ? px : axis == 1 ? py : pz) - h[axis];
      const T separation = above - r;
      if (separation > margin) continue;
      const T off = facing * (separation * 0.5 - above);
      toWorld(b, axis == 0 ? px + off : px, axis == 1 ? py + off : py, axis == 2 ? pz + off : pz);
      addPoint(out, world[0], world[1], world[2], separation, idBase + static_cast<uint32_t>(4 * face + 1 + e));
    }
    return out.count > 0;
  }
  // capsuleBoxDeep: src/collide.js:626-676.
  NW_HD void capsuleBoxDeep(const Shape& a, const Shape& b, T margin, T tolerance, Manifold& out) {
    const T* h = b.half;
    const T r = a.half[0];
    const T dx = local[3] - local[0], dy = local[4] - local[1], dz = local[5] - local[2];
    T bestSep = -INF, nx = 0, ny = 0, nz = 0;
    int bestAxis = -1;
    for (int c = 0; c < 6; c++) {
      T x = 0, y = 0, z = 0;
      if (c < 3) {
        if (c == 0) x = 1; else if (c == 1) y = 1; else z = 1;
      } else {
        const int e = c - 3;
        const T l = normalize(e == 0 ? 0 : e == 1 ? -dz : dy, e == 0 ? dz : e == 1 ? 0 : -dx,
                                   e == 0 ? -dy : e == 1 ? dx : 0);
        if (!(l > PARALLEL * sqrt(dx * dx + dy * dy + dz * dz))) continue;
        x = unit[0]; y = unit[1]; z = unit[2];
      }
      const T support = h[0] * fabs(x) + h[1] * fabs(y) + h[2] * fabs(z);
      const T p0 = local[0] * x + local[1] * y + local[2] * z, p1 = local[3] * x + local[4] * y + local[5] * z;
      const T lo = jmin(p0, p1), hi = jmax(p0, p1);
      const T plus = lo - support, minus = -support - hi;
      const T sep = jmax(plus, minus) - r;
      if (sep > bestSep + (c >= 3 && bestAxis < 3 ? tolerance : 0)) {
        bestSep = sep; bestAxis = c;
        const T s = plus >= minus ? -1 : 1;
        nx = x * s; ny = y * s; nz = z * s;
      }
    }
    if (bestAxis < 3) {
      const T facing = -(bestAxis == 0 ? nx : bestAxis == 1 ? ny : nz);
      clipToFace(b, bestAxis, sgn(facing), r, margin, out, 0);
      return;
    }
    const int i = bestAxis - 3, j = (i + 1) % 3, k = (i + 2) % 3;
    const T mj = j == 0 ? -nx : j == 1 ? -ny : -nz, mk = k == 0 ? -nx : k == 1 ? -ny : -nz;
    edge[i] = -h[i]; edge[3 + i] = h[i];
    edge[j] = edge[3 + j] = sgn(mj) * h[j];
    edge[k] = edge[3 + k] = sgn(mk) * h[k];
    closestSegments(local, edge);
    const T px = local[0] + dx * segS, py = local[1] + dy * segS, pz = local[2] + dz * segS;
    const T ex = edge[0] + (edge[3] - edge[0]) * segT, ey = edge[1] + (edge[4] - edge[1]) * segT,
                 ez = edge[2] + (edge[5] - edge[2]) * segT;
    const T separation = (ex - px) * nx + (ey - py) * ny + (ez - pz) * nz - r;
    const T* ax = b.axes;
    setNormal(out, ax[0] * nx + ax[3] * ny + ax[6] * nz, ax[1] * nx + ax[4] * ny + ax[7] * nz,
              ax[2] * nx + ax[5] * ny + ax[8] * nz);
    const T mm = r + separation * 0.5;
    toWorld(b, px + nx * mm, py + ny * mm, pz + nz * mm);
    addPoint(out, world[0], world[1], world[2], separation, static_cast<uint32_t>(32 + i));
  }
  // capsuleBox: src/collide.js:497-547.
  NW_HD void capsuleBox(const Shape& a, const Shape& b, T margin, T tolerance, Manifold& out) {
    segment(a, segA);
    const T* bx = b.axes;
    const T* h = b.half;
    const T r = a.half[0];
    for (int e = 0; e < 2; e++) {
      const T dx = segA[3 * e] - b.center[0], dy = segA[3 * e + 1] - b.center[1], dz = segA[3 * e + 2] - b.center[2];
      local[3 * e] = dx * bx[0] + dy * bx[1] + dz * bx[2];
      local[3 * e + 1] = dx * bx[3] + dy * bx[4] + dz * bx[5];
      local[3 * e + 2] = dx * bx[6] + dy * bx[7] + dz * bx[8];
    }
    if (segmentHitsBox(local, h)) { capsuleBoxDeep(a, b, margin, tolerance, out); return; }
    T best = INF, sx = 0, sy = 0, sz = 0, qx = 0, qy = 0, qz = 0;
    for (int e = 0; e < 2; e++) {
      const T px = local[3 * e], py = local[3 * e + 1], pz = local[3 * e + 2];
      const T cx = jmax(-h[0], jmin(h[0], px)), cy = jmax(-h[1], jmin(h[1], py)), cz = jmax(-h[2], jmin(h[2], pz));
      const T d = (px - cx) * (px - cx) + (py - cy) * (py - cy) + (pz - cz) * (pz - cz);
      if (d < best) { best = d; sx = px; sy = py; sz = pz; qx = cx; qy = cy; qz = cz; }
    }
    for (int i = 0; i < 3; i++) {
      const int j = (i + 1) % 3, k = (i + 2) % 3;
      for (int c = 0; c < 4; c++) {
        edge[i] = -h[i]; edge[3 + i] = h[i];
        edge[j] = edge[3 + j] = (c & 1) ? h[j] : -h[j];
        edge[k] = edge[3 + k] = (c & 2) ? h[k] : -h[k];
        closestSegments(local, edge);
        const T px = local[0] + (local[3] - local[0]) * segS, py = local[1] + (local[4] - local[1]) * segS,
                     pz = local[2] + (local[5] - local[2]) * segS;
        const T ex = edge[0] + (edge[3] - edge[0]) * segT, ey = edge[1] + (edge[4] - edge[1]) * segT,
                     ez = edge[2] + (edge[5] - edge[2]) * segT;
        const T d = (px - ex) * (px - ex) + (py - ey) * (py - ey) + (pz - ez) * (pz - ez);
        if (d < best) { best = d; sx = px; sy = py; sz = pz; qx = ex; qy = ey; qz = ez; }
      }
    }
    const T dist = normalize(qx - sx, qy - sy, qz - sz);
    if (dist - r > margin) return;
    const T nlx = unit[0], nly = unit[1], nlz = unit[2];
    setNormal(out, bx[0] * nlx + bx[3] * nly + bx[6] * nlz, bx[1] * nlx + bx[4] * nly + bx[7] * nlz,
              bx[2] * nlx + bx[5] * nly + bx[8] * nlz);
    const bool onX = fabs(qx) == h[0], onY = fabs(qy) == h[1], onZ = fabs(qz) == h[2];
    if (static_cast<int>(onX) + static_cast<int>(onY) + static_cast<int>(onZ) == 1) {
      const int axis = onX ? 0 : onY ? 1 : 2;
      const T facing = sgn(axis == 0 ? qx : axis == 1 ? qy : qz);
      if (clipToFace(b, axis, facing, r, margin, out, 0)) return;
    }
    const T separation = dist - r;
    const T m = r + separation * 0.5;
    toWorld(b, sx + nlx * m, sy + nly * m, sz + nlz * m);
    addPoint(out, world[0], world[1], world[2], separation, 0);
  }

  // support: src/collide.js:840-844.
  NW_HD static T support(const T* X, const T* h, T nx, T ny, T nz) {
    return h[0] * fabs(X[0] * nx + X[1] * ny + X[2] * nz)
      + h[1] * fabs(X[3] * nx + X[4] * ny + X[5] * nz)
      + h[2] * fabs(X[6] * nx + X[7] * ny + X[8] * nz);
  }
  // corners: src/collide.js:780-788.
  NW_HD static void corners(const Shape& x, T* c) {
    const T* X = x.axes;
    const T* h = x.half;
    for (int k = 0; k < 8; k++) {
      const T sx = (k & 1) ? h[0] : -h[0], sy = (k & 2) ? h[1] : -h[1], sz = (k & 4) ? h[2] : -h[2];
      c[3 * k] = x.center[0] + X[0] * sx + X[3] * sy + X[6] * sz;
      c[3 * k + 1] = x.center[1] + X[1] * sx + X[4] * sy + X[7] * sz;
      c[3 * k + 2] = x.center[2] + X[2] * sx + X[5] * sy + X[8] * sz;
    }
  }
  // boxBoxClosest: src/collide.js:800-837.
  NW_HD void boxBoxClosest(const Shape& a, const Shape& b, T margin, Manifold& out) {
    corners(a, cornerA);
    corners(b, cornerB);
    T best = INF, ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0;
    for (int side = 0; side < 2; side++) {
      const T* from = side == 0 ? cornerA : cornerB;
      const Shape& box = side == 0 ? b : a;
      const T* X = box.axes;
      const T* h = box.half;
      for (int k = 0; k < 8; k++) {
        const T dx = from[3 * k] - box.center[0], dy = from[3 * k + 1] - box.center[1], dz = from[3 * k + 2] - box.center[2];
        const T lx = jmax(-h[0], jmin(h[0], dx * X[0] + dy * X[1] + dz * X[2]));
        const T ly = jmax(-h[1], jmin(h[1], dx * X[3] + dy * X[4] + dz * X[5]));
        const T lz = jmax(-h[2], jmin(h[2], dx * X[6] + dy * X[7] + dz * X[8]));
        toWorld(box, lx, ly, lz);
        const T ex = world[0] - from[3 * k], ey = world[1] - from[3 * k + 1], ez = world[2] - from[3 * k + 2];
        const T d = ex * ex + ey * ey + ez * ez;
        if (d < best) {
          best = d;
          if (side == 0) { ax = from[3 * k]; ay = from[3 * k + 1]; az = from[3 * k + 2]; bx = world[0]; by = world[1]; bz = world[2]; }
          else { bx = from[3 * k]; by = from[3 * k + 1]; bz = from[3 * k + 2]; ax = world[0]; ay = world[1]; az = world[2]; }
        }
      }
    }
    for (int i = 0; i < 12; i++) {
      for (int k = 0; k < 3; k++) { segA[k] = cornerA[3 * edge_from(i) + k]; segA[3 + k] = cornerA[3 * edge_to(i) + k]; }
      for (int j = 0; j < 12; j++) {
        for (int k = 0; k < 3; k++) { segB[k] = cornerB[3 * edge_from(j) + k]; segB[3 + k] = cornerB[3 * edge_to(j) + k]; }
        closestSegments(segA, segB);
        const T px = segA[0] + (segA[3] - segA[0]) * segS, py = segA[1] + (segA[4] - segA[1]) * segS,
                     pz = segA[2] + (segA[5] - segA[2]) * segS;
        const T qx = segB[0] + (segB[3] - segB[0]) * segT, qy = segB[1] + (segB[4] - segB[1]) * segT,
                     qz = segB[2] + (segB[5] - segB[2]) * segT;
        const T d = (qx - px) * (qx - px) + (qy - py) * (qy - py) + (qz - pz) * (qz - pz);
        if (d < best) { best = d; ax = px; ay = py; az = pz; bx = qx; by = qy; bz = qz; }
      }
    }
    const T dist = normalize(bx - ax, by - ay, bz - az);
    if (dist > margin || dist == 0) return;
    setNormal(out, unit[0], unit[1], unit[2]);
    addPoint(out, (ax + bx) * 0.5, (ay + by) * 0.5, (az + bz) * 0.5, dist, 1u << 14);
  }

  // clipPolygon: src/collide.js:966-999.
  NW_HD static int clipPolygon(const T* src, const int* sf, const int* sl, int count, T* dst, int* df, int* dl,
                         T px, T py, T pz, T offset, int plane, T slack) {
    int n = 0;
    for (int v = 0; v < count; v++) {
      const int w = (v + 1) % count;
      const T ax = src[3 * v], ay = src[3 * v + 1], az = src[3 * v + 2];
      const T bx = src[3 * w], by = src[3 * w + 1], bz = src[3 * w + 2];
      const T da = ax * px + ay * py + az * pz - offset, db = bx * px + by * py + bz * pz - offset;
      const int line = sl[v];
      if (da <= slack) {
        if (da > 0) {
          dst[3 * n] = ax - px * da; dst[3 * n + 1] = ay - py * da; dst[3 * n + 2] = az - pz * da;
        } else {
          dst[3 * n] = ax; dst[3 * n + 1] = ay; dst[3 * n + 2] = az;
        }
        df[n] = sf[v];
        dl[n] = da > 0 && db > slack ? 4 + plane : line;
        n++;
      }
      if ((da <= 0 && db > slack) || (da > slack && db <= 0)) {
        const T t = da / (da - db);
        dst[3 * n] = ax + (bx - ax) * t; dst[3 * n + 1] = ay + (by - ay) * t; dst[3 * n + 2] = az + (bz - az) * t;
        const int lo = line - 4 < plane ? line - 4 : plane, hi = line - 4 > plane ? line - 4 : plane;
        df[n] = line < 4 ? 4 + 4 * line + plane : 20 + 4 * lo + hi;
        dl[n] = da <= 0 ? 4 + plane : line;
        n++;
      }
    }
    return n;
  }

  // four: src/collide.js:1116-1141.
  NW_HD void four(int n, int a, T nx, T ny, T nz, T pressed, T touching) {
    int b = -1;
    T far = -1;
    for (int pass = 0; pass < 3 && b < 0; pass++) {
      const T within = pass == 0 ? pressed : pass == 1 ? touching : INF;
      for (int k = 0; k < n; k++) {
        if (k == a || keptSep[k] > within) continue;
        const T x = kept[3 * k] - kept[3 * a], y = kept[3 * k + 1] - kept[3 * a + 1], z = kept[3 * k + 2] - kept[3 * a + 2];
        const T d = x * x + y * y + z * z;
        if (d > far) { far = d; b = k; }
      }
    }
    int c = -1, d = -1;
    T most = 0, least = 0;
    const T abx = kept[3 * b] - kept[3 * a], aby = kept[3 * b + 1] - kept[3 * a + 1], abz = kept[3 * b + 2] - kept[3 * a + 2];
    for (int pass = 0; pass < 3 && (c < 0 || d < 0); pass++) {
      const T within = pass == 0 ? pressed : pass == 1 ? touching : INF;
      const bool left = c < 0, right = d < 0;
      for (int k = 0; k < n; k++) {
        if (k == a || k == b || keptSep[k] > within) continue;
        const T x = kept[3 * k] - kept[3 * a], y = kept[3 * k + 1] - kept[3 * a + 1], z = kept[3 * k + 2] - kept[3 * a + 2];
        const T area = (aby * z - abz * y) * nx + (abz * x - abx * z) * ny + (abx * y - aby * x) * nz;
        if (left && area > most) { most = area; c = k; }
        if (right && area < least) { least = area; d = k; }
      }
    }
    FOUR[0] = a; FOUR[1] = d; FOUR[2] = b; FOUR[3] = c;
  }
  // foot: src/collide.js:1171-1178.
  NW_HD bool foot(const Shape& s, T nx, T ny, T nz) {
    const T* w = s.weight;
    const T* c = s.center;
    const T alongN = w[0] * nx + w[1] * ny + w[2] * nz;
    const int o = FOUR[0];
    if (alongN == 0) return false;
    const T t = ((kept[3 * o] - c[0]) * nx + (kept[3 * o + 1] - c[1]) * ny + (kept[3 * o + 2] - c[2]) * nz) / alongN;
    if (!(t > 0)) return false;
    FOOT[0] = c[0] + w[0] * t; FOOT[1] = c[1] + w[1] * t; FOOT[2] = c[2] + w[2] * t;
    return true;
  }
  // rests: src/collide.js:1151-1164.
  NW_HD bool rests(const Shape& s, T nx, T ny, T nz) {
    if (!foot(s, nx, ny, nz)) return false;
    const T px = FOOT[0], py = FOOT[1], pz = FOOT[2];
    int from = FOUR[0];
    for (int e = 1; e <= 4; e++) {
      const int to = FOUR[e & 3];
      if (to < 0) continue;
      const T ax = kept[3 * from] - px, ay = kept[3 * from + 1] - py, az = kept[3 * from + 2] - pz;
      const T bx = kept[3 * to] - px, by = kept[3 * to + 1] - py, bz = kept[3 * to + 2] - pz;
      if ((ay * bz - az * by) * nx + (az * bx - ax * bz) * ny + (ax * by - ay * bx) * nz < 0) return false;
      from = to;
    }
    return true;
  }
  // under: src/collide.js:1185-1194.
  NW_HD int under(int n, T nx, T ny, T nz, T pressed) {
    int start = -1;
    T nearest = INF;
    for (int k = 0; k < n; k++) {
      if (keptSep[k] > pressed) continue;
      const T x = kept[3 * k] - FOOT[0], y = kept[3 * k + 1] - FOOT[1], z = kept[3 * k + 2] - FOOT[2],
                   alongN = x * nx + y * ny + z * nz;
      const T d = x * x + y * y + z * z - alongN * alongN;
      if (d < nearest) { nearest = d; start = k; }
    }
    return start;
  }
  // reducePoints: src/collide.js:1077-1104.
  NW_HD void reducePoints(int n, T nx, T ny, T nz, T tolerance, Manifold& out) {
    if (n <= MAX_POINTS) {
      for (int k = 0; k < n; k++) addPoint(out, kept[3 * k], kept[3 * k + 1], kept[3 * k + 2], keptSep[k], keptId[k]);
      return;
    }
    T deepest = keptSep[0];
    int deep = 0;
    for (int k = 1; k < n; k++) if (keptSep[k] < deepest) { deepest = keptSep[k]; deep = k; }
    const T pressed = jmax(deepest, 0), touching = pressed + tolerance;
    int a = -1;
    for (int k = 0; k < n; k++) if (keptSep[k] <= deepest + tolerance && (a < 0 || keptId[k] < keptId[a])) a = k;
    four(n, a, nx, ny, nz, pressed, touching);
    if (!rests(*shapeA, nx, ny, nz) && !rests(*shapeB, nx, ny, nz)) {
      const bool weighed = foot(*shapeA, nx, ny, nz) || foot(*shapeB, nx, ny, nz);
      bool left = false;
      for (int k = 0; k < n && !left; k++) {
        left = (weighed ? keptSep[k] <= pressed : k == deep) && k != FOUR[0] && k != FOUR[1] && k != FOUR[2] && k != FOUR[3];
      }
      if (left) four(n, weighed ? under(n, nx, ny, nz, pressed) : deep, nx, ny, nz, pressed, touching);
    }
    const int s = FOUR[0], b = FOUR[2], c = FOUR[3], d = FOUR[1];
    addPoint(out, kept[3 * s], kept[3 * s + 1], kept[3 * s + 2], keptSep[s], keptId[s]);
    addPoint(out, kept[3 * b], kept[3 * b + 1], kept[3 * b + 2], keptSep[b], keptId[b]);
    if (c >= 0) addPoint(out, kept[3 * c], kept[3 * c + 1], kept[3 * c + 2], keptSep[c], keptId[c]);
    if (d >= 0) addPoint(out, kept[3 * d], kept[3 * d + 1], kept[3 * d + 2], keptSep[d], keptId[d]);
  }
  // faceContact: src/collide.js:884-945.
  NW_HD void faceContact(const Shape& ref, const Shape& inc, int axis, bool flipped, T margin, T tolerance,
                   Manifold& out) {
    const T* R = ref.axes;
    const T* I = inc.axes;
    const T* hr = ref.half;
    const T* hi = inc.half;
    const T dx = inc.center[0] - ref.center[0], dy = inc.center[1] - ref.center[1], dz = inc.center[2] - ref.center[2];
    const T s = sgn(dx * R[3 * axis] + dy * R[3 * axis + 1] + dz * R[3 * axis + 2]);
    const T nx = R[3 * axis] * s, ny = R[3 * axis + 1] * s, nz = R[3 * axis + 2] * s;
    const int refFace = 2 * axis + (s > 0 ? 1 : 0);
    int incAxis = 0;
    T best = -1;
    for (int j = 0; j < 3; j++) {
      const T d = fabs(I[3 * j] * nx + I[3 * j + 1] * ny + I[3 * j + 2] * nz);
      if (d > best) { best = d; incAxis = j; }
    }
    const T incSign = -sgn(I[3 * incAxis] * nx + I[3 * incAxis + 1] * ny + I[3 * incAxis + 2] * nz);
    const int incFace = 2 * incAxis + (incSign > 0 ? 1 : 0);
    const int p = (incAxis + 1) % 3, q = (incAxis + 2) % 3;
    const T cx = inc.center[0] + I[3 * incAxis] * incSign * hi[incAxis];
    const T cy = inc.center[1] + I[3 * incAxis + 1] * incSign * hi[incAxis];
    const T cz = inc.center[2] + I[3 * incAxis + 2] * incSign * hi[incAxis];
    for (int v = 0; v < 4; v++) {
      const T sp = corner_p(v), sq = corner_q(v);
      polyA[3 * v] = cx + I[3 * p] * sp * hi[p] + I[3 * q] * sq * hi[q];
      polyA[3 * v + 1] = cy + I[3 * p + 1] * sp * hi[p] + I[3 * q + 1] * sq * hi[q];
      polyA[3 * v + 2] = cz + I[3 * p + 2] * sp * hi[p] + I[3 * q + 2] * sq * hi[q];
      featA[v] = v;
      lineA[v] = v;
    }
    const int u = (axis + 1) % 3, w = (axis + 2) % 3;
    int count = 4, src = 0;
    for (int plane = 0; plane < 4 && count > 0; plane++) {
      const int c = plane < 2 ? u : w;
      const T side = plane % 2 == 0 ? 1 : -1;
      const T px = R[3 * c] * side, py = R[3 * c + 1] * side, pz = R[3 * c + 2] * side;
      const T offset = px * ref.center[0] + py * ref.center[1] + pz * ref.center[2] + hr[c];
      count = src == 0
        ? clipPolygon(polyA, featA, lineA, count, polyB, featB, lineB, px, py, pz, offset, plane, tolerance)
        : clipPolygon(polyB, featB, lineB, count, polyA, featA, lineA, px, py, pz, offset, plane, tolerance);
      src = 1 - src;
    }
    const T* poly = src == 0 ? polyA : polyB;
    const int* feat = src == 0 ? featA : featB;
    const T fx = ref.center[0] + nx * hr[axis], fy = ref.center[1] + ny * hr[axis], fz = ref.center[2] + nz * hr[axis];
    int n = 0;
    for (int v = 0; v < count; v++) {
      const T vx = poly[3 * v], vy = poly[3 * v + 1], vz = poly[3 * v + 2];
      const T separation = (vx - fx) * nx + (vy - fy) * ny + (vz - fz) * nz;
      if (separation > margin) continue;
      const T m = separation * 0.5;
      kept[3 * n] = vx - nx * m; kept[3 * n + 1] = vy - ny * m; kept[3 * n + 2] = vz - nz * m;
      keptSep[n] = separation;
      keptId[n] = flipped ? (static_cast<uint32_t>(incFace) << 9) | (static_cast<uint32_t>(refFace) << 6) | static_cast<uint32_t>(swapped_feature(feat[v]))
                          : (static_cast<uint32_t>(refFace) << 9) | (static_cast<uint32_t>(incFace) << 6) | static_cast<uint32_t>(feat[v]);
      n++;
    }
    if (n == 0) return;
    if (flipped) setNormal(out, -nx, -ny, -nz);
    else setNormal(out, nx, ny, nz);
    reducePoints(n, nx, ny, nz, tolerance, out);
  }
  // boxEdge: src/collide.js:1218-1229.
  NW_HD static void boxEdge(const Shape& x, int i, T nx, T ny, T nz, T* s) {
    const T* X = x.axes;
    const T* h = x.half;
    T cx = x.center[0], cy = x.center[1], cz = x.center[2];
    for (int k = 0; k < 3; k++) {
      if (k == i) continue;
      const T t = sgn(X[3 * k] * nx + X[3 * k + 1] * ny + X[3 * k + 2] * nz) * h[k];
      cx += X[3 * k] * t; cy += X[3 * k + 1] * t; cz += X[3 * k + 2] * t;
    }
    const T ex = X[3 * i] * h[i], ey = X[3 * i + 1] * h[i], ez = X[3 * i + 2] * h[i];
    s[0] = cx - ex; s[1] = cy - ey; s[2] = cz - ez;
    s[3] = cx + ex; s[4] = cy + ey; s[5] = cz + ez;
  }
  // edgeContact: src/collide.js:1201-1215.
  NW_HD void edgeContact(const Shape& a, const Shape& b, int i, int j, T nx, T ny, T nz, T margin,
                   Manifold& out) {
    boxEdge(a, i, nx, ny, nz, segA);
    boxEdge(b, j, -nx, -ny, -nz, segB);
    closestSegments(segA, segB);
    const T pax = segA[0] + (segA[3] - segA[0]) * segS, pay = segA[1] + (segA[4] - segA[1]) * segS,
                 paz = segA[2] + (segA[5] - segA[2]) * segS;
    const T pbx = segB[0] + (segB[3] - segB[0]) * segT, pby = segB[1] + (segB[4] - segB[1]) * segT,
                 pbz = segB[2] + (segB[5] - segB[2]) * segT;
    const T separation = (pbx - pax) * nx + (pby - pay) * ny + (pbz - paz) * nz;
    if (separation > margin) return;
    if (separation > 0 && (segS == 0 || segS == 1 || segT == 0 || segT == 1)) return;
    setNormal(out, nx, ny, nz);
    addPoint(out, (pax + pbx) * 0.5, (pay + pby) * 0.5, (paz + pbz) * 0.5, separation,
             (1u << 13) | static_cast<uint32_t>(3 * i + j));
  }
  // boxBox: src/collide.js:713-775.
  NW_HD void boxBox(const Shape& a, const Shape& b, T margin, T tolerance, Manifold& out) {
    const T* A = a.axes;
    const T* B = b.axes;
    const T* ha = a.half;
    const T* hb = b.half;
    const T dx = b.center[0] - a.center[0], dy = b.center[1] - a.center[1], dz = b.center[2] - a.center[2];
    T* R = cosines;
    T faceA = -INF;
    int axisA = 0;
    for (int i = 0; i < 3; i++) {
      const T nx = A[3 * i], ny = A[3 * i + 1], nz = A[3 * i + 2];
      const T r0 = fabs(B[0] * nx + B[1] * ny + B[2] * nz);
      const T r1 = fabs(B[3] * nx + B[4] * ny + B[5] * nz);
      const T r2 = fabs(B[6] * nx + B[7] * ny + B[8] * nz);
      R[3 * i] = r0; R[3 * i + 1] = r1; R[3 * i + 2] = r2;
      const T s = fabs(dx * nx + dy * ny + dz * nz) - ha[i] - (hb[0] * r0 + hb[1] * r1 + hb[2] * r2);
      if (s > margin) return;
      if (s > faceA) { faceA = s; axisA = i; }
    }
    T faceB = -INF;
    int axisB = 0;
    for (int j = 0; j < 3; j++) {
      const T nx = B[3 * j], ny = B[3 * j + 1], nz = B[3 * j + 2];
      const T s = fabs(dx * nx + dy * ny + dz * nz) - hb[j] - (ha[0] * R[j] + ha[1] * R[3 + j] + ha[2] * R[6 + j]);
      if (s > margin) return;
      if (s > faceB) { faceB = s; axisB = j; }
    }
    T edgeSep = -INF, enx = 0, eny = 0, enz = 0;
    int edgeI = -1, edgeJ = -1;
    for (int i = 0; i < 3; i++) {
      const T ux = A[3 * i], uy = A[3 * i + 1], uz = A[3 * i + 2];
      for (int j = 0; j < 3; j++) {
        const T vx = B[3 * j], vy = B[3 * j + 1], vz = B[3 * j + 2];
        const T l = normalize(uy * vz - uz * vy, uz * vx - ux * vz, ux * vy - uy * vx);
        if (!(l > PARALLEL)) continue;
        T nx = unit[0], ny = unit[1], nz = unit[2];
        const T d = dx * nx + dy * ny + dz * nz;
        if (d < 0) { nx = -nx; ny = -ny; nz = -nz; }
        const T s = fabs(d) - support(A, ha, nx, ny, nz) - support(B, hb, nx, ny, nz);
        if (s > margin) return;
        if (s > edgeSep) { edgeSep = s; edgeI = i; edgeJ = j; enx = nx; eny = ny; enz = nz; }
      }
    }
    if (edgeI >= 0 && edgeSep > jmax(faceA, faceB) + tolerance) {
      edgeContact(a, b, edgeI, edgeJ, enx, eny, enz, margin, out);
    } else if (faceB > faceA + tolerance) {
      faceContact(b, a, axisB, true, margin, tolerance, out);
    } else {
      faceContact(a, b, axisA, false, margin, tolerance, out);
    }
    if (out.count == 0 && jmax(jmax(faceA, faceB), edgeSep) > 0) boxBoxClosest(a, b, margin, out);
  }

  // pair: src/collide.js:225-242 (spheres, capsules and boxes).
  NW_HD void pair(const Shape& a, const Shape& b, T margin, T tolerance, Manifold& out) {
    if (a.kind == K_SPHERE) {
      if (b.kind == K_SPHERE) sphereSphere(a, b, margin, out);
      else if (b.kind == K_CAPSULE) sphereCapsule(a, b, margin, out);
      else sphereBox(a, b, margin, out);
    } else if (a.kind == K_CAPSULE) {
      if (b.kind == K_CAPSULE) capsuleCapsule(a, b, margin, tolerance, out);
      else capsuleBox(a, b, margin, tolerance, out);
    } else {
      boxBox(a, b, margin, tolerance, out);
    }
  }
};


}  // namespace narrow_detail

// collide(a, b, margin, tolerance, out): src/collide.js:204-218.  Returns the point count.
template <class T>
NW_HD int collideT(const ShapeT<T>& a, const ShapeT<T>& b, double margin, double tolerance, ManifoldT<T>& out) {
  narrow_detail::NarrowT<T> nw;
  out.count = 0;
  out.loss = 0;
  nw.shapeA = &a;
  nw.shapeB = &b;
  if (a.kind > b.kind) {
    nw.pair(b, a, margin, tolerance, out);
    out.normal[0] = -out.normal[0]; out.normal[1] = -out.normal[1]; out.normal[2] = -out.normal[2];
  } else {
    nw.pair(a, b, margin, tolerance, out);
  }
  return out.count;
}

}  // namespace bearing
