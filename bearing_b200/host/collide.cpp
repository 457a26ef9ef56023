// Sphere, capsule and box contacts, in the reference narrowphase's operation order
// (src/collide.js).  Each function cites the lines it follows.  The reference keeps its
// scratch in module variables; here they live in one Narrow object per call, so calls on
// different threads never share them.
#include "collide.hpp"

#include <cmath>
#include <limits>

namespace bearing {
namespace {

constexpr double INF = std::numeric_limits<double>::infinity();
constexpr double PARALLEL = 7.450580596923828e-9;   // 2^-27, src/collide.js:686

inline double sgn(double x) { return x < 0 ? -1 : 1; }                 // src/collide.js:246
inline double clamp01(double x) { return x < 0 ? 0 : x > 1 ? 1 : x; }  // src/collide.js:247

// Math.max / Math.min with JavaScript's NaN and signed-zero rules.
inline double jmax(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a > b) return a;
  if (b > a) return b;
  if (a == 0 && b == 0) return std::signbit(a) ? b : a;
  return a;
}
inline double jmin(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a < b) return a;
  if (b < a) return b;
  if (a == 0 && b == 0) return std::signbit(a) ? a : b;
  return a;
}

const int CORNER_P[4] = {-1, 1, 1, -1}, CORNER_Q[4] = {-1, -1, 1, 1};   // src/collide.js:703
const int EDGE_FROM[12] = {0, 2, 4, 6, 0, 1, 4, 5, 0, 1, 2, 3};        // src/collide.js:791
const int EDGE_TO[12] = {1, 3, 5, 7, 2, 3, 6, 7, 4, 5, 6, 7};
const int EDGE_PLANE[4] = {3, 0, 2, 1}, PLANE_EDGE[4] = {1, 3, 2, 0};  // src/collide.js:869

// SWAPPED: src/collide.js:870-877.
struct Swapped {
  uint8_t f[32];
  Swapped() {
    for (int i = 0; i < 32; i++) f[i] = static_cast<uint8_t>(i);
    for (int v = 0; v < 4; v++) {
      const int j = CORNER_P[v] > 0 ? 0 : 1, k = CORNER_Q[v] > 0 ? 2 : 3;
      f[v] = static_cast<uint8_t>(20 + 4 * j + k);
      f[20 + 4 * j + k] = static_cast<uint8_t>(v);
    }
    for (int e = 0; e < 4; e++)
      for (int k = 0; k < 4; k++) f[4 + 4 * e + k] = static_cast<uint8_t>(4 + 4 * PLANE_EDGE[k] + EDGE_PLANE[e]);
  }
};
const Swapped SWAPPED;

struct Narrow {
  const Shape* shapeA = nullptr;
  const Shape* shapeB = nullptr;
  double unit[3] = {0, 0, 0};
  double segS = 0, segT = 0;
  double segA[6], segB[6], local[6], edge[6], world[3];
  double polyA[24], polyB[24];
  int featA[8], featB[8], lineA[8], lineB[8];
  double kept[24], keptSep[8];
  uint32_t keptId[8];
  double cosines[9];
  double cornerA[24], cornerB[24];
  int FOUR[4];
  double FOOT[3];

  // normalize: src/collide.js:257-264.
  double normalize(double x, double y, double z) {
    const double m = jmax(jmax(std::fabs(x), std::fabs(y)), std::fabs(z));
    if (m == 0) return 0;
    const double sx = x / m, sy = y / m, sz = z / m;
    const double l = std::sqrt(sx * sx + sy * sy + sz * sz);
    unit[0] = sx / l; unit[1] = sy / l; unit[2] = sz / l;
    return l * m;
  }
  // perpendicular: src/collide.js:272-277.
  void perpendicular(double vx, double vy, double vz) {
    const double ax = std::fabs(vx), ay = std::fabs(vy), az = std::fabs(vz);
    if (ax <= ay && ax <= az) normalize(0, vz, -vy);
    else if (ay <= az) normalize(-vz, 0, vx);
    else normalize(vy, -vx, 0);
  }
  static void setNormal(Manifold& out, double x, double y, double z) {
    out.normal[0] = x; out.normal[1] = y; out.normal[2] = z;
  }
  static void addPoint(Manifold& out, double x, double y, double z, double separation, uint32_t id) {
    const int k = out.count++;
    out.points[3 * k] = x; out.points[3 * k + 1] = y; out.points[3 * k + 2] = z;
    out.separations[k] = separation;
    out.ids[k] = id;
  }
  // balls: src/collide.js:296-306.
  bool balls(double ax, double ay, double az, double ra, double bx, double by, double bz, double rb,
             double fx, double fy, double fz, double margin, Manifold& out, uint32_t id) {
    const double dist = normalize(bx - ax, by - ay, bz - az);
    const double separation = dist - ra - rb;
    if (separation > margin) return false;
    const double nx = dist > 0 ? unit[0] : fx, ny = dist > 0 ? unit[1] : fy, nz = dist > 0 ? unit[2] : fz;
    setNormal(out, nx, ny, nz);
    const double t = ra + separation * 0.5;
    addPoint(out, ax + nx * t, ay + ny * t, az + nz * t, separation, id);
    return true;
  }
  // segment: src/collide.js:309-313.
  static void segment(const Shape& c, double* out) {
    const double h = c.half[1];
    const double* y = c.axes;
    out[0] = c.center[0] - y[3] * h; out[1] = c.center[1] - y[4] * h; out[2] = c.center[2] - y[5] * h;
    out[3] = c.center[0] + y[3] * h; out[4] = c.center[1] + y[4] * h; out[5] = c.center[2] + y[5] * h;
  }
  // nearestOnSegment: src/collide.js:316-321.
  static double nearestOnSegment(const double* s, double x, double y, double z) {
    const double dx = s[3] - s[0], dy = s[4] - s[1], dz = s[5] - s[2];
    const double dd = dx * dx + dy * dy + dz * dz;
    if (dd == 0) return 0;
    return clamp01(((x - s[0]) * dx + (y - s[1]) * dy + (z - s[2]) * dz) / dd);
  }
  // closestSegments: src/collide.js:332-349.
  void closestSegments(const double* p, const double* q) {
    const double d1x = p[3] - p[0], d1y = p[4] - p[1], d1z = p[5] - p[2];
    const double d2x = q[3] - q[0], d2y = q[4] - q[1], d2z = q[5] - q[2];
    const double rx = p[0] - q[0], ry = p[1] - q[1], rz = p[2] - q[2];
    const double a = d1x * d1x + d1y * d1y + d1z * d1z;
    const double e = d2x * d2x + d2y * d2y + d2z * d2z;
    const double f = d2x * rx + d2y * ry + d2z * rz;
    if (a == 0 && e == 0) { segS = 0; segT = 0; return; }
    if (a == 0) { segS = 0; segT = clamp01(f / e); return; }
    const double c = d1x * rx + d1y * ry + d1z * rz;
    if (e == 0) { segT = 0; segS = clamp01(-c / a); return; }
    const double b = d1x * d2x + d1y * d2y + d1z * d2z;
    const double denom = a * e - b * b;
    double s = denom != 0 ? clamp01((b * f - c * e) / denom) : 0;
    double t = (b * s + f) / e;
    if (t < 0) { t = 0; s = clamp01(-c / a); } else if (t > 1) { t = 1; s = clamp01((b - c) / a); }
    segS = s; segT = t;
  }

  // sphereSphere: src/collide.js:353-357.
  void sphereSphere(const Shape& a, const Shape& b, double margin, Manifold& out) {
    balls(a.center[0], a.center[1], a.center[2], a.half[0], b.center[0], b.center[1], b.center[2], b.half[0],
          0, 1, 0, margin, out, 0);
  }
  // sphereCapsule: src/collide.js:361-369.
  void sphereCapsule(const Shape& a, const Shape& b, double margin, Manifold& out) {
    const double* c = a.center;
    segment(b, segB);
    const double t = nearestOnSegment(segB, c[0], c[1], c[2]);
    const double qx = segB[0] + (segB[3] - segB[0]) * t, qy = segB[1] + (segB[4] - segB[1]) * t,
                 qz = segB[2] + (segB[5] - segB[2]) * t;
    perpendicular(b.axes[3], b.axes[4], b.axes[5]);
    balls(c[0], c[1], c[2], a.half[0], qx, qy, qz, b.half[0], unit[0], unit[1], unit[2], margin, out, 0);
  }
  // sphereBox: src/collide.js:371-403.
  void sphereBox(const Shape& a, const Shape& b, double margin, Manifold& out) {
    const double* ax = b.axes;
    const double* h = b.half;
    const double r = a.half[0];
    const double dx = a.center[0] - b.center[0], dy = a.center[1] - b.center[1], dz = a.center[2] - b.center[2];
    const double lx = dx * ax[0] + dy * ax[1] + dz * ax[2];
    const double ly = dx * ax[3] + dy * ax[4] + dz * ax[5];
    const double lz = dx * ax[6] + dy * ax[7] + dz * ax[8];
    const bool inside = std::fabs(lx) <= h[0] && std::fabs(ly) <= h[1] && std::fabs(lz) <= h[2];
    if (!inside) {
      const double qx = jmax(-h[0], jmin(h[0], lx));
      const double qy = jmax(-h[1], jmin(h[1], ly));
      const double qz = jmax(-h[2], jmin(h[2], lz));
      const double wx = b.center[0] + ax[0] * qx + ax[3] * qy + ax[6] * qz;
      const double wy = b.center[1] + ax[1] * qx + ax[4] * qy + ax[7] * qz;
      const double wz = b.center[2] + ax[2] * qx + ax[5] * qy + ax[8] * qz;
      balls(a.center[0], a.center[1], a.center[2], r, wx, wy, wz, 0, 0, 1, 0, margin, out, 0);
      return;
    }
    int axis = 0;
    double depth = h[0] - std::fabs(lx);
    if (h[1] - std::fabs(ly) < depth) { axis = 1; depth = h[1] - std::fabs(ly); }
    if (h[2] - std::fabs(lz) < depth) { axis = 2; depth = h[2] - std::fabs(lz); }
    const double l = axis == 0 ? lx : axis == 1 ? ly : lz;
    const double s = -sgn(l);
    const double nx = ax[3 * axis] * s, ny = ax[3 * axis + 1] * s, nz = ax[3 * axis + 2] * s;
    setNormal(out, nx, ny, nz);
    const double separation = -(depth + r);
    const double t = r + separation * 0.5;
    addPoint(out, a.center[0] + nx * t, a.center[1] + ny * t, a.center[2] + nz * t, separation, 0);
  }

  // capsuleCapsule: src/collide.js:424-482.
  void capsuleCapsule(const Shape& a, const Shape& b, double margin, double tolerance, Manifold& out) {
    segment(a, segA);
    segment(b, segB);
    closestSegments(segA, segB);
    const double s = segS, t = segT;
    const double pax = segA[0] + (segA[3] - segA[0]) * s, pay = segA[1] + (segA[4] - segA[1]) * s,
                 paz = segA[2] + (segA[5] - segA[2]) * s;
    const double pbx = segB[0] + (segB[3] - segB[0]) * t, pby = segB[1] + (segB[4] - segB[1]) * t,
                 pbz = segB[2] + (segB[5] - segB[2]) * t;
    const double ra = a.half[0], rb = b.half[0];
    const double* ya = a.axes;
    const double* yb = b.axes;
    if (normalize(ya[4] * yb[5] - ya[5] * yb[4], ya[5] * yb[3] - ya[3] * yb[5], ya[3] * yb[4] - ya[4] * yb[3]) == 0) {
      perpendicular(ya[3], ya[4], ya[5]);
    }
    const double fx = unit[0], fy = unit[1], fz = unit[2];
    if (!balls(pax, pay, paz, ra, pbx, pby, pbz, rb, fx, fy, fz, margin, out, 0)) return;
    const double closest = out.separations[0];
    const double cx = out.points[0], cy = out.points[1], cz = out.points[2];
    out.count = 0;
    const double h = a.half[1];
    if (h > 0 && b.half[1] > 0) {
      const double k0 = (segB[0] - a.center[0]) * ya[3] + (segB[1] - a.center[1]) * ya[4] + (segB[2] - a.center[2]) * ya[5];
      const double k1 = (segB[3] - segB[0]) * ya[3] + (segB[4] - segB[1]) * ya[4] + (segB[5] - segB[2]) * ya[5];
      double u0 = 0, u1 = 1;
      if (k1 != 0) {
        const double ua = (-h - k0) / k1, ub = (h - k0) / k1;
        u0 = jmax(0, jmin(ua, ub));
        u1 = jmin(1, jmax(ua, ub));
      } else if (k0 < -h || k0 > h) {
        u1 = -1;
      }
      if (u1 > u0) {
        const double* n = out.normal;
        double deepest = INF;
        for (int e = 0; e < 2; e++) {
          const double u = e == 0 ? u0 : u1;
          const double bx = segB[0] + (segB[3] - segB[0]) * u, by = segB[1] + (segB[4] - segB[1]) * u,
                       bz = segB[2] + (segB[5] - segB[2]) * u;
          const double alongA = jmax(-h, jmin(h, k0 + k1 * u));
          const double ax = a.center[0] + ya[3] * alongA, ay = a.center[1] + ya[4] * alongA,
                       az = a.center[2] + ya[5] * alongA;
          const double gx = bx - ax, gy = by - ay, gz = bz - az;
          const double normalGap = gx * n[0] + gy * n[1] + gz * n[2];
          const double separation = normalGap - ra - rb;
          if (separation > margin) continue;
          if (gx * gx + gy * gy + gz * gz - normalGap * normalGap > tolerance * tolerance) continue;
          deepest = jmin(deepest, separation);
          const double m = ra + separation * 0.5;
          addPoint(out, ax + n[0] * m, ay + n[1] * m, az + n[2] * m, separation, static_cast<uint32_t>(1 + e));
        }
        if (out.count > 0 && closest < deepest) addPoint(out, cx, cy, cz, closest, 0);
        if (out.count > 0) return;
      }
    }
    addPoint(out, cx, cy, cz, closest, 0);
  }

  // toWorld: src/collide.js:552-557.
  void toWorld(const Shape& b, double x, double y, double z) {
    const double* ax = b.axes;
    world[0] = b.center[0] + ax[0] * x + ax[3] * y + ax[6] * z;
    world[1] = b.center[1] + ax[1] * x + ax[4] * y + ax[7] * z;
    world[2] = b.center[2] + ax[2] * x + ax[5] * y + ax[8] * z;
  }
  // segmentHitsBox: src/collide.js:560-575.
  static bool segmentHitsBox(const double* s, const double* h) {
    double t0 = 0, t1 = 1;
    for (int i = 0; i < 3; i++) {
      const double p = s[i], d = s[3 + i] - s[i];
      if (d == 0) {
        if (p < -h[i] || p > h[i]) return false;
        continue;
      }
      double ta = (-h[i] - p) / d, tb = (h[i] - p) / d;
      if (ta > tb) { const double x = ta; ta = tb; tb = x; }
      if (ta > t0) t0 = ta;
      if (tb < t1) t1 = tb;
      if (t0 > t1) return false;
    }
    return true;
  }
  // clipToFace: src/collide.js:583-615.
  bool clipToFace(const Shape& b, int axis, double facing, double r, double margin, Manifold& out, uint32_t idBase) {
    const double* h = b.half;
    const int j = (axis + 1) % 3, k = (axis + 2) % 3;
    double u0 = 0, u1 = 1;
    for (int pass = 0; pass < 2; pass++) {
      const int c = pass == 0 ? j : k;
      const double p = local[c], d = local[3 + c] - local[c];
      if (d == 0) {
        if (p < -h[c] || p > h[c]) return false;
        continue;
      }
      double ta = (-h[c] - p) / d, tb = (h[c] - p) / d;
      if (ta > tb) { const double x = ta; ta = tb; tb = x; }
      if (ta > u0) u0 = ta;
      if (tb < u1) u1 = tb;
    }
    if (u0 > u1) return false;
    const double* ax = b.axes;
    setNormal(out, -facing * ax[3 * axis], -facing * ax[3 * axis + 1], -facing * ax[3 * axis + 2]);
    const int face = 2 * axis + (facing > 0 ? 1 : 0);
    for (int e = 0; e < (u1 > u0 ? 2 : 1); e++) {
      const double u = e == 0 ? u0 : u1;
      const double px = local[0] + (local[3] - local[0]) * u, py = local[1] + (local[4] - local[1]) * u,
                   pz = local[2] + (local[5] - local[2]) * u;
      const double above = facing * (axis == 0 ? px : axis == 1 ? py : pz) - h[axis];
      const double separation = above - r;
      if (separation > margin) continue;
      const double off = facing * (separation * 0.5 - above);
      toWorld(b, axis == 0 ? px + off : px, axis == 1 ? py + off : py, axis == 2 ? pz + off : pz);
      addPoint(out, world[0], world[1], world[2], separation, idBase + static_cast<uint32_t>(4 * face + 1 + e));
    }
    return out.count > 0;
  }
  // capsuleBoxDeep: src/collide.js:626-676.
  void capsuleBoxDeep(const Shape& a, const Shape& b, double margin, double tolerance, Manifold& out) {
    const double* h = b.half;
    const double r = a.half[0];
    const double dx = local[3] - local[0], dy = local[4] - local[1], dz = local[5] - local[2];
    double bestSep = -INF, nx = 0, ny = 0, nz = 0;
    int bestAxis = -1;
    for (int c = 0; c < 6; c++) {
      double x = 0, y = 0, z = 0;
      if (c < 3) {
        if (c == 0) x = 1; else if (c == 1) y = 1; else z = 1;
      } else {
        const int e = c - 3;
        const double l = normalize(e == 0 ? 0 : e == 1 ? -dz : dy, e == 0 ? dz : e == 1 ? 0 : -dx,
                                   e == 0 ? -dy : e == 1 ? dx : 0);
        if (!(l > PARALLEL * std::sqrt(dx * dx + dy * dy + dz * dz))) continue;
        x = unit[0]; y = unit[1]; z = unit[2];
      }
      const double support = h[0] * std::fabs(x) + h[1] * std::fabs(y) + h[2] * std::fabs(z);
      const double p0 = local[0] * x + local[1] * y + local[2] * z, p1 = local[3] * x + local[4] * y + local[5] * z;
      const double lo = jmin(p0, p1), hi = jmax(p0, p1);
      const double plus = lo - support, minus = -support - hi;
      const double sep = jmax(plus, minus) - r;
      if (sep > bestSep + (c >= 3 && bestAxis < 3 ? tolerance : 0)) {
        bestSep = sep; bestAxis = c;
        const double s = plus >= minus ? -1 : 1;
        nx = x * s; ny = y * s; nz = z * s;
      }
    }
    if (bestAxis < 3) {
      const double facing = -(bestAxis == 0 ? nx : bestAxis == 1 ? ny : nz);
      clipToFace(b, bestAxis, sgn(facing), r, margin, out, 0);
      return;
    }
    const int i = bestAxis - 3, j = (i + 1) % 3, k = (i + 2) % 3;
    const double mj = j == 0 ? -nx : j == 1 ? -ny : -nz, mk = k == 0 ? -nx : k == 1 ? -ny : -nz;
    edge[i] = -h[i]; edge[3 + i] = h[i];
    edge[j] = edge[3 + j] = sgn(mj) * h[j];
    edge[k] = edge[3 + k] = sgn(mk) * h[k];
    closestSegments(local, edge);
    const double px = local[0] + dx * segS, py = local[1] + dy * segS, pz = local[2] + dz * segS;
    const double ex = edge[0] + (edge[3] - edge[0]) * segT, ey = edge[1] + (edge[4] - edge[1]) * segT,
                 ez = edge[2] + (edge[5] - edge[2]) * segT;
    const double separation = (ex - px) * nx + (ey - py) * ny + (ez - pz) * nz - r;
    const double* ax = b.axes;
    setNormal(out, ax[0] * nx + ax[3] * ny + ax[6] * nz, ax[1] * nx + ax[4] * ny + ax[7] * nz,
              ax[2] * nx + ax[5] * ny + ax[8] * nz);
    const double mm = r + separation * 0.5;
    toWorld(b, px + nx * mm, py + ny * mm, pz + nz * mm);
    addPoint(out, world[0], world[1], world[2], separation, static_cast<uint32_t>(32 + i));
  }
  // capsuleBox: src/collide.js:497-547.
  void capsuleBox(const Shape& a, const Shape& b, double margin, double tolerance, Manifold& out) {
    segment(a, segA);
    const double* bx = b.axes;
    const double* h = b.half;
    const double r = a.half[0];
    for (int e = 0; e < 2; e++) {
      const double dx = segA[3 * e] - b.center[0], dy = segA[3 * e + 1] - b.center[1], dz = segA[3 * e + 2] - b.center[2];
      local[3 * e] = dx * bx[0] + dy * bx[1] + dz * bx[2];
      local[3 * e + 1] = dx * bx[3] + dy * bx[4] + dz * bx[5];
      local[3 * e + 2] = dx * bx[6] + dy * bx[7] + dz * bx[8];
    }
    if (segmentHitsBox(local, h)) { capsuleBoxDeep(a, b, margin, tolerance, out); return; }
    double best = INF, sx = 0, sy = 0, sz = 0, qx = 0, qy = 0, qz = 0;
    for (int e = 0; e < 2; e++) {
      const double px = local[3 * e], py = local[3 * e + 1], pz = local[3 * e + 2];
      const double cx = jmax(-h[0], jmin(h[0], px)), cy = jmax(-h[1], jmin(h[1], py)), cz = jmax(-h[2], jmin(h[2], pz));
      const double d = (px - cx) * (px - cx) + (py - cy) * (py - cy) + (pz - cz) * (pz - cz);
      if (d < best) { best = d; sx = px; sy = py; sz = pz; qx = cx; qy = cy; qz = cz; }
    }
    for (int i = 0; i < 3; i++) {
      const int j = (i + 1) % 3, k = (i + 2) % 3;
      for (int c = 0; c < 4; c++) {
        edge[i] = -h[i]; edge[3 + i] = h[i];
        edge[j] = edge[3 + j] = (c & 1) ? h[j] : -h[j];
        edge[k] = edge[3 + k] = (c & 2) ? h[k] : -h[k];
        closestSegments(local, edge);
        const double px = local[0] + (local[3] - local[0]) * segS, py = local[1] + (local[4] - local[1]) * segS,
                     pz = local[2] + (local[5] - local[2]) * segS;
        const double ex = edge[0] + (edge[3] - edge[0]) * segT, ey = edge[1] + (edge[4] - edge[1]) * segT,
                     ez = edge[2] + (edge[5] - edge[2]) * segT;
        const double d = (px - ex) * (px - ex) + (py - ey) * (py - ey) + (pz - ez) * (pz - ez);
        if (d < best) { best = d; sx = px; sy = py; sz = pz; qx = ex; qy = ey; qz = ez; }
      }
    }
    const double dist = normalize(qx - sx, qy - sy, qz - sz);
    if (dist - r > margin) return;
    const double nlx = unit[0], nly = unit[1], nlz = unit[2];
    setNormal(out, bx[0] * nlx + bx[3] * nly + bx[6] * nlz, bx[1] * nlx + bx[4] * nly + bx[7] * nlz,
              bx[2] * nlx + bx[5] * nly + bx[8] * nlz);
    const bool onX = std::fabs(qx) == h[0], onY = std::fabs(qy) == h[1], onZ = std::fabs(qz) == h[2];
    if (static_cast<int>(onX) + static_cast<int>(onY) + static_cast<int>(onZ) == 1) {
      const int axis = onX ? 0 : onY ? 1 : 2;
      const double facing = sgn(axis == 0 ? qx : axis == 1 ? qy : qz);
      if (clipToFace(b, axis, facing, r, margin, out, 0)) return;
    }
    const double separation = dist - r;
    const double m = r + separation * 0.5;
    toWorld(b, sx + nlx * m, sy + nly * m, sz + nlz * m);
    addPoint(out, world[0], world[1], world[2], separation, 0);
  }

  // support: src/collide.js:840-844.
  static double support(const double* X, const double* h, double nx, double ny, double nz) {
    return h[0] * std::fabs(X[0] * nx + X[1] * ny + X[2] * nz)
      + h[1] * std::fabs(X[3] * nx + X[4] * ny + X[5] * nz)
      + h[2] * std::fabs(X[6] * nx + X[7] * ny + X[8] * nz);
  }
  // corners: src/collide.js:780-788.
  static void corners(const Shape& x, double* c) {
    const double* X = x.axes;
    const double* h = x.half;
    for (int k = 0; k < 8; k++) {
      const double sx = (k & 1) ? h[0] : -h[0], sy = (k & 2) ? h[1] : -h[1], sz = (k & 4) ? h[2] : -h[2];
      c[3 * k] = x.center[0] + X[0] * sx + X[3] * sy + X[6] * sz;
      c[3 * k + 1] = x.center[1] + X[1] * sx + X[4] * sy + X[7] * sz;
      c[3 * k + 2] = x.center[2] + X[2] * sx + X[5] * sy + X[8] * sz;
    }
  }
  // boxBoxClosest: src/collide.js:800-837.
  void boxBoxClosest(const Shape& a, const Shape& b, double margin, Manifold& out) {
    corners(a, cornerA);
    corners(b, cornerB);
    double best = INF, ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0;
    for (int side = 0; side < 2; side++) {
      const double* from = side == 0 ? cornerA : cornerB;
      const Shape& box = side == 0 ? b : a;
      const double* X = box.axes;
      const double* h = box.half;
      for (int k = 0; k < 8; k++) {
        const double dx = from[3 * k] - box.center[0], dy = from[3 * k + 1] - box.center[1], dz = from[3 * k + 2] - box.center[2];
        const double lx = jmax(-h[0], jmin(h[0], dx * X[0] + dy * X[1] + dz * X[2]));
        const double ly = jmax(-h[1], jmin(h[1], dx * X[3] + dy * X[4] + dz * X[5]));
        const double lz = jmax(-h[2], jmin(h[2], dx * X[6] + dy * X[7] + dz * X[8]));
        toWorld(box, lx, ly, lz);
        const double ex = world[0] - from[3 * k], ey = world[1] - from[3 * k + 1], ez = world[2] - from[3 * k + 2];
        const double d = ex * ex + ey * ey + ez * ez;
        if (d < best) {
          best = d;
          if (side == 0) { ax = from[3 * k]; ay = from[3 * k + 1]; az = from[3 * k + 2]; bx = world[0]; by = world[1]; bz = world[2]; }
          else { bx = from[3 * k]; by = from[3 * k + 1]; bz = from[3 * k + 2]; ax = world[0]; ay = world[1]; az = world[2]; }
        }
      }
    }
    for (int i = 0; i < 12; i++) {
      for (int k = 0; k < 3; k++) { segA[k] = cornerA[3 * EDGE_FROM[i] + k]; segA[3 + k] = cornerA[3 * EDGE_TO[i] + k]; }
      for (int j = 0; j < 12; j++) {
        for (int k = 0; k < 3; k++) { segB[k] = cornerB[3 * EDGE_FROM[j] + k]; segB[3 + k] = cornerB[3 * EDGE_TO[j] + k]; }
        closestSegments(segA, segB);
        const double px = segA[0] + (segA[3] - segA[0]) * segS, py = segA[1] + (segA[4] - segA[1]) * segS,
                     pz = segA[2] + (segA[5] - segA[2]) * segS;
        const double qx = segB[0] + (segB[3] - segB[0]) * segT, qy = segB[1] + (segB[4] - segB[1]) * segT,
                     qz = segB[2] + (segB[5] - segB[2]) * segT;
        const double d = (qx - px) * (qx - px) + (qy - py) * (qy - py) + (qz - pz) * (qz - pz);
        if (d < best) { best = d; ax = px; ay = py; az = pz; bx = qx; by = qy; bz = qz; }
      }
    }
    const double dist = normalize(bx - ax, by - ay, bz - az);
    if (dist > margin || dist == 0) return;
    setNormal(out, unit[0], unit[1], unit[2]);
    addPoint(out, (ax + bx) * 0.5, (ay + by) * 0.5, (az + bz) * 0.5, dist, 1u << 14);
  }

  // clipPolygon: src/collide.js:966-999.
  static int clipPolygon(const double* src, const int* sf, const int* sl, int count, double* dst, int* df, int* dl,
                         double px, double py, double pz, double offset, int plane, double slack) {
    int n = 0;
    for (int v = 0; v < count; v++) {
      const int w = (v + 1) % count;
      const double ax = src[3 * v], ay = src[3 * v + 1], az = src[3 * v + 2];
      const double bx = src[3 * w], by = src[3 * w + 1], bz = src[3 * w + 2];
      const double da = ax * px + ay * py + az * pz - offset, db = bx * px + by * py + bz * pz - offset;
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
        const double t = da / (da - db);
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
  void four(int n, int a, double nx, double ny, double nz, double pressed, double touching) {
    int b = -1;
    double far = -1;
    for (int pass = 0; pass < 3 && b < 0; pass++) {
      const double within = pass == 0 ? pressed : pass == 1 ? touching : INF;
      for (int k = 0; k < n; k++) {
        if (k == a || keptSep[k] > within) continue;
        const double x = kept[3 * k] - kept[3 * a], y = kept[3 * k + 1] - kept[3 * a + 1], z = kept[3 * k + 2] - kept[3 * a + 2];
        const double d = x * x + y * y + z * z;
        if (d > far) { far = d; b = k; }
      }
    }
    int c = -1, d = -1;
    double most = 0, least = 0;
    const double abx = kept[3 * b] - kept[3 * a], aby = kept[3 * b + 1] - kept[3 * a + 1], abz = kept[3 * b + 2] - kept[3 * a + 2];
    for (int pass = 0; pass < 3 && (c < 0 || d < 0); pass++) {
      const double within = pass == 0 ? pressed : pass == 1 ? touching : INF;
      const bool left = c < 0, right = d < 0;
      for (int k = 0; k < n; k++) {
        if (k == a || k == b || keptSep[k] > within) continue;
        const double x = kept[3 * k] - kept[3 * a], y = kept[3 * k + 1] - kept[3 * a + 1], z = kept[3 * k + 2] - kept[3 * a + 2];
        const double area = (aby * z - abz * y) * nx + (abz * x - abx * z) * ny + (abx * y - aby * x) * nz;
        if (left && area > most) { most = area; c = k; }
        if (right && area < least) { least = area; d = k; }
      }
    }
    FOUR[0] = a; FOUR[1] = d; FOUR[2] = b; FOUR[3] = c;
  }
  // foot: src/collide.js:1171-1178.
  bool foot(const Shape& s, double nx, double ny, double nz) {
    const double* w = s.weight;
    const double* c = s.center;
    const double alongN = w[0] * nx + w[1] * ny + w[2] * nz;
    const int o = FOUR[0];
    if (alongN == 0) return false;
    const double t = ((kept[3 * o] - c[0]) * nx + (kept[3 * o + 1] - c[1]) * ny + (kept[3 * o + 2] - c[2]) * nz) / alongN;
    if (!(t > 0)) return false;
    FOOT[0] = c[0] + w[0] * t; FOOT[1] = c[1] + w[1] * t; FOOT[2] = c[2] + w[2] * t;
    return true;
  }
  // rests: src/collide.js:1151-1164.
  bool rests(const Shape& s, double nx, double ny, double nz) {
    if (!foot(s, nx, ny, nz)) return false;
    const double px = FOOT[0], py = FOOT[1], pz = FOOT[2];
    int from = FOUR[0];
    for (int e = 1; e <= 4; e++) {
      const int to = FOUR[e & 3];
      if (to < 0) continue;
      const double ax = kept[3 * from] - px, ay = kept[3 * from + 1] - py, az = kept[3 * from + 2] - pz;
      const double bx = kept[3 * to] - px, by = kept[3 * to + 1] - py, bz = kept[3 * to + 2] - pz;
      if ((ay * bz - az * by) * nx + (az * bx - ax * bz) * ny + (ax * by - ay * bx) * nz < 0) return false;
      from = to;
    }
    return true;
  }
  // under: src/collide.js:1185-1194.
  int under(int n, double nx, double ny, double nz, double pressed) {
    int start = -1;
    double nearest = INF;
    for (int k = 0; k < n; k++) {
      if (keptSep[k] > pressed) continue;
      const double x = kept[3 * k] - FOOT[0], y = kept[3 * k + 1] - FOOT[1], z = kept[3 * k + 2] - FOOT[2],
                   alongN = x * nx + y * ny + z * nz;
      const double d = x * x + y * y + z * z - alongN * alongN;
      if (d < nearest) { nearest = d; start = k; }
    }
    return start;
  }
  // reducePoints: src/collide.js:1077-1104.
  void reducePoints(int n, double nx, double ny, double nz, double tolerance, Manifold& out) {
    if (n <= MAX_POINTS) {
      for (int k = 0; k < n; k++) addPoint(out, kept[3 * k], kept[3 * k + 1], kept[3 * k + 2], keptSep[k], keptId[k]);
      return;
    }
    double deepest = keptSep[0];
    int deep = 0;
    for (int k = 1; k < n; k++) if (keptSep[k] < deepest) { deepest = keptSep[k]; deep = k; }
    const double pressed = jmax(deepest, 0), touching = pressed + tolerance;
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
  void faceContact(const Shape& ref, const Shape& inc, int axis, bool flipped, double margin, double tolerance,
                   Manifold& out) {
    const double* R = ref.axes;
    const double* I = inc.axes;
    const double* hr = ref.half;
    const double* hi = inc.half;
    const double dx = inc.center[0] - ref.center[0], dy = inc.center[1] - ref.center[1], dz = inc.center[2] - ref.center[2];
    const double s = sgn(dx * R[3 * axis] + dy * R[3 * axis + 1] + dz * R[3 * axis + 2]);
    const double nx = R[3 * axis] * s, ny = R[3 * axis + 1] * s, nz = R[3 * axis + 2] * s;
    const int refFace = 2 * axis + (s > 0 ? 1 : 0);
    int incAxis = 0;
    double best = -1;
    for (int j = 0; j < 3; j++) {
      const double d = std::fabs(I[3 * j] * nx + I[3 * j + 1] * ny + I[3 * j + 2] * nz);
      if (d > best) { best = d; incAxis = j; }
    }
    const double incSign = -sgn(I[3 * incAxis] * nx + I[3 * incAxis + 1] * ny + I[3 * incAxis + 2] * nz);
    const int incFace = 2 * incAxis + (incSign > 0 ? 1 : 0);
    const int p = (incAxis + 1) % 3, q = (incAxis + 2) % 3;
    const double cx = inc.center[0] + I[3 * incAxis] * incSign * hi[incAxis];
    const double cy = inc.center[1] + I[3 * incAxis + 1] * incSign * hi[incAxis];
    const double cz = inc.center[2] + I[3 * incAxis + 2] * incSign * hi[incAxis];
    for (int v = 0; v < 4; v++) {
      const double sp = CORNER_P[v], sq = CORNER_Q[v];
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
      const double side = plane % 2 == 0 ? 1 : -1;
      const double px = R[3 * c] * side, py = R[3 * c + 1] * side, pz = R[3 * c + 2] * side;
      const double offset = px * ref.center[0] + py * ref.center[1] + pz * ref.center[2] + hr[c];
      count = src == 0
        ? clipPolygon(polyA, featA, lineA, count, polyB, featB, lineB, px, py, pz, offset, plane, tolerance)
        : clipPolygon(polyB, featB, lineB, count, polyA, featA, lineA, px, py, pz, offset, plane, tolerance);
      src = 1 - src;
    }
    const double* poly = src == 0 ? polyA : polyB;
    const int* feat = src == 0 ? featA : featB;
    const double fx = ref.center[0] + nx * hr[axis], fy = ref.center[1] + ny * hr[axis], fz = ref.center[2] + nz * hr[axis];
    int n = 0;
    for (int v = 0; v < count; v++) {
      const double vx = poly[3 * v], vy = poly[3 * v + 1], vz = poly[3 * v + 2];
      const double separation = (vx - fx) * nx + (vy - fy) * ny + (vz - fz) * nz;
      if (separation > margin) continue;
      const double m = separation * 0.5;
      kept[3 * n] = vx - nx * m; kept[3 * n + 1] = vy - ny * m; kept[3 * n + 2] = vz - nz * m;
      keptSep[n] = separation;
      keptId[n] = flipped ? (static_cast<uint32_t>(incFace) << 9) | (static_cast<uint32_t>(refFace) << 6) | SWAPPED.f[feat[v]]
                          : (static_cast<uint32_t>(refFace) << 9) | (static_cast<uint32_t>(incFace) << 6) | static_cast<uint32_t>(feat[v]);
      n++;
    }
    if (n == 0) return;
    if (flipped) setNormal(out, -nx, -ny, -nz);
    else setNormal(out, nx, ny, nz);
    reducePoints(n, nx, ny, nz, tolerance, out);
  }
  // boxEdge: src/collide.js:1218-1229.
  static void boxEdge(const Shape& x, int i, double nx, double ny, double nz, double* s) {
    const double* X = x.axes;
    const double* h = x.half;
    double cx = x.center[0], cy = x.center[1], cz = x.center[2];
    for (int k = 0; k < 3; k++) {
      if (k == i) continue;
      const double t = sgn(X[3 * k] * nx + X[3 * k + 1] * ny + X[3 * k + 2] * nz) * h[k];
      cx += X[3 * k] * t; cy += X[3 * k + 1] * t; cz += X[3 * k + 2] * t;
    }
    const double ex = X[3 * i] * h[i], ey = X[3 * i + 1] * h[i], ez = X[3 * i + 2] * h[i];
    s[0] = cx - ex; s[1] = cy - ey; s[2] = cz - ez;
    s[3] = cx + ex; s[4] = cy + ey; s[5] = cz + ez;
  }
  // edgeContact: src/collide.js:1201-1215.
  void edgeContact(const Shape& a, const Shape& b, int i, int j, double nx, double ny, double nz, double margin,
                   Manifold& out) {
    boxEdge(a, i, nx, ny, nz, segA);
    boxEdge(b, j, -nx, -ny, -nz, segB);
    closestSegments(segA, segB);
    const double pax = segA[0] + (segA[3] - segA[0]) * segS, pay = segA[1] + (segA[4] - segA[1]) * segS,
                 paz = segA[2] + (segA[5] - segA[2]) * segS;
    const double pbx = segB[0] + (segB[3] - segB[0]) * segT, pby = segB[1] + (segB[4] - segB[1]) * segT,
                 pbz = segB[2] + (segB[5] - segB[2]) * segT;
    const double separation = (pbx - pax) * nx + (pby - pay) * ny + (pbz - paz) * nz;
    if (separation > margin) return;
    if (separation > 0 && (segS == 0 || segS == 1 || segT == 0 || segT == 1)) return;
    setNormal(out, nx, ny, nz);
    addPoint(out, (pax + pbx) * 0.5, (pay + pby) * 0.5, (paz + pbz) * 0.5, separation,
             (1u << 13) | static_cast<uint32_t>(3 * i + j));
  }
  // boxBox: src/collide.js:713-775.
  void boxBox(const Shape& a, const Shape& b, double margin, double tolerance, Manifold& out) {
    const double* A = a.axes;
    const double* B = b.axes;
    const double* ha = a.half;
    const double* hb = b.half;
    const double dx = b.center[0] - a.center[0], dy = b.center[1] - a.center[1], dz = b.center[2] - a.center[2];
    double* R = cosines;
    double faceA = -INF;
    int axisA = 0;
    for (int i = 0; i < 3; i++) {
      const double nx = A[3 * i], ny = A[3 * i + 1], nz = A[3 * i + 2];
      const double r0 = std::fabs(B[0] * nx + B[1] * ny + B[2] * nz);
      const double r1 = std::fabs(B[3] * nx + B[4] * ny + B[5] * nz);
      const double r2 = std::fabs(B[6] * nx + B[7] * ny + B[8] * nz);
      R[3 * i] = r0; R[3 * i + 1] = r1; R[3 * i + 2] = r2;
      const double s = std::fabs(dx * nx + dy * ny + dz * nz) - ha[i] - (hb[0] * r0 + hb[1] * r1 + hb[2] * r2);
      if (s > margin) return;
      if (s > faceA) { faceA = s; axisA = i; }
    }
    double faceB = -INF;
    int axisB = 0;
    for (int j = 0; j < 3; j++) {
      const double nx = B[3 * j], ny = B[3 * j + 1], nz = B[3 * j + 2];
      const double s = std::fabs(dx * nx + dy * ny + dz * nz) - hb[j] - (ha[0] * R[j] + ha[1] * R[3 + j] + ha[2] * R[6 + j]);
      if (s > margin) return;
      if (s > faceB) { faceB = s; axisB = j; }
    }
    double edgeSep = -INF, enx = 0, eny = 0, enz = 0;
    int edgeI = -1, edgeJ = -1;
    for (int i = 0; i < 3; i++) {
      const double ux = A[3 * i], uy = A[3 * i + 1], uz = A[3 * i + 2];
      for (int j = 0; j < 3; j++) {
        const double vx = B[3 * j], vy = B[3 * j + 1], vz = B[3 * j + 2];
        const double l = normalize(uy * vz - uz * vy, uz * vx - ux * vz, ux * vy - uy * vx);
        if (!(l > PARALLEL)) continue;
        double nx = unit[0], ny = unit[1], nz = unit[2];
        const double d = dx * nx + dy * ny + dz * nz;
        if (d < 0) { nx = -nx; ny = -ny; nz = -nz; }
        const double s = std::fabs(d) - support(A, ha, nx, ny, nz) - support(B, hb, nx, ny, nz);
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
  void pair(const Shape& a, const Shape& b, double margin, double tolerance, Manifold& out) {
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

}  // namespace

int collide(const Shape& a, const Shape& b, double margin, double tolerance, Manifold& out) {
  Narrow nw;
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
