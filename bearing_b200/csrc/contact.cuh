// A step's contacts kept on the device, from the pair list to the stored contact memory: the rows
// a step's manifolds become (src/contact.js:889-921 emit, 1283-1292 basis, 999-1036 carry,
// 1318-1329 rest), the order the solve stage takes them in, and what store() keeps of them for the
// next step (src/contact.js:1067-1115 store/keep, 2178-2213 touched).  bg_contact_step
// (bearing_gpu.cu) runs these around the narrowphase (bg_collide's kernels), the colouring
// (colour.cuh) and the solve stage (stage.cuh).
//
// Every value is worked out with the host's expressions in the host's order (the library is
// built with -fmad=false), so the rows, and with them the solve, are the host path's to the bit.
//
// The contact memory (src/pairs.js:50-58: a pair's remembered point count, point ids and normal
// impulses, and its friction, twist and slip as world vectors) is kept as one record per pair of
// the last call's list, in two banks: the call reads the last call's bank and writes the other.
// With reuse on, a record also keeps the pair's manifold and touching flag (src/pairs.js:55-80),
// and a pair whose kept manifold still holds by REUSE's rules (src/contact.js:388-537) takes it
// rebuilt from the bodies' poses instead of a fresh one from the narrowphase (ct_reuse).
#pragma once

#include <stdint.h>

namespace bgct {

constexpr int P = 4;
constexpr double PIXEL = 1.0 / 200.0;   // src/contact.js:125
constexpr uint8_t kDynamic = 0;
constexpr int kOverflow = 32, kResting = 33;
// The solve order's keys: colour k < 32 and point count c give 4k + c - 1; the overflow run 128,
// the resting run 129.
constexpr int kKeys = 130;
constexpr int kOrderThreads = 1024;   // one block a tile, one row a thread

// Math.max / Math.min (NaN first, -0 below +0), as the host's jmax / jmin.
__device__ __forceinline__ double ct_max(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a > b) return a;
  if (b > a) return b;
  if (a == 0 && b == 0) return signbit(a) ? b : a;
  return a;
}
__device__ __forceinline__ double ct_min(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a < b) return a;
  if (b < a) return b;
  if (a == 0 && b == 0) return signbit(a) ? a : b;
  return a;
}

// One bank of contact memory, `cap` records: what the pair remembers for carry() (src/pairs.js:
// 50-58), its touching flag, and the manifold it keeps for reused() (src/pairs.js:55-80).
struct Memory {
  uint8_t* points;    // remembered point count (0: nothing remembered)
  uint32_t* pid;      // P per record
  double* ni;         // P per record: normal impulses
  double* friction;   // 3 per record
  double* twist;      // 3 per record
  double* slip;       // 3 per record
  uint8_t* touching;  // touched()'s flag as of the call that wrote the record
  uint8_t* cached;    // 1: a kept manifold follows
  uint8_t* cache_points;
  double* pose;       // 7 per record: the pose it was found at (relative())
  double* loss;
  double* local_normal;   // 3 per record: its normal in a's frame
  double* local;      // 6 P per record: each point's end on a (a's frame) and on b (b's frame)
  uint32_t* cache_id; // P per record
};

// ---- the kept manifold: src/contact.js:388-595 (REUSE) ----

// What the reuse rules read of a body, besides the pair's record.
struct Poses {
  const double *p, *q, *v, *w, *dims, *reach, *gscale;
  const uint8_t *type, *shape;
  const int32_t* joint_head;
  double gravity[3];
  double dt;
};

// axesOf: src/core/math.js:222-227.
__device__ __forceinline__ void ct_axes(const double* q, double* ax) {
  const double x = q[0], y = q[1], z = q[2], w = q[3];
  ax[0] = 1 - 2 * (y * y + z * z); ax[1] = 2 * (x * y + z * w); ax[2] = 2 * (x * z - y * w);
  ax[3] = 2 * (x * y - z * w); ax[4] = 1 - 2 * (x * x + z * z); ax[5] = 2 * (y * z + x * w);
  ax[6] = 2 * (x * z + y * w); ax[7] = 2 * (y * z - x * w); ax[8] = 1 - 2 * (x * x + y * y);
}

// relative(): src/contact.js:596-610.  Returns the smaller body.
__device__ __forceinline__ int ct_relative(const Poses& s, int a, int b, double* pose) {
  const int h = s.reach[a] >= s.reach[b] ? a : b, g = h == a ? b : a;
  double A[9];
  ct_axes(s.q + 4 * h, A);
  const double dx = s.p[3 * g] - s.p[3 * h], dy = s.p[3 * g + 1] - s.p[3 * h + 1], dz = s.p[3 * g + 2] - s.p[3 * h + 2];
  pose[0] = A[0] * dx + A[1] * dy + A[2] * dz;
  pose[1] = A[3] * dx + A[4] * dy + A[5] * dz;
  pose[2] = A[6] * dx + A[7] * dy + A[8] * dz;
  const double ax = -s.q[4 * h], ay = -s.q[4 * h + 1], az = -s.q[4 * h + 2], aw = s.q[4 * h + 3];
  const double bx = s.q[4 * g], by = s.q[4 * g + 1], bz = s.q[4 * g + 2], bw = s.q[4 * g + 3];
  pose[3] = aw * bx + ax * bw + ay * bz - az * by;
  pose[4] = aw * by + ay * bw + az * bx - ax * bz;
  pose[5] = aw * bz + az * bw + ax * by - ay * bx;
  pose[6] = aw * bw - ax * bx - ay * by - az * bz;
  return g;
}

// moving(): src/contact.js:695-703.
__device__ __forceinline__ double ct_moving(const Poses& s, int a, int b) {
  const int a3 = 3 * a, b3 = 3 * b;
  const double ga = s.type[a] == kDynamic ? s.gscale[a] : 0, gb = s.type[b] == kDynamic ? s.gscale[b] : 0;
  const double dx = s.v[b3] - s.v[a3], dy = s.v[b3 + 1] - s.v[a3 + 1], dz = s.v[b3 + 2] - s.v[a3 + 2];
  const double gs = gb - ga;
  const double gl = sqrt(s.gravity[0] * s.gravity[0] + s.gravity[1] * s.gravity[1] + s.gravity[2] * s.gravity[2]) * fabs(gs);
  const double* w = s.w;
  const double turning = sqrt(w[a3] * w[a3] + w[a3 + 1] * w[a3 + 1] + w[a3 + 2] * w[a3 + 2]) * s.reach[a]
    + sqrt(w[b3] * w[b3] + w[b3 + 1] * w[b3 + 1] + w[b3 + 2] * w[b3 + 2]) * s.reach[b];
  return (sqrt(dx * dx + dy * dy + dz * dz) + 0.5 * gl * s.dt + turning) * s.dt;
}

// keeps(): src/contact.js:516-537, for record j.
__device__ __forceinline__ bool ct_keeps(const Poses& s, const Memory& m, int j, int a, int b, double tolerance) {
  const double* pose = m.pose + 7 * j;
  double now[7];
  const int g = ct_relative(s, a, b, now);
  const double ex = now[0] - pose[0], ey = now[1] - pose[1], ez = now[2] - pose[2];
  const double cx = -pose[3], cy = -pose[4], cz = -pose[5], cw = pose[6];
  const double rx = now[3], ry = now[4], rz = now[5], rw = now[6];
  const double ux = cw * rx + cx * rw + cy * rz - cz * ry;
  const double uy = cw * ry + cy * rw + cz * rx - cx * rz;
  const double uz = cw * rz + cz * rw + cx * ry - cy * rx;
  const double drift = sqrt(ex * ex + ey * ey + ez * ez) + 2 * sqrt(ux * ux + uy * uy + uz * uz) * s.reach[g];
  if (m.loss[j] + 2 * drift > tolerance) return false;
  if (s.joint_head[a] != 0 || s.joint_head[b] != 0) return false;
  return m.touching[j] == 1 || drift + ct_moving(s, a, b) <= tolerance;
}

// rounded(): src/contact.js:571-575.
__device__ __forceinline__ double ct_rounded(const Poses& s, int x) {
  return s.shape[x] == BG_SPHERE || s.shape[x] == BG_CAPSULE ? s.dims[3 * x] : 0;
}

// cored(): src/contact.js:578-585.
__device__ __forceinline__ void ct_cored(const Poses& s, int x, double* local) {
  if (s.shape[x] == BG_SPHERE) { local[0] = 0; local[1] = 0; local[2] = 0; return; }
  if (s.shape[x] != BG_CAPSULE) return;
  const double half = (s.dims[3 * x + 1] - 2 * s.dims[3 * x]) * 0.5, y = local[1];
  local[0] = 0; local[1] = y < -half ? -half : y > half ? half : y; local[2] = 0;
}

struct ReuseParams {
  int32_t np;
  const int32_t *a, *b;
  const double *margin, *tol;
  const int32_t* memory;
  Poses s;
  Memory old;
  uint8_t* kept;                    // per pair: 1 if its manifold was reused
  uint8_t* points;                  // the manifolds, per pair (kept ones written here)
  double *normal, *point, *separation;
  uint32_t* pid;
};

// reused() (src/contact.js:468-510, never shifted) for each pair with a kept manifold: the manifold
// rebuilt from the bodies' poses now, or not kept (the narrowphase then finds it afresh).
__global__ void ct_reuse(ReuseParams r) {
  const Poses& s = r.s;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.np; i += gridDim.x * blockDim.x) {
    r.kept[i] = 0;
    const int j = r.memory[i];
    if (j < 0 || r.old.cached[j] == 0) continue;
    const int a = r.a[i], b = r.b[i];
    if (!ct_keeps(s, r.old, j, a, b, r.tol[i])) continue;
    const int count = r.old.cache_points[j];
    double A[9], Bx[9];
    ct_axes(s.q + 4 * a, A);
    ct_axes(s.q + 4 * b, Bx);
    const double* ln = r.old.local_normal + 3 * j;
    const double lx = ln[0], ly = ln[1], lz = ln[2];
    const double nx = A[0] * lx + A[3] * ly + A[6] * lz;
    const double ny = A[1] * lx + A[4] * ly + A[7] * lz;
    const double nz = A[2] * lx + A[5] * ly + A[8] * lz;
    const double ra = ct_rounded(s, a), rb = -ct_rounded(s, b);
    const double* pa0 = s.p + 3 * a;
    const double* pb0 = s.p + 3 * b;
    double sep[P], pt[3 * P];
    double least = __longlong_as_double(0x7ff0000000000000LL);   // +Infinity
    for (int k = 0; k < count; k++) {
      const double* l = r.old.local + 6 * (P * j + k);
      const double ax = l[0], ay = l[1], az = l[2], bx = l[3], by = l[4], bz = l[5];
      const double pax = pa0[0] + A[0] * ax + A[3] * ay + A[6] * az + nx * ra;
      const double pay = pa0[1] + A[1] * ax + A[4] * ay + A[7] * az + ny * ra;
      const double paz = pa0[2] + A[2] * ax + A[5] * ay + A[8] * az + nz * ra;
      const double pbx = pb0[0] + Bx[0] * bx + Bx[3] * by + Bx[6] * bz + nx * rb;
      const double pby = pb0[1] + Bx[1] * bx + Bx[4] * by + Bx[7] * bz + ny * rb;
      const double pbz = pb0[2] + Bx[2] * bx + Bx[5] * by + Bx[8] * bz + nz * rb;
      const double sp = (pbx - pax) * nx + (pby - pay) * ny + (pbz - paz) * nz, half = 0.5 * sp;
      sep[k] = sp;
      if (rb != 0) {
        pt[3 * k] = pbx - nx * half; pt[3 * k + 1] = pby - ny * half; pt[3 * k + 2] = pbz - nz * half;
      } else if (ra != 0) {
        pt[3 * k] = pax + nx * half; pt[3 * k + 1] = pay + ny * half; pt[3 * k + 2] = paz + nz * half;
      } else {
        pt[3 * k] = (pax + pbx) * 0.5; pt[3 * k + 1] = (pay + pby) * 0.5; pt[3 * k + 2] = (paz + pbz) * 0.5;
      }
      if (sp < least) least = sp;
    }
    if (least > r.margin[i]) continue;   // least(): src/contact.js:684-688
    r.kept[i] = 1;
    r.points[i] = static_cast<uint8_t>(count);
    r.normal[3 * i] = nx; r.normal[3 * i + 1] = ny; r.normal[3 * i + 2] = nz;
    for (int k = 0; k < P; k++) {
      const bool used = k < count;
      for (int e = 0; e < 3; e++) r.point[3 * (P * i + k) + e] = used ? pt[3 * k + e] : 0.0;
      r.separation[P * i + k] = used ? sep[k] : 0.0;
      r.pid[P * i + k] = used ? r.old.cache_id[P * j + k] : 0u;
    }
  }
}

// The step's rows in found order, in the caller's row layout (bg_rows), so the solve stage's
// unpack kernel reads them as it reads an upload.
struct FoundRows {
  int32_t *row, *a, *b, *pair;
  uint8_t* points;
  uint32_t* pid;
  double *normal, *t1, *t2, *friction, *restitution, *tolerance, *patch, *separation, *point, *shift;
  double *ni, *ti1, *ti2, *ri1, *ri2, *si, *drift1, *drift2, *maxni, *relvel, *gap;
};

struct EmitParams {
  int32_t np;                       // pairs in the list
  const int32_t *a, *b;             // per pair
  const double* tol;                // per pair
  const int32_t* memory;            // per pair: its record in `old`, or -1
  const uint8_t* points;            // the narrowphase's manifolds, per pair
  const double *normal, *point, *separation;
  const uint32_t* pid;
  const double *friction, *restitution, *size;   // per slot
  const uint8_t* type;                           // per slot
  int32_t* rowof;                   // np + 1: (points > 0), then its exclusive scan (found row)
  Memory old;
  FoundRows r;
  // the kept manifolds, with reuse on: which pairs reused theirs, and the next bank, which keeps
  // each touching pair's (remember(), src/contact.js:540-569, for a fresh one)
  int32_t reuse;
  const uint8_t* kept;
  Memory next;
  Poses s;
};

// Which pairs emit a row.
__global__ void ct_flags(EmitParams e) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < e.np; i += gridDim.x * blockDim.x)
    e.rowof[i] = e.points[i] > 0 ? 1 : 0;
}

// basis(): src/contact.js:1283-1292.
__device__ __forceinline__ void ct_basis(const FoundRows& r, int m) {
  const double nx = r.normal[3 * m], ny = r.normal[3 * m + 1], nz = r.normal[3 * m + 2];
  const double ax = fabs(nx), ay = fabs(ny), az = fabs(nz);
  double tx, ty, tz;
  if (ax <= ay && ax <= az) { tx = 0; ty = nz; tz = -ny; } else if (ay <= az) { tx = -nz; ty = 0; tz = nx; } else { tx = ny; ty = -nx; tz = 0; }
  const double l = 1 / sqrt(tx * tx + ty * ty + tz * tz);
  tx *= l; ty *= l; tz *= l;
  r.t1[3 * m] = tx; r.t1[3 * m + 1] = ty; r.t1[3 * m + 2] = tz;
  r.t2[3 * m] = ny * tz - nz * ty; r.t2[3 * m + 1] = nz * tx - nx * tz; r.t2[3 * m + 2] = nx * ty - ny * tx;
}

// emit() (src/contact.js:889-921: whole bodies, sign 1, no parts, never shifted), basis(), then
// carry() (999-1036) from the pair's record: one thread a pair that touches.
__global__ void ct_emit(EmitParams e) {
  const FoundRows& r = e.r;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < e.np; i += gridDim.x * blockDim.x) {
    const int count = e.points[i];
    if (count == 0) continue;
    const int m = e.rowof[i];
    const int a = e.a[i], b = e.b[i];
    r.row[m] = m;
    r.a[m] = a; r.b[m] = b; r.pair[m] = i;
    r.points[m] = static_cast<uint8_t>(count);
    for (int k = 0; k < 3; k++) r.normal[3 * m + k] = 1 * e.normal[3 * i + k];
    r.friction[m] = sqrt(e.friction[a] * e.friction[b]);
    r.restitution[m] = ct_max(e.restitution[a], e.restitution[b]);
    r.tolerance[m] = e.tol[i];
    r.patch[m] = PIXEL * (e.type[a] != kDynamic ? e.size[b] : e.type[b] != kDynamic ? e.size[a] : ct_min(e.size[a], e.size[b]));
    r.ri1[m] = 0; r.ri2[m] = 0; r.si[m] = 0; r.ti1[m] = 0; r.ti2[m] = 0; r.drift1[m] = 0; r.drift2[m] = 0;
    r.gap[m] = 0;
    for (int k = 0; k < P; k++) {
      const int o = m * P + k, q = i * P + k;
      const bool used = k < count;
      r.pid[o] = used ? e.pid[q] : 0u;
      r.separation[o] = used ? e.separation[q] : 0.0;
      for (int c = 0; c < 3; c++) {
        r.point[3 * o + c] = used ? e.point[3 * q + c] : 0.0;
        r.shift[3 * o + c] = 0;
      }
      r.ni[o] = 0; r.maxni[o] = 0; r.relvel[o] = 0;
    }
    ct_basis(r, m);
    const int j = e.memory[i];
    if (e.reuse) {
      Memory& n = e.next;
      n.cached[i] = 1;
      n.cache_points[i] = static_cast<uint8_t>(count);
      if (e.kept[i]) {   // the record's kept manifold goes on as it was
        for (int k = 0; k < 7; k++) n.pose[7 * i + k] = e.old.pose[7 * j + k];
        n.loss[i] = e.old.loss[j];
        for (int k = 0; k < 3; k++) n.local_normal[3 * i + k] = e.old.local_normal[3 * j + k];
        for (int k = 0; k < 6 * P; k++) n.local[6 * P * i + k] = e.old.local[6 * P * j + k];
        for (int k = 0; k < P; k++) n.cache_id[P * i + k] = e.old.cache_id[P * j + k];
      } else {           // remember(): the manifold collide() just found
        const Poses& s = e.s;
        ct_relative(s, a, b, n.pose + 7 * i);
        n.loss[i] = 0;   // collide() of boxes, spheres and capsules falls short of nothing
        double A[9], Bx[9];
        ct_axes(s.q + 4 * a, A);
        ct_axes(s.q + 4 * b, Bx);
        const double nx = r.normal[3 * m], ny = r.normal[3 * m + 1], nz = r.normal[3 * m + 2];
        n.local_normal[3 * i] = A[0] * nx + A[1] * ny + A[2] * nz;
        n.local_normal[3 * i + 1] = A[3] * nx + A[4] * ny + A[5] * nz;
        n.local_normal[3 * i + 2] = A[6] * nx + A[7] * ny + A[8] * nz;
        for (int k = 0; k < count; k++) {
          double* l = n.local + 6 * (P * i + k);
          const double half = 0.5 * r.separation[m * P + k];
          const double px = r.point[3 * (m * P + k)], py = r.point[3 * (m * P + k) + 1], pz = r.point[3 * (m * P + k) + 2];
          const double ax = px - nx * half - s.p[3 * a], ay = py - ny * half - s.p[3 * a + 1], az = pz - nz * half - s.p[3 * a + 2];
          const double bx = px + nx * half - s.p[3 * b], by = py + ny * half - s.p[3 * b + 1], bz = pz + nz * half - s.p[3 * b + 2];
          l[0] = A[0] * ax + A[1] * ay + A[2] * az;
          l[1] = A[3] * ax + A[4] * ay + A[5] * az;
          l[2] = A[6] * ax + A[7] * ay + A[8] * az;
          l[3] = Bx[0] * bx + Bx[1] * by + Bx[2] * bz;
          l[4] = Bx[3] * bx + Bx[4] * by + Bx[5] * bz;
          l[5] = Bx[6] * bx + Bx[7] * by + Bx[8] * bz;
          ct_cored(s, a, l);
          ct_cored(s, b, l + 3);
          n.cache_id[P * i + k] = r.pid[m * P + k];
        }
      }
    }
    // carry(), from the pair's record
    const int remembered = j < 0 ? 0 : e.old.points[j];
    if (remembered == 0) continue;
    const int m3 = 3 * m, j3 = 3 * j;
    const double t1x = r.t1[m3], t1y = r.t1[m3 + 1], t1z = r.t1[m3 + 2];
    const double t2x = r.t2[m3], t2y = r.t2[m3 + 1], t2z = r.t2[m3 + 2];
    const double lx = e.old.twist[j3], ly = e.old.twist[j3 + 1], lz = e.old.twist[j3 + 2];
    if (count <= 2) {
      r.ri1[m] = lx * t1x + ly * t1y + lz * t1z;
      r.ri2[m] = lx * t2x + ly * t2y + lz * t2z;
    }
    r.si[m] = lx * r.normal[m3] + ly * r.normal[m3 + 1] + lz * r.normal[m3 + 2];
    const double fx = e.old.friction[j3], fy = e.old.friction[j3 + 1], fz = e.old.friction[j3 + 2];
    r.ti1[m] = fx * t1x + fy * t1y + fz * t1z;
    r.ti2[m] = fx * t2x + fy * t2y + fz * t2z;
    bool same = false;
    for (int k = 0; k < count; k++) {
      const uint32_t id = r.pid[m * P + k];
      for (int q = 0; q < remembered; q++) {
        if (e.old.pid[j * P + q] != id) continue;
        r.ni[m * P + k] = e.old.ni[j * P + q];
        same = true;
        break;
      }
    }
    if (same) {
      const double sx = e.old.slip[j3], sy = e.old.slip[j3 + 1], sz = e.old.slip[j3 + 2];
      r.drift1[m] = sx * t1x + sy * t1y + sz * t1z;
      r.drift2[m] = sx * t2x + sy * t2y + sz * t2z;
    }
  }
}

// rest() (src/contact.js:1318-1329) for the rows coloured RESTING (between frozen or static
// bodies): the solve passes them through with these.
__global__ void ct_rest(FoundRows r, const int32_t* colour, int n) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    if (colour[m] != kResting) continue;
    double least = __longlong_as_double(0x7ff0000000000000LL);   // +Infinity
    for (int k = 0; k < r.points[m]; k++) {
      const int i = m * P + k;
      if (r.separation[i] < least) least = r.separation[i];
      r.maxni[i] = r.ni[i];
      r.relvel[i] = 0;
    }
    r.gap[m] = least;
  }
}

// ---- the order the solve stage takes the rows in ----
//
// Within each colour the rows go by point count, ties in arrange()'s order (a colour's rows move
// no body in common, so their order inside the colour changes no result, src/graph.js:1-33, and a
// warp of rows with one point count runs one row solver); the overflow and resting runs keep
// arrange()'s order.  That is a stable counting sort of arrange()'s order on kKeys keys: each
// tile of kOrderThreads rows counts its keys, the (key, tile) counts are scanned, and each tile
// places its rows, each row after the rows of its key in earlier tiles, earlier warps of its tile
// and earlier lanes of its warp.

struct OrderParams {
  int32_t n;                 // rows
  int32_t tiles;
  const int32_t* order;      // n: arrange()'s order (found index of row o)
  const int32_t* colour;     // n, found order
  const uint8_t* points;     // n, found order
  int32_t* counts;           // kKeys * tiles + 1: (key, tile) counts, then their exclusive scan
  int32_t* perm;             // n: device row d holds found row perm[d]
  int32_t* iperm;            // n: found row f is device row iperm[f]
  int32_t* groups;           // kKeys + 1: where each key's rows begin (device rows)
  int2* chunks;              // the solve's runs (see below)
  int32_t* chunk_base;       // kKeys + 1: each key's first run; [kKeys] the number of runs
};

__device__ __forceinline__ int ct_key(const OrderParams& p, int o) {
  const int f = p.order[o];
  const int k = p.colour[f];
  if (k >= kOverflow) return 128 + (k - kOverflow);
  int c = p.points[f];
  c = c < 1 ? 1 : c > P ? P : c;
  return 4 * k + c - 1;
}

__global__ void __launch_bounds__(kOrderThreads) ct_order_count(OrderParams p) {
  __shared__ int32_t hist[kKeys];
  for (int k = threadIdx.x; k < kKeys; k += blockDim.x) hist[k] = 0;
  __syncthreads();
  const int o = blockIdx.x * kOrderThreads + threadIdx.x;
  if (o < p.n) atomicAdd(&hist[ct_key(p, o)], 1);
  __syncthreads();
  for (int k = threadIdx.x; k < kKeys; k += blockDim.x) p.counts[k * p.tiles + blockIdx.x] = hist[k];
}

__global__ void __launch_bounds__(kOrderThreads) ct_order_place(OrderParams p) {
  constexpr int kWarps = kOrderThreads / 32;
  __shared__ int32_t warp_counts[kWarps][kKeys];
  for (int i = threadIdx.x; i < kWarps * kKeys; i += blockDim.x) (&warp_counts[0][0])[i] = 0;
  __syncthreads();
  const int o = blockIdx.x * kOrderThreads + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int key = o < p.n ? ct_key(p, o) : -1;
  const unsigned peers = __match_any_sync(0xffffffffu, key);
  const int before = __popc(peers & ((1u << lane) - 1u));
  if (key >= 0 && before == 0) warp_counts[warp][key] = __popc(peers);
  __syncthreads();
  if (key < 0) return;
  int at = p.counts[key * p.tiles + blockIdx.x] + before;
  for (int w = 0; w < warp; w++) at += warp_counts[w][key];
  const int f = p.order[o];
  p.perm[at] = f;
  p.iperm[f] = at;
}

// Each key's first device row, and the runs the grid's dataflow takes: each colour's rows of one
// point count in runs of 32 (the last shorter), then the overflow's rows one a run, in order (as
// the host's order_rows() makes them).  One block: a thread a key, then one thread adds them up.
constexpr int kRunThreads = 160;
__global__ void __launch_bounds__(kRunThreads) ct_order_runs(OrderParams p) {
  __shared__ int32_t runs_of[kKeys];
  const int k = threadIdx.x;
  if (k < kKeys) {
    const int first = p.counts[k * p.tiles];
    const int size = (k + 1 < kKeys ? p.counts[(k + 1) * p.tiles] : p.n) - first;
    p.groups[k] = first;
    runs_of[k] = k < 128 ? (size + 31) / 32 : k == 128 ? size : 0;
  }
  __syncthreads();
  if (k != 0) return;
  int runs = 0;
  for (int j = 0; j < kKeys; j++) {
    p.chunk_base[j] = runs;
    runs += runs_of[j];
  }
  p.groups[kKeys] = p.n;
  p.chunk_base[kKeys] = runs;
}

__global__ void ct_order_chunks(OrderParams p) {
  const int runs = p.chunk_base[kKeys];
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < runs; c += gridDim.x * blockDim.x) {
    int lo = 0, hi = kKeys - 1;   // the last key whose first run is at or before c
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.chunk_base[mid] <= c) lo = mid; else hi = mid - 1;
    }
    const int j = c - p.chunk_base[lo];
    const int first = p.groups[lo], size = p.groups[lo + 1] - first;
    if (lo == 128) {
      p.chunks[c] = make_int2(first + j, 1);
    } else {
      const int at = first + 32 * j;
      p.chunks[c] = make_int2(at, min(32, first + size - at));
    }
  }
}

// ---- the grid's dataflow tables (stage.cuh, flow_pass) ----
//
// Each solved row's place among the solved rows on each body it moves (a body with an inverse
// mass), in device order, and each body's count of them, as order_rows() makes them on the host.

struct FlowParams {
  int32_t solved, nrows, nb;
  const int32_t* perm;
  const int32_t *a, *b;          // found order
  const double* inv_mass;        // per slot
  int32_t* deg;                  // nb (zeroed)
  int32_t* off;                  // nb + 1
  int32_t* cursor;               // nb (zeroed)
  int32_t* list;                 // 2 * solved: 2d + side
  int32_t* rank;                 // 2 * nrows: on a, then on b (-1: not moved)
};

__global__ void ct_flow_degrees(FlowParams f) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < f.nrows; d += gridDim.x * blockDim.x) {
    f.rank[d] = -1;
    f.rank[f.nrows + d] = -1;
    if (d >= f.solved) continue;
    const int m = f.perm[d];
    const int x = f.a[m], y = f.b[m];
    if (f.inv_mass[x] != 0) atomicAdd(&f.deg[x], 1);
    if (f.inv_mass[y] != 0) atomicAdd(&f.deg[y], 1);
  }
}

__global__ void ct_flow_fill(FlowParams f) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < f.solved; d += gridDim.x * blockDim.x) {
    const int m = f.perm[d];
    const int x = f.a[m], y = f.b[m];
    if (f.inv_mass[x] != 0) f.list[f.off[x] + atomicAdd(&f.cursor[x], 1)] = 2 * d;
    if (f.inv_mass[y] != 0) f.list[f.off[y] + atomicAdd(&f.cursor[y], 1)] = 2 * d + 1;
  }
}

// Each body's rows in device order (an insertion sort: a moving body has at most a few dozen
// rows), then their ranks.
__global__ void ct_flow_ranks(FlowParams f) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < f.nb; x += gridDim.x * blockDim.x) {
    int32_t* l = f.list + f.off[x];
    const int d = f.off[x + 1] - f.off[x];
    for (int i = 1; i < d; i++) {
      const int32_t v = l[i];
      int j = i - 1;
      while (j >= 0 && l[j] > v) {
        l[j + 1] = l[j];
        j--;
      }
      l[j + 1] = v;
    }
    for (int i = 0; i < d; i++) {
      const int e = l[i];
      f.rank[(e & 1) ? f.nrows + (e >> 1) : (e >> 1)] = i;
    }
  }
}

// ---- store() and touched() after the solve ----

struct KeepParams {
  int32_t np, solved;
  const uint8_t* points;         // per pair (the narrowphase's)
  const int32_t* rowof;          // per pair: its found row
  const int32_t* memory;         // per pair: its record in `old`, or -1
  const int32_t* iperm;          // found row -> device row
  const uint32_t* pid;           // found rows' point ids
  bg::RowsDev R;                 // the solved rows (device layout)
  Memory old, next;
  uint8_t* touching;             // per pair
  int32_t* points_solved;        // sum of the solved rows' points
  int32_t reuse;
};

// For each pair of the list: its record for the next call (keep(), src/contact.js:1091-1115, for a
// solved row; the record it had for a resting row, which store() skips; nothing for a pair apart)
// and touched()'s flag (src/contact.js:2178-2213: the gap within tolerance, or a point pushed).
__global__ void ct_keep(KeepParams k) {
  const bg::RowsDev& R = k.R;
  const int64_t cap = R.cap;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k.np; i += gridDim.x * blockDim.x) {
    const int count = k.points[i];
    if (count == 0) {
      k.next.points[i] = 0;
      k.next.touching[i] = 0;
      k.next.cached[i] = 0;   // forget() uncaches: src/pairs.js:236
      k.touching[i] = 0;
      continue;
    }
    const int m = k.rowof[i];
    const int d = k.iperm[m];
    bool meets = R.gap[d] <= R.tolerance[d];
    for (int q = 0; q < count && !meets; q++) meets = R.maxni[q * cap + d] > 0;
    k.touching[i] = meets ? 1 : 0;
    k.next.touching[i] = meets ? 1 : 0;
    if (!k.reuse) k.next.cached[i] = 0;
    if (d >= k.solved) {
      const int j = k.memory[i];
      const int have = j < 0 ? 0 : k.old.points[j];
      k.next.points[i] = static_cast<uint8_t>(have);
      if (have == 0) continue;
      for (int q = 0; q < P; q++) {
        k.next.pid[i * P + q] = k.old.pid[j * P + q];
        k.next.ni[i * P + q] = k.old.ni[j * P + q];
      }
      for (int c = 0; c < 3; c++) {
        k.next.friction[3 * i + c] = k.old.friction[3 * j + c];
        k.next.twist[3 * i + c] = k.old.twist[3 * j + c];
        k.next.slip[3 * i + c] = k.old.slip[3 * j + c];
      }
      continue;
    }
    atomicAdd(k.points_solved, count);
    k.next.points[i] = static_cast<uint8_t>(count);
    const double t1x = R.t1[d], t1y = R.t1[cap + d], t1z = R.t1[2 * cap + d];
    const double t2x = R.t2[d], t2y = R.t2[cap + d], t2z = R.t2[2 * cap + d];
    const double nx = R.n[d], ny = R.n[cap + d], nz = R.n[2 * cap + d];
    const double r1 = R.ri1[d], r2 = R.ri2[d], sp = R.si[d];
    k.next.twist[3 * i] = t1x * r1 + t2x * r2 + nx * sp;
    k.next.twist[3 * i + 1] = t1y * r1 + t2y * r2 + ny * sp;
    k.next.twist[3 * i + 2] = t1z * r1 + t2z * r2 + nz * sp;
    const double l1 = R.ti1[d], l2 = R.ti2[d];
    k.next.friction[3 * i] = t1x * l1 + t2x * l2;
    k.next.friction[3 * i + 1] = t1y * l1 + t2y * l2;
    k.next.friction[3 * i + 2] = t1z * l1 + t2z * l2;
    const double d1 = R.drift1[d], d2 = R.drift2[d];
    k.next.slip[3 * i] = t1x * d1 + t2x * d2;
    k.next.slip[3 * i + 1] = t1y * d1 + t2y * d2;
    k.next.slip[3 * i + 2] = t1z * d1 + t2z * d2;
    for (int q = 0; q < count; q++) {
      k.next.pid[i * P + q] = k.pid[m * P + q];
      k.next.ni[i * P + q] = R.ni[q * cap + d];
    }
  }
}

}  // namespace bgct
