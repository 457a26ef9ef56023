// The host side of World.step around the solve stage, for boxes, spheres and capsules.
// Restates, for the parts it covers:
//   src/world.js     addBody/_write 2152-2274 (mass, inertia, size, reach), _bounds/_boundsOf
//                    1574-1630, step 880-1072 (order of the step), transforms 1040-1057
//   src/shapes.js    volume 14-21, inertia 37-56
//   src/core/check.js quat 106-117
//   src/broadphase.js fat boxes (fat 206-219, FAT 1/4, AHEAD 16), update 121-137, overlap 176-181
//   src/pairs.js     found 180-215, remove 217-232, forget 235-241, holds 340-357
//   src/contact.js   narrow 296-327, find 334-368, emit 889-921, carry 999-1036, basis 1283-1292,
//                    load 1244-1276, rest 1318-1329, store 1067-1088, keep 1091-1115,
//                    touched 2178-2213 (the touching flags; no event list)
//   src/graph.js     colour 105-170, arrange 178-214
// The broadphase files fat boxes in a uniform grid instead of the reference's two AABB trees
// (src/tree.js): the same pairs are found, offered in ascending slot order rather than tree
// order, so pair order (and with it row order and colours) can differ from the reference's.
#include "../../include/bearing_world.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "collide_impl.hpp"
#include "../csrc/tape.hpp"

namespace {

using bearing::Manifold;
using bearing::Shape;

constexpr int P = 4;
constexpr int COLOURS = 32;
constexpr int OVERFLOW_ = 32;
constexpr int RESTING = 33;
constexpr int DIGIT = 12;
constexpr int DIGITS = 1 << DIGIT;
constexpr double PIXEL = 1.0 / 200.0;     // src/contact.js:125
constexpr double FAT = 1.0 / 4.0;         // src/broadphase.js:15
constexpr double AHEAD = 16;              // src/broadphase.js:37
constexpr double PI = 3.141592653589793;
constexpr double INF = std::numeric_limits<double>::infinity();
constexpr int KINEMATIC = 2;

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

// axesOf: src/core/math.js:222-227.
inline void axesOf(const double* q, double* ax) {
  const double x = q[0], y = q[1], z = q[2], w = q[3];
  ax[0] = 1 - 2 * (y * y + z * z); ax[1] = 2 * (x * y + z * w); ax[2] = 2 * (x * z - y * w);
  ax[3] = 2 * (x * y - z * w); ax[4] = 1 - 2 * (x * x + z * z); ax[5] = 2 * (y * z + x * w);
  ax[6] = 2 * (x * z + y * w); ax[7] = 2 * (y * z - x * w); ax[8] = 1 - 2 * (x * x + y * y);
}

template <class T>
void grow(std::vector<T>& v, size_t n, T fill = T()) {
  if (v.size() < n) v.resize(n, fill);
}

// The step's manifolds: src/contact.js:149-269, the columns this path uses.
struct Contacts {
  int count = 0, solved = 0, capacity = 0;
  int starts[COLOURS + 3] = {};
  std::vector<int32_t> a, b, pair, colour, order, row;
  std::vector<uint8_t> points, sliding;
  std::vector<double> normal, t1, t2, friction, restitution, tolerance, patch;
  std::vector<double> rollImpulse1, rollImpulse2, spinImpulse, tangentImpulse1, tangentImpulse2, drift1, drift2;
  std::vector<double> separation, normalImpulse, point, shift, gap, maxNormalImpulse, relativeVelocity;
  std::vector<double> anchorA, anchorB;
  std::vector<uint32_t> pid;
  std::vector<double> room;
  std::vector<int32_t> digits;

  void alloc(int c) {
    const size_t m = static_cast<size_t>(c), p = m * P;
    a.resize(m); b.resize(m); pair.resize(m); colour.resize(m); order.resize(m); row.resize(m);
    points.resize(m); sliding.resize(m);
    normal.resize(3 * m); t1.resize(3 * m); t2.resize(3 * m);
    friction.resize(m); restitution.resize(m); tolerance.resize(m); patch.resize(m);
    rollImpulse1.resize(m); rollImpulse2.resize(m); spinImpulse.resize(m);
    tangentImpulse1.resize(m); tangentImpulse2.resize(m); drift1.resize(m); drift2.resize(m);
    separation.resize(p); normalImpulse.resize(p); point.resize(3 * p); shift.resize(3 * p);
    gap.resize(m); maxNormalImpulse.resize(p); relativeVelocity.resize(p);
    anchorA.resize(3 * m); anchorB.resize(3 * m);
    pid.resize(p);
    room.resize(3 * p);
    capacity = c;
  }
  // ensure: src/contact.js:250-255.
  void ensure(int n) {
    if (n <= capacity) return;
    int c = capacity > 1 ? capacity : 1;
    while (c < n) c *= 2;
    alloc(c);
  }
};

// Where each pair is in the list, by its key (the reference's Map from pair key to pair,
// src/pairs.js): open addressing with linear probing in two flat arrays, at most half full, keys
// spread by MurmurHash3's 64-bit finaliser.  A removal shifts the entries after it back into the
// hole where their probe path allows, so no deleted marks build up over a long run.
struct PairIndex {
  static constexpr uint64_t kEmpty = ~0ull;   // no pair key is all ones (slots are below 2^31)
  std::vector<uint64_t> keys;
  std::vector<int32_t> vals;
  size_t used = 0;

  static size_t spread(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return static_cast<size_t>(k);
  }
  size_t mask() const { return keys.size() - 1; }
  // The key's entry, or the empty entry where it would go.
  size_t find(uint64_t k) const {
    size_t i = spread(k) & mask();
    while (keys[i] != kEmpty && keys[i] != k) i = (i + 1) & mask();
    return i;
  }
  bool contains(uint64_t k) const { return !keys.empty() && keys[find(k)] == k; }
  void set(uint64_t k, int32_t v) {
    if (2 * (used + 1) > keys.size()) rehash(keys.empty() ? 64 : 2 * keys.size());
    const size_t i = find(k);
    if (keys[i] == kEmpty) {
      keys[i] = k;
      used++;
    }
    vals[i] = v;
  }
  void erase(uint64_t k) {
    if (keys.empty()) return;
    size_t hole = find(k);
    if (keys[hole] != k) return;
    for (size_t j = (hole + 1) & mask(); keys[j] != kEmpty; j = (j + 1) & mask()) {
      // The entry at j may fill the hole if the hole lies on its probe path, from its home to j.
      const size_t home = spread(keys[j]) & mask();
      if (((j - home) & mask()) >= ((j - hole) & mask())) {
        keys[hole] = keys[j];
        vals[hole] = vals[j];
        hole = j;
      }
    }
    keys[hole] = kEmpty;
    used--;
  }
  void rehash(size_t capacity) {
    std::vector<uint64_t> oldKeys(capacity, kEmpty);
    std::vector<int32_t> oldVals(capacity, 0);
    oldKeys.swap(keys);
    oldVals.swap(vals);
    for (size_t i = 0; i < oldKeys.size(); i++) {
      if (oldKeys[i] == kEmpty) continue;
      const size_t at = find(oldKeys[i]);
      keys[at] = oldKeys[i];
      vals[at] = oldVals[i];
    }
  }
};

// The pair list: src/pairs.js (awake pairs only: every pair here has an awake body).
struct Pairs {
  int count = 0, active = 0;
  std::vector<int32_t> a, b;
  std::vector<uint8_t> points, touching;
  std::vector<uint32_t> pid;
  std::vector<double> normalImpulse, friction, slip, twist;
  // with the contact step on another device (bw_set_contact_step): where the pair's memory is, its
  // index in the last list handed over, or -1 (nothing remembered)
  std::vector<int32_t> record;
  // The kept manifold (src/pairs.js:55-80, contact.js reused/remember), by pair rather than in rows
  // of its own (which rows hold which pair changes no result): whether one is kept, its point count,
  // the pose it was found at (7), how far it fell short of exact, its normal in a's frame (3), each
  // point's end on a in a's frame and on b in b's frame (6 a point) and feature ids.
  std::vector<uint8_t> cached, cachePoints;
  std::vector<double> cachePose, cacheLoss, cacheNormal, cacheLocal;
  std::vector<uint32_t> cacheId;
  PairIndex index;

  static uint64_t key(int x, int y) { return (static_cast<uint64_t>(x) << 32) | static_cast<uint32_t>(y); }
  void reserve(int n) {
    const size_t c = static_cast<size_t>(n);
    if (a.size() >= c) return;
    size_t cap = a.size() > 16 ? a.size() : 16;
    while (cap < c) cap *= 2;
    a.resize(cap); b.resize(cap); points.resize(cap); touching.resize(cap); record.resize(cap, -1);
    cached.resize(cap); cachePoints.resize(cap); cachePose.resize(7 * cap); cacheLoss.resize(cap);
    cacheNormal.resize(3 * cap); cacheLocal.resize(6 * P * cap); cacheId.resize(P * cap);
    pid.resize(P * cap); normalImpulse.resize(P * cap);
    friction.resize(3 * cap); slip.resize(3 * cap); twist.resize(3 * cap);
  }
  // found: src/pairs.js:180-215 (whole bodies, no sensors or filters).
  void found(int x, int y, const uint8_t* type) {
    if (type[x] != BG_DYNAMIC && type[y] != BG_DYNAMIC) return;
    const int lo = x < y ? x : y, hi = x < y ? y : x;
    if (index.contains(key(lo, hi))) return;
    const int p = count;
    reserve(p + 1);
    a[p] = lo; b[p] = hi; points[p] = 0; touching[p] = 0; record[p] = -1; cached[p] = 0;
    index.set(key(lo, hi), p);
    count++;
    active = count;
  }
  void moveTo(int from, int to) {
    a[to] = a[from]; b[to] = b[from]; points[to] = points[from]; touching[to] = touching[from];
    record[to] = record[from];
    cached[to] = cached[from];
    cachePoints[to] = cachePoints[from];
    cacheLoss[to] = cacheLoss[from];
    for (int k = 0; k < 7; k++) cachePose[7 * to + k] = cachePose[7 * from + k];
    for (int k = 0; k < 3; k++) cacheNormal[3 * to + k] = cacheNormal[3 * from + k];
    for (int k = 0; k < 6 * P; k++) cacheLocal[6 * P * to + k] = cacheLocal[6 * P * from + k];
    for (int k = 0; k < P; k++) cacheId[P * to + k] = cacheId[P * from + k];
    for (int k = 0; k < P; k++) { pid[P * to + k] = pid[P * from + k]; normalImpulse[P * to + k] = normalImpulse[P * from + k]; }
    for (int k = 0; k < 3; k++) {
      friction[3 * to + k] = friction[3 * from + k];
      slip[3 * to + k] = slip[3 * from + k];
      twist[3 * to + k] = twist[3 * from + k];
    }
    index.set(key(a[to], b[to]), to);
  }
  // remove: src/pairs.js:217-232 (one run).
  void remove(int p) {
    index.erase(key(a[p], b[p]));
    const int last = --count;
    if (p != last) moveTo(last, p);
    active = count;
  }
  // forget: src/pairs.js:235-241.
  void forget(int p) {
    points[p] = 0;
    touching[p] = 0;
    record[p] = -1;
    cached[p] = 0;   // uncache: src/pairs.js:236
  }
};

}  // namespace

// colour(): src/graph.js:105-170 over cnt manifolds in found order (A[m], Bs[m]): each manifold's
// colour, then the row order (order: row o holds manifold order[o]; `scratch` cnt entries,
// `count` DIGITS + 1) and the colour starts, as the reference lays them out.
static void colour_manifolds(int cnt, const int32_t* A, const int32_t* Bs, const uint8_t* type, const uint8_t* frozen,
                             int nslots, int32_t* colour, int32_t* order, int32_t* scratch, int32_t* count,
                             int32_t* starts) {
  std::vector<int32_t> used(static_cast<size_t>(nslots), 0);
  const bool anyFrozen = std::any_of(frozen, frozen + nslots, [](uint8_t f) { return f != 0; });
  for (int m = 0; m < cnt; m++) {
    const int a = A[m], b = Bs[m];
    bool da = type[a] == BG_DYNAMIC, db = type[b] == BG_DYNAMIC;
    if (anyFrozen) {
      const bool fa = frozen[a] != 0, fb = frozen[b] != 0;
      if ((fa || type[a] == BG_STATIC) && (fb || type[b] == BG_STATIC)) {
        colour[m] = RESTING;
        continue;
      }
      if (fa) da = false;
      if (fb) db = false;
    }
    const int32_t held = (da ? used[a] : 0) | (db ? used[b] : 0);
    if (held == -1) {
      colour[m] = OVERFLOW_;
      continue;
    }
    const uint32_t uheld = static_cast<uint32_t>(held);
    const uint32_t bit = ~uheld & (uheld + 1u);
    colour[m] = 31 - __builtin_clz(bit);
    if (da) used[a] |= static_cast<int32_t>(bit);
    if (db) used[b] |= static_cast<int32_t>(bit);
  }
  // stable counting sorts by b's low digit, its high one (past DIGITS slots), then colour
  std::fill(count, count + DIGITS + 1, 0);
  const bool high = nslots > DIGITS;
  int32_t* from = high ? order : scratch;
  for (int m = 0; m < cnt; m++) count[(Bs[m] & (DIGITS - 1)) + 1]++;
  for (int k = 0; k < DIGITS; k++) count[k + 1] += count[k];
  for (int m = 0; m < cnt; m++) from[count[Bs[m] & (DIGITS - 1)]++] = m;
  if (high) {
    std::fill(count, count + DIGITS + 1, 0);
    for (int i = 0; i < cnt; i++) count[(static_cast<uint32_t>(Bs[order[i]]) >> DIGIT) + 1]++;
    for (int k = 0; k < DIGITS; k++) count[k + 1] += count[k];
    for (int i = 0; i < cnt; i++) {
      const int m = order[i];
      scratch[count[static_cast<uint32_t>(Bs[m]) >> DIGIT]++] = m;
    }
    from = scratch;
  }
  std::fill(starts, starts + COLOURS + 3, 0);
  for (int m = 0; m < cnt; m++) starts[colour[m] + 1]++;
  for (int k = 0; k <= RESTING; k++) starts[k + 1] += starts[k];
  for (int i = 0; i < cnt; i++) {
    const int m = from[i];
    order[starts[colour[m]]++] = m;
  }
  for (int k = RESTING; k > 0; k--) starts[k] = starts[k - 1];
  starts[0] = 0;
}

struct bw_world {
  std::string error;
  double gravity[3] = {0, -9.81, 0};
  int substeps = 8;
  int64_t stepCount = 0;
  double stepDt = 0;
  int n = 0;   // slots in use
  // Per-slot columns: src/world.js:228-311.
  std::vector<double> position, rotation, velocity, angular, dims, mass, inertia, invInertia, tumbled, ceiling;
  std::vector<double> friction, restitution, damping, angularDamping, gravityScale, invMass, size, reach;
  std::vector<double> axes, box, motion, invI, start, startQ;
  std::vector<uint8_t> type, shape, framed, lock, frozen, awake;
  std::vector<int32_t> jointHead, awakeList;
  std::vector<float> transforms;
  // Broadphase: each slot's fat box (src/broadphase.js), filed in a uniform grid.
  std::vector<double> fat;
  std::vector<uint8_t> filed, isMoved, large;
  std::vector<int32_t> moved;
  double cell = 0;
  std::unordered_map<uint64_t, std::vector<int32_t>> grid;
  std::vector<int32_t> largeList;
  std::vector<int32_t> seen;
  int32_t seenMark = 0;
  Pairs pairs;
  Contacts c;
  bw_solver solver = nullptr;
  void* solverUser = nullptr;
  // the narrowphase over the step's pair list on another device (bw_set_narrowphase), or none
  bw_narrowphase narrowFn = nullptr;
  void* narrowUser = nullptr;
  std::vector<uint8_t> nmPoints;
  std::vector<uint32_t> nmPid;
  std::vector<double> nmNormal, nmPoint, nmSeparation;
  std::vector<int32_t> nmPair;
  // the whole contact side of the step on another device (bw_set_contact_step), or none
  bw_contact_solver contactFn = nullptr;
  void* contactUser = nullptr;
  std::vector<int32_t> nmRecord;
  std::vector<uint8_t> nmTouching;
  bool begun = false;
  bw_stats stats = {};

  void resize(int slots) {
    const size_t s = static_cast<size_t>(slots);
    grow(position, 3 * s); grow(rotation, 4 * s); grow(velocity, 3 * s); grow(angular, 3 * s);
    grow(dims, 3 * s); grow(mass, s); grow(inertia, 3 * s); grow(invInertia, 3 * s);
    grow(tumbled, 3 * s); grow(ceiling, s); grow(friction, s); grow(restitution, s); grow(damping, s);
    grow(angularDamping, s); grow(gravityScale, s); grow(invMass, s); grow(size, s); grow(reach, s);
    grow(axes, 9 * s); grow(box, 6 * s); grow(motion, s); grow(invI, 6 * s); grow(start, 3 * s); grow(startQ, 4 * s);
    grow(type, s); grow(shape, s); grow(framed, s); grow(lock, s); grow(frozen, s); grow(awake, s);
    grow(jointHead, s); grow(awakeList, s); grow(transforms, 7 * s);
    grow(fat, 6 * s); grow(filed, s); grow(isMoved, s); grow(large, s); grow(seen, s);
  }

  // _boundsOf: src/world.js:1581-1630 (boxes, spheres, capsules).
  void boundsOf(int s, double dt, double gl) {
    const int s3 = s * 3, s4 = s * 4, a9 = s * 9, b6 = s * 6;
    double* ax = &axes[a9];
    axesOf(&rotation[s4], ax);
    double m = 0;
    if (type[s] != BG_STATIC) {
      const double* v = &velocity[s3];
      const double* w = &angular[s3];
      const double speed = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
        + (type[s] == BG_DYNAMIC ? gl * std::fabs(gravityScale[s]) * dt : 0)
        + std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]) * reach[s];
      m = speed * dt;
    }
    motion[s] = m;
    double ex, ey, ez;
    const double* d = &dims[s3];
    if (shape[s] == BG_BOX) {
      const double hx = d[0] * 0.5, hy = d[1] * 0.5, hz = d[2] * 0.5;
      ex = std::fabs(ax[0]) * hx + std::fabs(ax[3]) * hy + std::fabs(ax[6]) * hz;
      ey = std::fabs(ax[1]) * hx + std::fabs(ax[4]) * hy + std::fabs(ax[7]) * hz;
      ez = std::fabs(ax[2]) * hx + std::fabs(ax[5]) * hy + std::fabs(ax[8]) * hz;
    } else if (shape[s] == BG_SPHERE) {
      ex = ey = ez = d[0];
    } else {
      const double r = d[0], hl = (d[1] - 2 * r) * 0.5;
      ex = std::fabs(ax[3]) * hl + r; ey = std::fabs(ax[4]) * hl + r; ez = std::fabs(ax[5]) * hl + r;
    }
    const double g = m + size[s] * PIXEL;
    const double cx = position[s3], cy = position[s3 + 1], cz = position[s3 + 2];
    box[b6] = cx - ex - g; box[b6 + 1] = cy - ey - g; box[b6 + 2] = cz - ez - g;
    box[b6 + 3] = cx + ex + g; box[b6 + 4] = cy + ey + g; box[b6 + 5] = cz + ez + g;
  }

  // fat(): src/broadphase.js:206-219.
  void fatten(int s, double time) {
    const int b = 6 * s;
    if (type[s] == BG_STATIC) {
      for (int k = 0; k < 6; k++) fat[b + k] = box[b + k];
      return;
    }
    const double mg = size[s] * FAT;
    for (int k = 0; k < 3; k++) {
      const double d = velocity[3 * s + k] * time;
      fat[b + k] = box[b + k] - mg + (d < 0 ? d : 0);
      fat[b + k + 3] = box[b + k + 3] + mg + (d > 0 ? d : 0);
    }
  }

  // The grid the fat boxes are filed in.
  void cellRange(int s, int64_t* lo, int64_t* hi) const {
    for (int k = 0; k < 3; k++) {
      lo[k] = static_cast<int64_t>(std::floor(fat[6 * s + k] / cell));
      hi[k] = static_cast<int64_t>(std::floor(fat[6 * s + k + 3] / cell));
    }
  }
  static uint64_t cellKey(int64_t x, int64_t y, int64_t z) {
    return (static_cast<uint64_t>(x & 0x1fffff) << 42) | (static_cast<uint64_t>(y & 0x1fffff) << 21) |
           static_cast<uint64_t>(z & 0x1fffff);
  }
  void fileIn(int s) {
    int64_t lo[3], hi[3];
    cellRange(s, lo, hi);
    const int64_t cells = (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
    if (cells > 64) {
      large[s] = 1;
      largeList.push_back(s);
      return;
    }
    large[s] = 0;
    for (int64_t x = lo[0]; x <= hi[0]; x++)
      for (int64_t y = lo[1]; y <= hi[1]; y++)
        for (int64_t z = lo[2]; z <= hi[2]; z++) grid[cellKey(x, y, z)].push_back(s);
  }
  void fileOut(int s) {
    if (large[s]) {
      largeList.erase(std::find(largeList.begin(), largeList.end(), s));
      large[s] = 0;
      return;
    }
    int64_t lo[3], hi[3];
    cellRange(s, lo, hi);
    for (int64_t x = lo[0]; x <= hi[0]; x++)
      for (int64_t y = lo[1]; y <= hi[1]; y++)
        for (int64_t z = lo[2]; z <= hi[2]; z++) {
          auto it = grid.find(cellKey(x, y, z));
          if (it == grid.end()) continue;
          auto& v = it->second;
          v.erase(std::find(v.begin(), v.end(), s));
          if (v.empty()) grid.erase(it);
        }
  }
  void mark(int s) {
    if (isMoved[s]) return;
    isMoved[s] = 1;
    moved.push_back(s);
  }
  bool fatOverlap(int x, int y) const {
    const double* fa = &fat[6 * x];
    const double* fb = &fat[6 * y];
    return fa[0] <= fb[3] && fa[3] >= fb[0] && fa[1] <= fb[4] && fa[4] >= fb[1] && fa[2] <= fb[5] && fa[5] >= fb[2];
  }

  // Broadphase.update (src/broadphase.js:121-137) and candidates (146-165).
  void broadphase(double dt) {
    if (cell == 0) {
      double sum = 0;
      int count = 0;
      for (int s = 0; s < n; s++)
        if (type[s] != BG_STATIC) { sum += reach[s]; count++; }
      cell = count > 0 ? jmax(4 * sum / count, 0.25) : 1;
      for (int s = 0; s < n; s++) if (filed[s]) fileIn(s);
    }
    for (int i = 0; i < static_cast<int>(awakeList.size()) && i < awakeCount; i++) {
      const int s = awakeList[i], o = 6 * s;
      if (type[s] == BG_STATIC) continue;
      if (box[o] >= fat[o] && box[o + 1] >= fat[o + 1] && box[o + 2] >= fat[o + 2]
          && box[o + 3] <= fat[o + 3] && box[o + 4] <= fat[o + 4] && box[o + 5] <= fat[o + 5]) continue;
      fileOut(s);
      fatten(s, AHEAD * dt);
      fileIn(s);
      mark(s);
    }
    std::vector<int32_t> found;
    for (size_t i = 0; i < moved.size(); i++) {
      const int a = moved[i];
      isMoved[a] = 0;
      const bool aStatic = type[a] == BG_STATIC;
      found.clear();
      seenMark++;
      auto consider = [&](int b) {
        if (b == a || seen[b] == seenMark) return;
        seen[b] = seenMark;
        if (aStatic && type[b] == BG_STATIC) return;
        if (fatOverlap(a, b)) found.push_back(b);
      };
      if (large[a]) {
        for (auto& kv : grid)
          for (int b : kv.second) consider(b);
      } else {
        int64_t lo[3], hi[3];
        cellRange(a, lo, hi);
        for (int64_t x = lo[0]; x <= hi[0]; x++)
          for (int64_t y = lo[1]; y <= hi[1]; y++)
            for (int64_t z = lo[2]; z <= hi[2]; z++) {
              auto it = grid.find(cellKey(x, y, z));
              if (it == grid.end()) continue;
              for (int b : it->second) consider(b);
            }
      }
      for (int b : largeList) consider(b);
      std::sort(found.begin(), found.end());
      for (int b : found) pairs.found(a, b, type.data());
    }
    moved.clear();
  }

  int awakeCount = 0;

  // load(): src/contact.js:1244-1276 (box, sphere, capsule).
  void load(int slot, Shape& s) const {
    const int s3 = slot * 3;
    const double* d = &dims[s3];
    if (shape[slot] == BG_BOX) {
      s.kind = bearing::K_BOX;
      s.half[0] = d[0] * 0.5; s.half[1] = d[1] * 0.5; s.half[2] = d[2] * 0.5;
    } else if (shape[slot] == BG_SPHERE) {
      s.kind = bearing::K_SPHERE;
      s.half[0] = d[0];
    } else {
      s.kind = bearing::K_CAPSULE;
      s.half[0] = d[0];
      s.half[1] = (d[1] - 2 * d[0]) * 0.5;
    }
    s.center[0] = position[s3]; s.center[1] = position[s3 + 1]; s.center[2] = position[s3 + 2];
    const double scale = type[slot] == BG_DYNAMIC ? gravityScale[slot] : 0;
    s.weight[0] = gravity[0] * scale; s.weight[1] = gravity[1] * scale; s.weight[2] = gravity[2] * scale;
    for (int k = 0; k < 9; k++) s.axes[k] = axes[9 * slot + k];
  }

  // ---- the kept manifold: src/contact.js:388-595 (REUSE) ----

  // relative(): src/contact.js:596-610.  The smaller body's centre in the larger's frame and the
  // larger's rotation undone from the smaller's, into pose; returns the smaller body.
  int relative(int a, int b, double* pose) const {
    const int h = reach[a] >= reach[b] ? a : b, g = h == a ? b : a;
    const double* A = axes.data();
    const int h3 = 3 * h, g3 = 3 * g, h9 = 9 * h, h4 = 4 * h, g4 = 4 * g;
    const double dx = position[g3] - position[h3], dy = position[g3 + 1] - position[h3 + 1],
                 dz = position[g3 + 2] - position[h3 + 2];
    pose[0] = A[h9] * dx + A[h9 + 1] * dy + A[h9 + 2] * dz;
    pose[1] = A[h9 + 3] * dx + A[h9 + 4] * dy + A[h9 + 5] * dz;
    pose[2] = A[h9 + 6] * dx + A[h9 + 7] * dy + A[h9 + 8] * dz;
    const double ax = -rotation[h4], ay = -rotation[h4 + 1], az = -rotation[h4 + 2], aw = rotation[h4 + 3];
    const double bx = rotation[g4], by = rotation[g4 + 1], bz = rotation[g4 + 2], bw = rotation[g4 + 3];
    pose[3] = aw * bx + ax * bw + ay * bz - az * by;
    pose[4] = aw * by + ay * bw + az * bx - ax * bz;
    pose[5] = aw * bz + az * bw + ax * by - ay * bx;
    pose[6] = aw * bw - ax * bx - ay * by - az * bz;
    return g;
  }

  // moving(): src/contact.js:695-703.
  double moving(int a, int b) const {
    const double dt = stepDt;
    const int a3 = 3 * a, b3 = 3 * b;
    const double ga = type[a] == BG_DYNAMIC ? gravityScale[a] : 0, gb = type[b] == BG_DYNAMIC ? gravityScale[b] : 0;
    const double dx = velocity[b3] - velocity[a3], dy = velocity[b3 + 1] - velocity[a3 + 1],
                 dz = velocity[b3 + 2] - velocity[a3 + 2];
    const double gs = gb - ga, gl = std::sqrt(gravity[0] * gravity[0] + gravity[1] * gravity[1] + gravity[2] * gravity[2]) * std::fabs(gs);
    const double* w = angular.data();
    const double turning = std::sqrt(w[a3] * w[a3] + w[a3 + 1] * w[a3 + 1] + w[a3 + 2] * w[a3 + 2]) * reach[a]
      + std::sqrt(w[b3] * w[b3] + w[b3 + 1] * w[b3 + 1] + w[b3 + 2] * w[b3 + 2]) * reach[b];
    return (std::sqrt(dx * dx + dy * dy + dz * dz) + 0.5 * gl * dt + turning) * dt;
  }

  // keeps(): src/contact.js:516-537.
  bool keeps(int p, int a, int b, double tolerance) const {
    const double* pose = &pairs.cachePose[7 * p];
    double now[7];
    const int g = relative(a, b, now);
    const double ex = now[0] - pose[0], ey = now[1] - pose[1], ez = now[2] - pose[2];
    const double cx = -pose[3], cy = -pose[4], cz = -pose[5], cw = pose[6];
    const double rx = now[3], ry = now[4], rz = now[5], rw = now[6];
    const double ux = cw * rx + cx * rw + cy * rz - cz * ry;
    const double uy = cw * ry + cy * rw + cz * rx - cx * rz;
    const double uz = cw * rz + cz * rw + cx * ry - cy * rx;
    const double drift = std::sqrt(ex * ex + ey * ey + ez * ez) + 2 * std::sqrt(ux * ux + uy * uy + uz * uz) * reach[g];
    if (pairs.cacheLoss[p] + 2 * drift > tolerance) return false;
    if (jointHead[a] != 0 || jointHead[b] != 0) return false;
    return pairs.touching[p] == 1 || drift + moving(a, b) <= tolerance;
  }

  // rounded(): src/contact.js:571-575.
  double rounded(int s) const { return shape[s] == BG_SPHERE || shape[s] == BG_CAPSULE ? dims[3 * s] : 0; }

  // cored(): src/contact.js:578-585.
  void cored(int s, double* local) const {
    if (shape[s] == BG_SPHERE) { local[0] = 0; local[1] = 0; local[2] = 0; return; }
    if (shape[s] != BG_CAPSULE) return;
    const double half = (dims[3 * s + 1] - 2 * dims[3 * s]) * 0.5, y = local[1];
    local[0] = 0; local[1] = y < -half ? -half : y > half ? half : y; local[2] = 0;
  }

  // reused(): src/contact.js:468-510 (never shifted: no time of impact here).
  bool reused(int p, int a, int b, double tolerance, double margin, Manifold& mf) const {
    if (pairs.cached[p] == 0 || !keeps(p, a, b, tolerance)) return false;
    const int count = pairs.cachePoints[p];
    const double* A = axes.data();
    const int a3 = 3 * a, b3 = 3 * b, a9 = 9 * a, b9 = 9 * b;
    const double* ln = &pairs.cacheNormal[3 * p];
    const double lx = ln[0], ly = ln[1], lz = ln[2];
    const double nx = A[a9] * lx + A[a9 + 3] * ly + A[a9 + 6] * lz;
    const double ny = A[a9 + 1] * lx + A[a9 + 4] * ly + A[a9 + 7] * lz;
    const double nz = A[a9 + 2] * lx + A[a9 + 5] * ly + A[a9 + 8] * lz;
    mf.normal[0] = nx; mf.normal[1] = ny; mf.normal[2] = nz;
    const double ra = rounded(a), rb = -rounded(b);
    mf.count = count;
    double least = INF;
    for (int k = 0; k < count; k++) {
      const double* l = &pairs.cacheLocal[6 * (P * p + k)];
      const double ax = l[0], ay = l[1], az = l[2], bx = l[3], by = l[4], bz = l[5];
      const double pax = position[a3] + A[a9] * ax + A[a9 + 3] * ay + A[a9 + 6] * az + nx * ra;
      const double pay = position[a3 + 1] + A[a9 + 1] * ax + A[a9 + 4] * ay + A[a9 + 7] * az + ny * ra;
      const double paz = position[a3 + 2] + A[a9 + 2] * ax + A[a9 + 5] * ay + A[a9 + 8] * az + nz * ra;
      const double pbx = position[b3] + A[b9] * bx + A[b9 + 3] * by + A[b9 + 6] * bz + nx * rb;
      const double pby = position[b3 + 1] + A[b9 + 1] * bx + A[b9 + 4] * by + A[b9 + 7] * bz + ny * rb;
      const double pbz = position[b3 + 2] + A[b9 + 2] * bx + A[b9 + 5] * by + A[b9 + 8] * bz + nz * rb;
      const double sep = (pbx - pax) * nx + (pby - pay) * ny + (pbz - paz) * nz, half = 0.5 * sep;
      mf.separations[k] = sep;
      double* q = &mf.points[3 * k];
      if (rb != 0) {
        q[0] = pbx - nx * half; q[1] = pby - ny * half; q[2] = pbz - nz * half;
      } else if (ra != 0) {
        q[0] = pax + nx * half; q[1] = pay + ny * half; q[2] = paz + nz * half;
      } else {
        q[0] = (pax + pbx) * 0.5; q[1] = (pay + pby) * 0.5; q[2] = (paz + pbz) * 0.5;
      }
      mf.ids[k] = pairs.cacheId[P * p + k];
      if (sep < least) least = sep;
    }
    return !(least > margin);   // least(): src/contact.js:684-688
  }

  // remember(): src/contact.js:540-569, with the manifold collide() just found.
  void remember(int p, int a, int b, const Manifold& mf) {
    const int count = mf.count;
    pairs.cached[p] = 1;
    pairs.cachePoints[p] = static_cast<uint8_t>(count);
    relative(a, b, &pairs.cachePose[7 * p]);
    pairs.cacheLoss[p] = mf.loss;
    const double* A = axes.data();
    const int a3 = 3 * a, b3 = 3 * b, a9 = 9 * a, b9 = 9 * b;
    const double nx = mf.normal[0], ny = mf.normal[1], nz = mf.normal[2];
    double* ln = &pairs.cacheNormal[3 * p];
    ln[0] = A[a9] * nx + A[a9 + 1] * ny + A[a9 + 2] * nz;
    ln[1] = A[a9 + 3] * nx + A[a9 + 4] * ny + A[a9 + 5] * nz;
    ln[2] = A[a9 + 6] * nx + A[a9 + 7] * ny + A[a9 + 8] * nz;
    for (int k = 0; k < count; k++) {
      double* l = &pairs.cacheLocal[6 * (P * p + k)];
      const double half = 0.5 * mf.separations[k];
      const double px = mf.points[3 * k], py = mf.points[3 * k + 1], pz = mf.points[3 * k + 2];
      const double ax = px - nx * half - position[a3], ay = py - ny * half - position[a3 + 1], az = pz - nz * half - position[a3 + 2];
      const double bx = px + nx * half - position[b3], by = py + ny * half - position[b3 + 1], bz = pz + nz * half - position[b3 + 2];
      l[0] = A[a9] * ax + A[a9 + 1] * ay + A[a9 + 2] * az;
      l[1] = A[a9 + 3] * ax + A[a9 + 4] * ay + A[a9 + 5] * az;
      l[2] = A[a9 + 6] * ax + A[a9 + 7] * ay + A[a9 + 8] * az;
      l[3] = A[b9] * bx + A[b9 + 1] * by + A[b9 + 2] * bz;
      l[4] = A[b9 + 3] * bx + A[b9 + 4] * by + A[b9 + 5] * bz;
      l[5] = A[b9 + 6] * bx + A[b9 + 7] * by + A[b9 + 8] * bz;
      cored(a, l);
      cored(b, l + 3);
      pairs.cacheId[P * p + k] = mf.ids[k];
    }
  }

  // basis(): src/contact.js:1283-1292.
  void basis(int m) {
    const double nx = c.normal[3 * m], ny = c.normal[3 * m + 1], nz = c.normal[3 * m + 2];
    const double ax = std::fabs(nx), ay = std::fabs(ny), az = std::fabs(nz);
    double tx, ty, tz;
    if (ax <= ay && ax <= az) { tx = 0; ty = nz; tz = -ny; } else if (ay <= az) { tx = -nz; ty = 0; tz = nx; } else { tx = ny; ty = -nx; tz = 0; }
    const double l = 1 / std::sqrt(tx * tx + ty * ty + tz * tz);
    tx *= l; ty *= l; tz *= l;
    c.t1[3 * m] = tx; c.t1[3 * m + 1] = ty; c.t1[3 * m + 2] = tz;
    c.t2[3 * m] = ny * tz - nz * ty; c.t2[3 * m + 1] = nz * tx - nx * tz; c.t2[3 * m + 2] = nx * ty - ny * tx;
  }

  // emit(): src/contact.js:889-921 (whole bodies, sign 1, no parts, never shifted).
  int emit(int p, int a, int b, const Manifold& mf, double tol) {
    const int m = c.count++;
    c.ensure(c.count);
    c.a[m] = a; c.b[m] = b; c.pair[m] = p;
    c.points[m] = static_cast<uint8_t>(mf.count);
    for (int k = 0; k < 3; k++) c.normal[3 * m + k] = 1 * mf.normal[k];
    c.friction[m] = std::sqrt(friction[a] * friction[b]);
    c.restitution[m] = jmax(restitution[a], restitution[b]);
    c.tolerance[m] = tol;
    c.patch[m] = PIXEL * (type[a] != BG_DYNAMIC ? size[b] : type[b] != BG_DYNAMIC ? size[a] : jmin(size[a], size[b]));
    c.rollImpulse1[m] = 0; c.rollImpulse2[m] = 0; c.spinImpulse[m] = 0;
    c.tangentImpulse1[m] = 0; c.tangentImpulse2[m] = 0; c.drift1[m] = 0; c.drift2[m] = 0;
    for (int k = 0; k < mf.count; k++) {
      const int i = m * P + k;
      c.pid[i] = mf.ids[k];
      c.separation[i] = mf.separations[k];
      for (int q = 0; q < 3; q++) c.point[3 * i + q] = mf.points[3 * k + q];
      for (int q = 0; q < 3; q++) c.shift[3 * i + q] = 0;
      c.normalImpulse[i] = 0;
    }
    basis(m);
    return m;
  }

  // carry(): src/contact.js:999-1036, from the pair list.
  void carry(int p, int m) {
    const int remembered = pairs.points[p];
    if (remembered == 0) return;
    const int m3 = 3 * m;
    const double t1x = c.t1[m3], t1y = c.t1[m3 + 1], t1z = c.t1[m3 + 2];
    const double t2x = c.t2[m3], t2y = c.t2[m3 + 1], t2z = c.t2[m3 + 2];
    const int count = c.points[m], p3 = 3 * p;
    const double lx = pairs.twist[p3], ly = pairs.twist[p3 + 1], lz = pairs.twist[p3 + 2];
    if (count <= 2) {
      c.rollImpulse1[m] = lx * t1x + ly * t1y + lz * t1z;
      c.rollImpulse2[m] = lx * t2x + ly * t2y + lz * t2z;
    }
    c.spinImpulse[m] = lx * c.normal[m3] + ly * c.normal[m3 + 1] + lz * c.normal[m3 + 2];
    const double fx = pairs.friction[p3], fy = pairs.friction[p3 + 1], fz = pairs.friction[p3 + 2];
    c.tangentImpulse1[m] = fx * t1x + fy * t1y + fz * t1z;
    c.tangentImpulse2[m] = fx * t2x + fy * t2y + fz * t2z;
    bool same = false;
    for (int k = 0; k < count; k++) {
      const int i = m * P + k;
      const uint32_t id = c.pid[i];
      for (int j = 0; j < remembered; j++) {
        const int o = p * P + j;
        if (pairs.pid[o] != id) continue;
        c.normalImpulse[i] = pairs.normalImpulse[o];
        same = true;
        break;
      }
    }
    if (same) {
      const double sx = pairs.slip[p3], sy = pairs.slip[p3 + 1], sz = pairs.slip[p3 + 2];
      c.drift1[m] = sx * t1x + sy * t1y + sz * t1z;
      c.drift2[m] = sx * t2x + sy * t2y + sz * t2z;
    }
  }

  // The pairs narrow() handed to collide() this step, with the margin and tolerance it passed.
  std::vector<int32_t> narrowA, narrowB;
  std::vector<double> narrowMargin, narrowTol;
  // The pairs whose boxes meet (listPairs), and for the two-pass walk which of them kept their
  // manifold (nmKept) and where the others are in the list handed to the narrowphase.
  std::vector<int32_t> listA, listB, nmSent;
  std::vector<double> listMargin, listTol;
  std::vector<Manifold> nmKept;
  bool reuse = false;   // the kept-manifold cache (REUSE) on

  // narrow() with the narrowphase itself on another device (bw_set_narrowphase): the same walk
  // over the pairs (src/contact.js:312-327), in two passes.  The first drops the pairs whose fat
  // boxes no longer meet (each removal moves the last pair into its place, as in one pass) and
  // forgets those whose boxes miss, listing the rest with their margins; the device finds their
  // manifolds; the second emits and carries the pairs that touch and forgets the others, in pair
  // order.  No decision of the first pass depends on a manifold, so the rows, their order and the
  // pairs' memory are the one-pass walk's.
  // The first pass: the list of pairs whose boxes meet, each with its slot, margin, tolerance and
  // contact record (nmRecord, for bw_set_contact_step).
  // Each pair's fate depends only on its two bodies' boxes, so the boxes are compared first, on
  // several threads when the list is long (kGone: the fat boxes part, kApart: the boxes miss,
  // kMeet).  The removals then run in the walk's order over those marks alone: the walk removes
  // the pair at its position by moving the last pair (and its mark) there and looking again, and
  // never moves a pair it has passed, so every pair it keeps ends where the walk handles it.  Last,
  // the kept pairs are forgotten or listed by position, on the same threads: the walk's list, in
  // its order, with each pair's final position.
  enum : uint8_t { kGone = 0, kApart = 1, kMeet = 2 };
  // World.workers (src/world.js:501-524): how many threads besides the caller's a step may use
  // (bw_set_workers); -1, 'auto', is the machine's cores up to 16.  Results do not depend on it.
  int workers = -1;
  int hostThreads() const {
    if (workers >= 0) return std::min(workers + 1, 64);
    return std::min(16, static_cast<int>(std::max(1u, std::thread::hardware_concurrency())));
  }
  std::vector<uint8_t> fate;
  std::vector<int32_t> meetBefore;
  void handle(int lo, int hi, int at) {
    for (int p = lo; p < hi; p++) {
      if (fate[p] == kApart) {
        pairs.forget(p);
        continue;
      }
      const int a = pairs.a[p], b = pairs.b[p];
      const double tol = jmin(size[a], size[b]) * PIXEL;
      listA[at] = a; listB[at] = b; listMargin[at] = motion[a] + motion[b] + tol; listTol[at] = tol;
      nmPair[at] = p; nmRecord[at] = pairs.record[p];
      at++;
    }
  }
  uint8_t fateOf(int p) const {
    const int a = pairs.a[p], b = pairs.b[p];
    if (!fatOverlap(a, b)) return kGone;
    const int a6 = a * 6, b6 = b * 6;
    return box[a6] > box[b6 + 3] || box[b6] > box[a6 + 3] || box[a6 + 1] > box[b6 + 4] || box[b6 + 1] > box[a6 + 4]
               || box[a6 + 2] > box[b6 + 5] || box[b6 + 2] > box[a6 + 5]
           ? kApart
           : kMeet;
  }
  // Runs f(t, lo, hi) over `threads` consecutive ranges of [0, n), on threads when more than one.
  template <class F>
  static void ranges(int n, int threads, F f) {
    if (threads <= 1) {
      f(0, 0, n);
      return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++)
      pool.emplace_back([&f, t, threads, n] {
        f(t, static_cast<int>(static_cast<int64_t>(n) * t / threads),
          static_cast<int>(static_cast<int64_t>(n) * (t + 1) / threads));
      });
    for (auto& th : pool) th.join();
  }
  void listPairs() {
    constexpr int kPerThread = 1 << 16;
    const int hw = hostThreads();
    const int before = pairs.active;
    fate.resize(static_cast<size_t>(std::max(before, 1)));
    ranges(before, std::min(hw, before / kPerThread), [this](int, int lo, int hi) {
      for (int p = lo; p < hi; p++) fate[p] = fateOf(p);
    });
    for (int p = 0; p < pairs.active; p++)
      while (p < pairs.active && fate[p] == kGone) {
        fate[p] = fate[pairs.active - 1];   // the last pair moves into p
        pairs.remove(p);
      }
    const int active = pairs.active;
    const int chunks = std::max(1, std::min(hw, active / kPerThread));
    meetBefore.assign(static_cast<size_t>(chunks) + 1, 0);
    ranges(active, chunks, [this](int t, int lo, int hi) {
      int m = 0;
      for (int p = lo; p < hi; p++) m += fate[p] == kMeet;
      meetBefore[t + 1] = m;
    });
    for (int t = 0; t < chunks; t++) meetBefore[t + 1] += meetBefore[t];
    const size_t listed = static_cast<size_t>(meetBefore[chunks]);
    listA.resize(listed); listB.resize(listed); listMargin.resize(listed); listTol.resize(listed);
    nmPair.resize(listed); nmRecord.resize(listed);
    ranges(active, chunks, [this](int t, int lo, int hi) { handle(lo, hi, meetBefore[t]); });
  }

  int narrowOnDevice() {
    listPairs();
    // The pairs that keep their manifold (reused(), src/contact.js:356) need no narrowphase; the
    // rest go to the device, in list order.
    const size_t listed = listA.size();
    narrowA.clear(); narrowB.clear(); narrowMargin.clear(); narrowTol.clear();
    nmSent.assign(listed, -1);
    nmKept.resize(listed);
    for (size_t i = 0; i < listed; i++) {
      if (reuse && reused(nmPair[i], listA[i], listB[i], listTol[i], listMargin[i], nmKept[i])) continue;
      nmSent[i] = static_cast<int32_t>(narrowA.size());
      narrowA.push_back(listA[i]); narrowB.push_back(listB[i]);
      narrowMargin.push_back(listMargin[i]); narrowTol.push_back(listTol[i]);
    }
    const size_t n = narrowA.size();
    nmPoints.resize(std::max<size_t>(n, 1)); nmPid.resize(P * std::max<size_t>(n, 1));
    nmNormal.resize(3 * std::max<size_t>(n, 1)); nmPoint.resize(3 * P * std::max<size_t>(n, 1));
    nmSeparation.resize(P * std::max<size_t>(n, 1));
    if (n > 0) {
      bg_bodies B;
      fillBodies(&B);
      const bg_pairs list = {static_cast<int32_t>(n), narrowA.data(), narrowB.data(), narrowMargin.data(),
                             narrowTol.data()};
      bg_manifolds out = {nmPoints.data(), nmNormal.data(), nmPoint.data(), nmSeparation.data(), nmPid.data()};
      const int32_t rc = narrowFn(narrowUser, &B, gravity, &list, &out);
      if (rc != BG_OK) return rc;
    }
    Manifold mf;
    for (size_t i = 0; i < listed; i++) {
      const int p = nmPair[i];
      const int j = nmSent[i];
      if (j < 0) {
        const int m = emit(p, listA[i], listB[i], nmKept[i], listTol[i]);
        carry(p, m);
        continue;
      }
      const int count = nmPoints[j];
      if (count == 0) {
        pairs.forget(p);
        continue;
      }
      mf.count = count;
      mf.loss = 0;   // collide() of boxes, spheres and capsules falls short of nothing
      for (int k = 0; k < 3; k++) mf.normal[k] = nmNormal[3 * j + k];
      for (int k = 0; k < count; k++) {
        for (int q = 0; q < 3; q++) mf.points[3 * k + q] = nmPoint[3 * (P * j + k) + q];
        mf.separations[k] = nmSeparation[P * j + k];
        mf.ids[k] = nmPid[P * j + k];
      }
      if (reuse) remember(p, listA[i], listB[i], mf);
      const int m = emit(p, listA[i], listB[i], mf, listTol[i]);
      carry(p, m);
    }
    return BG_OK;
  }

  // narrow(): src/contact.js:296-327 with find() 334-368 (the reuse cache when `reuse` is on; no
  // time of impact).  narrowA.. list the pairs handed to collide().
  void narrow() {
    Shape sa, sb;
    Manifold mf;
    narrowA.clear(); narrowB.clear(); narrowMargin.clear(); narrowTol.clear();
    for (int p = 0; p < pairs.active;) {
      const int a = pairs.a[p], b = pairs.b[p];
      if (!fatOverlap(a, b)) {
        pairs.remove(p);
        continue;
      }
      const double tol = jmin(size[a], size[b]) * PIXEL;
      const int a6 = a * 6, b6 = b * 6;
      bool met = true;
      if (box[a6] > box[b6 + 3] || box[b6] > box[a6 + 3] || box[a6 + 1] > box[b6 + 4]
          || box[b6 + 1] > box[a6 + 4] || box[a6 + 2] > box[b6 + 5] || box[b6 + 2] > box[a6 + 5]) {
        pairs.forget(p);
        met = false;
      } else {
        const double margin = motion[a] + motion[b] + tol;
        if (!(reuse && reused(p, a, b, tol, margin, mf))) {
          narrowA.push_back(a); narrowB.push_back(b); narrowMargin.push_back(margin); narrowTol.push_back(tol);
          load(a, sa);
          load(b, sb);
          if (bearing::collide(sa, sb, margin, tol, mf) == 0) {
            pairs.forget(p);
            met = false;
          } else if (reuse) {
            remember(p, a, b, mf);
          }
        }
      }
      if (met) {
        const int m = emit(p, a, b, mf, tol);
        carry(p, m);
      }
      p++;
    }
  }

  // colour(): src/graph.js:105-170, and arrange() 178-214.
  void colourRows() {
    const int cnt = c.count;
    c.digits.assign(DIGITS + 1, 0);
    colour_manifolds(cnt, c.a.data(), c.b.data(), type.data(), frozen.data(), n, c.colour.data(), c.order.data(),
                     c.row.data(), c.digits.data(), c.starts);
    c.solved = c.starts[RESTING];
    arrange(cnt);
  }
  template <class T>
  void moveColumn(std::vector<T>& column, int per, int cnt) {
    std::vector<T> tmp(column.begin(), column.begin() + static_cast<size_t>(cnt) * per);
    for (int o = 0; o < cnt; o++) {
      const int f = c.order[o] * per, t = o * per;
      for (int i = 0; i < per; i++) column[t + i] = tmp[f + i];
    }
  }
  void arrange(int cnt) {
    moveColumn(c.normal, 3, cnt); moveColumn(c.t1, 3, cnt); moveColumn(c.t2, 3, cnt);
    moveColumn(c.friction, 1, cnt); moveColumn(c.restitution, 1, cnt); moveColumn(c.tolerance, 1, cnt);
    moveColumn(c.patch, 1, cnt); moveColumn(c.rollImpulse1, 1, cnt); moveColumn(c.rollImpulse2, 1, cnt);
    moveColumn(c.spinImpulse, 1, cnt); moveColumn(c.tangentImpulse1, 1, cnt); moveColumn(c.tangentImpulse2, 1, cnt);
    moveColumn(c.drift1, 1, cnt); moveColumn(c.drift2, 1, cnt); moveColumn(c.separation, P, cnt);
    moveColumn(c.normalImpulse, P, cnt); moveColumn(c.point, 3 * P, cnt); moveColumn(c.shift, 3 * P, cnt);
    moveColumn(c.a, 1, cnt); moveColumn(c.b, 1, cnt); moveColumn(c.pair, 1, cnt); moveColumn(c.colour, 1, cnt);
    moveColumn(c.pid, P, cnt); moveColumn(c.points, 1, cnt);
    for (int o = 0; o < cnt; o++) c.row[c.order[o]] = o;
  }

  // rest(): src/contact.js:1318-1329.
  void rest() {
    for (int m = c.solved; m < c.count; m++) {
      double least = INF;
      for (int k = 0; k < c.points[m]; k++) {
        const int i = m * P + k;
        if (c.separation[i] < least) least = c.separation[i];
        c.maxNormalImpulse[i] = c.normalImpulse[i];
        c.relativeVelocity[i] = 0;
      }
      c.gap[m] = least;
    }
  }

  // keep(): src/contact.js:1091-1115, into the pair list.
  void keep(int p, int m) {
    const int count = c.points[m], m3 = 3 * m, p3 = 3 * p;
    pairs.points[p] = static_cast<uint8_t>(count);
    const double t1x = c.t1[m3], t1y = c.t1[m3 + 1], t1z = c.t1[m3 + 2];
    const double t2x = c.t2[m3], t2y = c.t2[m3 + 1], t2z = c.t2[m3 + 2];
    const double r1 = c.rollImpulse1[m], r2 = c.rollImpulse2[m], sp = c.spinImpulse[m];
    pairs.twist[p3] = t1x * r1 + t2x * r2 + c.normal[m3] * sp;
    pairs.twist[p3 + 1] = t1y * r1 + t2y * r2 + c.normal[m3 + 1] * sp;
    pairs.twist[p3 + 2] = t1z * r1 + t2z * r2 + c.normal[m3 + 2] * sp;
    const double l1 = c.tangentImpulse1[m], l2 = c.tangentImpulse2[m];
    pairs.friction[p3] = t1x * l1 + t2x * l2;
    pairs.friction[p3 + 1] = t1y * l1 + t2y * l2;
    pairs.friction[p3 + 2] = t1z * l1 + t2z * l2;
    const double d1 = c.drift1[m], d2 = c.drift2[m];
    pairs.slip[p3] = t1x * d1 + t2x * d2;
    pairs.slip[p3 + 1] = t1y * d1 + t2y * d2;
    pairs.slip[p3 + 2] = t1z * d1 + t2z * d2;
    for (int k = 0; k < count; k++) {
      pairs.pid[p * P + k] = c.pid[m * P + k];
      pairs.normalImpulse[p * P + k] = c.normalImpulse[m * P + k];
    }
  }

  // Per row after begin_step: what narrow() used besides the row's columns (bw_row_memory).
  void rowMemory(int m, uint32_t* pidOut, double* marginOut, uint8_t* rememberedOut, uint32_t* memPid,
                 double* memory) const {
    const int p = c.pair[m], a = c.a[m], b = c.b[m];
    for (int k = 0; k < P; k++) pidOut[k] = k < c.points[m] ? c.pid[m * P + k] : 0;
    *marginOut = motion[a] + motion[b] + c.tolerance[m];
    *rememberedOut = pairs.points[p];
    for (int k = 0; k < P; k++) {
      memPid[k] = pairs.pid[p * P + k];
      memory[k] = pairs.normalImpulse[p * P + k];
    }
    for (int k = 0; k < 3; k++) {
      memory[4 + k] = pairs.friction[3 * p + k];
      memory[7 + k] = pairs.twist[3 * p + k];
      memory[10 + k] = pairs.slip[3 * p + k];
    }
    memory[13] = memory[14] = memory[15] = 0;
  }

  // The end of a step: transforms (src/world.js:1040-1057) and the step's stats.
  void finish(int rows, int solved, int points, const int32_t* starts) {
    for (int i = 0; i < awakeCount; i++) {
      const int s = awakeList[i], t7 = 7 * s;
      if (frozen[s] == 1) continue;
      for (int k = 0; k < 3; k++) transforms[t7 + k] = static_cast<float>(position[3 * s + k]);
      for (int k = 0; k < 4; k++) transforms[t7 + 3 + k] = static_cast<float>(rotation[4 * s + k]);
    }
    bw_stats& st = stats;
    st.bodies = n;
    st.awake = awakeCount;
    st.pairs = pairs.count;
    st.rows = rows;
    st.solved = solved;
    st.points = points;
    int colours = 0;
    for (int k = 0; k < COLOURS; k++) if (starts[k + 1] > starts[k]) colours++;
    st.colours = colours;
    st.overflow = rows > 0 ? starts[OVERFLOW_ + 1] - starts[OVERFLOW_] : 0;
    st.step = stepCount;
    stepDt = 0;
  }

  // A step with its contact side on another device (bw_set_contact_step): the host's share of
  // narrow() (src/contact.js:312-327: the pair list's upkeep), then everything from the narrowphase
  // to store() in one call, then the pairs reported apart forgotten and the touching flags kept.
  int32_t contactStep(double dt) {
    if (!(dt > 0) || !std::isfinite(dt)) {
      error = "step: dt must be a positive number of seconds";
      return BG_EINVAL;
    }
    stepCount++;
    stepDt = dt;
    const double gl = std::sqrt(gravity[0] * gravity[0] + gravity[1] * gravity[1] + gravity[2] * gravity[2]);
    for (int i = 0; i < awakeCount; i++) boundsOf(awakeList[i], dt, gl);
    broadphase(dt);
    c.count = 0;
    c.solved = 0;
    std::fill(c.starts, c.starts + COLOURS + 3, 0);
    listPairs();
    narrowA = listA; narrowB = listB; narrowMargin = listMargin; narrowTol = listTol;
    const size_t np = narrowA.size();
    nmPoints.assign(std::max<size_t>(np, 1), 0);
    nmTouching.assign(std::max<size_t>(np, 1), 0);
    bg_bodies B;
    fillBodies(&B);
    const bg_materials M = {friction.data(), restitution.data(), size.data(), reach.data()};
    const bg_contact_pairs CP = {{static_cast<int32_t>(np), narrowA.data(), narrowB.data(), narrowMargin.data(),
                                  narrowTol.data()},
                                 nmRecord.data(), reuse ? 1 : 0};
    bg_step S;
    S.dt = dt;
    S.substeps = substeps;
    for (int k = 0; k < 3; k++) S.gravity[k] = gravity[k];
    bg_contact_result R = {};
    R.points = nmPoints.data();
    R.touching = nmTouching.data();
    const int32_t rc = contactFn(contactUser, &B, &M, &CP, &S, &R);
    if (rc != BG_OK) {
      error = "step: the contact step failed";
      stepDt = 0;
      return rc;
    }
    for (size_t i = 0; i < np; i++) {
      const int p = nmPair[i];
      if (nmPoints[i] == 0) {
        pairs.forget(p);
        continue;
      }
      pairs.record[p] = static_cast<int32_t>(i);
      pairs.touching[p] = nmTouching[i];
    }
    finish(R.rows, R.solved, R.points_solved, R.starts);
    return BG_OK;
  }

  void fillBodies(bg_bodies* B) {
    B->capacity = n;
    B->awake_count = awakeCount;
    B->awake_list = awakeList.data();
    B->awake = awake.data();
    B->position = position.data(); B->rotation = rotation.data(); B->velocity = velocity.data();
    B->angular = angular.data(); B->tumbled = tumbled.data(); B->ceiling = ceiling.data();
    B->start = start.data(); B->start_q = startQ.data(); B->inv_i = invI.data();
    B->inv_mass = invMass.data(); B->inertia = inertia.data(); B->inv_inertia = invInertia.data();
    B->dims = dims.data(); B->damping = damping.data(); B->angular_damping = angularDamping.data();
    B->gravity_scale = gravityScale.data(); B->type = type.data(); B->shape = shape.data();
    B->frozen = frozen.data(); B->framed = framed.data(); B->lock = lock.data(); B->joint_head = jointHead.data();
  }
  void fillRows(bg_rows* R) {
    c.ensure(1);
    R->count = c.count;
    R->solved = c.solved;
    for (int k = 0; k < COLOURS + 3; k++) R->starts[k] = c.starts[k];
    R->row = c.row.data(); R->a = c.a.data(); R->b = c.b.data(); R->points = c.points.data();
    R->normal = c.normal.data(); R->t1 = c.t1.data(); R->t2 = c.t2.data();
    R->friction = c.friction.data(); R->restitution = c.restitution.data(); R->tolerance = c.tolerance.data();
    R->patch = c.patch.data(); R->separation = c.separation.data(); R->point = c.point.data(); R->shift = c.shift.data();
    R->normal_impulse = c.normalImpulse.data(); R->tangent_impulse1 = c.tangentImpulse1.data();
    R->tangent_impulse2 = c.tangentImpulse2.data(); R->roll_impulse1 = c.rollImpulse1.data();
    R->roll_impulse2 = c.rollImpulse2.data(); R->spin_impulse = c.spinImpulse.data();
    R->drift1 = c.drift1.data(); R->drift2 = c.drift2.data(); R->gap = c.gap.data();
    R->max_normal_impulse = c.maxNormalImpulse.data(); R->relative_velocity = c.relativeVelocity.data();
    R->sliding = c.sliding.data(); R->anchor_a = c.anchorA.data(); R->anchor_b = c.anchorB.data();
  }
};

extern "C" {

bw_world* bw_create(const bw_options* options) {
  bw_world* w = new bw_world();
  if (options != nullptr) {
    for (int k = 0; k < 3; k++) w->gravity[k] = options->gravity[k];
    w->substeps = options->substeps > 0 ? options->substeps : 8;
    w->reuse = options->reuse != 0;
  }
  w->c.alloc(0);
  return w;
}

void bw_destroy(bw_world* world) { delete world; }

const char* bw_last_error(const bw_world* world) { return world == nullptr ? "no world" : world->error.c_str(); }

int32_t bw_add_body(bw_world* w, const bw_body* spec) {
  if (w == nullptr || spec == nullptr) return BG_EINVAL;
  if (spec->shape < BG_BOX || spec->shape > BG_CAPSULE) {
    w->error = "addBody: only box, sphere and capsule shapes are on this path";
    return BG_EUNSUPPORTED;
  }
  if (spec->type != BG_DYNAMIC && spec->type != BG_STATIC && spec->type != KINEMATIC) {
    w->error = "addBody: type must be dynamic, static or kinematic";
    return BG_EINVAL;
  }
  // quat(): src/core/check.js:106-117.
  const double* r = spec->rotation;
  const double mq = jmax(jmax(jmax(std::fabs(r[0]), std::fabs(r[1])), std::fabs(r[2])), std::fabs(r[3]));
  if (!(mq > 0) || !std::isfinite(mq)) {
    w->error = "addBody: rotation must be 4 finite numbers, not all zero";
    return BG_EINVAL;
  }
  const int s = w->n++;
  w->resize(w->n);
  const int s3 = 3 * s, s4 = 4 * s;
  w->type[s] = static_cast<uint8_t>(spec->type);
  w->shape[s] = static_cast<uint8_t>(spec->shape);
  double* d = &w->dims[s3];
  const double rad = spec->radius;
  if (spec->shape == BG_BOX) { d[0] = spec->size[0]; d[1] = spec->size[1]; d[2] = spec->size[2]; }
  else { d[0] = rad; d[1] = spec->shape == BG_CAPSULE ? spec->height : 0; d[2] = 0; }
  // volume(): src/shapes.js:14-21.
  double v;
  if (spec->shape == BG_BOX) v = spec->size[0] * spec->size[1] * spec->size[2];
  else {
    const double ball = (4.0 / 3.0) * PI * rad * rad * rad;
    v = spec->shape == BG_SPHERE ? ball : PI * rad * rad * (spec->height - 2 * rad) + ball;
  }
  w->mass[s] = spec->mass > 0 ? spec->mass : spec->density * v;
  const double mass = w->mass[s];
  // inertia(): src/shapes.js:37-56.
  double* I = &w->inertia[s3];
  if (spec->shape == BG_BOX) {
    const double wd = spec->size[0], h = spec->size[1], dd = spec->size[2];
    I[0] = mass * (h * h + dd * dd) / 12;
    I[1] = mass * (wd * wd + dd * dd) / 12;
    I[2] = mass * (wd * wd + h * h) / 12;
  } else if (spec->shape == BG_SPHERE) {
    I[0] = I[1] = I[2] = 0.4 * mass * rad * rad;
  } else {
    const double L = spec->height - 2 * rad;
    const double cylinder = PI * rad * rad * L, ball = (4.0 / 3.0) * PI * rad * rad * rad;
    const double mc = mass * cylinder / (cylinder + ball), ms = mass * ball / (cylinder + ball);
    I[1] = mc * rad * rad / 2 + ms * 0.4 * rad * rad;
    I[0] = I[2] = mc * (L * L / 12 + rad * rad / 4) + ms * (0.4 * rad * rad + L * L / 4 + 3 * L * rad / 8);
  }
  for (int k = 0; k < 3; k++) w->invInertia[s3 + k] = I[k] > 0 ? 1 / I[k] : 0;
  w->invMass[s] = spec->type == BG_DYNAMIC ? 1 / mass : 0;
  if (spec->shape == BG_BOX) {
    w->size[s] = jmin(jmin(spec->size[0], spec->size[1]), spec->size[2]);
    w->reach[s] = 0.5 * std::sqrt(spec->size[0] * spec->size[0] + spec->size[1] * spec->size[1] + spec->size[2] * spec->size[2]);
  } else {
    w->size[s] = 2 * rad;
    w->reach[s] = spec->shape == BG_CAPSULE ? spec->height * 0.5 : rad;
  }
  w->friction[s] = spec->friction;
  w->restitution[s] = spec->restitution;
  w->damping[s] = spec->damping;
  w->angularDamping[s] = spec->angular_damping;
  w->gravityScale[s] = spec->gravity_scale;
  const double x = r[0] / mq, y = r[1] / mq, z = r[2] / mq, ww = r[3] / mq;
  const double sc = 1 / std::sqrt(x * x + y * y + z * z + ww * ww);
  for (int k = 0; k < 3; k++) w->position[s3 + k] = spec->position[k];
  w->rotation[s4] = x * sc; w->rotation[s4 + 1] = y * sc; w->rotation[s4 + 2] = z * sc; w->rotation[s4 + 3] = ww * sc;
  for (int k = 0; k < 3; k++) {
    w->velocity[s3 + k] = spec->velocity[k];
    w->angular[s3 + k] = spec->angular[k];
    w->tumbled[s3 + k] = std::numeric_limits<double>::quiet_NaN();
  }
  w->ceiling[s] = 0;
  // Where the solver measures a step's movement from, for a body not moving in it: _place,
  // src/world.js:2294-2296.
  for (int k = 0; k < 3; k++) w->start[s3 + k] = w->position[s3 + k];
  // Transform as placed.
  for (int k = 0; k < 3; k++) w->transforms[7 * s + k] = static_cast<float>(w->position[s3 + k]);
  for (int k = 0; k < 4; k++) w->transforms[7 * s + 3 + k] = static_cast<float>(w->rotation[s4 + k]);
  // Bounds, the broadphase, and the awake list (src/world.js:563-578).
  w->boundsOf(s, 0, 0);
  w->fatten(s, 0);
  w->filed[s] = 1;
  if (w->cell != 0) w->fileIn(s);
  w->mark(s);
  if (spec->type != BG_STATIC) {
    w->awakeList[w->awakeCount++] = s;
    w->awake[s] = 1;
  }
  return s;
}

int32_t bw_set_workers(bw_world* w, int32_t workers) {
  if (w == nullptr || workers < -1) return BG_EINVAL;
  w->workers = workers;
  return BG_OK;
}

int32_t bw_set_narrowphase(bw_world* w, bw_narrowphase fn, void* user) {
  if (w == nullptr) return BG_EINVAL;
  w->narrowFn = fn;
  w->narrowUser = user;
  return BG_OK;
}

int32_t bw_set_solver(bw_world* w, bw_solver solver, void* user) {
  if (w == nullptr) return BG_EINVAL;
  w->solver = solver;
  w->solverUser = user;
  return BG_OK;
}

int32_t bw_set_contact_step(bw_world* w, bw_contact_solver fn, void* user) {
  if (w == nullptr) return BG_EINVAL;
  if (w->stepCount > 0) {
    w->error = "set_contact_step: the contact memory would be lost; set it before the first step";
    return BG_EINVAL;
  }
  w->contactFn = fn;
  w->contactUser = user;
  return BG_OK;
}

int32_t bw_begin_step(bw_world* w, double dt) {
  if (w == nullptr) return BG_EINVAL;
  if (w->contactFn != nullptr) {
    w->error = "begin_step: the world's rows live on the contact step's device (bw_set_contact_step)";
    return BG_EUNSUPPORTED;
  }
  if (!(dt > 0) || !std::isfinite(dt)) {
    w->error = "step: dt must be a positive number of seconds";
    return BG_EINVAL;
  }
  w->stepCount++;
  w->stepDt = dt;
  const double* g = w->gravity;
  const double gl = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  for (int i = 0; i < w->awakeCount; i++) w->boundsOf(w->awakeList[i], dt, gl);
  w->broadphase(dt);
  w->c.count = 0;
  if (w->narrowFn != nullptr) {
    const int32_t rc = w->narrowOnDevice();
    if (rc != BG_OK) {
      w->error = "step: the narrowphase failed";
      return rc;
    }
  } else {
    w->narrow();
  }
  if (w->c.count > 0) {
    w->colourRows();
    if (w->c.solved < w->c.count) w->rest();
  } else {
    std::fill(w->c.starts, w->c.starts + COLOURS + 3, 0);
    w->c.solved = 0;
  }
  w->begun = true;
  return BG_OK;
}

int32_t bw_end_step(bw_world* w) {
  if (w == nullptr || !w->begun) return BG_EINVAL;
  w->begun = false;
  Contacts& c = w->c;
  // store(): src/contact.js:1067-1088 (slipped() ran in the solve stage).
  for (int f = 0; f < c.count; f++) {
    const int m = c.row[f];
    if (m >= c.solved) continue;
    w->keep(c.pair[m], m);
  }
  // touched(): src/contact.js:2178-2213, the touching flags only.
  for (int f = 0; f < c.count; f++) {
    const int m = c.row[f];
    bool meets = c.gap[m] <= c.tolerance[m];
    for (int k = 0; k < c.points[m] && !meets; k++) meets = c.maxNormalImpulse[m * P + k] > 0;
    w->pairs.touching[c.pair[m]] = meets ? 1 : 0;
  }
  int pts = 0;
  for (int m = 0; m < c.solved; m++) pts += c.points[m];
  w->finish(c.count, c.solved, pts, c.starts);
  return BG_OK;
}

int32_t bw_row_memory_get(const bw_world* w, bw_row_memory* out) {
  if (w == nullptr || out == nullptr || !w->begun) return BG_EINVAL;
  const int n = w->c.count;
  if (n > 0 && (out->pid == nullptr || out->margin == nullptr || out->remembered == nullptr ||
                out->memory_pid == nullptr || out->memory == nullptr))
    return BG_EINVAL;
  for (int m = 0; m < n; m++)
    w->rowMemory(m, out->pid + P * m, out->margin + m, out->remembered + m, out->memory_pid + P * m,
                 out->memory + BW_MEMORY * m);
  return BG_OK;
}

int32_t bw_materials(const bw_world* w, double* friction, double* restitution) {
  if (w == nullptr || friction == nullptr || restitution == nullptr) return BG_EINVAL;
  for (int s = 0; s < w->n; s++) {
    friction[s] = w->friction[static_cast<size_t>(s)];
    restitution[s] = w->restitution[static_cast<size_t>(s)];
  }
  return BG_OK;
}

bw_world* bw_clone(const bw_world* w) {
  if (w == nullptr) return nullptr;
  try {
    return new bw_world(*w);
  } catch (const std::exception&) {
    return nullptr;
  }
}

int32_t bw_copy(bw_world* dst, const bw_world* src) {
  if (dst == nullptr || src == nullptr) return BG_EINVAL;
  if (dst == src) return BG_OK;
  try {
    *dst = *src;
  } catch (const std::exception&) {
    return BG_ENOMEM;
  }
  return BG_OK;
}

int32_t bw_colour_rows(const bg_bodies* B, int32_t count, const int32_t* a, const int32_t* b, int32_t* colour,
                       int32_t* order, int32_t* starts, int32_t* solved) {
  if (B == nullptr || starts == nullptr || solved == nullptr || count < 0 || B->capacity < 0) return BG_EINVAL;
  if (count > 0 && (a == nullptr || b == nullptr || colour == nullptr || order == nullptr || B->type == nullptr ||
                    B->frozen == nullptr))
    return BG_EINVAL;
  for (int m = 0; m < count; m++)
    if (a[m] < 0 || a[m] >= B->capacity || b[m] < 0 || b[m] >= B->capacity || a[m] == b[m]) return BG_EINVAL;
  std::vector<int32_t> scratch(static_cast<size_t>(std::max(count, 1))), digits(DIGITS + 1);
  colour_manifolds(count, a, b, B->type, B->frozen, B->capacity, colour, order, scratch.data(), digits.data(), starts);
  *solved = starts[RESTING];
  return BG_OK;
}

int32_t bw_narrow_pairs(const bw_world* w, bg_pairs* out) {
  if (w == nullptr || out == nullptr) return BG_EINVAL;
  out->count = static_cast<int32_t>(w->narrowA.size());
  out->a = w->narrowA.data();
  out->b = w->narrowB.data();
  out->margin = w->narrowMargin.data();
  out->tolerance = w->narrowTol.data();
  return BG_OK;
}

int32_t bw_collide_pairs(const bg_bodies* B, const double* gravity, const bg_pairs* pairs, bg_manifolds* out,
                         int32_t threads) {
  if (B == nullptr || gravity == nullptr || pairs == nullptr || out == nullptr || pairs->count < 0) return BG_EINVAL;
  const int n = pairs->count;
  if (n > 0 && (pairs->a == nullptr || pairs->b == nullptr || pairs->margin == nullptr || pairs->tolerance == nullptr ||
                out->points == nullptr || out->normal == nullptr || out->point == nullptr ||
                out->separation == nullptr || out->pid == nullptr || B->position == nullptr ||
                B->rotation == nullptr || B->dims == nullptr || B->shape == nullptr || B->type == nullptr ||
                B->gravity_scale == nullptr))
    return BG_EINVAL;
  for (int i = 0; i < n; i++)
    if (pairs->a[i] < 0 || pairs->a[i] >= B->capacity || pairs->b[i] < 0 || pairs->b[i] >= B->capacity) return BG_EINVAL;
  // load(), from the columns: the same shapes the step's narrowphase builds
  auto shape_of = [&](int slot, Shape& s) {
    const double* d = B->dims + 3 * slot;
    if (B->shape[slot] == BG_BOX) {
      s.kind = bearing::K_BOX;
      s.half[0] = d[0] * 0.5; s.half[1] = d[1] * 0.5; s.half[2] = d[2] * 0.5;
    } else if (B->shape[slot] == BG_SPHERE) {
      s.kind = bearing::K_SPHERE;
      s.half[0] = d[0]; s.half[1] = 0; s.half[2] = 0;
    } else {
      s.kind = bearing::K_CAPSULE;
      s.half[0] = d[0]; s.half[1] = (d[1] - 2 * d[0]) * 0.5; s.half[2] = 0;
    }
    for (int k = 0; k < 3; k++) s.center[k] = B->position[3 * slot + k];
    const double scale = B->type[slot] == BG_DYNAMIC ? B->gravity_scale[slot] : 0;
    for (int k = 0; k < 3; k++) s.weight[k] = gravity[k] * scale;
    axesOf(B->rotation + 4 * slot, s.axes);
  };
  const int nt = std::max(1, std::min<int>(threads, 64));
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; t++)
    pool.emplace_back([&, t]() {
      Shape sa, sb;
      Manifold mf;
      for (int i = static_cast<int>(static_cast<int64_t>(n) * t / nt); i < static_cast<int64_t>(n) * (t + 1) / nt; i++) {
        shape_of(pairs->a[i], sa);
        shape_of(pairs->b[i], sb);
        const int count = bearing::collide(sa, sb, pairs->margin[i], pairs->tolerance[i], mf);
        out->points[i] = static_cast<uint8_t>(count);
        for (int k = 0; k < 3; k++) out->normal[3 * i + k] = count > 0 ? mf.normal[k] : 0;
        for (int k = 0; k < P; k++) {
          const bool used = k < count;
          for (int q = 0; q < 3; q++) out->point[3 * (P * i + k) + q] = used ? mf.points[3 * k + q] : 0;
          out->separation[P * i + k] = used ? mf.separations[k] : 0;
          out->pid[P * i + k] = used ? mf.ids[k] : 0;
        }
      }
    });
  for (auto& th : pool) th.join();
  return BG_OK;
}

int32_t bw_bodies_view(bw_world* w, bg_bodies* out) {
  if (w == nullptr || out == nullptr) return BG_EINVAL;
  w->fillBodies(out);
  return BG_OK;
}

int32_t bw_rows_view(bw_world* w, bg_rows* out) {
  if (w == nullptr || out == nullptr) return BG_EINVAL;
  w->fillRows(out);
  return BG_OK;
}

int32_t bw_step_params(const bw_world* w, bg_step* out) {
  if (w == nullptr || out == nullptr) return BG_EINVAL;
  out->dt = w->stepDt;
  out->substeps = w->substeps;
  for (int k = 0; k < 3; k++) out->gravity[k] = w->gravity[k];
  return BG_OK;
}

int32_t bw_step(bw_world* w, double dt) {
  if (w == nullptr) return BG_EINVAL;
  if (w->contactFn != nullptr) return w->contactStep(dt);
  if (w->solver == nullptr) {
    w->error = "step: no solve stage set (bw_set_solver)";
    return BG_EUNSUPPORTED;
  }
  int32_t rc = bw_begin_step(w, dt);
  if (rc != BG_OK) return rc;
  bg_bodies B;
  bg_rows R;
  bg_step S;
  w->fillBodies(&B);
  w->fillRows(&R);
  bw_step_params(w, &S);
  rc = w->solver(w->solverUser, &B, &R, &S);
  if (rc != BG_OK) {
    w->begun = false;
    w->error = "step: the solve stage failed";
    return rc;
  }
  return bw_end_step(w);
}

const float* bw_transforms(const bw_world* w) { return w == nullptr ? nullptr : w->transforms.data(); }

int32_t bw_stats_get(const bw_world* w, bw_stats* out) {
  if (w == nullptr || out == nullptr) return BG_EINVAL;
  *out = w->stats;
  return BG_OK;
}

}  // extern "C"

// ---- batches of worlds ----

namespace {

// Runs f(i) for i in [0, n) on up to `threads` threads, each taking every threads-th index.
template <class F>
void parallel(int n, int threads, F f) {
  if (threads <= 1 || n <= 1) {
    for (int i = 0; i < n; i++) f(i);
    return;
  }
  const int t = threads < n ? threads : n;
  std::vector<std::thread> pool;
  for (int k = 0; k < t; k++)
    pool.emplace_back([&, k] {
      for (int i = k; i < n; i += t) f(i);
    });
  for (auto& th : pool) th.join();
}

template <class T>
struct Col {
  std::vector<T> v;
  T* at(size_t off) { return v.data() + off; }
};

}  // namespace

struct bw_batch {
  std::vector<bw_world*> worlds;
  std::vector<int32_t> body_off, awake_off, row_off, starts;
  // bodies, end to end
  std::vector<double> position, rotation, velocity, angular, tumbled, ceiling, start, startQ, invI, invMass, inertia,
      invInertia, dims, damping, angularDamping, gravityScale;
  std::vector<uint8_t> type, shape, frozen, framed, lock, awake;
  std::vector<int32_t> jointHead, awakeList;
  // rows, end to end
  std::vector<int32_t> row, a, b;
  std::vector<uint8_t> points, sliding;
  std::vector<double> normal, t1, t2, friction, restitution, tolerance, patch, separation, point, shift, normalImpulse,
      tangentImpulse1, tangentImpulse2, rollImpulse1, rollImpulse2, spinImpulse, drift1, drift2, gap, maxNormalImpulse,
      relativeVelocity, anchorA, anchorB;
  double dt = 0;
  bool begun = false;
};

namespace {

template <class T>
void put(std::vector<T>& dst, size_t off, const T* src, size_t n) {
  if (n) std::memcpy(dst.data() + off, src, n * sizeof(T));
}
template <class T>
void take(const std::vector<T>& src, size_t off, T* dst, size_t n) {
  if (n) std::memcpy(dst, src.data() + off, n * sizeof(T));
}

}  // namespace

extern "C" {

bw_batch* bw_batch_create(bw_world* const* worlds, int32_t count) {
  if (worlds == nullptr || count < 1) return nullptr;
  bw_batch* b = new bw_batch();
  b->worlds.assign(worlds, worlds + count);
  for (bw_world* w : b->worlds)
    if (w == nullptr) {
      delete b;
      return nullptr;
    }
  return b;
}

void bw_batch_destroy(bw_batch* b) { delete b; }

int32_t bw_batch_begin_step(bw_batch* b, double dt, int32_t threads) {
  if (b == nullptr) return BG_EINVAL;
  const int n = static_cast<int>(b->worlds.size());
  std::vector<int32_t> rcs(static_cast<size_t>(n), 0);
  parallel(n, threads, [&](int i) { rcs[static_cast<size_t>(i)] = bw_begin_step(b->worlds[static_cast<size_t>(i)], dt); });
  for (int32_t rc : rcs)
    if (rc != BG_OK) return rc;
  b->body_off.assign(static_cast<size_t>(n) + 1, 0);
  b->awake_off.assign(static_cast<size_t>(n) + 1, 0);
  b->row_off.assign(static_cast<size_t>(n) + 1, 0);
  b->starts.assign(static_cast<size_t>(n) * BG_STARTS, 0);
  for (int i = 0; i < n; i++) {
    bw_world* w = b->worlds[static_cast<size_t>(i)];
    b->body_off[i + 1] = b->body_off[i] + w->n;
    b->awake_off[i + 1] = b->awake_off[i] + w->awakeCount;
    b->row_off[i + 1] = b->row_off[i] + w->c.count;
    for (int k = 0; k < BG_STARTS; k++) b->starts[static_cast<size_t>(i) * BG_STARTS + k] = w->c.starts[k];
  }
  const size_t nb = static_cast<size_t>(b->body_off[n]), na = static_cast<size_t>(b->awake_off[n]),
               nr = static_cast<size_t>(b->row_off[n]);
  auto sz = [](auto& v, size_t k) { v.resize(k > 0 ? k : 1); };
  sz(b->position, 3 * nb); sz(b->rotation, 4 * nb); sz(b->velocity, 3 * nb); sz(b->angular, 3 * nb);
  sz(b->tumbled, 3 * nb); sz(b->ceiling, nb); sz(b->start, 3 * nb); sz(b->startQ, 4 * nb); sz(b->invI, 6 * nb);
  sz(b->invMass, nb); sz(b->inertia, 3 * nb); sz(b->invInertia, 3 * nb); sz(b->dims, 3 * nb); sz(b->damping, nb);
  sz(b->angularDamping, nb); sz(b->gravityScale, nb); sz(b->type, nb); sz(b->shape, nb); sz(b->frozen, nb);
  sz(b->framed, nb); sz(b->lock, nb); sz(b->awake, nb); sz(b->jointHead, nb); sz(b->awakeList, na);
  sz(b->row, nr); sz(b->a, nr); sz(b->b, nr); sz(b->points, nr); sz(b->sliding, nr); sz(b->normal, 3 * nr);
  sz(b->t1, 3 * nr); sz(b->t2, 3 * nr); sz(b->friction, nr); sz(b->restitution, nr); sz(b->tolerance, nr);
  sz(b->patch, nr); sz(b->separation, 4 * nr); sz(b->point, 12 * nr); sz(b->shift, 12 * nr); sz(b->normalImpulse, 4 * nr);
  sz(b->tangentImpulse1, nr); sz(b->tangentImpulse2, nr); sz(b->rollImpulse1, nr); sz(b->rollImpulse2, nr);
  sz(b->spinImpulse, nr); sz(b->drift1, nr); sz(b->drift2, nr); sz(b->gap, nr); sz(b->maxNormalImpulse, 4 * nr);
  sz(b->relativeVelocity, 4 * nr); sz(b->anchorA, 3 * nr); sz(b->anchorB, 3 * nr);
  parallel(n, threads, [&](int i) {
    bw_world* w = b->worlds[static_cast<size_t>(i)];
    const size_t o = static_cast<size_t>(b->body_off[i]), q = static_cast<size_t>(b->awake_off[i]),
                 r = static_cast<size_t>(b->row_off[i]), s = static_cast<size_t>(w->n), m = static_cast<size_t>(w->c.count);
    put(b->position, 3 * o, w->position.data(), 3 * s); put(b->rotation, 4 * o, w->rotation.data(), 4 * s);
    put(b->velocity, 3 * o, w->velocity.data(), 3 * s); put(b->angular, 3 * o, w->angular.data(), 3 * s);
    put(b->tumbled, 3 * o, w->tumbled.data(), 3 * s); put(b->ceiling, o, w->ceiling.data(), s);
    put(b->start, 3 * o, w->start.data(), 3 * s); put(b->startQ, 4 * o, w->startQ.data(), 4 * s);
    put(b->invI, 6 * o, w->invI.data(), 6 * s); put(b->invMass, o, w->invMass.data(), s);
    put(b->inertia, 3 * o, w->inertia.data(), 3 * s); put(b->invInertia, 3 * o, w->invInertia.data(), 3 * s);
    put(b->dims, 3 * o, w->dims.data(), 3 * s); put(b->damping, o, w->damping.data(), s);
    put(b->angularDamping, o, w->angularDamping.data(), s); put(b->gravityScale, o, w->gravityScale.data(), s);
    put(b->type, o, w->type.data(), s); put(b->shape, o, w->shape.data(), s); put(b->frozen, o, w->frozen.data(), s);
    put(b->framed, o, w->framed.data(), s); put(b->lock, o, w->lock.data(), s); put(b->awake, o, w->awake.data(), s);
    put(b->jointHead, o, w->jointHead.data(), s);
    put(b->awakeList, q, w->awakeList.data(), static_cast<size_t>(w->awakeCount));
    Contacts& c = w->c;
    put(b->row, r, c.row.data(), m); put(b->a, r, c.a.data(), m); put(b->b, r, c.b.data(), m);
    put(b->points, r, c.points.data(), m); put(b->sliding, r, c.sliding.data(), m);
    put(b->normal, 3 * r, c.normal.data(), 3 * m); put(b->t1, 3 * r, c.t1.data(), 3 * m); put(b->t2, 3 * r, c.t2.data(), 3 * m);
    put(b->friction, r, c.friction.data(), m); put(b->restitution, r, c.restitution.data(), m);
    put(b->tolerance, r, c.tolerance.data(), m); put(b->patch, r, c.patch.data(), m);
    put(b->separation, 4 * r, c.separation.data(), 4 * m); put(b->point, 12 * r, c.point.data(), 12 * m);
    put(b->shift, 12 * r, c.shift.data(), 12 * m); put(b->normalImpulse, 4 * r, c.normalImpulse.data(), 4 * m);
    put(b->tangentImpulse1, r, c.tangentImpulse1.data(), m); put(b->tangentImpulse2, r, c.tangentImpulse2.data(), m);
    put(b->rollImpulse1, r, c.rollImpulse1.data(), m); put(b->rollImpulse2, r, c.rollImpulse2.data(), m);
    put(b->spinImpulse, r, c.spinImpulse.data(), m); put(b->drift1, r, c.drift1.data(), m); put(b->drift2, r, c.drift2.data(), m);
    put(b->gap, r, c.gap.data(), m); put(b->maxNormalImpulse, 4 * r, c.maxNormalImpulse.data(), 4 * m);
    put(b->relativeVelocity, 4 * r, c.relativeVelocity.data(), 4 * m);
    put(b->anchorA, 3 * r, c.anchorA.data(), 3 * m); put(b->anchorB, 3 * r, c.anchorB.data(), 3 * m);
  });
  b->dt = dt;
  b->begun = true;
  return BG_OK;
}

int32_t bw_batch_views(bw_batch* b, bg_bodies* B, bg_rows* R, bg_worlds* W, bg_step* S) {
  if (b == nullptr || !b->begun || B == nullptr || R == nullptr || W == nullptr || S == nullptr) return BG_EINVAL;
  const size_t n = b->worlds.size();
  B->capacity = b->body_off[n];
  B->awake_count = b->awake_off[n];
  B->awake_list = b->awakeList.data(); B->awake = b->awake.data();
  B->position = b->position.data(); B->rotation = b->rotation.data(); B->velocity = b->velocity.data();
  B->angular = b->angular.data(); B->tumbled = b->tumbled.data(); B->ceiling = b->ceiling.data();
  B->start = b->start.data(); B->start_q = b->startQ.data(); B->inv_i = b->invI.data();
  B->inv_mass = b->invMass.data(); B->inertia = b->inertia.data(); B->inv_inertia = b->invInertia.data();
  B->dims = b->dims.data(); B->damping = b->damping.data(); B->angular_damping = b->angularDamping.data();
  B->gravity_scale = b->gravityScale.data(); B->type = b->type.data(); B->shape = b->shape.data();
  B->frozen = b->frozen.data(); B->framed = b->framed.data(); B->lock = b->lock.data(); B->joint_head = b->jointHead.data();
  R->count = b->row_off[n];
  R->solved = 0;
  for (int k = 0; k < BG_STARTS; k++) R->starts[k] = 0;
  R->row = b->row.data(); R->a = b->a.data(); R->b = b->b.data(); R->points = b->points.data();
  R->normal = b->normal.data(); R->t1 = b->t1.data(); R->t2 = b->t2.data(); R->friction = b->friction.data();
  R->restitution = b->restitution.data(); R->tolerance = b->tolerance.data(); R->patch = b->patch.data();
  R->separation = b->separation.data(); R->point = b->point.data(); R->shift = b->shift.data();
  R->normal_impulse = b->normalImpulse.data(); R->tangent_impulse1 = b->tangentImpulse1.data();
  R->tangent_impulse2 = b->tangentImpulse2.data(); R->roll_impulse1 = b->rollImpulse1.data();
  R->roll_impulse2 = b->rollImpulse2.data(); R->spin_impulse = b->spinImpulse.data(); R->drift1 = b->drift1.data();
  R->drift2 = b->drift2.data(); R->gap = b->gap.data(); R->max_normal_impulse = b->maxNormalImpulse.data();
  R->relative_velocity = b->relativeVelocity.data(); R->sliding = b->sliding.data(); R->anchor_a = b->anchorA.data();
  R->anchor_b = b->anchorB.data();
  W->count = static_cast<int32_t>(n);
  W->body_offset = b->body_off.data();
  W->awake_offset = b->awake_off.data();
  W->row_offset = b->row_off.data();
  W->starts = b->starts.data();
  W->gravity = nullptr;
  bw_step_params(b->worlds[0], S);
  S->dt = b->dt;
  return BG_OK;
}

int32_t bw_batch_row_memory(const bw_batch* b, bw_row_memory* out) {
  if (b == nullptr || !b->begun || out == nullptr) return BG_EINVAL;
  const size_t n = b->worlds.size();
  for (size_t i = 0; i < n; i++) {
    const size_t r = static_cast<size_t>(b->row_off[i]);
    bw_row_memory part = {out->pid + P * r, out->margin + r, out->remembered + r, out->memory_pid + P * r,
                          out->memory + BW_MEMORY * r};
    const int32_t rc = bw_row_memory_get(b->worlds[i], &part);
    if (rc != BG_OK) return rc;
  }
  return BG_OK;
}

int32_t bw_batch_end_step(bw_batch* b, int32_t threads) {
  if (b == nullptr || !b->begun) return BG_EINVAL;
  b->begun = false;
  const int n = static_cast<int>(b->worlds.size());
  std::vector<int32_t> rcs(static_cast<size_t>(n), 0);
  parallel(n, threads, [&](int i) {
    bw_world* w = b->worlds[static_cast<size_t>(i)];
    const size_t o = static_cast<size_t>(b->body_off[i]), r = static_cast<size_t>(b->row_off[i]),
                 s = static_cast<size_t>(w->n), m = static_cast<size_t>(w->c.count);
    take(b->position, 3 * o, w->position.data(), 3 * s); take(b->rotation, 4 * o, w->rotation.data(), 4 * s);
    take(b->velocity, 3 * o, w->velocity.data(), 3 * s); take(b->angular, 3 * o, w->angular.data(), 3 * s);
    take(b->tumbled, 3 * o, w->tumbled.data(), 3 * s); take(b->ceiling, o, w->ceiling.data(), s);
    take(b->start, 3 * o, w->start.data(), 3 * s); take(b->startQ, 4 * o, w->startQ.data(), 4 * s);
    take(b->invI, 6 * o, w->invI.data(), 6 * s);
    Contacts& c = w->c;
    take(b->normalImpulse, 4 * r, c.normalImpulse.data(), 4 * m);
    take(b->tangentImpulse1, r, c.tangentImpulse1.data(), m); take(b->tangentImpulse2, r, c.tangentImpulse2.data(), m);
    take(b->rollImpulse1, r, c.rollImpulse1.data(), m); take(b->rollImpulse2, r, c.rollImpulse2.data(), m);
    take(b->spinImpulse, r, c.spinImpulse.data(), m); take(b->drift1, r, c.drift1.data(), m); take(b->drift2, r, c.drift2.data(), m);
    take(b->gap, r, c.gap.data(), m); take(b->maxNormalImpulse, 4 * r, c.maxNormalImpulse.data(), 4 * m);
    take(b->relativeVelocity, 4 * r, c.relativeVelocity.data(), 4 * m); take(b->sliding, r, c.sliding.data(), m);
    take(b->anchorA, 3 * r, c.anchorA.data(), 3 * m); take(b->anchorB, 3 * r, c.anchorB.data(), 3 * m);
    rcs[static_cast<size_t>(i)] = bw_end_step(w);
  });
  for (int32_t rc : rcs)
    if (rc != BG_OK) return rc;
  return BG_OK;
}

}  // extern "C"

// ---- the host side's share of a step's adjoint ----

namespace bgad {
namespace {
thread_local Tape* t_tape = nullptr;
}
Tape* thread_tape() { return t_tape; }
}  // namespace bgad

namespace {

using bgad::TV;

// A tape of the calling host thread's own, for the life of one object.
struct HostTape {
  std::vector<int32_t> pa, pb;
  std::vector<double> da, db, adj;
  bgad::Tape t{};
  explicit HostTape(int cap) : pa(static_cast<size_t>(cap)), pb(static_cast<size_t>(cap)), da(static_cast<size_t>(cap)),
                               db(static_cast<size_t>(cap)), adj(static_cast<size_t>(cap)) {
    t = bgad::Tape{0, cap, pa.data(), pb.data(), da.data(), db.data(), adj.data(), 0, 0};
    bgad::t_tape = &t;
  }
  ~HostTape() { bgad::t_tape = nullptr; }
};

// Math.max with JavaScript's NaN and signed-zero rules, for recorded values.
TV jmax_tv(const TV& a, const TV& b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a > b) return a;
  if (b > a) return b;
  if (a == 0 && b == 0) return std::signbit(a.v) ? b : a;
  return a;
}

// axesOf: src/core/math.js:222-227.
void axes_tv(const TV* q, TV* ax) {
  const TV x = q[0], y = q[1], z = q[2], w = q[3];
  ax[0] = 1 - 2 * (y * y + z * z); ax[1] = 2 * (x * y + z * w); ax[2] = 2 * (x * z - y * w);
  ax[3] = 2 * (x * y - z * w); ax[4] = 1 - 2 * (x * x + z * z); ax[5] = 2 * (y * z + x * w);
  ax[6] = 2 * (x * z + y * w); ax[7] = 2 * (y * z - x * w); ax[8] = 1 - 2 * (x * x + y * y);
}

// World w of a batch (or the one world): its first slot, first row and row count.
struct Part {
  int body0, row0, nrows, solved;
};

std::vector<Part> parts_of(const bg_rows* R, const bg_worlds* W) {
  std::vector<Part> out;
  if (W == nullptr) {
    out.push_back(Part{0, 0, R->count, R->solved});
    return out;
  }
  for (int i = 0; i < W->count; i++)
    out.push_back(Part{W->body_offset[i], W->row_offset[i], W->row_offset[i + 1] - W->row_offset[i],
                       W->starts[BG_STARTS * i + RESTING]});
  return out;
}

}  // namespace

extern "C" {

int32_t bw_keep_backward(const bg_rows* R, const bg_worlds* W, const double* g, bg_row_grads* o) {
  if (R == nullptr || g == nullptr || o == nullptr) return BG_EINVAL;
  for (const Part& part : parts_of(R, W)) {
    for (int j = 0; j < part.nrows; j++) {
      const int m = part.row0 + j, m3 = 3 * m;
      const double* gm = g + BW_MEMORY * static_cast<size_t>(m);
      for (int k = 0; k < P; k++) o->normal_impulse[P * m + k] = 0;
      o->tangent_impulse1[m] = 0; o->tangent_impulse2[m] = 0; o->roll_impulse1[m] = 0; o->roll_impulse2[m] = 0;
      o->spin_impulse[m] = 0; o->drift1[m] = 0; o->drift2[m] = 0;
      if (j >= part.solved) continue;   // a resting row: its pair keeps what it had
      const double* t1 = R->t1 + m3;
      const double* t2 = R->t2 + m3;
      const double* n = R->normal + m3;
      const double r1 = R->roll_impulse1[m], r2 = R->roll_impulse2[m], sp = R->spin_impulse[m];
      const double l1 = R->tangent_impulse1[m], l2 = R->tangent_impulse2[m];
      const double d1 = R->drift1[m], d2 = R->drift2[m];
      const double* gt = gm + 7;   // twist = t1 r1 + t2 r2 + n sp
      const double* gf = gm + 4;   // friction = t1 l1 + t2 l2
      const double* gs = gm + 10;  // slip = t1 d1 + t2 d2
      for (int c = 0; c < 3; c++) {
        o->roll_impulse1[m] += t1[c] * gt[c];
        o->roll_impulse2[m] += t2[c] * gt[c];
        o->spin_impulse[m] += n[c] * gt[c];
        o->tangent_impulse1[m] += t1[c] * gf[c];
        o->tangent_impulse2[m] += t2[c] * gf[c];
        o->drift1[m] += t1[c] * gs[c];
        o->drift2[m] += t2[c] * gs[c];
        o->t1[m3 + c] += r1 * gt[c] + l1 * gf[c] + d1 * gs[c];
        o->t2[m3 + c] += r2 * gt[c] + l2 * gf[c] + d2 * gs[c];
        o->normal[m3 + c] += sp * gt[c];
      }
      for (int k = 0; k < R->points[m]; k++) o->normal_impulse[P * m + k] = gm[k];
    }
  }
  return BG_OK;
}

int32_t bw_narrow_backward(const bg_bodies* B, const bg_rows* R, const bg_worlds* W, const bw_row_memory* M,
                           const double* gravity, const double* friction, const double* restitution,
                           const bg_row_grads* g, double* gp, double* gq, double* gfr, double* gre, double* gmem,
                           int32_t threads) {
  if (B == nullptr || R == nullptr || M == nullptr || gravity == nullptr || friction == nullptr || restitution == nullptr ||
      g == nullptr || gp == nullptr || gq == nullptr || gfr == nullptr || gre == nullptr || gmem == nullptr)
    return BG_EINVAL;
  const std::vector<Part> parts = parts_of(R, W);
  std::vector<int32_t> rcs(parts.size(), BG_OK);
  parallel(static_cast<int>(parts.size()), threads, [&](int wi) {
    const Part& part = parts[static_cast<size_t>(wi)];
    HostTape tape(1 << 16);
    bgad::Tape* t = &tape.t;
    for (int j = 0; j < part.nrows; j++) {
      const int m = part.row0 + j, m3 = 3 * m;
      double* gm = gmem + BW_MEMORY * static_cast<size_t>(m);
      for (int k = 0; k < BW_MEMORY; k++) gm[k] = 0;
      const int a = part.body0 + R->a[m], b = part.body0 + R->b[m];
      bgad::reset(t);
      TV pose[2][7];
      bearing::ShapeT<TV> sh[2];
      for (int e = 0; e < 2; e++) {
        const int s = e == 0 ? a : b;
        for (int k = 0; k < 3; k++) pose[e][k] = bgad::leaf(B->position[3 * s + k]);
        for (int k = 0; k < 4; k++) pose[e][3 + k] = bgad::leaf(B->rotation[4 * s + k]);
        const double* d = B->dims + 3 * s;
        bearing::ShapeT<TV>& x = sh[e];
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
        for (int k = 0; k < 3; k++) x.center[k] = pose[e][k];
        const double scale = B->type[s] == BG_DYNAMIC ? B->gravity_scale[s] : 0;
        for (int k = 0; k < 3; k++) x.weight[k] = gravity[k] * scale;
        axes_tv(pose[e] + 3, x.axes);
      }
      const TV fa = bgad::leaf(friction[a]), fb = bgad::leaf(friction[b]);
      const TV ea = bgad::leaf(restitution[a]), eb = bgad::leaf(restitution[b]);
      // narrowphase: src/collide.js:204-218
      bearing::ManifoldT<TV> mf;
      bearing::collideT<TV>(sh[0], sh[1], M->margin[m], R->tolerance[m], mf);
      const int count = R->points[m];
      bool same_points = mf.count == count;
      for (int k = 0; k < count && same_points; k++) same_points = mf.ids[k] == M->pid[P * m + k];
      if (!same_points || t->overflow) {
        rcs[static_cast<size_t>(wi)] = BG_EFAULT;
        return;
      }
      // emit: src/contact.js:901-921, basis: 1283-1292
      const TV fr = sqrt(fa * fb);
      const TV re = jmax_tv(ea, eb);
      const TV nx = mf.normal[0], ny = mf.normal[1], nz = mf.normal[2];
      const TV ax = fabs(nx), ay = fabs(ny), az = fabs(nz);
      TV tx, ty, tz;
      if (ax <= ay && ax <= az) { tx = 0; ty = nz; tz = -ny; } else if (ay <= az) { tx = -nz; ty = 0; tz = nx; } else { tx = ny; ty = -nx; tz = 0; }
      const TV l = 1 / sqrt(tx * tx + ty * ty + tz * tz);
      tx *= l; ty *= l; tz *= l;
      const TV T1[3] = {tx, ty, tz};
      const TV T2[3] = {ny * tz - nz * ty, nz * tx - nx * tz, nx * ty - ny * tx};
      const TV N[3] = {nx, ny, nz};
      // carry: src/contact.js:999-1036
      const int remembered = M->remembered[m];
      TV mem[13];
      TV ni[P], ti1, ti2, ri1, ri2, si, dr1, dr2;
      if (remembered > 0) {
        const double* src = M->memory + BW_MEMORY * static_cast<size_t>(m);
        for (int k = 0; k < 13; k++) mem[k] = bgad::leaf(src[k]);
        const TV* twist = mem + 7;
        const TV* fric = mem + 4;
        const TV* slip = mem + 10;
        if (count <= 2) {
          ri1 = twist[0] * T1[0] + twist[1] * T1[1] + twist[2] * T1[2];
          ri2 = twist[0] * T2[0] + twist[1] * T2[1] + twist[2] * T2[2];
        }
        si = twist[0] * N[0] + twist[1] * N[1] + twist[2] * N[2];
        ti1 = fric[0] * T1[0] + fric[1] * T1[1] + fric[2] * T1[2];
        ti2 = fric[0] * T2[0] + fric[1] * T2[1] + fric[2] * T2[2];
        bool same = false;
        for (int k = 0; k < count; k++) {
          for (int q = 0; q < remembered; q++) {
            if (M->memory_pid[P * m + q] != M->pid[P * m + k]) continue;
            ni[k] = mem[q];
            same = true;
            break;
          }
        }
        if (same) {
          dr1 = slip[0] * T1[0] + slip[1] * T1[1] + slip[2] * T1[2];
          dr2 = slip[0] * T2[0] + slip[1] * T2[1] + slip[2] * T2[2];
        }
      }
      if (t->overflow) {
        rcs[static_cast<size_t>(wi)] = BG_ENOMEM;
        return;
      }
      bgad::clear_adjoints(t);
      for (int c = 0; c < 3; c++) {
        bgad::seed(t, N[c], g->normal[m3 + c]);
        bgad::seed(t, T1[c], g->t1[m3 + c]);
        bgad::seed(t, T2[c], g->t2[m3 + c]);
      }
      bgad::seed(t, fr, g->friction[m]);
      bgad::seed(t, re, g->restitution[m]);
      for (int k = 0; k < count; k++) {
        bgad::seed(t, mf.separations[k], g->separation[P * m + k]);
        for (int c = 0; c < 3; c++) bgad::seed(t, mf.points[3 * k + c], g->point[12 * m + 3 * k + c]);
        bgad::seed(t, ni[k], g->normal_impulse[P * m + k]);
      }
      bgad::seed(t, ti1, g->tangent_impulse1[m]);
      bgad::seed(t, ti2, g->tangent_impulse2[m]);
      bgad::seed(t, ri1, g->roll_impulse1[m]);
      bgad::seed(t, ri2, g->roll_impulse2[m]);
      bgad::seed(t, si, g->spin_impulse[m]);
      bgad::seed(t, dr1, g->drift1[m]);
      bgad::seed(t, dr2, g->drift2[m]);
      bgad::sweep(t);
      for (int e = 0; e < 2; e++) {
        const int s = e == 0 ? a : b;
        if (B->type[s] != BG_DYNAMIC || B->inv_mass[s] == 0) continue;
        for (int k = 0; k < 3; k++) gp[3 * s + k] += bgad::adjoint(t, pose[e][k]);
        for (int k = 0; k < 4; k++) gq[4 * s + k] += bgad::adjoint(t, pose[e][3 + k]);
      }
      gfr[a] += bgad::adjoint(t, fa);
      gfr[b] += bgad::adjoint(t, fb);
      gre[a] += bgad::adjoint(t, ea);
      gre[b] += bgad::adjoint(t, eb);
      if (remembered > 0)
        for (int k = 0; k < 13; k++) gm[k] = bgad::adjoint(t, mem[k]);
    }
  });
  for (int32_t rc : rcs)
    if (rc != BG_OK) return rc;
  return BG_OK;
}

}  // extern "C"
