// The narrowphase for spheres, capsules and boxes: where two placed shapes touch, as one
// normal and up to four points (src/collide.js:1-1229, restated for the host side of the
// step; hulls, meshes and parts are not on this path).
#pragma once

#include <cstdint>

namespace bearing {

// Shape kinds in dispatch order: src/collide.js:44 (a pair is handled lower kind first).
enum Kind { K_SPHERE = 0, K_CAPSULE = 1, K_BOX = 2 };

// One placed shape: src/collide.js:52-93.  T is the scalar (double for the step itself; see
// collide_impl.hpp).
template <class T>
struct ShapeT {
  int kind = K_BOX;
  T center[3] = {0, 0, 0};
  T axes[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  T half[3] = {0, 0, 0};
  T weight[3] = {0, 0, 0};
};
using Shape = ShapeT<double>;

constexpr int MAX_POINTS = 4;

// src/collide.js:181-197.
template <class T>
struct ManifoldT {
  int count = 0;
  T normal[3] = {0, 0, 0};
  T points[3 * MAX_POINTS] = {};
  T separations[MAX_POINTS] = {};
  uint32_t ids[MAX_POINTS] = {};
  T loss = 0;
};
using Manifold = ManifoldT<double>;

// collide(a, b, margin, tolerance, out): src/collide.js:204-218.  Returns the point count.
int collide(const Shape& a, const Shape& b, double margin, double tolerance, Manifold& out);

}  // namespace bearing
