// The narrowphase for the step itself: collideT (collide_impl.hpp) in double.
#include "collide_impl.hpp"

namespace bearing {

int collide(const Shape& a, const Shape& b, double margin, double tolerance, Manifold& out) {
  return collideT<double>(a, b, margin, tolerance, out);
}

}  // namespace bearing
