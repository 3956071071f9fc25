// href_bounds.cpp -- TEST INFRASTRUCTURE ONLY: the reference's GenRBFBounds compute program
// (deviceCodeBounds.hlsl, rewritten to C++ by hlsl2cpp.py, unchanged otherwise) over every leaf.
#include "href_common.h"

namespace bounds_module {
#include "deviceCodeBounds.hlsl.cpp"

void href_intersection(int) {}
void href_any_hit(void *, const void *) {}
}  // namespace bounds_module

using namespace bounds_module;

// boxes: 6 floats per leaf (lo xyz, hi xyz), ceil(n / ppl) leaves; radiusmap: decoded texels
extern "C" void href_bounds(const float *particles, uint32_t n, uint32_t ppl, float rbf_radius,
                            const float *radiusmap, int nr, float *boxes) {
  static Texture1D rm;
  rm = Texture1D{radiusmap, nr, 1};
  const uint32_t nleaves = (n + ppl - 1) / ppl;
  pc.aabbs = gprt::Buffer{boxes};
  pc.numAABBs = nleaves;
  pc.particles = gprt::Buffer{const_cast<float *>(particles)};
  pc.numParticles = n;
  pc.particlesPerLeaf = (uint16_t)ppl;
  pc.rbfRadius = rbf_radius;
  pc.radiusmap = gprt::Texture{&rm};
  UnusedRecord rec{};
  for (uint32_t l = 0; l < nleaves; ++l) {
    href_thread().dispatch_thread = uint3(l, 0, 0);
    GenRBFBounds(rec);
  }
}
