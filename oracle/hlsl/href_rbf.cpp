// href_rbf.cpp -- TEST INFRASTRUCTURE ONLY: the reference's ParticleRBFRayGen with its
// ParticleRBFIntersection / ParticleRBFAnyHit programs (deviceCodeRBF.hlsl, rewritten to C++ by
// hlsl2cpp.py, unchanged otherwise), run on the CPU over the leaf boxes of the reference's own
// bounds program. One call renders spp successive launches (frameID + k, accumID + k), as the
// reference's frame loop does one per frame (hostCode.cpp:800-815).
#include "href_common.h"

namespace rbf_module {
#include "deviceCodeRBF.hlsl.cpp"

void href_intersection(int) {
  UnusedRecord r{};
  ParticleRBFIntersection(r);
}
void href_any_hit(void *payload, const void *attribute) {
  UnusedRecord r{};
  ParticleRBFAnyHit(r, *static_cast<RBFPayload *>(payload), *static_cast<const RBFAttribute *>(attribute));
}
}  // namespace rbf_module

using namespace rbf_module;

// ip: accum_id, frame_id, enable_blue_noise, show_noise, visualize_attributes, particles_per_leaf,
//     spp, reverse traversal order
// fp: light azimuth, elevation, ambient, camera pos[3], dir_00[3], dir_du[3], dir_dv[3],
//     rbf_radius, unit, global AABB min[3], max[3]
// textures: decoded texel values (colormap RGBA x nc, radiusmap x nr, densitymap x nd); stbn:
// RGBA floats (UNORM values) or NULL
extern "C" void href_rbf_render(const float *particles, uint32_t n, const float *boxes, uint32_t nleaves,
                                const int32_t *ip, const float *fp, const float *colormap, int nc,
                                const float *radiusmap, int nr, const float *densitymap, int nd,
                                const float *stbn, int stbn_w, int stbn_h, int w, int h, float *accum,
                                float *image, int threads) {
  static Texture1D cm, rm, dm;
  static Texture2D noise;
  cm = Texture1D{colormap, nc, 4};
  rm = Texture1D{radiusmap, nr, 1};
  dm = Texture1D{densitymap, nd, 1};
  static const float black[4] = {0, 0, 0, 0};
  noise = stbn ? Texture2D{stbn, stbn_w, stbn_h} : Texture2D{black, 1, 1};
  href_scene() = HrefScene{boxes, nleaves, ip[7] != 0};
  pc.enableBlueNoise = (uint16_t)ip[2];
  pc.showNoise = (uint16_t)ip[3];
  pc.visualizeAttributes = (uint16_t)ip[4];
  pc.particlesPerLeaf = (uint16_t)ip[5];
  pc.light.azimuth = fp[0];
  pc.light.elevation = fp[1];
  pc.light.ambient = fp[2];
  pc.camera.pos = float3(fp[3], fp[4], fp[5]);
  pc.camera.dir_00 = float3(fp[6], fp[7], fp[8]);
  pc.camera.dir_du = float3(fp[9], fp[10], fp[11]);
  pc.camera.dir_dv = float3(fp[12], fp[13], fp[14]);
  pc.rbfRadius = fp[15];
  pc.unit = fp[16];
  pc.particles = gprt::Buffer{const_cast<float *>(particles)};
  pc.numParticles = n;
  pc.colormap = gprt::Texture{&cm};
  pc.radiusmap = gprt::Texture{&rm};
  pc.densitymap = gprt::Texture{&dm};
  RayGenData rec;
  rec.stbnTexture = gprt::Texture{&noise};
  rec.imageBuffer = gprt::Buffer{image};
  rec.accumBuffer = gprt::Buffer{accum};
  rec.fbSize = int2(w, h);
  rec.globalAABBMin = float3(fp[17], fp[18], fp[19]);
  rec.globalAABBMax = float3(fp[20], fp[21], fp[22]);
  const int spp = ip[6] > 0 ? ip[6] : 1;
  for (int k = 0; k < spp; ++k) {
    pc.accumID = (uint16_t)(ip[0] + k);
    pc.frameID = (uint16_t)(ip[1] + k);
    const long total = (long)w * (long)h;
#pragma omp parallel for schedule(dynamic, 8) num_threads(href_threads(threads))
    for (long q = 0; q < total; ++q) {
      HrefThread &th = href_thread();
      th.launch_index = uint3(q % w, q / w, 0);
      th.launch_dims = uint3(w, h, 1);
      ParticleRBFRayGen(rec);
    }
  }
}
