// href_splat.cpp -- TEST INFRASTRUCTURE ONLY: the reference's ParticleSplatRayGen with its
// ParticleSplatIntersection / ParticleSplatAnyHit programs (deviceCodeSplat.hlsl, rewritten to
// C++ by hlsl2cpp.py, unchanged otherwise), run on the CPU over the leaf boxes of the reference's
// own bounds program.
#include "href_common.h"

namespace splat_module {
#include "deviceCodeSplat.hlsl.cpp"

void href_intersection(int) {
  UnusedRecord r{};
  ParticleSplatIntersection(r);
}
void href_any_hit(void *payload, const void *attribute) {
  UnusedRecord r{};
  ParticleSplatAnyHit(r, *static_cast<SplatPayload *>(payload), *static_cast<const ParticleSample *>(attribute));
}
}  // namespace splat_module

using namespace splat_module;

// ip / fp / textures as href_rbf_render (ip[6] unused)
extern "C" void href_splat_render(const float *particles, uint32_t n, const float *boxes, uint32_t nleaves,
                                  const int32_t *ip, const float *fp, const float *colormap, int nc,
                                  const float *densitymap, int nd, int w, int h, float *image, int threads) {
  static Texture1D cm, dm;
  cm = Texture1D{colormap, nc, 4};
  dm = Texture1D{densitymap, nd, 1};
  href_scene() = HrefScene{boxes, nleaves, ip[7] != 0};
  pc.accumID = (uint16_t)ip[0];
  pc.frameID = (uint16_t)ip[1];
  pc.enableBlueNoise = (uint16_t)ip[2];
  pc.showNoise = (uint16_t)ip[3];
  pc.visualizeAttributes = (uint16_t)ip[4];
  pc.particlesPerLeaf = (uint16_t)ip[5];
  pc.camera.pos = float3(fp[3], fp[4], fp[5]);
  pc.camera.dir_00 = float3(fp[6], fp[7], fp[8]);
  pc.camera.dir_du = float3(fp[9], fp[10], fp[11]);
  pc.camera.dir_dv = float3(fp[12], fp[13], fp[14]);
  pc.rbfRadius = fp[15];
  pc.unit = fp[16];
  pc.particles = gprt::Buffer{const_cast<float *>(particles)};
  pc.numParticles = n;
  pc.colormap = gprt::Texture{&cm};
  pc.densitymap = gprt::Texture{&dm};
  RayGenData rec;
  rec.imageBuffer = gprt::Buffer{image};
  rec.fbSize = int2(w, h);
  rec.globalAABBMin = float3(fp[17], fp[18], fp[19]);
  rec.globalAABBMax = float3(fp[20], fp[21], fp[22]);
  const long total = (long)w * (long)h;
#pragma omp parallel for schedule(dynamic, 8) num_threads(href_threads(threads))
  for (long q = 0; q < total; ++q) {
    HrefThread &th = href_thread();
    th.launch_index = uint3(q % w, q / w, 0);
    th.launch_dims = uint3(w, h, 1);
    ParticleSplatRayGen(rec);
  }
}
