// href_taa.cpp -- TEST INFRASTRUCTURE ONLY: the reference's CompositeGui compute program
// (deviceCodeCommon.hlsl, rewritten to C++ by hlsl2cpp.py, unchanged otherwise) over every pixel,
// with an empty (transparent) GUI layer.
#include "href_common.h"

namespace taa_module {
#include "deviceCodeCommon.hlsl.cpp"

void href_intersection(int) {}
void href_any_hit(void *, const void *) {}
}  // namespace taa_module

using namespace taa_module;

extern "C" void href_taa(const float *image, const float *prev, float *taa, uint32_t *bgra, int w, int h,
                         int disable) {
  static Texture2D img, gui;
  static float *zeros = nullptr;
  static size_t nz = 0;
  const size_t np = (size_t)w * (size_t)h;
  if (nz < np) {
    delete[] zeros;
    zeros = new float[4 * np]();
    nz = np;
  }
  img = Texture2D{image, w, h};
  gui = Texture2D{zeros, w, h};
  pc.disableTAA = (uint16_t)disable;
  pc.showNoise = 0;
  pc.fbSize = int2(w, h);
  pc.imageTexture = gprt::Texture{&img};
  pc.guiTexture = gprt::Texture{&gui};
  pc.frameBuffer = gprt::Buffer{bgra};
  pc.taaBuffer = gprt::Buffer{taa};
  pc.taaPrevBuffer = gprt::Buffer{const_cast<float *>(prev)};
  UnusedRecord rec{};
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      href_thread().dispatch_thread = uint3(x, y, 0);
      CompositeGui(rec);
    }
}
