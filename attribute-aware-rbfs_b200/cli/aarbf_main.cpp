// aarbf -- headless command-line front end, the argparse CLI of the reference's hostCode.cpp
// (:103-131) on top of the C ABI: --particles PATH, --camera 10 floats, --radius F,
// --particles-per-leaf U, plus headless options (--out, --frames, --spp, --width, --height,
// --mode track|march|splat, --taa, --start-frame, --rebuild).
//
// Pipeline per hostCode.cpp: load the series (or the built-in synthetic one, :147-168), compute
// the space-time domain over all frames (:183-193), then per frame: upload, build the BVH on the
// first frame (Hilbert sort, bounds, LBVH) and refit it on a frame change of the same particle
// count (the frame sorted along the curve, its leaves refitting the first build's topology, as the
// reference's gprtAccelUpdate path, :751-794; --rebuild builds every frame instead), render and
// optionally resolve TAA, writing <out>_<frame>.pfm.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "aarbf.h"

namespace {

struct Args {
  std::string particles;
  std::vector<float> camera;
  float radius = 0.0f;
  unsigned ppl = 0;
  std::string out = "aarbf";
  int frames = 1, start = 0, spp = 1, width = 1920, height = 1080;
  std::string mode = "track";
  bool taa = false;
  bool rebuild = false;
};

void usage() {
  fprintf(stderr,
          "Usage: aarbf [--particles PATH] [--camera px py pz ax ay az ux uy uz fovy] [--radius R]\n"
          "             [--particles-per-leaf N] [--out PREFIX] [--frames N] [--start-frame F]\n"
          "             [--spp N] [--width W] [--height H] [--mode track|march|splat] [--taa]\n"
          "             [--rebuild]\n");
}

bool parse(int argc, char** argv, Args& a) {
  for (int i = 1; i < argc; ++i) {
    std::string k = argv[i];
    auto need = [&](int n) {
      if (i + n >= argc) {
        fprintf(stderr, "%s: expected %d value(s)\n", k.c_str(), n);
        return false;
      }
      return true;
    };
    if (k == "--particles") {
      if (!need(1)) return false;
      a.particles = argv[++i];
    } else if (k == "--camera") {
      if (!need(10)) return false;
      for (int j = 0; j < 10; ++j) a.camera.push_back(std::strtof(argv[++i], nullptr));
    } else if (k == "--radius") {
      if (!need(1)) return false;
      a.radius = std::strtof(argv[++i], nullptr);
    } else if (k == "--particles-per-leaf") {
      if (!need(1)) return false;
      a.ppl = (unsigned)std::strtoul(argv[++i], nullptr, 10);
    } else if (k == "--out") {
      if (!need(1)) return false;
      a.out = argv[++i];
    } else if (k == "--frames") {
      if (!need(1)) return false;
      a.frames = std::atoi(argv[++i]);
    } else if (k == "--start-frame") {
      if (!need(1)) return false;
      a.start = std::atoi(argv[++i]);
    } else if (k == "--spp") {
      if (!need(1)) return false;
      a.spp = std::atoi(argv[++i]);
    } else if (k == "--width") {
      if (!need(1)) return false;
      a.width = std::atoi(argv[++i]);
    } else if (k == "--height") {
      if (!need(1)) return false;
      a.height = std::atoi(argv[++i]);
    } else if (k == "--mode") {
      if (!need(1)) return false;
      a.mode = argv[++i];
    } else if (k == "--taa") {
      a.taa = true;
    } else if (k == "--rebuild") {
      a.rebuild = true;
    } else if (k == "-h" || k == "--help") {
      usage();
      exit(0);
    } else {
      fprintf(stderr, "unknown argument %s\n", k.c_str());
      return false;
    }
  }
  return true;
}

bool write_pfm(const std::string& path, const std::vector<float>& rgba, int w, int h) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  fprintf(f, "PF\n%d %d\n-1.0\n", w, h);
  std::vector<float> row(3 * (size_t)w);
  for (int y = h - 1; y >= 0; --y) {  // PFM rows run bottom to top
    for (int x = 0; x < w; ++x)
      for (int c = 0; c < 3; ++c) row[3 * x + c] = rgba[4 * ((size_t)y * w + x) + c];
    fwrite(row.data(), sizeof(float), row.size(), f);
  }
  return fclose(f) == 0;
}

#define CHECK(ctx, call)                                                                           \
  do {                                                                                             \
    aarbf_status _s = (call);                                                                      \
    if (_s != AARBF_OK) {                                                                          \
      fprintf(stderr, "%s failed: %s %s\n", #call, aarbf_status_string(_s), aarbf_last_error(ctx)); \
      return 1;                                                                                    \
    }                                                                                              \
  } while (0)

}  // namespace

int main(int argc, char** argv) {
  Args a;
  if (!parse(argc, argv, a)) {
    usage();
    return 1;
  }
  // particles: importParticles or the reference's synthetic series
  std::vector<std::vector<float>> frames;
  bool synthetic = a.particles.empty();
  if (!synthetic) {
    aarbf_series* s = nullptr;
    if (aarbf_series_load(a.particles.c_str(), &s) != AARBF_OK) {
      fprintf(stderr, "cannot load %s\n", a.particles.c_str());
      return 1;
    }
    uint64_t nf = 0;
    aarbf_series_num_frames(s, &nf);
    for (uint64_t k = 0; k < nf; ++k) {
      const float* p;
      uint64_t n;
      aarbf_series_frame(s, k, &p, &n);
      frames.emplace_back(p, p + 4 * n);
    }
    aarbf_series_free(s);
  } else {
    frames.resize(500);
    for (uint32_t f = 0; f < frames.size(); ++f) {
      frames[f].resize(4 * 1000);
      for (int z = 0; z < 10; ++z)
        for (int y = 0; y < 10; ++y)
          for (int x = 0; x < 10; ++x) {
            uint32_t i = x + y * 10 + z * 100;
            float t1 = float(y) / float(10.f);
            float t2 = float(f) / float(frames.size());
            float s = (float)(std::sin(t2 * 2.f * 3.14) + 1.5f);
            frames[f][4 * i + 0] = s * ((x - 5.f) / 10.f);
            frames[f][4 * i + 1] = s * ((y - 5.f) / 10.f);
            frames[f][4 * i + 2] = s * ((z - 5.f) / 10.f);
            frames[f][4 * i + 3] = t1;
          }
    }
  }
  if (frames.empty()) {
    fprintf(stderr, "no frames\n");
    return 1;
  }
  aarbf_ctx* ctx = nullptr;
  if (aarbf_create(&ctx, 0) != AARBF_OK) {
    fprintf(stderr, "no CUDA device\n");
    return 1;
  }
  // space-time domain over every frame (hostCode.cpp:183-193, :227-240)
  float dom[8];
  aarbf_domain_init(dom);
  for (auto& f : frames) CHECK(ctx, aarbf_domain_accumulate(ctx, f.data(), f.size() / 4, dom, nullptr));
  CHECK(ctx, aarbf_set_domain(ctx, dom));
  float diag = std::sqrt((dom[3] - dom[0]) * (dom[3] - dom[0]) + (dom[4] - dom[1]) * (dom[4] - dom[1]) +
                         (dom[5] - dom[2]) * (dom[5] - dom[2]));
  float radius = (synthetic ? 0.05f : 0.01f) * diag;  // hostCode.cpp:474
  if (a.radius > 0.0f) radius = a.radius;             // applied directly (the reference needs a UI edit)
  float from[3], at[3], up[3], cosfovy;
  if (a.camera.size() == 10) {
    for (int k = 0; k < 3; ++k) {
      from[k] = a.camera[k];
      at[k] = a.camera[3 + k];
      up[k] = a.camera[6 + k];
    }
    cosfovy = a.camera[9];
  } else {  // hostCode.cpp:261-271
    up[0] = 0.f, up[1] = -1.f, up[2] = 0.f;
    for (int k = 0; k < 3; ++k) {
      at[k] = (dom[3 + k] + dom[k]) * .5f;
      from[k] = dom[3 + k];
    }
    if (synthetic) {
      at[0] = at[1] = at[2] = 0.f;
      from[0] = -3.f, from[1] = 3.f, from[2] = 3.f;
    }
    cosfovy = 0.66f;
  }
  aarbf_params p;
  memset(&p, 0, sizeof(p));
  CHECK(ctx, aarbf_camera(from, at, up, cosfovy, a.width, a.height, p.cam_pos, p.cam_dir00, p.cam_du, p.cam_dv));
  p.rbf_radius = radius;
  p.unit = std::fmax(radius * 0.1f, 0.0001f);  // hostCode.cpp:482, :740
  p.flags = AARBF_FLAG_VISUALIZE_ATTRIBUTES | (a.mode == "march" ? AARBF_FLAG_BLUE_NOISE : 0u);
  p.light_ambient = 0.5f;
  p.spp = (uint32_t)(a.spp > 0 ? a.spp : 1);
  for (int k = 0; k < 3; ++k) {
    p.aabb_min[k] = dom[k];
    p.aabb_max[k] = dom[3 + k];
  }
  float *accum = nullptr, *image = nullptr, *taa = nullptr, *taa_prev = nullptr;
  size_t fb = sizeof(float) * 4 * (size_t)a.width * a.height;
  CHECK(ctx, aarbf_get_framebuffers(ctx, a.width, a.height, &accum, &image));
  if (a.taa) {
    CHECK(ctx, aarbf_device_alloc(ctx, fb, (void**)&taa));
    CHECK(ctx, aarbf_device_alloc(ctx, fb, (void**)&taa_prev));
    CHECK(ctx, aarbf_memset(ctx, taa_prev, 0, fb, nullptr));
  }
  std::vector<float> host(4 * (size_t)a.width * a.height);
  uint32_t frame_id = 0;
  size_t built_count = 0;
  for (int k = 0; k < a.frames; ++k) {
    auto& f = frames[(size_t)(a.start + k) % frames.size()];
    CHECK(ctx, aarbf_set_particles(ctx, f.data(), f.size() / 4, nullptr, nullptr));
    if (k == 0 || a.rebuild || f.size() / 4 != built_count) {
      CHECK(ctx, aarbf_build(ctx, radius, a.ppl, nullptr));
      built_count = f.size() / 4;
    } else {
      CHECK(ctx, aarbf_refit_frame(ctx, 0, nullptr));
    }
    p.accum_id = 1;
    p.frame_id = frame_id;
    if (a.mode == "splat") CHECK(ctx, aarbf_render_splat(ctx, &p, a.width, a.height, image, nullptr));
    else CHECK(ctx, aarbf_render(ctx, &p, a.width, a.height, accum, image, nullptr));
    frame_id += p.spp;
    const float* src = image;
    if (a.taa) {
      CHECK(ctx, aarbf_taa_resolve(ctx, image, taa_prev, taa, nullptr, a.width, a.height, 0, nullptr));
      std::swap(taa, taa_prev);
      src = taa_prev;
    }
    CHECK(ctx, aarbf_memcpy(ctx, host.data(), src, fb, nullptr));
    CHECK(ctx, aarbf_sync(ctx, nullptr));
    char name[512];
    snprintf(name, sizeof(name), "%s_%04d.pfm", a.out.c_str(), a.start + k);
    if (!write_pfm(name, host, a.width, a.height)) {
      fprintf(stderr, "cannot write %s\n", name);
      return 1;
    }
    printf("wrote %s\n", name);
  }
  aarbf_device_free(ctx, taa);
  aarbf_device_free(ctx, taa_prev);
  aarbf_destroy(ctx);
  return 0;
}
