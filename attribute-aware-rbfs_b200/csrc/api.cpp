// api.cpp -- the C ABI of include/aarbf.h: context, uploads, the build pipeline that replaces
// GenRBFBounds + the driver's acceleration-structure build (hostCode.cpp:755-799), and the
// launches that replace gprtRayGenLaunch2D / gprtComputeLaunch2D (hostCode.cpp:813, :822).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "aarbf_internal.h"

using namespace aarbf;

namespace {

aarbf_status fail(aarbf_ctx* ctx, aarbf_status s, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return s;
}

aarbf_status cuda_fail(aarbf_ctx* ctx, cudaError_t e, const char* where) {
  std::string m = std::string(where) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return fail(ctx, AARBF_ERR_OUT_OF_MEMORY, m);
  return fail(ctx, AARBF_ERR_CUDA, m);
}

#define CK(call, where)                                  \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, where); \
  } while (0)

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

cudaError_t upload(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (!bytes) return cudaSuccess;
  return cudaMemcpyAsync(dst, src, bytes, is_device_ptr(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                         st);
}

float srgb_decode8(uint8_t v) {
  double c = (double)v / 255.0;
  double l = (c <= 0.04045) ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4);
  return (float)l;
}

uint8_t make_8bit(float f) {
  int v = (int)(f * 256.0f);
  if (v < 0) v = 0;
  if (v > 255) v = 255;
  return (uint8_t)v;
}

// default transfer functions of hostCode.cpp:416-436 as 64-texel RGBA8 textures
void default_tf_rgba8(std::vector<uint8_t>& cm, std::vector<uint8_t>& rm, std::vector<uint8_t>& dm) {
  const float cpos[5] = {0.0f, 0.25f, 0.5f, 0.75f, 1.0f};
  const float ccol[20] = {0.f, 0.f, 1.f, 1.f, 0.f, 0.972549f, 1.f, 1.f, 0.f, 1.f, 0.00784314f, 1.f,
                          0.996078f, 1.f, 0.f, 1.f, 1.f, 0.f, 0.f, 1.f};
  const float gpos[2] = {0.0f, 1.0f};
  const float rcol[8] = {1.f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f};
  const float dcol[8] = {0.f, 0.f, 0.f, 0.f, 1.f, 1.f, 1.f, 1.f};
  cm.assign(64 * 4, 0);
  rm.assign(64 * 4, 0);
  dm.assign(64 * 4, 0);
  aarbf_marks_to_rgba8(cpos, ccol, 5, 1, cm.data(), 64);
  aarbf_marks_to_rgba8(gpos, rcol, 2, 0, rm.data(), 64);
  aarbf_marks_to_rgba8(gpos, dcol, 2, 0, dm.data(), 64);
}

aarbf_status install_tf_f32(aarbf_ctx* ctx, const float* color, int nc, const float* radius, int nr,
                            const float* density, int nd, cudaStream_t st) {
  CK(ctx->tf_color.reserve(sizeof(float) * 4 * nc), "tf alloc");
  CK(ctx->tf_radius.reserve(sizeof(float) * nr), "tf alloc");
  CK(ctx->tf_density.reserve(sizeof(float) * nd), "tf alloc");
  CK(upload(ctx->tf_color.ptr, color, sizeof(float) * 4 * nc, st), "tf upload");
  CK(upload(ctx->tf_radius.ptr, radius, sizeof(float) * nr, st), "tf upload");
  CK(upload(ctx->tf_density.ptr, density, sizeof(float) * nd, st), "tf upload");
  CK(cudaStreamSynchronize(st), "tf upload");
  ctx->nc = nc;
  ctx->nr = nr;
  ctx->nd = nd;
  ctx->has_tf = true;
  std::vector<float> rh(nr);
  CK(cudaMemcpy(rh.data(), ctx->tf_radius.ptr, sizeof(float) * nr, cudaMemcpyDeviceToHost), "tf read");
  ctx->radius_map_unit = true;
  for (float v : rh) ctx->radius_map_unit = ctx->radius_map_unit && v == 1.0f;
  return AARBF_OK;
}

aarbf_status install_tf_rgba8(aarbf_ctx* ctx, const uint8_t* cm, int nc, const uint8_t* rm, int nr, const uint8_t* dm,
                              int nd, cudaStream_t st) {
  std::vector<float> c(4 * (size_t)nc), r(nr), d(nd);
  for (int i = 0; i < nc; ++i) {
    for (int k = 0; k < 3; ++k) c[4 * i + k] = srgb_decode8(cm[4 * i + k]);
    c[4 * i + 3] = (float)((double)cm[4 * i + 3] / 255.0);  // alpha of an sRGB format is linear
  }
  for (int i = 0; i < nr; ++i) r[i] = srgb_decode8(rm[4 * i]);
  for (int i = 0; i < nd; ++i) d[i] = srgb_decode8(dm[4 * i]);
  return install_tf_f32(ctx, c.data(), nc, r.data(), nr, d.data(), nd, st);
}

aarbf_status ensure_tf(aarbf_ctx* ctx, cudaStream_t st) {
  if (ctx->has_tf) return AARBF_OK;
  std::vector<uint8_t> cm, rm, dm;
  default_tf_rgba8(cm, rm, dm);
  return install_tf_rgba8(ctx, cm.data(), 64, rm.data(), 64, dm.data(), 64, st);
}

// prepass + leaf bounds + refit, then read back the root box and the largest radius
aarbf_status run_refit(aarbf_ctx* ctx, cudaStream_t st) {
  const uint64_t n = ctx->n;
  aarbf_status s = ensure_tf(ctx, st);
  if (s != AARBF_OK) return s;
  CK(launch_prepass(ctx->xyzw.as<float4>(), ctx->has_radii ? ctx->radii.as<float>() : nullptr, n,
                    ctx->tf_color.as<float4>(), ctx->nc, ctx->tf_radius.as<float>(), ctx->nr, ctx->rbf_radius,
                    ctx->alpha_floor, ctx->rec0.as<float4>(), ctx->w4.as<float4>(), ctx->rgeom.as<float>(), st),
     "prepass");
  if (ctx->built_fp16)
    CK(launch_quantize_weights(ctx->w4.as<float4>(), ctx->rec0.as<float4>(), n, ctx->posq.as<uint2>(),
                               ctx->colq.as<uint2>(), ctx->reval.as<float>(), st),
       "fp16 weights");
  CK(launch_refit(ctx->rec0.as<float4>(), ctx->rgeom.as<float>(), n, ctx->ppl, ctx->nleaves, ctx->nodes.as<Node>(),
                  ctx->nodes_ref.as<Node>(), ctx->leaf_parent.as<uint32_t>(), ctx->counters.as<uint32_t>(),
                  ctx->leaf_box.as<float>(), ctx->leaf_eff.as<float>(), ctx->root_box.as<float>(),
                  ctx->status.as<uint32_t>(), st),
     "refit");
  if (ctx->nleaves > 1) {
    const size_t wb = sizeof(WideNode) * (size_t)(ctx->nleaves - 1);
    CK(ctx->wide.reserve(wb), "alloc");
    CK(ctx->wide_ref.reserve(wb), "alloc");
    CK(launch_collapse(ctx->nodes.as<Node>(), ctx->nleaves, ctx->wide.as<WideNode>(), st), "collapse");
    CK(launch_collapse(ctx->nodes_ref.as<Node>(), ctx->nleaves, ctx->wide_ref.as<WideNode>(), st), "collapse");
  }
  // root box (6 floats) and the largest bounds radius (slot 6), read back in one copy
  float* rb = ctx->root_box.as<float>();
  CK(launch_max_radius(ctx->rgeom.as<float>(), n, rb + 6, st), "max radius");
  float host[7] = {0, 0, 0, 0, 0, 0, 0};
  CK(cudaMemcpyAsync(host, rb, sizeof(host), cudaMemcpyDeviceToHost, st), "root box");
  CK(cudaStreamSynchronize(st), "refit sync");
  if (ctx->nleaves) memcpy(ctx->root_box_host, host, 6 * sizeof(float));
  ctx->max_radius = host[6];
  ctx->built = true;
  return AARBF_OK;
}

float scene_eps(const aarbf_ctx* ctx, const float* cam) {
  float m = 1e-20f;
  for (int a = 0; a < 6; ++a)
    if (std::isfinite(ctx->root_box_host[a])) m = std::fmax(m, std::fabs(ctx->root_box_host[a]));
  if (cam)
    for (int a = 0; a < 3; ++a) m = std::fmax(m, std::fabs(cam[a]));
  return m * 0x1p-18f;
}

void light_dir(float az, float el, float* dir) {
  // getLightDirection, sharedCode.h:127-132
  float a = el * 3.14f - 0.5f * 3.14f;
  float b = (az * 2.0f) * 3.14f;
  float s = std::sin(a);
  dir[0] = s * std::cos(b);
  dir[1] = s * std::sin(b);
  dir[2] = std::cos(a);
}

void fill_scene_view(const aarbf_ctx* ctx, const float* cam_pos, SceneView& s) {
  memset(&s, 0, sizeof(s));
  s.rec0 = ctx->rec0.as<float4>();
  s.w4 = ctx->w4.as<float4>();
  s.xyzw = ctx->xyzw.as<float4>();
  s.rgeom = ctx->rgeom.as<float>();
  s.nodes = ctx->nodes.as<Node>();
  s.nodes_ref = ctx->nodes_ref.as<Node>();
  s.wide = ctx->wide.as<WideNode>();
  s.wide_ref = ctx->wide_ref.as<WideNode>();
  s.tf_color = ctx->tf_color.as<float4>();
  s.tf_density = ctx->tf_density.as<float>();
  s.n = ctx->n;
  s.ppl = ctx->ppl;
  s.nleaves = ctx->nleaves;
  s.root = ctx->nleaves == 1 ? (0u | kLeafBit) : 0u;
  s.nc = ctx->nc;
  s.nd = ctx->nd;
  for (int a = 0; a < 3; ++a) {
    s.root_lo[a] = ctx->root_box_host[a];
    s.root_hi[a] = ctx->root_box_host[3 + a];
  }
  s.eps = scene_eps(ctx, cam_pos);
  s.per_particle_radius = ctx->has_radii;
  if (ctx->built_fp16) {
    s.posq = ctx->posq.as<uint2>();
    s.colq = ctx->colq.as<uint2>();
    s.origin = ctx->origin.as<float4>();
    s.reval = ctx->reval.as<float>();
  }
}

// context_planes: the per-sample colour planes and the noise plane are the context's (false: the
// caller supplies them, as a batch does from its own memory)
aarbf_status fill_launch(aarbf_ctx* ctx, const aarbf_params* p, int w, int h, float* accum, float* image,
                         RenderLaunch& L, bool context_planes = true) {
  if (!ctx->built) return fail(ctx, AARBF_ERR_NOT_READY, "render before aarbf_build");
  if (!p || w <= 0 || h <= 0) return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "bad render arguments");
  memset(&L, 0, sizeof(L));
  fill_scene_view(ctx, p->cam_pos, L.s);
  L.accum_id = p->accum_id;
  L.frame_id = p->frame_id;
  L.spp = p->spp ? p->spp : 1;
  L.flags = p->flags;
  L.ambient = p->light_ambient;
  light_dir(p->light_azimuth, p->light_elevation, L.light);
  for (int a = 0; a < 3; ++a) {
    L.cam_pos[a] = p->cam_pos[a];
    L.cam_d00[a] = p->cam_dir00[a];
    L.cam_du[a] = p->cam_du[a];
    L.cam_dv[a] = p->cam_dv[a];
    L.aabb_min[a] = p->aabb_min[a];
    L.aabb_max[a] = p->aabb_max[a];
  }
  L.rbf_radius = p->rbf_radius;
  L.unit = p->unit;
  L.density_gain = p->density_gain;
  L.jitter_x = p->jitter_x;
  L.jitter_y = p->jitter_y;
  L.noise = ctx->noise.as<uchar4>();
  L.noise_w = ctx->noise_w;
  L.noise_h = ctx->noise_h;
  L.width = w;
  L.height = h;
  L.accum = reinterpret_cast<float4*>(accum);
  L.image = reinterpret_cast<float4*>(image);
  L.status = ctx->status.as<uint32_t>();
  L.s.loop_cap = p->loop_cap;
  L.traversal = p->traversal;
  L.splat_rmax = (p->flags & kFlagSplatParticleRadius) ? ctx->max_radius : p->rbf_radius;
  L.density_scale = p->density_scale;
  L.bin_length = p->bin_length;
  L.stage_bins = p->stage_bins;
  if (L.stage_bins < 0 || L.stage_bins > 64)
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "stage_bins must lie in 1..64 (0 = default)");
  L.candidate_cap = p->candidate_cap;
  {
    const bool warp = render_uses_warp_kernel(L);
    const int c = p->candidate_cap;
    if (L.stage_bins == 0) L.stage_bins = warp ? 4 : 16;
    if (c == 0) {
      L.candidate_cap = warp ? 256 : 32;
    } else if (warp ? (c != 256 && c != 512 && c != 1024) : (c != 16 && c != 32 && c != 64 && c != 128)) {
      return fail(ctx, AARBF_ERR_INVALID_ARGUMENT,
                  warp ? "candidate_cap must be 256, 512 or 1024 for the warp kernel"
                       : "candidate_cap must be 16, 32, 64 or 128");
    }
  }
  if (!(p->unit > 0.0f)) return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "unit must be > 0");
  {
    // the persistent kernels count work items (one sample of one pixel, pixels padded to 8 x 4
    // tiles) in 32 bits, and every resident warp or thread takes one item past the end
    const uint64_t items = (uint64_t)((w + 7) / 8) * (uint64_t)((h + 3) / 4) * 32u * L.spp;
    if (items > 0xfff00000ull)
      return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "width x height x spp exceeds the 32-bit work-item count");
  }
  if ((p->flags & kFlagMajorantTracking) && !(p->bin_length > 0.0f && p->density_scale >= 0.0f))
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "majorant tracking needs bin_length > 0, density_scale >= 0");
  if (!ctx->work.ptr) CK(ctx->work.reserve(256), "work counter");
  L.work_counter = ctx->work.as<uint32_t>();
  if (context_planes) {
    CK(ctx->samples.reserve(sizeof(float) * 4 * (size_t)w * (size_t)h * L.spp), "sample planes");
    CK(ctx->noise_buf.reserve(sizeof(float) * (size_t)w * (size_t)h), "noise plane");
    L.samples = ctx->samples.as<float4>();
    L.noise_buf = ctx->noise_buf.as<float>();
  }
  if (render_uses_warp_kernel(L)) {
    size_t words = 0;
    CK(render_warp_stack_words(&words), "warp kernel setup");
    CK(ctx->warp_stacks.reserve(4 * words), "warp stacks");
    L.warp_stacks = ctx->warp_stacks.as<uint32_t>();
  }
  return AARBF_OK;
}

aarbf_status ensure_fb(aarbf_ctx* ctx, int w, int h) {
  size_t bytes = sizeof(float) * 4 * (size_t)w * (size_t)h;
  if (ctx->fb_w != w || ctx->fb_h != h || !ctx->fb_accum.ptr) {
    CK(ctx->fb_accum.reserve(bytes), "framebuffer alloc");
    CK(ctx->fb_image.reserve(bytes), "framebuffer alloc");
    CK(cudaMemset(ctx->fb_accum.ptr, 0, bytes), "framebuffer clear");
    CK(cudaMemset(ctx->fb_image.ptr, 0, bytes), "framebuffer clear");
    ctx->fb_w = w;
    ctx->fb_h = h;
  }
  return AARBF_OK;
}

// the frame's Hilbert keys and sort permutation (ctx->sorted_keys, ctx->perm), as the reference
// sorts each frame along the curve of the space-time box (hostCode.cpp:195-222)
aarbf_status sort_frame(aarbf_ctx* ctx, const float* dom, cudaStream_t st) {
  const uint64_t n = ctx->n;
  const float4* in = ctx->in_xyzw.as<float4>();
  uint64_t* keys = ctx->keys.as<uint64_t>();
  uint32_t* perm = ctx->perm.as<uint32_t>();
  const size_t hw = ctx->hist.bytes / 4;
  bool alt = false;
  {
    CK(launch_hilbert_keys(in, n, dom, keys, perm, st), "hilbert keys");
    CK(radix_sort_pairs(keys, perm, ctx->keys_alt.as<uint64_t>(), ctx->perm_alt.as<uint32_t>(), n, 48,
                        ctx->hist.as<uint32_t>(), hw, st, &alt),
       "radix sort");
    if (alt) {
      keys = ctx->keys_alt.as<uint64_t>();
      perm = ctx->perm_alt.as<uint32_t>();
    }
    // equal keys: short runs are ordered in place; a run longer than the in-place limit redoes
    // the sort as an LSD chain over (w, z, y, x) then the key, each pass stable
    CK(cudaMemsetAsync(ctx->flag.ptr, 0, 4, st), "flag");
    CK(launch_tie_runs(keys, in, perm, n, ctx->flag.as<uint32_t>(), st), "tie runs");
    uint32_t tie = 0;
    CK(cudaMemcpyAsync(&tie, ctx->flag.ptr, 4, cudaMemcpyDeviceToHost, st), "tie read");
    CK(cudaStreamSynchronize(st), "tie sync");
    if (tie & 2u) {
      uint64_t* k0 = ctx->keys.as<uint64_t>();
      uint64_t* k1 = ctx->keys_alt.as<uint64_t>();
      uint32_t* p0 = ctx->perm.as<uint32_t>();
      uint32_t* p1 = ctx->perm_alt.as<uint32_t>();
      // identity permutation via a key pass with ident output
      CK(launch_hilbert_keys(in, n, dom, k0, p0, st), "ident");
      for (int comp = 3; comp >= -1; --comp) {
        if (comp >= 0) CK(launch_orderable_component(in, p0, n, comp, k0, st), "tie keys");
        else CK(launch_hilbert_keys_perm(in, p0, n, dom, k0, st), "tie keys");
        bool a2 = false;
        CK(radix_sort_pairs(k0, p0, k1, p1, n, comp >= 0 ? 32 : 48, ctx->hist.as<uint32_t>(), hw, st, &a2),
           "tie sort");
        if (a2) {
          uint64_t* tk = k0; k0 = k1; k1 = tk;
          uint32_t* tp = p0; p0 = p1; p1 = tp;
        }
      }
      keys = k0;
      perm = p0;
    }
    CK(cudaMemcpyAsync(ctx->sorted_keys.ptr, keys, 8 * n, cudaMemcpyDeviceToDevice, st), "keys");
    if (perm != ctx->perm.as<uint32_t>())
      CK(cudaMemcpyAsync(ctx->perm.ptr, perm, 4 * n, cudaMemcpyDeviceToDevice, st), "perm");
  }
  return AARBF_OK;
}

// the frame's particles in the order of ctx->perm, attributes normalised over dom; FP16 records
aarbf_status gather_frame(aarbf_ctx* ctx, const float* dom, cudaStream_t st) {
  const uint64_t n = ctx->n, nn = n ? n : 1;
  CK(launch_gather_normalize(ctx->in_xyzw.as<float4>(), ctx->has_radii ? ctx->in_radii.as<float>() : nullptr,
                             ctx->perm.as<uint32_t>(), n, dom[6], dom[7], ctx->xyzw.as<float4>(),
                             ctx->radii.as<float>(), st),
     "gather");
  if (ctx->storage_fp16) {
    CK(ctx->posq.reserve(8 * nn), "alloc");
    CK(ctx->colq.reserve(8 * nn), "alloc");
    CK(ctx->reval.reserve(4 * nn), "alloc");
    CK(ctx->origin.reserve(16 * ((nn + 255) / 256)), "alloc");
    CK(launch_quantize_positions(ctx->xyzw.as<float4>(), n, ctx->posq.as<uint2>(), ctx->origin.as<float4>(), st),
       "fp16 positions");
  }
  return AARBF_OK;
}
}  // namespace

extern "C" {

const char* aarbf_status_string(aarbf_status s) {
  switch (s) {
    case AARBF_OK: return "ok";
    case AARBF_ERR_INVALID_ARGUMENT: return "invalid argument";
    case AARBF_ERR_OUT_OF_MEMORY: return "out of memory";
    case AARBF_ERR_CUDA: return "CUDA error";
    case AARBF_ERR_DEVICE_LIMIT: return "device-side limit exceeded";
    case AARBF_ERR_NOT_READY: return "not ready";
    case AARBF_ERR_IO: return "I/O error";
    case AARBF_ERR_UNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

aarbf_status aarbf_get_version(int* major, int* minor) {
  if (major) *major = AARBF_VERSION_MAJOR;
  if (minor) *minor = AARBF_VERSION_MINOR;
  return AARBF_OK;
}

aarbf_status aarbf_create(aarbf_ctx** out, int device) {
  if (!out) return AARBF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return AARBF_ERR_CUDA;
  }
  if (cudaSetDevice(device) != cudaSuccess) return AARBF_ERR_CUDA;
  aarbf_ctx* ctx = new (std::nothrow) aarbf_ctx();
  if (!ctx) return AARBF_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  if (ctx->status.reserve(64) != cudaSuccess || cudaMemset(ctx->status.ptr, 0, 64) != cudaSuccess) {
    delete ctx;
    return AARBF_ERR_CUDA;
  }
  *out = ctx;
  return AARBF_OK;
}

aarbf_status aarbf_destroy(aarbf_ctx* ctx) {
  if (!ctx) return AARBF_OK;
  cudaSetDevice(ctx->device);
  DevBuf* bufs[] = {&ctx->in_xyzw, &ctx->in_radii, &ctx->keys, &ctx->keys_alt, &ctx->perm, &ctx->perm_alt,
                    &ctx->hist, &ctx->tmp_keys, &ctx->flag, &ctx->xyzw, &ctx->radii, &ctx->rec0, &ctx->w4,
                    &ctx->rgeom, &ctx->nodes, &ctx->nodes_ref, &ctx->leaf_eff, &ctx->leaf_parent, &ctx->counters,
                    &ctx->leaf_box, &ctx->root_box,
                    &ctx->sorted_keys, &ctx->tf_color, &ctx->tf_radius, &ctx->tf_density, &ctx->noise,
                    &ctx->fb_accum, &ctx->fb_image, &ctx->status, &ctx->work, &ctx->samples,
                    &ctx->noise_buf, &ctx->warp_stacks, &ctx->diff_views, &ctx->diff_ckpt, &ctx->diff_grad,
                    &ctx->posq, &ctx->colq, &ctx->origin, &ctx->reval, &ctx->splat_slabs, &ctx->wide,
                    &ctx->wide_ref};
  for (DevBuf* b : bufs) b->release();
  for (auto* v : {&ctx->ev_pending, &ctx->ev_free})
    for (auto& ev : *v)
      for (cudaEvent_t e : ev) cudaEventDestroy(e);
  delete ctx;
  return AARBF_OK;
}

const char* aarbf_last_error(const aarbf_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

aarbf_status aarbf_sync(aarbf_ctx* ctx, void* stream) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaStreamSynchronize(st), "sync");
  uint32_t bits = 0;
  CK(cudaMemcpy(&bits, ctx->status.ptr, sizeof(bits), cudaMemcpyDeviceToHost), "status read");
  if (bits) {
    CK(cudaMemset(ctx->status.ptr, 0, sizeof(bits)), "status clear");
    char msg[160];
    snprintf(msg, sizeof(msg), "device status bits 0x%x (1 = traversal stack overflow, 2 = bad input, 4 = loop cap)",
             bits);
    return fail(ctx, (bits & kStatusBadInput) ? AARBF_ERR_INVALID_ARGUMENT : AARBF_ERR_DEVICE_LIMIT, msg);
  }
  return AARBF_OK;
}

aarbf_status aarbf_set_particles(aarbf_ctx* ctx, const float* xyzw, uint64_t n, const float* radii, void* stream) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (n && !xyzw) return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "null particle pointer");
  if (n >= 0xffffffffull) return fail(ctx, AARBF_ERR_UNSUPPORTED, "more than 2^32-1 particles per frame");
  cudaSetDevice(ctx->device);
  cudaStream_t st = (cudaStream_t)stream;
  CK(ctx->in_xyzw.reserve(16 * (n ? n : 1)), "particle alloc");
  CK(upload(ctx->in_xyzw.ptr, xyzw, 16 * n, st), "particle upload");
  ctx->has_radii = radii != nullptr;
  if (radii) {
    CK(ctx->in_radii.reserve(4 * (n ? n : 1)), "radius alloc");
    CK(upload(ctx->in_radii.ptr, radii, 4 * n, st), "radius upload");
  }
  ctx->n = n;
  ctx->built = false;
  return AARBF_OK;
}

aarbf_status aarbf_domain_init(float* dom) {
  if (!dom) return AARBF_ERR_INVALID_ARGUMENT;
  dom[0] = dom[1] = dom[2] = 1e38f;  // hostCode.cpp:183
  dom[3] = dom[4] = dom[5] = -1e38f;
  dom[6] = 1e20f;  // hostCode.cpp:227-228
  dom[7] = -1e20f;
  return AARBF_OK;
}

aarbf_status aarbf_set_domain(aarbf_ctx* ctx, const float* dom) {
  if (!ctx || !dom) return AARBF_ERR_INVALID_ARGUMENT;
  memcpy(ctx->dom, dom, sizeof(ctx->dom));
  ctx->has_domain = true;
  return AARBF_OK;
}

aarbf_status aarbf_domain_accumulate(aarbf_ctx* ctx, const float* xyzw, uint64_t n, float* dom, void* stream) {
  if (!ctx || !dom) return AARBF_ERR_INVALID_ARGUMENT;
  if (!n) return AARBF_OK;
  if (!xyzw) return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "null particle pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t st = (cudaStream_t)stream;
  const float4* src = reinterpret_cast<const float4*>(xyzw);
  DevBuf tmp;
  if (!is_device_ptr(xyzw)) {
    CK(tmp.reserve(16 * n), "domain alloc");
    CK(cudaMemcpyAsync(tmp.ptr, xyzw, 16 * n, cudaMemcpyHostToDevice, st), "domain upload");
    src = tmp.as<float4>();
  }
  int nb = (int)std::min<uint64_t>((n + 255) / 256, 1184);
  DevBuf part;
  if (part.reserve(sizeof(float) * 9 * nb) != cudaSuccess) {
    tmp.release();
    return fail(ctx, AARBF_ERR_OUT_OF_MEMORY, "domain alloc");
  }
  std::vector<float> h(9 * (size_t)nb);
  cudaError_t e = launch_domain_reduce(src, n, part.as<float>(), nb, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part.ptr, h.size() * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  part.release();
  tmp.release();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "domain reduce");
  bool bad = false;
  for (int b = 0; b < nb; ++b) {
    const float* v = h.data() + 9 * b;
    for (int a = 0; a < 3; ++a) {
      dom[a] = std::fmin(dom[a], v[a]);
      dom[3 + a] = std::fmax(dom[3 + a], v[3 + a]);
    }
    dom[6] = std::fmin(dom[6], v[6]);
    dom[7] = std::fmax(dom[7], v[7]);
    bad = bad || v[8] != 0.0f;
  }
  if (bad) return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "non-finite particle coordinates or attributes");
  return AARBF_OK;
}

aarbf_status aarbf_set_transfer_functions_rgba8(aarbf_ctx* ctx, const uint8_t* cm, int nc, const uint8_t* rm, int nr,
                                                const uint8_t* dm, int nd) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (!cm || !rm || !dm || nc < 1 || nr < 1 || nd < 1 || nc > 65536 || nr > 65536 || nd > 65536)
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "bad transfer-function textures");
  cudaSetDevice(ctx->device);
  aarbf_status s = install_tf_rgba8(ctx, cm, nc, rm, nr, dm, nd, nullptr);
  if (s == AARBF_OK && ctx->built) ctx->built = false, s = AARBF_OK;
  return s;
}

aarbf_status aarbf_set_transfer_functions_f32(aarbf_ctx* ctx, const float* cm, int nc, const float* rm, int nr,
                                              const float* dm, int nd) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (!cm || !rm || !dm || nc < 1 || nr < 1 || nd < 1 || nc > 65536 || nr > 65536 || nd > 65536)
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "bad transfer-function tables");
  cudaSetDevice(ctx->device);
  aarbf_status s = install_tf_f32(ctx, cm, nc, rm, nr, dm, nd, nullptr);
  if (s == AARBF_OK && ctx->built) ctx->built = false;
  return s;
}

aarbf_status aarbf_marks_to_rgba8(const float* pos, const float* rgba, int nmarks, int gamma, uint8_t* out,
                                  int ntexels) {
  if (!pos || !rgba || !out || nmarks < 1 || ntexels < 1) return AARBF_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < ntexels; ++i) {
    float u = (ntexels > 1) ? (float)i / (float)(ntexels - 1) : 0.0f;
    float c[4];
    // piecewise-linear gradient between marks, constant outside (imgui_gradient's gradient.at)
    if (u <= pos[0]) {
      for (int k = 0; k < 4; ++k) c[k] = rgba[k];
    } else if (u >= pos[nmarks - 1]) {
      for (int k = 0; k < 4; ++k) c[k] = rgba[4 * (nmarks - 1) + k];
    } else {
      int j = 0;
      while (j + 1 < nmarks && !(u < pos[j + 1])) ++j;
      float span = pos[j + 1] - pos[j];
      float a = span > 0.0f ? (u - pos[j]) / span : 0.0f;
      for (int k = 0; k < 4; ++k) c[k] = rgba[4 * j + k] + a * (rgba[4 * (j + 1) + k] - rgba[4 * j + k]);
    }
    if (gamma) {
      for (int k = 0; k < 3; ++k) out[4 * i + k] = make_8bit(std::pow(c[k], 1.0f / 2.2f));
      out[4 * i + 3] = make_8bit(c[3]);
    } else {
      out[4 * i + 0] = make_8bit(c[0]);
      out[4 * i + 1] = out[4 * i + 2] = out[4 * i + 3] = 0;
    }
  }
  return AARBF_OK;
}

aarbf_status aarbf_build(aarbf_ctx* ctx, float rbf_radius, uint32_t ppl, void* stream) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (ppl == 0) ppl = 1;  // hostCode.cpp:65, :170-171
  if (!(rbf_radius >= 0.0f) || !std::isfinite(rbf_radius))
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "rbf_radius must be finite and >= 0");
  cudaSetDevice(ctx->device);
  cudaStream_t st = (cudaStream_t)stream;
  const uint64_t n = ctx->n;
  ctx->ppl = ppl;
  ctx->rbf_radius = rbf_radius;
  ctx->nleaves = (uint32_t)((n + ppl - 1) / ppl);
  ctx->has_topology = false;
  // domain: the caller's space-time box, else this frame's own bounds
  float dom[8];
  if (ctx->has_domain) {
    memcpy(dom, ctx->dom, sizeof(dom));
  } else {
    aarbf_domain_init(dom);
    aarbf_status s = aarbf_domain_accumulate(ctx, ctx->in_xyzw.as<float>(), n, dom, stream);
    if (s != AARBF_OK) return s;
  }
  const uint64_t nn = n ? n : 1;
  CK(ctx->keys.reserve(8 * nn), "alloc");
  CK(ctx->keys_alt.reserve(8 * nn), "alloc");
  CK(ctx->perm.reserve(4 * nn), "alloc");
  CK(ctx->perm_alt.reserve(4 * nn), "alloc");
  CK(ctx->hist.reserve(4 * radix_sort_hist_words(nn)), "alloc");
  CK(ctx->flag.reserve(16), "alloc");
  CK(ctx->xyzw.reserve(16 * nn), "alloc");
  CK(ctx->rec0.reserve(16 * nn), "alloc");
  CK(ctx->w4.reserve(16 * nn), "alloc");
  CK(ctx->rgeom.reserve(4 * nn), "alloc");
  if (ctx->has_radii) CK(ctx->radii.reserve(4 * nn), "alloc");
  const uint64_t nl = ctx->nleaves ? ctx->nleaves : 1;
  CK(ctx->nodes.reserve(sizeof(Node) * nl), "alloc");
  CK(ctx->nodes_ref.reserve(sizeof(Node) * nl), "alloc");
  CK(ctx->leaf_eff.reserve(24 * nl), "alloc");
  CK(ctx->leaf_parent.reserve(4 * nl), "alloc");
  CK(ctx->counters.reserve(4 * nl), "alloc");
  CK(ctx->leaf_box.reserve(24 * nl), "alloc");
  CK(ctx->root_box.reserve(64), "alloc");
  CK(ctx->sorted_keys.reserve(8 * nn), "alloc");

  if (n) {
    aarbf_status s = sort_frame(ctx, dom, st);
    if (s != AARBF_OK) return s;
    s = gather_frame(ctx, dom, st);
    if (s != AARBF_OK) return s;
    CK(launch_karras(ctx->sorted_keys.as<uint64_t>(), n, ppl, ctx->nleaves, ctx->nodes.as<Node>(),
                     ctx->nodes_ref.as<Node>(), ctx->leaf_parent.as<uint32_t>(), st),
       "karras");
  }
  memcpy(ctx->dom, dom, sizeof(dom));
  ctx->built_fp16 = ctx->storage_fp16 && n > 0;
  ctx->built_n = n;
  ctx->built_has_radii = ctx->has_radii;
  aarbf_status s = run_refit(ctx, st);
  if (s != AARBF_OK) return s;
  ctx->has_topology = true;
  if (!n)
    for (int a = 0; a < 6; ++a) ctx->root_box_host[a] = NAN;
  return AARBF_OK;
}


aarbf_status aarbf_refit_frame(aarbf_ctx* ctx, int keep_order, void* stream) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  // a new frame clears `built` (the scene is stale until refit); the topology of the last
  // completed aarbf_build is what this call needs
  if (!ctx->has_topology || !ctx->nodes.ptr) return fail(ctx, AARBF_ERR_NOT_READY, "refit_frame before build");
  if (ctx->n != ctx->built_n || ctx->has_radii != ctx->built_has_radii)
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT,
                "refit_frame needs a frame of the built particle count (and radii iff the build had them); "
                "call aarbf_build for a new count");
  if (ctx->storage_fp16 != ctx->built_fp16 && ctx->n)
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "storage form changed since the build: call aarbf_build");
  cudaSetDevice(ctx->device);
  cudaStream_t st = (cudaStream_t)stream;
  if (ctx->n) {
    if (!keep_order) {
      aarbf_status s = sort_frame(ctx, ctx->dom, st);
      if (s != AARBF_OK) return s;
    }
    aarbf_status s = gather_frame(ctx, ctx->dom, st);
    if (s != AARBF_OK) return s;
  }
  return run_refit(ctx, st);
}

aarbf_status aarbf_refit(aarbf_ctx* ctx, float rbf_radius, void* stream) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (!ctx->nodes.ptr) return fail(ctx, AARBF_ERR_NOT_READY, "refit before build");
  if (!(rbf_radius >= 0.0f) || !std::isfinite(rbf_radius))
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "rbf_radius must be finite and >= 0");
  cudaSetDevice(ctx->device);
  ctx->rbf_radius = rbf_radius;
  return run_refit(ctx, (cudaStream_t)stream);
}

aarbf_status aarbf_get_framebuffers(aarbf_ctx* ctx, int w, int h, float** accum, float** image) {
  if (!ctx || w <= 0 || h <= 0) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  aarbf_status s = ensure_fb(ctx, w, h);
  if (s != AARBF_OK) return s;
  if (accum) *accum = ctx->fb_accum.as<float>();
  if (image) *image = ctx->fb_image.as<float>();
  return AARBF_OK;
}

aarbf_status aarbf_render(aarbf_ctx* ctx, const aarbf_params* p, int w, int h, float* accum, float* image,
                          void* stream) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (!accum || !image) {
    aarbf_status s = ensure_fb(ctx, w, h);
    if (s != AARBF_OK) return s;
    if (!accum) accum = ctx->fb_accum.as<float>();
    if (!image) image = ctx->fb_image.as<float>();
  }
  RenderLaunch L;
  aarbf_status s = fill_launch(ctx, p, w, h, accum, image, L);
  if (s != AARBF_OK) return s;
  if ((p->flags & kFlagBlueNoise) && !ctx->noise.ptr) {
    std::vector<uint8_t> atlas(2048ull * 4096ull * 4ull);
    aarbf_generate_noise_atlas(atlas.data(), 2048, 4096);
    s = aarbf_set_noise_atlas(ctx, atlas.data(), 2048, 4096);
    if (s != AARBF_OK) return s;
    L.noise = ctx->noise.as<uchar4>();
    L.noise_w = ctx->noise_w;
    L.noise_h = ctx->noise_h;
  }
  if (!ctx->kernel_timing) {
    CK(launch_render(L, (cudaStream_t)stream), "render launch");
    return AARBF_OK;
  }
  std::array<cudaEvent_t, 3> ev{};
  if (!ctx->ev_free.empty()) {
    ev = ctx->ev_free.back();
    ctx->ev_free.pop_back();
  } else {
    for (auto& e : ev) CK(cudaEventCreate(&e), "timing event");
  }
  ctx->ev_pending.push_back(ev);
  CK(launch_render(L, (cudaStream_t)stream, ev.data()), "render launch");
  return AARBF_OK;
}

aarbf_status aarbf_set_kernel_timing(aarbf_ctx* ctx, int enable) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  ctx->kernel_timing = enable != 0;
  return AARBF_OK;
}

aarbf_status aarbf_get_kernel_times(aarbf_ctx* ctx, double* render_ms, double* accumulate_ms,
                                    uint32_t* renders) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  double r = 0.0, a = 0.0;
  uint32_t k = 0;
  cudaError_t err = cudaSuccess;
  for (auto& ev : ctx->ev_pending) {
    float t01 = 0.0f, t12 = 0.0f;
    if (err == cudaSuccess) err = cudaEventSynchronize(ev[2]);
    if (err == cudaSuccess) err = cudaEventElapsedTime(&t01, ev[0], ev[1]);
    if (err == cudaSuccess) err = cudaEventElapsedTime(&t12, ev[1], ev[2]);
    r += t01;
    a += t12;
    ++k;
    ctx->ev_free.push_back(ev);
  }
  ctx->ev_pending.clear();
  if (err != cudaSuccess) return cuda_fail(ctx, err, "kernel times");
  if (render_ms) *render_ms = r;
  if (accumulate_ms) *accumulate_ms = a;
  if (renders) *renders = k;
  return AARBF_OK;
}

aarbf_status aarbf_render_count(aarbf_ctx* ctx, const aarbf_params* p, int w, int h, float* accum, float* image,
                                uint64_t* counts, void* stream) {
  if (!ctx || !counts) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (!accum || !image) {
    aarbf_status s = ensure_fb(ctx, w, h);
    if (s != AARBF_OK) return s;
    if (!accum) accum = ctx->fb_accum.as<float>();
    if (!image) image = ctx->fb_image.as<float>();
  }
  RenderLaunch L;
  aarbf_status s = fill_launch(ctx, p, w, h, accum, image, L);
  if (s != AARBF_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  DevBuf c;
  unsigned long long h2[AARBF_COUNT_SLOTS] = {};
  CK(c.reserve(sizeof(h2)), "count alloc");
  cudaError_t e = cudaMemsetAsync(c.ptr, 0, sizeof(h2), st);
  L.counters = c.as<unsigned long long>();
  if (e == cudaSuccess) e = launch_render(L, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h2, c.ptr, sizeof(h2), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  c.release();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "render count");
  for (int k = 0; k < AARBF_COUNT_SLOTS; ++k) counts[k] = h2[k];
  return AARBF_OK;
}

// ---- batched rendering ---------------------------------------------------------------------

struct aarbf_batch {
  int device = 0;
  int nscenes = 0;
  uint64_t total_pixels = 0;
  DevBuf dev;           // launch blocks, item and pixel prefix sums, work counter
  DevBuf planes;        // every scene's per-sample colour planes, then every scene's noise plane
  uint32_t* warp_stacks = nullptr;
  bool fp16 = false;
  int blocks_per_sm = 0;  // launch shape (aarbf_batch_set_shape)
  int sample_major = 0;
  std::vector<RenderLaunch> launches;  // host copies: the batched kernel takes them as parameters
  std::vector<uint64_t> items;         // nscenes + 1 prefix sums of work items
  std::string last_error;
};

// the batch's device block: launch blocks (read by the accumulation pass), pixel prefix sums,
// 64 per-scene item counters
struct BatchLayout {
  size_t launch_bytes, pix_bytes, off_pix, off_ctr, bytes;
  explicit BatchLayout(int nscenes)
      : launch_bytes(sizeof(RenderLaunch) * (size_t)nscenes), pix_bytes(sizeof(uint64_t) * ((size_t)nscenes + 1)) {
    off_pix = (launch_bytes + 255) / 256 * 256;
    off_ctr = off_pix + (pix_bytes + 255) / 256 * 256;
    bytes = off_ctr + 64 * sizeof(uint32_t);
  }
};

aarbf_status aarbf_batch_set_shape(aarbf_batch* b, int blocks_per_sm, int sample_major) {
  if (!b) return AARBF_ERR_INVALID_ARGUMENT;
  if (blocks_per_sm < 0 || blocks_per_sm > 64 || (sample_major != 0 && sample_major != 1)) {
    b->last_error = "blocks_per_sm must lie in 0..64 and sample_major be 0 or 1";
    return AARBF_ERR_INVALID_ARGUMENT;
  }
  b->blocks_per_sm = blocks_per_sm;
  b->sample_major = sample_major;
  return AARBF_OK;
}

aarbf_status aarbf_batch_create(aarbf_batch** out, aarbf_ctx* const* ctxs, const aarbf_params* params, int nscenes,
                                const int* widths, const int* heights, float* const* accums, float* const* images) {
  if (!out || !ctxs || !params || nscenes <= 0 || !widths || !heights || !accums || !images)
    return AARBF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  aarbf_ctx* c0 = ctxs[0];
  if (!c0) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c0->device);
  std::vector<RenderLaunch> Ls((size_t)nscenes);
  std::vector<uint64_t> items((size_t)nscenes + 1, 0), pix((size_t)nscenes + 1, 0);
  for (int i = 0; i < nscenes; ++i) {
    aarbf_ctx* ctx = ctxs[i];
    if (!ctx || ctx->device != c0->device)
      return fail(c0, AARBF_ERR_INVALID_ARGUMENT, "batched scenes need contexts on one device");
    if (ctx->built_fp16 != c0->built_fp16)
      return fail(c0, AARBF_ERR_UNSUPPORTED, "batched scenes need one storage form");
    if (!accums[i] || !images[i]) return fail(c0, AARBF_ERR_INVALID_ARGUMENT, "batched scenes need framebuffers");
    const aarbf_params& p = params[i];
    if (!(p.flags & kFlagMajorantTracking) || (p.flags & kFlagBlueNoise) || p.traversal != AARBF_TRAVERSAL_AUTO)
      return fail(c0, AARBF_ERR_UNSUPPORTED, "batched rendering runs majorant tracking with AARBF_TRAVERSAL_AUTO");
    aarbf_params q = p;
    q.candidate_cap = 0;
    aarbf_status s = fill_launch(ctx, &q, widths[i], heights[i], accums[i], images[i], Ls[(size_t)i], false);
    if (s != AARBF_OK) {
      c0->last_error = ctx->last_error;
      return s;
    }
    const uint64_t tiles = (uint64_t)((widths[i] + 7) / 8) * (uint64_t)((heights[i] + 3) / 4);
    items[(size_t)i + 1] = items[(size_t)i] + tiles * 32u * Ls[(size_t)i].spp;
    pix[(size_t)i + 1] = pix[(size_t)i] + (uint64_t)widths[i] * (uint64_t)heights[i];
  }
  size_t words = 0;
  cudaError_t e0 = render_warp_stack_words(&words);
  if (e0 == cudaSuccess) e0 = c0->warp_stacks.reserve(4 * words);
  if (e0 != cudaSuccess) return cuda_fail(c0, e0, "warp stacks");
  aarbf_batch* b = new aarbf_batch();
  b->device = c0->device;
  b->nscenes = nscenes;
  b->total_pixels = pix.back();
  b->warp_stacks = c0->warp_stacks.as<uint32_t>();
  b->fp16 = c0->built_fp16;
  // the batch's own sample and noise planes: a context may appear more than once, and a single
  // render through a context (which may reallocate the context's planes) leaves the batch intact
  size_t sample_bytes = 0;
  for (int i = 0; i < nscenes; ++i) sample_bytes += sizeof(float4) * (size_t)widths[i] * (size_t)heights[i] * Ls[(size_t)i].spp;
  cudaError_t e = b->planes.reserve(sample_bytes + sizeof(float) * (size_t)b->total_pixels);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(c0, e, "batch sample planes");
  }
  {
    float4* sp = b->planes.as<float4>();
    float* np = reinterpret_cast<float*>(static_cast<char*>(b->planes.ptr) + sample_bytes);
    for (int i = 0; i < nscenes; ++i) {
      RenderLaunch& L = Ls[(size_t)i];
      L.samples = sp;
      L.noise_buf = np;
      sp += (size_t)widths[i] * (size_t)heights[i] * L.spp;
      np += (size_t)widths[i] * (size_t)heights[i];
    }
  }
  const BatchLayout lay(nscenes);
  e = b->dev.reserve(lay.bytes);
  if (e == cudaSuccess) e = cudaMemcpy(b->dev.ptr, Ls.data(), lay.launch_bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(static_cast<char*>(b->dev.ptr) + lay.off_pix, pix.data(), lay.pix_bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    b->dev.release();
    b->planes.release();
    delete b;
    return cuda_fail(c0, e, "batch upload");
  }
  b->launches = std::move(Ls);
  b->items = std::move(items);
  *out = b;
  return AARBF_OK;
}

aarbf_status aarbf_batch_render(aarbf_batch* b, int candidate_cap, void* stream) {
  if (!b) return AARBF_ERR_INVALID_ARGUMENT;
  if (candidate_cap != 0 && candidate_cap != 256 && candidate_cap != 512 && candidate_cap != 1024) {
    b->last_error = "candidate_cap must be 0, 256, 512 or 1024";
    return AARBF_ERR_INVALID_ARGUMENT;
  }
  cudaSetDevice(b->device);
  const BatchLayout lay(b->nscenes);
  char* base = static_cast<char*>(b->dev.ptr);
  BatchArgs B;
  B.launches = reinterpret_cast<const RenderLaunch*>(base);
  B.host_launches = b->launches.data();
  B.host_items = b->items.data();
  B.pix_ofs = reinterpret_cast<const uint64_t*>(base + lay.off_pix);
  B.nscenes = b->nscenes;
  B.total_pixels = b->total_pixels;
  B.candidate_cap = candidate_cap;
  B.work_counters = reinterpret_cast<uint32_t*>(base + lay.off_ctr);
  B.warp_stacks = b->warp_stacks;
  B.fp16 = b->fp16;
  B.blocks_per_sm = b->blocks_per_sm;
  B.sample_major = b->sample_major;
  cudaError_t e = launch_render_batched(B, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    b->last_error = std::string("batch render: ") + cudaGetErrorString(e);
    return AARBF_ERR_CUDA;
  }
  return AARBF_OK;
}

aarbf_status aarbf_batch_destroy(aarbf_batch* b) {
  if (!b) return AARBF_OK;
  cudaSetDevice(b->device);
  b->dev.release();
  b->planes.release();
  delete b;
  return AARBF_OK;
}

const char* aarbf_batch_last_error(const aarbf_batch* b) { return b ? b->last_error.c_str() : ""; }

// ---- differentiable form ------------------------------------------------------------------

static aarbf_status diff_setup(aarbf_ctx* ctx, const aarbf_params* views, int nviews, int w, int h, DiffArgs& A,
                               cudaStream_t st) {
  if (!ctx->built) return fail(ctx, AARBF_ERR_NOT_READY, "differentiable render before aarbf_build");
  if (!views || nviews <= 0 || w <= 0 || h <= 0) return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "bad views or size");
  if (!ctx->radius_map_unit)
    return fail(ctx, AARBF_ERR_UNSUPPORTED, "differentiable render needs a radius map of ones");
  if (ctx->nc > 2048) return fail(ctx, AARBF_ERR_UNSUPPORTED, "differentiable render needs <= 2048 colour texels");
  if (!(ctx->dom[7] > ctx->dom[6])) return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "empty attribute range");
  const uint32_t spp0 = views[0].spp ? views[0].spp : 1u;
  std::vector<float> hv(22 * (size_t)nviews);
  for (int v = 0; v < nviews; ++v) {
    const aarbf_params* p = views + v;
    if (!(p->unit > 0.0f)) return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "unit must be > 0");
    const uint32_t fid = p->frame_id, spp = p->spp ? p->spp : 1u;
    if (spp != spp0) return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "all views need the same spp");
    float* o = hv.data() + 22 * (size_t)v;
    for (int a = 0; a < 3; ++a) {
      o[a] = p->cam_pos[a];
      o[3 + a] = p->cam_dir00[a];
      o[6 + a] = p->cam_du[a];
      o[9 + a] = p->cam_dv[a];
      o[12 + a] = p->aabb_min[a] - 2.0f * p->rbf_radius;
      o[15 + a] = p->aabb_max[a] + 2.0f * p->rbf_radius;
    }
    o[18] = p->unit;
    o[19] = p->density_gain;
    memcpy(o + 20, &fid, 4);
    memcpy(o + 21, &spp, 4);
  }
  CK(ctx->diff_views.reserve(sizeof(float) * hv.size()), "views alloc");
  CK(cudaMemcpyAsync(ctx->diff_views.ptr, hv.data(), sizeof(float) * hv.size(), cudaMemcpyHostToDevice, st),
     "views upload");
  CK(cudaStreamSynchronize(st), "views upload");
  memset(&A, 0, sizeof(A));
  fill_scene_view(ctx, views[0].cam_pos, A.s);
  A.s.loop_cap = views[0].loop_cap;
  for (int v = 1; v < nviews; ++v) A.s.eps = std::fmax(A.s.eps, scene_eps(ctx, views[v].cam_pos));
  A.views = ctx->diff_views.ptr;
  A.nviews = nviews;
  A.width = w;
  A.height = h;
  if (!ctx->work.ptr) CK(ctx->work.reserve(256), "work counter");
  A.work_counter = ctx->work.as<uint32_t>();
  A.status = ctx->status.as<uint32_t>();
  {
    size_t words = 0;
    CK(diff_stack_words(&words), "differentiable kernel setup");
    CK(ctx->warp_stacks.reserve(4 * words), "warp stacks");
  }
  A.warp_stacks = ctx->warp_stacks.as<uint32_t>();
  ctx->diff_samples = (size_t)nviews * (size_t)w * (size_t)h * spp0;
  ctx->diff_spp = spp0;
  return AARBF_OK;
}

aarbf_status aarbf_render_diff_forward(aarbf_ctx* ctx, const aarbf_params* views, int nviews, int w, int h,
                                       float* images, void* stream) {
  if (!ctx || !images) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  cudaStream_t st = (cudaStream_t)stream;
  DiffArgs A;
  ctx->diff_ready = false;
  aarbf_status s = diff_setup(ctx, views, nviews, w, h, A, st);
  if (s != AARBF_OK) return s;
  CK(ctx->diff_ckpt.reserve(16 * ctx->diff_samples), "checkpoint alloc");
  A.image = reinterpret_cast<float4*>(images);
  A.ckpt = ctx->diff_ckpt.as<float4>();
  CK(launch_diff(A, st), "diff forward");
  ctx->diff_ready = true;
  ctx->diff_nviews = nviews;
  ctx->diff_w = w;
  ctx->diff_h = h;
  return AARBF_OK;
}

aarbf_status aarbf_render_diff_backward(aarbf_ctx* ctx, const aarbf_params* views, int nviews, int w, int h,
                                        const float* grad_images, float* grad_xyz, float* grad_radius,
                                        float* grad_attr, float* grad_tf, void* stream) {
  if (!ctx || !grad_images || !grad_xyz || !grad_radius || !grad_attr || !grad_tf) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (!ctx->diff_ready || ctx->diff_nviews != nviews || ctx->diff_w != w || ctx->diff_h != h || !views ||
      (views[0].spp ? views[0].spp : 1u) != ctx->diff_spp)
    return fail(ctx, AARBF_ERR_NOT_READY, "backward without a matching aarbf_render_diff_forward");
  cudaStream_t st = (cudaStream_t)stream;
  DiffArgs A;
  aarbf_status s = diff_setup(ctx, views, nviews, w, h, A, st);
  if (s != AARBF_OK) return s;
  const uint64_t n = ctx->n;
  const size_t nn = n ? n : 1;
  CK(ctx->diff_grad.reserve(sizeof(float) * 8 * nn), "gradient alloc");
  float* gp = ctx->diff_grad.as<float>();
  CK(cudaMemsetAsync(gp, 0, sizeof(float) * 8 * nn, st), "gradient clear");
  CK(cudaMemsetAsync(grad_tf, 0, sizeof(float) * 4 * (size_t)ctx->nc, st), "gradient clear");
  A.backward = true;
  A.ckpt = ctx->diff_ckpt.as<float4>();
  A.grad_image = reinterpret_cast<const float4*>(grad_images);
  A.g_pos = gp;
  A.g_rad = gp + 3 * nn;
  A.g_w = gp + 4 * nn;
  CK(launch_diff(A, st), "diff backward");
  const float scale = 1.0f / (ctx->dom[7] - ctx->dom[6]);  // attribute normalisation
  CK(launch_diff_finish(ctx->xyzw.as<float4>(), ctx->perm.as<uint32_t>(), n, ctx->tf_color.as<float4>(), ctx->nc,
                        scale, A.g_pos, A.g_rad, A.g_w, grad_xyz, grad_radius, grad_attr, grad_tf, st),
     "diff finish");
  return AARBF_OK;
}

aarbf_status aarbf_render_splat(aarbf_ctx* ctx, const aarbf_params* p, int w, int h, float* image, void* stream) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (!image) {
    aarbf_status s = ensure_fb(ctx, w, h);
    if (s != AARBF_OK) return s;
    image = ctx->fb_image.as<float>();
  }
  RenderLaunch L;
  aarbf_status s = fill_launch(ctx, p, w, h, nullptr, image, L);
  if (s != AARBF_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  if (p->traversal == AARBF_TRAVERSAL_THREAD) {
    CK(launch_splat(L, st), "splat launch");
    return AARBF_OK;
  }
  // slab starts of the ray-per-warp kernel: the running sum t += spacing from 0, tabulated until
  // it passes the farthest corner of the padded box (every ray's exit lies before it)
  const float spacing = (float)(15 / 8) * p->unit;
  double far2 = 0.0;
  for (int c = 0; c < 8; ++c) {
    double d2 = 0.0;
    for (int a = 0; a < 3; ++a) {
      double v = ((c >> a) & 1) ? (double)p->aabb_max[a] + p->rbf_radius : (double)p->aabb_min[a] - p->rbf_radius;
      d2 += (v - p->cam_pos[a]) * (v - p->cam_pos[a]);
    }
    far2 = std::fmax(far2, d2);
  }
  const float tfar = (float)(std::sqrt(far2) * 1.001) + 2.0f * spacing;
  std::vector<float> tab;
  bool ok = spacing > 0.0f && std::isfinite(tfar);
  if (ok) {
    float t = 0.0f;
    tab.push_back(t);
    while (t < tfar) {
      const float nt = t + spacing;
      if (!(nt > t) || tab.size() >= (1u << 20)) {
        ok = false;
        break;
      }
      t = nt;
      tab.push_back(t);
    }
  }
  if (!ok) {  // too many slabs for the table: thread-per-pixel kernel
    CK(launch_splat(L, st), "splat launch");
    return AARBF_OK;
  }
  if (ctx->splat_spacing != spacing || ctx->splat_nslabs < (int)tab.size()) {
    CK(ctx->splat_slabs.reserve(sizeof(float) * tab.size()), "slab table alloc");
    CK(cudaMemcpyAsync(ctx->splat_slabs.ptr, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, st),
       "slab table upload");
    CK(cudaStreamSynchronize(st), "slab table upload");
    ctx->splat_spacing = spacing;
    ctx->splat_nslabs = (int)tab.size();
  }
  if (!ctx->work.ptr) CK(ctx->work.reserve(256), "work counter");
  L.work_counter = ctx->work.as<uint32_t>();
  {
    size_t words = 0;
    CK(splat_stack_words(&words), "splat kernel setup");
    CK(ctx->warp_stacks.reserve(4 * words), "warp stacks");
  }
  L.warp_stacks = ctx->warp_stacks.as<uint32_t>();
  CK(launch_splat(L, st, ctx->splat_slabs.as<float>(), ctx->splat_nslabs), "splat launch");
  return AARBF_OK;
}

aarbf_status aarbf_taa_resolve(aarbf_ctx* ctx, const float* image, const float* prev, float* taa, uint32_t* bgra,
                               int w, int h, int disable, void* stream) {
  if (!image || w <= 0 || h <= 0 || (!disable && (!prev || !taa)))
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "bad TAA arguments");
  if (ctx) cudaSetDevice(ctx->device);
  CK(launch_taa(reinterpret_cast<const float4*>(image), reinterpret_cast<const float4*>(prev),
                reinterpret_cast<float4*>(taa), bgra, w, h, disable, (cudaStream_t)stream),
     "taa launch");
  return AARBF_OK;
}

aarbf_status aarbf_device_alloc(aarbf_ctx* ctx, size_t bytes, void** ptr) {
  if (!ctx || !ptr) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  *ptr = nullptr;
  CK(cudaMalloc(ptr, bytes ? bytes : 1), "device alloc");
  return AARBF_OK;
}

aarbf_status aarbf_device_free(aarbf_ctx* ctx, void* ptr) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (ptr) CK(cudaFree(ptr), "device free");
  return AARBF_OK;
}

aarbf_status aarbf_memcpy(aarbf_ctx* ctx, void* dst, const void* src, size_t bytes, void* stream) {
  if (!ctx || (bytes && (!dst || !src))) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, (cudaStream_t)stream), "memcpy");
  return AARBF_OK;
}

aarbf_status aarbf_memset(aarbf_ctx* ctx, void* dst, int value, size_t bytes, void* stream) {
  if (!ctx || (bytes && !dst)) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  CK(cudaMemsetAsync(dst, value, bytes, (cudaStream_t)stream), "memset");
  return AARBF_OK;
}

aarbf_status aarbf_set_noise_atlas(aarbf_ctx* ctx, const uint8_t* rgba8, int w, int h) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  std::vector<uint8_t> gen;
  if (!rgba8) {
    w = 2048;
    h = 4096;
    gen.resize((size_t)w * h * 4);
    aarbf_generate_noise_atlas(gen.data(), w, h);
    rgba8 = gen.data();
  }
  if (w <= 0 || h <= 0) return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "bad noise atlas size");
  size_t bytes = (size_t)w * h * 4;
  CK(ctx->noise.reserve(bytes), "noise alloc");
  CK(upload(ctx->noise.ptr, rgba8, bytes, nullptr), "noise upload");
  CK(cudaStreamSynchronize(nullptr), "noise upload");
  ctx->noise_w = w;
  ctx->noise_h = h;
  return AARBF_OK;
}


aarbf_status aarbf_camera(const float* from, const float* at, const float* up, float cos_fovy, int w, int h,
                          float* pos, float* d00, float* du, float* dv) {
  if (!from || !at || !up || !pos || !d00 || !du || !dv || w <= 0 || h <= 0) return AARBF_ERR_INVALID_ARGUMENT;
  auto normalize = [](const float* a, float* o) {
    float len = std::sqrt((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2]);
    o[0] = a[0] / len;
    o[1] = a[1] / len;
    o[2] = a[2] / len;
  };
  auto cross = [](const float* a, const float* b, float* o) {
    float x = a[1] * b[2] - a[2] * b[1];
    float y = a[2] * b[0] - a[0] * b[2];
    float z = a[0] * b[1] - a[1] * b[0];
    o[0] = x;
    o[1] = y;
    o[2] = z;
  };
  float diff[3] = {at[0] - from[0], at[1] - from[1], at[2] - from[2]};
  float dir[3], c[3], nrm[3];
  normalize(diff, dir);
  float aspect = (float)w / (float)h;
  cross(dir, up, c);
  normalize(c, nrm);
  float su = cos_fovy * aspect;
  float ddu[3] = {su * nrm[0], su * nrm[1], su * nrm[2]};
  cross(ddu, dir, c);
  normalize(c, nrm);
  float ddv[3] = {cos_fovy * nrm[0], cos_fovy * nrm[1], cos_fovy * nrm[2]};
  for (int a = 0; a < 3; ++a) {
    float d = dir[a] - 0.5f * ddu[a];
    d = d - 0.5f * ddv[a];
    pos[a] = from[a];
    d00[a] = d;
    du[a] = ddu[a];
    dv[a] = ddv[a];
  }
  return AARBF_OK;
}

// ---- debug getters ----------------------------------------------------------------------------

aarbf_status aarbf_get_num_particles(const aarbf_ctx* ctx, uint64_t* n, uint32_t* nl) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (n) *n = ctx->n;
  if (nl) *nl = ctx->nleaves;
  return AARBF_OK;
}

aarbf_status aarbf_get_hilbert_keys(aarbf_ctx* ctx, uint64_t* keys, uint32_t* perm) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (!ctx->built) return fail(ctx, AARBF_ERR_NOT_READY, "not built");
  cudaSetDevice(ctx->device);
  if (keys && ctx->n) CK(cudaMemcpy(keys, ctx->sorted_keys.ptr, 8 * ctx->n, cudaMemcpyDeviceToHost), "keys");
  if (perm && ctx->n) CK(cudaMemcpy(perm, ctx->perm.ptr, 4 * ctx->n, cudaMemcpyDeviceToHost), "perm");
  return AARBF_OK;
}

aarbf_status aarbf_get_sorted_particles(aarbf_ctx* ctx, float* xyzw) {
  if (!ctx || !xyzw) return AARBF_ERR_INVALID_ARGUMENT;
  if (!ctx->built) return fail(ctx, AARBF_ERR_NOT_READY, "not built");
  cudaSetDevice(ctx->device);
  if (ctx->n) CK(cudaMemcpy(xyzw, ctx->xyzw.ptr, 16 * ctx->n, cudaMemcpyDeviceToHost), "particles");
  return AARBF_OK;
}

aarbf_status aarbf_get_prepass(aarbf_ctx* ctx, float* rec0, float* w4, float* rgeom) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (!ctx->built) return fail(ctx, AARBF_ERR_NOT_READY, "not built");
  cudaSetDevice(ctx->device);
  const uint64_t n = ctx->n;
  if (!n) return AARBF_OK;
  if (rec0) CK(cudaMemcpy(rec0, ctx->rec0.ptr, 16 * n, cudaMemcpyDeviceToHost), "rec0");
  if (w4) CK(cudaMemcpy(w4, ctx->w4.ptr, 16 * n, cudaMemcpyDeviceToHost), "w4");
  if (rgeom) CK(cudaMemcpy(rgeom, ctx->rgeom.ptr, 4 * n, cudaMemcpyDeviceToHost), "rgeom");
  return AARBF_OK;
}

aarbf_status aarbf_set_storage(aarbf_ctx* ctx, int format) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (format != AARBF_STORAGE_FP32 && format != AARBF_STORAGE_FP16)
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "unknown storage format");
  ctx->storage_fp16 = format == AARBF_STORAGE_FP16;
  ctx->built = false;
  return AARBF_OK;
}

aarbf_status aarbf_set_opacity_floor(aarbf_ctx* ctx, float alpha_floor) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (!(alpha_floor >= 0.0f && alpha_floor <= 1.0f))
    return fail(ctx, AARBF_ERR_INVALID_ARGUMENT, "opacity floor must lie in [0, 1]");
  if (alpha_floor != ctx->alpha_floor) {
    ctx->alpha_floor = alpha_floor;
    ctx->built = false;
  }
  return AARBF_OK;
}

aarbf_status aarbf_get_bvh(aarbf_ctx* ctx, uint32_t* left, uint32_t* right, float* node_box, float* leaf_box,
                           float* leaf_eff, float* root_box) {
  if (!ctx) return AARBF_ERR_INVALID_ARGUMENT;
  if (!ctx->built) return fail(ctx, AARBF_ERR_NOT_READY, "not built");
  cudaSetDevice(ctx->device);
  const uint32_t L = ctx->nleaves;
  const uint32_t ni = L > 0 ? L - 1 : 0;
  std::vector<Node> nodes(ni);
  if (ni) CK(cudaMemcpy(nodes.data(), ctx->nodes.ptr, sizeof(Node) * ni, cudaMemcpyDeviceToHost), "nodes");
  for (uint32_t i = 0; i < ni; ++i) {
    if (left) left[i] = nodes[i].d.x;
    if (right) right[i] = nodes[i].d.y;
    if (node_box) {
      const float* f = reinterpret_cast<const float*>(&nodes[i]);
      for (int a = 0; a < 3; ++a) {
        node_box[6 * i + a] = std::fmin(f[a], f[6 + a]);
        node_box[6 * i + 3 + a] = std::fmax(f[3 + a], f[9 + a]);
      }
    }
  }
  if (leaf_box && L) CK(cudaMemcpy(leaf_box, ctx->leaf_box.ptr, 24 * (size_t)L, cudaMemcpyDeviceToHost), "leaf box");
  if (leaf_eff && L) CK(cudaMemcpy(leaf_eff, ctx->leaf_eff.ptr, 24 * (size_t)L, cudaMemcpyDeviceToHost), "leaf box");
  if (root_box) memcpy(root_box, ctx->root_box_host, 6 * sizeof(float));
  return AARBF_OK;
}

}  // extern "C"
