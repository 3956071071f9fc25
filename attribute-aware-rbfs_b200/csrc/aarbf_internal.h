// aarbf_internal.h -- context state and kernel launchers shared by the library's sources.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/aarbf.h"
#include "aarbf_device.cuh"

namespace aarbf {

// Grow-only device buffer.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaError_t reserve(size_t want) {
    if (want <= bytes) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t alloc = want < 256 ? 256 : want;
    cudaError_t e = cudaMalloc(&ptr, alloc);
    if (e == cudaSuccess) bytes = alloc;
    return e;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  template <class T>
  T* as() const { return static_cast<T*>(ptr); }
};

// Launch configuration that belongs to one device: kernel attributes such as the dynamic
// shared-memory limit are set per device context, and grid sizes follow the device's SM count.
// Each value is computed once per device, under a lock, by init(device, &value) with that device
// current; a value of 0 means "not computed yet".
constexpr int kMaxDevices = 64;
struct PerDevice {
  std::mutex mu;
  int value[kMaxDevices] = {};
};
template <class Init>
cudaError_t per_device(PerDevice& c, int* out, Init&& init) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(c.mu);
  if (c.value[dev] == 0) {
    int v = 0;
    e = init(dev, &v);
    if (e != cudaSuccess) return e;
    c.value[dev] = v > 0 ? v : 1;
  }
  *out = c.value[dev];
  return cudaSuccess;
}

// Everything the tracking / marching / splat kernels read about a built scene.
struct SceneView {
  const float4* rec0;  // x, y, z, r_eval
  const float4* w4;    // a^3, pow(rgb, 2.2) a^3
  const float4* xyzw;  // sorted particles (attribute normalised)
  const float* rgeom;  // bounds radius, -1 = skipped by the bounds program
  const Node* nodes;      // traversal bounds (particles that can be hit)
  const Node* nodes_ref;  // reference bounds (splatting)
  const WideNode* wide;      // wide form of nodes (what the warp traversals read)
  const WideNode* wide_ref;  // wide form of nodes_ref
  const float4* tf_color;
  const float* tf_density;
  uint64_t n;
  uint32_t ppl;
  uint32_t nleaves;
  uint32_t root;  // child code of the root
  int nc, nd;
  float root_lo[3], root_hi[3];
  float eps;      // absolute slack used by conservative culling tests
  int per_particle_radius;
  uint32_t loop_cap;  // 0, or a lower iteration bound for every device loop (loop_bound)
  // FP16 storage form (null in the fp32 form): packed records the tracking kernels read
  const uint2* posq;     // FP16 offsets x, y, z from the run origin, FP16 radius rounded up (culling)
  const uint2* colq;     // FP16 rgb^2.2 a^3 and a^3
  const float4* origin;  // fp32 origin of every run of 256 particles
  const float* reval;    // fp32 r_eval
};

struct RenderLaunch {
  SceneView s;
  uint32_t accum_id, frame_id, spp, flags;
  float ambient;
  float light[3];
  float cam_pos[3], cam_d00[3], cam_du[3], cam_dv[3];
  float rbf_radius, unit, density_gain, jitter_x, jitter_y;
  float aabb_min[3], aabb_max[3];
  const uchar4* noise;
  int noise_w, noise_h;
  int width, height;
  float4* accum;
  float4* image;
  uint32_t* status;
  int traversal;
  float splat_rmax;                // largest splat radius of the scene
  unsigned long long* counters;    // count mode: [particles on traversed segments, node visits]
  float density_scale, bin_length; // majorant tracking
  uint32_t* work_counter;          // persistent kernel: next pixel tile item (zeroed per launch)
  int candidate_cap;               // staging buffer depth per ray (template instance)
  int stage_bins;                  // majorant tracking: bins staged first (1..64)
  float4* samples;                 // spp planes of per-sample colours (width * height each)
  float* noise_buf;                // per pixel: noise value of the last sample (showNoise)
  uint32_t* warp_stacks;           // ray-per-warp kernel: one traversal stack per resident warp
};

// launchers (defined in the .cu files)
cudaError_t launch_domain_reduce(const float4* p, uint64_t n, float* d_partial, int nblocks,
                                 cudaStream_t st);
cudaError_t launch_hilbert_keys(const float4* p, uint64_t n, const float* dom, uint64_t* keys,
                                uint32_t* perm, cudaStream_t st);
cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                             uint64_t n, int key_bits, uint32_t* hist, size_t hist_words,
                             cudaStream_t st, bool* result_in_alt);
size_t radix_sort_hist_words(uint64_t n);
// orders every run of equal sorted keys of at most 64 entries by (x, y, z, w, input index) in
// place on perm; *flag |= 1 if any run exists, |= 2 if a longer run needs the full chain
cudaError_t launch_tie_runs(const uint64_t* keys, const float4* p, uint32_t* perm, uint64_t n, uint32_t* flag,
                            cudaStream_t st);
cudaError_t launch_orderable_component(const float4* p, const uint32_t* perm, uint64_t n, int comp,
                                       uint64_t* out, cudaStream_t st);
cudaError_t launch_hilbert_keys_perm(const float4* p, const uint32_t* perm, uint64_t n, const float* dom,
                                     uint64_t* keys, cudaStream_t st);
cudaError_t launch_gather_normalize(const float4* in, const float* radii_in, const uint32_t* perm,
                                    uint64_t n, float amin, float amax, float4* out,
                                    float* radii_out, cudaStream_t st);
cudaError_t launch_prepass(const float4* xyzw, const float* radii, uint64_t n, const float4* tf_color,
                           int nc, const float* tf_radius, int nr, float rbf_radius, float alpha_floor,
                           float4* rec0, float4* w4, float* rgeom, cudaStream_t st);
cudaError_t launch_karras(const uint64_t* sorted_keys, uint64_t n, uint32_t ppl, uint32_t nleaves,
                          Node* nodes, Node* nodes_ref, uint32_t* leaf_parent, cudaStream_t st);
// largest bounds radius of the scene into *out (device)
cudaError_t launch_max_radius(const float* rgeom, uint64_t n, float* out, cudaStream_t st);
// wide nodes (several binary levels per node) of the binary tree; nleaves - 1 of them
cudaError_t launch_collapse(const Node* nodes, uint32_t nleaves, WideNode* wide, cudaStream_t st);
cudaError_t launch_refit(const float4* rec0, const float* rgeom, uint64_t n, uint32_t ppl,
                         uint32_t nleaves, Node* nodes, Node* nodes_ref, const uint32_t* leaf_parent,
                         uint32_t* counters, float* leaf_box, float* leaf_eff, float* root_box,
                         uint32_t* status, cudaStream_t st);
// the tracking kernels, built for the fp32 records (r32) and the FP16 storage form (r16)
struct BatchArgs;
#define AARBF_RENDER_DECLS                                                                      \
  cudaError_t launch_render(const RenderLaunch& L, cudaStream_t st, const cudaEvent_t* marks); \
  bool render_uses_warp_kernel(const RenderLaunch& L);                                          \
  cudaError_t render_warp_stack_words(size_t* words);                                           \
  cudaError_t launch_render_batched(const BatchArgs& B, cudaStream_t st);
namespace r32 { AARBF_RENDER_DECLS }
namespace r16 { AARBF_RENDER_DECLS }
#undef AARBF_RENDER_DECLS

// marks (optional): three events recorded before the tracking kernel, between it and the
// accumulation pass, and after the accumulation pass.
inline cudaError_t launch_render(const RenderLaunch& L, cudaStream_t st, const cudaEvent_t* marks = nullptr) {
  return L.s.posq ? r16::launch_render(L, st, marks) : r32::launch_render(L, st, marks);
}
inline bool render_uses_warp_kernel(const RenderLaunch& L) { return r32::render_uses_warp_kernel(L); }
// stack words for the largest grid of either build
inline cudaError_t render_warp_stack_words(size_t* words) {
  size_t a = 0, b = 0;
  cudaError_t e = r32::render_warp_stack_words(&a);
  if (e == cudaSuccess) e = r16::render_warp_stack_words(&b);
  *words = a > b ? a : b;
  return e;
}
// slabs: the splat slab starts (nslabs entries, the last beyond every ray's exit) for the
// ray-per-warp splat kernel; NULL selects the thread-per-pixel kernel
cudaError_t launch_splat(const RenderLaunch& L, cudaStream_t st, const float* slabs = nullptr, int nslabs = 0);
cudaError_t splat_stack_words(size_t* words);

// several scenes in one persistent launch of the ray-per-warp kernel (render.cu)
struct BatchArgs {
  const RenderLaunch* launches;  // device: one launch block per scene
  const RenderLaunch* host_launches;  // host copies of the launch blocks (kernel parameters)
  const uint64_t* host_items;    // host: nscenes + 1 prefix sums of work items
  const uint64_t* pix_ofs;       // device: nscenes + 1 prefix sums of pixels
  int nscenes;
  uint64_t total_pixels;
  int candidate_cap;
  uint32_t* work_counters;        // device: 64 per-scene item counters (256 bytes)
  uint32_t* warp_stacks;
  bool fp16;                     // every scene is in the FP16 storage form
  int blocks_per_sm;             // resident blocks per SM (0 = the occupancy limit)
  int sample_major;              // work items sample by sample (1) or tile by tile (0)
};
inline cudaError_t launch_render_batched(const BatchArgs& B, cudaStream_t st) {
  return B.fp16 ? r16::launch_render_batched(B, st) : r32::launch_render_batched(B, st);
}

// FP16 storage form (fp16.cu)
cudaError_t launch_quantize_positions(float4* xyzw, uint64_t n, uint2* posq, float4* origin, cudaStream_t st);
cudaError_t launch_quantize_weights(float4* w4, const float4* rec0, uint64_t n, uint2* posq, uint2* colq,
                                   float* reval, cudaStream_t st);

// differentiable form (diff.cu)
struct DiffArgs {
  SceneView s;
  const void* views;         // device array: per view 22 words (camera, padded box, unit, gain, frame, spp)
  int nviews, width, height;
  float4* image;             // forward output
  float4* ckpt;              // per-sample checkpoint
  const float4* grad_image;  // backward input
  float* g_pos;              // backward accumulators, sorted order
  float* g_rad;
  float* g_w;
  uint32_t* work_counter;
  uint32_t* status;
  uint32_t* warp_stacks;
  bool backward;
};
cudaError_t launch_diff(const DiffArgs& A, cudaStream_t st);
cudaError_t diff_stack_words(size_t* words);
cudaError_t launch_diff_finish(const float4* xyzw, const uint32_t* perm, uint64_t n, const float4* tf, int nc,
                               float attr_scale, const float* g_pos, const float* g_rad, const float* g_w,
                               float* out_pos, float* out_rad, float* out_attr, float* out_tf, cudaStream_t st);
cudaError_t launch_taa(const float4* image, const float4* prev, float4* taa, uint32_t* bgra, int w,
                       int h, int disable, cudaStream_t st);

}  // namespace aarbf

struct aarbf_ctx {
  int device = 0;
  std::string last_error;
  // input frame
  aarbf::DevBuf in_xyzw, in_radii;
  uint64_t n = 0;
  bool has_radii = false;
  // domain
  float dom[8] = {0, 0, 0, 1, 1, 1, 0, 1};
  bool has_domain = false;
  // sort
  aarbf::DevBuf keys, keys_alt, perm, perm_alt, hist, tmp_keys, flag;
  // sorted scene
  aarbf::DevBuf xyzw, radii, rec0, w4, rgeom, nodes, nodes_ref, leaf_parent, counters, leaf_box, leaf_eff,
      root_box;
  float alpha_floor = 0.0f;  // opacity below this counts as transparent
  aarbf::DevBuf sorted_keys;  // Hilbert keys in sorted order
  uint32_t ppl = 1, nleaves = 0;
  float rbf_radius = 0.0f;
  bool built = false;
  uint64_t built_n = 0;          // particle count and radii presence of the last aarbf_build
  bool built_has_radii = false;
  bool has_topology = false;     // the last aarbf_build completed: its BVH topology can be refit
  float root_box_host[6] = {0, 0, 0, 0, 0, 0};
  // transfer functions
  aarbf::DevBuf tf_color, tf_radius, tf_density;
  int nc = 0, nr = 0, nd = 0;
  bool has_tf = false;
  // noise atlas
  aarbf::DevBuf noise;
  int noise_w = 0, noise_h = 0;
  // framebuffers owned by the context
  aarbf::DevBuf fb_accum, fb_image;
  int fb_w = 0, fb_h = 0;
  // status word, persistent-kernel work counter, per-sample colour planes
  aarbf::DevBuf status, work, samples, noise_buf, warp_stacks;
  float max_radius = 0.0f;
  aarbf::DevBuf wide, wide_ref;  // wide forms of nodes / nodes_ref
  aarbf::DevBuf splat_slabs;      // slab starts of the splat kernel, for splat_spacing
  float splat_spacing = 0.0f;
  int splat_nslabs = 0;
  bool storage_fp16 = false;     // FP16 storage form (takes effect at the next build)
  bool built_fp16 = false;       // the built scene is in the FP16 form
  aarbf::DevBuf posq, colq, origin, reval;
  bool radius_map_unit = false;  // every radius-map texel is 1 (required by the differentiable form)
  // differentiable form: views, per-sample checkpoints, gradient accumulators
  aarbf::DevBuf diff_views, diff_ckpt, diff_grad;
  size_t diff_samples = 0;
  bool diff_ready = false;
  int diff_nviews = 0, diff_w = 0, diff_h = 0;
  uint32_t diff_spp = 0;
  // kernel timing: event triples of timed renders not yet read, and recycled ones
  bool kernel_timing = false;
  std::vector<std::array<cudaEvent_t, 3>> ev_pending, ev_free;
};
