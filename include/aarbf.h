/*
 * aarbf.h -- C ABI of the B200 attribute-aware Gaussian-RBF particle-volume renderer.
 *
 * This is the drop-in boundary for the reference's GPU path (gprt-org/attribute-aware-rbfs):
 * the GPRT program registration and launches of hostCode.cpp (bounds compute program,
 * hardware BVH build/refit, the RBF ray-generation program with its intersection/any-hit
 * programs, the splat ray-generation program, the CompositeGui TAA pass). Each entry point
 * below names the reference interface it replaces (file:line in the reference tree).
 *
 * Conventions
 *  - Plain pointers and sizes; no C++ or torch types. All functions return aarbf_status and
 *    never abort; aarbf_last_error() gives a message for the last failing call on a context.
 *  - A context is bound to one CUDA device and is not internally locked: use one context per
 *    host thread. GPU work is enqueued on the caller's stream (`stream` is a cudaStream_t;
 *    NULL = the legacy default stream). aarbf_render* do not synchronise.
 *  - Particle and transfer-function inputs may be host or device pointers (detected).
 *    Render targets are caller-owned device pointers (float4 per pixel, row-major,
 *    offset = x + width * y as in deviceCodeRBF.hlsl:210) or NULL for context-owned ones.
 */
#ifndef AARBF_H
#define AARBF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AARBF_VERSION_MAJOR 0
#define AARBF_VERSION_MINOR 1

typedef enum aarbf_status {
  AARBF_OK = 0,
  AARBF_ERR_INVALID_ARGUMENT = 1,
  AARBF_ERR_OUT_OF_MEMORY = 2,
  AARBF_ERR_CUDA = 3,
  AARBF_ERR_DEVICE_LIMIT = 4, /* a device-side cap was hit (traversal stack, loop cap) */
  AARBF_ERR_NOT_READY = 5,    /* e.g. render before build */
  AARBF_ERR_IO = 6,
  AARBF_ERR_UNSUPPORTED = 7
} aarbf_status;

typedef struct aarbf_ctx aarbf_ctx;

/* Render flags: PushConstants booleans (sharedCode.h:37-40) plus native-mode switches. */
enum {
  AARBF_FLAG_BLUE_NOISE = 1u << 0,           /* enableBlueNoise -> stochastic marching */
  AARBF_FLAG_SHOW_NOISE = 1u << 1,           /* showNoise */
  AARBF_FLAG_VISUALIZE_ATTRIBUTES = 1u << 2, /* visualizeAttributes (reference default: on) */
  AARBF_FLAG_TRACK_FROM_ENTRY = 1u << 3,     /* native: delta tracking starts at tenter + unit*xi */
  AARBF_FLAG_DENSITY_LINEAR = 1u << 4,       /* native: density = min(D * density_gain, 1) */
  AARBF_FLAG_SPLAT_PARTICLE_RADIUS = 1u << 5, /* native: splats use the per-particle radius */
  AARBF_FLAG_MAJORANT_TRACKING = 1u << 6,     /* native: delta tracking with per-bin majorants
                                                 (extinction = density_scale * D, unclamped) */
  AARBF_FLAG_COST_IMAGE = 1u << 7             /* diagnostic: image alpha = SM clock cycles the
                                                 pixel's samples took */
};

/* Traversal strategies of the render kernel; every choice gives bit-identical results. */
enum {
  AARBF_TRAVERSAL_AUTO = 0,  /* one warp per ray (cooperative traversal, staged candidate lists
                                and fixed-point sums) for every estimator */
  AARBF_TRAVERSAL_POINT = 1, /* one BVH point query per tracking step (reference shape) */
  AARBF_TRAVERSAL_THREAD = 2 /* per-thread staged segments for every estimator */
};

/*
 * Per-launch parameters. Mirrors PushConstants (sharedCode.h:33-74) and the RayGenData record
 * (sharedCode.h:108-117): accumID/frameID are taken modulo 2^16 like the reference's uint16.
 * spp > 1 renders spp consecutive frames (frameID+k, accumID+k) in one launch; the result is
 * bit-identical to spp launches of one frame each.
 */
typedef struct aarbf_params {
  uint32_t accum_id;
  uint32_t frame_id;
  uint32_t spp;
  uint32_t flags;
  float light_azimuth, light_elevation, light_ambient;
  float cam_pos[3], cam_dir00[3], cam_du[3], cam_dv[3];
  float rbf_radius;  /* global radius (per-particle radii multiply nothing into it) */
  float unit;        /* delta-tracking / marching step unit */
  float aabb_min[3]; /* RayGenData.globalAABBMin / Max: the space-time box */
  float aabb_max[3];
  float density_gain; /* AARBF_FLAG_DENSITY_LINEAR: density scale * unit */
  float jitter_x, jitter_y; /* sub-pixel camera jitter in pixels (0 = reference) */
  int32_t traversal;        /* AARBF_TRAVERSAL_* */
  float density_scale;      /* AARBF_FLAG_MAJORANT_TRACKING: extinction per unit length per unit D */
  float bin_length;         /* AARBF_FLAG_MAJORANT_TRACKING: majorant bin length along a ray */
  int32_t candidate_cap;    /* staged candidates per ray: 16, 32, 64 or 128 per thread (0 = 32),
                               or 256, 512 or 1024 per warp for the warp kernel (0 = 256);
                               tuning only, results are identical for every value */
  int32_t stage_bins;       /* bins staged by the first traversal of a ray (1..64; 0 = 4 for the
                               warp kernel, 16 per thread; later stagings double, the warp
                               kernel's at most to 64 bins and to half a buffer of candidates at
                               the last staging's density); the
                               bins are bin_length long (16 units when bin_length is 0 and majorant
                               tracking is off); tuning only */
  uint32_t loop_cap;        /* 0 = the built-in iteration bounds of the device loops (the
                               reference's MAX_DEPTH step budget is not one of them). A positive
                               value lowers every bound to it, so the status path can be
                               exercised: a loop that runs out of iterations leaves its pixel
                               incomplete and makes the next aarbf_sync return
                               AARBF_ERR_DEVICE_LIMIT (the reference caps its loops silently at
                               MAX_DEPTH, sharedCode.h:27). */
} aarbf_params;

/* ---- context -------------------------------------------------------------------------- */

/* replaces gprtContextCreate (hostCode.cpp:280-281): bind a context to CUDA device `device` */
aarbf_status aarbf_create(aarbf_ctx **out, int device);
/* replaces the gprt*Destroy calls (hostCode.cpp:834-848) */
aarbf_status aarbf_destroy(aarbf_ctx *ctx);
const char *aarbf_last_error(const aarbf_ctx *ctx);
const char *aarbf_status_string(aarbf_status s);
aarbf_status aarbf_get_version(int *major, int *minor);
/* waits for the stream, then reports (and clears) device-side error bits */
aarbf_status aarbf_sync(aarbf_ctx *ctx, void *stream);

/* ---- particles and domain --------------------------------------------------------------- */

/* Upload one frame of particles: float4 (x, y, z, attribute) x n, as importParticles
 * (importParticles.h:8-31) yields them; replaces the particle buffer upload
 * (hostCode.cpp:759-763). radii: optional per-particle radius (n floats) or NULL. */
aarbf_status aarbf_set_particles(aarbf_ctx *ctx, const float *xyzw, uint64_t n, const float *radii,
                                 void *stream);

/* Space-time domain used to quantise Hilbert keys and normalise attributes
 * (hostCode.cpp:183-193, :227-250). dom = {minx,miny,minz,maxx,maxy,maxz,attr_min,attr_max}. */
aarbf_status aarbf_set_domain(aarbf_ctx *ctx, const float *dom);
/* Reduce frames on the device into a running domain (initialise dom with aarbf_domain_init). */
aarbf_status aarbf_domain_init(float *dom);
aarbf_status aarbf_domain_accumulate(aarbf_ctx *ctx, const float *xyzw, uint64_t n, float *dom,
                                     void *stream);

/* ---- transfer functions (hostCode.cpp:355-365, :416-436, :524-572) ------------------------ */

/* 8-bit textures exactly as the reference uploads them (R8G8B8A8_SRGB): colormap RGBA x nc,
 * radiusmap and densitymap use their R channel (RGBA x nr / x nd). */
aarbf_status aarbf_set_transfer_functions_rgba8(aarbf_ctx *ctx, const uint8_t *colormap, int nc,
                                                const uint8_t *radiusmap, int nr,
                                                const uint8_t *densitymap, int nd);
/* fp32 tables (native mode): colormap RGBA x nc (rgb linear), radiusmap x nr, densitymap x nd. */
aarbf_status aarbf_set_transfer_functions_f32(aarbf_ctx *ctx, const float *colormap, int nc,
                                              const float *radiusmap, int nr,
                                              const float *densitymap, int nd);
/* Opacity below alpha_floor counts as transparent, as opacity 0 does in the any-hit program
 * (deviceCodeRBF.hlsl:369-372). Default 0 (the reference). With fp32 transfer functions, 1/255
 * reproduces the resolution of the reference's 8-bit textures. Takes effect at the next
 * aarbf_build / aarbf_refit. */
aarbf_status aarbf_set_opacity_floor(aarbf_ctx *ctx, float alpha_floor);
/* Gradient marks -> 64-entry RGBA8 texture as hostCode.cpp:528-542 (gamma 1/2.2 on rgb when
 * gamma != 0) and :544-572 (grey maps). marks: npos positions + npos RGBA colours. */
aarbf_status aarbf_marks_to_rgba8(const float *pos, const float *rgba, int nmarks, int gamma,
                                  uint8_t *out, int ntexels);

/* ---- acceleration structure -------------------------------------------------------------- */

/* Hilbert keys, device radix sort, attribute normalisation, per-particle shading prepass,
 * leaf bounds (GenRBFBounds, deviceCodeBounds.hlsl:29-82), Karras LBVH and refit. Replaces
 * GenRBFBounds + gprtAccelBuild (hostCode.cpp:770-789). Synchronises `stream` once. */
aarbf_status aarbf_build(aarbf_ctx *ctx, float rbf_radius, uint32_t particles_per_leaf, void *stream);
/* New radius / transfer functions, same particles: prepass + leaf bounds + refit
 * (replaces gprtAccelUpdate, hostCode.cpp:791-794). */
aarbf_status aarbf_refit(aarbf_ctx *ctx, float rbf_radius, void *stream);

/* A new frame of the same particle count (aarbf_set_particles, radii given iff the build had
 * them), same radius and transfer functions: the BVH keeps the topology of the last aarbf_build
 * and is refit to the new frame's leaves, as the reference refits on a frame change
 * (hostCode.cpp:751-794: the frame upload, GenRBFBounds and gprtAccelUpdate when the radius did
 * not change). keep_order = 0: the new frame is sorted along the Hilbert curve of the build's
 * space-time box, as the reference pre-sorts every frame (hostCode.cpp:195-222), and its leaves
 * refit the old topology; keep_order = 1: the frame's particles keep the previous frame's order
 * (particle i of every frame is the same particle), so nothing is sorted; aarbf_get_hilbert_keys
 * then still returns the keys of the last sort. Renders are bit-identical to a full aarbf_build
 * of the frame in either case (the sums are exact and the traversal only culls). A different
 * count or storage form returns AARBF_ERR_INVALID_ARGUMENT: call aarbf_build. Synchronises
 * `stream` once (root box read-back, and the tie check of the sort when keep_order = 0). */
aarbf_status aarbf_refit_frame(aarbf_ctx *ctx, int keep_order, void *stream);

/* ---- rendering --------------------------------------------------------------------------- */

/* ParticleRBFRayGen (deviceCodeRBF.hlsl:206-336) with the intersection/any-hit programs
 * (:338-389) fused in; replaces gprtRayGenLaunch2D(ParticleRBFRayGen) (hostCode.cpp:813).
 * accum is read-modify-written (running mean over accum_id), image receives the frame. */
aarbf_status aarbf_render(aarbf_ctx *ctx, const aarbf_params *p, int width, int height,
                          float *accum, float *image, void *stream);
/* aarbf_render plus accounting (no counterpart in the reference; for roofline figures).
 * counts has AARBF_COUNT_SLOTS entries: [0] particles whose sphere meets a traversed ray segment
 * (primary [start, termination] and shadow), [1] BVH nodes those segment queries visit, then the
 * kernel's own work: [2] tracking steps, [3] segment stagings, [4] staging overflows, [5] point
 * queries, [6] staged-candidate checks, [7] particle evaluations, [8] node visits while staging,
 * [9] node visits of point queries. The ray-per-warp kernels (AARBF_TRAVERSAL_AUTO) fill [2..9]
 * with their own work instead: [2] tentative steps, [3] segment stagings, [4] staging overflows,
 * [5] direct (unstaged) bin sums or point queries, [6] candidates staged, [7] bins and sub-bins
 * visited (majorant tracking), [8] warp traversal iterations, [9] particles tested by the
 * traversals. Count-mode launches use the timed instances' grid (their larger frames fit fewer
 * blocks per SM, so they run oversubscribed; work comes from an atomic counter either way).
 * Synchronises `stream`. */
#define AARBF_COUNT_SLOTS 10
aarbf_status aarbf_render_count(aarbf_ctx *ctx, const aarbf_params *p, int width, int height,
                                float *accum, float *image, uint64_t *counts, void *stream);
/* Kernel timing (no counterpart in the reference; for roofline figures). While enabled, every
 * aarbf_render records CUDA events on its stream around its two kernels: the tracking kernel
 * and the in-order accumulation pass. aarbf_get_kernel_times waits for the recorded events,
 * returns the summed milliseconds of each kernel and the number of renders timed, and clears
 * the record. */
aarbf_status aarbf_set_kernel_timing(aarbf_ctx *ctx, int enable);
aarbf_status aarbf_get_kernel_times(aarbf_ctx *ctx, double *render_ms, double *accumulate_ms,
                                    uint32_t *renders);
/* ---- FP16 storage form (no counterpart in the reference) -------------------------------- */

/* Storage of the scene the next aarbf_build makes. AARBF_STORAGE_FP16: positions as FP16
 * offsets from the centre of each run of 256 Hilbert-sorted particles (fp32 centre per run),
 * attribute and per-particle colour weights in FP16, radii fp32; the tracking kernels read the
 * packed records. Results are exact for the rounded scene (every kernel sees the same decoded
 * values); the rounding itself changes the image slightly. */
enum { AARBF_STORAGE_FP32 = 0, AARBF_STORAGE_FP16 = 1 };
aarbf_status aarbf_set_storage(aarbf_ctx *ctx, int format);

/* ---- batched rendering (no counterpart in the reference) -------------------------------- */

/* Many scenes, views and resolutions in one persistent launch of the ray-per-warp kernel plus
 * one accumulation launch. aarbf_batch_create binds nscenes contexts (each with its own built
 * scene and transfer functions, all on one device), their parameters (majorant tracking with
 * AARBF_TRAVERSAL_AUTO; per-scene frame, spp, camera, stage_bins), resolutions and caller-owned
 * framebuffers, reserves every scene's working memory and uploads the launch blocks
 * (synchronous). aarbf_batch_render then only enqueues the two kernels on `stream`: it allocates
 * nothing and does not synchronise, so it can be called repeatedly or captured; candidate_cap
 * (0, 256, 512, 1024) picks the staging-buffer depth. Results equal aarbf_render of each scene.
 * The batch holds its own per-sample colour planes, so one context may appear several times
 * (other views of the same scene) and may render on its own between batch renders. The
 * contexts must outlive the batch, and their scenes, transfer functions and noise atlases must
 * not be rebuilt or replaced while it is used. Up to 64 scenes run in one persistent launch;
 * larger batches take one launch per 64 scenes. */
typedef struct aarbf_batch aarbf_batch;
aarbf_status aarbf_batch_create(aarbf_batch **out, aarbf_ctx *const *ctxs, const aarbf_params *params,
                                int nscenes, const int *widths, const int *heights,
                                float *const *accums, float *const *images);
aarbf_status aarbf_batch_render(aarbf_batch *batch, int candidate_cap, void *stream);
/* Launch shape of the next aarbf_batch_render calls (tuning only: results are identical for every
 * shape). blocks_per_sm: resident blocks of four warps per SM (0 = as many as fit; 1..64 caps the
 * grid); sample_major: 1 hands out the work items sample by sample over all 8 x 4 pixel tiles,
 * 0 (default) tile by tile with a tile's samples in sequence. */
aarbf_status aarbf_batch_set_shape(aarbf_batch *batch, int blocks_per_sm, int sample_major);
aarbf_status aarbf_batch_destroy(aarbf_batch *batch);
const char *aarbf_batch_last_error(const aarbf_batch *batch);

/* ---- differentiable form (no counterpart in the reference) ------------------------------- */

/* Expected stochastic marching: the reference's stochasticMarching (deviceCodeRBF.hlsl:67-139)
 * with ambient 1 and its random stopping threshold integrated in closed form, with the
 * truncated Gaussian shifted to zero at the cut-off radius (continuous in positions and radii).
 * views: nviews parameter blocks (camera, unit, density_gain, aabb, rbf_radius as the box
 * padding, frame_id, spp; the same spp in every view; other fields ignored). images: device
 * float4 nviews x height x width, mean RGB over spp, alpha 1. Keeps a 16-byte checkpoint per
 * sample for aarbf_render_diff_backward. Needs a built scene whose radius map is all ones and
 * at most 2048 colour texels. Synchronises `stream` once (view upload). */
aarbf_status aarbf_render_diff_forward(aarbf_ctx *ctx, const aarbf_params *views, int nviews, int width,
                                       int height, float *images, void *stream);
/* Adjoint of the last aarbf_render_diff_forward (same views) by path replay. grad_images:
 * dL/dimages (device, same layout). Writes, in the caller's particle order: grad_xyz (n x 3),
 * grad_radius (n), grad_attr (n, the raw attribute: normalisation chained in), and grad_tf
 * (nc x 4, the RGBA colour table). Accumulation uses float atomics (summation order varies). */
aarbf_status aarbf_render_diff_backward(aarbf_ctx *ctx, const aarbf_params *views, int nviews, int width,
                                        int height, const float *grad_images, float *grad_xyz,
                                        float *grad_radius, float *grad_attr, float *grad_tf, void *stream);

/* ParticleSplatRayGen (deviceCodeSplat.hlsl:58-193); writes image only. One warp per pixel
 * (AARBF_TRAVERSAL_AUTO; the first call with a new `unit` uploads a table of slab starts and
 * synchronises `stream` once) or one thread per pixel (AARBF_TRAVERSAL_THREAD); identical bits. */
aarbf_status aarbf_render_splat(aarbf_ctx *ctx, const aarbf_params *p, int width, int height,
                                float *image, void *stream);
/* CompositeGui TAA resolve (deviceCodeCommon.hlsl:67-115). Writes taa unless disable; bgra
 * (optional) receives the BGRA8 frame. The reference's taa->taaPrev copy
 * (hostCode.cpp:829-830) is a pointer swap for the caller. ctx may be NULL. */
aarbf_status aarbf_taa_resolve(aarbf_ctx *ctx, const float *image, const float *taa_prev,
                               float *taa, uint32_t *bgra, int width, int height, int disable,
                               void *stream);
/* Device buffers owned by the context (GPRT device buffers, hostCode.cpp:314-322). */
aarbf_status aarbf_get_framebuffers(aarbf_ctx *ctx, int width, int height, float **accum,
                                    float **image);

/* Device buffers for callers without their own CUDA runtime: gprtDeviceBufferCreate /
 * gprtBufferDestroy (hostCode.cpp:314-325, :834-836). aarbf_memcpy copies between any mix of
 * host and device pointers on `stream` (replaces gprtBufferMap + memcpy, hostCode.cpp:759-763). */
aarbf_status aarbf_device_alloc(aarbf_ctx *ctx, size_t bytes, void **ptr);
aarbf_status aarbf_device_free(aarbf_ctx *ctx, void *ptr);
aarbf_status aarbf_memcpy(aarbf_ctx *ctx, void *dst, const void *src, size_t bytes, void *stream);
aarbf_status aarbf_memset(aarbf_ctx *ctx, void *dst, int value, size_t bytes, void *stream);

/* Blue-noise atlas for the marching mode: RGBA8, 8 x 16 tiles of 256 x 256 (stbn.png layout,
 * hostCode.cpp:337-352). NULL selects a generated substitute (aarbf_generate_noise_atlas: one
 * void-and-cluster blue-noise tile, frame f's tile offset by f times the golden-ratio conjugate
 * modulo 1; every tile holds each 8-bit value 256 times; the first call takes a few seconds of
 * host time, later calls reuse the tile). */
aarbf_status aarbf_set_noise_atlas(aarbf_ctx *ctx, const uint8_t *rgba8, int width, int height);
aarbf_status aarbf_generate_noise_atlas(uint8_t *rgba8_out, int width, int height);

/* ---- host helpers ------------------------------------------------------------------------ */

/* Camera basis of hostCode.cpp:669-676 (cos_fovy is the reference's --camera 10th value). */
aarbf_status aarbf_camera(const float *look_from, const float *look_at, const float *look_up,
                          float cos_fovy, int width, int height, float *pos, float *dir00,
                          float *du, float *dv);

/* importParticles (importParticles.h:8-31): header text file of timestep names, each
 * `path + "_" + name` holding u64 count + count float4. Unlike the reference every read is
 * checked. */
typedef struct aarbf_series aarbf_series;
aarbf_status aarbf_series_load(const char *path, aarbf_series **out);
aarbf_status aarbf_series_num_frames(const aarbf_series *s, uint64_t *frames);
aarbf_status aarbf_series_frame(const aarbf_series *s, uint64_t frame, const float **xyzw,
                                uint64_t *n);
aarbf_status aarbf_series_free(aarbf_series *s);
/* writer of the same format (names are "0", "1", ...) */
aarbf_status aarbf_series_save(const char *path, const float *const *frames, const uint64_t *counts,
                               uint64_t nframes);

/* ---- allocation-free Hilbert sort ---------------------------------------------------------- */

/* No counterpart in the reference. For callers that cannot allocate device memory -- device
 * memory handed out by the application's own pool or arena, which forbids other allocations,
 * real-time loops that must not reach the allocator (it can synchronise the device): the
 * Hilbert keys and sort permutation that aarbf_build computes, without calling cudaMalloc or
 * cudaFree. xyzw: device pointer to n float4 particles; dom: HOST pointer to the 8-float domain of aarbf_set_domain;
 * keys (n x u64) and perm (n x u32): device outputs, equal to aarbf_get_hilbert_keys' results.
 * Working space is a fixed array in device memory that every GPU loading the library holds
 * until the process exits (about 12.5 MiB), so n is limited to AARBF_NOALLOC_MAX_PARTICLES;
 * larger n returns AARBF_ERR_INVALID_ARGUMENT. All calls share that array: calls whose GPU work
 * overlaps (other streams, other host threads) race and must be ordered by the caller. The first
 * call on a device looks up the array's address; make it before any stream capture. That address
 * is cached for the life of the device's primary context: do not keep calling across a
 * cudaDeviceReset. Host pointers for xyzw, keys or perm are refused with
 * AARBF_ERR_INVALID_ARGUMENT before any GPU work. The call
 * synchronises `stream` once (to read the tie flag), like aarbf_build. */
#define AARBF_NOALLOC_MAX_PARTICLES (1u << 20)
aarbf_status aarbf_hilbert_sort_noalloc(const float *xyzw, uint64_t n, const float *dom,
                                        uint64_t *keys, uint32_t *perm, void *stream);

/* ---- debug getters (bit-exact tests) ------------------------------------------------------ */

aarbf_status aarbf_get_num_particles(const aarbf_ctx *ctx, uint64_t *n, uint32_t *num_leaves);
/* Hilbert keys (in sorted order) and the sort permutation (sorted -> input index) */
aarbf_status aarbf_get_hilbert_keys(aarbf_ctx *ctx, uint64_t *keys, uint32_t *perm);
/* sorted, normalised particles (float4 x n) */
aarbf_status aarbf_get_sorted_particles(aarbf_ctx *ctx, float *xyzw);
/* prepass records: rec0 = (x,y,z,r_eval) x n, w4 = (a^3, pow(rgb,2.2) a^3) x n, rgeom x n */
aarbf_status aarbf_get_prepass(aarbf_ctx *ctx, float *rec0, float *w4, float *rgeom);
/* BVH: child codes (bit31 = leaf) of the L-1 internal nodes, their traversal boxes (6 floats
 * each: lo xyz, hi xyz), the leaf boxes of the reference's bounds program (6 x L,
 * GenRBFBounds), the traversal leaf boxes (6 x L, particles that can be hit) and the root
 * traversal box (6) */
aarbf_status aarbf_get_bvh(aarbf_ctx *ctx, uint32_t *left, uint32_t *right, float *node_box,
                           float *leaf_box, float *leaf_eff, float *root_box);

#ifdef __cplusplus
}
#endif
#endif /* AARBF_H */
