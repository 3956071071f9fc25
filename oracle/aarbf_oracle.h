/*
 * aarbf_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's attribute-aware RBF particle-volume path
 * (gprt-org/attribute-aware-rbfs). It is the checker for the CUDA product path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 * Nothing in the product library includes, links or calls this code.
 *
 * Pinning: the Hilbert encoder and the RNG are pinned bit-for-bit against the
 * reference's own hilbert.h and rng.h compiled unchanged by oracle/Makefile
 * (oracle/_ref/libaarbf_ref.so) and against committed golden vectors in
 * tests/golden/. The renderer (the reference's HLSL) cannot be compiled here,
 * so its restatement is pinned by analytic known-answer tests only; where the
 * reference's result depends on the un-vendored GPRT runtime (texture sampler,
 * any-hit order, sort tie-break) the oracle fixes one documented model.
 */
#ifndef AARBF_ORACLE_H
#define AARBF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- deterministic float math (same operation sequence as the CUDA path) ---- */
float orc_logf(float x);
float orc_expf(float x);
float orc_powf(float x, float y);

/* ---- Hilbert curve (hilbert.h:16-88,124-166,181-225) ---- */
uint64_t orc_hilbert_c2i(unsigned nDims, unsigned nBits, const uint64_t *coord);
void orc_hilbert_i2c(unsigned nDims, unsigned nBits, uint64_t index, uint64_t *coord);

/* ---- RNG (rng.h:24-70) ---- */
uint32_t orc_murmur_mix(uint32_t hash, uint32_t k);
uint32_t orc_murmur_finalize(uint32_t hash);
uint32_t orc_get_rng(int frame_id, uint32_t px, uint32_t py, uint32_t dimx);
uint32_t orc_lcg_next(uint32_t *state);
float orc_lcg_randomf(uint32_t *state);

/* ---- host preprocessing (hostCode.cpp:183-250) ---- */
/* dom = {minx,miny,minz,maxx,maxy,maxz,attr_min,attr_max}; accumulates into dom. */
void orc_domain_accumulate(const float *xyzw, uint64_t n, float *dom);
void orc_domain_init(float *dom);
void orc_hilbert_keys(const float *xyzw, uint64_t n, const float *dom, uint64_t *keys);
/* order = stable sort by (key, x, y, z, w, original index) */
void orc_sort_perm(const uint64_t *keys, const float *xyzw, uint64_t n, uint32_t *perm);
void orc_gather_normalize(const float *xyzw, const float *radii, const uint32_t *perm, uint64_t n,
                          float attr_min, float attr_max, float *out_xyzw, float *out_radii);

/* ---- transfer functions (hostCode.cpp:355-365,524-572) ---- */
/* decode an RGBA8 texture of n texels; srgb!=0 decodes R,G,B (alpha stays linear) */
void orc_decode_rgba8(const uint8_t *rgba8, int n, int srgb, float *out4);
float orc_tex_sample(const float *tex, int n, int stride, int channel, float u);
uint8_t orc_make_8bit(float f);

/* ---- camera and light (hostCode.cpp:669-676, sharedCode.h:127-132) ---- */
void orc_camera(const float *look_from, const float *look_at, const float *look_up, float cos_fovy,
                int width, int height, float *pos, float *d00, float *du, float *dv);
void orc_light_dir(float azimuth, float elevation, float *dir);

/* ---- scene: prepass, leaf bounds, LBVH, refit ---- */
typedef struct orc_scene orc_scene;

typedef struct orc_tf_desc {
  const float *color; int nc;    /* RGBA table, nc texels */
  const float *radius; int nr;   /* R table */
  const float *density; int nd;  /* R table */
  float alpha_floor;             /* opacity below this counts as transparent (0: only alpha == 0) */
  int storage_fp16;              /* scene option: positions (relative to the centre of each run of
                                    256 sorted particles), attributes and the per-particle weights
                                    a^3, rgb^2.2 a^3 are rounded to FP16 */
} orc_tf_desc;

/* IEEE binary16 conversions: round to nearest even, and exact widening */
uint16_t orc_f2h(float f);
float orc_h2f(uint16_t h);

/* xyzw: Hilbert-sorted particles with normalised attribute; radii may be NULL.
 * keys: Hilbert keys of the sorted particles. */
orc_scene *orc_scene_create(const float *xyzw, const float *radii, const uint64_t *keys, uint64_t n,
                            uint32_t ppl, float rbf_radius, const orc_tf_desc *tf);
void orc_scene_destroy(orc_scene *s);
uint32_t orc_scene_num_leaves(const orc_scene *s);
/* copies out the BVH: left/right child codes (bit31 = leaf), internal boxes (6 floats each;
 * unions of the traversal leaf boxes), leaf boxes of the reference's bounds program, traversal
 * leaf boxes (particles that can be hit), root box (6 floats) */
void orc_scene_get_bvh(const orc_scene *s, uint32_t *left, uint32_t *right, float *node_box,
                       float *leaf_box, float *leaf_eff, float *root_box);
void orc_scene_get_prepass(const orc_scene *s, float *rec0, float *w4, float *rgeom);
/* the scene's sorted particles as rendered (after FP16 rounding in the FP16 storage form) */
void orc_scene_get_particles(const orc_scene *s, float *xyzw);

/* point query at x: returns hit count; acc = {D, R, G, B} fixed point (2^-40 units) */
int orc_point_query(const orc_scene *s, const float *x, int64_t *acc);
int orc_point_query_brute(const orc_scene *s, const float *x, int64_t *acc);

/* ---- render parameters (PushConstants sharedCode.h:33-74 + RayGenData :108-117) ---- */
enum {
  ORC_FLAG_BLUE_NOISE = 1u << 0,          /* enableBlueNoise: stochastic marching */
  ORC_FLAG_SHOW_NOISE = 1u << 1,          /* showNoise */
  ORC_FLAG_VISUALIZE_ATTRIBUTES = 1u << 2,/* visualizeAttributes */
  ORC_FLAG_TRACK_FROM_ENTRY = 1u << 3,    /* native: tracking starts at tenter+unit*xi_y */
  ORC_FLAG_DENSITY_LINEAR = 1u << 4,      /* native: density = min(D*gain, 1) */
  ORC_FLAG_SPLAT_PARTICLE_RADIUS = 1u << 5,/* native: splat uses per-particle radius */
  ORC_FLAG_MAJORANT_TRACKING = 1u << 6    /* native: delta tracking with per-bin majorants */
};

typedef struct orc_params {
  uint32_t accum_id;
  uint32_t frame_id;
  uint32_t spp;
  uint32_t flags;
  float light_azimuth, light_elevation, light_ambient;
  float cam_pos[3], cam_dir00[3], cam_du[3], cam_dv[3];
  float rbf_radius;
  float unit;
  float aabb_min[3], aabb_max[3];
  float density_gain;
  float jitter_x, jitter_y;
  float density_scale; /* majorant tracking: extinction = density_scale * D per unit length */
  float bin_length;    /* majorant tracking: length of the majorant bins along a ray */
  const uint8_t *noise; /* RGBA8 atlas of 8x16 tiles of 256x256 (blue-noise mode) */
  int noise_w, noise_h;
} orc_params;

/* accum/image: float4 per pixel; accum is read-modify-write as in deviceCodeRBF.hlsl:326-335 */
void orc_render(const orc_scene *s, const orc_params *p, int w, int h, float *accum, float *image,
                int nthreads);
/* render only rows [y0,y1) x cols [x0,x1) (bounded CPU-baseline samples) */
void orc_render_region(const orc_scene *s, const orc_params *p, int w, int h, int x0, int x1,
                       int y0, int y1, float *accum, float *image, int nthreads);
/* the same, plus per pixel (w x h, written inside the region) the smallest relative gap
 * |a - b| / |b| between the two sides of any random decision its samples took (the collision
 * test, the marching threshold, the shadow opacity cap): a pixel whose gap is tiny can change
 * with the rounding of the reference's float any-hit sums, whose order the hardware decides */
void orc_render_region_gaps(const orc_scene *s, const orc_params *p, int w, int h, int x0, int x1,
                            int y0, int y1, float *accum, float *image, float *gaps, int nthreads);
void orc_render_splat(const orc_scene *s, const orc_params *p, int w, int h, float *image,
                      int nthreads);
/* CompositeGui TAA (deviceCodeCommon.hlsl:67-115); bgra may be NULL */
void orc_taa(const float *image, const float *prev, float *taa, uint32_t *bgra, int w, int h,
             int disable);

/* FP64 twin of the native-mode volume model (converged reference images): mean RGB over spp
 * samples of pixels [x0,x1) x [y0,y1) of a w x h frame, rgb_out 3 floats per pixel, row-major
 * over the region. clamp_plain: extinction min(density_scale D, 1/unit) of the plain native
 * estimator instead of density_scale D. Independent random stream (seed). */
void orc_render_f64(const orc_scene *s, const orc_params *p, int w, int h, int x0, int x1, int y0,
                    int y1, int spp, int clamp_plain, uint64_t seed, float *rgb_out, int nthreads);

/* Differentiable form (expected stochastic marching, ambient 1), double precision, brute-force
 * candidate search: particles by position (3n), radius, attribute in [0, 1], and an RGBA
 * transfer function of nc texels. images: nviews x h x w x 3. The backward takes dL/dimage of
 * the same shape and writes dL/d(position, radius, attribute, transfer function). Each view's
 * params give camera, unit, density_gain, aabb, rbf_radius (box padding), frame_id and spp. */
typedef struct orc_diff_scene {
  const double *pos, *radius, *attr, *tf;
  int n, nc;
} orc_diff_scene;
double orc_diff_forward(const orc_diff_scene *sc, const orc_params *views, int nviews, int w, int h,
                        double *images, int nthreads);
void orc_diff_backward(const orc_diff_scene *sc, const orc_params *views, int nviews, int w, int h,
                       const double *grad_images, double *g_pos, double *g_radius, double *g_attr,
                       double *g_tf, int nthreads);

/* per-pixel statistics of the last orc_render call on this thread (steps, queries) */
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
