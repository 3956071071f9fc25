/*
 * aarbf_oracle.c -- TEST INFRASTRUCTURE ONLY (see aarbf_oracle.h).
 *
 * A plain-C restatement of the reference's particle-volume path, written from the
 * reference's semantics. Each function cites the reference file:line it restates.
 * Compiled with -ffp-contract=off: every float operation below is one IEEE
 * round-to-nearest operation, fmaf() is written out where a fused step is meant.
 *
 * Parity model fixed here (the reference leaves these to the un-vendored GPRT runtime
 * or to hardware; the CUDA path makes the same choices):
 *   - exp/log/pow: Cody-Waite reduction + Taylor / atanh series (orc_expf/orc_logf);
 *   - textures: linear filter at texel centres, clamp-to-edge, sRGB decode of R,G,B;
 *   - any-hit accumulation: exact fixed-point sums (2^-40 units), order independent;
 *   - sort ties: (key, x, y, z, w, original index);
 *   - splat: the 15 kept samples of a slab are the 15 smallest (t, index).
 */
#include "aarbf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_DEPTH 10000 /* sharedCode.h:27 */
#define ORC_FIX_SCALE 0x1p40f
#define ORC_FIX_INV 0x1p-40f
#define ORC_LEAF_BIT 0x80000000u

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }

/* ------------------------------------------------------------------------------------------ */
/* deterministic math                                                                          */
/* ------------------------------------------------------------------------------------------ */

/* ln 2 split so that k*LN2_HI is exact for |k| < 2^8 (16 significant bits in LN2_HI). */
static const float LN2_HI = 0x1.62e4p-1f;
static const float LN2_LO = 0x1.7f7d1cp-20f;
static const float INV_LN2 = 0x1.715476p+0f;
static const float SQRT2F = 0x1.6a09e6p+0f;

static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline float pow2i(int k) { return u2f((uint32_t)(k + 127) << 23); } /* -126 <= k <= 127 */

/* natural log: x = m * 2^e with m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(s), s=(m-1)/(m+1),
 * atanh by its Taylor series through s^9. */
float orc_logf(float x) {
  if (x != x || x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (x == INFINITY) return INFINITY;
  int e = 0;
  uint32_t b = f2u(x);
  if (b < 0x00800000u) { x = x * 0x1p23f; b = f2u(x); e = -23; }
  e += (int)(b >> 23) - 127;
  float m = u2f((b & 0x007fffffu) | 0x3f800000u);
  if (m > SQRT2F) { m = m * 0.5f; e += 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float z = s * s;
  float p = 0x1.c71c72p-3f;          /* 2/9 */
  p = fmaf(p, z, 0x1.24924ap-2f);   /* 2/7 */
  p = fmaf(p, z, 0x1.99999ap-2f);   /* 2/5 */
  p = fmaf(p, z, 0x1.555556p-1f);   /* 2/3 */
  p = fmaf(p, z, 2.0f);
  float lm = s * p;
  float ef = (float)e;
  return fmaf(ef, LN2_HI, fmaf(ef, LN2_LO, lm));
}

/* exp: k = rint(x/ln2), r = x - k ln2 (two fused steps), Taylor series through r^7,
 * scaled by 2^k in two exact power-of-two multiplies (one rounding for subnormals). */
float orc_expf(float x) {
  if (x != x) return x;
  if (x > 88.72284f) return INFINITY;
  if (x < -103.972084f) return 0.0f;
  float kf = rintf(x * INV_LN2);
  float r = fmaf(-kf, LN2_HI, x);
  r = fmaf(-kf, LN2_LO, r);
  float p = 0x1.a01a02p-13f;        /* 1/5040 */
  p = fmaf(p, r, 0x1.6c16c2p-10f);  /* 1/720 */
  p = fmaf(p, r, 0x1.111112p-7f);   /* 1/120 */
  p = fmaf(p, r, 0x1.555556p-5f);   /* 1/24 */
  p = fmaf(p, r, 0x1.555556p-3f);   /* 1/6 */
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  int k = (int)kf;
  int k1 = k / 2;
  int k2 = k - k1;
  return (p * pow2i(k1)) * pow2i(k2);
}

/* pow for x >= 0 as used by the shaders (colour gamma 2.2 and 1/2.2) */
float orc_powf(float x, float y) {
  if (x != x || y != y) return NAN;
  if (x == 0.0f) return (y > 0.0f) ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
  if (x < 0.0f) return NAN;
  return orc_expf(y * orc_logf(x));
}

static inline float orc_minf(float a, float b) { return fminf(a, b); }
static inline float orc_maxf(float a, float b) { return fmaxf(a, b); }

/* ------------------------------------------------------------------------------------------ */
/* Hilbert curve: restates hilbert.h hilbert_c2i (181-225) and hilbert_i2c (124-166),          */
/* with the bit transpose (37-88) written as an explicit bit loop.                             */
/* ------------------------------------------------------------------------------------------ */

static inline uint64_t ones64(unsigned k) { return k >= 64 ? ~0ull : ((1ull << k) - 1ull); }

static inline uint64_t rot_right(uint64_t v, unsigned n, unsigned w) {
  return ((v >> n) | (v << (w - n))) & ones64(w);
}
static inline uint64_t rot_left(uint64_t v, unsigned n, unsigned w) {
  return ((v << n) | (v >> (w - n))) & ones64(w);
}

/* rotation bookkeeping of hilbert.h:16-24: advance by 1 + index of the lowest set bit of the
 * digit when that bit lies below the top axis, modulo nDims */
static inline unsigned next_rotation(unsigned rotation, unsigned nDims, uint64_t digit) {
  uint64_t low = digit & (~digit + 1ull) & (ones64(nDims) >> 1);
  while (low) { low >>= 1; ++rotation; }
  ++rotation;
  if (rotation >= nDims) rotation -= nDims;
  return rotation;
}

uint64_t orc_hilbert_c2i(unsigned nDims, unsigned nBits, const uint64_t *coord) {
  if (nDims <= 1) return coord[0];
  const unsigned total = nDims * nBits;
  /* OR-packing: field d at bits [d*nBits, (d+1)*nBits); a coordinate equal to 2^nBits spills
   * its top bit into field d+1 exactly as the reference packing does (hilbert.h:189-193) */
  uint64_t packed = 0;
  for (int d = (int)nDims - 1; d >= 0; --d) packed = (packed << nBits) | coord[d];
  uint64_t index;
  if (nBits > 1) {
    uint64_t inter = 0;
    for (unsigned d = 0; d < nDims; ++d) {
      uint64_t field = (d * nBits < 64) ? ((packed >> (d * nBits)) & ones64(nBits)) : 0;
      for (unsigned b = 0; b < nBits; ++b)
        inter |= ((field >> b) & 1ull) << (b * nDims + d);
    }
    inter ^= inter >> nDims;
    index = 0;
    unsigned rotation = 0;
    uint64_t flip = 0;
    for (int b = (int)total - (int)nDims; b >= 0; b -= (int)nDims) {
      uint64_t digit = (inter >> b) & ones64(nDims);
      digit = rot_right(flip ^ digit, rotation, nDims);
      index = (index << nDims) | digit;
      flip = 1ull << rotation;
      rotation = next_rotation(rotation, nDims, digit);
    }
    index ^= (ones64(total) / ones64(nDims)) >> 1;
  } else {
    index = packed;
  }
  for (unsigned d = 1; d < total; d *= 2) index ^= index >> d;
  return index;
}

void orc_hilbert_i2c(unsigned nDims, unsigned nBits, uint64_t index, uint64_t *coord) {
  if (nDims <= 1) { coord[0] = index; return; }
  const unsigned total = nDims * nBits;
  uint64_t coords;
  if (nBits > 1) {
    const uint64_t nth = ones64(total) / ones64(nDims);
    index ^= (index ^ nth) >> 1;
    uint64_t inter = 0;
    unsigned rotation = 0;
    uint64_t flip = 0;
    for (int b = (int)total - (int)nDims; b >= 0; b -= (int)nDims) {
      uint64_t digit = (index >> b) & ones64(nDims);
      inter = (inter << nDims) | (rot_left(digit, rotation, nDims) ^ flip);
      flip = 1ull << rotation;
      rotation = next_rotation(rotation, nDims, digit);
    }
    for (unsigned b = nDims; b < total; b *= 2) inter ^= inter >> b;
    coords = 0;
    for (unsigned d = 0; d < nDims; ++d)
      for (unsigned b = 0; b < nBits; ++b)
        coords |= ((inter >> (b * nDims + d)) & 1ull) << (d * nBits + b);
  } else {
    coords = index ^ (index >> 1);
  }
  for (unsigned d = 0; d < nDims; ++d) {
    coord[d] = coords & ones64(nBits);
    coords >>= nBits;
  }
}

/* ------------------------------------------------------------------------------------------ */
/* RNG: rng.h:24-70                                                                            */
/* ------------------------------------------------------------------------------------------ */

static inline uint32_t rotl32(uint32_t v, unsigned r) { return (v << r) | (v >> (32u - r)); }

uint32_t orc_murmur_mix(uint32_t hash, uint32_t k) {
  k *= 0xcc9e2d51u;
  k = rotl32(k, 15);
  k *= 0x1b873593u;
  hash ^= k;
  return rotl32(hash, 13) * 5u + 0xe6546b64u;
}

uint32_t orc_murmur_finalize(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

uint32_t orc_get_rng(int frame_id, uint32_t px, uint32_t py, uint32_t dimx) {
  uint32_t s = orc_murmur_mix(0u, px + py * dimx);
  s = orc_murmur_mix(s, (uint32_t)frame_id);
  return orc_murmur_finalize(s);
}

uint32_t orc_lcg_next(uint32_t *state) {
  *state = *state * 1664525u + 1013904223u;
  return *state;
}

/* ldexp((float)u, -32): the u32 -> float conversion rounds, the scaling is exact */
float orc_lcg_randomf(uint32_t *state) { return (float)orc_lcg_next(state) * 0x1p-32f; }

/* ------------------------------------------------------------------------------------------ */
/* host preprocessing: hostCode.cpp:183-250                                                    */
/* ------------------------------------------------------------------------------------------ */

void orc_domain_init(float *dom) {
  /* hostCode.cpp:183 starts from +-1e38; attribute range from +-1e20 (:227-228) */
  dom[0] = dom[1] = dom[2] = 1e38f;
  dom[3] = dom[4] = dom[5] = -1e38f;
  dom[6] = 1e20f;
  dom[7] = -1e20f;
}

void orc_domain_accumulate(const float *p, uint64_t n, float *dom) {
  for (uint64_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) {
      dom[a] = orc_minf(dom[a], p[4 * i + a]);
      dom[3 + a] = orc_maxf(dom[3 + a], p[4 * i + a]);
    }
    dom[6] = orc_minf(dom[6], p[4 * i + 3]);
    dom[7] = orc_maxf(dom[7], p[4 * i + 3]);
  }
}

/* quantise to 16 bits per axis, (p-min)/(max-min)*65536 truncated (hostCode.cpp:200-206).
 * A degenerate axis (max == min) and coordinates outside the domain are clamped to [0, 65536]
 * (the reference leaves both undefined). */
static inline uint64_t quantise16(float v, float lo, float hi) {
  float t = (v - lo) / (hi - lo);
  t = t * 65536.0f;
  if (!(t >= 0.0f)) return 0;
  if (t >= 65536.0f) return 65536;
  return (uint64_t)t;
}

void orc_hilbert_keys(const float *p, uint64_t n, const float *dom, uint64_t *keys) {
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t c[3];
    for (int a = 0; a < 3; ++a) c[a] = quantise16(p[4 * i + a], dom[a], dom[3 + a]);
    keys[i] = orc_hilbert_c2i(3, 16, c);
  }
}

/* total order used for the Hilbert sort: key, then x, y, z, w compared as floats, then index */
static const uint64_t *g_sort_keys;
static const float *g_sort_p;
static int cmp_perm(const void *a, const void *b) {
  uint32_t i = *(const uint32_t *)a, j = *(const uint32_t *)b;
  if (g_sort_keys[i] != g_sort_keys[j]) return g_sort_keys[i] < g_sort_keys[j] ? -1 : 1;
  for (int c = 0; c < 4; ++c) {
    float x = g_sort_p[4 * (uint64_t)i + c], y = g_sort_p[4 * (uint64_t)j + c];
    if (x < y) return -1;
    if (y < x) return 1;
  }
  return (i < j) ? -1 : (i > j ? 1 : 0);
}

void orc_sort_perm(const uint64_t *keys, const float *p, uint64_t n, uint32_t *perm) {
  for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
  g_sort_keys = keys;
  g_sort_p = p;
  qsort(perm, (size_t)n, sizeof(uint32_t), cmp_perm);
}

void orc_gather_normalize(const float *p, const float *radii, const uint32_t *perm, uint64_t n,
                          float amin, float amax, float *out, float *out_r) {
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t s = perm[i];
    out[4 * i + 0] = p[4 * s + 0];
    out[4 * i + 1] = p[4 * s + 1];
    out[4 * i + 2] = p[4 * s + 2];
    float w = p[4 * s + 3];
    if (amax > amin) w = (w - amin) / (amax - amin); /* hostCode.cpp:243-250 */
    out[4 * i + 3] = w;
    if (radii && out_r) out_r[i] = radii[s];
  }
}

/* ------------------------------------------------------------------------------------------ */
/* transfer functions                                                                          */
/* ------------------------------------------------------------------------------------------ */

/* hostCode.cpp:524-526 */
uint8_t orc_make_8bit(float f) {
  int v = (int)(f * 256.0f);
  if (v < 0) v = 0;
  if (v > 255) v = 255;
  return (uint8_t)v;
}

static float srgb_decode8(uint8_t v) {
  double c = (double)v / 255.0;
  double l = (c <= 0.04045) ? c / 12.92 : pow((c + 0.055) / 1.055, 2.4);
  return (float)l;
}

/* R8G8B8A8_SRGB textures (hostCode.cpp:355-365): R,G,B decoded, alpha linear */
void orc_decode_rgba8(const uint8_t *t, int n, int srgb, float *out) {
  for (int i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c)
      out[4 * i + c] = srgb ? srgb_decode8(t[4 * i + c]) : (float)((double)t[4 * i + c] / 255.0);
    out[4 * i + 3] = (float)((double)t[4 * i + 3] / 255.0);
  }
}

/* SampleGrad with zero gradients: linear filter between texel centres, clamp to edge */
float orc_tex_sample(const float *tex, int n, int stride, int channel, float u) {
  float f = u * (float)n - 0.5f;
  if (!(f > -1.0f)) f = -1.0f;
  if (f > (float)n) f = (float)n;
  float fl = floorf(f);
  float a = f - fl;
  int i0 = (int)fl;
  int i1 = i0 + 1;
  if (i0 < 0) i0 = 0;
  if (i0 > n - 1) i0 = n - 1;
  if (i1 < 0) i1 = 0;
  if (i1 > n - 1) i1 = n - 1;
  float v0 = tex[i0 * stride + channel];
  float v1 = tex[i1 * stride + channel];
  return v0 + a * (v1 - v0);
}

/* ------------------------------------------------------------------------------------------ */
/* camera (hostCode.cpp:669-676) and light (sharedCode.h:127-132)                               */
/* ------------------------------------------------------------------------------------------ */

static void v3_normalize(const float *a, float *o) {
  float len = sqrtf((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2]);
  o[0] = a[0] / len;
  o[1] = a[1] / len;
  o[2] = a[2] / len;
}
static void v3_cross(const float *a, const float *b, float *o) {
  float x = a[1] * b[2] - a[2] * b[1];
  float y = a[2] * b[0] - a[0] * b[2];
  float z = a[0] * b[1] - a[1] * b[0];
  o[0] = x; o[1] = y; o[2] = z;
}

void orc_camera(const float *from, const float *at, const float *up, float cos_fovy, int width,
                int height, float *pos, float *d00, float *du, float *dv) {
  float diff[3] = {at[0] - from[0], at[1] - from[1], at[2] - from[2]};
  float dir[3], c[3], n[3];
  v3_normalize(diff, dir);
  float aspect = (float)width / (float)height;
  v3_cross(dir, up, c);
  v3_normalize(c, n);
  float su = cos_fovy * aspect;
  float ddu[3] = {su * n[0], su * n[1], su * n[2]};
  v3_cross(ddu, dir, c);
  v3_normalize(c, n);
  float ddv[3] = {cos_fovy * n[0], cos_fovy * n[1], cos_fovy * n[2]};
  for (int a = 0; a < 3; ++a) {
    float d = dir[a] - 0.5f * ddu[a];
    d = d - 0.5f * ddv[a];
    pos[a] = from[a];
    d00[a] = d;
    du[a] = ddu[a];
    dv[a] = ddv[a];
  }
}

void orc_light_dir(float az, float el, float *dir) {
  float a = el * 3.14f - 0.5f * 3.14f;
  float b = (az * 2.0f) * 3.14f;
  float s = sinf(a);
  dir[0] = s * cosf(b);
  dir[1] = s * sinf(b);
  dir[2] = cosf(a);
}

/* ------------------------------------------------------------------------------------------ */
/* scene: per-particle prepass, leaf bounds (deviceCodeBounds.hlsl:29-82), Karras LBVH, refit  */
/* ------------------------------------------------------------------------------------------ */

struct orc_scene {
  uint64_t n;
  uint32_t ppl, nleaves;
  float rbf_radius;
  float *xyzw;     /* 4n sorted particles (attribute normalised) */
  float *rec0;     /* 4n: x, y, z, r_eval (0 when the particle can never be hit) */
  float *w4;       /* 4n: alpha^3, pow(r,2.2) a^3, pow(g,2.2) a^3, pow(b,2.2) a^3 */
  float *rgeom;    /* n: bounds radius, -1 when radiusmap == 0 (skipped by the bounds program) */
  uint64_t *leaf_key;
  float *leaf_box; /* 6 per leaf: the reference's bounds program (radius from radiusmap) */
  float *leaf_eff; /* 6 per leaf: traversal box from r_eval (particles that can be hit) */
  uint32_t *left, *right;
  float *node_box; /* 6 per internal node (union of leaf_eff) */
  float root_box[6];
  uint32_t root;   /* child code of the root */
  /* transfer functions for rendering */
  float *color; int nc;
  float *density; int nd;
};

static float *dupf(const float *src, size_t cnt) {
  float *d = (float *)malloc(cnt * sizeof(float));
  memcpy(d, src, cnt * sizeof(float));
  return d;
}

/* ---- FP16 storage form (no counterpart in the reference) ---------------------------------- */

uint16_t orc_f2h(float f) {
  uint32_t x = f2u(f);
  uint32_t sign = (x >> 16) & 0x8000u, ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return (uint16_t)(sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u));
  if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u); /* >= 65520 rounds to infinity */
  if (ax <= 0x33000000u) return (uint16_t)sign;            /* <= 2^-25 rounds to zero (tie to even) */
  int e = (int)(ax >> 23) - 127;
  uint32_t mant = (ax & 0x7fffffu) | 0x800000u;
  int shift = e < -14 ? -e - 1 : 13; /* bits dropped: subnormal results keep fewer */
  uint32_t q = mant >> shift, rem = mant & ((1u << shift) - 1u), halfway = 1u << (shift - 1);
  if (rem > halfway || (rem == halfway && (q & 1u))) ++q;
  if (e < -14) return (uint16_t)(sign | q); /* q == 0x400 is the smallest normal, encoded alike */
  return (uint16_t)(sign | (((uint32_t)(e + 15) << 10) + (q - 0x400u)));
}

float orc_h2f(uint16_t h) {
  uint32_t sign = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
  if (e == 0x1f) return u2f(sign | 0x7f800000u | (m << 13));
  if (e == 0) {
    float v = (float)m * 0x1p-24f; /* exact */
    return sign ? -v : v;
  }
  return u2f(sign | ((e + 112u) << 23) | (m << 13));
}

#define ORC_FP16_RUN 256 /* particles sharing one fp32 origin */

/* positions relative to the centre of their run's bounding box, and the attribute, through FP16 */
static void quantize_positions(orc_scene *s) {
  for (uint64_t b = 0; b < s->n; b += ORC_FP16_RUN) {
    uint64_t e = b + ORC_FP16_RUN < s->n ? b + ORC_FP16_RUN : s->n;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint64_t i = b; i < e; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[a] = fminf(lo[a], s->xyzw[4 * i + a]);
        hi[a] = fmaxf(hi[a], s->xyzw[4 * i + a]);
      }
    float o[3];
    for (int a = 0; a < 3; ++a) o[a] = (lo[a] + hi[a]) * 0.5f;
    for (uint64_t i = b; i < e; ++i) {
      for (int a = 0; a < 3; ++a) s->xyzw[4 * i + a] = o[a] + orc_h2f(orc_f2h(s->xyzw[4 * i + a] - o[a]));
      s->xyzw[4 * i + 3] = orc_h2f(orc_f2h(s->xyzw[4 * i + 3]));
    }
  }
}

static void quantize_weights(orc_scene *s) {
  for (uint64_t i = 0; i < 4 * s->n; ++i) s->w4[i] = orc_h2f(orc_f2h(s->w4[i]));
}

/* deviceCodeRBF.hlsl:349-351 (radius), :366-376 (colour weights), deviceCodeBounds.hlsl:59-65 */
static void prepass(orc_scene *s, const float *radii, const orc_tf_desc *tf) {
  for (uint64_t i = 0; i < s->n; ++i) {
    const float *p = s->xyzw + 4 * i;
    float w = p[3];
    float rp = orc_tex_sample(tf->radius, tf->nr, 1, 0, w);
    float base = radii ? radii[i] : s->rbf_radius;
    float r = base * rp;
    float col[4];
    for (int c = 0; c < 4; ++c) col[c] = orc_tex_sample(tf->color, tf->nc, 4, c, w);
    s->rgeom[i] = (rp == 0.0f) ? -1.0f : r;
    s->rec0[4 * i + 0] = p[0];
    s->rec0[4 * i + 1] = p[1];
    s->rec0[4 * i + 2] = p[2];
    float a = col[3];
    if (a == 0.0f || a < tf->alpha_floor) { /* transparent: ignored by the any-hit program */
      s->rec0[4 * i + 3] = 0.0f;
      s->w4[4 * i + 0] = s->w4[4 * i + 1] = s->w4[4 * i + 2] = s->w4[4 * i + 3] = 0.0f;
    } else {
      float a3 = (a * a) * a;
      s->rec0[4 * i + 3] = r;
      s->w4[4 * i + 0] = a3;
      for (int c = 0; c < 3; ++c) s->w4[4 * i + 1 + c] = orc_powf(col[c], 2.2f) * a3;
    }
  }
}

static void leaf_bounds(orc_scene *s) {
  for (uint32_t l = 0; l < s->nleaves; ++l) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t k = 0; k < s->ppl; ++k) {
      uint64_t i = (uint64_t)l * s->ppl + k;
      if (i >= s->n) break;
      float r = s->rgeom[i];
      if (r < 0.0f) continue; /* radiusPercent == 0 */
      for (int a = 0; a < 3; ++a) {
        float c = s->rec0[4 * i + a];
        lo[a] = orc_minf(lo[a], c - r);
        hi[a] = orc_maxf(hi[a], c + r);
      }
    }
    int empty = (lo[0] > hi[0]) || (lo[1] > hi[1]) || (lo[2] > hi[2]);
    for (int a = 0; a < 3; ++a) {
      s->leaf_box[6 * l + a] = empty ? NAN : lo[a];
      s->leaf_box[6 * l + 3 + a] = empty ? NAN : hi[a];
    }
    /* traversal box: the particles that can be hit, p +- r_eval */
    float el[3] = {INFINITY, INFINITY, INFINITY}, eh[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t k = 0; k < s->ppl; ++k) {
      uint64_t i = (uint64_t)l * s->ppl + k;
      if (i >= s->n) break;
      float r = s->rec0[4 * i + 3];
      if (!(r > 0.0f)) continue;
      for (int a = 0; a < 3; ++a) {
        float c = s->rec0[4 * i + a];
        el[a] = orc_minf(el[a], c - r);
        eh[a] = orc_maxf(eh[a], c + r);
      }
    }
    empty = (el[0] > eh[0]) || (el[1] > eh[1]) || (el[2] > eh[2]);
    for (int a = 0; a < 3; ++a) {
      s->leaf_eff[6 * l + a] = empty ? NAN : el[a];
      s->leaf_eff[6 * l + 3 + a] = empty ? NAN : eh[a];
    }
  }
}

/* Karras (HPG 2012) radix tree over leaf keys; equal keys are ordered by leaf index */
static int delta(const uint64_t *k, int64_t L, int64_t i, int64_t j) {
  if (j < 0 || j >= L) return -1;
  uint64_t x = k[i] ^ k[j];
  if (x == 0) return 64 + __builtin_clz((uint32_t)(i ^ j));
  return __builtin_clzll(x);
}

static void karras(orc_scene *s) {
  const int64_t L = s->nleaves;
  const uint64_t *k = s->leaf_key;
  for (int64_t i = 0; i < L - 1; ++i) {
    int d = (delta(k, L, i, i + 1) - delta(k, L, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(k, L, i, i - d);
    int64_t lmax = 2;
    while (delta(k, L, i, i + lmax * d) > dmin) lmax *= 2;
    int64_t l = 0;
    for (int64_t t = lmax / 2; t >= 1; t /= 2)
      if (delta(k, L, i, i + (l + t) * d) > dmin) l += t;
    int64_t j = i + l * d;
    int dnode = delta(k, L, i, j);
    int64_t sp = 0, step = l;
    do {
      step = (step + 1) >> 1;
      if (delta(k, L, i, i + (sp + step) * d) > dnode) sp += step;
    } while (step > 1);
    int64_t g = i + sp * d + (d < 0 ? -1 : 0);
    int64_t lo = i < j ? i : j, hi = i < j ? j : i;
    s->left[i] = (lo == g) ? ((uint32_t)g | ORC_LEAF_BIT) : (uint32_t)g;
    s->right[i] = (hi == g + 1) ? ((uint32_t)(g + 1) | ORC_LEAF_BIT) : (uint32_t)(g + 1);
  }
}

static const float *child_box(const orc_scene *s, uint32_t c) {
  return (c & ORC_LEAF_BIT) ? s->leaf_eff + 6 * (c & ~ORC_LEAF_BIT) : s->node_box + 6 * c;
}

static void refit_node(orc_scene *s, uint32_t node) {
  /* post-order over the internal nodes; explicit stack */
  uint32_t *stack = (uint32_t *)malloc(sizeof(uint32_t) * 2 * (s->nleaves + 1));
  uint8_t *state = (uint8_t *)calloc(s->nleaves, 1);
  int sp = 0;
  stack[sp++] = node;
  while (sp) {
    uint32_t nd = stack[sp - 1];
    if (!state[nd]) {
      state[nd] = 1;
      if (!(s->left[nd] & ORC_LEAF_BIT)) stack[sp++] = s->left[nd];
      if (!(s->right[nd] & ORC_LEAF_BIT)) stack[sp++] = s->right[nd];
      continue;
    }
    --sp;
    const float *a = child_box(s, s->left[nd]);
    const float *b = child_box(s, s->right[nd]);
    for (int c = 0; c < 3; ++c) {
      s->node_box[6 * nd + c] = orc_minf(a[c], b[c]);
      s->node_box[6 * nd + 3 + c] = orc_maxf(a[3 + c], b[3 + c]);
    }
  }
  free(stack);
  free(state);
}

orc_scene *orc_scene_create(const float *xyzw, const float *radii, const uint64_t *keys, uint64_t n,
                            uint32_t ppl, float rbf_radius, const orc_tf_desc *tf) {
  orc_scene *s = (orc_scene *)calloc(1, sizeof(orc_scene));
  s->n = n;
  s->ppl = ppl ? ppl : 1;
  s->rbf_radius = rbf_radius;
  s->nleaves = (uint32_t)((n + s->ppl - 1) / s->ppl);
  size_t nn = n ? n : 1, nl = s->nleaves ? s->nleaves : 1;
  s->xyzw = dupf(xyzw ? xyzw : (const float[4]){0, 0, 0, 0}, n ? 4 * n : 4);
  s->rec0 = (float *)calloc(4 * nn, sizeof(float));
  s->w4 = (float *)calloc(4 * nn, sizeof(float));
  s->rgeom = (float *)calloc(nn, sizeof(float));
  s->leaf_key = (uint64_t *)calloc(nl, sizeof(uint64_t));
  s->leaf_box = (float *)calloc(6 * nl, sizeof(float));
  s->leaf_eff = (float *)calloc(6 * nl, sizeof(float));
  s->left = (uint32_t *)calloc(nl, sizeof(uint32_t));
  s->right = (uint32_t *)calloc(nl, sizeof(uint32_t));
  s->node_box = (float *)calloc(6 * nl, sizeof(float));
  s->color = dupf(tf->color, 4 * (size_t)tf->nc);
  s->nc = tf->nc;
  s->density = dupf(tf->density, (size_t)tf->nd);
  s->nd = tf->nd;
  if (tf->storage_fp16) quantize_positions(s);
  prepass(s, radii, tf);
  if (tf->storage_fp16) quantize_weights(s);
  for (uint32_t l = 0; l < s->nleaves; ++l) s->leaf_key[l] = keys[(uint64_t)l * s->ppl];
  leaf_bounds(s);
  if (s->nleaves == 0) {
    for (int a = 0; a < 6; ++a) s->root_box[a] = NAN;
    s->root = ORC_LEAF_BIT; /* unused */
  } else if (s->nleaves == 1) {
    s->root = 0 | ORC_LEAF_BIT;
    memcpy(s->root_box, s->leaf_eff, 6 * sizeof(float));
  } else {
    karras(s);
    refit_node(s, 0);
    s->root = 0;
    memcpy(s->root_box, s->node_box, 6 * sizeof(float));
  }
  return s;
}

void orc_scene_destroy(orc_scene *s) {
  if (!s) return;
  free(s->xyzw); free(s->rec0); free(s->w4); free(s->rgeom);
  free(s->leaf_key); free(s->leaf_box); free(s->leaf_eff); free(s->left); free(s->right);
  free(s->node_box);
  free(s->color); free(s->density);
  free(s);
}

uint32_t orc_scene_num_leaves(const orc_scene *s) { return s->nleaves; }

void orc_scene_get_bvh(const orc_scene *s, uint32_t *left, uint32_t *right, float *node_box,
                       float *leaf_box, float *leaf_eff, float *root_box) {
  uint32_t ni = s->nleaves > 0 ? s->nleaves - 1 : 0;
  if (left) memcpy(left, s->left, ni * sizeof(uint32_t));
  if (right) memcpy(right, s->right, ni * sizeof(uint32_t));
  if (node_box) memcpy(node_box, s->node_box, 6 * (size_t)ni * sizeof(float));
  if (leaf_box) memcpy(leaf_box, s->leaf_box, 6 * (size_t)s->nleaves * sizeof(float));
  if (leaf_eff) memcpy(leaf_eff, s->leaf_eff, 6 * (size_t)s->nleaves * sizeof(float));
  if (root_box) memcpy(root_box, s->root_box, 6 * sizeof(float));
}

void orc_scene_get_particles(const orc_scene *s, float *xyzw) { memcpy(xyzw, s->xyzw, 16 * s->n); }

void orc_scene_get_prepass(const orc_scene *s, float *rec0, float *w4, float *rgeom) {
  if (rec0) memcpy(rec0, s->rec0, 4 * s->n * sizeof(float));
  if (w4) memcpy(w4, s->w4, 4 * s->n * sizeof(float));
  if (rgeom) memcpy(rgeom, s->rgeom, s->n * sizeof(float));
}

/* ------------------------------------------------------------------------------------------ */
/* point query = ParticleRBFIntersection + ParticleRBFAnyHit (deviceCodeRBF.hlsl:338-389)      */
/* ------------------------------------------------------------------------------------------ */

static inline int64_t fix40(float v) { return llrintf(v * ORC_FIX_SCALE); }

static inline void eval_particle(const orc_scene *s, uint64_t i, const float *x, int *count,
                                 int64_t *acc) {
  const float *r = s->rec0 + 4 * i;
  float dx = r[0] - x[0], dy = r[1] - x[1], dz = r[2] - x[2];
  float dist = sqrtf((dx * dx + dy * dy) + dz * dz);
  if (!(dist < r[3])) return;
  /* evaluate_rbf, sharedCode.h:137-140, sigma = 3 */
  float q = (dist * 3.0f) / r[3];
  float rho = orc_expf(-0.5f * (q * q));
  const float *w = s->w4 + 4 * i;
  *count += 1;
  acc[0] += fix40(rho * w[0]);
  acc[1] += fix40(rho * w[1]);
  acc[2] += fix40(rho * w[2]);
  acc[3] += fix40(rho * w[3]);
}

static inline int box_contains(const float *b, const float *x) {
  return x[0] >= b[0] && x[0] <= b[3] && x[1] >= b[1] && x[1] <= b[4] && x[2] >= b[2] &&
         x[2] <= b[5];
}

static void leaf_eval(const orc_scene *s, uint32_t leaf, const float *x, int *count,
                      int64_t *acc) {
  for (uint32_t k = 0; k < s->ppl; ++k) {
    uint64_t i = (uint64_t)leaf * s->ppl + k;
    if (i >= s->n) break;
    eval_particle(s, i, x, count, acc);
  }
}

int orc_point_query(const orc_scene *s, const float *x, int64_t *acc) {
  int count = 0;
  acc[0] = acc[1] = acc[2] = acc[3] = 0;
  if (s->nleaves == 0 || !box_contains(s->root_box, x)) return 0;
  if (s->root & ORC_LEAF_BIT) {
    leaf_eval(s, s->root & ~ORC_LEAF_BIT, x, &count, acc);
    return count;
  }
  uint32_t stack[128];
  int sp = 0;
  stack[sp++] = s->root;
  while (sp) {
    uint32_t nd = stack[--sp];
    uint32_t ch[2] = {s->left[nd], s->right[nd]};
    for (int c = 0; c < 2; ++c) {
      if (!box_contains(child_box(s, ch[c]), x)) continue;
      if (ch[c] & ORC_LEAF_BIT) leaf_eval(s, ch[c] & ~ORC_LEAF_BIT, x, &count, acc);
      else if (sp < 128) stack[sp++] = ch[c];
      else abort(); /* tree deeper than any 64-bit key prefix allows */
    }
  }
  return count;
}

int orc_point_query_brute(const orc_scene *s, const float *x, int64_t *acc) {
  int count = 0;
  acc[0] = acc[1] = acc[2] = acc[3] = 0;
  for (uint64_t i = 0; i < s->n; ++i) eval_particle(s, i, x, &count, acc);
  return count;
}

/* ------------------------------------------------------------------------------------------ */
/* tracker: ParticleTracker (deviceCodeRBF.hlsl:40-204)                                         */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
  float o[3], d[3], tmin, tmax;
} orc_ray;

typedef struct {
  int i;
  float random;
  uint32_t rng;
  float albedo[4];
  float t;
  float lhs;
  int shadow;
  int marching;
  float gap; /* smallest relative gap between the two sides of any random decision so far */
} orc_tracker;

/* records how close a decision a < b (or a > b) came to going the other way */
static inline void note_gap(orc_tracker *tr, float a, float b) {
  float g = fabsf(a - b) / fmaxf(fabsf(b), 1e-30f);
  if (g < tr->gap) tr->gap = g;
}

/* sharedCode.h:151-185 */
static int aabb_intersect(const orc_ray *r, const float *lb, const float *rt, float *tenter,
                          float *texit) {
  float fx = 1.0f / r->d[0], fy = 1.0f / r->d[1], fz = 1.0f / r->d[2];
  float t2 = (rt[0] - r->o[0]) * fx;
  float t4 = (rt[1] - r->o[1]) * fy;
  float t6 = (rt[2] - r->o[2]) * fz;
  float t1 = (lb[0] - r->o[0]) * fx;
  float t3 = (lb[1] - r->o[1]) * fy;
  float t5 = (lb[2] - r->o[2]) * fz;
  float te = orc_maxf(orc_maxf(orc_minf(t1, t2), orc_minf(t3, t4)), orc_minf(t5, t6));
  float tx = orc_minf(orc_minf(orc_maxf(t1, t2), orc_maxf(t3, t4)), orc_maxf(t5, t6));
  te = orc_maxf(te, r->tmin);
  tx = orc_minf(tx, r->tmax);
  *tenter = te;
  *texit = tx;
  int hit = 1;
  if (tx < 0.0f) hit = 0;
  if (te >= tx) hit = 0;
  return hit;
}

typedef struct {
  int count;
  float density; /* D */
  float c[3];    /* C (not yet divided) */
} orc_sample;

static void sample_at(const orc_scene *s, const float *x, orc_sample *out) {
  int64_t acc[4];
  out->count = orc_point_query(s, x, acc);
  out->density = (float)acc[0] * ORC_FIX_INV;
  out->c[0] = (float)acc[1] * ORC_FIX_INV;
  out->c[1] = (float)acc[2] * ORC_FIX_INV;
  out->c[2] = (float)acc[3] * ORC_FIX_INV;
}

/* colour of a sample, deviceCodeRBF.hlsl:184-186 (+:192-194 when not visualising attributes) */
static void sample_color(const orc_scene *s, const orc_params *p, const orc_sample *smp,
                         float *rgb) {
  if (p->flags & ORC_FLAG_VISUALIZE_ATTRIBUTES) {
    for (int c = 0; c < 3; ++c) rgb[c] = orc_powf(smp->c[c] / smp->density, 1.0f / 2.2f);
  } else {
    for (int c = 0; c < 3; ++c) rgb[c] = orc_tex_sample(s->color, s->nc, 4, c, smp->density);
  }
}

/* densitymap(D) (:190), or the native linear transform min(D*gain, 1) */
static float sample_density(const orc_scene *s, const orc_params *p, float D) {
  if (p->flags & ORC_FLAG_DENSITY_LINEAR) return orc_minf(D * p->density_gain, 1.0f);
  return orc_tex_sample(s->density, s->nd, 1, 0, D);
}

/* stochasticTracking, deviceCodeRBF.hlsl:141-203 */
static void track_delta(const orc_scene *s, const orc_params *p, orc_tracker *tr,
                        const orc_ray *ray, int from_entry) {
  if (!from_entry) tr->t = ray->tmin;
  for (; tr->i < ORC_MAX_DEPTH; ++tr->i) {
    float u = orc_lcg_randomf(&tr->rng);
    float step = (orc_logf(1.0f - u) / 1.0f) * p->unit;
    tr->t = tr->t - step;
    if (tr->t >= ray->tmax) return;
    float x[3] = {ray->o[0] + tr->t * ray->d[0], ray->o[1] + tr->t * ray->d[1],
                  ray->o[2] + tr->t * ray->d[2]};
    orc_sample smp;
    sample_at(s, x, &smp);
    if (smp.count == 0) continue;
    float density = sample_density(s, p, smp.density);
    float xi = orc_lcg_randomf(&tr->rng);
    note_gap(tr, xi, density / 1.0f);
    if (xi < density / 1.0f) {
      float rgb[3];
      sample_color(s, p, &smp, rgb);
      tr->albedo[0] = rgb[0];
      tr->albedo[1] = rgb[1];
      tr->albedo[2] = rgb[2];
      tr->albedo[3] = 1.0f;
      return;
    }
  }
}

/* stochasticMarching, deviceCodeRBF.hlsl:67-139 */
static void track_march(const orc_scene *s, const orc_params *p, orc_tracker *tr,
                        const orc_ray *ray) {
  float rhs = -orc_logf(1.0f - tr->random * 0.99f);
  for (; tr->i < ORC_MAX_DEPTH; ++tr->i) {
    tr->t = tr->t + p->unit;
    if (tr->t >= ray->tmax) return;
    float x[3] = {ray->o[0] + tr->t * ray->d[0], ray->o[1] + tr->t * ray->d[1],
                  ray->o[2] + tr->t * ray->d[2]};
    orc_sample smp;
    sample_at(s, x, &smp);
    if (!(smp.count > 0 && smp.density > 0.0f)) continue;
    float density = sample_density(s, p, smp.density);
    tr->lhs = tr->lhs + density;
    if (!tr->shadow) note_gap(tr, tr->lhs, rhs);
    if (tr->lhs > rhs && !tr->shadow) {
      float rgb[3];
      sample_color(s, p, &smp, rgb);
      tr->albedo[0] = rgb[0];
      tr->albedo[1] = rgb[1];
      tr->albedo[2] = rgb[2];
      tr->albedo[3] = 1.0f;
      return;
    }
    if (tr->shadow) {
      tr->albedo[3] = tr->albedo[3] + (1.0f - orc_expf(-density));
      note_gap(tr, tr->albedo[3], 1.0f);
      if (tr->albedo[3] >= 1.0f) {
        tr->albedo[3] = 1.0f;
        return;
      }
    }
  }
}

/* ---- delta tracking with per-bin majorants (native mode; no counterpart in the reference) ----
 * The ray from its start t0 is cut into bins [t0 + k L, t0 + (k+1) L). The majorant of a bin is
 * density_scale * (1 + 2^-7) * sum over particles whose sphere meets the bin's segment of
 * a^3 * rho at the particle's closest approach to the segment (fixed-point sum). Delta tracking
 * then runs bin by bin: empty bins are crossed without drawing, a tentative step beyond the bin
 * restarts at the bin boundary (memoryless), a tentative collision at t is real with probability
 * density_scale * D(t) / majorant. */

typedef struct {
  uint32_t *idx;
  size_t n, cap;
} orc_cands;

static void cands_push(orc_cands *c, uint32_t i) {
  if (c->n == c->cap) {
    c->cap = c->cap ? 2 * c->cap : 256;
    c->idx = (uint32_t *)realloc(c->idx, c->cap * sizeof(uint32_t));
  }
  c->idx[c->n++] = i;
}

static int seg_box_hit(const float *b, const orc_ray *r, const float *inv, float t0, float t1, float e) {
  float ax = (b[0] - e - r->o[0]) * inv[0], bx = (b[3] + e - r->o[0]) * inv[0];
  float ay = (b[1] - e - r->o[1]) * inv[1], by = (b[4] + e - r->o[1]) * inv[1];
  float az = (b[2] - e - r->o[2]) * inv[2], bz = (b[5] + e - r->o[2]) * inv[2];
  float tn = orc_maxf(orc_maxf(orc_minf(ax, bx), orc_minf(ay, by)), orc_maxf(orc_minf(az, bz), t0));
  float tf = orc_minf(orc_minf(orc_maxf(ax, bx), orc_maxf(ay, by)), orc_minf(orc_maxf(az, bz), t1));
  return tn <= tf;
}

/* every particle whose (slightly inflated) sphere meets [t0, t1]: a superset of the particles
 * that meet any bin inside the segment by the exact test of bin_contrib */
static void seg_collect(const orc_scene *s, const orc_ray *ray, float t0, float t1, orc_cands *c) {
  c->n = 0;
  if (s->nleaves == 0) return;
  float m = 1.0f;
  for (int a = 0; a < 3; ++a) m = orc_maxf(m, orc_maxf(fabsf(ray->o[a]), fabsf(s->root_box[a])));
  for (int a = 3; a < 6; ++a) m = orc_maxf(m, fabsf(s->root_box[a]));
  const float e = m * 0x1p-14f;
  float inv[3] = {1.0f / ray->d[0], 1.0f / ray->d[1], 1.0f / ray->d[2]};
  uint32_t stack[128];
  int sp = 0;
  uint32_t todo[2];
  int nt = 0;
  if (s->root & ORC_LEAF_BIT) todo[nt++] = s->root;
  else stack[sp++] = s->root;
  for (;;) {
    for (int k = 0; k < nt; ++k) {
      uint32_t leaf = todo[k] & ~ORC_LEAF_BIT;
      for (uint32_t j = 0; j < s->ppl; ++j) {
        uint64_t i = (uint64_t)leaf * s->ppl + j;
        if (i >= s->n) break;
        const float *r = s->rec0 + 4 * i;
        if (!(r[3] > 0.0f)) continue;
        float vx = r[0] - ray->o[0], vy = r[1] - ray->o[1], vz = r[2] - ray->o[2];
        float tc = (vx * ray->d[0] + vy * ray->d[1]) + vz * ray->d[2];
        float wx = vx - tc * ray->d[0], wy = vy - tc * ray->d[1], wz = vz - tc * ray->d[2];
        float h2 = (wx * wx + wy * wy) + wz * wz;
        float R = r[3] * (1.0f + 0x1p-8f) + e;
        if (h2 > R * R) continue;
        float half = sqrtf(R * R - h2) + e;
        if (tc + half < t0 || tc - half > t1) continue;
        cands_push(c, (uint32_t)i);
      }
    }
    nt = 0;
    if (!sp) break;
    uint32_t nd = stack[--sp];
    uint32_t ch[2] = {s->left[nd], s->right[nd]};
    for (int k = 0; k < 2; ++k) {
      if (!seg_box_hit(child_box(s, ch[k]), ray, inv, t0, t1, e)) continue;
      if (ch[k] & ORC_LEAF_BIT) todo[nt++] = ch[k];
      else if (sp < 128) stack[sp++] = ch[k];
      else abort();
    }
  }
}

/* a^3 rho at the closest approach of particle i to the ray segment [b0, b1], 0 when its sphere
 * does not meet the segment */
static float bin_contrib(const orc_scene *s, const orc_ray *ray, uint64_t i, float b0, float b1) {
  const float *r = s->rec0 + 4 * i;
  float vx = r[0] - ray->o[0], vy = r[1] - ray->o[1], vz = r[2] - ray->o[2];
  float tc = (vx * ray->d[0] + vy * ray->d[1]) + vz * ray->d[2];
  float wx = vx - tc * ray->d[0], wy = vy - tc * ray->d[1], wz = vz - tc * ray->d[2];
  float h2 = (wx * wx + wy * wy) + wz * wz;
  float tcl = orc_minf(orc_maxf(tc, b0), b1);
  float dt = tcl - tc;
  float d2 = h2 + dt * dt;
  float r2 = r[3] * r[3];
  if (!(d2 < r2)) return 0.0f;
  float q2 = (9.0f * d2) / r2;
  return orc_expf(-0.5f * q2) * s->w4[4 * i];
}

#define ORC_BIN_SPLIT_STEPS 4.0f /* split a bin while majorant * length exceeds this */
#define ORC_BIN_SPLIT_DEPTH 10

typedef struct {
  const orc_scene *s;
  const orc_params *p;
  orc_tracker *tr;
  const orc_ray *ray;
  const orc_cands *c;
  float scale, minf;
} orc_bin_ctx;

static float bin_majorant(const orc_bin_ctx *b, float lo, float hi) {
  int64_t acc = 0;
  for (size_t j = 0; j < b->c->n; ++j) acc += fix40(bin_contrib(b->s, b->ray, b->c->idx[j], lo, hi));
  return ((float)acc * ORC_FIX_INV) * b->minf;
}

/* delta tracking across [lo, hi); a bin whose expected number of tentative steps exceeds
 * ORC_BIN_SPLIT_STEPS is split in halves (front half first), at most ORC_BIN_SPLIT_DEPTH times.
 * Returns 1 when the tracker is done (collision or step cap). */
static int track_bin(const orc_bin_ctx *b, float lo, float hi, int depth, float *tp) {
  float M = bin_majorant(b, lo, hi);
  if (!(M > 0.0f)) return 0;
  float mid = lo + 0.5f * (hi - lo);
  if (M * (hi - lo) > ORC_BIN_SPLIT_STEPS && depth < ORC_BIN_SPLIT_DEPTH && mid > lo && mid < hi) {
    if (track_bin(b, lo, mid, depth + 1, tp)) return 1;
    return track_bin(b, mid, hi, depth + 1, tp);
  }
  orc_tracker *tr = b->tr;
  const orc_ray *ray = b->ray;
  float t = lo;
  for (;;) {
    if (tr->i >= ORC_MAX_DEPTH) {
      *tp = t;
      return 1;
    }
    tr->i += 1;
    float u = orc_lcg_randomf(&tr->rng);
    float step = -orc_logf(1.0f - u) / M;
    t = t + step;
    if (t >= hi || t >= ray->tmax) return 0;
    float x[3] = {ray->o[0] + t * ray->d[0], ray->o[1] + t * ray->d[1], ray->o[2] + t * ray->d[2]};
    orc_sample smp;
    sample_at(b->s, x, &smp);
    float sigma = smp.density * b->scale;
    float xi = orc_lcg_randomf(&tr->rng);
    note_gap(tr, xi, sigma / M);
    if (xi < sigma / M) {
      float rgb[3];
      sample_color(b->s, b->p, &smp, rgb);
      tr->albedo[0] = rgb[0];
      tr->albedo[1] = rgb[1];
      tr->albedo[2] = rgb[2];
      tr->albedo[3] = 1.0f;
      *tp = t;
      return 1;
    }
  }
}

static void track_majorant(const orc_scene *s, const orc_params *p, orc_tracker *tr, const orc_ray *ray) {
  const float L = p->bin_length;
  const float t0 = tr->t;
  orc_cands c = {0, 0, 0};
  orc_bin_ctx b = {s, p, tr, ray, &c, p->density_scale, p->density_scale * 1.0078125f};
  /* (1 + 2^-7) on the majorant: slack for rounding in the bound */
  int seg_end = 0; /* bins [.., seg_end) are covered by c */
  int k = 0;
  float t = t0;
  for (;;) {
    float b0 = t0 + (float)k * L;
    float b1 = t0 + (float)(k + 1) * L;
    if (!(b0 < ray->tmax) || !(b1 > b0)) break;
    if (k >= seg_end) {
      seg_collect(s, ray, b0, t0 + (float)(k + 16) * L, &c);
      seg_end = k + 16;
    }
    float tp = b1;
    if (track_bin(&b, b0, b1, 0, &tp)) {
      tr->t = tp;
      free(c.idx);
      return;
    }
    k += 1;
    t = b1;
  }
  tr->t = t;
  free(c.idx);
}

static void track(const orc_scene *s, const orc_params *p, orc_tracker *tr, const orc_ray *ray,
                  int from_entry) {
  if (tr->marching) track_march(s, p, tr, ray);
  else if (p->flags & ORC_FLAG_MAJORANT_TRACKING) track_majorant(s, p, tr, ray);
  else track_delta(s, p, tr, ray, from_entry);
}

/* sharedCode.h:142-150 */
static void over(const float *a, const float *b, float *res) {
  float ra = a[3] + b[3] * (1.0f - a[3]);
  if (ra == 0.0f) {
    res[0] = a[0]; res[1] = a[1]; res[2] = a[2]; res[3] = a[3];
    return;
  }
  for (int c = 0; c < 3; ++c) res[c] = (a[c] * a[3] + (b[c] * b[3]) * (1.0f - a[3])) / ra;
  res[3] = ra;
}

static float noise_at(const orc_params *p, uint32_t frame, uint32_t px, uint32_t py) {
  /* deviceCodeRBF.hlsl:243-251: 8 x 16 grid of 256x256 tiles, UNORM8 .x */
  uint32_t gx = frame % 8u, gy = (frame / 8u) % 16u;
  uint32_t cx = gx * 256u + px % 256u, cy = gy * 256u + py % 256u;
  if (!p->noise || (int)cx >= p->noise_w || (int)cy >= p->noise_h) return 0.0f;
  uint8_t v = p->noise[4 * ((size_t)cy * (size_t)p->noise_w + cx)];
  return (float)v / 255.0f;
}

/* ParticleRBFRayGen, deviceCodeRBF.hlsl:206-336, one sample; returns colour (pre-accumulation)
 * and the noise value used for showNoise */
static void raygen_sample(const orc_scene *s, const orc_params *p, const float *light, uint32_t frame,
                          int px, int py, int w, int h, float *color, float *noise_out, float *gap_out) {
  uint32_t rng = orc_get_rng((int)frame, (uint32_t)px, (uint32_t)py, (uint32_t)w);
  float sx = ((float)px + 0.5f + p->jitter_x) / (float)w;
  float sy = ((float)py + 0.5f + p->jitter_y) / (float)h;
  float rt[3], lb[3];
  for (int a = 0; a < 3; ++a) {
    rt[a] = p->aabb_max[a] + 2.0f * p->rbf_radius;
    lb[a] = p->aabb_min[a] - 2.0f * p->rbf_radius;
  }
  orc_ray ray;
  float dir[3];
  for (int a = 0; a < 3; ++a) {
    ray.o[a] = p->cam_pos[a];
    dir[a] = (p->cam_dir00[a] + sx * p->cam_du[a]) + sy * p->cam_dv[a];
  }
  v3_normalize(dir, ray.d);
  ray.tmin = 0.0f;
  ray.tmax = 10000.0f;
  float tenter, texit;
  aabb_intersect(&ray, lb, rt, &tenter, &texit);

  orc_tracker tr;
  memset(&tr, 0, sizeof(tr));
  float rnd[3];
  int blue = (p->flags & ORC_FLAG_BLUE_NOISE) != 0;
  if (blue) {
    rnd[0] = noise_at(p, frame, (uint32_t)px, (uint32_t)py);
    tr.marching = 1;
  } else {
    rnd[0] = orc_lcg_randomf(&rng);
    tr.marching = 0;
    tr.rng = rng;
  }
  rnd[1] = orc_lcg_randomf(&rng);
  rnd[2] = orc_lcg_randomf(&rng);
  tr.i = 0;
  tr.lhs = 0.0f;
  tr.random = rnd[0];
  tr.shadow = 0;
  tr.gap = INFINITY;
  float col[4] = {0, 0, 0, 0};
  *noise_out = rnd[0];

  if (tenter < texit) {
    ray.tmax = texit;
    tr.t = tenter + p->unit * rnd[1];
    track(s, p, &tr, &ray, (p->flags & ORC_FLAG_TRACK_FROM_ENTRY) != 0);
    float albedo[4] = {tr.albedo[0], tr.albedo[1], tr.albedo[2], tr.albedo[3]};
    float t = tr.t;
    float vis = 1.0f;
    if (albedo[3] > 0.0f && p->light_ambient != 1.0f) {
      orc_ray sr;
      for (int a = 0; a < 3; ++a) {
        sr.o[a] = ray.o[a] + ray.d[a] * t;
        sr.d[a] = light[a];
      }
      sr.tmin = 0.0f;
      sr.tmax = 10000.0f;
      float ste, stx;
      aabb_intersect(&sr, lb, rt, &ste, &stx);
      sr.tmax = stx;
      tr.albedo[0] = tr.albedo[1] = tr.albedo[2] = tr.albedo[3] = 0.0f;
      tr.lhs = 0.0f;
      tr.shadow = 1;
      tr.t = blue ? -p->unit * rnd[2] : 0.0f;
      track(s, p, &tr, &sr, 0);
      vis = 1.0f - tr.albedo[3];
    }
    if (albedo[3] == 1.0f) {
      for (int c = 0; c < 3; ++c)
        col[c] = (albedo[c] * vis) * (1.0f - p->light_ambient) + albedo[c] * p->light_ambient;
      col[3] = 1.0f;
    }
  }
  float bg[4] = {0.0f, 0.0f, 0.0f, 1.0f};
  over(col, bg, color);
  *gap_out = tr.gap;
}

static void render_pixel(const orc_scene *s, const orc_params *p, const float *light, int px,
                         int py, int w, int h, float *accum, float *image, float *gaps) {
  size_t ofs = (size_t)py * (size_t)w + (size_t)px;
  float prev[4] = {accum[4 * ofs], accum[4 * ofs + 1], accum[4 * ofs + 2], accum[4 * ofs + 3]};
  float fin[4] = {prev[0], prev[1], prev[2], prev[3]};
  float noise = 0.0f;
  uint32_t spp = p->spp ? p->spp : 1;
  float gap = INFINITY;
  for (uint32_t k = 0; k < spp; ++k) {
    uint32_t frame = (p->frame_id + k) & 0xffffu;
    uint32_t aid = (p->accum_id + k) & 0xffffu;
    float color[4], g;
    raygen_sample(s, p, light, frame, px, py, w, h, color, &noise, &g);
    if (g < gap) gap = g;
    /* deviceCodeRBF.hlsl:326-328 */
    float fa = (float)aid;
    float wa = 1.0f / fa, wb = (float)((int)aid - 1) / fa;
    for (int c = 0; c < 4; ++c) fin[c] = wa * color[c] + wb * prev[c];
    memcpy(prev, fin, sizeof(prev));
  }
  memcpy(accum + 4 * ofs, fin, sizeof(fin));
  if (p->flags & ORC_FLAG_SHOW_NOISE) {
    fin[0] = fin[1] = fin[2] = noise;
    fin[3] = 1.0f;
  }
  memcpy(image + 4 * ofs, fin, sizeof(fin));
  if (gaps) gaps[ofs] = gap;
}

void orc_render_region_gaps(const orc_scene *s, const orc_params *p, int w, int h, int x0, int x1,
                            int y0, int y1, float *accum, float *image, float *gaps, int nthreads) {
  float light[3];
  orc_light_dir(p->light_azimuth, p->light_elevation, light);
  int nt = nthreads > 0 ? nthreads : g_threads;
  int rows = y1 - y0, cols = x1 - x0;
  long total = (long)rows * (long)cols;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(nt > 0 ? nt : omp_get_max_threads())
#endif
  for (long k = 0; k < total; ++k) {
    int py = y0 + (int)(k / cols), px = x0 + (int)(k % cols);
    render_pixel(s, p, light, px, py, w, h, accum, image, gaps);
  }
  (void)nt;
}

void orc_render_region(const orc_scene *s, const orc_params *p, int w, int h, int x0, int x1,
                       int y0, int y1, float *accum, float *image, int nthreads) {
  orc_render_region_gaps(s, p, w, h, x0, x1, y0, y1, accum, image, NULL, nthreads);
}

void orc_render(const orc_scene *s, const orc_params *p, int w, int h, float *accum, float *image,
                int nthreads) {
  orc_render_region(s, p, w, h, 0, w, 0, h, accum, image, nthreads);
}

/* ------------------------------------------------------------------------------------------ */
/* splatting: ParticleSplatRayGen / Intersection / AnyHit (deviceCodeSplat.hlsl:29-193)         */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
  float t;
  uint32_t id;
} orc_splat_sample;

static int cmp_splat(const void *a, const void *b) {
  const orc_splat_sample *x = (const orc_splat_sample *)a, *y = (const orc_splat_sample *)b;
  if (x->t < y->t) return -1;
  if (x->t > y->t) return 1;
  return (x->id < y->id) ? -1 : (x->id > y->id ? 1 : 0);
}

/* splat radius: the global rbfRadius as in deviceCodeSplat.hlsl:166, or the per-particle radius
 * in native mode; particles whose radiusmap value is 0 are not splatted */
static float splat_radius(const orc_scene *s, const orc_params *p, uint64_t i) {
  if (s->rgeom[i] < 0.0f) return 0.0f;
  return (p->flags & ORC_FLAG_SPLAT_PARTICLE_RADIUS) ? s->rgeom[i] : p->rbf_radius;
}

static void splat_pixel(const orc_scene *s, const orc_params *p, int px, int py, int w, int h,
                        float *image) {
  float sx = ((float)px + 0.5f + p->jitter_x) / (float)w;
  float sy = ((float)py + 0.5f + p->jitter_y) / (float)h;
  float rt[3], lb[3];
  for (int a = 0; a < 3; ++a) {
    rt[a] = p->aabb_max[a] + p->rbf_radius;
    lb[a] = p->aabb_min[a] - p->rbf_radius;
  }
  orc_ray ray;
  float dir[3];
  for (int a = 0; a < 3; ++a) {
    ray.o[a] = p->cam_pos[a];
    dir[a] = (p->cam_dir00[a] + sx * p->cam_du[a]) + sy * p->cam_dv[a];
  }
  v3_normalize(dir, ray.d);
  ray.tmin = 0.0f;
  ray.tmax = 10000.0f;
  float tenter, texit;
  aabb_intersect(&ray, lb, rt, &tenter, &texit);
  float res[4] = {0, 0, 0, 0};
  if (tenter < texit) {
    /* every candidate: t = |c - o|; accept if |c - (o + t d)|^2 < r^2 (:165-179); the slab
     * condition TMin <= t < TMax is applied per slab below. Particles of leaves whose bounds
     * box is inactive and particles with radiusmap == 0 are not candidates. */
    size_t cap = 64, cnt = 0;
    orc_splat_sample *cand = (orc_splat_sample *)malloc(cap * sizeof(orc_splat_sample));
    for (uint64_t i = 0; i < s->n; ++i) {
      float r = splat_radius(s, p, i);
      if (!(r > 0.0f)) continue;
      const float *c = s->xyzw + 4 * i;
      float vx = c[0] - ray.o[0], vy = c[1] - ray.o[1], vz = c[2] - ray.o[2];
      float t = sqrtf((vx * vx + vy * vy) + vz * vz);
      float sp[3] = {ray.o[0] + t * ray.d[0], ray.o[1] + t * ray.d[1], ray.o[2] + t * ray.d[2]};
      float ox = c[0] - sp[0], oy = c[1] - sp[1], oz = c[2] - sp[2];
      if (!(((ox * ox + oy * oy) + oz * oz) < r * r)) continue;
      if (cnt == cap) {
        cap *= 2;
        cand = (orc_splat_sample *)realloc(cand, cap * sizeof(orc_splat_sample));
      }
      cand[cnt].t = t;
      cand[cnt].id = (uint32_t)i;
      ++cnt;
    }
    qsort(cand, cnt, sizeof(orc_splat_sample), cmp_splat);
    const float per_slab = (float)(15 / 8); /* PARTICLE_BUFFER_SIZE / 8 in integers = 1 */
    const float spacing = per_slab * p->unit;
    const float atten = orc_expf(-p->unit * per_slab);
    float tslab = 0.0f;
    size_t cursor = 0;
    while (tslab < texit) {
      if (res[3] > 0.99f) break;
      float tmin = orc_maxf(tenter, tslab);
      float tmax = orc_minf(texit, tslab + spacing);
      if (tmax > tenter) {
        while (cursor < cnt && cand[cursor].t < tmin) ++cursor;
        size_t k = cursor;
        int taken = 0;
        while (k < cnt && taken < 15 && cand[k].t < tmax) {
          const float *P = s->xyzw + 4 * (uint64_t)cand[k].id;
          float X[3] = {ray.o[0] + ray.d[0] * cand[k].t, ray.o[1] + ray.d[1] * cand[k].t,
                        ray.o[2] + ray.d[2] * cand[k].t};
          float dx = X[0] - P[0], dy = X[1] - P[1], dz = X[2] - P[2];
          float dist = sqrtf((dx * dx + dy * dy) + dz * dz);
          float r = splat_radius(s, p, cand[k].id);
          float q = (dist * 3.0f) / r;
          float drbf = orc_expf(-0.5f * (q * q));
          float col[4];
          if (p->flags & ORC_FLAG_VISUALIZE_ATTRIBUTES) {
            for (int c = 0; c < 4; ++c) col[c] = orc_tex_sample(s->color, s->nc, 4, c, P[3]);
            drbf = orc_tex_sample(s->density, s->nd, 1, 0, drbf);
            col[3] = col[3] * drbf;
          } else {
            for (int c = 0; c < 3; ++c) col[c] = orc_tex_sample(s->color, s->nc, 4, c, drbf);
            col[3] = orc_tex_sample(s->density, s->nd, 1, 0, drbf);
          }
          col[3] = col[3] * atten;
          float nr[4];
          over(res, col, nr);
          memcpy(res, nr, sizeof(res));
          ++k;
          ++taken;
        }
      }
      tslab = tslab + spacing;
    }
    free(cand);
  }
  float bg[4] = {0.0f, 0.0f, 0.0f, 1.0f};
  float out[4];
  over(res, bg, out);
  memcpy(image + 4 * ((size_t)py * (size_t)w + (size_t)px), out, sizeof(out));
}

void orc_render_splat(const orc_scene *s, const orc_params *p, int w, int h, float *image,
                      int nthreads) {
  int nt = nthreads > 0 ? nthreads : g_threads;
  long total = (long)w * (long)h;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(nt > 0 ? nt : omp_get_max_threads())
#endif
  for (long k = 0; k < total; ++k) splat_pixel(s, p, (int)(k % w), (int)(k / w), w, h, image);
  (void)nt;
}

/* ------------------------------------------------------------------------------------------ */
/* TAA resolve (deviceCodeCommon.hlsl:27-43, 67-115)                                           */
/* ------------------------------------------------------------------------------------------ */

static void rgb2ycocg(const float *c, float *o) {
  float co = c[0] - c[2];
  float t = c[2] + co / 2.0f;
  float cg = c[1] - t;
  float y = t + cg / 2.0f;
  o[0] = y; o[1] = co; o[2] = cg;
}
static void ycocg2rgb(const float *c, float *o) {
  float t = c[0] - c[2] / 2.0f;
  float g = c[2] + t;
  float b = t - c[1] / 2.0f;
  float r = c[1] + b;
  o[0] = r; o[1] = g; o[2] = b;
}

static uint8_t unorm8(float v) {
  if (!(v > 0.0f)) v = 0.0f;
  if (v > 1.0f) v = 1.0f;
  return (uint8_t)(v * 255.0f + 0.5f);
}

void orc_taa(const float *image, const float *prev, float *taa, uint32_t *bgra, int w, int h,
             int disable) {
  for (int py = 0; py < h; ++py) {
    for (int px = 0; px < w; ++px) {
      size_t ofs = (size_t)py * (size_t)w + (size_t)px;
      const float *center = image + 4 * ofs;
      float pix[4];
      if (!disable) {
        float mn[3], mx[3];
        rgb2ycocg(center, mn);
        rgb2ycocg(center, mx);
        for (int iy = -1; iy <= 1; ++iy) {
          for (int ix = -1; ix <= 1; ++ix) {
            if (ix == 0 && iy == 0) continue;
            int qx = px + ix, qy = py + iy;
            if (qx < 0) qx = 0;
            if (qx > w - 1) qx = w - 1;
            if (qy < 0) qy = 0;
            if (qy > h - 1) qy = h - 1;
            float y[3];
            rgb2ycocg(image + 4 * ((size_t)qy * (size_t)w + (size_t)qx), y);
            for (int c = 0; c < 3; ++c) {
              mn[c] = orc_minf(mn[c], y[c]);
              mx[c] = orc_maxf(mx[c], y[c]);
            }
          }
        }
        float old[4] = {prev[4 * ofs], prev[4 * ofs + 1], prev[4 * ofs + 2], prev[4 * ofs + 3]};
        float y[3], rgb[3];
        rgb2ycocg(old, y);
        for (int c = 0; c < 3; ++c) y[c] = orc_maxf(y[c], mn[c]);
        ycocg2rgb(y, rgb);
        rgb2ycocg(rgb, y);
        for (int c = 0; c < 3; ++c) y[c] = orc_minf(y[c], mx[c]);
        ycocg2rgb(y, rgb);
        old[0] = rgb[0]; old[1] = rgb[1]; old[2] = rgb[2];
        for (int c = 0; c < 4; ++c) pix[c] = old[c] + 0.2f * (center[c] - old[c]);
        memcpy(taa + 4 * ofs, pix, sizeof(pix));
      } else {
        memcpy(pix, center, sizeof(pix));
      }
      if (bgra) {
        /* GUI layer is empty: over((0,0,0,0), pixel) (:193-195), then BGRA8 */
        float gui[4] = {0, 0, 0, 0}, o[4];
        over(gui, pix, o);
        bgra[ofs] = (uint32_t)unorm8(o[2]) | ((uint32_t)unorm8(o[1]) << 8) |
                    ((uint32_t)unorm8(o[0]) << 16) | ((uint32_t)unorm8(o[3]) << 24);
      }
    }
  }
}

/* ------------------------------------------------------------------------------------------ */
/* FP64 twin: converged reference images of the native-mode volume model                        */
/* ------------------------------------------------------------------------------------------ */
/* The same model as the native estimators (extinction sigma = density_scale * D with
 * D = sum a^3 exp(-4.5 d^2 / r^2) over the particles whose sphere contains the point; colour
 * pow(C / D, 1 / 2.2); one shadow ray; ambient shading, raygen as deviceCodeRBF.hlsl:206-324),
 * evaluated in double precision with libm exp/log/pow and an independent 64-bit random stream
 * (splitmix64). Transfer-function values are interpolated in double from the fp32 tables.
 * clamp_plain selects the extinction of the plain native estimator, min(sigma, 1/unit).
 * Delta tracking with per-bin majorants (unbiased for any valid majorant): the expected image
 * is the model's, whatever the bins. The float BVH only culls: seg_collect inflates every
 * sphere by 2^-8 r plus an absolute slack far above the float/double ray difference. */

typedef struct {
  double o[3], d[3], tmax;
} ray64;

typedef struct {
  double a, b, tc, h2, r2, w[4];
  double c[3]; /* centre */
} cand64;

static uint64_t splitmix64(uint64_t *s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static double u01(uint64_t *s) { return (double)(splitmix64(s) >> 11) * 0x1p-53; }

static double tex64(const float *tex, int n, int stride, int channel, double u) {
  /* linear between texel centres, clamp to edge (the parity model of orc_tex_sample) */
  if (n <= 0) return 0.0;
  double x = u * (double)n - 0.5;
  if (!(x > 0.0)) return (double)tex[channel];
  if (x >= (double)(n - 1)) return (double)tex[(size_t)(n - 1) * stride + channel];
  int i = (int)floor(x);
  double f = x - (double)i;
  double a = (double)tex[(size_t)i * stride + channel], b = (double)tex[(size_t)(i + 1) * stride + channel];
  return a + (b - a) * f;
}

static int cmp_cand64(const void *x, const void *y) {
  double a = ((const cand64 *)x)->a, b = ((const cand64 *)y)->a;
  return a < b ? -1 : (a > b ? 1 : 0);
}

typedef struct {
  cand64 *v;
  size_t n, cap;
  orc_cands idx;
} cand64_set;

static void collect64(const orc_scene *s, const ray64 *r, double t0, double t1, cand64_set *cs) {
  orc_ray fr;
  for (int a = 0; a < 3; ++a) {
    fr.o[a] = (float)r->o[a];
    fr.d[a] = (float)r->d[a];
  }
  fr.tmin = 0.0f;
  fr.tmax = 1e30f;
  float m = 1.0f;
  for (int a = 0; a < 3; ++a) m = fmaxf(m, fabsf(fr.o[a]));
  seg_collect(s, &fr, (float)t0 - m * 0x1p-12f, (float)t1 + m * 0x1p-12f, &cs->idx);
  cs->n = 0;
  for (size_t j = 0; j < cs->idx.n; ++j) {
    uint64_t i = cs->idx.idx[j];
    const float *q = s->rec0 + 4 * i;
    double rr = (double)q[3];
    if (!(rr > 0.0)) continue;
    double v[3] = {(double)q[0] - r->o[0], (double)q[1] - r->o[1], (double)q[2] - r->o[2]};
    double tc = v[0] * r->d[0] + v[1] * r->d[1] + v[2] * r->d[2];
    double w[3] = {v[0] - tc * r->d[0], v[1] - tc * r->d[1], v[2] - tc * r->d[2]};
    double h2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    double r2 = rr * rr;
    if (!(h2 < r2)) continue;
    double half = sqrt(r2 - h2);
    if (tc + half < t0 || tc - half > t1) continue;
    if (cs->n == cs->cap) {
      cs->cap = cs->cap ? 2 * cs->cap : 256;
      cs->v = (cand64 *)realloc(cs->v, cs->cap * sizeof(cand64));
    }
    cand64 *c = cs->v + cs->n++;
    c->a = tc - half;
    c->b = tc + half;
    c->tc = tc;
    c->h2 = h2;
    c->r2 = r2;
    for (int a = 0; a < 3; ++a) c->c[a] = (double)q[a];
    double attr = (double)s->xyzw[4 * i + 3];
    double al = tex64(s->color, s->nc, 4, 3, attr);
    double a3 = al * al * al;
    c->w[0] = a3;
    for (int k = 0; k < 3; ++k) c->w[1 + k] = pow(tex64(s->color, s->nc, 4, k, attr), 2.2) * a3;
  }
  qsort(cs->v, cs->n, sizeof(cand64), cmp_cand64);
}

/* delta tracking along r from t; returns 1 on a collision (rgb set) */
static int track64(const orc_scene *s, const orc_params *p, int clamp_plain, const ray64 *r, double t,
                   uint64_t *rng, cand64_set *cs, size_t **act, size_t *act_cap, double *t_hit,
                   double *rgb) {
  const double Lb = (double)p->bin_length > 0.0 ? (double)p->bin_length : 4.0 * (double)p->unit;
  const double scale = (double)p->density_scale;
  const double cap = clamp_plain ? 1.0 / (double)p->unit : INFINITY;
  double chunk = 2.0 * Lb; /* candidates are collected a chunk at a time, chunks growing to 64 bins */
  while (t < r->tmax) {
    double c1 = fmin(t + chunk, r->tmax);
    if (chunk < 64.0 * Lb) chunk *= 2.0;
    collect64(s, r, t, c1, cs);
    size_t next = 0, na = 0;
    if (*act_cap < cs->n + 1) {
      *act_cap = cs->n + 1;
      *act = (size_t *)realloc(*act, *act_cap * sizeof(size_t));
    }
    size_t *A = *act;
    for (double lo = t; lo < c1;) {
      double hi = fmin(lo + Lb, c1);
      while (next < cs->n && cs->v[next].a <= hi) A[na++] = next++;
      size_t keep = 0;
      for (size_t k = 0; k < na; ++k)
        if (cs->v[A[k]].b >= lo) A[keep++] = A[k];
      na = keep;
      if (na == 0) {
        if (next == cs->n) break; /* nothing further in this chunk */
        lo = hi;
        continue;
      }
      double M = 0.0;
      for (size_t k = 0; k < na; ++k) {
        const cand64 *c = cs->v + A[k];
        double tcl = fmin(fmax(c->tc, lo), hi), dt = tcl - c->tc;
        M += c->w[0] * exp(-4.5 * (c->h2 + dt * dt) / c->r2);
      }
      M = fmin(M * scale * (1.0 + 1e-9), cap);
      double tt = lo;
      while (M > 0.0) {
        tt += -log(1.0 - u01(rng)) / M;
        if (tt >= hi) break;
        double x[3] = {r->o[0] + tt * r->d[0], r->o[1] + tt * r->d[1], r->o[2] + tt * r->d[2]};
        double acc[4] = {0, 0, 0, 0};
        for (size_t k = 0; k < na; ++k) {
          const cand64 *c = cs->v + A[k];
          double dx = c->c[0] - x[0], dy = c->c[1] - x[1], dz = c->c[2] - x[2];
          double d2 = dx * dx + dy * dy + dz * dz;
          if (!(d2 < c->r2)) continue;
          double rho = exp(-4.5 * d2 / c->r2);
          for (int q = 0; q < 4; ++q) acc[q] += rho * c->w[q];
        }
        double sigma = fmin(acc[0] * scale, cap);
        if (u01(rng) * M < sigma) {
          for (int q = 0; q < 3; ++q) rgb[q] = pow(acc[1 + q] / acc[0], 1.0 / 2.2);
          *t_hit = tt;
          return 1;
        }
      }
      lo = hi;
    }
    t = c1;
  }
  return 0;
}

static void pixel64(const orc_scene *s, const orc_params *p, const double *light, int clamp_plain, int px,
                    int py, int w, int h, int spp, uint64_t seed, cand64_set *cs, size_t **act,
                    size_t *act_cap, double *out) {
  double sum[3] = {0, 0, 0};
  double lb[3], rt[3];
  for (int a = 0; a < 3; ++a) {
    rt[a] = (double)p->aabb_max[a] + 2.0 * (double)p->rbf_radius;
    lb[a] = (double)p->aabb_min[a] - 2.0 * (double)p->rbf_radius;
  }
  uint64_t rng = seed ^ (((uint64_t)(uint32_t)py << 32) | (uint32_t)px) * 0xD1B54A32D192ED03ull;
  splitmix64(&rng);
  double sx = ((double)px + 0.5 + (double)p->jitter_x) / (double)w;
  double sy = ((double)py + 0.5 + (double)p->jitter_y) / (double)h;
  ray64 r;
  double n2 = 0.0;
  for (int a = 0; a < 3; ++a) {
    r.o[a] = (double)p->cam_pos[a];
    r.d[a] = (double)p->cam_dir00[a] + sx * (double)p->cam_du[a] + sy * (double)p->cam_dv[a];
    n2 += r.d[a] * r.d[a];
  }
  for (int a = 0; a < 3; ++a) r.d[a] /= sqrt(n2);
  double te = -INFINITY, tx = INFINITY;
  for (int a = 0; a < 3; ++a) {
    double t1 = (lb[a] - r.o[a]) / r.d[a], t2 = (rt[a] - r.o[a]) / r.d[a];
    te = fmax(te, fmin(t1, t2));
    tx = fmin(tx, fmax(t1, t2));
  }
  te = fmax(te, 0.0);
  const double amb = (double)p->light_ambient;
  for (int k = 0; k < spp; ++k) {
    if (!(te < tx)) break;
    r.tmax = tx;
    double rgb[3], th;
    double t_start = te + (double)p->unit * u01(&rng);
    if (!track64(s, p, clamp_plain, &r, t_start, &rng, cs, act, act_cap, &th, rgb)) continue;
    double vis = 1.0;
    if (amb != 1.0) {
      ray64 sr;
      for (int a = 0; a < 3; ++a) {
        sr.o[a] = r.o[a] + r.d[a] * th;
        sr.d[a] = light[a];
      }
      double ste = -INFINITY, stx = INFINITY;
      for (int a = 0; a < 3; ++a) {
        double t1 = (lb[a] - sr.o[a]) / sr.d[a], t2 = (rt[a] - sr.o[a]) / sr.d[a];
        ste = fmax(ste, fmin(t1, t2));
        stx = fmin(stx, fmax(t1, t2));
      }
      sr.tmax = stx;
      double srgb[3], sth;
      if (track64(s, p, clamp_plain, &sr, 0.0, &rng, cs, act, act_cap, &sth, srgb)) vis = 0.0;
    }
    for (int q = 0; q < 3; ++q) sum[q] += rgb[q] * vis * (1.0 - amb) + rgb[q] * amb;
  }
  for (int q = 0; q < 3; ++q) out[q] = sum[q] / (double)spp;
}

void orc_render_f64(const orc_scene *s, const orc_params *p, int w, int h, int x0, int x1, int y0, int y1,
                    int spp, int clamp_plain, uint64_t seed, float *rgb_out, int nthreads) {
  double az = (double)p->light_azimuth, el = (double)p->light_elevation;
  double a = el * 3.14 - 0.5 * 3.14, b = (az * 2.0) * 3.14; /* sharedCode.h:127-132 (3.14 as written) */
  double light[3] = {sin(a) * cos(b), sin(a) * sin(b), cos(a)};
  int cols = x1 - x0, rows = y1 - y0;
  long total = (long)rows * (long)cols;
  int nt = nthreads > 0 ? nthreads : g_threads;
#ifdef _OPENMP
#pragma omp parallel num_threads(nt > 0 ? nt : omp_get_max_threads())
#endif
  {
    cand64_set cs = {0, 0, 0, {0, 0, 0}};
    size_t *act = 0, act_cap = 0;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
    for (long k = 0; k < total; ++k) {
      int py = y0 + (int)(k / cols), px = x0 + (int)(k % cols);
      double out[3];
      pixel64(s, p, light, clamp_plain, px, py, w, h, spp, seed, &cs, &act, &act_cap, out);
      for (int q = 0; q < 3; ++q) rgb_out[3 * k + q] = (float)out[q];
    }
    free(cs.v);
    free(cs.idx.idx);
    free(act);
  }
  (void)nt;
}

/* ------------------------------------------------------------------------------------------ */
/* Differentiable form: expected stochastic marching, FP64 forward and adjoint                  */
/* ------------------------------------------------------------------------------------------ */
/* The reference's stochasticMarching (deviceCodeRBF.hlsl:67-139) stops at the first step where
 * the accumulated density exceeds -log(1 - 0.99 xi). With ambient = 1 (no shadow ray) the
 * expectation of its colour over xi has a closed form, which is the differentiable model:
 *   t_k = t0 + (k + 1) unit,  t0 = tenter + unit u   (u: first LCG draw of the pixel seed)
 *   D_k = sum rho_i a_i^3,  C_k = sum rho_i a_i^3 rgb_i^2.2  over particles with |x_k - p_i| < r_i,
 *   rho_i = (exp(-4.5 q^2) - e^-4.5) / (1 - e^-4.5), q = |x_k - p_i| / r_i: the reference's
 *   truncated Gaussian (evaluate_rbf, sharedCode.h:137-140) shifted to reach 0 at the cut-off, so
 *   that images are continuous in positions and radii (the unshifted kernel jumps by e^-4.5 at r,
 *   a change no adjoint sees and finite differences do),
 *   (rgb_i, a_i) = transfer function at attribute w_i,
 *   dens_k = min(gain D_k, 1),  tau_k = sum_{j<=k} dens_j,  G_k = min(1, (1 - exp(-tau_k)) / 0.99)
 *   c_k = (C_k / D_k)^(1/2.2),  E = sum_k (G_k - G_{k-1}) c_k,  pixel = mean of E over spp.
 * Adjoint (path replay): dE/d dens_j = g'_j c_j + sum_{k>j} B_k with g'_k = dG_k/dtau_k and
 * B_k = (g'_k - g'_{prev(k)}) c_k, prev(k) the previous step with D > 0; the forward keeps only
 * B_total = sum_k B_k per sample, the backward replays the ray and subtracts the prefix.
 * Everything here is double precision: the reference values for the GPU's float kernels and the
 * subject of the finite-difference checks. Candidates are found by brute force. */

#define DIFF_E45 0.011108996538242306 /* exp(-4.5) */
#define DIFF_INV (1.0 / (1.0 - DIFF_E45))

typedef struct {
  int idx;
  double lo, hi;
} dcand;

typedef struct {
  const orc_diff_scene *sc;
  double *rgb22a3; /* 4 per particle: a^3, rgb^2.2 a^3 */
} dctx;

static void tf64(const double *tf, int nc, double w, double *out4, int *i0, double *f) {
  double x = w * (double)nc - 0.5;
  if (!(x > 0.0)) {
    *i0 = 0; *f = 0.0;
  } else if (x >= (double)(nc - 1)) {
    *i0 = nc - 1; *f = 0.0;
  } else {
    *i0 = (int)floor(x); *f = x - (double)*i0;
  }
  int j = *i0 + 1 < nc ? *i0 + 1 : *i0;
  for (int c = 0; c < 4; ++c) out4[c] = tf[4 * *i0 + c] + (tf[4 * j + c] - tf[4 * *i0 + c]) * *f;
}

typedef struct {
  double o[3], d[3], t0, tmax;
  int valid;
} dray;

static dray diff_ray(const orc_params *p, int px, int py, int w, int h, uint32_t s) {
  dray r;
  uint32_t rng = orc_get_rng((int)((p->frame_id + s) & 0xffffu), (uint32_t)px, (uint32_t)py, (uint32_t)w);
  double u = (double)orc_lcg_next(&rng) * 0x1p-32;
  double sx = ((double)px + 0.5) / (double)w, sy = ((double)py + 0.5) / (double)h, n2 = 0.0;
  for (int a = 0; a < 3; ++a) {
    r.o[a] = (double)p->cam_pos[a];
    r.d[a] = (double)p->cam_dir00[a] + sx * (double)p->cam_du[a] + sy * (double)p->cam_dv[a];
    n2 += r.d[a] * r.d[a];
  }
  double te = 0.0, tx = 10000.0;
  for (int a = 0; a < 3; ++a) {
    r.d[a] /= sqrt(n2);
    double lb = (double)p->aabb_min[a] - 2.0 * (double)p->rbf_radius;
    double rt = (double)p->aabb_max[a] + 2.0 * (double)p->rbf_radius;
    double t1 = (lb - r.o[a]) / r.d[a], t2 = (rt - r.o[a]) / r.d[a];
    te = fmax(te, fmin(t1, t2));
    tx = fmin(tx, fmax(t1, t2));
  }
  r.valid = te < tx;
  r.t0 = te + (double)p->unit * u;
  r.tmax = tx;
  return r;
}

/* particles whose sphere meets the ray within [t0, tmax] */
static int diff_cands(const orc_diff_scene *sc, const dray *r, dcand *out) {
  int n = 0;
  for (int i = 0; i < sc->n; ++i) {
    const double *p = sc->pos + 3 * i;
    double rr = sc->radius[i];
    if (!(rr > 0.0)) continue;
    double v[3] = {p[0] - r->o[0], p[1] - r->o[1], p[2] - r->o[2]};
    double tc = v[0] * r->d[0] + v[1] * r->d[1] + v[2] * r->d[2];
    double h2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] - tc * tc;
    if (!(h2 < rr * rr)) continue;
    double half = sqrt(rr * rr - h2);
    if (tc + half < r->t0 || tc - half > r->tmax) continue;
    out[n].idx = i;
    out[n].lo = tc - half;
    out[n].hi = tc + half;
    ++n;
  }
  return n;
}

/* one step: D, C and the members (index; kernel value in rho[m], derivative factor in rho[n + m]) */
static void diff_eval(const dctx *dc, const dray *r, const dcand *cands, int ncand, double t, double *D, double *C,
                      int *mem, double *rho, int *nm) {
  const orc_diff_scene *sc = dc->sc;
  const int n_ = sc->n;
  double x[3] = {r->o[0] + t * r->d[0], r->o[1] + t * r->d[1], r->o[2] + t * r->d[2]};
  *D = 0.0;
  C[0] = C[1] = C[2] = 0.0;
  *nm = 0;
  for (int k = 0; k < ncand; ++k) {
    if (t < cands[k].lo || t > cands[k].hi) continue;
    int i = cands[k].idx;
    const double *p = sc->pos + 3 * i;
    double dx = x[0] - p[0], dy = x[1] - p[1], dz = x[2] - p[2];
    double d2 = dx * dx + dy * dy + dz * dz, r2 = sc->radius[i] * sc->radius[i];
    if (!(d2 < r2)) continue;
    double e = exp(-4.5 * d2 / r2);
    double q = (e - DIFF_E45) * DIFF_INV;
    const double *w = dc->rgb22a3 + 4 * i;
    *D += q * w[0];
    for (int c = 0; c < 3; ++c) C[c] += q * w[1 + c];
    if (mem) {
      mem[*nm] = i;
      rho[*nm] = q;
      rho[n_ + *nm] = e * DIFF_INV;
    }
    ++*nm;
  }
}

/* forward of one sample: colour E and B_total */
static void diff_sample_fwd(const dctx *dc, const orc_params *p, const dray *r, const dcand *cands, int ncand,
                            double *E, double *Btot) {
  double tau = 0.0, G = 0.0, gprev = 0.0;
  E[0] = E[1] = E[2] = 0.0;
  Btot[0] = Btot[1] = Btot[2] = 0.0;
  const double unit = (double)p->unit, gain = (double)p->density_gain;
  for (int k = 0;; ++k) {
    double t = r->t0 + (double)(k + 1) * unit;
    if (t >= r->tmax) break;
    double D, C[3];
    int nm;
    diff_eval(dc, r, cands, ncand, t, &D, C, 0, 0, &nm);
    if (!(D > 0.0)) continue;
    double dens = fmin(gain * D, 1.0);
    tau += dens;
    double Gk = fmin(1.0, (1.0 - exp(-tau)) / 0.99);
    double gk = ((1.0 - exp(-tau)) / 0.99 < 1.0) ? exp(-tau) / 0.99 : 0.0;
    for (int c = 0; c < 3; ++c) {
      double ck = pow(C[c] / D, 1.0 / 2.2);
      E[c] += (Gk - G) * ck;
      Btot[c] += (gk - gprev) * ck;
    }
    G = Gk;
    gprev = gk;
    if (G >= 1.0) break;
  }
}

static void diff_prepare(dctx *dc, const orc_diff_scene *sc) {
  dc->sc = sc;
  dc->rgb22a3 = (double *)malloc(sizeof(double) * 4 * (size_t)(sc->n > 0 ? sc->n : 1));
  for (int i = 0; i < sc->n; ++i) {
    double t4[4], f;
    int i0;
    tf64(sc->tf, sc->nc, sc->attr[i], t4, &i0, &f);
    double a3 = t4[3] * t4[3] * t4[3];
    dc->rgb22a3[4 * i] = a3;
    for (int c = 0; c < 3; ++c) dc->rgb22a3[4 * i + 1 + c] = pow(t4[c], 2.2) * a3;
  }
}

double orc_diff_forward(const orc_diff_scene *sc, const orc_params *views, int nviews, int w, int h,
                        double *images, int nthreads) {
  dctx dc;
  diff_prepare(&dc, sc);
  long total = (long)nviews * w * h;
  int nt = nthreads > 0 ? nthreads : g_threads;
#ifdef _OPENMP
#pragma omp parallel num_threads(nt > 0 ? nt : omp_get_max_threads())
#endif
  {
    dcand *cands = (dcand *)malloc(sizeof(dcand) * (size_t)(sc->n > 0 ? sc->n : 1));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 8)
#endif
    for (long k = 0; k < total; ++k) {
      int v = (int)(k / ((long)w * h)), pix = (int)(k % ((long)w * h));
      int px = pix % w, py = pix / w;
      const orc_params *p = views + v;
      uint32_t spp = p->spp ? p->spp : 1u;
      double acc[3] = {0, 0, 0};
      for (uint32_t s = 0; s < spp; ++s) {
        dray r = diff_ray(p, px, py, w, h, s);
        if (!r.valid) continue;
        int ncand = diff_cands(sc, &r, cands);
        double E[3], B[3];
        diff_sample_fwd(&dc, p, &r, cands, ncand, E, B);
        for (int c = 0; c < 3; ++c) acc[c] += E[c];
      }
      for (int c = 0; c < 3; ++c) images[3 * k + c] = acc[c] / (double)spp;
    }
    free(cands);
  }
  free(dc.rgb22a3);
  (void)nt;
  return 0.0;
}

void orc_diff_backward(const orc_diff_scene *sc, const orc_params *views, int nviews, int w, int h,
                       const double *grad_images, double *g_pos, double *g_radius, double *g_attr, double *g_tf,
                       int nthreads) {
  dctx dc;
  diff_prepare(&dc, sc);
  const int n = sc->n, nc = sc->nc;
  /* per-particle upstream: dL/d(a^3 weight) and dL/d(rgb^2.2 a^3 weight), chained to the TF at the end */
  size_t nacc = 4 * (size_t)n;
  memset(g_pos, 0, sizeof(double) * 3 * (size_t)n);
  memset(g_radius, 0, sizeof(double) * (size_t)n);
  memset(g_attr, 0, sizeof(double) * (size_t)n);
  memset(g_tf, 0, sizeof(double) * 4 * (size_t)nc);
  double *g_w = (double *)calloc(nacc > 0 ? nacc : 1, sizeof(double));
  long total = (long)nviews * w * h;
  int nt = nthreads > 0 ? nthreads : g_threads;
#ifdef _OPENMP
#pragma omp parallel num_threads(nt > 0 ? nt : omp_get_max_threads())
#endif
  {
    dcand *cands = (dcand *)malloc(sizeof(dcand) * (size_t)(n > 0 ? n : 1));
    int *mem = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    double *rho = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    double *lp = (double *)calloc(3 * (size_t)n + 1, sizeof(double));
    double *lr = (double *)calloc((size_t)n + 1, sizeof(double));
    double *lw = (double *)calloc(nacc + 1, sizeof(double));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 8)
#endif
    for (long k = 0; k < total; ++k) {
      int v = (int)(k / ((long)w * h)), pix = (int)(k % ((long)w * h));
      int px = pix % w, py = pix / w;
      const orc_params *p = views + v;
      uint32_t spp = p->spp ? p->spp : 1u;
      const double unit = (double)p->unit, gain = (double)p->density_gain;
      double g[3];
      for (int c = 0; c < 3; ++c) g[c] = grad_images[3 * k + c] / (double)spp;
      for (uint32_t s = 0; s < spp; ++s) {
        dray r = diff_ray(p, px, py, w, h, s);
        if (!r.valid) continue;
        int ncand = diff_cands(sc, &r, cands);
        double E[3], Btot[3];
        diff_sample_fwd(&dc, p, &r, cands, ncand, E, Btot);
        double tau = 0.0, G = 0.0, gprev = 0.0, P[3] = {0, 0, 0};
        for (int st = 0;; ++st) {
          double t = r.t0 + (double)(st + 1) * unit;
          if (t >= r.tmax) break;
          double D, C[3];
          int nm;
          diff_eval(&dc, &r, cands, ncand, t, &D, C, mem, rho, &nm);
          if (!(D > 0.0)) continue;
          double dens = fmin(gain * D, 1.0);
          tau += dens;
          double Gk = fmin(1.0, (1.0 - exp(-tau)) / 0.99);
          double gk = ((1.0 - exp(-tau)) / 0.99 < 1.0) ? exp(-tau) / 0.99 : 0.0;
          double ck[3], grho = 0.0, gD, gC[3];
          for (int c = 0; c < 3; ++c) {
            ck[c] = pow(C[c] / D, 1.0 / 2.2);
            P[c] += (gk - gprev) * ck[c];
            double S = gk * ck[c] + (Btot[c] - P[c]);
            grho += g[c] * S;
          }
          double wk = Gk - G;
          gD = (gain * D < 1.0) ? grho * gain : 0.0;
          for (int c = 0; c < 3; ++c) {
            double gc = g[c] * wk;
            gD -= gc * ck[c] / (2.2 * D);
            gC[c] = (C[c] > 0.0) ? gc * ck[c] / (2.2 * C[c]) : 0.0;
          }
          double x[3] = {r.o[0] + t * r.d[0], r.o[1] + t * r.d[1], r.o[2] + t * r.d[2]};
          for (int m = 0; m < nm; ++m) {
            int i = mem[m];
            const double *wi = dc.rgb22a3 + 4 * i;
            double gr = gD * wi[0] + gC[0] * wi[1] + gC[1] * wi[2] + gC[2] * wi[3];
            const double *pp = sc->pos + 3 * i;
            double r2 = sc->radius[i] * sc->radius[i], d2 = 0.0;
            for (int a = 0; a < 3; ++a) {
              double dx = x[a] - pp[a];
              d2 += dx * dx;
              lp[3 * i + a] += gr * rho[n + m] * 9.0 * dx / r2;
            }
            lr[i] += gr * rho[n + m] * 9.0 * d2 / (r2 * sc->radius[i]);
            lw[4 * i] += gD * rho[m];
            for (int c = 0; c < 3; ++c) lw[4 * i + 1 + c] += gC[c] * rho[m];
          }
          G = Gk;
          gprev = gk;
          if (G >= 1.0) break;
        }
      }
    }
#ifdef _OPENMP
#pragma omp critical
#endif
    {
      for (size_t j = 0; j < 3 * (size_t)n; ++j) g_pos[j] += lp[j];
      for (int j = 0; j < n; ++j) g_radius[j] += lr[j];
      for (size_t j = 0; j < nacc; ++j) g_w[j] += lw[j];
    }
    free(cands); free(mem); free(rho); free(lp); free(lr); free(lw);
  }
  /* chain the weight gradients to the transfer function and the attribute: the D weight is a^3
   * and the C weights rgb_c^2.2 a^3, so d/da = 3 a^2 (dA3 + sum_c dC_c rgb_c^2.2) and
   * d/drgb_c = dC_c 2.2 rgb_c^1.2 a^3 */
  for (int i = 0; i < n; ++i) {
    double t4[4], f;
    int i0;
    tf64(sc->tf, nc, sc->attr[i], t4, &i0, &f);
    double a = t4[3], a2 = a * a, a3 = a2 * a;
    double gtf[4];
    double ga = g_w[4 * i];
    for (int c = 0; c < 3; ++c) {
      double dC = g_w[4 * i + 1 + c];
      ga += dC * pow(t4[c], 2.2);
      gtf[c] = (t4[c] > 0.0) ? dC * 2.2 * pow(t4[c], 1.2) * a3 : 0.0;
    }
    gtf[3] = ga * 3.0 * a2;
    int j = i0 + 1 < nc ? i0 + 1 : i0;
    double x = sc->attr[i] * (double)nc - 0.5;
    int interior = x > 0.0 && x < (double)(nc - 1);
    for (int c = 0; c < 4; ++c) {
      g_tf[4 * i0 + c] += gtf[c] * (1.0 - f);
      if (j != i0) g_tf[4 * j + c] += gtf[c] * f;
      if (interior) g_attr[i] += gtf[c] * (sc->tf[4 * j + c] - sc->tf[4 * i0 + c]) * (double)nc;
    }
  }
  free(g_w);
  free(dc.rgb22a3);
  (void)nt;
}
