// aarbf_device.cuh -- device-side building blocks shared by the aarbf kernels.
//
// Every float operation here is a single IEEE round-to-nearest operation: the library is
// compiled with -fmad=false and writes fmaf() where a fused step is meant, so a kernel's
// result does not depend on the compiler's contraction choices. exp/log/pow are this
// library's own (Cody-Waite argument reduction + Taylor / atanh series), not CUDA's.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace aarbf {

constexpr int kMaxDepth = 10000;            // MAX_DEPTH, sharedCode.h:27
constexpr uint32_t kLeafBit = 0x80000000u;  // child code: leaf index | kLeafBit
constexpr float kFixScale = 0x1p40f;        // any-hit sums are exact fixed point, 2^-40 units
constexpr float kFixInv = 0x1p-40f;
constexpr int kStackSize = 96;              // >= 48 key bits + 32 index bits of tree depth

// device status bits (or-ed into the context's status word, read by aarbf_sync)
enum : uint32_t {
  kStatusStackOverflow = 1u,
  kStatusBadInput = 2u,
  kStatusLoopCap = 4u,
};

// Iteration bound of a device loop: its built-in bound, or the lower one a launch asks for
// (aarbf_params.loop_cap, which exists to exercise this path). A loop that runs out of
// iterations ors kStatusLoopCap into the status word, so the caller's aarbf_sync reports
// AARBF_ERR_DEVICE_LIMIT instead of returning a truncated result as if it were complete.
__host__ __device__ __forceinline__ int loop_bound(uint32_t requested, int builtin) {
  return (requested != 0u && requested < (uint32_t)builtin) ? (int)requested : builtin;
}

// render flags (match AARBF_FLAG_* in include/aarbf.h)
enum : uint32_t {
  kFlagBlueNoise = 1u << 0,
  kFlagShowNoise = 1u << 1,
  kFlagVisualizeAttributes = 1u << 2,
  kFlagTrackFromEntry = 1u << 3,
  kFlagDensityLinear = 1u << 4,
  kFlagSplatParticleRadius = 1u << 5,
  kFlagMajorantTracking = 1u << 6,
  kFlagCostImage = 1u << 7,
};

// Internal BVH node: the boxes of both children live in the parent, so a traversal step reads
// one 64-byte node and tests two boxes.
struct __align__(16) Node {
  float4 a;  // c0.lo.x c0.lo.y c0.lo.z c0.hi.x
  float4 b;  // c0.hi.y c0.hi.z c1.lo.x c1.lo.y
  float4 c;  // c1.lo.z c1.hi.x c1.hi.y c1.hi.z
  uint4 d;   // child0 code, child1 code, parent, unused
};

// Wide node derived from the binary tree: node n lists up to kBvhWidth descendants of binary
// node n that together cover its subtree (its children, with the inner ones of largest surface
// area replaced by their own children until the node is full), so one traversal step descends
// several binary levels. One 32-byte slot per child: lo.xyz, hi.xyz, child code (bit 31 = leaf;
// 0xffffffff = empty slot). Every binary inner node has its wide node (the same index).
#ifndef AARBF_BVH_WIDTH
#define AARBF_BVH_WIDTH 4
#endif
constexpr int kBvhWidth = AARBF_BVH_WIDTH;
struct __align__(16) WideNode {
  float4 s[2 * kBvhWidth];  // slot k: s[2k] = (lo.x, lo.y, lo.z, hi.x), s[2k+1] = (hi.y, hi.z, code, 0)
};

// ------------------------------------------------------------------------------------------
// deterministic math
// ------------------------------------------------------------------------------------------

__host__ __device__ __forceinline__ float ln2_hi() { return 0x1.62e4p-1f; }
__host__ __device__ __forceinline__ float ln2_lo() { return 0x1.7f7d1cp-20f; }

__device__ __forceinline__ float pow2i(int k) { return __uint_as_float((uint32_t)(k + 127) << 23); }

// natural log: x = m 2^e, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh((m-1)/(m+1)) by series
__device__ __forceinline__ float dlog(float x) {
  if (x != x || x < 0.0f) return __int_as_float(0x7fc00000);
  if (x == 0.0f) return -__int_as_float(0x7f800000);
  if (x == __int_as_float(0x7f800000)) return x;
  int e = 0;
  uint32_t b = __float_as_uint(x);
  if (b < 0x00800000u) {
    x = x * 0x1p23f;
    b = __float_as_uint(x);
    e = -23;
  }
  e += (int)(b >> 23) - 127;
  float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
  if (m > 0x1.6a09e6p+0f) {
    m = m * 0.5f;
    e += 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float z = s * s;
  float p = 0x1.c71c72p-3f;
  p = fmaf(p, z, 0x1.24924ap-2f);
  p = fmaf(p, z, 0x1.99999ap-2f);
  p = fmaf(p, z, 0x1.555556p-1f);
  p = fmaf(p, z, 2.0f);
  float lm = s * p;
  float ef = (float)e;
  return fmaf(ef, ln2_hi(), fmaf(ef, ln2_lo(), lm));
}

// exp: k = rint(x / ln2), r = x - k ln2, Taylor series through r^7, scale by 2^k exactly
__device__ __forceinline__ float dexp(float x) {
  if (x != x) return x;
  if (x > 88.72284f) return __int_as_float(0x7f800000);
  if (x < -103.972084f) return 0.0f;
  float kf = rintf(x * 0x1.715476p+0f);
  float r = fmaf(-kf, ln2_hi(), x);
  r = fmaf(-kf, ln2_lo(), r);
  float p = 0x1.a01a02p-13f;
  p = fmaf(p, r, 0x1.6c16c2p-10f);
  p = fmaf(p, r, 0x1.111112p-7f);
  p = fmaf(p, r, 0x1.555556p-5f);
  p = fmaf(p, r, 0x1.555556p-3f);
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  int k = (int)kf;
  int k1 = k / 2;
  int k2 = k - k1;
  return (p * pow2i(k1)) * pow2i(k2);
}

__device__ __forceinline__ float dpow(float x, float y) {
  if (x != x || y != y) return __int_as_float(0x7fc00000);
  if (x == 0.0f) return (y > 0.0f) ? 0.0f : (y == 0.0f ? 1.0f : __int_as_float(0x7f800000));
  if (x < 0.0f) return __int_as_float(0x7fc00000);
  return dexp(y * dlog(x));
}

__device__ __forceinline__ long long fix40(float v) { return __float2ll_rn(v * kFixScale); }

// ------------------------------------------------------------------------------------------
// small vector helpers (explicit operation order)
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return (ax * bx + ay * by) + az * bz;
}

// v / |v| per component (normalize as v / length(v))
__device__ __forceinline__ float3 normalize3(float3 v) {
  float len = sqrtf(dot3(v.x, v.y, v.z, v.x, v.y, v.z));
  return make_float3(v.x / len, v.y / len, v.z / len);
}

// ------------------------------------------------------------------------------------------
// RNG: murmur3-seeded LCG (rng.h:24-70)
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t rotl32(uint32_t v, unsigned r) { return (v << r) | (v >> (32u - r)); }

__device__ __forceinline__ uint32_t murmur_mix(uint32_t hash, uint32_t k) {
  k *= 0xcc9e2d51u;
  k = rotl32(k, 15);
  k *= 0x1b873593u;
  hash ^= k;
  return rotl32(hash, 13) * 5u + 0xe6546b64u;
}

__device__ __forceinline__ uint32_t murmur_finalize(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

__device__ __forceinline__ uint32_t pixel_seed(uint32_t frame, uint32_t px, uint32_t py, uint32_t w) {
  uint32_t s = murmur_mix(0u, px + py * w);
  s = murmur_mix(s, frame);
  return murmur_finalize(s);
}

__device__ __forceinline__ float lcg_f(uint32_t& state) {
  state = state * 1664525u + 1013904223u;
  return (float)state * 0x1p-32f;
}

// ------------------------------------------------------------------------------------------
// 1-D lookup tables: linear filter between texel centres, clamp to edge
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ void tex_coords(float u, int n, int& i0, int& i1, float& a) {
  float f = u * (float)n - 0.5f;
  if (!(f > -1.0f)) f = -1.0f;
  if (f > (float)n) f = (float)n;
  float fl = floorf(f);
  a = f - fl;
  i0 = (int)fl;
  i1 = i0 + 1;
  i0 = min(max(i0, 0), n - 1);
  i1 = min(max(i1, 0), n - 1);
}

__device__ __forceinline__ float tex1(const float* __restrict__ t, int n, float u) {
  int i0, i1;
  float a;
  tex_coords(u, n, i0, i1, a);
  float v0 = __ldg(t + i0), v1 = __ldg(t + i1);
  return v0 + a * (v1 - v0);
}

__device__ __forceinline__ float4 tex4(const float4* __restrict__ t, int n, float u) {
  int i0, i1;
  float a;
  tex_coords(u, n, i0, i1, a);
  float4 v0 = __ldg(t + i0), v1 = __ldg(t + i1);
  return make_float4(v0.x + a * (v1.x - v0.x), v0.y + a * (v1.y - v0.y), v0.z + a * (v1.z - v0.z),
                     v0.w + a * (v1.w - v0.w));
}

// ------------------------------------------------------------------------------------------
// Hilbert index, 3 axes x 16 bits (hilbert.h:181-225 with nDims = 3, nBits = 16)
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ uint64_t hilbert3x16(uint64_t c0, uint64_t c1, uint64_t c2) {
  // OR-packing lets a coordinate equal to 65536 spill into the next axis field, as in the
  // reference; bits above 48 are dropped by the transpose
  uint64_t packed = (((c2 << 16) | c1) << 16) | c0;
  // bit b of field d goes to bit 3b + d (the reference's bitTranspose), spread by masks
  uint64_t inter = 0;
#pragma unroll
  for (unsigned d = 0; d < 3; ++d) {
    uint64_t x = (packed >> (d * 16)) & 0xffffull;
    x = (x | (x << 16)) & 0x0000ff0000ffull;
    x = (x | (x << 8)) & 0x00f00f00f00full;
    x = (x | (x << 4)) & 0x0c30c30c30c3ull;
    x = (x | (x << 2)) & 0x249249249249ull;
    inter |= x << d;
  }
  inter ^= inter >> 3;
  uint64_t index = 0;
  unsigned rotation = 0;
  uint32_t flip = 0;
#pragma unroll
  for (int b = 45; b >= 0; b -= 3) {
    uint32_t digit = (uint32_t)(inter >> b) & 7u;
    uint32_t v = flip ^ digit;
    digit = ((v >> rotation) | (v << (3u - rotation))) & 7u;
    index = (index << 3) | digit;
    flip = 1u << rotation;
    uint32_t low = digit & (~digit + 1u) & 3u;
    rotation += (low == 1u) ? 1u : ((low == 2u) ? 2u : 0u);
    rotation += 1u;
    if (rotation >= 3u) rotation -= 3u;
  }
  index ^= (0xffffffffffffull / 7ull) >> 1;
#pragma unroll
  for (unsigned d = 1; d < 48; d *= 2) index ^= index >> d;
  return index;
}

// (p - lo) / (hi - lo) * 65536 truncated, clamped to [0, 65536] (hostCode.cpp:200-206)
__device__ __forceinline__ uint64_t quantise16(float v, float lo, float hi) {
  float t = (v - lo) / (hi - lo);
  t = t * 65536.0f;
  if (!(t >= 0.0f)) return 0;
  if (t >= 65536.0f) return 65536;
  return (uint64_t)t;
}

// ------------------------------------------------------------------------------------------
// "over" compositing (sharedCode.h:142-150)
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ float4 over4(float4 a, float4 b) {
  float ra = a.w + b.w * (1.0f - a.w);
  if (ra == 0.0f) return a;
  float4 r;
  r.x = (a.x * a.w + (b.x * b.w) * (1.0f - a.w)) / ra;
  r.y = (a.y * a.w + (b.y * b.w) * (1.0f - a.w)) / ra;
  r.z = (a.z * a.w + (b.z * b.w) * (1.0f - a.w)) / ra;
  r.w = ra;
  return r;
}

// slab test of sharedCode.h:151-185
__device__ __forceinline__ void aabb_clip(float3 o, float3 d, float3 lb, float3 rt, float tmin,
                                          float tmax, float& tenter, float& texit) {
  float fx = 1.0f / d.x, fy = 1.0f / d.y, fz = 1.0f / d.z;
  float t2 = (rt.x - o.x) * fx;
  float t4 = (rt.y - o.y) * fy;
  float t6 = (rt.z - o.z) * fz;
  float t1 = (lb.x - o.x) * fx;
  float t3 = (lb.y - o.y) * fy;
  float t5 = (lb.z - o.z) * fz;
  float te = fmaxf(fmaxf(fminf(t1, t2), fminf(t3, t4)), fminf(t5, t6));
  float tx = fminf(fminf(fmaxf(t1, t2), fmaxf(t3, t4)), fmaxf(t5, t6));
  tenter = fmaxf(te, tmin);
  texit = fminf(tx, tmax);
}

}  // namespace aarbf
