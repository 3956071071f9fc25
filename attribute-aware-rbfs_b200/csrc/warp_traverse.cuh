// warp_traverse.cuh -- ray type, culling tests and the warp-wide BVH traversal shared by the
// tracking kernels (render.cu) and the differentiable kernels (diff.cu).
#pragma once

#include "aarbf_internal.h"

namespace aarbf {

struct Ray {
  float3 o, d;
  float tmin, tmax;
};

__device__ __forceinline__ bool inside(float lx, float ly, float lz, float hx, float hy, float hz, float3 x) {
  return x.x >= lx && x.x <= hx && x.y >= ly && x.y <= hy && x.z >= lz && x.z <= hz;
}

// slab test of a (slack-inflated) box against the ray segment [t0, t1]
__device__ __forceinline__ bool seg_box(float lx, float ly, float lz, float hx, float hy, float hz, float3 o,
                                        float3 inv, float t0, float t1, float eps) {
  float ax = (lx - eps - o.x) * inv.x, bx = (hx + eps - o.x) * inv.x;
  float ay = (ly - eps - o.y) * inv.y, by = (hy + eps - o.y) * inv.y;
  float az = (lz - eps - o.z) * inv.z, bz = (hz + eps - o.z) * inv.z;
  float tn = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), t0));
  float tf = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fminf(fmaxf(az, bz), t1));
  return tn <= tf;
}

// The same test with the per-ray terms folded so each slab end is one fused multiply-add:
// (l - eps - o) inv = l inv + clo, (h + eps - o) inv = h inv + chi. It only culls: its slab ends
// differ from seg_box's by a few ulps of |o inv|, far inside the eps slack (eps >= 2^-18 of every
// coordinate and of the camera position). inv is clamped to +-1e30 so an axis-parallel ray meets
// no inf - inf.
struct SegSlab {
  float3 inv, clo, chi;
  float t0, t1;
  __device__ __forceinline__ void init(float3 o, float3 inv_ray, float eps, float a, float b) {
    inv = make_float3(fminf(fmaxf(inv_ray.x, -1e30f), 1e30f), fminf(fmaxf(inv_ray.y, -1e30f), 1e30f),
                      fminf(fmaxf(inv_ray.z, -1e30f), 1e30f));
    clo = make_float3(-(o.x + eps) * inv.x, -(o.y + eps) * inv.y, -(o.z + eps) * inv.z);
    chi = make_float3((eps - o.x) * inv.x, (eps - o.y) * inv.y, (eps - o.z) * inv.z);
    t0 = a;
    t1 = b;
  }
  __device__ __forceinline__ bool hit(float lx, float ly, float lz, float hx, float hy, float hz) const {
    const float ax = fmaf(lx, inv.x, clo.x), bx = fmaf(hx, inv.x, chi.x);
    const float ay = fmaf(ly, inv.y, clo.y), by = fmaf(hy, inv.y, chi.y);
    const float az = fmaf(lz, inv.z, clo.z), bz = fmaf(hz, inv.z, chi.z);
    const float tn = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), t0));
    const float tf = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fminf(fmaxf(az, bz), t1));
    return tn <= tf;
  }
};

// Conservative [a, b] of the ray parameters at which particle (c, r) can hold a point of the ray
// (sphere inflated by 2^-10 r + eps, interval by eps); false when the ray misses it. Culling only:
// fused steps round differently from the plain ones by far less than the slack.
__device__ __forceinline__ bool sphere_span(float4 c, float3 o, float3 d, float eps, float& a, float& b) {
  const float vx = c.x - o.x, vy = c.y - o.y, vz = c.z - o.z;
  const float tc = fmaf(vz, d.z, fmaf(vy, d.y, vx * d.x));
  const float wx = fmaf(-tc, d.x, vx), wy = fmaf(-tc, d.y, vy), wz = fmaf(-tc, d.z, vz);
  const float h2 = fmaf(wz, wz, fmaf(wy, wy, wx * wx));
  const float R = fmaf(c.w, 1.0f + 0x1p-10f, eps);
  const float R2 = R * R;
  if (h2 > R2) return false;
  const float half = sqrtf(R2 - h2) + eps;
  a = tc - half;
  b = tc + half;
  return true;
}

constexpr int kWarpStack = 8192;      // traversal stack entries per warp (global memory: a shared-memory
                                      // stack costs L1 capacity and measured slower)
constexpr int kMaxSegBins = 64;       // bins per staged segment
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t lane_lt_mask() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Exact warp sums (every lane gets the total). A 64-bit value is cut into limbs of 26, 26 and 12
// bits whose 32-lane sums fit 32 bits, summed by the warp-reduce instruction and put back
// together modulo 2^64: the same integer as a shuffle tree, in three reductions instead of five
// rounds of two shuffles and an add.
__device__ __forceinline__ long long warp_sum(long long v) {
  const unsigned long long u = (unsigned long long)v;
  const unsigned long long s0 = __reduce_add_sync(kFull, (unsigned)(u & 0x3ffffffull));
  const unsigned long long s1 = __reduce_add_sync(kFull, (unsigned)((u >> 26) & 0x3ffffffull));
  const unsigned long long s2 = __reduce_add_sync(kFull, (unsigned)(u >> 52));
  return (long long)(s0 + (s1 << 26) + (s2 << 52));
}

__device__ __forceinline__ int warp_sum(int v) { return __reduce_add_sync(kFull, v); }

// warp-kernel count-mode slots (lane 0 adds warp-uniform values)
enum { kWcSteps = 2, kWcStages = 3, kWcOverflows = 4, kWcDirect = 5, kWcCands = 6, kWcBins = 7,
       kWcIters = 8, kWcParticles = 9 };

__device__ __forceinline__ void wctr(unsigned long long* c, int i, unsigned long long v) {
  if (c && (threadIdx.x & 31u) == 0) atomicAdd(c + i, v);
}

// Warp-wide traversal of a BVH in its wide form (WideNode: kBvhWidth children per node). Each
// step takes up to 32 / kBvhWidth nodes from the warp's stack; lane kBvhWidth j + k tests child k
// of node j with
// box_test(child box) and pushes the inner children it enters (ballot-compacted);
// on_particle(valid, i) is then called by all lanes together for the particles of every entered
// leaf (valid false on padding lanes) and returns false to abort. Returns false on abort or
// stack overflow.
template <class BoxTest, class OnParticle>
__device__ bool warp_traverse_wide(const SceneView& s, const WideNode* wide, uint32_t* stk, uint32_t* leafbuf,
                                   uint32_t* status, BoxTest&& box_test, OnParticle&& on_particle,
                                   unsigned long long* ctr = nullptr) {
  const uint32_t lane = threadIdx.x & 31u, lt = lane_lt_mask();
  if (s.nleaves == 0) return true;
  const uint32_t ppl = s.ppl;
  const bool pow2 = (ppl & (ppl - 1u)) == 0u;
  const uint32_t shift = pow2 ? (uint32_t)__ffs((int)ppl) - 1u : 0u;
  if (s.root & kLeafBit) {
    for (uint32_t b = 0; b < ppl; b += 32) {
      uint32_t j = b + lane;
      bool v = j < ppl && (uint64_t)j < s.n;
      if (!on_particle(v, j)) return false;
    }
    return true;
  }
  if (lane == 0) stk[0] = s.root;
  int sp = 1;
  __syncwarp();
  for (int budget = loop_bound(s.loop_cap, 1 << 24); sp > 0 && budget > 0; --budget) {
    constexpr int kPer = 32 / kBvhWidth;
    const int take = sp < kPer ? sp : kPer;
    const int base = sp - take;
    const int slot = (int)lane / kBvhWidth;
    const bool valid = slot < take;
    const uint32_t node = valid ? stk[base + slot] : 0u;
    __syncwarp();
    sp = base;
    bool hit = false;
    uint32_t code = 0xffffffffu;
    if (valid) {
      const float4* p = wide[node].s + 2 * ((int)lane % kBvhWidth);
      const float4 a = __ldg(p), b = __ldg(p + 1);
      code = __float_as_uint(b.z);
      hit = code != 0xffffffffu && box_test(a.x, a.y, a.z, a.w, b.x, b.y);
    }
    const bool inner = hit && !(code & kLeafBit), leaf = hit && (code & kLeafBit);
    const uint32_t m = __ballot_sync(kFull, inner);
    const int ni = __popc(m);
    if (sp + ni > kWarpStack) {
      if (lane == 0) atomicOr(status, kStatusStackOverflow);
      return false;
    }
    if (inner) stk[sp + __popc(m & lt)] = code;
    sp += ni;
    const uint32_t q = __ballot_sync(kFull, leaf);
    const int nl = __popc(q);
    if (leaf) leafbuf[__popc(q & lt)] = code & ~kLeafBit;
    __syncwarp();
    const uint32_t total = (uint32_t)nl * ppl;
    wctr(ctr, kWcIters, 1);
    wctr(ctr, kWcParticles, total);
    for (uint32_t b = 0; b < total; b += 32) {
      uint32_t j = b + lane;
      bool v = j < total;
      uint64_t i = 0;
      if (v) {
        // leaf slot and offset of entry j: a shift and a mask when ppl is a power of two
        const uint32_t q = pow2 ? j >> shift : j / ppl, r = pow2 ? j & (ppl - 1u) : j - q * ppl;
        i = (uint64_t)leafbuf[q] * ppl + r;
        v = i < s.n;
      }
      if (!on_particle(v, (uint32_t)i)) return false;
    }
    __syncwarp();
  }
  if (sp > 0) {  // the iteration bound ran out: a truncated traversal, reported
    if (lane == 0) atomicOr(status, kStatusLoopCap);
    return false;
  }
  return true;
}

// the traversal-bounds BVH (particles that can be hit)
template <class BoxTest, class OnParticle>
__device__ __forceinline__ bool warp_traverse(const SceneView& s, uint32_t* stk, uint32_t* leafbuf, uint32_t* status,
                                              BoxTest&& box_test, OnParticle&& on_particle,
                                              unsigned long long* ctr = nullptr) {
  return warp_traverse_wide(s, s.wide, stk, leafbuf, status, box_test, on_particle, ctr);
}

}  // namespace aarbf
