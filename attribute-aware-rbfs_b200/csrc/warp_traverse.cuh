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

constexpr int kWarpStack = 8192;      // traversal stack entries per warp (global memory: a shared-memory
                                      // stack costs L1 capacity and measured slower)
constexpr int kMaxSegBins = 64;       // bins per staged segment
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t lane_lt_mask() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ long long warp_sum(long long v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// warp-kernel count-mode slots (lane 0 adds warp-uniform values)
enum { kWcSteps = 2, kWcStages = 3, kWcOverflows = 4, kWcDirect = 5, kWcCands = 6, kWcBins = 7,
       kWcIters = 8, kWcParticles = 9 };

__device__ __forceinline__ void wctr(unsigned long long* c, int i, unsigned long long v) {
  if (c && (threadIdx.x & 31u) == 0) atomicAdd(c + i, v);
}

// Warp-wide traversal of a BVH over the scene's topology: `nodes` is one of its node arrays
// (traversal bounds s.nodes, reference bounds s.nodes_ref). box_test(child box) decides which
// children to enter; on_particle(valid, i) is called by all lanes together for the particles of
// every entered leaf (valid false on padding lanes) and returns false to abort. Returns false on
// abort or stack overflow.
template <class BoxTest, class OnParticle>
__device__ bool warp_traverse_nodes(const SceneView& s, const Node* nodes, uint32_t* stk, uint32_t* leafbuf,
                                    uint32_t* status, BoxTest&& box_test, OnParticle&& on_particle,
                                    unsigned long long* ctr = nullptr) {
  const uint32_t lane = threadIdx.x & 31u, lt = lane_lt_mask();
  if (s.nleaves == 0) return true;
  const uint32_t ppl = s.ppl;
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
  for (int guard = 0; sp > 0 && guard < (1 << 24); ++guard) {
    const int take = sp < 32 ? sp : 32;
    const int base = sp - take;
    const bool valid = (int)lane < take;
    uint32_t node = valid ? stk[base + lane] : 0u;
    __syncwarp();
    sp = base;
    bool h0 = false, h1 = false;
    uint2 ch = make_uint2(0u, 0u);
    if (valid) {
      const Node* nd = nodes + node;
      float4 a = __ldg(&nd->a), b = __ldg(&nd->b), c = __ldg(&nd->c);
      ch = __ldg(reinterpret_cast<const uint2*>(&nd->d));
      h0 = box_test(a.x, a.y, a.z, a.w, b.x, b.y);
      h1 = box_test(b.z, b.w, c.x, c.y, c.z, c.w);
    }
    const bool i0 = h0 && !(ch.x & kLeafBit), i1 = h1 && !(ch.y & kLeafBit);
    const bool l0 = h0 && (ch.x & kLeafBit), l1 = h1 && (ch.y & kLeafBit);
    const uint32_t m0 = __ballot_sync(kFull, i0), m1 = __ballot_sync(kFull, i1);
    const int n0 = __popc(m0), n1 = __popc(m1);
    if (sp + n0 + n1 > kWarpStack) {
      if (lane == 0) atomicOr(status, kStatusStackOverflow);
      return false;
    }
    if (i0) stk[sp + __popc(m0 & lt)] = ch.x;
    if (i1) stk[sp + n0 + __popc(m1 & lt)] = ch.y;
    sp += n0 + n1;
    const uint32_t q0 = __ballot_sync(kFull, l0), q1 = __ballot_sync(kFull, l1);
    const int c0 = __popc(q0), nl = c0 + __popc(q1);
    if (l0) leafbuf[__popc(q0 & lt)] = ch.x & ~kLeafBit;
    if (l1) leafbuf[c0 + __popc(q1 & lt)] = ch.y & ~kLeafBit;
    __syncwarp();
    const uint32_t total = (uint32_t)nl * ppl;
    wctr(ctr, kWcIters, 1);
    wctr(ctr, kWcParticles, total);
    for (uint32_t b = 0; b < total; b += 32) {
      uint32_t j = b + lane;
      bool v = j < total;
      uint64_t i = 0;
      if (v) {
        uint32_t leaf = leafbuf[j / ppl];
        i = (uint64_t)leaf * ppl + (j % ppl);
        v = i < s.n;
      }
      if (!on_particle(v, (uint32_t)i)) return false;
    }
    __syncwarp();
  }
  return true;
}

// the traversal-bounds BVH (particles that can be hit)
template <class BoxTest, class OnParticle>
__device__ __forceinline__ bool warp_traverse(const SceneView& s, uint32_t* stk, uint32_t* leafbuf, uint32_t* status,
                                              BoxTest&& box_test, OnParticle&& on_particle,
                                              unsigned long long* ctr = nullptr) {
  return warp_traverse_nodes(s, s.nodes, stk, leafbuf, status, box_test, on_particle, ctr);
}

}  // namespace aarbf
