// render.cu -- ParticleRBFRayGen + ParticleTracker + ParticleRBFIntersection/AnyHit
// (deviceCodeRBF.hlsl:40-389) as one CUDA kernel.
//
// The reference issues one zero-length ray per tracking step and lets the RT cores find every
// leaf box containing the step point. Here the density at a step point is the exact sum over
// particles with |x - p| < r, accumulated in 64-bit fixed point (2^-40 units), so the result does
// not depend on the order particles are visited. Two traversal strategies give identical bits:
//   STAGED: a ray is cut into segments; one BVH traversal per segment stages every particle whose
//           (slightly inflated) sphere meets the segment, with its ray-parameter interval, in
//           shared memory; each step then only scans the staged list. A segment whose candidates
//           overflow the buffer is halved; below a minimum length the steps fall back to POINT.
//   POINT:  one stack-based BVH point query per step (the reference's shape).
#include <cuda_fp16.h>

#include "aarbf_internal.h"
#include "warp_traverse.cuh"

#include <memory>

// Compiled twice: AARBF_RENDER_NS = r32 reads the fp32 prepass records, r16 the packed FP16
// storage form (AARBF_FP16_RECORDS); each build has no branch on the format in its hot loops.
#ifndef AARBF_RENDER_NS
#define AARBF_RENDER_NS r32
#endif
#ifndef AARBF_FP16_RECORDS
#define AARBF_FP16_RECORDS 0
#endif

namespace aarbf {
namespace AARBF_RENDER_NS {

namespace {

constexpr int kBlock = 128;  // 16 x 8 pixel tile per block


// count-mode instrumentation: indices into RenderLaunch::counters
enum { kCtrSteps = 2, kCtrStages = 3, kCtrOverflows = 4, kCtrPointQueries = 5, kCtrCandChecks = 6,
       kCtrEvals = 7, kCtrStageNodes = 8, kCtrPointNodes = 9 };

__device__ __forceinline__ void ctr_add(unsigned long long* c, int i, unsigned long long v) {
  if (c) atomicAdd(c + i, v);
}

// Particle records: the fp32 prepass arrays, or the packed FP16 storage form (fp16.cu); both
// decode to the same floats.
#if AARBF_FP16_RECORDS
__device__ __forceinline__ float hval16(uint32_t b) { return __half2float(__ushort_as_half((unsigned short)b)); }

__device__ __forceinline__ float4 part_rec(const SceneView& s, uint32_t i) {
  const uint2 q = __ldg(s.posq + i);
  const float4 o = __ldg(s.origin + (i >> 8));
  return make_float4(o.x + hval16(q.x & 0xffffu), o.y + hval16(q.x >> 16), o.z + hval16(q.y & 0xffffu),
                     __ldg(s.reval + i));
}

// the staging test's record: the position and the FP16 radius rounded up, so the staged spans
// are a superset of the exact ones (the sums evaluate every candidate with the fp32 radius)
__device__ __forceinline__ float4 part_cull(const SceneView& s, uint32_t i) {
  const uint2 q = __ldg(s.posq + i);
  const float4 o = __ldg(s.origin + (i >> 8));
  return make_float4(o.x + hval16(q.x & 0xffffu), o.y + hval16(q.x >> 16), o.z + hval16(q.y & 0xffffu),
                     hval16(q.y >> 16));
}

__device__ __forceinline__ float part_a3(const SceneView& s, uint32_t i) { return hval16(__ldg(&s.colq[i].y) >> 16); }

__device__ __forceinline__ float4 part_w(const SceneView& s, uint32_t i) {
  const uint2 c = __ldg(s.colq + i);
  return make_float4(hval16(c.y >> 16), hval16(c.x & 0xffffu), hval16(c.x >> 16), hval16(c.y & 0xffffu));
}
#else
__device__ __forceinline__ float4 part_rec(const SceneView& s, uint32_t i) { return __ldg(s.rec0 + i); }
__device__ __forceinline__ float4 part_cull(const SceneView& s, uint32_t i) { return part_rec(s, i); }
__device__ __forceinline__ float part_a3(const SceneView& s, uint32_t i) { return __ldg(&s.w4[i].x); }
__device__ __forceinline__ float4 part_w(const SceneView& s, uint32_t i) { return __ldg(s.w4 + i); }
#endif

struct Sample {
  int count;
  long long a0, a1, a2, a3;
};

__device__ __forceinline__ void sample_clear(Sample& s) {
  s.count = 0;
  s.a0 = s.a1 = s.a2 = s.a3 = 0;
}

__device__ __forceinline__ void eval_particle(const SceneView& s, uint32_t i, float3 x, Sample& acc) {
  float4 r = part_rec(s, i);
  float dx = r.x - x.x, dy = r.y - x.y, dz = r.z - x.z;
  float dist = sqrtf((dx * dx + dy * dy) + dz * dz);
  if (!(dist < r.w)) return;
  float q = (dist * 3.0f) / r.w;  // evaluate_rbf, sigma = 3 (sharedCode.h:137-140)
  float rho = dexp(-0.5f * (q * q));
  float4 w = part_w(s, i);
  acc.count += 1;
  acc.a0 += fix40(rho * w.x);
  acc.a1 += fix40(rho * w.y);
  acc.a2 += fix40(rho * w.z);
  acc.a3 += fix40(rho * w.w);
}

// the density part of eval_particle only: the hot loops need the colour sums only at a collision
__device__ __forceinline__ void eval_density(const SceneView& s, uint32_t i, float3 x, int& count, long long& a0) {
  float4 r = part_rec(s, i);
  float dx = r.x - x.x, dy = r.y - x.y, dz = r.z - x.z;
  float dist = sqrtf((dx * dx + dy * dy) + dz * dz);
  if (!(dist < r.w)) return;
  float q = (dist * 3.0f) / r.w;
  float rho = dexp(-0.5f * (q * q));
  count += 1;
  a0 += fix40(rho * part_a3(s, i));
}

__device__ __forceinline__ void eval_leaf(const SceneView& s, uint32_t leaf, float3 x, Sample& acc) {
  uint64_t b = (uint64_t)leaf * s.ppl;
  uint64_t e = b + s.ppl;
  if (e > s.n) e = s.n;
  for (uint64_t i = b; i < e; ++i) eval_particle(s, (uint32_t)i, x, acc);
}


// POINT: every leaf whose box contains x, then the exact particle test
__device__ void point_query(const SceneView& s, float3 x, Sample& acc, uint32_t* status,
                            unsigned long long* ctr = nullptr) {
  sample_clear(acc);
  ctr_add(ctr, kCtrPointQueries, 1);
  if (s.nleaves == 0) return;
  if (!inside(s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1], s.root_hi[2], x)) return;
  if (s.root & kLeafBit) {
    eval_leaf(s, s.root & ~kLeafBit, x, acc);
    return;
  }
  uint32_t stack[kStackSize];
  int sp = 0;
  uint32_t node = s.root;
  unsigned long long visits = 0;
  while (true) {
    ++visits;
    const Node* nd = s.nodes + node;
    float4 a = __ldg(&nd->a), b = __ldg(&nd->b), c = __ldg(&nd->c);
    uint2 ch = __ldg(reinterpret_cast<const uint2*>(&nd->d));
    bool h0 = inside(a.x, a.y, a.z, a.w, b.x, b.y, x);
    bool h1 = inside(b.z, b.w, c.x, c.y, c.z, c.w, x);
    if (h0 && (ch.x & kLeafBit)) {
      eval_leaf(s, ch.x & ~kLeafBit, x, acc);
      h0 = false;
    }
    if (h1 && (ch.y & kLeafBit)) {
      eval_leaf(s, ch.y & ~kLeafBit, x, acc);
      h1 = false;
    }
    if (h0 && h1) {
      if (sp == kStackSize) {
        atomicOr(status, kStatusStackOverflow);
        return;
      }
      stack[sp++] = ch.y;
      node = ch.x;
    } else if (h0) {
      node = ch.x;
    } else if (h1) {
      node = ch.y;
    } else {
      if (sp == 0) break;
      node = stack[--sp];
    }
  }
  ctr_add(ctr, kCtrPointNodes, visits);
}


// Per-thread staged candidate buffer, structure-of-arrays in shared memory:
// entry j of thread t lives at [j * kBlock + t].
template <int CAP>
struct Stager {
  uint32_t* idx;
  float* lo;
  float* hi;
  int ncand;       // -1: point-query mode for the current segment
  float seg_end;   // the staged segment covers steps with t < seg_end
  float len;       // current segment length
  float len_min, len_max;
  float rb_enter, rb_exit;  // ray interval inside the inflated root box
  float3 inv;
  unsigned long long* ctr;  // count mode only

  __device__ void init(const SceneView& s, const Ray& ray, float unit, char* smem, unsigned long long* counters) {
    const int t = threadIdx.x;
    ctr = counters;
    idx = reinterpret_cast<uint32_t*>(smem) + t;
    lo = reinterpret_cast<float*>(smem + sizeof(uint32_t) * CAP * kBlock) + t;
    hi = reinterpret_cast<float*>(smem + (sizeof(uint32_t) + sizeof(float)) * CAP * kBlock) + t;
    ncand = 0;
    seg_end = -__int_as_float(0x7f800000);
    len_min = unit * 0.25f;
    len_max = unit * 64.0f;
    len = unit * 16.0f;
    inv = make_float3(1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z);
    float e = s.eps * 4.0f;
    float ax = (s.root_lo[0] - e - ray.o.x) * inv.x, bx = (s.root_hi[0] + e - ray.o.x) * inv.x;
    float ay = (s.root_lo[1] - e - ray.o.y) * inv.y, by = (s.root_hi[1] + e - ray.o.y) * inv.y;
    float az = (s.root_lo[2] - e - ray.o.z) * inv.z, bz = (s.root_hi[2] + e - ray.o.z) * inv.z;
    rb_enter = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz));
    rb_exit = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
    if (s.nleaves == 0 || !(rb_enter <= rb_exit)) {
      rb_enter = __int_as_float(0x7f800000);
      rb_exit = -__int_as_float(0x7f800000);
    }
  }

  __device__ __forceinline__ bool push(uint32_t i, float a, float b) {
    if (ncand == CAP) return false;
    idx[ncand * kBlock] = i;
    lo[ncand * kBlock] = a;
    hi[ncand * kBlock] = b;
    ++ncand;
    return true;
  }

  // stage all particles whose inflated sphere meets [t0, t1]; false on buffer overflow
  __device__ bool stage(const SceneView& s, const Ray& ray, float t0, float t1, uint32_t* status) {
    ncand = 0;
    ctr_add(ctr, kCtrStages, 1);
    const float eps = s.eps;
    uint32_t stack[kStackSize];
    int sp = 0;
    uint32_t node = s.root;
    const bool root_leaf = (s.root & kLeafBit) != 0;
    uint32_t leaves[2];
    while (true) {
      int nl = 0;
      uint32_t next0 = 0xffffffffu, next1 = 0xffffffffu;
      if (root_leaf) {
        leaves[nl++] = s.root & ~kLeafBit;
      } else {
        ctr_add(ctr, kCtrStageNodes, 1);
        const Node* nd = s.nodes + node;
        float4 a = __ldg(&nd->a), b = __ldg(&nd->b), c = __ldg(&nd->c);
        uint2 ch = __ldg(reinterpret_cast<const uint2*>(&nd->d));
        bool h0 = seg_box(a.x, a.y, a.z, a.w, b.x, b.y, ray.o, inv, t0, t1, eps);
        bool h1 = seg_box(b.z, b.w, c.x, c.y, c.z, c.w, ray.o, inv, t0, t1, eps);
        if (h0) {
          if (ch.x & kLeafBit) leaves[nl++] = ch.x & ~kLeafBit;
          else next0 = ch.x;
        }
        if (h1) {
          if (ch.y & kLeafBit) leaves[nl++] = ch.y & ~kLeafBit;
          else next1 = ch.y;
        }
      }
      for (int k = 0; k < nl; ++k) {
        uint64_t b0 = (uint64_t)leaves[k] * s.ppl;
        uint64_t e0 = b0 + s.ppl;
        if (e0 > s.n) e0 = s.n;
        for (uint64_t i = b0; i < e0; ++i) {
          float4 r = part_rec(s, i);
          if (!(r.w > 0.0f)) continue;
          float vx = r.x - ray.o.x, vy = r.y - ray.o.y, vz = r.z - ray.o.z;
          float tc = (vx * ray.d.x + vy * ray.d.y) + vz * ray.d.z;
          float wx = vx - tc * ray.d.x, wy = vy - tc * ray.d.y, wz = vz - tc * ray.d.z;
          float h2 = (wx * wx + wy * wy) + wz * wz;
          float R = r.w * (1.0f + 0x1p-10f) + eps;
          float R2 = R * R;
          if (h2 > R2) continue;
          float half = sqrtf(R2 - h2) + eps;
          float a = tc - half, b = tc + half;
          if (b < t0 || a > t1) continue;
          if (!push((uint32_t)i, a, b)) return false;
        }
      }
      if (root_leaf) return true;
      if (next0 != 0xffffffffu && next1 != 0xffffffffu) {
        if (sp == kStackSize) {
          atomicOr(status, kStatusStackOverflow);
          return true;
        }
        stack[sp++] = next1;
        node = next0;
      } else if (next0 != 0xffffffffu) {
        node = next0;
      } else if (next1 != 0xffffffffu) {
        node = next1;
      } else {
        if (sp == 0) return true;
        node = stack[--sp];
      }
    }
  }

  // make sure the step at t is covered by the staged segment
  __device__ void cover(const SceneView& s, const Ray& ray, float t, uint32_t* status) {
    if (t < seg_end) return;
    if (t < rb_enter) {  // before the scene: nothing can be hit
      ncand = 0;
      seg_end = rb_enter;
      return;
    }
    if (t > rb_exit) {  // past the scene
      ncand = 0;
      seg_end = __int_as_float(0x7f800000);
      return;
    }
    for (int guard = 0; guard < 64; ++guard) {
      float te = t + len;
      if (!(te > t)) break;
      if (stage(s, ray, t, te, status)) {
        seg_end = te;
        len = fminf(len * 2.0f, len_max);
        return;
      }
      ctr_add(ctr, kCtrOverflows, 1);
      len = len * 0.5f;
      if (len < len_min) break;
    }
    // dense or degenerate: point queries until t + len_min
    ncand = -1;
    float te = t + len_min;
    seg_end = (te > t) ? te : t;
    len = len_min * 4.0f;
  }

  __device__ __forceinline__ void sample(const SceneView& s, float t, float3 x, Sample& acc, uint32_t* status) {
    if (ncand < 0) {
      point_query(s, x, acc, status, ctr);
      return;
    }
    sample_clear(acc);
    unsigned long long ev = 0;
    for (int j = 0; j < ncand; ++j) {
      float a = lo[j * kBlock], b = hi[j * kBlock];
      if (t < a || t > b) continue;
      ++ev;
      eval_particle(s, idx[j * kBlock], x, acc);
    }
    ctr_add(ctr, kCtrCandChecks, (unsigned long long)ncand);
    ctr_add(ctr, kCtrEvals, ev);
  }
};

// Count mode (roofline accounting, not timed): the particles whose sphere meets the traversed
// segment [t0, t1] of a ray (exact test, no slack) and the BVH nodes a segment query visits.
// out of line: count mode only, kept out of the tracking kernels' instruction stream and frame
__device__ __noinline__ void count_segment(const RenderLaunch& L, const Ray ray, float t0, float t1) {
  const SceneView& s = L.s;
  if (s.nleaves == 0 || !(t1 >= t0)) return;
  const float3 inv = make_float3(1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z);
  unsigned long long parts = 0, visits = 0;
  uint32_t stack[kStackSize];
  int sp = 0;
  uint32_t node = s.root;
  const bool root_leaf = (s.root & kLeafBit) != 0;
  while (true) {
    uint32_t leaves[2];
    int nl = 0;
    uint32_t n0 = 0xffffffffu, n1 = 0xffffffffu;
    if (root_leaf) {
      leaves[nl++] = s.root & ~kLeafBit;
    } else {
      ++visits;
      const Node* nd = s.nodes + node;
      float4 a = __ldg(&nd->a), b = __ldg(&nd->b), c = __ldg(&nd->c);
      uint2 ch = __ldg(reinterpret_cast<const uint2*>(&nd->d));
      if (seg_box(a.x, a.y, a.z, a.w, b.x, b.y, ray.o, inv, t0, t1, 0.0f)) {
        if (ch.x & kLeafBit) leaves[nl++] = ch.x & ~kLeafBit;
        else n0 = ch.x;
      }
      if (seg_box(b.z, b.w, c.x, c.y, c.z, c.w, ray.o, inv, t0, t1, 0.0f)) {
        if (ch.y & kLeafBit) leaves[nl++] = ch.y & ~kLeafBit;
        else n1 = ch.y;
      }
    }
    for (int k = 0; k < nl; ++k) {
      uint64_t b0 = (uint64_t)leaves[k] * s.ppl, e0 = b0 + s.ppl;
      if (e0 > s.n) e0 = s.n;
      for (uint64_t i = b0; i < e0; ++i) {
        float4 r = part_rec(s, i);
        if (!(r.w > 0.0f)) continue;
        float vx = r.x - ray.o.x, vy = r.y - ray.o.y, vz = r.z - ray.o.z;
        float tc = (vx * ray.d.x + vy * ray.d.y) + vz * ray.d.z;
        float wx = vx - tc * ray.d.x, wy = vy - tc * ray.d.y, wz = vz - tc * ray.d.z;
        float h2 = (wx * wx + wy * wy) + wz * wz;
        float R2 = r.w * r.w;
        if (h2 >= R2) continue;
        float half = sqrtf(R2 - h2);
        if (tc + half < t0 || tc - half > t1) continue;
        ++parts;
      }
    }
    if (root_leaf) break;
    if (n0 != 0xffffffffu && n1 != 0xffffffffu) {
      if (sp == kStackSize) break;
      stack[sp++] = n1;
      node = n0;
    } else if (n0 != 0xffffffffu) {
      node = n0;
    } else if (n1 != 0xffffffffu) {
      node = n1;
    } else {
      if (sp == 0) break;
      node = stack[--sp];
    }
  }
  atomicAdd(L.counters + 0, parts);
  atomicAdd(L.counters + 1, visits);
}

struct Tracker {
  int i;
  float random;
  uint32_t rng;
  float4 albedo;
  float t;
  float lhs;
  bool shadow;
  bool marching;
};

__device__ __forceinline__ float sample_density(const RenderLaunch& L, float D) {
  if (L.flags & kFlagDensityLinear) return fminf(D * L.density_gain, 1.0f);
  return tex1(L.s.tf_density, L.s.nd, D);
}

// out of line: runs once per collision, and keeps three pow expansions out of the hot loops
__device__ __noinline__ float3 sample_color(const RenderLaunch& L, const Sample acc, float D) {
  if (L.flags & kFlagVisualizeAttributes) {
    const float g = 1.0f / 2.2f;
    float c0 = (float)acc.a1 * kFixInv, c1 = (float)acc.a2 * kFixInv, c2 = (float)acc.a3 * kFixInv;
    return make_float3(dpow(c0 / D, g), dpow(c1 / D, g), dpow(c2 / D, g));
  }
  float4 c = tex4(L.s.tf_color, L.s.nc, D);
  return make_float3(c.x, c.y, c.z);
}

template <int CAP>
__device__ __forceinline__ void do_sample(const RenderLaunch& L, Stager<CAP>& st, const Ray& ray, float t, float3 x,
                                          Sample& acc) {
  if (L.traversal == AARBF_TRAVERSAL_POINT) {
    point_query(L.s, x, acc, L.status, L.counters);
  } else {
    st.cover(L.s, ray, t, L.status);
    st.sample(L.s, t, x, acc, L.status);
  }
}

// stochasticTracking (deviceCodeRBF.hlsl:141-203)
template <int CAP>
__device__ void track_delta(const RenderLaunch& L, Tracker& tr, const Ray& ray, bool from_entry, char* smem) {
  Stager<CAP> st;
  st.init(L.s, ray, L.unit, smem, L.counters);
  if (!from_entry) tr.t = ray.tmin;
  for (; tr.i < kMaxDepth; ++tr.i) {
    float u = lcg_f(tr.rng);
    float step = (dlog(1.0f - u) / 1.0f) * L.unit;
    tr.t = tr.t - step;
    if (tr.t >= ray.tmax) return;
    float3 x = make_float3(ray.o.x + tr.t * ray.d.x, ray.o.y + tr.t * ray.d.y, ray.o.z + tr.t * ray.d.z);
    Sample acc;
    do_sample<CAP>(L, st, ray, tr.t, x, acc);
    if (acc.count == 0) continue;
    float D = (float)acc.a0 * kFixInv;
    float density = sample_density(L, D);
    if (lcg_f(tr.rng) < density / 1.0f) {
      float3 c = sample_color(L, acc, D);
      tr.albedo = make_float4(c.x, c.y, c.z, 1.0f);
      return;
    }
  }
}

// stochasticMarching (deviceCodeRBF.hlsl:67-139)
template <int CAP>
__device__ void track_march(const RenderLaunch& L, Tracker& tr, const Ray& ray, char* smem) {
  Stager<CAP> st;
  st.init(L.s, ray, L.unit, smem, L.counters);
  float rhs = -dlog(1.0f - tr.random * 0.99f);
  for (; tr.i < kMaxDepth; ++tr.i) {
    tr.t = tr.t + L.unit;
    if (tr.t >= ray.tmax) return;
    float3 x = make_float3(ray.o.x + tr.t * ray.d.x, ray.o.y + tr.t * ray.d.y, ray.o.z + tr.t * ray.d.z);
    Sample acc;
    do_sample<CAP>(L, st, ray, tr.t, x, acc);
    float D = (float)acc.a0 * kFixInv;
    if (!(acc.count > 0 && D > 0.0f)) continue;
    float density = sample_density(L, D);
    tr.lhs = tr.lhs + density;
    if (tr.lhs > rhs && !tr.shadow) {
      float3 c = sample_color(L, acc, D);
      tr.albedo = make_float4(c.x, c.y, c.z, 1.0f);
      return;
    }
    if (tr.shadow) {
      tr.albedo.w = tr.albedo.w + (1.0f - dexp(-density));
      if (tr.albedo.w >= 1.0f) {
        tr.albedo.w = 1.0f;
        return;
      }
    }
  }
}

// ---- delta tracking with per-bin majorants (native mode) -----------------------------------
// Bins [t0 + k L, t0 + (k+1) L) along the ray. Majorant of a bin = density_scale (1 + 2^-7) times
// the exact fixed-point sum over particles whose sphere meets the bin's segment of a^3 rho at
// their closest approach to the segment. The staged candidates of a run of bins serve both the
// majorants and the density at tentative collisions; runs of empty bins are skipped without
// drawing random numbers, which leaves the sample stream unchanged.

// a bin is split in halves while majorant * length (its expected number of tentative steps)
// exceeds kSplitSteps, at most kSplitDepth times: tight majorants across steep density gradients
constexpr float kSplitSteps = 4.0f;
constexpr int kSplitDepth = 10;

// a^3 rho at particle i's closest approach to [b0, b1]; 0 when its sphere misses the segment
__device__ __forceinline__ float bin_contrib(const SceneView& s, const Ray& ray, uint32_t i, float b0, float b1) {
  float4 r = part_rec(s, i);
  float vx = r.x - ray.o.x, vy = r.y - ray.o.y, vz = r.z - ray.o.z;
  float tc = (vx * ray.d.x + vy * ray.d.y) + vz * ray.d.z;
  float wx = vx - tc * ray.d.x, wy = vy - tc * ray.d.y, wz = vz - tc * ray.d.z;
  float h2 = (wx * wx + wy * wy) + wz * wz;
  float tcl = fminf(fmaxf(tc, b0), b1);
  float dt = tcl - tc;
  float d2 = h2 + dt * dt;
  float r2 = r.w * r.w;
  if (!(d2 < r2)) return 0.0f;
  float q2 = (9.0f * d2) / r2;
  return dexp(-0.5f * q2) * part_a3(s, i);
}

// majorant sum of one bin without a buffer: every particle of every leaf whose inflated box
// meets the bin (used when a single bin holds more candidates than the staging buffer)
__device__ long long bin_sum_direct(const SceneView& s, const Ray& ray, float3 inv, float b0, float b1,
                                    uint32_t* status, unsigned long long* ctr) {
  long long acc = 0;
  if (s.nleaves == 0) return 0;
  uint32_t stack[kStackSize];
  int sp = 0;
  uint32_t node = s.root;
  const bool root_leaf = (s.root & kLeafBit) != 0;
  while (true) {
    uint32_t leaves[2];
    int nl = 0;
    uint32_t n0 = 0xffffffffu, n1 = 0xffffffffu;
    if (root_leaf) {
      leaves[nl++] = s.root & ~kLeafBit;
    } else {
      ctr_add(ctr, kCtrStageNodes, 1);
      const Node* nd = s.nodes + node;
      float4 a = __ldg(&nd->a), b = __ldg(&nd->b), c = __ldg(&nd->c);
      uint2 ch = __ldg(reinterpret_cast<const uint2*>(&nd->d));
      if (seg_box(a.x, a.y, a.z, a.w, b.x, b.y, ray.o, inv, b0, b1, s.eps)) {
        if (ch.x & kLeafBit) leaves[nl++] = ch.x & ~kLeafBit;
        else n0 = ch.x;
      }
      if (seg_box(b.z, b.w, c.x, c.y, c.z, c.w, ray.o, inv, b0, b1, s.eps)) {
        if (ch.y & kLeafBit) leaves[nl++] = ch.y & ~kLeafBit;
        else n1 = ch.y;
      }
    }
    for (int k = 0; k < nl; ++k) {
      uint64_t e0 = (uint64_t)leaves[k] * s.ppl + s.ppl;
      if (e0 > s.n) e0 = s.n;
      for (uint64_t i = (uint64_t)leaves[k] * s.ppl; i < e0; ++i) acc += fix40(bin_contrib(s, ray, (uint32_t)i, b0, b1));
    }
    if (root_leaf) break;
    if (n0 != 0xffffffffu && n1 != 0xffffffffu) {
      if (sp == kStackSize) {
        atomicOr(status, kStatusStackOverflow);
        break;
      }
      stack[sp++] = n1;
      node = n0;
    } else if (n0 != 0xffffffffu) {
      node = n0;
    } else if (n1 != 0xffffffffu) {
      node = n1;
    } else {
      if (sp == 0) break;
      node = stack[--sp];
    }
  }
  return acc;
}

template <int CAP>
__device__ void track_majorant(const RenderLaunch& L, Tracker& tr, const Ray& ray, char* smem) {
  Stager<CAP> st;
  st.init(L.s, ray, L.unit, smem, L.counters);
  const float Lb = L.bin_length;
  const float scale = L.density_scale;
  const float minf = scale * 1.0078125f;
  const float t0 = tr.t;
  int k = 0;
  float t = t0;
  int seg_end = 0;   // bins below seg_end are covered by the staged candidates
  int nb = L.stage_bins;  // bins per staging
  bool direct = false;
  const int cap = loop_bound(L.s.loop_cap, 1 << 26);
  int guard = 0;
  for (; guard < cap; ++guard) {
    float b0 = t0 + (float)k * Lb;
    float b1 = t0 + (float)(k + 1) * Lb;
    if (!(b0 < ray.tmax) || !(b1 > b0)) break;
    if (k >= seg_end) {
      // bins ending before the scene's root box are empty
      if (b1 < st.rb_enter) {
        int ks = (int)floorf((st.rb_enter - t0) / Lb) - 1;
        if (ks > k) {
          k = ks;
          t = t0 + (float)k * Lb;
          continue;
        }
      }
      if (b0 > st.rb_exit) break;  // nothing further along the ray
      direct = false;
      for (;;) {
        float te = t0 + (float)(k + nb) * Lb;
        if (st.stage(L.s, ray, b0, te, L.status)) {
          seg_end = k + nb;
          if (nb < 64) nb *= 2;
          break;
        }
        ctr_add(L.counters, kCtrOverflows, 1);
        nb >>= 1;
        if (nb == 0) {
          direct = true;
          seg_end = k + 1;
          nb = 1;
          break;
        }
      }
      if (!direct) {
        if (st.ncand == 0) {  // the whole staged run is empty
          k = seg_end;
          t = t0 + (float)k * Lb;
          continue;
        }
        float lo_min = __int_as_float(0x7f800000);
        for (int j = 0; j < st.ncand; ++j) lo_min = fminf(lo_min, st.lo[j * kBlock]);
        int ks = (int)floorf((lo_min - t0) / Lb) - 1;
        if (ks > k && ks < seg_end) {
          k = ks;
          t = t0 + (float)k * Lb;
          continue;
        }
      }
    }
    // [b0, b1), split in halves (front first) while majorant * length > kSplitSteps
    // [b0, b1) and its halves: path bit l set = the interval at level l + 1 is the upper half;
    // a pending upper half is replayed from [b0, b1) by the same midpoint operations, so its
    // floats are those a stack of pending intervals would hold
    float lo = b0, hi = b1;
    int depth = 0;
    uint32_t path = 0;
    for (;;) {
      long long acc = 0;
      if (direct) {
        acc = bin_sum_direct(L.s, ray, st.inv, lo, hi, L.status, L.counters);
      } else {
        for (int j = 0; j < st.ncand; ++j) {
          if (st.hi[j * kBlock] < lo || st.lo[j * kBlock] > hi) continue;
          acc += fix40(bin_contrib(L.s, ray, st.idx[j * kBlock], lo, hi));
        }
      }
      float M = ((float)acc * kFixInv) * minf;
      if (M > 0.0f) {
        float mid = lo + 0.5f * (hi - lo);
        if (M * (hi - lo) > kSplitSteps && depth < kSplitDepth && mid > lo && mid < hi) {
          hi = mid;
          depth += 1;
          continue;
        }
        t = lo;
        for (;;) {
          if (tr.i >= kMaxDepth) {
            tr.t = t;
            return;
          }
          tr.i += 1;
          float u = lcg_f(tr.rng);
          float step = -dlog(1.0f - u) / M;
          t = t + step;
          if (t >= hi || t >= ray.tmax) break;
          float3 x = make_float3(ray.o.x + t * ray.d.x, ray.o.y + t * ray.d.y, ray.o.z + t * ray.d.z);
          Sample smp;
          if (direct) {
            point_query(L.s, x, smp, L.status, L.counters);
          } else {
            st.sample(L.s, t, x, smp, L.status);
          }
          float D = (float)smp.a0 * kFixInv;
          float sigma = D * scale;
          if (lcg_f(tr.rng) < sigma / M) {
            float3 c = sample_color(L, smp, D);
            tr.albedo = make_float4(c.x, c.y, c.z, 1.0f);
            tr.t = t;
            return;
          }
        }
      }
      const uint32_t pending = ~path & ((1u << depth) - 1u);  // lower halves whose upper half waits
      if (!pending) break;
      const int d = 31 - __clz(pending);
      path = (path | (1u << d)) & ((2u << d) - 1u);
      depth = d + 1;
      lo = b0;
      hi = b1;
      for (int l = 0; l < depth; ++l) {
        const float m = lo + 0.5f * (hi - lo);
        if ((path >> l) & 1u) lo = m;
        else hi = m;
      }
    }
    k += 1;
    t = b1;
  }
  if (guard == cap) atomicOr(L.status, kStatusLoopCap);
  tr.t = t;
}

template <int CAP>
__device__ __forceinline__ void track(const RenderLaunch& L, Tracker& tr, const Ray& ray, bool from_entry,
                                      char* smem) {
  const int i0 = tr.i;
  if (tr.marching) track_march<CAP>(L, tr, ray, smem);
  else if (L.flags & kFlagMajorantTracking) track_majorant<CAP>(L, tr, ray, smem);
  else track_delta<CAP>(L, tr, ray, from_entry, smem);
  ctr_add(L.counters, kCtrSteps, (unsigned long long)(tr.i - i0 + 1));
}

// ParticleRBFRayGen body for one sample (deviceCodeRBF.hlsl:206-324); track_fn runs the tracker
// (per thread or per warp), count_lane selects the lane that does count-mode accounting. BLUE:
// the blue-noise flag when the caller knows it at compile time (0 or 1), else -1 (read from L)
template <int BLUE = -1, class TrackFn>
__device__ float4 raygen_generic(const RenderLaunch& L, uint32_t frame, int px, int py, float& noise,
                                 bool count_lane, TrackFn&& track_fn) {
  uint32_t rng = pixel_seed(frame, (uint32_t)px, (uint32_t)py, (uint32_t)L.width);
  float sx = ((float)px + 0.5f + L.jitter_x) / (float)L.width;
  float sy = ((float)py + 0.5f + L.jitter_y) / (float)L.height;
  float3 rt = make_float3(L.aabb_max[0] + 2.0f * L.rbf_radius, L.aabb_max[1] + 2.0f * L.rbf_radius,
                          L.aabb_max[2] + 2.0f * L.rbf_radius);
  float3 lb = make_float3(L.aabb_min[0] - 2.0f * L.rbf_radius, L.aabb_min[1] - 2.0f * L.rbf_radius,
                          L.aabb_min[2] - 2.0f * L.rbf_radius);
  Ray ray;
  ray.o = make_float3(L.cam_pos[0], L.cam_pos[1], L.cam_pos[2]);
  float3 dir = make_float3((L.cam_d00[0] + sx * L.cam_du[0]) + sy * L.cam_dv[0],
                           (L.cam_d00[1] + sx * L.cam_du[1]) + sy * L.cam_dv[1],
                           (L.cam_d00[2] + sx * L.cam_du[2]) + sy * L.cam_dv[2]);
  ray.d = normalize3(dir);
  ray.tmin = 0.0f;
  ray.tmax = 10000.0f;
  float tenter, texit;
  aabb_clip(ray.o, ray.d, lb, rt, ray.tmin, ray.tmax, tenter, texit);

  Tracker tr;
  const bool blue = BLUE >= 0 ? BLUE != 0 : (L.flags & kFlagBlueNoise) != 0;
  float r0;
  if (blue) {
    uint32_t gx = frame % 8u, gy = (frame / 8u) % 16u;
    uint32_t cx = gx * 256u + (uint32_t)px % 256u, cy = gy * 256u + (uint32_t)py % 256u;
    r0 = 0.0f;
    if (L.noise && (int)cx < L.noise_w && (int)cy < L.noise_h)
      r0 = (float)L.noise[(size_t)cy * (size_t)L.noise_w + cx].x / 255.0f;
    tr.marching = true;
    tr.rng = 0u;
  } else {
    r0 = lcg_f(rng);
    tr.marching = false;
    tr.rng = rng;
  }
  float r1 = lcg_f(rng);
  float r2 = lcg_f(rng);
  tr.i = 0;
  tr.lhs = 0.0f;
  tr.random = r0;
  tr.albedo = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  tr.shadow = false;
  noise = r0;
  float4 color = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (tenter < texit) {
    ray.tmax = texit;
    tr.t = tenter + L.unit * r1;
    const bool from_entry = (L.flags & kFlagTrackFromEntry) != 0;
    const float t_start = (blue || from_entry) ? tr.t : ray.tmin;
    float4 albedo = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float t = 0.0f, vis = 1.0f, ts0 = 0.0f;
    Ray cur = ray;
    bool cur_from_entry = from_entry;
    // the tracker has one call site: pass 0 tracks the primary ray, pass 1 the shadow ray (NEE,
    // deviceCodeRBF.hlsl:288-314), so an inlined tracker exists once in the kernel
    for (int pass = 0; pass < 2; ++pass) {
      track_fn(tr, cur, cur_from_entry);
      if (pass == 1) {
        vis = 1.0f - tr.albedo.w;
        if (L.counters && count_lane) count_segment(L, cur, fmaxf(ts0, 0.0f), fminf(tr.t, cur.tmax));
        break;
      }
      albedo = tr.albedo;
      t = tr.t;
      if (L.counters && count_lane) count_segment(L, ray, t_start, fminf(t, ray.tmax));
      if (!(albedo.w > 0.0f && L.ambient != 1.0f)) break;
      cur.o = make_float3(ray.o.x + ray.d.x * t, ray.o.y + ray.d.y * t, ray.o.z + ray.d.z * t);
      cur.d = make_float3(L.light[0], L.light[1], L.light[2]);
      cur.tmin = 0.0f;
      cur.tmax = 10000.0f;
      float ste, stx;
      aabb_clip(cur.o, cur.d, lb, rt, cur.tmin, cur.tmax, ste, stx);
      cur.tmax = stx;
      cur_from_entry = false;
      tr.albedo = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      tr.lhs = 0.0f;
      tr.shadow = true;
      tr.t = blue ? -L.unit * r2 : 0.0f;
      ts0 = tr.t;
    }
    if (albedo.w == 1.0f) {
      color.x = (albedo.x * vis) * (1.0f - L.ambient) + albedo.x * L.ambient;
      color.y = (albedo.y * vis) * (1.0f - L.ambient) + albedo.y * L.ambient;
      color.z = (albedo.z * vis) * (1.0f - L.ambient) + albedo.z * L.ambient;
      color.w = 1.0f;
    }
  }
  return over4(color, make_float4(0.0f, 0.0f, 0.0f, 1.0f));
}

template <int CAP>
__device__ float4 raygen_sample(const RenderLaunch& L, uint32_t frame, int px, int py, float& noise, char* smem) {
  return raygen_generic(L, frame, px, py, noise, true,
                        [&](Tracker& tr, const Ray& r, bool from_entry) { track<CAP>(L, tr, r, from_entry, smem); });
}

// ============================================================================================
// Ray-per-warp kernel for majorant tracking. All 32 lanes of a warp work on one ray: the
// sequential tracker logic runs uniformly on every lane (identical values), and the heavy parts
// are split across lanes -- BVH traversal as a warp-wide frontier compacted with ballots,
// candidate staging into a per-warp shared buffer bucketed by majorant bin, and the fixed-point
// sums of majorants and densities, which lanes accumulate over disjoint particles and combine
// with shuffles (integer sums, so the lane split cannot change a bit).
// ============================================================================================

constexpr int kWarpsPerBlock = 4;
// resident blocks per SM the ray-per-warp kernels are compiled for (caps registers at
// 65536 / (128 * kWarpMinBlocks)); the tracker is out of line unless AARBF_TRACK_INLINE
#ifndef AARBF_WARP_MIN_BLOCKS
#define AARBF_WARP_MIN_BLOCKS 8
#endif
#ifndef AARBF_TRACK_INLINE
#define AARBF_TRACK_INLINE 0
#endif
constexpr int kWarpMinBlocks = AARBF_WARP_MIN_BLOCKS;

// per-warp shared memory: staged candidates, then per-bin lists of candidate slots (CSR)
template <int CAPW>
struct WarpBuf {
  uint32_t idx[CAPW];
  float lo[CAPW];
  float hi[CAPW];
  uint16_t list[2 * CAPW];
  uint32_t start[kMaxSegBins + 1];
  uint32_t leaves[64];
};

// this warp's buffer, addressed in the shared window (out-of-line functions receiving the buffer
// as a generic pointer would reach it with generic loads and stores)
template <int CAPW>
__device__ __forceinline__ WarpBuf<CAPW>* warp_buf() {
  extern __shared__ __align__(16) char smem[];
  return reinterpret_cast<WarpBuf<CAPW>*>(smem) + (threadIdx.x >> 5);
}

__device__ __forceinline__ void warp_sum_sample(Sample& s) {
  s.count = warp_sum(s.count);
  s.a0 = warp_sum(s.a0);
  s.a1 = warp_sum(s.a1);
  s.a2 = warp_sum(s.a2);
  s.a3 = warp_sum(s.a3);
}



template <int CAPW>
struct WarpStager {
  WarpBuf<CAPW>* buf;
  uint32_t* stk;
  int ncand;
  int kseg, nbins;   // the staged segment covers bins [kseg, kseg + nbins)
  bool lists;        // per-bin lists are valid
  float rb_enter, rb_exit;
  float3 inv;
  unsigned long long* ctr;

  __device__ void init(const SceneView& s, const Ray& ray) {
    ncand = 0;
    kseg = 0;
    nbins = 0;
    lists = false;
    inv = make_float3(1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z);
    float e = s.eps * 4.0f;
    float ax = (s.root_lo[0] - e - ray.o.x) * inv.x, bx = (s.root_hi[0] + e - ray.o.x) * inv.x;
    float ay = (s.root_lo[1] - e - ray.o.y) * inv.y, by = (s.root_hi[1] + e - ray.o.y) * inv.y;
    float az = (s.root_lo[2] - e - ray.o.z) * inv.z, bz = (s.root_hi[2] + e - ray.o.z) * inv.z;
    rb_enter = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz));
    rb_exit = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
    if (s.nleaves == 0 || !(rb_enter <= rb_exit)) {
      rb_enter = __int_as_float(0x7f800000);
      rb_exit = -__int_as_float(0x7f800000);
    }
  }

  // conservative range of segment bins a candidate interval [a, b] may touch
  __device__ __forceinline__ void bin_span(float a, float b, float t0, float Lb, int& j0, int& j1) const {
    float fa = floorf((a - t0) / Lb), fb = floorf((b - t0) / Lb);
    float lo = (float)(kseg - 1), hi = (float)(kseg + nbins);
    fa = fminf(fmaxf(fa, lo), hi);
    fb = fminf(fmaxf(fb, lo), hi);
    j0 = max((int)fa - 1 - kseg, 0);
    j1 = min((int)fb + 1 - kseg, nbins - 1);
  }

  // stage every particle whose (slightly inflated) sphere meets bins [k, k + nb) and bucket the
  // candidates by bin; false on overflow
  __device__ bool stage(const SceneView& s, const Ray& ray, int k, int nb, float t0, float Lb, uint32_t* status) {
    const uint32_t lane = threadIdx.x & 31u, lt = lane_lt_mask();
    wctr(ctr, kWcStages, 1);
    const float eps = s.eps;
    const float ts = t0 + (float)k * Lb, te = t0 + (float)(k + nb) * Lb;
    SegSlab slab;
    slab.init(ray.o, inv, eps, ts, te);
    int n = 0;
    bool ok = warp_traverse(
        s, stk, buf->leaves, status,
        [&](float lx, float ly, float lz, float hx, float hy, float hz) { return slab.hit(lx, ly, lz, hx, hy, hz); },
        [&](bool v, uint32_t i) -> bool {
          bool keep = false;
          float a = 0.0f, b = 0.0f;
          if (v) {
            const float4 r = part_cull(s, i);
            if (r.w > 0.0f && sphere_span(r, ray.o, ray.d, eps, a, b)) keep = !(b < ts || a > te);
          }
          const uint32_t m = __ballot_sync(kFull, keep);
          const int cnt = __popc(m);
          if (n + cnt > CAPW) return false;
          if (keep) {
            int p = n + __popc(m & lt);
            buf->idx[p] = i;
            buf->lo[p] = a;
            buf->hi[p] = b;
          }
          n += cnt;
          return true;
        },
        ctr);
    __syncwarp();
    if (!ok) {
      wctr(ctr, kWcOverflows, 1);
      ncand = 0;
      return false;
    }
    wctr(ctr, kWcCands, n);
    ncand = n;
    kseg = k;
    nbins = nb;
    // per-bin lists: count, exclusive scan, fill
    for (int j = (int)lane; j <= nb; j += 32) buf->start[j] = 0u;
    __syncwarp();
    for (int c = (int)lane; c < n; c += 32) {
      int j0, j1;
      bin_span(buf->lo[c], buf->hi[c], t0, Lb, j0, j1);
      for (int j = j0; j <= j1; ++j) atomicAdd(&buf->start[j + 1], 1u);
    }
    __syncwarp();
    uint32_t c0 = lane < (uint32_t)nb ? buf->start[lane + 1] : 0u;
    uint32_t c1 = lane + 32u < (uint32_t)nb ? buf->start[lane + 33] : 0u;
    uint32_t x0 = c0, x1 = c1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y0 = __shfl_up_sync(kFull, x0, o), y1 = __shfl_up_sync(kFull, x1, o);
      if ((int)lane >= o) {
        x0 += y0;
        x1 += y1;
      }
    }
    const uint32_t tot0 = __shfl_sync(kFull, x0, 31);
    const uint32_t total = tot0 + __shfl_sync(kFull, x1, 31);
    __syncwarp();
    // start[j] = first slot of bin j (exclusive prefix); start[nb] = total
    if (lane < (uint32_t)nb) buf->start[lane] = x0 - c0;
    if (lane + 32u < (uint32_t)nb) buf->start[lane + 32] = tot0 + x1 - c1;
    if (lane == 0) buf->start[nb] = total;
    lists = total <= 2u * CAPW;
    __syncwarp();
    if (lists) {
      // fill with per-bin cursors kept in the upper half of list[] scratch: reuse start[] by
      // counting down from the bin end
      uint32_t* cur = buf->leaves;  // 64 cursors (nb <= 64)
      for (int j = (int)lane; j < nb; j += 32) cur[j] = buf->start[j];
      __syncwarp();
      for (int c = (int)lane; c < n; c += 32) {
        int j0, j1;
        bin_span(buf->lo[c], buf->hi[c], t0, Lb, j0, j1);
        for (int j = j0; j <= j1; ++j) buf->list[atomicAdd(&cur[j], 1u)] = (uint16_t)c;
      }
      __syncwarp();
    }
    return true;
  }

  // candidate slots for top-level bin kbin: [first, last) in list[] (or all candidates)
  __device__ __forceinline__ void range(int kbin, int& first, int& last) const {
    if (lists) {
      int j = kbin - kseg;
      first = (int)buf->start[j];
      last = (int)buf->start[j + 1];
    } else {
      first = 0;
      last = ncand;
    }
  }

  __device__ __forceinline__ int slot(int p) const { return lists ? (int)buf->list[p] : p; }

  __device__ long long bin_sum(const SceneView& s, const Ray& ray, int kbin, float lo, float hi) const {
    int first, last;
    range(kbin, first, last);
    long long acc = 0;
    for (int p = first + (int)(threadIdx.x & 31u); p < last; p += 32) {
      int j = slot(p);
      if (buf->hi[j] < lo || buf->lo[j] > hi) continue;
      acc += fix40(bin_contrib(s, ray, buf->idx[j], lo, hi));
    }
    return warp_sum(acc);
  }

  __device__ void sample(const SceneView& s, int kbin, float t, float3 x, Sample& acc) const {
    int first, last;
    range(kbin, first, last);
    sample_clear(acc);
    if (first >= last) return;  // no candidate in this bin (warp-uniform): nothing to sum
    for (int p = first + (int)(threadIdx.x & 31u); p < last; p += 32) {
      int j = slot(p);
      if (t < buf->lo[j] || t > buf->hi[j]) continue;
      eval_particle(s, buf->idx[j], x, acc);
    }
    warp_sum_sample(acc);
  }

  // the density sum at step point x (t on the ray) over bin kbin's candidates, warp-reduced;
  // any: some particle holds x. The colour sums are left to sample() (once per collision).
  __device__ long long sample_density(const SceneView& s, int kbin, float t, float3 x, bool& any) const {
    int first, last;
    range(kbin, first, last);
    if (first >= last) {  // no candidate in this bin (warp-uniform)
      any = false;
      return 0;
    }
    long long a0 = 0;
    int count = 0;
    for (int p = first + (int)(threadIdx.x & 31u); p < last; p += 32) {
      int j = slot(p);
      if (t < buf->lo[j] || t > buf->hi[j]) continue;
      eval_density(s, buf->idx[j], x, count, a0);
    }
    any = __any_sync(kFull, count > 0);
    return any ? warp_sum(a0) : 0;
  }

  // first bin >= k of the staged segment whose list is not empty (kseg + nbins if none)
  __device__ int next_nonempty(int k) const {
    if (!lists) return k;
    for (int j = k - kseg; j < nbins; j += 32) {
      int jj = j + (int)(threadIdx.x & 31u);
      bool ne = jj < nbins && buf->start[jj + 1] > buf->start[jj];
      uint32_t m = __ballot_sync(kFull, ne);
      if (m) return kseg + j + __ffs(m) - 1;
    }
    return kseg + nbins;
  }
};

// Length of a ray's next staging after one of nb bins that staged n candidates: twice as long
// (at most kMaxSegBins, the size of the per-bin list arrays), but no longer than this staging's
// candidate density predicts fills half the buffer, so a dense run of bins is not staged long
// enough to overflow and be staged again. Only the cost depends on it: a bin's candidates are
// the same whatever segment it was staged with. With nb in [1, kMaxSegBins] the result is too.
template <int CAPW>
__device__ __forceinline__ int next_stage_bins(int nb, int n) {
  int next = 2 * nb < kMaxSegBins ? 2 * nb : kMaxSegBins;
  if (n > 0) {
    const int fit = (CAPW * nb) / (2 * n);
    next = fit < next ? (fit > 1 ? fit : 1) : next;
  }
  return next;
}

// direct (unbuffered) majorant sum of one bin; out of line (rare path, instruction-cache footprint)
template <int CAPW>
__device__ __noinline__ long long warp_bin_sum_direct(const SceneView& s, const Ray ray, const float3 inv, float lo,
                                                      float hi, WarpBuf<CAPW>* buf, uint32_t* stk, uint32_t* status,
                                                      unsigned long long* ctr) {
  (void)buf;
  long long acc = 0;
  SegSlab slab;
  slab.init(ray.o, inv, s.eps, lo, hi);
  warp_traverse(
      s, stk, warp_buf<CAPW>()->leaves, status,
      [&](float lx, float ly, float lz, float hx, float hy, float hz) { return slab.hit(lx, ly, lz, hx, hy, hz); },
      [&](bool v, uint32_t i) -> bool {
        if (v) acc += fix40(bin_contrib(s, ray, i, lo, hi));
        return true;
      },
      ctr);
  wctr(ctr, kWcDirect, 1);
  return warp_sum(acc);
}

// direct point query; out of line (rare path)
template <int CAPW>
__device__ __noinline__ Sample warp_point(const SceneView& s, const float3 x, WarpBuf<CAPW>* buf, uint32_t* stk,
                                          uint32_t* status, unsigned long long* ctr) {
  (void)buf;
  Sample acc;
  sample_clear(acc);
  warp_traverse(
      s, stk, warp_buf<CAPW>()->leaves, status,
      [&](float lx, float ly, float lz, float hx, float hy, float hz) { return inside(lx, ly, lz, hx, hy, hz, x); },
      [&](bool v, uint32_t i) -> bool {
        if (v) eval_particle(s, i, x, acc);
        return true;
      },
      ctr);
  wctr(ctr, kWcDirect, 1);
  warp_sum_sample(acc);
  return acc;
}

// track_majorant with the warp-cooperative stager; same decisions, same random-number stream
// out of line: one copy serves the primary and the shadow ray (instruction-cache footprint);
// the tracker state and the ray cross the call by value (references would pin the caller's
// copies in local memory)
template <int CAPW, bool COUNT>
__device__ __forceinline__ void track_majorant_warp_body(const RenderLaunch& L, Tracker& tr, const Ray& ray,
                                                         WarpBuf<CAPW>* buf, uint32_t* stk) {
  WarpStager<CAPW> st;
  st.buf = buf;
  st.stk = stk;
  unsigned long long* const ctr = COUNT ? L.counters : nullptr;  // count mode has its own instance
  st.ctr = ctr;
  st.init(L.s, ray);
  const float Lb = L.bin_length;
  const float scale = L.density_scale;
  const float minf = scale * 1.0078125f;
  const float t0 = tr.t;
  int k = 0;
  float t = t0;
  int seg_end = 0;
  int nb = L.stage_bins;
  bool direct = false;
  int budget = loop_bound(L.s.loop_cap, 1 << 26);  // iterations left
  for (; budget > 0; --budget) {
    float b0 = t0 + (float)k * Lb;
    float b1 = t0 + (float)(k + 1) * Lb;
    if (!(b0 < ray.tmax) || !(b1 > b0)) break;
    if (k >= seg_end) {
      if (b1 < st.rb_enter) {
        int ks = (int)floorf((st.rb_enter - t0) / Lb) - 1;
        if (ks > k) {
          k = ks;
          t = t0 + (float)k * Lb;
          continue;
        }
      }
      if (b0 > st.rb_exit) break;
      direct = false;
      for (;;) {
        if (st.stage(L.s, ray, k, nb, t0, Lb, L.status)) {
          seg_end = k + nb;
          nb = next_stage_bins<CAPW>(nb, st.ncand);
          break;
        }
        nb >>= 1;
        if (nb == 0) {
          direct = true;
          seg_end = k + 1;
          nb = 1;
          break;
        }
      }
      if (!direct) {
        if (st.ncand == 0) {
          k = seg_end;
          t = t0 + (float)k * Lb;
          continue;
        }
      }
    }
    if (!direct) {
      // bins whose candidate list is empty have majorant 0: skip them without drawing
      int kn = st.next_nonempty(k);
      if (kn > k) {
        k = kn;
        t = t0 + (float)k * Lb;
        continue;
      }
    }
    float lo = b0, hi = b1;
    int depth = 0, np = 0;
    float pend_hi[kSplitDepth];
    int pend_depth[kSplitDepth];
    for (;;) {
      wctr(ctr, kWcBins, 1);
      long long acc = direct ? warp_bin_sum_direct<CAPW>(L.s, ray, st.inv, lo, hi, buf, stk, L.status, ctr)
                             : st.bin_sum(L.s, ray, k, lo, hi);
      float M = ((float)acc * kFixInv) * minf;
      if (M > 0.0f) {
        float mid = lo + 0.5f * (hi - lo);
        if (M * (hi - lo) > kSplitSteps && depth < kSplitDepth && mid > lo && mid < hi) {
          pend_hi[np] = hi;
          pend_depth[np] = depth + 1;
          ++np;
          hi = mid;
          depth += 1;
          continue;
        }
        t = lo;
        for (;;) {
          if (tr.i >= kMaxDepth) {
            tr.t = t;
            return;
          }
          tr.i += 1;
          wctr(ctr, kWcSteps, 1);
          float u = lcg_f(tr.rng);
          float step = -dlog(1.0f - u) / M;
          t = t + step;
          if (t >= hi || t >= ray.tmax) break;
          float3 x = make_float3(ray.o.x + t * ray.d.x, ray.o.y + t * ray.d.y, ray.o.z + t * ray.d.z);
          Sample smp;
          if (direct) smp = warp_point<CAPW>(L.s, x, buf, stk, L.status, ctr);
          else st.sample(L.s, k, t, x, smp);
          float D = (float)smp.a0 * kFixInv;
          float sigma = D * scale;
          if (lcg_f(tr.rng) < sigma / M) {
            float3 c = sample_color(L, smp, D);
            tr.albedo = make_float4(c.x, c.y, c.z, 1.0f);
            tr.t = t;
            return;
          }
        }
      }
      if (np == 0) break;
      lo = hi;
      --np;
      hi = pend_hi[np];
      depth = pend_depth[np];
    }
    k += 1;
    t = b1;
  }
  if (budget == 0 && (threadIdx.x & 31u) == 0) atomicOr(L.status, kStatusLoopCap);
  tr.t = t;
}

template <int CAPW, bool COUNT>
#if AARBF_TRACK_INLINE
__device__ __forceinline__
#else
__device__ __noinline__
#endif
Tracker track_majorant_warp(const RenderLaunch& L, Tracker tr, const Ray ray, uint32_t* stk) {
  track_majorant_warp_body<CAPW, COUNT>(L, tr, ray, warp_buf<CAPW>(), stk);
  return tr;
}

// stochasticTracking (deviceCodeRBF.hlsl:141-203) with the warp: the reference's step sequence
// (t -= log(1 - xi) unit with the global majorant 1, then the collision draw only where a particle
// holds the step point) runs uniformly on every lane with the reference's draw order; the density
// at a step point is a lane-parallel fixed-point sum over the particles staged for the point's bin
// (bins of bin_length along the ray, staged by warp traversals as in the majorant tracker), so
// every float equals the sequential tracker's. A bin with more candidates than the buffer takes
// direct warp point queries. Out of line for the same reason as the majorant tracker.
template <int CAPW, bool COUNT>
__device__ __forceinline__ void track_delta_warp_body(const RenderLaunch& L, Tracker& tr, const Ray& ray,
                                                      bool from_entry, WarpBuf<CAPW>* buf, uint32_t* stk) {
  WarpStager<CAPW> st;
  st.buf = buf;
  st.stk = stk;
  unsigned long long* const ctr = COUNT ? L.counters : nullptr;
  st.ctr = ctr;
  st.init(L.s, ray);
  if (!from_entry) tr.t = ray.tmin;
  const float t0 = tr.t;
  const float Lb = L.bin_length > 0.0f ? L.bin_length : 16.0f * L.unit;  // staging granularity only
  int seg_begin = 0, seg_end = 0;  // staged bins [seg_begin, seg_end)
  int nb = L.stage_bins;
  bool direct = false;
  for (; tr.i < kMaxDepth; ++tr.i) {
    wctr(ctr, kWcSteps, 1);
    const float u = lcg_f(tr.rng);
    const float step = (dlog(1.0f - u) / 1.0f) * L.unit;
    tr.t = tr.t - step;
    if (tr.t >= ray.tmax) return;
    const float t = tr.t;
    // outside the (inflated) root box no particle holds the step point
    if (t < st.rb_enter || t > st.rb_exit) continue;
    const float fk = floorf((t - t0) / Lb);
    const int kb = fk < 1.0e9f ? (int)fk : 1000000000;
    if (kb < seg_begin || kb >= seg_end) {
      direct = false;
      for (;;) {
        if (st.stage(L.s, ray, kb, nb, t0, Lb, L.status)) {
          seg_begin = kb;
          seg_end = kb + nb;
          nb = next_stage_bins<CAPW>(nb, st.ncand);
          break;
        }
        nb >>= 1;
        if (nb == 0) {
          direct = true;
          seg_begin = kb;
          seg_end = kb + 1;
          nb = 1;
          break;
        }
      }
    }
    const float3 x = make_float3(ray.o.x + t * ray.d.x, ray.o.y + t * ray.d.y, ray.o.z + t * ray.d.z);
    Sample smp;
    long long a0;
    bool any;
    if (direct) {
      smp = warp_point<CAPW>(L.s, x, buf, stk, L.status, ctr);
      a0 = smp.a0;
      any = smp.count > 0;
    } else {
      a0 = st.sample_density(L.s, kb, t, x, any);
    }
    if (!any) continue;
    const float D = (float)a0 * kFixInv;
    const float density = sample_density(L, D);
    if (lcg_f(tr.rng) < density / 1.0f) {
      if (!direct) st.sample(L.s, kb, t, x, smp);  // the colour sums of the collision
      const float3 c = sample_color(L, smp, D);
      tr.albedo = make_float4(c.x, c.y, c.z, 1.0f);
      return;
    }
  }
}

template <int CAPW, bool COUNT>
__device__ __noinline__ Tracker track_delta_warp(const RenderLaunch& L, Tracker tr, const Ray ray, bool from_entry,
                                                 uint32_t* stk) {
  track_delta_warp_body<CAPW, COUNT>(L, tr, ray, from_entry, warp_buf<CAPW>(), stk);
  return tr;
}

// stochasticMarching (deviceCodeRBF.hlsl:67-139) with the warp: the steps of a chunk (up to 32)
// are evaluated one per lane against the particles staged for the chunk's segment; the step
// positions are the reference's running sum t += unit and the accumulated density / shadow
// opacity and the stopping test run in step order (all lanes, values by shuffle), so every float
// matches the sequential tracker. A chunk whose candidates overflow the buffer is halved; a single
// step that still overflows is evaluated by a direct warp traversal.
template <int CAPW>
__device__ bool stage_segment(const SceneView& s, const Ray& ray, float3 inv, float ta, float tb, WarpBuf<CAPW>* buf,
                              uint32_t* stk, uint32_t* status, int& n) {
  const uint32_t lt = lane_lt_mask();
  const float eps = s.eps;
  SegSlab slab;
  slab.init(ray.o, inv, eps, ta, tb);
  n = 0;
  const bool ok = warp_traverse(
      s, stk, buf->leaves, status,
      [&](float lx, float ly, float lz, float hx, float hy, float hz) { return slab.hit(lx, ly, lz, hx, hy, hz); },
      [&](bool v, uint32_t i) -> bool {
        bool keep = false;
        float a = 0.0f, b = 0.0f;
        if (v) {
          const float4 r = part_cull(s, i);
          if (r.w > 0.0f && sphere_span(r, ray.o, ray.d, eps, a, b)) keep = !(b < ta || a > tb);
        }
        const uint32_t m = __ballot_sync(kFull, keep);
        const int cnt = __popc(m);
        if (n + cnt > CAPW) return false;
        if (keep) {
          int p = n + __popc(m & lt);
          buf->idx[p] = i;
          buf->lo[p] = a;
          buf->hi[p] = b;
        }
        n += cnt;
        return true;
      });
  __syncwarp();
  return ok;
}

template <int CAPW>
__device__ __forceinline__ void track_march_warp_body(const RenderLaunch& L, Tracker& tr, const Ray& ray,
                                                      WarpBuf<CAPW>* buf, uint32_t* stk) {
  const uint32_t lane = threadIdx.x & 31u;
  const SceneView& s = L.s;
  const float rhs = -dlog(1.0f - tr.random * 0.99f);
  const float3 inv = make_float3(1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z);
  int m = 32;
  const int cap = loop_bound(s.loop_cap, 1 << 22);
  for (int guard = 0; guard < cap; ++guard) {
    if (tr.i >= kMaxDepth) return;
    // the chunk's step positions: the running sum, lane j keeps step j
    float tj = 0.0f, t = tr.t;
    for (int j = 0; j < m; ++j) {
      t = t + L.unit;
      if ((int)lane == j) tj = t;
    }
    const float tfirst = __shfl_sync(kFull, tj, 0);
    if (!(tfirst < ray.tmax)) {
      tr.t = tfirst;
      return;
    }
    const float tb = fminf(t, ray.tmax);
    int n = 0;
    bool direct = false;
    if (!stage_segment<CAPW>(s, ray, inv, tfirst, tb, buf, stk, L.status, n)) {
      if (m > 1) {
        m >>= 1;
        continue;
      }
      direct = true;
    }
    const bool active = (int)lane < m;
    const float3 x = make_float3(ray.o.x + tj * ray.d.x, ray.o.y + tj * ray.d.y, ray.o.z + tj * ray.d.z);
    Sample smp;
    sample_clear(smp);
    if (!direct) {  // each lane its step's density; the colour sums only for the stopping step
      for (int c = 0; c < n; ++c) {
        const bool in = active && tj < ray.tmax && tj >= buf->lo[c] && tj <= buf->hi[c];
        if (in) eval_density(s, buf->idx[c], x, smp.count, smp.a0);
      }
    } else {
      const float3 x0 = make_float3(__shfl_sync(kFull, x.x, 0), __shfl_sync(kFull, x.y, 0), __shfl_sync(kFull, x.z, 0));
      Sample d0 = warp_point<CAPW>(s, x0, buf, stk, L.status, L.counters);
      if (lane == 0) smp = d0;
    }
    const float D = (float)smp.a0 * kFixInv;
    const bool ne = active && smp.count > 0 && D > 0.0f;
    const float dens = ne ? sample_density(L, D) : 0.0f;
    const float op = (ne && tr.shadow) ? (1.0f - dexp(-dens)) : 0.0f;
    // the sequential tracker over the chunk's steps
    int stop = -1;
    float lhs = tr.lhs, alpha = tr.albedo.w;
    for (int j = 0; j < m; ++j) {
      if (tr.i + j >= kMaxDepth) {  // the step budget runs out before step j
        tr.i = kMaxDepth;
        tr.t = j ? __shfl_sync(kFull, tj, j - 1) : tr.t;
        tr.lhs = lhs;
        tr.albedo.w = alpha;
        return;
      }
      const float tjj = __shfl_sync(kFull, tj, j);
      if (tjj >= ray.tmax) {
        tr.t = tjj;
        tr.i += j;
        tr.lhs = lhs;
        tr.albedo.w = alpha;
        return;
      }
      if (!__shfl_sync(kFull, ne, j)) continue;
      lhs = lhs + __shfl_sync(kFull, dens, j);
      if (lhs > rhs && !tr.shadow) {
        stop = j;
        break;
      }
      if (tr.shadow) {
        alpha = alpha + __shfl_sync(kFull, op, j);
        if (alpha >= 1.0f) {
          alpha = 1.0f;
          stop = j;
          break;
        }
      }
    }
    if (stop >= 0) {
      tr.t = __shfl_sync(kFull, tj, stop);
      tr.i += stop;
      tr.lhs = lhs;
      if (tr.shadow) {
        tr.albedo.w = alpha;
      } else {
        float3 c = make_float3(0.0f, 0.0f, 0.0f);
        if ((int)lane == stop) {
          if (!direct) {  // the stopping step's colour sums over the same candidates
            sample_clear(smp);
            for (int q = 0; q < n; ++q)
              if (tj >= buf->lo[q] && tj <= buf->hi[q]) eval_particle(s, buf->idx[q], x, smp);
          }
          c = sample_color(L, smp, D);
        }
        tr.albedo = make_float4(__shfl_sync(kFull, c.x, stop), __shfl_sync(kFull, c.y, stop),
                                __shfl_sync(kFull, c.z, stop), 1.0f);
      }
      return;
    }
    tr.t = t;
    tr.i += m;
    tr.lhs = lhs;
    tr.albedo.w = alpha;
    if (m < 32) m <<= 1;
  }
  if (lane == 0) atomicOr(L.status, kStatusLoopCap);  // the loop bound ran out
}

template <int CAPW>
__device__ __noinline__ Tracker track_march_warp(const RenderLaunch& L, Tracker tr, const Ray ray, uint32_t* stk) {
  track_march_warp_body<CAPW>(L, tr, ray, warp_buf<CAPW>(), stk);
  return tr;
}

// persistent warps; an item is one sample of one pixel, ordered as in k_render
// items of one render: one sample of one pixel, 32 consecutive items = one sample of an 8x4 tile
__device__ __forceinline__ uint32_t warp_items(const RenderLaunch& L) {
  const uint32_t tiles_x = (uint32_t)(L.width + 7) / 8u;
  const uint32_t spp = L.spp ? L.spp : 1u;
  return tiles_x * ((uint32_t)(L.height + 3) / 4u) * 32u * spp;
}

// estimators of the ray-per-warp kernel, each in its own kernel instance so none carries another's
// code: delta tracking with per-bin majorants (native), stochastic marching (blue-noise mode), and
// the reference's delta tracking with the global majorant
enum { kWarpMajorant = 0, kWarpMarch = 1, kWarpDelta = 2 };

// one work item of the ray-per-warp kernel (all lanes of the warp); COUNT: the count-mode instance
// (render_count), so the timed instance carries no accounting code. sample_major: items run over
// every 8 x 4 tile for one sample before the next sample (else a tile's samples follow each
// other); the image is the same either way
template <int CAPW, int MODE, bool COUNT>
__device__ __forceinline__ void render_warp_item(const RenderLaunch& L, uint32_t item, WarpBuf<CAPW>* buf,
                                                 uint32_t* stk, bool sample_major = false) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t tiles_x = (uint32_t)(L.width + 7) / 8u;
  const uint32_t spp = L.spp ? L.spp : 1u;
  const size_t plane = (size_t)L.width * (size_t)L.height;
  const bool cost = (L.flags & kFlagCostImage) != 0;
  uint32_t group = item >> 5, in = item & 31u;
  uint32_t tile = group / spp, k = group % spp;
  if (sample_major) {
    const uint32_t ntiles = tiles_x * ((uint32_t)(L.height + 3) / 4u);
    k = group / ntiles;
    tile = group % ntiles;
  }
  const int px = (int)((tile % tiles_x) * 8u + (in & 7u));
  const int py = (int)((tile / tiles_x) * 4u + (in >> 3));
  if (px >= L.width || py >= L.height) return;
  const size_t ofs = (size_t)px + (size_t)L.width * (size_t)py;
  const long long c0 = cost ? clock64() : 0;
  float noise = 0.0f;
  float4 c = raygen_generic<MODE == kWarpMarch ? 1 : 0>(
      L, (L.frame_id + k) & 0xffffu, px, py, noise, COUNT && lane == 0, [&](Tracker& tr, const Ray& r, bool from_entry) {
        if (MODE == kWarpMarch) tr = track_march_warp<CAPW>(L, tr, r, stk);
        else if (MODE == kWarpDelta) tr = track_delta_warp<CAPW, COUNT>(L, tr, r, from_entry, stk);
        else tr = track_majorant_warp<CAPW, COUNT>(L, tr, r, stk);
      });
  if (cost) c.w = (float)(clock64() - c0);
  if (lane == 0) {
    L.samples[(size_t)k * plane + ofs] = c;
    if (k + 1 == spp) L.noise_buf[ofs] = noise;
  }
}

template <int CAPW, int MODE, bool COUNT>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kWarpMinBlocks) k_render_warp(const __grid_constant__ RenderLaunch L) {
  extern __shared__ __align__(16) char smem[];
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  WarpBuf<CAPW>* buf = reinterpret_cast<WarpBuf<CAPW>*>(smem) + wib;
  uint32_t* stk = L.warp_stacks + ((size_t)blockIdx.x * kWarpsPerBlock + wib) * kWarpStack;
  const uint32_t total = warp_items(L);
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(L.work_counter, 1u);
    // broadcast by a warp reduction: its result is known warp-uniform, so the item's pixel and
    // ray setup can use uniform registers
    item = __reduce_max_sync(kFull, item);
    if (item >= total) break;
    render_warp_item<CAPW, MODE, COUNT>(L, item, buf, stk);
  }
}

// Several scenes in one persistent launch. The scenes' launch blocks are one kernel parameter (as
// the single-scene kernel's launch block is), so the raygen reads them from the constant bank and
// the out-of-line trackers through a pointer into the parameter block, as in the single-scene
// kernel. Every warp walks the scenes in order and takes items of the current scene from that
// scene's counter until they run out, then moves on to the next scene: no warp waits for a scene
// to finish, and the scene index is a loop counter every lane agrees on (warp-uniform, like the
// item, which is broadcast by a warp reduction), so scene fields are read with uniform addresses.
// At most kBatchPerLaunch scenes per launch (the parameter block stays under the 32 KB
// kernel-parameter limit); larger batches take several launches.
constexpr int kBatchPerLaunch = 64;
struct BatchLaunch {
  RenderLaunch L[kBatchPerLaunch];
  uint32_t items[kBatchPerLaunch];  // work items of each scene
  uint32_t* counters;               // kBatchPerLaunch per-scene item counters, zeroed per launch
  uint32_t* warp_stacks;
  int nscenes;
};
static_assert(sizeof(BatchLaunch) <= 32000, "batched kernel parameters exceed the 32 KB limit");

// SMAJ: work items sample by sample over all tiles (a compile-time choice, as in the single-scene
// kernel, so the item decode carries one form)
template <int CAPW, bool SMAJ>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kWarpMinBlocks)
    k_render_warp_batched(const __grid_constant__ BatchLaunch P) {
  extern __shared__ __align__(16) char smem[];
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  WarpBuf<CAPW>* buf = reinterpret_cast<WarpBuf<CAPW>*>(smem) + wib;
  uint32_t* stk = P.warp_stacks + ((size_t)blockIdx.x * kWarpsPerBlock + wib) * kWarpStack;
  for (int s = 0; s < P.nscenes; ++s) {
    const uint32_t total = P.items[s];
    for (;;) {
      uint32_t item = 0;
      if (lane == 0) item = atomicAdd(P.counters + s, 1u);
      item = __reduce_max_sync(kFull, item);
      if (item >= total) break;
      render_warp_item<CAPW, kWarpMajorant, false>(P.L[s], item, buf, stk, SMAJ);
    }
  }
}

// Persistent kernel: each thread repeatedly takes the next work item from a global counter.
// An item is one sample of one pixel; 32 consecutive items are one sample of an 8x4 pixel tile
// and the spp groups of a tile follow each other, so the samples of an expensive pixel run on
// different threads at the same time. Each sample's colour goes to its own plane of L.samples;
// k_accumulate then forms the running mean in sample order (bit-identical to spp launches).
template <int CAP>
__global__ void __launch_bounds__(kBlock) k_render(const __grid_constant__ RenderLaunch L) {
  extern __shared__ __align__(16) char smem[];
  const uint32_t tiles_x = (uint32_t)(L.width + 7) / 8u;
  const uint32_t spp = L.spp ? L.spp : 1u;
  const uint32_t total = tiles_x * ((uint32_t)(L.height + 3) / 4u) * 32u * spp;
  const size_t plane = (size_t)L.width * (size_t)L.height;
  const bool cost = (L.flags & kFlagCostImage) != 0;
  for (;;) {
    uint32_t item = atomicAdd(L.work_counter, 1u);
    if (item >= total) break;
    uint32_t group = item >> 5, in = item & 31u;
    uint32_t tile = group / spp, k = group % spp;
    const int px = (int)((tile % tiles_x) * 8u + (in & 7u));
    const int py = (int)((tile / tiles_x) * 4u + (in >> 3));
    if (px >= L.width || py >= L.height) continue;
    const size_t ofs = (size_t)px + (size_t)L.width * (size_t)py;
    const long long c0 = cost ? clock64() : 0;
    float noise = 0.0f;
    float4 c = raygen_sample<CAP>(L, (L.frame_id + k) & 0xffffu, px, py, noise, smem);
    if (cost) c.w = (float)(clock64() - c0);
    L.samples[(size_t)k * plane + ofs] = c;
    if (k + 1 == spp) L.noise_buf[ofs] = noise;
  }
}

// running mean over the samples in order, deviceCodeRBF.hlsl:326-335
// running mean of one pixel's samples in sample order (deviceCodeRBF.hlsl:326-335)
__device__ __forceinline__ void accumulate_pixel(const RenderLaunch& L, size_t ofs) {
  const size_t plane = (size_t)L.width * (size_t)L.height;
  const uint32_t spp = L.spp ? L.spp : 1u;
  const bool cost = (L.flags & kFlagCostImage) != 0;
  float4 prev = L.accum[ofs];
  float4 fin = prev;
  float cycles = 0.0f;
  for (uint32_t k = 0; k < spp; ++k) {
    float4 c = L.samples[(size_t)k * plane + ofs];
    if (cost) {
      cycles += c.w;
      c.w = 1.0f;
    }
    uint32_t aid = (L.accum_id + k) & 0xffffu;
    float fa = (float)aid;
    float wa = 1.0f / fa, wb = (float)((int)aid - 1) / fa;
    fin.x = wa * c.x + wb * prev.x;
    fin.y = wa * c.y + wb * prev.y;
    fin.z = wa * c.z + wb * prev.z;
    fin.w = wa * c.w + wb * prev.w;
    prev = fin;
  }
  L.accum[ofs] = fin;
  if (L.flags & kFlagShowNoise) {
    float noise = L.noise_buf[ofs];
    fin = make_float4(noise, noise, noise, 1.0f);
  }
  // diagnostic: the image's alpha channel receives the pixel's cost in SM clock cycles
  if (cost) fin.w = cycles;
  L.image[ofs] = fin;
}

__global__ void k_accumulate(const RenderLaunch L) {
  const size_t plane = (size_t)L.width * (size_t)L.height;
  const size_t ofs = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (ofs >= plane) return;
  accumulate_pixel(L, ofs);
}

// the accumulation pass of every scene of a batch: pixels [pix_ofs[s], pix_ofs[s + 1]) are scene s's
__global__ void k_accumulate_batched(const RenderLaunch* __restrict__ Ls, const uint64_t* __restrict__ pix_ofs,
                                     int nscenes) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= pix_ofs[nscenes]) return;
  int lo = 0, hi = nscenes;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pix_ofs[mid] <= i) lo = mid;
    else hi = mid;
  }
  accumulate_pixel(Ls[lo], (size_t)(i - pix_ofs[lo]));
}

template <int CAP>
cudaError_t launch_cap(const RenderLaunch& L, cudaStream_t st, const cudaEvent_t* marks) {
  const size_t smem = (sizeof(uint32_t) + 2 * sizeof(float)) * CAP * kBlock;
  static PerDevice cache;
  int blocks = 0;
  cudaError_t e = per_device(cache, &blocks, [&](int dev, int* v) {
    cudaError_t r = cudaFuncSetAttribute(k_render<CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int sms = 0, per_sm = 0;
    if (r == cudaSuccess) r = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (r == cudaSuccess) r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_render<CAP>, kBlock, smem);
    *v = sms * (per_sm > 0 ? per_sm : 1);
    return r;
  });
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(L.work_counter, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  uint64_t items = (uint64_t)((L.width + 7) / 8) * (uint64_t)((L.height + 3) / 4) * 32u * (L.spp ? L.spp : 1u);
  int grid = (int)((items + kBlock - 1) / kBlock);
  if (grid > blocks) grid = blocks;
  if (marks) cudaEventRecord(marks[0], st);
  k_render<CAP><<<grid, kBlock, smem, st>>>(L);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (marks) cudaEventRecord(marks[1], st);
  size_t plane = (size_t)L.width * (size_t)L.height;
  k_accumulate<<<(unsigned)((plane + 255) / 256), 256, 0, st>>>(L);
  if (marks) cudaEventRecord(marks[2], st);
  return cudaGetLastError();
}

}  // namespace

namespace {

// Grid of the ray-per-warp kernels on the current device: the occupancy of the timed instances
// (the count-mode instances have larger frames and run oversubscribed on the same grid; work comes
// from an atomic counter, so that is still correct). Also sets the shared-memory limit of every
// instance, including the batched kernel, on this device.
template <int CAPW>
cudaError_t warp_grid(int* blocks) {
  static PerDevice cache;
  return per_device(cache, blocks, [](int dev, int* v) {
    const int smem = (int)(sizeof(WarpBuf<CAPW>) * kWarpsPerBlock);
    const cudaFuncAttribute attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e = cudaSuccess;
    for (auto f : {k_render_warp<CAPW, kWarpMajorant, false>, k_render_warp<CAPW, kWarpMajorant, true>,
                   k_render_warp<CAPW, kWarpMarch, false>, k_render_warp<CAPW, kWarpMarch, true>,
                   k_render_warp<CAPW, kWarpDelta, false>, k_render_warp<CAPW, kWarpDelta, true>})
      if (e == cudaSuccess) e = cudaFuncSetAttribute(f, attr, smem);
    for (auto f : {k_render_warp_batched<CAPW, false>, k_render_warp_batched<CAPW, true>})
      if (e == cudaSuccess) e = cudaFuncSetAttribute(f, attr, smem);
    int sms = 0, per_sm = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (auto f : {k_render_warp<CAPW, kWarpMajorant, false>, k_render_warp<CAPW, kWarpMarch, false>,
                   k_render_warp<CAPW, kWarpDelta, false>}) {
      int per = 0;
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, f, kWarpsPerBlock * 32, smem);
      per_sm = per > per_sm ? per : per_sm;
    }
    *v = sms * (per_sm > 0 ? per_sm : 1);
    return e;
  });
}

template <int CAPW>
cudaError_t launch_warp(const RenderLaunch& L, cudaStream_t st, const cudaEvent_t* marks) {
  int blocks = 0;
  cudaError_t e = warp_grid<CAPW>(&blocks);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(L.work_counter, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  if (marks) cudaEventRecord(marks[0], st);
  const size_t smem = sizeof(WarpBuf<CAPW>) * kWarpsPerBlock;
  const int mode = (L.flags & kFlagBlueNoise) ? kWarpMarch : (L.flags & kFlagMajorantTracking) ? kWarpMajorant
                                                                                                  : kWarpDelta;
  auto f = L.counters ? (mode == kWarpMarch ? k_render_warp<CAPW, kWarpMarch, true>
                         : mode == kWarpDelta ? k_render_warp<CAPW, kWarpDelta, true>
                                              : k_render_warp<CAPW, kWarpMajorant, true>)
                      : (mode == kWarpMarch ? k_render_warp<CAPW, kWarpMarch, false>
                         : mode == kWarpDelta ? k_render_warp<CAPW, kWarpDelta, false>
                                              : k_render_warp<CAPW, kWarpMajorant, false>);
  f<<<blocks, kWarpsPerBlock * 32, smem, st>>>(L);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (marks) cudaEventRecord(marks[1], st);
  size_t plane = (size_t)L.width * (size_t)L.height;
  k_accumulate<<<(unsigned)((plane + 255) / 256), 256, 0, st>>>(L);
  if (marks) cudaEventRecord(marks[2], st);
  return cudaGetLastError();
}

}  // namespace

bool render_uses_warp_kernel(const RenderLaunch& L) { return L.traversal == AARBF_TRAVERSAL_AUTO; }

cudaError_t render_warp_stack_words(size_t* words) {
  // enough stacks for the largest grid of any buffer depth
  int b0 = 0, b1 = 0, b2 = 0;
  cudaError_t e = warp_grid<256>(&b0);
  if (e == cudaSuccess) e = warp_grid<512>(&b1);
  if (e == cudaSuccess) e = warp_grid<1024>(&b2);
  int blocks = max(b0, max(b1, b2));
  *words = (size_t)blocks * kWarpsPerBlock * kWarpStack;
  return e;
}

namespace {
template <int CAPW>
cudaError_t launch_warp_batched(const BatchArgs& B, cudaStream_t st) {
  int blocks = 0;
  cudaError_t e = warp_grid<CAPW>(&blocks);
  if (e != cudaSuccess) return e;
  if (B.blocks_per_sm > 0) {  // fewer resident blocks than the occupancy limit
    int dev = 0, sms = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    if (sms * B.blocks_per_sm < blocks) blocks = sms * B.blocks_per_sm;
  }
  std::unique_ptr<BatchLaunch> P(new BatchLaunch());
  P->counters = B.work_counters;
  P->warp_stacks = B.warp_stacks;
  for (int c0 = 0; c0 < B.nscenes; c0 += kBatchPerLaunch) {
    const int n = B.nscenes - c0 < kBatchPerLaunch ? B.nscenes - c0 : kBatchPerLaunch;
    P->nscenes = n;
    for (int i = 0; i < n; ++i) {
      P->L[i] = B.host_launches[c0 + i];
      P->items[i] = (uint32_t)(B.host_items[c0 + i + 1] - B.host_items[c0 + i]);  // < 2^32: fill_launch
    }
    e = cudaMemsetAsync(B.work_counters, 0, sizeof(uint32_t) * kBatchPerLaunch, st);
    if (e != cudaSuccess) return e;
    auto f = B.sample_major ? k_render_warp_batched<CAPW, true> : k_render_warp_batched<CAPW, false>;
    f<<<blocks, kWarpsPerBlock * 32, sizeof(WarpBuf<CAPW>) * kWarpsPerBlock, st>>>(*P);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (B.total_pixels)
    k_accumulate_batched<<<(unsigned)((B.total_pixels + 255) / 256), 256, 0, st>>>(B.launches, B.pix_ofs, B.nscenes);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_render_batched(const BatchArgs& B, cudaStream_t st) {
  if (B.nscenes <= 0) return cudaSuccess;
  switch (B.candidate_cap) {
    case 512: return launch_warp_batched<512>(B, st);
    case 1024: return launch_warp_batched<1024>(B, st);
    default: return launch_warp_batched<256>(B, st);
  }
}

cudaError_t launch_render(const RenderLaunch& L, cudaStream_t st, const cudaEvent_t* marks) {
  if (L.width <= 0 || L.height <= 0) return cudaSuccess;
  if (AARBF_RENDER_NS::render_uses_warp_kernel(L)) {
    switch (L.candidate_cap) {
      case 512: return launch_warp<512>(L, st, marks);
      case 1024: return launch_warp<1024>(L, st, marks);
      default: return launch_warp<256>(L, st, marks);
    }
  }
  switch (L.candidate_cap) {
    case 16: return launch_cap<16>(L, st, marks);
    case 64: return launch_cap<64>(L, st, marks);
    case 128: return launch_cap<128>(L, st, marks);
    default: return launch_cap<32>(L, st, marks);
  }
}

}  // namespace AARBF_RENDER_NS
}  // namespace aarbf
