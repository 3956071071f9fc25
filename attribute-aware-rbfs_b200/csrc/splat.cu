// splat.cu -- ParticleSplatRayGen / ParticleSplatIntersection / ParticleSplatAnyHit
// (deviceCodeSplat.hlsl:29-193): Knoll/Wald-style slab-sorted splatting.
//
// The ray is cut into slabs of width unit (PARTICLE_BUFFER_SIZE / 8 = 1 in integer arithmetic,
// deviceCodeSplat.hlsl:80). A slab keeps at most 15 samples; which 15 the reference keeps depends
// on hardware traversal order, here they are the 15 smallest (t, particle index). Candidates of
// a run of slabs are staged once per BVH traversal in shared memory and sorted; a slab with more
// than the buffer holds is resolved by a streaming top-15 traversal of that slab alone.
#include "aarbf_internal.h"
#include "warp_traverse.cuh"

namespace aarbf {

namespace {

constexpr int kBlock = 128;
constexpr int kCap = 32;
constexpr int kKeep = 15;  // PARTICLE_BUFFER_SIZE, deviceCodeSplat.hlsl:36

__device__ __forceinline__ float splat_radius(const RenderLaunch& L, uint32_t i) {
  float rg = __ldg(L.s.rgeom + i);
  if (rg < 0.0f) return 0.0f;  // radiusmap == 0: not splatted
  return (L.flags & kFlagSplatParticleRadius) ? rg : L.rbf_radius;
}

// ParticleSplatIntersection test (deviceCodeSplat.hlsl:165-179) without the slab condition;
// returns t = |c - o| when accepted, -1 otherwise
__device__ __forceinline__ float splat_t(const RenderLaunch& L, uint32_t i, float3 o, float3 d) {
  float r = splat_radius(L, i);
  if (!(r > 0.0f)) return -1.0f;
  float4 c = __ldg(L.s.xyzw + i);
  float vx = c.x - o.x, vy = c.y - o.y, vz = c.z - o.z;
  float t = sqrtf((vx * vx + vy * vy) + vz * vz);
  float sx = o.x + t * d.x, sy = o.y + t * d.y, sz = o.z + t * d.z;
  float ox = c.x - sx, oy = c.y - sy, oz = c.z - sz;
  if (!(((ox * ox + oy * oy) + oz * oz) < r * r)) return -1.0f;
  return t;
}

__device__ __forceinline__ bool less_ti(float ta, uint32_t ia, float tb, uint32_t ib) {
  return ta < tb || (ta == tb && ia < ib);
}

// visit every particle of every leaf whose padded box meets [t0, t1]; f(i) returns false to stop
template <class F>
__device__ bool traverse(const RenderLaunch& L, float3 o, float3 inv, float t0, float t1, float pad, F&& f) {
  const SceneView& s = L.s;
  if (s.nleaves == 0) return true;
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
      const Node* nd = s.nodes_ref + node;  // reference bounds: splatting ignores opacity
      float4 a = __ldg(&nd->a), b = __ldg(&nd->b), c = __ldg(&nd->c);
      uint2 ch = __ldg(reinterpret_cast<const uint2*>(&nd->d));
      if (seg_box(a.x, a.y, a.z, a.w, b.x, b.y, o, inv, t0, t1, pad)) {
        if (ch.x & kLeafBit) leaves[nl++] = ch.x & ~kLeafBit;
        else n0 = ch.x;
      }
      if (seg_box(b.z, b.w, c.x, c.y, c.z, c.w, o, inv, t0, t1, pad)) {
        if (ch.y & kLeafBit) leaves[nl++] = ch.y & ~kLeafBit;
        else n1 = ch.y;
      }
    }
    for (int k = 0; k < nl; ++k) {
      uint64_t b0 = (uint64_t)leaves[k] * s.ppl, e0 = b0 + s.ppl;
      if (e0 > s.n) e0 = s.n;
      for (uint64_t i = b0; i < e0; ++i)
        if (!f((uint32_t)i)) return false;
    }
    if (root_leaf) return true;
    if (n0 != 0xffffffffu && n1 != 0xffffffffu) {
      if (sp == kStackSize) {
        atomicOr(L.status, kStatusStackOverflow);
        return true;
      }
      stack[sp++] = n1;
      node = n0;
    } else if (n0 != 0xffffffffu) {
      node = n0;
    } else if (n1 != 0xffffffffu) {
      node = n1;
    } else {
      if (sp == 0) return true;
      node = stack[--sp];
    }
  }
}

__device__ __forceinline__ float4 shade_sample(const RenderLaunch& L, uint32_t id, float t, float3 o, float3 d,
                                               float atten) {
  float4 P = __ldg(L.s.xyzw + id);
  float r = splat_radius(L, id);
  float X0 = o.x + d.x * t, X1 = o.y + d.y * t, X2 = o.z + d.z * t;
  float dx = X0 - P.x, dy = X1 - P.y, dz = X2 - P.z;
  float dist = sqrtf((dx * dx + dy * dy) + dz * dz);
  float q = (dist * 3.0f) / r;
  float drbf = dexp(-0.5f * (q * q));
  float4 col;
  if (L.flags & kFlagVisualizeAttributes) {
    col = tex4(L.s.tf_color, L.s.nc, P.w);
    drbf = tex1(L.s.tf_density, L.s.nd, drbf);
    col.w = col.w * drbf;
  } else {
    float4 c = tex4(L.s.tf_color, L.s.nc, drbf);
    col = make_float4(c.x, c.y, c.z, tex1(L.s.tf_density, L.s.nd, drbf));
  }
  col.w = col.w * atten;
  return col;
}

__global__ void __launch_bounds__(kBlock) k_splat(const RenderLaunch L, float pad) {
  __shared__ float sh_t[kCap][kBlock];
  __shared__ uint32_t sh_i[kCap][kBlock];
  const int tid = threadIdx.x;
  const int px = blockIdx.x * 16 + (tid & 15);
  const int py = blockIdx.y * 8 + (tid >> 4);
  if (px >= L.width || py >= L.height) return;
  float sx = ((float)px + 0.5f + L.jitter_x) / (float)L.width;
  float sy = ((float)py + 0.5f + L.jitter_y) / (float)L.height;
  float3 rt = make_float3(L.aabb_max[0] + L.rbf_radius, L.aabb_max[1] + L.rbf_radius, L.aabb_max[2] + L.rbf_radius);
  float3 lb = make_float3(L.aabb_min[0] - L.rbf_radius, L.aabb_min[1] - L.rbf_radius, L.aabb_min[2] - L.rbf_radius);
  float3 o = make_float3(L.cam_pos[0], L.cam_pos[1], L.cam_pos[2]);
  float3 d = normalize3(make_float3((L.cam_d00[0] + sx * L.cam_du[0]) + sy * L.cam_dv[0],
                                    (L.cam_d00[1] + sx * L.cam_du[1]) + sy * L.cam_dv[1],
                                    (L.cam_d00[2] + sx * L.cam_du[2]) + sy * L.cam_dv[2]));
  float tenter, texit;
  aabb_clip(o, d, lb, rt, 0.0f, 10000.0f, tenter, texit);
  float4 res = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (tenter < texit) {
    const float3 inv = make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    const float spacing = (float)(kKeep / 8) * L.unit;
    const float atten = dexp(-L.unit * (float)(kKeep / 8));
    float tslab = 0.0f;
    int run = 16;  // slabs staged per traversal
    const int cap = loop_bound(L.s.loop_cap, 1 << 24);
    int guard = 0;
    while (tslab < texit) {
      if (guard++ == cap) {  // the loop bound ran out: report the truncated pixel
        atomicOr(L.status, kStatusLoopCap);
        break;
      }
      if (res.w > 0.99f) break;
      // skip slabs that end before the entry point
      float tmax0 = fminf(texit, tslab + spacing);
      if (!(tmax0 > tenter)) {
        tslab = tslab + spacing;
        continue;
      }
      // stage the next `run` slabs
      float s_end = tslab;
      int nslab = 0;
      for (; nslab < run && s_end < texit; ++nslab) s_end = s_end + spacing;
      float lo = fmaxf(tenter, tslab), hi = fminf(texit, s_end);
      int cnt = 0;
      bool ok = traverse(L, o, inv, lo, hi, pad, [&](uint32_t i) {
        float t = splat_t(L, i, o, d);
        if (t < 0.0f || !(t >= lo && t < hi)) return true;
        if (cnt == kCap) return false;
        sh_t[cnt][tid] = t;
        sh_i[cnt][tid] = i;
        ++cnt;
        return true;
      });
      if (!ok && nslab > 1) {
        run = nslab / 2;
        continue;
      }
      if (ok) {
        // insertion sort by (t, id)
        for (int a = 1; a < cnt; ++a) {
          float ta = sh_t[a][tid];
          uint32_t ia = sh_i[a][tid];
          int b = a - 1;
          while (b >= 0 && less_ti(ta, ia, sh_t[b][tid], sh_i[b][tid])) {
            sh_t[b + 1][tid] = sh_t[b][tid];
            sh_i[b + 1][tid] = sh_i[b][tid];
            --b;
          }
          sh_t[b + 1][tid] = ta;
          sh_i[b + 1][tid] = ia;
        }
        int cur = 0;
        for (int k = 0; k < nslab; ++k) {
          if (!(tslab < texit)) break;
          if (res.w > 0.99f) break;
          float tmin = fmaxf(tenter, tslab), tmax = fminf(texit, tslab + spacing);
          if (tmax > tenter) {
            while (cur < cnt && sh_t[cur][tid] < tmin) ++cur;
            int taken = 0;
            while (cur < cnt && taken < kKeep && sh_t[cur][tid] < tmax) {
              float4 col = shade_sample(L, sh_i[cur][tid], sh_t[cur][tid], o, d, atten);
              res = over4(res, col);
              ++cur;
              ++taken;
            }
          }
          tslab = tslab + spacing;
        }
        if (run < 64) run *= 2;
      } else {
        // a single slab with more candidates than the buffer: streaming top-15 of the slab
        float tmin = fmaxf(tenter, tslab), tmax = fminf(texit, tslab + spacing);
        float kt[kKeep];
        uint32_t ki[kKeep];
        int kc = 0;
        traverse(L, o, inv, tmin, tmax, pad, [&](uint32_t i) {
          float t = splat_t(L, i, o, d);
          if (t < 0.0f || !(t >= tmin && t < tmax)) return true;
          if (kc == kKeep && !less_ti(t, i, kt[kKeep - 1], ki[kKeep - 1])) return true;
          int b = (kc < kKeep) ? kc : kKeep - 1;
          if (kc < kKeep) ++kc;
          while (b > 0 && less_ti(t, i, kt[b - 1], ki[b - 1])) {
            kt[b] = kt[b - 1];
            ki[b] = ki[b - 1];
            --b;
          }
          kt[b] = t;
          ki[b] = i;
          return true;
        });
        for (int k = 0; k < kc; ++k) res = over4(res, shade_sample(L, ki[k], kt[k], o, d, atten));
        tslab = tslab + spacing;
        run = 1;
      }
    }
  }
  res = over4(res, make_float4(0.0f, 0.0f, 0.0f, 1.0f));
  L.image[(size_t)px + (size_t)L.width * (size_t)py] = res;
}

// ---- one warp per pixel --------------------------------------------------------------------
// The slab starts are the reference's running sum t_{k+1} = t_k + spacing from t_0 = 0, the same
// floats for every ray, so they are tabulated once per launch (slabs[]); a ray finds its first
// slab by binary search. A run of slabs is staged by one warp-wide traversal of the
// reference-bounds BVH (accepted samples with t in the run), sorted by (t, index) with a bitonic
// network in shared memory, and then composited slab by slab (lanes shade the up to 15 samples
// of a slab in parallel, the "over" chain runs in order); slabs without samples are skipped by a
// binary search for the next sample's slab. A single slab with more samples than the buffer
// takes its 15 smallest (t, index) by repeated minimum traversals.

constexpr int kSplatWarps = 4;
constexpr int kSplatCap = 512;

struct SplatBuf {
  float t[kSplatCap];
  uint32_t id[kSplatCap];
  uint32_t leaves[64];
};

struct SplatWarpArgs {
  const float* slabs;  // slab starts, nslabs entries (the last one >= every ray's texit)
  int nslabs;
  float pad;
  uint32_t* work_counter;
  uint32_t* warp_stacks;
};

// first j in [lo, hi) with slabs[j] > x (hi if none)
__device__ __forceinline__ int first_above(const float* slabs, int lo, int hi, float x) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(slabs + mid) > x) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

__device__ __forceinline__ void bitonic_sort(SplatBuf* b, int n, uint32_t lane) {
  int P = 1;
  while (P < n) P <<= 1;
  for (int j = n + (int)lane; j < P; j += 32) {
    b->t[j] = __int_as_float(0x7f800000);
    b->id[j] = 0xffffffffu;
  }
  __syncwarp();
  for (int size = 2; size <= P; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int p = (int)lane; p < P / 2; p += 32) {
        const int a = 2 * p - (p & (stride - 1)), c = a + stride;
        const bool up = (a & size) == 0;
        const float ta = b->t[a], tc = b->t[c];
        const uint32_t ia = b->id[a], ic = b->id[c];
        if (less_ti(tc, ic, ta, ia) == up) {
          b->t[a] = tc;
          b->id[a] = ic;
          b->t[c] = ta;
          b->id[c] = ia;
        }
      }
      __syncwarp();
    }
}

__global__ void __launch_bounds__(kSplatWarps * 32) k_splat_warp(const __grid_constant__ RenderLaunch L,
                                                                 const SplatWarpArgs A) {
  extern __shared__ __align__(16) char smem[];
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, lt = lane_lt_mask();
  SplatBuf* buf = reinterpret_cast<SplatBuf*>(smem) + wib;
  uint32_t* stk = A.warp_stacks + ((size_t)blockIdx.x * kSplatWarps + wib) * kWarpStack;
  const uint32_t total = (uint32_t)L.width * (uint32_t)L.height;
  const float spacing = (float)(kKeep / 8) * L.unit;
  const float atten = dexp(-L.unit * (float)(kKeep / 8));
  const float3 rt = make_float3(L.aabb_max[0] + L.rbf_radius, L.aabb_max[1] + L.rbf_radius, L.aabb_max[2] + L.rbf_radius);
  const float3 lb = make_float3(L.aabb_min[0] - L.rbf_radius, L.aabb_min[1] - L.rbf_radius, L.aabb_min[2] - L.rbf_radius);
  const float3 o = make_float3(L.cam_pos[0], L.cam_pos[1], L.cam_pos[2]);
  (void)spacing;
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(A.work_counter, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= total) break;
    const int px = (int)(item % (uint32_t)L.width), py = (int)(item / (uint32_t)L.width);
    const float sx = ((float)px + 0.5f + L.jitter_x) / (float)L.width;
    const float sy = ((float)py + 0.5f + L.jitter_y) / (float)L.height;
    const float3 d = normalize3(make_float3((L.cam_d00[0] + sx * L.cam_du[0]) + sy * L.cam_dv[0],
                                            (L.cam_d00[1] + sx * L.cam_du[1]) + sy * L.cam_dv[1],
                                            (L.cam_d00[2] + sx * L.cam_du[2]) + sy * L.cam_dv[2]));
    float tenter, texit;
    aabb_clip(o, d, lb, rt, 0.0f, 10000.0f, tenter, texit);
    float4 res = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (tenter < texit && L.s.nleaves > 0) {
      const float3 inv = make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
      // first slab whose end lies beyond the entry point
      int k = first_above(A.slabs, 1, A.nslabs, tenter) - 1;
      int run = 64;
      const int cap = loop_bound(L.s.loop_cap, 1 << 22);
      for (int guard = 0; k + 1 < A.nslabs; ++guard) {
        if (guard == cap) {  // the loop bound ran out: report the truncated pixel
          if (lane == 0) atomicOr(L.status, kStatusLoopCap);
          break;
        }
        const float ts = __ldg(A.slabs + k);
        if (!(ts < texit) || res.w > 0.99f) break;
        const int kend = min(k + run, A.nslabs - 1);
        const float lo = fmaxf(tenter, ts), hi = fminf(texit, __ldg(A.slabs + kend));
        int n = 0;
        const bool ok = warp_traverse_wide(
            L.s, L.s.wide_ref, stk, buf->leaves, L.status,
            [&](float bx0, float by0, float bz0, float bx1, float by1, float bz1) {
              return seg_box(bx0, by0, bz0, bx1, by1, bz1, o, inv, lo, hi, A.pad);
            },
            [&](bool v, uint32_t i) -> bool {
              float t = v ? splat_t(L, i, o, d) : -1.0f;
              const bool keep = t >= 0.0f && t >= lo && t < hi;
              const uint32_t m = __ballot_sync(kFull, keep);
              if (n + __popc(m) > kSplatCap) return false;
              if (keep) {
                const int p = n + __popc(m & lt);
                buf->t[p] = t;
                buf->id[p] = i;
              }
              n += __popc(m);
              return true;
            });
        __syncwarp();
        if (!ok) {
          if (run > 1) {
            run >>= 1;
            continue;
          }
          // one slab with more samples than the buffer: its 15 smallest (t, index), one by one
          const float tmin = lo, tmax = hi;
          float pt = -__int_as_float(0x7f800000);
          uint32_t pi = 0u;
          bool first = true;
          for (int taken = 0; taken < kKeep; ++taken) {
            float bt = __int_as_float(0x7f800000);
            uint32_t bi = 0xffffffffu;
            warp_traverse_wide(
                L.s, L.s.wide_ref, stk, buf->leaves, L.status,
                [&](float bx0, float by0, float bz0, float bx1, float by1, float bz1) {
                  return seg_box(bx0, by0, bz0, bx1, by1, bz1, o, inv, tmin, tmax, A.pad);
                },
                [&](bool v, uint32_t i) -> bool {
                  float t = v ? splat_t(L, i, o, d) : -1.0f;
                  if (t >= 0.0f && t >= tmin && t < tmax && (first || less_ti(pt, pi, t, i)) && less_ti(t, i, bt, bi)) {
                    bt = t;
                    bi = i;
                  }
                  return true;
                });
            for (int off = 16; off; off >>= 1) {
              const float ot = __shfl_xor_sync(kFull, bt, off);
              const uint32_t oi = __shfl_xor_sync(kFull, bi, off);
              if (less_ti(ot, oi, bt, bi)) {
                bt = ot;
                bi = oi;
              }
            }
            if (bi == 0xffffffffu) break;
            res = over4(res, shade_sample(L, bi, bt, o, d, atten));
            pt = bt;
            pi = bi;
            first = false;
          }
          k += 1;
          continue;
        }
        if (n == 0) {
          k = kend;
          if (run < 4096) run <<= 1;
          continue;
        }
        bitonic_sort(buf, n, lane);
        // composite the slabs of the run
        int cur = 0;
        while (k < kend) {
          const float tk = __ldg(A.slabs + k);
          if (!(tk < texit) || res.w > 0.99f) break;
          const float tmin = fmaxf(tenter, tk), tmax = fminf(texit, __ldg(A.slabs + k + 1));
          // skip samples below this slab (beyond the 15 kept by an earlier slab)
          for (;;) {
            const int j = cur + (int)lane;
            const uint32_t below = __ballot_sync(kFull, j < n && buf->t[j] < tmin);
            const int c = __popc(below);
            cur += c;
            if (c < 32) break;
          }
          if (cur >= n) {
            k = kend;
            break;
          }
          const int j = cur + (int)lane;
          const uint32_t inside = __ballot_sync(kFull, j < n && (int)lane < kKeep && buf->t[j] < tmax);
          const int m = __popc(inside);
          if (m == 0) {
            // the next sample's slab: first slab whose end lies beyond it
            const float tn = buf->t[cur];
            k = max(k + 1, min(kend, first_above(A.slabs, k + 1, kend + 1, tn) - 1));
            continue;
          }
          float4 col = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          if ((int)lane < m) col = shade_sample(L, buf->id[j], buf->t[j], o, d, atten);
          for (int q = 0; q < m; ++q) {
            const float4 c = make_float4(__shfl_sync(kFull, col.x, q), __shfl_sync(kFull, col.y, q),
                                         __shfl_sync(kFull, col.z, q), __shfl_sync(kFull, col.w, q));
            res = over4(res, c);
          }
          cur += m;
          k += 1;
        }
        if (n < kSplatCap / 4 && run < 4096) run <<= 1;
      }
    }
    res = over4(res, make_float4(0.0f, 0.0f, 0.0f, 1.0f));
    if (lane == 0) L.image[(size_t)px + (size_t)L.width * (size_t)py] = res;
  }
}

// grid of the ray-per-warp splat kernel on the current device (sets its shared-memory limit there)
cudaError_t splat_grid_blocks(int* blocks) {
  static PerDevice cache;
  return per_device(cache, blocks, [](int dev, int* v) {
    const int smem = (int)(sizeof(SplatBuf) * kSplatWarps);
    cudaError_t e = cudaFuncSetAttribute(k_splat_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int sms = 0, per = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_splat_warp, kSplatWarps * 32, smem);
    *v = sms * (per > 0 ? per : 1);
    return e;
  });
}

}  // namespace

cudaError_t launch_splat(const RenderLaunch& L, cudaStream_t st, const float* slabs, int nslabs) {
  if (L.width <= 0 || L.height <= 0) return cudaSuccess;
  // An accepted sample point lies within the splat radius of its particle's centre, on the ray
  // segment being staged. The reference-bounds box holds the sphere of the bounds radius, so
  // with per-particle splat radii (= bounds radii) the unpadded box already meets the segment;
  // with the global rbfRadius the sphere can exceed the box by at most rbfRadius. eps covers
  // the rounding of the sample point and of the box corners.
  const bool own_radius = (L.flags & kFlagSplatParticleRadius) != 0;
  float pad = (own_radius ? 0.0f : L.splat_rmax) + 4.0f * L.s.eps;
  if (slabs && nslabs >= 2 && L.traversal != AARBF_TRAVERSAL_THREAD) {
    SplatWarpArgs A;
    A.slabs = slabs;
    A.nslabs = nslabs;
    A.pad = pad;
    A.work_counter = L.work_counter;
    A.warp_stacks = L.warp_stacks;
    cudaError_t e = cudaMemsetAsync(L.work_counter, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    int blocks = 0;
    e = splat_grid_blocks(&blocks);
    if (e != cudaSuccess) return e;
    k_splat_warp<<<blocks, kSplatWarps * 32, sizeof(SplatBuf) * kSplatWarps, st>>>(L, A);
    return cudaGetLastError();
  }
  dim3 grid((L.width + 15) / 16, (L.height + 7) / 8);
  k_splat<<<grid, kBlock, 0, st>>>(L, pad);
  return cudaGetLastError();
}

cudaError_t splat_stack_words(size_t* words) {
  int blocks = 0;
  cudaError_t e = splat_grid_blocks(&blocks);
  *words = (size_t)blocks * kSplatWarps * kWarpStack;
  return e;
}

}  // namespace aarbf
