// diff.cu -- the differentiable form: expected stochastic marching and its adjoint.
//
// Forward model (the reference's stochasticMarching, deviceCodeRBF.hlsl:67-139, with ambient 1,
// its random threshold -log(1 - 0.99 xi) integrated over xi in closed form):
//   steps t_k = t0 + (k + 1) unit from t0 = tenter + unit u (u: first LCG draw of the pixel seed),
//   D_k = sum rho a^3, C_k = sum rho a^3 rgb^2.2 over particles with |x_k - p| < r,
//   rho = (exp(-4.5 |x_k - p|^2 / r^2) - e^-4.5) / (1 - e^-4.5)   (zero at the cut-off radius),
//   dens_k = min(gain D_k, 1), tau_k = sum_{j<=k} dens_j, G_k = min(1, (1 - exp(-tau_k)) / 0.99),
//   c_k = (C_k / D_k)^(1/2.2), sample colour E = sum_k (G_k - G_{k-1}) c_k, pixel = mean over spp.
// Adjoint by path replay: dE/d dens_j = g'_j c_j + sum_{k>j} B_k with g'_k = dG_k/dtau_k and
// B_k = (g'_k - g'_prev(k)) c_k. The forward keeps B_total per sample (the checkpoint); the
// backward replays the ray, forms the prefix of B and scatters dL/d(position, radius, a^3,
// rgb^2.2 a^3) to the particles; a last pass chains the weights to the transfer function and
// the attribute and maps the gradients back to the caller's particle order.
//
// One warp per pixel. The ray is processed in chunks of up to 32 steps: one warp-wide BVH
// traversal stages every particle whose sphere meets the chunk's segment (index, ray interval,
// centre and radius) in shared memory, then lane j evaluates step j of the chunk against the
// staged list, and the optical depth is an inclusive warp scan. A chunk whose candidates
// overflow the buffer is halved; a single step that still overflows is evaluated by a direct
// warp traversal.
#include "aarbf_internal.h"
#include "warp_traverse.cuh"

namespace aarbf {

namespace {

constexpr int kDiffWarps = 4;
constexpr int kDiffCap = 256;
constexpr float kE45 = 0.011108996538242306f;  // exp(-4.5)
constexpr float kKernInv = 1.0f / (1.0f - 0.011108996538242306f);

struct DiffBuf {
  uint32_t idx[kDiffCap];
  float lo[kDiffCap];
  float hi[kDiffCap];
  float4 rec[kDiffCap];
  uint32_t leaves[64];
};

__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ float warp_scanf(float v, uint32_t lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    float y = __shfl_up_sync(kFull, v, o);
    if ((int)lane >= o) v += y;
  }
  return v;
}

__device__ __forceinline__ float g_of(float tau) { return fminf(1.0f, (1.0f - dexp(-tau)) / 0.99f); }

// stage the particles whose (inflated) sphere meets [ta, tb]; false on overflow
__device__ bool diff_stage(const SceneView& s, const Ray& ray, float3 inv, float ta, float tb, DiffBuf* buf,
                           uint32_t* stk, uint32_t* status, int& n) {
  const uint32_t lt = lane_lt_mask();
  const float eps = s.eps;
  n = 0;
  bool ok = warp_traverse(
      s, stk, buf->leaves, status,
      [&](float lx, float ly, float lz, float hx, float hy, float hz) {
        return seg_box(lx, ly, lz, hx, hy, hz, ray.o, inv, ta, tb, eps);
      },
      [&](bool v, uint32_t i) -> bool {
        bool keep = false;
        float a = 0.0f, b = 0.0f;
        float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (v) {
          r = __ldg(s.rec0 + i);
          if (r.w > 0.0f) {
            float vx = r.x - ray.o.x, vy = r.y - ray.o.y, vz = r.z - ray.o.z;
            float tc = (vx * ray.d.x + vy * ray.d.y) + vz * ray.d.z;
            float wx = vx - tc * ray.d.x, wy = vy - tc * ray.d.y, wz = vz - tc * ray.d.z;
            float h2 = (wx * wx + wy * wy) + wz * wz;
            float R = r.w * (1.0f + 0x1p-10f) + eps;
            if (!(h2 > R * R)) {
              float half = sqrtf(R * R - h2) + eps;
              a = tc - half;
              b = tc + half;
              keep = !(b < ta || a > tb);
            }
          }
        }
        const uint32_t m = __ballot_sync(kFull, keep);
        const int cnt = __popc(m);
        if (n + cnt > kDiffCap) return false;
        if (keep) {
          int p = n + __popc(m & lt);
          buf->idx[p] = i;
          buf->lo[p] = a;
          buf->hi[p] = b;
          buf->rec[p] = r;
        }
        n += cnt;
        return true;
      });
  __syncwarp();
  return ok;
}

// kernel value and derivative factor of particle rec at x (false outside the sphere)
__device__ __forceinline__ bool kern(float4 r, float3 x, float& rho, float& deriv, float& d2, float3& dx) {
  dx = make_float3(x.x - r.x, x.y - r.y, x.z - r.z);
  d2 = (dx.x * dx.x + dx.y * dx.y) + dx.z * dx.z;
  float r2 = r.w * r.w;
  if (!(d2 < r2)) return false;
  float e = dexp(-4.5f * (d2 / r2));
  rho = (e - kE45) * kKernInv;
  deriv = e * kKernInv;
  return true;
}

struct DiffView {
  float pos[3], d00[3], du[3], dv[3];
  float lb[3], rt[3];
  float unit, gain;
  uint32_t frame_id, spp;
};

struct DiffLaunch {
  SceneView s;
  const DiffView* views;
  int nviews, width, height;
  float4* image;             // forward: nviews x h x w, (mean rgb, 1)
  float4* ckpt;              // per sample: B_total (xyz)
  const float4* grad_image;  // backward: dL/dimage
  float* g_pos;              // backward, sorted order: 3 n
  float* g_rad;              // n
  float* g_w;                // 4 n: dL/d(a^3 weight), dL/d(rgb^2.2 a^3 weights)
  uint32_t* work_counter;
  uint32_t* status;
  uint32_t* warp_stacks;
};

// gradient of one (step, particle) pair: position (3), radius, a^3 weight, colour weights (3)
__device__ __forceinline__ void pair_grad(const SceneView& s, uint32_t i, float4 r, float rho, float deriv, float d2,
                                          float3 dx, float gD, float gC0, float gC1, float gC2, float* v) {
  const float4 w = __ldg(s.w4 + i);
  const float gr = ((gD * w.x + gC0 * w.y) + gC1 * w.z) + gC2 * w.w;
  const float f = gr * deriv * 9.0f / (r.w * r.w);
  v[0] = f * dx.x;
  v[1] = f * dx.y;
  v[2] = f * dx.z;
  v[3] = f * d2 / r.w;
  v[4] = gD * rho;
  v[5] = gC0 * rho;
  v[6] = gC1 * rho;
  v[7] = gC2 * rho;
}

__device__ __forceinline__ void add_grad(const DiffLaunch& L, uint32_t i, const float* v) {
  atomicAdd(L.g_pos + 3 * (size_t)i, v[0]);
  atomicAdd(L.g_pos + 3 * (size_t)i + 1, v[1]);
  atomicAdd(L.g_pos + 3 * (size_t)i + 2, v[2]);
  atomicAdd(L.g_rad + i, v[3]);
#pragma unroll
  for (int q = 0; q < 4; ++q) atomicAdd(L.g_w + 4 * (size_t)i + q, v[4 + q]);
}

// One sample of one pixel. Forward: returns E, writes B_total to bt. Backward: g = upstream
// gradient of this sample's colour, bt = its checkpoint; scatters the particle gradients.
template <bool BWD>
__device__ float3 diff_sample(const DiffLaunch& L, const DiffView& V, int px, int py, uint32_t smp, DiffBuf* buf,
                              uint32_t* stk, float3& bt, float3 g) {
  const uint32_t lane = threadIdx.x & 31u, lt = lane_lt_mask();
  const SceneView& s = L.s;
  uint32_t rng = pixel_seed((V.frame_id + smp) & 0xffffu, (uint32_t)px, (uint32_t)py, (uint32_t)L.width);
  const float u = lcg_f(rng);
  const float sx = ((float)px + 0.5f) / (float)L.width, sy = ((float)py + 0.5f) / (float)L.height;
  Ray ray;
  ray.o = make_float3(V.pos[0], V.pos[1], V.pos[2]);
  ray.d = normalize3(make_float3((V.d00[0] + sx * V.du[0]) + sy * V.dv[0], (V.d00[1] + sx * V.du[1]) + sy * V.dv[1],
                                 (V.d00[2] + sx * V.du[2]) + sy * V.dv[2]));
  float tenter, texit;
  aabb_clip(ray.o, ray.d, make_float3(V.lb[0], V.lb[1], V.lb[2]), make_float3(V.rt[0], V.rt[1], V.rt[2]), 0.0f,
            10000.0f, tenter, texit);
  float3 E = make_float3(0.0f, 0.0f, 0.0f);
  float3 B = make_float3(0.0f, 0.0f, 0.0f);
  if (!(tenter < texit) || s.nleaves == 0) {
    if (!BWD) bt = B;
    return E;
  }
  const float unit = V.unit, gain = V.gain;
  const float t0 = tenter + unit * u;
  const float3 inv = make_float3(1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z);
  float tau_c = 0.0f, gp_c = 0.0f;              // carries: optical depth, g' of the last step with D > 0
  float3 P_c = make_float3(0.0f, 0.0f, 0.0f);   // backward: prefix of B
  int k0 = 0, m = 32;
  const int cap = loop_bound(s.loop_cap, 1 << 22);
  for (int guard = 0;; ++guard) {
    if (guard == cap) {  // the loop bound ran out: report the truncated ray
      if (lane == 0) atomicOr(L.status, kStatusLoopCap);
      break;
    }
    const float ta = t0 + (float)(k0 + 1) * unit;
    if (!(ta < texit)) break;
    const float tb = fminf(t0 + (float)(k0 + m) * unit, texit);
    int n = 0;
    bool direct = false;
    if (!diff_stage(s, ray, inv, ta, tb, buf, stk, L.status, n)) {
      if (m > 1) {
        m >>= 1;
        continue;
      }
      direct = true;
    }
    const float t = t0 + (float)(k0 + (int)lane + 1) * unit;
    const bool active = (int)lane < m && t < texit;
    float D = 0.0f, C0 = 0.0f, C1 = 0.0f, C2 = 0.0f;
    const float3 x = make_float3(ray.o.x + t * ray.d.x, ray.o.y + t * ray.d.y, ray.o.z + t * ray.d.z);
    const float3 x0 = make_float3(__shfl_sync(kFull, x.x, 0), __shfl_sync(kFull, x.y, 0), __shfl_sync(kFull, x.z, 0));
    if (!direct) {
      for (int c = 0; c < n; ++c) {
        const bool in = active && t >= buf->lo[c] && t <= buf->hi[c];
        if (!__any_sync(kFull, in)) continue;
        float rho, deriv, d2;
        float3 dx;
        if (in && kern(buf->rec[c], x, rho, deriv, d2, dx)) {
          float4 w = __ldg(s.w4 + buf->idx[c]);
          D += rho * w.x;
          C0 += rho * w.y;
          C1 += rho * w.z;
          C2 += rho * w.w;
        }
      }
    } else {
      // one step (lane 0's point, m = 1) with more candidates than the buffer: direct traversal
      float d = 0.0f, a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
      warp_traverse(
          s, stk, buf->leaves, L.status,
          [&](float lx, float ly, float lz, float hx, float hy, float hz) { return inside(lx, ly, lz, hx, hy, hz, x0); },
          [&](bool v, uint32_t i) -> bool {
            float rho, deriv, d2;
            float3 dx;
            if (v && kern(__ldg(s.rec0 + i), x0, rho, deriv, d2, dx)) {
              float4 w = __ldg(s.w4 + i);
              d += rho * w.x;
              a0 += rho * w.y;
              a1 += rho * w.z;
              a2 += rho * w.w;
            }
            return true;
          });
      d = warp_sumf(d);
      a0 = warp_sumf(a0);
      a1 = warp_sumf(a1);
      a2 = warp_sumf(a2);
      if (lane == 0 && active) {
        D = d;
        C0 = a0;
        C1 = a1;
        C2 = a2;
      }
    }
    // optical depth, stopping probability, colours
    const bool ne = active && D > 0.0f;
    const float dens = ne ? fminf(gain * D, 1.0f) : 0.0f;
    const float tau = warp_scanf(dens, lane) + tau_c;
    float tau_x = __shfl_up_sync(kFull, tau, 1);
    if (lane == 0) tau_x = tau_c;
    const float e = dexp(-tau);
    const float G = fminf(1.0f, (1.0f - e) / 0.99f);
    const float Gp = g_of(tau_x);
    const float gpr = ((1.0f - e) / 0.99f < 1.0f) ? e / 0.99f : 0.0f;
    float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
    if (ne) {
      const float k = 1.0f / 2.2f;
      c0 = dpow(C0 / D, k);
      c1 = dpow(C1 / D, k);
      c2 = dpow(C2 / D, k);
    }
    const float wgt = ne ? (G - Gp) : 0.0f;
    const uint32_t nem = __ballot_sync(kFull, ne);
    const uint32_t before = nem & lt;
    const int pl = before ? 31 - __clz((int)before) : 0;
    float gprev = __shfl_sync(kFull, gpr, pl);
    if (!before) gprev = gp_c;
    const float dB = ne ? (gpr - gprev) : 0.0f;
    const float B0 = dB * c0, B1 = dB * c1, B2 = dB * c2;
    if (!BWD) {
      E.x += warp_sumf(wgt * c0);
      E.y += warp_sumf(wgt * c1);
      E.z += warp_sumf(wgt * c2);
      B.x += warp_sumf(B0);
      B.y += warp_sumf(B1);
      B.z += warp_sumf(B2);
    } else {
      const float3 P = make_float3(warp_scanf(B0, lane) + P_c.x, warp_scanf(B1, lane) + P_c.y,
                                   warp_scanf(B2, lane) + P_c.z);
      P_c = make_float3(__shfl_sync(kFull, P.x, 31), __shfl_sync(kFull, P.y, 31), __shfl_sync(kFull, P.z, 31));
      float gD = 0.0f, gC0 = 0.0f, gC1 = 0.0f, gC2 = 0.0f;
      if (ne) {
        const float S0 = gpr * c0 + (bt.x - P.x), S1 = gpr * c1 + (bt.y - P.y), S2 = gpr * c2 + (bt.z - P.z);
        const float grho = (g.x * S0 + g.y * S1) + g.z * S2;
        gD = (gain * D < 1.0f) ? grho * gain : 0.0f;
        const float q0 = g.x * wgt, q1 = g.y * wgt, q2 = g.z * wgt;
        gD -= ((q0 * c0 + q1 * c1) + q2 * c2) / (2.2f * D);
        gC0 = C0 > 0.0f ? q0 * c0 / (2.2f * C0) : 0.0f;
        gC1 = C1 > 0.0f ? q1 * c1 / (2.2f * C1) : 0.0f;
        gC2 = C2 > 0.0f ? q2 * c2 / (2.2f * C2) : 0.0f;
      }
      const bool want = ne && (gD != 0.0f || gC0 != 0.0f || gC1 != 0.0f || gC2 != 0.0f);
      if (!direct) {
        for (int c = 0; c < n; ++c) {
          const bool in = want && t >= buf->lo[c] && t <= buf->hi[c];
          float rho = 0.0f, deriv = 0.0f, d2 = 0.0f;
          float3 dx = make_float3(0.0f, 0.0f, 0.0f);
          const float4 r = buf->rec[c];
          const bool member = in && kern(r, x, rho, deriv, d2, dx);
          if (!__any_sync(kFull, member)) continue;
          const uint32_t i = buf->idx[c];
          float v[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
          if (member) pair_grad(s, i, r, rho, deriv, d2, dx, gD, gC0, gC1, gC2, v);
#pragma unroll
          for (int q = 0; q < 8; ++q) v[q] = warp_sumf(v[q]);
          if (lane == 0) add_grad(L, i, v);
        }
      } else if (__shfl_sync(kFull, want, 0)) {
        // lane 0's step: the lanes take the particles of a direct traversal with lane 0's upstream
        gD = __shfl_sync(kFull, gD, 0);
        gC0 = __shfl_sync(kFull, gC0, 0);
        gC1 = __shfl_sync(kFull, gC1, 0);
        gC2 = __shfl_sync(kFull, gC2, 0);
        warp_traverse(
            s, stk, buf->leaves, L.status,
            [&](float lx, float ly, float lz, float hx, float hy, float hz) { return inside(lx, ly, lz, hx, hy, hz, x0); },
            [&](bool v, uint32_t i) -> bool {
              float rho = 0.0f, deriv = 0.0f, d2 = 0.0f;
              float3 dx = make_float3(0.0f, 0.0f, 0.0f);
              const float4 r = v ? __ldg(s.rec0 + i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
              if (v && kern(r, x0, rho, deriv, d2, dx)) {  // lanes hold different particles
                float q[8];
                pair_grad(s, i, r, rho, deriv, d2, dx, gD, gC0, gC1, gC2, q);
                add_grad(L, i, q);
              }
              return true;
            });
      }
    }
    // carries into the next chunk
    tau_c = __shfl_sync(kFull, tau, 31);
    if (nem) gp_c = __shfl_sync(kFull, gpr, 31 - __clz((int)nem));
    const float Glast = __shfl_sync(kFull, G, 31);
    k0 += m;
    if (m < 32) m <<= 1;
    if (Glast >= 1.0f) break;
  }
  if (!BWD) bt = B;
  return E;
}

template <bool BWD>
__global__ void __launch_bounds__(kDiffWarps * 32) k_diff(const __grid_constant__ DiffLaunch L) {
  extern __shared__ __align__(16) char smem[];
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  DiffBuf* buf = reinterpret_cast<DiffBuf*>(smem) + wib;
  uint32_t* stk = L.warp_stacks + ((size_t)blockIdx.x * kDiffWarps + wib) * kWarpStack;
  const size_t plane = (size_t)L.width * (size_t)L.height;
  const uint32_t total = (uint32_t)(plane * (size_t)L.nviews);
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(L.work_counter, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= total) break;
    const uint32_t view = item / (uint32_t)plane;
    const uint32_t pix = item % (uint32_t)plane;
    const int px = (int)(pix % (uint32_t)L.width), py = (int)(pix / (uint32_t)L.width);
    const DiffView& V = L.views[view];
    const uint32_t spp = V.spp ? V.spp : 1u;
    const size_t ofs = (size_t)view * plane + pix;
    if (!BWD) {
      float3 acc = make_float3(0.0f, 0.0f, 0.0f);
      for (uint32_t k = 0; k < spp; ++k) {
        float3 bt;
        float3 e = diff_sample<false>(L, V, px, py, k, buf, stk, bt, make_float3(0.0f, 0.0f, 0.0f));
        acc.x += e.x;
        acc.y += e.y;
        acc.z += e.z;
        if (lane == 0) L.ckpt[ofs * spp + k] = make_float4(bt.x, bt.y, bt.z, 0.0f);
      }
      const float is = 1.0f / (float)spp;
      if (lane == 0) L.image[ofs] = make_float4(acc.x * is, acc.y * is, acc.z * is, 1.0f);
    } else {
      const float4 gi = L.grad_image[ofs];
      const float is = 1.0f / (float)spp;
      const float3 g = make_float3(gi.x * is, gi.y * is, gi.z * is);
      if (g.x == 0.0f && g.y == 0.0f && g.z == 0.0f) continue;
      for (uint32_t k = 0; k < spp; ++k) {
        const float4 c = L.ckpt[ofs * spp + k];
        float3 bt = make_float3(c.x, c.y, c.z);
        diff_sample<true>(L, V, px, py, k, buf, stk, bt, g);
      }
    }
  }
}

// chain the per-particle weight gradients to the transfer function and the attribute, and write
// every gradient in the caller's particle order
__global__ void k_diff_finish(const float4* __restrict__ xyzw, const uint32_t* __restrict__ perm, uint64_t n,
                              const float4* __restrict__ tf, int nc, float attr_scale, const float* __restrict__ g_pos,
                              const float* __restrict__ g_rad, const float* __restrict__ g_w, float* __restrict__ out_pos,
                              float* __restrict__ out_rad, float* __restrict__ out_attr, float* __restrict__ out_tf) {
  extern __shared__ float sh_tf[];  // nc x 4
  for (int j = threadIdx.x; j < 4 * nc; j += blockDim.x) sh_tf[j] = 0.0f;
  __syncthreads();
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) {
    const float w = __ldg(xyzw + i).w;
    int i0, i1;
    float a;
    tex_coords(w, nc, i0, i1, a);
    const float4 v0 = __ldg(tf + i0), v1 = __ldg(tf + i1);
    const float col[4] = {v0.x + a * (v1.x - v0.x), v0.y + a * (v1.y - v0.y), v0.z + a * (v1.z - v0.z),
                          v0.w + a * (v1.w - v0.w)};
    const float slope[4] = {v1.x - v0.x, v1.y - v0.y, v1.z - v0.z, v1.w - v0.w};
    const float al = col[3], a3 = (al * al) * al;
    float gt[4];
    float ga = g_w[4 * i];
    for (int c = 0; c < 3; ++c) {
      const float gc = g_w[4 * i + 1 + c];
      ga += gc * dpow(col[c], 2.2f);
      gt[c] = col[c] > 0.0f ? gc * 2.2f * dpow(col[c], 1.2f) * a3 : 0.0f;
    }
    gt[3] = ga * 3.0f * (al * al);
    float gattr = 0.0f;
    for (int c = 0; c < 4; ++c) {
      atomicAdd(sh_tf + 4 * i0 + c, gt[c] * (1.0f - a));
      atomicAdd(sh_tf + 4 * i1 + c, gt[c] * a);
      if (i0 != i1) gattr += gt[c] * slope[c] * (float)nc;
    }
    const uint32_t o = perm[i];
    out_pos[3 * (size_t)o] = g_pos[3 * i];
    out_pos[3 * (size_t)o + 1] = g_pos[3 * i + 1];
    out_pos[3 * (size_t)o + 2] = g_pos[3 * i + 2];
    out_rad[o] = g_rad[i];
    out_attr[o] = gattr * attr_scale;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < 4 * nc; j += blockDim.x)
    if (sh_tf[j] != 0.0f) atomicAdd(out_tf + j, sh_tf[j]);
}

// grid of the differentiable kernels on the current device (sets their shared-memory limit there)
cudaError_t diff_grid_blocks(int* blocks) {
  static PerDevice cache;
  return per_device(cache, blocks, [](int dev, int* v) {
    const int smem = (int)(sizeof(DiffBuf) * kDiffWarps);
    cudaError_t e = cudaFuncSetAttribute(k_diff<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_diff<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int sms = 0, a = 0, b = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_diff<false>, kDiffWarps * 32, smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_diff<true>, kDiffWarps * 32, smem);
    *v = sms * max(1, min(a, b));
    return e;
  });
}

static_assert(sizeof(DiffView) == sizeof(float) * 22, "DiffView layout");

}  // namespace

cudaError_t diff_stack_words(size_t* words) {
  int blocks = 0;
  cudaError_t e = diff_grid_blocks(&blocks);
  *words = (size_t)blocks * kDiffWarps * kWarpStack;
  return e;
}

cudaError_t launch_diff(const DiffArgs& A, cudaStream_t st) {
  if (A.width <= 0 || A.height <= 0 || A.nviews <= 0) return cudaSuccess;
  DiffLaunch L;
  L.s = A.s;
  L.views = reinterpret_cast<const DiffView*>(A.views);
  L.nviews = A.nviews;
  L.width = A.width;
  L.height = A.height;
  L.image = A.image;
  L.ckpt = A.ckpt;
  L.grad_image = A.grad_image;
  L.g_pos = A.g_pos;
  L.g_rad = A.g_rad;
  L.g_w = A.g_w;
  L.work_counter = A.work_counter;
  L.status = A.status;
  L.warp_stacks = A.warp_stacks;
  int blocks = 0;
  cudaError_t eg = diff_grid_blocks(&blocks);
  if (eg != cudaSuccess) return eg;
  cudaError_t e = cudaMemsetAsync(A.work_counter, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  const size_t smem = sizeof(DiffBuf) * kDiffWarps;
  if (A.backward) k_diff<true><<<blocks, kDiffWarps * 32, smem, st>>>(L);
  else k_diff<false><<<blocks, kDiffWarps * 32, smem, st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_diff_finish(const float4* xyzw, const uint32_t* perm, uint64_t n, const float4* tf, int nc,
                               float attr_scale, const float* g_pos, const float* g_rad, const float* g_w,
                               float* out_pos, float* out_rad, float* out_attr, float* out_tf, cudaStream_t st) {
  if (!n) return cudaSuccess;
  const int threads = 256;
  k_diff_finish<<<(unsigned)((n + threads - 1) / threads), threads, sizeof(float) * 4 * nc, st>>>(
      xyzw, perm, n, tf, nc, attr_scale, g_pos, g_rad, g_w, out_pos, out_rad, out_attr, out_tf);
  return cudaGetLastError();
}

}  // namespace aarbf
