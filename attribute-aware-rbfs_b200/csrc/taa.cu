// taa.cu -- CompositeGui (deviceCodeCommon.hlsl:67-115): temporal anti-aliasing resolve with a
// YCoCg 3x3 neighbourhood clamp of the history, lerp(old, new, 0.2), then the (empty) GUI layer
// composited with "over" and a BGRA8 pack. The reference launches it with one-thread work groups
// (deviceCodeCommon.hlsl:67); here 16x16 pixel tiles stage the image tile plus a one-pixel halo
// in shared memory so each image texel is read from HBM once.
#include "aarbf_internal.h"

namespace aarbf {

namespace {

constexpr int kTile = 16;

__device__ __forceinline__ float3 rgb2ycocg(float3 c) {
  float co = c.x - c.z;
  float t = c.z + co / 2.0f;
  float cg = c.y - t;
  float y = t + cg / 2.0f;
  return make_float3(y, co, cg);
}

__device__ __forceinline__ float3 ycocg2rgb(float3 c) {
  float t = c.x - c.z / 2.0f;
  float g = c.z + t;
  float b = t - c.y / 2.0f;
  float r = c.y + b;
  return make_float3(r, g, b);
}

__device__ __forceinline__ uint32_t unorm8(float v) {
  if (!(v > 0.0f)) v = 0.0f;
  if (v > 1.0f) v = 1.0f;
  return (uint32_t)(v * 255.0f + 0.5f);
}

__global__ void __launch_bounds__(kTile* kTile) k_taa(const float4* __restrict__ image, const float4* __restrict__ prev,
                                                       float4* __restrict__ taa, uint32_t* __restrict__ bgra, int w,
                                                       int h, int disable) {
  __shared__ float4 tile[kTile + 2][kTile + 2];
  const int x0 = blockIdx.x * kTile, y0 = blockIdx.y * kTile;
  // clamp-to-edge halo load
  for (int k = threadIdx.x; k < (kTile + 2) * (kTile + 2); k += kTile * kTile) {
    int ty = k / (kTile + 2), tx = k % (kTile + 2);
    int gx = min(max(x0 + tx - 1, 0), w - 1), gy = min(max(y0 + ty - 1, 0), h - 1);
    tile[ty][tx] = __ldg(image + (size_t)gy * (size_t)w + (size_t)gx);
  }
  __syncthreads();
  const int lx = threadIdx.x % kTile, ly = threadIdx.x / kTile;
  const int px = x0 + lx, py = y0 + ly;
  if (px >= w || py >= h) return;
  const size_t ofs = (size_t)py * (size_t)w + (size_t)px;
  float4 center = tile[ly + 1][lx + 1];
  float4 pix;
  if (!disable) {
    float3 mn = rgb2ycocg(make_float3(center.x, center.y, center.z));
    float3 mx = mn;
#pragma unroll
    for (int iy = -1; iy <= 1; ++iy) {
#pragma unroll
      for (int ix = -1; ix <= 1; ++ix) {
        if (ix == 0 && iy == 0) continue;
        float4 q = tile[ly + 1 + iy][lx + 1 + ix];
        float3 y = rgb2ycocg(make_float3(q.x, q.y, q.z));
        mn = make_float3(fminf(mn.x, y.x), fminf(mn.y, y.y), fminf(mn.z, y.z));
        mx = make_float3(fmaxf(mx.x, y.x), fmaxf(mx.y, y.y), fmaxf(mx.z, y.z));
      }
    }
    float4 old = __ldg(prev + ofs);
    float3 y = rgb2ycocg(make_float3(old.x, old.y, old.z));
    float3 c = ycocg2rgb(make_float3(fmaxf(y.x, mn.x), fmaxf(y.y, mn.y), fmaxf(y.z, mn.z)));
    y = rgb2ycocg(c);
    c = ycocg2rgb(make_float3(fminf(y.x, mx.x), fminf(y.y, mx.y), fminf(y.z, mx.z)));
    old.x = c.x;
    old.y = c.y;
    old.z = c.z;
    pix.x = old.x + 0.2f * (center.x - old.x);
    pix.y = old.y + 0.2f * (center.y - old.y);
    pix.z = old.z + 0.2f * (center.z - old.z);
    pix.w = old.w + 0.2f * (center.w - old.w);
    taa[ofs] = pix;
  } else {
    pix = center;
  }
  if (bgra) {
    float4 o = over4(make_float4(0.0f, 0.0f, 0.0f, 0.0f), pix);
    bgra[ofs] = unorm8(o.z) | (unorm8(o.y) << 8) | (unorm8(o.x) << 16) | (unorm8(o.w) << 24);
  }
}

}  // namespace

cudaError_t launch_taa(const float4* image, const float4* prev, float4* taa, uint32_t* bgra, int w, int h,
                       int disable, cudaStream_t st) {
  if (w <= 0 || h <= 0) return cudaSuccess;
  dim3 grid((w + kTile - 1) / kTile, (h + kTile - 1) / kTile);
  k_taa<<<grid, kTile * kTile, 0, st>>>(image, prev, taa, bgra, w, h, disable);
  return cudaGetLastError();
}

}  // namespace aarbf
