// fp16.cu -- the FP16 storage form of a scene (no counterpart in the reference).
//
// Positions are stored as FP16 offsets from the centre of the bounding box of each run of 256
// consecutive (Hilbert-sorted) particles, whose fp32 centre is kept once per run; the attribute
// and the per-particle weights a^3 and rgb^2.2 a^3 are rounded to FP16; radii stay fp32. The
// rounded values are also written back into the fp32 arrays (sorted particles, prepass records),
// so every other kernel, the BVH and the oracle see exactly what the FP16 records decode to.
// The tracking kernels read the packed records instead: 8 bytes of position + the radius rounded
// up to FP16 (what the staging test reads: a conservative sphere), the fp32 radius (what the
// density evaluation reads) and 8 bytes of a^3 + colour weights.
#include <cuda_fp16.h>

#include "aarbf_internal.h"

namespace aarbf {

namespace {

constexpr int kRun = 256;

__device__ __forceinline__ uint32_t hbits(float v) { return (uint32_t)__half_as_ushort(__float2half_rn(v)); }
__device__ __forceinline__ float hval(uint32_t b) { return __half2float(__ushort_as_half((unsigned short)b)); }

// one block per run of 256 particles
__global__ void __launch_bounds__(kRun) k_quantize_positions(float4* __restrict__ xyzw, uint64_t n,
                                                             uint2* __restrict__ posq, float4* __restrict__ origin) {
  __shared__ float lo[3][kRun], hi[3][kRun];
  const uint64_t i = blockIdx.x * (uint64_t)kRun + threadIdx.x;
  const bool v = i < n;
  float4 p = v ? xyzw[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float inf = __int_as_float(0x7f800000);
  lo[0][threadIdx.x] = v ? p.x : inf;
  lo[1][threadIdx.x] = v ? p.y : inf;
  lo[2][threadIdx.x] = v ? p.z : inf;
  hi[0][threadIdx.x] = v ? p.x : -inf;
  hi[1][threadIdx.x] = v ? p.y : -inf;
  hi[2][threadIdx.x] = v ? p.z : -inf;
  __syncthreads();
  for (int s = kRun / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int a = 0; a < 3; ++a) {
        lo[a][threadIdx.x] = fminf(lo[a][threadIdx.x], lo[a][threadIdx.x + s]);
        hi[a][threadIdx.x] = fmaxf(hi[a][threadIdx.x], hi[a][threadIdx.x + s]);
      }
    __syncthreads();
  }
  const float ox = (lo[0][0] + hi[0][0]) * 0.5f, oy = (lo[1][0] + hi[1][0]) * 0.5f, oz = (lo[2][0] + hi[2][0]) * 0.5f;
  if (threadIdx.x == 0) origin[blockIdx.x] = make_float4(ox, oy, oz, 0.0f);
  if (!v) return;
  const uint32_t hx = hbits(p.x - ox), hy = hbits(p.y - oy), hz = hbits(p.z - oz), hw = hbits(p.w);
  xyzw[i] = make_float4(ox + hval(hx), oy + hval(hy), oz + hval(hz), hval(hw));
  posq[i] = make_uint2(hx | (hy << 16), hz);  // the high half of .y receives the culling radius later
}

__global__ void k_quantize_weights(float4* __restrict__ w4, const float4* __restrict__ rec0, uint64_t n,
                                   uint2* __restrict__ posq, uint2* __restrict__ colq, float* __restrict__ reval) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 w = w4[i];
  const uint32_t a = hbits(w.x), r = hbits(w.y), g = hbits(w.z), b = hbits(w.w);
  w4[i] = make_float4(hval(a), hval(r), hval(g), hval(b));
  const uint2 q = posq[i];
  const float re = rec0[i].w;
  const uint32_t rc = (uint32_t)__half_as_ushort(__float2half_ru(re));  // rounded up: culling only
  posq[i] = make_uint2(q.x, (q.y & 0xffffu) | (rc << 16));
  colq[i] = make_uint2(r | (g << 16), b | (a << 16));
  reval[i] = re;
}

}  // namespace

cudaError_t launch_quantize_positions(float4* xyzw, uint64_t n, uint2* posq, float4* origin, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_quantize_positions<<<(unsigned)((n + kRun - 1) / kRun), kRun, 0, st>>>(xyzw, n, posq, origin);
  return cudaGetLastError();
}

cudaError_t launch_quantize_weights(float4* w4, const float4* rec0, uint64_t n, uint2* posq, uint2* colq,
                                   float* reval, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_quantize_weights<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(w4, rec0, n, posq, colq, reval);
  return cudaGetLastError();
}

}  // namespace aarbf
