// preprocess.cu -- device side of the reference's host preprocessing (hostCode.cpp:183-250):
// space-time domain reduction, 16-bit quantisation + 3-D Hilbert keys, a stable LSD radix
// sort (hand written: per-tile histogram, exclusive scan, stable warp-multisplit scatter through
// shared memory), the in-place ordering of equal-key runs (the lexicographic LSD chain for long
// runs) and the gather that normalises attributes.
#include <cfloat>

#include "aarbf_internal.h"

namespace aarbf {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per tile
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---- domain reduction ---------------------------------------------------------------------

__global__ void k_domain_partial(const float4* __restrict__ p, uint64_t n, float* __restrict__ part) {
  float v[8] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX};
  float bad = 0.0f;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    float4 q = __ldg(p + i);
    if (!(fabsf(q.x) <= FLT_MAX && fabsf(q.y) <= FLT_MAX && fabsf(q.z) <= FLT_MAX &&
          fabsf(q.w) <= FLT_MAX))
      bad = 1.0f;
    v[0] = fminf(v[0], q.x); v[1] = fminf(v[1], q.y); v[2] = fminf(v[2], q.z);
    v[3] = fmaxf(v[3], q.x); v[4] = fmaxf(v[4], q.y); v[5] = fmaxf(v[5], q.z);
    v[6] = fminf(v[6], q.w); v[7] = fmaxf(v[7], q.w);
  }
  __shared__ float sh[8][32];
  __shared__ float shbad[32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    float x = v[k];
    for (int o = 16; o; o >>= 1) {
      float y = __shfl_xor_sync(0xffffffffu, x, o);
      x = (k < 3 || k == 6) ? fminf(x, y) : fmaxf(x, y);
    }
    if (lane == 0) sh[k][warp] = x;
  }
  for (int o = 16; o; o >>= 1) bad = fmaxf(bad, __shfl_xor_sync(0xffffffffu, bad, o));
  if (lane == 0) shbad[warp] = bad;
  __syncthreads();
  if (threadIdx.x < 8) {
    int k = threadIdx.x;
    float x = sh[k][0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      x = (k < 3 || k == 6) ? fminf(x, sh[k][w]) : fmaxf(x, sh[k][w]);
    part[9 * blockIdx.x + k] = x;
  }
  if (threadIdx.x == 8) {
    float b = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = fmaxf(b, shbad[w]);
    part[9 * blockIdx.x + 8] = b;
  }
}

// ---- Hilbert keys -------------------------------------------------------------------------

__global__ void k_hilbert_keys(const float4* __restrict__ p, const uint32_t* __restrict__ perm,
                               uint64_t n, float d0, float d1, float d2, float d3, float d4, float d5,
                               uint64_t* __restrict__ keys, uint32_t* __restrict__ ident) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t src = perm ? perm[i] : (uint32_t)i;
  float4 q = __ldg(p + src);
  uint64_t c0 = quantise16(q.x, d0, d3);
  uint64_t c1 = quantise16(q.y, d1, d4);
  uint64_t c2 = quantise16(q.z, d2, d5);
  keys[i] = hilbert3x16(c0, c1, c2);
  if (ident) ident[i] = (uint32_t)i;
}

// float -> order-preserving u32 (+0 and -0 map to the same value, as float compare treats them)
__device__ __forceinline__ uint32_t orderable(float f) {
  if (f == 0.0f) return 0x80000000u;
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_orderable(const float4* __restrict__ p, const uint32_t* __restrict__ perm, uint64_t n,
                            int comp, uint64_t* __restrict__ out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 q = __ldg(p + perm[i]);
  float f = comp == 0 ? q.x : (comp == 1 ? q.y : (comp == 2 ? q.z : q.w));
  out[i] = orderable(f);
}

// (x, y, z, w, input index) of particle a before that of particle b, each coordinate compared as
// floats compare (orderable() maps +0 and -0 together)
__device__ __forceinline__ bool tie_less(float4 a, uint32_t ia, float4 b, uint32_t ib) {
  uint32_t ua = orderable(a.x), ub = orderable(b.x);
  if (ua != ub) return ua < ub;
  ua = orderable(a.y), ub = orderable(b.y);
  if (ua != ub) return ua < ub;
  ua = orderable(a.z), ub = orderable(b.z);
  if (ua != ub) return ua < ub;
  ua = orderable(a.w), ub = orderable(b.w);
  if (ua != ub) return ua < ub;
  return ia < ib;
}

// Runs of equal keys after the stable key sort from the identity hold their particles in input
// order. The reference sorts (key, float4) pairs (hostCode.cpp:212-222), so equal keys are
// ordered by x, then y, z, w; equal particles keep input order here. The thread at the start of
// each run sorts a run of at most kMaxTieRun entries in place (insertion sort on perm); a longer
// run sets bit 1 of *flag and is left to the full LSD chain over (w, z, y, x, key). Bit 0 is set
// when any run exists.
constexpr int kMaxTieRun = 64;

__global__ void k_tie_runs(const uint64_t* __restrict__ keys, const float4* __restrict__ p,
                           uint32_t* __restrict__ perm, uint64_t n, uint32_t* flag) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i + 1 >= n) return;
  const uint64_t k = keys[i];
  if (keys[i + 1] != k || (i > 0 && keys[i - 1] == k)) return;
  uint64_t e = i + 2;
  while (e < n && e - i <= (uint64_t)kMaxTieRun && keys[e] == k) ++e;
  if (e - i > (uint64_t)kMaxTieRun) {
    atomicOr(flag, 3u);
    return;
  }
  atomicOr(flag, 1u);
  for (uint64_t a = i + 1; a < e; ++a) {
    const uint32_t v = perm[a];
    const float4 q = __ldg(p + v);
    uint64_t b = a;
    while (b > i) {
      const uint32_t u = perm[b - 1];
      if (!tie_less(q, v, __ldg(p + u), u)) break;
      perm[b] = u;
      --b;
    }
    perm[b] = v;
  }
}

__global__ void k_gather_normalize(const float4* __restrict__ in, const float* __restrict__ rin,
                                   const uint32_t* __restrict__ perm, uint64_t n, float amin, float amax,
                                   float4* __restrict__ out, float* __restrict__ rout) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t s = perm[i];
  float4 q = __ldg(in + s);
  if (amax > amin) q.w = (q.w - amin) / (amax - amin);
  out[i] = q;
  if (rin) rout[i] = __ldg(rin + s);
}

// ---- radix sort ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint64_t* __restrict__ keys, uint64_t n,
                                                             int shift, uint32_t* __restrict__ hist,
                                                             uint32_t ntiles) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    uint64_t idx = base + (uint64_t)k * kSortThreads + threadIdx.x;
    if (idx < n) atomicAdd(&h[(uint32_t)(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// block-wide exclusive scan of one value per thread; returns the block total in *total
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums, uint32_t* total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < nw ? warp_sums[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_sums[lane] = s;  // inclusive warp prefix
  }
  __syncthreads();
  uint32_t warp_off = warp ? warp_sums[warp - 1] : 0u;
  *total = warp_sums[nw - 1];
  __syncthreads();
  return warp_off + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t* __restrict__ in, uint64_t n,
                                                              uint32_t* __restrict__ sums) {
  __shared__ uint32_t ws[32];
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += in[base + k];
  uint32_t total;
  block_exclusive_scan(s, ws, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// single block: exclusive scan of the tile sums, carried across chunks
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(uint32_t* sums, uint64_t m) {
  __shared__ uint32_t ws[32];
  uint32_t carry = 0;
  for (uint64_t base = 0; base < m; base += kScanThreads) {
    uint64_t i = base + threadIdx.x;
    uint32_t v = i < m ? sums[i] : 0u;
    uint32_t total;
    uint32_t ex = block_exclusive_scan(v, ws, &total);
    if (i < m) sums[i] = carry + ex;
    carry += total;
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(uint32_t* __restrict__ data, uint64_t n,
                                                             const uint32_t* __restrict__ sums) {
  __shared__ uint32_t ws[32];
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? data[base + k] : 0u;
    s += v[k];
  }
  uint32_t total;
  uint32_t ex = block_exclusive_scan(s, ws, &total) + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) data[base + k] = ex;
    ex += v[k];
  }
}

// stable scatter: warp w of a tile owns keys [w*256, (w+1)*256) of the tile and walks them in
// 8 batches of 32 in input order; ranks inside a batch come from __match_any_sync. The tile is
// first reordered by digit in shared memory, then written out by consecutive threads, so that a
// warp's stores fall into few runs of consecutive addresses (one per digit it covers).
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(
    const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint64_t* __restrict__ kout,
    uint32_t* __restrict__ vout, uint64_t n, int shift, const uint32_t* __restrict__ offs, uint32_t ntiles) {
  constexpr int kWarps = kSortThreads / 32;
  static_assert(kSortThreads == 256, "one thread per digit");
  __shared__ uint32_t cnt[kWarps][256];
  __shared__ uint32_t gofs[256];
  __shared__ uint32_t lstart[256];
  __shared__ uint32_t ws[32];
  __shared__ uint64_t sk[kSortTile];
  __shared__ uint32_t sv[kSortTile];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) cnt[w][threadIdx.x] = 0;
  gofs[threadIdx.x] = offs[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
  __syncthreads();
  const uint64_t tile0 = (uint64_t)blockIdx.x * kSortTile;
  const uint64_t base = tile0 + (uint64_t)warp * (32 * kSortItems);
  uint64_t k[kSortItems];
  uint32_t v[kSortItems], pos[kSortItems], dig[kSortItems];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int b = 0; b < kSortItems; ++b) {
    uint64_t idx = base + (uint64_t)b * 32 + lane;
    bool valid = idx < n;
    k[b] = valid ? kin[idx] : 0ull;
    v[b] = valid ? vin[idx] : 0u;
    uint32_t d = valid ? ((uint32_t)(k[b] >> shift) & 255u) : 256u;
    dig[b] = d;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t rank = __popc(peers & lt);
    uint32_t before = valid ? cnt[warp][d] : 0u;
    __syncwarp();
    if (valid && rank == 0) cnt[warp][d] = before + __popc(peers);
    __syncwarp();
    pos[b] = before + rank;
  }
  __syncthreads();
  // per digit (thread = digit): exclusive prefix over the warps, then over the digits
  uint32_t run = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    uint32_t c = cnt[w][threadIdx.x];
    cnt[w][threadIdx.x] = run;
    run += c;
  }
  uint32_t tile_total;
  lstart[threadIdx.x] = block_exclusive_scan(run, ws, &tile_total);
  __syncthreads();
#pragma unroll
  for (int b = 0; b < kSortItems; ++b) {
    if (dig[b] < 256u) {
      uint32_t lp = lstart[dig[b]] + cnt[warp][dig[b]] + pos[b];
      sk[lp] = k[b];
      sv[lp] = v[b];
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    uint32_t j = (uint32_t)r * kSortThreads + threadIdx.x;
    if (j < tile_total) {
      uint64_t key = sk[j];
      uint32_t d = (uint32_t)(key >> shift) & 255u;
      uint32_t dst = gofs[d] + (j - lstart[d]);
      kout[dst] = key;
      vout[dst] = sv[j];
    }
  }
}

cudaError_t exclusive_scan(uint32_t* data, uint64_t n, uint32_t* sums, cudaStream_t st) {
  uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 0) return cudaSuccess;
  k_scan_reduce<<<(unsigned)tiles, kScanThreads, 0, st>>>(data, n, sums);
  k_scan_sums<<<1, kScanThreads, 0, st>>>(sums, tiles);
  k_scan_apply<<<(unsigned)tiles, kScanThreads, 0, st>>>(data, n, sums);
  return cudaGetLastError();
}

inline unsigned blocks_for(uint64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

size_t radix_sort_hist_words(uint64_t n) {
  uint64_t ntiles = (n + kSortTile - 1) / kSortTile;
  uint64_t hw = 256 * ntiles;
  uint64_t scan_tiles = (hw + kScanTile - 1) / kScanTile;
  return (size_t)(hw + scan_tiles + 64);
}

cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                             uint64_t n, int key_bits, uint32_t* hist, size_t hist_words, cudaStream_t st,
                             bool* result_in_alt) {
  *result_in_alt = false;
  if (n <= 1) return cudaSuccess;
  uint32_t ntiles = (uint32_t)((n + kSortTile - 1) / kSortTile);
  uint64_t hw = 256ull * ntiles;
  if (hist_words < radix_sort_hist_words(n)) return cudaErrorInvalidValue;
  uint32_t* sums = hist + hw;
  uint64_t *ki = keys, *ko = keys_alt;
  uint32_t *vi = vals, *vo = vals_alt;
  for (int shift = 0; shift < key_bits; shift += 8) {
    k_radix_hist<<<ntiles, kSortThreads, 0, st>>>(ki, n, shift, hist, ntiles);
    cudaError_t e = exclusive_scan(hist, hw, sums, st);
    if (e != cudaSuccess) return e;
    k_radix_scatter<<<ntiles, kSortThreads, 0, st>>>(ki, vi, ko, vo, n, shift, hist, ntiles);
    uint64_t* tk = ki; ki = ko; ko = tk;
    uint32_t* tv = vi; vi = vo; vo = tv;
  }
  *result_in_alt = (ki == keys_alt);
  return cudaGetLastError();
}

cudaError_t launch_domain_reduce(const float4* p, uint64_t n, float* d_partial, int nblocks, cudaStream_t st) {
  k_domain_partial<<<nblocks, 256, 0, st>>>(p, n, d_partial);
  return cudaGetLastError();
}

cudaError_t launch_hilbert_keys(const float4* p, uint64_t n, const float* dom, uint64_t* keys, uint32_t* perm,
                                cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_hilbert_keys<<<blocks_for(n, 256), 256, 0, st>>>(p, nullptr, n, dom[0], dom[1], dom[2], dom[3], dom[4],
                                                    dom[5], keys, perm);
  return cudaGetLastError();
}

cudaError_t launch_hilbert_keys_perm(const float4* p, const uint32_t* perm, uint64_t n, const float* dom,
                                     uint64_t* keys, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_hilbert_keys<<<blocks_for(n, 256), 256, 0, st>>>(p, perm, n, dom[0], dom[1], dom[2], dom[3], dom[4],
                                                    dom[5], keys, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_tie_runs(const uint64_t* keys, const float4* p, uint32_t* perm, uint64_t n, uint32_t* flag,
                            cudaStream_t st) {
  if (n < 2) return cudaSuccess;
  k_tie_runs<<<blocks_for(n, 256), 256, 0, st>>>(keys, p, perm, n, flag);
  return cudaGetLastError();
}

cudaError_t launch_orderable_component(const float4* p, const uint32_t* perm, uint64_t n, int comp,
                                       uint64_t* out, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_orderable<<<blocks_for(n, 256), 256, 0, st>>>(p, perm, n, comp, out);
  return cudaGetLastError();
}

cudaError_t launch_gather_normalize(const float4* in, const float* radii_in, const uint32_t* perm, uint64_t n,
                                    float amin, float amax, float4* out, float* radii_out, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_gather_normalize<<<blocks_for(n, 256), 256, 0, st>>>(in, radii_in, perm, n, amin, amax, out, radii_out);
  return cudaGetLastError();
}

}  // namespace aarbf
