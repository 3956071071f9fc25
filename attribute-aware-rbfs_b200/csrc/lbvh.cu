// lbvh.cu -- the reference's bounds program (deviceCodeBounds.hlsl:29-82) turned into an LBVH
// builder: per-particle shading prepass, Karras (HPG 2012) radix tree over the leaf clusters'
// Hilbert keys, and a bottom-up refit with atomic arrival counters.
//
// The refit produces two box sets over one topology:
//  - reference bounds: leaf boxes exactly as GenRBFBounds computes them (radius from the radius
//    map, every particle whose radius-map value is non-zero) -- the bounds output, and the tree
//    the splat kernel traverses (splatting ignores opacity, deviceCodeSplat.hlsl:156-187);
//  - traversal bounds: leaf boxes over the particles that can be hit (r_eval > 0), the tree the
//    tracking kernels traverse. Particles outside it never contribute, so results are unchanged.
#include "aarbf_internal.h"

namespace aarbf {

namespace {

inline unsigned blocks_for(uint64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// radius (deviceCodeRBF.hlsl:349-351, deviceCodeBounds.hlsl:59) and the per-particle any-hit
// weights (deviceCodeRBF.hlsl:366-376), evaluated once per particle instead of once per hit.
// Opacity 0, or below alpha_floor, marks a particle transparent (deviceCodeRBF.hlsl:369-372).
__global__ void k_prepass(const float4* __restrict__ xyzw, const float* __restrict__ radii, uint64_t n,
                          const float4* __restrict__ tf_color, int nc, const float* __restrict__ tf_radius,
                          int nr, float rbf_radius, float alpha_floor, float4* __restrict__ rec0,
                          float4* __restrict__ w4, float* __restrict__ rgeom) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = __ldg(xyzw + i);
  float rp = tex1(tf_radius, nr, p.w);
  float base = radii ? __ldg(radii + i) : rbf_radius;
  float r = base * rp;
  float4 col = tex4(tf_color, nc, p.w);
  rgeom[i] = (rp == 0.0f) ? -1.0f : r;
  if (col.w == 0.0f || col.w < alpha_floor) {
    rec0[i] = make_float4(p.x, p.y, p.z, 0.0f);
    w4[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  } else {
    float a3 = (col.w * col.w) * col.w;
    rec0[i] = make_float4(p.x, p.y, p.z, r);
    w4[i] = make_float4(a3, dpow(col.x, 2.2f) * a3, dpow(col.y, 2.2f) * a3, dpow(col.z, 2.2f) * a3);
  }
}

__device__ __forceinline__ int delta(const uint64_t* __restrict__ keys, uint32_t ppl, int64_t L, int64_t i,
                                     int64_t j) {
  if (j < 0 || j >= L) return -1;
  uint64_t a = __ldg(keys + (uint64_t)i * ppl), b = __ldg(keys + (uint64_t)j * ppl);
  uint64_t x = a ^ b;
  if (x == 0) return 64 + __clz((int)((uint32_t)i ^ (uint32_t)j));
  return __clzll((long long)x);
}

// leaf l's key is the key of its first particle; equal keys are ordered by leaf index
__global__ void k_karras(const uint64_t* __restrict__ keys, uint32_t ppl, uint32_t nleaves, Node* nodes,
                         Node* nodes_ref, uint32_t* leaf_parent) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t L = nleaves;
  if (i >= L - 1) return;
  int d = (delta(keys, ppl, L, i, i + 1) - delta(keys, ppl, L, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = delta(keys, ppl, L, i, i - d);
  int64_t lmax = 2;
  while (delta(keys, ppl, L, i, i + lmax * d) > dmin) lmax *= 2;
  int64_t l = 0;
  for (int64_t t = lmax / 2; t >= 1; t /= 2)
    if (delta(keys, ppl, L, i, i + (l + t) * d) > dmin) l += t;
  int64_t j = i + l * d;
  int dnode = delta(keys, ppl, L, i, j);
  int64_t s = 0, step = l;
  do {
    step = (step + 1) >> 1;
    if (delta(keys, ppl, L, i, i + (s + step) * d) > dnode) s += step;
  } while (step > 1);
  int64_t g = i + s * d + (d < 0 ? -1 : 0);
  int64_t lo = i < j ? i : j, hi = i < j ? j : i;
  uint32_t left = (lo == g) ? ((uint32_t)g | kLeafBit) : (uint32_t)g;
  uint32_t right = (hi == g + 1) ? ((uint32_t)(g + 1) | kLeafBit) : (uint32_t)(g + 1);
  Node* trees[2] = {nodes, nodes_ref};
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    Node* nd = trees[t];
    nd[i].d.x = left;
    nd[i].d.y = right;
    nd[i].d.w = (uint32_t)j;  // the other end of the node's leaf range [min(i, j), max(i, j)]
    if (i == 0) nd[0].d.z = 0xffffffffu;
    if (!(left & kLeafBit)) nd[left].d.z = (uint32_t)i;
    if (!(right & kLeafBit)) nd[right].d.z = (uint32_t)i;
  }
  if (left & kLeafBit) leaf_parent[left & ~kLeafBit] = (uint32_t)i;
  if (right & kLeafBit) leaf_parent[right & ~kLeafBit] = (uint32_t)i;
}

__device__ __forceinline__ void write_slot(Node* node, int slot, const float* lo, const float* hi) {
  float* f = reinterpret_cast<float*>(node) + 6 * slot;
  f[0] = lo[0]; f[1] = lo[1]; f[2] = lo[2];
  f[3] = hi[0]; f[4] = hi[1]; f[5] = hi[2];
}

__device__ __forceinline__ void read_union(const Node* node, float* lo, float* hi) {
  const float* f = reinterpret_cast<const float*>(node);
  float v[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) v[k] = __ldcg(f + k);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = fminf(v[a], v[6 + a]);
    hi[a] = fmaxf(v[3 + a], v[9 + a]);
  }
}

__device__ __forceinline__ void nan_if_empty(float* lo, float* hi) {
  if (lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]) {
    const float nan = __int_as_float(0x7fc00000);
    lo[0] = lo[1] = lo[2] = hi[0] = hi[1] = hi[2] = nan;
  }
}

// one thread per leaf: GenRBFBounds (deviceCodeBounds.hlsl:45-81) and the traversal box, then
// walk up the tree; the second child to arrive at an internal node computes both of its boxes.
constexpr int kRefitBlock = 256;  // threads (leaves) per refit block

__global__ void __launch_bounds__(kRefitBlock) k_refit(const float4* __restrict__ rec0, const float* __restrict__ rgeom, uint64_t n,
                        uint32_t ppl, uint32_t nleaves, Node* nodes, Node* nodes_ref,
                        const uint32_t* __restrict__ leaf_parent, uint32_t* counters, float* __restrict__ leaf_box,
                        float* __restrict__ leaf_eff, float* __restrict__ root_box, uint32_t* status) {
  // per inner node of this block's window: both children's boxes of both trees, arrival count
  __shared__ float s_box[kRefitBlock * 24];
  __shared__ uint32_t s_cnt[kRefitBlock];
  s_cnt[threadIdx.x] = 0u;
  __syncthreads();
  uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (l >= nleaves) return;
  const float inf = __int_as_float(0x7f800000);
  float lo[3] = {inf, inf, inf}, hi[3] = {-inf, -inf, -inf};     // reference bounds
  float elo[3] = {inf, inf, inf}, ehi[3] = {-inf, -inf, -inf};   // traversal bounds
  for (uint32_t k = 0; k < ppl; ++k) {
    uint64_t i = l * ppl + k;
    if (i >= n) break;
    float4 p = __ldg(rec0 + i);
    float r = __ldg(rgeom + i);
    if (r >= 0.0f) {  // radiusPercent != 0
      lo[0] = fminf(lo[0], p.x - r); lo[1] = fminf(lo[1], p.y - r); lo[2] = fminf(lo[2], p.z - r);
      hi[0] = fmaxf(hi[0], p.x + r); hi[1] = fmaxf(hi[1], p.y + r); hi[2] = fmaxf(hi[2], p.z + r);
    }
    if (p.w > 0.0f) {
      elo[0] = fminf(elo[0], p.x - p.w); elo[1] = fminf(elo[1], p.y - p.w); elo[2] = fminf(elo[2], p.z - p.w);
      ehi[0] = fmaxf(ehi[0], p.x + p.w); ehi[1] = fmaxf(ehi[1], p.y + p.w); ehi[2] = fmaxf(ehi[2], p.z + p.w);
    }
  }
  nan_if_empty(lo, hi);
  nan_if_empty(elo, ehi);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    leaf_box[6 * l + a] = lo[a];
    leaf_box[6 * l + 3 + a] = hi[a];
    leaf_eff[6 * l + a] = elo[a];
    leaf_eff[6 * l + 3 + a] = ehi[a];
  }
  if (nleaves == 1) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      root_box[a] = elo[a];
      root_box[3 + a] = ehi[a];
    }
    return;
  }
  // Climb. An inner node whose leaf range lies in this block's leaves [b0, b0 + blockDim) has
  // index in that window too and only this block's threads arrive at it: those nodes meet in
  // shared memory (block-scope fences, shared arrival counters). The first node reaching outside
  // the window, and every ancestor of it, meets in global memory (device-scope fences).
  const uint32_t b0 = blockIdx.x * blockDim.x;
  bool local = true;
  uint32_t child = (uint32_t)l | kLeafBit;
  uint32_t parent = leaf_parent[l];
  for (int guard = 0; guard < 256; ++guard) {
    Node* pn = nodes + parent;
    Node* pr = nodes_ref + parent;
    int slot = (pn->d.x == child) ? 0 : 1;
    write_slot(pn, slot, elo, ehi);
    write_slot(pr, slot, lo, hi);
    if (local) {
      const uint32_t j = pn->d.w;
      const uint32_t first = parent < j ? parent : j, last = parent < j ? j : parent;
      local = first >= b0 && last < b0 + blockDim.x;
    }
    if (local) {
      const uint32_t q = parent - b0;  // first <= parent <= last: inside the window
      float* mine = s_box + q * 24u + (uint32_t)slot * 12u;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        mine[a] = elo[a];
        mine[3 + a] = ehi[a];
        mine[6 + a] = lo[a];
        mine[9 + a] = hi[a];
      }
      __threadfence_block();
      if (atomicAdd(s_cnt + q, 1u) == 0u) return;
      __threadfence_block();
      const float* other = s_box + q * 24u + (uint32_t)(1 - slot) * 12u;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        elo[a] = fminf(elo[a], other[a]);
        ehi[a] = fmaxf(ehi[a], other[3 + a]);
        lo[a] = fminf(lo[a], other[6 + a]);
        hi[a] = fmaxf(hi[a], other[9 + a]);
      }
    } else {
      // release the slot before the arrival count, acquire the sibling's slot after it
      // (acquire-release fences: the message-passing pattern needs no sequentially consistent fence)
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      if (atomicAdd(counters + parent, 1u) == 0u) return;
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      read_union(pn, elo, ehi);
      read_union(pr, lo, hi);
    }
    uint32_t up = pn->d.z;
    if (up == 0xffffffffu) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        root_box[a] = elo[a];
        root_box[3 + a] = ehi[a];
      }
      return;
    }
    child = parent;
    parent = up;
  }
  // a Karras tree over 48-bit keys with index tie-breaks is at most 80 levels deep, so the
  // climb cannot run out of its 256 iterations on a well-formed tree; report it if it does
  atomicOr(status, kStatusLoopCap);
}

// largest non-negative bounds radius (max over the float bits, which order like the values)
__global__ void k_max_radius(const float* __restrict__ rgeom, uint64_t n, int* __restrict__ out) {
  float m = 0.0f;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    m = fmaxf(m, __ldg(rgeom + i));
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(out, __float_as_int(m));
}

// one thread per binary inner node: its wide node
__global__ void k_collapse(const Node* __restrict__ nodes, uint32_t ninternal, WideNode* __restrict__ wide) {
  const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= ninternal) return;
  constexpr int W = kBvhWidth;
  float box[W][6];
  uint32_t code[W];
  int k = 0;
  auto take = [&](const Node& nd, int c, int at) {
    const float* f = reinterpret_cast<const float*>(&nd);
    for (int q = 0; q < 6; ++q) box[at][q] = f[6 * c + q];
    code[at] = c == 0 ? nd.d.x : nd.d.y;
  };
  const Node root = nodes[n];
  take(root, 0, k++);
  take(root, 1, k++);
  // open the inner entry of largest surface area until the node is full
  while (k < W) {
    int best = -1;
    float barea = -1.0f;
    for (int j = 0; j < k; ++j) {
      if (code[j] & kLeafBit) continue;
      const float dx = box[j][3] - box[j][0], dy = box[j][4] - box[j][1], dz = box[j][5] - box[j][2];
      const float area = (dx * dy + dy * dz) + dz * dx;
      if (area > barea) {  // empty (NaN) subtrees are never opened
        barea = area;
        best = j;
      }
    }
    if (best < 0) break;
    const Node g = nodes[code[best]];
    take(g, 0, best);
    take(g, 1, k++);
  }
  WideNode w;
  for (int j = 0; j < W; ++j) {
    if (j < k) {
      w.s[2 * j] = make_float4(box[j][0], box[j][1], box[j][2], box[j][3]);
      w.s[2 * j + 1] = make_float4(box[j][4], box[j][5], __uint_as_float(code[j]), 0.0f);
    } else {
      w.s[2 * j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      w.s[2 * j + 1] = make_float4(0.0f, 0.0f, __uint_as_float(0xffffffffu), 0.0f);
    }
  }
  wide[n] = w;
}

}  // namespace

cudaError_t launch_prepass(const float4* xyzw, const float* radii, uint64_t n, const float4* tf_color, int nc,
                           const float* tf_radius, int nr, float rbf_radius, float alpha_floor, float4* rec0,
                           float4* w4, float* rgeom, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_prepass<<<blocks_for(n, 256), 256, 0, st>>>(xyzw, radii, n, tf_color, nc, tf_radius, nr, rbf_radius,
                                                alpha_floor, rec0, w4, rgeom);
  return cudaGetLastError();
}

cudaError_t launch_max_radius(const float* rgeom, uint64_t n, float* out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float), st);
  if (e != cudaSuccess || !n) return e;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 4096) blocks = 4096;
  k_max_radius<<<blocks, 256, 0, st>>>(rgeom, n, reinterpret_cast<int*>(out));
  return cudaGetLastError();
}

cudaError_t launch_collapse(const Node* nodes, uint32_t nleaves, WideNode* wide, cudaStream_t st) {
  if (nleaves < 2) return cudaSuccess;
  const uint32_t ni = nleaves - 1;
  k_collapse<<<(ni + 255) / 256, 256, 0, st>>>(nodes, ni, wide);
  return cudaGetLastError();
}

cudaError_t launch_karras(const uint64_t* sorted_keys, uint64_t n, uint32_t ppl, uint32_t nleaves, Node* nodes,
                          Node* nodes_ref, uint32_t* leaf_parent, cudaStream_t st) {
  (void)n;
  if (nleaves < 2) return cudaSuccess;
  k_karras<<<blocks_for(nleaves - 1, 256), 256, 0, st>>>(sorted_keys, ppl, nleaves, nodes, nodes_ref, leaf_parent);
  return cudaGetLastError();
}

cudaError_t launch_refit(const float4* rec0, const float* rgeom, uint64_t n, uint32_t ppl, uint32_t nleaves,
                         Node* nodes, Node* nodes_ref, const uint32_t* leaf_parent, uint32_t* counters,
                         float* leaf_box, float* leaf_eff, float* root_box, uint32_t* status, cudaStream_t st) {
  if (!nleaves) return cudaSuccess;
  if (nleaves > 1) {
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(uint32_t) * (nleaves - 1), st);
    if (e != cudaSuccess) return e;
  }
  k_refit<<<blocks_for(nleaves, kRefitBlock), kRefitBlock, 0, st>>>(rec0, rgeom, n, ppl, nleaves, nodes, nodes_ref, leaf_parent,
                                                   counters, leaf_box, leaf_eff, root_box, status);
  return cudaGetLastError();
}

}  // namespace aarbf
