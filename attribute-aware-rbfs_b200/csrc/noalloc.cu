// noalloc.cu -- an allocation-free variant of the Hilbert-key sort that aarbf_build runs.
//
// Some callers cannot call cudaMalloc: applications whose device memory is handed out by their
// own pool or arena, which forbids allocations made behind its back, and real-time render loops
// that must not reach the allocator (cudaMalloc and cudaFree can synchronise the whole device)
// once they are running. aarbf_hilbert_sort_noalloc serves them: the caller passes the particles
// and the two outputs; the sort's working space (the radix sort's second key/index buffers, its
// histograms and a flag) is one file-scope __device__ array of a fixed size, so nothing is
// allocated per call.
//
// Limits and sharing rules:
//  - at most kNoallocMaxParticles particles per call; larger inputs are rejected;
//  - the array exists once per device that loads the library and stays allocated until the
//    process exits (about 12.5 MiB);
//  - every call on a device uses the same array, and it keeps whatever the last call left in it:
//    the call clears the one part that must start at zero (the tie flag); two calls whose GPU
//    work overlaps in time (different streams, or host threads) race on it and must be ordered
//    by the caller;
//  - the first call on a device resolves the array's device address (cudaGetSymbolAddress, with
//    that device current) and caches it; make that first call before any stream capture. The
//    cached address belongs to the device's primary context: it must not outlive a
//    cudaDeviceReset of that device;
//  - xyzw, keys and perm must be device (or managed) memory: host pointers are refused with
//    AARBF_ERR_INVALID_ARGUMENT before any GPU work (cudaPointerGetAttributes, which allocates
//    nothing).
#include <cstring>
#include <mutex>

#include "aarbf_internal.h"

namespace aarbf {

namespace {

constexpr uint64_t kNoallocMaxParticles = 1ull << 20;
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
// hist words of radix_sort_hist_words(kNoallocMaxParticles): 256 per 2048-key tile, one scan
// sum per 4096 words, plus 64 spare
constexpr size_t kHistWords = 256 * (kNoallocMaxParticles / 2048) + (256 * (kNoallocMaxParticles / 2048)) / 4096 + 64;
constexpr size_t kOffKeysAlt = 0;
constexpr size_t kOffPermAlt = kOffKeysAlt + align256(8 * kNoallocMaxParticles);
constexpr size_t kOffHist = kOffPermAlt + align256(4 * kNoallocMaxParticles);
constexpr size_t kOffFlag = kOffHist + align256(4 * kHistWords);
constexpr size_t kScratchBytes = kOffFlag + 256;

// The working space. In host code this name is a host-side stand-in, not a device address; the
// device address comes from cudaGetSymbolAddress below.
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// true for memory a kernel on the current device may read and write
bool device_accessible(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the (non-sticky) error the query recorded
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

}  // namespace aarbf

using namespace aarbf;

extern "C" aarbf_status aarbf_hilbert_sort_noalloc(const float* xyzw, uint64_t n, const float* dom, uint64_t* keys,
                                                   uint32_t* perm, void* stream) {
  if (n > kNoallocMaxParticles) return AARBF_ERR_INVALID_ARGUMENT;
  if (n && (!xyzw || !dom || !keys || !perm)) return AARBF_ERR_INVALID_ARGUMENT;
  if (!n) return AARBF_OK;
  if (!device_accessible(xyzw) || !device_accessible(keys) || !device_accessible(perm))
    return AARBF_ERR_INVALID_ARGUMENT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return AARBF_ERR_CUDA;
  unsigned char* base;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) return AARBF_ERR_CUDA;
      g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    }
    base = g_scratch_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  uint64_t* keys_alt = reinterpret_cast<uint64_t*>(base + kOffKeysAlt);
  uint32_t* perm_alt = reinterpret_cast<uint32_t*>(base + kOffPermAlt);
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + kOffHist);
  uint32_t* flag = reinterpret_cast<uint32_t*>(base + kOffFlag);
  const float4* in = reinterpret_cast<const float4*>(xyzw);
  if (radix_sort_hist_words(n) > kHistWords) return AARBF_ERR_INVALID_ARGUMENT;

  // same steps as aarbf_build: keys + identity, 48-bit radix sort, short runs of equal keys
  // ordered in place, and for a longer run the stable LSD chain over (w, z, y, x) then the key
  bool alt = false;
  if (launch_hilbert_keys(in, n, dom, keys, perm, st) != cudaSuccess) return AARBF_ERR_CUDA;
  if (radix_sort_pairs(keys, perm, keys_alt, perm_alt, n, 48, hist, kHistWords, st, &alt) != cudaSuccess)
    return AARBF_ERR_CUDA;
  if (alt) {
    if (cudaMemcpyAsync(keys, keys_alt, 8 * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(perm, perm_alt, 4 * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return AARBF_ERR_CUDA;
  }
  uint32_t tie = 0;
  if (cudaMemsetAsync(flag, 0, 4, st) != cudaSuccess || launch_tie_runs(keys, in, perm, n, flag, st) != cudaSuccess ||
      cudaMemcpyAsync(&tie, flag, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return AARBF_ERR_CUDA;
  if (!(tie & 2u)) return AARBF_OK;
  uint64_t *k0 = keys, *k1 = keys_alt;
  uint32_t *p0 = perm, *p1 = perm_alt;
  if (launch_hilbert_keys(in, n, dom, k0, p0, st) != cudaSuccess) return AARBF_ERR_CUDA;
  for (int comp = 3; comp >= -1; --comp) {
    cudaError_t e = comp >= 0 ? launch_orderable_component(in, p0, n, comp, k0, st)
                              : launch_hilbert_keys_perm(in, p0, n, dom, k0, st);
    if (e != cudaSuccess) return AARBF_ERR_CUDA;
    bool a2 = false;
    if (radix_sort_pairs(k0, p0, k1, p1, n, comp >= 0 ? 32 : 48, hist, kHistWords, st, &a2) != cudaSuccess)
      return AARBF_ERR_CUDA;
    if (a2) {
      uint64_t* tk = k0;
      k0 = k1;
      k1 = tk;
      uint32_t* tp = p0;
      p0 = p1;
      p1 = tp;
    }
  }
  if (k0 != keys) {
    if (cudaMemcpyAsync(keys, k0, 8 * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(perm, p0, 4 * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return AARBF_ERR_CUDA;
  }
  return AARBF_OK;
}
