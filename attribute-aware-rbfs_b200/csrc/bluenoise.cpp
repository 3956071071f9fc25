// bluenoise.cpp -- the blue-noise threshold atlas of the stochastic-marching mode.
//
// The reference drives stochastic marching with spatio-temporal blue noise: an RGBA8 atlas of
// 8 x 16 tiles of 256 x 256 texels, frame f reading tile (f % 8, (f / 8) % 16)
// (deviceCodeRBF.hlsl:243-251, hostCode.cpp:337-352). Its stbn.png is not part of the reference
// snapshot, so the library generates an atlas of the same layout:
//  - one 256 x 256 blue-noise threshold tile by the void-and-cluster method (Ulichney 1993):
//    energy = the pattern convolved with a toroidal Gaussian (sigma 1.9); an initial random 10 %
//    pattern is relaxed by moving its tightest cluster into its largest void until stable; ranks
//    are then given by removing tightest clusters (down from the initial count) and by filling
//    largest voids (up to every texel); the texel value is rank / 256;
//  - frame f's tile is that tile offset by f times the golden-ratio conjugate, modulo 1, so each
//    texel's values over successive frames form the additive recurrence (R1) sequence, which is
//    well spread in time, while every frame stays a shifted blue-noise tile with exactly 256
//    texels of every 8-bit value.
// The tile is computed once per process (a few seconds of host time) and cached.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "aarbf_internal.h"

namespace aarbf {
namespace {

constexpr int kTile = 256;
constexpr int kTexels = kTile * kTile;
constexpr int kRadius = 8;  // Gaussian truncated at 8 texels (exp(-64 / (2 sigma^2)) < 2e-4)
constexpr double kSigma = 1.9;

// argmin / argmax over the texels by a tournament tree (ties: the lower index)
struct Tournament {
  std::vector<double> key;
  std::vector<int> node;  // node[1] = best leaf; leaves at kTexels + i
  bool max_wins;
  explicit Tournament(bool want_max) : key(kTexels), node(2 * kTexels), max_wins(want_max) {}
  bool better(int a, int b) const {
    if (key[a] != key[b]) return max_wins ? key[a] > key[b] : key[a] < key[b];
    return a < b;
  }
  void build() {
    for (int i = 0; i < kTexels; ++i) node[kTexels + i] = i;
    for (int i = kTexels - 1; i >= 1; --i) {
      const int l = node[2 * i], r = node[2 * i + 1];
      node[i] = better(l, r) ? l : r;
    }
  }
  void set(int i, double v) {
    key[i] = v;
    for (int p = (kTexels + i) >> 1; p >= 1; p >>= 1) {
      const int l = node[2 * p], r = node[2 * p + 1];
      node[p] = better(l, r) ? l : r;
    }
  }
  int best() const { return node[1]; }
};

struct VoidAndCluster {
  std::vector<double> energy;
  std::vector<uint8_t> on;
  Tournament cluster{true};  // over set texels: their energy; unset: -inf
  Tournament hole{false};    // over unset texels: their energy; set: +inf
  double kernel[2 * kRadius + 1][2 * kRadius + 1];

  VoidAndCluster() : energy(kTexels, 0.0), on(kTexels, 0) {
    for (int dy = -kRadius; dy <= kRadius; ++dy)
      for (int dx = -kRadius; dx <= kRadius; ++dx)
        kernel[dy + kRadius][dx + kRadius] = std::exp(-(double)(dx * dx + dy * dy) / (2.0 * kSigma * kSigma));
  }
  // add (sign +1) or remove (-1) a texel's Gaussian from the energy field (toroidal); only the
  // tree a texel competes in (set: clusters, unset: holes) sees its energy change
  void splat(int i, double sign) {
    const int x0 = i % kTile, y0 = i / kTile;
    for (int dy = -kRadius; dy <= kRadius; ++dy) {
      const int y = (y0 + dy + kTile) % kTile;
      for (int dx = -kRadius; dx <= kRadius; ++dx) {
        const int x = (x0 + dx + kTile) % kTile, j = y * kTile + x;
        energy[j] += sign * kernel[dy + kRadius][dx + kRadius];
        if (on[j]) cluster.set(j, energy[j]);
        else hole.set(j, energy[j]);
      }
    }
  }
  void turn_on(int i) {
    on[i] = 1;
    hole.set(i, INFINITY);
    splat(i, 1.0);
  }
  void turn_off(int i) {
    on[i] = 0;
    cluster.set(i, -INFINITY);
    splat(i, -1.0);
  }
};

// ranks 0 .. kTexels-1 of the void-and-cluster ordering
std::vector<int> void_and_cluster_ranks() {
  VoidAndCluster vc;
  // initial pattern: 10 % of the texels from a fixed splitmix64 stream
  uint64_t s = 0x243f6a8885a308d3ull;
  auto next = [&s]() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  };
  int ones = 0;
  while (ones < kTexels / 10) {
    const int i = (int)(next() % (uint64_t)kTexels);
    if (!vc.on[i]) {
      vc.on[i] = 1;
      ++ones;
    }
  }
  for (int i = 0; i < kTexels; ++i)
    if (vc.on[i]) {
      const int x0 = i % kTile, y0 = i / kTile;
      for (int dy = -kRadius; dy <= kRadius; ++dy)
        for (int dx = -kRadius; dx <= kRadius; ++dx)
          vc.energy[((y0 + dy + kTile) % kTile) * kTile + (x0 + dx + kTile) % kTile] +=
              vc.kernel[dy + kRadius][dx + kRadius];
    }
  for (int i = 0; i < kTexels; ++i) {
    vc.cluster.key[i] = vc.on[i] ? vc.energy[i] : -INFINITY;
    vc.hole.key[i] = vc.on[i] ? INFINITY : vc.energy[i];
  }
  vc.cluster.build();
  vc.hole.build();
  // relax: move the tightest cluster into the largest void until that changes nothing
  for (int guard = 0; guard < 4 * kTexels; ++guard) {
    const int c = vc.cluster.best();
    vc.turn_off(c);
    const int v = vc.hole.best();
    vc.turn_on(v);
    if (v == c) break;
  }
  const std::vector<double> energy0 = vc.energy;
  const std::vector<uint8_t> on0 = vc.on;
  std::vector<int> rank(kTexels, -1);
  // ranks below the initial count: remove tightest clusters
  for (int r = ones - 1; r >= 0; --r) {
    const int c = vc.cluster.best();
    vc.turn_off(c);
    rank[c] = r;
  }
  // ranks from the initial count up: fill largest voids (the inverted pattern's tightest clusters)
  vc.energy = energy0;
  vc.on = on0;
  for (int i = 0; i < kTexels; ++i) {
    vc.cluster.key[i] = vc.on[i] ? vc.energy[i] : -INFINITY;
    vc.hole.key[i] = vc.on[i] ? INFINITY : vc.energy[i];
  }
  vc.cluster.build();
  vc.hole.build();
  for (int r = ones; r < kTexels; ++r) {
    const int v = vc.hole.best();
    vc.turn_on(v);
    rank[v] = r;
  }
  return rank;
}

const std::vector<int>& cached_ranks() {
  static std::once_flag once;
  static std::vector<int> ranks;
  std::call_once(once, [] { ranks = void_and_cluster_ranks(); });
  return ranks;
}

}  // namespace
}  // namespace aarbf

extern "C" aarbf_status aarbf_generate_noise_atlas(uint8_t* out, int w, int h) {
  if (!out || w <= 0 || h <= 0) return AARBF_ERR_INVALID_ARGUMENT;
  const std::vector<int>& rank = aarbf::cached_ranks();
  // rank / kTexels + f * golden-ratio conjugate, modulo 1, in 2^-16 units (exact integer arithmetic)
  const uint32_t phi16 = 40503u;  // round(0.6180339887 * 65536)
  for (int y = 0; y < h; ++y) {
    for (int x = 0; x < w; ++x) {
      const uint32_t f = (uint32_t)(y / aarbf::kTile) * 8u + (uint32_t)(x / aarbf::kTile);
      const uint32_t r = (uint32_t)rank[(size_t)(y % aarbf::kTile) * aarbf::kTile + (size_t)(x % aarbf::kTile)];
      const uint32_t v = ((r + f * phi16) & 0xffffu) >> 8;
      uint8_t* t = out + 4 * ((size_t)y * (size_t)w + (size_t)x);
      t[0] = t[1] = t[2] = (uint8_t)v;
      t[3] = 255;
    }
  }
  return AARBF_OK;
}
