// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own hilbert.h and rng.h, unchanged, from where they lie in the
// reference tree (include path given by oracle/Makefile), and exports them under ref_* names
// so the oracle's restatements can be pinned against them. Output goes to oracle/_ref/ only.
//
// rng.h is HLSL-flavoured C: it needs the HLSL scalar/vector names `uint` and `uint2` and the
// parameter qualifier `inout`. `inout` is defined away, so lcg_random() works on a copy of its
// argument; the wrappers below therefore advance the state one step per call themselves.
#include <cmath>
#include <cstdint>

typedef unsigned int uint;
struct uint2 {
  uint x, y;
};
#define inout

#include "hilbert.h"
#include "rng.h"

extern "C" {

unsigned long long ref_hilbert_c2i(unsigned nDims, unsigned nBits, const unsigned long long *coord) {
  return hilbert_c2i(nDims, nBits, coord);
}

void ref_hilbert_i2c(unsigned nDims, unsigned nBits, unsigned long long index,
                     unsigned long long *coord) {
  hilbert_i2c(nDims, nBits, index, coord);
}

unsigned long long ref_bit_transpose(unsigned nDims, unsigned nBits, unsigned long long in) {
  return bitTranspose(nDims, nBits, in);
}

uint32_t ref_murmur_mix(uint32_t h, uint32_t k) { return murmur_hash3_mix(h, k); }
uint32_t ref_murmur_finalize(uint32_t h) { return murmur_hash3_finalize(h); }

uint32_t ref_get_rng(int frame_id, uint32_t px, uint32_t py, uint32_t dx, uint32_t dy) {
  uint2 p = {px, py}, d = {dx, dy};
  return get_rng(frame_id, p, d).state;
}

// one LCG step: returns the new state; *f receives lcg_randomf of the old state
uint32_t ref_lcg_step(uint32_t state, float *f) {
  LCGRand r;
  r.state = state;
  *f = lcg_randomf(r);
  r.state = state;
  return lcg_random(r);
}

}  // extern "C"
