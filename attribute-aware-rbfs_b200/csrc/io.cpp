// io.cpp -- the reference's particle importer (importParticles.h:8-31) with every read checked,
// and a writer of the same format.
//
// Format: a header text file; each line names a timestep. The binary file `path + "_" + name`
// holds a u64 particle count followed by count float4 (x, y, z, attribute).
#include <cstdio>
#include <fstream>
#include <new>
#include <string>
#include <vector>

#include "../../include/aarbf.h"

struct aarbf_series {
  std::vector<std::vector<float>> frames;  // 4 floats per particle
};

extern "C" {

aarbf_status aarbf_series_load(const char* path, aarbf_series** out) {
  if (!path || !out) return AARBF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::ifstream hdr(path);
  if (!hdr) return AARBF_ERR_IO;
  aarbf_series* s = new (std::nothrow) aarbf_series();
  if (!s) return AARBF_ERR_OUT_OF_MEMORY;
  std::string name;
  while (std::getline(hdr, name)) {
    std::string fn = std::string(path) + "_" + name;
    std::ifstream f(fn, std::ios::binary);
    if (!f) {
      delete s;
      return AARBF_ERR_IO;
    }
    f.seekg(0, std::ios::end);
    std::streamoff size = f.tellg();
    f.seekg(0, std::ios::beg);
    uint64_t count = 0;
    if (size < 8 || !f.read(reinterpret_cast<char*>(&count), sizeof(count))) {
      delete s;
      return AARBF_ERR_IO;
    }
    // the count must match the bytes present (truncated files are rejected)
    if (count > (uint64_t)(size - 8) / 16ull) {
      delete s;
      return AARBF_ERR_IO;
    }
    try {
      s->frames.emplace_back(count * 4);
    } catch (...) {
      delete s;
      return AARBF_ERR_OUT_OF_MEMORY;
    }
    if (count && !f.read(reinterpret_cast<char*>(s->frames.back().data()), (std::streamsize)(count * 16))) {
      delete s;
      return AARBF_ERR_IO;
    }
  }
  *out = s;
  return AARBF_OK;
}

aarbf_status aarbf_series_num_frames(const aarbf_series* s, uint64_t* frames) {
  if (!s || !frames) return AARBF_ERR_INVALID_ARGUMENT;
  *frames = s->frames.size();
  return AARBF_OK;
}

aarbf_status aarbf_series_frame(const aarbf_series* s, uint64_t frame, const float** xyzw, uint64_t* n) {
  if (!s || !xyzw || !n || frame >= s->frames.size()) return AARBF_ERR_INVALID_ARGUMENT;
  *xyzw = s->frames[frame].data();
  *n = s->frames[frame].size() / 4;
  return AARBF_OK;
}

aarbf_status aarbf_series_free(aarbf_series* s) {
  delete s;
  return AARBF_OK;
}

aarbf_status aarbf_series_save(const char* path, const float* const* frames, const uint64_t* counts,
                               uint64_t nframes) {
  if (!path || (nframes && (!frames || !counts))) return AARBF_ERR_INVALID_ARGUMENT;
  std::ofstream hdr(path);
  if (!hdr) return AARBF_ERR_IO;
  for (uint64_t k = 0; k < nframes; ++k) {
    std::string name = std::to_string(k);
    hdr << name << "\n";
    std::ofstream f(std::string(path) + "_" + name, std::ios::binary);
    if (!f) return AARBF_ERR_IO;
    uint64_t c = counts[k];
    f.write(reinterpret_cast<const char*>(&c), sizeof(c));
    if (c) f.write(reinterpret_cast<const char*>(frames[k]), (std::streamsize)(c * 16));
    if (!f) return AARBF_ERR_IO;
  }
  return hdr ? AARBF_OK : AARBF_ERR_IO;
}

}  // extern "C"
