// dataset.cu -- the reference's real-dataset readers, host side.
//
// baseline+filter+beta+shuffle/RealDatasets/BinaryDataset/main.cu:109-148
// reads its keys from a score file in one of two forms, chosen at compile
// time there (#define readBinary) and by a format code here:
//
//   DRTOPK_DATASET_BIN_I32 (main.cu:109-123): n raw little-endian int32
//     values, each kept as its 32-bit pattern (vec[i] = value).  The
//     reference reads with an istream whose target keeps its last value
//     once the stream runs dry, so a short file repeats its last value to n.
//   DRTOPK_DATASET_TXT_REF (main.cu:125-148, the reference's default build):
//     whitespace-separated decimal scores read with fscanf("%f") into the
//     reference's unsigned key slots, so a slot holds the float's bit
//     pattern u, and then vec[i] = (1 - vec[i]) * 1000000000 runs in
//     unsigned 32-bit arithmetic: key = (1 - u) * 10^9 mod 2^32.  At most
//     2^26 scores are read; keys past them repeat the scores in order
//     (vec[i] = vec[i mod 2^26]).  A file with fewer scores than that is
//     tiled by the count it holds (the reference would read uninitialised
//     memory there).
//   DRTOPK_DATASET_TXT_SCORE: the same file and tiling with the map the
//     reference's authors meant, in float arithmetic: key = (1 - s) * 1e9,
//     truncated toward zero and clamped to [0, 2^32 - 1].
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/drtopk.h"

namespace {

constexpr uint64_t kTextTile = 1ull << 26;  // main.cu:134 reads 67108864 scores

drtopk_status_t load_bin_i32(const char* path, uint64_t n, uint32_t* out, uint64_t* n_read) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return DRTOPK_EINVAL;
  uint64_t got = 0;
  const size_t chunk = 1 << 16;
  while (got < n) {
    const size_t want = (size_t)std::min<uint64_t>(chunk, n - got);
    const size_t r = std::fread(out + got, 4, want, f);
    got += r;
    if (r < want) break;
  }
  std::fclose(f);
  if (got == 0) return DRTOPK_EINVAL;
  // keys are the int32 bit patterns; on a little-endian host fread already
  // holds them, elsewhere swap
  const uint16_t probe = 1;
  if (*reinterpret_cast<const uint8_t*>(&probe) != 1)
    for (uint64_t i = 0; i < got; ++i) {
      const uint32_t v = out[i];
      out[i] = (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24);
    }
  for (uint64_t i = got; i < n; ++i) out[i] = out[got - 1];
  if (n_read) *n_read = got;
  return DRTOPK_OK;
}

drtopk_status_t load_text(const char* path, uint64_t n, bool ref_arith, uint32_t* out, uint64_t* n_read) {
  FILE* f = std::fopen(path, "r");
  if (!f) return DRTOPK_EINVAL;
  const uint64_t lim = std::min<uint64_t>(n, kTextTile);
  uint64_t got = 0;
  float s = 0.0f;
  while (got < lim && std::fscanf(f, "%f", &s) == 1) {
    if (ref_arith) {
      uint32_t u;
      std::memcpy(&u, &s, 4);
      out[got] = (uint32_t)((1u - u) * 1000000000u);
    } else {
      const float v = (1.0f - s) * 1000000000.0f;
      double d = std::trunc((double)v);
      if (!(d >= 0.0)) d = 0.0;  // negative scores above 1, and NaN
      if (d > 4294967295.0) d = 4294967295.0;
      out[got] = (uint32_t)d;
    }
    ++got;
  }
  std::fclose(f);
  if (got == 0) return DRTOPK_EINVAL;
  for (uint64_t i = got; i < n; ++i) out[i] = out[i % got];
  if (n_read) *n_read = got;
  return DRTOPK_OK;
}

}  // namespace

extern "C" drtopk_status_t drtopk_load_dataset(const char* path, int format, uint64_t n, uint32_t* h_keys,
                                               uint64_t* n_read) {
  if (!path || !h_keys || n == 0) return DRTOPK_EINVAL;
  if (n_read) *n_read = 0;
  switch (format) {
    case DRTOPK_DATASET_BIN_I32: return load_bin_i32(path, n, h_keys, n_read);
    case DRTOPK_DATASET_TXT_REF: return load_text(path, n, true, h_keys, n_read);
    case DRTOPK_DATASET_TXT_SCORE: return load_text(path, n, false, h_keys, n_read);
    default: return DRTOPK_EINVAL;
  }
}
