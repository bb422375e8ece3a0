// Golden-vector harness (test infrastructure): compiled against the reference's own
// MortonLUT.h (encode/decode tables) and MarchingCubes/LookTable.h (case tables) by
// oracle/build_ref.py, writing JSON to stdout. Nothing here is shipped.
#define __constant__
#define _CUDA_GENERAL_CALL_
#include <cstdio>
#include <cstdint>
#include "MortonLUT.h"
#include "LookTable.h"

static uint32_t lcg(uint32_t& s) { s = s * 1664525u + 1013904223u; return s >> 8; }

int main() {
  std::printf("{\n\"encode\": [");
  bool first = true;
  // Every (x,y,z) in [0,16)^3, then 4000 pseudo-random triples in [0,1024)^3.
  auto emit = [&](unsigned x, unsigned y, unsigned z) {
    uint32_t m = morton::mortonEncode_LUT((uint16_t)x, (uint16_t)y, (uint16_t)z);
    uint16_t dx, dy, dz;
    morton::morton3D_32_decode(m, dx, dy, dz);
    std::printf("%s[%u,%u,%u,%u,%u,%u,%u]", first ? "" : ",", x, y, z, m, dx, dy, dz);
    first = false;
  };
  for (unsigned z = 0; z < 16; ++z)
    for (unsigned y = 0; y < 16; ++y)
      for (unsigned x = 0; x < 16; ++x) emit(x, y, z);
  uint32_t s = 12345u;
  for (int i = 0; i < 4000; ++i) {
    unsigned x = lcg(s) % 1024, y = lcg(s) % 1024, z = lcg(s) % 1024;
    emit(x, y, z);
  }
  std::printf("],\n\"triTable\": [");
  for (int c = 0; c < 256; ++c) {
    std::printf("%s[", c ? "," : "");
    for (int k = 0; k < 16; ++k) std::printf("%s%d", k ? "," : "", MC::triTable[c][k]);
    std::printf("]");
  }
  std::printf("],\n\"nVertsTable\": [");
  for (int c = 0; c < 256; ++c) std::printf("%s%d", c ? "," : "", MC::nVertsTable[c]);
  std::printf("],\n\"edgeTable\": [");
  for (int c = 0; c < 256; ++c) std::printf("%s%d", c ? "," : "", MC::edgeTable[c]);
  std::printf("]\n}\n");
  return 0;
}
