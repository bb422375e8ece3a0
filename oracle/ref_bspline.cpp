// Golden-vector harness (test infrastructure): compiled against the reference's own
// src/BSpline.hpp (with the stand-in BasicDataType.h of oracle/ref_stub) by
// oracle/build_ref.py; prints the reference's hat values and hat gradients at known-answer
// points as JSON on stdout. Nothing here is shipped.
#include <cstdint>
#include <cstdio>

#include "BSpline.hpp"

static uint32_t lcg(uint32_t& s) { s = s * 1664525u + 1013904223u; return s >> 8; }
static double unit(uint32_t& s) { return (double)(lcg(s) & 0xFFFFFF) / (double)0x1000000; }

int main() {
  std::printf("{\"hat\": [");
  bool first = true;
  auto emit = [&](double px, double py, double pz, double w, double qx, double qy, double qz) {
    const V3d p(px, py, pz), q(qx, qy, qz);
    const double v = BaseFunction4Point(p, w, q);
    const V3d g = de_BaseFunction4Point(p, w, q);
    std::printf("%s[%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g]", first ? "" : ",", px, py, pz,
                w, qx, qy, qz, v, g.x(), g.y(), g.z());
    first = false;
  };
  // known answers on one axis: the node, the support ends, half-way, just inside and outside
  const double p = 0.375, w = 0.125;
  const double offs[] = {0.0, 1.0, -1.0, 0.5, -0.5, 1.0 - 1e-10, -1.0 + 1e-10, 1.0 - 1e-8, 1.0 + 1e-8, 0.25, -0.75, 2.0};
  for (double a : offs)
    for (double b : offs) emit(p, p, p, w, p + a * w, p + b * w, p + 0.25 * w);
  // lattice points of octree-like widths and arbitrary query points around them
  uint32_t s = 2024u;
  for (int i = 0; i < 600; ++i) {
    const int d = (int)(lcg(s) % 8);
    const double wd = 1.0 / (double)(256 >> d);
    const double cx = (double)(lcg(s) % (256 >> d)) * wd, cy = (double)(lcg(s) % (256 >> d)) * wd,
                 cz = (double)(lcg(s) % (256 >> d)) * wd;
    double qx = cx + (2.4 * unit(s) - 1.2) * wd, qy = cy + (2.4 * unit(s) - 1.2) * wd,
           qz = cz + (2.4 * unit(s) - 1.2) * wd;
    if (i % 5 == 0) qx = cx + (double)((int)(lcg(s) % 5) - 2) * 0.5 * wd;  // on half-lattice planes
    emit(cx, cy, cz, wd, qx, qy, qz);
  }
  std::printf("]}\n");
  return 0;
}
