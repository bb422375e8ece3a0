// CPU oracle for the ITS thin-shell path -- TEST INFRASTRUCTURE ONLY.
//
// This library restates, on the CPU, the reference algorithm of Alan-Leo-Wong/ITS
// ("3DThinShell") for the hot path: unit-cube normalisation, cubic bounding box,
// triangle attributes, conservative surface voxelisation, the Morton-coded sparse
// voxel octree (levels, 27-neighbours, per-depth corner vertices, fine-node edges),
// shell-sample intersections, signed distance RHS, hierarchical hat-basis assembly,
// Eigen-style LSCG (CGLS with column-norm Jacobi scaling), field evaluation and
// GPU marching-cubes semantics. Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load it, and only as the checker or the timed CPU baseline.
//
// Arithmetic conventions (shared with the CUDA product so that both are bit-exact):
//   * no FMA contraction (built with -ffp-contract=off), except where the reference
//     itself writes fma() (the MC vertex lerp, MarchingCubes.h:18);
//   * three-term dot products and squared norms are summed left to right,
//     (a0*b0 + a1*b1) + a2*b2;
//   * positions derived from the lattice: origin = g + w*X (one multiply, one add).
// Parity pinning: Morton encode/decode, the neighbour/sharing LUTs and the MC case
// tables are checked against the reference's own headers (tests/golden). The remaining
// stages have no reference test, golden file or runnable binary (Eigen and libigl are
// absent), so their parity is unpinned beyond this restatement.
#pragma once
#include <cstdint>
#include <cmath>
#include <vector>
#include <limits>

namespace orc {

constexpr uint32_t kMortonFlag = 0x80000000u;  // E_MORTON_32_FLAG, MortonLUT.h:7
constexpr uint32_t kMortonMask = 0x7FFFFFFFu;  // D_MORTON_32_FLAG, MortonLUT.h:8
constexpr uint32_t kNone = 0xFFFFFFFFu;        // UINT_MAX "no node", SVO.h:25-27
constexpr double kDInf = std::numeric_limits<double>::max();  // DINF, BasicDataType.h:15

struct V3 {
  double x, y, z;
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot3(V3 a, V3 b) {
  double s = a.x * b.x;
  s = s + a.y * b.y;
  return s + a.z * b.z;
}
inline V3 cross3(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// fminf/fmaxf double overloads of the reference (CUDAMath.hpp:131-139).
inline double dmin(double a, double b) { return a < b ? a : b; }
inline double dmax(double a, double b) { return a > b ? a : b; }
inline V3 vmin(V3 a, V3 b) { return {dmin(a.x, b.x), dmin(a.y, b.y), dmin(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {dmax(a.x, b.x), dmax(a.y, b.y), dmax(a.z, b.z)}; }
inline int clampi(int f, int a, int b) { return f < a ? a : (f > b ? b : f); }

// Tolerant lexicographic compare of std::less<V3d> (BasicDataType.h:44-56) and
// lessPoint (SVO.cu:1012-1023): coordinates within 1e-9 count as equal.
inline int lessPoint(const V3& a, const V3& b) {
  for (int i = 0; i < 3; ++i) {
    if (std::fabs(a[i] - b[i]) < 1e-9) continue;
    if (a[i] < b[i]) return 1;
    if (a[i] > b[i]) return -1;
  }
  return 0;
}
// Eigen isApprox: ||a-b||^2 <= prec^2 * min(||a||^2, ||b||^2).
inline bool isApprox(const V3& a, const V3& b, double prec) {
  V3 d = a - b;
  double na = dot3(a, a), nb = dot3(b, b);
  return dot3(d, d) <= prec * prec * (na < nb ? na : nb);
}

// ---- Morton codes (MortonLUT.h:292-343) --------------------------------------
// The reference encodes through 8-bit -> 24-bit spread tables (x at bit 3i, y at
// 3i+1, z at 3i+2) and decodes through 9-bit tables. We spread bits arithmetically;
// tests/golden pins both directions against the reference's own tables.
inline uint32_t spread3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
inline uint32_t compact3(uint32_t v) {
  v &= 0x09249249u;
  v = (v | (v >> 2)) & 0x030C30C3u;
  v = (v | (v >> 4)) & 0x0300F00Fu;
  v = (v | (v >> 8)) & 0x030000FFu;
  v = (v | (v >> 16)) & 0x000003FFu;
  return v;
}
inline uint32_t mortonEncode(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}
inline void mortonDecode(uint32_t m, uint32_t& x, uint32_t& y, uint32_t& z) {
  x = compact3(m);
  y = compact3(m >> 1);
  z = compact3(m >> 2);
}

// Neighbour slot of offset (dx,dy,dz) in {-1,0,1}^3: s = (dx+1) + 3(dy+1) + 9(dz+1);
// slot 13 is the node itself (SVO.cu:242-304 tables use this order).
inline int nbSlot(int dx, int dy, int dz) { return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1); }

// neighbor_LUTparent / neighbor_LUTchild (SVO.cu:242-304), derived: child key
// k = kx | ky<<1 | kz<<2; neighbour at offset d lies in the parent's neighbour
// floor((k+d)/2) as that parent's child ((k+d) mod 2).
inline void neighborLUTs(short parentLUT[8][27], short childLUT[8][27]) {
  for (int k = 0; k < 8; ++k) {
    int kb[3] = {k & 1, (k >> 1) & 1, (k >> 2) & 1};
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int d[3] = {dx, dy, dz}, P[3], C[3];
          for (int a = 0; a < 3; ++a) {
            int t = kb[a] + d[a];           // in {-1,0,1,2}
            P[a] = (t < 0) ? -1 : (t > 1 ? 1 : 0);
            C[a] = t & 1;
          }
          int s = nbSlot(dx, dy, dz);
          parentLUT[k][s] = (short)nbSlot(P[0], P[1], P[2]);
          childLUT[k][s] = (short)(C[0] | (C[1] << 1) | (C[2] << 2));
        }
  }
}
// d_vertSharedLUT (SVO.cu:330-347): the 8 cells sharing corner k, ascending slots.
inline void vertSharedLUT(short lut[64]) {
  for (int k = 0; k < 8; ++k) {
    int c[3] = {k & 1, (k >> 1) & 1, (k >> 2) & 1};
    int j = 0;
    for (int dz = c[2] - 1; dz <= c[2]; ++dz)
      for (int dy = c[1] - 1; dy <= c[1]; ++dy)
        for (int dx = c[0] - 1; dx <= c[0]; ++dx) lut[k * 8 + j++] = (short)nbSlot(dx, dy, dz);
  }
}
// Fine-node edge list of determineNodeEdge (SVO.cu:974-990), corner pairs
// "02 23 31 10 46 67 75 54 04 26 37 15" written lower corner first.
constexpr int kEdgeCorners[12][2] = {{0, 2}, {2, 3}, {1, 3}, {0, 1}, {4, 6}, {6, 7},
                                     {5, 7}, {4, 5}, {0, 4}, {2, 6}, {3, 7}, {1, 5}};
// d_edgeSharedLUT (SVO.cu:312-327): the 4 cells sharing edge i, ascending slots.
inline void edgeSharedLUT(short lut[48]) {
  for (int e = 0; e < 12; ++e) {
    int a = kEdgeCorners[e][0], b = kEdgeCorners[e][1];
    int ca[3] = {a & 1, (a >> 1) & 1, (a >> 2) & 1}, cb[3] = {b & 1, (b >> 1) & 1, (b >> 2) & 1};
    int lo[3], hi[3];
    for (int t = 0; t < 3; ++t) {
      if (ca[t] == cb[t]) { lo[t] = ca[t] - 1; hi[t] = ca[t]; }  // shared across this axis
      else { lo[t] = 0; hi[t] = 0; }                             // along the edge
    }
    int j = 0;
    for (int dz = lo[2]; dz <= hi[2]; ++dz)
      for (int dy = lo[1]; dy <= hi[1]; ++dy)
        for (int dx = lo[0]; dx <= hi[0]; ++dx) lut[e * 4 + j++] = (short)nbSlot(dx, dy, dz);
  }
}

// ---- degree-1 hat basis (BSpline.hpp:4-22) ------------------------------------
inline double baseFunction(double x, double p, double w) {
  if (std::fabs(x - (p - w)) < 1e-9 || x < p - w || std::fabs(x - (p + w)) < 1e-9 || x > p + w)
    return 0.0;
  if (x <= p) return 1 + (x - p) / w;
  return 1 - (x - p) / w;
}
// de_BaseFunction (BSpline.hpp:30-35): 1/w left of the node, -1/w right of it, 0 outside.
inline double deBaseFunction(double x, double p, double w) {
  if (std::fabs(x - (p - w)) < 1e-9 || x < p - w || std::fabs(x - (p + w)) < 1e-9 || x > p + w) return 0.0;
  if (x <= p) return 1 / w;
  return -1 / w;
}
inline double baseFunction4Point(const V3& p, double w, const V3& q) {
  double x = baseFunction(q.x, p.x, w);
  if (x <= 0.0) return 0.0;
  double y = baseFunction(q.y, p.y, w);
  if (y <= 0.0) return 0.0;
  double z = baseFunction(q.z, p.z, w);
  if (z <= 0.0) return 0.0;
  return x * y * z;
}

}  // namespace orc
