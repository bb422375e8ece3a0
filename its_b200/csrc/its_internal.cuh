// Internal definitions shared by the sm_100a kernels of libits.
//
// Arithmetic conventions (the oracle follows the same ones, so that integer topology
// and the assembled operator are bit-exact between the two): the library is compiled
// with -fmad=false; three-term dot products sum left to right; lattice positions are
// g + w*X (one multiply, one add); explicit fma() appears only where the reference
// writes it (marching-cubes lerp, MarchingCubes.h:18).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "its/its.h"

namespace its {

constexpr uint32_t kNone = 0xFFFFFFFFu;  // "no node" (UINT_MAX in SVO.h:25-27)
constexpr int kMaxDepth = 12;            // res <= 1024 gives at most 11 levels

// ---- Morton codes: x at bit 3i, y at 3i+1, z at 3i+2 (MortonLUT.h:292-343) ---------
__host__ __device__ inline uint32_t spread3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__host__ __device__ inline uint32_t compact3(uint32_t v) {
  v &= 0x09249249u;
  v = (v | (v >> 2)) & 0x030C30C3u;
  v = (v | (v >> 4)) & 0x0300F00Fu;
  v = (v | (v >> 8)) & 0x030000FFu;
  v = (v | (v >> 16)) & 0x000003FFu;
  return v;
}
__host__ __device__ inline uint32_t mortonEncode(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}
__host__ __device__ inline void mortonDecode(uint32_t m, uint32_t& x, uint32_t& y, uint32_t& z) {
  x = compact3(m);
  y = compact3(m >> 1);
  z = compact3(m >> 2);
}

// Scalar helpers with the reference's semantics: fminf/fmaxf double overloads
// (CUDAMath.hpp:131-139) and clamp(int) (CUDAMath.hpp:193-196).
__host__ __device__ inline double dmin(double a, double b) { return a < b ? a : b; }
__host__ __device__ inline double dmax(double a, double b) { return a > b ? a : b; }
__host__ __device__ inline double fmax0(double b) { return 0.0 > b ? 0.0 : b; }
__host__ __device__ inline int clampi(int f, int a, int b) { return f < a ? a : (f > b ? b : f); }

// ---- degree-1 hat basis (BSpline.hpp:4-22) -----------------------------------------
__host__ __device__ inline double hat1(double x, double p, double w) {
  if (fabs(x - (p - w)) < 1e-9 || x < p - w || fabs(x - (p + w)) < 1e-9 || x > p + w) return 0.0;
  if (x <= p) return 1 + (x - p) / w;
  return 1 - (x - p) / w;
}
// Correctly rounded quotient a / b from y = RN(1 / b) (Markstein's theorem: with y the
// correctly rounded reciprocal and q = RN(a y) within one ulp of a / b, the exact remainder
// r = a - q b (one FMA) gives RN(a / b) = RN(q + r y)). Valid without overflow or underflow,
// which the octree's coordinates (|a|, |b| in [1e-300, 1e300]) never approach. Bit-identical
// to a / b; a multiply and two FMAs instead of a division.
__device__ __forceinline__ double divRn(double a, double b, double y) {
  const double q = a * y;
  const double r = fma(-q, b, a);
  return fma(r, y, q);
}
// hat1 with the quotient formed by divRn (same result bit for bit).
__device__ __forceinline__ double hat1r(double x, double p, double w, double winv) {
  if (fabs(x - (p - w)) < 1e-9 || x < p - w || fabs(x - (p + w)) < 1e-9 || x > p + w) return 0.0;
  if (x <= p) return 1 + divRn(x - p, w, winv);
  return 1 - divRn(x - p, w, winv);
}
// hat3 with the quotients formed by divRn (same result bit for bit).
__device__ __forceinline__ double hat3r(double px, double py, double pz, double w, double winv, double qx, double qy,
                                        double qz) {
  const double x = hat1r(qx, px, w, winv);
  if (x <= 0.0) return 0.0;
  const double y = hat1r(qy, py, w, winv);
  if (y <= 0.0) return 0.0;
  const double z = hat1r(qz, pz, w, winv);
  if (z <= 0.0) return 0.0;
  return x * y * z;
}
__host__ __device__ inline double hat3(double px, double py, double pz, double w, double qx, double qy,
                                       double qz) {
  const double x = hat1(qx, px, w);
  if (x <= 0.0) return 0.0;
  const double y = hat1(qy, py, w);
  if (y <= 0.0) return 0.0;
  const double z = hat1(qz, pz, w);
  if (z <= 0.0) return 0.0;
  return x * y * z;
}

// ---- per-depth corner-vertex index: bitmap over the (res_d+1)^3 lattice + rank -------
// Lattice point (X,Y,Z) at depth d has linear index (X*M + Y)*M + Z, M = (res>>d)+1, which
// is the reference's lexicographic (x, y, z) vertex order (SVO.cu:1012-1096).
struct LatticeIndex {
  const unsigned long long* bits;  // M^3 bits
  const uint32_t* rank;            // exclusive popcount prefix per 64-bit word
  uint32_t M;
  uint32_t base;                   // global index of the depth's first vertex
};
__device__ __forceinline__ bool latticeHas(const LatticeIndex& L, uint32_t lin) {
  return (L.bits[lin >> 6] >> (lin & 63)) & 1ull;
}
__device__ __forceinline__ uint32_t latticeRank(const LatticeIndex& L, uint32_t lin) {
  const unsigned long long w = L.bits[lin >> 6];
  const unsigned long long below = w & ((1ull << (lin & 63)) - 1ull);
  return L.base + L.rank[lin >> 6] + (uint32_t)__popcll(below);
}

// ---- packed vertex key: X | Y << 11 | Z << 22 | depth << 33 | owner corner bits 37-39 ----
struct VertCoord {
  uint32_t X, Y, Z;     // lattice coordinates at the vertex's depth
  int d;                // depth
  uint32_t Xo, Yo, Zo;  // the owner node's coordinates (the vertex is its corner X-Xo, Y-Yo, Z-Zo)
};
__host__ __device__ inline VertCoord decodeVertKey(uint64_t k) {
  VertCoord c;
  c.X = (uint32_t)k & 2047u;
  c.Y = (uint32_t)(k >> 11) & 2047u;
  c.Z = (uint32_t)(k >> 22) & 2047u;
  c.d = (int)((k >> 33) & 15u);
  c.Xo = c.X - ((uint32_t)(k >> 37) & 1u);
  c.Yo = c.Y - ((uint32_t)(k >> 38) & 1u);
  c.Zo = c.Z - ((uint32_t)(k >> 39) & 1u);
  return c;
}
__host__ __device__ inline uint64_t encodeVertKey(uint32_t X, uint32_t Y, uint32_t Z, int d, uint32_t Xo, uint32_t Yo,
                                                  uint32_t Zo) {
  return (uint64_t)X | ((uint64_t)Y << 11) | ((uint64_t)Z << 22) | ((uint64_t)d << 33) | ((uint64_t)(X - Xo) << 37) |
         ((uint64_t)(Y - Yo) << 38) | ((uint64_t)(Z - Zo) << 39);
}

// ---- octree on the device (structure of arrays; finest depth first, root last) ------
struct SvoDevice {
  int res = 0, depth = 0;
  double origin[3] = {0, 0, 0};
  double unit[3] = {0, 0, 0};  // unitVoxelSize per axis; node widths use unit[0]
  int64_t numVoxels = 0, numNodes = 0, numVerts = 0, numEdges = 0;
  int64_t levelCount[kMaxDepth] = {0}, levelStart[kMaxDepth + 1] = {0};
  int64_t vertCount[kMaxDepth] = {0}, vertStart[kMaxDepth + 1] = {0};
  uint32_t* voxels = nullptr;      // surface voxels, ascending Morton
  uint32_t* nodeMorton = nullptr;
  uint32_t* nodeParent = nullptr;
  uint32_t* nodeChild0 = nullptr;  // first of 8 consecutive children, kNone for leaves
  uint8_t* nodeLeaf = nullptr;
  uint32_t* nodeNb = nullptr;      // 27 per node, slot (dx+1)+3(dy+1)+9(dz+1)
  unsigned long long* vbits[kMaxDepth] = {nullptr};
  uint32_t* vrank[kMaxDepth] = {nullptr};
  uint32_t* vertLin = nullptr;     // lattice index within its depth
  uint64_t* vertKey = nullptr;     // lattice coordinates, depth and the vertex's corner of its owner:
                                   // X | Y << 11 | Z << 22 | depth << 33 | (X - Xo) << 37 | (Y - Yo) << 38 | (Z - Zo) << 39
  uint32_t* vertOwner = nullptr;   // lowest-index node having the corner
  double* vertPos = nullptr;       // 3 per vertex
  unsigned long long* ebits = nullptr;  // fine edges: bit (lin*3 + {z:0,y:1,x:2})
  uint32_t* erank = nullptr;
  uint32_t* edgeKey = nullptr;
  uint32_t* edgeOwner = nullptr;
  uint64_t* fineOcc = nullptr;     // res^3-bit Morton bitset of depth-0 nodes
  uint32_t* fineRank = nullptr;    // exclusive popcount prefix per word of fineOcc: node index by rank
  // face samples (centroids, unit normals) summed per node, finest depth first
  float* nodeSampleCnt = nullptr;  // per node
  double* nodeSamplePos = nullptr; // 3 per node: sum of centroids
  double* nodeSampleNrm = nullptr; // 3 per node: sum of unit normals
  int64_t* coincIds = nullptr;     // vertices coincident with a coarser corner, ascending
  int64_t numCoinc = 0;
  float* coincGeom = nullptr;      // share-network features 38-45 of each coincident vertex (the
                                   // face samples around its owner: octree and mesh only)
  void* rowParams = nullptr;       // device copy of the octree's RowParams (its_rows.cuh)
  float buildMs = 0.0f;            // device time of the whole build
  float learnedTablesMs = 0.0f;    // of which the learned fit's octree-only tables
  LatticeIndex lattice(int d) const {
    LatticeIndex L;
    L.bits = vbits[d];
    L.rank = vrank[d];
    L.M = (uint32_t)(res >> d) + 1u;
    L.base = (uint32_t)vertStart[d];
    return L;
  }
};

// Index of the depth-0 node with Morton code m (depth-0 nodes are stored in Morton order), or
// kNone: a bit test and a rank in the fine-node bitset instead of a binary search.
__device__ __forceinline__ uint32_t fineNodeOf(const unsigned long long* occ, const uint32_t* rank, uint32_t m) {
  const unsigned long long w = occ[m >> 6];
  if (!((w >> (m & 63)) & 1ull)) return kNone;
  return rank[m >> 6] + (uint32_t)__popcll(w & ((1ull << (m & 63)) - 1ull));
}

// Lattice position g + w*X per axis (createNode_1/2, SVO.cu:573-576).
__host__ __device__ inline double latticePos(double g, double w, uint32_t X) { return g + w * (double)X; }

// ---- small device utilities -----------------------------------------------------------
__device__ __forceinline__ double warpSum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Error plumbing shared by the C-ABI translation units.
struct Error {
  its_status code;
  std::string msg;
};
its_status setError(its_ctx* ctx, its_status code, const std::string& msg);
its_status cudaFail(its_ctx* ctx, cudaError_t e, const char* what);

}  // namespace its

#define ITS_CU(ctx, call)                                   \
  do {                                                      \
    cudaError_t e__ = (call);                               \
    if (e__ != cudaSuccess) return ::its::cudaFail((ctx), e__, #call); \
  } while (0)
