// Marching-cubes device code shared by the marching-cubes entry points (MarchingCubes.cu:164-377
// of the reference): case index with bit i = f(corner i) < iso in the reference's corner order,
// vertex counts from the case table, and the triangle soup written in voxel order by an
// exclusive scan's downsweep.
#pragma once
#include <stdint.h>

namespace its {

__device__ __constant__ uint64_t cMcCase[256] = {
#include "mc_tables.inc"
};
// corner order of MarchingCubes.cu:233-241: 0 (0,0,0) 1 (0,1,0) 2 (1,1,0) 3 (1,0,0), 4..7 at z+1
__device__ __constant__ int8_t cMcCorner[8][3] = {{0, 0, 0}, {0, 1, 0}, {1, 1, 0}, {1, 0, 0},
                                                 {0, 0, 1}, {0, 1, 1}, {1, 1, 1}, {1, 0, 1}};
__device__ __constant__ int8_t cMcEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                               {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

// Per-voxel vertex count (the scan's input): 8 corners of the (R+1)^3 lattice field, x fastest.
// Voxel v = x + R (y + R z) to its coordinates: 32-bit division while R^3 < 2^32 (R <= 1625),
// 64-bit beyond (64-bit division costs several times more and dominated the scan).
__device__ __forceinline__ void voxelXYZ(int64_t v, int R, int64_t& x, int64_t& y, int64_t& z) {
  if ((uint64_t)R * R * R <= 0xFFFFFFFFull) {
    const uint32_t u = (uint32_t)v, r = (uint32_t)R;
    const uint32_t q = u / r;
    x = u - q * r;
    y = q % r;
    z = q / r;
  } else {
    x = v % R;
    y = (v / R) % R;
    z = v / ((int64_t)R * R);
  }
}

template <typename T>
struct McCaseT {
  const T* field;
  int R;
  double iso;
  __device__ unsigned cube(int64_t v) const {
    const int64_t M = (int64_t)R + 1;
    int64_t x, y, z;
    voxelXYZ(v, R, x, y, z);
    unsigned ci = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const double f = (double)field[((z + cMcCorner[k][2]) * M + (y + cMcCorner[k][1])) * M + (x + cMcCorner[k][0])];
      ci |= (unsigned)(f < iso) << k;
    }
    return ci;
  }
  __device__ unsigned long long operator()(int64_t v) const { return cMcCase[cube(v)] & 15ull; }
};
using McCase = McCaseT<double>;

__device__ inline void vertexLerp(const double* p0, const double* p1, double s0, double s1, double iso, double* out) {
  if (fabs(iso - s0) < 1e-6) { out[0] = p0[0]; out[1] = p0[1]; out[2] = p0[2]; return; }
  if (fabs(iso - s1) < 1e-6) { out[0] = p1[0]; out[1] = p1[1]; out[2] = p1[2]; return; }
  if (fabs(s1 - s0) < 1e-6) { out[0] = p0[0]; out[1] = p0[1]; out[2] = p0[2]; return; }
  const double t = (iso - s0) / (s1 - s0);
#pragma unroll
  for (int a = 0; a < 3; ++a) out[a] = fma(t, p1[a], fma(-t, p0[a], p0[a]));  // MCKernel::lerp
}

// The triangle vertices of voxel v (case ci, count vertices) written from offset on.
template <typename T>
__device__ inline void mcEmitVoxel(const McCaseT<T>& mc, double3 o, double3 vs, double* tri, unsigned long long capacity,
                                   int64_t v, unsigned ci, unsigned long long offset, unsigned long long count) {
  const int R = mc.R;
  const int64_t M = (int64_t)R + 1;
  int64_t x, y, z;
  voxelXYZ(v, R, x, y, z);
  const double vp[3] = {(double)x * vs.x + o.x, (double)y * vs.y + o.y, (double)z * vs.z + o.z};
  const double vsz[3] = {vs.x, vs.y, vs.z};
  double corner[8][3], sdf[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    for (int a = 0; a < 3; ++a) corner[k][a] = cMcCorner[k][a] ? vp[a] + vsz[a] : vp[a];
    sdf[k] = (double)mc.field[((z + cMcCorner[k][2]) * M + (y + cMcCorner[k][1])) * M + (x + cMcCorner[k][0])];
  }
  const uint64_t cw = cMcCase[ci];
  for (unsigned i = 0; i < (unsigned)count; ++i) {
    const unsigned long long dst = offset + i;
    if (dst >= capacity) break;
    const int e = (int)((cw >> (4 * (i + 1))) & 15u);
    double q[3];
    vertexLerp(corner[cMcEdge[e][0]], corner[cMcEdge[e][1]], sdf[cMcEdge[e][0]], sdf[cMcEdge[e][1]], mc.iso, q);
    tri[3 * dst] = q[0];
    tri[3 * dst + 1] = q[1];
    tri[3 * dst + 2] = q[2];
  }
}

// The scan's write step: case byte (optional) and the voxel's triangle vertices at its offset.
template <typename T>
struct McEmitT {
  McCaseT<T> mc;
  double3 o, vs;
  uint8_t* cubeOut;
  double* tri;
  unsigned long long capacity;
  __device__ void operator()(int64_t v, unsigned long long offset, unsigned long long count) const {
    const unsigned ci = (cubeOut || count) ? mc.cube(v) : 0u;
    if (cubeOut) cubeOut[v] = (uint8_t)ci;
    if (!count || !tri) return;
    mcEmitVoxel(mc, o, vs, tri, capacity, v, ci, offset, count);
  }
};
using McEmit = McEmitT<double>;

}  // namespace its
