// Welded marching-cubes mesh (the "next" step after the reference's triangle soup,
// MarchingCubes.cu:635-661 writes three fresh vertices per triangle).
//
// Every MC vertex lies on one edge of the (R+1)^3 lattice. An edge (lower lattice point i,
// axis a) is active when its two field values fall on different sides of iso (f < iso test of
// MarchingCubes.cu:184-187). Active edges are marked in a bitmap over the 3 (R+1)^3 edge ids
// id = 3 * lin(i) + a and ranked by popcount, which numbers the welded vertices in edge-id
// order; triangles are the case table's edge lists mapped to those ranks. A welded vertex
// is the reference's lerp from the lower to the upper lattice point (explicit fma as in
// MarchingCubes.h:18), both end points at origin + index * voxel size.
#include "its_mc.cuh"
#include "its_scan.cuh"

namespace its {

struct MeshGrid {
  const double* field;
  int R;
  double iso;
  double3 o, vs;
  __device__ int64_t M() const { return (int64_t)R + 1; }
  __device__ double f(int64_t x, int64_t y, int64_t z) const { return field[(z * M() + y) * M() + x]; }
};

__global__ void kMarkActiveEdges(MeshGrid G, unsigned long long* __restrict__ bits) {
  const int64_t M = G.M(), total = 3 * M * M * M;
  for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < total; id += (int64_t)gridDim.x * blockDim.x) {
    const int64_t lin = id / 3;
    const int a = (int)(id % 3);
    const int64_t x = lin % M, y = (lin / M) % M, z = lin / (M * M);
    const int64_t x1 = x + (a == 0), y1 = y + (a == 1), z1 = z + (a == 2);
    if (x1 >= M || y1 >= M || z1 >= M) continue;
    if ((G.f(x, y, z) < G.iso) != (G.f(x1, y1, z1) < G.iso)) atomicOr(bits + (id >> 6), 1ull << (id & 63));
  }
}

__global__ void kWeldedVertices(MeshGrid G, const unsigned long long* __restrict__ bits,
                                const unsigned long long* __restrict__ rank, int64_t words, double* __restrict__ verts) {
  const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (w >= words) return;
  unsigned long long b = bits[w];
  unsigned long long r = rank[w];
  const int64_t M = G.M();
  while (b) {
    const int k = __ffsll((long long)b) - 1;
    b &= b - 1;
    const int64_t id = w * 64 + k;
    const int64_t lin = id / 3;
    const int a = (int)(id % 3);
    const int64_t x = lin % M, y = (lin / M) % M, z = lin / (M * M);
    const int64_t x1 = x + (a == 0), y1 = y + (a == 1), z1 = z + (a == 2);
    const double p0[3] = {G.o.x + (double)x * G.vs.x, G.o.y + (double)y * G.vs.y, G.o.z + (double)z * G.vs.z};
    const double p1[3] = {G.o.x + (double)x1 * G.vs.x, G.o.y + (double)y1 * G.vs.y, G.o.z + (double)z1 * G.vs.z};
    vertexLerp(p0, p1, G.f(x, y, z), G.f(x1, y1, z1), G.iso, verts + 3 * r);
    ++r;
  }
}

struct MeshTris {
  McCase mc;
  const unsigned long long* bits;
  const unsigned long long* rank;
  int32_t* tris;
  unsigned long long capacity;  // triangles
  __device__ unsigned long long operator()(int64_t v) const { return (cMcCase[mc.cube(v)] & 15ull) / 3; }
  __device__ void operator()(int64_t v, unsigned long long offset, unsigned long long count) const {
    if (!count || !tris) return;
    const int R = mc.R;
    const int64_t M = (int64_t)R + 1;
    int64_t x, y, z;
    voxelXYZ(v, R, x, y, z);
    const uint64_t cw = cMcCase[mc.cube(v)];
    for (unsigned t = 0; t < (unsigned)count; ++t) {
      if (offset + t >= capacity) break;
      for (int j = 0; j < 3; ++j) {
        const int e = (int)((cw >> (4 * (3 * t + j + 1))) & 15u);
        const int ca = cMcEdge[e][0], cb = cMcEdge[e][1];
        const int64_t ax = x + cMcCorner[ca][0], ay = y + cMcCorner[ca][1], az = z + cMcCorner[ca][2];
        const int64_t bx = x + cMcCorner[cb][0], by = y + cMcCorner[cb][1], bz = z + cMcCorner[cb][2];
        const int64_t lx = ax < bx ? ax : bx, ly = ay < by ? ay : by, lz = az < bz ? az : bz;
        const int axis = ax != bx ? 0 : (ay != by ? 1 : 2);
        const unsigned long long id = (unsigned long long)(((lz * M + ly) * M + lx) * 3 + axis);
        const unsigned long long word = bits[id >> 6];
        tris[3 * (offset + t) + j] =
            (int32_t)(rank[id >> 6] + (unsigned long long)__popcll(word & ((1ull << (id & 63)) - 1ull)));
      }
    }
  }
};
// scan input / write adapters over the two-role functor above
struct MeshTrisCount {
  MeshTris m;
  __device__ unsigned long long operator()(int64_t v) const { return m(v); }
};
struct MeshTrisWrite {
  MeshTris m;
  __device__ void operator()(int64_t v, unsigned long long offset, unsigned long long count) const { m(v, offset, count); }
};

}  // namespace its

using namespace its;

extern "C" {

its_status its_marching_cubes_mesh(its_ctx* ctx, const double* field, int res, const double origin[3],
                                   const double width[3], double iso, double* verts, int64_t vert_capacity,
                                   int64_t* num_verts, int32_t* tris, int64_t tri_capacity, int64_t* num_tris) {
  if (!ctx) return ITS_ERR_INVALID;
  if (!field || !origin || !width || !num_verts || !num_tris || res < 1 || res > 1024 || vert_capacity < 0 ||
      tri_capacity < 0)
    return setError(ctx, ITS_ERR_INVALID, "its_marching_cubes_mesh: bad arguments");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  const int64_t M = (int64_t)res + 1, nvox = (int64_t)res * res * res;
  const int64_t edges = 3 * M * M * M, words = (edges + 63) / 64;
  InArg<double> F;
  its_status st;
  if ((st = F.stage(ctx, field, M * M * M)) != ITS_OK) return st;
  DevBuf<unsigned long long> bits, rank, tot;
  if ((st = bits.zeros(ctx, words)) != ITS_OK || (st = rank.alloc(ctx, words)) != ITS_OK ||
      (st = tot.alloc(ctx, 2)) != ITS_OK)
    return st;
  MeshGrid G{F.d, res, iso, make_double3(origin[0], origin[1], origin[2]),
             make_double3(width[0] / res, width[1] / res, width[2] / res)};
  const unsigned blocks = (unsigned)std::min<int64_t>(gridFor(edges, 256), (int64_t)ctx->numSMs * 32);
  kMarkActiveEdges<<<blocks, 256, 0, ctx->stream>>>(G, bits.p);
  ITS_LAUNCHED(ctx);
  const unsigned long long* bp = bits.p;
  auto pc = [bp] __device__(int64_t i) -> unsigned long long { return (unsigned long long)__popcll(bp[i]); };
  if ((st = scanExclusiveAlloc<unsigned long long>(ctx, pc, words, StorePrefix<unsigned long long>{rank.p}, tot.p)) != ITS_OK)
    return st;
  MeshTris mt{McCase{F.d, res, iso}, bits.p, rank.p, nullptr, 0};
  auto nowrite = [] __device__(int64_t, unsigned long long, unsigned long long) {};
  if ((st = scanExclusiveAlloc<unsigned long long>(ctx, MeshTrisCount{mt}, nvox, nowrite, tot.p + 1)) != ITS_OK) return st;
  unsigned long long h[2];
  ITS_CU(ctx, cudaMemcpyAsync(h, tot.p, 16, cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  *num_verts = (int64_t)h[0];
  *num_tris = (int64_t)h[1];
  if (verts && vert_capacity >= (int64_t)h[0] && h[0]) {
    OutArg<double> Vo;
    if ((st = Vo.stage(ctx, verts, 3 * h[0])) != ITS_OK) return st;
    kWeldedVertices<<<gridFor(words, 256), 256, 0, ctx->stream>>>(G, bits.p, rank.p, words, Vo.d);
    ITS_LAUNCHED(ctx);
    if ((st = Vo.finish(ctx)) != ITS_OK) return st;
  } else if (verts && h[0]) {
    return setError(ctx, ITS_ERR_INVALID, "its_marching_cubes_mesh: vertex capacity too small");
  }
  if (tris && tri_capacity >= (int64_t)h[1] && h[1]) {
    OutArg<int32_t> To;
    if ((st = To.stage(ctx, tris, 3 * h[1])) != ITS_OK) return st;
    mt.tris = To.d;
    mt.capacity = h[1];
    if ((st = scanExclusiveAlloc<unsigned long long>(ctx, MeshTrisCount{mt}, nvox, MeshTrisWrite{mt}, tot.p + 1)) != ITS_OK)
      return st;
    if ((st = To.finish(ctx)) != ITS_OK) return st;
  } else if (tris && h[1]) {
    return setError(ctx, ITS_ERR_INVALID, "its_marching_cubes_mesh: triangle capacity too small");
  }
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // extern "C"
