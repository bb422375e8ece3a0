// Sparse voxel octree on the GPU (replaces SparseVoxelOctree::createOctree and
// constructNodeAtrributes, SVO.cu:366-1110 of the reference).
//
// Layout (structure of arrays, depth 0 = voxels first, root last; same node order as the
// reference's svoNodeArray):
//   * occupancy of the res^3 voxel grid is a Morton-indexed bitset (res^3/8 bytes) instead
//     of a dense uint32 array; surface voxels are compacted from it in Morton order;
//   * each level's occupied codes O_L are sorted, so the next level is unique(O_L >> 3):
//     no dense per-level arrays and no sort;
//   * nodes: morton / parent / first-child / leaf flag / 27 neighbours;
//   * per-depth corner vertices are a bitmap over the (res_d+1)^3 corner lattice with a
//     popcount rank per 64-bit word, which gives the reference's sorted (x,y,z) vertex order
//     and an O(1) corner -> column lookup without hashing or tolerant compares;
//   * fine-node edges are a bitmap over (lattice point, axis) with the same rank.
#include <algorithm>
#include <cmath>
#include <vector>

#include "its_scan.cuh"
#include "its_rows.cuh"
#include "its_svo.cuh"

namespace its {

// ---- voxelisation: surfaceVoxelize (SVO.cu:366-493), one thread per triangle -------------
struct E2 { double a, b, d; };
__device__ inline E2 edgeTest(double a, double b, bool flip, double pa, double pb, double ua, double ub) {
  if (flip) { a = -a; b = -b; }
  double d = (-1.0 * (a * pa + b * pb)) + fmax0(ua * a);
  d = d + fmax0(ub * b);
  return E2{a, b, d};
}

__global__ void kVoxelize(const double* __restrict__ V, const int32_t* __restrict__ F, int64_t nf, int res,
                          double3 g, double3 u, unsigned long long* __restrict__ occ) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nf; t += (int64_t)gridDim.x * blockDim.x) {
    const int32_t i0 = F[3 * t], i1 = F[3 * t + 1], i2 = F[3 * t + 2];
    const double v0x = V[3 * i0] - g.x, v0y = V[3 * i0 + 1] - g.y, v0z = V[3 * i0 + 2] - g.z;
    const double v1x = V[3 * i1] - g.x, v1y = V[3 * i1 + 1] - g.y, v1z = V[3 * i1 + 2] - g.z;
    const double v2x = V[3 * i2] - g.x, v2y = V[3 * i2 + 1] - g.y, v2z = V[3 * i2 + 2] - g.z;
    const double e0x = v1x - v0x, e0y = v1y - v0y, e0z = v1z - v0z;
    const double e1x = v2x - v1x, e1y = v2y - v1y, e1z = v2z - v1z;
    const double e2x = v0x - v2x, e2y = v0y - v2y, e2z = v0z - v2z;
    double nx = e0y * e1z - e0z * e1y, ny = e0z * e1x - e0x * e1z, nz = e0x * e1y - e0y * e1x;
    {
      double z = nx * nx;
      z = z + ny * ny;
      z = z + nz * nz;
      if (z > 0.0) {
        const double s = sqrt(z);
        nx = nx / s; ny = ny / s; nz = nz / s;
      }
    }
    const double bminx = dmin(v0x, dmin(v1x, v2x)), bminy = dmin(v0y, dmin(v1y, v2y)), bminz = dmin(v0z, dmin(v1z, v2z));
    const double bmaxx = dmax(v0x, dmax(v1x, v2x)), bmaxy = dmax(v0y, dmax(v1y, v2y)), bmaxz = dmax(v0z, dmax(v1z, v2z));
    const int gx0 = clampi((int)(bminx / u.x), 0, res - 1), gy0 = clampi((int)(bminy / u.y), 0, res - 1),
              gz0 = clampi((int)(bminz / u.z), 0, res - 1);
    const int gx1 = clampi((int)(bmaxx / u.x), 0, res - 1), gy1 = clampi((int)(bmaxy / u.y), 0, res - 1),
              gz1 = clampi((int)(bmaxz / u.z), 0, res - 1);
    const double cx = nx > 0.0 ? u.x : 0.0, cy = ny > 0.0 ? u.y : 0.0, cz = nz > 0.0 ? u.z : 0.0;
    double d1 = nx * (cx - v0x);
    d1 = d1 + ny * (cy - v0y);
    d1 = d1 + nz * (cz - v0z);
    double d2 = nx * ((u.x - cx) - v0x);
    d2 = d2 + ny * ((u.y - cy) - v0y);
    d2 = d2 + nz * ((u.z - cz) - v0z);
    const E2 xy0 = edgeTest(-1.0 * e0y, e0x, nz < 0.0, v0x, v0y, u.x, u.y);
    const E2 xy1 = edgeTest(-1.0 * e1y, e1x, nz < 0.0, v1x, v1y, u.x, u.y);
    const E2 xy2 = edgeTest(-1.0 * e2y, e2x, nz < 0.0, v2x, v2y, u.x, u.y);
    const E2 yz0 = edgeTest(-1.0 * e0z, e0y, nx < 0.0, v0y, v0z, u.y, u.z);
    const E2 yz1 = edgeTest(-1.0 * e1z, e1y, nx < 0.0, v1y, v1z, u.y, u.z);
    const E2 yz2 = edgeTest(-1.0 * e2z, e2y, nx < 0.0, v2y, v2z, u.y, u.z);
    const E2 zx0 = edgeTest(-1.0 * e0x, e0z, ny < 0.0, v0z, v0x, u.z, u.x);
    const E2 zx1 = edgeTest(-1.0 * e1x, e1z, ny < 0.0, v1z, v1x, u.z, u.x);
    const E2 zx2 = edgeTest(-1.0 * e2x, e2z, ny < 0.0, v2z, v2x, u.z, u.x);
    for (int z = gz0; z <= gz1; ++z)
      for (int y = gy0; y <= gy1; ++y)
        for (int x = gx0; x <= gx1; ++x) {
          const double px = (double)x * u.x, py = (double)y * u.y, pz = (double)z * u.z;
          double nd = nx * px;
          nd = nd + ny * py;
          nd = nd + nz * pz;
          if ((nd + d1) * (nd + d2) > 0.0) continue;
          if ((xy0.a * px + xy0.b * py) + xy0.d < 0.0) continue;
          if ((xy1.a * px + xy1.b * py) + xy1.d < 0.0) continue;
          if ((xy2.a * px + xy2.b * py) + xy2.d < 0.0) continue;
          if ((yz0.a * py + yz0.b * pz) + yz0.d < 0.0) continue;
          if ((yz1.a * py + yz1.b * pz) + yz1.d < 0.0) continue;
          if ((yz2.a * py + yz2.b * pz) + yz2.d < 0.0) continue;
          if ((zx0.a * pz + zx0.b * px) + zx0.d < 0.0) continue;
          if ((zx1.a * pz + zx1.b * px) + zx1.d < 0.0) continue;
          if ((zx2.a * pz + zx2.b * px) + zx2.d < 0.0) continue;
          const uint32_t m = mortonEncode((uint32_t)x, (uint32_t)y, (uint32_t)z);
          atomicOr(occ + (m >> 6), 1ull << (m & 63));
        }
  }
}

// ---- level build ---------------------------------------------------------------------------
__global__ void kFillGroups(int64_t G, const uint32_t* __restrict__ next, uint32_t* morton, uint32_t* parent,
                            uint32_t* child0, uint8_t* leaf, int64_t start) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // node within the level
  if (i >= 8 * G) return;
  const int64_t g = i >> 3;
  morton[start + i] = (next[g] << 3) | (uint32_t)(i & 7);
  parent[start + i] = kNone;
  child0[start + i] = kNone;
  leaf[start + i] = 1;
}
// Occupied nodes of level L >= 1 (createNode_2, SVO.cu:596-638): not leaves, children are the
// i-th sibling group of level L-1, which point back at them.
__global__ void kFillOccupied(int64_t c, const uint32_t* __restrict__ O, const uint32_t* __restrict__ grp,
                              int64_t start, int64_t childStart, uint32_t* parent, uint32_t* child0,
                              uint8_t* leaf) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= c) return;
  const uint32_t node = (uint32_t)(start + 8 * (int64_t)grp[i] + (O[i] & 7u));
  leaf[node] = 0;
  child0[node] = (uint32_t)(childStart + 8 * i);
#pragma unroll
  for (int k = 0; k < 8; ++k) parent[childStart + 8 * i + k] = node;
}
__global__ void kFillRoot(uint32_t O0, int64_t start, int64_t childStart, int hasChildren, uint32_t* morton,
                          uint32_t* parent, uint32_t* child0, uint8_t* leaf, uint32_t* nb) {
  const int k = threadIdx.x;
  if (k == 0) {
    morton[start] = O0;
    parent[start] = kNone;
    child0[start] = hasChildren ? (uint32_t)childStart : kNone;
    leaf[start] = hasChildren ? 0 : 1;
  }
  if (k < 27) nb[start * 27 + k] = (k == 13) ? (uint32_t)start : kNone;
  if (hasChildren && k < 8) parent[childStart + k] = (uint32_t)start;
}

// 27-neighbours top-down (findNeighbors, SVO.cu:861-890): the neighbour at offset d of the
// child with key k is child ((k+d) mod 2) of the parent's neighbour floor((k+d)/2).
__global__ void kNeighbors(int64_t count, int64_t start, const uint32_t* __restrict__ morton,
                           const uint32_t* __restrict__ parent, const uint32_t* __restrict__ child0,
                           uint32_t* nb) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= count * 27) return;
  const int64_t t = start + idx / 27;
  const int s = (int)(idx % 27);
  const uint32_t key = morton[t] & 7u;
  const int d[3] = {s % 3 - 1, (s / 3) % 3 - 1, s / 9 - 1};
  int P[3], C = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int tt = (int)((key >> a) & 1u) + d[a];
    P[a] = tt < 0 ? -1 : (tt > 1 ? 1 : 0);
    C |= (tt & 1) << a;
  }
  const uint32_t p = parent[t];
  const uint32_t pn = nb[(int64_t)p * 27 + (P[0] + 1) + 3 * (P[1] + 1) + 9 * (P[2] + 1)];
  uint32_t r = kNone;
  if (pn != kNone) {
    const uint32_t c0 = child0[pn];
    if (c0 != kNone) r = c0 + (uint32_t)C;
  }
  nb[t * 27 + s] = r;
}

// ---- corner vertices (determineNodeVertex + sort + unique, SVO.cu:913-963, 1064-1096) -------
__global__ void kMarkCorners(int64_t count, int64_t start, const uint32_t* __restrict__ morton, uint32_t M,
                             unsigned long long* bits) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= count * 8) return;
  const int64_t t = start + (idx >> 3);
  const int k = (int)(idx & 7);
  uint32_t X, Y, Z;
  mortonDecode(morton[t], X, Y, Z);
  const uint32_t lin = ((X + (k & 1)) * M + (Y + ((k >> 1) & 1))) * M + (Z + ((k >> 2) & 1));
  atomicOr(bits + (lin >> 6), 1ull << (lin & 63));
}
__global__ void kEmitBits(int64_t words, const unsigned long long* __restrict__ bits,
                          const uint32_t* __restrict__ rank, uint32_t* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= words) return;
  unsigned long long w = bits[i];
  uint32_t r = rank[i];
  while (w) {
    const int b = __ffsll((long long)w) - 1;
    out[r++] = (uint32_t)(i * 64 + b);
    w &= w - 1;
  }
}
__global__ void kOwnerCorners(int64_t count, int64_t start, const uint32_t* __restrict__ morton, LatticeIndex L,
                              uint32_t* owner) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= count * 8) return;
  const int64_t t = start + (idx >> 3);
  const int k = (int)(idx & 7);
  uint32_t X, Y, Z;
  mortonDecode(morton[t], X, Y, Z);
  const uint32_t lin = ((X + (k & 1)) * L.M + (Y + ((k >> 1) & 1))) * L.M + (Z + ((k >> 2) & 1));
  atomicMin(owner + latticeRank(L, lin), (uint32_t)t);
}
// Representative position of a corner: taken from its owner node, corner = origin (+ w),
// origin = g + w*X (the surviving entry of the reference's stable sort + unique).
// Also the vertex's packed key (lattice coordinates, depth, corner of the owner).
__global__ void kVertexPositions(int64_t count, int64_t vstart, uint32_t M, int depth, double3 g, double w,
                                 const uint32_t* __restrict__ lin, const uint32_t* __restrict__ owner,
                                 const uint32_t* __restrict__ morton, double* __restrict__ pos,
                                 uint64_t* __restrict__ key) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int64_t v = vstart + i;
  const uint32_t l = lin[v];
  const uint32_t X = l / (M * M), Y = (l / M) % M, Z = l % M;
  uint32_t Xo, Yo, Zo;
  mortonDecode(morton[owner[v]], Xo, Yo, Zo);
  key[v] = encodeVertKey(X, Y, Z, depth, Xo, Yo, Zo);
  const double bx = latticePos(g.x, w, Xo), by = latticePos(g.y, w, Yo), bz = latticePos(g.z, w, Zo);
  pos[3 * v] = (X != Xo) ? bx + w : bx;
  pos[3 * v + 1] = (Y != Yo) ? by + w : by;
  pos[3 * v + 2] = (Z != Zo) ? bz + w : bz;
}

// ---- fine-node edges (determineNodeEdge + sort + unique, SVO.cu:965-1008, 1098-1110) --------
// Edge key = lin(lower end)*3 + {z:0, y:1, x:2}: the reference's lexicographic order of
// (first point, second point).
__device__ __constant__ int8_t cEdgeCorners[12][2] = {{0, 2}, {2, 3}, {1, 3}, {0, 1}, {4, 6}, {6, 7},
                                                    {5, 7}, {4, 5}, {0, 4}, {2, 6}, {3, 7}, {1, 5}};
__device__ inline uint32_t fineEdgeKey(uint32_t X, uint32_t Y, uint32_t Z, int e, uint32_t M) {
  const int a = cEdgeCorners[e][0], b = cEdgeCorners[e][1];
  const uint32_t sx = X + (a & 1), sy = Y + ((a >> 1) & 1), sz = Z + ((a >> 2) & 1);
  const int diff = a ^ b;  // 1: x, 2: y, 4: z
  const uint32_t ord = diff == 4 ? 0u : (diff == 2 ? 1u : 2u);
  return ((sx * M + sy) * M + sz) * 3u + ord;
}
__global__ void kMarkEdges(int64_t count, const uint32_t* __restrict__ morton, uint32_t M,
                           unsigned long long* bits) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= count * 12) return;
  const int64_t t = idx / 12;
  const int e = (int)(idx % 12);
  uint32_t X, Y, Z;
  mortonDecode(morton[t], X, Y, Z);
  const uint32_t key = fineEdgeKey(X, Y, Z, e, M);
  atomicOr(bits + (key >> 6), 1ull << (key & 63));
}
__global__ void kOwnerEdges(int64_t count, const uint32_t* __restrict__ morton, uint32_t M,
                            const unsigned long long* __restrict__ bits, const uint32_t* __restrict__ rank,
                            uint32_t* owner) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= count * 12) return;
  const int64_t t = idx / 12;
  const int e = (int)(idx % 12);
  uint32_t X, Y, Z;
  mortonDecode(morton[t], X, Y, Z);
  const uint32_t key = fineEdgeKey(X, Y, Z, e, M);
  const unsigned long long w = bits[key >> 6];
  const uint32_t r = rank[key >> 6] + (uint32_t)__popcll(w & ((1ull << (key & 63)) - 1ull));
  atomicMin(owner + r, (uint32_t)t);
}
__global__ void kMarkFine(int64_t count, const uint32_t* __restrict__ morton, unsigned long long* occ) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count) return;
  const uint32_t m = morton[t];
  atomicOr(occ + (m >> 6), 1ull << (m & 63));
}

// ---- getters -------------------------------------------------------------------------------------
__global__ void kNodeGeometry(int64_t count, int64_t start, double3 g, double w, const uint32_t* __restrict__ morton,
                              double* origin, double* width) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int64_t t = start + i;
  uint32_t X, Y, Z;
  mortonDecode(morton[t], X, Y, Z);
  if (origin) {
    origin[3 * t] = latticePos(g.x, w, X);
    origin[3 * t + 1] = latticePos(g.y, w, Y);
    origin[3 * t + 2] = latticePos(g.z, w, Z);
  }
  if (width) width[t] = w;
}
__global__ void kExpandChildren(int64_t n, const uint32_t* __restrict__ child0, uint32_t* childs) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * 8) return;
  const uint32_t c = child0[i >> 3];
  childs[i] = (c == kNone) ? kNone : c + (uint32_t)(i & 7);
}
__global__ void kEdgePositions(int64_t E, uint32_t M, double3 g, double w, const uint32_t* __restrict__ key,
                               const uint32_t* __restrict__ owner, const uint32_t* __restrict__ morton,
                               double* p0, double* p1) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= E) return;
  const uint32_t k = key[i];
  const uint32_t lin = k / 3, ord = k % 3;
  const uint32_t X = lin / (M * M), Y = (lin / M) % M, Z = lin % M;
  uint32_t Xo, Yo, Zo;
  mortonDecode(morton[owner[i]], Xo, Yo, Zo);
  const double bx = latticePos(g.x, w, Xo), by = latticePos(g.y, w, Yo), bz = latticePos(g.z, w, Zo);
  const uint32_t E1[3] = {X + (ord == 2), Y + (ord == 1), Z + (ord == 0)};
  const uint32_t S[3] = {X, Y, Z}, O[3] = {Xo, Yo, Zo};
  const double B[3] = {bx, by, bz};
  for (int a = 0; a < 3; ++a) {
    if (p0) p0[3 * i + a] = (S[a] != O[a]) ? B[a] + w : B[a];
    if (p1) p1[3 * i + a] = (E1[a] != O[a]) ? B[a] + w : B[a];
  }
}

}  // namespace its

// =====================================================================================
using namespace its;

static void svoRelease(its_svo* s) {
  if (!s) return;
  its::destroyPlan(s->plan);
  s->plan = nullptr;
  its_ctx* c = s->ctx;
  SvoDevice& d = s->d;
  void* ptrs[] = {d.voxels, d.nodeMorton, d.nodeParent, d.nodeChild0, d.nodeLeaf, d.nodeNb, d.vertLin, d.vertKey,
                  d.vertOwner, d.vertPos, d.ebits, d.erank, d.edgeKey, d.edgeOwner, d.fineOcc, d.fineRank,
                  d.nodeSampleCnt, d.nodeSamplePos, d.nodeSampleNrm, d.coincIds, d.rowParams, d.coincGeom};
  for (void* p : ptrs) devFree(c, p);
  for (int i = 0; i < kMaxDepth; ++i) { devFree(c, d.vbits[i]); devFree(c, d.vrank[i]); }
  d = SvoDevice();
}

namespace its {

its_status svoBuild(its_ctx* ctx, const double* dV, int64_t nv, const int32_t* dF, int64_t nf, int res,
                    const double origin[3], const double width[3], its_svo* s) {
  (void)nv;
  SvoDevice& d = s->d;
  d.res = res;
  for (int a = 0; a < 3; ++a) { d.origin[a] = origin[a]; d.unit[a] = width[a] / res; }
  const double3 g = make_double3(origin[0], origin[1], origin[2]);
  const double3 u = make_double3(d.unit[0], d.unit[1], d.unit[2]);
  const int64_t gridBits = (int64_t)res * res * res;
  const int64_t gridWords = (gridBits + 63) / 64;
  its_status st;
  // device time of the build and of the learned fit's tables (reported by its_svo_get_info)
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  for (auto& e : ev) ITS_CU(ctx, cudaEventCreate(&e));
  struct EvFree {
    cudaEvent_t* e;
    ~EvFree() { for (int k = 0; k < 3; ++k) if (e[k]) cudaEventDestroy(e[k]); }
  } evFree{ev};
  ITS_CU(ctx, cudaEventRecord(ev[0], ctx->stream));

  // 1. voxelise into the Morton bitset
  DevBuf<unsigned long long> occ;
  if ((st = occ.zeros(ctx, gridWords)) != ITS_OK) return st;
  if (nf > 0) {
    const int block = 128;
    const unsigned grid = (unsigned)std::min<int64_t>(gridFor(nf, block), (int64_t)ctx->numSMs * 64);
    kVoxelize<<<grid, block, 0, ctx->stream>>>(dV, dF, nf, res, g, u, occ.p);
    ITS_LAUNCHED(ctx);
  }
  // 2. compact to the sorted list of surface voxels
  DevBuf<uint32_t> dCount;
  if ((st = dCount.alloc(ctx, 1)) != ITS_OK) return st;
  {
    const unsigned long long* bits = occ.p;
    auto f = [bits] __device__(int64_t i) -> uint32_t { return (uint32_t)__popcll(bits[i]); };
    DevBuf<uint32_t> wordRank;
    if ((st = wordRank.alloc(ctx, gridWords)) != ITS_OK) return st;
    uint32_t* wr = wordRank.p;
    if ((st = scanExclusiveAlloc<uint32_t>(ctx, f, gridWords, StorePrefix<uint32_t>{wr}, dCount.p)) != ITS_OK) return st;
    uint32_t nvox = 0;
    if ((st = readScalar(ctx, dCount.p, &nvox)) != ITS_OK) return st;
    d.numVoxels = nvox;
    if (nvox == 0) return setError(ctx, ITS_ERR_INVALID, "no surface voxel: the mesh does not meet the grid");
    if ((st = devAlloc(ctx, (void**)&d.voxels, nvox * sizeof(uint32_t))) != ITS_OK) return st;
    kEmitBits<<<gridFor(gridWords, 256), 256, 0, ctx->stream>>>(gridWords, occ.p, wr, d.voxels);
    ITS_LAUNCHED(ctx);
  }
  occ.reset();

  // 3. levels: O_{L+1} = unique(O_L >> 3); group index of every element
  std::vector<DevBuf<uint32_t>> O, grp;  // levels >= 1 and per-level group indices
  std::vector<int64_t> cnt;
  const uint32_t* cur = d.voxels;
  int64_t c = d.numVoxels;
  std::vector<const uint32_t*> Optr;
  Optr.push_back(cur);
  cnt.push_back(c);
  while (c > 1) {
    if ((int)cnt.size() >= kMaxDepth) return setError(ctx, ITS_ERR_INVALID, "octree deeper than supported");
    DevBuf<uint32_t> g1(ctx), nx(ctx);
    if ((st = g1.alloc(ctx, c)) != ITS_OK) return st;
    if ((st = nx.alloc(ctx, c)) != ITS_OK) return st;
    const uint32_t* Oc = cur;
    uint32_t* gp = g1.p;
    uint32_t* np = nx.p;
    auto head = [Oc] __device__(int64_t i) -> uint32_t { return (i == 0 || (Oc[i] >> 3) != (Oc[i - 1] >> 3)) ? 1u : 0u; };
    auto wr = [Oc, gp, np] __device__(int64_t i, uint32_t prefix, uint32_t v) {
      gp[i] = prefix + v - 1u;
      if (v) np[prefix] = Oc[i] >> 3;
    };
    if ((st = scanExclusiveAlloc<uint32_t>(ctx, head, c, wr, dCount.p)) != ITS_OK) return st;
    uint32_t G = 0;
    if ((st = readScalar(ctx, dCount.p, &G)) != ITS_OK) return st;
    grp.push_back(std::move(g1));
    O.push_back(std::move(nx));
    cur = O.back().p;
    Optr.push_back(cur);
    c = G;
    cnt.push_back(c);
  }
  const int top = (int)cnt.size() - 1;  // root level
  d.depth = top + 1;
  int64_t total = 0;
  for (int L = 0; L <= top; ++L) {
    d.levelStart[L] = total;
    d.levelCount[L] = (L < top) ? 8 * cnt[L + 1] : 1;
    total += d.levelCount[L];
  }
  d.levelStart[top + 1] = total;
  d.numNodes = total;
  if ((st = devAlloc(ctx, (void**)&d.nodeMorton, total * 4)) != ITS_OK) return st;
  if ((st = devAlloc(ctx, (void**)&d.nodeParent, total * 4)) != ITS_OK) return st;
  if ((st = devAlloc(ctx, (void**)&d.nodeChild0, total * 4)) != ITS_OK) return st;
  if ((st = devAlloc(ctx, (void**)&d.nodeLeaf, total)) != ITS_OK) return st;
  if ((st = devAlloc(ctx, (void**)&d.nodeNb, total * 27 * 4)) != ITS_OK) return st;
  for (int L = 0; L < top; ++L) {
    const int64_t G = cnt[L + 1];
    kFillGroups<<<gridFor(8 * G, 256), 256, 0, ctx->stream>>>(G, Optr[L + 1], d.nodeMorton, d.nodeParent,
                                                              d.nodeChild0, d.nodeLeaf, d.levelStart[L]);
    ITS_LAUNCHED(ctx);
  }
  for (int L = 1; L < top; ++L) {
    kFillOccupied<<<gridFor(cnt[L], 256), 256, 0, ctx->stream>>>(cnt[L], Optr[L], grp[L].p, d.levelStart[L],
                                                                  d.levelStart[L - 1], d.nodeParent,
                                                                  d.nodeChild0, d.nodeLeaf);
    ITS_LAUNCHED(ctx);
  }
  {
    uint32_t O0 = 0;
    ITS_CU(ctx, cudaMemcpyAsync(&O0, Optr[top], 4, cudaMemcpyDeviceToHost, ctx->stream));
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
    kFillRoot<<<1, 32, 0, ctx->stream>>>(O0, d.levelStart[top], top >= 1 ? d.levelStart[top - 1] : 0, top >= 1 ? 1 : 0,
                                         d.nodeMorton, d.nodeParent, d.nodeChild0, d.nodeLeaf, d.nodeNb);
    ITS_LAUNCHED(ctx);
  }
  O.clear();
  grp.clear();

  // 4. neighbours, top-down
  for (int L = top - 1; L >= 0; --L) {
    const int64_t n27 = d.levelCount[L] * 27;
    kNeighbors<<<gridFor(n27, 256), 256, 0, ctx->stream>>>(d.levelCount[L], d.levelStart[L], d.nodeMorton,
                                                           d.nodeParent, d.nodeChild0, d.nodeNb);
    ITS_LAUNCHED(ctx);
  }

  // 5. corner vertices per depth
  DevBuf<uint32_t> vcnt;
  if ((st = vcnt.zeros(ctx, d.depth)) != ITS_OK) return st;
  for (int L = 0; L < d.depth; ++L) {
    const uint32_t M = (uint32_t)(res >> L) + 1u;
    const int64_t words = ((int64_t)M * M * M + 63) / 64;
    if ((st = devAlloc(ctx, (void**)&d.vbits[L], words * 8)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&d.vrank[L], words * 4)) != ITS_OK) return st;
    ITS_CU(ctx, cudaMemsetAsync(d.vbits[L], 0, words * 8, ctx->stream));
    kMarkCorners<<<gridFor(d.levelCount[L] * 8, 256), 256, 0, ctx->stream>>>(d.levelCount[L], d.levelStart[L],
                                                                              d.nodeMorton, M, d.vbits[L]);
    ITS_LAUNCHED(ctx);
    const unsigned long long* bits = d.vbits[L];
    auto f = [bits] __device__(int64_t i) -> uint32_t { return (uint32_t)__popcll(bits[i]); };
    if ((st = scanExclusiveAlloc<uint32_t>(ctx, f, words, StorePrefix<uint32_t>{d.vrank[L]}, vcnt.p + L)) != ITS_OK)
      return st;
  }
  {
    std::vector<uint32_t> hv(d.depth);
    ITS_CU(ctx, cudaMemcpyAsync(hv.data(), vcnt.p, 4 * d.depth, cudaMemcpyDeviceToHost, ctx->stream));
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
    int64_t t = 0;
    for (int L = 0; L < d.depth; ++L) { d.vertStart[L] = t; d.vertCount[L] = hv[L]; t += hv[L]; }
    d.vertStart[d.depth] = t;
    d.numVerts = t;
  }
  if ((st = devAlloc(ctx, (void**)&d.vertLin, d.numVerts * 4)) != ITS_OK) return st;
  if ((st = devAlloc(ctx, (void**)&d.vertOwner, d.numVerts * 4)) != ITS_OK) return st;
  if ((st = devAlloc(ctx, (void**)&d.vertPos, d.numVerts * 24)) != ITS_OK) return st;
  if ((st = devAlloc(ctx, (void**)&d.vertKey, d.numVerts * 8)) != ITS_OK) return st;
  ITS_CU(ctx, cudaMemsetAsync(d.vertOwner, 0xFF, d.numVerts * 4, ctx->stream));
  for (int L = 0; L < d.depth; ++L) {
    const uint32_t M = (uint32_t)(res >> L) + 1u;
    const int64_t words = ((int64_t)M * M * M + 63) / 64;
    kEmitBits<<<gridFor(words, 256), 256, 0, ctx->stream>>>(words, d.vbits[L], d.vrank[L], d.vertLin + d.vertStart[L]);
    ITS_LAUNCHED(ctx);
    kOwnerCorners<<<gridFor(d.levelCount[L] * 8, 256), 256, 0, ctx->stream>>>(d.levelCount[L], d.levelStart[L],
                                                                               d.nodeMorton, d.lattice(L), d.vertOwner);
    ITS_LAUNCHED(ctx);
    const double w = d.unit[0] * (double)(1u << L);
    kVertexPositions<<<gridFor(d.vertCount[L], 256), 256, 0, ctx->stream>>>(d.vertCount[L], d.vertStart[L], M, L, g,
                                                                             w, d.vertLin, d.vertOwner, d.nodeMorton,
                                                                             d.vertPos, d.vertKey);
    ITS_LAUNCHED(ctx);
  }

  // 6. fine-node edges and the fine-node occupancy bitset
  {
    const uint32_t M = (uint32_t)res + 1u;
    const int64_t ebitsN = 3ll * M * M * M;
    const int64_t words = (ebitsN + 63) / 64;
    if ((st = devAlloc(ctx, (void**)&d.ebits, words * 8)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&d.erank, words * 4)) != ITS_OK) return st;
    ITS_CU(ctx, cudaMemsetAsync(d.ebits, 0, words * 8, ctx->stream));
    const int64_t nf0 = d.levelCount[0];
    kMarkEdges<<<gridFor(nf0 * 12, 256), 256, 0, ctx->stream>>>(nf0, d.nodeMorton, M, d.ebits);
    ITS_LAUNCHED(ctx);
    const unsigned long long* bits = d.ebits;
    auto f = [bits] __device__(int64_t i) -> uint32_t { return (uint32_t)__popcll(bits[i]); };
    if ((st = scanExclusiveAlloc<uint32_t>(ctx, f, words, StorePrefix<uint32_t>{d.erank}, dCount.p)) != ITS_OK) return st;
    uint32_t ne = 0;
    if ((st = readScalar(ctx, dCount.p, &ne)) != ITS_OK) return st;
    d.numEdges = ne;
    if ((st = devAlloc(ctx, (void**)&d.edgeKey, (size_t)ne * 4)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&d.edgeOwner, (size_t)ne * 4)) != ITS_OK) return st;
    ITS_CU(ctx, cudaMemsetAsync(d.edgeOwner, 0xFF, (size_t)ne * 4, ctx->stream));
    kEmitBits<<<gridFor(words, 256), 256, 0, ctx->stream>>>(words, d.ebits, d.erank, d.edgeKey);
    ITS_LAUNCHED(ctx);
    kOwnerEdges<<<gridFor(nf0 * 12, 256), 256, 0, ctx->stream>>>(nf0, d.nodeMorton, M, d.ebits, d.erank, d.edgeOwner);
    ITS_LAUNCHED(ctx);
    if ((st = devAlloc(ctx, (void**)&d.fineOcc, gridWords * 8)) != ITS_OK) return st;
    ITS_CU(ctx, cudaMemsetAsync(d.fineOcc, 0, gridWords * 8, ctx->stream));
    kMarkFine<<<gridFor(nf0, 256), 256, 0, ctx->stream>>>(nf0, d.nodeMorton, (unsigned long long*)d.fineOcc);
    ITS_LAUNCHED(ctx);
    if ((st = devAlloc(ctx, (void**)&d.fineRank, gridWords * 4)) != ITS_OK) return st;
    const unsigned long long* occBits = (const unsigned long long*)d.fineOcc;
    auto pc = [occBits] __device__(int64_t i) -> uint32_t { return (uint32_t)__popcll(occBits[i]); };
    if ((st = scanExclusiveAlloc<uint32_t>(ctx, pc, gridWords, StorePrefix<uint32_t>{d.fineRank}, (uint32_t*)nullptr)) !=
        ITS_OK)
      return st;
  }
  // per-node sums of the face samples (features of the share network)
  ITS_CU(ctx, cudaEventRecord(ev[1], ctx->stream));
  if ((st = nodeSampleStats(ctx, d, dV, dF, nf)) != ITS_OK) return st;
  // the coincident vertices (the shares of the exact start)
  if ((st = devAlloc(ctx, (void**)&d.coincIds, std::max<int64_t>(d.numVerts, 1) * 8)) != ITS_OK) return st;
  if ((st = coincidentIds(ctx, d, d.coincIds, &d.numCoinc)) != ITS_OK) return st;
  if ((st = coincidentGeometry(ctx, d)) != ITS_OK) return st;
  // the row parameters of the matrix-free kernels, on the device for the octree's lifetime
  const RowParams hp = rowParams(d);
  if ((st = devAlloc(ctx, &d.rowParams, sizeof(RowParams))) != ITS_OK) return st;
  ITS_CU(ctx, cudaMemcpyAsync(d.rowParams, &hp, sizeof(RowParams), cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaEventRecord(ev[2], ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  cudaEventElapsedTime(&d.buildMs, ev[0], ev[2]);
  cudaEventElapsedTime(&d.learnedTablesMs, ev[1], ev[2]);
  return ITS_OK;
}

}  // namespace its

// ================================ C ABI ===============================================
extern "C" {

its_status its_svo_build(its_ctx* ctx, const double* verts, int64_t nverts, const int32_t* faces, int64_t nfaces,
                         int res, const double origin[3], const double width[3], its_svo** out) {
  if (!ctx || !out) return ITS_ERR_INVALID;
  *out = nullptr;
  if (!verts || !faces || nverts <= 0 || nfaces <= 0 || !origin || !width)
    return setError(ctx, ITS_ERR_INVALID, "its_svo_build: empty mesh or missing arguments");
  if (res < 1 || res > 1024 || (res & (res - 1)))
    return setError(ctx, ITS_ERR_INVALID, "its_svo_build: res must be a power of two in [1, 1024]");
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(origin[a]) || !(width[a] > 0.0) || !std::isfinite(width[a]))
      return setError(ctx, ITS_ERR_INVALID, "its_svo_build: bounding box must be finite with positive width");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> V;
  InArg<int32_t> F;
  its_status st;
  if ((st = V.stage(ctx, verts, 3 * nverts)) != ITS_OK) return st;
  if ((st = F.stage(ctx, faces, 3 * nfaces)) != ITS_OK) return st;
  if ((st = validateMesh(ctx, V.d, nverts, F.d, nfaces)) != ITS_OK) return st;
  its_svo* s = new its_svo;
  s->ctx = ctx;
  st = svoBuild(ctx, V.d, nverts, F.d, nfaces, res, origin, width, s);
  if (st != ITS_OK) {
    svoRelease(s);
    delete s;
    return st;
  }
  *out = s;
  return ITS_OK;
}

its_status its_svo_free(its_svo* s) {
  if (!s) return ITS_OK;
  its_ctx* c = s->ctx;
  svoRelease(s);
  cudaStreamSynchronize(c->stream);
  delete s;
  return ITS_OK;
}

its_status its_svo_get_info(const its_svo* s, its_svo_info* info) {
  if (!s || !info) return ITS_ERR_INVALID;
  const SvoDevice& d = s->d;
  *info = its_svo_info{};
  info->res = d.res;
  info->depth = d.depth;
  info->num_voxels = d.numVoxels;
  info->num_fine_nodes = d.levelCount[0];
  info->num_nodes = d.numNodes;
  info->num_vertices = d.numVerts;
  info->num_edges = d.numEdges;
  for (int L = 0; L < d.depth && L < 16; ++L) {
    info->nodes_per_depth[L] = d.levelCount[L];
    info->vertices_per_depth[L] = d.vertCount[L];
  }
  for (int a = 0; a < 3; ++a) { info->origin[a] = d.origin[a]; info->unit[a] = d.unit[a]; }
  info->build_ms = d.buildMs;
  info->learned_tables_ms = d.learnedTablesMs;
  return ITS_OK;
}

its_status its_svo_get_voxels(its_svo* s, uint32_t* morton) {
  if (!s || !morton) return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  ITS_CU(ctx, cudaMemcpyAsync(morton, s->d.voxels, s->d.numVoxels * 4, cudaMemcpyDefault, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_svo_get_nodes(its_svo* s, uint32_t* morton, uint32_t* parent, uint32_t* childs, uint8_t* is_leaf,
                             double* origin, double* width, uint32_t* neighbors) {
  if (!s) return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  const SvoDevice& d = s->d;
  const int64_t N = d.numNodes;
  if (morton) ITS_CU(ctx, cudaMemcpyAsync(morton, d.nodeMorton, N * 4, cudaMemcpyDefault, ctx->stream));
  if (parent) ITS_CU(ctx, cudaMemcpyAsync(parent, d.nodeParent, N * 4, cudaMemcpyDefault, ctx->stream));
  if (is_leaf) ITS_CU(ctx, cudaMemcpyAsync(is_leaf, d.nodeLeaf, N, cudaMemcpyDefault, ctx->stream));
  if (neighbors) ITS_CU(ctx, cudaMemcpyAsync(neighbors, d.nodeNb, N * 27 * 4, cudaMemcpyDefault, ctx->stream));
  its_status st;
  if (childs) {
    OutArg<uint32_t> o;
    if ((st = o.stage(ctx, childs, N * 8)) != ITS_OK) return st;
    kExpandChildren<<<gridFor(N * 8, 256), 256, 0, ctx->stream>>>(N, d.nodeChild0, o.d);
    ITS_LAUNCHED(ctx);
    if ((st = o.finish(ctx)) != ITS_OK) return st;
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  }
  if (origin || width) {
    OutArg<double> o, w;
    if ((st = o.stage(ctx, origin, N * 3)) != ITS_OK) return st;
    if ((st = w.stage(ctx, width, N)) != ITS_OK) return st;
    const double3 g = make_double3(d.origin[0], d.origin[1], d.origin[2]);
    for (int L = 0; L < d.depth; ++L) {
      kNodeGeometry<<<gridFor(d.levelCount[L], 256), 256, 0, ctx->stream>>>(
          d.levelCount[L], d.levelStart[L], g, d.unit[0] * (double)(1u << L), d.nodeMorton, o.d, w.d);
      ITS_LAUNCHED(ctx);
    }
    if ((st = o.finish(ctx)) != ITS_OK) return st;
    if ((st = w.finish(ctx)) != ITS_OK) return st;
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  }
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_svo_get_vertices(its_svo* s, double* pos, uint32_t* owner) {
  if (!s) return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  if (pos) ITS_CU(ctx, cudaMemcpyAsync(pos, s->d.vertPos, s->d.numVerts * 24, cudaMemcpyDefault, ctx->stream));
  if (owner) ITS_CU(ctx, cudaMemcpyAsync(owner, s->d.vertOwner, s->d.numVerts * 4, cudaMemcpyDefault, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_svo_get_edges(its_svo* s, double* p0, double* p1, uint32_t* owner) {
  if (!s) return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  const SvoDevice& d = s->d;
  const int64_t E = d.numEdges;
  its_status st;
  if (owner) ITS_CU(ctx, cudaMemcpyAsync(owner, d.edgeOwner, E * 4, cudaMemcpyDefault, ctx->stream));
  if ((p0 || p1) && E > 0) {
    OutArg<double> a, b;
    if ((st = a.stage(ctx, p0, E * 3)) != ITS_OK) return st;
    if ((st = b.stage(ctx, p1, E * 3)) != ITS_OK) return st;
    kEdgePositions<<<gridFor(E, 256), 256, 0, ctx->stream>>>(E, (uint32_t)d.res + 1u,
                                                             make_double3(d.origin[0], d.origin[1], d.origin[2]),
                                                             d.unit[0], d.edgeKey, d.edgeOwner, d.nodeMorton, a.d, b.d);
    ITS_LAUNCHED(ctx);
    if ((st = a.finish(ctx)) != ITS_OK) return st;
    if ((st = b.finish(ctx)) != ITS_OK) return st;
  }
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // extern "C"
