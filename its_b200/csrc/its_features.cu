// Per-vertex features of the share network and the learned start.
//
// For every corner vertex v coincident with a coarser corner (lattice coordinates all even
// below the root depth; these are the free shares of the exact start) 64 FP32 features:
//   0  b_v (signed distance at v)            1  s: zero-share surplus of v's coarsest copy
//   2  zero-share value of the copy one depth up
//   3  depth / (depth count - 1)             4, 5  coarser / finer copies of v, / depth count
//   6-11  same-depth axis neighbours present (+x -x +y -y +z -z)
//   12-17 their b minus b_v                  18-23 their zero-share values
//   24-29 finer-depth odd neighbours (2X +- e) present   30-35 their zero-share values
//   36 cell width w_d                        37 b_v / w_d
//   38 log(1 + samples in the owner node's 27-neighbourhood)
//   39-41 mean sample offset from v / w_d    42-44 mean sample normal
//   45 curvature proxy 1 - |mean normal|     46-63 zero
// Samples are the mesh's face centroids with unit face normals; their per-node sums are
// formed finest depth first (a stable sort of the samples by fine node, a segmented sum in
// sample order, then each node sums its 8 children), so the features are deterministic.
// Features 38-45 depend on the octree and the mesh only and are computed with the octree
// (its_svo_build); the rest, which depend on b, with every fit.
// Features are optionally normalised, (f - mean) * scale, as the network was trained.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "its_op.cuh"
#include "its_scan.cuh"
#include "its_umma.cuh"

namespace its {

constexpr int kFeat = 64;

struct NodeStats {
  float* cnt;  // per node
  double* sp;  // 3 per node: sum of sample positions
  double* sn;  // 3 per node: sum of unit normals
};

// Face centroid, unit normal and fine node (fineCount when no fine node holds the centroid).
__global__ void kFaceSamples(const double* __restrict__ V, const int32_t* __restrict__ F, int64_t nf, double3 g,
                             double w0, int res, const unsigned long long* __restrict__ occ,
                             const uint32_t* __restrict__ occRank, int64_t fineCount,
                             double* __restrict__ cent, double* __restrict__ nrm, uint32_t* __restrict__ node,
                             uint32_t* __restrict__ ids) {
  const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const double* a = V + 3 * (int64_t)F[3 * f];
  const double* b = V + 3 * (int64_t)F[3 * f + 1];
  const double* c = V + 3 * (int64_t)F[3 * f + 2];
  const double cx = (a[0] + b[0] + c[0]) / 3.0, cy = (a[1] + b[1] + c[1]) / 3.0, cz = (a[2] + b[2] + c[2]) / 3.0;
  const double ux = b[0] - a[0], uy = b[1] - a[1], uz = b[2] - a[2];
  const double vx = c[0] - a[0], vy = c[1] - a[1], vz = c[2] - a[2];
  double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
  const double len = sqrt(nx * nx + ny * ny + nz * nz);
  if (len > 0.0) {
    nx /= len;
    ny /= len;
    nz /= len;
  }
  cent[3 * f] = cx;
  cent[3 * f + 1] = cy;
  cent[3 * f + 2] = cz;
  nrm[3 * f] = nx;
  nrm[3 * f + 1] = ny;
  nrm[3 * f + 2] = nz;
  ids[f] = (uint32_t)f;
  uint32_t t = (uint32_t)fineCount;  // "no fine node" sorts after every node
  const int dx = (int)((cx - g.x) / w0), dy = (int)((cy - g.y) / w0), dz = (int)((cz - g.z) / w0);
  if (dx >= 0 && dy >= 0 && dz >= 0 && dx < res && dy < res && dz < res) {
    const uint32_t k = fineNodeOf(occ, occRank, mortonEncode((uint32_t)dx, (uint32_t)dy, (uint32_t)dz));
    if (k != kNone) t = k;
  }
  node[f] = t;
}

// Fine-node sums over the samples sorted by node (each node's run in sample order).
__global__ void kFineSums(const uint32_t* __restrict__ sortedNode, const uint32_t* __restrict__ sortedId,
                          int64_t nf, int64_t fineCount, const double* __restrict__ cent, const double* __restrict__ nrm,
                          NodeStats S) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const uint32_t t = sortedNode[i];
  if (t >= fineCount || (i > 0 && sortedNode[i - 1] == t)) return;  // first sample of the run only
  float c = 0.0f;
  double p[3] = {0, 0, 0}, q[3] = {0, 0, 0};
  for (int64_t k = i; k < nf && sortedNode[k] == t; ++k) {
    const uint32_t f = sortedId[k];
    c += 1.0f;
    for (int a = 0; a < 3; ++a) {
      p[a] += cent[3 * (int64_t)f + a];
      q[a] += nrm[3 * (int64_t)f + a];
    }
  }
  S.cnt[t] = c;
  for (int a = 0; a < 3; ++a) {
    S.sp[3 * (int64_t)t + a] = p[a];
    S.sn[3 * (int64_t)t + a] = q[a];
  }
}

// Nodes of one depth sum their 8 children (children 0..7 in order).
__global__ void kParentSums(int64_t begin, int64_t count, const uint32_t* __restrict__ child0, NodeStats S) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int64_t t = begin + i;
  const uint32_t c0 = child0[t];
  float c = 0.0f;
  double p[3] = {0, 0, 0}, q[3] = {0, 0, 0};
  if (c0 != kNone) {
    for (int k = 0; k < 8; ++k) {
      const int64_t ch = (int64_t)c0 + k;
      c += S.cnt[ch];
      for (int a = 0; a < 3; ++a) {
        p[a] += S.sp[3 * ch + a];
        q[a] += S.sn[3 * ch + a];
      }
    }
  }
  S.cnt[t] = c;
  for (int a = 0; a < 3; ++a) {
    S.sp[3 * t + a] = p[a];
    S.sn[3 * t + a] = q[a];
  }
}

struct FeatParams {
  int depth, res;
  double w0;
  LatticeIndex lat[kMaxDepth];
  int64_t vertStart[kMaxDepth + 1];
  const uint32_t* vertLin;
  const uint64_t* vertKey;
  const uint32_t* vertOwner;
  const double* vertPos;
  const uint32_t* nodeNb;
};

__device__ __forceinline__ int vertDepth(const FeatParams& P, int64_t v) {
  int d = 0;
  while (d + 1 < P.depth && P.vertStart[d + 1] <= v) ++d;
  return d;
}
__device__ __forceinline__ bool coincidentVertex(const FeatParams& P, int64_t v, int d) {
  if (d + 1 >= P.depth) return false;
  const uint32_t M = P.lat[d].M, lin = P.vertLin[v];
  return (((lin / (M * M)) | ((lin / M) % M) | (lin % M)) & 1u) == 0u;
}
// Vertex index of lattice point (X,Y,Z) at depth d, or -1.
__device__ __forceinline__ int64_t latticeVertex(const FeatParams& P, int d, int64_t X, int64_t Y, int64_t Z) {
  if (d < 0 || d >= P.depth) return -1;
  const LatticeIndex& L = P.lat[d];
  if (X < 0 || Y < 0 || Z < 0 || X >= L.M || Y >= L.M || Z >= L.M) return -1;
  const uint32_t lin = (uint32_t)((X * L.M + Y) * L.M + Z);
  return latticeHas(L, lin) ? (int64_t)latticeRank(L, lin) : -1;
}

// latticeVertex with both words (presence bits and rank) loaded up front, so that independent
// lookups issued together overlap their memory latency; -1 where no vertex is.
__device__ __forceinline__ int64_t latticeVertexIlp(const FeatParams& P, int d, int64_t X, int64_t Y, int64_t Z) {
  if (d < 0 || d >= P.depth) return -1;
  const LatticeIndex& L = P.lat[d];
  if (X < 0 || Y < 0 || Z < 0 || X >= L.M || Y >= L.M || Z >= L.M) return -1;
  const uint32_t lin = (uint32_t)((X * L.M + Y) * L.M + Z);
  const unsigned long long word = L.bits[lin >> 6];
  const uint32_t rank = L.rank[lin >> 6];
  if (!((word >> (lin & 63)) & 1ull)) return -1;
  return (int64_t)(L.base + rank + (uint32_t)__popcll(word & ((1ull << (lin & 63)) - 1ull)));
}

__global__ void kMarkCoincident(const __grid_constant__ FeatParams P, int64_t n, uint32_t* __restrict__ flag) {
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= n) return;
  flag[v] = coincidentVertex(P, v, vertDepth(P, v)) ? 1u : 0u;
}

// Feature normalisation (mean[64], scale[64]) passed by value with the launch.
struct FeatNorm {
  float v[2 * kFeat];
  int on;
};

constexpr int kFeatLanes = 4;                       // lanes per vertex
constexpr int kFeatThreads = 128;
constexpr int kFeatRows = kFeatThreads / kFeatLanes;  // vertices per block

// Four lanes per vertex: lane 0 the coincident copies above and the scalar features, lane 1
// the copies below, the face neighbours split over the lanes, lane 3 also the sample features
// of the owner's 27-neighbourhood (computed with the octree, kCoincGeom). The block's rows go
// through shared memory so that the normalised features leave in coalesced stores.
__global__ void __launch_bounds__(kFeatThreads) kShareFeatures(const __grid_constant__ FeatParams P,
                                                               const int64_t* __restrict__ ids, int64_t count,
                                                               const double* __restrict__ b,
                                                               const double* __restrict__ lam0,
                                                               const float* __restrict__ geom,
                                                               const __grid_constant__ FeatNorm norm,
                                                               float* __restrict__ out, __nv_bfloat16* __restrict__ tiles,
                                                               int64_t tileRow0) {
  gridDependencyWait();
  gridDependents();
  __shared__ __align__(16) float sf[kFeatRows][kFeat];
  const int sub = threadIdx.x & (kFeatLanes - 1), slot = threadIdx.x / kFeatLanes;
  const int64_t i0 = (int64_t)blockIdx.x * kFeatRows, i = i0 + slot;
  float* f = sf[slot];
#pragma unroll
  for (int k = 0; k < kFeat / kFeatLanes; ++k) f[sub * (kFeat / kFeatLanes) + k] = 0.0f;
  __syncwarp();
  const bool valid = i < count;
  int64_t v = 0;
  int d = 0;
  double w = 0.0;
  if (valid) {
    v = ids[i];
    const VertCoord vc = decodeVertKey(P.vertKey[v]);
    d = vc.d;
    const int64_t X = vc.X, Y = vc.Y, Z = vc.Z;
    w = P.w0 * (double)(1u << d);
    const double bv = b[v];
    if (sub == 0) {  // the coincident copies above
      // depth d + k holds a copy while the low k bits of X, Y and Z are all zero and every
      // depth in between has one: the candidates' lookups are independent, so they are issued
      // together and the chain is cut at the first missing copy afterwards
      const uint64_t xyz = (uint64_t)(X | Y | Z);
      const int even = xyz ? __ffsll((long long)xyz) - 1 : kMaxDepth;  // trailing zeros
      const int maxUp = min(even, P.depth - 1 - d);
      int64_t cand[kMaxDepth];
#pragma unroll
      for (int k = 1; k < kMaxDepth; ++k)
        cand[k] = k <= maxUp ? latticeVertexIlp(P, d + k, X >> k, Y >> k, Z >> k) : -1;
      int up = 0;
      int64_t top = v;
#pragma unroll
      for (int k = 1; k < kMaxDepth; ++k)
        if (up == k - 1 && cand[k] >= 0) {
          up = k;
          top = cand[k];
        }
      const double oneUp = up >= 1 ? lam0[cand[1]] : 0.0;
      f[0] = (float)bv;
      f[1] = (float)lam0[top];
      f[2] = (float)oneUp;
      f[3] = P.depth > 1 ? (float)d / (float)(P.depth - 1) : 0.0f;
      f[4] = (float)up / (float)P.depth;
      f[36] = (float)w;
      f[37] = (float)(bv / w);
    } else if (sub == 1) {  // the coincident copies below: independent lookups, then the chain
      bool has[kMaxDepth];
#pragma unroll
      for (int s = 1; s < kMaxDepth; ++s) has[s] = s <= d && latticeVertexIlp(P, d - s, X << s, Y << s, Z << s) >= 0;
      int down = 0;
#pragma unroll
      for (int s = 1; s < kMaxDepth; ++s)
        if (down == s - 1 && has[s]) down = s;
      f[5] = (float)down / (float)P.depth;
    }
    // face neighbours: lanes 0, 1 one each, lanes 2, 3 two each
    const int ex[6] = {1, -1, 0, 0, 0, 0}, ey[6] = {0, 0, 1, -1, 0, 0}, ez[6] = {0, 0, 0, 0, 1, -1};
    const int k0 = sub < 2 ? sub : 2 * sub - 2, k1 = sub < 2 ? sub + 1 : 2 * sub;
    for (int k = k0; k < k1; ++k) {
      const int64_t u = latticeVertex(P, d, X + ex[k], Y + ey[k], Z + ez[k]);
      if (u >= 0) {
        f[6 + k] = 1.0f;
        f[12 + k] = (float)(b[u] - bv);
        f[18 + k] = (float)lam0[u];
      }
      if (d > 0) {
        const int64_t qv = latticeVertex(P, d - 1, 2 * X + ex[k], 2 * Y + ey[k], 2 * Z + ez[k]);
        if (qv >= 0) {
          f[24 + k] = 1.0f;
          f[30 + k] = (float)lam0[qv];
        }
      }
    }
    // the samples around the owner (octree and mesh only): computed with the octree
    if (sub == 3) {
#pragma unroll
      for (int k = 0; k < 8; ++k) f[38 + k] = geom[8 * i + k];
    }
  }
  __syncthreads();
  const int64_t rows = count - i0 < kFeatRows ? count - i0 : kFeatRows;
  if (tiles) {
    // the network's input tiles: row R = tileRow0 + i of 128-row tile R / 128, 64 BF16 (128 B)
    // per row in 16-byte chunks at their 128-byte-swizzled places (umma::swizzledChunk)
    for (int e = threadIdx.x; e < rows * 8; e += kFeatThreads) {
      const int r = e >> 3, c = e & 7;
      const int64_t R = tileRow0 + i0 + r;
      __align__(16) __nv_bfloat16 q[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        float x = sf[r][8 * c + k];
        if (norm.on) x = (x - norm.v[8 * c + k]) * norm.v[kFeat + 8 * c + k];
        q[k] = __float2bfloat16_rn(x);
      }
      *(uint4*)((uint8_t*)tiles + (R >> 7) * 16384 + umma::swizzledChunk((uint32_t)(R & 127), (uint32_t)c)) =
          *(const uint4*)q;
    }
    return;
  }
  // the block's rows are consecutive in out: float4 stores over all of them
  for (int e = threadIdx.x; e < rows * (kFeat / 4); e += kFeatThreads) {
    const int r = e / (kFeat / 4), k = 4 * (e % (kFeat / 4));
    float4 x = *(const float4*)&sf[r][k];
    if (norm.on) {
      x.x = (x.x - norm.v[k]) * norm.v[kFeat + k];
      x.y = (x.y - norm.v[k + 1]) * norm.v[kFeat + k + 1];
      x.z = (x.z - norm.v[k + 2]) * norm.v[kFeat + k + 2];
      x.w = (x.w - norm.v[k + 3]) * norm.v[kFeat + k + 3];
    }
    float* dst = out + (i0 + r) * kFeat + k;
    if (((uintptr_t)out & 15) == 0) {
      *(float4*)dst = x;
    } else {
      dst[0] = x.x;
      dst[1] = x.y;
      dst[2] = x.z;
      dst[3] = x.w;
    }
  }
}

// Learned shares of the coincident vertices: share[ids[i]] = pred[i] * scale + mean.
__global__ void kScatterShares(const int64_t* __restrict__ ids, int64_t count, const float* __restrict__ pred,
                               float scale, float mean, double* __restrict__ shares) {
  gridDependencyWait();
  gridDependents();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  shares[ids[i]] = (double)pred[i] * (double)scale + (double)mean;
}

static FeatParams featParams(const SvoDevice& d) {
  FeatParams P;
  P.depth = d.depth;
  P.res = d.res;
  P.w0 = d.unit[0];
  for (int L = 0; L < kMaxDepth; ++L) P.lat[L] = L < d.depth ? d.lattice(L) : LatticeIndex{};
  for (int L = 0; L <= kMaxDepth; ++L) P.vertStart[L] = L <= d.depth ? d.vertStart[L] : d.numVerts;
  P.vertLin = d.vertLin;
  P.vertKey = d.vertKey;
  P.vertOwner = d.vertOwner;
  P.vertPos = d.vertPos;
  P.nodeNb = d.nodeNb;
  return P;
}

// Coincident vertices (ascending) into ids (capacity n); *count their number.
its_status coincidentIds(its_ctx* ctx, const SvoDevice& d, int64_t* ids, int64_t* count) {
  const int64_t n = d.numVerts;
  its_status st;
  DevBuf<uint32_t> flag;
  DevBuf<int64_t> tot;
  if ((st = flag.alloc(ctx, n)) != ITS_OK || (st = tot.alloc(ctx, 1)) != ITS_OK) return st;
  const FeatParams P = featParams(d);
  kMarkCoincident<<<gridFor(n, 256), 256, 0, ctx->stream>>>(P, n, flag.p);
  ITS_LAUNCHED(ctx);
  const uint32_t* fl = flag.p;
  auto fv = [fl] __device__(int64_t i) -> int64_t { return (int64_t)fl[i]; };
  auto wr = [fl, ids] __device__(int64_t i, int64_t prefix, int64_t) {
    if (fl[i]) ids[prefix] = i;
  };
  if ((st = scanExclusiveAlloc<int64_t>(ctx, fv, n, wr, tot.p)) != ITS_OK) return st;
  return readScalar(ctx, tot.p, count);
}

// Features 38-45 of coincident vertex i (one thread each): the samples of the 27 nodes around
// its owner, summed in neighbour order.
__global__ void kCoincGeom(const __grid_constant__ FeatParams P, const int64_t* __restrict__ ids, int64_t count,
                           NodeStats S, float* __restrict__ geom) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int64_t v = ids[i];
  const VertCoord vc = decodeVertKey(P.vertKey[v]);
  const double w = P.w0 * (double)(1u << vc.d);
  const uint32_t o = P.vertOwner[v];
  double c = 0.0, p[3] = {0, 0, 0}, q[3] = {0, 0, 0};
  for (int k = 0; k < 27; ++k) {
    const uint32_t t = P.nodeNb[27 * (int64_t)o + k];
    if (t == kNone) continue;
    c += (double)S.cnt[t];
    for (int a = 0; a < 3; ++a) {
      p[a] += S.sp[3 * (int64_t)t + a];
      q[a] += S.sn[3 * (int64_t)t + a];
    }
  }
  float f[8] = {(float)log1p(c), 0, 0, 0, 0, 0, 0, 0};
  if (c > 0.0) {
    const double* x = P.vertPos + 3 * v;
    double nn = 0.0;
    for (int a = 0; a < 3; ++a) {
      f[1 + a] = (float)((p[a] / c - x[a]) / w);
      const double m = q[a] / c;
      f[4 + a] = (float)m;
      nn += m * m;
    }
    f[7] = (float)(1.0 - sqrt(nn));
  }
  for (int k = 0; k < 8; ++k) geom[8 * i + k] = f[k];
}

its_status coincidentGeometry(its_ctx* ctx, SvoDevice& d) {
  its_status st;
  if ((st = devAlloc(ctx, (void**)&d.coincGeom, std::max<int64_t>(d.numCoinc, 1) * 8 * sizeof(float))) != ITS_OK)
    return st;
  if (d.numCoinc > 0) {
    NodeStats S{d.nodeSampleCnt, d.nodeSamplePos, d.nodeSampleNrm};
    kCoincGeom<<<gridFor(d.numCoinc, 128), 128, 0, ctx->stream>>>(featParams(d), d.coincIds, d.numCoinc, S,
                                                                  d.coincGeom);
    ITS_LAUNCHED(ctx);
  }
  return ITS_OK;
}

its_status nodeSampleStats(its_ctx* ctx, SvoDevice& d, const double* V, const int32_t* F, int64_t nf) {
  its_status st;
  const int64_t nn = d.numNodes;
  if ((st = devAlloc(ctx, (void**)&d.nodeSampleCnt, std::max<int64_t>(nn, 1) * 4)) != ITS_OK ||
      (st = devAlloc(ctx, (void**)&d.nodeSamplePos, std::max<int64_t>(nn, 1) * 24)) != ITS_OK ||
      (st = devAlloc(ctx, (void**)&d.nodeSampleNrm, std::max<int64_t>(nn, 1) * 24)) != ITS_OK)
    return st;
  ITS_CU(ctx, cudaMemsetAsync(d.nodeSampleCnt, 0, nn * 4, ctx->stream));
  ITS_CU(ctx, cudaMemsetAsync(d.nodeSamplePos, 0, nn * 24, ctx->stream));
  ITS_CU(ctx, cudaMemsetAsync(d.nodeSampleNrm, 0, nn * 24, ctx->stream));
  if (nf <= 0 || nn <= 0) return ITS_OK;
  DevBuf<double> cent, nrm;
  DevBuf<uint32_t> node, fid, sNode, sId, tk, tv;
  if ((st = cent.alloc(ctx, 3 * nf)) != ITS_OK || (st = nrm.alloc(ctx, 3 * nf)) != ITS_OK ||
      (st = node.alloc(ctx, nf)) != ITS_OK || (st = fid.alloc(ctx, nf)) != ITS_OK ||
      (st = sNode.alloc(ctx, nf)) != ITS_OK || (st = sId.alloc(ctx, nf)) != ITS_OK ||
      (st = tk.alloc(ctx, nf)) != ITS_OK || (st = tv.alloc(ctx, nf)) != ITS_OK)
    return st;
  const int64_t fineCount = d.levelCount[0];
  kFaceSamples<<<gridFor(nf, 256), 256, 0, ctx->stream>>>(V, F, nf, make_double3(d.origin[0], d.origin[1], d.origin[2]),
                                                         d.unit[0], d.res, (const unsigned long long*)d.fineOcc,
                                                         d.fineRank, fineCount, cent.p, nrm.p,
                                                         node.p, fid.p);
  ITS_LAUNCHED(ctx);
  // stable sort by fine node ("none" = fineCount sorts last)
  int bits = 1;
  while (bits < 32 && (1ll << bits) <= fineCount) ++bits;
  if ((st = radixSortPairs(ctx, node.p, fid.p, sNode.p, sId.p, tk.p, tv.p, nf, bits)) != ITS_OK) return st;
  NodeStats S{d.nodeSampleCnt, d.nodeSamplePos, d.nodeSampleNrm};
  kFineSums<<<gridFor(nf, 256), 256, 0, ctx->stream>>>(sNode.p, sId.p, nf, fineCount, cent.p, nrm.p, S);
  ITS_LAUNCHED(ctx);
  for (int L = 1; L < d.depth; ++L) {
    if (!d.levelCount[L]) continue;
    kParentSums<<<gridFor(d.levelCount[L], 256), 256, 0, ctx->stream>>>(d.levelStart[L], d.levelCount[L],
                                                                        d.nodeChild0, S);
    ITS_LAUNCHED(ctx);
  }
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));  // the sample scratch is freed on return
  return ITS_OK;
}

// Features of the octree's coincident vertices (ids = d.coincIds, count = d.numCoinc: row i
// is coincident vertex i) (see the file comment); hostNorm (host memory, may be null) the
// normalisation.
its_status shareFeatures(its_ctx* ctx, const SvoDevice& d, const double* b, const double* lam0, const int64_t* ids,
                         int64_t count, const float* hostNorm, float* out, bool afterKernel, __nv_bfloat16* tiles,
                         int64_t tileRow0) {
  const FeatParams P = featParams(d);
  FeatNorm norm;
  norm.on = hostNorm != nullptr;
  for (int k = 0; k < 2 * kFeat; ++k) norm.v[k] = hostNorm ? hostNorm[k] : 0.0f;
  if (count > 0) {
    its_status st = launchDependent(ctx, afterKernel, kShareFeatures, gridFor(count, kFeatRows), kFeatThreads, 0, ctx->stream, P, ids,
                                    count, b, lam0, (const float*)d.coincGeom, norm, out, tiles, tileRow0);
    if (st != ITS_OK) return st;
  }
  return ITS_OK;
}

// Learned shares of the coincident vertices (the exact start reads shares nowhere else).
its_status scatterShares(its_ctx* ctx, const int64_t* ids, int64_t count, const float* pred, float scale, float mean,
                         double* shares) {
  if (count > 0) {
    its_status st = launchDependent(ctx, true, kScatterShares, gridFor(count, 256), 256, 0, ctx->stream, ids, count, pred, scale,
                                    mean, shares);
    if (st != ITS_OK) return st;
  }
  return ITS_OK;
}

}  // namespace its

namespace its {
its_status exactStart(its_ctx* ctx, its_svo* const* svos, int64_t count, const double* const* b,
                      const double* const* shares, double* const* lam, bool afterKernel, double* gScratch,
                      unsigned long long* stamp);
}

using namespace its;

namespace its {
its_status mlpInfer(its_mlp* mlp, const float* X, int64_t n, float* out, bool afterKernel);
its_status mlpInferTiles(its_mlp* h, const __nv_bfloat16* tiles, int64_t n, float* out, const int64_t* ids,
                         float scale, float mean, double* shares, bool afterKernel);
its_status mlpCheck(its_mlp* mlp);
}  // namespace its

namespace its {

// The 130 normalisation values in host memory (norm may be host or device memory).
its_status hostNorm(its_ctx* ctx, const float* norm, float* hn) {
  const MemKind k = memKind(norm, ctx->device);
  if (k == MemKind::OtherDevice) return otherDeviceError(ctx);
  if (k == MemKind::Device) {
    ITS_CU(ctx, cudaMemcpyAsync(hn, norm, (2 * kFeat + 2) * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  } else {
    std::memcpy(hn, norm, (2 * kFeat + 2) * sizeof(float));
  }
  return ITS_OK;
}

// Learned starts of count octrees, device vectors, everything queued on the context's stream
// without a host wait or a copy from host memory (norm hn is passed with the launches): the
// zero-share starts (feature inputs), the features of every mesh into one array, one network
// pass, the shares, the exact starts with them.
its_status learnedStart(its_ctx* ctx, its_svo* const* svos, int64_t count, its_mlp* mlp, const double* const* b,
                        const float* hn, double* const* lam, unsigned long long* stamp) {
  its_status st;
  std::vector<DevBuf<double>> lam0(count), shares(count);
  std::vector<const double*> sp(count);
  std::vector<double*> l0(count);
  std::vector<int64_t> cnt(count);
  int64_t total = 0, verts = 0;
  for (int64_t m = 0; m < count; ++m) {
    const int64_t n = svos[m]->d.numVerts;
    if ((st = lam0[m].alloc(ctx, n)) != ITS_OK || (st = shares[m].alloc(ctx, n)) != ITS_OK) return st;
    l0[m] = lam0[m].p;
    sp[m] = shares[m].p;
    cnt[m] = svos[m]->d.numCoinc;
    total += cnt[m];
    verts += n;
  }
  // every buffer up front: from the first kernel on, each launch follows a kernel (dependent
  // launches, gridDependencyWait at the top of each kernel)
  // the features go straight into the network's BF16 input tiles (128 rows x 128 B each)
  DevBuf<__nv_bfloat16> feat;
  DevBuf<float> pred;
  DevBuf<double> G;
  if ((st = feat.alloc(ctx, std::max<int64_t>((total + 127) / 128, 1) * 128 * kFeat)) != ITS_OK ||
      (st = pred.alloc(ctx, std::max<int64_t>(total, 1))) != ITS_OK ||
      (st = G.alloc(ctx, std::max<int64_t>(verts, 1))) != ITS_OK)
    return st;
  if ((st = exactStart(ctx, svos, count, b, nullptr, l0.data(), false, nullptr, stamp)) != ITS_OK) return st;
  int64_t off = 0;
  for (int64_t m = 0; m < count; ++m) {
    if ((st = shareFeatures(ctx, svos[m]->d, b[m], l0[m], svos[m]->d.coincIds, cnt[m], hn, nullptr, true, feat.p,
                            off)) != ITS_OK)
      return st;
    off += cnt[m];
  }
  if (count == 1) {  // one octree: the network writes the shares itself
    if (total > 0 && (st = mlpInferTiles(mlp, feat.p, total, nullptr, svos[0]->d.coincIds, hn[2 * kFeat + 1],
                                         hn[2 * kFeat], shares[0].p, true)) != ITS_OK)
      return st;
  } else {
    if (total > 0 &&
        (st = mlpInferTiles(mlp, feat.p, total, pred.p, nullptr, 0.0f, 0.0f, nullptr, true)) != ITS_OK)
      return st;
    off = 0;
    for (int64_t m = 0; m < count; ++m) {
      if ((st = scatterShares(ctx, svos[m]->d.coincIds, cnt[m], pred.p + off, hn[2 * kFeat + 1], hn[2 * kFeat],
                              shares[m].p)) != ITS_OK)
        return st;
      off += cnt[m];
    }
  }
  return exactStart(ctx, svos, count, b, sp.data(), lam, total > 0, G.p, nullptr);
}

}  // namespace its

extern "C" {

its_status its_share_features(its_svo* svo, const double* b, const float* norm, float* features, int64_t capacity,
                              int64_t* ids, int64_t* count) {
  if (!svo || !b || !count) return ITS_ERR_INVALID;
  its_ctx* ctx = svo->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  const SvoDevice& d = svo->d;
  const int64_t n = d.numVerts;
  its_status st;
  InArg<double> db;
  if ((st = db.stage(ctx, b, n)) != ITS_OK) return st;
  float hn[2 * kFeat];
  if (norm && memKind(norm, ctx->device) == MemKind::OtherDevice) return otherDeviceError(ctx);
  if (norm && isDevicePtr(ctx, norm)) {
    ITS_CU(ctx, cudaMemcpyAsync(hn, norm, sizeof(hn), cudaMemcpyDeviceToHost, ctx->stream));
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  } else if (norm) {
    std::memcpy(hn, norm, sizeof(hn));
  }
  const int64_t cnt = d.numCoinc;
  const int64_t* dIds = d.coincIds;
  *count = cnt;
  if (!features) return ITS_OK;
  if (capacity < cnt) return setError(ctx, ITS_ERR_INVALID, "its_share_features: capacity below the count");
  DevBuf<double> lam0;
  if ((st = lam0.alloc(ctx, n)) != ITS_OK) return st;
  const double* bp = db.d;
  double* lp = lam0.p;
  if ((st = exactStart(ctx, &svo, 1, &bp, nullptr, &lp, false, nullptr, nullptr)) != ITS_OK) return st;
  OutArg<float> out;
  if ((st = out.stage(ctx, features, cnt * kFeat)) != ITS_OK) return st;
  if ((st = shareFeatures(ctx, d, db.d, lam0.p, dIds, cnt, norm ? hn : nullptr, out.d, false, nullptr, 0)) != ITS_OK)
    return st;
  if ((st = out.finish(ctx)) != ITS_OK) return st;
  if (ids) ITS_CU(ctx, cudaMemcpyAsync(ids, dIds, cnt * 8, cudaMemcpyDefault, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_learned_start_batch(its_svo* const* svos, int64_t count, its_mlp* mlp, const double* const* b,
                                   const float* norm, double* const* lambda) {
  if (!svos || count <= 0 || !mlp || !b || !norm || !lambda) return ITS_ERR_INVALID;
  its_ctx* ctx = svos[0] ? svos[0]->ctx : nullptr;
  if (!ctx) return ITS_ERR_INVALID;
  for (int64_t m = 0; m < count; ++m)
    if (!svos[m] || svos[m]->ctx != ctx || !b[m] || !lambda[m])
      return setError(ctx, ITS_ERR_INVALID, "its_learned_start: bad octree or vector");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  its_status st;
  float hn[2 * kFeat + 2];
  if ((st = hostNorm(ctx, norm, hn)) != ITS_OK) return st;
  std::vector<InArg<double>> B(count);
  std::vector<OutArg<double>> L(count);
  std::vector<const double*> bp(count);
  std::vector<double*> lp(count);
  for (int64_t m = 0; m < count; ++m) {
    const int64_t n = svos[m]->d.numVerts;
    if ((st = B[m].stage(ctx, b[m], n)) != ITS_OK || (st = L[m].stage(ctx, lambda[m], n)) != ITS_OK) return st;
    bp[m] = B[m].d;
    lp[m] = L[m].d;
  }
  if ((st = learnedStart(ctx, svos, count, mlp, bp.data(), hn, lp.data(), nullptr)) != ITS_OK) return st;
  bool host = false;
  for (int64_t m = 0; m < count; ++m) {
    host = host || L[m].host;
    if ((st = L[m].finish(ctx)) != ITS_OK) return st;
  }
  // device outputs: ordered on the context's stream (a tensor-core wait that ran out shows at
  // the network's next checked call); host outputs: complete on return, network checked
  if (host) return mlpCheck(mlp);
  return ITS_OK;
}

its_status its_learned_start(its_svo* svo, its_mlp* mlp, const double* b, const float* norm, double* lambda) {
  return its_learned_start_batch(&svo, 1, mlp, &b, norm, &lambda);
}

}  // extern "C"
