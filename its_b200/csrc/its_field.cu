#include <cmath>
// Field evaluation and marching cubes.
//
// * Points (ThinShells::cpLatentBSplineValue, ThinShells.cpp:655-755): a point's fine node
//   is found by binary search of its voxel's Morton code in the sorted depth-0 node list;
//   the field is sum(lambda * hat) over the 8 corners of that node and of every ancestor,
//   corners in order k = x|y<<1|z<<2, ancestors from fine to coarse (the reference's order).
// * Lattice (the MC input of MarchingCubes.cu:464-536 / CUDACompute.cu:435-510): the
//   reference sums lambda_j * hat_j over ALL n corner vertices for 8 duplicated corners per
//   voxel, O(8 R^3 n). Only the 8 corners of the depth-d cell holding p can be non-zero, so
//   each lattice point of the (R+1)^3 grid is evaluated once from at most 8 corners per depth,
//   their existence and column read from the per-depth lattice bitmaps: O(8 D) per point.
// * Marching cubes (MarchingCubes.cu:164-377): case index with bit i = f(corner i) < iso in
//   the reference's corner order, vertex counts from the case table, an exclusive scan of the
//   counts, and the triangle soup written in voxel order by the scan's own downsweep (no
//   compaction pass, no 18 R^3 preallocation).
#include <algorithm>
#include <cfloat>
#include <vector>

#include "its_mc.cuh"
#include "its_tune.cuh"
#include "its_op.cuh"

namespace its {

struct EvalParams {
  int depth, res;
  double3 g;
  double w0;
  LatticeIndex lat[kMaxDepth];
  int64_t fineCount;
  const uint32_t* morton;
  const uint32_t* parent;
  const double* vertPos;
  const uint64_t* vertKey;  // packed lattice coordinates and the vertex's corner of its owner
  const unsigned long long* fineOcc;  // depth-0 nodes: Morton bitset and its word ranks
  const uint32_t* fineRank;
  double winv[kMaxDepth];  // RN(1 / w_d), for divRn
};

static EvalParams evalParams(const SvoDevice& d) {
  EvalParams P;
  P.depth = d.depth;
  P.res = d.res;
  P.g = make_double3(d.origin[0], d.origin[1], d.origin[2]);
  P.w0 = d.unit[0];
  for (int L = 0; L < kMaxDepth; ++L) P.lat[L] = L < d.depth ? d.lattice(L) : LatticeIndex{};
  P.fineCount = d.levelCount[0];
  P.morton = d.nodeMorton;
  P.parent = d.nodeParent;
  P.vertPos = d.vertPos;
  P.vertKey = d.vertKey;
  P.fineOcc = (const unsigned long long*)d.fineOcc;
  P.fineRank = d.fineRank;
  for (int L = 0; L < kMaxDepth; ++L) P.winv[L] = 1.0 / (P.w0 * (double)(1u << L));
  return P;
}

// Chain evaluation of one point; returns false when no fine node holds it.
__device__ inline bool evalChain(const EvalParams& P, const double* __restrict__ lambda, double px, double py,
                                 double pz, double& out) {
  const int dx = (int)((px - P.g.x) / P.w0), dy = (int)((py - P.g.y) / P.w0), dz = (int)((pz - P.g.z) / P.w0);
  if (dx < 0 || dy < 0 || dz < 0 || dx >= P.res || dy >= P.res || dz >= P.res) return false;
  uint32_t t = fineNodeOf(P.fineOcc, P.fineRank, mortonEncode((uint32_t)dx, (uint32_t)dy, (uint32_t)dz));
  if (t == kNone) return false;
  double sum = 0.0;
  for (int d = 0; d < P.depth && t != kNone; ++d) {
    uint32_t X, Y, Z;
    mortonDecode(P.morton[t], X, Y, Z);
    const double w = P.w0 * (double)(1u << d), wi = P.winv[d];
    const double bx = latticePos(P.g.x, w, X), by = latticePos(P.g.y, w, Y), bz = latticePos(P.g.z, w, Z);
    const LatticeIndex& L = P.lat[d];
    // hat3's three factors for the cell's two corner positions per axis (the 8 corners share
    // them); each term is hat3's value: 0 once a factor is not positive, else x * y * z
    const double fx[2] = {hat1r(px, bx, w, wi), hat1r(px, bx + w, w, wi)};
    const double fy[2] = {hat1r(py, by, w, wi), hat1r(py, by + w, w, wi)};
    const double fz[2] = {hat1r(pz, bz, w, wi), hat1r(pz, bz + w, w, wi)};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
      const uint32_t col = latticeRank(L, ((X + ox) * L.M + (Y + oy)) * L.M + (Z + oz));
      const double h = (fx[ox] <= 0.0 || fy[oy] <= 0.0 || fz[oz] <= 0.0) ? 0.0 : fx[ox] * fy[oy] * fz[oz];
      sum += lambda[col] * h;
    }
    t = P.parent[t];
  }
  out = sum;
  return true;
}

__global__ void kEvalPoints(const __grid_constant__ EvalParams P, const double* __restrict__ lambda,
                            const double* __restrict__ pts, int64_t m, double* __restrict__ out,
                            uint8_t* __restrict__ missing) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  double v = 0.0;
  const bool ok = evalChain(P, lambda, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], v);
  out[i] = ok ? v : 0.0;
  if (missing) missing[i] = ok ? 0 : 1;
}

// min / max over the found points, count of missing ones; one partial per block.
__global__ void kIsoPartials(const __grid_constant__ EvalParams P, const double* __restrict__ lambda,
                             const double* __restrict__ pts, int64_t m, double* __restrict__ pmin,
                             double* __restrict__ pmax, unsigned long long* __restrict__ pmiss) {
  double lo = DBL_MAX, hi = -DBL_MAX;
  unsigned long long miss = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    double v;
    if (evalChain(P, lambda, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], v)) {
      lo = fmin(lo, v);
      hi = fmax(hi, v);
    } else {
      ++miss;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, o));
    miss += __shfl_down_sync(0xffffffffu, miss, o);
  }
  __shared__ double slo[8], shi[8];
  __shared__ unsigned long long smiss[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { slo[w] = lo; shi[w] = hi; smiss[w] = miss; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
      lo = fmin(lo, slo[k]);
      hi = fmax(hi, shi[k]);
      miss += smiss[k];
    }
    pmin[blockIdx.x] = lo;
    pmax[blockIdx.x] = hi;
    pmiss[blockIdx.x] = miss;
  }
}

// The field at any point: sum over every corner vertex of lambda * hat, restricted to the
// only terms that can be non-zero -- at each depth the 8 corners of the cell holding p that
// exist as vertices of that depth -- summed depth 0..D-1, corners k = x|y<<1|z<<2.
__device__ inline double fieldAt(const EvalParams& P, const double* __restrict__ lambda, double px, double py,
                                 double pz) {
  double sum = 0.0;
  for (int d = 0; d < P.depth; ++d) {
    const double w = P.w0 * (double)(1u << d), wi = P.winv[d];
    const LatticeIndex& L = P.lat[d];
    const int64_t lim = (int64_t)(P.res >> d);
    const int64_t cx = (int64_t)floor(divRn(px - P.g.x, w, wi)), cy = (int64_t)floor(divRn(py - P.g.y, w, wi)),
                  cz = (int64_t)floor(divRn(pz - P.g.z, w, wi));
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int64_t Lx = cx + (k & 1), Ly = cy + ((k >> 1) & 1), Lz = cz + ((k >> 2) & 1);
      if (Lx < 0 || Ly < 0 || Lz < 0 || Lx > lim || Ly > lim || Lz > lim) continue;
      const uint32_t lin = (uint32_t)((Lx * L.M + Ly) * L.M + Lz);
      if (!latticeHas(L, lin)) continue;
      const uint32_t v = latticeRank(L, lin);
      sum += lambda[v] * hat3r(P.vertPos[3 * v], P.vertPos[3 * v + 1], P.vertPos[3 * v + 2], w, wi, px, py, pz);
    }
  }
  return sum;
}

// Field on the (R+1)^3 lattice in bricks of 32 x 4 x 2 points (one per thread). For each
// depth the brick's points fall in a small box of cells; the corners of that box (presence,
// coefficient, representative position) are staged in shared memory once, and every point
// then sums its 8 corners from there -- the same additions in the same order as fieldAt, so
// the result is bit-identical, without the per-point lattice lookups (bitmap, rank, vertex
// position) that made the point-wise kernel L2-bound. Depths whose corner box exceeds the
// tile (grids much coarser than the octree) fall back to the point-wise lookups.
constexpr int kBrickThreads = 256, kTileCap = 640;

// Field on the (R+1)^3 lattice in bricks of 32 x 4 x 8 points; a thread evaluates a column of
// 4 points along z. For each depth the brick's points fall in a small box of cells; the
// corners of that box (presence, coefficient, representative position) are staged in shared
// memory once, and every point then sums its 8 corners from there -- the same additions in
// the same order as fieldAt, so the result is bit-identical, without per-point lattice
// lookups. The x and y hat factors of a corner are shared by the thread's 4 points (equal
// inputs, equal IEEE results); all quotients use divRn. Depths whose corner box has no
// corner are skipped; depths whose box exceeds the tile (grids much coarser than the octree)
// fall back to per-point lookups.
template <typename T>
__device__ __forceinline__ T quotT(T a, T w, T wi) {
  if constexpr (sizeof(T) == 8) return divRn(a, w, wi);
  else return a * wi;
}
template <typename T>
__device__ __forceinline__ T hatT(T x, T p, T w, T wi) {
  if constexpr (sizeof(T) == 8) {
    return hat1r(x, p, w, wi);
  } else {
    if (x <= p - w || x >= p + w) return T(0);
    return x <= p ? T(1) + (x - p) * wi : T(1) - (x - p) * wi;
  }
}

template <typename T, int kBrickX, int kBrickY, int kZPer>
__global__ void __launch_bounds__(kBrickThreads, 2)
    kEvalGridBricks(const __grid_constant__ EvalParams P, const double* __restrict__ lambda, double3 o, double3 vs,
                    int R, T* __restrict__ field) {
  constexpr int kBrickZ = (kBrickThreads / (kBrickX * kBrickY)) * kZPer;
  __shared__ T tLam[kTileCap], tPx[kTileCap], tPy[kTileCap], tPz[kTileCap];
  __shared__ unsigned char tHas[kTileCap];
  __shared__ int64_t box[6];  // first and last cell per axis at the current depth
  const int64_t M = (int64_t)R + 1;
  const int tid = threadIdx.x;
  const int64_t x0 = (int64_t)blockIdx.x * kBrickX, y0 = (int64_t)blockIdx.y * kBrickY,
                z0 = (int64_t)blockIdx.z * kBrickZ;
  const int64_t xi = x0 + (tid % kBrickX), yj = y0 + ((tid / kBrickX) % kBrickY);
  const int64_t zb = z0 + (int64_t)(tid / (kBrickX * kBrickY)) * kZPer;
  const bool inXY = xi < M && yj < M;
  const T px = (T)(o.x + (double)xi * vs.x), py = (T)(o.y + (double)yj * vs.y);
  const T gx = (T)P.g.x, gy = (T)P.g.y, gz = (T)P.g.z;
  T pz[kZPer], sum[kZPer];
#pragma unroll
  for (int q = 0; q < kZPer; ++q) {
    pz[q] = (T)(o.z + (double)(zb + q) * vs.z);
    sum[q] = T(0);
  }
  for (int d = 0; d < P.depth; ++d) {
    const double wd = P.w0 * (double)(1u << d), wid = P.winv[d];
    const T w = (T)wd, wi = (T)wid;
    const LatticeIndex& L = P.lat[d];
    const int64_t lim = (int64_t)(P.res >> d);
    if (tid < 6) {
      const int a = tid >> 1;
      const int64_t idx = (a == 0 ? x0 : a == 1 ? y0 : z0) +
                          ((tid & 1) ? (a == 0 ? kBrickX : a == 1 ? kBrickY : kBrickZ) - 1 : 0);
      const int64_t cl = idx < M ? idx : M - 1;
      const double oa = a == 0 ? o.x : a == 1 ? o.y : o.z, va = a == 0 ? vs.x : a == 1 ? vs.y : vs.z;
      const double ga = a == 0 ? P.g.x : a == 1 ? P.g.y : P.g.z;
      const double pa = oa + (double)cl * va;
      box[tid] = sizeof(T) == 8 ? (int64_t)floor(divRn(pa - ga, wd, wid))
                                : (int64_t)floorf(quotT<T>((T)pa - (T)ga, w, wi));
    }
    __syncthreads();
    const int64_t cx0 = box[0], cy0 = box[2], cz0 = box[4];
    const int nx = (int)(box[1] - cx0 + 2), ny = (int)(box[3] - cy0 + 2), nz = (int)(box[5] - cz0 + 2);
    const bool tiled = (int64_t)nx * ny * nz <= kTileCap;  // block-uniform
    int any = 1;
    if (tiled) {
      int mine = 0;
      for (int t = tid; t < nx * ny * nz; t += kBrickThreads) {
        const int64_t Lx = cx0 + t / (ny * nz), Ly = cy0 + (t / nz) % ny, Lz = cz0 + t % nz;
        unsigned char has = 0;
        if (Lx >= 0 && Ly >= 0 && Lz >= 0 && Lx <= lim && Ly <= lim && Lz <= lim) {
          const uint32_t lin = (uint32_t)((Lx * L.M + Ly) * L.M + Lz);
          if (latticeHas(L, lin)) {
            const uint32_t v = latticeRank(L, lin);
            const double qx = P.vertPos[3 * v], qy = P.vertPos[3 * v + 1], qz = P.vertPos[3 * v + 2];
            tLam[t] = (T)lambda[v];
            tPx[t] = (T)qx;
            tPy[t] = (T)qy;
            tPz[t] = (T)qz;
            // bit 0: present; bits 1-3: the x / y / z coordinate is the lattice coordinate
            // g + w X, so the column's shared factor for that axis applies (FP32: always)
            has = (unsigned char)(1 | ((sizeof(T) == 4 || qx == latticePos(P.g.x, wd, (uint32_t)Lx)) ? 2 : 0) |
                                  ((sizeof(T) == 4 || qy == latticePos(P.g.y, wd, (uint32_t)Ly)) ? 4 : 0) |
                                  ((sizeof(T) == 4 || qz == latticePos(P.g.z, wd, (uint32_t)Lz)) ? 8 : 0));
          }
        }
        tHas[t] = has;
        mine |= has;
      }
      any = __syncthreads_or(mine);
    } else {
      __syncthreads();
    }
    if (any && inXY) {
      const int64_t cx = (int64_t)floor(quotT<T>(px - gx, w, wi)), cy = (int64_t)floor(quotT<T>(py - gy, w, wi));
      // the lattice factors of this column's cell: x and y shared by its 4 points
      const T fx[2] = {hatT<T>(px, (T)latticePos(P.g.x, wd, (uint32_t)cx), w, wi),
                       hatT<T>(px, (T)latticePos(P.g.x, wd, (uint32_t)(cx + 1)), w, wi)};
      const T fy[2] = {hatT<T>(py, (T)latticePos(P.g.y, wd, (uint32_t)cy), w, wi),
                       hatT<T>(py, (T)latticePos(P.g.y, wd, (uint32_t)(cy + 1)), w, wi)};
#pragma unroll
      for (int q = 0; q < kZPer; ++q) {
        if (zb + q >= M) break;
        const T pzq = pz[q];
        const int64_t cz = (int64_t)floor(quotT<T>(pzq - gz, w, wi));
        const T fz[2] = {hatT<T>(pzq, (T)latticePos(P.g.z, wd, (uint32_t)cz), w, wi),
                         hatT<T>(pzq, (T)latticePos(P.g.z, wd, (uint32_t)(cz + 1)), w, wi)};
        T s = sum[q];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
          T lam;
          unsigned f;
          int t = 0;
          uint32_t vv = 0;
          if (tiled) {
            t = ((int)(cx - cx0) + ox) * ny * nz + ((int)(cy - cy0) + oy) * nz + ((int)(cz - cz0) + oz);
            f = tHas[t];
            if (!f) continue;
            lam = tLam[t];
          } else {
            const int64_t Lx = cx + ox, Ly = cy + oy, Lz = cz + oz;
            if (Lx < 0 || Ly < 0 || Lz < 0 || Lx > lim || Ly > lim || Lz > lim) continue;
            const uint32_t lin = (uint32_t)((Lx * L.M + Ly) * L.M + Lz);
            if (!latticeHas(L, lin)) continue;
            vv = latticeRank(L, lin);
            lam = (T)lambda[vv];
            f = sizeof(T) == 4 ? 15u : 1u;  // FP64: positions from the vertex array
          }
          // hat3 as the reference forms it: x, y, z factors with early exits; a factor at the
          // lattice coordinate is the column's shared one (equal inputs, equal IEEE result)
          T hx, hy, hz;
          if (f & 2) hx = fx[ox];
          else hx = hatT<T>(px, tiled ? tPx[t] : (T)P.vertPos[3 * (int64_t)vv], w, wi);
          if (hx <= T(0)) continue;
          if (f & 4) hy = fy[oy];
          else hy = hatT<T>(py, tiled ? tPy[t] : (T)P.vertPos[3 * (int64_t)vv + 1], w, wi);
          if (hy <= T(0)) continue;
          if (f & 8) hz = fz[oz];
          else hz = hatT<T>(pzq, tiled ? tPz[t] : (T)P.vertPos[3 * (int64_t)vv + 2], w, wi);
          if (hz <= T(0)) continue;
          s += lam * (hx * hy * hz);
        }
        sum[q] = s;
      }
    }
    __syncthreads();
  }
  if (inXY) {
#pragma unroll
    for (int q = 0; q < kZPer; ++q)
      if (zb + q < M) field[xi + M * (yj + M * (zb + q))] = sum[q];
  }
}

// The FP64 field again, separably. A corner vertex's position along one axis is one of two
// values: g + w X (the owner node's corner bit is 0 on that axis) or (g + w (X - 1)) + w (the
// bit is 1; SVO.cu:573-576 forms corners from the owner's origin). So the hat factor of a
// point and a corner along an axis is one of two values that depend only on the point's
// coordinate on that axis, the corner's lattice coordinate and that bit. kSepTables forms
// them once per grid coordinate and depth (the reference's hat arithmetic, quotients by
// divRn); each block copies its brick's slices and stages each corner of the brick's cell box
// at every depth as its coefficient and a flag byte (present, the three corner bits). A point
// then sums, for d = 0..D-1 and k = x|y<<1|z<<2, lambda * ((hx * hy) * hz) over its present
// corners -- fieldAt's additions in fieldAt's order, so the field is bit-identical, at a few
// table reads and three FP64 operations per term (the x*y factor is shared by a column's
// points where they lie in one cell).
constexpr int kSepX = 32, kSepY = 8, kSepThreads = kSepX * kSepY, kSepTileCap = 1024, kSepStageCap = 2048;
template <typename T> struct Pair { typedef double2 type; };
template <> struct Pair<float> { typedef float2 type; };

// The hat tables of every lattice coordinate of the grid, once per depth and axis (a grid of
// (R+1)^3 points has only 3 (R+1) coordinates per depth, which every brick would otherwise
// form again): tabC the coordinate's cell c = floor((p - g) / w), tabH its factors
// [corner side * 2 + corner bit] against the corner at c + side, whose position is g + w X for
// an owner bit 0 and (g + w (X - 1)) + w for an owner bit 1. Entry ((d * 3 + axis) * M + i).
__global__ void kSepTables(const __grid_constant__ EvalParams P, double3 o, double3 vs, int64_t M,
                           double* __restrict__ tabH, int* __restrict__ tabC) {
  const int64_t item = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (item >= (int64_t)P.depth * 3 * M) return;
  const int d = (int)(item / (3 * M)), a = (int)((item / M) % 3);
  const int64_t idx = item % M;
  const double w = P.w0 * (double)(1u << d), wi = P.winv[d];
  const double oa = a == 0 ? o.x : a == 1 ? o.y : o.z, va = a == 0 ? vs.x : a == 1 ? vs.y : vs.z;
  const double ga = a == 0 ? P.g.x : a == 1 ? P.g.y : P.g.z;
  const double pa = oa + (double)idx * va;
  const int64_t c = (int64_t)floor(divRn(pa - ga, w, wi));
  double h[4];
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int64_t X = c + side;
    const double pA = latticePos(ga, w, (uint32_t)(X < 0 ? 0 : X));
    const double pB = X >= 1 ? latticePos(ga, w, (uint32_t)(X - 1)) + w : pA;
    h[2 * side] = hat1r(pa, pA, w, wi);
    h[2 * side + 1] = hat1r(pa, pB, w, wi);
  }
  double2* dst = (double2*)(tabH + 4 * item);
  dst[0] = make_double2(h[0], h[1]);
  dst[1] = make_double2(h[2], h[3]);
  tabC[item] = (int)c;
}

// One brick's hat tables and cell boxes: the hat factors and cells of the brick's coordinates
// for every depth ([corner side * 2 + corner bit]; hZ is [depth][that index][point], so a
// corner's factors for a thread's points lie side by side and come in pairs), and the corner
// boxes of every depth staged together in one pass (their lattice lookups are dependent loads:
// in one pass their latencies overlap).
template <typename T, int kSepZ>
struct alignas(16) SepStage {
  T hX[kMaxDepth][4][kSepX];  // [depth][corner side * 2 + corner bit][x]: a warp's x run reads side by side
  T hY[kMaxDepth][kSepY][4];
  T hZ[kMaxDepth][4][kSepZ];
  T tLam[kSepStageCap];
  int cX[kMaxDepth][kSepX], cY[kMaxDepth][kSepY], cZ[kMaxDepth][kSepZ];
  int tOff[kMaxDepth], tEnd[kMaxDepth];  // depth d's tile: [tOff[d], tEnd[d]); tOff -1: per-point
  int cOff[kMaxDepth], cEnd[kMaxDepth];  // its (x, y) columns: [cOff[d], cEnd[d])
  int bny[kMaxDepth], bnz[kMaxDepth];  // the box's corners along y and z
  int tAny[kMaxDepth], tCols;
  unsigned char tFlag[kSepStageCap];
  __device__ int boxOf(int d, int& nx, int& ny, int& nz) const {
    nx = cX[d][kSepX - 1] - cX[d][0] + 2;
    ny = cY[d][kSepY - 1] - cY[d][0] + 2;
    nz = cZ[d][kSepZ - 1] - cZ[d][0] + 2;
    return nx * ny * nz;
  }
};

// The brick's slices of kSepTables' tables (threads i = 0, n, 2n, ... of the calling group).
template <typename T, int kSepZ>
__device__ void sepTables(SepStage<T, kSepZ>& S, int D, int64_t M, int64_t x0, int64_t y0, int64_t z0,
                          const double* __restrict__ tabH, const int* __restrict__ tabC, int i, int n) {
  constexpr int kCoords = kSepX + kSepY + kSepZ, kBatch = 4;  // a thread's items in batches, loads first
  const int total = kCoords * D;
  for (int item0 = i; item0 < total; item0 += kBatch * n) {
    double2 h01[kBatch], h23[kBatch];
    int c[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int item = item0 + u * n;
      if (item >= total) break;
      const int d = item / kCoords, j = item % kCoords;
      const int a = j < kSepX ? 0 : (j < kSepX + kSepY ? 1 : 2);
      const int k = a == 0 ? j : (a == 1 ? j - kSepX : j - kSepX - kSepY);
      int64_t idx = (a == 0 ? x0 : a == 1 ? y0 : z0) + k;
      if (idx > M - 1) idx = M - 1;  // clamped to the grid
      const int64_t r = ((int64_t)d * 3 + a) * M + idx;
      h01[u] = __ldg((const double2*)(tabH + 4 * r));
      h23[u] = __ldg((const double2*)(tabH + 4 * r) + 1);
      c[u] = __ldg(tabC + r);
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int item = item0 + u * n;
      if (item >= total) break;
      const int d = item / kCoords, j = item % kCoords;
      const int a = j < kSepX ? 0 : (j < kSepX + kSepY ? 1 : 2);
      const int k = a == 0 ? j : (a == 1 ? j - kSepX : j - kSepX - kSepY);
      if (a == 2) {
        S.hZ[d][0][k] = (T)h01[u].x;
        S.hZ[d][1][k] = (T)h01[u].y;
        S.hZ[d][2][k] = (T)h23[u].x;
        S.hZ[d][3][k] = (T)h23[u].y;
      } else if (a == 0) {
        S.hX[d][0][k] = (T)h01[u].x;
        S.hX[d][1][k] = (T)h01[u].y;
        S.hX[d][2][k] = (T)h23[u].x;
        S.hX[d][3][k] = (T)h23[u].y;
      } else {
        T* dst = S.hY[d][k];
        dst[0] = (T)h01[u].x;
        dst[1] = (T)h01[u].y;
        dst[2] = (T)h23[u].x;
        dst[3] = (T)h23[u].y;
      }
      (a == 0 ? S.cX[d] : a == 1 ? S.cY[d] : S.cZ[d])[k] = c[u];
    }
  }
}

// Where each depth's box goes (a box over the capacity: per-point lookups), by one warp: lane d
// sizes depth d's box, then every lane runs the greedy placement in depth order on the
// shuffled sizes (registers only) and lane d keeps depth d's place.
template <typename T, int kSepZ>
__device__ void sepPlace(SepStage<T, kSepZ>& S, int D, int lane) {
  int n = 0, c = 0, ny = 0, nz = 0;
  if (lane < D) {
    int nx;
    n = S.boxOf(lane, nx, ny, nz);
    c = nx * ny;
  }
  int off = 0, cols = 0, myOff = -1, myCol = 0, myEnd = 0, myColEnd = 0;
  for (int d = 0; d < D; ++d) {
    const int nd = __shfl_sync(0xffffffffu, n, d), cd = __shfl_sync(0xffffffffu, c, d);
    const bool fits = nd <= kSepTileCap && off + nd <= kSepStageCap;
    if (lane == d) {
      myOff = fits ? off : -1;
      myCol = cols;
    }
    if (fits) {
      off += (nd + 1) & ~1;  // boxes start at even entries: a column's z pairs are aligned
      cols += cd;
    }
    if (lane == d) {
      myEnd = off;
      myColEnd = cols;
    }
  }
  if (lane < D) {
    S.tOff[lane] = myOff;
    S.tEnd[lane] = myEnd;
    S.cOff[lane] = myCol;
    S.cEnd[lane] = myColEnd;
    S.bny[lane] = ny;
    S.bnz[lane] = nz;
    S.tAny[lane] = 0;
  }
  if (lane == 0) S.tCols = cols;
}

// The corners of every depth's cell box: coefficient and flag byte (bit 0 present, bits 1-3
// the owner corner bits); tAny[d]: whether depth d has any. A thread per (x, y) column of a
// box, eight z entries at a time: their lattice indices are consecutive, so they lie in one or
// two words of the lattice bits, and the loads of those words, then of the present corners'
// coefficients and keys, go out together. The box entry (x, y, z) sits at (x ny + y) nz + z.
template <typename T, int kSepZ>
__device__ void sepStageBoxes(SepStage<T, kSepZ>& S, const EvalParams& P, const double* __restrict__ lambda, int i,
                              int n) {
  for (int e = i; e < S.tCols; e += n) {
    // the columns lie in depth order (a depth without a tile: an empty range): e's depth is the
    // number of depths whose columns end at or before it
    int d = 0;
#pragma unroll
    for (int j = 0; j < kMaxDepth; ++j) d += (j < P.depth && e >= S.cEnd[j]) ? 1 : 0;
    const int ny = S.bny[d], nz = S.bnz[d];
    const int col = e - S.cOff[d], ix = col / ny, iy = col - ix * ny;
    const LatticeIndex& L = P.lat[d];
    const int lim = P.res >> d;
    const int Lx = S.cX[d][0] + ix, Ly = S.cY[d][0] + iy;
    const bool inBox = Lx >= 0 && Ly >= 0 && Lx <= lim && Ly <= lim;
    const uint32_t colBase = inBox ? ((uint32_t)Lx * L.M + (uint32_t)Ly) * L.M : 0u;
    bool any = false;
    for (int z8 = 0; z8 < nz; z8 += 8) {
      const int zA = S.cZ[d][0] + z8;
      const int zLo = zA < 0 ? 0 : zA, zHi = min(min(zA + 7, S.cZ[d][0] + nz - 1), lim);
      unsigned long long wLo = 0, wHi = 0;
      uint32_t rLo = 0, rHi = 0, wIdx = 0;
      const bool live = inBox && zLo <= zHi;
      if (live) {
        wIdx = (colBase + (uint32_t)zLo) >> 6;
        const uint32_t wLast = (colBase + (uint32_t)zHi) >> 6;
        wLo = L.bits[wIdx];
        rLo = L.rank[wIdx];
        if (wLast != wIdx) {
          wHi = L.bits[wLast];
          rHi = L.rank[wLast];
        }
      }
      uint32_t v[8];
      unsigned hasMask = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int Lz = zA + j;
        v[j] = 0;
        if (live && Lz >= zLo && Lz <= zHi) {
          const uint32_t lin = colBase + (uint32_t)Lz;
          const bool lo = (lin >> 6) == wIdx;
          const unsigned long long word = lo ? wLo : wHi;
          if ((word >> (lin & 63)) & 1ull) {  // latticeHas / latticeRank on the kept words
            v[j] = L.base + (lo ? rLo : rHi) + (uint32_t)__popcll(word & ((1ull << (lin & 63)) - 1ull));
            hasMask |= 1u << j;
          }
        }
      }
      double lv[8];
      uint32_t keyHi[8];  // the key's upper word: the owner corner bits 37-39 are its bits 5-7
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        lv[j] = 0.0;
        keyHi[j] = 0;
        if (hasMask >> j & 1u) {
          lv[j] = lambda[v[j]];
          keyHi[j] = ((const uint32_t*)P.vertKey)[2 * (size_t)v[j] + 1];
        }
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (z8 + j >= nz) break;
        const int t = S.tOff[d] + col * nz + z8 + j;
        unsigned char f = 0;
        if (hasMask >> j & 1u) {
          S.tLam[t] = (T)lv[j];
          f = (unsigned char)(1u | (((keyHi[j] >> 5) & 7u) << 1));
        }
        S.tFlag[t] = f;
      }
      any |= hasMask != 0;
    }
    if (any) S.tAny[d] = 1;  // benign race: every writer stores 1
  }
}

// The terms of G consecutive points q0.. of a thread's column that lie in one cell (box-relative
// z cell rz): each present corner's coefficient, bits and x*y factor are read once for them,
// and each point adds lambda * ((hx * hy) * hz) in corner order. colT[c]: the box entry of the
// (x, y) corner column c = x | y << 1 at z = 0.
template <int G, typename T, int kSepZ>
__device__ __forceinline__ void sepCellTerms(const SepStage<T, kSepZ>& S, int d, const T* hx, const T* hy,
                                             const T* lamT, const unsigned char* flagT, const int (&colT)[4], int rz,
                                             int q0, T (&sum)[kSepZ]) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
    const int t = colT[k & 3] + rz + oz;
    const unsigned f = flagT[t];
    if (!(f & 1u)) continue;
    const T lam = lamT[t];
    const T fxy = hx[kSepX * (2 * ox + ((f >> 1) & 1u))] * hy[2 * oy + ((f >> 2) & 1u)];
    const T* hz = S.hZ[d][2 * oz + ((f >> 3) & 1u)];
#pragma unroll
    for (int g = 0; g < G; ++g) sum[q0 + g] += lam * (fxy * hz[q0 + g]);
  }
}

// The terms of one thread's column of kSepZ points (brick column tx, ty) over every depth, in
// fieldAt's order: for d = 0..D-1 and k = x|y<<1|z<<2, lambda * ((hx * hy) * hz).
template <typename T, int kSepZ>
__device__ void sepTerms(const SepStage<T, kSepZ>& S, const EvalParams& P, const double* __restrict__ lambda,
                         double3 o, double3 vs, int tx, int ty, int64_t xi, int64_t yj, int64_t z0, T (&sum)[kSepZ]) {
#pragma unroll
  for (int q = 0; q < kSepZ; ++q) sum[q] = T(0);
  for (int d = 0; d < P.depth; ++d) {
    const double w = P.w0 * (double)(1u << d), wi = P.winv[d];
    const int ny = S.bny[d], nz = S.bnz[d];
    if (S.tOff[d] < 0) {  // the box does not fit the tile: per-point lookups
      const LatticeIndex& L = P.lat[d];
      const int64_t lim = (int64_t)(P.res >> d);
      const double px = o.x + (double)xi * vs.x, py = o.y + (double)yj * vs.y;
#pragma unroll
      for (int q = 0; q < kSepZ; ++q) {
        const double pz = o.z + (double)(z0 + q) * vs.z;
        const int64_t cx = S.cX[d][tx], cy = S.cY[d][ty], cz = S.cZ[d][q];
        T s = sum[q];
        for (int k = 0; k < 8; ++k) {
          const int64_t Lx = cx + (k & 1), Ly = cy + ((k >> 1) & 1), Lz = cz + ((k >> 2) & 1);
          if (Lx < 0 || Ly < 0 || Lz < 0 || Lx > lim || Ly > lim || Lz > lim) continue;
          const uint32_t lin = (uint32_t)((Lx * L.M + Ly) * L.M + Lz);
          if (!latticeHas(L, lin)) continue;
          const uint32_t v = latticeRank(L, lin);
          const double fx = hat1r(px, P.vertPos[3 * (int64_t)v], w, wi);
          if (fx <= 0.0) continue;
          const double fy = hat1r(py, P.vertPos[3 * (int64_t)v + 1], w, wi);
          if (fy <= 0.0) continue;
          const double fz = hat1r(pz, P.vertPos[3 * (int64_t)v + 2], w, wi);
          if (fz <= 0.0) continue;
          s += (T)lambda[v] * ((T)fx * (T)fy * (T)fz);
        }
        sum[q] = s;
      }
    } else if (S.tAny[d]) {
      const int rx = S.cX[d][tx] - S.cX[d][0], ry = S.cY[d][ty] - S.cY[d][0];
      const T* hx = &S.hX[d][0][tx];  // hx[kSepX * e]: factor e of the thread's x
      const T* hy = S.hY[d][ty];
      const T* lamT = S.tLam + S.tOff[d];
      const unsigned char* flagT = S.tFlag + S.tOff[d];
      // A present corner adds lambda * ((hx * hy) * hz) even where a factor is 0: the term is
      // then +-0 (NaN for a non-finite coefficient), as fieldAt's sum over the corners adds it,
      // and a running sum that starts at +0 is never -0, so a +-0 term leaves it unchanged.
      if (nz == 2) {
        // Every point of the brick's z run lies in one cell (block-uniform): a corner is the
        // same vertex for all of the thread's points, so its coefficient, bits and x*y factor
        // are read once and its terms cost two products and a sum per point. The four (x, y)
        // corner columns' flag and coefficient pairs (z = 0, 1 side by side, at an even entry)
        // are read up front.
        typedef typename Pair<T>::type P2;
        unsigned fp[4];
        P2 lp[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int t0 = ((rx + (c & 1)) * ny + (ry + (c >> 1))) * 2;
          fp[c] = *(const unsigned short*)(flagT + t0);
          lp[c] = *(const P2*)(lamT + t0);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
          const unsigned f = (fp[k & 3] >> (8 * oz)) & 0xffu;
          if (!(f & 1u)) continue;
          const T lam = oz ? lp[k & 3].y : lp[k & 3].x;
          const T fxy = hx[kSepX * (2 * ox + ((f >> 1) & 1u))] * hy[2 * oy + ((f >> 2) & 1u)];
          const T* hz = S.hZ[d][2 * oz + (int)((f >> 3) & 1u)];
#pragma unroll
          for (int q = 0; q < kSepZ; q += 2) {
            const typename Pair<T>::type h2 = *(const typename Pair<T>::type*)(hz + q);
            sum[q] += lam * (fxy * h2.x);
            sum[q + 1] += lam * (fxy * h2.y);
          }
        }
      } else {
        // The thread's z run spans several cells (the finest depths): the points are taken in
        // runs of four, two or one that lie in one cell (the runs are the same for the whole
        // block), so a corner's reads and x*y factor serve every point of its run.
        int colT[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) colT[c] = ((rx + (c & 1)) * ny + (ry + (c >> 1))) * nz;
        const int zc = S.cZ[d][0];
#pragma unroll
        for (int q0 = 0; q0 < kSepZ; q0 += 4) {
          const int ra = S.cZ[d][q0] - zc, rb = S.cZ[d][q0 + 1] - zc, rc = S.cZ[d][q0 + 2] - zc,
                    rd = S.cZ[d][q0 + 3] - zc;
          if (ra == rd) {
            sepCellTerms<4>(S, d, hx, hy, lamT, flagT, colT, ra, q0, sum);
          } else {
            if (ra == rb) {
              sepCellTerms<2>(S, d, hx, hy, lamT, flagT, colT, ra, q0, sum);
            } else {
              sepCellTerms<1>(S, d, hx, hy, lamT, flagT, colT, ra, q0, sum);
              sepCellTerms<1>(S, d, hx, hy, lamT, flagT, colT, rb, q0 + 1, sum);
            }
            if (rc == rd) {
              sepCellTerms<2>(S, d, hx, hy, lamT, flagT, colT, rc, q0 + 2, sum);
            } else {
              sepCellTerms<1>(S, d, hx, hy, lamT, flagT, colT, rc, q0 + 2, sum);
              sepCellTerms<1>(S, d, hx, hy, lamT, flagT, colT, rd, q0 + 3, sum);
            }
          }
        }
      }
    }
  }
}

// T = float is the precision form's FP32 field: the same tables (formed in FP64, rounded once)
// and the same terms, summed in FP32. One block per brick of kSepX x kSepY x kSepZ points.
template <typename T, int kSepZ>  // points per thread along z (the brick's depth)
__global__ void __launch_bounds__(kSepThreads, 4) kEvalGridSep(const __grid_constant__ EvalParams P,
                                                            const double* __restrict__ lambda, double3 o, double3 vs,
                                                            const double* __restrict__ tabH,
                                                            const int* __restrict__ tabC, int R,
                                                            T* __restrict__ field) {
  __shared__ SepStage<T, kSepZ> S;
  const int64_t M = (int64_t)R + 1;
  const int tid = threadIdx.x, tx = tid % kSepX, ty = tid / kSepX;
  const int64_t x0 = (int64_t)blockIdx.x * kSepX, y0 = (int64_t)blockIdx.y * kSepY, z0 = (int64_t)blockIdx.z * kSepZ;
  const int64_t xi = x0 + tx, yj = y0 + ty;
  sepTables(S, P.depth, M, x0, y0, z0, tabH, tabC, tid, kSepThreads);
  __syncthreads();
  if (tid < 32) sepPlace(S, P.depth, tid);
  __syncthreads();
  sepStageBoxes(S, P, lambda, tid, kSepThreads);
  __syncthreads();
  if (xi < M && yj < M) {
    T sum[kSepZ];
    sepTerms(S, P, lambda, o, vs, tx, ty, xi, yj, z0, sum);
#pragma unroll
    for (int q = 0; q < kSepZ; ++q)
      if (z0 + q < M) field[xi + M * (yj + M * (z0 + q))] = sum[q];
  }
}

// ---- marching cubes in three launches -----------------------------------------------------
// Classify: each thread takes 8 consecutive voxels (x fastest) and slides along x, loading one
// column of 4 corner values per voxel (each field value is read about once), writes the case
// bytes and reduces the vertex counts per block. The block sums are scanned (kScanSpine);
// Emit re-reads only the case bytes, scans the counts inside the block and writes the
// triangle vertices of the non-empty voxels in voxel order, as the reference's compaction does.
template <typename T, int ITEMS>
__global__ void __launch_bounds__(kScanThreads) kMcClassify(const T* __restrict__ field, int R, double iso,
                                                             uint8_t* __restrict__ cube,
                                                             unsigned long long* __restrict__ blockSums) {
  const int64_t nvox = (int64_t)R * R * R, M = (int64_t)R + 1;
  const int64_t base = (int64_t)blockIdx.x * (kScanThreads * ITEMS) + (int64_t)threadIdx.x * ITEMS;
  unsigned long long cnt = 0;
  int64_t x = 0, y = 0, z = 0;
  if (base < nvox) voxelXYZ(base, R, x, y, z);
  if (base + ITEMS <= nvox && x + ITEMS <= R) {
    // the run stays in one row: all 4 x (ITEMS + 1) corner values are loaded up front
    const int64_t r0 = (z * M + y) * M + x, r1 = (z * M + y + 1) * M + x, r2 = ((z + 1) * M + y) * M + x,
                  r3 = ((z + 1) * M + y + 1) * M + x;
    double fa[ITEMS + 1], fb[ITEMS + 1], fc[ITEMS + 1], fd[ITEMS + 1];
#pragma unroll
    for (int j = 0; j <= ITEMS; ++j) {
      fa[j] = (double)field[r0 + j];
      fb[j] = (double)field[r1 + j];
      fc[j] = (double)field[r2 + j];
      fd[j] = (double)field[r3 + j];
    }
    unsigned long long packed = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const unsigned ci = (unsigned)(fa[j] < iso) | (unsigned)(fb[j] < iso) << 1 | (unsigned)(fb[j + 1] < iso) << 2 |
                          (unsigned)(fa[j + 1] < iso) << 3 | (unsigned)(fc[j] < iso) << 4 |
                          (unsigned)(fd[j] < iso) << 5 | (unsigned)(fd[j + 1] < iso) << 6 |
                          (unsigned)(fc[j + 1] < iso) << 7;
      cnt += cMcCase[ci] & 15ull;
      packed |= (unsigned long long)ci << (8 * (j & 7));
      if (ITEMS != 8 || (((uintptr_t)(cube + base)) & 7u)) cube[base + j] = (uint8_t)ci;
    }
    // one 8-byte store when the caller's buffer allows it (base is a multiple of 8)
    if (ITEMS == 8 && !(((uintptr_t)(cube + base)) & 7u)) *(unsigned long long*)(cube + base) = packed;
  } else if (base < nvox) {
    double a = 0, b = 0, c = 0, d = 0;  // column x: (y,z) (y+1,z) (y,z+1) (y+1,z+1)
    bool have = false;
    for (int j = 0; j < ITEMS && base + j < nvox; ++j) {
      const int64_t r0 = (z * M + y) * M, r1 = (z * M + y + 1) * M, r2 = ((z + 1) * M + y) * M,
                    r3 = ((z + 1) * M + y + 1) * M;
      if (!have) {
        a = (double)field[r0 + x];
        b = (double)field[r1 + x];
        c = (double)field[r2 + x];
        d = (double)field[r3 + x];
      }
      const double a1 = (double)field[r0 + x + 1], b1 = (double)field[r1 + x + 1], c1 = (double)field[r2 + x + 1],
                   d1 = (double)field[r3 + x + 1];
      // corner order 0 (0,0,0) 1 (0,1,0) 2 (1,1,0) 3 (1,0,0) 4 (0,0,1) 5 (0,1,1) 6 (1,1,1) 7 (1,0,1)
      const unsigned ci = (unsigned)(a < iso) | (unsigned)(b < iso) << 1 | (unsigned)(b1 < iso) << 2 |
                          (unsigned)(a1 < iso) << 3 | (unsigned)(c < iso) << 4 | (unsigned)(d < iso) << 5 |
                          (unsigned)(d1 < iso) << 6 | (unsigned)(c1 < iso) << 7;
      cube[base + j] = (uint8_t)ci;
      cnt += cMcCase[ci] & 15ull;
      a = a1;
      b = b1;
      c = c1;
      d = d1;
      have = true;
      if (++x == R) {  // next row
        x = 0;
        have = false;
        if (++y == R) {
          y = 0;
          ++z;
        }
      }
    }
  }
  unsigned long long total;
  blockExclusiveScan<unsigned long long>(cnt, total);
  if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

// kMcClassify for R a multiple of 256 (tiles of 8 voxels per thread): the same case bytes and
// block sums with coalesced loads. A warp takes 256 consecutive voxels of one row, lane l the
// voxels x0 + l + 32 j; each of the 4 corner rows is read 32 values per load, compared with
// the iso level, and the comparison of the x+1 corner comes from the next lane's bit of the
// row's ballot (lane 31: the next round's bit 0, or one extra value).
template <typename T>
__global__ void __launch_bounds__(kScanThreads) kMcClassifyRows(const T* __restrict__ field, int R, double iso,
                                                               uint8_t* __restrict__ cube,
                                                               unsigned long long* __restrict__ blockSums) {
  const int64_t M = (int64_t)R + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t s = (int64_t)blockIdx.x * (kScanThreads * 8) + (int64_t)warp * 256;  // the warp's first voxel
  int64_t x0, y, z;
  voxelXYZ(s, R, x0, y, z);
  const int64_t r[4] = {(z * M + y) * M + x0, (z * M + y + 1) * M + x0, ((z + 1) * M + y) * M + x0,
                        ((z + 1) * M + y + 1) * M + x0};
  double v[4][9];  // corner rows: v[k][j] at x0 + lane + 32 j; v[k][8] at x0 + 256 (all lanes)
#pragma unroll
  for (int k = 0; k < 4; ++k) {
#pragma unroll
    for (int j = 0; j < 8; ++j) v[k][j] = (double)field[r[k] + lane + 32 * j];
    v[k][8] = (double)field[r[k] + 256];
  }
  // each corner row's comparisons as warp ballots: the x+1 corner of lane l is bit l+1 (lane
  // 31: bit 0 of the next round, or the extra value)
  unsigned bal[4][8];
  unsigned ext = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
#pragma unroll
    for (int j = 0; j < 8; ++j) bal[k][j] = __ballot_sync(0xffffffffu, v[k][j] < iso);
    ext |= (unsigned)(v[k][8] < iso) << k;
  }
  unsigned long long cnt = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    unsigned c[4], n[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      c[k] = (bal[k][j] >> lane) & 1u;
      n[k] = lane < 31 ? (bal[k][j] >> (lane + 1)) & 1u : (j < 7 ? bal[k][j < 7 ? j + 1 : 0] & 1u : (ext >> k) & 1u);
    }
    // corner order 0 (0,0,0) 1 (0,1,0) 2 (1,1,0) 3 (1,0,0) 4 (0,0,1) 5 (0,1,1) 6 (1,1,1) 7 (1,0,1)
    const unsigned ci = c[0] | c[1] << 1 | n[1] << 2 | n[0] << 3 | c[2] << 4 | c[3] << 5 | n[3] << 6 | n[2] << 7;
    cube[s + lane + 32 * j] = (uint8_t)ci;
    cnt += cMcCase[ci] & 15ull;
  }
  unsigned long long total;
  blockExclusiveScan<unsigned long long>(cnt, total);
  if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

template <typename T, int ITEMS>
__global__ void __launch_bounds__(kScanThreads) kMcEmit(McCaseT<T> mc, double3 o, double3 vs,
                                                         const uint8_t* __restrict__ cube,
                                                         const unsigned long long* __restrict__ blockOffsets,
                                                         const unsigned long long* __restrict__ grandTotal,
                                                         double* __restrict__ tri, unsigned long long capacity) {
  // a block whose voxels emit nothing (most of them: the surface crosses few tiles) leaves at once
  const unsigned long long next = blockIdx.x + 1 < gridDim.x ? blockOffsets[blockIdx.x + 1] : *grandTotal;
  if (next == blockOffsets[blockIdx.x]) return;
  const int64_t nvox = (int64_t)mc.R * mc.R * mc.R;
  const int64_t base = (int64_t)blockIdx.x * (kScanThreads * ITEMS) + (int64_t)threadIdx.x * ITEMS;
  unsigned char ci[ITEMS];
  unsigned long long cnt = 0;
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    ci[j] = base + j < nvox ? cube[base + j] : 0;
    cnt += cMcCase[ci[j]] & 15ull;
  }
  unsigned long long total;
  const unsigned long long tileBase = blockOffsets[blockIdx.x];
  unsigned long long run = blockExclusiveScan<unsigned long long>(cnt, total);  // within the tile
  if (!total || !tri) return;
  // The tile's voxels with vertices are listed (place in the tile | offset within the tile's
  // output << 12: at most 15 vertices per voxel, so the offset stays below 2^16) and the block
  // emits the list round-robin, instead of each thread its own ITEMS voxels one after another.
  // Every voxel writes at its own offset: the order of the list does not matter.
  static_assert(kScanThreads * ITEMS <= 4096 && 15 * kScanThreads * ITEMS < 65536, "list entry packing");
  __shared__ uint32_t sList[kScanThreads * ITEMS];
  __shared__ unsigned sCount;
  if (threadIdx.x == 0) sCount = 0;
  __syncthreads();
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const unsigned c = cMcCase[ci[j]] & 15u;
    if (c) sList[atomicAdd(&sCount, 1u)] = (uint32_t)(threadIdx.x * ITEMS + j) | (uint32_t)run << 12;
    run += c;
  }
  __syncthreads();
  const int64_t tile0 = (int64_t)blockIdx.x * (kScanThreads * ITEMS);
  for (unsigned e = threadIdx.x; e < sCount; e += kScanThreads) {
    const uint32_t item = sList[e];
    const int64_t v = tile0 + (item & 4095u);
    const unsigned char c8 = cube[v];
    mcEmitVoxel(mc, o, vs, tri, capacity, v, c8, tileBase + (item >> 12), cMcCase[c8] & 15ull);
  }
}

// Dense-field launch shapes (bricks of BX x BY x BZ points, a thread per column of ZPER
// points); every shape computes the same bits, the autotuner picks the fastest.
template <typename T, int BX, int BY, int ZPER>
static its_status launchBricks(its_ctx* ctx, const EvalParams& P, const double* lam, double3 o, double3 vs, int res,
                               T* field) {
  constexpr int BZ = (kBrickThreads / (BX * BY)) * ZPER;
  const int64_t M = (int64_t)res + 1;
  const dim3 grid((unsigned)((M + BX - 1) / BX), (unsigned)((M + BY - 1) / BY), (unsigned)((M + BZ - 1) / BZ));
  kEvalGridBricks<T, BX, BY, ZPER><<<grid, kBrickThreads, 0, ctx->stream>>>(P, lam, o, vs, res, field);
  ITS_LAUNCHED(ctx);
  return ITS_OK;
}

// Corners per axis of the cell box that n consecutive lattice points span at the finest depth
// (one more than the exact bound, for the rounding of the cell quotients).
static int64_t boxCorners(int n, double v, double w0) { return (int64_t)std::floor((n - 1) * v / w0) + 3; }

template <typename T>
static its_status evalGridTuned(its_ctx* ctx, const SvoDevice& d, const double* lam, double3 o, double3 vs, int res,
                                T* field) {
  const EvalParams P = evalParams(d);
  // four brick shapes of the point-wise kernel and the separable kernel with 4 or 8 points per
  // thread along z (FP64, when the brick's cell box fits its tile): every candidate computes
  // the same bits
  auto sepFits = [&](int z) {
    return boxCorners(kSepX, vs.x, d.unit[0]) * boxCorners(kSepY, vs.y, d.unit[0]) * boxCorners(z, vs.z, d.unit[0]) <=
           kSepTileCap;
  };
  // Candidates, each computing the same bits for its type: FP64, four brick shapes of the
  // point-wise kernel and the separable kernel with 4 or 8 points per thread along z (when the
  // brick's cell box fits its tile); FP32, the separable kernel's two shapes where it fits (its
  // rounding differs from the point-wise FP32 kernel's), else the brick shapes.
  std::vector<int> cand;
  if (sizeof(T) == 8 || !sepFits(4)) cand = {0, 1, 2, 3};
  if (sepFits(4)) cand.push_back(4);
  if (sepFits(8)) cand.push_back(5);
  DevBuf<double> tabH;
  DevBuf<int> tabC;
  if (sepFits(4)) {  // the separable kernel's hat tables, formed once for all its launches here
    const int64_t M = (int64_t)res + 1, n = (int64_t)d.depth * 3 * M;
    its_status st = tabH.alloc(ctx, 4 * n);
    if (st == ITS_OK) st = tabC.alloc(ctx, n);
    if (st != ITS_OK) return st;
    kSepTables<<<gridFor(n, 256), 256, 0, ctx->stream>>>(P, o, vs, M, tabH.p, tabC.p);
    ITS_LAUNCHED(ctx);
  }
  auto run = [&](int j) -> its_status {
    switch (cand[j]) {
      case 1: return launchBricks<T, 32, 8, 2>(ctx, P, lam, o, vs, res, field);
      case 2: return launchBricks<T, 64, 4, 2>(ctx, P, lam, o, vs, res, field);
      case 3: return launchBricks<T, 16, 4, 4>(ctx, P, lam, o, vs, res, field);
      case 4:
      case 5: {
        const int z = cand[j] == 5 ? 8 : 4;
        const int64_t M = (int64_t)res + 1;
        const dim3 grid((unsigned)((M + kSepX - 1) / kSepX), (unsigned)((M + kSepY - 1) / kSepY),
                        (unsigned)((M + z - 1) / z));
        if (z == 8)
          kEvalGridSep<T, 8><<<grid, kSepThreads, 0, ctx->stream>>>(P, lam, o, vs, tabH.p, tabC.p, res, field);
        else
          kEvalGridSep<T, 4><<<grid, kSepThreads, 0, ctx->stream>>>(P, lam, o, vs, tabH.p, tabC.p, res, field);
        ITS_LAUNCHED(ctx);
        return ITS_OK;
      }
      default: return launchBricks<T, 32, 4, 4>(ctx, P, lam, o, vs, res, field);
    }
  };
  const std::string key = std::string("eval_grid/") + (sizeof(T) == 8 ? "f64" : "f32") + "/grid=" +
                          std::to_string(res) + "/octree=" + std::to_string(d.res) + "/depth=" + std::to_string(d.depth);
  int choice = 0;
  its_status st = tuneChoice(ctx, key, (int)cand.size(), cand.back() >= 4 ? (int)cand.size() - 1 : 0, run, &choice);
  if (st != ITS_OK) return st;
  return run(choice);
}

// divRn against the hardware-correct quotient (a test hook: out[i] = 1 where they differ).
__global__ void kCheckDivRn(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                            unsigned char* __restrict__ differ) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double y = 1.0 / b[i];
  const double q1 = divRn(a[i], b[i], y), q2 = a[i] / b[i];
  differ[i] = __double_as_longlong(q1) != __double_as_longlong(q2);
}

// ThinShells::getPointValGradient (ThinShells.cpp:1800-1866): a point outside the model box
// moves halfway towards its previous position until inside (at most 64 halvings; no move
// without previous positions), then the field and its gradient over its fine node's chain,
// with de_BaseFunction (BSpline.hpp:30-57) for the derivative factors.
__device__ __forceinline__ double deHat1(double x, double p, double w) {
  if (fabs(x - (p - w)) < 1e-9 || x < p - w || fabs(x - (p + w)) < 1e-9 || x > p + w) return 0.0;
  if (x <= p) return 1 / w;
  return -1 / w;
}

__global__ void kPointGradient(const __grid_constant__ EvalParams P, const double* __restrict__ lambda,
                               const double* __restrict__ pts, const double* __restrict__ before, int64_t m, double3 lo,
                               double3 hi, double* __restrict__ val, double* __restrict__ grad,
                               uint8_t* __restrict__ missing) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  double px = pts[3 * i], py = pts[3 * i + 1], pz = pts[3 * i + 2];
  if (before) {
    const double bx = before[3 * i], by = before[3 * i + 1], bz = before[3 * i + 2];
    for (int it = 0; it < 64; ++it) {
      if (!(px < lo.x || py < lo.y || pz < lo.z || px > hi.x || py > hi.y || pz > hi.z)) break;
      px = (px + bx) / 2.0;
      py = (py + by) / 2.0;
      pz = (pz + bz) / 2.0;
    }
  }
  double sum = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
  bool found = false;
  const int dx = (int)((px - P.g.x) / P.w0), dy = (int)((py - P.g.y) / P.w0), dz = (int)((pz - P.g.z) / P.w0);
  if (dx >= 0 && dy >= 0 && dz >= 0 && dx < P.res && dy < P.res && dz < P.res) {
    const uint32_t t0 = fineNodeOf(P.fineOcc, P.fineRank, mortonEncode((uint32_t)dx, (uint32_t)dy, (uint32_t)dz));
    if (t0 != kNone) {
      found = true;
      uint32_t t = t0;
      for (int d = 0; d < P.depth && t != kNone; ++d) {
        uint32_t X, Y, Z;
        mortonDecode(P.morton[t], X, Y, Z);
        const double w = P.w0 * (double)(1u << d);
        const double bx = latticePos(P.g.x, w, X), by = latticePos(P.g.y, w, Y), bz = latticePos(P.g.z, w, Z);
        const LatticeIndex& L = P.lat[d];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
          const double cx = ox ? bx + w : bx, cy = oy ? by + w : by, cz = oz ? bz + w : bz;
          const double lam = lambda[latticeRank(L, ((X + ox) * L.M + (Y + oy)) * L.M + (Z + oz))];
          sum += lam * hat3(cx, cy, cz, w, px, py, pz);
          const double hx = hat1(px, cx, w), hy = hat1(py, cy, w), hz = hat1(pz, cz, w);
          gx += lam * (deHat1(px, cx, w) * hy * hz);
          gy += lam * (hx * deHat1(py, cy, w) * hz);
          gz += lam * (hx * hy * deHat1(pz, cz, w));
        }
        t = P.parent[t];
      }
    }
  }
  val[i] = sum;
  grad[3 * i] = gx;
  grad[3 * i + 1] = gy;
  grad[3 * i + 2] = gz;
  if (missing) missing[i] = found ? 0 : 1;
}

// Point queries (ThinShells::multiPointQuery, ThinShells.cpp:1183-1420, CUDA branch
// cuAcc::cpPointQuery, CUDACompute.cu:1070-1156): points outside the model box grown by one
// box width on every side take the outer iso value; the others the field. Label: 1 when the
// value >= outer, -1 when <= inner, else 0 (inside the shell).
__global__ void kPointQuery(const __grid_constant__ EvalParams P, const double* __restrict__ lambda,
                            const double* __restrict__ pts, int64_t m, double3 lo, double3 hi, double inner,
                            double outer, double* __restrict__ values, int8_t* __restrict__ labels) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double px = pts[3 * i], py = pts[3 * i + 1], pz = pts[3 * i + 2];
  const bool outside = px < lo.x || py < lo.y || pz < lo.z || px > hi.x || py > hi.y || pz > hi.z;
  const double v = outside ? outer : fieldAt(P, lambda, px, py, pz);
  if (values) values[i] = v;
  if (labels) labels[i] = (int8_t)(v >= outer ? 1 : (v <= inner ? -1 : 0));
}

}  // namespace its

using namespace its;

extern "C" {

its_status its_eval_points(its_svo* s, const double* lambda, const double* points, int64_t npoints, double* out,
                           uint8_t* missing) {
  if (!s || !lambda || (!points && npoints) || (!out && npoints) || npoints < 0) return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  if (npoints == 0) return ITS_OK;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> L, P;
  OutArg<double> O;
  OutArg<uint8_t> Mi;
  its_status st;
  if ((st = L.stage(ctx, lambda, s->d.numVerts)) != ITS_OK) return st;
  if ((st = P.stage(ctx, points, 3 * npoints)) != ITS_OK) return st;
  if ((st = O.stage(ctx, out, npoints)) != ITS_OK) return st;
  if ((st = Mi.stage(ctx, missing, npoints)) != ITS_OK) return st;
  kEvalPoints<<<gridFor(npoints, 128), 128, 0, ctx->stream>>>(evalParams(s->d), L.d, P.d, npoints, O.d, Mi.d);
  ITS_LAUNCHED(ctx);
  if ((st = O.finish(ctx)) != ITS_OK) return st;
  if ((st = Mi.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_shell_iso_values(its_svo* s, const double* lambda, const double* points, int64_t npoints, double* inner,
                                double* outer, int64_t* num_missing) {
  if (!s || !lambda || !points || npoints <= 0 || !inner || !outer) return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> L, P;
  its_status st;
  if ((st = L.stage(ctx, lambda, s->d.numVerts)) != ITS_OK) return st;
  if ((st = P.stage(ctx, points, 3 * npoints)) != ITS_OK) return st;
  const unsigned blocks = (unsigned)std::min<int64_t>(gridFor(npoints, 256), (int64_t)ctx->numSMs * 8);
  DevBuf<double> pmin, pmax;
  DevBuf<unsigned long long> pmiss;
  if ((st = pmin.alloc(ctx, blocks)) != ITS_OK) return st;
  if ((st = pmax.alloc(ctx, blocks)) != ITS_OK) return st;
  if ((st = pmiss.alloc(ctx, blocks)) != ITS_OK) return st;
  kIsoPartials<<<blocks, 256, 0, ctx->stream>>>(evalParams(s->d), L.d, P.d, npoints, pmin.p, pmax.p, pmiss.p);
  ITS_LAUNCHED(ctx);
  std::vector<double> hmin(blocks), hmax(blocks);
  std::vector<unsigned long long> hmiss(blocks);
  ITS_CU(ctx, cudaMemcpyAsync(hmin.data(), pmin.p, blocks * 8, cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(hmax.data(), pmax.p, blocks * 8, cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(hmiss.data(), pmiss.p, blocks * 8, cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  double lo = DBL_MAX, hi = -DBL_MAX;
  unsigned long long miss = 0;
  for (unsigned k = 0; k < blocks; ++k) {
    lo = std::min(lo, hmin[k]);
    hi = std::max(hi, hmax[k]);
    miss += hmiss[k];
  }
  if (miss == (unsigned long long)npoints) return setError(ctx, ITS_ERR_INVALID, "no point lies in a fine node");
  *inner = lo;
  *outer = hi;
  if (num_missing) *num_missing = (int64_t)miss;
  return ITS_OK;
}

its_status its_point_query(its_svo* s, const double* lambda, const double* points, int64_t npoints,
                           const double box_origin[3], const double box_end[3], double inner, double outer,
                           double* values, int8_t* labels) {
  if (!s || !lambda || !box_origin || !box_end || npoints < 0 || (npoints && !points)) return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  if (npoints == 0) return ITS_OK;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> L, P;
  OutArg<double> Va;
  OutArg<int8_t> La;
  its_status st;
  if ((st = L.stage(ctx, lambda, s->d.numVerts)) != ITS_OK) return st;
  if ((st = P.stage(ctx, points, 3 * npoints)) != ITS_OK) return st;
  if ((st = Va.stage(ctx, values, npoints)) != ITS_OK) return st;
  if ((st = La.stage(ctx, labels, npoints)) != ITS_OK) return st;
  // minRange = boxOrigin - boxWidth, maxRange = boxEnd + boxWidth (ThinShells.cpp:1198-1199)
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    const double w = box_end[a] - box_origin[a];
    lo[a] = box_origin[a] - w;
    hi[a] = box_end[a] + w;
  }
  kPointQuery<<<gridFor(npoints, 128), 128, 0, ctx->stream>>>(evalParams(s->d), L.d, P.d, npoints,
                                                             make_double3(lo[0], lo[1], lo[2]),
                                                             make_double3(hi[0], hi[1], hi[2]), inner, outer, Va.d, La.d);
  ITS_LAUNCHED(ctx);
  if ((st = Va.finish(ctx)) != ITS_OK) return st;
  if ((st = La.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_point_value_gradient(its_svo* s, const double* lambda, const double* points, const double* before,
                                   int64_t npoints, const double box_origin[3], const double box_end[3], double* values,
                                   double* gradients, uint8_t* missing) {
  if (!s || !lambda || npoints < 0 || (npoints && (!points || !values || !gradients)) || !box_origin || !box_end)
    return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  if (npoints == 0) return ITS_OK;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> L, P, B;
  OutArg<double> Vo, G;
  OutArg<uint8_t> Mi;
  its_status st;
  if ((st = L.stage(ctx, lambda, s->d.numVerts)) != ITS_OK || (st = P.stage(ctx, points, 3 * npoints)) != ITS_OK ||
      (st = B.stage(ctx, before, before ? 3 * npoints : 0)) != ITS_OK || (st = Vo.stage(ctx, values, npoints)) != ITS_OK ||
      (st = G.stage(ctx, gradients, 3 * npoints)) != ITS_OK || (st = Mi.stage(ctx, missing, npoints)) != ITS_OK)
    return st;
  kPointGradient<<<gridFor(npoints, 128), 128, 0, ctx->stream>>>(
      evalParams(s->d), L.d, P.d, B.d, npoints, make_double3(box_origin[0], box_origin[1], box_origin[2]),
      make_double3(box_end[0], box_end[1], box_end[2]), Vo.d, G.d, Mi.d);
  ITS_LAUNCHED(ctx);
  if ((st = Vo.finish(ctx)) != ITS_OK || (st = G.finish(ctx)) != ITS_OK || (st = Mi.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_eval_grid(its_svo* s, const double* lambda, const double origin[3], const double width[3], int res,
                         double* field) {
  if (!s || !lambda || !origin || !width || !field || res < 1 || res > 2048) return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  const int64_t M = (int64_t)res + 1, total = M * M * M;
  InArg<double> L;
  OutArg<double> F;
  its_status st;
  if ((st = L.stage(ctx, lambda, s->d.numVerts)) != ITS_OK) return st;
  if ((st = F.stage(ctx, field, total)) != ITS_OK) return st;
  const double3 o = make_double3(origin[0], origin[1], origin[2]);
  const double3 vs = make_double3(width[0] / res, width[1] / res, width[2] / res);
  if ((st = evalGridTuned<double>(ctx, s->d, L.d, o, vs, res, F.d)) != ITS_OK) return st;
  if ((st = F.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_eval_grid_f32(its_svo* s, const double* lambda, const double origin[3], const double width[3], int res,
                             float* field) {
  if (!s || !lambda || !origin || !width || !field || res < 1 || res > 2048) return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  const int64_t M = (int64_t)res + 1, total = M * M * M;
  InArg<double> L;
  OutArg<float> F;
  its_status st;
  if ((st = L.stage(ctx, lambda, s->d.numVerts)) != ITS_OK) return st;
  if ((st = F.stage(ctx, field, total)) != ITS_OK) return st;
  const double3 o = make_double3(origin[0], origin[1], origin[2]);
  const double3 vs = make_double3(width[0] / res, width[1] / res, width[2] / res);
  if ((st = evalGridTuned<float>(ctx, s->d, L.d, o, vs, res, F.d)) != ITS_OK) return st;
  if ((st = F.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

// Counts the pairs (a[i], b[i]) whose quotient by divRn differs from a[i] / b[i] (device or
// host arrays). A self-check of the division the field kernels use.
its_status its_check_division(its_ctx* ctx, const double* a, const double* b, int64_t n, int64_t* mismatches) {
  if (!ctx || !a || !b || n <= 0 || !mismatches) return ITS_ERR_INVALID;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> A, B;
  its_status st;
  if ((st = A.stage(ctx, a, n)) != ITS_OK || (st = B.stage(ctx, b, n)) != ITS_OK) return st;
  DevBuf<unsigned char> diff;
  if ((st = diff.alloc(ctx, n)) != ITS_OK) return st;
  kCheckDivRn<<<gridFor(n, 256), 256, 0, ctx->stream>>>(A.d, B.d, n, diff.p);
  ITS_LAUNCHED(ctx);
  std::vector<unsigned char> h(n);
  ITS_CU(ctx, cudaMemcpyAsync(h.data(), diff.p, n, cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  int64_t c = 0;
  for (int64_t i = 0; i < n; ++i) c += h[i];
  *mismatches = c;
  return ITS_OK;
}

}  // extern "C"

namespace {
template <typename FT>
its_status marchingCubesT(its_ctx* ctx, const FT* field, int res, const double origin[3], const double width[3],
                          double iso, uint8_t* cube_index, double* tri_verts, int64_t capacity, int64_t* num_verts) {
  if (!ctx) return ITS_ERR_INVALID;
  if (!field || !origin || !width || res < 1 || res > 2048 || !num_verts)
    return setError(ctx, ITS_ERR_INVALID, "its_marching_cubes: bad arguments");
  if (tri_verts && capacity < 0) return setError(ctx, ITS_ERR_INVALID, "negative capacity");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  const int64_t M = (int64_t)res + 1, nvox = (int64_t)res * res * res;
  InArg<FT> F;
  OutArg<uint8_t> Cb;
  OutArg<double> T;
  its_status st;
  if ((st = F.stage(ctx, field, M * M * M)) != ITS_OK) return st;
  if ((st = Cb.stage(ctx, cube_index, nvox)) != ITS_OK) return st;
  if ((st = T.stage(ctx, tri_verts, tri_verts ? 3 * capacity : 0)) != ITS_OK) return st;
  McCaseT<FT> mc{F.d, res, iso};
  // case bytes: the caller's buffer when it is on the device, else scratch copied back
  DevBuf<uint8_t> cubeTmp;
  uint8_t* cubeD = Cb.d;
  if (!cubeD) {
    if ((st = cubeTmp.alloc(ctx, nvox)) != ITS_OK) return st;
    cubeD = cubeTmp.p;
  }
  // tile of 256 threads x ITEMS voxels; the autotuner picks ITEMS (same bits for every choice)
  const int itemsOf[3] = {8, 16, 4};
  const int64_t nbMax = (nvox + kScanThreads * 4 - 1) / (kScanThreads * 4);
  DevBuf<unsigned long long> sums, tot;
  if ((st = sums.alloc(ctx, nbMax + spineTops(nbMax))) != ITS_OK || (st = tot.alloc(ctx, 1)) != ITS_OK) return st;
  const double3 o3 = make_double3(origin[0], origin[1], origin[2]);
  const double3 v3 = make_double3(width[0] / res, width[1] / res, width[2] / res);
  auto run = [&](int i) -> its_status {
    const int items = itemsOf[i];
    const int64_t nb = (nvox + kScanThreads * items - 1) / (kScanThreads * items);
    if (items == 16)
      kMcClassify<FT, 16><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(F.d, res, iso, cubeD, sums.p);
    else if (items == 4)
      kMcClassify<FT, 4><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(F.d, res, iso, cubeD, sums.p);
    else if (res % 256 == 0)
      kMcClassifyRows<FT><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(F.d, res, iso, cubeD, sums.p);
    else
      kMcClassify<FT, 8><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(F.d, res, iso, cubeD, sums.p);
    ITS_LAUNCHED(ctx);
    if ((st = scanSpine<unsigned long long>(ctx, sums.p, nb, tot.p, sums.p + nbMax)) != ITS_OK) return st;
    if (T.d) {
      const unsigned long long cap = (unsigned long long)capacity;
      if (items == 16)
        kMcEmit<FT, 16><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(mc, o3, v3, cubeD, sums.p, tot.p, T.d, cap);
      else if (items == 4)
        kMcEmit<FT, 4><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(mc, o3, v3, cubeD, sums.p, tot.p, T.d, cap);
      else
        kMcEmit<FT, 8><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(mc, o3, v3, cubeD, sums.p, tot.p, T.d, cap);
      ITS_LAUNCHED(ctx);
    }
    return ITS_OK;
  };
  const std::string key = std::string("marching_cubes/") + (sizeof(FT) == 8 ? "f64" : "f32") + "/res=" +
                          std::to_string(res) + (T.d ? "/soup" : "/cases");
  int choice = 0;
  if ((st = tuneChoice(ctx, key, 3, 0, run, &choice)) != ITS_OK) return st;
  if ((st = run(choice)) != ITS_OK) return st;
  unsigned long long total = 0;
  if ((st = readScalar(ctx, tot.p, &total)) != ITS_OK) return st;
  *num_verts = (int64_t)total;
  // only the vertices written leave the device (the rest of a host buffer is left untouched)
  T.count = 3 * (size_t)std::min<int64_t>(capacity, (int64_t)total);
  if ((st = Cb.finish(ctx)) != ITS_OK) return st;
  if ((st = T.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}
}  // namespace

extern "C" {

its_status its_marching_cubes(its_ctx* ctx, const double* field, int res, const double origin[3],
                              const double width[3], double iso, uint8_t* cube_index, double* tri_verts,
                              int64_t capacity, int64_t* num_verts) {
  return marchingCubesT<double>(ctx, field, res, origin, width, iso, cube_index, tri_verts, capacity, num_verts);
}

its_status its_marching_cubes_f32(its_ctx* ctx, const float* field, int res, const double origin[3],
                                  const double width[3], double iso, uint8_t* cube_index, double* tri_verts,
                                  int64_t capacity, int64_t* num_verts) {
  return marchingCubesT<float>(ctx, field, res, origin, width, iso, cube_index, tri_verts, capacity, num_verts);
}

}  // extern "C"
