// Accelerated signed distance: a linear BVH over the triangles (Karras 2012: Morton codes of
// centroids, radix sort, binary radix tree, bottom-up boxes) answers
//   * the exact unsigned distance: nearest-first traversal with box lower bounds; a node is
//     skipped only when its box is farther than the best squared distance times (1 + 1e-12),
//     so the minimum is the same IEEE value the brute force finds (same per-triangle code);
//   * the sign from the fast winding number (Barill et al. 2018): a node farther than beta = 2
//     times its radius contributes the second-order expansion of its triangles' solid angles
//     about its area centroid (the area-weighted normal sum as a dipole, plus the tensor
//     M = sum_t an_t (c_t - c)^T), nearer nodes recurse, leaves add the exact solid angle.
//     libigl's signed_distance(FAST_WINDING_NUMBER), which the reference calls
//     (ThinShells.cpp:501), uses the same expansion order and accuracy scale; inside if w > 1/2.
#include <cmath>

#include "its_scan.cuh"
#include "its_sdf.cuh"
#include "its_sparse.cuh"
#include <vector>
#include <algorithm>

namespace its {

constexpr int kBvhStack = 64;
constexpr double kFwnBeta = 2.0;  // far-field test |q - c| > beta * r

struct BvhDevice {
  int64_t nf = 0;
  int32_t* left = nullptr;   // internal nodes: child index; >= 0 internal, < 0 leaf -(k+1)
  int32_t* right = nullptr;
  int32_t* parent = nullptr; // 2F-1 entries: internal 0..F-2, leaves F-1..2F-2
  uint32_t* leafTri = nullptr;
  double* lo = nullptr;      // 3 per node (2F-1)
  double* hi = nullptr;
  double* an = nullptr;      // area-weighted normal sum (3 per node)
  double* ac = nullptr;      // area-weighted centroid sum (3 per node)
  double* sm = nullptr;      // sum over the node's triangles of an_t c_t^T (9 per node, row-major)
  double* area = nullptr;
  unsigned* flag = nullptr;
  int32_t* range = nullptr;  // internal node i covers sorted leaves range[2i] .. range[2i+1]
};

// The traversal's view of the tree, in three arrays:
//   * TravNode, one 64-byte line per internal node: both children's boxes (FP32, rounded
//     outward, so a box distance from them is a lower bound of the exact box's) and the
//     children. A nearest-distance visit reads this one line; for 10^6 triangles the array
//     (64 MB) stays in L2.
//   * FwnNode, two lines per internal node: the fast winding number's expansion centre
//     (area-weighted centroid sum / area), squared radius (+inf for a node without area, which
//     the far-field test then never accepts), normal sum and second-order tensor.
//   * the leaves' triangles (9 doubles each, in leaf order).
// The FP64 values are those the traversal used to form per visit from the build's arrays
// (same operations), and a pruned node is one whose exact box is also beyond the best
// distance, so results are unchanged.
constexpr int kBucket = 4;  // a child whose subtree holds at most this many leaves is tested leaf by leaf
struct __align__(64) TravNode {
  float lo[2][3], hi[2][3];
  int32_t child[2];   // >= 0 internal, < 0 leaf -(k+1)
  uint32_t bucket[2]; // an internal child of <= kBucket leaves: (count << 29) | first leaf; else 0
};
static_assert(sizeof(TravNode) == 64, "one line per node");
struct __align__(64) FwnNode {
  double c[3];
  double r2;
  double an[3];
  double m[9];  // sum_t an_t (c_t - c)^T about the node's centre c
};
static_assert(sizeof(FwnNode) == 128, "two lines per node");

__global__ void kCentroidBounds(const double* __restrict__ V, const int32_t* __restrict__ F, int64_t nf,
                                double* __restrict__ partial) {
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nf; t += (int64_t)gridDim.x * blockDim.x) {
    for (int a = 0; a < 3; ++a) {
      const double c = (V[3 * F[3 * t] + a] + V[3 * F[3 * t + 1] + a] + V[3 * F[3 * t + 2] + a]) / 3.0;
      mn[a] = fmin(mn[a], c);
      mx[a] = fmax(mx[a], c);
    }
  }
  for (int a = 0; a < 3; ++a)
    for (int o = 16; o > 0; o >>= 1) {
      mn[a] = fmin(mn[a], __shfl_down_sync(0xffffffffu, mn[a], o));
      mx[a] = fmax(mx[a], __shfl_down_sync(0xffffffffu, mx[a], o));
    }
  __shared__ double s[8][6];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
    for (int a = 0; a < 3; ++a) { s[w][a] = mn[a]; s[w][3 + a] = mx[a]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
      for (int a = 0; a < 3; ++a) { mn[a] = fmin(mn[a], s[k][a]); mx[a] = fmax(mx[a], s[k][3 + a]); }
    for (int a = 0; a < 3; ++a) { partial[6 * blockIdx.x + a] = mn[a]; partial[6 * blockIdx.x + 3 + a] = mx[a]; }
  }
}

__global__ void kMortonCodes(const double* __restrict__ V, const int32_t* __restrict__ F, int64_t nf, double3 lo,
                             double3 inv, uint32_t* __restrict__ codes, uint32_t* __restrict__ idx) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nf) return;
  const double c[3] = {(V[3 * F[3 * t]] + V[3 * F[3 * t + 1]] + V[3 * F[3 * t + 2]]) / 3.0,
                       (V[3 * F[3 * t] + 1] + V[3 * F[3 * t + 1] + 1] + V[3 * F[3 * t + 2] + 1]) / 3.0,
                       (V[3 * F[3 * t] + 2] + V[3 * F[3 * t + 1] + 2] + V[3 * F[3 * t + 2] + 2]) / 3.0};
  const double L[3] = {lo.x, lo.y, lo.z}, I[3] = {inv.x, inv.y, inv.z};
  uint32_t q[3];
  for (int a = 0; a < 3; ++a) {
    const double u = (c[a] - L[a]) * I[a];
    q[a] = (uint32_t)fmin(fmax(u * 1024.0, 0.0), 1023.0);
  }
  codes[t] = mortonEncode(q[0], q[1], q[2]);
  idx[t] = (uint32_t)t;
}

// Length of the common prefix of keys i and j (index bits break ties), -1 out of range.
__device__ inline int delta(const uint32_t* codes, int64_t n, int64_t i, int64_t j) {
  if (j < 0 || j >= n) return -1;
  const uint32_t a = codes[i], b = codes[j];
  if (a != b) return __clz(a ^ b);
  return 32 + __clzll((unsigned long long)(i ^ j));
}

__global__ void kBuildInternal(const uint32_t* __restrict__ codes, int64_t n, int32_t* __restrict__ left,
                               int32_t* __restrict__ right, int32_t* __restrict__ parent, int32_t* __restrict__ range) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = delta(codes, n, i, i + 1) - delta(codes, n, i, i - 1) >= 0 ? 1 : -1;
  const int dmin = delta(codes, n, i, i - d);
  int64_t lmax = 2;
  while (delta(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int64_t l = 0;
  for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
  const int64_t j = i + l * d;
  const int dnode = delta(codes, n, i, j);
  int64_t s = 0;
  for (int64_t t = (l + 1) >> 1;; t = (t + 1) >> 1) {
    if (delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
    if (t == 1) break;
  }
  const int64_t g = i + s * d + (d < 0 ? d : 0);
  const int64_t lo = i < j ? i : j, hi = i < j ? j : i;
  const int32_t L = (lo == g) ? -(int32_t)(g + 1) : (int32_t)g;
  const int32_t R = (hi == g + 1) ? -(int32_t)(g + 2) : (int32_t)(g + 1);
  left[i] = L;
  right[i] = R;
  range[2 * i] = (int32_t)lo;
  range[2 * i + 1] = (int32_t)hi;
  parent[L < 0 ? (n - 1) + (-L - 1) : L] = (int32_t)i;
  parent[R < 0 ? (n - 1) + (-R - 1) : R] = (int32_t)i;
}

// Leaf data, then climb: the second child to arrive at a node merges both children.
__global__ void kBottomUp(const double* __restrict__ V, const int32_t* __restrict__ F, int64_t n,
                          const uint32_t* __restrict__ leafTri, BvhDevice B) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t node = (n - 1) + k;
  {
    const uint32_t t = leafTri[k];
    double p[3][3];
    for (int c = 0; c < 3; ++c)
      for (int a = 0; a < 3; ++a) p[c][a] = V[3 * F[3 * t + c] + a];
    const double u[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    const double v[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    const double nx = 0.5 * (u[1] * v[2] - u[2] * v[1]), ny = 0.5 * (u[2] * v[0] - u[0] * v[2]),
                 nz = 0.5 * (u[0] * v[1] - u[1] * v[0]);
    const double ar = sqrt(nx * nx + ny * ny + nz * nz);
    for (int a = 0; a < 3; ++a) {
      B.lo[3 * node + a] = fmin(p[0][a], fmin(p[1][a], p[2][a]));
      B.hi[3 * node + a] = fmax(p[0][a], fmax(p[1][a], p[2][a]));
      B.ac[3 * node + a] = ar * (p[0][a] + p[1][a] + p[2][a]) / 3.0;
    }
    const double an3[3] = {nx, ny, nz};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) B.sm[9 * node + 3 * i + j] = an3[i] * ((p[0][j] + p[1][j] + p[2][j]) / 3.0);
    B.an[3 * node] = nx;
    B.an[3 * node + 1] = ny;
    B.an[3 * node + 2] = nz;
    B.area[node] = ar;
  }
  __threadfence();
  while (true) {
    const int32_t par = B.parent[node];
    if (par < 0) break;
    if (atomicAdd(B.flag + par, 1u) == 0) return;  // first arrival: the sibling finishes the merge
    __threadfence();
    const int32_t L = B.left[par], R = B.right[par];
    const int64_t a = L < 0 ? (n - 1) + (-L - 1) : L, b = R < 0 ? (n - 1) + (-R - 1) : R;
    for (int c = 0; c < 3; ++c) {
      B.lo[3 * par + c] = fmin(((volatile double*)B.lo)[3 * a + c], ((volatile double*)B.lo)[3 * b + c]);
      B.hi[3 * par + c] = fmax(((volatile double*)B.hi)[3 * a + c], ((volatile double*)B.hi)[3 * b + c]);
      B.an[3 * par + c] = ((volatile double*)B.an)[3 * a + c] + ((volatile double*)B.an)[3 * b + c];
      B.ac[3 * par + c] = ((volatile double*)B.ac)[3 * a + c] + ((volatile double*)B.ac)[3 * b + c];
    }
    B.area[par] = ((volatile double*)B.area)[a] + ((volatile double*)B.area)[b];
    for (int e = 0; e < 9; ++e)
      B.sm[9 * par + e] = ((volatile double*)B.sm)[9 * a + e] + ((volatile double*)B.sm)[9 * b + e];
    __threadfence();
    node = par;
  }
}

__global__ void kPackNodes(const double* __restrict__ V, const int32_t* __restrict__ F, BvhDevice B,
                           TravNode* __restrict__ trav, FwnNode* __restrict__ fwn, double* __restrict__ tris) {
  const int64_t n = B.nf;
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= 2 * n - 1) return;
  if (k >= n - 1) {  // leaf: its triangle's corners
    const uint32_t t = B.leafTri[k - (n - 1)];
    double* dst = tris + 9 * (k - (n - 1));
    for (int c = 0; c < 3; ++c)
      for (int a = 0; a < 3; ++a) dst[3 * c + a] = V[3 * (int64_t)F[3 * t + c] + a];
    return;
  }
  TravNode r;
  const int32_t ch[2] = {B.left[k], B.right[k]};
  for (int j = 0; j < 2; ++j) {
    const int64_t cn = ch[j] < 0 ? (n - 1) + (-ch[j] - 1) : ch[j];
    for (int a = 0; a < 3; ++a) {
      r.lo[j][a] = __double2float_rd(B.lo[3 * cn + a]);
      r.hi[j][a] = __double2float_ru(B.hi[3 * cn + a]);
    }
    r.child[j] = ch[j];
    r.bucket[j] = 0;
    if (ch[j] >= 0) {
      const int32_t first = B.range[2 * ch[j]], count = B.range[2 * ch[j] + 1] - first + 1;
      if (count <= kBucket && first < (1 << 29)) r.bucket[j] = ((uint32_t)count << 29) | (uint32_t)first;
    }
  }
  trav[k] = r;
  FwnNode f;
  const double A = B.area[k];
  const double lo[3] = {B.lo[3 * k], B.lo[3 * k + 1], B.lo[3 * k + 2]};
  const double hi[3] = {B.hi[3 * k], B.hi[3 * k + 1], B.hi[3 * k + 2]};
  for (int a = 0; a < 3; ++a) {
    f.an[a] = B.an[3 * k + a];
    f.c[a] = A > 0.0 ? B.ac[3 * k + a] / A : 0.0;
  }
  f.r2 = __longlong_as_double(0x7ff0000000000000ll);  // +inf: no far-field term without area
  if (A > 0.0) {
    double r2 = 0.0;
    for (int a = 0; a < 3; ++a) {
      const double e = fmax(f.c[a] - lo[a], hi[a] - f.c[a]);
      r2 += e * e;
    }
    f.r2 = r2;
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) f.m[3 * i + j] = B.sm[9 * k + 3 * i + j] - f.an[i] * f.c[j];
  fwn[k] = f;
}

__device__ inline double boxDist2(const double* lo, const double* hi, const double* q) {
  double s = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double d = q[a] < lo[a] ? lo[a] - q[a] : (q[a] > hi[a] ? q[a] - hi[a] : 0.0);
    s = s + d * d;
  }
  return s;
}

// Squared distance from q to a box given in FP32 (promoted exactly to FP64).
__device__ inline double boxDist2f(const float* lo, const float* hi, const double* q) {
  double s = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double l = lo[a], h = hi[a];
    const double d = q[a] < l ? l - q[a] : (q[a] > h ? q[a] - h : 0.0);
    s = s + d * d;
  }
  return s;
}

// One query per thread, queries taken in the Morton order of their positions (order[i] is the
// i-th query), so that a warp's traversals follow nearby paths through the tree.
__global__ void __launch_bounds__(128) kSdfBvh(const double* __restrict__ P, int64_t m,
                                               const uint32_t* __restrict__ order, const TravNode* __restrict__ T,
                                               const FwnNode* __restrict__ W, const double* __restrict__ tris,
                                               int64_t n, double* __restrict__ out, unsigned* __restrict__ overflow) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= m) return;
  const int64_t i = order[s];
  const double q[3] = {P[3 * i], P[3 * i + 1], P[3 * i + 2]};
  const D3 qd{q[0], q[1], q[2]};
  auto tri = [&](int32_t leafCode, D3* t) {
    const double* v = tris + 9 * (int64_t)(-leafCode - 1);
    for (int c = 0; c < 3; ++c) t[c] = D3{v[3 * c], v[3 * c + 1], v[3 * c + 2]};
  };
  // exact unsigned distance: nearest-first, each stacked node with its box distance (tested
  // again against the best distance when popped)
  double best = 1.7976931348623157e308;
  int32_t stack[kBvhStack];
  double sdist[kBvhStack];
  int sp = 0;
  if (n == 1) {
    D3 t[3];
    tri(-1, t);
    best = pointTriSqDist(qd, t[0], t[1], t[2]);
  } else {
    stack[0] = 0;
    sdist[0] = 0.0;
    sp = 1;
    while (sp > 0) {
      --sp;
      if (sdist[sp] > best * (1.0 + 1e-12)) continue;
      const TravNode& nd = T[stack[sp]];
      const double dc[2] = {boxDist2f(nd.lo[0], nd.hi[0], q), boxDist2f(nd.lo[1], nd.hi[1], q)};
      const int32_t c[2] = {nd.child[0], nd.child[1]};
      const uint32_t bk[2] = {nd.bucket[0], nd.bucket[1]};
      const int first = dc[1] < dc[0] ? 1 : 0;
      for (int kk = 1; kk >= 0; --kk) {  // push the farther child first
        const int k = kk == 1 ? 1 - first : first;
        if (dc[k] > best * (1.0 + 1e-12)) continue;
        if (c[k] < 0) {
          D3 t[3];
          tri(c[k], t);
          best = fmin(best, pointTriSqDist(qd, t[0], t[1], t[2]));
        } else if (bk[k]) {  // a small subtree: its leaves' triangles directly
          const int32_t f0 = (int32_t)(bk[k] & ((1u << 29) - 1u)), cnt = (int32_t)(bk[k] >> 29);
          for (int32_t l = 0; l < cnt; ++l) {
            D3 t[3];
            tri(-(f0 + l) - 1, t);
            best = fmin(best, pointTriSqDist(qd, t[0], t[1], t[2]));
          }
        } else {
          if (sp >= kBvhStack) { atomicOr(overflow, 1u); continue; }
          stack[sp] = c[k];
          sdist[sp] = dc[k];
          ++sp;
        }
      }
    }
  }
  // fast winding number
  double w = 0.0;
  sp = 0;
  stack[sp++] = n == 1 ? -1 : 0;
  while (sp > 0) {
    const int32_t cur = stack[--sp];
    if (cur < 0) {
      D3 t[3];
      tri(cur, t);
      w += solidAngle(qd, t[0], t[1], t[2]);
      continue;
    }
    const FwnNode& nd = W[cur];
    const double d[3] = {nd.c[0] - q[0], nd.c[1] - q[1], nd.c[2] - q[2]};
    const double R2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (R2 > kFwnBeta * kFwnBeta * nd.r2) {  // the powers of 1/R from one reciprocal
      const double iR = 1.0 / sqrt(R2);
      const double iR2 = iR * iR, iR3 = iR2 * iR, iR5 = iR3 * iR2;
      const double* mm = nd.m;
      const double tr = mm[0] + mm[4] + mm[8];
      const double dmd = d[0] * (mm[0] * d[0] + mm[1] * d[1] + mm[2] * d[2]) +
                         d[1] * (mm[3] * d[0] + mm[4] * d[1] + mm[5] * d[2]) +
                         d[2] * (mm[6] * d[0] + mm[7] * d[1] + mm[8] * d[2]);
      w += (nd.an[0] * d[0] + nd.an[1] * d[1] + nd.an[2] * d[2]) * iR3 + (tr * iR3 - 3.0 * dmd * iR5);
      continue;
    }
    if (sp + 2 > kBvhStack) { atomicOr(overflow, 1u); continue; }
    stack[sp++] = T[cur].child[0];
    stack[sp++] = T[cur].child[1];
  }
  const double wn = w / (4.0 * 3.14159265358979323846);
  const double dist = sqrt(best);
  out[i] = (wn > 0.5) ? -dist : dist;
}

// Morton code of a query position in the triangles' centroid box (clamped), for the traversal order.
__global__ void kQueryCodes(const double* __restrict__ P, int64_t m, double3 lo, double3 inv,
                            uint32_t* __restrict__ codes, uint32_t* __restrict__ idx) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double L[3] = {lo.x, lo.y, lo.z}, I[3] = {inv.x, inv.y, inv.z};
  uint32_t qc[3];
  for (int a = 0; a < 3; ++a) {
    const double u = (P[3 * i + a] - L[a]) * I[a];
    qc[a] = (uint32_t)fmin(fmax(u * 1024.0, 0.0), 1023.0);
  }
  codes[i] = mortonEncode(qc[0], qc[1], qc[2]);
  idx[i] = (uint32_t)i;
}

its_status sdfBvh(its_ctx* ctx, const double* dP, int64_t m, const double* dV, const int32_t* dF, int64_t nf, double* dOut) {
  its_status st;
  const int64_t nodes = 2 * nf - 1;
  BvhDevice B;
  B.nf = nf;
  DevBuf<int32_t> left, right, parent;
  DevBuf<uint32_t> codes, idx, sc, leafTri, tk, tv;
  DevBuf<double> lo, hi, an, ac, area, smom;
  DevBuf<unsigned> flag, overflow;
  DevBuf<int32_t> range;
  if ((st = left.alloc(ctx, nf)) != ITS_OK || (st = right.alloc(ctx, nf)) != ITS_OK ||
      (st = parent.alloc(ctx, nodes)) != ITS_OK || (st = codes.alloc(ctx, nf)) != ITS_OK ||
      (st = idx.alloc(ctx, nf)) != ITS_OK || (st = sc.alloc(ctx, nf)) != ITS_OK ||
      (st = leafTri.alloc(ctx, nf)) != ITS_OK || (st = tk.alloc(ctx, nf)) != ITS_OK ||
      (st = tv.alloc(ctx, nf)) != ITS_OK || (st = lo.alloc(ctx, 3 * nodes)) != ITS_OK ||
      (st = hi.alloc(ctx, 3 * nodes)) != ITS_OK || (st = an.alloc(ctx, 3 * nodes)) != ITS_OK ||
      (st = ac.alloc(ctx, 3 * nodes)) != ITS_OK || (st = area.alloc(ctx, nodes)) != ITS_OK ||
      (st = smom.alloc(ctx, 9 * nodes)) != ITS_OK ||
      (st = flag.zeros(ctx, nf)) != ITS_OK || (st = overflow.zeros(ctx, 1)) != ITS_OK ||
      (st = range.alloc(ctx, 2 * nf)) != ITS_OK)
    return st;
  // centroid bounds for the Morton quantisation
  const unsigned pb = 256;
  DevBuf<double> part;
  if ((st = part.alloc(ctx, 6 * pb)) != ITS_OK) return st;
  kCentroidBounds<<<pb, 256, 0, ctx->stream>>>(dV, dF, nf, part.p);
  ITS_LAUNCHED(ctx);
  std::vector<double> hp(6 * pb);
  ITS_CU(ctx, cudaMemcpyAsync(hp.data(), part.p, 6 * pb * 8, cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  double bl[3] = {1e300, 1e300, 1e300}, bh[3] = {-1e300, -1e300, -1e300};
  for (unsigned k = 0; k < pb; ++k)
    for (int a = 0; a < 3; ++a) { bl[a] = std::min(bl[a], hp[6 * k + a]); bh[a] = std::max(bh[a], hp[6 * k + 3 + a]); }
  double inv[3];
  for (int a = 0; a < 3; ++a) inv[a] = bh[a] > bl[a] ? 1.0 / (bh[a] - bl[a]) : 0.0;
  kMortonCodes<<<gridFor(nf, 256), 256, 0, ctx->stream>>>(dV, dF, nf, make_double3(bl[0], bl[1], bl[2]),
                                                         make_double3(inv[0], inv[1], inv[2]), codes.p, idx.p);
  ITS_LAUNCHED(ctx);
  if ((st = radixSortPairs(ctx, codes.p, idx.p, sc.p, leafTri.p, tk.p, tv.p, nf, 30)) != ITS_OK) return st;
  B.left = left.p;
  B.right = right.p;
  B.parent = parent.p;
  B.leafTri = leafTri.p;
  B.lo = lo.p;
  B.hi = hi.p;
  B.an = an.p;
  B.ac = ac.p;
  B.area = area.p;
  B.sm = smom.p;
  B.flag = flag.p;
  B.range = range.p;
  ITS_CU(ctx, cudaMemsetAsync(parent.p, 0xFF, nodes * 4, ctx->stream));
  if (nf > 1) {
    kBuildInternal<<<gridFor(nf - 1, 256), 256, 0, ctx->stream>>>(sc.p, nf, left.p, right.p, parent.p, range.p);
    ITS_LAUNCHED(ctx);
  }
  kBottomUp<<<gridFor(nf, 256), 256, 0, ctx->stream>>>(dV, dF, nf, leafTri.p, B);
  ITS_LAUNCHED(ctx);
  DevBuf<TravNode> trav;
  DevBuf<FwnNode> fwn;
  DevBuf<double> tris;
  if ((st = trav.alloc(ctx, nf > 1 ? nf - 1 : 1)) != ITS_OK || (st = fwn.alloc(ctx, nf > 1 ? nf - 1 : 1)) != ITS_OK ||
      (st = tris.alloc(ctx, 9 * nf)) != ITS_OK)
    return st;
  kPackNodes<<<gridFor(nodes, 128), 128, 0, ctx->stream>>>(dV, dF, B, trav.p, fwn.p, tris.p);
  ITS_LAUNCHED(ctx);
  // the queries in Morton order (the tree's build buffers are reused for the sort)
  DevBuf<uint32_t> qc, qi, qsc, qorder, qtk, qtv;
  if ((st = qc.alloc(ctx, m)) != ITS_OK || (st = qi.alloc(ctx, m)) != ITS_OK || (st = qsc.alloc(ctx, m)) != ITS_OK ||
      (st = qorder.alloc(ctx, m)) != ITS_OK || (st = qtk.alloc(ctx, m)) != ITS_OK || (st = qtv.alloc(ctx, m)) != ITS_OK)
    return st;
  kQueryCodes<<<gridFor(m, 256), 256, 0, ctx->stream>>>(dP, m, make_double3(bl[0], bl[1], bl[2]),
                                                       make_double3(inv[0], inv[1], inv[2]), qc.p, qi.p);
  ITS_LAUNCHED(ctx);
  if ((st = radixSortPairs(ctx, qc.p, qi.p, qsc.p, qorder.p, qtk.p, qtv.p, m, 30)) != ITS_OK) return st;
  kSdfBvh<<<gridFor(m, 128), 128, 0, ctx->stream>>>(dP, m, qorder.p, trav.p, fwn.p, tris.p, nf, dOut,
                                                   overflow.p);
  ITS_LAUNCHED(ctx);
  unsigned ov = 0;
  ITS_CU(ctx, cudaMemcpyAsync(&ov, overflow.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  if (ov) return setError(ctx, ITS_ERR_INVALID, "BVH traversal stack overflow (degenerate triangle distribution)");
  return ITS_OK;
}

}  // namespace its
