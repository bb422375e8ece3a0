// CPU oracle (test infrastructure): the signed distance of ThinShells::cpSDFOfTreeNodes
// (ThinShells.cpp:481-509, libigl signed_distance with SIGNED_DISTANCE_TYPE_FAST_WINDING_NUMBER)
// restated with a linear BVH so that million-triangle meshes finish on the host in seconds:
//   * tree: Karras 2012 -- Morton codes of the triangle centroids quantised to 10 bits per axis
//     over the centroids' box, a stable sort by code (ties keep triangle order), the binary
//     radix tree over the sorted codes (index bits break equal codes), node boxes, area-weighted
//     normal sums and area-weighted centroid sums formed bottom-up as left + right;
//   * distance: the exact minimum over all triangles of the per-triangle squared distance
//     (pointTriSqDist, Ericson 5.1.5); subtrees whose box is farther than the best so far
//     (times 1 + 1e-12) are skipped, so the minimum is the brute force's IEEE value;
//   * sign: the fast winding number (Barill et al. 2018): a node whose area centroid c is
//     farther than beta = 2 times its box radius contributes the second-order expansion of its
//     triangles' solid angles about c -- the normal sum as a dipole plus the tensor
//     M = sum_t an_t (c_t - c)^T (formed as sum_t an_t c_t^T - AN c^T), the powers of 1/R from
//     one reciprocal of sqrt(R^2) -- nearer nodes recurse
//     (right child first), leaves add the exact solid angle; inside if w > 1/2.
// The same tree, the same traversal order and the same IEEE operations as libits' kSdfBvh, so
// distances are bit-identical and the winding numbers agree to the last bits of atan2.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "orc_fit.hpp"

namespace orc {
namespace {

constexpr double kBeta = 2.0;

struct Bvh {
  int64_t n = 0;
  std::vector<int32_t> left, right;  // internal nodes; child >= 0 internal, < 0 leaf -(k+1)
  std::vector<uint32_t> leafTri;
  std::vector<double> lo, hi, an, ac, area;  // 2n-1 nodes: internal 0..n-2, leaves n-1..2n-2
  std::vector<double> sm;                    // sum_t an_t c_t^T, 9 per node (row-major)
  int64_t nodeOf(int32_t c) const { return c < 0 ? (n - 1) + (-c - 1) : c; }
};

int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }
int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

int delta(const std::vector<uint32_t>& codes, int64_t n, int64_t i, int64_t j) {
  if (j < 0 || j >= n) return -1;
  const uint32_t a = codes[i], b = codes[j];
  if (a != b) return clz32(a ^ b);
  return 32 + clz64((uint64_t)(i ^ j));
}

V3 vert(const double* V, int32_t k) { return {V[3 * k], V[3 * k + 1], V[3 * k + 2]}; }

Bvh build(const double* V, const int32_t* F, int64_t nf) {
  Bvh B;
  B.n = nf;
  std::vector<double> cen(3 * nf);
  double bl[3] = {1e300, 1e300, 1e300}, bh[3] = {-1e300, -1e300, -1e300};
  for (int64_t t = 0; t < nf; ++t)
    for (int a = 0; a < 3; ++a) {
      const double c = (V[3 * F[3 * t] + a] + V[3 * F[3 * t + 1] + a] + V[3 * F[3 * t + 2] + a]) / 3.0;
      cen[3 * t + a] = c;
      bl[a] = std::min(bl[a], c);
      bh[a] = std::max(bh[a], c);
    }
  double inv[3];
  for (int a = 0; a < 3; ++a) inv[a] = bh[a] > bl[a] ? 1.0 / (bh[a] - bl[a]) : 0.0;
  std::vector<uint32_t> code(nf);
  for (int64_t t = 0; t < nf; ++t) {
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
      const double u = (cen[3 * t + a] - bl[a]) * inv[a];
      q[a] = (uint32_t)std::fmin(std::fmax(u * 1024.0, 0.0), 1023.0);
    }
    code[t] = mortonEncode(q[0], q[1], q[2]);
  }
  std::vector<uint32_t> order(nf);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return code[x] < code[y]; });
  std::vector<uint32_t> sc(nf);
  for (int64_t k = 0; k < nf; ++k) sc[k] = code[order[k]];
  B.leafTri = order;
  const int64_t nodes = 2 * nf - 1;
  B.left.assign(std::max<int64_t>(nf - 1, 0), 0);
  B.right.assign(std::max<int64_t>(nf - 1, 0), 0);
  for (int64_t i = 0; i + 1 < nf; ++i) {
    const int d = delta(sc, nf, i, i + 1) - delta(sc, nf, i, i - 1) >= 0 ? 1 : -1;
    const int dmin = delta(sc, nf, i, i - d);
    int64_t lmax = 2;
    while (delta(sc, nf, i, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
      if (delta(sc, nf, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(sc, nf, i, j);
    int64_t s = 0;
    for (int64_t t = (l + 1) >> 1;; t = (t + 1) >> 1) {
      if (delta(sc, nf, i, i + (s + t) * d) > dnode) s += t;
      if (t == 1) break;
    }
    const int64_t g = i + s * d + (d < 0 ? d : 0);
    const int64_t lo = std::min(i, j), hi = std::max(i, j);
    B.left[i] = (lo == g) ? -(int32_t)(g + 1) : (int32_t)g;
    B.right[i] = (hi == g + 1) ? -(int32_t)(g + 2) : (int32_t)(g + 1);
  }
  B.lo.assign(3 * nodes, 0.0);
  B.hi.assign(3 * nodes, 0.0);
  B.an.assign(3 * nodes, 0.0);
  B.ac.assign(3 * nodes, 0.0);
  B.area.assign(nodes, 0.0);
  B.sm.assign(9 * nodes, 0.0);
  for (int64_t k = 0; k < nf; ++k) {
    const int64_t node = (nf - 1) + k;
    const uint32_t t = B.leafTri[k];
    double p[3][3];
    for (int c = 0; c < 3; ++c)
      for (int a = 0; a < 3; ++a) p[c][a] = V[3 * F[3 * t + c] + a];
    const double u[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    const double v[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    const double nx = 0.5 * (u[1] * v[2] - u[2] * v[1]), ny = 0.5 * (u[2] * v[0] - u[0] * v[2]),
                 nz = 0.5 * (u[0] * v[1] - u[1] * v[0]);
    const double ar = std::sqrt(nx * nx + ny * ny + nz * nz);
    for (int a = 0; a < 3; ++a) {
      B.lo[3 * node + a] = std::fmin(p[0][a], std::fmin(p[1][a], p[2][a]));
      B.hi[3 * node + a] = std::fmax(p[0][a], std::fmax(p[1][a], p[2][a]));
      B.ac[3 * node + a] = ar * (p[0][a] + p[1][a] + p[2][a]) / 3.0;
    }
    B.an[3 * node] = nx;
    B.an[3 * node + 1] = ny;
    B.an[3 * node + 2] = nz;
    B.area[node] = ar;
    const double an3[3] = {nx, ny, nz};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) B.sm[9 * node + 3 * i + j] = an3[i] * ((p[0][j] + p[1][j] + p[2][j]) / 3.0);
  }
  // internal nodes bottom-up (children before parents: a post-order walk from the root)
  if (nf > 1) {
    std::vector<std::pair<int32_t, int>> st;
    st.push_back({0, 0});
    while (!st.empty()) {
      auto& top = st.back();
      const int32_t i = top.first;
      if (top.second == 0) {
        top.second = 1;
        if (B.left[i] >= 0) st.push_back({B.left[i], 0});
        if (B.right[i] >= 0) st.push_back({B.right[i], 0});
        continue;
      }
      st.pop_back();
      const int64_t a = B.nodeOf(B.left[i]), b = B.nodeOf(B.right[i]);
      for (int c = 0; c < 3; ++c) {
        B.lo[3 * i + c] = std::fmin(B.lo[3 * a + c], B.lo[3 * b + c]);
        B.hi[3 * i + c] = std::fmax(B.hi[3 * a + c], B.hi[3 * b + c]);
        B.an[3 * i + c] = B.an[3 * a + c] + B.an[3 * b + c];
        B.ac[3 * i + c] = B.ac[3 * a + c] + B.ac[3 * b + c];
      }
      B.area[i] = B.area[a] + B.area[b];
      for (int e = 0; e < 9; ++e) B.sm[9 * i + e] = B.sm[9 * a + e] + B.sm[9 * b + e];
    }
  }
  return B;
}

double boxDist2(const double* lo, const double* hi, const double* q) {
  double s = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double d = q[a] < lo[a] ? lo[a] - q[a] : (q[a] > hi[a] ? q[a] - hi[a] : 0.0);
    s = s + d * d;
  }
  return s;
}

double queryOne(const Bvh& B, const double* V, const int32_t* F, const double* q, std::vector<int32_t>& stack) {
  const int64_t n = B.n;
  const V3 qd{q[0], q[1], q[2]};
  auto tri = [&](int64_t node, V3* t) {
    const uint32_t ti = B.leafTri[node - (n - 1)];
    for (int c = 0; c < 3; ++c) t[c] = vert(V, F[3 * ti + c]);
  };
  double best = kDInf;
  stack.clear();
  if (n == 1) {
    V3 t[3];
    tri(0, t);
    best = pointTriSqDist(qd, t[0], t[1], t[2]);
  } else {
    stack.push_back(0);
    while (!stack.empty()) {
      const int64_t node = stack.back();
      stack.pop_back();
      if (boxDist2(&B.lo[3 * node], &B.hi[3 * node], q) > best * (1.0 + 1e-12)) continue;
      const int32_t c[2] = {B.left[node], B.right[node]};
      double dc[2];
      for (int k = 0; k < 2; ++k) {
        const int64_t cn = B.nodeOf(c[k]);
        dc[k] = boxDist2(&B.lo[3 * cn], &B.hi[3 * cn], q);
      }
      const int first = dc[1] < dc[0] ? 1 : 0;
      for (int kk = 1; kk >= 0; --kk) {
        const int k = kk == 1 ? 1 - first : first;
        if (dc[k] > best * (1.0 + 1e-12)) continue;
        if (c[k] < 0) {
          V3 t[3];
          tri(B.nodeOf(c[k]), t);
          best = std::fmin(best, pointTriSqDist(qd, t[0], t[1], t[2]));
        } else {
          stack.push_back(c[k]);
        }
      }
    }
  }
  double w = 0.0;
  stack.clear();
  stack.push_back(n == 1 ? -1 : 0);
  while (!stack.empty()) {
    const int32_t cur = stack.back();
    stack.pop_back();
    const int64_t node = B.nodeOf(cur);
    if (cur < 0) {
      V3 t[3];
      tri(node, t);
      w += solidAngle(qd, t[0], t[1], t[2]);
      continue;
    }
    const double A = B.area[node];
    const double* lo = &B.lo[3 * node];
    const double* hi = &B.hi[3 * node];
    if (A > 0.0) {
      const double c[3] = {B.ac[3 * node] / A, B.ac[3 * node + 1] / A, B.ac[3 * node + 2] / A};
      double r2 = 0.0;
      for (int a = 0; a < 3; ++a) {
        const double e = std::fmax(c[a] - lo[a], hi[a] - c[a]);
        r2 += e * e;
      }
      const double d[3] = {c[0] - q[0], c[1] - q[1], c[2] - q[2]};
      const double R2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (R2 > kBeta * kBeta * r2) {
        const double iR = 1.0 / std::sqrt(R2);
        const double iR2 = iR * iR, iR3 = iR2 * iR, iR5 = iR3 * iR2;
        double m[9];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) m[3 * i + j] = B.sm[9 * node + 3 * i + j] - B.an[3 * node + i] * c[j];
        const double tr = m[0] + m[4] + m[8];
        const double dmd = d[0] * (m[0] * d[0] + m[1] * d[1] + m[2] * d[2]) +
                           d[1] * (m[3] * d[0] + m[4] * d[1] + m[5] * d[2]) +
                           d[2] * (m[6] * d[0] + m[7] * d[1] + m[8] * d[2]);
        w += (B.an[3 * node] * d[0] + B.an[3 * node + 1] * d[1] + B.an[3 * node + 2] * d[2]) * iR3 +
             (tr * iR3 - 3.0 * dmd * iR5);
        continue;
      }
    }
    stack.push_back(B.left[node]);
    stack.push_back(B.right[node]);
  }
  const double wn = w / (4.0 * 3.14159265358979323846);
  const double dist = std::sqrt(best);
  return (wn > 0.5) ? -dist : dist;
}

}  // namespace

void signedDistanceBvh(const double* P, int64_t m, const double* V, const int32_t* F, int64_t nf, double* out) {
  if (nf <= 0) {
    for (int64_t i = 0; i < m; ++i) out[i] = kDInf;
    return;
  }
  const Bvh B = build(V, F, nf);
#pragma omp parallel
  {
    std::vector<int32_t> stack;
    stack.reserve(256);
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < m; ++i) out[i] = queryOne(B, V, F, P + 3 * i, stack);
  }
}

}  // namespace orc
