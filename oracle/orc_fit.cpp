// CPU oracle (test infrastructure): shell samples, signed-distance RHS, basis assembly,
// LSCG, field evaluation and marching cubes. Restates ThinShells.cpp:38-755,
// CUDACompute.cu:435-510 and MarchingCubes.cu:72-377 of the reference on the CPU.
#include "orc_fit.hpp"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <set>
#include <stdexcept>
#include <unordered_map>

namespace orc {

namespace {
struct TolLess {  // std::less<V3d> of the reference (BasicDataType.h:44-56)
  bool operator()(const V3& a, const V3& b) const { return lessPoint(a, b) == 1; }
};
using VertMap = std::map<V3, size_t, TolLess>;

std::vector<VertMap> depthVert2Idx(const Svo& s) {
  std::vector<VertMap> m(s.treeDepth);
  for (int d = 0; d < s.treeDepth; ++d)
    for (size_t i = 0; i < s.depthVerts[d].size(); ++i)
      m[d].emplace(s.depthVerts[d][i].pos, s.esumVerts[d] + i);
  return m;
}

V3 cornerOf(const Node& n, int k) {
  return {n.origin.x + n.width * (double)(k & 1), n.origin.y + n.width * (double)((k >> 1) & 1),
          n.origin.z + n.width * (double)((k >> 2) & 1)};
}
inline bool inRange(double l, double r, double q) { return l <= q && q <= r; }
inline bool isLargeDouble(double l, double r, double eps) { return !(std::fabs(l - r) < eps) && l > r; }
}  // namespace

// ---- shell samples: ThinShells::cpIntersectionPoints (ThinShells.cpp:38-479) ----------
std::vector<V3> intersections(const Svo& s, const double* V, int64_t nv, const int32_t* F, int64_t nf,
                              size_t* nEdgePoints) {
  (void)nv;
  // BaseModel::extractEdges (BaseModel.cpp:291-313): sorted unique (min,max) pairs.
  std::set<std::pair<int, int>> uset;
  for (int64_t t = 0; t < nf; ++t) {
    int a = F[3 * t], b = F[3 * t + 1], c = F[3 * t + 2];
    int mx = std::max(a, std::max(b, c)), mn = std::min(a, std::min(b, c)), md = a + b + c - mx - mn;
    uset.insert({mn, md});
    uset.insert({md, mx});
    uset.insert({mn, mx});
  }
  std::map<uint32_t, size_t> morton2Fine;
  for (size_t i = 0; i < s.numFineNodes; ++i) morton2Fine.emplace(s.nodes[i].morton, i);
  const V3 org = s.gridOrigin;
  const double vw = s.nodes[0].width;
  const int gsz = s.res;
  auto pointDis = [&](const V3& p, int out[3]) {
    for (int a = 0; a < 3; ++a) out[a] = (int)((p[a] - org[a]) / vw);
  };

  std::vector<std::pair<int, int>> edges(uset.begin(), uset.end());
  std::vector<std::vector<V3>> perEdge(edges.size());
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < (int64_t)edges.size(); ++i) {
    const V3 p1{V[3 * edges[i].first], V[3 * edges[i].first + 1], V[3 * edges[i].first + 2]};
    const V3 p2{V[3 * edges[i].second], V[3 * edges[i].second + 1], V[3 * edges[i].second + 2]};
    const V3 dir = p2 - p1;
    int d1[3], d2[3], lo[3], hi[3];
    pointDis(p1, d1);
    pointDis(p2, d2);
    for (int a = 0; a < 3; ++a) {
      lo[a] = clampi(std::min(d1[a], d2[a]) - 1, 0, gsz - 1);
      hi[a] = clampi(std::max(d1[a], d2[a]) + 1, 0, gsz - 1);
    }
    std::vector<V3>& out = perEdge[i];
    for (int z = lo[2]; z <= hi[2]; ++z)
      for (int y = lo[1]; y <= hi[1]; ++y)
        for (int x = lo[0]; x <= hi[0]; ++x) {
          auto it = morton2Fine.find(mortonEncode(x, y, z));
          if (it == morton2Fine.end()) continue;
          const V3 lbb = s.nodes[it->second].origin;
          const double w = s.nodes[it->second].width;
          double back_t = kDInf, left_t = kDInf, bottom_t = kDInf;
          if (dir.x != 0) back_t = (lbb.x - p1.x) / dir.x;
          if (dir.y != 0) left_t = (lbb.y - p1.y) / dir.y;
          if (dir.z != 0) bottom_t = (lbb.z - p1.z) / dir.z;
          auto at = [&](double t) { return V3{p1.x + t * dir.x, p1.y + t * dir.y, p1.z + t * dir.z}; };
          if (inRange(0.0, 1.0, back_t)) {
            V3 q = at(back_t);
            if (inRange(lbb.y, lbb.y + w, q.y) && inRange(lbb.z, lbb.z + w, q.z)) out.push_back(q);
          }
          if (inRange(0.0, 1.0, left_t)) {
            V3 q = at(left_t);
            if (inRange(lbb.x, lbb.x + w, q.x) && inRange(lbb.z, lbb.z + w, q.z)) out.push_back(q);
          }
          if (inRange(0.0, 1.0, bottom_t)) {
            V3 q = at(bottom_t);
            if (inRange(lbb.x, lbb.x + w, q.x) && inRange(lbb.y, lbb.y + w, q.y)) out.push_back(q);
          }
        }
  }
  std::vector<V3> edgePts;
  for (auto& v : perEdge) edgePts.insert(edgePts.end(), v.begin(), v.end());
  std::sort(edgePts.begin(), edgePts.end(), TolLess());
  edgePts.erase(std::unique(edgePts.begin(), edgePts.end(),
                            [](const V3& a, const V3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }),
                edgePts.end());
  if (nEdgePoints) *nEdgePoints = edgePts.size();

  // Face step: fine-node edges per axis, swept against each triangle.
  std::vector<EdgeRec> ax[3];
  for (const EdgeRec& e : s.edges) {
    EdgeRec t = e;
    if (lessPoint(t.p0, t.p1) != 1) std::swap(t.p0, t.p1);
    int axis;
    if (std::fabs(t.p0.y - t.p1.y) < 1e-9 && std::fabs(t.p0.z - t.p1.z) < 1e-9) axis = 0;
    else if (std::fabs(t.p0.x - t.p1.x) < 1e-9 && std::fabs(t.p0.z - t.p1.z) < 1e-9) axis = 1;
    else axis = 2;
    ax[axis].push_back(t);
  }
  // x_sortEdge / y_sortEdge / z_sortEdge (ThinShells.cpp:170-207) on the second end point.
  const int order[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};
  for (int a = 0; a < 3; ++a) {
    const int* o = order[a];
    std::sort(ax[a].begin(), ax[a].end(), [o](const EdgeRec& p, const EdgeRec& q) {
      if (std::fabs(p.p1[o[0]] - q.p1[o[0]]) < 1e-9) {
        if (std::fabs(p.p1[o[1]] - q.p1[o[1]]) < 1e-9) return p.p1[o[2]] < q.p1[o[2]];
        return p.p1[o[1]] < q.p1[o[1]];
      }
      return p.p1[o[0]] < q.p1[o[0]];
    });
  }
  std::vector<double> nrm(3 * nf), area(nf), dirv(nf);
  triAttributes(V, F, nf, nrm.data(), area.data(), dirv.data());
  std::vector<std::vector<V3>> perTri(nf);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t t = 0; t < nf; ++t) {
    const V3 p1{V[3 * F[3 * t]], V[3 * F[3 * t] + 1], V[3 * F[3 * t] + 2]};
    const V3 p2{V[3 * F[3 * t + 1]], V[3 * F[3 * t + 1] + 1], V[3 * F[3 * t + 1] + 2]};
    const V3 p3{V[3 * F[3 * t + 2]], V[3 * F[3 * t + 2] + 1], V[3 * F[3 * t + 2] + 2]};
    const V3 te1 = p2 - p1, te2 = p3 - p2, te3 = p1 - p3;
    const V3 tn{nrm[3 * t], nrm[3 * t + 1], nrm[3 * t + 2]};
    const double tdir = dirv[t];
    const V3 bo = vmin(p1, vmin(p2, p3)), be = vmax(p1, vmax(p2, p3));
    for (int a = 0; a < 3; ++a) {
      const std::vector<EdgeRec>& L = ax[a];
      // lower_bound with lessXVal: first edge whose second point is not below bo[a] (1e-9).
      auto lower = std::lower_bound(L.begin(), L.end(), bo[a], [a](const EdgeRec& e, double q) {
        return isLargeDouble(q, e.p1[a], 1e-9);
      });
      for (auto it = lower; it != L.end(); ++it) {
        const V3 ep1 = it->p0, ep2 = it->p1;
        if (isLargeDouble(ep1[a], be[a], 1e-9)) break;
        const V3 ed = ep2 - ep1;
        const double nd = dot3(tn, ed);
        if ((double)std::fabs((float)nd) < 1e-9) continue;  // fabsf on a double (ThinShells.cpp:268)
        const double tt = (-tdir - dot3(tn, ep1)) / nd;
        if (tt < 0. || tt > 1.) continue;
        const V3 ip = ep1 + ed * tt;
        if (dot3(cross3(te1, ip - p1), tn) < 0) continue;
        if (dot3(cross3(te2, ip - p2), tn) < 0) continue;
        if (dot3(cross3(te3, ip - p3), tn) < 0) continue;
        perTri[t].push_back(ip);
      }
    }
  }
  std::vector<V3> all = edgePts;
  for (auto& v : perTri) all.insert(all.end(), v.begin(), v.end());
  return all;
}

// ---- RHS: signed distance at the corner vertices (ThinShells.cpp:481-509) -------------
// libigl's signed_distance(FAST_WINDING_NUMBER) is not available; this restates it as the
// exact point-triangle distance (Ericson, Real-Time Collision Detection 5.1.5) with the
// sign of the exact generalised winding number (Jacobson et al. 2013): inside if w > 0.5.
double pointTriSqDist(const V3& p, const V3& a, const V3& b, const V3& c) {
  const V3 ab = b - a, ac = c - a, ap = p - a;
  const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return dot3(ap, ap);
  const V3 bp = p - b;
  const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) return dot3(bp, bp);
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
    const double v = d1 / (d1 - d3);
    const V3 q = p - (a + ab * v);
    return dot3(q, q);
  }
  const V3 cp = p - c;
  const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return dot3(cp, cp);
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
    const double w = d2 / (d2 - d6);
    const V3 q = p - (a + ac * w);
    return dot3(q, q);
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
    const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    const V3 q = p - (b + (c - b) * w);
    return dot3(q, q);
  }
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom, w = vc * denom;
  const V3 q = p - (a + ab * v + ac * w);
  return dot3(q, q);
}
// Solid angle of triangle (a,b,c) seen from p (Van Oosterom & Strackee 1983).
double solidAngle(const V3& p, const V3& a0, const V3& b0, const V3& c0) {
  const V3 a = a0 - p, b = b0 - p, c = c0 - p;
  const double la = std::sqrt(dot3(a, a)), lb = std::sqrt(dot3(b, b)), lc = std::sqrt(dot3(c, c));
  const double num = dot3(a, cross3(b, c));
  const double den = la * lb * lc + dot3(a, b) * lc + dot3(b, c) * la + dot3(c, a) * lb;
  return 2.0 * std::atan2(num, den);
}
void signedDistance(const double* P, int64_t m, const double* V, const int32_t* F, int64_t nf, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < m; ++i) {
    const V3 p{P[3 * i], P[3 * i + 1], P[3 * i + 2]};
    double best = kDInf, wsum = 0.0;
    for (int64_t t = 0; t < nf; ++t) {
      const V3 a{V[3 * F[3 * t]], V[3 * F[3 * t] + 1], V[3 * F[3 * t] + 2]};
      const V3 b{V[3 * F[3 * t + 1]], V[3 * F[3 * t + 1] + 1], V[3 * F[3 * t + 1] + 2]};
      const V3 c{V[3 * F[3 * t + 2]], V[3 * F[3 * t + 2] + 1], V[3 * F[3 * t + 2] + 2]};
      best = std::min(best, pointTriSqDist(p, a, b, c));
      wsum += solidAngle(p, a, b, c);
    }
    const double w = wsum / (4.0 * M_PI);
    const double d = std::sqrt(best);
    out[i] = (w > 0.5) ? -d : d;
  }
}

// ---- operator assembly: ThinShells::cpCoefficients (ThinShells.cpp:511-606) ----------
// Row v: the diagonal 1, coincident finer vertices (value 1, the chain stops at the first
// depth without one), and the hat values of the 8 corners of every ancestor of v's owner
// node (SparseVoxelOctree::setInDomainPoints, SVO.cu:1160-1193). Returned as CSR with
// ascending columns (Eigen's setFromTriplets sorts; no duplicates arise).
Csr assemble(const Svo& s) {
  const std::vector<VertMap> m = depthVert2Idx(s);
  const size_t n = s.numVerts;
  std::vector<std::vector<std::pair<int32_t, double>>> rows(n);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t r = 0; r < (int64_t)n; ++r) {
    int d = 0;
    while (s.esumVerts[d + 1] <= (size_t)r) ++d;
    const VertexRec& vr = s.depthVerts[d][r - s.esumVerts[d]];
    const size_t row = m[d].at(vr.pos);
    auto& R = rows[row];
    R.push_back({(int32_t)row, 1.0});
    for (int j = d - 1; j >= 0; --j) {
      auto it = m[j].find(vr.pos);
      if (it == m[j].end()) break;
      R.push_back({(int32_t)it->second, 1.0});
    }
    uint32_t nodeIdx = s.nodes[vr.owner].parent;
    int depth = d + 1;
    while (depth < s.treeDepth && nodeIdx != kNone) {
      const Node& nd = s.nodes[nodeIdx];
      for (int k = 0; k < 8; ++k) {
        const V3 c = cornerOf(nd, k);
        const size_t col = m[depth].at(c);
        const double val = baseFunction4Point(c, nd.width, vr.pos);
        if (val != 0) R.push_back({(int32_t)col, val});
      }
      nodeIdx = nd.parent;
      ++depth;
    }
    std::sort(R.begin(), R.end());
  }
  Csr A;
  A.n = (int64_t)n;
  A.rowptr.assign(n + 1, 0);
  for (size_t r = 0; r < n; ++r) A.rowptr[r + 1] = A.rowptr[r] + (int64_t)rows[r].size();
  A.col.resize(A.rowptr[n]);
  A.val.resize(A.rowptr[n]);
  for (size_t r = 0; r < n; ++r)
    for (size_t k = 0; k < rows[r].size(); ++k) {
      A.col[A.rowptr[r] + k] = rows[r][k].first;
      A.val[A.rowptr[r] + k] = rows[r][k].second;
    }
  return A;
}

Csr transpose(const Csr& A) {  // stable: rows ascending inside each column
  Csr T;
  T.n = A.n;
  T.rowptr.assign(A.n + 1, 0);
  for (int32_t c : A.col) T.rowptr[c + 1]++;
  for (int64_t i = 0; i < A.n; ++i) T.rowptr[i + 1] += T.rowptr[i];
  T.col.resize(A.col.size());
  T.val.resize(A.val.size());
  std::vector<int64_t> fill(T.rowptr.begin(), T.rowptr.end() - 1);
  for (int64_t r = 0; r < A.n; ++r)
    for (int64_t k = A.rowptr[r]; k < A.rowptr[r + 1]; ++k) {
      const int64_t dst = fill[A.col[k]]++;
      T.col[dst] = (int32_t)r;
      T.val[dst] = A.val[k];
    }
  return T;
}

// ---- LSCG: Eigen::LeastSquaresConjugateGradient (ThinShells.cpp:615-617) ------------
// Eigen 3.x LeastSquaresConjugateGradient (version unpinned: the reference vendors no
// Eigen): CGLS with the LeastSquareDiagonalPreconditioner (inverse squared column norms,
// 1 for empty columns), initial guess x (zero for solve()), stop when
// ||A^T r||^2 < tol^2 ||A^T b||^2 (stop == 0) or ||r||^2 < tol^2 ||b||^2 (stop == 1).
// Vector reductions here are sequential left-to-right sums.
static void spmv(const Csr& A, const double* x, double* y) {
#pragma omp parallel for schedule(static, 4096)
  for (int64_t r = 0; r < A.n; ++r) {
    double s = 0.0;
    for (int64_t k = A.rowptr[r]; k < A.rowptr[r + 1]; ++k) s += A.val[k] * x[A.col[k]];
    y[r] = s;
  }
}
static double dotv(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}
CglsReport cgls(const Csr& A, const Csr& T, const double* b, double* x, double tol, int64_t maxIters, int stop) {
  const int64_t n = A.n;
  CglsReport rep{};
  std::vector<double> invdiag(n), res(n), nres(n), p(n), z(n), tmp(n), atb(n);
  for (int64_t j = 0; j < n; ++j) {
    double sum = 0.0;
    bool first = true;
    for (int64_t k = T.rowptr[j]; k < T.rowptr[j + 1]; ++k) {
      const double a2 = T.val[k] * T.val[k];
      sum = first ? a2 : sum + a2;
      first = false;
    }
    invdiag[j] = sum > 0.0 ? 1.0 / sum : 1.0;
  }
  spmv(A, x, tmp.data());
  for (int64_t i = 0; i < n; ++i) res[i] = b[i] - tmp[i];
  spmv(T, res.data(), nres.data());
  spmv(T, b, atb.data());
  const double rhsNorm2 = dotv(atb, atb);
  double bNorm2 = 0.0;
  for (int64_t i = 0; i < n; ++i) bNorm2 += b[i] * b[i];
  rep.rhs_norm2 = rhsNorm2;
  if (rhsNorm2 == 0) {
    for (int64_t i = 0; i < n; ++i) x[i] = 0.0;
    rep.converged = 1;
    return rep;
  }
  const double threshold = stop == 0 ? tol * tol * rhsNorm2 : tol * tol * bNorm2;
  auto measure = [&]() { return stop == 0 ? dotv(nres, nres) : dotv(res, res); };
  double residualNorm2 = measure();
  rep.normal_residual_norm2 = dotv(nres, nres);
  if (residualNorm2 < threshold) {
    rep.converged = 1;
    rep.iterations = 0;
  } else {
    for (int64_t i = 0; i < n; ++i) p[i] = invdiag[i] * nres[i];
    double absNew = dotv(nres, p);
    int64_t i = 0;
    while (i < maxIters) {
      spmv(A, p.data(), tmp.data());
      const double tn = dotv(tmp, tmp);
      if (!(tn > 0.0)) { rep.breakdown = 1; break; }
      const double alpha = absNew / tn;
      for (int64_t k = 0; k < n; ++k) x[k] += alpha * p[k];
      for (int64_t k = 0; k < n; ++k) res[k] -= alpha * tmp[k];
      spmv(T, res.data(), nres.data());
      residualNorm2 = measure();
      if (residualNorm2 < threshold) { rep.converged = 1; break; }
      for (int64_t k = 0; k < n; ++k) z[k] = invdiag[k] * nres[k];
      const double absOld = absNew;
      absNew = dotv(nres, z);
      const double beta = absNew / absOld;
      for (int64_t k = 0; k < n; ++k) p[k] = z[k] + beta * p[k];
      ++i;
    }
    rep.iterations = i;
    rep.normal_residual_norm2 = dotv(nres, nres);
  }
  spmv(A, x, tmp.data());
  double rn = 0.0;
  for (int64_t k = 0; k < n; ++k) rn += (b[k] - tmp[k]) * (b[k] - tmp[k]);
  rep.rel_residual = bNorm2 > 0 ? std::sqrt(rn / bNorm2) : 0.0;
  rep.normal_rel_residual = std::sqrt(rep.normal_residual_norm2 / rhsNorm2);
  return rep;
}

// ---- field at points through the owner chain (ThinShells.cpp:655-755) ----------------
void evalPoints(const Svo& s, const double* lambda, const double* P, int64_t m, double* out, uint8_t* missing) {
  const std::vector<VertMap> vm = depthVert2Idx(s);
  std::map<uint32_t, size_t> morton2Fine;
  for (size_t i = 0; i < s.numFineNodes; ++i) morton2Fine.emplace(s.nodes[i].morton, i);
  const double vw = s.nodes[0].width;
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < m; ++i) {
    const V3 p{P[3 * i], P[3 * i + 1], P[3 * i + 2]};
    int dis[3];
    for (int a = 0; a < 3; ++a) dis[a] = (int)((p[a] - s.gridOrigin[a]) / vw);
    auto it = morton2Fine.find(mortonEncode((uint16_t)dis[0], (uint16_t)dis[1], (uint16_t)dis[2]));
    if (it == morton2Fine.end()) {  // std::map::at would throw in the reference
      out[i] = 0.0;
      if (missing) missing[i] = 1;
      continue;
    }
    if (missing) missing[i] = 0;
    double sum = 0.0;
    uint32_t nodeIdx = (uint32_t)it->second;
    int depth = 0;
    while (depth < s.treeDepth && nodeIdx != kNone) {
      const Node& nd = s.nodes[nodeIdx];
      for (int k = 0; k < 8; ++k) {
        const V3 c = cornerOf(nd, k);
        sum += lambda[vm[depth].at(c)] * baseFunction4Point(c, nd.width, p);
      }
      nodeIdx = nd.parent;
      ++depth;
    }
    out[i] = sum;
  }
}

void pointValGradient(const Svo& s, const double* lambda, const double* P, const double* before, int64_t m,
                      const double boxOrigin[3], const double boxEnd[3], double* val, double* grad, uint8_t* missing) {
  const std::vector<VertMap> vm = depthVert2Idx(s);
  std::map<uint32_t, size_t> morton2Fine;
  for (size_t i = 0; i < s.numFineNodes; ++i) morton2Fine.emplace(s.nodes[i].morton, i);
  const double vw = s.nodes[0].width;
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < m; ++i) {
    V3 p{P[3 * i], P[3 * i + 1], P[3 * i + 2]};
    if (before) {
      const V3 b{before[3 * i], before[3 * i + 1], before[3 * i + 2]};
      for (int it = 0; it < 64; ++it) {
        bool out = false;
        for (int a = 0; a < 3; ++a) out = out || p[a] < boxOrigin[a] || p[a] > boxEnd[a];
        if (!out) break;
        for (int a = 0; a < 3; ++a) p[a] = (p[a] + b[a]) / 2.0;
      }
    }
    int dis[3];
    for (int a = 0; a < 3; ++a) dis[a] = (int)((p[a] - s.gridOrigin[a]) / vw);
    val[i] = 0.0;
    grad[3 * i] = grad[3 * i + 1] = grad[3 * i + 2] = 0.0;
    const bool inGrid = dis[0] >= 0 && dis[1] >= 0 && dis[2] >= 0 && dis[0] < s.res && dis[1] < s.res && dis[2] < s.res;
    auto it = inGrid ? morton2Fine.find(mortonEncode((uint16_t)dis[0], (uint16_t)dis[1], (uint16_t)dis[2]))
                     : morton2Fine.end();
    if (it == morton2Fine.end()) {
      if (missing) missing[i] = 1;
      continue;
    }
    if (missing) missing[i] = 0;
    double sum = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    uint32_t nodeIdx = (uint32_t)it->second;
    int depth = 0;
    while (depth < s.treeDepth && nodeIdx != kNone) {
      const Node& nd = s.nodes[nodeIdx];
      const double w = nd.width;
      for (int k = 0; k < 8; ++k) {
        const V3 c = cornerOf(nd, k);
        const double lam = lambda[vm[depth].at(c)];
        sum += lam * baseFunction4Point(c, w, p);
        const double bx = baseFunction(p.x, c.x, w), by = baseFunction(p.y, c.y, w), bz = baseFunction(p.z, c.z, w);
        gx += lam * (deBaseFunction(p.x, c.x, w) * by * bz);
        gy += lam * (bx * deBaseFunction(p.y, c.y, w) * bz);
        gz += lam * (bx * by * deBaseFunction(p.z, c.z, w));
      }
      nodeIdx = nd.parent;
      ++depth;
    }
    val[i] = sum;
    grad[3 * i] = gx;
    grad[3 * i + 1] = gy;
    grad[3 * i + 2] = gz;
  }
}

// Brute-force field (CUDACompute.cu:435-510 semantics): sum over every corner vertex,
// in index order; width = width of the vertex's owner node.
void evalBrute(const Svo& s, const double* lambda, const double* P, int64_t m, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < m; ++i) {
    const V3 p{P[3 * i], P[3 * i + 1], P[3 * i + 2]};
    double sum = 0.0;
    for (int d = 0; d < s.treeDepth; ++d)
      for (size_t j = 0; j < s.depthVerts[d].size(); ++j) {
        const VertexRec& v = s.depthVerts[d][j];
        sum += lambda[s.esumVerts[d] + j] * baseFunction4Point(v.pos, s.nodes[v.owner].width, p);
      }
    out[i] = sum;
  }
}

// Dense field on the (R+1)^3 MC lattice, the sparse equivalent of the brute force: at
// each depth only the 8 corners of the depth-d cell holding p can be non-zero. Terms are
// summed depth 0..D-1, corners k = x|y<<1|z<<2 in order. Lattice point (i,j,k) sits at
// origin + index*voxelSize per axis, voxelSize = width/R; x is the fastest index.
void evalGrid(const Svo& s, const double* lambda, const double origin[3], const double width[3], int R,
              double* out) {
  std::vector<std::unordered_map<uint64_t, size_t>> key2v(s.treeDepth);
  for (int d = 0; d < s.treeDepth; ++d) {
    const double w = s.unit.x * (double)(1u << d);
    for (size_t j = 0; j < s.depthVerts[d].size(); ++j) {
      const V3 pos = s.depthVerts[d][j].pos;
      uint64_t key = 0;
      for (int a = 0; a < 3; ++a) key = key * 4096 + (uint64_t)std::llround((pos[a] - s.gridOrigin[a]) / w);
      key2v[d].emplace(key, s.esumVerts[d] + j);
    }
  }
  const double vs[3] = {width[0] / R, width[1] / R, width[2] / R};
  const int64_t M = R + 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t zk = 0; zk < M; ++zk)
    for (int64_t yj = 0; yj < M; ++yj)
      for (int64_t xi = 0; xi < M; ++xi) {
        const V3 p{origin[0] + (double)xi * vs[0], origin[1] + (double)yj * vs[1], origin[2] + (double)zk * vs[2]};
        double sum = 0.0;
        for (int d = 0; d < s.treeDepth; ++d) {
          const double w = s.unit.x * (double)(1u << d);
          const int64_t lim = (int64_t)(s.res >> d);
          int64_t c[3];
          for (int a = 0; a < 3; ++a) c[a] = (int64_t)std::floor((p[a] - s.gridOrigin[a]) / w);
          for (int k = 0; k < 8; ++k) {
            const int64_t L[3] = {c[0] + (k & 1), c[1] + ((k >> 1) & 1), c[2] + ((k >> 2) & 1)};
            if (L[0] < 0 || L[1] < 0 || L[2] < 0 || L[0] > lim || L[1] > lim || L[2] > lim) continue;
            const uint64_t key = ((uint64_t)L[0] * 4096 + (uint64_t)L[1]) * 4096 + (uint64_t)L[2];
            auto it = key2v[d].find(key);
            if (it == key2v[d].end()) continue;
            const size_t j = it->second;
            const VertexRec& v = s.depthVerts[d][j - s.esumVerts[d]];
            sum += lambda[j] * baseFunction4Point(v.pos, w, p);
          }
        }
        out[(zk * M + yj) * M + xi] = sum;
      }
}

// Point queries (ThinShells::multiPointQuery, ThinShells.cpp:1183-1420, CUDA branch):
// outside [boxOrigin - boxWidth, boxEnd + boxWidth] the value is the outer iso level, else
// the field (the sparse equivalent of the sum over all corner vertices, as in evalGrid);
// label 1 if value >= outer, -1 if value <= inner, 0 otherwise.
void pointQuery(const Svo& s, const double* lambda, const double* P, int64_t m, const double boxOrigin[3],
                const double boxEnd[3], double inner, double outer, double* values, int8_t* labels) {
  std::vector<std::unordered_map<uint64_t, size_t>> key2v(s.treeDepth);
  for (int d = 0; d < s.treeDepth; ++d) {
    const double w = s.unit.x * (double)(1u << d);
    for (size_t j = 0; j < s.depthVerts[d].size(); ++j) {
      const V3 pos = s.depthVerts[d][j].pos;
      uint64_t key = 0;
      for (int a = 0; a < 3; ++a) key = key * 4096 + (uint64_t)std::llround((pos[a] - s.gridOrigin[a]) / w);
      key2v[d].emplace(key, s.esumVerts[d] + j);
    }
  }
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    const double w = boxEnd[a] - boxOrigin[a];
    lo[a] = boxOrigin[a] - w;
    hi[a] = boxEnd[a] + w;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    const V3 p{P[3 * i], P[3 * i + 1], P[3 * i + 2]};
    double v;
    if (p.x < lo[0] || p.y < lo[1] || p.z < lo[2] || p.x > hi[0] || p.y > hi[1] || p.z > hi[2]) {
      v = outer;
    } else {
      double sum = 0.0;
      for (int d = 0; d < s.treeDepth; ++d) {
        const double w = s.unit.x * (double)(1u << d);
        const int64_t lim = (int64_t)(s.res >> d);
        int64_t c[3];
        for (int a = 0; a < 3; ++a) c[a] = (int64_t)std::floor((p[a] - s.gridOrigin[a]) / w);
        for (int k = 0; k < 8; ++k) {
          const int64_t L[3] = {c[0] + (k & 1), c[1] + ((k >> 1) & 1), c[2] + ((k >> 2) & 1)};
          if (L[0] < 0 || L[1] < 0 || L[2] < 0 || L[0] > lim || L[1] > lim || L[2] > lim) continue;
          auto it = key2v[d].find(((uint64_t)L[0] * 4096 + (uint64_t)L[1]) * 4096 + (uint64_t)L[2]);
          if (it == key2v[d].end()) continue;
          const VertexRec& vr = s.depthVerts[d][it->second - s.esumVerts[d]];
          sum += lambda[it->second] * baseFunction4Point(vr.pos, w, p);
        }
      }
      v = sum;
    }
    if (values) values[i] = v;
    if (labels) labels[i] = (int8_t)(v >= outer ? 1 : (v <= inner ? -1 : 0));
  }
}

// ---- marching cubes: MarchingCubes.cu:164-377 on a shared-corner lattice --------------
static const uint64_t kMcCase[256] = {
#include "../its_b200/csrc/mc_tables.inc"
};
static const int kMcCorner[8][3] = {{0, 0, 0}, {0, 1, 0}, {1, 1, 0}, {1, 0, 0},
                                    {0, 0, 1}, {0, 1, 1}, {1, 1, 1}, {1, 0, 1}};
static const int kMcEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                   {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
static V3 vertexLerp(const V3& p0, const V3& p1, double s0, double s1, double iso) {
  if (std::fabs(iso - s0) < 1e-6) return p0;
  if (std::fabs(iso - s1) < 1e-6) return p1;
  if (std::fabs(s1 - s0) < 1e-6) return p0;
  const double t = (iso - s0) / (s1 - s0);
  auto lerp = [t](double a, double b) { return std::fma(t, b, std::fma(-t, a, a)); };
  return {lerp(p0.x, p1.x), lerp(p0.y, p1.y), lerp(p0.z, p1.z)};
}
int64_t marchingCubes(const double* field, int R, const double origin[3], const double width[3], double iso,
                      uint8_t* cubeIndex, double* tri, int64_t maxVerts) {
  const int64_t M = R + 1;
  const double vs[3] = {width[0] / R, width[1] / R, width[2] / R};
  const int64_t nVox = (int64_t)R * R * R;
  std::vector<uint32_t> nv(nVox);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < nVox; ++v) {
    const int64_t x = v % R, y = (v / R) % R, z = v / ((int64_t)R * R);
    unsigned ci = 0;
    for (int k = 0; k < 8; ++k) {
      const double f = field[((z + kMcCorner[k][2]) * M + (y + kMcCorner[k][1])) * M + (x + kMcCorner[k][0])];
      ci |= (unsigned)(f < iso) << k;
    }
    if (cubeIndex) cubeIndex[v] = (uint8_t)ci;
    nv[v] = (uint32_t)(kMcCase[ci] & 15u);
  }
  int64_t total = 0;
  std::vector<int64_t> off(nVox);
  for (int64_t v = 0; v < nVox; ++v) { off[v] = total; total += nv[v]; }
  if (!tri) return total;
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < nVox; ++v) {
    if (!nv[v]) continue;
    const int64_t x = v % R, y = (v / R) % R, z = v / ((int64_t)R * R);
    const V3 vp{(double)x * vs[0] + origin[0], (double)y * vs[1] + origin[1], (double)z * vs[2] + origin[2]};
    V3 corner[8];
    double sdf[8];
    unsigned ci = 0;
    for (int k = 0; k < 8; ++k) {
      corner[k] = {kMcCorner[k][0] ? vp.x + vs[0] : vp.x, kMcCorner[k][1] ? vp.y + vs[1] : vp.y,
                   kMcCorner[k][2] ? vp.z + vs[2] : vp.z};
      sdf[k] = field[((z + kMcCorner[k][2]) * M + (y + kMcCorner[k][1])) * M + (x + kMcCorner[k][0])];
      ci |= (unsigned)(sdf[k] < iso) << k;
    }
    V3 tv[12];
    for (int e = 0; e < 12; ++e)
      tv[e] = vertexLerp(corner[kMcEdge[e][0]], corner[kMcEdge[e][1]], sdf[kMcEdge[e][0]], sdf[kMcEdge[e][1]], iso);
    const uint64_t cw = kMcCase[ci];
    for (uint32_t i = 0; i < nv[v]; ++i) {
      const int64_t dst = off[v] + i;
      if (dst >= maxVerts) break;
      const V3 q = tv[(cw >> (4 * (i + 1))) & 15u];
      tri[3 * dst] = q.x;
      tri[3 * dst + 1] = q.y;
      tri[3 * dst + 2] = q.z;
    }
  }
  return total;
}

// Welded marching-cubes mesh: one vertex per active lattice edge (the two end values on
// different sides of iso), numbered in edge-id order id = 3*lin(lower end) + axis, placed by
// the reference's lerp from the lower to the upper end point; triangles from the case table.
void marchingCubesMesh(const double* field, int R, const double origin[3], const double width[3], double iso,
                       std::vector<double>& verts, std::vector<int32_t>& tris) {
  const int64_t M = R + 1;
  const double vs[3] = {width[0] / R, width[1] / R, width[2] / R};
  auto f = [&](int64_t x, int64_t y, int64_t z) { return field[(z * M + y) * M + x]; };
  std::vector<int32_t> index(3 * M * M * M, -1);
  verts.clear();
  tris.clear();
  for (int64_t id = 0; id < 3 * M * M * M; ++id) {
    const int64_t lin = id / 3;
    const int a = (int)(id % 3);
    const int64_t x = lin % M, y = (lin / M) % M, z = lin / (M * M);
    const int64_t x1 = x + (a == 0), y1 = y + (a == 1), z1 = z + (a == 2);
    if (x1 >= M || y1 >= M || z1 >= M) continue;
    if ((f(x, y, z) < iso) == (f(x1, y1, z1) < iso)) continue;
    const V3 p0{origin[0] + (double)x * vs[0], origin[1] + (double)y * vs[1], origin[2] + (double)z * vs[2]};
    const V3 p1{origin[0] + (double)x1 * vs[0], origin[1] + (double)y1 * vs[1], origin[2] + (double)z1 * vs[2]};
    const V3 q = vertexLerp(p0, p1, f(x, y, z), f(x1, y1, z1), iso);
    index[id] = (int32_t)(verts.size() / 3);
    verts.insert(verts.end(), {q.x, q.y, q.z});
  }
  for (int64_t v = 0; v < (int64_t)R * R * R; ++v) {
    const int64_t x = v % R, y = (v / R) % R, z = v / ((int64_t)R * R);
    unsigned ci = 0;
    for (int k = 0; k < 8; ++k)
      ci |= (unsigned)(f(x + kMcCorner[k][0], y + kMcCorner[k][1], z + kMcCorner[k][2]) < iso) << k;
    const uint64_t cw = kMcCase[ci];
    const unsigned n = (unsigned)(cw & 15u);
    for (unsigned i = 0; i < n; ++i) {
      const int e = (int)((cw >> (4 * (i + 1))) & 15u);
      const int* A = kMcCorner[kMcEdge[e][0]];
      const int* B = kMcCorner[kMcEdge[e][1]];
      const int64_t lx = x + std::min(A[0], B[0]), ly = y + std::min(A[1], B[1]), lz = z + std::min(A[2], B[2]);
      const int axis = A[0] != B[0] ? 0 : (A[1] != B[1] ? 1 : 2);
      tris.push_back(index[((lz * M + ly) * M + lx) * 3 + axis]);
    }
  }
}

}  // namespace orc

namespace orc {

// Coincident flags and depth starts of the corner vertices. A vertex of depth d below the
// root whose lattice coordinates (recovered from its position, (p - gridOrigin) /
// (unit * 2^d), to the nearest integer) are all even coincides with a corner of depth d + 1.
static void startTables(const Svo& s, int64_t n, std::vector<int64_t>& start, std::vector<char>& coincident) {
  const int depth = s.treeDepth;
  start.assign(depth + 1, 0);
  for (int d = 0; d < depth; ++d) start[d + 1] = start[d] + (int64_t)s.depthVerts[d].size();
  coincident.assign(n, 0);
  for (int d = 0; d + 1 < depth; ++d) {
    const double w = s.unit.x * (double)(1u << d);
    for (size_t k = 0; k < s.depthVerts[d].size(); ++k) {
      const V3& p = s.depthVerts[d][k].pos;
      const long long X = std::llround((p.x - s.gridOrigin.x) / w), Y = std::llround((p.y - s.gridOrigin.y) / w),
                      Z = std::llround((p.z - s.gridOrigin.z) / w);
      coincident[start[d] + (int64_t)k] = ((X | Y | Z) & 1) == 0;
    }
  }
}

// Exact start of A lambda = b in explicit form, read off the assembled rows. Coincident
// vertices keep their shares. With G_r = b_r - (row r's finer coincident columns, value 1,
// times their shares), every other row is
//   lambda_r = G_r - sum over row r's entries of depth d+1 (its owner's parent cell) of A(r,c) G_c,
// both sums in column order: the coarser depths' part of the field is trilinear on that cell,
// and its values at the cell's corners are G.
void exactStart(const Svo& s, const Csr& A, const double* b, const double* shares, double* lambda) {
  std::vector<int64_t> start;
  std::vector<char> coincident;
  startTables(s, A.n, start, coincident);
  const int depth = s.treeDepth;
  std::vector<double> G(A.n);
  std::vector<int> rowDepth(A.n);
  for (int d = 0; d < depth; ++d)
    for (int64_t r = start[d]; r < start[d + 1]; ++r) rowDepth[r] = d;
  for (int64_t r = 0; r < A.n; ++r) {
    double acc = 0.0;
    if (shares)
      for (int64_t k = A.rowptr[r]; k < A.rowptr[r + 1]; ++k)
        if (A.col[k] < start[rowDepth[r]]) acc += A.val[k] * shares[A.col[k]];
    G[r] = b[r] - acc;
  }
  for (int64_t r = 0; r < A.n; ++r) {
    const int d = rowDepth[r];
    if (coincident[r]) {
      lambda[r] = shares ? shares[r] : 0.0;
      continue;
    }
    double acc = 0.0;
    if (d + 1 < depth)
      for (int64_t k = A.rowptr[r]; k < A.rowptr[r + 1]; ++k)
        if (A.col[k] >= start[d + 1] && A.col[k] < start[d + 2]) acc += A.val[k] * G[A.col[k]];
    lambda[r] = G[r] - acc;
  }
}

// The same solution by the sequential definition, coarse depths first: every non-coincident
// row solves lambda_v = b_v - sum_{u != v} A(v,u) lambda_u, its entries summed in column order.
void exactStartSurplus(const Svo& s, const Csr& A, const double* b, const double* shares, double* lambda) {
  std::vector<int64_t> start;
  std::vector<char> coincident;
  startTables(s, A.n, start, coincident);
  for (int64_t r = 0; r < A.n; ++r) lambda[r] = (coincident[r] && shares) ? shares[r] : 0.0;
  for (int d = s.treeDepth - 1; d >= 0; --d) {
    for (int64_t r = start[d]; r < start[d + 1]; ++r) {
      if (coincident[r]) continue;
      double acc = 0.0;
      for (int64_t k = A.rowptr[r]; k < A.rowptr[r + 1]; ++k)
        if (A.col[k] != r) acc += A.val[k] * lambda[A.col[k]];
      lambda[r] = b[r] - acc;
    }
  }
}

}  // namespace orc
