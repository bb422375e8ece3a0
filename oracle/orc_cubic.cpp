// CPU oracle (test infrastructure): the cubic tensor-product B-spline basis over the octree's
// corner vertices and the offset shell samples. Neither has a counterpart in the reference,
// whose basis is the degree-1 hat of BSpline.hpp:4-22 and whose fit samples are the corner
// vertices themselves (ThinShells.cpp:481-606); the closest ancestor of extra sample rows is
// the uncompiled ThinShellsOctree.deprecated.cpp:139-187, which appends one row per sample
// point to A. This file defines the extension that libits' its_cubic.cu implements, and both
// follow the same operation order so that their results compare bit for bit:
//
//   * vertex v at depth d, lattice coordinates (X, Y, Z), sits at origin + (X, Y, Z) * w_d with
//     w_d = unit * 2^d; its basis function is beta3((x - p_x) / w_d) beta3(..y..) beta3(..z..),
//     beta3 the uniform cubic B-spline (support |t| < 2; 2/3 - t^2 + |t|^3/2 inside |t| < 1,
//     (2 - |t|)^3 / 6 beyond);
//   * the field at x is the sum over every depth d (finest first) and every lattice point k of
//     that depth with |u - k| < 2 on each axis (u = (x - origin) / w_d), in ascending lattice
//     order, of lambda_k * (bx * by) * bz, where a vertex exists at k;
//   * a corner vertex's own row uses its exact lattice coordinates (u = X * 2^(d_v - d)), so the
//     rows of the corner vertices carry no position rounding;
//   * extra sample rows (offset shell samples) follow the corner vertices' rows; the system is
//     stored square, padded with empty columns past the last vertex.
#include <cmath>
#include <vector>

#include "orc_fit.hpp"

namespace orc {

double bspline3(double t) {
  const double a = std::fabs(t);
  if (a >= 2.0) return 0.0;
  if (a < 1.0) return (4.0 + a * a * (3.0 * a - 6.0)) / 6.0;
  const double b = 2.0 - a;
  return b * b * b / 6.0;
}

namespace {

struct CubicIndex {
  int depth = 0;
  double origin[3] = {0, 0, 0};
  double unit = 0;
  std::vector<int64_t> M;
  std::vector<std::vector<int64_t>> col;  // per depth: lattice index -> column, -1 where no vertex
  std::vector<uint32_t> vx, vy, vz;
  std::vector<int> vd;
};

CubicIndex makeIndex(const Svo& s) {
  CubicIndex I;
  I.depth = s.treeDepth;
  I.origin[0] = s.gridOrigin.x;
  I.origin[1] = s.gridOrigin.y;
  I.origin[2] = s.gridOrigin.z;
  I.unit = s.unit.x;
  I.M.resize(I.depth);
  I.col.resize(I.depth);
  for (int d = 0; d < I.depth; ++d) {
    const int64_t M = (int64_t)(s.res >> d) + 1;
    I.M[d] = M;
    I.col[d].assign(M * M * M, -1);
    const double w = std::ldexp(s.unit.x, d);
    for (size_t i = 0; i < s.depthVerts[d].size(); ++i) {
      const V3 p = s.depthVerts[d][i].pos;
      const uint32_t X = (uint32_t)std::lrint((p.x - s.gridOrigin.x) / w);
      const uint32_t Y = (uint32_t)std::lrint((p.y - s.gridOrigin.y) / w);
      const uint32_t Z = (uint32_t)std::lrint((p.z - s.gridOrigin.z) / w);
      I.col[d][((int64_t)X * M + Y) * M + Z] = (int64_t)(s.esumVerts[d] + i);
      I.vx.push_back(X);
      I.vy.push_back(Y);
      I.vz.push_back(Z);
      I.vd.push_back(d);
    }
  }
  return I;
}

// Entries of the row at lattice coordinates u(d) (one triple per depth), in emission order.
template <typename U, typename Emit>
void cubicRow(const CubicIndex& I, U uOf, Emit emit) {
  for (int d = 0; d < I.depth; ++d) {
    double u[3];
    uOf(d, u);
    const int64_t M = I.M[d];
    int64_t base[3];
    double wt[3][4];
    for (int a = 0; a < 3; ++a) {
      base[a] = (int64_t)std::floor(u[a]) - 1;
      for (int j = 0; j < 4; ++j) wt[a][j] = bspline3(u[a] - (double)(base[a] + j));
    }
    for (int jx = 0; jx < 4; ++jx) {
      const int64_t kx = base[0] + jx;
      if (kx < 0 || kx >= M || wt[0][jx] == 0.0) continue;
      for (int jy = 0; jy < 4; ++jy) {
        const int64_t ky = base[1] + jy;
        if (ky < 0 || ky >= M || wt[1][jy] == 0.0) continue;
        const double wxy = wt[0][jx] * wt[1][jy];
        for (int jz = 0; jz < 4; ++jz) {
          const int64_t kz = base[2] + jz;
          if (kz < 0 || kz >= M || wt[2][jz] == 0.0) continue;
          const int64_t c = I.col[d][(kx * M + ky) * M + kz];
          if (c >= 0) emit(c, wxy * wt[2][jz]);
        }
      }
    }
  }
}

void pointU(const CubicIndex& I, const double* x, int d, double* u) {
  const double w = std::ldexp(I.unit, d);
  for (int a = 0; a < 3; ++a) u[a] = (x[a] - I.origin[a]) / w;
}

}  // namespace

Csr cubicAssemble(const Svo& s, const double* samples, int64_t m) {
  const CubicIndex I = makeIndex(s);
  const int64_t n = (int64_t)I.vd.size();
  Csr A;
  A.n = n + m;
  A.rowptr.assign(A.n + 1, 0);
  for (int64_t r = 0; r < A.n; ++r) {
    auto emit = [&](int64_t c, double v) {
      A.col.push_back((int32_t)c);
      A.val.push_back(v);
    };
    if (r < n) {
      const int dv = I.vd[r];
      const double X = I.vx[r], Y = I.vy[r], Z = I.vz[r];
      cubicRow(I, [&](int d, double* u) {
        u[0] = std::ldexp(X, dv - d);
        u[1] = std::ldexp(Y, dv - d);
        u[2] = std::ldexp(Z, dv - d);
      }, emit);
    } else {
      const double* x = samples + 3 * (r - n);
      cubicRow(I, [&](int d, double* u) { pointU(I, x, d, u); }, emit);
    }
    A.rowptr[r + 1] = (int64_t)A.col.size();
  }
  return A;
}

void cubicEval(const Svo& s, const double* lambda, const double* P, int64_t m, double* out) {
  const CubicIndex I = makeIndex(s);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < m; ++i) {
    double acc = 0.0;
    cubicRow(I, [&](int d, double* u) { pointU(I, P + 3 * i, d, u); },
             [&](int64_t c, double v) { acc = acc + v * lambda[c]; });
    out[i] = acc;
  }
}

void cubicEvalGrid(const Svo& s, const double* lambda, const double origin[3], const double width[3], int R,
                   double* out) {
  const int64_t M = (int64_t)R + 1;
  const double vs[3] = {width[0] / R, width[1] / R, width[2] / R};
  std::vector<double> P(3 * M * M);
  for (int64_t z = 0; z < M; ++z) {
    for (int64_t y = 0; y < M; ++y)
      for (int64_t x = 0; x < M; ++x) {
        const int64_t k = y * M + x;
        P[3 * k] = origin[0] + (double)x * vs[0];
        P[3 * k + 1] = origin[1] + (double)y * vs[1];
        P[3 * k + 2] = origin[2] + (double)z * vs[2];
      }
    cubicEval(s, lambda, P.data(), M * M, out + z * M * M);
  }
}

// Offset shell samples: at every mesh vertex, the area-weighted normal (the sum of the
// unnormalised face normals (p1 - p0) x (p2 - p0) of its faces, in face order) made unit, and
// the points v + eps n (target +eps, outside) for all vertices, then v - eps n (target -eps).
// A vertex with a zero normal gets both points at v.
void offsetSamples(const double* V, int64_t nv, const int32_t* F, int64_t nf, double eps, double* pts, double* tgt) {
  std::vector<V3> acc(nv, V3{0, 0, 0});
  for (int64_t f = 0; f < nf; ++f) {
    const V3 a{V[3 * F[3 * f]], V[3 * F[3 * f] + 1], V[3 * F[3 * f] + 2]};
    const V3 b{V[3 * F[3 * f + 1]], V[3 * F[3 * f + 1] + 1], V[3 * F[3 * f + 1] + 2]};
    const V3 c{V[3 * F[3 * f + 2]], V[3 * F[3 * f + 2] + 1], V[3 * F[3 * f + 2] + 2]};
    const V3 nrm = cross3(b - a, c - a);
    for (int k = 0; k < 3; ++k) acc[F[3 * f + k]] = acc[F[3 * f + k]] + nrm;
  }
  for (int64_t i = 0; i < nv; ++i) {
    const V3 nrm = acc[i];
    const double len = std::sqrt(dot3(nrm, nrm));
    V3 u{0, 0, 0};
    if (len > 0.0) u = V3{nrm.x / len, nrm.y / len, nrm.z / len};
    for (int a = 0; a < 3; ++a) {
      pts[3 * i + a] = V[3 * i + a] + eps * u[a];
      pts[3 * (nv + i) + a] = V[3 * i + a] - eps * u[a];
    }
    tgt[i] = eps;
    tgt[nv + i] = -eps;
  }
}

}  // namespace orc
