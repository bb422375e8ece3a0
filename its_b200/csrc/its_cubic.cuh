// The cubic tensor-product B-spline basis over the octree's corner vertices (no counterpart in
// the reference, whose basis is the degree-1 hat of BSpline.hpp:4-22).
//
// Vertex v at depth d, lattice coordinates (X, Y, Z), sits at origin + (X, Y, Z) w_d with
// w_d = unit * 2^d; its basis function is the product over the axes of beta3((x - p) / w_d),
// beta3 the uniform cubic B-spline (support |t| < 2). The field at x sums, depth by depth
// (finest first) and over the lattice points k of each depth with |u - k| < 2 on every axis
// (u = (x - origin) / w_d) in ascending lattice order, lambda_k (bx by) bz where a vertex
// exists at k. A corner vertex's own row uses its exact lattice coordinates
// (u = X 2^(d_v - d)); extra sample rows (offset shell samples) follow the vertices' rows.
// Every sum runs in this order, so rows, matrix-free evaluation and the oracle's restatement
// (oracle/orc_cubic.cpp) agree bit for bit.
#pragma once
#include "its_svo.cuh"

namespace its {

__host__ __device__ inline double bspline3(double t) {
  const double a = fabs(t);
  if (a >= 2.0) return 0.0;
  if (a < 1.0) return (4.0 + a * a * (3.0 * a - 6.0)) / 6.0;
  const double b = 2.0 - a;
  return b * b * b / 6.0;
}

struct CubicGen {
  int depth;
  double origin[3];
  double unit;
  LatticeIndex lat[kMaxDepth];
  int64_t numVerts;
  const uint64_t* vertKey;
  const double* samples;  // 3 per extra row (rows numVerts ...)

  // Entries of the row whose lattice coordinates at depth dd are u(dd, u).
  template <typename U, typename E>
  __device__ void row(U uOf, E emit) const {
    for (int dd = 0; dd < depth; ++dd) {
      double u[3];
      uOf(dd, u);
      const LatticeIndex L = lat[dd];
      const int64_t M = L.M;
      int64_t base[3];
      double wt[3][4];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        base[a] = (int64_t)floor(u[a]) - 1;
#pragma unroll
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
            const uint32_t lin = (uint32_t)((kx * M + ky) * M + kz);
            if (latticeHas(L, lin)) emit((int32_t)latticeRank(L, lin), wxy * wt[2][jz]);
          }
        }
      }
    }
  }

  __device__ void pointU(const double* x, int dd, double* u) const {
    const double w = ldexp(unit, dd);
    u[0] = (x[0] - origin[0]) / w;
    u[1] = (x[1] - origin[1]) / w;
    u[2] = (x[2] - origin[2]) / w;
  }

  // Row r of the assembled system: a corner vertex (r < numVerts) or an extra sample point.
  template <typename E>
  __device__ void operator()(int64_t r, E emit) const {
    if (r < numVerts) {
      const VertCoord c = decodeVertKey(vertKey[r]);
      const double X = c.X, Y = c.Y, Z = c.Z;
      const int dv = c.d;
      row([&](int dd, double* u) {
        u[0] = ldexp(X, dv - dd);
        u[1] = ldexp(Y, dv - dd);
        u[2] = ldexp(Z, dv - dd);
      }, emit);
    } else {
      const double* x = samples + 3 * (r - numVerts);
      row([&](int dd, double* u) { pointU(x, dd, u); }, emit);
    }
  }

  // The field at x: sum of lambda_c * value in emission order.
  __device__ double eval(const double* x, const double* lambda) const {
    double acc = 0.0;
    row([&](int dd, double* u) { pointU(x, dd, u); }, [&](int32_t c, double v) { acc = acc + v * lambda[c]; });
    return acc;
  }
};

inline CubicGen cubicGen(const SvoDevice& d, const double* samples) {
  CubicGen g;
  g.depth = d.depth;
  for (int a = 0; a < 3; ++a) g.origin[a] = d.origin[a];
  g.unit = d.unit[0];
  for (int L = 0; L < kMaxDepth; ++L) g.lat[L] = L < d.depth ? d.lattice(L) : LatticeIndex{};
  g.numVerts = d.numVerts;
  g.vertKey = d.vertKey;
  g.samples = samples;
  return g;
}

}  // namespace its
