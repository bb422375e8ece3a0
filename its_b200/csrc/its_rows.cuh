// The rows of the thin-shell basis matrix A, generated on the fly from the octree.
//
// Row v (a corner vertex at depth d, lattice point P, owner node o) evaluates the fitted
// field at v (ThinShells::cpCoefficients, ThinShells.cpp:511-606; setInDomainPoints,
// SVO.cu:1160-1193):
//   * the coincident vertices at depths j0..d-1 (value 1; the chain stops at the first finer
//     depth without that corner), found by a bit test in each depth's lattice bitmap;
//   * the diagonal (value 1);
//   * for every ancestor of o, the non-zero hats of its 8 corners at v, with the corner
//     positions origin (+ w) of that ancestor, exactly as the reference computes them.
//     (An ancestor exists at every coarser depth: the level build keeps every parent.)
// Columns are lattice ranks, so a row comes out sorted: chain < diagonal < ancestors, corners
// in x-major order. The assembly writes these entries into CSR; the matrix-free kernels
// (exact start, residual) consume them directly in the same order.
#pragma once
#include "its_svo.cuh"

namespace its {

struct RowParams {
  int depth;
  double3 g;
  double w0;
  LatticeIndex lat[kMaxDepth];
  int64_t vertStart[kMaxDepth + 1];
  const uint32_t* parent;
  const uint32_t* morton;
  const uint32_t* vertLin;
  const uint64_t* vertKey;
  const uint32_t* vertOwner;
  const double* vertPos;
  double winv[kMaxDepth];  // RN(1 / w_d): the hat quotients by divRn (bit-identical, no division)
};

inline RowParams rowParams(const SvoDevice& d) {
  RowParams P;
  P.depth = d.depth;
  P.g = make_double3(d.origin[0], d.origin[1], d.origin[2]);
  P.w0 = d.unit[0];
  for (int L = 0; L < kMaxDepth; ++L) P.lat[L] = L < d.depth ? d.lattice(L) : LatticeIndex{};
  for (int L = 0; L <= kMaxDepth; ++L) P.vertStart[L] = L <= d.depth ? d.vertStart[L] : d.numVerts;
  P.parent = d.nodeParent;
  P.morton = d.nodeMorton;
  P.vertLin = d.vertLin;
  P.vertKey = d.vertKey;
  P.vertOwner = d.vertOwner;
  P.vertPos = d.vertPos;
  for (int L = 0; L < kMaxDepth; ++L) P.winv[L] = 1.0 / (P.w0 * (double)(1u << L));
  return P;
}

// Lattice coordinates, depth and owner coordinates of vertex r (one 8-byte load). The
// owner (the lowest-index node with that corner) has the vertex at its corner (X - Xo,
// Y - Yo, Z - Zo); its ancestor k depths up has coordinates (Xo, Yo, Zo) >> k, because the
// octree's levels are O_{L+1} = O_L >> 3 -- no walk along the parent links.
__device__ __forceinline__ VertCoord vertCoord(const RowParams& P, int64_t r) { return decodeVertKey(P.vertKey[r]); }

// A vertex whose lattice coordinates are all even below the root depth coincides with a
// corner of the next coarser depth.
__device__ __forceinline__ bool coordCoincident(const RowParams& P, const VertCoord& v) {
  return v.d + 1 < P.depth && ((v.X | v.Y | v.Z) & 1u) == 0u;
}

// The coincident vertices of the finer depths at the point of a depth-d vertex with lattice
// coordinates (X, Y, Z): visit(col) for depths j0..d-1, finest first (their value in the row
// is 1). The chain stops at the first finer depth without a corner there.
template <class Visit>
__device__ __forceinline__ void walkChain(const RowParams& P, int d, uint32_t X, uint32_t Y, uint32_t Z,
                                          Visit&& visit) {
  int j0 = d;
  for (int j = d - 1; j >= 0; --j) {
    const int s = d - j;
    const uint32_t Mj = P.lat[j].M;
    const uint32_t lj = ((X << s) * Mj + (Y << s)) * Mj + (Z << s);
    if (!latticeHas(P.lat[j], lj)) break;
    j0 = j;
  }
  for (int j = j0; j < d; ++j) {
    const int s = d - j;
    const uint32_t Mj = P.lat[j].M;
    const uint32_t lj = ((X << s) * Mj + (Y << s)) * Mj + (Z << s);
    visit((int32_t)latticeRank(P.lat[j], lj));
  }
}

// hat1r(x, b, w) and hat1r(x, b + w, w) for a coordinate x of a point in the cell [b, b + w]
// (to rounding: the point is a corner of a node inside it). Of hat1r's four zero tests, two
// per corner can only hold a cell width away from the cell, so only the others are made; the
// values are hat1r's bit for bit.
__device__ __forceinline__ void hatPair(double x, double b, double w, double wi, double h[2]) {
  const double b1 = b + w;
  const double e0 = b + w, e1 = b1 - w;  // hat1r's far support ends of the two corners
  h[0] = (fabs(x - e0) < 1e-9 || x > e0) ? 0.0 : (x <= b ? 1 + divRn(x - b, w, wi) : 1 - divRn(x - b, w, wi));
  h[1] = (fabs(x - e1) < 1e-9 || x < e1) ? 0.0 : (x <= b1 ? 1 + divRn(x - b1, w, wi) : 1 - divRn(x - b1, w, wi));
}

// visit(col, val) for the non-zero hats at (qx, qy, qz) of the 8 corners of the depth-dd
// ancestor of the depth-d vertex c's owner, corners in x-major order. (Corner positions are
// the cell's origin (+ w), as the reference forms them, so the cell must be the owner's
// ancestor itself: a neighbouring cell sharing the corner would place it an ulp away.)
template <class Visit>
__device__ __forceinline__ void walkAncestor(const RowParams& P, const VertCoord& c, int dd, double qx, double qy,
                                             double qz, Visit&& visit) {
  const int up = dd - c.d;
  const LatticeIndex& L = P.lat[dd];
  const uint32_t Xa = c.Xo >> up, Ya = c.Yo >> up, Za = c.Zo >> up;
  const double w = P.w0 * (double)(1u << dd), wi = P.winv[dd];
  const double bx = latticePos(P.g.x, w, Xa), by = latticePos(P.g.y, w, Ya), bz = latticePos(P.g.z, w, Za);
  // the six axis factors once (the corners share them)
  double hxs[2], hys[2], hzs[2];
  hatPair(qx, bx, w, wi, hxs);
  hatPair(qy, by, w, wi, hys);
  hatPair(qz, bz, w, wi, hzs);
#pragma unroll
  for (int ox = 0; ox < 2; ++ox) {
    const double hx = hxs[ox];
    if (hx <= 0.0) continue;
#pragma unroll
    for (int oy = 0; oy < 2; ++oy) {
      const double hy = hys[oy];
      if (hy <= 0.0) continue;
#pragma unroll
      for (int oz = 0; oz < 2; ++oz) {
        const double hz = hzs[oz];
        if (hz <= 0.0) continue;
        const double v = hx * hy * hz;
        if (v == 0.0) continue;
        visit((int32_t)latticeRank(L, ((Xa + ox) * L.M + (Ya + oy)) * L.M + (Za + oz)), v);
      }
    }
  }
}

// visit(col, val) for every entry of row r in column order: the finer coincident vertices,
// the diagonal, then the corners of every ancestor of the owner, coarser last.
template <class Visit>
__device__ __forceinline__ void walkRow(const RowParams& P, int64_t r, Visit&& visit) {
  const VertCoord c = vertCoord(P, r);
  const double qx = P.vertPos[3 * r], qy = P.vertPos[3 * r + 1], qz = P.vertPos[3 * r + 2];
  walkChain(P, c.d, c.X, c.Y, c.Z, [&](int32_t k) { visit(k, 1.0); });
  visit((int32_t)r, 1.0);
  for (int dd = c.d + 1; dd < P.depth; ++dd) walkAncestor(P, c, dd, qx, qy, qz, visit);
}

}  // namespace its
