// CPU oracle (test infrastructure): fit-side stages. See orc_common.hpp.
#pragma once
#include <vector>

#include "orc_svo.hpp"

namespace orc {

struct Csr {
  int64_t n = 0;
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  std::vector<double> val;
};
struct CglsReport {
  int64_t iterations = 0;
  int converged = 0, breakdown = 0;
  double rel_residual = 0, normal_rel_residual = 0, rhs_norm2 = 0, normal_residual_norm2 = 0;
};

std::vector<V3> intersections(const Svo& s, const double* V, int64_t nv, const int32_t* F, int64_t nf,
                              size_t* nEdgePoints);
void signedDistance(const double* P, int64_t m, const double* V, const int32_t* F, int64_t nf, double* out);
// The same signed distance accelerated as libits computes it (orc_bvh.cpp): a linear BVH,
// exact nearest-triangle distance, the sign from the fast winding number.
void signedDistanceBvh(const double* P, int64_t m, const double* V, const int32_t* F, int64_t nf, double* out);
double pointTriSqDist(const V3& p, const V3& a, const V3& b, const V3& c);
// Cubic B-spline basis over the corner vertices and offset shell samples (orc_cubic.cpp).
double bspline3(double t);
Csr cubicAssemble(const Svo& s, const double* samples, int64_t m);
void cubicEval(const Svo& s, const double* lambda, const double* P, int64_t m, double* out);
void cubicEvalGrid(const Svo& s, const double* lambda, const double origin[3], const double width[3], int R,
                   double* out);
void offsetSamples(const double* V, int64_t nv, const int32_t* F, int64_t nf, double eps, double* pts, double* tgt);
double solidAngle(const V3& p, const V3& a0, const V3& b0, const V3& c0);
Csr assemble(const Svo& s);
Csr transpose(const Csr& A);
CglsReport cgls(const Csr& A, const Csr& T, const double* b, double* x, double tol, int64_t maxIters, int stop);
void exactStart(const Svo& s, const Csr& A, const double* b, const double* shares, double* lambda);
void exactStartSurplus(const Svo& s, const Csr& A, const double* b, const double* shares, double* lambda);
void evalPoints(const Svo& s, const double* lambda, const double* P, int64_t m, double* out, uint8_t* missing);
// ThinShells::getPointValGradient (ThinShells.cpp:1800-1866): a point outside the box is moved
// halfway towards its previous position until inside (before may be null: no move), then the
// field and its gradient over its fine node's chain; missing as in evalPoints.
void pointValGradient(const Svo& s, const double* lambda, const double* P, const double* before, int64_t m,
                      const double boxOrigin[3], const double boxEnd[3], double* val, double* grad, uint8_t* missing);
void evalBrute(const Svo& s, const double* lambda, const double* P, int64_t m, double* out);
void evalGrid(const Svo& s, const double* lambda, const double origin[3], const double width[3], int R, double* out);
void pointQuery(const Svo& s, const double* lambda, const double* P, int64_t m, const double boxOrigin[3],
                const double boxEnd[3], double inner, double outer, double* values, int8_t* labels);
int64_t marchingCubes(const double* field, int R, const double origin[3], const double width[3], double iso,
                      uint8_t* cubeIndex, double* tri, int64_t maxVerts);
void marchingCubesMesh(const double* field, int R, const double origin[3], const double width[3], double iso,
                       std::vector<double>& verts, std::vector<int32_t>& tris);

}  // namespace orc
