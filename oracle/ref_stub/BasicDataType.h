// Stand-in for the reference's BasicDataType.h (test infrastructure): the reference's own
// header pulls in Eigen, which is not available here. Only what src/BSpline.hpp uses is
// provided -- a 3-vector of doubles with x()/y()/z()/operator(), and a row-major matrix of
// such rows -- so that BSpline.hpp itself compiles unchanged for the golden-vector harness.
#pragma once
#include <cmath>
#include <vector>

struct MXd;
struct V3d {
  double v[3] = {0.0, 0.0, 0.0};
  V3d() = default;
  V3d(double a, double b, double c) : v{a, b, c} {}
  V3d(const MXd& m);  // NOLINT: BSpline.hpp passes a matrix where a point is expected
  double& x() { return v[0]; }
  double& y() { return v[1]; }
  double& z() { return v[2]; }
  const double& x() const { return v[0]; }
  const double& y() const { return v[1]; }
  const double& z() const { return v[2]; }
  double& operator()(int i) { return v[i]; }
  const double& operator()(int i) const { return v[i]; }
};
struct MXd {
  std::vector<V3d> r;
  MXd(int rows, int) : r(rows) {}
  int rows() const { return (int)r.size(); }
  V3d& row(int i) { return r[i]; }
  const V3d& row(int i) const { return r[i]; }
};
inline V3d::V3d(const MXd& m) : V3d(m.rows() ? m.row(0) : V3d()) {}
