// Per-triangle geometry shared by the signed-distance paths: exact point-triangle squared
// distance (Ericson, Real-Time Collision Detection 5.1.5) and the solid angle of a triangle
// seen from a point (Van Oosterom and Strackee 1983). Three-term dots sum left to right.
#pragma once

namespace its {

struct D3 { double x, y, z; };
__device__ inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ inline D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ inline D3 mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ inline double dot(D3 a, D3 b) {
  double s = a.x * b.x;
  s = s + a.y * b.y;
  return s + a.z * b.z;
}
__device__ inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

__device__ inline double pointTriSqDist(D3 p, D3 a, D3 b, D3 c) {
  const D3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return dot(ap, ap);
  const D3 bp = sub(p, b);
  const double d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) return dot(bp, bp);
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
    const double v = d1 / (d1 - d3);
    const D3 q = sub(p, add(a, mul(ab, v)));
    return dot(q, q);
  }
  const D3 cp = sub(p, c);
  const double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return dot(cp, cp);
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
    const double w = d2 / (d2 - d6);
    const D3 q = sub(p, add(a, mul(ac, w)));
    return dot(q, q);
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
    const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    const D3 q = sub(p, add(b, mul(sub(c, b), w)));
    return dot(q, q);
  }
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom, w = vc * denom;
  const D3 q = sub(p, add(add(a, mul(ab, v)), mul(ac, w)));
  return dot(q, q);
}
__device__ inline double solidAngle(D3 p, D3 a0, D3 b0, D3 c0) {
  const D3 a = sub(a0, p), b = sub(b0, p), c = sub(c0, p);
  const double la = sqrt(dot(a, a)), lb = sqrt(dot(b, b)), lc = sqrt(dot(c, c));
  const double num = dot(a, cross(b, c));
  const double den = la * lb * lc + dot(a, b) * lc + dot(b, c) * la + dot(c, a) * lb;
  return 2.0 * atan2(num, den);
}

}  // namespace its
