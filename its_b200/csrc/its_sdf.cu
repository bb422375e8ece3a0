// Right-hand side: signed distance at the corner vertices (replaces ThinShells::cpSDFOfTreeNodes,
// ThinShells.cpp:481-509, which calls libigl::signed_distance with the fast winding number).
// Exact point-triangle distance (Ericson, Real-Time Collision Detection 5.1.5) and the sign of
// the generalised winding number (Jacobson et al. 2013; solid angles by Van Oosterom and
// Strackee 1983): negative where w > 1/2. Brute force over triangle tiles staged in shared
// memory, one thread per query point.
#include <cmath>

#include "its_ctx.cuh"

namespace its {

constexpr int kSdfThreads = 128;
constexpr int kSdfTile = 128;

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

__global__ void __launch_bounds__(kSdfThreads) kSignedDistance(const double* __restrict__ P, int64_t m,
                                                               const double* __restrict__ V,
                                                               const int32_t* __restrict__ F, int64_t nf,
                                                               double* __restrict__ out) {
  __shared__ D3 tri[kSdfTile][3];
  const int64_t i = blockIdx.x * (int64_t)kSdfThreads + threadIdx.x;
  const bool active = i < m;
  const D3 p = active ? D3{P[3 * i], P[3 * i + 1], P[3 * i + 2]} : D3{0, 0, 0};
  double best = 1.7976931348623157e308, wsum = 0.0;
  for (int64_t t0 = 0; t0 < nf; t0 += kSdfTile) {
    const int cnt = (int)((nf - t0) < kSdfTile ? (nf - t0) : kSdfTile);
    __syncthreads();
    for (int k = threadIdx.x; k < 3 * cnt; k += kSdfThreads) {
      const int tt = k / 3, c = k % 3;
      const int32_t vi = F[3 * (t0 + tt) + c];
      tri[tt][c] = D3{V[3 * vi], V[3 * vi + 1], V[3 * vi + 2]};
    }
    __syncthreads();
    if (active)
      for (int tt = 0; tt < cnt; ++tt) {
        best = fmin(best, pointTriSqDist(p, tri[tt][0], tri[tt][1], tri[tt][2]));
        wsum += solidAngle(p, tri[tt][0], tri[tt][1], tri[tt][2]);
      }
  }
  if (active) {
    const double w = wsum / (4.0 * 3.14159265358979323846);
    const double d = sqrt(best);
    out[i] = (w > 0.5) ? -d : d;
  }
}

its_status validateMesh(its_ctx* ctx, const double* dV, int64_t nv, const int32_t* dF, int64_t nf);

}  // namespace its

using namespace its;

extern "C" {

its_status its_signed_distance(its_ctx* ctx, const double* points, int64_t npoints, const double* verts, int64_t nverts,
                               const int32_t* faces, int64_t nfaces, double* out) {
  if (!ctx) return ITS_ERR_INVALID;
  if (!points || !verts || !faces || !out || npoints < 0 || nverts <= 0 || nfaces <= 0)
    return setError(ctx, ITS_ERR_INVALID, "its_signed_distance: bad arguments");
  if (npoints == 0) return ITS_OK;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> P, V;
  InArg<int32_t> F;
  OutArg<double> O;
  its_status st;
  if ((st = P.stage(ctx, points, 3 * npoints)) != ITS_OK) return st;
  if ((st = V.stage(ctx, verts, 3 * nverts)) != ITS_OK) return st;
  if ((st = F.stage(ctx, faces, 3 * nfaces)) != ITS_OK) return st;
  if ((st = validateMesh(ctx, V.d, nverts, F.d, nfaces)) != ITS_OK) return st;
  if ((st = O.stage(ctx, out, npoints)) != ITS_OK) return st;
  kSignedDistance<<<gridFor(npoints, kSdfThreads), kSdfThreads, 0, ctx->stream>>>(P.d, npoints, V.d, F.d, nfaces, O.d);
  ITS_LAUNCHED(ctx);
  if ((st = O.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // extern "C"
