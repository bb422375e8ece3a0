// Cubic B-spline basis (its_cubic.cuh): the field at points and on a lattice, and the offset
// shell samples. No counterpart in the reference (degree-1 hats, corner-vertex samples).
#include "its_cubic.cuh"
#include "its_scan.cuh"
#include "its_sparse.cuh"

namespace its {

__global__ void __launch_bounds__(128) kCubicEvalPoints(const __grid_constant__ CubicGen g,
                                                        const double* __restrict__ lambda,
                                                        const double* __restrict__ P, int64_t m,
                                                        double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double x[3] = {P[3 * i], P[3 * i + 1], P[3 * i + 2]};
  out[i] = g.eval(x, lambda);
}

// Lattice point i (x fastest) at origin + (ix, iy, iz) * vs, vs = width / res.
__global__ void __launch_bounds__(128) kCubicEvalGrid(const __grid_constant__ CubicGen g,
                                                      const double* __restrict__ lambda, double3 o, double3 vs,
                                                      int64_t M, double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= M * M * M) return;
  const int64_t ix = i % M, iy = (i / M) % M, iz = i / (M * M);
  const double x[3] = {o.x + (double)ix * vs.x, o.y + (double)iy * vs.y, o.z + (double)iz * vs.z};
  out[i] = g.eval(x, lambda);
}

// Start of each vertex's run in the vertex-sorted face corners (every pointer written once).
__global__ void kRunStarts(int64_t n, const uint32_t* __restrict__ keys, int64_t nv, int64_t* __restrict__ start) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i > n) return;
  const int64_t c = (i < n) ? (int64_t)keys[i] : nv;
  const int64_t prev = (i == 0) ? -1 : (int64_t)keys[i - 1];
  for (int64_t k = prev + 1; k <= c; ++k) start[k] = i;
}

// Unit area-weighted normal of every vertex (its faces' unnormalised normals summed in face
// order) and the two offset points with their targets.
__global__ void kOffsetSamples(const double* __restrict__ V, int64_t nv, const int32_t* __restrict__ F,
                               const int64_t* __restrict__ start, const uint32_t* __restrict__ corner, double eps,
                               double* __restrict__ pts, double* __restrict__ tgt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double n[3] = {0.0, 0.0, 0.0};
  for (int64_t k = start[i]; k < start[i + 1]; ++k) {
    const int64_t f = corner[k] / 3;
    double p[3][3];
    for (int c = 0; c < 3; ++c)
      for (int a = 0; a < 3; ++a) p[c][a] = V[3 * (int64_t)F[3 * f + c] + a];
    const double u[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    const double v[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    n[0] = n[0] + (u[1] * v[2] - u[2] * v[1]);
    n[1] = n[1] + (u[2] * v[0] - u[0] * v[2]);
    n[2] = n[2] + (u[0] * v[1] - u[1] * v[0]);
  }
  double len = n[0] * n[0];
  len = len + n[1] * n[1];
  len = sqrt(len + n[2] * n[2]);
  double un[3] = {0.0, 0.0, 0.0};
  if (len > 0.0)
    for (int a = 0; a < 3; ++a) un[a] = n[a] / len;
  if (pts)
    for (int a = 0; a < 3; ++a) {
      pts[3 * i + a] = V[3 * i + a] + eps * un[a];
      pts[3 * (nv + i) + a] = V[3 * i + a] - eps * un[a];
    }
  if (tgt) {
    tgt[i] = eps;
    tgt[nv + i] = -eps;
  }
}

__global__ void kCornerKeys(const int32_t* __restrict__ F, int64_t n3, uint32_t* __restrict__ keys,
                            uint32_t* __restrict__ vals) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n3) return;
  keys[k] = (uint32_t)F[k];
  vals[k] = (uint32_t)k;
}

}  // namespace its

using namespace its;

extern "C" {

its_status its_eval_points_cubic(its_svo* svo, const double* lambda, const double* points, int64_t npoints,
                                 double* out) {
  if (!svo || !lambda || (npoints > 0 && (!points || !out)) || npoints < 0) return ITS_ERR_INVALID;
  its_ctx* ctx = svo->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  if (npoints == 0) return ITS_OK;
  InArg<double> L, P;
  OutArg<double> O;
  its_status st;
  if ((st = L.stage(ctx, lambda, svo->d.numVerts)) != ITS_OK || (st = P.stage(ctx, points, 3 * npoints)) != ITS_OK ||
      (st = O.stage(ctx, out, npoints)) != ITS_OK)
    return st;
  kCubicEvalPoints<<<gridFor(npoints, 128), 128, 0, ctx->stream>>>(cubicGen(svo->d, nullptr), L.d, P.d, npoints, O.d);
  ITS_LAUNCHED(ctx);
  if ((st = O.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_eval_grid_cubic(its_svo* svo, const double* lambda, const double origin[3], const double width[3],
                               int res, double* field) {
  if (!svo || !lambda || !origin || !width || !field || res < 1 || res > 2048) return ITS_ERR_INVALID;
  its_ctx* ctx = svo->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  const int64_t M = (int64_t)res + 1;
  InArg<double> L;
  OutArg<double> O;
  its_status st;
  if ((st = L.stage(ctx, lambda, svo->d.numVerts)) != ITS_OK || (st = O.stage(ctx, field, M * M * M)) != ITS_OK)
    return st;
  const double3 o = make_double3(origin[0], origin[1], origin[2]);
  const double3 vs = make_double3(width[0] / res, width[1] / res, width[2] / res);
  kCubicEvalGrid<<<gridFor(M * M * M, 128), 128, 0, ctx->stream>>>(cubicGen(svo->d, nullptr), L.d, o, vs, M, O.d);
  ITS_LAUNCHED(ctx);
  if ((st = O.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_offset_samples(its_ctx* ctx, const double* verts, int64_t nverts, const int32_t* faces, int64_t nfaces,
                              double eps, double* points, double* targets) {
  if (!ctx) return ITS_ERR_INVALID;
  if (!verts || nverts < 1 || nfaces < 0 || (nfaces > 0 && !faces) || !(eps == eps) || 3 * nfaces >= (1ll << 32) ||
      nverts >= (1ll << 32))
    return setError(ctx, ITS_ERR_INVALID, "its_offset_samples: bad arguments");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> V;
  InArg<int32_t> F;
  OutArg<double> P, T;
  its_status st;
  if ((st = V.stage(ctx, verts, 3 * nverts)) != ITS_OK || (st = F.stage(ctx, faces, 3 * nfaces)) != ITS_OK ||
      (st = P.stage(ctx, points, 6 * nverts)) != ITS_OK || (st = T.stage(ctx, targets, 2 * nverts)) != ITS_OK)
    return st;
  if (nfaces > 0 && (st = validateMesh(ctx, V.d, nverts, F.d, nfaces)) != ITS_OK) return st;
  const int64_t n3 = 3 * nfaces;
  DevBuf<uint32_t> keys, vals, sk, sv, tk, tv;
  DevBuf<int64_t> start;
  if ((st = start.alloc(ctx, nverts + 1)) != ITS_OK) return st;
  if (n3 > 0) {
    if ((st = keys.alloc(ctx, n3)) != ITS_OK || (st = vals.alloc(ctx, n3)) != ITS_OK ||
        (st = sk.alloc(ctx, n3)) != ITS_OK || (st = sv.alloc(ctx, n3)) != ITS_OK || (st = tk.alloc(ctx, n3)) != ITS_OK ||
        (st = tv.alloc(ctx, n3)) != ITS_OK)
      return st;
    kCornerKeys<<<gridFor(n3, 256), 256, 0, ctx->stream>>>(F.d, n3, keys.p, vals.p);
    ITS_LAUNCHED(ctx);
    int bits = 1;
    while (bits < 32 && (1ll << bits) < nverts) ++bits;
    if ((st = radixSortPairs(ctx, keys.p, vals.p, sk.p, sv.p, tk.p, tv.p, n3, bits)) != ITS_OK) return st;
    kRunStarts<<<gridFor(n3 + 1, 256), 256, 0, ctx->stream>>>(n3, sk.p, nverts, start.p);
    ITS_LAUNCHED(ctx);
  } else {
    ITS_CU(ctx, cudaMemsetAsync(start.p, 0, (nverts + 1) * 8, ctx->stream));
  }
  kOffsetSamples<<<gridFor(nverts, 128), 128, 0, ctx->stream>>>(V.d, nverts, F.d, start.p, sv.p, eps, P.d, T.d);
  ITS_LAUNCHED(ctx);
  if ((st = P.finish(ctx)) != ITS_OK || (st = T.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // extern "C"
