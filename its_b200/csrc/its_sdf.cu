// Right-hand side: signed distance at the corner vertices (replaces ThinShells::cpSDFOfTreeNodes,
// ThinShells.cpp:481-509, which calls libigl::signed_distance with the fast winding number).
// The work is in its_bvh.cu: exact distance through a linear BVH, sign from the fast winding
// number; negative where w > 1/2.
#include "its_ctx.cuh"

namespace its {
its_status validateMesh(its_ctx* ctx, const double* dV, int64_t nv, const int32_t* dF, int64_t nf);
its_status sdfBvh(its_ctx* ctx, const double* dP, int64_t m, const double* dV, const int32_t* dF, int64_t nf,
                  double* dOut);
}  // namespace its

using namespace its;

extern "C" {

its_status its_signed_distance(its_ctx* ctx, const double* points, int64_t npoints, const double* verts, int64_t nverts,
                               const int32_t* faces, int64_t nfaces, double* out) {
  if (!ctx) return ITS_ERR_INVALID;
  if (!points || !verts || !faces || !out || npoints < 0 || nverts <= 0 || nfaces <= 0)
    return setError(ctx, ITS_ERR_INVALID, "its_signed_distance: bad arguments");
  if (nfaces >= (1ll << 31)) return setError(ctx, ITS_ERR_INVALID, "its_signed_distance: too many faces");
  if (npoints >= (1ll << 32)) return setError(ctx, ITS_ERR_INVALID, "its_signed_distance: too many points");
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
  if ((st = sdfBvh(ctx, P.d, npoints, V.d, F.d, nfaces, O.d)) != ITS_OK) return st;
  if ((st = O.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // extern "C"
