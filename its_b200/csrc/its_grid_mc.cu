// its_eval_grid_mc: the marching-cubes driver of ThinShells::mcVisualization
// (src/ThinShells.cpp:1086-1129 -> MC::marching_cubes, src/cuAcc/MarchingCubes/MarchingCubes.cu:672-714)
// in one call: the dense field of lambda on the (res+1)^3 lattice is evaluated once into device
// scratch and stays there, then marching cubes runs at every requested iso level and only the
// triangle soups leave the device. The reference evaluates the field per call, copies the
// 8-corners-per-voxel field array back to the host and forth again; here the field never
// leaves HBM.
#include "its_ctx.cuh"
#include "its_svo.cuh"

using namespace its;

extern "C" {

its_status its_eval_grid_mc(its_svo* svo, const double* lambda, const double origin[3], const double width[3], int res,
                            int field_mode, const double* iso, int n_iso, double* const* tri_verts,
                            const int64_t* capacity, int64_t* num_verts) {
  if (!svo) return ITS_ERR_INVALID;
  its_ctx* ctx = svo->ctx;
  if (!lambda || !origin || !width || !iso || !num_verts || n_iso < 1 || n_iso > 64 || res < 1 || res > 2048 ||
      (field_mode != 0 && field_mode != 1))
    return setError(ctx, ITS_ERR_INVALID, "its_eval_grid_mc: bad arguments");
  if (tri_verts && !capacity) return setError(ctx, ITS_ERR_INVALID, "its_eval_grid_mc: capacities missing");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  const int64_t M = (int64_t)res + 1;
  DevBuf<double> field;
  its_status st;
  if ((st = field.alloc(ctx, M * M * M)) != ITS_OK) return st;
  st = field_mode == 1 ? its_eval_grid_fast(svo, lambda, origin, width, res, field.p)
                       : its_eval_grid(svo, lambda, origin, width, res, field.p);
  if (st != ITS_OK) return st;
  for (int k = 0; k < n_iso; ++k) {
    double* out = tri_verts ? tri_verts[k] : nullptr;
    const int64_t cap = out ? capacity[k] : 0;
    if ((st = its_marching_cubes(ctx, field.p, res, origin, width, iso[k], nullptr, out, cap, &num_verts[k])) != ITS_OK)
      return st;
  }
  return ITS_OK;
}

}  // extern "C"
