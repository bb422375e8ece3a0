// Dense field on a lattice aligned with the octree, by prolongation.
//
// The field of MC::launch_computSDFKernel (MarchingCubes.cu:464-536, CUDACompute.cu:435-510)
// is F = sum over depths d of f_d, f_d(p) = sum over the depth-d corner vertices v of
// lambda_v * hat_v(p): on each depth-d lattice cell, the trilinear interpolant of the cell's
// corner coefficients (0 where the corner is not a vertex). When the output lattice is the
// octree's own box at res * 2^k points per axis, every output point sits on a dyadic point of
// every depth's lattice, and F can be built coarse to fine on dense per-depth lattices:
//   D_{root} = lambda at the root corners;   D_d = lambda at the depth-d corners + P(D_{d+1});
//   out = P^k(D_0),
// P the trilinear prolongation to the next finer lattice (a point between coarse points takes
// their mean: weights 1, 1/2, 1/4, 1/8 per point, exact in floating point). Each level is one
// pass over its lattice that reads an eighth as much: the cost is that of writing the output
// once (8 B per point), where evaluating every point from its cells at all depths
// (its_eval_grid, bit-identical to the reference's sums) is bound by hat arithmetic. The sums
// differ from the reference's by rounding only: the hats are centred on the exact lattice
// positions, the representative vertex positions of the octree differ from them by ulps.
#include <cmath>
#include <vector>

#include "its_op.cuh"
#include "its_svo.cuh"

namespace its {

template <typename T>
__global__ void kScatterCorners(int64_t n, const uint64_t* __restrict__ vertKey, const double* __restrict__ lambda,
                                const int64_t* __restrict__ off, const int64_t* __restrict__ Ms, T* __restrict__ D) {
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= n) return;
  const VertCoord c = decodeVertKey(vertKey[v]);
  const int64_t M = Ms[c.d];
  D[off[c.d] + c.X + M * (c.Y + M * (int64_t)c.Z)] = (T)lambda[v];
}

// fine = (accumulate ? fine : 0) + the trilinear prolongation of coarse by the factor 2^s
// (fine has Mf = (Mc - 1) 2^s + 1 points per axis, x fastest). One thread per coarse x
// interval and fine (y, z): it reads the interval's ends on the <= 4 coarse rows around
// (y, z) and writes the 2^s fine points of the interval (the last coarse point: one), so a
// warp's stores are contiguous. Blocks of 32 intervals x 8 fine rows; z per block.
template <typename T, int S>
__global__ void __launch_bounds__(256) kProlong(const T* __restrict__ coarse, int Mc, T* __restrict__ fine,
                                                int accumulate) {
  constexpr int F = 1 << S;
  const int Mf = (Mc - 1) * F + 1;
  const int xc = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
  if (xc >= Mc || y >= Mf) return;
  const int ry = y & (F - 1), rz = z & (F - 1);
  const int cy = y >> S, cz = z >> S;
  const T wy1 = (T)ry / (T)F, wz1 = (T)rz / (T)F;  // exact: F is a power of two
  const bool xr = xc + 1 < Mc;                       // the interval has a right end
  const T* base = coarse + ((int64_t)cz * Mc + cy) * Mc + xc;
  const int64_t rowY = Mc, rowZ = (int64_t)Mc * Mc;
  // the coarse field at x = xc and xc + 1, interpolated in y and z
  T a0 = base[0], a1 = xr ? base[1] : T(0);
  if (ry) {
    a0 = (T(1) - wy1) * a0 + wy1 * base[rowY];
    if (xr) a1 = (T(1) - wy1) * a1 + wy1 * base[rowY + 1];
  }
  if (rz) {
    T b0 = base[rowZ], b1 = xr ? base[rowZ + 1] : T(0);
    if (ry) {
      b0 = (T(1) - wy1) * b0 + wy1 * base[rowZ + rowY];
      if (xr) b1 = (T(1) - wy1) * b1 + wy1 * base[rowZ + rowY + 1];
    }
    a0 = (T(1) - wz1) * a0 + wz1 * b0;
    a1 = (T(1) - wz1) * a1 + wz1 * b1;
  }
  T* out = fine + ((int64_t)z * Mf + y) * Mf + (int64_t)xc * F;
#pragma unroll
  for (int r = 0; r < F; ++r) {
    if (r > 0 && !xr) break;
    const T w1 = (T)r / (T)F;
    const T v = r ? (T(1) - w1) * a0 + w1 * a1 : a0;
    out[r] = accumulate ? out[r] + v : v;
  }
}

template <typename T>
static its_status prolong(its_ctx* ctx, const T* coarse, int64_t Mc, T* fine, int s, int accumulate) {
  const int64_t Mf = (Mc - 1) * ((int64_t)1 << s) + 1;
  const dim3 grid((unsigned)((Mc + 31) / 32), (unsigned)((Mf + 7) / 8), (unsigned)Mf), block(32, 8);
  switch (s) {
    case 1: kProlong<T, 1><<<grid, block, 0, ctx->stream>>>(coarse, (int)Mc, fine, accumulate); break;
    case 2: kProlong<T, 2><<<grid, block, 0, ctx->stream>>>(coarse, (int)Mc, fine, accumulate); break;
    default: kProlong<T, 3><<<grid, block, 0, ctx->stream>>>(coarse, (int)Mc, fine, accumulate); break;
  }
  ITS_LAUNCHED(ctx);
  return ITS_OK;
}

// Whether the lattice (origin, width, res) is the octree's box at res_octree * 2^s points: per
// axis the octree's origin and cell width (the octree sizes its cells by its first axis) to
// within 1e-6 of a cell. Boxes padded in single precision (BaseModel.cpp:24-51) have axes a
// few 1e-9 apart; the cascade's points are then the octree's lattice points, at most that far
// from the requested ones.
static bool alignedLattice(const SvoDevice& d, const double origin[3], const double width[3], int res, int* s) {
  const double u = d.unit[0];
  for (int a = 0; a < 3; ++a)
    if (fabs(origin[a] - d.origin[a]) > 1e-6 * u || fabs(width[a] / d.res - u) > 1e-6 * u) return false;
  for (int k = 0; k <= 3; ++k)
    if ((int64_t)d.res << k == res) {
      *s = k;
      return true;
    }
  return false;
}

template <typename T>
static its_status cascade(its_ctx* ctx, const SvoDevice& d, const double* lambda, int res, int s, T* out) {
  its_status st;
  const int D = d.depth;
  std::vector<int64_t> M(D), off(D + 1, 0);
  for (int k = 0; k < D; ++k) {
    M[k] = (int64_t)(d.res >> k) + 1;
    off[k + 1] = off[k] + M[k] * M[k] * M[k];
  }
  // with s == 0 the output is depth 0's lattice itself
  const int64_t inner = s == 0 ? off[D] - off[1] : off[D];
  DevBuf<T> lat;
  DevBuf<int64_t> tab;
  if ((st = lat.alloc(ctx, std::max<int64_t>(inner, 1))) != ITS_OK || (st = tab.alloc(ctx, 2 * (D + 1))) != ITS_OK)
    return st;
  std::vector<int64_t> h(2 * (D + 1), 0);
  for (int k = 0; k < D; ++k) h[k] = M[k];
  for (int k = 0; k < D; ++k) h[D + 1 + k] = s == 0 ? (k == 0 ? 0 : off[k] - off[1]) : off[k];
  ITS_CU(ctx, cudaMemcpyAsync(tab.p, h.data(), h.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  auto level = [&](int k) -> T* { return s == 0 ? (k == 0 ? out : lat.p + (off[k] - off[1])) : lat.p + off[k]; };
  ITS_CU(ctx, cudaMemsetAsync(lat.p, 0, std::max<int64_t>(inner, 1) * sizeof(T), ctx->stream));
  if (s == 0) ITS_CU(ctx, cudaMemsetAsync(out, 0, M[0] * M[0] * M[0] * sizeof(T), ctx->stream));
  if (d.numVerts > 0) {
    if (s == 0) {
      // depth 0 goes to the output, the rest to the scratch lattices (offsets already shifted)
      kScatterCorners<T><<<gridFor(d.vertCount[0], 256), 256, 0, ctx->stream>>>(d.vertCount[0], d.vertKey, lambda,
                                                                               tab.p + D + 1, tab.p, out);
      ITS_LAUNCHED(ctx);
      const int64_t rest = d.numVerts - d.vertStart[1 < D ? 1 : D];
      if (rest > 0) {
        kScatterCorners<T><<<gridFor(rest, 256), 256, 0, ctx->stream>>>(rest, d.vertKey + d.vertStart[1], lambda +
                                                                         d.vertStart[1], tab.p + D + 1, tab.p, lat.p);
        ITS_LAUNCHED(ctx);
      }
    } else {
      kScatterCorners<T><<<gridFor(d.numVerts, 256), 256, 0, ctx->stream>>>(d.numVerts, d.vertKey, lambda,
                                                                           tab.p + D + 1, tab.p, lat.p);
      ITS_LAUNCHED(ctx);
    }
  }
  for (int k = D - 2; k >= 0; --k)
    if ((st = prolong<T>(ctx, level(k + 1), M[k + 1], level(k), 1, 1)) != ITS_OK) return st;
  if (s > 0 && (st = prolong<T>(ctx, level(0), M[0], out, s, 0)) != ITS_OK) return st;
  return ITS_OK;
}

template <typename T>
static its_status evalGridFast(its_svo* sv, const double* lambda, const double origin[3], const double width[3],
                               int res, T* field) {
  if (!sv || !lambda || !origin || !width || !field || res < 1 || res > 2048) return ITS_ERR_INVALID;
  its_ctx* ctx = sv->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  int s = 0;
  if (!alignedLattice(sv->d, origin, width, res, &s)) {  // any other lattice: point by point
    if (sizeof(T) == 8) return its_eval_grid(sv, lambda, origin, width, res, (double*)field);
    return its_eval_grid_f32(sv, lambda, origin, width, res, (float*)field);
  }
  const int64_t Mo = (int64_t)res + 1;
  InArg<double> L;
  OutArg<T> F;
  its_status st;
  if ((st = L.stage(ctx, lambda, sv->d.numVerts)) != ITS_OK || (st = F.stage(ctx, field, Mo * Mo * Mo)) != ITS_OK)
    return st;
  if ((st = cascade<T>(ctx, sv->d, L.d, res, s, F.d)) != ITS_OK) return st;
  if ((st = F.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // namespace its

using namespace its;

extern "C" {

its_status its_eval_grid_fast(its_svo* svo, const double* lambda, const double origin[3], const double width[3],
                              int res, double* field) {
  return evalGridFast<double>(svo, lambda, origin, width, res, field);
}

its_status its_eval_grid_fast_f32(its_svo* svo, const double* lambda, const double origin[3], const double width[3],
                                  int res, float* field) {
  return evalGridFast<float>(svo, lambda, origin, width, res, field);
}

}  // extern "C"
