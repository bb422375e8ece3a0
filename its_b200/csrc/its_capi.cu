// C ABI core: context lifetime, errors, host-side model pre-processing (BaseModel.cpp),
// triangle attributes and mesh validation.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "its_ctx.cuh"
#include "its_svo.cuh"

namespace its {

void saveTuneCache(its_ctx* ctx) {
  if (ctx->tuneCache.empty()) return;
  if (FILE* f = std::fopen(ctx->tuneCache.c_str(), "w")) {
    for (const auto& kv : ctx->tuned) std::fprintf(f, "%s %d\n", kv.first.c_str(), kv.second);
    std::fclose(f);
  }
}


its_status setError(its_ctx* ctx, its_status code, const std::string& msg) {
  if (ctx) ctx->lastError = msg;
  return code;
}
its_status cudaFail(its_ctx* ctx, cudaError_t e, const char* what) {
  const std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return setError(ctx, e == cudaErrorMemoryAllocation ? ITS_ERR_OOM : ITS_ERR_CUDA, m);
}

__global__ void kValidateMesh(const double* __restrict__ V, int64_t nv, const int32_t* __restrict__ F, int64_t nf,
                              unsigned* bad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < nv * 3 && !isfinite(V[i])) atomicOr(bad, 1u);
  if (i < nf * 3 && (F[i] < 0 || (int64_t)F[i] >= nv)) atomicOr(bad, 2u);
}

its_status validateMesh(its_ctx* ctx, const double* dV, int64_t nv, const int32_t* dF, int64_t nf) {
  DevBuf<unsigned> bad;
  its_status st;
  if ((st = bad.zeros(ctx, 1)) != ITS_OK) return st;
  const int64_t n = std::max(nv, nf) * 3;
  kValidateMesh<<<gridFor(n, 256), 256, 0, ctx->stream>>>(dV, nv, dF, nf, bad.p);
  ITS_LAUNCHED(ctx);
  unsigned h = 0;
  ITS_CU(ctx, cudaMemcpyAsync(&h, bad.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  if (h & 1u) return setError(ctx, ITS_ERR_INVALID, "mesh has non-finite vertex coordinates");
  if (h & 2u) return setError(ctx, ITS_ERR_INVALID, "mesh has face indices outside [0, nverts)");
  return ITS_OK;
}

// modelTriAttributeKernel (CUDACompute.cu:79-96).
__global__ void kTriAttributes(const double* __restrict__ V, const int32_t* __restrict__ F, int64_t nf,
                               double* normal, double* area, double* dir) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nf) return;
  const int32_t a = F[3 * t], b = F[3 * t + 1], c = F[3 * t + 2];
  const double p1x = V[3 * a], p1y = V[3 * a + 1], p1z = V[3 * a + 2];
  const double ux = V[3 * b] - p1x, uy = V[3 * b + 1] - p1y, uz = V[3 * b + 2] - p1z;
  const double vx = V[3 * c] - p1x, vy = V[3 * c + 1] - p1y, vz = V[3 * c + 2] - p1z;
  const double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
  if (normal) { normal[3 * t] = nx; normal[3 * t + 1] = ny; normal[3 * t + 2] = nz; }
  if (area) {
    double s = nx * nx;
    s = s + ny * ny;
    s = s + nz * nz;
    area[t] = 0.5 * sqrt(s);
  }
  if (dir) {
    double s = -nx * p1x;
    s = s + -ny * p1y;
    s = s + -nz * p1z;
    dir[t] = s;
  }
}

}  // namespace its

using namespace its;

extern "C" {

const char* its_version(void) { return "its-b200 0.1 (sm_100a)"; }

its_status its_create(its_ctx** out, int device) {
  if (!out) return ITS_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return ITS_ERR_CUDA;
  }
  if (device < 0 || device >= n) return ITS_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return ITS_ERR_CUDA;
  its_ctx* c = new its_ctx;
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->ownStream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return ITS_ERR_CUDA;
  }
  c->stream = c->ownStream;
  cudaDeviceGetAttribute(&c->numSMs, cudaDevAttrMultiProcessorCount, device);
  // The context's own stream-ordered pool keeps freed blocks across synchronisations: with a
  // release threshold of 0 every sync would hand memory back and the next allocation would
  // map it again, which costs far more than the fit's kernels.
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  if (cudaMemPoolCreate(&c->pool, &props) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  } else {
    cudaGetLastError();
    c->pool = nullptr;
  }
  if (cudaMallocHost((void**)&c->pinned, 256) != cudaSuccess) {
    cudaGetLastError();
    if (c->pool) cudaMemPoolDestroy(c->pool);
    cudaStreamDestroy(c->ownStream);
    delete c;
    return ITS_ERR_CUDA;
  }
  *out = c;
  return ITS_OK;
}

its_status its_destroy(its_ctx* c) {
  if (!c) return ITS_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  its::hostIoRelease(c);
  if (c->mapSlab) cudaFreeHost(c->mapSlab);
  if (c->ownStream) cudaStreamDestroy(c->ownStream);
  if (c->pool) cudaMemPoolDestroy(c->pool);  // released once nothing allocated from it is live
  if (c->pinned) cudaFreeHost(c->pinned);
  delete c;
  return ITS_OK;
}

const char* its_last_error(const its_ctx* c) { return c ? c->lastError.c_str() : "no context"; }

its_status its_set_stream(its_ctx* c, void* s) {
  if (!c) return ITS_ERR_INVALID;
  c->stream = s ? (cudaStream_t)s : c->ownStream;
  return ITS_OK;
}

its_status its_synchronize(its_ctx* c) {
  if (!c) return ITS_ERR_INVALID;
  ITS_CU(c, cudaStreamSynchronize(c->stream));
  return ITS_OK;
}

int64_t its_kernel_launches(const its_ctx* c) { return c ? c->launches : 0; }

its_status its_set_autotune(its_ctx* c, int enable, const char* cache_path) {
  if (!c) return ITS_ERR_INVALID;
  c->autotune = enable ? 1 : 0;
  c->tuneCache = cache_path ? cache_path : "";
  if (!c->tuneCache.empty()) {  // load earlier choices: one "key value" pair per line
    if (FILE* f = std::fopen(c->tuneCache.c_str(), "r")) {
      char key[512];
      int v;
      while (std::fscanf(f, "%511s %d", key, &v) == 2) c->tuned[key] = v;
      std::fclose(f);
    }
  }
  return ITS_OK;
}

its_status its_autotune_choices(const its_ctx* c, char* buf, int64_t size, int64_t* length) {
  if (!c || !length) return ITS_ERR_INVALID;
  std::string out;
  for (const auto& kv : c->tuned) out += kv.first + " " + std::to_string(kv.second) + "\n";
  *length = (int64_t)out.size();
  if (buf && size > 0) {
    const int64_t k = std::min<int64_t>(size - 1, (int64_t)out.size());
    std::memcpy(buf, out.data(), (size_t)k);
    buf[k] = 0;
  }
  return ITS_OK;
}

// BaseModel::calcUnitCubeTransformMatrix + model2UnitCube (BaseModel.cpp:54-92): host code in
// the reference as well; centre the box, scale its longest side to scale_factor^-1.
its_status its_model_to_unit_cube(double* V, int64_t nv, double scaleFactor) {
  if (!V || nv <= 0 || !(scaleFactor > 0.0)) return ITS_ERR_INVALID;
  double bmin[3] = {V[0], V[1], V[2]}, bmax[3] = {V[0], V[1], V[2]};
  for (int64_t i = 1; i < nv; ++i)
    for (int a = 0; a < 3; ++a) {
      bmin[a] = std::min(bmin[a], V[3 * i + a]);
      bmax[a] = std::max(bmax[a], V[3 * i + a]);
    }
  double scale = bmax[0] - bmin[0];
  for (int d = 1; d < 3; ++d) scale = std::max<double>(scale, bmax[d] - bmin[d]);
  scale *= scaleFactor;
  if (!(scale > 0.0) || !std::isfinite(scale)) return ITS_ERR_INVALID;
  double center[3];
  for (int a = 0; a < 3; ++a) center[a] = 0.5 * bmax[a] + 0.5 * bmin[a];
  for (int a = 0; a < 3; ++a) center[a] -= scale / 2;
  const double inv = 1. / scale;
  for (int64_t i = 0; i < nv; ++i)
    for (int a = 0; a < 3; ++a) V[3 * i + a] = (V[3 * i + a] + (-center[a])) * inv;
  return ITS_OK;
}

// BaseModel::setUniformBoundingBox (BaseModel.cpp:24-51): pad the short axes by half the
// FLOAT difference to the longest one, then every side by width/11.
its_status its_uniform_bbox(const double* V, int64_t nv, double origin[3], double end[3], double width[3]) {
  if (!V || nv <= 0 || !origin) return ITS_ERR_INVALID;
  double mn[3] = {V[0], V[1], V[2]}, mx[3] = {V[0], V[1], V[2]};
  for (int64_t i = 1; i < nv; ++i)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], V[3 * i + a]);
      mx[a] = std::max(mx[a], V[3 * i + a]);
    }
  double o[3], e[3], len[3];
  for (int a = 0; a < 3; ++a) { o[a] = mn[a]; e[a] = mx[a]; len[a] = mx[a] - mn[a]; }
  const float maxLen = (float)dmax(len[0], dmax(len[1], len[2]));
  for (int a = 0; a < 3; ++a) {
    if ((double)maxLen == len[a]) continue;
    const float delta = (float)((double)maxLen - len[a]);
    o[a] = mn[a] - (double)(delta / 2.0f);
    e[a] = mx[a] + (double)(delta / 2.0f);
  }
  double eps[3];
  for (int a = 0; a < 3; ++a) eps[a] = (e[a] - o[a]) / 11;
  for (int a = 0; a < 3; ++a) {
    o[a] = o[a] - eps[a];
    e[a] = e[a] + eps[a];
    origin[a] = o[a];
    if (end) end[a] = e[a];
    if (width) width[a] = e[a] - o[a];
  }
  return ITS_OK;
}

its_status its_tri_attributes(its_ctx* ctx, const double* verts, int64_t nverts, const int32_t* faces, int64_t nfaces,
                              double* normal, double* area, double* dir) {
  if (!ctx) return ITS_ERR_INVALID;
  if (!verts || !faces || nverts <= 0 || nfaces <= 0) return setError(ctx, ITS_ERR_INVALID, "its_tri_attributes: empty mesh");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> V;
  InArg<int32_t> F;
  OutArg<double> N, A, D;
  its_status st;
  if ((st = V.stage(ctx, verts, 3 * nverts)) != ITS_OK) return st;
  if ((st = F.stage(ctx, faces, 3 * nfaces)) != ITS_OK) return st;
  if ((st = validateMesh(ctx, V.d, nverts, F.d, nfaces)) != ITS_OK) return st;
  if ((st = N.stage(ctx, normal, 3 * nfaces)) != ITS_OK) return st;
  if ((st = A.stage(ctx, area, nfaces)) != ITS_OK) return st;
  if ((st = D.stage(ctx, dir, nfaces)) != ITS_OK) return st;
  kTriAttributes<<<gridFor(nfaces, 256), 256, 0, ctx->stream>>>(V.d, F.d, nfaces, N.d, A.d, D.d);
  ITS_LAUNCHED(ctx);
  if ((st = N.finish(ctx)) != ITS_OK) return st;
  if ((st = A.finish(ctx)) != ITS_OK) return st;
  if ((st = D.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // extern "C"
