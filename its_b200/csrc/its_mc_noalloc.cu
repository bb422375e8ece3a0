// its_marching_cubes_noalloc: marching cubes that allocates no device memory.
//
// Some callers of this library cannot let it call cudaMalloc: a host application that
// reserves the GPU's memory for its own allocator at start-up and runs every later frame
// inside that fixed budget (an allocation there can fail, or take memory the application has
// promised elsewhere), and a frame loop that must not stall, since cudaMalloc and cudaFree can
// synchronise the device. For them this entry point computes the same case indices and
// triangle soup as its_marching_cubes, but its scan scratch (one block sum per 2,048 voxels
// plus the grand total) lives in a fixed file-scope device array instead of being allocated
// per call.
//
// Limits and rules:
//   * res <= 256 (16,777,216 voxels): the array holds 8,193 64-bit words (64 KiB) and every
//     GPU that loads libits keeps it until the process exits;
//   * field, cube_index and tri_verts must already be device memory of the context's GPU (a
//     host pointer would need a staging allocation) -- anything else is rejected with
//     ITS_ERR_INVALID;
//   * every call on a device shares the one array, which keeps the last call's contents (each
//     call rewrites every word it reads); calls that overlap on the GPU (two streams, two host
//     threads) race on it;
//   * the call waits for its stream to read the vertex count back to the host;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress,
//     with that device current) and keeps it for the life of the process: calling
//     cudaDeviceReset on that device afterwards is not supported.
#include <mutex>

#include "its_mc.cuh"
#include "its_scan.cuh"

namespace its {
namespace {

constexpr int64_t kNoAllocMaxRes = 256;
constexpr int64_t kNoAllocMaxVoxels = kNoAllocMaxRes * kNoAllocMaxRes * kNoAllocMaxRes;
constexpr int64_t kNoAllocSpine = (kNoAllocMaxVoxels + kScanTile - 1) / kScanTile;  // 8,192 block sums

// Block sums of the count scan, then the grand total in the last word.
static __device__ __align__(256) unsigned long long gMcScratch[kNoAllocSpine + 1];

constexpr int kMaxDevices = 64;
std::mutex gScratchMu;
unsigned long long* gScratchAddr[kMaxDevices] = {};

// Device address of gMcScratch on the context's device (looked up once per device).
its_status scratchFor(its_ctx* ctx, unsigned long long** out) {
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return setError(ctx, ITS_ERR_INVALID, "its_marching_cubes_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(gScratchMu);
  if (!gScratchAddr[ctx->device]) {
    ITS_CU(ctx, cudaSetDevice(ctx->device));
    void* p = nullptr;
    ITS_CU(ctx, cudaGetSymbolAddress(&p, gMcScratch));
    gScratchAddr[ctx->device] = static_cast<unsigned long long*>(p);
  }
  *out = gScratchAddr[ctx->device];
  return ITS_OK;
}

}  // namespace
}  // namespace its

using namespace its;

extern "C" {

its_status its_marching_cubes_noalloc(its_ctx* ctx, const double* field, int res, const double origin[3],
                                      const double width[3], double iso, uint8_t* cube_index, double* tri_verts,
                                      int64_t capacity, int64_t* num_verts) {
  if (!ctx) return ITS_ERR_INVALID;
  if (!field || !origin || !width || !num_verts || res < 1 || capacity < 0)
    return setError(ctx, ITS_ERR_INVALID, "its_marching_cubes_noalloc: bad arguments");
  if (res > kNoAllocMaxRes)
    return setError(ctx, ITS_ERR_INVALID,
                    "its_marching_cubes_noalloc: res " + std::to_string(res) + " exceeds the maximum of 256 "
                    "(fixed scratch of 8,193 words); use its_marching_cubes");
  if (!isDevicePtr(ctx, field) || (cube_index && !isDevicePtr(ctx, cube_index)) ||
      (tri_verts && !isDevicePtr(ctx, tri_verts)))
    return setError(ctx, ITS_ERR_INVALID,
                    "its_marching_cubes_noalloc: field and outputs must be device memory of the context's GPU");
  // the vertex count is read back with a stream synchronisation, which a capturing stream
  // does not allow: refuse before anything is queued rather than break the caller's capture
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  ITS_CU(ctx, cudaStreamIsCapturing(ctx->stream, &cap));
  if (cap != cudaStreamCaptureStatusNone)
    return setError(ctx, ITS_ERR_INVALID,
                    "its_marching_cubes_noalloc: the stream is capturing; this call waits for the vertex count");
  unsigned long long* scratch = nullptr;
  its_status st = scratchFor(ctx, &scratch);
  if (st != ITS_OK) return st;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  const int64_t nvox = (int64_t)res * res * res;
  McCase mc{field, res, iso};
  McEmit em{mc, make_double3(origin[0], origin[1], origin[2]),
            make_double3(width[0] / res, width[1] / res, width[2] / res), cube_index, tri_verts,
            (unsigned long long)(tri_verts ? capacity : 0)};
  unsigned long long* total = scratch + kNoAllocSpine;
  if ((st = scanExclusive<unsigned long long>(ctx, mc, nvox, em, total, scratch)) != ITS_OK) return st;
  unsigned long long h = 0;
  ITS_CU(ctx, cudaMemcpyAsync(&h, total, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  *num_verts = (int64_t)h;
  return ITS_OK;
}

}  // extern "C"
