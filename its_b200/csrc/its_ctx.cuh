// Context, device buffers and host/device argument staging for the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <utility>

#include "its_internal.cuh"

namespace its {
struct HostIo;  // pinned staging and host threads for large copies into pageable memory (its_hostio.cu)
}

struct its_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t ownStream = nullptr;
  std::string lastError;
  int64_t launches = 0;
  int numSMs = 148;
  cudaMemPool_t pool = nullptr;  // the context's stream-ordered allocator
  int* pinned = nullptr;         // 256 bytes of pinned host memory for small device reads
  // autotuner: launch shapes chosen by measurement (its_tune.cuh)
  int autotune = 0;                  // 0: built-in defaults, 1: measure candidates on first use
  std::map<std::string, int> tuned;  // shape key -> chosen candidate
  std::string tuneCache;             // file the choices persist to ("" = none)
  // while a CUDA graph is captured, device buffers come from this bump arena (owned by the
  // graph's plan) instead of the pool, so the graph holds no allocation nodes
  uint8_t* arena = nullptr;
  size_t arenaCap = 0, arenaOff = 0;
  its::HostIo* hostio = nullptr;  // created on the first large copy into pageable memory
  // mapped pinned words handed out in 64-byte slots (learned-fit plans: residual, flags, clocks)
  double* mapSlab = nullptr;
  uint64_t mapUsed = 0;  // one bit per slot
};

namespace its {

// Count and check a kernel launch on the context's stream.
#define ITS_LAUNCHED(ctx)                                          \
  do {                                                             \
    (ctx)->launches++;                                             \
    cudaError_t e__ = cudaGetLastError();                          \
    if (e__ != cudaSuccess) return ::its::cudaFail((ctx), e__, "kernel launch"); \
  } while (0)

inline its_status devAlloc(its_ctx* ctx, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return ITS_OK;
  if (ctx->arena) {
    const size_t off = (ctx->arenaOff + 255) & ~(size_t)255;
    if (off + bytes > ctx->arenaCap) return setError(ctx, ITS_ERR_OOM, "capture arena exhausted");
    *p = ctx->arena + off;
    ctx->arenaOff = off + bytes;
    return ITS_OK;
  }
  cudaError_t e = ctx->pool ? cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream)
                            : cudaMallocAsync(p, bytes, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return setError(ctx, e == cudaErrorMemoryAllocation ? ITS_ERR_OOM : ITS_ERR_CUDA,
                    std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " +
                        cudaGetErrorString(e));
  }
  return ITS_OK;
}
inline void devFree(its_ctx* ctx, void* p) {
  if (ctx->arena && (uint8_t*)p >= ctx->arena && (uint8_t*)p < ctx->arena + ctx->arenaCap) return;
  if (p) cudaFreeAsync(p, ctx->stream);
}

// Stream-ordered device buffer owned by one C-ABI call (or by an object).
template <typename T>
struct DevBuf {
  its_ctx* ctx = nullptr;
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(its_ctx* c) : ctx(c) {}
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ctx(o.ctx), p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { reset(); ctx = o.ctx; p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { reset(); }
  its_status alloc(its_ctx* c, size_t count) {
    reset();
    ctx = c;
    n = count;
    return devAlloc(c, (void**)&p, count * sizeof(T));
  }
  its_status zeros(its_ctx* c, size_t count) {
    its_status s = alloc(c, count);
    if (s != ITS_OK) return s;
    if (count) ITS_CU(c, cudaMemsetAsync(p, 0, count * sizeof(T), c->stream));
    return ITS_OK;
  }
  void reset() {
    if (p && ctx) devFree(ctx, p);
    p = nullptr;
    n = 0;
  }
  T* release() { T* q = p; p = nullptr; n = 0; return q; }
};

// Where an argument lives, seen from the context's device: its own device memory (or managed
// memory, which every GPU can reach), host memory, or device memory of another GPU -- which a
// kernel of this device may not be able to read, so callers reject it.
enum class MemKind { Host, Device, OtherDevice };
inline MemKind memKind(const void* p, int device) {
  if (!p) return MemKind::Host;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return MemKind::Host;
  }
  if (a.type == cudaMemoryTypeManaged) return MemKind::Device;
  if (a.type == cudaMemoryTypeDevice) return a.device == device ? MemKind::Device : MemKind::OtherDevice;
  return MemKind::Host;
}
// The same with host memory split into page-locked and pageable, from one attribute query.
enum class PtrClass { Pageable, Pinned, Device, OtherDevice };
inline PtrClass ptrClass(const void* p, int device) {
  if (!p) return PtrClass::Pageable;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return PtrClass::Pageable;
  }
  if (a.type == cudaMemoryTypeManaged) return PtrClass::Device;
  if (a.type == cudaMemoryTypeDevice) return a.device == device ? PtrClass::Device : PtrClass::OtherDevice;
  return a.type == cudaMemoryTypeHost ? PtrClass::Pinned : PtrClass::Pageable;
}
// True when p is device (or managed) memory the context's device can use directly.
inline bool isDevicePtr(const its_ctx* ctx, const void* p) { return memKind(p, ctx->device) == MemKind::Device; }
inline its_status otherDeviceError(its_ctx* ctx) {
  return setError(ctx, ITS_ERR_INVALID, "an argument is device memory of another GPU than the context's");
}

// True when p is page-locked host memory the GPU can copy from and to asynchronously.
inline bool isPinnedHostPtr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// A read-only argument on the device: the caller's pointer if it already is device
// memory, else a staged copy.
// Large copies between pageable host memory and the device through two pinned chunks, the
// host side of each chunk copied by several host threads (its_hostio.cu). To the host: returns
// with the data in dst. To the device: returns once the last chunk is queued on the context's
// stream (later work on the stream sees the data).
constexpr size_t kStagedCopyMin = 8u << 20;     // to the host: parallel first touch of the pages
constexpr size_t kStagedUploadMin = 32u << 20;  // to the device: below this the driver's path is as fast
its_status copyToHostStaged(its_ctx* ctx, void* dst, const void* src, size_t bytes);
its_status copyToDeviceStaged(its_ctx* ctx, void* dst, const void* src, size_t bytes);
void hostIoRelease(its_ctx* ctx);

template <typename T>
struct InArg {
  const T* d = nullptr;
  DevBuf<T> tmp;
  its_status stage(its_ctx* ctx, const T* src, size_t count) {
    if (!src || count == 0) { d = nullptr; return ITS_OK; }
    const MemKind k = memKind(src, ctx->device);
    if (k == MemKind::OtherDevice) return otherDeviceError(ctx);
    if (k == MemKind::Device) { d = src; return ITS_OK; }
    its_status s = tmp.alloc(ctx, count);
    if (s != ITS_OK) return s;
    d = tmp.p;
    if (count * sizeof(T) >= kStagedUploadMin && !ctx->arena && ptrClass(src, ctx->device) == PtrClass::Pageable)
      return copyToDeviceStaged(ctx, tmp.p, src, count * sizeof(T));
    ITS_CU(ctx, cudaMemcpyAsync(tmp.p, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return ITS_OK;
  }
};

// A written argument: device scratch copied back to a host destination by finish().
template <typename T>
struct OutArg {
  T* d = nullptr;
  T* host = nullptr;
  size_t count = 0;
  DevBuf<T> tmp;
  its_status stage(its_ctx* ctx, T* dst, size_t n) {
    count = n;
    host = nullptr;
    if (!dst || n == 0) { d = nullptr; return ITS_OK; }
    const MemKind k = memKind(dst, ctx->device);
    if (k == MemKind::OtherDevice) return otherDeviceError(ctx);
    if (k == MemKind::Device) { d = dst; return ITS_OK; }
    its_status s = tmp.alloc(ctx, n);
    if (s != ITS_OK) return s;
    d = tmp.p;
    host = dst;
    return ITS_OK;
  }
  // Large results into pageable memory go through copyToHostStaged (synchronous), the rest
  // by one asynchronous copy that the caller's stream synchronisation completes.
  its_status finish(its_ctx* ctx) {
    if (!host || !count) return ITS_OK;
    const size_t bytes = count * sizeof(T);
    if (bytes >= kStagedCopyMin && !ctx->arena && ptrClass(host, ctx->device) == PtrClass::Pageable)
      return copyToHostStaged(ctx, host, d, bytes);
    ITS_CU(ctx, cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return ITS_OK;
  }
};

inline unsigned gridFor(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }

// Programmatic dependent launch: a kernel launched by launchDependent may be scheduled while
// the kernel before it in the stream is still running, once every block of that kernel has
// passed gridDependents(). It must call gridDependencyWait() before it reads anything earlier
// work writes or writes anything earlier work reads; past that call all earlier work is
// complete and visible. (Launched the ordinary way, both calls return at once.)
// The device's global nanosecond clock.
__device__ __forceinline__ unsigned long long globalTimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void gridDependencyWait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void gridDependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// dependent = false launches the ordinary way. Only a launch whose previous operation in the
// stream is a kernel may be dependent: the relaxed ordering does not cover copies, memsets,
// event waits or stream-ordered allocations in between.
template <typename... KArgs, typename... Args>
its_status launchDependent(its_ctx* ctx, bool dependent, void (*kernel)(KArgs...), dim3 grid, dim3 block,
                           size_t smem, cudaStream_t stream, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = dependent ? 1 : 0;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
  ctx->launches++;
  if (e != cudaSuccess) {
    cudaGetLastError();
    return cudaFail(ctx, e, "kernel launch");
  }
  return ITS_OK;
}

}  // namespace its
