// Large device-to-host copies into pageable memory. A plain cudaMemcpy to pageable memory
// goes through the driver's staging buffer and one host thread, and the destination's pages
// are first touched (faulted in and zeroed by the kernel) inside that copy: for a fresh
// buffer of tens of MB that first touch, not the PCIe/C2C transfer, sets the time. Here the
// device data goes by DMA into two pinned chunks in turn, and each chunk is copied on into the
// destination by a pool of host threads, so the page faults of different parts of the buffer
// are taken in parallel while the next chunk is in flight.
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "its_ctx.cuh"

namespace its {

namespace {
constexpr size_t kChunk = 16u << 20;  // bytes per pinned chunk (two of them)
constexpr size_t kPage = 4096;

// A fixed pool of host threads running one parallel-for at a time.
class HostPool {
 public:
  explicit HostPool(int n) {
    for (int i = 0; i < n; ++i) workers_.emplace_back([this, i] { loop(i); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  int size() const { return (int)workers_.size() + 1; }
  // Runs fn(part) for part = 0..parts-1 on the workers and the calling thread.
  void run(int parts, const std::function<void(int)>& fn) {
    {
      std::lock_guard<std::mutex> g(m_);
      fn_ = &fn;
      parts_ = parts;
      next_ = 0;
      busy_ = (int)workers_.size();
      ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> l(m_);
    done_.wait(l, [this] { return busy_ == 0; });
    fn_ = nullptr;
  }

 private:
  void work() {
    for (;;) {
      int p;
      {
        std::lock_guard<std::mutex> g(m_);
        if (!fn_ || next_ >= parts_) return;
        p = next_++;
      }
      (*fn_)(p);
    }
  }
  void loop(int) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      work();
      {
        std::lock_guard<std::mutex> g(m_);
        if (--busy_ == 0) done_.notify_all();
      }
    }
  }
  std::vector<std::thread> workers_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* fn_ = nullptr;
  int parts_ = 0, next_ = 0, busy_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};
}  // namespace

struct HostIo {
  uint8_t* stage[2] = {nullptr, nullptr};
  cudaEvent_t ready[2] = {nullptr, nullptr};
  HostPool* pool = nullptr;
};

void hostIoRelease(its_ctx* ctx) {
  HostIo* h = ctx->hostio;
  if (!h) return;
  for (int b = 0; b < 2; ++b) {
    if (h->stage[b]) cudaFreeHost(h->stage[b]);
    if (h->ready[b]) cudaEventDestroy(h->ready[b]);
  }
  delete h->pool;
  delete h;
  ctx->hostio = nullptr;
}

static its_status hostIoInit(its_ctx* ctx) {
  if (ctx->hostio) return ITS_OK;
  HostIo* h = new HostIo;
  ctx->hostio = h;
  for (int b = 0; b < 2; ++b) {
    if (cudaHostAlloc((void**)&h->stage[b], kChunk, cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ready[b], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      hostIoRelease(ctx);
      return setError(ctx, ITS_ERR_OOM, "pinned staging for host copies");
    }
  }
  unsigned hw = std::thread::hardware_concurrency();
  const int threads = (int)(hw > 16 ? 16 : (hw > 1 ? hw : 1));
  h->pool = new HostPool(threads - 1);
  return ITS_OK;
}

its_status copyToHostStaged(its_ctx* ctx, void* dst, const void* src, size_t bytes) {
  its_status st = hostIoInit(ctx);
  if (st != ITS_OK) return st;
  HostIo* h = ctx->hostio;
  const size_t chunks = (bytes + kChunk - 1) / kChunk;
  auto issue = [&](size_t c) -> its_status {
    const size_t off = c * kChunk, len = bytes - off < kChunk ? bytes - off : kChunk;
    ITS_CU(ctx, cudaMemcpyAsync(h->stage[c & 1], (const uint8_t*)src + off, len, cudaMemcpyDeviceToHost, ctx->stream));
    ITS_CU(ctx, cudaEventRecord(h->ready[c & 1], ctx->stream));
    return ITS_OK;
  };
  if ((st = issue(0)) != ITS_OK) return st;
  for (size_t c = 0; c < chunks; ++c) {
    // the other buffer's chunk was copied out in the previous iteration: refill it now
    if (c + 1 < chunks && (st = issue(c + 1)) != ITS_OK) return st;
    ITS_CU(ctx, cudaEventSynchronize(h->ready[c & 1]));
    const size_t off = c * kChunk, len = bytes - off < kChunk ? bytes - off : kChunk;
    const uint8_t* from = h->stage[c & 1];
    uint8_t* to = (uint8_t*)dst + off;
    const int parts = h->pool->size();
    const size_t per = ((len + parts - 1) / parts + kPage - 1) / kPage * kPage;
    h->pool->run(parts, [&](int p) {
      const size_t a = (size_t)p * per;
      if (a >= len) return;
      const size_t n = len - a < per ? len - a : per;
      memcpy(to + a, from + a, n);
    });
  }
  return ITS_OK;
}

its_status copyToDeviceStaged(its_ctx* ctx, void* dst, const void* src, size_t bytes) {
  its_status st = hostIoInit(ctx);
  if (st != ITS_OK) return st;
  HostIo* h = ctx->hostio;
  // pieces of a quarter of the copy (at least 4 MB, at most a chunk), so that the host's copy
  // into one buffer overlaps the transfer from the other
  size_t piece = bytes / 4;
  piece = piece < (4u << 20) ? (4u << 20) : (piece > kChunk ? kChunk : piece);
  const size_t chunks = (bytes + piece - 1) / piece;
  for (size_t c = 0; c < chunks; ++c) {
    const int b = (int)(c & 1);
    // the buffer's previous transfer (of this call or an earlier one) has left it
    ITS_CU(ctx, cudaEventSynchronize(h->ready[b]));
    const size_t off = c * piece, len = bytes - off < piece ? bytes - off : piece;
    const uint8_t* from = (const uint8_t*)src + off;
    uint8_t* to = h->stage[b];
    const int parts = h->pool->size();
    const size_t per = ((len + parts - 1) / parts + kPage - 1) / kPage * kPage;
    h->pool->run(parts, [&](int p) {
      const size_t a = (size_t)p * per;
      if (a >= len) return;
      const size_t n = len - a < per ? len - a : per;
      memcpy(to + a, from + a, n);
    });
    ITS_CU(ctx, cudaMemcpyAsync((uint8_t*)dst + off, to, len, cudaMemcpyHostToDevice, ctx->stream));
    ITS_CU(ctx, cudaEventRecord(h->ready[b], ctx->stream));
  }
  return ITS_OK;
}

}  // namespace its

using namespace its;

extern "C" {

its_status its_copy_to_device(its_ctx* ctx, void* dst, const void* src, int64_t bytes) {
  if (!ctx || bytes < 0 || (bytes > 0 && (!dst || !src))) return ITS_ERR_INVALID;
  if (bytes == 0) return ITS_OK;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  if (ptrClass(dst, ctx->device) != PtrClass::Device)
    return setError(ctx, ITS_ERR_INVALID, "its_copy_to_device: the destination must be device memory of the context's GPU");
  const PtrClass k = ptrClass(src, ctx->device);
  its_status st = ITS_OK;
  if (k == PtrClass::Pageable && (size_t)bytes >= kStagedUploadMin)
    st = copyToDeviceStaged(ctx, dst, src, (size_t)bytes);
  else
    ITS_CU(ctx, cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDefault, ctx->stream));
  if (st != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // extern "C"
