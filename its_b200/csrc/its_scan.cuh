// Exclusive prefix sums (reduce-then-scan, three launches, no inter-block waiting).
// The input is produced by a functor so that flags, popcounts or counts need not be
// materialised. Used for stream compaction of Morton codes, lattice ranks, CSR row
// pointers and marching-cubes offsets.
#pragma once
#include "its_ctx.cuh"

namespace its {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one value per thread; returns the block total.
template <typename T>
__device__ inline T blockExclusiveScan(T v, T& total) {
  __shared__ T warpTot[kScanThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warpTot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    T t = (lane < kScanThreads / 32) ? warpTot[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < kScanThreads / 32) warpTot[lane] = t;
  }
  __syncthreads();
  total = warpTot[kScanThreads / 32 - 1];
  T excl = x - v + (wid > 0 ? warpTot[wid - 1] : T(0));
  __syncthreads();
  return excl;
}

template <typename T, typename F>
__global__ void kScanUpsweep(F f, int64_t n, T* blockSums) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  T s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j)
    if (base + j < n) s += f(base + j);
  T total;
  blockExclusiveScan<T>(s, total);
  if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

// Single block: exclusive scan of the block sums in place; grand total to *total. Thread t
// takes the t-th contiguous run of ceil(nb / threads) sums: it adds them, the block scans the
// run totals once, and the thread writes its run's prefixes (integer sums: any grouping gives
// the same values).
// Both passes read eight sums per step, so that the loads of a run are in flight together.
template <typename T>
__global__ void kScanSpine(T* blockSums, int64_t nb, T* total) {
  const int64_t per = (nb + kScanThreads - 1) / kScanThreads;
  const int64_t b0 = (int64_t)threadIdx.x * per, b1 = b0 + per < nb ? b0 + per : nb;
  T s = 0;
  int64_t i = b0;
  for (; i + 8 <= b1; i += 8) {
    T v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = blockSums[i + k];
#pragma unroll
    for (int k = 0; k < 8; ++k) s += v[k];
  }
  for (; i < b1; ++i) s += blockSums[i];
  T tot;
  T run = blockExclusiveScan<T>(s, tot);
  for (i = b0; i + 8 <= b1; i += 8) {
    T v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = blockSums[i + k];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      blockSums[i + k] = run;
      run += v[k];
    }
  }
  for (; i < b1; ++i) {
    const T v = blockSums[i];
    blockSums[i] = run;
    run += v;
  }
  if (threadIdx.x == 0 && total) *total = tot;
}

// The spine above kSpineOneBlock block sums, in three launches: tiles of kSpineTile sums
// scanned in place by a block each (eight consecutive sums per thread) with each tile's total
// in tops; the totals scanned by kScanSpine (one block); each tile's offset added.
constexpr int64_t kSpineOneBlock = 8192;
constexpr int kSpineTile = kScanThreads * 8;
inline int64_t spineTops(int64_t nb) { return nb > kSpineOneBlock ? (nb + kSpineTile - 1) / kSpineTile : 0; }
template <typename T>
__global__ void __launch_bounds__(kScanThreads) kSpineTiles(T* __restrict__ sums, int64_t nb, T* __restrict__ tops) {
  const int64_t i0 = (int64_t)blockIdx.x * kSpineTile + (int64_t)threadIdx.x * 8;
  T v[8];
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    v[k] = i0 + k < nb ? sums[i0 + k] : T(0);
    s += v[k];
  }
  T tot;
  T run = blockExclusiveScan<T>(s, tot);
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (i0 + k < nb) {
      sums[i0 + k] = run;
      run += v[k];
    }
  if (threadIdx.x == 0) tops[blockIdx.x] = tot;
}
template <typename T>
__global__ void __launch_bounds__(kScanThreads) kSpineAdd(T* __restrict__ sums, int64_t nb,
                                                         const T* __restrict__ tops) {
  const T add = tops[blockIdx.x];
  const int64_t i0 = (int64_t)blockIdx.x * kSpineTile;
  for (int k = threadIdx.x; k < kSpineTile; k += kScanThreads)
    if (i0 + k < nb) sums[i0 + k] += add;
}

template <typename T, typename F, typename W>
__global__ void kScanDownsweep(F f, int64_t n, const T* blockOffsets, W write) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = (base + j < n) ? f(base + j) : T(0);
    s += v[j];
  }
  T total;
  T run = blockExclusiveScan<T>(s, total) + blockOffsets[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kScanItems; ++j)
    if (base + j < n) {
      write(base + j, run, v[j]);
      run += v[j];
    }
}

// Writes the exclusive prefix to out[i].
template <typename T>
struct StorePrefix {
  T* out;
  __device__ void operator()(int64_t i, T prefix, T) const { out[i] = prefix; }
};

// The spine: nb block sums scanned in place (exclusive), their total to *total (may be NULL);
// above kSpineOneBlock sums tops holds spineTops(nb) elements of scratch.
template <typename T>
its_status scanSpine(its_ctx* ctx, T* sums, int64_t nb, T* total, T* tops) {
  if (nb <= kSpineOneBlock) {
    kScanSpine<T><<<1, kScanThreads, 0, ctx->stream>>>(sums, nb, total);
    ITS_LAUNCHED(ctx);
    return ITS_OK;
  }
  const int64_t nt = spineTops(nb);
  kSpineTiles<T><<<(unsigned)nt, kScanThreads, 0, ctx->stream>>>(sums, nb, tops);
  ITS_LAUNCHED(ctx);
  kScanSpine<T><<<1, kScanThreads, 0, ctx->stream>>>(tops, nt, total);
  ITS_LAUNCHED(ctx);
  kSpineAdd<T><<<(unsigned)nt, kScanThreads, 0, ctx->stream>>>(sums, nb, tops);
  ITS_LAUNCHED(ctx);
  return ITS_OK;
}

// Exclusive scan of f(0..n-1); write(i, prefix, value) receives each element's prefix.
// The total lands in *dTotal (device memory, may be NULL). scratch must hold
// scanScratchSize(n) elements of T (the block sums, then the spine's tile totals).
inline int64_t scanBlocks(int64_t n) { return (n + kScanTile - 1) / kScanTile; }
inline int64_t scanScratchSize(int64_t n) {
  const int64_t nb = scanBlocks(n > 0 ? n : 1);
  return nb + spineTops(nb);
}
template <typename T, typename F, typename W>
its_status scanExclusive(its_ctx* ctx, F f, int64_t n, W write, T* dTotal, T* scratch) {
  if (n <= 0) {
    if (dTotal) ITS_CU(ctx, cudaMemsetAsync(dTotal, 0, sizeof(T), ctx->stream));
    return ITS_OK;
  }
  const int64_t nb = scanBlocks(n);
  kScanUpsweep<T, F><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(f, n, scratch);
  ITS_LAUNCHED(ctx);
  its_status st = scanSpine<T>(ctx, scratch, nb, dTotal, scratch + nb);
  if (st != ITS_OK) return st;
  kScanDownsweep<T, F, W><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(f, n, scratch, write);
  ITS_LAUNCHED(ctx);
  return ITS_OK;
}
// Convenience: allocates its own spine scratch.
template <typename T, typename F, typename W>
its_status scanExclusiveAlloc(its_ctx* ctx, F f, int64_t n, W write, T* dTotal) {
  DevBuf<T> spine;
  its_status s = spine.alloc(ctx, (size_t)scanScratchSize(n));
  if (s != ITS_OK) return s;
  return scanExclusive<T>(ctx, f, n, write, dTotal, spine.p);
}

// Read one device scalar into host memory (synchronises the stream).
template <typename T>
its_status readScalar(its_ctx* ctx, const T* d, T* h) {
  ITS_CU(ctx, cudaMemcpyAsync(h, d, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // namespace its
