// SpMV row classes and the stable radix sort used to transpose the operator.
#include "its_sparse.cuh"

namespace its {

// ---- row classes --------------------------------------------------------------------------
__host__ __device__ inline uint32_t rowClass(int64_t len) {
  for (int c = 0; c < kLongClass; ++c)
    if (len <= classMaxLen(c)) return (uint32_t)c;
  return kLongClass;
}
__global__ void kRowClass(int64_t n, const int64_t* __restrict__ rowptr, uint32_t* __restrict__ cls,
                          uint32_t* __restrict__ ids) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  cls[r] = rowClass(rowptr[r + 1] - rowptr[r]);
  ids[r] = (uint32_t)r;
}
// Class boundaries in the class-sorted list: entry i opens classes (cls[i-1], cls[i]].
__global__ void kClassBounds(int64_t n, const uint32_t* __restrict__ cls, int64_t* __restrict__ bounds) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i > n) return;
  const int64_t c = (i < n) ? (int64_t)cls[i] : kNumClasses;
  const int64_t prev = (i == 0) ? -1 : (int64_t)cls[i - 1];
  for (int64_t k = prev + 1; k <= c; ++k) bounds[k] = i;
}
__global__ void kSegCounts(int64_t nLong, const uint32_t* __restrict__ longRows, const int64_t* __restrict__ rowptr,
                           uint32_t* __restrict__ cnt) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= nLong) return;
  const int64_t l = rowptr[longRows[j] + 1] - rowptr[longRows[j]];
  cnt[j] = (uint32_t)((l + kSegLen - 1) / kSegLen);
}
// Long row j is cut into segments first[j] .. first[j+1]-1 of kSegLen entries each.
__global__ void kFillSegments(int64_t nLong, const uint32_t* __restrict__ longRows,
                              const uint32_t* __restrict__ first, const int64_t* __restrict__ rowptr,
                              uint32_t* __restrict__ segRow, int64_t* __restrict__ segBeg) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= nLong) return;
  const uint32_t row = longRows[j];
  const int64_t beg = rowptr[row];
  for (uint32_t s = first[j]; s < first[j + 1]; ++s) {
    segRow[s] = row;
    segBeg[s] = beg + (int64_t)(s - first[j]) * kSegLen;
  }
}

its_status buildSpmvPlan(its_ctx* ctx, int64_t n, const int64_t* rowptr, SpmvPlan* P) {
  *P = SpmvPlan();
  its_status st;
  DevBuf<uint32_t> cls, ids, sortedCls, tk, tv;
  DevBuf<int64_t> bounds;
  if ((st = cls.alloc(ctx, n)) != ITS_OK || (st = ids.alloc(ctx, n)) != ITS_OK ||
      (st = sortedCls.alloc(ctx, n)) != ITS_OK || (st = tk.alloc(ctx, n)) != ITS_OK ||
      (st = tv.alloc(ctx, n)) != ITS_OK || (st = bounds.alloc(ctx, kNumClasses + 1)) != ITS_OK)
    return st;
  if ((st = devAlloc(ctx, (void**)&P->rows, n * 4)) != ITS_OK) return st;
  kRowClass<<<gridFor(n, 256), 256, 0, ctx->stream>>>(n, rowptr, cls.p, ids.p);
  ITS_LAUNCHED(ctx);
  // one stable 8-bit pass groups the rows by class, ascending inside each class
  if ((st = radixSortPairs(ctx, cls.p, ids.p, sortedCls.p, P->rows, tk.p, tv.p, n, 3)) != ITS_OK) return st;
  kClassBounds<<<gridFor(n + 1, 256), 256, 0, ctx->stream>>>(n, sortedCls.p, bounds.p);
  ITS_LAUNCHED(ctx);
  int64_t hb[kNumClasses + 1];
  ITS_CU(ctx, cudaMemcpyAsync(hb, bounds.p, sizeof(hb), cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  unsigned blk = 0;
  for (int c = 0; c < kNumClasses; ++c) {
    P->offset[c] = hb[c];
    P->count[c] = hb[c + 1] - hb[c];
    P->blockStart[c] = blk;
    if (c < kLongClass) {
      P->blocks[c] = (unsigned)((P->count[c] * classLanes(c) + kSpmvThreads - 1) / kSpmvThreads);
      blk += P->blocks[c];
    }
  }
  const int64_t nLong = P->nLong();
  if (nLong) {
    DevBuf<uint32_t> segCnt, tot;
    if ((st = segCnt.alloc(ctx, nLong)) != ITS_OK || (st = tot.alloc(ctx, 1)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&P->longFirstSeg, (nLong + 1) * 4)) != ITS_OK) return st;
    const uint32_t* longRows = P->rows + P->offset[kLongClass];
    kSegCounts<<<gridFor(nLong, 128), 128, 0, ctx->stream>>>(nLong, longRows, rowptr, segCnt.p);
    ITS_LAUNCHED(ctx);
    const uint32_t* sc = segCnt.p;
    auto fc = [sc] __device__(int64_t i) -> uint32_t { return sc[i]; };
    if ((st = scanExclusiveAlloc<uint32_t>(ctx, fc, nLong, StorePrefix<uint32_t>{P->longFirstSeg}, tot.p)) != ITS_OK)
      return st;
    ITS_CU(ctx, cudaMemcpyAsync(P->longFirstSeg + nLong, tot.p, 4, cudaMemcpyDeviceToDevice, ctx->stream));
    uint32_t nseg = 0;
    if ((st = readScalar(ctx, tot.p, &nseg)) != ITS_OK) return st;
    P->nSeg = nseg;
    if ((st = devAlloc(ctx, (void**)&P->segRow, nseg * 4)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&P->segBeg, nseg * 8)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&P->segPartial, nseg * 8)) != ITS_OK) return st;
    kFillSegments<<<gridFor(nLong, 128), 128, 0, ctx->stream>>>(nLong, longRows, P->longFirstSeg, rowptr, P->segRow,
                                                              P->segBeg);
    ITS_LAUNCHED(ctx);
  }
  P->blocks[kLongClass] = (unsigned)P->nSeg;
  P->blockStart[kLongClass] = blk;
  P->blockStart[kNumClasses] = blk + (unsigned)P->nSeg;
  return ITS_OK;
}

void releasePlan(its_ctx* ctx, SpmvPlan* P) {
  void* ptrs[] = {P->rows, P->longFirstSeg, P->segRow, P->segBeg, P->segPartial};
  for (void* p : ptrs) devFree(ctx, p);
  *P = SpmvPlan();
}

// ---- stable LSD radix sort (8-bit digits) ----------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;

__global__ void __launch_bounds__(kRsThreads) kRadixUpsweep(const uint32_t* __restrict__ keys, int64_t n, int shift,
                                                            uint32_t* __restrict__ blockHist, int64_t nb) {
  __shared__ uint32_t hist[256];
  hist[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRsTile;
#pragma unroll 4
  for (int j = 0; j < kRsItems; ++j) {
    const int64_t i = base + (int64_t)j * kRsThreads + threadIdx.x;
    if (i < n) atomicAdd(&hist[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  blockHist[(int64_t)threadIdx.x * nb + blockIdx.x] = hist[threadIdx.x];
}

// Stable scatter: items of a tile are ranked in (round, warp, lane) order, which is their
// order in the input; warps find same-digit peers with __match_any_sync.
__global__ void __launch_bounds__(kRsThreads) kRadixDownsweep(const uint32_t* __restrict__ keys,
                                                              const uint32_t* __restrict__ vals, int64_t n, int shift,
                                                              const uint32_t* __restrict__ offsets, int64_t nb,
                                                              uint32_t* __restrict__ keysOut,
                                                              uint32_t* __restrict__ valsOut) {
  __shared__ uint32_t base[256];
  __shared__ uint32_t roundBase[256];
  __shared__ uint32_t warpCnt[kRsThreads / 32][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  base[threadIdx.x] = offsets[(int64_t)threadIdx.x * nb + blockIdx.x];
  for (int w = 0; w < kRsThreads / 32; ++w) warpCnt[w][threadIdx.x] = 0;
  __syncthreads();
  const int64_t tile = (int64_t)blockIdx.x * kRsTile;
  const unsigned ltMask = (1u << lane) - 1u;
  for (int j = 0; j < kRsItems; ++j) {
    const int64_t i = tile + (int64_t)j * kRsThreads + threadIdx.x;
    const bool valid = i < n;
    const uint32_t key = valid ? keys[i] : 0u;
    const uint32_t val = valid ? vals[i] : 0u;
    const uint32_t digit = valid ? ((key >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, digit);
    const unsigned rank = __popc(peers & ltMask);
    const bool leader = (peers & ltMask) == 0;
    if (valid && leader) warpCnt[warp][digit] = __popc(peers);
    __syncthreads();
    {
      const int t = threadIdx.x;  // digit
      uint32_t s = 0;
#pragma unroll
      for (int w = 0; w < kRsThreads / 32; ++w) {
        const uint32_t c = warpCnt[w][t];
        warpCnt[w][t] = s;
        s += c;
      }
      roundBase[t] = base[t];
      base[t] += s;
    }
    __syncthreads();
    if (valid) {
      const uint32_t dst = roundBase[digit] + warpCnt[warp][digit] + rank;
      keysOut[dst] = key;
      valsOut[dst] = val;
    }
    __syncthreads();
    // every entry now holds a prefix value: clear them all for the next round
    for (int w = 0; w < kRsThreads / 32; ++w) warpCnt[w][threadIdx.x] = 0;
    __syncthreads();
  }
}

its_status radixSortPairs(its_ctx* ctx, const uint32_t* keys, const uint32_t* vals, uint32_t* keysOut,
                          uint32_t* valsOut, uint32_t* tmpK, uint32_t* tmpV, int64_t n, int keyBits) {
  if (n <= 0) return ITS_OK;
  const int passes = keyBits <= 0 ? 1 : (keyBits + 7) / 8;
  const int64_t nb = (n + kRsTile - 1) / kRsTile;
  its_status st;
  DevBuf<uint32_t> hist, spine;
  if ((st = hist.alloc(ctx, 256 * nb)) != ITS_OK) return st;
  if ((st = spine.alloc(ctx, scanScratchSize(256 * nb))) != ITS_OK) return st;
  const uint32_t* sk = keys;
  const uint32_t* sv = vals;
  for (int p = 0; p < passes; ++p) {
    const bool toOut = ((passes - p) & 1) == 1;
    uint32_t* dk = toOut ? keysOut : tmpK;
    uint32_t* dv = toOut ? valsOut : tmpV;
    kRadixUpsweep<<<(unsigned)nb, kRsThreads, 0, ctx->stream>>>(sk, n, 8 * p, hist.p, nb);
    ITS_LAUNCHED(ctx);
    uint32_t* hp = hist.p;
    auto f = [hp] __device__(int64_t i) -> uint32_t { return hp[i]; };
    if ((st = scanExclusive<uint32_t>(ctx, f, 256 * nb, StorePrefix<uint32_t>{hp}, (uint32_t*)nullptr, spine.p)) != ITS_OK)
      return st;
    kRadixDownsweep<<<(unsigned)nb, kRsThreads, 0, ctx->stream>>>(sk, sv, n, 8 * p, hist.p, nb, dk, dv);
    ITS_LAUNCHED(ctx);
    sk = dk;
    sv = dv;
  }
  return ITS_OK;
}

}  // namespace its
