// SpMV row binning and the stable radix sort used to transpose the operator.
#include <vector>

#include "its_sparse.cuh"

namespace its {

// ---- row bins ---------------------------------------------------------------------------
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
  DevBuf<uint32_t> tShort, tMid, tLong, tot;
  DevBuf<uint32_t> segCount;  // per long row
  if ((st = tShort.alloc(ctx, n)) != ITS_OK) return st;
  if ((st = tMid.alloc(ctx, n)) != ITS_OK) return st;
  if ((st = tLong.alloc(ctx, n)) != ITS_OK) return st;
  if ((st = tot.zeros(ctx, 4)) != ITS_OK) return st;
  const int64_t* rp = rowptr;
  uint32_t* ps = tShort.p;
  uint32_t* pm = tMid.p;
  uint32_t* pl = tLong.p;
  auto fs = [rp] __device__(int64_t i) -> uint32_t { return (rp[i + 1] - rp[i]) <= kShortMax ? 1u : 0u; };
  auto fm = [rp] __device__(int64_t i) -> uint32_t {
    const int64_t l = rp[i + 1] - rp[i];
    return (l > kShortMax && l <= kMidMax) ? 1u : 0u;
  };
  auto fl = [rp] __device__(int64_t i) -> uint32_t { return (rp[i + 1] - rp[i]) > kMidMax ? 1u : 0u; };
  auto ws = [ps] __device__(int64_t i, uint32_t pre, uint32_t v) { if (v) ps[pre] = (uint32_t)i; };
  auto wm = [pm] __device__(int64_t i, uint32_t pre, uint32_t v) { if (v) pm[pre] = (uint32_t)i; };
  auto wl = [pl] __device__(int64_t i, uint32_t pre, uint32_t v) { if (v) pl[pre] = (uint32_t)i; };
  if ((st = scanExclusiveAlloc<uint32_t>(ctx, fs, n, ws, tot.p + 0)) != ITS_OK) return st;
  if ((st = scanExclusiveAlloc<uint32_t>(ctx, fm, n, wm, tot.p + 1)) != ITS_OK) return st;
  if ((st = scanExclusiveAlloc<uint32_t>(ctx, fl, n, wl, tot.p + 2)) != ITS_OK) return st;
  uint32_t h[4] = {0, 0, 0, 0};
  ITS_CU(ctx, cudaMemcpyAsync(h, tot.p, 16, cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  P->nShort = h[0];
  P->nMid = h[1];
  P->nLong = h[2];
  if ((st = devAlloc(ctx, (void**)&P->shortRows, P->nShort * 4)) != ITS_OK) return st;
  if ((st = devAlloc(ctx, (void**)&P->midRows, P->nMid * 4)) != ITS_OK) return st;
  if ((st = devAlloc(ctx, (void**)&P->longRows, P->nLong * 4)) != ITS_OK) return st;
  if (P->nShort) ITS_CU(ctx, cudaMemcpyAsync(P->shortRows, tShort.p, P->nShort * 4, cudaMemcpyDeviceToDevice, ctx->stream));
  if (P->nMid) ITS_CU(ctx, cudaMemcpyAsync(P->midRows, tMid.p, P->nMid * 4, cudaMemcpyDeviceToDevice, ctx->stream));
  if (P->nLong) ITS_CU(ctx, cudaMemcpyAsync(P->longRows, tLong.p, P->nLong * 4, cudaMemcpyDeviceToDevice, ctx->stream));
  P->shortBlocks = (unsigned)((P->nShort * 8 + kSpmvThreads - 1) / kSpmvThreads);
  P->midBlocks = (unsigned)((P->nMid + kSpmvThreads / 32 - 1) / (kSpmvThreads / 32));
  if (P->nLong) {
    if ((st = devAlloc(ctx, (void**)&P->longFirstSeg, (P->nLong + 1) * 4)) != ITS_OK) return st;
    const uint32_t* lr = P->longRows;
    uint32_t* lfs = P->longFirstSeg;
    auto fc = [rp, lr] __device__(int64_t i) -> uint32_t {
      const int64_t l = rp[lr[i] + 1] - rp[lr[i]];
      return (uint32_t)((l + kSegLen - 1) / kSegLen);
    };
    if ((st = scanExclusiveAlloc<uint32_t>(ctx, fc, P->nLong, StorePrefix<uint32_t>{lfs}, tot.p + 3)) != ITS_OK) return st;
    ITS_CU(ctx, cudaMemcpyAsync(lfs + P->nLong, tot.p + 3, 4, cudaMemcpyDeviceToDevice, ctx->stream));
    uint32_t nseg = 0;
    if ((st = readScalar(ctx, tot.p + 3, &nseg)) != ITS_OK) return st;
    P->nSeg = nseg;
    if ((st = devAlloc(ctx, (void**)&P->segRow, nseg * 4)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&P->segBeg, nseg * 8)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&P->segPartial, nseg * 8)) != ITS_OK) return st;
    kFillSegments<<<gridFor(P->nLong, 128), 128, 0, ctx->stream>>>(P->nLong, P->longRows, P->longFirstSeg, rowptr,
                                                                 P->segRow, P->segBeg);
    ITS_LAUNCHED(ctx);
  }
  return ITS_OK;
}

void releasePlan(its_ctx* ctx, SpmvPlan* P) {
  void* ptrs[] = {P->shortRows, P->midRows, P->longRows, P->longFirstSeg, P->segRow, P->segBeg, P->segPartial};
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
  if ((st = spine.alloc(ctx, scanBlocks(256 * nb))) != ITS_OK) return st;
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
