// Deterministic CSR SpMV for the thin-shell operator and its transpose.
//
// A has short rows (at most 1 + (D-1) + 8(D-1) entries), but A^T has a few enormous rows:
// a corner of the root cell is touched by almost every row of A. Rows are therefore
// binned once per matrix:
//   short  (len <= 64):   8 lanes per row, 4 rows per warp;
//   medium (len <= 4096): one warp per row;
//   long   (len > 4096):  fixed 4096-entry segments, one block each, partial sums combined
//                         in segment order by a second pass.
// Every sum has a fixed order, so results are bit-reproducible run to run. All three bins
// run in one launch (block ranges pick the role); long rows need one extra combine launch.
#pragma once
#include "its_scan.cuh"

namespace its {

constexpr int kShortMax = 64;
constexpr int kMidMax = 4096;
constexpr int kSegLen = 4096;
constexpr int kSpmvThreads = 256;

struct SpmvPlan {
  int64_t nShort = 0, nMid = 0, nLong = 0, nSeg = 0;
  uint32_t* shortRows = nullptr;
  uint32_t* midRows = nullptr;
  uint32_t* longRows = nullptr;
  uint32_t* longFirstSeg = nullptr;  // per long row: first segment (nLong+1 entries)
  uint32_t* segRow = nullptr;        // per segment: row
  int64_t* segBeg = nullptr;         // per segment: first entry
  double* segPartial = nullptr;      // per segment: partial sum
  unsigned shortBlocks = 0, midBlocks = 0, segBlocks = 0;
};

// One SpMV operand set: y = M x with values of type VT and x of type XT, summed in AT.
template <typename VT, typename XT>
struct CsrView {
  int64_t n = 0;
  const int64_t* rowptr = nullptr;
  const int32_t* col = nullptr;
  const VT* val = nullptr;
};

template <typename VT, typename XT, typename YT>
__global__ void __launch_bounds__(kSpmvThreads) kSpmvBinned(CsrView<VT, XT> A, SpmvPlan P, const XT* __restrict__ x,
                                                            YT* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  unsigned b = blockIdx.x;
  if (b < P.shortBlocks) {
    // 8 lanes per row
    const int64_t slot = ((int64_t)b * kSpmvThreads + threadIdx.x) >> 3;
    const int sub = threadIdx.x & 7;
    double s = 0.0;
    uint32_t row = 0;
    const bool valid = slot < P.nShort;
    if (valid) {
      row = P.shortRows[slot];
      const int64_t beg = A.rowptr[row], end = A.rowptr[row + 1];
      for (int64_t k = beg + sub; k < end; k += 8) s += (double)A.val[k] * (double)x[A.col[k]];
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, 8);
    if (valid && sub == 0) y[row] = (YT)s;
    return;
  }
  b -= P.shortBlocks;
  if (b < P.midBlocks) {
    const int64_t slot = (int64_t)b * (kSpmvThreads / 32) + warp;
    if (slot >= P.nMid) return;
    const uint32_t row = P.midRows[slot];
    const int64_t beg = A.rowptr[row], end = A.rowptr[row + 1];
    double s = 0.0;
    for (int64_t k = beg + lane; k < end; k += 32) s += (double)A.val[k] * (double)x[A.col[k]];
    s = warpSum(s);
    if (lane == 0) y[row] = (YT)s;
    return;
  }
  b -= P.midBlocks;
  {
    // one long-row segment per block
    const int64_t seg = b;
    if (seg >= P.nSeg) return;
    const uint32_t row = P.segRow[seg];
    const int64_t beg = P.segBeg[seg];
    const int64_t rowEnd = A.rowptr[row + 1];
    const int64_t end = beg + kSegLen < rowEnd ? beg + kSegLen : rowEnd;
    double s = 0.0;
    for (int64_t k = beg + threadIdx.x; k < end; k += kSpmvThreads) s += (double)A.val[k] * (double)x[A.col[k]];
    s = warpSum(s);
    __shared__ double ws[kSpmvThreads / 32];
    if (lane == 0) ws[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < kSpmvThreads / 32; ++w) t += ws[w];
      P.segPartial[seg] = t;
    }
  }
}

template <typename YT>
__global__ void kSpmvCombine(SpmvPlan P, YT* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int64_t r = blockIdx.x * (int64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= P.nLong) return;
  const uint32_t s0 = P.longFirstSeg[r], s1 = P.longFirstSeg[r + 1];
  double s = 0.0;
  for (uint32_t k = s0 + lane; k < s1; k += 32) s += P.segPartial[k];
  s = warpSum(s);
  if (lane == 0) y[P.longRows[r]] = (YT)s;
}

// Build the row bins of a CSR matrix (device rowptr) into plan (device allocations owned
// by the caller through releasePlan).
its_status buildSpmvPlan(its_ctx* ctx, int64_t n, const int64_t* rowptr, SpmvPlan* plan);
void releasePlan(its_ctx* ctx, SpmvPlan* plan);

template <typename VT, typename XT, typename YT>
its_status spmv(its_ctx* ctx, const CsrView<VT, XT>& A, const SpmvPlan& P, const XT* x, YT* y,
                const int* skip = nullptr) {
  const unsigned blocks = P.shortBlocks + P.midBlocks + (unsigned)P.nSeg;
  if (blocks) {
    kSpmvBinned<VT, XT, YT><<<blocks, kSpmvThreads, 0, ctx->stream>>>(A, P, x, y, skip);
    ITS_LAUNCHED(ctx);
  }
  if (P.nLong) {
    kSpmvCombine<YT><<<gridFor(P.nLong, 8), 256, 0, ctx->stream>>>(P, y, skip);
    ITS_LAUNCHED(ctx);
  }
  return ITS_OK;
}

// Stable LSD radix sort of (key, value) pairs on the low keyBits bits of the keys.
// keys/vals are sorted into keysOut/valsOut; tmpK/tmpV are scratch of n elements.
its_status radixSortPairs(its_ctx* ctx, const uint32_t* keys, const uint32_t* vals, uint32_t* keysOut,
                          uint32_t* valsOut, uint32_t* tmpK, uint32_t* tmpV, int64_t n, int keyBits);

}  // namespace its
