// Deterministic CSR SpMV for the thin-shell operator and its transpose.
//
// A has short rows (at most 1 + (D-1) + 8(D-1) entries) while A^T mixes ~10^5 rows of one to
// nine entries (fine-level columns) with a few enormous ones (a corner of the root cell is
// touched by almost every row of A). Rows are therefore classed once per matrix by length and
// each class gets the lane count that keeps every lane busy with a few entries:
//   class 0..5: 1, 2, 4, 8, 8, 32 lanes for rows of <= 4, 8, 16, 32, 64, 512 entries;
//   class 6:    rows above 512 entries, cut into 4096-entry segments (one block each) whose
//               partial sums a second pass adds in segment order.
// (A warp per row up to 4096 entries left the longest of those rows -- 128 entries per lane
// -- as the launch's stragglers: A^T took 79 us at 1e7 entries; cut at 512, 48 us.)
// Each lane keeps two accumulators (alternate entries) so that two loads are in flight.
// Every sum has a fixed order, so results are bit-reproducible run to run. All classes run in
// one launch (block ranges pick the class); long rows need one extra combine launch.
#pragma once
#include "its_scan.cuh"

namespace its {

constexpr int kNumClasses = 7;  // 6 lane widths + long rows
constexpr int kLongClass = 6;
constexpr int kMidMax = 512;
constexpr int kSegLen = 4096;
constexpr int kSpmvThreads = 256;

// lanes per row of classes 0..5: 33..64-entry rows take 8 lanes (4 to 8 entries each, two in
// flight per lane), which measured faster than 16 for A's dominant class (43 vs 48 us)
__host__ __device__ constexpr int classLanes(int c) { return c == 4 ? 8 : 1 << c; }
__host__ __device__ constexpr int classMaxLen(int c) { return c == 5 ? kMidMax : 4 << c; }

struct SpmvPlan {
  int64_t count[kNumClasses] = {0};  // rows per class (class 6: long rows)
  int64_t offset[kNumClasses] = {0}; // first row of the class in `rows`
  unsigned blocks[kNumClasses] = {0};// blocks per class (class 6: segments)
  unsigned blockStart[kNumClasses + 1] = {0};
  uint32_t* rows = nullptr;          // row ids grouped by class, ascending inside a class
  int64_t nSeg = 0;
  uint32_t* longFirstSeg = nullptr;  // per long row: first segment (count[6]+1 entries)
  uint32_t* segRow = nullptr;        // per segment: row
  int64_t* segBeg = nullptr;         // per segment: first entry
  double* segPartial = nullptr;      // per segment: partial sum
  __host__ __device__ int64_t nLong() const { return count[kLongClass]; }
  __host__ __device__ unsigned totalBlocks() const { return blockStart[kNumClasses]; }
};

// One SpMV operand set: y = M x with values of type VT and x of type XT, summed in FP64.
template <typename VT, typename XT>
struct CsrView {
  int64_t n = 0;
  const int64_t* rowptr = nullptr;
  const int32_t* col = nullptr;
  const VT* val = nullptr;
};

template <int W, typename VT, typename XT>
__device__ __forceinline__ double rowDot(const CsrView<VT, XT>& A, const XT* __restrict__ x, int64_t beg, int64_t end,
                                         int sub) {
  double s0 = 0.0, s1 = 0.0;
  int64_t k = beg + sub;
  for (; k + W < end; k += 2 * W) {
    const int32_t c0 = __ldg(A.col + k), c1 = __ldg(A.col + k + W);
    const VT v0 = __ldg(A.val + k), v1 = __ldg(A.val + k + W);
    s0 += (double)v0 * (double)__ldg(x + c0);
    s1 += (double)v1 * (double)__ldg(x + c1);
  }
  if (k < end) s0 += (double)__ldg(A.val + k) * (double)__ldg(x + __ldg(A.col + k));
  double s = s0 + s1;
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, W);
  return s;
}

template <int W, typename VT, typename XT, typename YT>
__device__ __forceinline__ void spmvClass(const CsrView<VT, XT>& A, const SpmvPlan& P, int c, unsigned b,
                                          const XT* __restrict__ x, YT* __restrict__ y) {
  const int64_t slot = ((int64_t)b * kSpmvThreads + threadIdx.x) / W;
  const int sub = threadIdx.x & (W - 1);
  const bool valid = slot < P.count[c];
  uint32_t row = 0;
  int64_t beg = 0, end = 0;
  if (valid) {
    row = P.rows[P.offset[c] + slot];
    beg = A.rowptr[row];
    end = A.rowptr[row + 1];
  }
  const double s = rowDot<W>(A, x, beg, end, sub);  // all lanes take part in the shuffles
  if (valid && sub == 0) y[row] = (YT)s;
}

template <typename VT, typename XT, typename YT>
__global__ void __launch_bounds__(kSpmvThreads) kSpmvBinned(CsrView<VT, XT> A, SpmvPlan P, const XT* __restrict__ x,
                                                            YT* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const unsigned b = blockIdx.x;
  if (b < P.blockStart[1]) return spmvClass<1>(A, P, 0, b - P.blockStart[0], x, y);
  if (b < P.blockStart[2]) return spmvClass<2>(A, P, 1, b - P.blockStart[1], x, y);
  if (b < P.blockStart[3]) return spmvClass<4>(A, P, 2, b - P.blockStart[2], x, y);
  if (b < P.blockStart[4]) return spmvClass<8>(A, P, 3, b - P.blockStart[3], x, y);
  if (b < P.blockStart[5]) return spmvClass<classLanes(4)>(A, P, 4, b - P.blockStart[4], x, y);
  if (b < P.blockStart[6]) return spmvClass<32>(A, P, 5, b - P.blockStart[5], x, y);
  // one long-row segment per block
  const int64_t seg = b - P.blockStart[6];
  if (seg >= P.nSeg) return;
  const uint32_t row = P.segRow[seg];
  const int64_t beg = P.segBeg[seg];
  const int64_t rowEnd = A.rowptr[row + 1];
  const int64_t end = beg + kSegLen < rowEnd ? beg + kSegLen : rowEnd;
  double s0 = 0.0, s1 = 0.0;
  int64_t k = beg + threadIdx.x;
  for (; k + kSpmvThreads < end; k += 2 * kSpmvThreads) {
    s0 += (double)__ldg(A.val + k) * (double)__ldg(x + __ldg(A.col + k));
    s1 += (double)__ldg(A.val + k + kSpmvThreads) * (double)__ldg(x + __ldg(A.col + k + kSpmvThreads));
  }
  if (k < end) s0 += (double)__ldg(A.val + k) * (double)__ldg(x + __ldg(A.col + k));
  double s = warpSum(s0 + s1);
  __shared__ double ws[kSpmvThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) ws[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kSpmvThreads / 32; ++w) t += ws[w];
    P.segPartial[seg] = t;
  }
}

template <typename YT>
__global__ void kSpmvCombine(SpmvPlan P, YT* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int64_t r = blockIdx.x * (int64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= P.nLong()) return;
  const uint32_t s0 = P.longFirstSeg[r], s1 = P.longFirstSeg[r + 1];
  double s = 0.0;
  for (uint32_t k = s0 + lane; k < s1; k += 32) s += P.segPartial[k];
  s = warpSum(s);
  if (lane == 0) y[P.rows[P.offset[kLongClass] + r]] = (YT)s;
}

// Build the row classes of a CSR matrix (device rowptr) into plan (device allocations
// released by releasePlan).
its_status buildSpmvPlan(its_ctx* ctx, int64_t n, const int64_t* rowptr, SpmvPlan* plan);
void releasePlan(its_ctx* ctx, SpmvPlan* plan);

template <typename VT, typename XT, typename YT>
its_status spmv(its_ctx* ctx, const CsrView<VT, XT>& A, const SpmvPlan& P, const XT* x, YT* y,
                const int* skip = nullptr) {
  const unsigned blocks = P.totalBlocks();
  if (blocks) {
    kSpmvBinned<VT, XT, YT><<<blocks, kSpmvThreads, 0, ctx->stream>>>(A, P, x, y, skip);
    ITS_LAUNCHED(ctx);
  }
  if (P.nLong()) {
    kSpmvCombine<YT><<<gridFor(P.nLong(), 8), 256, 0, ctx->stream>>>(P, y, skip);
    ITS_LAUNCHED(ctx);
  }
  return ITS_OK;
}

// Stable LSD radix sort of (key, value) pairs on the low keyBits bits of the keys.
// keys/vals are sorted into keysOut/valsOut; tmpK/tmpV are scratch of n elements.
its_status radixSortPairs(its_ctx* ctx, const uint32_t* keys, const uint32_t* vals, uint32_t* keysOut,
                          uint32_t* valsOut, uint32_t* tmpK, uint32_t* tmpV, int64_t n, int keyBits);

}  // namespace its
