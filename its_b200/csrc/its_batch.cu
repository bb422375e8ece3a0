// Batched LSCG: many independent operators (one per mesh) fitted together.
//
// The meshes' vectors are concatenated (mesh i owns rows off_i .. off_i + n_i - 1). One SpMV
// launch covers every mesh: each operator's row classes (its SpmvPlan) are merged into one
// work list of (mesh, row) items per class, plus the long-row segments. Dot products are
// segmented: every mesh's range is cut into fixed chunks; the last chunk of a mesh to finish
// (per-mesh ticket, no waiting) folds that mesh's chunk partials in order and runs the same
// scalar update as the single solve (its_cgls.cu), so each mesh follows exactly Eigen's CGLS
// with its own alpha, beta, stopping test and iteration count. Converged meshes drop out of
// every kernel; `check_every` iterations of the whole batch are one CUDA graph.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "its_cgls.cuh"
#include "its_op.cuh"

namespace its {

constexpr int64_t kChunk = 8192;  // rows per reduction chunk

struct BatchOp {
  int64_t n, off;
  CsrView<double, double> A, T;
  const double* invdiag;
};

// Merged work list of one SpMV side.
struct BatchList {
  int64_t count[kNumClasses] = {0};
  int64_t offset[kNumClasses] = {0};
  unsigned blockStart[kNumClasses + 1] = {0};
  const uint32_t* op = nullptr;   // item -> mesh
  const uint32_t* row = nullptr;  // item -> local row
  int64_t nSeg = 0, nLong = 0;
  const uint32_t* segOp = nullptr;
  const uint32_t* segRow = nullptr;
  const int64_t* segBeg = nullptr;
  double* segPartial = nullptr;
  const uint32_t* longOp = nullptr;
  const uint32_t* longRow = nullptr;
  const uint32_t* longFirstSeg = nullptr;
};

struct Chunks {
  int64_t count = 0;
  const uint32_t* op = nullptr;
  const int64_t* beg = nullptr;
  const int64_t* end = nullptr;
  const uint32_t* opFirst = nullptr;  // per mesh: first chunk
  const uint32_t* opCount = nullptr;  // per mesh: chunks
};

template <int W>
__device__ __forceinline__ void batchClass(const BatchOp* __restrict__ ops, const BatchList& L, int c, unsigned b,
                                           bool tr, const double* __restrict__ x, double* __restrict__ y,
                                           const CgScalars* __restrict__ S) {
  const int64_t slot = ((int64_t)b * kSpmvThreads + threadIdx.x) / W;
  const int sub = threadIdx.x & (W - 1);
  bool valid = slot < L.count[c];
  uint32_t m = 0, row = 0;
  CsrView<double, double> M;
  int64_t beg = 0, end = 0, off = 0;
  if (valid) {
    m = L.op[L.offset[c] + slot];
    row = L.row[L.offset[c] + slot];
    valid = !(S && S[m].done);
    if (valid) {
      M = tr ? ops[m].T : ops[m].A;
      off = ops[m].off;
      beg = M.rowptr[row];
      end = M.rowptr[row + 1];
    }
  }
  const double s = rowDot<W>(M, x + off, beg, end, sub);  // every lane joins the shuffles
  if (valid && sub == 0) y[off + row] = s;
}

__global__ void __launch_bounds__(kSpmvThreads) kBatchSpmv(const BatchOp* __restrict__ ops, BatchList L, int tr,
                                                           const double* __restrict__ x, double* __restrict__ y,
                                                           const CgScalars* __restrict__ S) {
  const unsigned b = blockIdx.x;
  if (b < L.blockStart[1]) return batchClass<1>(ops, L, 0, b - L.blockStart[0], tr, x, y, S);
  if (b < L.blockStart[2]) return batchClass<2>(ops, L, 1, b - L.blockStart[1], tr, x, y, S);
  if (b < L.blockStart[3]) return batchClass<4>(ops, L, 2, b - L.blockStart[2], tr, x, y, S);
  if (b < L.blockStart[4]) return batchClass<8>(ops, L, 3, b - L.blockStart[3], tr, x, y, S);
  if (b < L.blockStart[5]) return batchClass<classLanes(4)>(ops, L, 4, b - L.blockStart[4], tr, x, y, S);
  if (b < L.blockStart[6]) return batchClass<32>(ops, L, 5, b - L.blockStart[5], tr, x, y, S);
  const int64_t seg = b - L.blockStart[6];
  if (seg >= L.nSeg) return;
  const uint32_t m = L.segOp[seg];
  if (S && S[m].done) return;
  const CsrView<double, double> M = tr ? ops[m].T : ops[m].A;
  const uint32_t row = L.segRow[seg];
  const int64_t beg = L.segBeg[seg], rowEnd = M.rowptr[row + 1];
  const int64_t end = beg + kSegLen < rowEnd ? beg + kSegLen : rowEnd;
  const double* xo = x + ops[m].off;
  double s0 = 0.0, s1 = 0.0;
  int64_t k = beg + threadIdx.x;
  for (; k + kSpmvThreads < end; k += 2 * kSpmvThreads) {
    s0 += __ldg(M.val + k) * __ldg(xo + __ldg(M.col + k));
    s1 += __ldg(M.val + k + kSpmvThreads) * __ldg(xo + __ldg(M.col + k + kSpmvThreads));
  }
  if (k < end) s0 += __ldg(M.val + k) * __ldg(xo + __ldg(M.col + k));
  double s = warpSum(s0 + s1);
  __shared__ double ws[kSpmvThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kSpmvThreads / 32; ++w) t += ws[w];
    L.segPartial[seg] = t;
  }
}

__global__ void kBatchCombine(const BatchOp* __restrict__ ops, BatchList L, double* __restrict__ y,
                              const CgScalars* __restrict__ S) {
  const int64_t r = blockIdx.x * (int64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= L.nLong) return;
  const uint32_t m = L.longOp[r];
  if (S && S[m].done) return;
  double s = 0.0;
  for (uint32_t k = L.longFirstSeg[r] + lane; k < L.longFirstSeg[r + 1]; k += 32) s += L.segPartial[k];
  s = warpSum(s);
  if (lane == 0) y[ops[m].off + L.longRow[r]] = s;
}

// Segmented reduction with a per-mesh last-chunk finalize (see kReduce in its_cgls.cu).
template <class Op>
__global__ void __launch_bounds__(kRedThreads) kBatchReduce(Op op, Chunks C, double* __restrict__ partials,
                                                            CgScalars* __restrict__ S, unsigned* __restrict__ tickets,
                                                            unsigned* __restrict__ numDone, int honorDone) {
  const int64_t k = blockIdx.x;
  const uint32_t m = C.op[k];
  if (honorDone && S[m].done) return;
  double a = 0.0, b = 0.0;
  for (int64_t i = C.beg[k] + threadIdx.x; i < C.end[k]; i += kRedThreads) op.terms(i, S[m], a, b);
  blockSum2(a, b);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partials[2 * k] = a;
    partials[2 * k + 1] = b;
    __threadfence();
    const unsigned t = atomicAdd(tickets + m, 1u);
    last = (t == C.opCount[m] - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double ta = 0.0, tb = 0.0;
  const uint32_t f = C.opFirst[m], cnt = C.opCount[m];
  for (uint32_t j = threadIdx.x; j < cnt; j += kRedThreads) {
    ta += ((volatile double*)partials)[2 * (f + j)];
    tb += ((volatile double*)partials)[2 * (f + j) + 1];
  }
  blockSum2(ta, tb);
  if (threadIdx.x == 0) {
    const int wasDone = S[m].done;
    op.finalize(S + m, ta, tb);
    if (!wasDone && S[m].done) atomicAdd(numDone, 1u);
    tickets[m] = 0;
  }
}

// Batched forms of the scalar steps (terms get the mesh's scalars).
struct BInitResidual {
  const double* b;
  const double* t;
  double* r;
  __device__ void terms(int64_t i, const CgScalars&, double& a, double& c) const {
    const double v = t ? b[i] - t[i] : b[i];
    r[i] = v;
    a += v * v;
    c += b[i] * b[i];
  }
  __device__ void finalize(CgScalars* S, double rr, double bb) const { OpInitResidual{}.finalize(S, rr, bb); }
};
struct BRhsNorm {
  const double* atb;
  __device__ void terms(int64_t i, const CgScalars&, double& a, double&) const { a += atb[i] * atb[i]; }
  __device__ void finalize(CgScalars* S, double v, double) const { S->rhsNorm2 = v; }
};
struct BInitNormal {
  const double* nr;
  const double* invdiag;
  double* p;
  __device__ void terms(int64_t i, const CgScalars&, double& a, double& c) const {
    const double z = invdiag[i] * nr[i];
    p[i] = z;
    a += nr[i] * nr[i];
    c += nr[i] * z;
  }
  __device__ void finalize(CgScalars* S, double nrr, double nrz) const { OpInitNormal{}.finalize(S, nrr, nrz); }
};
struct BTmpNorm {
  const double* t;
  __device__ void terms(int64_t i, const CgScalars&, double& a, double&) const { a += t[i] * t[i]; }
  __device__ void finalize(CgScalars* S, double tn, double) const { OpTmpNorm{}.finalize(S, tn, 0.0); }
};
struct BUpdateXR {
  double* x;
  double* r;
  const double* p;
  const double* t;
  __device__ void terms(int64_t i, const CgScalars& S, double& a, double&) const {
    const double al = S.alpha;
    x[i] += al * p[i];
    const double v = r[i] - al * t[i];
    r[i] = v;
    a += v * v;
  }
  __device__ void finalize(CgScalars* S, double rr, double) const { S->rr = rr; }
};
struct BNormal {
  const double* nr;
  const double* invdiag;
  __device__ void terms(int64_t i, const CgScalars&, double& a, double& c) const {
    const double z = invdiag[i] * nr[i];
    a += nr[i] * nr[i];
    c += nr[i] * z;
  }
  __device__ void finalize(CgScalars* S, double nrr, double nrz) const { OpNormal{}.finalize(S, nrr, nrz); }
};
struct BUpdateP {
  const double* nr;
  const double* invdiag;
  double* p;
  __device__ void terms(int64_t i, const CgScalars& S, double&, double&) const {
    p[i] = invdiag[i] * nr[i] + S.beta * p[i];
  }
  __device__ void finalize(CgScalars*, double, double) const {}
};

__global__ void kBatchSetScalars(CgScalars* S, int64_t count, double tol, long long maxIters, int stopRule,
                                 unsigned* numDone) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i == 0) *numDone = 0;
  if (i >= count) return;
  CgScalars& s = S[i];
  s.tol = tol;
  s.maxIters = maxIters;
  s.stopRule = stopRule;
  s.done = 0;
  s.converged = 0;
  s.breakdown = 0;
  s.iter = 0;
}
__global__ void kBatchZeroEmpty(const BatchOp* __restrict__ ops, int64_t count, double* __restrict__ x,
                                const CgScalars* __restrict__ S) {
  const int64_t m = blockIdx.x;
  if (m >= count || S[m].rhsNorm2 != 0.0) return;
  for (int64_t i = threadIdx.x; i < ops[m].n; i += blockDim.x) x[ops[m].off + i] = 0.0;
}
// Count meshes already finished by the initial test (rhs = 0 or residual below threshold).
__global__ void kBatchCountDone(const CgScalars* __restrict__ S, int64_t count, unsigned* numDone) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < count && S[i].done) atomicAdd(numDone, 1u);
}
__global__ void kFillItems(int64_t total, const uint32_t* __restrict__ srcOff, const uint64_t* __restrict__ dstOff,
                           const uint32_t* const* __restrict__ srcRows, int64_t count, uint32_t* __restrict__ itemOp,
                           uint32_t* __restrict__ itemRow) {
  // dstOff[m] .. dstOff[m+1]: items of mesh m, copied from srcRows[m] + srcOff[m]
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= total) return;
  int64_t lo = 0, hi = count;  // last m with dstOff[m] <= j
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if ((int64_t)dstOff[mid] <= j) lo = mid;
    else hi = mid;
  }
  itemOp[j] = (uint32_t)lo;
  itemRow[j] = srcRows[lo][srcOff[lo] + (j - (int64_t)dstOff[lo])];
}

// Host-side construction of one side's merged work list.
struct BatchSide {
  BatchList L;
  DevBuf<uint32_t> op, row, segOp, segRow, longOp, longRow, longFirst;
  DevBuf<int64_t> segBeg;
  DevBuf<double> segPartial;
};

static its_status buildSide(its_ctx* ctx, its_op* const* ops, int64_t count, bool tr, BatchSide& B) {
  its_status st;
  std::vector<const SpmvPlan*> plans(count);
  for (int64_t m = 0; m < count; ++m) plans[m] = tr ? &ops[m]->planT : &ops[m]->planA;
  int64_t total = 0;
  unsigned blk = 0;
  for (int c = 0; c < kLongClass; ++c) {
    B.L.offset[c] = total;
    int64_t cnt = 0;
    for (int64_t m = 0; m < count; ++m) cnt += plans[m]->count[c];
    B.L.count[c] = cnt;
    total += cnt;
    B.L.blockStart[c] = blk;
    blk += (unsigned)((cnt * classLanes(c) + kSpmvThreads - 1) / kSpmvThreads);
  }
  B.L.blockStart[kLongClass] = blk;
  if ((st = B.op.alloc(ctx, std::max<int64_t>(total, 1))) != ITS_OK) return st;
  if ((st = B.row.alloc(ctx, std::max<int64_t>(total, 1))) != ITS_OK) return st;
  // per class: gather every mesh's class rows
  DevBuf<uint32_t> srcOff;
  DevBuf<uint64_t> dstOff;
  DevBuf<const uint32_t*> srcRows;
  if ((st = srcOff.alloc(ctx, count)) != ITS_OK || (st = dstOff.alloc(ctx, count + 1)) != ITS_OK ||
      (st = srcRows.alloc(ctx, count)) != ITS_OK)
    return st;
  std::vector<const uint32_t*> hRows(count);
  for (int64_t m = 0; m < count; ++m) hRows[m] = plans[m]->rows;
  ITS_CU(ctx, cudaMemcpyAsync(srcRows.p, hRows.data(), count * sizeof(void*), cudaMemcpyHostToDevice, ctx->stream));
  std::vector<uint32_t> hOff(count);
  std::vector<uint64_t> hDst(count + 1);
  for (int c = 0; c < kLongClass; ++c) {
    if (!B.L.count[c]) continue;
    uint64_t acc = 0;
    for (int64_t m = 0; m < count; ++m) {
      hOff[m] = (uint32_t)plans[m]->offset[c];
      hDst[m] = acc;
      acc += plans[m]->count[c];
    }
    hDst[count] = acc;
    ITS_CU(ctx, cudaMemcpyAsync(srcOff.p, hOff.data(), count * 4, cudaMemcpyHostToDevice, ctx->stream));
    ITS_CU(ctx, cudaMemcpyAsync(dstOff.p, hDst.data(), (count + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    kFillItems<<<gridFor(B.L.count[c], 256), 256, 0, ctx->stream>>>(B.L.count[c], srcOff.p, dstOff.p, srcRows.p, count,
                                                                   B.op.p + B.L.offset[c], B.row.p + B.L.offset[c]);
    ITS_LAUNCHED(ctx);
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));  // host arrays are reused for the next class
  }
  // long rows and their segments (few): assembled on the host from each plan
  int64_t nLong = 0, nSeg = 0;
  for (int64_t m = 0; m < count; ++m) {
    nLong += plans[m]->nLong();
    nSeg += plans[m]->nSeg;
  }
  B.L.nLong = nLong;
  B.L.nSeg = nSeg;
  if (nLong) {
    std::vector<uint32_t> lOp, lRow, lFirst, sOp, sRow;
    std::vector<int64_t> sBeg;
    for (int64_t m = 0; m < count; ++m) {
      const SpmvPlan& P = *plans[m];
      if (!P.nLong()) continue;
      std::vector<uint32_t> rows(P.nLong()), first(P.nLong() + 1), segRow(P.nSeg);
      std::vector<int64_t> segBeg(P.nSeg);
      ITS_CU(ctx, cudaMemcpyAsync(rows.data(), P.rows + P.offset[kLongClass], P.nLong() * 4, cudaMemcpyDeviceToHost, ctx->stream));
      ITS_CU(ctx, cudaMemcpyAsync(first.data(), P.longFirstSeg, (P.nLong() + 1) * 4, cudaMemcpyDeviceToHost, ctx->stream));
      ITS_CU(ctx, cudaMemcpyAsync(segRow.data(), P.segRow, P.nSeg * 4, cudaMemcpyDeviceToHost, ctx->stream));
      ITS_CU(ctx, cudaMemcpyAsync(segBeg.data(), P.segBeg, P.nSeg * 8, cudaMemcpyDeviceToHost, ctx->stream));
      ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
      const uint32_t base = (uint32_t)sOp.size();
      for (int64_t r = 0; r < P.nLong(); ++r) {
        lOp.push_back((uint32_t)m);
        lRow.push_back(rows[r]);
        lFirst.push_back(base + first[r]);
      }
      for (int64_t s = 0; s < P.nSeg; ++s) {
        sOp.push_back((uint32_t)m);
        sRow.push_back(segRow[s]);
        sBeg.push_back(segBeg[s]);
      }
    }
    lFirst.push_back((uint32_t)sOp.size());
    if ((st = B.longOp.alloc(ctx, nLong)) != ITS_OK || (st = B.longRow.alloc(ctx, nLong)) != ITS_OK ||
        (st = B.longFirst.alloc(ctx, nLong + 1)) != ITS_OK || (st = B.segOp.alloc(ctx, nSeg)) != ITS_OK ||
        (st = B.segRow.alloc(ctx, nSeg)) != ITS_OK || (st = B.segBeg.alloc(ctx, nSeg)) != ITS_OK ||
        (st = B.segPartial.alloc(ctx, nSeg)) != ITS_OK)
      return st;
    ITS_CU(ctx, cudaMemcpyAsync(B.longOp.p, lOp.data(), nLong * 4, cudaMemcpyHostToDevice, ctx->stream));
    ITS_CU(ctx, cudaMemcpyAsync(B.longRow.p, lRow.data(), nLong * 4, cudaMemcpyHostToDevice, ctx->stream));
    ITS_CU(ctx, cudaMemcpyAsync(B.longFirst.p, lFirst.data(), (nLong + 1) * 4, cudaMemcpyHostToDevice, ctx->stream));
    ITS_CU(ctx, cudaMemcpyAsync(B.segOp.p, sOp.data(), nSeg * 4, cudaMemcpyHostToDevice, ctx->stream));
    ITS_CU(ctx, cudaMemcpyAsync(B.segRow.p, sRow.data(), nSeg * 4, cudaMemcpyHostToDevice, ctx->stream));
    ITS_CU(ctx, cudaMemcpyAsync(B.segBeg.p, sBeg.data(), nSeg * 8, cudaMemcpyHostToDevice, ctx->stream));
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  }
  B.L.blockStart[kNumClasses] = blk + (unsigned)nSeg;
  B.L.op = B.op.p;
  B.L.row = B.row.p;
  B.L.segOp = B.segOp.p;
  B.L.segRow = B.segRow.p;
  B.L.segBeg = B.segBeg.p;
  B.L.segPartial = B.segPartial.p;
  B.L.longOp = B.longOp.p;
  B.L.longRow = B.longRow.p;
  B.L.longFirstSeg = B.longFirst.p;
  return ITS_OK;
}

static its_status batchSpmv(its_ctx* ctx, const BatchOp* ops, const BatchSide& B, bool tr, const double* x, double* y,
                            const CgScalars* S) {
  if (B.L.blockStart[kNumClasses]) {
    kBatchSpmv<<<B.L.blockStart[kNumClasses], kSpmvThreads, 0, ctx->stream>>>(ops, B.L, tr ? 1 : 0, x, y, S);
    ITS_LAUNCHED(ctx);
  }
  if (B.L.nLong) {
    kBatchCombine<<<gridFor(B.L.nLong, 8), 256, 0, ctx->stream>>>(ops, B.L, y, S);
    ITS_LAUNCHED(ctx);
  }
  return ITS_OK;
}

struct BatchRun {
  its_ctx* ctx;
  int64_t count, N;
  const BatchOp* ops;
  BatchSide* A;
  BatchSide* T;
  Chunks C;
  double *x, *r, *nr, *p, *t, *b, *d, *invdiag;
  CgScalars* S;
  double* partials;
  unsigned* tickets;  // 8 slots x count
  unsigned* numDone;
};

template <class Op>
static its_status breduce(const BatchRun& R, int slot, const Op& op, int honorDone) {
  kBatchReduce<Op><<<(unsigned)R.C.count, kRedThreads, 0, R.ctx->stream>>>(op, R.C, R.partials + slot * 2 * R.C.count, R.S,
                                                                            R.tickets + slot * R.count, R.numDone, honorDone);
  ITS_LAUNCHED(R.ctx);
  return ITS_OK;
}

static its_status batchIteration(const BatchRun& R) {
  its_status st;
  if ((st = batchSpmv(R.ctx, R.ops, *R.A, false, R.p, R.t, R.S)) != ITS_OK) return st;
  if ((st = breduce(R, 3, BTmpNorm{R.t}, 1)) != ITS_OK) return st;
  if ((st = breduce(R, 4, BUpdateXR{R.x, R.r, R.p, R.t}, 1)) != ITS_OK) return st;
  if ((st = batchSpmv(R.ctx, R.ops, *R.T, true, R.r, R.nr, R.S)) != ITS_OK) return st;
  if ((st = breduce(R, 5, BNormal{R.nr, R.invdiag}, 1)) != ITS_OK) return st;
  return breduce(R, 6, BUpdateP{R.nr, R.invdiag, R.p}, 1);
}

__global__ void kGatherInvdiag(const BatchOp* __restrict__ ops, int64_t count, double* __restrict__ out) {
  const int64_t m = blockIdx.x;
  if (m >= count) return;
  for (int64_t i = threadIdx.x; i < ops[m].n; i += blockDim.x) out[ops[m].off + i] = ops[m].invdiag[i];
}

its_status solveBatch(its_ctx* ctx, its_op* const* ops, int64_t count, const double* const* b, double* const* x,
                      const its_solve_opts& o, its_solve_report* reports) {
  its_status st;
  std::vector<BatchOp> h(count);
  int64_t N = 0;
  for (int64_t m = 0; m < count; ++m) {
    h[m] = BatchOp{ops[m]->n, N, ops[m]->A64(), ops[m]->T64(), ops[m]->invdiag};
    N += ops[m]->n;
  }
  DevBuf<BatchOp> dOps;
  DevBuf<double> vec, partials;
  DevBuf<CgScalars> S;
  DevBuf<unsigned> tickets, numDone;
  if ((st = dOps.alloc(ctx, count)) != ITS_OK || (st = vec.alloc(ctx, 8 * N)) != ITS_OK ||
      (st = S.alloc(ctx, count)) != ITS_OK || (st = tickets.zeros(ctx, 8 * count)) != ITS_OK ||
      (st = numDone.zeros(ctx, 1)) != ITS_OK)
    return st;
  ITS_CU(ctx, cudaMemcpyAsync(dOps.p, h.data(), count * sizeof(BatchOp), cudaMemcpyHostToDevice, ctx->stream));
  // reduction chunks
  std::vector<uint32_t> cOp, cFirst(count), cCount(count);
  std::vector<int64_t> cBeg, cEnd;
  for (int64_t m = 0; m < count; ++m) {
    cFirst[m] = (uint32_t)cOp.size();
    const int64_t nc = std::max<int64_t>(1, (h[m].n + kChunk - 1) / kChunk);
    cCount[m] = (uint32_t)nc;
    for (int64_t k = 0; k < nc; ++k) {
      cOp.push_back((uint32_t)m);
      cBeg.push_back(h[m].off + k * kChunk);
      cEnd.push_back(std::min(h[m].off + (k + 1) * kChunk, h[m].off + h[m].n));
    }
  }
  const int64_t nc = (int64_t)cOp.size();
  DevBuf<uint32_t> dcOp, dcFirst, dcCount;
  DevBuf<int64_t> dcBeg, dcEnd;
  if ((st = dcOp.alloc(ctx, nc)) != ITS_OK || (st = dcFirst.alloc(ctx, count)) != ITS_OK ||
      (st = dcCount.alloc(ctx, count)) != ITS_OK || (st = dcBeg.alloc(ctx, nc)) != ITS_OK ||
      (st = dcEnd.alloc(ctx, nc)) != ITS_OK || (st = partials.alloc(ctx, 8 * 2 * nc)) != ITS_OK)
    return st;
  ITS_CU(ctx, cudaMemcpyAsync(dcOp.p, cOp.data(), nc * 4, cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dcFirst.p, cFirst.data(), count * 4, cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dcCount.p, cCount.data(), count * 4, cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dcBeg.p, cBeg.data(), nc * 8, cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dcEnd.p, cEnd.data(), nc * 8, cudaMemcpyHostToDevice, ctx->stream));
  BatchSide sideA, sideT;
  if ((st = buildSide(ctx, ops, count, false, sideA)) != ITS_OK) return st;
  if ((st = buildSide(ctx, ops, count, true, sideT)) != ITS_OK) return st;
  BatchRun R;
  R.ctx = ctx;
  R.count = count;
  R.N = N;
  R.ops = dOps.p;
  R.A = &sideA;
  R.T = &sideT;
  R.C = Chunks{nc, dcOp.p, dcBeg.p, dcEnd.p, dcFirst.p, dcCount.p};
  R.x = vec.p;
  R.r = R.x + N;
  R.nr = R.r + N;
  R.p = R.nr + N;
  R.t = R.p + N;
  R.b = R.t + N;
  R.d = R.b + N;
  R.invdiag = R.d + N;
  R.S = S.p;
  R.partials = partials.p;
  R.tickets = tickets.p;
  R.numDone = numDone.p;

  cudaEvent_t e0, e1;
  ITS_CU(ctx, cudaEventCreate(&e0));
  ITS_CU(ctx, cudaEventCreate(&e1));
  ITS_CU(ctx, cudaEventRecord(e0, ctx->stream));
  for (int64_t m = 0; m < count; ++m) {
    ITS_CU(ctx, cudaMemcpyAsync(R.b + h[m].off, b[m], h[m].n * 8, cudaMemcpyDefault, ctx->stream));
    if (o.x0) ITS_CU(ctx, cudaMemcpyAsync(R.x + h[m].off, ((const double* const*)o.x0)[m], h[m].n * 8, cudaMemcpyDefault, ctx->stream));
  }
  if (!o.x0) ITS_CU(ctx, cudaMemsetAsync(R.x, 0, N * 8, ctx->stream));
  kGatherInvdiag<<<(unsigned)count, 256, 0, ctx->stream>>>(R.ops, count, R.invdiag);
  ITS_LAUNCHED(ctx);
  const long long maxIters = o.max_iters > 0 ? o.max_iters : 0;  // 0: per mesh 2n (set below)
  kBatchSetScalars<<<gridFor(count, 128), 128, 0, ctx->stream>>>(R.S, count, o.tol, maxIters > 0 ? maxIters : (1ll << 62),
                                                                 o.stop_rule, R.numDone);
  ITS_LAUNCHED(ctx);
  if (maxIters <= 0) {  // Eigen's default: twice the number of columns of each mesh
    std::vector<long long> mi(count);
    for (int64_t m = 0; m < count; ++m) mi[m] = 2 * h[m].n;
    for (int64_t m = 0; m < count; ++m)
      ITS_CU(ctx, cudaMemcpyAsync(&R.S[m].maxIters, &mi[m], sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  }
  if (o.x0) {
    if ((st = batchSpmv(ctx, R.ops, sideA, false, R.x, R.t, R.S)) != ITS_OK) return st;
  }
  if ((st = breduce(R, 0, BInitResidual{R.b, o.x0 ? R.t : nullptr, R.r}, 0)) != ITS_OK) return st;
  if ((st = batchSpmv(ctx, R.ops, sideT, true, R.b, R.d, R.S)) != ITS_OK) return st;
  if ((st = breduce(R, 1, BRhsNorm{R.d}, 0)) != ITS_OK) return st;
  if ((st = batchSpmv(ctx, R.ops, sideT, true, R.r, R.nr, R.S)) != ITS_OK) return st;
  if ((st = breduce(R, 2, BInitNormal{R.nr, R.invdiag, R.p}, 0)) != ITS_OK) return st;
  kBatchZeroEmpty<<<(unsigned)count, 256, 0, ctx->stream>>>(R.ops, count, R.x, R.S);
  ITS_LAUNCHED(ctx);
  ITS_CU(ctx, cudaMemsetAsync(R.numDone, 0, 4, ctx->stream));
  kBatchCountDone<<<gridFor(count, 128), 128, 0, ctx->stream>>>(R.S, count, R.numDone);
  ITS_LAUNCHED(ctx);

  // iterations: graphs of `every` batch iterations until every mesh is done
  const int every = o.check_every > 0 ? o.check_every : 8;
  cudaGraph_t g;
  cudaGraphExec_t ge = nullptr;
  ITS_CU(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  const int64_t before = ctx->launches;
  st = ITS_OK;
  for (int k = 0; k < every && st == ITS_OK; ++k) st = batchIteration(R);
  const int64_t perGraph = ctx->launches - before;
  ctx->launches = before;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (st != ITS_OK) return st;
  if (e != cudaSuccess) return cudaFail(ctx, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cudaFail(ctx, e, "cudaGraphInstantiate");
  for (int64_t guard = 0;; ++guard) {
    ITS_CU(ctx, cudaMemcpyAsync(ctx->pinned, R.numDone, 4, cudaMemcpyDeviceToHost, ctx->stream));
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if ((int64_t)(unsigned)ctx->pinned[0] >= count) break;
    ITS_CU(ctx, cudaGraphLaunch(ge, ctx->stream));
    ctx->launches += perGraph;
  }
  cudaGraphExecDestroy(ge);
  // true residuals and results (every mesh is done: the SpMV ignores the done flags)
  if ((st = batchSpmv(ctx, R.ops, sideA, false, R.x, R.t, nullptr)) != ITS_OK) return st;
  std::vector<CgScalars> hs(count);
  ITS_CU(ctx, cudaMemcpyAsync(hs.data(), R.S, count * sizeof(CgScalars), cudaMemcpyDeviceToHost, ctx->stream));
  // the residual reduction overwrites rr/bNorm2: read the solver state first
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  // S[m].done is set for every mesh; force the residual pass to run for all
  if ((st = breduce(R, 7, BInitResidual{R.b, R.t, R.d}, 0)) != ITS_OK) return st;
  for (int64_t m = 0; m < count; ++m) ITS_CU(ctx, cudaMemcpyAsync(x[m], R.x + h[m].off, h[m].n * 8, cudaMemcpyDefault, ctx->stream));
  ITS_CU(ctx, cudaEventRecord(e1, ctx->stream));
  std::vector<CgScalars> hr(count);
  ITS_CU(ctx, cudaMemcpyAsync(hr.data(), R.S, count * sizeof(CgScalars), cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (int64_t m = 0; m < count; ++m) {
    its_solve_report& rp = reports[m];
    rp = its_solve_report{};
    rp.iterations = hs[m].iter;
    rp.converged = hs[m].converged;
    rp.breakdown = hs[m].breakdown;
    rp.normal_rel_residual = hs[m].rhsNorm2 > 0 ? std::sqrt(hs[m].nrr / hs[m].rhsNorm2) : 0.0;
    rp.rel_residual = hr[m].bNorm2 > 0 ? std::sqrt(hr[m].rr / hr[m].bNorm2) : 0.0;
    rp.ms = ms;
  }
  return ITS_OK;
}

}  // namespace its

using namespace its;

extern "C" {

its_status its_lscg_solve_batch(its_op* const* ops, int64_t count, const double* const* b, double* const* lambda,
                                const its_solve_opts* opts, its_solve_report* reports) {
  if (!ops || count <= 0 || !b || !lambda || !reports) return ITS_ERR_INVALID;
  its_ctx* ctx = ops[0] ? ops[0]->ctx : nullptr;
  if (!ctx) return ITS_ERR_INVALID;
  for (int64_t m = 0; m < count; ++m) {
    if (!ops[m] || ops[m]->ctx != ctx || !b[m] || !lambda[m])
      return setError(ctx, ITS_ERR_INVALID, "its_lscg_solve_batch: every operator must share one context");
  }
  its_solve_opts o;
  its_solve_opts_default(&o);
  if (opts) o = *opts;
  if (!(o.tol > 0.0) || !std::isfinite(o.tol)) return setError(ctx, ITS_ERR_INVALID, "tol must be positive");
  if (o.precision != ITS_PREC_FP64) return setError(ctx, ITS_ERR_INVALID, "the batched solve runs in FP64");
  if (o.stop_rule != ITS_STOP_NORMAL && o.stop_rule != ITS_STOP_RESIDUAL)
    return setError(ctx, ITS_ERR_INVALID, "unknown stop rule");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  its_status st = solveBatch(ctx, ops, count, b, lambda, o, reports);
  if (st != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // extern "C"
