// Exact start of the thin-shell least-squares system (hierarchical surplus).
//
// Row v of A evaluates the fitted field at corner vertex v: the coincident vertices of the
// finer depths (value 1), v itself (1), and the non-zero hats of the corners of every
// ancestor of v's owner (ThinShells.cpp:511-606). Two vertices at the same point (one per
// depth that has a corner there) therefore have identical rows: the system is consistent
// and rank deficient, one constraint per distinct point. Its exact solutions are
// parametrised by how each point's value is split among its coincident vertices:
//
//   * a vertex whose lattice coordinates are all even (below the root depth) coincides with
//     a corner of the next coarser depth; its coefficient is a free "share" (0 by default,
//     or the value given, e.g. a learned prediction);
//   * every other vertex, coarse depths first, takes the surplus
//       lambda_v = b_v - sum_{u != v} A(v,u) lambda_u,
//     whose terms are all known by then: coarser columns are final, and the finer columns
//     of row v are coincident (even) vertices holding their shares.
//
// The result satisfies A lambda = b up to rounding for any shares: one pass over the rows of
// A (one launch per depth), instead of the CGLS iterations. CGLS started there stops at once
// (Eigen's solve with a guess tests the initial residual first), and because CGLS only moves
// inside the row space of A, the shares fix the null-space component of the final
// coefficients. The field at the corner vertices, and hence in every finest cell, is the
// same for every exact solution; coarser cells differ by that null-space component.
//
// Both passes here are matrix-free: the rows are generated from the octree by walkRow
// (its_rows.cuh), in the assembled operator's column order, so no CSR is needed.
#include <algorithm>
#include <cmath>
#include <vector>

#include "its_op.cuh"
#include "its_rows.cuh"

namespace its {

// One depth (or, for the residual, one chunk of rows) of one octree.
struct RowSeg {
  const RowParams* P;    // the octree's row parameters (device)
  int d;                 // depth of the rows (exact start)
  int64_t rowBegin, rows;
  const double* b;
  const double* shares;  // may be null (all shares 0)
  double* lam;
};

__device__ __forceinline__ int findSeg(const int64_t* __restrict__ prefix, int nseg, int64_t i) {
  int lo = 0, hi = nseg - 1;  // last segment with prefix[seg] <= i
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Shares of the coincident vertices, zeros elsewhere (segments: whole octrees).
__global__ void kStartShares(const RowSeg* __restrict__ segs, const int64_t* __restrict__ prefix, int nseg,
                             int64_t total) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int g = findSeg(prefix, nseg, i);
  const RowSeg& s = segs[g];
  const int64_t r = s.rowBegin + (i - prefix[g]);
  const RowParams& P = *s.P;
  s.lam[r] = (s.shares && rowCoincident(P, r, rowDepth(P, r))) ? s.shares[r] : 0.0;
}

// Surplus of one non-coincident row, the row summed in column order.
__device__ __forceinline__ void startRow(const RowSeg& s, int64_t r) {
  const RowParams& P = *s.P;
  if (rowCoincident(P, r, s.d)) return;
  const double* lam = s.lam;
  double acc = 0.0;
  walkRow(P, r, s.d, [&](int32_t c, double v) {
    if (c != (int32_t)r) acc += v * lam[c];
  });
  s.lam[r] = s.b[r] - acc;
}

// One depth per octree (segments = that depth of every octree).
__global__ void kStartLevel(const RowSeg* __restrict__ segs, const int64_t* __restrict__ prefix, int nseg,
                            int64_t total) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int g = findSeg(prefix, nseg, i);
  startRow(segs[g], segs[g].rowBegin + (i - prefix[g]));
}

// The coarse depths, whose few rows would leave a launch per depth mostly idle: one block
// walks depths t0..t1-1 in order (a block barrier between depths makes each depth's values
// visible to the next), the rows of a depth spread over its threads.
constexpr int kSmallLevelRows = 4096;
__global__ void __launch_bounds__(1024) kStartLevelsSmall(const RowSeg* __restrict__ segs,
                                                          const int64_t* __restrict__ prefix,
                                                          const int* __restrict__ levelFirst,
                                                          const int64_t* __restrict__ levelRows, int t0, int t1) {
  for (int t = t0; t < t1; ++t) {
    const int g0 = levelFirst[t], ng = levelFirst[t + 1] - g0;
    for (int64_t i = threadIdx.x; i < levelRows[t]; i += blockDim.x) {
      const int g = g0 + findSeg(prefix + g0, ng, i);
      startRow(segs[g], segs[g].rowBegin + (i - prefix[g]));
    }
    __syncthreads();
  }
}

constexpr int kResThreads = 256;
constexpr int64_t kResChunk = 256;  // rows per block (one per thread): enough blocks to fill the GPU

// ||b - A lambda||^2 and ||b||^2 of one chunk of rows (segments = chunks, one block each).
__global__ void __launch_bounds__(kResThreads) kResidualChunks(const RowSeg* __restrict__ segs, double* __restrict__ part) {
  const RowSeg& s = segs[blockIdx.x];
  const RowParams& P = *s.P;
  double rr = 0.0, bb = 0.0;
  for (int64_t i = threadIdx.x; i < s.rows; i += kResThreads) {
    const int64_t r = s.rowBegin + i;
    double acc = 0.0;
    const double* lam = s.lam;
    walkRow(P, r, rowDepth(P, r), [&](int32_t c, double v) { acc += v * lam[c]; });
    const double e = s.b[r] - acc;
    rr += e * e;
    bb += s.b[r] * s.b[r];
  }
  __shared__ double srr[kResThreads / 32], sbb[kResThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    rr += __shfl_down_sync(0xffffffffu, rr, o);
    bb += __shfl_down_sync(0xffffffffu, bb, o);
  }
  if ((threadIdx.x & 31) == 0) {
    srr[threadIdx.x >> 5] = rr;
    sbb[threadIdx.x >> 5] = bb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, c = 0.0;
    for (int w = 0; w < kResThreads / 32; ++w) {
      a += srr[w];
      c += sbb[w];
    }
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = c;
  }
}

// One block per mesh: the mesh's chunk partials in a fixed order (strided per thread, then a
// fixed tree), so the result does not depend on timing.
__global__ void __launch_bounds__(kResThreads) kResidualFinish(const double* __restrict__ part,
                                                               const int64_t* __restrict__ first,
                                                               double* __restrict__ rel) {
  const int64_t m = blockIdx.x;
  double a = 0.0, c = 0.0;
  for (int64_t k = first[m] + threadIdx.x; k < first[m + 1]; k += kResThreads) {
    a += part[2 * k];
    c += part[2 * k + 1];
  }
  __shared__ double sa[kResThreads], sc[kResThreads];
  sa[threadIdx.x] = a;
  sc[threadIdx.x] = c;
  __syncthreads();
  for (int s = kResThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sa[threadIdx.x] += sa[threadIdx.x + s];
      sc[threadIdx.x] += sc[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) rel[m] = sc[0] > 0.0 ? sqrt(sa[0] / sc[0]) : sqrt(sa[0]);
}

// Row parameters of count octrees on the device.
static its_status uploadParams(its_ctx* ctx, its_svo* const* svos, int64_t count, DevBuf<RowParams>& dP) {
  its_status st;
  std::vector<RowParams> h(count);
  for (int64_t m = 0; m < count; ++m) h[m] = rowParams(svos[m]->d);
  if ((st = dP.alloc(ctx, count)) != ITS_OK) return st;
  // from pageable memory: the call returns once the source is staged, so h may go away
  ITS_CU(ctx, cudaMemcpyAsync(dP.p, h.data(), count * sizeof(RowParams), cudaMemcpyHostToDevice, ctx->stream));
  return ITS_OK;
}

// Exact starts of count octrees (device vectors), matrix-free: one launch for the shares and
// one per depth (root first) for all octrees together.
its_status exactStart(its_ctx* ctx, its_svo* const* svos, int64_t count, const double* const* b,
                      const double* const* shares, double* const* lam) {
  its_status st;
  DevBuf<RowParams> dP;
  if ((st = uploadParams(ctx, svos, count, dP)) != ITS_OK) return st;
  int maxDepth = 0;
  for (int64_t m = 0; m < count; ++m) maxDepth = std::max(maxDepth, svos[m]->d.depth);
  std::vector<RowSeg> segs;
  std::vector<int64_t> prefix;
  std::vector<int> first(maxDepth + 2, 0);
  std::vector<int64_t> rows(maxDepth + 1, 0);
  // level 0: whole octrees (shares); level t+1: depth (depth-1-t) of every octree
  for (int t = -1; t < maxDepth; ++t) {
    first[t + 1] = (int)segs.size();
    int64_t acc = 0;
    for (int64_t m = 0; m < count; ++m) {
      const SvoDevice& d = svos[m]->d;
      RowSeg s;
      s.P = dP.p + m;
      s.b = b[m];
      s.shares = shares ? shares[m] : nullptr;
      s.lam = lam[m];
      if (t < 0) {
        s.d = -1;
        s.rowBegin = 0;
        s.rows = d.numVerts;
      } else {
        const int dep = d.depth - 1 - t;
        if (dep < 0 || d.vertCount[dep] == 0) continue;
        s.d = dep;
        s.rowBegin = d.vertStart[dep];
        s.rows = d.vertCount[dep];
      }
      if (!s.rows) continue;
      segs.push_back(s);
      prefix.push_back(acc);
      acc += s.rows;
    }
    rows[t + 1] = acc;
  }
  first[maxDepth + 1] = (int)segs.size();
  const int nseg = (int)segs.size();
  if (!nseg) return ITS_OK;
  DevBuf<RowSeg> dSegs;
  DevBuf<int64_t> dPrefix, dLevelRows;
  DevBuf<int> dLevelFirst;
  if ((st = dSegs.alloc(ctx, nseg)) != ITS_OK || (st = dPrefix.alloc(ctx, nseg)) != ITS_OK ||
      (st = dLevelFirst.alloc(ctx, maxDepth + 1)) != ITS_OK || (st = dLevelRows.alloc(ctx, maxDepth)) != ITS_OK)
    return st;
  ITS_CU(ctx, cudaMemcpyAsync(dSegs.p, segs.data(), nseg * sizeof(RowSeg), cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dPrefix.p, prefix.data(), nseg * 8, cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dLevelFirst.p, first.data() + 1, (maxDepth + 1) * sizeof(int), cudaMemcpyHostToDevice,
                              ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dLevelRows.p, rows.data() + 1, maxDepth * 8, cudaMemcpyHostToDevice, ctx->stream));
  // leading run of small depths (from the root): one launch for all of them
  int tSmall = 0;
  while (tSmall < maxDepth && rows[tSmall + 1] <= kSmallLevelRows) ++tSmall;
  for (int t = -1; t < maxDepth; ++t) {
    if (t == 0 && tSmall >= 2) {
      // shares first (t = -1 above), then the small depths together
      kStartLevelsSmall<<<1, 1024, 0, ctx->stream>>>(dSegs.p, dPrefix.p, dLevelFirst.p, dLevelRows.p, 0, tSmall);
      ITS_LAUNCHED(ctx);
      t = tSmall - 1;
      continue;
    }
    const int g0 = first[t + 1], ng = first[t + 2] - g0;
    const int64_t total = rows[t + 1];
    if (!ng || !total) continue;
    if (t < 0)
      kStartShares<<<gridFor(total, 256), 256, 0, ctx->stream>>>(dSegs.p + g0, dPrefix.p + g0, ng, total);
    else
      kStartLevel<<<gridFor(total, 128), 128, 0, ctx->stream>>>(dSegs.p + g0, dPrefix.p + g0, ng, total);
    ITS_LAUNCHED(ctx);
  }
  return ITS_OK;  // the tables were copied from pageable memory (staged at the call)
}

// ||b - A lambda|| / ||b|| of count octrees (device vectors), matrix-free, into rel[count]
// (host), each mesh's sum in a fixed order.
its_status fitResidual(its_ctx* ctx, its_svo* const* svos, int64_t count, const double* const* b,
                       const double* const* lam, double* rel) {
  its_status st;
  DevBuf<RowParams> dP;
  if ((st = uploadParams(ctx, svos, count, dP)) != ITS_OK) return st;
  std::vector<RowSeg> segs;
  std::vector<int64_t> first(count + 1, 0);
  for (int64_t m = 0; m < count; ++m) {
    first[m] = (int64_t)segs.size();
    const int64_t n = svos[m]->d.numVerts;
    for (int64_t r0 = 0; r0 < n; r0 += kResChunk) {
      RowSeg s;
      s.P = dP.p + m;
      s.d = -1;
      s.rowBegin = r0;
      s.rows = std::min(kResChunk, n - r0);
      s.b = b[m];
      s.shares = nullptr;
      s.lam = const_cast<double*>(lam[m]);
      segs.push_back(s);
    }
  }
  first[count] = (int64_t)segs.size();
  const int64_t nseg = (int64_t)segs.size();
  DevBuf<RowSeg> dSegs;
  DevBuf<int64_t> dFirst;
  DevBuf<double> part, dRel;
  if ((st = dSegs.alloc(ctx, std::max<int64_t>(nseg, 1))) != ITS_OK || (st = dFirst.alloc(ctx, count + 1)) != ITS_OK ||
      (st = part.alloc(ctx, 2 * std::max<int64_t>(nseg, 1))) != ITS_OK || (st = dRel.alloc(ctx, count)) != ITS_OK)
    return st;
  ITS_CU(ctx, cudaMemcpyAsync(dSegs.p, segs.data(), nseg * sizeof(RowSeg), cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dFirst.p, first.data(), (count + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (nseg) {
    kResidualChunks<<<(unsigned)nseg, kResThreads, 0, ctx->stream>>>(dSegs.p, part.p);
    ITS_LAUNCHED(ctx);
  } else {
    ITS_CU(ctx, cudaMemsetAsync(part.p, 0, 16, ctx->stream));
  }
  kResidualFinish<<<(unsigned)count, kResThreads, 0, ctx->stream>>>(part.p, dFirst.p, dRel.p);
  ITS_LAUNCHED(ctx);
  ITS_CU(ctx, cudaMemcpyAsync(rel, dRel.p, count * 8, cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // namespace its

using namespace its;

namespace {
its_status checkSvos(its_svo* const* svos, int64_t count, its_ctx** ctxOut) {
  if (!svos || count <= 0 || !svos[0]) return ITS_ERR_INVALID;
  its_ctx* ctx = svos[0]->ctx;
  for (int64_t m = 0; m < count; ++m)
    if (!svos[m] || svos[m]->ctx != ctx) return setError(ctx, ITS_ERR_INVALID, "octrees must share one context");
  *ctxOut = ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  return ITS_OK;
}
}  // namespace

extern "C" {

its_status its_exact_start_batch(its_svo* const* svos, int64_t count, const double* const* b,
                                 const double* const* shares, double* const* lambda) {
  its_ctx* ctx = nullptr;
  its_status st = checkSvos(svos, count, &ctx);
  if (st != ITS_OK) return st;
  if (!b || !lambda) return ITS_ERR_INVALID;
  std::vector<InArg<double>> B(count), S(count);
  std::vector<OutArg<double>> L(count);
  std::vector<const double*> db(count), ds(count);
  std::vector<double*> dl(count);
  for (int64_t m = 0; m < count; ++m) {
    if (!b[m] || !lambda[m]) return ITS_ERR_INVALID;
    const int64_t n = svos[m]->d.numVerts;
    if ((st = B[m].stage(ctx, b[m], n)) != ITS_OK) return st;
    ds[m] = nullptr;
    if (shares && shares[m]) {
      if ((st = S[m].stage(ctx, shares[m], n)) != ITS_OK) return st;
      ds[m] = S[m].d;
    }
    if ((st = L[m].stage(ctx, lambda[m], n)) != ITS_OK) return st;
    db[m] = B[m].d;
    dl[m] = L[m].d;
  }
  if ((st = exactStart(ctx, svos, count, db.data(), ds.data(), dl.data())) != ITS_OK) return st;
  bool host = false;
  for (int64_t m = 0; m < count; ++m) {
    host = host || L[m].host;
    if ((st = L[m].finish(ctx)) != ITS_OK) return st;
  }
  // device outputs: ordered on the context's stream; host outputs: complete on return
  if (host) ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_exact_start(its_svo* svo, const double* b, const double* shares, double* lambda) {
  return its_exact_start_batch(&svo, 1, &b, &shares, &lambda);
}

its_status its_fit_residual_batch(its_svo* const* svos, int64_t count, const double* const* b,
                                  const double* const* lambda, double* rel_residual) {
  its_ctx* ctx = nullptr;
  its_status st = checkSvos(svos, count, &ctx);
  if (st != ITS_OK) return st;
  if (!b || !lambda || !rel_residual) return ITS_ERR_INVALID;
  std::vector<InArg<double>> B(count), L(count);
  std::vector<const double*> db(count), dl(count);
  for (int64_t m = 0; m < count; ++m) {
    if (!b[m] || !lambda[m]) return ITS_ERR_INVALID;
    const int64_t n = svos[m]->d.numVerts;
    if ((st = B[m].stage(ctx, b[m], n)) != ITS_OK || (st = L[m].stage(ctx, lambda[m], n)) != ITS_OK) return st;
    db[m] = B[m].d;
    dl[m] = L[m].d;
  }
  return fitResidual(ctx, svos, count, db.data(), dl.data(), rel_residual);
}

its_status its_fit_residual(its_svo* svo, const double* b, const double* lambda, double* rel_residual) {
  return its_fit_residual_batch(&svo, 1, &b, &lambda, rel_residual);
}

}  // extern "C"
