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
#include <algorithm>
#include <vector>

#include "its_op.cuh"

namespace its {

// One depth of one operator.
struct StartSeg {
  const int64_t* rowptr;
  const int32_t* col;
  const double* val;
  const double* b;
  const double* shares;  // may be null (all shares 0)
  double* lam;
  const uint32_t* vertLin;
  int64_t rowBegin, rows;  // rows of this depth within the operator
  uint32_t M;              // lattice points per axis at this depth
  int root;                // the root depth: no coarser corner
};

constexpr int kStartLanes = 8;  // lanes per row (rows hold at most 1 + 9 (depth - 1) entries)

__device__ __forceinline__ bool evenVertex(const StartSeg& s, int64_t r) {
  if (s.root) return false;
  const uint32_t lin = s.vertLin[r], M = s.M;
  const uint32_t X = lin / (M * M), Y = (lin / M) % M, Z = lin % M;
  return ((X | Y | Z) & 1u) == 0u;
}

__device__ __forceinline__ int findSeg(const int64_t* __restrict__ prefix, int nseg, int64_t i) {
  int lo = 0, hi = nseg - 1;  // last segment with prefix[seg] <= i
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Shares of the even vertices (every depth of every operator).
__global__ void kStartShares(const StartSeg* __restrict__ segs, const int64_t* __restrict__ prefix, int nseg,
                             int64_t total) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int g = findSeg(prefix, nseg, i);
  const StartSeg& s = segs[g];
  const int64_t r = s.rowBegin + (i - prefix[g]);
  s.lam[r] = (evenVertex(s, r) && s.shares) ? s.shares[r] : 0.0;
}

// Surplus of the non-even rows of one depth per operator (segments = one depth each).
__global__ void kStartLevel(const StartSeg* __restrict__ segs, const int64_t* __restrict__ prefix, int nseg,
                            int64_t total) {
  const int64_t item = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kStartLanes;
  const int sub = threadIdx.x & (kStartLanes - 1);
  bool valid = item < total;
  const StartSeg* s = nullptr;
  int64_t r = 0, beg = 0, end = 0;
  if (valid) {
    const int g = findSeg(prefix, nseg, item);
    s = &segs[g];
    r = s->rowBegin + (item - prefix[g]);
    valid = !evenVertex(*s, r);
    if (valid) {
      beg = s->rowptr[r];
      end = s->rowptr[r + 1];
    }
  }
  double acc = 0.0;
  for (int64_t k = beg + sub; k < end; k += kStartLanes) {
    const int32_t c = s->col[k];
    if (c != (int32_t)r) acc += s->val[k] * s->lam[c];
  }
#pragma unroll
  for (int o = kStartLanes / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, kStartLanes);
  if (valid && sub == 0) s->lam[r] = s->b[r] - acc;
}

// Exact starts of count operators: b[m], shares[m] (may be null) and lam[m] are device
// vectors of operator m.
its_status exactStart(its_ctx* ctx, its_op* const* ops, int64_t count, const double* const* b,
                      const double* const* shares, double* const* lam) {
  its_status st;
  int maxDepth = 0;
  for (int64_t m = 0; m < count; ++m) maxDepth = std::max(maxDepth, ops[m]->svo->d.depth);
  // segments: level t (from the root down) of every operator, then all levels for the shares
  std::vector<StartSeg> segs;
  std::vector<int64_t> prefix;
  std::vector<int> levelFirst(maxDepth + 1);
  std::vector<int64_t> levelRows(maxDepth);
  for (int t = 0; t < maxDepth; ++t) {
    levelFirst[t] = (int)segs.size();
    int64_t acc = 0;
    for (int64_t m = 0; m < count; ++m) {
      const SvoDevice& d = ops[m]->svo->d;
      const int dep = d.depth - 1 - t;  // depth index (0 = finest)
      if (dep < 0 || d.vertCount[dep] == 0) continue;
      StartSeg s;
      s.rowptr = ops[m]->rowptr;
      s.col = ops[m]->col;
      s.val = ops[m]->val;
      s.b = b[m];
      s.shares = shares ? shares[m] : nullptr;
      s.lam = lam[m];
      s.vertLin = d.vertLin;
      s.rowBegin = d.vertStart[dep];
      s.rows = d.vertCount[dep];
      s.M = (uint32_t)(d.res >> dep) + 1u;
      s.root = dep == d.depth - 1;
      segs.push_back(s);
      prefix.push_back(acc);
      acc += s.rows;
    }
    levelRows[t] = acc;
  }
  levelFirst[maxDepth] = (int)segs.size();
  const int nseg = (int)segs.size();
  if (!nseg) return ITS_OK;
  DevBuf<StartSeg> dSegs;
  DevBuf<int64_t> dPrefix, dAll;
  if ((st = dSegs.alloc(ctx, nseg)) != ITS_OK || (st = dPrefix.alloc(ctx, nseg)) != ITS_OK ||
      (st = dAll.alloc(ctx, nseg)) != ITS_OK)
    return st;
  // prefix over all segments for the shares pass
  std::vector<int64_t> all(nseg);
  int64_t total = 0;
  for (int g = 0; g < nseg; ++g) {
    all[g] = total;
    total += segs[g].rows;
  }
  ITS_CU(ctx, cudaMemcpyAsync(dSegs.p, segs.data(), nseg * sizeof(StartSeg), cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dPrefix.p, prefix.data(), nseg * 8, cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dAll.p, all.data(), nseg * 8, cudaMemcpyHostToDevice, ctx->stream));
  kStartShares<<<gridFor(total, 256), 256, 0, ctx->stream>>>(dSegs.p, dAll.p, nseg, total);
  ITS_LAUNCHED(ctx);
  for (int t = 0; t < maxDepth; ++t) {
    const int g0 = levelFirst[t], ng = levelFirst[t + 1] - g0;
    if (!ng || !levelRows[t]) continue;
    const int64_t threads = levelRows[t] * kStartLanes;
    kStartLevel<<<(unsigned)((threads + 255) / 256), 256, 0, ctx->stream>>>(dSegs.p + g0, dPrefix.p + g0, ng,
                                                                          levelRows[t]);
    ITS_LAUNCHED(ctx);
  }
  // the host vectors above are read by the copies: wait before they go out of scope
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // namespace its

using namespace its;

extern "C" {

its_status its_exact_start_batch(its_op* const* ops, int64_t count, const double* const* b,
                                 const double* const* shares, double* const* lambda) {
  if (!ops || count <= 0 || !b || !lambda) return ITS_ERR_INVALID;
  its_ctx* ctx = ops[0] ? ops[0]->ctx : nullptr;
  if (!ctx) return ITS_ERR_INVALID;
  for (int64_t m = 0; m < count; ++m)
    if (!ops[m] || ops[m]->ctx != ctx || !b[m] || !lambda[m] || !ops[m]->svo)
      return setError(ctx, ITS_ERR_INVALID, "its_exact_start: operators must share one context");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  // stage host vectors on the device
  std::vector<InArg<double>> B(count), S(count);
  std::vector<OutArg<double>> L(count);
  std::vector<const double*> db(count), ds(count);
  std::vector<double*> dl(count);
  its_status st;
  for (int64_t m = 0; m < count; ++m) {
    const int64_t n = ops[m]->n;
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
  if ((st = exactStart(ctx, ops, count, db.data(), ds.data(), dl.data())) != ITS_OK) return st;
  for (int64_t m = 0; m < count; ++m)
    if ((st = L[m].finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_exact_start(its_op* op, const double* b, const double* shares, double* lambda) {
  if (!op) return ITS_ERR_INVALID;
  return its_exact_start_batch(&op, 1, &b, &shares, &lambda);
}

}  // extern "C"
