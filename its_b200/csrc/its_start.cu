// Exact start of the thin-shell least-squares system.
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
//   * every other vertex v takes its hierarchical surplus, the value at v minus what the
//     coarser depths already put there.
//
// The surplus needs no sweep over the depths. The coarser depths' part of the field,
// F_{>d} = sum over depths dd > d of the hats of the depth-dd corners, is trilinear on the
// cell P of depth d+1 that holds v (each depth-dd term is trilinear on its own cell, which
// contains P), so it is the trilinear interpolant -- row v's hats of P's corners -- of its
// values at P's corners c. Those values follow from row c alone: the row says
// F_{>=d+1}(c) = b_c - (the finer coincident vertices at c), i.e. b_c minus shares. With
//   G_u = b_u - sum of the shares of the finer coincident vertices at u's point,
// every surplus is explicit:
//   lambda_v = G_v - sum_{corners c of P} hat_c(v) G_c        (lambda_v = G_v at the root),
// one independent row per vertex: two launches (G, then lambda) for any number of octrees,
// one when the shares are zero (G = b). The result satisfies A lambda = b up to rounding
// for any shares. CGLS started there stops at once (Eigen's solve with a guess tests the
// initial residual first), and because CGLS only moves inside the row space of A, the
// shares fix the null-space component of the final coefficients. The field at the corner
// vertices, and hence in every finest cell, is the same for every exact solution; coarser
// cells differ by that null-space component.
//
// Both the start and the residual check are matrix-free: rows and their parts come from the
// octree (walkRow, walkChain, walkAncestor in its_rows.cuh) in the assembled operator's
// column order, so no CSR is needed.
#include <algorithm>
#include <cmath>
#include <vector>

#include "its_op.cuh"
#include "its_rows.cuh"

namespace its {

// One octree (exact start) or one chunk of rows of an octree (residual).
struct RowSeg {
  const RowParams* P;    // the octree's row parameters (device)
  int64_t rowBegin, rows;
  const double* b;
  const double* shares;  // may be null (all shares 0)
  double* g;             // values less the finer shares (b itself when there are no shares)
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

// G_r = b_r - the shares of the finer coincident vertices at r's point (finest first).
__global__ void kStartValues(const RowSeg* __restrict__ segs, const int64_t* __restrict__ prefix, int nseg,
                             int64_t total) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int k = findSeg(prefix, nseg, i);
  const RowSeg& s = segs[k];
  const int64_t r = s.rowBegin + (i - prefix[k]);
  const RowParams& P = *s.P;
  const int d = rowDepth(P, r);
  const uint32_t M = P.lat[d].M, lin = P.vertLin[r];
  double acc = 0.0;
  if (s.shares) walkChain(P, d, lin / (M * M), (lin / M) % M, lin % M, [&](int32_t c) { acc += s.shares[c]; });
  s.g[r] = s.b[r] - acc;
}

// lambda_r: the share of a coincident vertex; otherwise G_r less the interpolant of G over
// the corners of the owner's parent cell (the row's hats of that depth, in column order).
__global__ void kStartInterp(const RowSeg* __restrict__ segs, const int64_t* __restrict__ prefix, int nseg,
                             int64_t total) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int k = findSeg(prefix, nseg, i);
  const RowSeg& s = segs[k];
  const int64_t r = s.rowBegin + (i - prefix[k]);
  const RowParams& P = *s.P;
  const int d = rowDepth(P, r);
  if (rowCoincident(P, r, d)) {
    s.lam[r] = s.shares ? s.shares[r] : 0.0;
    return;
  }
  const double* __restrict__ g = s.g;
  double acc = 0.0;
  if (d + 1 < P.depth) {
    uint32_t Xo, Yo, Zo;
    mortonDecode(P.morton[P.vertOwner[r]], Xo, Yo, Zo);
    walkAncestor(P, d, d + 1, Xo, Yo, Zo, P.vertPos[3 * r], P.vertPos[3 * r + 1], P.vertPos[3 * r + 2],
                 [&](int32_t c, double v) { acc += v * g[c]; });
  }
  s.lam[r] = g[r] - acc;
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

// Exact starts of count octrees (device vectors), matrix-free: G (when there are shares),
// then lambda, each one launch for all octrees together.
its_status exactStart(its_ctx* ctx, its_svo* const* svos, int64_t count, const double* const* b,
                      const double* const* shares, double* const* lam) {
  its_status st;
  DevBuf<RowParams> dP;
  if ((st = uploadParams(ctx, svos, count, dP)) != ITS_OK) return st;
  bool anyShares = false;
  int64_t total = 0;
  for (int64_t m = 0; m < count; ++m) {
    anyShares = anyShares || (shares && shares[m]);
    total += svos[m]->d.numVerts;
  }
  DevBuf<double> G;
  if (anyShares && (st = G.alloc(ctx, std::max<int64_t>(total, 1))) != ITS_OK) return st;
  std::vector<RowSeg> segs;
  std::vector<int64_t> prefix;
  int64_t acc = 0;
  for (int64_t m = 0; m < count; ++m) {
    const int64_t n = svos[m]->d.numVerts;
    if (!n) continue;
    RowSeg s;
    s.P = dP.p + m;
    s.rowBegin = 0;
    s.rows = n;
    s.b = b[m];
    s.shares = shares ? shares[m] : nullptr;
    s.g = anyShares ? G.p + acc : const_cast<double*>(b[m]);  // no shares anywhere: G = b
    s.lam = lam[m];
    segs.push_back(s);
    prefix.push_back(acc);
    acc += n;
  }
  const int nseg = (int)segs.size();
  if (!nseg) return ITS_OK;
  DevBuf<RowSeg> dSegs;
  DevBuf<int64_t> dPrefix;
  if ((st = dSegs.alloc(ctx, nseg)) != ITS_OK || (st = dPrefix.alloc(ctx, nseg)) != ITS_OK) return st;
  ITS_CU(ctx, cudaMemcpyAsync(dSegs.p, segs.data(), nseg * sizeof(RowSeg), cudaMemcpyHostToDevice, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(dPrefix.p, prefix.data(), nseg * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (anyShares) {
    kStartValues<<<gridFor(total, 256), 256, 0, ctx->stream>>>(dSegs.p, dPrefix.p, nseg, total);
    ITS_LAUNCHED(ctx);
  }
  kStartInterp<<<gridFor(total, 256), 256, 0, ctx->stream>>>(dSegs.p, dPrefix.p, nseg, total);
  ITS_LAUNCHED(ctx);
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
      s.rowBegin = r0;
      s.rows = std::min(kResChunk, n - r0);
      s.b = b[m];
      s.shares = nullptr;
      s.g = nullptr;
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
