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
#include <cstring>
#include <vector>

#include "its_op.cuh"
#include "its_rows.cuh"
#include "its_tune.cuh"

namespace its {

// One octree of an exact start.
struct RowSeg {
  const RowParams* P;    // the octree's row parameters (device)
  int64_t rowBegin, rows;
  const double* b;
  const double* shares;  // may be null (all shares 0)
  double* g;             // values less the finer shares (b itself when there are no shares)
  double* lam;
};

// A segment table and its prefix. Up to kInlineSegs segments travel with the launch as a
// kernel parameter (no copy, nothing to wait for); a larger table is copied to the device once
// (from pageable memory, staged at the call) into keep, which the caller holds until the
// launches are queued.
constexpr int kInlineSegs = 16;
template <class Seg>
struct SegArgs {
  int nseg = 0;
  const Seg* dsegs = nullptr;
  const int64_t* dprefix = nullptr;
  unsigned long long* stamp = nullptr;  // when set: the device clock (ns) at the kernel's start
  Seg segs[kInlineSegs];
  int64_t prefix[kInlineSegs + 1];
  __device__ __forceinline__ const Seg& seg(int k) const { return dsegs ? dsegs[k] : segs[k]; }
  __device__ __forceinline__ int64_t pre(int k) const { return dsegs ? dprefix[k] : prefix[k]; }
  // last segment whose first item is <= i
  __device__ __forceinline__ int find(int64_t i) const {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pre(mid) <= i) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
};

template <class Seg>
static its_status makeSegArgs(its_ctx* ctx, const std::vector<Seg>& segs, const std::vector<int64_t>& prefix,
                              SegArgs<Seg>& A, DevBuf<uint8_t>& keep) {
  A.nseg = (int)segs.size();
  if (A.nseg <= kInlineSegs) {
    for (int k = 0; k < A.nseg; ++k) {
      A.segs[k] = segs[k];
      A.prefix[k] = prefix[k];
    }
    A.prefix[A.nseg] = prefix[A.nseg];
    return ITS_OK;
  }
  const size_t a = segs.size() * sizeof(Seg), b = (segs.size() + 1) * sizeof(int64_t);
  std::vector<uint8_t> h(a + b);
  std::memcpy(h.data(), segs.data(), a);
  std::memcpy(h.data() + a, prefix.data(), b);
  its_status st;
  if ((st = keep.alloc(ctx, a + b)) != ITS_OK) return st;
  ITS_CU(ctx, cudaMemcpyAsync(keep.p, h.data(), a + b, cudaMemcpyHostToDevice, ctx->stream));
  A.dsegs = (const Seg*)keep.p;
  A.dprefix = (const int64_t*)(keep.p + a);
  return ITS_OK;
}

// G_r = b_r - the shares of the finer coincident vertices at r's point (finest first).
__global__ void __launch_bounds__(256) kStartValues(const __grid_constant__ SegArgs<RowSeg> A, int64_t total) {
  gridDependencyWait();
  gridDependents();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int k = A.find(i);
  const RowSeg& s = A.seg(k);
  const int64_t r = s.rowBegin + (i - A.pre(k));
  const RowParams& P = *s.P;
  double acc = 0.0;
  if (s.shares) {
    const VertCoord v = vertCoord(P, r);
    walkChain(P, v.d, v.X, v.Y, v.Z, [&](int32_t c) { acc += s.shares[c]; });
  }
  s.g[r] = s.b[r] - acc;
}

// lambda_r: the share of a coincident vertex; otherwise G_r less the interpolant of G over
// the corners of the owner's parent cell (the row's hats of that depth, in column order).
__global__ void __launch_bounds__(256) kStartInterp(const __grid_constant__ SegArgs<RowSeg> A, int64_t total) {
  gridDependencyWait();
  gridDependents();
  if (A.stamp && blockIdx.x == 0 && threadIdx.x == 0) *A.stamp = globalTimer();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int k = A.find(i);
  const RowSeg& s = A.seg(k);
  const int64_t r = s.rowBegin + (i - A.pre(k));
  const RowParams& P = *s.P;
  const VertCoord v = vertCoord(P, r);
  if (coordCoincident(P, v)) {
    s.lam[r] = s.shares ? s.shares[r] : 0.0;
    return;
  }
  const double* __restrict__ g = s.g;
  double acc = 0.0;
  if (v.d + 1 < P.depth)
    walkAncestor(P, v, v.d + 1, P.vertPos[3 * r], P.vertPos[3 * r + 1], P.vertPos[3 * r + 2],
                 [&](int32_t c, double h) { acc += h * g[c]; });
  s.lam[r] = g[r] - acc;
}

// ---- residual ||b - A lambda|| ---------------------------------------------------------
// (A lambda)_v = (the finer coincident columns: their lambdas) + H_v, where H_v = lambda_v +
// F_{>d}(v) is the field of v's own and the coarser depths at v. F_{>d} is trilinear on the
// owner's parent cell (the argument of the exact start), so
//   H_v = lambda_v + sum_{corners c of the parent cell} hat_c(v) H_c:
// the same operator with 8 hats per row instead of 8 per ancestor. Two bands, each one launch
// for all octrees: the vertices above the finest depth sum H_v as row v has it (the hats of
// every ancestor's corners); then the finest depth -- most of the rows, with the most
// ancestors -- interpolates H from the band above. Every chunk of rows (32 in the coarse band,
// 256 at the finest depth) leaves its sums of e^2 and b^2 in a slot of its own, a mesh's slots
// contiguous, and kResidualFinish adds a mesh's slots in a fixed order.
constexpr int kResThreads = 256;

struct ResSeg {
  const RowParams* P;
  int64_t rowBegin, rows;  // one band of one octree
  const double* b;
  const double* lam;
  double* H;
  int64_t slot;            // slot of the segment's first chunk
};

// The finest depth: one row per thread, H interpolated from the parent cell's corners.
__global__ void __launch_bounds__(kResThreads) kResidualFine(const __grid_constant__ SegArgs<ResSeg> A,
                                                            double* __restrict__ part) {
  gridDependencyWait();
  gridDependents();
  const int k = A.find(blockIdx.x);
  const ResSeg& s = A.seg(k);
  const int64_t j = blockIdx.x - A.pre(k);
  const RowParams& P = *s.P;
  const int64_t i = j * kResThreads + threadIdx.x;
  double rr = 0.0, bb = 0.0;
  if (i < s.rows) {
    const int64_t r = s.rowBegin + i;
    const VertCoord v = vertCoord(P, r);
    const double* __restrict__ lam = s.lam;
    const double* __restrict__ H = s.H;
    double acc = 0.0;
    if (v.d + 1 < P.depth)
      walkAncestor(P, v, v.d + 1, P.vertPos[3 * r], P.vertPos[3 * r + 1], P.vertPos[3 * r + 2],
                   [&](int32_t c, double h) { acc += h * H[c]; });
    const double h = lam[r] + acc;
    double chain = 0.0;
    walkChain(P, v.d, v.X, v.Y, v.Z, [&](int32_t c) { chain += lam[c]; });
    const double e = s.b[r] - (chain + h);
    rr = e * e;
    bb = s.b[r] * s.b[r];
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
    part[2 * (s.slot + j)] = a;
    part[2 * (s.slot + j) + 1] = c;
  }
}

// The coarse band: 32 rows per block, lane l of every warp on row l, warp w summing the hats
// of the ancestors at depths d+1+w, d+9+w, ... (a warp's loads stay on one depth of
// neighbouring rows; these rows are few, so the ancestors, not the rows, fill the GPU). The
// last warp also takes the row's finer coincident columns; the parts are added in warp order.
constexpr int kResCoarseRows = 32;
constexpr int kResWarps = kResThreads / 32;
__global__ void __launch_bounds__(kResThreads) kResidualCoarse(const __grid_constant__ SegArgs<ResSeg> A,
                                                              double* __restrict__ part) {
  gridDependencyWait();
  gridDependents();
  __shared__ double sacc[kResWarps][kResCoarseRows];
  __shared__ double schain[kResCoarseRows];
  const int k = A.find(blockIdx.x);
  const ResSeg& s = A.seg(k);
  const int64_t j = blockIdx.x - A.pre(k);
  const RowParams& P = *s.P;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i = j * kResCoarseRows + lane;
  const double* __restrict__ lam = s.lam;
  double acc = 0.0;
  if (i < s.rows) {
    const int64_t r = s.rowBegin + i;
    const VertCoord v = vertCoord(P, r);
    if (v.d + 1 + warp < P.depth) {
      const double qx = P.vertPos[3 * r], qy = P.vertPos[3 * r + 1], qz = P.vertPos[3 * r + 2];
      for (int dd = v.d + 1 + warp; dd < P.depth; dd += kResWarps)
        walkAncestor(P, v, dd, qx, qy, qz, [&](int32_t c, double h) { acc += h * lam[c]; });
    }
    if (warp == kResWarps - 1) {  // the last warp has the fewest ancestors: it walks the chain too
      double chain = 0.0;
      walkChain(P, v.d, v.X, v.Y, v.Z, [&](int32_t c) { chain += lam[c]; });
      schain[lane] = chain;
    }
  }
  sacc[warp][lane] = acc;
  __syncthreads();
  if (warp == 0) {
    double rr = 0.0, bb = 0.0;
    if (i < s.rows) {
      const int64_t r = s.rowBegin + i;
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < kResWarps; ++w) t += sacc[w][lane];
      const double h = lam[r] + t;
      s.H[r] = h;
      const double e = s.b[r] - (schain[lane] + h);
      rr = e * e;
      bb = s.b[r] * s.b[r];
    }
    for (int o = 16; o > 0; o >>= 1) {
      rr += __shfl_down_sync(0xffffffffu, rr, o);
      bb += __shfl_down_sync(0xffffffffu, bb, o);
    }
    if (lane == 0) {
      part[2 * (s.slot + j)] = rr;
      part[2 * (s.slot + j) + 1] = bb;
    }
  }
}

// Slot ranges of the meshes for kResidualFinish (inline up to kInlineSegs meshes).
struct SlotArgs {
  const int64_t* dfirst = nullptr;
  int64_t first[kInlineSegs + 1];
  const int* flagSrc = nullptr;  // optional: one flag copied to flagDst with the results
  int* flagDst = nullptr;
  unsigned long long* stampEnd = nullptr;  // optional: the device clock (ns) when the results are out
  __device__ __forceinline__ int64_t at(int64_t m) const { return dfirst ? dfirst[m] : first[m]; }
};

// One block per mesh: the mesh's chunk partials in a fixed order (strided per thread, then a
// fixed tree), so the result does not depend on timing.
__global__ void __launch_bounds__(kResThreads) kResidualFinish(const double* __restrict__ part,
                                                               const __grid_constant__ SlotArgs F,
                                                               double* __restrict__ rel) {
  gridDependencyWait();
  gridDependents();
  const int64_t m = blockIdx.x;
  if (m == 0 && threadIdx.x == 0 && F.flagSrc) *F.flagDst = *F.flagSrc;
  double a = 0.0, c = 0.0;
  for (int64_t k = F.at(m) + threadIdx.x; k < F.at(m + 1); k += kResThreads) {
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
  if (threadIdx.x == 0) {
    rel[m] = sc[0] > 0.0 ? sqrt(sa[0] / sc[0]) : sqrt(sa[0]);
    if (m == 0 && F.stampEnd) *F.stampEnd = globalTimer();
  }
}

static const RowParams* rowParamsOf(its_svo* s) { return (const RowParams*)s->d.rowParams; }

// Exact starts of count octrees (device vectors), matrix-free: G (when there are shares),
// then lambda, each one launch for all octrees together.
its_status exactStart(its_ctx* ctx, its_svo* const* svos, int64_t count, const double* const* b,
                      const double* const* shares, double* const* lam, bool afterKernel, double* gScratch,
                      unsigned long long* stamp) {
  its_status st;
  bool anyShares = false;
  int64_t total = 0;
  for (int64_t m = 0; m < count; ++m) {
    anyShares = anyShares || (shares && shares[m]);
    total += svos[m]->d.numVerts;
  }
  DevBuf<double> G;
  if (anyShares && !gScratch && (st = G.alloc(ctx, std::max<int64_t>(total, 1))) != ITS_OK) return st;
  double* g = gScratch ? gScratch : G.p;
  std::vector<RowSeg> segs;
  std::vector<int64_t> prefix;
  int64_t acc = 0;
  for (int64_t m = 0; m < count; ++m) {
    const int64_t n = svos[m]->d.numVerts;
    if (!n) continue;
    RowSeg s;
    s.P = rowParamsOf(svos[m]);
    s.rowBegin = 0;
    s.rows = n;
    s.b = b[m];
    s.shares = shares ? shares[m] : nullptr;
    s.g = anyShares ? g + acc : const_cast<double*>(b[m]);  // no shares anywhere: G = b
    s.lam = lam[m];
    segs.push_back(s);
    prefix.push_back(acc);
    acc += n;
  }
  if (segs.empty()) return ITS_OK;
  prefix.push_back(acc);
  SegArgs<RowSeg> A;
  DevBuf<uint8_t> keep;
  if ((st = makeSegArgs(ctx, segs, prefix, A, keep)) != ITS_OK) return st;
  A.stamp = stamp;
  // dependent launches only straight after a kernel (no segment table copied in between; not
  // while the autotuner times candidates, which records events between them)
  bool timing = true;
  const bool dep = afterKernel && !A.dsegs;
  // a thread per row, no block-level sums: the block size is result-neutral and tuned
  static const int kStartBlocks[3] = {256, 128, 64};
  auto run = [&](int c) -> its_status {
    const int bs = kStartBlocks[c];
    if (anyShares &&
        (st = launchDependent(ctx, dep && !timing, kStartValues, gridFor(total, bs), bs, 0, ctx->stream, A, total)) !=
            ITS_OK)
      return st;
    return launchDependent(ctx, anyShares || (dep && !timing), kStartInterp, gridFor(total, bs), bs, 0, ctx->stream, A,
                           total);
  };
  const std::string key = std::string("exact_start/rows=") + std::to_string(total) + "/octrees=" +
                          std::to_string(count) + (anyShares ? "/shares" : "/zero");
  // the tuner measures on the first uncaptured call of a key when tuning is on; its last
  // stream operation is then an event, so the launch that follows is not a dependent one
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess) cudaGetLastError();
  const bool measures = ctx->autotune && cs == cudaStreamCaptureStatusNone && ctx->tuned.find(key) == ctx->tuned.end();
  int choice = 0;
  if ((st = tuneChoice(ctx, key, 3, 0, run, &choice)) != ITS_OK) return st;
  timing = measures;
  return run(choice);  // a copied table came from pageable memory (staged at the call)
}

// ||b - A lambda|| / ||b|| of count octrees (device vectors), matrix-free, into relDev[count]
// (device), each mesh's sum in a fixed order: two bands, then the sums; queued on the
// context's stream without a host wait.
its_status fitResidualEnqueue(its_ctx* ctx, its_svo* const* svos, int64_t count, const double* const* b,
                              const double* const* lam, double* relDev, const int* flagSrc, int* flagDst,
                              bool afterKernel, unsigned long long* stampEnd) {
  its_status st;
  int64_t total = 0;
  for (int64_t m = 0; m < count; ++m) total += svos[m]->d.numVerts;
  DevBuf<double> H;
  if ((st = H.alloc(ctx, std::max<int64_t>(total, 1))) != ITS_OK) return st;
  // band 0: depths >= 1; band 1: the finest depth. Mesh m owns slots [mFirst[m], mFirst[m+1]):
  // its band 0 chunks, then band 1's.
  constexpr int kBands = 2;
  std::vector<ResSeg> segs[kBands];
  std::vector<int64_t> cf[kBands];
  int64_t chunks[kBands] = {0, 0};
  std::vector<int64_t> mFirst(count + 1, 0);
  for (int64_t m = 0, h = 0; m < count; ++m) {
    const SvoDevice& d = svos[m]->d;
    auto vs = [&](int k) { return d.vertStart[k < d.depth ? k : d.depth]; };
    const int64_t lo[kBands] = {vs(1), 0}, hi[kBands] = {d.numVerts, vs(1)};
    int64_t slot = mFirst[m];
    for (int band = 0; band < kBands; ++band) {
      ResSeg s;
      s.P = rowParamsOf(svos[m]);
      s.rowBegin = lo[band];
      s.rows = hi[band] - lo[band];
      s.b = b[m];
      s.lam = lam[m];
      s.H = H.p + h;
      s.slot = slot;
      const int64_t per = band == 0 ? kResCoarseRows : kResThreads;  // rows per chunk
      const int64_t c = (s.rows + per - 1) / per;
      if (!c) continue;
      segs[band].push_back(s);
      cf[band].push_back(chunks[band]);
      chunks[band] += c;
      slot += c;
    }
    mFirst[m + 1] = slot;
    h += d.numVerts;
  }
  const int64_t slots = mFirst[count];
  SegArgs<ResSeg> A[kBands];
  DevBuf<uint8_t> keep[kBands + 1];
  for (int band = 0; band < kBands; ++band) {
    cf[band].push_back(chunks[band]);
    if ((st = makeSegArgs(ctx, segs[band], cf[band], A[band], keep[band])) != ITS_OK) return st;
  }
  SlotArgs F;
  F.flagSrc = flagSrc;
  F.flagDst = flagDst;
  F.stampEnd = stampEnd;
  if (count <= kInlineSegs) {
    for (int64_t m = 0; m <= count; ++m) F.first[m] = mFirst[m];
  } else {
    if ((st = keep[kBands].alloc(ctx, (count + 1) * 8)) != ITS_OK) return st;
    ITS_CU(ctx, cudaMemcpyAsync(keep[kBands].p, mFirst.data(), (count + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    F.dfirst = (const int64_t*)keep[kBands].p;
  }
  DevBuf<double> part;
  if ((st = part.alloc(ctx, 2 * std::max<int64_t>(slots, 1))) != ITS_OK) return st;
  // the coarse band first: the finest rows interpolate the H values it writes
  if (chunks[0]) {
    // dependent only straight after the caller's kernel (no table copied in between)
    const bool dep = afterKernel && !A[0].dsegs && !F.dfirst;
    if ((st = launchDependent(ctx, dep, kResidualCoarse, (unsigned)chunks[0], kResThreads, 0, ctx->stream, A[0],
                              part.p)) != ITS_OK)
      return st;
  }
  for (int band = 1; band < kBands; ++band) {
    if (!chunks[band]) continue;
    if ((st = launchDependent(ctx, chunks[0] > 0, kResidualFine, (unsigned)chunks[band], kResThreads, 0, ctx->stream,
                              A[band], part.p)) != ITS_OK)
      return st;
  }
  if (!slots) ITS_CU(ctx, cudaMemsetAsync(part.p, 0, 16, ctx->stream));
  if ((st = launchDependent(ctx, slots > 0, kResidualFinish, (unsigned)count, kResThreads, 0, ctx->stream, (const double*)part.p,
                            F, relDev)) != ITS_OK)
    return st;
  return ITS_OK;
}

// The same into rel[count] in host memory (complete on return).
its_status fitResidual(its_ctx* ctx, its_svo* const* svos, int64_t count, const double* const* b,
                       const double* const* lam, double* rel) {
  its_status st;
  DevBuf<double> dRel;
  if ((st = dRel.alloc(ctx, count)) != ITS_OK) return st;
  if ((st = fitResidualEnqueue(ctx, svos, count, b, lam, dRel.p, nullptr, nullptr, false, nullptr)) != ITS_OK)
    return st;
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
  if ((st = exactStart(ctx, svos, count, db.data(), ds.data(), dl.data(), false, nullptr, nullptr)) != ITS_OK)
    return st;
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
