// LSCG on the GPU (replaces Eigen::LeastSquaresConjugateGradient, ThinShells.cpp:615-617).
//
// Eigen's algorithm (CGLS with the LeastSquareDiagonalPreconditioner): r = b - A x,
// n = A^T r, p = D n, then per iteration
//   t = A p; alpha = |n|_D^2 / |t|^2; x += alpha p; r -= alpha t; n = A^T r;
//   stop if |n|^2 < tol^2 |A^T b|^2; z = D n; beta = n.z / old; p = z + beta p.
// Scalars never leave the GPU: each reduction writes per-block partials and the last block
// to arrive (ticket counter, no waiting) folds them in a fixed order and updates the
// scalar state, so runs are bit-reproducible. A done flag makes every later kernel of the
// captured iteration a no-op, which lets `check_every` iterations run as one CUDA graph
// between host checks.
//
// Mixed precision: FP32 copies of the values and of the gathered vectors (p, r) feed the
// SpMVs (accumulated in FP64); dot products, x and the residual stay FP64, and an outer
// loop recomputes r = b - A x with the FP64 operator (iterative refinement).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "its_op.cuh"

#include "its_cgls.cuh"

namespace its {


template <class Op>
__global__ void __launch_bounds__(kRedThreads) kReduce(Op op, int64_t n, double* __restrict__ partials,
                                                       CgScalars* __restrict__ S, int honorDone) {
  if (honorDone && S->done) return;
  double a = 0.0, b = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads)
    op.terms(i, a, b);
  blockSum2(a, b);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
    __threadfence();
    const unsigned t = atomicAdd(&S->tickets[op.slot], 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double ta = 0.0, tb = 0.0;
  for (unsigned k = threadIdx.x; k < gridDim.x; k += kRedThreads) {
    ta += ((volatile double*)partials)[2 * k];
    tb += ((volatile double*)partials)[2 * k + 1];
  }
  blockSum2(ta, tb);
  if (threadIdx.x == 0) {
    op.finalize(S, ta, tb);
    S->tickets[op.slot] = 0;
  }
}

// ---- initial state ------------------------------------------------------------------------
__global__ void kUpdateP(int64_t n, const double* __restrict__ nr, const double* __restrict__ invdiag,
                         double* __restrict__ p, float* __restrict__ pf, const CgScalars* __restrict__ S) {
  if (S->done) return;
  const double beta = S->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double z = invdiag[i] * nr[i];
    const double v = z + beta * p[i];
    p[i] = v;
    if (pf) pf[i] = (float)v;
  }
}
__global__ void kCopyToFloat(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void kZeroIfEmptyRhs(int64_t n, double* __restrict__ x, const CgScalars* __restrict__ S) {
  if (S->rhsNorm2 != 0.0) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] = 0.0;
}
__global__ void kAxpy(int64_t n, double* __restrict__ x, const double* __restrict__ d) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] += d[i];
}
__global__ void kSetScalars(CgScalars* S, double tol, long long maxIters, int stopRule) {
  S->tol = tol;
  S->maxIters = maxIters;
  S->stopRule = stopRule;
  S->done = 0;
  S->converged = 0;
  S->breakdown = 0;
  S->iter = 0;
  for (int k = 0; k < 8; ++k) S->tickets[k] = 0;
}

// Workspace layout (doubles): x, r, nr, p, t, b, d (7n); floats: pf, rf (2n).
struct Work {
  double *x, *r, *nr, *p, *t, *b, *d;
  float *pf, *rf;
};

static its_status ensureWork(its_op* op) {
  its_ctx* ctx = op->ctx;
  its_status st;
  if (!op->work && (st = devAlloc(ctx, (void**)&op->work, 7 * op->n * 8)) != ITS_OK) return st;
  if (!op->workf && (st = devAlloc(ctx, (void**)&op->workf, 2 * op->n * 4)) != ITS_OK) return st;
  if (!op->scalars && (st = devAlloc(ctx, &op->scalars, sizeof(CgScalars))) != ITS_OK) return st;
  if (!op->partials && (st = devAlloc(ctx, (void**)&op->partials, 2 * 8 * 4096 * 8)) != ITS_OK) return st;
  op->hostDone = ctx->pinned;
  if (!op->hostDone) return setError(ctx, ITS_ERR_STATE, "context has no pinned scratch");
  return ITS_OK;
}
static Work workOf(its_op* op) {
  const int64_t n = op->n;
  Work w;
  w.x = op->work;
  w.r = w.x + n;
  w.nr = w.r + n;
  w.p = w.nr + n;
  w.t = w.p + n;
  w.b = w.t + n;
  w.d = w.b + n;
  w.pf = op->workf;
  w.rf = w.pf + n;
  return w;
}

struct SolveCtx {
  its_op* op;
  Work w;
  CgScalars* S;
  double* part[6];
  unsigned redBlocks;
};

template <class Op>
static its_status reduce(its_ctx* ctx, const SolveCtx& sc, const Op& o, int honorDone) {
  kReduce<Op><<<sc.redBlocks, kRedThreads, 0, ctx->stream>>>(o, sc.op->n, sc.part[o.slot], sc.S, honorDone);
  ITS_LAUNCHED(ctx);
  return ITS_OK;
}

// CGLS on A x = rhs (FP64 values, or FP32 copies when f32), starting from x (in w.x).
// Enqueues the initial phase; the caller then runs iterations.
static its_status cglsInit(its_ctx* ctx, const SolveCtx& sc, const double* rhs, bool hasX0, bool f32) {
  its_op* op = sc.op;
  const Work& w = sc.w;
  its_status st;
  if (hasX0) {
    if ((st = spmv(ctx, op->A64(), op->planA, (const double*)w.x, w.t)) != ITS_OK) return st;
  }
  if ((st = reduce(ctx, sc, OpInitResidual{rhs, hasX0 ? w.t : nullptr, w.r}, 0)) != ITS_OK) return st;
  // A^T rhs -> w.d (scratch), |A^T rhs|^2
  if ((st = spmv(ctx, op->T64(), op->planT, rhs, w.d)) != ITS_OK) return st;
  if ((st = reduce(ctx, sc, OpRhsNorm{w.d}, 0)) != ITS_OK) return st;
  if ((st = spmv(ctx, op->T64(), op->planT, (const double*)w.r, w.nr)) != ITS_OK) return st;
  if ((st = reduce(ctx, sc, OpInitNormal{w.nr, op->invdiag, w.p, f32 ? w.pf : nullptr}, 0)) != ITS_OK) return st;
  if (f32) {
    kCopyToFloat<<<sc.redBlocks, 256, 0, ctx->stream>>>(op->n, w.r, w.rf);
    ITS_LAUNCHED(ctx);
  }
  return ITS_OK;
}

static its_status cglsIteration(its_ctx* ctx, const SolveCtx& sc, bool f32) {
  its_op* op = sc.op;
  const Work& w = sc.w;
  its_status st;
  const int* skip = &sc.S->done;
  if (f32) st = spmv(ctx, op->A32(), op->planA, (const float*)w.pf, w.t, skip);
  else st = spmv(ctx, op->A64(), op->planA, (const double*)w.p, w.t, skip);
  if (st != ITS_OK) return st;
  if ((st = reduce(ctx, sc, OpTmpNorm{w.t}, 1)) != ITS_OK) return st;
  if ((st = reduce(ctx, sc, OpUpdateXR{sc.S, w.x, w.r, f32 ? w.rf : nullptr, w.p, w.t}, 1)) != ITS_OK) return st;
  if (f32) st = spmv(ctx, op->T32(), op->planT, (const float*)w.rf, w.nr, skip);
  else st = spmv(ctx, op->T64(), op->planT, (const double*)w.r, w.nr, skip);
  if (st != ITS_OK) return st;
  if ((st = reduce(ctx, sc, OpNormal{w.nr, op->invdiag}, 1)) != ITS_OK) return st;
  kUpdateP<<<sc.redBlocks, 256, 0, ctx->stream>>>(op->n, w.nr, op->invdiag, w.p, f32 ? w.pf : nullptr, sc.S);
  ITS_LAUNCHED(ctx);
  return ITS_OK;
}

// Runs iterations until the device sets done: graphs of `every` iterations.
static its_status cglsRun(its_ctx* ctx, const SolveCtx& sc, bool f32, int every) {
  its_op* op = sc.op;
  const int key[4] = {f32 ? 1 : 0, every, (int)(op->n & 0x7fffffff), 1};
  if (!op->graph || std::memcmp(key, op->graphKey, sizeof(key)) != 0) {
    if (op->graph) {
      cudaGraphExecDestroy(op->graph);
      op->graph = nullptr;
    }
    cudaGraph_t g;
    ITS_CU(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    its_status st = ITS_OK;
    const int64_t before = ctx->launches;
    for (int k = 0; k < every && st == ITS_OK; ++k) st = cglsIteration(ctx, sc, f32);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (st != ITS_OK) return st;
    if (e != cudaSuccess) return cudaFail(ctx, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&op->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cudaFail(ctx, e, "cudaGraphInstantiate");
    std::memcpy(op->graphKey, key, sizeof(key));
    op->graphLaunches = ctx->launches - before;
    ctx->launches = before;
  }
  for (int guard = 0; guard < (1 << 30); ++guard) {
    ITS_CU(ctx, cudaGraphLaunch(op->graph, ctx->stream));
    ctx->launches += op->graphLaunches;
    ITS_CU(ctx, cudaMemcpyAsync(op->hostDone, &sc.S->done, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if (*op->hostDone) break;
  }
  return ITS_OK;
}

static its_status readScalars(its_ctx* ctx, const SolveCtx& sc, CgScalars* h) {
  ITS_CU(ctx, cudaMemcpyAsync(h, sc.S, sizeof(CgScalars), cudaMemcpyDeviceToHost, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

// |b - A x|^2 into S->rr (uses w.t, w.d as scratch).
static its_status trueResidual(its_ctx* ctx, const SolveCtx& sc, const double* rhs, double* rOut) {
  its_status st;
  if ((st = spmv(ctx, sc.op->A64(), sc.op->planA, (const double*)sc.w.x, sc.w.t)) != ITS_OK) return st;
  return reduce(ctx, sc, OpInitResidual{rhs, sc.w.t, rOut}, 0);
}

its_status solve(its_op* op, const double* dB, double* dX, const its_solve_opts& o, its_solve_report* rep) {
  its_ctx* ctx = op->ctx;
  its_status st;
  if ((st = ensureWork(op)) != ITS_OK) return st;
  SolveCtx sc;
  sc.op = op;
  sc.w = workOf(op);
  sc.S = (CgScalars*)op->scalars;
  for (int k = 0; k < 6; ++k) sc.part[k] = op->partials + k * 2 * 4096;
  sc.redBlocks = (unsigned)std::min<int64_t>(4096, std::max<int64_t>(1, std::min<int64_t>((op->n + 255) / 256, ctx->numSMs * 4)));
  const int64_t n = op->n;
  const long long maxIters = o.max_iters > 0 ? o.max_iters : 2 * n;
  const int every = o.check_every > 0 ? o.check_every : 8;
  cudaEvent_t e0, e1;
  ITS_CU(ctx, cudaEventCreate(&e0));
  ITS_CU(ctx, cudaEventCreate(&e1));
  ITS_CU(ctx, cudaEventRecord(e0, ctx->stream));
  ITS_CU(ctx, cudaMemcpyAsync(sc.w.b, dB, n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  const bool hasX0 = o.x0 != nullptr;
  if (hasX0) ITS_CU(ctx, cudaMemcpyAsync(sc.w.x, o.x0, n * 8, cudaMemcpyDefault, ctx->stream));
  else ITS_CU(ctx, cudaMemsetAsync(sc.w.x, 0, n * 8, ctx->stream));
  CgScalars h{};
  *rep = its_solve_report{};
  if (o.precision == ITS_PREC_FP64) {
    kSetScalars<<<1, 1, 0, ctx->stream>>>(sc.S, o.tol, maxIters, o.stop_rule);
    ITS_LAUNCHED(ctx);
    if ((st = cglsInit(ctx, sc, sc.w.b, hasX0, false)) != ITS_OK) return st;
    kZeroIfEmptyRhs<<<sc.redBlocks, 256, 0, ctx->stream>>>(n, sc.w.x, sc.S);
    ITS_LAUNCHED(ctx);
    if ((st = readScalars(ctx, sc, &h)) != ITS_OK) return st;
    if (!h.done && (st = cglsRun(ctx, sc, false, every)) != ITS_OK) return st;
    if ((st = readScalars(ctx, sc, &h)) != ITS_OK) return st;
    rep->iterations = h.iter;
    rep->converged = h.converged;
    rep->breakdown = h.breakdown;
    rep->normal_rel_residual = h.rhsNorm2 > 0 ? std::sqrt(h.nrr / h.rhsNorm2) : 0.0;
  } else {
    // Iterative refinement: r = b - A x in FP64, correction d from FP32-SpMV CGLS on A d = r.
    const double innerTol = o.inner_tol > 0 ? o.inner_tol : 1e-3;
    const int steps = o.ir_steps > 0 ? o.ir_steps : 3;
    double bNorm2 = 0.0, rhsNorm2 = 0.0;
    DevBuf<double> rr(ctx), saveX(ctx);
    if ((st = rr.alloc(ctx, n)) != ITS_OK) return st;
    if ((st = saveX.alloc(ctx, n)) != ITS_OK) return st;
    int64_t inner = 0;
    bool conv = false;
    for (int s = 0; s < steps; ++s) {
      // outer residual in FP64
      kSetScalars<<<1, 1, 0, ctx->stream>>>(sc.S, o.tol, maxIters, o.stop_rule);
      ITS_LAUNCHED(ctx);
      if ((st = trueResidual(ctx, sc, sc.w.b, rr.p)) != ITS_OK) return st;
      if (s == 0) {  // ||A^T b||^2 once
        if ((st = spmv(ctx, op->T64(), op->planT, (const double*)sc.w.b, sc.w.d)) != ITS_OK) return st;
        if ((st = reduce(ctx, sc, OpRhsNorm{sc.w.d}, 0)) != ITS_OK) return st;
      }
      if (o.stop_rule == 0) {  // the normal-equation residual only where the stopping test uses it
        if ((st = spmv(ctx, op->T64(), op->planT, (const double*)rr.p, sc.w.nr)) != ITS_OK) return st;
        if ((st = reduce(ctx, sc, OpNormal{sc.w.nr, op->invdiag}, 0)) != ITS_OK) return st;
      }
      if ((st = readScalars(ctx, sc, &h)) != ITS_OK) return st;
      bNorm2 = h.bNorm2;
      if (s == 0) rhsNorm2 = h.rhsNorm2;
      const double m = o.stop_rule == 0 ? h.nrr / (rhsNorm2 > 0 ? rhsNorm2 : 1.0) : h.rr / (bNorm2 > 0 ? bNorm2 : 1.0);
      rep->normal_rel_residual = rhsNorm2 > 0 ? std::sqrt(h.nrr / rhsNorm2) : 0.0;
      if (bNorm2 == 0.0 || m < o.tol * o.tol) { conv = true; break; }
      // inner correction solve from zero on A d = rr
      ITS_CU(ctx, cudaMemcpyAsync(saveX.p, sc.w.x, n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      ITS_CU(ctx, cudaMemsetAsync(sc.w.x, 0, n * 8, ctx->stream));
      kSetScalars<<<1, 1, 0, ctx->stream>>>(sc.S, innerTol, maxIters, 1);
      ITS_LAUNCHED(ctx);
      if ((st = cglsInit(ctx, sc, rr.p, false, true)) != ITS_OK) return st;
      if ((st = readScalars(ctx, sc, &h)) != ITS_OK) return st;
      if (!h.done && (st = cglsRun(ctx, sc, true, every)) != ITS_OK) return st;
      if ((st = readScalars(ctx, sc, &h)) != ITS_OK) return st;
      inner += h.iter;
      rep->breakdown |= h.breakdown;
      kAxpy<<<sc.redBlocks, 256, 0, ctx->stream>>>(n, saveX.p, sc.w.x);
      ITS_LAUNCHED(ctx);
      ITS_CU(ctx, cudaMemcpyAsync(sc.w.x, saveX.p, n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    if (!conv || o.stop_rule != 0) {  // final check after the last correction; normal residual for the report
      if ((st = trueResidual(ctx, sc, sc.w.b, rr.p)) != ITS_OK) return st;
      if ((st = spmv(ctx, op->T64(), op->planT, (const double*)rr.p, sc.w.nr)) != ITS_OK) return st;
      if ((st = reduce(ctx, sc, OpNormal{sc.w.nr, op->invdiag}, 0)) != ITS_OK) return st;
      if ((st = readScalars(ctx, sc, &h)) != ITS_OK) return st;
      const double m = o.stop_rule == 0 ? h.nrr / (rhsNorm2 > 0 ? rhsNorm2 : 1.0) : h.rr / (bNorm2 > 0 ? bNorm2 : 1.0);
      if (!conv) conv = m < o.tol * o.tol;
      rep->normal_rel_residual = rhsNorm2 > 0 ? std::sqrt(h.nrr / rhsNorm2) : 0.0;
    }
    rep->iterations = inner;
    rep->inner_iterations = inner;
    rep->converged = conv ? 1 : 0;
  }
  // report the true residual of the returned x
  if ((st = trueResidual(ctx, sc, sc.w.b, sc.w.d)) != ITS_OK) return st;
  ITS_CU(ctx, cudaMemcpyAsync(dX, sc.w.x, n * 8, cudaMemcpyDefault, ctx->stream));
  ITS_CU(ctx, cudaEventRecord(e1, ctx->stream));
  if ((st = readScalars(ctx, sc, &h)) != ITS_OK) return st;
  rep->rel_residual = h.bNorm2 > 0 ? std::sqrt(h.rr / h.bNorm2) : 0.0;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  rep->ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ITS_OK;
}

void releaseSolver(its_op* op) {
  if (op->graph) {
    cudaGraphExecDestroy(op->graph);
    op->graph = nullptr;
  }
  devFree(op->ctx, op->work);
  devFree(op->ctx, op->workf);
  devFree(op->ctx, op->scalars);
  devFree(op->ctx, op->partials);
  op->work = nullptr;
  op->workf = nullptr;
  op->scalars = nullptr;
  op->partials = nullptr;
  op->hostDone = nullptr;
}

}  // namespace its

using namespace its;

extern "C" {

its_status its_solve_opts_default(its_solve_opts* o) {
  if (!o) return ITS_ERR_INVALID;
  o->tol = DBL_EPSILON;
  o->max_iters = 0;
  o->stop_rule = ITS_STOP_NORMAL;
  o->precision = ITS_PREC_FP64;
  o->ir_steps = 3;
  o->inner_tol = 1e-3;
  o->x0 = nullptr;
  o->check_every = 8;
  return ITS_OK;
}

its_status its_lscg_solve(its_op* op, const double* b, double* lambda, const its_solve_opts* opts,
                          its_solve_report* report) {
  if (!op || !b || !lambda) return ITS_ERR_INVALID;
  its_ctx* ctx = op->ctx;
  its_solve_opts o;
  its_solve_opts_default(&o);
  if (opts) o = *opts;
  if (!(o.tol > 0.0) || !std::isfinite(o.tol)) return setError(ctx, ITS_ERR_INVALID, "tol must be positive");
  if (o.stop_rule != ITS_STOP_NORMAL && o.stop_rule != ITS_STOP_RESIDUAL)
    return setError(ctx, ITS_ERR_INVALID, "unknown stop rule");
  if (o.precision != ITS_PREC_FP64 && o.precision != ITS_PREC_MIXED)
    return setError(ctx, ITS_ERR_INVALID, "unknown precision");
  if (o.precision == ITS_PREC_MIXED && !op->valf)
    return setError(ctx, ITS_ERR_STATE, "mixed precision needs an operator built with ITS_OP_FP32_VALUES");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> B;
  OutArg<double> X;
  its_status st;
  if ((st = B.stage(ctx, b, op->n)) != ITS_OK) return st;
  if ((st = X.stage(ctx, lambda, op->n)) != ITS_OK) return st;
  its_solve_report rep;
  if ((st = solve(op, B.d, X.d, o, &rep)) != ITS_OK) return st;
  if ((st = X.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  if (report) *report = rep;
  return ITS_OK;
}

}  // extern "C"
