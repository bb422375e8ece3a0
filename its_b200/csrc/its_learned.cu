// The learned fit as one call: learned start, FP64 residual check, plain LSCG fallback.
//
// ThinShells::creatShell (ThinShells.cpp:608-653) assembles the operator and runs Eigen's
// LSCG from zero. Here the fit is the learned start (zero-share start, features, share
// network, exact start with the predicted shares), checked by the matrix-free residual
// ||b - A lambda|| / ||b||; when that misses tol, the plain FP64 LSCG continues from it.
//
// The start and the check are a fixed sequence of about a dozen short launches per octree,
// so their launch and host costs rival the kernels. The sequence is captured once into a CUDA
// graph per octree (its "plan") and replayed while the octree, the network, the vectors'
// device addresses and the normalisation stay the same; any change captures a new one. The
// graph reads the inputs' memory at every replay, so new values of b (or of the network's
// parameters) are always used. Scratch buffers of the captured sequence live in an arena the
// plan owns (the graph holds no allocation nodes); host vectors are staged through plan-owned
// device buffers around the replay. The residual's last kernel writes its result, and the
// network's error flag beside it, straight to the plan's mapped pinned memory.
#include <cstring>
#include <vector>

#include "its_op.cuh"
#include "its_svo.cuh"

struct its_mlp;

namespace its {

its_status learnedStart(its_ctx* ctx, its_svo* const* svos, int64_t count, its_mlp* mlp, const double* const* b,
                        const float* hn, double* const* lam, unsigned long long* stamp);
its_status fitResidualEnqueue(its_ctx* ctx, its_svo* const* svos, int64_t count, const double* const* b,
                              const double* const* lam, double* relDev, const int* flagSrc, int* flagDst,
                              bool afterKernel, unsigned long long* stampEnd);
its_status hostNorm(its_ctx* ctx, const float* norm, float* hn);
const int* mlpErrFlag(its_mlp* mlp);
uint64_t mlpUid(const its_mlp* mlp);

constexpr int kNormValues = 130;

struct LearnedPlan {
  its_ctx* ctx = nullptr;
  // what the graph was captured for
  its_mlp* mlp = nullptr;
  uint64_t mlpUid = 0;  // the network's identity (its address may be reused after a free)
  const double* b = nullptr;
  double* lam = nullptr;
  const double* bHost = nullptr;  // pinned host vectors copied inside the graph (or null)
  double* lamHost = nullptr;
  cudaStream_t stream = nullptr;
  float norm[kNormValues];
  cudaGraphExec_t exec = nullptr;
  int64_t launches = 0;     // kernels per replay
  // owned memory
  uint8_t* arena = nullptr; // scratch of the captured sequence
  size_t arenaCap = 0;
  double* relHost = nullptr;  // pinned: the residual (written by the residual's last kernel
                              // through the mapped address), then the network's error flag
  double* relMapped = nullptr;  // relHost's device address

  cudaStream_t side = nullptr;  // the copy of lambda to pinned host memory, beside the residual
  cudaEvent_t fork = nullptr, join = nullptr;
  double* bStage = nullptr;   // device copies of host vectors
  double* lamStage = nullptr;
  int mapSlot = -1;            // relHost's slot in the context's mapped slab (-1: its own allocation)
  // the kinds of the last call's norm, b and lambda addresses (the graph is reused only for
  // the same addresses, so the kinds are looked up again only when an address changes)
  const void* kindOf[3] = {nullptr, nullptr, nullptr};
  PtrClass kind[3] = {PtrClass::Pageable, PtrClass::Pageable, PtrClass::Pageable};
};

static void dropGraph(LearnedPlan* p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  p->exec = nullptr;
}

void destroyPlan(LearnedPlan* p) {
  if (!p) return;
  cudaStreamSynchronize(p->ctx->stream);
  dropGraph(p);

  if (p->fork) cudaEventDestroy(p->fork);
  if (p->join) cudaEventDestroy(p->join);
  if (p->side) cudaStreamDestroy(p->side);
  devFree(p->ctx, p->arena);
  devFree(p->ctx, p->bStage);
  devFree(p->ctx, p->lamStage);
  if (p->mapSlot >= 0) p->ctx->mapUsed &= ~(1ull << p->mapSlot);
  else if (p->relHost) cudaFreeHost(p->relHost);
  delete p;
}

static its_status planFor(its_svo* svo, LearnedPlan** out) {
  its_ctx* ctx = svo->ctx;
  if (!svo->plan) {
    LearnedPlan* p = new LearnedPlan;
    p->ctx = ctx;
    const int64_t n = svo->d.numVerts, c = svo->d.numCoinc;
    // the captured sequence's buffers: zero-share start, shares, G, H (8 B per vertex each),
    // features and predictions (260 B per coincident vertex), chunk sums, 256-byte alignment
    p->arenaCap = (size_t)(40 * n + 264 * c + 16 * (n / 256 + 64) + (1 << 16));
    // from the context's stream-ordered pool (a plan per octree: cudaMalloc's device-wide
    // synchronisation and its cost on a busy device stay out of the fit's first call)
    its_status st = devAlloc(ctx, (void**)&p->arena, p->arenaCap);
    if (st != ITS_OK) {
      delete p;
      return st;
    }
    cudaError_t e = cudaSuccess;
    if (!ctx->mapSlab) e = cudaHostAlloc((void**)&ctx->mapSlab, 64 * 64, cudaHostAllocMapped);
    if (e == cudaSuccess && ctx->mapUsed != ~0ull) {  // a free 64-byte slot of the mapped slab
      const int slot = __builtin_ctzll(~ctx->mapUsed);
      ctx->mapUsed |= 1ull << slot;
      p->mapSlot = slot;
      p->relHost = ctx->mapSlab + 8 * slot;
    } else if (e == cudaSuccess) {
      e = cudaHostAlloc(&p->relHost, 64, cudaHostAllocMapped);
    }
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&p->relMapped, p->relHost, 0);

    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      cudaGetLastError();
      destroyPlan(p);
      return setError(ctx, ITS_ERR_OOM, "learned fit: plan buffers");
    }
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));  // the pool memory usable from any stream
    svo->plan = p;
  }
  *out = svo->plan;
  return ITS_OK;
}

// Queue the learned start and the residual check of one octree (device vectors), with the
// copies of pinned host vectors when given: b in first, lambda out on the side stream while
// the residual runs (the residual's last kernel also copies the network's error flag beside
// its result).
static its_status enqueueFit(its_svo* svo, LearnedPlan* p, its_mlp* mlp, const double* b, const float* hn, double* lam,
                             const double* bHost, double* lamHost) {
  its_ctx* ctx = svo->ctx;
  const int64_t n = svo->d.numVerts;
  its_status st;
  if (bHost) ITS_CU(ctx, cudaMemcpyAsync(const_cast<double*>(b), bHost, n * 8, cudaMemcpyHostToDevice, ctx->stream));
  // the plan's mapped words: residual, the network's error flag, first-kernel and last-kernel clocks
  unsigned long long* stamps = (unsigned long long*)(p->relMapped + 2);
  if ((st = learnedStart(ctx, &svo, 1, mlp, &b, hn, &lam, stamps)) != ITS_OK) return st;
  if (lamHost) {
    ITS_CU(ctx, cudaEventRecord(p->fork, ctx->stream));
    ITS_CU(ctx, cudaStreamWaitEvent(p->side, p->fork, 0));
    ITS_CU(ctx, cudaMemcpyAsync(lamHost, lam, n * 8, cudaMemcpyDeviceToHost, p->side));
    ITS_CU(ctx, cudaEventRecord(p->join, p->side));
  }
  // the residual follows the start's last kernel directly unless lambda's copy forks off first
  if ((st = fitResidualEnqueue(ctx, &svo, 1, &b, &lam, p->relMapped, mlpErrFlag(mlp), (int*)(p->relMapped + 1),
                               lamHost == nullptr, stamps + 1)) != ITS_OK)
    return st;
  if (lamHost) ITS_CU(ctx, cudaStreamWaitEvent(ctx->stream, p->join, 0));
  return ITS_OK;
}

// Capture the sequence for (mlp, b, lam, norm, pinned host vectors) into p->exec.
static its_status capture(its_svo* svo, LearnedPlan* p, its_mlp* mlp, const double* b, const float* hn, double* lam,
                          const double* bHost, double* lamHost) {
  its_ctx* ctx = svo->ctx;
  dropGraph(p);
  its_status st = ITS_OK;
  if (ctx->autotune) {  // a capture cannot time: the start's tunable launches are measured first
    if (bHost) ITS_CU(ctx, cudaMemcpyAsync(const_cast<double*>(b), bHost, svo->d.numVerts * 8, cudaMemcpyHostToDevice,
                                           ctx->stream));
    if ((st = learnedStart(ctx, &svo, 1, mlp, &b, hn, &lam, nullptr)) != ITS_OK) return st;
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  }
  const int64_t launches0 = ctx->launches;
  ctx->arena = p->arena;
  ctx->arenaCap = p->arenaCap;
  ctx->arenaOff = 0;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    st = enqueueFit(svo, p, mlp, b, hn, lam, bHost, lamHost);
    const cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &graph);
    if (e == cudaSuccess) e = e2;
  }
  ctx->arena = nullptr;
  ctx->arenaCap = ctx->arenaOff = 0;
  p->launches = ctx->launches - launches0;
  ctx->launches = launches0;  // nothing ran yet
  if (st == ITS_OK && e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (st != ITS_OK) return st;
  if (e != cudaSuccess) {
    cudaGetLastError();
    p->exec = nullptr;
    return cudaFail(ctx, e, "learned fit: graph capture");
  }
  p->mlp = mlp;
  p->mlpUid = mlpUid(mlp);
  p->b = b;
  p->lam = lam;
  p->bHost = bHost;
  p->lamHost = lamHost;
  p->stream = ctx->stream;
  std::memcpy(p->norm, hn, sizeof(p->norm));
  return ITS_OK;
}

}  // namespace its

using namespace its;

extern "C" {

its_status its_learned_fit(its_svo* svo, its_mlp* mlp, const double* b, const float* norm, double tol,
                           double* lambda, its_solve_report* report) {
  if (!svo || !mlp || !b || !norm || !lambda) return ITS_ERR_INVALID;
  its_ctx* ctx = svo->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  its_status st;
  LearnedPlan* p = nullptr;
  if ((st = planFor(svo, &p)) != ITS_OK) return st;
  if (report) std::memset(report, 0, sizeof(*report));
  const void* addr[3] = {norm, b, lambda};
  for (int k = 0; k < 3; ++k)
    if (p->kindOf[k] != addr[k]) {
      p->kind[k] = ptrClass(addr[k], ctx->device);
      p->kindOf[k] = addr[k];
    }
  const PtrClass cn = p->kind[0], cb = p->kind[1], cl = p->kind[2];
  if (cn == PtrClass::OtherDevice || cb == PtrClass::OtherDevice || cl == PtrClass::OtherDevice) {
    p->kindOf[0] = p->kindOf[1] = p->kindOf[2] = nullptr;
    return otherDeviceError(ctx);
  }
  float hn[kNormValues];
  if (cn == PtrClass::Device) {
    ITS_CU(ctx, cudaMemcpyAsync(hn, norm, sizeof(hn), cudaMemcpyDeviceToHost, ctx->stream));
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  } else {
    std::memcpy(hn, norm, sizeof(hn));
  }
  const int64_t n = svo->d.numVerts;
  // device addresses of the vectors: the caller's, or the plan's copies of host vectors
  const bool bHost = cb != PtrClass::Device, lamHost = cl != PtrClass::Device;
  if ((bHost && !p->bStage && (st = devAlloc(ctx, (void**)&p->bStage, std::max<int64_t>(n, 1) * 8)) != ITS_OK) ||
      (lamHost && !p->lamStage && (st = devAlloc(ctx, (void**)&p->lamStage, std::max<int64_t>(n, 1) * 8)) != ITS_OK))
    return st;
  const double* bd = bHost ? p->bStage : b;
  double* ld = lamHost ? p->lamStage : lambda;
  // page-locked host vectors are copied by the graph itself (lambda beside the residual);
  // pageable ones around it
  const double* bPin = cb == PtrClass::Pinned ? b : nullptr;
  double* lamPin = cl == PtrClass::Pinned ? lambda : nullptr;
  if (bHost && !bPin) ITS_CU(ctx, cudaMemcpyAsync(p->bStage, b, n * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (!p->exec || p->mlp != mlp || p->mlpUid != mlpUid(mlp) || p->b != bd || p->lam != ld || p->bHost != bPin ||
      p->lamHost != lamPin || p->stream != ctx->stream || std::memcmp(p->norm, hn, sizeof(hn)) != 0)
    if ((st = capture(svo, p, mlp, bd, hn, ld, bPin, lamPin)) != ITS_OK) return st;
  ITS_CU(ctx, cudaGraphLaunch(p->exec, ctx->stream));
  ctx->launches += p->launches;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  // device time of the start and the check: from the first kernel's start to the residual's end
  // (the device clock, written by those kernels to the plan's mapped words)
  const unsigned long long* stamps = (const unsigned long long*)(p->relHost + 2);
  double ms = stamps[1] > stamps[0] ? (double)(stamps[1] - stamps[0]) * 1e-6 : 0.0;
  int netErr = 0;
  std::memcpy(&netErr, p->relHost + 1, sizeof(int));
  if (netErr) return setError(ctx, ITS_ERR_TIMEOUT, "share network: a tensor-core wait ran out");
  double rel = *p->relHost;
  int64_t iters = 0;
  int converged = rel <= tol;
  const bool fellBack = !converged;
  if (fellBack) {  // the plain FP64 LSCG from the learned start
    its_op* op = nullptr;
    if ((st = its_operator_build(svo, 0, &op)) != ITS_OK) return st;
    its_solve_opts o;
    its_solve_opts_default(&o);
    o.tol = tol;
    o.stop_rule = ITS_STOP_RESIDUAL;
    o.x0 = ld;
    its_solve_report r;
    st = its_lscg_solve(op, bd, ld, &o, &r);
    its_operator_free(op);
    if (st != ITS_OK) return st;
    rel = r.rel_residual;
    iters = r.iterations;
    converged = r.converged;
    ms += r.ms;
  }
  if (lamHost && (!lamPin || fellBack)) {  // not copied by the graph, or changed since
    ITS_CU(ctx, cudaMemcpyAsync(lambda, ld, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  }
  if (report) {
    report->iterations = iters;
    report->converged = converged;
    report->rel_residual = rel;
    report->ms = ms;
  }
  return ITS_OK;
}

}  // extern "C"
