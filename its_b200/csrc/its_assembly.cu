// Operator assembly (replaces ThinShells::cpCoefficients' triplet build and
// SparseMatrix::setFromTriplets, ThinShells.cpp:511-606, and setInDomainPoints,
// SVO.cu:1160-1193).
//
// Rows are generated by walkRow (its_rows.cuh): chain < diagonal < ancestors, so every row
// comes out sorted. Two passes (count, fill) with an exclusive scan in between. The
// transpose is a stable radix sort of the entries by column.
#include <cmath>

#include "its_cubic.cuh"
#include "its_op.cuh"
#include "its_rows.cuh"

namespace its {

// Rows of the reference's hat-basis system (walkRow).
struct HatGen {
  RowParams P;
  template <typename E>
  __device__ void operator()(int64_t r, E emit) const { walkRow(P, r, emit); }
};

template <bool FILL, typename Gen>
__global__ void kAssembleRows(const __grid_constant__ Gen gen, int64_t n, int64_t* __restrict__ rowptrOrCount,
                              int32_t* __restrict__ col, double* __restrict__ val, uint32_t* __restrict__ rowIdx) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  int64_t k = FILL ? rowptrOrCount[r] : 0;
  gen(r, [&](int32_t c, double v) {
    if (FILL) {
      col[k] = c;
      val[k] = v;
      rowIdx[k] = (uint32_t)r;
    }
    ++k;
  });
  if (!FILL) rowptrOrCount[r] = k;
}

// Row pointers of A^T from the column-sorted keys: entry i opens every column in
// (key[i-1], key[i]]; the end sentinel closes the rest. Each pointer is written once, no
// atomics (a column count by atomicAdd would pile up on the few coarse corners that touch
// almost every row).
__global__ void kRowptrFromSorted(int64_t nnz, const uint32_t* __restrict__ keys, int64_t n,
                                  int64_t* __restrict__ rowptr) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i > nnz) return;
  const int64_t c = (i < nnz) ? (int64_t)keys[i] : n;
  const int64_t prev = (i == 0) ? -1 : (int64_t)keys[i - 1];
  for (int64_t k = prev + 1; k <= c; ++k) rowptr[k] = i;
}
__global__ void kGatherTranspose(int64_t nnz, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ rowIdx,
                                 const double* __restrict__ val, int32_t* __restrict__ tcol, double* __restrict__ tval) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nnz) return;
  const uint32_t k = perm[i];
  tcol[i] = (int32_t)rowIdx[k];
  tval[i] = val[k];
}
__global__ void kSquare(int64_t n, const double* __restrict__ a, double* __restrict__ b) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i] * a[i];
}
__global__ void kFill(int64_t n, double v, double* __restrict__ a) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}
__global__ void kInvDiag(int64_t n, double* __restrict__ d) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) d[i] = d[i] > 0.0 ? 1.0 / d[i] : 1.0;
}
__global__ void kToFloat(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

static void opRelease(its_op* op) {
  if (!op) return;
  its_ctx* c = op->ctx;
  releaseSolver(op);
  void* ptrs[] = {op->rowptr, op->col, op->val, op->trowptr, op->tcol, op->tval, op->valf, op->tvalf, op->invdiag};
  for (void* p : ptrs) devFree(c, p);
  releasePlan(c, &op->planA);
  releasePlan(c, &op->planT);
}

// Assembles the n x n system whose rows gen generates (columns < n; a system with more rows
// than unknowns is stored square, its columns past the unknowns empty).
template <typename Gen>
static its_status opBuild(its_op* op, int64_t n, const Gen& P) {
  its_ctx* ctx = op->ctx;
  op->n = n;
  its_status st;
  if ((st = devAlloc(ctx, (void**)&op->rowptr, (n + 1) * 8)) != ITS_OK) return st;
  kAssembleRows<false, Gen><<<gridFor(n, 128), 128, 0, ctx->stream>>>(P, n, op->rowptr, nullptr, nullptr, nullptr);
  ITS_LAUNCHED(ctx);
  DevBuf<int64_t> tot;
  if ((st = tot.alloc(ctx, 1)) != ITS_OK) return st;
  {
    int64_t* rp = op->rowptr;
    auto f = [rp] __device__(int64_t i) -> int64_t { return rp[i]; };
    if ((st = scanExclusiveAlloc<int64_t>(ctx, f, n, StorePrefix<int64_t>{rp}, tot.p)) != ITS_OK) return st;
    ITS_CU(ctx, cudaMemcpyAsync(rp + n, tot.p, 8, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  int64_t nnz = 0;
  if ((st = readScalar(ctx, tot.p, &nnz)) != ITS_OK) return st;
  if (nnz >= (1ll << 32)) return setError(ctx, ITS_ERR_INVALID, "operator has more than 2^32 entries");
  op->nnz = nnz;
  if ((st = devAlloc(ctx, (void**)&op->col, nnz * 4)) != ITS_OK) return st;
  if ((st = devAlloc(ctx, (void**)&op->val, nnz * 8)) != ITS_OK) return st;
  DevBuf<uint32_t> rowIdx;
  if ((st = rowIdx.alloc(ctx, nnz)) != ITS_OK) return st;
  kAssembleRows<true, Gen><<<gridFor(n, 128), 128, 0, ctx->stream>>>(P, n, op->rowptr, op->col, op->val, rowIdx.p);
  ITS_LAUNCHED(ctx);

  // transpose: stable sort of the entries by column keeps rows ascending within a column
  {
    DevBuf<uint32_t> iota, sk, sv, tk, tv;
    if ((st = iota.alloc(ctx, nnz)) != ITS_OK) return st;
    if ((st = sk.alloc(ctx, nnz)) != ITS_OK) return st;
    if ((st = sv.alloc(ctx, nnz)) != ITS_OK) return st;
    if ((st = tk.alloc(ctx, nnz)) != ITS_OK) return st;
    if ((st = tv.alloc(ctx, nnz)) != ITS_OK) return st;
    uint32_t* ip = iota.p;
    auto one = [] __device__(int64_t) -> uint32_t { return 1u; };
    if ((st = scanExclusiveAlloc<uint32_t>(ctx, one, nnz, StorePrefix<uint32_t>{ip}, (uint32_t*)nullptr)) != ITS_OK) return st;
    int bits = 1;
    while (bits < 32 && (1ll << bits) < n) ++bits;
    if ((st = radixSortPairs(ctx, (const uint32_t*)op->col, iota.p, sk.p, sv.p, tk.p, tv.p, nnz, bits)) != ITS_OK)
      return st;
    if ((st = devAlloc(ctx, (void**)&op->tcol, nnz * 4)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&op->tval, nnz * 8)) != ITS_OK) return st;
    kGatherTranspose<<<gridFor(nnz, 256), 256, 0, ctx->stream>>>(nnz, sv.p, rowIdx.p, op->val, op->tcol, op->tval);
    ITS_LAUNCHED(ctx);
    if ((st = devAlloc(ctx, (void**)&op->trowptr, (n + 1) * 8)) != ITS_OK) return st;
    kRowptrFromSorted<<<gridFor(nnz + 1, 256), 256, 0, ctx->stream>>>(nnz, sk.p, n, op->trowptr);
    ITS_LAUNCHED(ctx);
  }
  rowIdx.reset();
  if ((st = buildSpmvPlan(ctx, n, op->rowptr, &op->planA)) != ITS_OK) return st;
  if ((st = buildSpmvPlan(ctx, n, op->trowptr, &op->planT)) != ITS_OK) return st;

  // Jacobi column scaling of Eigen's LeastSquareDiagonalPreconditioner
  {
    DevBuf<double> sq, ones;
    if ((st = sq.alloc(ctx, nnz)) != ITS_OK) return st;
    if ((st = ones.alloc(ctx, n)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&op->invdiag, n * 8)) != ITS_OK) return st;
    kSquare<<<gridFor(nnz, 256), 256, 0, ctx->stream>>>(nnz, op->tval, sq.p);
    ITS_LAUNCHED(ctx);
    kFill<<<gridFor(n, 256), 256, 0, ctx->stream>>>(n, 1.0, ones.p);
    ITS_LAUNCHED(ctx);
    CsrView<double, double> S{n, op->trowptr, op->tcol, sq.p};
    if ((st = spmv(ctx, S, op->planT, (const double*)ones.p, op->invdiag)) != ITS_OK) return st;
    kInvDiag<<<gridFor(n, 256), 256, 0, ctx->stream>>>(n, op->invdiag);
    ITS_LAUNCHED(ctx);
  }
  if (op->mode == ITS_OP_FP32_VALUES) {
    if ((st = devAlloc(ctx, (void**)&op->valf, nnz * 4)) != ITS_OK) return st;
    if ((st = devAlloc(ctx, (void**)&op->tvalf, nnz * 4)) != ITS_OK) return st;
    kToFloat<<<gridFor(nnz, 256), 256, 0, ctx->stream>>>(nnz, op->val, op->valf);
    ITS_LAUNCHED(ctx);
    kToFloat<<<gridFor(nnz, 256), 256, 0, ctx->stream>>>(nnz, op->tval, op->tvalf);
    ITS_LAUNCHED(ctx);
  }
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // namespace its

using namespace its;

extern "C" {

its_status its_operator_build(its_svo* svo, int mode, its_op** out) {
  if (!svo || !out) return ITS_ERR_INVALID;
  *out = nullptr;
  its_ctx* ctx = svo->ctx;
  if (mode != ITS_OP_FP64 && mode != ITS_OP_FP32_VALUES) return setError(ctx, ITS_ERR_INVALID, "unknown operator mode");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  its_op* op = new its_op;
  op->ctx = ctx;
  op->svo = svo;
  op->mode = mode;
  op->unknowns = svo->d.numVerts;
  its_status st = opBuild(op, svo->d.numVerts, HatGen{rowParams(svo->d)});
  if (st != ITS_OK) {
    opRelease(op);
    cudaStreamSynchronize(ctx->stream);
    delete op;
    return st;
  }
  *out = op;
  return ITS_OK;
}

its_status its_operator_build_ex(its_svo* svo, int mode, const its_basis_opts* opts, its_op** out) {
  if (!svo || !out) return ITS_ERR_INVALID;
  *out = nullptr;
  its_ctx* ctx = svo->ctx;
  const int degree = opts ? opts->degree : 1;
  const int64_t m = opts ? opts->num_samples : 0;
  if (mode != ITS_OP_FP64 && mode != ITS_OP_FP32_VALUES) return setError(ctx, ITS_ERR_INVALID, "unknown operator mode");
  if (degree != 1 && degree != 3) return setError(ctx, ITS_ERR_INVALID, "basis degree must be 1 or 3");
  if (m < 0 || (m > 0 && !opts->samples)) return setError(ctx, ITS_ERR_INVALID, "bad extra samples");
  if (degree == 1 && m > 0)
    return setError(ctx, ITS_ERR_INVALID, "extra sample rows need the cubic basis (degree 3)");
  if (degree == 1) return its_operator_build(svo, mode, out);
  if (svo->d.numVerts + m >= (1ll << 31)) return setError(ctx, ITS_ERR_INVALID, "too many rows");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<double> S;
  its_status st;
  if ((st = S.stage(ctx, m > 0 ? opts->samples : nullptr, 3 * m)) != ITS_OK) return st;
  its_op* op = new its_op;
  op->ctx = ctx;
  op->svo = svo;
  op->mode = mode;
  op->degree = 3;
  op->unknowns = svo->d.numVerts;
  st = opBuild(op, svo->d.numVerts + m, cubicGen(svo->d, S.d));
  if (st != ITS_OK) {
    opRelease(op);
    cudaStreamSynchronize(ctx->stream);
    delete op;
    return st;
  }
  *out = op;
  return ITS_OK;
}

its_status its_operator_free(its_op* op) {
  if (!op) return ITS_OK;
  its_ctx* c = op->ctx;
  opRelease(op);
  cudaStreamSynchronize(c->stream);
  delete op;
  return ITS_OK;
}

its_status its_operator_info(const its_op* op, int64_t* rows, int64_t* nnz) {
  if (!op) return ITS_ERR_INVALID;
  if (rows) *rows = op->n;
  if (nnz) *nnz = op->nnz;
  return ITS_OK;
}

its_status its_operator_get_csr(its_op* op, int64_t* rowptr, int32_t* col, double* val) {
  if (!op) return ITS_ERR_INVALID;
  its_ctx* ctx = op->ctx;
  if (rowptr) ITS_CU(ctx, cudaMemcpyAsync(rowptr, op->rowptr, (op->n + 1) * 8, cudaMemcpyDefault, ctx->stream));
  if (col) ITS_CU(ctx, cudaMemcpyAsync(col, op->col, op->nnz * 4, cudaMemcpyDefault, ctx->stream));
  if (val) ITS_CU(ctx, cudaMemcpyAsync(val, op->val, op->nnz * 8, cudaMemcpyDefault, ctx->stream));
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

its_status its_operator_apply(its_op* op, const double* x, double* y, int transpose) {
  if (!op || !x || !y) return ITS_ERR_INVALID;
  its_ctx* ctx = op->ctx;
  InArg<double> X;
  OutArg<double> Y;
  its_status st;
  if ((st = X.stage(ctx, x, op->n)) != ITS_OK) return st;
  if ((st = Y.stage(ctx, y, op->n)) != ITS_OK) return st;
  if (transpose) st = spmv(ctx, op->T64(), op->planT, X.d, Y.d);
  else st = spmv(ctx, op->A64(), op->planA, X.d, Y.d);
  if (st != ITS_OK) return st;
  if ((st = Y.finish(ctx)) != ITS_OK) return st;
  // Device-to-device applies stay asynchronous on the context stream.
  if (Y.host || X.tmp.p) ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // extern "C"
