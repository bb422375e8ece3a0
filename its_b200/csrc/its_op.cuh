// Operator object: the assembled basis matrix A (CSR, ascending columns), its transpose,
// FP32 value copies for the mixed-precision solver, the Jacobi column scaling and the
// solver workspace.
#pragma once
#include "its_sparse.cuh"
#include "its_svo.cuh"

struct its_op {
  its_ctx* ctx = nullptr;
  its_svo* svo = nullptr;
  int mode = 0;
  int degree = 1;          // basis degree: 1 (the reference's hats) or 3 (cubic B-splines)
  int64_t n = 0, nnz = 0;  // rows (= stored columns: a system with extra sample rows is square-padded)
  int64_t unknowns = 0;    // columns that are corner vertices (the rest are empty padding)
  int64_t* rowptr = nullptr;
  int32_t* col = nullptr;
  double* val = nullptr;
  int64_t* trowptr = nullptr;
  int32_t* tcol = nullptr;
  double* tval = nullptr;
  float* valf = nullptr;
  float* tvalf = nullptr;
  double* invdiag = nullptr;  // 1 / ||A(:,j)||^2 (1 for empty columns)
  its::SpmvPlan planA, planT;
  // solver workspace, allocated on first solve
  double* work = nullptr;
  float* workf = nullptr;
  void* scalars = nullptr;
  double* partials = nullptr;
  int* hostDone = nullptr;  // the context's pinned scratch
  cudaGraphExec_t graph = nullptr;
  int64_t graphLaunches = 0;  // kernels per graph launch
  int graphKey[4] = {-1, -1, -1, -1};

  its::CsrView<double, double> A64() const { return {n, rowptr, col, val}; }
  its::CsrView<double, double> T64() const { return {n, trowptr, tcol, tval}; }
  its::CsrView<float, float> A32() const { return {n, rowptr, col, valf}; }
  its::CsrView<float, float> T32() const { return {n, trowptr, tcol, tvalf}; }
};

namespace its {
void releaseSolver(its_op* op);
}
