// Solver state and the scalar steps of Eigen's CGLS shared by the single and the batched
// solve: per-step reductions fold their terms with a fixed order, and each finalize is one
// line of Eigen's least_square_conjugate_gradient loop.
#pragma once
#include "its_internal.cuh"

namespace its {

constexpr int kRedThreads = 256;

struct CgScalars {
  double absNew, alpha, beta, tn, rr, nrr, nrz, rhsNorm2, bNorm2, threshold, tol;
  long long iter, maxIters;
  int done, converged, breakdown, stopRule;
  unsigned tickets[8];
};

// Two block-wide sums in a fixed order.
__device__ inline void blockSum2(double& a, double& b) {
  __shared__ double sa[kRedThreads / 32], sb[kRedThreads / 32];
  a = warpSum(a);
  b = warpSum(b);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { sa[w] = a; sb[w] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0, tb = 0;
#pragma unroll
    for (int i = 0; i < kRedThreads / 32; ++i) { ta += sa[i]; tb += sb[i]; }
    a = ta;
    b = tb;
  }
  __syncthreads();
}

// Grid reduction with a last-block finalize. Op provides
//   __device__ void terms(int64_t i, double& a, double& b) const  (may also update vectors)
//   __device__ void finalize(CgScalars* S, double a, double b) const
//   int slot

struct OpInitResidual {  // r = b - t (t = A x0), or r = b
  const double* b;
  const double* t;
  double* r;
  int slot = 0;
  __device__ void terms(int64_t i, double& a, double& c) const {
    const double v = t ? b[i] - t[i] : b[i];
    r[i] = v;
    a += v * v;      // |r|^2
    c += b[i] * b[i];  // |b|^2
  }
  __device__ void finalize(CgScalars* S, double rr, double bb) const {
    S->rr = rr;
    S->bNorm2 = bb;
  }
};
struct OpRhsNorm {  // |A^T b|^2
  const double* atb;
  int slot = 1;
  __device__ void terms(int64_t i, double& a, double&) const { a += atb[i] * atb[i]; }
  __device__ void finalize(CgScalars* S, double v, double) const { S->rhsNorm2 = v; }
};
struct OpInitNormal {  // |n|^2, n.Dn, decide the zero-iteration exit, p = D n
  const double* nr;
  const double* invdiag;
  double* p;
  float* pf;
  int slot = 2;
  __device__ void terms(int64_t i, double& a, double& c) const {
    const double z = invdiag[i] * nr[i];
    p[i] = z;
    if (pf) pf[i] = (float)z;
    a += nr[i] * nr[i];
    c += nr[i] * z;
  }
  __device__ void finalize(CgScalars* S, double nrr, double nrz) const {
    S->nrr = nrr;
    S->nrz = nrz;
    S->iter = 0;
    S->breakdown = 0;
    if (S->rhsNorm2 == 0.0) {  // Eigen: x = 0, iterations 0
      S->done = 1;
      S->converged = 1;
      return;
    }
    S->threshold = S->stopRule == 0 ? S->tol * S->tol * S->rhsNorm2 : S->tol * S->tol * S->bNorm2;
    const double m = S->stopRule == 0 ? nrr : S->rr;
    if (m < S->threshold) {
      S->done = 1;
      S->converged = 1;
      return;
    }
    S->done = 0;
    S->converged = 0;
    S->absNew = nrz;
  }
};

// ---- iteration ---------------------------------------------------------------------------
struct OpTmpNorm {
  const double* t;
  int slot = 3;
  __device__ void terms(int64_t i, double& a, double&) const { a += t[i] * t[i]; }
  __device__ void finalize(CgScalars* S, double tn, double) const {
    S->tn = tn;
    if (!(tn > 0.0)) {
      S->breakdown = 1;
      S->done = 1;
      return;
    }
    S->alpha = S->absNew / tn;
  }
};
struct OpUpdateXR {
  const CgScalars* S;
  double* x;
  double* r;
  float* rf;
  const double* p;
  const double* t;
  int slot = 4;
  __device__ void terms(int64_t i, double& a, double&) const {
    const double al = S->alpha;
    x[i] += al * p[i];
    const double v = r[i] - al * t[i];
    r[i] = v;
    if (rf) rf[i] = (float)v;
    a += v * v;
  }
  __device__ void finalize(CgScalars* Sm, double rr, double) const { Sm->rr = rr; }
};
struct OpNormal {
  const double* nr;
  const double* invdiag;
  int slot = 5;
  __device__ void terms(int64_t i, double& a, double& c) const {
    const double z = invdiag[i] * nr[i];
    a += nr[i] * nr[i];
    c += nr[i] * z;
  }
  __device__ void finalize(CgScalars* S, double nrr, double nrz) const {
    S->nrr = nrr;
    const double m = S->stopRule == 0 ? nrr : S->rr;
    if (m < S->threshold) {
      S->done = 1;
      S->converged = 1;
      return;
    }
    const double absOld = S->absNew;
    S->absNew = nrz;
    S->beta = nrz / absOld;
    S->iter += 1;
    if (S->iter >= S->maxIters) S->done = 1;
  }
};

}  // namespace its
