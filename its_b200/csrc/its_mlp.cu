// Share network: a small MLP that predicts, for every corner vertex coincident with a
// coarser corner, its coefficient in the minimum-norm solution of the shell system (the
// solution Eigen's CGLS reaches from zero). Those coefficients are exactly the free "shares"
// of the exact start, so a good prediction puts the exact solution close to the reference's.
//
// Network: 64 features -> 128 GELU -> 128 GELU -> 128 GELU -> 1, BF16 weights and
// activations, FP32 accumulation; FP32 master weights trained with Adam on a mean squared
// error. Every layer product is one tcgen05 GEMM (kUmmaGemm): 128 rows per CTA, operands
// staged in shared memory in the 128-byte-swizzled K-major layout, the accumulator in TMEM,
// the epilogue (bias, GELU, output dot product, loss gradient, GELU derivative) fused and
// read back with tcgen05.ld. Weight gradients are split-K GEMMs over the batch whose
// partials are summed in a fixed order, so a training step is deterministic.
//
// Parameters (flat FP32): W1[128x64] b1[128] W2[128x128] b2[128] W3[128x128] b3[128]
// w4[128] b4[1] (W[o][i]: output o, input i).
#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>

#include "its_ctx.cuh"
#include "its_umma.cuh"

namespace its {

constexpr int kIn = 64, kHid = 128;
constexpr int64_t kOffW1 = 0, kOffB1 = kOffW1 + kHid * kIn, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
                  kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kHid, kOffW4 = kOffB3 + kHid,
                  kOffB4 = kOffW4 + kHid, kNumParams = kOffB4 + 1;
constexpr int kSplitK = 128;  // weight-gradient partial sums per layer

using bf16 = __nv_bfloat16;

// GELU in its tanh form (Hendrycks & Gimpel, "Gaussian Error Linear Units", 2016):
//   gelu(z) = z/2 (1 + tanh(u)),  u = sqrt(2/pi) (z + 0.044715 z^3),
// with the tanh from the hardware's approximate unit: a handful of instructions where the
// erf form costs a few dozen, in the epilogues that bound the network's kernels.
constexpr float kGeluK0 = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluK1 = 0.044715f;
__device__ __forceinline__ float tanhApprox(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float geluF(float z) {
  const float u = z * fmaf(kGeluK0 * kGeluK1, z * z, kGeluK0);
  const float h = 0.5f * z;
  return fmaf(h, tanhApprox(u), h);
}
// Two lanes of geluF with the packed FP32 instructions (each lane one IEEE FP32 operation of
// geluF's, in geluF's order: the same bits at half the instructions).
__device__ __forceinline__ float2 geluF2(float2 z) {
  const float2 p = __ffma2_rn(make_float2(kGeluK0 * kGeluK1, kGeluK0 * kGeluK1), __fmul2_rn(z, z),
                              make_float2(kGeluK0, kGeluK0));
  const float2 u = __fmul2_rn(z, p);
  const float2 h = __fmul2_rn(make_float2(0.5f, 0.5f), z);
  return __ffma2_rn(h, make_float2(tanhApprox(u.x), tanhApprox(u.y)), h);
}
// d gelu / dz = (1 + t)/2 + z/2 (1 - t^2) sqrt(2/pi) (1 + 3 * 0.044715 z^2), t = tanh(u)
__device__ __forceinline__ float geluGrad(float z) {
  const float z2 = z * z;
  const float t = tanhApprox(z * fmaf(kGeluK0 * kGeluK1, z2, kGeluK0));
  const float du = fmaf(3.0f * kGeluK0 * kGeluK1, z2, kGeluK0);
  return fmaf(0.5f * z * du, fmaf(-t, t, 1.0f), 0.5f * (1.0f + t));
}

// ---- one tcgen05 GEMM: C[m][n] = sum_k A[m][k] B[n][k] over this CTA's K range -------------
// 128 rows per CTA and four warp groups: 64-wide K chunks are fetched by all 512 threads with
// cp.async into one of two stages while the tensor core multiplies the other; the accumulator
// (TMEM) is read back by each warp group for a quarter of the columns (thread = row, the TMEM
// lane of its warp) and handed to the epilogue functor with that quarter.
constexpr int kGemmGroups = 4;
constexpr int kGemmThreads = 128 * kGemmGroups;
template <int N>
struct GemmSmem {
  static constexpr int kA = 128 * 128, kB = N * 128, kStage = kA + kB;
  // two stages, the epilogue's per-group row partials and per-row value, mbarriers, TMEM slot
  static constexpr int kBytes = 2 * kStage + (kGemmGroups + 1) * 128 * 4 + 64 + 1024;
};

// 16 bytes global -> shared without staging through registers; bytes < 16 zero-fills the rest.
__device__ __forceinline__ void cpAsync16(uint32_t dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int Pending>
__device__ __forceinline__ void cpAsyncWait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(Pending) : "memory");
}

template <int N, class Epi>
__global__ void __launch_bounds__(kGemmThreads, 2) kUmmaGemm(const bf16* __restrict__ A, int64_t lda, int64_t M,
                                                             const bf16* __restrict__ B, int64_t ldb, int64_t K,
                                                             int64_t kPerSplit, Epi epi, int* __restrict__ err) {
  using namespace umma;
  extern __shared__ uint8_t smemRaw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smemRaw + 1023) & ~(uintptr_t)1023);
  float* sPart = (float*)(smem + 2 * GemmSmem<N>::kStage);  // [group][row]
  float* sRow = sPart + kGemmGroups * 128;                  // [row]
  uint64_t* mbar = (uint64_t*)(sRow + 128);                 // one per stage
  uint32_t* slot = (uint32_t*)(mbar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, grp = tid >> 7, row = tid & 127;
  const int64_t m0 = (int64_t)blockIdx.x * 128;
  const int64_t k0 = (int64_t)blockIdx.z * kPerSplit;
  const int64_t k1 = k0 + kPerSplit < K ? k0 + kPerSplit : K;
  constexpr uint32_t kCols = N < 32 ? 32 : N;
  if (warp == 0) tmemAlloc(smemAddr(slot), kCols);
  if (tid == 0) {
    mbarInit(smemAddr(mbar), 1);
    mbarInit(smemAddr(mbar + 1), 1);
  }
  fenceBefore();
  __syncthreads();
  fenceAfter();
  const uint32_t tmem = *slot;
  constexpr uint32_t idesc = idescBf16(128, N);
  // chunk kc into stage st; columns past the split's end (and rows past M) read as zeros
  auto load = [&](int st, int64_t kc) {
    uint8_t* sA = smem + st * GemmSmem<N>::kStage;
    uint8_t* sB = sA + GemmSmem<N>::kA;
    for (int i = tid; i < 128 * 8; i += kGemmThreads) {
      const int r = i >> 3, c = i & 7;
      const int64_t col = kc + c * 8, left = k1 - col;
      const uint32_t bytes = (m0 + r < M && left > 0) ? (uint32_t)(left >= 8 ? 16 : 2 * left) : 0u;
      cpAsync16(smemAddr(sA + swizzledChunk(r, c)), bytes ? (const void*)(A + (m0 + r) * lda + col) : (const void*)A,
                bytes);
    }
    for (int i = tid; i < N * 8; i += kGemmThreads) {
      const int r = i >> 3, c = i & 7;
      const int64_t col = kc + c * 8, left = k1 - col;
      const uint32_t bytes = left > 0 ? (uint32_t)(left >= 8 ? 16 : 2 * left) : 0u;
      cpAsync16(smemAddr(sB + swizzledChunk(r, c)), bytes ? (const void*)(B + (int64_t)r * ldb + col) : (const void*)B,
                bytes);
    }
    cpAsyncCommit();
  };
  const int nk = k1 > k0 ? (int)((k1 - k0 + 63) / 64) : 0;
  uint32_t ph[2] = {0u, 0u};
  bool ok = true;
  if (nk > 0) load(0, k0);
  for (int c = 0; c < nk; ++c) {
    const int st = c & 1;
    if (c + 1 < nk) {
      if (c >= 1) {  // the products of chunk c - 1 have read the stage chunk c + 1 goes into
        ok = mbarWait(smemAddr(mbar + (st ^ 1)), ph[st ^ 1]) && ok;
        ph[st ^ 1] ^= 1u;
      }
      load(st ^ 1, k0 + (int64_t)(c + 1) * 64);
      cpAsyncWait<1>();  // this chunk's copies (the next chunk's may still be in flight)
    } else {
      cpAsyncWait<0>();
    }
    fenceProxyAsync();
    __syncthreads();
    if (tid == 0) {
      fenceAfter();
      const uint8_t* sA = smem + st * GemmSmem<N>::kStage;
      const uint64_t da = descSw128(smemAddr(sA)), db = descSw128(smemAddr(sA + GemmSmem<N>::kA));
#pragma unroll
      for (int k = 0; k < 4; ++k) mma(tmem, da + 2 * k, db + 2 * k, idesc, (c > 0 || k > 0) ? 1u : 0u);
      commit(smemAddr(mbar + st));
    }
  }
  if (nk > 0) {  // the last chunk's products (and with them every earlier one)
    const int st = (nk - 1) & 1;
    ok = mbarWait(smemAddr(mbar + st), ph[st]) && ok;
  }
  fenceAfter();
  constexpr int C = N / kGemmGroups;
  static_assert(C == 16 || C == 32, "a quarter of the columns per warp group");
  float v[C];
  const uint32_t lane = (uint32_t)((warp & 3) * 32) << 16;
  if constexpr (C == 32) {
    tmemLoad32(tmem + lane + (uint32_t)(grp * C), v);
  } else {
    tmemLoad16(tmem + lane + (uint32_t)(grp * C), v);
  }
  if (k1 <= k0) {  // an empty split contributes zeros
#pragma unroll
    for (int j = 0; j < C; ++j) v[j] = 0.0f;
  }
  const int64_t m = m0 + row;
  epi(m, ok && m < M, grp * C, v, sPart, sRow, grp, smem, m0, M);  // the stages are free: the products are done
  fenceBefore();
  __syncthreads();
  if (warp == 0) tmemFree(tmem, kCols);
  if (!ok && tid == 0) atomicExch(err, 1);
}

// ---- epilogues ----------------------------------------------------------------------------
// Each is called by every thread with its row m, whether the row is written (valid), the first
// column j0 of its warp group's quarter and that quarter's accumulators. The row-major stores
// go out in 16-byte pieces (eight BF16 or four FP32 values per store); the transposed copies are
// coalesced across the warp as they are.
__device__ __forceinline__ uint4 packBf16x8(const float* v) {
  uint4 r;
  __nv_bfloat162* q = (__nv_bfloat162*)&r;
#pragma unroll
  for (int e = 0; e < 4; ++e) q[e] = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
  return r;
}
// The transposed copy of a 128-row tile goes through shared memory (sT[column][row], BF16):
// each thread stages its row's values, then the block writes whole rows of the transposed
// matrix (128 consecutive m) in 16-byte pieces.
__device__ __forceinline__ void stageT(bf16* sT, int row, int j, const uint4& vals) {
  const bf16* v = (const bf16*)&vals;
#pragma unroll
  for (int e = 0; e < 8; ++e) sT[(j + e) * 128 + row] = v[e];
}
__device__ __forceinline__ void storeT(const bf16* sT, bf16* dstT, int64_t ldt, int64_t m0, int64_t M) {
  for (int p = threadIdx.x; p < kHid * 16; p += blockDim.x) {
    const int j = p >> 4, r8 = (p & 15) * 8;
    const int64_t m = m0 + r8;
    bf16* dst = dstT + (int64_t)j * ldt + m;
    const bf16* src = sT + j * 128 + r8;
    if (m + 8 <= M) {
      *(uint4*)dst = *(const uint4*)src;
    } else {
      for (int e = 0; e < 8 && m + e < M; ++e) dst[e] = src[e];
    }
  }
}

// A row-major 128-row tile goes through shared memory too: each thread stages its row's 16-byte
// pieces (piece c of row r at slot c ^ (r mod pieces per row): no bank conflicts either way),
// then consecutive threads write consecutive pieces of whole rows, or, for loadRows, read them.
template <int RowBytes>
__device__ __forceinline__ void stageRow(uint8_t* sR, int row, int byteCol, const uint4& v) {
  constexpr int kPieces = RowBytes / 16;
  *(uint4*)(sR + row * RowBytes + (((byteCol >> 4) ^ (row % kPieces)) << 4)) = v;
}
template <int RowBytes>
__device__ __forceinline__ uint4 rowPiece(const uint8_t* sR, int row, int byteCol) {
  constexpr int kPieces = RowBytes / 16;
  return *(const uint4*)(sR + row * RowBytes + (((byteCol >> 4) ^ (row % kPieces)) << 4));
}
template <int RowBytes>
__device__ __forceinline__ void storeRows(const uint8_t* sR, void* dst, int64_t m0, int64_t M) {
  constexpr int kPieces = RowBytes / 16;
  for (int p = threadIdx.x; p < 128 * kPieces; p += blockDim.x) {
    const int row = p / kPieces, c = p % kPieces;
    if (m0 + row < M)
      *(uint4*)((uint8_t*)dst + (m0 + row) * RowBytes + c * 16) = rowPiece<RowBytes>(sR, row, c * 16);
  }
}
template <int RowBytes, int kThreads>  // a thread's loads go out four at a time before their shared stores
__device__ __forceinline__ void loadRows(uint8_t* sR, const void* src, int64_t m0, int64_t M) {
  constexpr int kPieces = RowBytes / 16, kPer = 128 * kPieces / kThreads, kBatch = 4;
  static_assert(kPer * kThreads == 128 * kPieces && kPer % kBatch == 0, "whole batches of pieces per thread");
#pragma unroll
  for (int i0 = 0; i0 < kPer; i0 += kBatch) {
    uint4 q[kBatch];
#pragma unroll
    for (int i = 0; i < kBatch; ++i) {
      const int p = threadIdx.x + (i0 + i) * kThreads, row = p / kPieces, c = p % kPieces;
      q[i] = m0 + row < M ? *(const uint4*)((const uint8_t*)src + (m0 + row) * RowBytes + c * 16)
                          : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int i = 0; i < kBatch; ++i) {
      const int p = threadIdx.x + (i0 + i) * kThreads;
      stageRow<RowBytes>(sR, p / kPieces, (p % kPieces) * 16, q[i]);
    }
  }
}

// Hidden layer: z = acc + b, h = gelu(z); Z (FP32, for the backward pass), H row-major and
// its transpose (the operands of the next layer and of the weight gradient). Ht and H go out
// through the two halves of the stage area, then Z through all of it.
struct EpiHidden {
  const float* bias;
  float* Z;
  bf16* H;
  bf16* Ht;
  int64_t ldt;
  template <int C>
  __device__ void operator()(int64_t m, bool valid, int j0, float (&v)[C], float*, float*, int, uint8_t* stage,
                             int64_t m0, int64_t M) const {
    bf16* sT = (bf16*)stage;
    uint8_t* sH = stage + kHid * 128 * 2;  // the second half: H row-major
    const int row = threadIdx.x & 127;
    if (valid) {
#pragma unroll
      for (int jb = 0; jb < C; jb += 8) {
        const int j = j0 + jb;
        float h[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          v[jb + e] += bias[j + e];  // z, kept for Z
          h[e] = geluF(v[jb + e]);
        }
        const uint4 hb = packBf16x8(h);
        stageRow<kHid * 2>(sH, row, j * 2, hb);
        if (Ht) stageT(sT, row, j, hb);
      }
    }
    __syncthreads();
    storeRows<kHid * 2>(sH, H, m0, M);
    if (Ht) storeT(sT, Ht, ldt, m0, M);
    if (!Z) return;
    __syncthreads();
    if (valid) {
#pragma unroll
      for (int jb = 0; jb < C; jb += 4)
        stageRow<kHid * 4>(stage, row, (j0 + jb) * 4,
                           make_uint4(__float_as_uint(v[jb]), __float_as_uint(v[jb + 1]), __float_as_uint(v[jb + 2]),
                                      __float_as_uint(v[jb + 3])));
    }
    __syncthreads();
    storeRows<kHid * 4>(stage, Z, m0, M);
  }
};

constexpr int kOutParts = 4;  // partial sums of the output unit (one per quarter of the columns)
static_assert(kOutParts == kGemmGroups, "the output unit's partial sums follow the warp groups");

// Last hidden layer plus the output unit. Inference: out = sum_j h_j w4_j + b4. Training also
// forms the loss gradient d = scale (out - y) and dZ3 = d w4 gelu'(z3), H3 transposed (for
// the w4 gradient) and the per-row squared error. The output unit sums each quarter of the
// columns in order (one per warp group), then the four partial sums in order -- the fused
// inference kernel's split, so both give the same bits.
struct EpiOutput {
  const float* bias;
  const float* w4;  // BF16-rounded values
  const float* b4;
  float* out;
  // training only
  const float* y;
  float scale;
  bf16* H3t;  // H3 transposed (for the w4 gradient)
  bf16* dZ;
  bf16* dZt;
  int64_t ldt;
  float* dOut;
  float* sqErr;
  template <int C>
  __device__ void operator()(int64_t m, bool valid, int j0, float (&v)[C], float* sPart, float* sRow, int grp,
                             uint8_t* stage, int64_t m0, int64_t M) const {
    const int row = threadIdx.x & 127;
    bf16* sT3 = (bf16*)stage + kHid * 128;  // H3's transposed tile (the stage area's second half)
    float o = 0.0f;
    if (valid) {
#pragma unroll
      for (int jb = 0; jb < C; jb += 8) {
        float h[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int j = j0 + jb + e;
          v[jb + e] += bias[j];
          h[e] = __bfloat162float(__float2bfloat16_rn(geluF(v[jb + e])));
          o += h[e] * w4[j];
        }
        if (H3t) stageT(sT3, row, j0 + jb, packBf16x8(h));
      }
    }
    sPart[grp * 128 + row] = o;
    __syncthreads();
    if (H3t) storeT(sT3, H3t, ldt, m0, M);
    if (grp == 0) {
      float d = 0.0f;
      if (valid) {
        float oo = sPart[row];
#pragma unroll
        for (int g = 1; g < kOutParts; ++g) oo += sPart[g * 128 + row];
        oo += b4[0];
        if (out) out[m] = oo;
        if (y) {
          const float e = oo - y[m];
          d = scale * e;
          dOut[m] = d;
          sqErr[m] = e * e;
        }
      }
      sRow[row] = d;
    }
    __syncthreads();
    if (!y) return;
    bf16* sT = (bf16*)stage;  // dZt; dZ row-major in the second half (H3t's copy is out)
    if (valid) {
      const float d = sRow[row];
#pragma unroll
      for (int jb = 0; jb < C; jb += 8) {
        const int j = j0 + jb;
        float g[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) g[k] = d * w4[j + k] * geluGrad(v[jb + k]);
        const uint4 gb = packBf16x8(g);
        stageRow<kHid * 2>((uint8_t*)sT3, row, j * 2, gb);
        stageT(sT, row, j, gb);
      }
    }
    __syncthreads();
    storeRows<kHid * 2>((const uint8_t*)sT3, dZ, m0, M);
    storeT(sT, dZt, ldt, m0, M);
  }
};

// Backward through a hidden layer: dZ = acc * gelu'(Z) (acc = dH of that layer).
struct EpiBack {
  const float* Z;
  bf16* dZ;
  bf16* dZt;
  int64_t ldt;
  template <int C>
  __device__ void operator()(int64_t m, bool valid, int j0, float (&v)[C], float*, float*, int, uint8_t* stage,
                             int64_t m0, int64_t M) const {
    // Z's tile comes in through all of the stage area (whole rows per warp), then dZt and dZ go
    // out through its two halves
    bf16* sT = (bf16*)stage;
    uint8_t* sD = stage + kHid * 128 * 2;
    const int row = threadIdx.x & 127;
    loadRows<kHid * 4, kGemmThreads>(stage, Z, m0, M);
    __syncthreads();
    if (valid) {  // dZ in place of the accumulators
#pragma unroll
      for (int jb = 0; jb < C; jb += 4) {
        const uint4 zq = rowPiece<kHid * 4>(stage, row, (j0 + jb) * 4);
        v[jb] *= geluGrad(__uint_as_float(zq.x));
        v[jb + 1] *= geluGrad(__uint_as_float(zq.y));
        v[jb + 2] *= geluGrad(__uint_as_float(zq.z));
        v[jb + 3] *= geluGrad(__uint_as_float(zq.w));
      }
    }
    __syncthreads();
    if (valid) {
#pragma unroll
      for (int jb = 0; jb < C; jb += 8) {
        const int j = j0 + jb;
        const uint4 gb = packBf16x8(v + jb);
        if (dZ) stageRow<kHid * 2>(sD, row, j * 2, gb);
        stageT(sT, row, j, gb);
      }
    }
    __syncthreads();
    if (dZ) storeRows<kHid * 2>(sD, dZ, m0, M);
    storeT(sT, dZt, ldt, m0, M);
  }
};

// Split-K partial of a weight gradient: partial[split][m][n].
template <int N>
struct EpiPartial {
  float* partial;
  int64_t rows;
  template <int C>
  __device__ void operator()(int64_t m, bool valid, int j0, float (&v)[C], float*, float*, int, uint8_t*, int64_t,
                             int64_t) const {
    if (!valid) return;
    float* p = partial + ((int64_t)blockIdx.z * rows + m) * N + j0;
#pragma unroll
    for (int j = 0; j < C; j += 4) *(float4*)(p + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
  }
};

// ---- fused inference ------------------------------------------------------------------------
// The whole network for 128-row tiles in one persistent kernel: the three weight matrices
// stay in shared memory (80 KB, loaded once per CTA), the features of a tile are converted to
// BF16 into shared memory, and each layer's activations go from TMEM through the epilogue
// straight back into shared memory as the next layer's A operand -- nothing but the features
// and the outputs touches global memory. The MMA sequence and the epilogue arithmetic are
// those of the layer-by-layer kernels, so the outputs are identical.
constexpr int kFusedSlots = 2;                                 // 128-row tiles in flight per CTA
constexpr int kFusedGroups = 4;                                // warp groups per tile, one per quarter of the columns
constexpr int kSlotThreads = 128 * kFusedGroups;
constexpr int kFusedThreads = kSlotThreads * kFusedSlots;
constexpr int kGroupCols = 128 / kFusedGroups;
static_assert(kFusedGroups == kOutParts, "the output unit's partial sums follow the warp groups in both kernels");
constexpr int kFusedSmem = 16384 /*W1*/ + 32768 /*W2*/ + 32768 /*W3*/ + kFusedSlots * (16384 /*X*/ + 32768 /*H*/) +
                           4 * 128 * 4 /*b1 b2 b3 w4*/ + kFusedSlots * kFusedGroups * 128 * 4 /*partial sums*/ + 64 +
                           1024;

// The fused kernel's shared-memory image of the weights, built once per parameter update:
// W1 (16 KB), W2 and W3 (32 KB each) as 128 x K bf16 K-major B operands in 128-byte-swizzled
// blocks of 128 x 64, then b1, b2, b3 and the BF16-rounded w4 (512 floats). A CTA fetches it
// with a few bulk copies.
constexpr int kImgWeights = 16384 + 32768 + 32768, kImgBytes = kImgWeights + 4 * 128 * 4;
__global__ void kPackFusedImage(const float* __restrict__ P, const bf16* __restrict__ W1, const bf16* __restrict__ W2,
                                const bf16* __restrict__ W3, const float* __restrict__ w4r, uint8_t* __restrict__ img) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // one 16-byte chunk of a weight row
  if (i < 128 * 8 + 2 * 128 * 16) {
    const bf16* W = i < 1024 ? W1 : (i < 1024 + 2048 ? W2 : W3);
    const int K = i < 1024 ? kIn : kHid;
    const int j = i < 1024 ? i : (i - 1024) % 2048;
    const int r = j / (K / 8), c = j % (K / 8);
    uint8_t* dst = img + (i < 1024 ? 0 : (i < 1024 + 2048 ? 16384 : 16384 + 32768));
    *(uint4*)(dst + (c >> 3) * 16384 + umma::swizzledChunk(r, c & 7)) = *(const uint4*)(W + (int64_t)r * K + c * 8);
  }
  if (i < 512) {
    float* b = (float*)(img + kImgWeights);
    b[i] = i < 384 ? P[(i < 128 ? kOffB1 : (i < 256 ? kOffB2 : kOffB3)) + (i & 127)] : w4r[i - 384];
  }
}

// Barrier of one tile slot (256 threads), ids 1 and 2 (0 is __syncthreads').
__device__ __forceinline__ void slotSync(int s) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + s), "n"(kSlotThreads) : "memory");
}

// Share-network inference: persistent, one CTA per SM, two 128-row tiles in flight. A tile's
// 512 threads load its features, one of them issues each layer's MMAs, and the four warp
// groups run the epilogue of a quarter of the 128 columns each (thread = row, the TMEM lane of
// its warp). Biases and output weights sit in shared memory. The output unit sums each
// group's quarter of the columns in order and the first group adds the four partial sums in
// order, as the layer-by-layer kernels do, so the result is theirs bit for bit.
__global__ void __launch_bounds__(kFusedThreads, 1)
    kMlpForwardFused(const float* __restrict__ X, int64_t n, const uint8_t* __restrict__ img,
                     const float* __restrict__ P, float* __restrict__ out, int* __restrict__ err, const int64_t* __restrict__ shareIds,
                     double* __restrict__ shares, float shareScale, float shareMean, const bf16* __restrict__ Xt) {
  using namespace umma;
  extern __shared__ uint8_t smemRaw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smemRaw + 1023) & ~(uintptr_t)1023);
  uint8_t* sW1 = smem;
  uint8_t* sW2 = sW1 + 16384;
  uint8_t* sW3 = sW2 + 32768;
  const int tid = threadIdx.x, s = tid / kSlotThreads, st = tid % kSlotThreads, grp = st >> 7, row = tid & 127,
            warp = tid >> 5;
  uint8_t* sX = sW3 + 32768 + s * (16384 + 32768);
  uint8_t* sH = sX + 16384;
  float* sBias = (float*)(sW3 + 32768 + kFusedSlots * (16384 + 32768));  // b1, b2, b3, w4 (128 each)
  float* sPart = sBias + 4 * 128 + s * kFusedGroups * 128;               // [group][row] partial sums
  uint64_t* mbar = (uint64_t*)(sBias + 4 * 128 + kFusedSlots * kFusedGroups * 128);  // MMA, input loads, weights
  uint32_t* tslot = (uint32_t*)(mbar + 2 * kFusedSlots + 1);
  volatile uint32_t* slot0Started = tslot + 1;  // set once slot 0's first layer-1 product is done
  const uint32_t barW = smemAddr(mbar + 2 * kFusedSlots);
  if (warp == 0) tmemAlloc(smemAddr(tslot), 128 * kFusedSlots);
  if (tid == 0) {
    *slot0Started = 0;
    for (int k = 0; k < 2 * kFusedSlots + 1; ++k) mbarInit(smemAddr(mbar + k), 1);
    // the weight image in five 16 KB bulk copies and the biases in one; the image was written
    // before the previous kernel started (only the features are its output)
    mbarArriveExpectTx(barW, kImgBytes);
#pragma unroll
    for (int k = 0; k < kImgWeights / 16384; ++k) bulkLoad(smemAddr(sW1 + k * 16384), img + k * 16384, 16384, barW);
    bulkLoad(smemAddr(sBias), img + kImgWeights, kImgBytes - kImgWeights, barW);
  }
  gridDependencyWait();
  gridDependents();
  const int64_t tiles = (n + 127) / 128;
  if (tid == 0 && Xt)  // each slot's first input tile (the previous kernel's output), beside the weights
    for (int s2 = 0; s2 < kFusedSlots; ++s2) {
      const int64_t t0 = (int64_t)blockIdx.x * kFusedSlots + s2;
      if (t0 >= tiles) break;
      const uint32_t b2 = smemAddr(mbar + kFusedSlots + s2);
      mbarArriveExpectTx(b2, 16384);
      bulkLoad(smemAddr(sW3 + 32768 + s2 * (16384 + 32768)), (const uint8_t*)Xt + t0 * 16384, 16384, b2);
    }
  fenceBefore();
  __syncthreads();
  fenceAfter();
  bool ok = mbarWait(barW, 0);
  const uint32_t tmem = *tslot + 128u * s;                 // this tile slot's 128 columns
  const uint32_t lane = (uint32_t)((warp & 3) * 32) << 16;  // the warp's TMEM lanes
  constexpr uint32_t idesc = idescBf16(128, kHid);
  const uint32_t bar = smemAddr(mbar + s), barX = smemAddr(mbar + kFusedSlots + s);
  uint32_t phase = 0, phaseX = 0;
  const float* b1 = sBias;
  const float* b2 = sBias + 128;
  const float* b3 = sBias + 256;
  const float* w4 = sBias + 384;
  const bool xVec = ((uintptr_t)X & 15) == 0;  // rows are 256 B apart: 16-byte loads when the base allows
  for (int64_t t = (int64_t)blockIdx.x * kFusedSlots + s; t < tiles; t += (int64_t)gridDim.x * kFusedSlots) {
    const int64_t m = t * 128 + row;
    if (Xt) {  // the tile already in BF16 and swizzled: one bulk copy by the TMA engine
      if (st == 0 && t != (int64_t)blockIdx.x * kFusedSlots + s) {  // (the first was issued above)
        mbarArriveExpectTx(barX, 16384);
        bulkLoad(smemAddr(sX), (const uint8_t*)Xt + t * 16384, 16384, barX);
      }
      ok = mbarWait(barX, phaseX) && ok;
      phaseX ^= 1u;
    }
    // features -> BF16: the tile's 128 rows x 256 B read in coalesced 32-byte pieces, each one
    // 16-byte chunk of a row in the swizzled A tile
#pragma unroll 2
    for (int p = st; p < (Xt ? 0 : 128 * 8); p += kSlotThreads) {
      const int pr = p >> 3, pc = p & 7;
      const int64_t mr = t * 128 + pr;
      float4 f0 = make_float4(0.f, 0.f, 0.f, 0.f), f1 = f0;
      if (mr < n) {
        const float* src = X + mr * kIn + pc * 8;
        if (xVec) {
          f0 = ((const float4*)src)[0];
          f1 = ((const float4*)src)[1];
        } else {
          f0 = make_float4(src[0], src[1], src[2], src[3]);
          f1 = make_float4(src[4], src[5], src[6], src[7]);
        }
      }
      __align__(16) bf16 v[8] = {__float2bfloat16_rn(f0.x), __float2bfloat16_rn(f0.y), __float2bfloat16_rn(f0.z),
                                 __float2bfloat16_rn(f0.w), __float2bfloat16_rn(f1.x), __float2bfloat16_rn(f1.y),
                                 __float2bfloat16_rn(f1.z), __float2bfloat16_rn(f1.w)};
      *(uint4*)(sX + swizzledChunk(pr, pc)) = *(const uint4*)v;
    }
    // The two slots start half a layer apart: slot 1 begins once slot 0's first product is
    // done, so that one slot's epilogue (bound by the tanh unit and the issue rate) runs while
    // the other's MMA does. A bounded wait: past the bound slot 1 simply goes on.
    if (s == 1 && t == (int64_t)blockIdx.x * kFusedSlots + s)
      for (int spin = 0; spin < 20000 && *slot0Started == 0; ++spin) __nanosleep(32);
    float o = 0.0f;
    for (int layer = 0; layer < 3; ++layer) {
      fenceProxyAsync();
      fenceBefore();
      slotSync(s);
      if (st == 0) {
        fenceAfter();
        if (layer == 0) {
          const uint64_t da = descSw128(smemAddr(sX)), db = descSw128(smemAddr(sW1));
#pragma unroll
          for (int k = 0; k < 4; ++k) mma(tmem, da + 2 * k, db + 2 * k, idesc, k > 0 ? 1u : 0u);
        } else {
          const uint8_t* sW = layer == 1 ? sW2 : sW3;
#pragma unroll
          for (int kb = 0; kb < 2; ++kb) {
            const uint64_t da = descSw128(smemAddr(sH + kb * 16384)), db = descSw128(smemAddr(sW + kb * 16384));
#pragma unroll
            for (int k = 0; k < 4; ++k) mma(tmem, da + 2 * k, db + 2 * k, idesc, (kb > 0 || k > 0) ? 1u : 0u);
          }
        }
        commit(bar);
      }
      ok = mbarWait(bar, phase) && ok;
      phase ^= 1u;
      fenceAfter();
      if (s == 0 && st == 0 && layer == 0) *slot0Started = 1;
      // epilogue of this group's 32 columns: one TMEM load, one wait
      const float* bias = layer == 0 ? b1 : (layer == 1 ? b2 : b3);
      const int n0 = kGroupCols * grp;
      float v[kGroupCols];
      tmemLoad32(tmem + lane + (uint32_t)n0, v);
      // two columns per packed FP32 instruction; the output unit's sum stays in column order
      if (layer < 2) {  // hidden layer: the next layer's A operand
#pragma unroll
        for (int h = 0; h < kGroupCols / 8; ++h) {
          __align__(16) __nv_bfloat162 q[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int j = h * 8 + 2 * e;
            const float2 b = *(const float2*)(bias + n0 + j);
            q[e] = __float22bfloat162_rn(geluF2(__fadd2_rn(make_float2(v[j], v[j + 1]), b)));
          }
          const int c = (n0 >> 3) + h;
          *(uint4*)(sH + (c >> 3) * 16384 + swizzledChunk(row, c & 7)) = *(const uint4*)q;
        }
      } else {  // output unit: this group's quarter of the columns, in order
#pragma unroll
        for (int j = 0; j < kGroupCols; j += 2) {
          const float2 b = *(const float2*)(bias + n0 + j);
          const float2 g = __bfloat1622float2(__float22bfloat162_rn(geluF2(__fadd2_rn(make_float2(v[j], v[j + 1]), b))));
          const float2 t = __fmul2_rn(g, *(const float2*)(w4 + n0 + j));
          o += t.x;
          o += t.y;
        }
      }
    }
    if (grp > 0) sPart[grp * 128 + row] = o;
    slotSync(s);
    if (grp == 0) {
#pragma unroll
      for (int g = 1; g < kFusedGroups; ++g) o += sPart[g * 128 + row];
      if (m < n && ok) {
        const float pred = o + P[kOffB4];
        if (shares)  // the learned start's share of coincident vertex shareIds[m], de-normalised
          shares[shareIds[m]] = (double)pred * (double)shareScale + (double)shareMean;
        else
          out[m] = pred;
      }
    }
    fenceBefore();
    slotSync(s);  // TMEM read and sH free before the next tile
  }
  fenceBefore();
  __syncthreads();
  if (warp == 0) tmemFree(*tslot, 128 * kFusedSlots);
  if (!ok) atomicExch(err, 1);
}

// ---- small kernels ----------------------------------------------------------------------
// Features (FP32, n x 64, already normalised) to BF16 rows (and columns for training).
__global__ void kFeaturesBf16(const float* __restrict__ X, int64_t n, bf16* __restrict__ Xb, bf16* __restrict__ Xt,
                              int64_t ldt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * kIn) return;
  const int64_t m = i / kIn;
  const int k = (int)(i % kIn);
  const bf16 v = __float2bfloat16_rn(X[i]);
  Xb[i] = v;
  if (Xt) Xt[(int64_t)k * ldt + m] = v;
}

// BF16 weight copies (row-major and transposed) and the BF16-rounded output weights.
__global__ void kCastWeights(const float* __restrict__ P, bf16* __restrict__ W1, bf16* __restrict__ W1t,
                             bf16* __restrict__ W2, bf16* __restrict__ W2t, bf16* __restrict__ W3,
                             bf16* __restrict__ W3t, float* __restrict__ w4r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kHid * kIn) {
    const int o = i / kIn, k = i % kIn;
    const bf16 v = __float2bfloat16_rn(P[kOffW1 + i]);
    W1[i] = v;
    W1t[k * kHid + o] = v;
  }
  if (i < kHid * kHid) {
    const int o = i / kHid, k = i % kHid;
    const bf16 v2 = __float2bfloat16_rn(P[kOffW2 + i]);
    W2[i] = v2;
    W2t[k * kHid + o] = v2;
    const bf16 v3 = __float2bfloat16_rn(P[kOffW3 + i]);
    W3[i] = v3;
    W3t[k * kHid + o] = v3;
  }
  if (i < kHid) w4r[i] = __bfloat162float(__float2bfloat16_rn(P[kOffW4 + i]));
}

// Fixed-order block sum over a row of length n (one block per output).
__device__ __forceinline__ float blockSum256(float v) {
  __shared__ float sh[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  float t = 0.0f;
  if (threadIdx.x == 0)
    for (int w = 0; w < 8; ++w) t += sh[w];
  return t;
}

// Gradients not produced by a GEMM: biases of the hidden layers (row sums of dZ^T), the output
// weights (H3^T dOut), the output bias (sum dOut) and the loss (mean squared error).
// Block b: 0..383 hidden biases, 384..511 w4, 512 b4, 513 loss.
__global__ void __launch_bounds__(256) kSmallGrads(const bf16* __restrict__ dZ1t, const bf16* __restrict__ dZ2t,
                                                  const bf16* __restrict__ dZ3t, const bf16* __restrict__ H3t,
                                                  const float* __restrict__ dOut, const float* __restrict__ sqErr,
                                                  int64_t n, int64_t ldt, float* __restrict__ grad,
                                                  float* __restrict__ loss) {
  const int b = blockIdx.x;
  float s = 0.0f;
  if (b < 3 * kHid) {
    const bf16* row = (b < kHid ? dZ1t : b < 2 * kHid ? dZ2t : dZ3t) + (int64_t)(b % kHid) * ldt;
    for (int64_t m = threadIdx.x; m < n; m += 256) s += __bfloat162float(row[m]);
  } else if (b < 4 * kHid) {
    const int j = b - 3 * kHid;
    for (int64_t m = threadIdx.x; m < n; m += 256) s += dOut[m] * __bfloat162float(H3t[(int64_t)j * ldt + m]);
  } else if (b == 4 * kHid) {
    for (int64_t m = threadIdx.x; m < n; m += 256) s += dOut[m];
  } else {
    for (int64_t m = threadIdx.x; m < n; m += 256) s += sqErr[m];
  }
  const float t = blockSum256(s);
  if (threadIdx.x != 0) return;
  if (b < 3 * kHid) {
    const int64_t off = b < kHid ? kOffB1 : b < 2 * kHid ? kOffB2 : kOffB3;
    grad[off + b % kHid] = t;
  } else if (b < 4 * kHid) {
    grad[kOffW4 + (b - 3 * kHid)] = t;
  } else if (b == 4 * kHid) {
    grad[kOffB4] = t;
  } else {
    loss[0] = t / (float)n;
  }
}

// Weight gradients from the split-K partials (summed in split order).
__global__ void kSumPartials(const float* __restrict__ P1, const float* __restrict__ P2, const float* __restrict__ P3,
                             float* __restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kHid * kIn) {
    float s = 0.0f;
    for (int k = 0; k < kSplitK; ++k) s += P1[(int64_t)k * kHid * kIn + i];
    grad[kOffW1 + i] = s;
  }
  if (i < kHid * kHid) {
    float s2 = 0.0f, s3 = 0.0f;
    for (int k = 0; k < kSplitK; ++k) {
      s2 += P2[(int64_t)k * kHid * kHid + i];
      s3 += P3[(int64_t)k * kHid * kHid + i];
    }
    grad[kOffW2 + i] = s2;
    grad[kOffW3 + i] = s3;
  }
}

// Adam (Kingma & Ba): m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2; p -= lr mhat / (sqrt(vhat) + eps).
__global__ void kAdam(float* __restrict__ P, float* __restrict__ Mo, float* __restrict__ Ve,
                      const float* __restrict__ G, int64_t n, float lr, float b1, float b2, float eps, float c1,
                      float c2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  const float m = b1 * Mo[i] + (1.0f - b1) * g;
  const float v = b2 * Ve[i] + (1.0f - b2) * g * g;
  Mo[i] = m;
  Ve[i] = v;
  P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

// Random batch: rows idx of the dataset (features n x 64 FP32, targets n).
__global__ void kGatherBatch(const float* __restrict__ X, const float* __restrict__ y, int64_t n, uint64_t seed,
                             uint64_t step, int64_t B, bf16* __restrict__ Xb, bf16* __restrict__ Xt,
                             float* __restrict__ yb) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= B) return;
  // splitmix64 of (seed, step, i)
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * (step * (uint64_t)B + (uint64_t)i + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const int64_t r = (int64_t)(z % (uint64_t)n);
  yb[i] = y[r];
  const float* src = X + r * kIn;
  if (((uintptr_t)X & 15) == 0) {  // the row in 16-byte pieces, the BF16 row out in 16-byte pieces
#pragma unroll
    for (int k = 0; k < kIn; k += 8) {
      const float4 a = *(const float4*)(src + k), b = *(const float4*)(src + k + 4);
      const float f[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
      __align__(16) bf16 q[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        q[e] = __float2bfloat16_rn(f[e]);
        Xt[(int64_t)(k + e) * B + i] = q[e];
      }
      *(uint4*)(Xb + i * kIn + k) = *(const uint4*)q;
    }
  } else {
    for (int k = 0; k < kIn; ++k) {
      const bf16 v = __float2bfloat16_rn(src[k]);
      Xb[i * kIn + k] = v;
      Xt[(int64_t)k * B + i] = v;
    }
  }
}

template <int N, class Epi>
static its_status gemm(its_ctx* ctx, const bf16* A, int64_t lda, int64_t M, const bf16* B, int64_t ldb, int64_t K,
                       int splits, const Epi& epi, int* err) {
  static bool configured = false;
  if (!configured) {
    ITS_CU(ctx, cudaFuncSetAttribute(kUmmaGemm<N, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     GemmSmem<N>::kBytes));
    configured = true;
  }
  const int64_t kPer = ((K / splits + 63) / 64) * 64;
  dim3 grid((unsigned)((M + 127) / 128), 1, (unsigned)splits);
  kUmmaGemm<N, Epi><<<grid, kGemmThreads, GemmSmem<N>::kBytes, ctx->stream>>>(A, lda, M, B, ldb, K, kPer, epi, err);
  ITS_LAUNCHED(ctx);
  return ITS_OK;
}

}  // namespace its

using namespace its;

struct its_mlp {
  its_ctx* ctx = nullptr;
  uint64_t uid = 0;  // distinct for every network made (a later one may reuse a freed address)
  int64_t cap = 0;  // rows per batch
  float* P = nullptr;
  float* Mo = nullptr;
  float* Ve = nullptr;
  float* G = nullptr;
  float* loss = nullptr;
  int64_t step = 0;
  bf16 *W1, *W1t, *W2, *W2t, *W3, *W3t;
  float* w4r;
  uint8_t* img;  // the fused inference kernel's shared-memory image of the parameters
  // batch buffers
  bf16 *Xb, *Xt, *H1, *H1t, *H2, *H2t, *H3t, *dZ3, *dZ3t, *dZ2, *dZ2t, *dZ1t;
  float *Z1, *Z2, *yb, *dOut, *sqErr, *out, *part1, *part2, *part3;
  int* err;
  std::vector<void*> allocs;
  template <typename T>
  its_status alloc(T** p, int64_t count) {
    its_status s = devAlloc(ctx, (void**)p, (size_t)count * sizeof(T));
    if (s == ITS_OK) allocs.push_back((void*)*p);
    return s;
  }
};

namespace its {

static its_status mlpCast(its_mlp* h) {
  kCastWeights<<<gridFor(kHid * kHid, 256), 256, 0, h->ctx->stream>>>(h->P, h->W1, h->W1t, h->W2, h->W2t, h->W3,
                                                                      h->W3t, h->w4r);
  ITS_LAUNCHED(h->ctx);
  kPackFusedImage<<<gridFor(128 * 8 + 2 * 128 * 16, 256), 256, 0, h->ctx->stream>>>(h->P, h->W1, h->W2, h->W3, h->w4r,
                                                                                    h->img);
  ITS_LAUNCHED(h->ctx);
  return ITS_OK;
}

// Forward of n <= cap rows already in h->Xb; training forms the loss gradients too.
static its_status mlpForward(its_mlp* h, int64_t n, bool train, const float* y, float* out) {
  its_ctx* ctx = h->ctx;
  its_status st;
  const int64_t ldt = h->cap;
  EpiHidden e1{h->P + kOffB1, train ? h->Z1 : nullptr, h->H1, train ? h->H1t : nullptr, ldt};
  if ((st = gemm<kHid>(ctx, h->Xb, kIn, n, h->W1, kIn, kIn, 1, e1, h->err)) != ITS_OK) return st;
  EpiHidden e2{h->P + kOffB2, train ? h->Z2 : nullptr, h->H2, train ? h->H2t : nullptr, ldt};
  if ((st = gemm<kHid>(ctx, h->H1, kHid, n, h->W2, kHid, kHid, 1, e2, h->err)) != ITS_OK) return st;
  EpiOutput e3{h->P + kOffB3, h->w4r, h->P + kOffB4, out, y, 2.0f / (float)n, train ? h->H3t : nullptr,
               h->dZ3, h->dZ3t, ldt, h->dOut, h->sqErr};
  return gemm<kHid>(ctx, h->H2, kHid, n, h->W3, kHid, kHid, 1, e3, h->err);
}

// Gradient of the mean squared error over the n rows in h->Xb/h->Xt (targets yb) into h->G.
static its_status mlpGradient(its_mlp* h, int64_t n) {
  its_ctx* ctx = h->ctx;
  its_status st;
  const int64_t ldt = h->cap;
  if ((st = mlpForward(h, n, true, h->yb, nullptr)) != ITS_OK) return st;
  // dH2 = dZ3 W3 -> dZ2; dH1 = dZ2 W2 -> dZ1 (transposed only)
  EpiBack b2{h->Z2, h->dZ2, h->dZ2t, ldt};
  if ((st = gemm<kHid>(ctx, h->dZ3, kHid, n, h->W3t, kHid, kHid, 1, b2, h->err)) != ITS_OK) return st;
  EpiBack b1{h->Z1, nullptr, h->dZ1t, ldt};
  if ((st = gemm<kHid>(ctx, h->dZ2, kHid, n, h->W2t, kHid, kHid, 1, b1, h->err)) != ITS_OK) return st;
  // weight gradients dW_l = dZ_l^T H_{l-1}: split-K over the batch
  EpiPartial<kHid> p3{h->part3, kHid};
  if ((st = gemm<kHid>(ctx, h->dZ3t, ldt, kHid, h->H2t, ldt, n, kSplitK, p3, h->err)) != ITS_OK) return st;
  EpiPartial<kHid> p2{h->part2, kHid};
  if ((st = gemm<kHid>(ctx, h->dZ2t, ldt, kHid, h->H1t, ldt, n, kSplitK, p2, h->err)) != ITS_OK) return st;
  EpiPartial<kIn> p1{h->part1, kHid};
  if ((st = gemm<kIn>(ctx, h->dZ1t, ldt, kHid, h->Xt, ldt, n, kSplitK, p1, h->err)) != ITS_OK) return st;
  kSumPartials<<<gridFor(kHid * kHid, 256), 256, 0, ctx->stream>>>(h->part1, h->part2, h->part3, h->G);
  ITS_LAUNCHED(ctx);
  kSmallGrads<<<4 * kHid + 2, 256, 0, ctx->stream>>>(h->dZ1t, h->dZ2t, h->dZ3t, h->H3t, h->dOut, h->sqErr, n, ldt, h->G,
                                                     h->loss);
  ITS_LAUNCHED(ctx);
  return ITS_OK;
}

static its_status mlpAdam(its_mlp* h, float lr) {
  ++h->step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)h->step), c2 = 1.0f - powf(b2, (float)h->step);
  kAdam<<<gridFor(kNumParams, 256), 256, 0, h->ctx->stream>>>(h->P, h->Mo, h->Ve, h->G, kNumParams, lr, b1, b2, 1e-8f,
                                                              c1, c2);
  ITS_LAUNCHED(h->ctx);
  return mlpCast(h);
}

static its_status checkErr(its_mlp* h) {
  int e = 0;
  ITS_CU(h->ctx, cudaMemcpyAsync(&e, h->err, 4, cudaMemcpyDeviceToHost, h->ctx->stream));
  ITS_CU(h->ctx, cudaStreamSynchronize(h->ctx->stream));
  if (e) return setError(h->ctx, ITS_ERR_TIMEOUT, "share network: a tensor-core wait ran out");
  return ITS_OK;
}

// Predictions for n device rows into device out, launched on the context's stream without
// waiting (the caller checks the error flag at its next synchronisation).
static its_status launchFused(its_mlp* h, const float* X, int64_t n, float* out, const int64_t* ids, double* shares,
                              float scale, float mean, bool afterKernel, const bf16* Xt = nullptr) {
  its_ctx* ctx = h->ctx;
  if (n <= 0) return ITS_OK;
  const int64_t tiles = (n + 127) / 128, ctas = (tiles + kFusedSlots - 1) / kFusedSlots;
  const unsigned grid = (unsigned)(ctas < ctx->numSMs ? ctas : ctx->numSMs);
  return launchDependent(ctx, afterKernel, kMlpForwardFused, grid, kFusedThreads, kFusedSmem, ctx->stream, X, n,
                         (const uint8_t*)h->img, (const float*)h->P, out, h->err, ids, shares, scale, mean, Xt);
}
its_status mlpInfer(its_mlp* h, const float* X, int64_t n, float* out, bool afterKernel) {
  return launchFused(h, X, n, out, nullptr, nullptr, 0.0f, 0.0f, afterKernel);
}
// The same predictions written as shares: shares[ids[m]] = pred[m] * scale + mean (in FP64,
// as the share scatter of the learned start computes it).
// Predictions from input tiles that are already BF16 and swizzled (128 rows x 128 B each,
// whole tiles): into out, or, with shares set, as shares[ids[m]] = pred[m] * scale + mean (in
// FP64, as the share scatter of the learned start computes it).
its_status mlpInferTiles(its_mlp* h, const bf16* tiles, int64_t n, float* out, const int64_t* ids, float scale,
                         float mean, double* shares, bool afterKernel) {
  return launchFused(h, nullptr, n, out, ids, shares, scale, mean, afterKernel, tiles);
}

its_status mlpCheck(its_mlp* h) { return checkErr(h); }
// The network's (sticky) error flag in device memory, for callers that read it with their own copy.
const int* mlpErrFlag(its_mlp* h) { return h->err; }
uint64_t mlpUid(const its_mlp* h) { return h->uid; }

}  // namespace its

extern "C" {

its_status its_mlp_create(its_ctx* ctx, int64_t batch, its_mlp** out) {
  if (!ctx || !out || batch <= 0 || batch % 128) return ITS_ERR_INVALID;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  its_mlp* h = new its_mlp;
  h->ctx = ctx;
  static std::atomic<uint64_t> made{0};
  h->uid = ++made;
  h->cap = batch;
  const int64_t B = batch;
  its_status s = ITS_OK;
  auto A = [&](auto** p, int64_t c) {
    if (s == ITS_OK) s = h->alloc(p, c);
  };
  A(&h->P, kNumParams); A(&h->Mo, kNumParams); A(&h->Ve, kNumParams); A(&h->G, kNumParams); A(&h->loss, 1);
  A(&h->W1, kHid * kIn); A(&h->W1t, kHid * kIn); A(&h->W2, kHid * kHid); A(&h->W2t, kHid * kHid);
  A(&h->W3, kHid * kHid); A(&h->W3t, kHid * kHid); A(&h->w4r, kHid); A(&h->img, kImgBytes);
  A(&h->Xb, B * kIn); A(&h->Xt, B * kIn); A(&h->H1, B * kHid); A(&h->H1t, B * kHid); A(&h->H2, B * kHid);
  A(&h->H2t, B * kHid); A(&h->H3t, B * kHid); A(&h->dZ3, B * kHid); A(&h->dZ3t, B * kHid); A(&h->dZ2, B * kHid);
  A(&h->dZ2t, B * kHid); A(&h->dZ1t, B * kHid); A(&h->Z1, B * kHid); A(&h->Z2, B * kHid); A(&h->yb, B);
  A(&h->dOut, B); A(&h->sqErr, B); A(&h->out, B); A(&h->part1, (int64_t)kSplitK * kHid * kIn);
  A(&h->part2, (int64_t)kSplitK * kHid * kHid); A(&h->part3, (int64_t)kSplitK * kHid * kHid); A(&h->err, 1);
  if (s != ITS_OK) {
    for (void* p : h->allocs) devFree(ctx, p);
    delete h;
    return s;
  }
  cudaMemsetAsync(h->P, 0, kNumParams * 4, ctx->stream);
  cudaMemsetAsync(h->Mo, 0, kNumParams * 4, ctx->stream);
  cudaMemsetAsync(h->Ve, 0, kNumParams * 4, ctx->stream);
  cudaMemsetAsync(h->err, 0, 4, ctx->stream);
  cudaMemsetAsync(h->img, 0, kImgBytes, ctx->stream);
  // the fused inference kernel's shared memory, set here once (not inside a graph capture)
  ITS_CU(ctx, cudaFuncSetAttribute(kMlpForwardFused, cudaFuncAttributeMaxDynamicSharedMemorySize, kFusedSmem));
  *out = h;
  return ITS_OK;
}

its_status its_mlp_free(its_mlp* h) {
  if (!h) return ITS_ERR_INVALID;
  cudaStreamSynchronize(h->ctx->stream);
  for (void* p : h->allocs) devFree(h->ctx, p);
  delete h;
  return ITS_OK;
}

int64_t its_mlp_num_params(void) { return kNumParams; }

its_status its_mlp_set_params(its_mlp* h, const float* params) {
  if (!h || !params) return ITS_ERR_INVALID;
  ITS_CU(h->ctx, cudaMemcpyAsync(h->P, params, kNumParams * 4, cudaMemcpyDefault, h->ctx->stream));
  ITS_CU(h->ctx, cudaMemsetAsync(h->Mo, 0, kNumParams * 4, h->ctx->stream));
  ITS_CU(h->ctx, cudaMemsetAsync(h->Ve, 0, kNumParams * 4, h->ctx->stream));
  h->step = 0;
  its_status s = mlpCast(h);
  if (s != ITS_OK) return s;
  ITS_CU(h->ctx, cudaStreamSynchronize(h->ctx->stream));
  return ITS_OK;
}

its_status its_mlp_get_params(its_mlp* h, float* params) {
  if (!h || !params) return ITS_ERR_INVALID;
  ITS_CU(h->ctx, cudaMemcpyAsync(params, h->P, kNumParams * 4, cudaMemcpyDefault, h->ctx->stream));
  ITS_CU(h->ctx, cudaStreamSynchronize(h->ctx->stream));
  return ITS_OK;
}

// Predictions for n rows of features (n x 64 FP32, normalised), host or device memory.
its_status its_mlp_forward(its_mlp* h, const float* X, int64_t n, float* out) {
  if (!h || (n > 0 && (!X || !out)) || n < 0) return ITS_ERR_INVALID;
  its_ctx* ctx = h->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<float> x;
  OutArg<float> o;
  its_status st;
  if ((st = x.stage(ctx, X, n * kIn)) != ITS_OK) return st;
  if ((st = o.stage(ctx, out, n)) != ITS_OK) return st;
  if ((st = mlpInfer(h, x.d, n, o.d, false)) != ITS_OK) return st;
  if ((st = o.finish(ctx)) != ITS_OK) return st;
  return checkErr(h);
}

// The same predictions for device rows, queued on the context's stream without waiting; a
// tensor-core wait that ran out is reported by the next its_mlp_check (the flag is sticky).
its_status its_mlp_forward_async(its_mlp* h, const float* X, int64_t n, float* out) {
  if (!h || (n > 0 && (!X || !out)) || n < 0) return ITS_ERR_INVALID;
  its_ctx* ctx = h->ctx;
  if (n > 0 && (!isDevicePtr(ctx, X) || !isDevicePtr(ctx, out)))
    return setError(ctx, ITS_ERR_INVALID, "its_mlp_forward_async: features and output must be device memory");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  return mlpInfer(h, X, n, out, false);
}

its_status its_mlp_forward_tiles_async(its_mlp* h, const void* tiles, int64_t n, float* out, int after_kernel) {
  if (!h || (n > 0 && (!tiles || !out)) || n < 0) return ITS_ERR_INVALID;
  its_ctx* ctx = h->ctx;
  if (n > 0 && (!isDevicePtr(ctx, tiles) || !isDevicePtr(ctx, out) || ((uintptr_t)tiles & 15)))
    return setError(ctx, ITS_ERR_INVALID,
                    "its_mlp_forward_tiles_async: tiles (16-byte aligned) and output must be device memory");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  return mlpInferTiles(h, (const bf16*)tiles, n, out, nullptr, 0.0f, 0.0f, nullptr, after_kernel != 0);
}

// Waits for the context's stream and reports the network's error flag.
its_status its_mlp_check(its_mlp* h) {
  if (!h) return ITS_ERR_INVALID;
  ITS_CU(h->ctx, cudaSetDevice(h->ctx->device));
  return checkErr(h);
}

// The same predictions layer by layer (the training kernels' forward); identical to
// its_mlp_forward bit for bit (a test hook).
its_status its_mlp_forward_layers(its_mlp* h, const float* X, int64_t n, float* out) {
  if (!h || (n > 0 && (!X || !out)) || n < 0) return ITS_ERR_INVALID;
  its_ctx* ctx = h->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<float> x;
  OutArg<float> o;
  its_status st;
  if ((st = x.stage(ctx, X, n * kIn)) != ITS_OK) return st;
  if ((st = o.stage(ctx, out, n)) != ITS_OK) return st;
  for (int64_t r0 = 0; r0 < n; r0 += h->cap) {
    const int64_t rows = n - r0 < h->cap ? n - r0 : h->cap;
    kFeaturesBf16<<<gridFor(rows * kIn, 256), 256, 0, ctx->stream>>>(x.d + r0 * kIn, rows, h->Xb, nullptr, 0);
    ITS_LAUNCHED(ctx);
    if ((st = mlpForward(h, rows, false, nullptr, o.d + r0)) != ITS_OK) return st;
  }
  if ((st = o.finish(ctx)) != ITS_OK) return st;
  return checkErr(h);
}

// Gradient of the mean squared error over n rows (n <= batch, a multiple of 64; no update):
// grad has its_mlp_num_params() entries; loss may be NULL.
its_status its_mlp_gradient(its_mlp* h, const float* X, const float* y, int64_t n, float* grad, float* loss) {
  if (!h || !X || !y || !grad || n <= 0 || n > h->cap || n % 64) return ITS_ERR_INVALID;
  its_ctx* ctx = h->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<float> x, yy;
  its_status st;
  if ((st = x.stage(ctx, X, n * kIn)) != ITS_OK) return st;
  if ((st = yy.stage(ctx, y, n)) != ITS_OK) return st;
  // columns of the transposed operands are laid out with the batch capacity as leading size
  kFeaturesBf16<<<gridFor(n * kIn, 256), 256, 0, ctx->stream>>>(x.d, n, h->Xb, h->Xt, h->cap);
  ITS_LAUNCHED(ctx);
  ITS_CU(ctx, cudaMemcpyAsync(h->yb, yy.d, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
  if ((st = mlpGradient(h, n)) != ITS_OK) return st;
  ITS_CU(ctx, cudaMemcpyAsync(grad, h->G, kNumParams * 4, cudaMemcpyDefault, ctx->stream));
  if (loss) ITS_CU(ctx, cudaMemcpyAsync(loss, h->loss, 4, cudaMemcpyDefault, ctx->stream));
  return checkErr(h);
}

// steps Adam steps on random batches (batch = capacity) of a resident dataset (n x 64
// normalised features, n targets; host or device). loss_curve (may be NULL) gets the
// mean squared error of every step.
its_status its_mlp_train(its_mlp* h, const float* X, const float* y, int64_t n, int64_t steps, float lr,
                         uint64_t seed, float* loss_curve) {
  if (!h || !X || !y || n <= 0 || steps < 0) return ITS_ERR_INVALID;
  its_ctx* ctx = h->ctx;
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  InArg<float> x, yy;
  its_status st;
  if ((st = x.stage(ctx, X, n * kIn)) != ITS_OK) return st;
  if ((st = yy.stage(ctx, y, n)) != ITS_OK) return st;
  DevBuf<float> curve;
  if ((st = curve.alloc(ctx, steps > 0 ? steps : 1)) != ITS_OK) return st;
  for (int64_t s = 0; s < steps; ++s) {
    kGatherBatch<<<gridFor(h->cap, 256), 256, 0, ctx->stream>>>(x.d, yy.d, n, seed, (uint64_t)s, h->cap, h->Xb, h->Xt,
                                                               h->yb);
    ITS_LAUNCHED(ctx);
    if ((st = mlpGradient(h, h->cap)) != ITS_OK) return st;
    if ((st = mlpAdam(h, lr)) != ITS_OK) return st;
    ITS_CU(ctx, cudaMemcpyAsync(curve.p + s, h->loss, 4, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  if (loss_curve && steps > 0)
    ITS_CU(ctx, cudaMemcpyAsync(loss_curve, curve.p, steps * 4, cudaMemcpyDefault, ctx->stream));
  return checkErr(h);
}

}  // extern "C"
