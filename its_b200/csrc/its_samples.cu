// Shell samples on the GPU (replaces ThinShells::cpIntersectionPoints, ThinShells.cpp:38-479).
//
// Edge step (ThinShells.cpp:66-143): every unique mesh edge is tested against the min-x /
// min-y / min-z faces of the fine nodes in its voxel box grown by one; hits are kept once
// (exact duplicates removed). Unique edges and unique points come from open-addressing hash
// sets keyed on the exact bits; the first occurrence (lowest index) wins, so the output is
// deterministic.
// Face step (ThinShells.cpp:158-369): the reference sweeps, per triangle and axis, every fine
// edge whose axial span overlaps the triangle's box (within 1e-9) and keeps plane hits that
// pass the inside-triangle test. A hit lies inside the triangle, so the edge's two lateral
// coordinates lie in the triangle's box; candidates are therefore enumerated on the fine
// lattice lines of the box (and along the axis one cell either side of it, for the sweep's
// tolerance) and checked against the fine-edge bitmap, then the reference's own window and
// intersection tests decide. Same points, no slab sweep. Each step tests every item once to
// count its hits and again only where it has hits, to write them.
#include <algorithm>
#include <cmath>

#include "its_scan.cuh"
#include "its_svo.cuh"

namespace its {

// ---- exact hash sets -----------------------------------------------------------------------
__device__ inline uint64_t mix64(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}
constexpr unsigned long long kEmpty = ~0ull;

// Insert key (never kEmpty); keep the minimum owner index per key. Bounded probing: the
// table is at least twice the number of keys, so a free slot is always found.
__device__ inline void setInsertMin(unsigned long long* keys, unsigned* owner, uint64_t mask, unsigned long long key,
                                    unsigned idx) {
  uint64_t h = mix64(key) & mask;
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const unsigned long long prev = atomicCAS(keys + h, kEmpty, key);
    if (prev == kEmpty || prev == key) {
      atomicMin(owner + h, idx);
      return;
    }
    h = (h + 1) & mask;
  }
}
__device__ inline unsigned setOwner(const unsigned long long* keys, const unsigned* owner, uint64_t mask,
                                    unsigned long long key) {
  uint64_t h = mix64(key) & mask;
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const unsigned long long k = keys[h];
    if (k == key) return owner[h];
    if (k == kEmpty) return 0xFFFFFFFFu;
    h = (h + 1) & mask;
  }
  return 0xFFFFFFFFu;
}

__device__ inline unsigned long long edgeKeyOf(const int32_t* F, int64_t slot) {
  const int64_t t = slot / 3;
  const int k = (int)(slot % 3);
  const int32_t a = F[3 * t + k], b = F[3 * t + (k + 1) % 3];
  const uint32_t lo = (uint32_t)(a < b ? a : b), hi = (uint32_t)(a < b ? b : a);
  return ((unsigned long long)lo << 32) | hi;
}
__global__ void kEdgeInsert(const int32_t* __restrict__ F, int64_t slots, unsigned long long* keys, unsigned* owner,
                            uint64_t mask) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s < slots) setInsertMin(keys, owner, mask, edgeKeyOf(F, s), (unsigned)s);
}

struct SampleParams {
  double3 g;
  double w0;
  int res;
  const unsigned long long* fineOcc;
  const uint32_t* morton;
  int64_t fineCount;
  const unsigned long long* ebits;
  const uint32_t* erank;
  const uint32_t* edgeOwner;
};

__device__ inline bool inRange(double l, double r, double q) { return l <= q && q <= r; }
__device__ inline bool isLargeDouble(double l, double r) { return !(fabs(l - r) < 1e-9) && l > r; }

// Edge-step hits of mesh edge (p1,p2); emit == nullptr only counts.
__device__ int edgeHits(const SampleParams& S, const double* p1, const double* p2, double* emit) {
  const double dir[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
  const double org[3] = {S.g.x, S.g.y, S.g.z};
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    const int d1 = (int)((p1[a] - org[a]) / S.w0), d2 = (int)((p2[a] - org[a]) / S.w0);
    lo[a] = clampi((d1 < d2 ? d1 : d2) - 1, 0, S.res - 1);
    hi[a] = clampi((d1 > d2 ? d1 : d2) + 1, 0, S.res - 1);
  }
  int n = 0;
  for (int z = lo[2]; z <= hi[2]; ++z)
    for (int y = lo[1]; y <= hi[1]; ++y)
      for (int x = lo[0]; x <= hi[0]; ++x) {
        const uint32_t m = mortonEncode(x, y, z);
        if (!((S.fineOcc[m >> 6] >> (m & 63)) & 1ull)) continue;
        const double lbb[3] = {latticePos(org[0], S.w0, x), latticePos(org[1], S.w0, y), latticePos(org[2], S.w0, z)};
        const double w = S.w0;
        double tt[3];
        for (int a = 0; a < 3; ++a) tt[a] = dir[a] != 0 ? (lbb[a] - p1[a]) / dir[a] : 1.7976931348623157e308;
        for (int a = 0; a < 3; ++a) {  // back (x), left (y), bottom (z) planes
          if (!inRange(0.0, 1.0, tt[a])) continue;
          double q[3];
          for (int c = 0; c < 3; ++c) q[c] = p1[c] + tt[a] * dir[c];
          const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
          if (inRange(lbb[b], lbb[b] + w, q[b]) && inRange(lbb[c], lbb[c] + w, q[c])) {
            if (emit) { emit[3 * n] = q[0]; emit[3 * n + 1] = q[1]; emit[3 * n + 2] = q[2]; }
            ++n;
          }
        }
      }
  return n;
}

struct EdgeStep {
  SampleParams S;
  const double* V;
  const int32_t* F;
  const unsigned long long* keys;
  const unsigned* owner;
  uint64_t mask;
  __device__ bool isUnique(int64_t slot) const { return setOwner(keys, owner, mask, edgeKeyOf(F, slot)) == (unsigned)slot; }
  __device__ uint32_t operator()(int64_t slot) const {
    if (!isUnique(slot)) return 0;
    const unsigned long long key = edgeKeyOf(F, slot);
    const uint32_t a = (uint32_t)(key >> 32), b = (uint32_t)(key & 0xffffffffu);
    return (uint32_t)edgeHits(S, V + 3 * a, V + 3 * b, nullptr);
  }
};
struct EdgeEmit {
  EdgeStep es;
  double* out;
  __device__ void operator()(int64_t slot, uint32_t prefix, uint32_t count) const {
    if (!count) return;
    const unsigned long long key = edgeKeyOf(es.F, slot);
    const uint32_t a = (uint32_t)(key >> 32), b = (uint32_t)(key & 0xffffffffu);
    edgeHits(es.S, es.V + 3 * a, es.V + 3 * b, out + 3 * (int64_t)prefix);
  }
};

// Exact-duplicate removal of points: key = hash of the three coordinates' bits, owner =
// first index; a point is kept when it owns its key and matches its owner's coordinates (a
// rare 64-bit hash collision between different points keeps both).
__device__ inline unsigned long long pointKey(const double* p) {
  unsigned long long h = mix64(__double_as_longlong(p[0]));
  h = mix64(h ^ (unsigned long long)__double_as_longlong(p[1]));
  h = mix64(h ^ (unsigned long long)__double_as_longlong(p[2]));
  return h == kEmpty ? 0 : h;
}
__global__ void kPointInsert(const double* __restrict__ P, int64_t m, unsigned long long* keys, unsigned* owner,
                             uint64_t mask) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) setInsertMin(keys, owner, mask, pointKey(P + 3 * i), (unsigned)i);
}
struct PointKeep {
  const double* P;
  const unsigned long long* keys;
  const unsigned* owner;
  uint64_t mask;
  __device__ uint32_t operator()(int64_t i) const {
    const unsigned o = setOwner(keys, owner, mask, pointKey(P + 3 * i));
    if (o == (unsigned)i) return 1;
    const double* q = P + 3 * (int64_t)o;
    const double* p = P + 3 * i;
    return (q[0] == p[0] && q[1] == p[1] && q[2] == p[2]) ? 0 : 1;
  }
};
struct PointCompact {
  PointKeep keep;
  double* out;
  __device__ void operator()(int64_t i, uint32_t prefix, uint32_t v) const {
    if (!v) return;
    for (int c = 0; c < 3; ++c) out[3 * (int64_t)prefix + c] = keep.P[3 * i + c];
  }
};

// ---- face step -------------------------------------------------------------------------------
// Owner-derived end points of a fine edge (the representative kept by the reference's sort).
__device__ inline void fineEdgeEnds(const SampleParams& S, uint32_t X, uint32_t Y, uint32_t Z, int axis, uint32_t rank,
                                    double* e1, double* e2) {
  uint32_t Xo, Yo, Zo;
  mortonDecode(S.morton[S.edgeOwner[rank]], Xo, Yo, Zo);
  const double w = S.w0;
  const double base[3] = {latticePos(S.g.x, w, Xo), latticePos(S.g.y, w, Yo), latticePos(S.g.z, w, Zo)};
  const uint32_t st[3] = {X, Y, Z}, o[3] = {Xo, Yo, Zo};
  for (int a = 0; a < 3; ++a) {
    e1[a] = st[a] != o[a] ? base[a] + w : base[a];
    const uint32_t en = st[a] + (a == axis ? 1u : 0u);
    e2[a] = en != o[a] ? base[a] + w : base[a];
  }
}

__device__ int faceHits(const SampleParams& S, const double* V, const int32_t* F, int64_t t, double* emit) {
  const int32_t ia = F[3 * t], ib = F[3 * t + 1], ic = F[3 * t + 2];
  const double p1[3] = {V[3 * ia], V[3 * ia + 1], V[3 * ia + 2]};
  const double p2[3] = {V[3 * ib], V[3 * ib + 1], V[3 * ib + 2]};
  const double p3[3] = {V[3 * ic], V[3 * ic + 1], V[3 * ic + 2]};
  // triangle attributes as modelTriAttributeKernel (CUDACompute.cu:79-96)
  const double u[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
  const double v[3] = {p3[0] - p1[0], p3[1] - p1[1], p3[2] - p1[2]};
  const double tn[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
  double tdir = -tn[0] * p1[0];
  tdir = tdir + -tn[1] * p1[1];
  tdir = tdir + -tn[2] * p1[2];
  const double te1[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
  const double te2[3] = {p3[0] - p2[0], p3[1] - p2[1], p3[2] - p2[2]};
  const double te3[3] = {p1[0] - p3[0], p1[1] - p3[1], p1[2] - p3[2]};
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = dmin(p1[a], dmin(p2[a], p3[a]));
    hi[a] = dmax(p1[a], dmax(p2[a], p3[a]));
  }
  const double org[3] = {S.g.x, S.g.y, S.g.z};
  const uint32_t M = (uint32_t)S.res + 1u;
  int fl[3], fh[3];
  for (int a = 0; a < 3; ++a) {
    fl[a] = (int)floor((lo[a] - org[a]) / S.w0);
    fh[a] = (int)floor((hi[a] - org[a]) / S.w0);
  }
  auto dot3 = [](const double* a, const double* b) {
    double s = a[0] * b[0];
    s = s + a[1] * b[1];
    return s + a[2] * b[2];
  };
  auto insideTest = [&](const double* te, const double* pv, const double* ip) {
    const double d[3] = {ip[0] - pv[0], ip[1] - pv[1], ip[2] - pv[2]};
    const double c[3] = {te[1] * d[2] - te[2] * d[1], te[2] * d[0] - te[0] * d[2], te[0] * d[1] - te[1] * d[0]};
    return dot3(c, tn) >= 0;
  };
  int n = 0;
  for (int axis = 0; axis < 3; ++axis) {
    const uint32_t ord = axis == 2 ? 0u : (axis == 1 ? 1u : 2u);
    // Candidate fine edges along the axis. Along it: those whose span can meet the sweep window
    // [lo - 1e-9, hi + 1e-9] (start cells floor(lo) - 1 .. floor(hi) + 1). Across it: a hit is
    // the edge's own lateral coordinates (the edge direction has no lateral component) and lies
    // in the triangle, so the lattice lines in [lo, hi] to rounding: floor(lo) .. floor(hi) + 1.
    // (A cell quotient's rounding moves a floor by at most one, toward lines a cell outside.)
    int l0[3], l1[3];
    for (int a = 0; a < 3; ++a) {
      const int c0 = a == axis ? fl[a] - 1 : fl[a], c1 = fh[a] + 1;
      l0[a] = c0 < 0 ? 0 : c0;
      l1[a] = c1 > S.res ? S.res : c1;
    }
    if (l1[axis] > S.res - 1) l1[axis] = S.res - 1;  // edge start along its axis
    for (int X = l0[0]; X <= l1[0]; ++X)
      for (int Y = l0[1]; Y <= l1[1]; ++Y)
        for (int Z = l0[2]; Z <= l1[2]; ++Z) {
          const uint32_t key = (((uint32_t)X * M + (uint32_t)Y) * M + (uint32_t)Z) * 3u + ord;
          const unsigned long long wbits = S.ebits[key >> 6];
          if (!((wbits >> (key & 63)) & 1ull)) continue;
          const uint32_t rank = S.erank[key >> 6] + (uint32_t)__popcll(wbits & ((1ull << (key & 63)) - 1ull));
          double e1[3], e2[3];
          fineEdgeEnds(S, X, Y, Z, axis, rank, e1, e2);
          // the reference's sweep window on this axis (lower_bound / break, 1e-9 tolerance)
          if (isLargeDouble(lo[axis], e2[axis])) continue;
          if (isLargeDouble(e1[axis], hi[axis])) continue;
          const double ed[3] = {e2[0] - e1[0], e2[1] - e1[1], e2[2] - e1[2]};
          const double nd = dot3(tn, ed);
          if ((double)fabsf((float)nd) < 1e-9) continue;  // fabsf on a double, ThinShells.cpp:268
          const double tt = (-tdir - dot3(tn, e1)) / nd;
          if (tt < 0. || tt > 1.) continue;
          const double ip[3] = {e1[0] + ed[0] * tt, e1[1] + ed[1] * tt, e1[2] + ed[2] * tt};
          if (!insideTest(te1, p1, ip)) continue;
          if (!insideTest(te2, p2, ip)) continue;
          if (!insideTest(te3, p3, ip)) continue;
          if (emit) { emit[3 * n] = ip[0]; emit[3 * n + 1] = ip[1]; emit[3 * n + 2] = ip[2]; }
          ++n;
        }
  }
  return n;
}
struct FaceStep {
  SampleParams S;
  const double* V;
  const int32_t* F;
  __device__ uint32_t operator()(int64_t t) const { return (uint32_t)faceHits(S, V, F, t, nullptr); }
};
struct FaceEmit {
  FaceStep fs;
  double* out;
  __device__ void operator()(int64_t t, uint32_t prefix, uint32_t count) const {
    if (count) faceHits(fs.S, fs.V, fs.F, t, out + 3 * (int64_t)prefix);
  }
};

// The hit count of every item, evaluated once and stored; the scan of the stored counts writes
// each item's offset, and the emitting pass re-runs the hit test, one thread per item, only for
// items that have hits, writing them at that offset.
template <class Step>
__global__ void __launch_bounds__(128) kCountHits(Step f, int64_t n, uint32_t* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) cnt[i] = f(i);
}
template <class Emit>
__global__ void __launch_bounds__(128) kEmitHits(Emit e, int64_t n, const uint32_t* __restrict__ cnt,
                                                 const uint32_t* __restrict__ off) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = cnt[i];
  if (c) e(i, off[i], c);
}
struct StoredCount {
  const uint32_t* cnt;
  __device__ uint32_t operator()(int64_t i) const { return cnt[i]; }
};

static uint64_t tableSize(int64_t keys) {
  uint64_t s = 1024;
  while (s < (uint64_t)(2 * keys)) s <<= 1;
  return s;
}

its_status validateMesh(its_ctx* ctx, const double* dV, int64_t nv, const int32_t* dF, int64_t nf);

}  // namespace its

using namespace its;

extern "C" {

its_status its_shell_samples(its_svo* s, const double* verts, int64_t nverts, const int32_t* faces, int64_t nfaces,
                             double* out_points, int64_t capacity, int64_t* num_points, int64_t* num_edge_points) {
  if (!s || !verts || !faces || nverts <= 0 || nfaces <= 0 || !num_points) return ITS_ERR_INVALID;
  its_ctx* ctx = s->ctx;
  if (nfaces * 3 >= (1ll << 32)) return setError(ctx, ITS_ERR_INVALID, "too many faces");
  ITS_CU(ctx, cudaSetDevice(ctx->device));
  const SvoDevice& d = s->d;
  InArg<double> V;
  InArg<int32_t> F;
  its_status st;
  if ((st = V.stage(ctx, verts, 3 * nverts)) != ITS_OK) return st;
  if ((st = F.stage(ctx, faces, 3 * nfaces)) != ITS_OK) return st;
  if ((st = validateMesh(ctx, V.d, nverts, F.d, nfaces)) != ITS_OK) return st;
  SampleParams S;
  S.g = make_double3(d.origin[0], d.origin[1], d.origin[2]);
  S.w0 = d.unit[0];
  S.res = d.res;
  S.fineOcc = (const unsigned long long*)d.fineOcc;
  S.morton = d.nodeMorton;
  S.fineCount = d.levelCount[0];
  S.ebits = d.ebits;
  S.erank = d.erank;
  S.edgeOwner = d.edgeOwner;

  // unique mesh edges
  const int64_t slots = 3 * nfaces;
  const uint64_t tsz = tableSize(slots);
  DevBuf<unsigned long long> ekeys;
  DevBuf<unsigned> eown;
  if ((st = ekeys.alloc(ctx, tsz)) != ITS_OK) return st;
  if ((st = eown.alloc(ctx, tsz)) != ITS_OK) return st;
  ITS_CU(ctx, cudaMemsetAsync(ekeys.p, 0xFF, tsz * 8, ctx->stream));
  ITS_CU(ctx, cudaMemsetAsync(eown.p, 0xFF, tsz * 4, ctx->stream));
  kEdgeInsert<<<gridFor(slots, 256), 256, 0, ctx->stream>>>(F.d, slots, ekeys.p, eown.p, tsz - 1);
  ITS_LAUNCHED(ctx);
  EdgeStep es{S, V.d, F.d, ekeys.p, eown.p, tsz - 1};
  DevBuf<uint32_t> tot, ecnt, eoff;
  if ((st = tot.zeros(ctx, 3)) != ITS_OK || (st = ecnt.alloc(ctx, slots)) != ITS_OK ||
      (st = eoff.alloc(ctx, slots)) != ITS_OK)
    return st;
  kCountHits<<<gridFor(slots, 128), 128, 0, ctx->stream>>>(es, slots, ecnt.p);
  ITS_LAUNCHED(ctx);
  if ((st = scanExclusiveAlloc<uint32_t>(ctx, StoredCount{ecnt.p}, slots, StorePrefix<uint32_t>{eoff.p}, tot.p)) !=
      ITS_OK)
    return st;
  uint32_t nRaw = 0;
  if ((st = readScalar(ctx, tot.p, &nRaw)) != ITS_OK) return st;
  DevBuf<double> raw;
  if ((st = raw.alloc(ctx, 3 * (size_t)(nRaw ? nRaw : 1))) != ITS_OK) return st;
  kEmitHits<<<gridFor(slots, 128), 128, 0, ctx->stream>>>(EdgeEmit{es, raw.p}, slots, ecnt.p, eoff.p);
  ITS_LAUNCHED(ctx);
  ecnt.reset();
  eoff.reset();
  ekeys.reset();
  eown.reset();
  // exact-duplicate removal
  uint32_t nEdge = 0;
  DevBuf<double> edgePts;
  {
    const uint64_t psz = tableSize(nRaw);
    DevBuf<unsigned long long> pk;
    DevBuf<unsigned> po;
    if ((st = pk.alloc(ctx, psz)) != ITS_OK) return st;
    if ((st = po.alloc(ctx, psz)) != ITS_OK) return st;
    ITS_CU(ctx, cudaMemsetAsync(pk.p, 0xFF, psz * 8, ctx->stream));
    ITS_CU(ctx, cudaMemsetAsync(po.p, 0xFF, psz * 4, ctx->stream));
    if (nRaw) {
      kPointInsert<<<gridFor(nRaw, 256), 256, 0, ctx->stream>>>(raw.p, nRaw, pk.p, po.p, psz - 1);
      ITS_LAUNCHED(ctx);
    }
    PointKeep keep{raw.p, pk.p, po.p, psz - 1};
    if ((st = edgePts.alloc(ctx, 3 * (size_t)(nRaw ? nRaw : 1))) != ITS_OK) return st;
    if ((st = scanExclusiveAlloc<uint32_t>(ctx, keep, nRaw, PointCompact{keep, edgePts.p}, tot.p + 1)) != ITS_OK) return st;
    if ((st = readScalar(ctx, tot.p + 1, &nEdge)) != ITS_OK) return st;
  }
  raw.reset();
  // face step
  FaceStep fs{S, V.d, F.d};
  DevBuf<uint32_t> fcnt, foff;
  if ((st = fcnt.alloc(ctx, nfaces)) != ITS_OK || (st = foff.alloc(ctx, nfaces)) != ITS_OK) return st;
  kCountHits<<<gridFor(nfaces, 128), 128, 0, ctx->stream>>>(fs, nfaces, fcnt.p);
  ITS_LAUNCHED(ctx);
  if ((st = scanExclusiveAlloc<uint32_t>(ctx, StoredCount{fcnt.p}, nfaces, StorePrefix<uint32_t>{foff.p},
                                         tot.p + 2)) != ITS_OK)
    return st;
  uint32_t nFace = 0;
  if ((st = readScalar(ctx, tot.p + 2, &nFace)) != ITS_OK) return st;
  const int64_t total = (int64_t)nEdge + nFace;
  *num_points = total;
  if (num_edge_points) *num_edge_points = nEdge;
  if (!out_points) return ITS_OK;
  if (capacity < 0) return setError(ctx, ITS_ERR_INVALID, "its_shell_samples: negative capacity");
  // the first min(capacity, total) points: straight into the output when it holds them all,
  // else through a full-size scratch
  const int64_t keep = std::min<int64_t>(capacity, total);
  OutArg<double> O;
  if ((st = O.stage(ctx, out_points, 3 * keep)) != ITS_OK) return st;
  DevBuf<double> all;
  double* dst = O.d;
  if (keep < total) {
    if ((st = all.alloc(ctx, 3 * total)) != ITS_OK) return st;
    dst = all.p;
  }
  if (nEdge && dst) ITS_CU(ctx, cudaMemcpyAsync(dst, edgePts.p, (size_t)nEdge * 24, cudaMemcpyDeviceToDevice, ctx->stream));
  if (dst) {
    kEmitHits<<<gridFor(nfaces, 128), 128, 0, ctx->stream>>>(FaceEmit{fs, dst + 3 * (int64_t)nEdge}, nfaces, fcnt.p,
                                                             foff.p);
    ITS_LAUNCHED(ctx);
  }
  if (keep < total && keep > 0)
    ITS_CU(ctx, cudaMemcpyAsync(O.d, all.p, (size_t)keep * 24, cudaMemcpyDeviceToDevice, ctx->stream));
  if ((st = O.finish(ctx)) != ITS_OK) return st;
  ITS_CU(ctx, cudaStreamSynchronize(ctx->stream));
  return ITS_OK;
}

}  // extern "C"
