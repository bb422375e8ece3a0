// The project's autotuner: launch shapes picked by measurement.
//
// A tunable launch names its shape key (kernel, data type and the sizes that matter) and
// its candidates. With tuning off the built-in default runs. With tuning on, the first call
// for a key runs every candidate once to warm it, times two runs of each with CUDA events on
// the context's stream, keeps the fastest, and records the choice in the context (and in the
// cache file, when one is set, so that later processes start tuned). Only result-neutral
// choices are tuned -- every candidate computes the same bits -- so tuning never changes an
// output, only how fast it is produced.
#pragma once
#include <cstdio>
#include <string>

#include "its_ctx.cuh"

namespace its {

void saveTuneCache(its_ctx* ctx);

// The candidate to use for `key` (0..n-1). run(i) launches candidate i on ctx->stream.
template <class Run>
its_status tuneChoice(its_ctx* ctx, const std::string& key, int n, int def, Run&& run, int* choice) {
  auto it = ctx->tuned.find(key);
  if (it != ctx->tuned.end() && it->second >= 0 && it->second < n) {
    *choice = it->second;
    return ITS_OK;
  }
  if (!ctx->autotune || n <= 1) {
    *choice = def;
    return ITS_OK;
  }
  // inside a stream capture nothing can be timed: the default, until an uncaptured call tunes
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    *choice = def;
    return ITS_OK;
  }
  cudaEvent_t e0, e1;
  ITS_CU(ctx, cudaEventCreate(&e0));
  ITS_CU(ctx, cudaEventCreate(&e1));
  int best = def;
  float bestMs = 3.4e38f;
  its_status st = ITS_OK;
  for (int i = 0; i < n && st == ITS_OK; ++i) {
    if ((st = run(i)) != ITS_OK) break;  // warm-up
    cudaEventRecord(e0, ctx->stream);
    for (int r = 0; r < 2 && st == ITS_OK; ++r) st = run(i);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (st == ITS_OK && ms < bestMs) {
      bestMs = ms;
      best = i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != ITS_OK) return st;
  ctx->tuned[key] = best;
  saveTuneCache(ctx);
  *choice = best;
  return ITS_OK;
}

}  // namespace its
