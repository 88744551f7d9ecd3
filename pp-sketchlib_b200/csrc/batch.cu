// batch.cu -- batched persistent launches under CUDA graphs, and the tile-shape
// autotuner.
//
// A batch turns many independent distance jobs (different databases, sample
// counts, k-mer sets, sketch widths, all-vs-all or query-vs-reference) into one
// work list consumed by one persistent launch of the distance kernel, captured
// once in a CUDA graph and replayed.  The reference has no counterpart: it runs
// one blocking dispatchDists per job (src/gpu/dist.cu:408-489).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <fstream>
#include <vector>

#include "sk_runtime.h"

using namespace sk;

struct sk_batch {
  sk_ctx *ctx = nullptr;
  Plan plan;
  std::vector<JobParams> jobs;
  LaunchBuffers buf;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t pairs = 0;
};

namespace {

void free_buffers(LaunchBuffers &b) {
  if (b.meta) cudaFree(b.meta);
  if (b.cta) cudaFree(b.cta);
  if (b.split) cudaFree(b.split);
  b = LaunchBuffers{};
}

// The tile shape a batch uses: the context's forced shape, else the tuned
// shape of the class holding the most pair-block work, else the default.
const TileConfig *batch_config(sk_ctx *ctx, const std::vector<JobParams> &jobs,
                               const std::vector<int> &s64) {
  if (ctx->tile_cfg > 0) return tile_config(ctx->tile_cfg);
  std::map<std::pair<int, int>, double> work;
  for (size_t j = 0; j < jobs.size(); ++j)
    work[{jobs[j].n_kmers, s64[j]}] +=
        static_cast<double>(jobs[j].n_rows) * jobs[j].n_cols * jobs[j].n_kmers * jobs[j].nb;
  std::pair<int, int> top{0, 0};
  double best = -1;
  for (auto &w : work)
    if (w.second > best) {
      best = w.second;
      top = w.first;
    }
  auto it = ctx->tuning.find(top);
  if (it != ctx->tuning.end() && tile_config(it->second)) return tile_config(it->second);
  return tile_config(1);
}

// Builds one JobParams per job with the given tile shape.
sk_status build_jobs(sk_ctx *ctx, const sk_job *in, int n, const TileConfig &cfg,
                     std::vector<JobParams> &jobs, int64_t *pairs) {
  jobs.resize(n);
  *pairs = 0;
  for (int j = 0; j < n; ++j) {
    if (!in[j].out) return fail(ctx, SK_EINVAL, "job %d has no output buffer", j);
    if (in[j].out_mode != SK_OUT_CORE_ACC && in[j].out_mode != SK_OUT_JACCARD &&
        in[j].out_mode != SK_OUT_COUNTS)
      return fail(ctx, SK_EINVAL, "job %d: unknown output mode %d", j, in[j].out_mode);
    const TileConfig *used = nullptr;
    const int saved = ctx->tile_cfg;
    ctx->tile_cfg = cfg.id;   // build_job plans tiles for the batch's shape
    sk_status st = build_job(ctx, in[j].ref, in[j].query, in[j].random, in[j].out_mode, 0,
                             in[j].out, &used, &jobs[j]);
    ctx->tile_cfg = saved;
    if (st == SK_OK) st = attach_count_tables(ctx, &jobs[j]);
    if (st != SK_OK) return st;
    *pairs += n_pairs(in[j].ref, in[j].query);
  }
  return SK_OK;
}

// Times `repeats` launches of the plan (after one warm-up), in milliseconds.
sk_status time_plan(sk_ctx *ctx, const Plan &plan, const LaunchBuffers &buf, int repeats,
                    float *ms) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  sk_status st = enqueue_plan(ctx, plan, buf);
  cudaEventRecord(e0, ctx->stream);
  for (int r = 0; st == SK_OK && r < repeats; ++r) st = enqueue_plan(ctx, plan, buf);
  cudaEventRecord(e1, ctx->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != SK_OK) return st;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "autotune timing");
  *ms = t / std::max(1, repeats);
  return SK_OK;
}

}  // namespace

extern "C" {

sk_status sk_batch_create(sk_ctx *ctx, const sk_job *jobs, int32_t n_jobs, int32_t flags,
                          sk_batch **out) {
  if (!ctx) return SK_EINVAL;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  DeviceGuard g(ctx->device);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (!out || !jobs || n_jobs < 1) return fail(ctx, SK_EINVAL, "empty batch");
  *out = nullptr;
  std::vector<int> s64(n_jobs);
  for (int j = 0; j < n_jobs; ++j) {
    if (!jobs[j].ref) return fail(ctx, SK_EINVAL, "job %d has no reference database", j);
    s64[j] = jobs[j].ref->s64;
  }

  const TileConfig *cfg = nullptr;
  if (flags & SK_BATCH_AUTOTUNE) {
    // time every shape on the whole batch (results land in the real outputs)
    float best_ms = -1.0f;
    for (int id = 1; id <= tile_config_count(); ++id) {
      const TileConfig *c = tile_config(id);
      std::vector<JobParams> jp;
      int64_t pairs = 0;
      st = build_jobs(ctx, jobs, n_jobs, *c, jp, &pairs);
      if (st != SK_OK) return st;
      Plan plan;
      st = make_plan(ctx, jp, *c, plan);
      if (st != SK_OK) continue;
      LaunchBuffers buf;
      st = upload_plan(ctx, jp, plan, buf, false);
      if (st != SK_OK) return st;
      float ms = 0.0f;
      st = time_plan(ctx, plan, buf, 2, &ms);
      if (st != SK_OK) return st;
      if (best_ms < 0 || ms < best_ms) {
        best_ms = ms;
        cfg = c;
      }
    }
    st = finish_call(ctx);
    if (st != SK_OK) return st;
  } else {
    std::vector<JobParams> probe;
    int64_t pairs = 0;
    st = build_jobs(ctx, jobs, n_jobs, *tile_config(1), probe, &pairs);
    if (st != SK_OK) return st;
    cfg = batch_config(ctx, probe, s64);
  }
  if (!cfg) return fail(ctx, SK_ENOTSUP, "no tile configuration fits the device");

  sk_batch *b = new sk_batch();
  b->ctx = ctx;
  st = build_jobs(ctx, jobs, n_jobs, *cfg, b->jobs, &b->pairs);
  if (st == SK_OK) st = make_plan(ctx, b->jobs, *cfg, b->plan);
  if (st == SK_OK) st = upload_plan(ctx, b->jobs, b->plan, b->buf, true);
  if (st == SK_OK) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess)
      e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      st = enqueue_plan(ctx, b->plan, b->buf);
      cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &b->graph);
      if (st == SK_OK && e2 != cudaSuccess) st = cuda_fail(ctx, e2, "graph capture");
    } else {
      st = cuda_fail(ctx, e, "graph capture");
    }
    if (st == SK_OK) {
      e = cudaGraphInstantiate(&b->exec, b->graph, 0);
      if (e != cudaSuccess) st = cuda_fail(ctx, e, "graph instantiation");
    }
  }
  if (st != SK_OK) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    free_buffers(b->buf);
    delete b;
    return st;
  }
  ctx_retain(ctx);
  *out = b;
  return SK_OK;
}

sk_status sk_batch_launch(sk_batch *b) {
  if (!b) return SK_EINVAL;
  sk_ctx *ctx = b->ctx;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  DeviceGuard g(ctx->device);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  cudaError_t e = cudaGraphLaunch(b->exec, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "graph launch");
  return SK_OK;
}

sk_status sk_batch_run(sk_batch *b) {
  sk_status st = sk_batch_launch(b);
  if (st != SK_OK) return st;
  std::lock_guard<std::recursive_mutex> lock(b->ctx->mu);
  DeviceGuard g(b->ctx->device);
  return finish_call(b->ctx);
}

sk_status sk_batch_info(const sk_batch *b, int32_t *tile_config_id, int32_t *grid,
                        int64_t *n_items, int64_t *n_pairs_out) {
  if (!b) return SK_EINVAL;
  if (tile_config_id) *tile_config_id = b->plan.cfg->id;
  if (grid) *grid = b->plan.grid;
  if (n_items) *n_items = static_cast<int64_t>(b->plan.items.size());
  if (n_pairs_out) *n_pairs_out = b->pairs;
  return SK_OK;
}

sk_status sk_batch_destroy(sk_batch *b) {
  if (!b) return SK_EINVAL;
  sk_ctx *ctx = b->ctx;
  {
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    free_buffers(b->buf);
  }
  delete b;
  ctx_release(ctx);
  return SK_OK;
}

sk_status sk_autotune(sk_ctx *ctx, const sk_db *ref, const sk_db *query, const sk_random *random,
                      int32_t repeats, int32_t *best_config) {
  if (!ctx) return SK_EINVAL;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  DeviceGuard g(ctx->device);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (!ref) return fail(ctx, SK_EINVAL, "No reference database");
  const int64_t pairs = n_pairs(ref, query);
  void *d_out = nullptr;
  st = scratch(ctx, kSlotOut, std::max<int64_t>(pairs, 1) * 8, &d_out);
  if (st != SK_OK) return st;
  sk_job job{ref, query, random, SK_OUT_CORE_ACC, d_out};
  float best_ms = -1.0f;
  int best = 0;
  for (int id = 1; id <= tile_config_count(); ++id) {
    const TileConfig *c = tile_config(id);
    std::vector<JobParams> jp;
    int64_t p = 0;
    st = build_jobs(ctx, &job, 1, *c, jp, &p);
    if (st != SK_OK) return st;
    Plan plan;
    if (make_plan(ctx, jp, *c, plan) != SK_OK) continue;
    LaunchBuffers buf;
    st = upload_plan(ctx, jp, plan, buf, false);
    if (st != SK_OK) return st;
    float ms = 0.0f;
    st = time_plan(ctx, plan, buf, std::max(1, repeats), &ms);
    if (st != SK_OK) return st;
    if (best_ms < 0 || ms < best_ms) {
      best_ms = ms;
      best = id;
    }
  }
  st = finish_call(ctx);
  if (st != SK_OK) return st;
  if (best == 0) return fail(ctx, SK_ENOTSUP, "no tile configuration fits the device");
  ctx->tuning[{ref->K, ref->s64}] = best;
  if (best_config) *best_config = best;
  return SK_OK;
}

sk_status sk_ctx_save_tuning(sk_ctx *ctx, const char *path) {
  if (!ctx || !path) return SK_EINVAL;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  std::ofstream o(path);
  if (!o) return fail(ctx, SK_EINVAL, "Cannot write tuning table %s", path);
  o << "# n_kmers sketchsize64 tile_config  (written by sk_autotune)\n";
  for (auto &t : ctx->tuning) o << t.first.first << " " << t.first.second << " " << t.second << "\n";
  return SK_OK;
}

}  // extern "C"
