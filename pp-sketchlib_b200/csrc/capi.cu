// capi.cu -- the C ABI (include/sketchlib_b200.h): contexts, resident sketch
// databases, random-match models and the dense / kNN / sparse entry points.
//
// Host responsibilities mirror the reference's GPU host driver
// (src/gpu/gpu_api.cpp:166-531, src/gpu/dist.cu:326-489): parameter checks
// with the reference's messages, device selection, layout packing (here on the
// device instead of OpenMP flattening on the host), launch planning and result
// copies.  No C++ exception crosses the ABI; errors become sk_status codes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "sk_common.h"
#include "sk_launch.h"
#include "sketchlib_b200.h"
#include "sk_runtime.h"

using namespace sk;

// ------------------------------------------------------------------ helpers

namespace sk {

sk_status fail(sk_ctx *ctx, sk_status st, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return st;
}

sk_status cuda_fail(sk_ctx *ctx, cudaError_t e, const char *what) {
  const sk_status st = (e == cudaErrorMemoryAllocation) ? SK_ENOMEM : SK_ECUDA;
  return fail(ctx, st, "CUDA error in %s: %s", what, cudaGetErrorString(e));
}

static std::mutex g_ctx_refs_mu;

sk_status attach_count_tables(sk_ctx *ctx, JobParams *jp, bool alloc) {
  if (jp->rmode != kRandNone || jp->semantics == kSemRefGpu || jp->out_mode == kOutCounts ||
      jp->nchunk != 1)
    return SK_OK;
  const int64_t bins = static_cast<int64_t>(jp->union_bits);
  std::lock_guard<std::mutex> lock(ctx->count_tables_mu);
  auto it = ctx->count_tables.find(bins);
  if (it == ctx->count_tables.end()) {
    if (!alloc) return SK_OK;
    float *jt = nullptr;
    double *lt = nullptr;
    cudaError_t e = cudaMalloc(&jt, (bins + 1) * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&lt, (bins + 1) * sizeof(double));
    if (e == cudaSuccess) e = launch_count_tables(jp->union_bits, bins + 1, jt, lt, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      if (jt) cudaFree(jt);
      if (lt) cudaFree(lt);
      return cuda_fail(ctx, e, "count tables");
    }
    it = ctx->count_tables.emplace(bins, std::make_pair(jt, lt)).first;
  }
  jp->jtab = it->second.first;
  jp->ltab = it->second.second;
  return SK_OK;
}

static void ctx_free(sk_ctx *ctx) {
  {
    DeviceGuard g(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto &s : ctx->scratch)
      if (s.ptr) cudaFree(s.ptr);
    for (auto &t : ctx->count_tables) {
      cudaFree(t.second.first);
      cudaFree(t.second.second);
    }
    if (ctx->status_dev) cudaFree(ctx->status_dev);
    if (ctx->cancel_host) cudaFreeHost(ctx->cancel_host);
    if (ctx->stream && ctx->own_stream) cudaStreamDestroy(ctx->stream);
    if (ctx->copy_stream) {
      cudaStreamSynchronize(ctx->copy_stream);
      cudaStreamDestroy(ctx->copy_stream);
    }
    for (int b = 0; b < 2; ++b) {
      if (ctx->ev_ready[b]) cudaEventDestroy(ctx->ev_ready[b]);
      if (ctx->ev_free[b]) cudaEventDestroy(ctx->ev_free[b]);
    }
    for (cudaStream_t st : {ctx->stream_b, ctx->pack_stream, ctx->d2h_stream}) {
      if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
      }
    }
    for (cudaEvent_t ev : ctx->ev_chunk) cudaEventDestroy(ev);
    for (cudaEvent_t ev : ctx->ev_out) cudaEventDestroy(ev);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  }
  delete ctx;
}

void ctx_retain(sk_ctx *ctx) {
  std::lock_guard<std::mutex> g(g_ctx_refs_mu);
  ++ctx->refs;
}

void ctx_release(sk_ctx *ctx) {
  bool last = false;
  {
    std::lock_guard<std::mutex> g(g_ctx_refs_mu);
    last = --ctx->refs == 0;
  }
  if (last) ctx_free(ctx);
}

DeviceGuard::DeviceGuard(int dev) {
  cudaGetDevice(&prev_);
  if (prev_ != dev) cudaSetDevice(dev);
}
DeviceGuard::~DeviceGuard() { cudaSetDevice(prev_); }

// Grows the context's device scratch buffer `slot` to at least `bytes`.
sk_status scratch(sk_ctx *ctx, int slot, size_t bytes, void **out) {
  Scratch &s = ctx->scratch[slot];
  if (s.bytes < bytes) {
    if (s.ptr) {
      cudaStreamSynchronize(ctx->stream);
      cudaFree(s.ptr);
      s.ptr = nullptr;
      s.bytes = 0;
    }
    cudaError_t e = cudaMalloc(&s.ptr, bytes);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "scratch allocation");
    s.bytes = bytes;
  }
  *out = s.ptr;
  return SK_OK;
}

// Begins a public call: the context's device becomes current and the cancel
// word and device status are cleared.
sk_status begin_call(sk_ctx *ctx) {
  ctx->err.clear();
  *ctx->cancel_host = 0;
  cudaError_t e = cudaMemsetAsync(ctx->status_dev, 0, sizeof(DevStatus), ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "status reset");
  return SK_OK;
}

// Waits for the context's stream and turns the device status into a code.
sk_status finish_call(sk_ctx *ctx) {
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel execution");
  DevStatus st{};
  e = cudaMemcpy(&st, ctx->status_dev, sizeof(st), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "status readback");
  ctx->last_tiles = st.tiles_done;
  if (st.error & 2u) return fail(ctx, SK_ECANCELLED, "Distance calculation cancelled");
  if (st.error & 1u)
    return fail(ctx, SK_ETIMEDOUT, "A device-side bounded wait timed out (site %u)", st.where);
  if (st.error) return fail(ctx, SK_EKERNEL, "Device error flag 0x%x", st.error);
  return SK_OK;
}

const TileConfig *choose_config(sk_ctx *ctx, int K, int s64) {
  if (ctx->tile_cfg > 0) {
    const TileConfig *c = tile_config(ctx->tile_cfg);
    if (c && c->max_kmers >= K) return c;
  }
  auto it = ctx->tuning.find({K, s64});
  if (it != ctx->tuning.end()) {
    const TileConfig *c = tile_config(it->second);
    if (c && c->max_kmers >= K) return c;
  }
  return tile_config(1);
}

// Upper-triangle / rectangle tile counts for a tile shape.
void plan_tiles(JobParams &jp, const TileConfig &cfg) {
  jp.tile_rows = cfg.tile_rows;
  jp.tile_cols = cfg.tile_cols;
  if (jp.self) {
    const int64_t n = jp.n_rows;
    jp.n_row_tiles = static_cast<int32_t>(n > 1 ? (n - 1 + cfg.tile_rows - 1) / cfg.tile_rows : 0);
    jp.n_col_tiles = static_cast<int32_t>((n + cfg.tile_cols - 1) / cfg.tile_cols);
    const int64_t m = cfg.tile_rows / cfg.tile_cols;
    int64_t tiles = 0;
    for (int64_t ti = 0; ti < jp.n_row_tiles; ++ti) tiles += jp.n_col_tiles - ti * m;
    jp.n_tiles = tiles;
  } else {
    jp.n_row_tiles = static_cast<int32_t>((jp.n_rows + cfg.tile_rows - 1) / cfg.tile_rows);
    jp.n_col_tiles = static_cast<int32_t>((jp.n_cols + cfg.tile_cols - 1) / cfg.tile_cols);
    jp.n_tiles = static_cast<int64_t>(jp.n_row_tiles) * jp.n_col_tiles;
  }
}

// The reference GPU path's equal-base chances: csrs(k, use_rc, l0, l0) with l0
// the first sample's length, narrowed to float (flattened_random,
// src/random/random_match.cpp:278-310; csrs :318-336).
std::vector<float> equal_base_gpu(const sk_db *db, int use_rc) {
  std::vector<float> t(static_cast<size_t>(db->K), 0.0f);
  const double len = static_cast<double>(db->seq_len.empty() ? 0 : db->seq_len[0]);
  for (int k = 0; k < db->K; ++k) {
    const double match_chance = std::ldexp(1.0, (db->kmers[k] - 1) * 2 + (use_rc ? 1 : 0));
    const double j = 1 - std::pow(1 - (double)1 / match_chance, len);
    t[k] = j > 0 ? static_cast<float>((j * j) / (j + j - j * j)) : 0.0f;
  }
  return t;
}

// Equal-base random-match factors j(k, len) = 1 - (1 - 4^-k')^len per sample
// (csrs, src/random/random_match.cpp:318-336), computed with std::pow on the
// host exactly as the reference does: [K][padded samples] doubles.
std::vector<double> equal_base_factors(const sk_db *db, int use_rc) {
  const int64_t ld = static_cast<int64_t>(db->ng) * kGranule;
  std::vector<double> jv(static_cast<size_t>(db->K) * ld, 0.0);
  for (int k = 0; k < db->K; ++k) {
    const int shift = (db->kmers[k] - 1) * 2 + (use_rc ? 1 : 0);
    const double match_chance = std::ldexp(1.0, shift);
    for (int64_t s = 0; s < db->n; ++s) {
      const double len = static_cast<double>(db->seq_len.empty() ? 0 : db->seq_len[s]);
      jv[k * ld + s] = 1 - std::pow(1 - (double)1 / match_chance, len);
    }
  }
  return jv;
}

// The same factors, uploaded and cached on the database.
sk_status ensure_jv(sk_ctx *ctx, sk_db *db, int use_rc) {
  if (db->jv && db->jv_rc == use_rc) return SK_OK;
  const std::vector<double> jv = equal_base_factors(db, use_rc);
  if (!db->jv) {
    cudaError_t e = cudaMalloc(&db->jv, jv.size() * sizeof(double));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "random-match factors");
  }
  cudaError_t e = cudaMemcpy(db->jv, jv.data(), jv.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "random-match factors");
  db->jv_rc = use_rc;
  return SK_OK;
}

sk_status check_compatible(sk_ctx *ctx, const sk_db *a, const sk_db *b) {
  if (a->bbits != b->bbits) return fail(ctx, SK_EMISMATCH, "Mismatching bbits in sketches");
  if (a->s64 != b->s64) return fail(ctx, SK_EMISMATCH, "Mismatching sketchsize64 in sketches");
  if (a->kmers != b->kmers) return fail(ctx, SK_EMISMATCH, "Mismatching k-mer lengths in sketches");
  return SK_OK;
}

// Fills a JobParams for ref (columns) vs query (rows; NULL = all-vs-all).
sk_status build_job(sk_ctx *ctx, const sk_db *ref, const sk_db *query, const sk_random *random,
                    int out_mode, int out_col, void *d_out, const TileConfig **cfg_out,
                    JobParams *jp) {
  if (!ref) return fail(ctx, SK_EINVAL, "No reference database");
  if (ref->n < 1 || (query && query->n < 1))
    return fail(ctx, SK_EINVAL, "Query with empty ref or query list!");
  if (query) {
    sk_status st = check_compatible(ctx, ref, query);
    if (st != SK_OK) return st;
  }
  if (random && random->kmers != ref->kmers)
    return fail(ctx, SK_EMISMATCH, "Random match table k-mer lengths differ from the sketches");
  const TileConfig *cfg = choose_config(ctx, ref->K, ref->s64);
  // A query batch of at most 64 samples fills one 64-row tile: with the
  // default 128-row tile more than half of every tile's work would be padding
  // (serving slices of a few queries), so use the 64 x 64 shape unless a shape
  // was forced or tuned for this (K, sketchsize64).
  if (query && query->n <= 64 && cfg && cfg->tile_rows > 64 && ctx->tile_cfg == 0 &&
      ctx->tuning.find({ref->K, ref->s64}) == ctx->tuning.end()) {
    const TileConfig *small = tile_config(kSmallQueryConfig);
    if (small && small->tile_rows == 64 && small->max_kmers >= ref->K) cfg = small;
  }
  if (!cfg || cfg->max_kmers < ref->K)
    return fail(ctx, SK_ENOTSUP, "No tile configuration holds %d k-mer lengths (at most %d)",
                ref->K, cfg ? cfg->max_kmers : kMaxKmers);
  std::memset(jp, 0, sizeof(*jp));
  const sk_db *rows = query ? query : ref;
  jp->self = query ? 0 : 1;
  jp->row_words = rows->packed;
  jp->col_words = ref->packed;
  jp->n_rows = rows->n;
  jp->n_cols = ref->n;
  jp->ng_rows = rows->ng;
  jp->ng_cols = ref->ng;
  jp->n_kmers = ref->K;
  jp->nb = 2 * ref->s64;
  jp->nchunk = (jp->nb + kMaxChunkBlocks - 1) / kMaxChunkBlocks;
  jp->chunk_nb = jp->nchunk == 1 ? jp->nb : kMaxChunkBlocks;
  jp->out_mode = out_mode;
  jp->out_col = out_col;
  jp->out = d_out;
  jp->tol = 5.0 / (ref->s64 * 64);
  jp->union_bits = static_cast<double>(64 * ref->s64);
  jp->one = 1;
  jp->semantics = ctx->semantics;
  const bool gpu_sem = ctx->semantics == kSemRefGpu;
  for (int k = 0; k < ref->K; ++k) jp->kmers[k] = ref->kmers[k];
  jp->rmode = random ? random->mode : kRandNone;
  if (jp->rmode == kRandTable) {
    const int C = random->n_clusters;
    if ((ref->cluster && ref->max_cluster >= C) || (query && query->cluster && query->max_cluster >= C))
      return fail(ctx, SK_EINVAL, "Cluster id %d beyond the %d clusters of the random match table",
                  std::max(ref->max_cluster, query ? query->max_cluster : 0), C);
    jp->rtable = random->table;
    jp->rs_k = C * C;
    // CPU path, self: [k][cluster(i = row)][cluster(j = col)]  (random_match(r1=i, r2=j))
    // query (both paths) and GPU path self: [k][cluster(ref = col)][cluster(query = row)]
    // (src/api.cpp:264-266; src/gpu/dist.cu:262-267 with ref_idx = j, query_idx = i)
    const bool col_major = query || gpu_sem;
    jp->rs_row = col_major ? 1 : C;
    jp->rs_col = col_major ? C : 1;
    jp->cl_rows = rows->cluster;
    jp->cl_cols = ref->cluster;
  } else if (jp->rmode == kRandEqualBase && gpu_sem) {
    // GPU path: one chance per k from the first reference's length
    // (flattened_random(kmer_lengths, ref_sketches[0].seq_length()),
    // src/gpu/gpu_api.cpp:402-403, src/random/random_match.cpp:278-310)
    sk_db *r = const_cast<sk_db *>(ref);
    if (!r->jgpu || r->jgpu_rc != random->use_rc) {
      const std::vector<float> t = equal_base_gpu(r, random->use_rc);
      if (!r->jgpu) {
        cudaError_t e = cudaMalloc(&r->jgpu, t.size() * sizeof(float));
        if (e != cudaSuccess) return cuda_fail(ctx, e, "random-match chances");
      }
      cudaError_t e = cudaMemcpy(r->jgpu, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "random-match chances");
      r->jgpu_rc = random->use_rc;
    }
    jp->rmode = kRandTable;
    jp->rtable = r->jgpu;
    jp->rs_k = 1;
    jp->rs_row = jp->rs_col = 0;
  } else if (jp->rmode == kRandEqualBase) {
    sk_status st = ensure_jv(ctx, const_cast<sk_db *>(ref), random->use_rc);
    if (st != SK_OK) return st;
    if (query) {
      st = ensure_jv(ctx, const_cast<sk_db *>(query), random->use_rc);
      if (st != SK_OK) return st;
    }
    jp->jv_rows = rows->jv;
    jp->jv_cols = ref->jv;
    jp->jv_rows_ld = static_cast<int64_t>(rows->ng) * kGranule;
    jp->jv_cols_ld = static_cast<int64_t>(ref->ng) * kGranule;
  }
  plan_tiles(*jp, *cfg);
  *cfg_out = cfg;
  return SK_OK;
}

// Work list for one launch.  Jobs are visited in decreasing cost per tile
// (K x blocks, longest first) so the dynamic queue ends on the cheapest items.
// The tiles of the last, partial wave are cut into p parts along k (p chosen to
// minimise ceil(r p / W) * ceil(K / p), r tail tiles on W resident CTAs); the
// per-k counts are independent, so the parts need no reduction, only a shared
// count slot and an arrival counter.  When every part holds one k, narrow
// jobs' parts are cut further into block ranges (about 32 parts per tile), so
// the launch ends within a small fraction of a tile on every SM; the partial
// counts of one k's ranges are summed by the tile's finishing thread.
void plan_items(const std::vector<JobParams> &jobs, int grid, Plan &plan) {
  plan.items.clear();
  plan.n_splits = 0;
  plan.k_slots = 1;
  std::vector<int> order(jobs.size());
  for (size_t j = 0; j < jobs.size(); ++j) order[j] = static_cast<int>(j);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return static_cast<int64_t>(jobs[a].n_kmers) * jobs[a].nb >
           static_cast<int64_t>(jobs[b].n_kmers) * jobs[b].nb;
  });
  for (int j : order) {
    plan.k_slots = std::max(plan.k_slots, job_slots(jobs[j]));
    for (int64_t t = 0; t < jobs[j].n_tiles; ++t)
      plan.items.push_back(WorkItem{t, j, 0, static_cast<int16_t>(jobs[j].n_kmers), -1, 1});
  }
  split_tail(plan.items, 0, grid, &plan.n_splits, &jobs);
  plan.k_slots = items_slots(plan.items, plan.k_slots);
}

// Block ranges each k of a narrow job's tail tile is cut into: about 32 parts
// per tile with the k parts, each range a whole number of 2-block steps.
int32_t tail_block_parts(const JobParams &jp) {
  if (needs_wide(jp)) return 1;
  return std::max(1, std::min(32 / jp.n_kmers, jp.nb / 2));
}

// Count slots the items of a work list need: base (the jobs' K x nchunk), or
// K x block ranges for tail tiles cut into block ranges.
int32_t items_slots(const std::vector<WorkItem> &items, int32_t base) {
  for (const WorkItem &it : items)
    if (it.nbpart > 1) base = std::max<int32_t>(base, it.k1 * it.nbpart);
  return base;
}

// Splits the last partial wave of items[begin..end) (whole tiles, k range
// [0, K)) along k; split slots are numbered from 0 for this range.
void split_tail(std::vector<WorkItem> &items, size_t begin, int grid, int32_t *n_splits,
                const std::vector<JobParams> *jobs) {
  *n_splits = 0;
  const int64_t T = static_cast<int64_t>(items.size() - begin);
  if (T == 0 || grid <= 0) return;
  const int64_t r = T % grid == 0 ? 0 : T % grid;
  if (r == 0) return;
  // tail tiles: the last r items; k is split by the smallest K among them
  int kmin = kMaxKmers;
  for (size_t i = items.size() - r; i < items.size(); ++i) kmin = std::min<int>(kmin, items[i].k1);
  int best_p = 1;
  int64_t best = -1;
  for (int p = 1; p <= kmin; ++p) {
    const int64_t rounds = (r * p + grid - 1) / grid;
    const int64_t cost = rounds * ((kmin + p - 1) / p);
    if (best < 0 || cost < best) {
      best = cost;
      best_p = p;
    }
  }
  if (best_p == 1) return;
  std::vector<WorkItem> tail(items.end() - r, items.end());
  items.resize(items.size() - r);
  int32_t slot = 0;
  for (const WorkItem &it : tail) {
    const int K = it.k1;
    const int parts = std::min(best_p, K);
    // narrow jobs cut each k further into block ranges when the tile is
    // already cut into single k: about 32 parts per tile
    int q = 1, nb = 0;
    if (jobs && parts == K) {
      const JobParams &jp = (*jobs)[it.job];
      q = tail_block_parts(jp);
      nb = jp.nb;
    }
    for (int p = 0; p < parts; ++p) {
      const int k0 = K * p / parts, k1 = K * (p + 1) / parts;
      for (int b = 0; b < q; ++b) {
        WorkItem w{it.tile, it.job, static_cast<int16_t>(k0), static_cast<int16_t>(k1), slot,
                   parts * q};
        if (q > 1) {
          const int steps = nb / 2;
          w.b0 = 2 * (steps * b / q);
          w.b1 = 2 * (steps * (b + 1) / q);
          w.bpart = static_cast<int16_t>(b);
          w.nbpart = static_cast<int16_t>(q);
        }
        items.push_back(w);
      }
    }
    ++slot;
  }
  *n_splits = slot;
}

// Device buffers for a plan: job table, work list, control block (queue
// counter + split arrival counters, zeroed per launch) and count scratch.
MetaLayout meta_layout(size_t n_jobs, size_t n_items, int32_t n_splits, int threads) {
  MetaLayout m;
  m.items_off = (n_jobs * sizeof(JobParams) + 255) & ~static_cast<size_t>(255);
  m.ctrl_off = (m.items_off + n_items * sizeof(WorkItem) + 255) & ~static_cast<size_t>(255);
  m.ctrl_bytes = 8 + static_cast<size_t>(n_splits) * threads * 4;
  m.bytes = m.ctrl_off + m.ctrl_bytes;
  return m;
}

sk_status upload_plan(sk_ctx *ctx, const std::vector<JobParams> &jobs, Plan &plan,
                      LaunchBuffers &buf, bool owned) {
  const TileConfig &cfg = *plan.cfg;
  const size_t jobs_bytes = jobs.size() * sizeof(JobParams);
  const size_t items_bytes = plan.items.size() * sizeof(WorkItem);
  const MetaLayout ml = meta_layout(jobs.size(), plan.items.size(), plan.n_splits, cfg.threads);
  const size_t ctrl_bytes = ml.ctrl_bytes;
  const size_t jobs_off = 0;
  const size_t items_off = ml.items_off;
  const size_t ctrl_off = ml.ctrl_off;
  const size_t meta_bytes = ml.bytes;
  const size_t slot = count_slot_bytes(cfg, plan.k_slots);
  const size_t cta_bytes = static_cast<size_t>(plan.grid) * slot;
  const size_t split_bytes = std::max<size_t>(static_cast<size_t>(plan.n_splits) * slot, 16);
  void *meta = nullptr, *cta = nullptr, *split = nullptr;
  if (owned) {
    cudaError_t e = cudaMalloc(&meta, meta_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&cta, cta_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&split, split_bytes);
    if (e != cudaSuccess) {
      if (meta) cudaFree(meta);
      if (cta) cudaFree(cta);
      if (split) cudaFree(split);
      return cuda_fail(ctx, e, "batch buffers");
    }
  } else {
    sk_status st = scratch(ctx, kSlotLaunchMeta, meta_bytes, &meta);
    if (st == SK_OK) st = scratch(ctx, kSlotCounts, cta_bytes, &cta);
    if (st == SK_OK) st = scratch(ctx, kSlotSplitCounts, split_bytes, &split);
    if (st != SK_OK) return st;
  }
  char *m = static_cast<char *>(meta);
  cudaError_t e = cudaMemcpyAsync(m + jobs_off, jobs.data(), jobs_bytes, cudaMemcpyHostToDevice,
                                  ctx->stream);
  if (e == cudaSuccess && items_bytes)
    e = cudaMemcpyAsync(m + items_off, plan.items.data(), items_bytes, cudaMemcpyHostToDevice,
                        ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "work list upload");
  buf.meta = meta;
  buf.cta = cta;
  buf.split = split;
  buf.ctrl = m + ctrl_off;
  buf.ctrl_bytes = ctrl_bytes;
  LaunchParams &lp = buf.lp;
  lp.jobs = reinterpret_cast<const JobParams *>(m + jobs_off);
  lp.items = reinterpret_cast<const WorkItem *>(m + items_off);
  lp.n_items = static_cast<int64_t>(plan.items.size());
  lp.item_counter = reinterpret_cast<unsigned long long *>(m + ctrl_off);
  lp.split_done = reinterpret_cast<unsigned int *>(m + ctrl_off + 8);
  lp.cta_scratch = static_cast<uint16_t *>(cta);
  lp.split_scratch = static_cast<uint16_t *>(split);
  lp.k_slots = plan.k_slots;
  lp.wide = 0;
  for (const JobParams &jp : jobs) lp.wide |= needs_wide(jp) ? 1 : 0;
  lp.status = ctx->status_dev;
  lp.cancel = ctx->cancel_dev;
  return SK_OK;
}

sk_status enqueue_plan(sk_ctx *ctx, const Plan &plan, const LaunchBuffers &buf) {
  if (buf.lp.n_items == 0) return SK_OK;
  cudaError_t e = cudaMemsetAsync(buf.ctrl, 0, buf.ctrl_bytes, ctx->stream);
  if (e == cudaSuccess) e = plan.cfg->launch(buf.lp, plan.grid, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "distance kernel launch");
  return SK_OK;
}

int resident_grid(sk_ctx *ctx, const TileConfig &cfg) {
  const int per_sm = cfg.blocks_per_sm();
  return per_sm < 1 ? 0 : per_sm * ctx->sm_count;
}

sk_status make_plan(sk_ctx *ctx, const std::vector<JobParams> &jobs, const TileConfig &cfg,
                    Plan &plan) {
  plan.cfg = &cfg;
  const int resident = resident_grid(ctx, cfg);
  if (resident < 1) return fail(ctx, SK_ECUDA, "Tile configuration %d does not fit the device", cfg.id);
  int64_t tiles = 0;
  for (const JobParams &j : jobs) tiles += j.n_tiles;
  plan.grid = resident;
  plan_items(jobs, resident, plan);
  if (static_cast<int64_t>(plan.items.size()) < plan.grid)
    plan.grid = static_cast<int>(std::max<int64_t>(1, plan.items.size()));
  return SK_OK;
}

sk_status launch_job(sk_ctx *ctx, const JobParams &jp, const TileConfig &cfg) {
  if (jp.n_tiles == 0) return SK_OK;
  std::vector<JobParams> jobs{jp};
  Plan plan;
  sk_status st = make_plan(ctx, jobs, cfg, plan);
  if (st != SK_OK) return st;
  LaunchBuffers buf;
  st = upload_plan(ctx, jobs, plan, buf, false);
  if (st != SK_OK) return st;
  return enqueue_plan(ctx, plan, buf);
}

int64_t n_pairs(const sk_db *ref, const sk_db *query) {
  if (!ref) return 0;
  if (query) return query->n * ref->n;
  return ref->n * (ref->n - 1) / 2;
}

size_t out_bytes(int out_mode, int64_t pairs, int K) {
  switch (out_mode) {
    case kOutCoreAcc: return static_cast<size_t>(pairs) * 8;
    case kOutJaccard:
    case kOutCounts: return static_cast<size_t>(pairs) * 4 * K;
    default: return static_cast<size_t>(pairs) * 4;
  }
}

// Dense distances into device memory `d_out` (queued on the context stream).
sk_status dense_to_device(sk_ctx *ctx, const sk_db *ref, const sk_db *query,
                          const sk_random *random, int out_mode, int out_col, void *d_out) {
  JobParams jp;
  const TileConfig *cfg = nullptr;
  sk_status st = build_job(ctx, ref, query, random, out_mode, out_col, d_out, &cfg, &jp);
  if (st == SK_OK) st = attach_count_tables(ctx, &jp);
  if (st != SK_OK) return st;
  return launch_job(ctx, jp, *cfg);
}

// The context's second stream and its double-buffer events.
sk_status ensure_copy_stream(sk_ctx *ctx) {
  cudaError_t e = cudaSuccess;
  if (!ctx->copy_stream) e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
    if (!ctx->ev_ready[b]) e = cudaEventCreateWithFlags(&ctx->ev_ready[b], cudaEventDisableTiming);
    if (e == cudaSuccess && !ctx->ev_free[b])
      e = cudaEventCreateWithFlags(&ctx->ev_free[b], cudaEventDisableTiming);
  }
  return e == cudaSuccess ? SK_OK : cuda_fail(ctx, e, "copy stream setup");
}

// Device bytes a dense call may use to stage its output: the context's limit,
// else the free memory less a 2 GiB margin.  The output staging buffer the
// context already holds counts as available: growing it frees it first.
size_t dense_budget(sk_ctx *ctx) {
  if (ctx->mem_limit > 0) return static_cast<size_t>(ctx->mem_limit);
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
  free_b += ctx->scratch[kSlotOut].bytes;
  const size_t margin = size_t(2) << 30;
  return free_b > 2 * margin ? free_b - margin : free_b / 2;
}

// Dense distances to a host buffer in blocks of row tiles, for outputs larger
// than the device memory allowed for them (the reference's query_db_cuda
// estimates memory and splits the all-vs-all into chunks,
// src/gpu/gpu_api.cpp:357-389, and refuses query mode).  A block of row tiles
// is a contiguous range of tiles and of long-form rows, so each block is one
// persistent launch into one of two device buffers, copied back on the copy
// stream while the next block computes.
sk_status dense_blocked_to_host(sk_ctx *ctx, const sk_db *ref, const sk_db *query,
                                const sk_random *random, int out_mode, void *out, size_t budget) {
  JobParams base;
  const TileConfig *cfg = nullptr;
  sk_status st = build_job(ctx, ref, query, random, out_mode, 0, nullptr, &cfg, &base);
  if (st == SK_OK) st = attach_count_tables(ctx, &base);
  if (st != SK_OK) return st;
  st = ensure_copy_stream(ctx);
  if (st != SK_OK) return st;
  const int grid = resident_grid(ctx, *cfg);
  if (grid < 1) return fail(ctx, SK_ECUDA, "Tile configuration %d does not fit the device", cfg->id);
  const size_t elem = out_bytes(out_mode, 1, base.n_kmers);
  const int64_t nrt = base.n_row_tiles;
  const int64_t m = base.tile_rows / base.tile_cols;
  auto first_row = [&](int64_t ti) -> int64_t {   // first long-form row of row tile ti
    if (base.self) {
      const int64_t i = std::min<int64_t>(ti * base.tile_rows, base.n_rows - 1);
      return base.n_rows * i - i * (i + 1) / 2;
    }
    return std::min<int64_t>(ti * base.tile_rows, base.n_rows) * base.n_cols;
  };
  auto first_tile = [&](int64_t ti) -> int64_t {
    return base.self ? ti * base.n_col_tiles - m * ti * (ti - 1) / 2 : ti * base.n_col_tiles;
  };
  // blocks of whole row tiles, each within half the budget (two buffers)
  const int64_t cap = std::max<int64_t>(1, static_cast<int64_t>(budget / 2 / elem));
  std::vector<int64_t> cut{0};
  int64_t max_rows = 0;
  while (cut.back() < nrt) {
    const int64_t t0 = cut.back();
    int64_t t1 = t0 + 1;
    while (t1 < nrt && first_row(t1 + 1) - first_row(t0) <= cap) ++t1;
    max_rows = std::max(max_rows, first_row(t1) - first_row(t0));
    cut.push_back(t1);
  }
  const int nblk = static_cast<int>(cut.size() - 1);
  std::vector<JobParams> jobs(nblk, base);
  std::vector<WorkItem> items;
  std::vector<size_t> start(nblk), count(nblk);
  std::vector<int32_t> splits(nblk);
  for (int c = 0; c < nblk; ++c) {
    jobs[c].out_row0 = first_row(cut[c]);
    start[c] = items.size();
    for (int64_t t = first_tile(cut[c]); t < first_tile(cut[c + 1]); ++t)
      items.push_back(WorkItem{t, c, 0, static_cast<int16_t>(base.n_kmers), -1, 1});
    split_tail(items, start[c], grid, &splits[c], &jobs);
    count[c] = items.size() - start[c];
  }
  int32_t max_splits = *std::max_element(splits.begin(), splits.end());
  const int32_t k_slots = items_slots(items, job_slots(base));
  const size_t items_off = (jobs.size() * sizeof(JobParams) + 255) & ~static_cast<size_t>(255);
  const size_t ctrl_off = (items_off + items.size() * sizeof(WorkItem) + 255) & ~static_cast<size_t>(255);
  std::vector<size_t> ctrl_at(nblk);
  size_t meta_bytes = ctrl_off;
  for (int c = 0; c < nblk; ++c) {
    ctrl_at[c] = meta_bytes;
    meta_bytes += (8 + static_cast<size_t>(splits[c]) * cfg->threads * 4 + 255) & ~static_cast<size_t>(255);
  }
  const size_t slot = count_slot_bytes(*cfg, k_slots);
  void *meta = nullptr, *cta = nullptr, *split = nullptr, *obuf = nullptr;
  st = scratch(ctx, kSlotLaunchMeta, meta_bytes, &meta);
  if (st == SK_OK) st = scratch(ctx, kSlotCounts, static_cast<size_t>(grid) * slot, &cta);
  if (st == SK_OK)
    st = scratch(ctx, kSlotSplitCounts, std::max<size_t>(static_cast<size_t>(max_splits) * slot, 16), &split);
  if (st == SK_OK) st = scratch(ctx, kSlotOut, 2 * static_cast<size_t>(max_rows) * elem, &obuf);
  if (st != SK_OK) return st;
  char *buf[2] = {static_cast<char *>(obuf), static_cast<char *>(obuf) + max_rows * elem};
  for (int c = 0; c < nblk; ++c) jobs[c].out = buf[c & 1];
  char *mt = static_cast<char *>(meta);
  cudaError_t e = cudaMemcpyAsync(mt, jobs.data(), jobs.size() * sizeof(JobParams),
                                  cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(mt + items_off, items.data(), items.size() * sizeof(WorkItem),
                        cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(mt + ctrl_off, 0, meta_bytes - ctrl_off, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "work list upload");
  LaunchParams lp{};
  lp.jobs = reinterpret_cast<const JobParams *>(mt);
  lp.cta_scratch = static_cast<uint16_t *>(cta);
  lp.split_scratch = static_cast<uint16_t *>(split);
  lp.k_slots = k_slots;
  lp.wide = needs_wide(base) ? 1 : 0;
  lp.status = ctx->status_dev;
  lp.cancel = ctx->cancel_dev;
  // block c computes into buf[c & 1] once the copy of block c - 2 has left it;
  // its copy is queued after block c + 1's launch, so a pageable destination
  // (whose copy returns only when done) still overlaps the next block
  auto copy_back = [&](int c) -> cudaError_t {
    const int b = c & 1;
    const size_t rows = static_cast<size_t>(first_row(cut[c + 1]) - first_row(cut[c]));
    cudaError_t e2 = cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_ready[b], 0);
    if (e2 == cudaSuccess)
      e2 = cudaMemcpyAsync(static_cast<char *>(out) + first_row(cut[c]) * elem, buf[b], rows * elem,
                           cudaMemcpyDeviceToHost, ctx->copy_stream);
    if (e2 == cudaSuccess) e2 = cudaEventRecord(ctx->ev_free[b], ctx->copy_stream);
    return e2;
  };
  for (int c = 0; c <= nblk && e == cudaSuccess; ++c) {
    if (c < nblk) {
      const int b = c & 1;
      if (c >= 2) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_free[b], 0);
      if (e == cudaSuccess && count[c] > 0) {
        LaunchParams l = lp;
        l.items = reinterpret_cast<const WorkItem *>(mt + items_off) + start[c];
        l.n_items = static_cast<int64_t>(count[c]);
        l.item_counter = reinterpret_cast<unsigned long long *>(mt + ctrl_at[c]);
        l.split_done = reinterpret_cast<unsigned int *>(mt + ctrl_at[c] + 8);
        e = cfg->launch(l, static_cast<int>(std::min<int64_t>(grid, l.n_items)), ctx->stream);
      }
      if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_ready[b], ctx->stream);
    }
    if (e == cudaSuccess && c >= 1) e = copy_back(c - 1);
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "blocked distance computation");
  // the compute stream (whose completion finish_call reports) waits for the last copies
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_free[b], 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "blocked distance computation");
  return SK_OK;
}


// kNN over rows of `rows` against every column of `cols`, in blocks of rows
// whose distance columns fit `budget` bytes, for when the whole column does not
// fit (the reference's sparseDists likewise works in chunks,
// src/gpu/dist.cu:495-791).  A block is a view of the row database: the packed
// array offset by whole granules (the kernel strides by the full array's
// granule count), cluster ids and equal-base factors offset by the first row.
// self: rows and cols are the same database; each row's own column is +inf and
// random-table lookups keep the all-vs-all orientation (self_view), so the
// result is bit-identical to the one-column path, at twice its compute.
// Results go to d_j / d_d at [row][kNN]; everything is queued on the stream.
sk_status knn_blocked(sk_ctx *ctx, const sk_db *cols, const sk_db *rows, bool self,
                      const sk_random *random, int kNN, int out_col, int jaccard, int64_t *d_j,
                      float *d_d, size_t budget) {
  if (random && random->mode == kRandEqualBase) {
    sk_status st = ensure_jv(ctx, const_cast<sk_db *>(rows), random->use_rc);
    if (st == SK_OK) st = ensure_jv(ctx, const_cast<sk_db *>(cols), random->use_rc);
    if (st != SK_OK) return st;
  }
  const int64_t n_cols = cols->n;
  int64_t per = static_cast<int64_t>(budget / (static_cast<size_t>(n_cols) * 4));
  per = std::max<int64_t>(kSamplePad, per / kSamplePad * kSamplePad);
  void *d_vals = nullptr;
  sk_status st = scratch(ctx, kSlotOut, static_cast<size_t>(std::min(per, rows->n)) * n_cols * 4, &d_vals);
  if (st != SK_OK) return st;
  for (int64_t r0 = 0; r0 < rows->n; r0 += per) {
    sk_db view = *rows;
    view.n = std::min(per, rows->n - r0);
    view.packed = rows->packed + (r0 / kGranule) * kStripeWords;
    view.cluster = rows->cluster ? rows->cluster + r0 : nullptr;
    view.jv = rows->jv ? rows->jv + r0 : nullptr;
    view.jgpu = nullptr;
    JobParams jp;
    const TileConfig *cfg = nullptr;
    st = build_job(ctx, cols, &view, random, kOutColumn, out_col, d_vals, &cfg, &jp);
    if (st == SK_OK) st = attach_count_tables(ctx, &jp);
    if (st != SK_OK) return st;
    if (self) {
      jp.self_view = 1;
      jp.row_base = r0;
      if (jp.rmode == kRandTable && random && random->mode == kRandTable) {
        // the all-vs-all orientation: CPU path [k][cluster(i)][cluster(j)],
        // GPU path [k][cluster(j)][cluster(i)], i < j
        const int C = random->n_clusters;
        jp.rs_row = jp.semantics == kSemRefGpu ? 1 : C;
        jp.rs_col = jp.semantics == kSemRefGpu ? C : 1;
      }
    }
    st = launch_job(ctx, jp, *cfg);
    if (st != SK_OK) return st;
    cudaError_t e = launch_knn_rows(static_cast<float *>(d_vals), view.n, n_cols, kNN,
                                    self ? r0 : -1, jaccard, d_j + r0 * kNN, d_d + r0 * kNN,
                                    ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "kNN");
  }
  return SK_OK;
}

}  // namespace sk

// ------------------------------------------------------------------ context

#define SK_GUARD(ctx)                                      \
  if (!(ctx)) return SK_EINVAL;                            \
  std::lock_guard<std::recursive_mutex> lock_((ctx)->mu);  \
  DeviceGuard dev_guard_((ctx)->device)

extern "C" {

int32_t sk_abi_version(void) { return SK_ABI_VERSION; }

sk_status sk_ctx_create(int32_t device_id, sk_ctx **out) {
  if (!out) return SK_EINVAL;
  *out = nullptr;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev < 1) return SK_ECUDA;
  if (device_id < 0 || device_id >= n_dev) return SK_EINVAL;
  sk_ctx *ctx = new sk_ctx();
  ctx->device = device_id;
  DeviceGuard g(device_id);
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device_id);
  if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void **>(&ctx->cancel_host), sizeof(int), cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&ctx->cancel_dev), ctx->cancel_host, 0);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->status_dev, sizeof(DevStatus));
  if (e != cudaSuccess) {
    sk_ctx_destroy(ctx);
    return e == cudaErrorMemoryAllocation ? SK_ENOMEM : SK_ECUDA;
  }
  *ctx->cancel_host = 0;
  cudaMemset(ctx->status_dev, 0, sizeof(DevStatus));
  *out = ctx;
  return SK_OK;
}

sk_status sk_ctx_destroy(sk_ctx *ctx) {
  if (!ctx) return SK_EINVAL;
  {
    std::lock_guard<std::mutex> g(g_ctx_refs_mu);
    if (ctx->destroyed) return SK_EINVAL;
    ctx->destroyed = true;
  }
  ctx_release(ctx);
  return SK_OK;
}

const char *sk_last_error(const sk_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

sk_status sk_ctx_set_stream(sk_ctx *ctx, void *stream) {
  SK_GUARD(ctx);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  ctx->stream = static_cast<cudaStream_t>(stream);
  ctx->own_stream = false;
  return SK_OK;
}

sk_status sk_ctx_set_memory_limit(sk_ctx *ctx, int64_t bytes) {
  SK_GUARD(ctx);
  if (bytes < 0) return fail(ctx, SK_EINVAL, "negative memory limit");
  ctx->mem_limit = bytes;
  return SK_OK;
}

sk_status sk_ctx_set_semantics(sk_ctx *ctx, int32_t semantics) {
  SK_GUARD(ctx);
  if (semantics != kSemRefCpu && semantics != kSemRefGpu)
    return fail(ctx, SK_EINVAL, "Unknown semantics %d", semantics);
  ctx->semantics = semantics;
  return SK_OK;
}

sk_status sk_cancel(sk_ctx *ctx) {
  if (!ctx) return SK_EINVAL;
  // deliberately no lock: called from another thread while a call runs
  reinterpret_cast<volatile int *>(ctx->cancel_host)[0] = 1;
  return SK_OK;
}

sk_status sk_device_info(sk_ctx *ctx, int64_t *mem_free, int64_t *mem_total, int32_t *sm_count) {
  SK_GUARD(ctx);
  size_t f = 0, t = 0;
  cudaError_t e = cudaMemGetInfo(&f, &t);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemGetInfo");
  if (mem_free) *mem_free = static_cast<int64_t>(f);
  if (mem_total) *mem_total = static_cast<int64_t>(t);
  if (sm_count) *sm_count = ctx->sm_count;
  return SK_OK;
}

sk_status sk_ctx_synchronize(sk_ctx *ctx) {
  SK_GUARD(ctx);
  return finish_call(ctx);
}

sk_status sk_ctx_set_tile_config(sk_ctx *ctx, int32_t config_id) {
  SK_GUARD(ctx);
  if (config_id != 0 && !tile_config(config_id))
    return fail(ctx, SK_EINVAL, "Unknown tile configuration %d", config_id);
  ctx->tile_cfg = config_id;
  return SK_OK;
}

int32_t sk_tile_config_count(void) { return tile_config_count(); }

sk_status sk_tile_config_info(int32_t config_id, int32_t *tile_rows, int32_t *tile_cols,
                              int32_t *thread_rows, int32_t *thread_cols, int32_t *max_kmers) {
  const TileConfig *c = tile_config(config_id);
  if (!c) return SK_EINVAL;
  if (tile_rows) *tile_rows = c->tile_rows;
  if (tile_cols) *tile_cols = c->tile_cols;
  if (thread_rows) *thread_rows = c->thread_rows;
  if (thread_cols) *thread_cols = c->thread_cols;
  if (max_kmers) *max_kmers = c->max_kmers;
  return SK_OK;
}

sk_status sk_ctx_load_tuning(sk_ctx *ctx, const char *path) {
  SK_GUARD(ctx);
  std::ifstream in(path ? path : "");
  if (!in) return fail(ctx, SK_EINVAL, "Cannot open tuning table %s", path ? path : "(null)");
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ls(line);
    int K = 0, s64 = 0, id = 0;
    if (!(ls >> K >> s64 >> id)) continue;
    if (tile_config(id)) ctx->tuning[{K, s64}] = id;
  }
  return SK_OK;
}

// ------------------------------------------------------------------ databases

}  // extern "C"

namespace sk {

// A database with its packed array allocated (contents not yet written); with
// packed_slot >= 0 the array is that context scratch slot, kept across calls.
sk_status db_alloc(sk_ctx *ctx, int64_t n, const int32_t *kmers, int32_t K, int32_t s64,
                   int32_t bbits, sk_db **out, int packed_slot) {
  if (!out) return fail(ctx, SK_EINVAL, "null output handle");
  *out = nullptr;
  if (n < 0) return fail(ctx, SK_EINVAL, "negative sample count");
  if (bbits != kBbits)
    return fail(ctx, SK_ENOTSUP, "bbits %d not supported (sketches use %d bit planes)", bbits, kBbits);
  if (s64 < 1 || s64 > kMaxSketch64)
    return fail(ctx, SK_ERANGE, "sketchsize64 %d outside [1, %d]", s64, kMaxSketch64);
  if (K < 1 || K > kMaxKmers || !kmers)
    return fail(ctx, SK_ERANGE, "n_kmers %d outside [1, %d]", K, kMaxKmers);
  for (int k = 0; k < K; ++k)
    if (kmers[k] < 1 || kmers[k] > kMaxKmerLength)
      return fail(ctx, SK_EINVAL, "bad k-mer length %d", kmers[k]);
  sk_db *db = new sk_db();
  db->ctx = ctx;
  ctx_retain(ctx);
  db->n = n;
  db->K = K;
  db->s64 = s64;
  db->bbits = bbits;
  db->kmers.assign(kmers, kmers + K);
  const int64_t npad = ((n + kSamplePad - 1) / kSamplePad) * kSamplePad;
  db->ng = static_cast<int32_t>(std::max<int64_t>(npad, kSamplePad) / kGranule);
  const size_t packed_words = static_cast<size_t>(K) * 2 * s64 * db->ng * kStripeWords;
  if (packed_slot >= 0) {
    void *buf = nullptr;
    sk_status st = scratch(ctx, packed_slot, packed_words * 4, &buf);
    if (st != SK_OK) {
      delete db;
      ctx_release(ctx);
      return st;
    }
    db->packed = static_cast<uint32_t *>(buf);
    db->own_packed = false;
  } else {
    cudaError_t e = cudaMalloc(&db->packed, packed_words * 4);
    if (e != cudaSuccess) {
      delete db;
      ctx_release(ctx);
      return cuda_fail(ctx, e, "sketch database allocation");
    }
  }
  *out = db;
  return SK_OK;
}

// Frees a database made by db_alloc (the context's stream must be idle).
void db_free(sk_db *db) {
  sk_ctx *ctx = db->ctx;
  {
    DeviceGuard g(ctx->device);
    if (db->packed && db->own_packed) cudaFree(db->packed);
    if (db->cluster) cudaFree(db->cluster);
    if (db->jv) cudaFree(db->jv);
    if (db->jgpu) cudaFree(db->jgpu);
  }
  delete db;
  ctx_release(ctx);
}

}  // namespace sk

extern "C" {

static sk_status db_create_impl(sk_ctx *ctx, const uint64_t *words, bool on_device, int64_t n,
                                const int32_t *kmers, int32_t K, int32_t s64, int32_t bbits,
                                sk_db **out) {
  if (!out) return fail(ctx, SK_EINVAL, "null output handle");
  *out = nullptr;
  if (n > 0 && !words) return fail(ctx, SK_EINVAL, "null sketch words");
  sk_db *db = nullptr;
  sk_status st0 = db_alloc(ctx, n, kmers, K, s64, bbits, &db);
  if (st0 != SK_OK) return st0;
  cudaError_t e = cudaSuccess;
  const size_t in_words = static_cast<size_t>(n) * K * s64 * kBbits;
  const uint64_t *d_words = words;
  uint64_t *tmp = nullptr;
  if (!on_device && n > 0) {
    e = cudaMalloc(&tmp, in_words * 8);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tmp, words, in_words * 8, cudaMemcpyHostToDevice, ctx->stream);
    d_words = tmp;
  }
  if (e == cudaSuccess) e = launch_pack(d_words, n, K, s64, db->ng, db->packed, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (tmp) cudaFree(tmp);
  if (e != cudaSuccess) {
    sk_status st = cuda_fail(ctx, e, "sketch upload");
    db_free(db);
    return st;
  }
  *out = db;
  return SK_OK;
}

sk_status sk_db_create(sk_ctx *ctx, const uint64_t *words, int64_t n_samples, const int32_t *kmers,
                       int32_t n_kmers, int32_t sketchsize64, int32_t bbits, sk_db **out) {
  SK_GUARD(ctx);
  ctx->err.clear();
  return db_create_impl(ctx, words, false, n_samples, kmers, n_kmers, sketchsize64, bbits, out);
}

sk_status sk_db_create_device(sk_ctx *ctx, const uint64_t *d_words, int64_t n_samples,
                              const int32_t *kmers, int32_t n_kmers, int32_t sketchsize64,
                              int32_t bbits, sk_db **out) {
  SK_GUARD(ctx);
  ctx->err.clear();
  return db_create_impl(ctx, d_words, true, n_samples, kmers, n_kmers, sketchsize64, bbits, out);
}

sk_status sk_db_destroy(sk_db *db) {
  if (!db) return SK_EINVAL;
  {
    DeviceGuard g(db->ctx->device);
    cudaStreamSynchronize(db->ctx->stream);
  }
  db_free(db);
  return SK_OK;
}

sk_status sk_db_info(const sk_db *db, int64_t *n_samples, int32_t *n_kmers, int32_t *sketchsize64,
                     int32_t *bbits) {
  if (!db) return SK_EINVAL;
  if (n_samples) *n_samples = db->n;
  if (n_kmers) *n_kmers = db->K;
  if (sketchsize64) *sketchsize64 = db->s64;
  if (bbits) *bbits = db->bbits;
  return SK_OK;
}

sk_status sk_db_set_sample_info(sk_db *db, const uint16_t *cluster, const uint64_t *seq_len) {
  if (!db) return SK_EINVAL;
  sk_ctx *ctx = db->ctx;
  SK_GUARD(ctx);
  const int64_t npad = static_cast<int64_t>(db->ng) * kGranule;
  if (cluster) {
    std::vector<uint16_t> cl(npad, 0);
    std::copy(cluster, cluster + db->n, cl.begin());
    db->max_cluster = db->n > 0 ? *std::max_element(cluster, cluster + db->n) : 0;
    if (!db->cluster) {
      cudaError_t e = cudaMalloc(&db->cluster, npad * sizeof(uint16_t));
      if (e != cudaSuccess) return cuda_fail(ctx, e, "cluster ids");
    }
    cudaError_t e = cudaMemcpy(db->cluster, cl.data(), npad * sizeof(uint16_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cluster ids");
  }
  if (seq_len) {
    db->seq_len.assign(seq_len, seq_len + db->n);
    db->jv_rc = -1;  // factors depend on lengths
    db->jgpu_rc = -1;
  }
  return SK_OK;
}

sk_status sk_db_download(sk_ctx *ctx, const sk_db *db, uint64_t *words) {
  SK_GUARD(ctx);
  if (!db || (!words && db->n > 0)) return fail(ctx, SK_EINVAL, "null argument");
  const size_t n_words = static_cast<size_t>(db->n) * db->K * db->s64 * kBbits;
  if (n_words == 0) return SK_OK;
  void *tmp = nullptr;
  sk_status st = scratch(ctx, kSlotTemp, n_words * 8, &tmp);
  if (st != SK_OK) return st;
  cudaError_t e = launch_unpack(db->packed, db->n, db->K, db->s64, db->ng, static_cast<uint64_t *>(tmp), ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(words, tmp, n_words * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "sketch download");
  return SK_OK;
}

// ------------------------------------------------------------------- random

sk_status sk_random_create(sk_ctx *ctx, int32_t mode, int32_t use_rc, const int32_t *kmers,
                           int32_t n_kmers, int32_t n_clusters, const float *table,
                           sk_random **out) {
  SK_GUARD(ctx);
  ctx->err.clear();
  if (!out) return fail(ctx, SK_EINVAL, "null output handle");
  *out = nullptr;
  if (mode != kRandNone && mode != kRandEqualBase && mode != kRandTable)
    return fail(ctx, SK_EINVAL, "Unknown random-match mode %d", mode);
  if (n_kmers < 1 || n_kmers > kMaxKmers || !kmers)
    return fail(ctx, SK_EINVAL, "bad k-mer list for random matches");
  sk_random *r = new sk_random();
  r->ctx = ctx;
  ctx_retain(ctx);
  r->mode = mode;
  r->use_rc = use_rc ? 1 : 0;
  r->kmers.assign(kmers, kmers + n_kmers);
  if (mode == kRandTable) {
    if (n_clusters < 1 || !table) {
      delete r;
      ctx_release(ctx);
      return fail(ctx, SK_EINVAL, "Random match table needs n_clusters >= 1 and a table");
    }
    r->n_clusters = n_clusters;
    const size_t sz = static_cast<size_t>(n_kmers) * n_clusters * n_clusters * sizeof(float);
    cudaError_t e = cudaMalloc(&r->table, sz);
    if (e == cudaSuccess) e = cudaMemcpy(r->table, table, sz, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      if (r->table) cudaFree(r->table);
      delete r;
      sk_status st = cuda_fail(ctx, e, "random match table");
      ctx_release(ctx);
      return st;
    }
  }
  *out = r;
  return SK_OK;
}

sk_status sk_random_set_centroids(sk_random *random, const float *centroids,
                                  int32_t n_clusters) {
  if (!random) return SK_EINVAL;
  sk_ctx *ctx = random->ctx;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  ctx->err.clear();
  if (random->mode != kRandTable)
    return fail(ctx, SK_EINVAL, "Centroids belong to a Monte Carlo (table) random-match model");
  if (n_clusters != random->n_clusters || !centroids)
    return fail(ctx, SK_EINVAL, "Expected %d centroids of 4 base frequencies", random->n_clusters);
  random->centroids.assign(centroids, centroids + static_cast<size_t>(n_clusters) * 4);
  return SK_OK;
}

sk_status sk_closest_cluster(const float *centroids, int32_t n_clusters, int32_t use_rc,
                             const double *base_freq, int64_t n, uint16_t *cluster_out) {
  if (n < 0 || n_clusters < 0 || (n > 0 && (!base_freq || !cluster_out)) ||
      (n_clusters > 0 && !centroids))
    return SK_EINVAL;
  for (int64_t i = 0; i < n; ++i) {
    double b[4] = {base_freq[4 * i], base_freq[4 * i + 1], base_freq[4 * i + 2],
                   base_freq[4 * i + 3]};
    if (use_rc) {  // strand unknown: A/T and C/G cannot be told apart
      b[0] = 0.5 * (b[0] + b[3]);
      b[1] = 0.5 * (b[1] + b[2]);
      b[2] = b[1];
      b[3] = b[0];
    }
    int best = 0;
    float best_d = std::numeric_limits<float>::infinity();
    for (int c = 0; c < n_clusters; ++c) {
      float d = 0.0f;
      for (int j = 0; j < 4; ++j) {
        const float diff = centroids[c * 4 + j] - static_cast<float>(b[j]);
        d += diff * diff;
      }
      if (d < best_d) {
        best_d = d;
        best = c;
      }
    }
    cluster_out[i] = static_cast<uint16_t>(best);
  }
  return SK_OK;
}

sk_status sk_random_destroy(sk_random *random) {
  if (!random) return SK_EINVAL;
  sk_ctx *ctx = random->ctx;
  {
    DeviceGuard g(ctx->device);
    if (random->table) cudaFree(random->table);
  }
  delete random;
  ctx_release(ctx);
  return SK_OK;
}

// ------------------------------------------------------------------- dense

int64_t sk_dists_rows(const sk_db *ref, const sk_db *query) { return n_pairs(ref, query); }

sk_status sk_dists_dense(sk_ctx *ctx, const sk_db *ref, const sk_db *query, const sk_random *random,
                         int32_t out_mode, void *out, int32_t out_on_device) {
  SK_GUARD(ctx);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (out_mode != kOutCoreAcc && out_mode != kOutJaccard && out_mode != kOutCounts)
    return fail(ctx, SK_EINVAL, "Unknown output mode %d", out_mode);
  const int64_t pairs = n_pairs(ref, query);
  if (pairs > 0 && !out) return fail(ctx, SK_EINVAL, "null output buffer");
  const size_t bytes = ref ? out_bytes(out_mode, pairs, ref->K) : 0;
  if (!out_on_device && bytes > 0) {
    const size_t budget = dense_budget(ctx);
    if (bytes > budget) {
      st = dense_blocked_to_host(ctx, ref, query, random, out_mode, out, budget);
      if (st != SK_OK) return st;
      return finish_call(ctx);
    }
  }
  void *d_out = out;
  if (!out_on_device && bytes > 0) {
    st = scratch(ctx, kSlotOut, bytes, &d_out);
    if (st != SK_OK) return st;
  }
  st = dense_to_device(ctx, ref, query, random, out_mode, 0, d_out);
  if (st != SK_OK) return st;
  if (out_on_device) return SK_OK;
  if (bytes > 0) {
    cudaError_t e = cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "result copy");
  }
  return finish_call(ctx);
}

// --------------------------------------------------------------------- kNN

sk_status sk_dists_knn(sk_ctx *ctx, const sk_db *db, const sk_random *random, int32_t kNN,
                       int32_t dist_col, int32_t jaccard, int64_t *i_out, int64_t *j_out,
                       float *d_out) {
  SK_GUARD(ctx);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (!db || db->n < 1) return fail(ctx, SK_EINVAL, "Query with empty ref or query list!");
  // check_sparse_inputs (src/api.cpp:293-313)
  if ((jaccard && dist_col >= db->K) || (dist_col != 0 && dist_col != 1))
    return fail(ctx, SK_EINVAL, "dist_col out of range");
  if (kNN < 0 || kNN > db->n) return fail(ctx, SK_EINVAL, "kNN must be between 0 and the number of samples");
  if (kNN == 0) return SK_OK;
  const int64_t n = db->n, pairs = n_pairs(db, nullptr);
  void *d_vals = nullptr, *d_res = nullptr;
  const size_t res_elems = static_cast<size_t>(n) * kNN;
  st = scratch(ctx, kSlotResult, res_elems * 12, &d_res);
  if (st != SK_OK) return st;
  int64_t *d_j = static_cast<int64_t *>(d_res);
  float *d_d = reinterpret_cast<float *>(d_j + res_elems);
  const int out_col = jaccard ? 2 + dist_col : dist_col;
  const size_t budget = dense_budget(ctx);
  cudaError_t e = cudaSuccess;
  if (static_cast<size_t>(pairs) * 4 > budget || kNN > kKnnListMax) {
    // longer lists are selected over dense rows: rows in blocks against every column
    st = knn_blocked(ctx, db, db, true, random, kNN, out_col, jaccard, d_j, d_d, budget);
    if (st != SK_OK) return st;
  } else {
    st = scratch(ctx, kSlotOut, std::max<size_t>(pairs, 1) * 4, &d_vals);
    if (st != SK_OK) return st;
    if (pairs > 0) {
      st = dense_to_device(ctx, db, nullptr, random, kOutColumn, out_col, d_vals);
      if (st != SK_OK) return st;
    }
    e = launch_knn_self(static_cast<float *>(d_vals), n, kNN, jaccard, d_j, d_d, ctx->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(j_out, d_j, res_elems * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_out, d_d, res_elems * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "kNN");
  st = finish_call(ctx);
  if (st != SK_OK) return st;
  for (int64_t i = 0; i < n; ++i) std::fill_n(i_out + i * kNN, kNN, i);
  return SK_OK;
}

sk_status sk_query_knn(sk_ctx *ctx, const sk_db *ref, const sk_db *query, const sk_random *random,
                       int32_t kNN, int32_t dist_col, int64_t *r_out, float *d_out) {
  SK_GUARD(ctx);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (!ref || !query || ref->n < 1 || query->n < 1)
    return fail(ctx, SK_EINVAL, "Query with empty ref or query list!");
  if (dist_col != 0 && dist_col != 1) return fail(ctx, SK_EINVAL, "dist_col out of range");
  if (kNN < 0 || kNN > ref->n) return fail(ctx, SK_EINVAL, "kNN must be between 0 and the number of references");
  if (kNN == 0) return SK_OK;
  const int64_t pairs = n_pairs(ref, query);
  void *d_vals = nullptr, *d_res = nullptr;
  const size_t res_elems = static_cast<size_t>(query->n) * kNN;
  st = scratch(ctx, kSlotResult, res_elems * 12, &d_res);
  if (st != SK_OK) return st;
  int64_t *d_j = static_cast<int64_t *>(d_res);
  float *d_d = reinterpret_cast<float *>(d_j + res_elems);
  const size_t budget = dense_budget(ctx);
  cudaError_t e = cudaSuccess;
  if (static_cast<size_t>(pairs) * 4 > budget) {
    st = knn_blocked(ctx, ref, query, false, random, kNN, dist_col, 0, d_j, d_d, budget);
    if (st != SK_OK) return st;
  } else {
    st = scratch(ctx, kSlotOut, pairs * 4, &d_vals);
    if (st != SK_OK) return st;
    st = dense_to_device(ctx, ref, query, random, kOutColumn, dist_col, d_vals);
    if (st != SK_OK) return st;
    e = launch_knn_rows(static_cast<float *>(d_vals), query->n, ref->n, kNN, -1, 0, d_j, d_d,
                        ctx->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(r_out, d_j, res_elems * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_out, d_d, res_elems * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "query kNN");
  return finish_call(ctx);
}

// ---------------------------------------------------------- threshold sparse

static sk_status threshold_device(sk_ctx *ctx, const float *d_vals, int64_t n, int stride, int col,
                                  float cutoff, sk_sparse **out) {
  void *d_cnt = nullptr;
  sk_status st = scratch(ctx, kSlotResult, static_cast<size_t>(n + 1) * 16, &d_cnt);
  if (st != SK_OK) return st;
  int64_t *counts = static_cast<int64_t *>(d_cnt);
  int64_t *offsets = counts + (n + 1);
  cudaError_t e = cudaMemsetAsync(counts, 0, (n + 1) * 8, ctx->stream);
  if (e == cudaSuccess) e = launch_threshold_count(d_vals, n, stride, col, cutoff, counts, ctx->stream);
  size_t tmp_bytes = 0;
  if (e == cudaSuccess) e = exclusive_scan_i64(counts, offsets, n + 1, nullptr, &tmp_bytes, ctx->stream);
  void *tmp = nullptr;
  if (e == cudaSuccess) {
    st = scratch(ctx, kSlotTemp, std::max<size_t>(tmp_bytes, 16), &tmp);
    if (st != SK_OK) return st;
    e = exclusive_scan_i64(counts, offsets, n + 1, tmp, &tmp_bytes, ctx->stream);
  }
  int64_t total = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&total, offsets + n, 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "threshold count");
  sk_sparse *sp = new sk_sparse();
  sp->i.resize(total);
  sp->j.resize(total);
  sp->d.resize(total);
  if (total > 0) {
    void *d_res = nullptr;
    st = scratch(ctx, kSlotTemp, static_cast<size_t>(total) * 20, &d_res);
    if (st != SK_OK) { delete sp; return st; }
    int64_t *di = static_cast<int64_t *>(d_res);
    int64_t *dj = di + total;
    float *dd = reinterpret_cast<float *>(dj + total);
    e = launch_threshold_fill(d_vals, n, stride, col, cutoff, offsets, di, dj, dd, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sp->i.data(), di, total * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sp->j.data(), dj, total * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sp->d.data(), dd, total * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) { delete sp; return cuda_fail(ctx, e, "threshold fill"); }
  }
  st = finish_call(ctx);
  if (st != SK_OK) { delete sp; return st; }
  *out = sp;
  return SK_OK;
}

sk_status sk_sparse_threshold(sk_ctx *ctx, const float *long_form, int64_t n_samples, int32_t n_cols,
                              int32_t col, float cutoff, sk_sparse **out) {
  SK_GUARD(ctx);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (!out) return fail(ctx, SK_EINVAL, "null output handle");
  *out = nullptr;
  if (cutoff < 0) return fail(ctx, SK_EINVAL, "Distance threshold must be at least 0");
  if (n_samples < 0 || n_cols < 1 || col < 0 || col >= n_cols)
    return fail(ctx, SK_EINVAL, "bad long-form shape");
  const int64_t pairs = n_samples * (n_samples - 1) / 2;
  void *d_vals = nullptr;
  st = scratch(ctx, kSlotOut, std::max<int64_t>(pairs, 1) * n_cols * 4, &d_vals);
  if (st != SK_OK) return st;
  if (pairs > 0) {
    cudaError_t e = cudaMemcpyAsync(d_vals, long_form, pairs * n_cols * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "long-form upload");
  }
  return threshold_device(ctx, static_cast<float *>(d_vals), n_samples, n_cols, col, cutoff, out);
}

sk_status sk_dists_threshold(sk_ctx *ctx, const sk_db *db, const sk_random *random, int32_t dist_col,
                             float cutoff, sk_sparse **out) {
  SK_GUARD(ctx);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (!out) return fail(ctx, SK_EINVAL, "null output handle");
  *out = nullptr;
  if (cutoff < 0) return fail(ctx, SK_EINVAL, "Distance threshold must be at least 0");
  if (!db || db->n < 1) return fail(ctx, SK_EINVAL, "Query with empty ref or query list!");
  if (dist_col != 0 && dist_col != 1) return fail(ctx, SK_EINVAL, "dist_col out of range");
  const int64_t pairs = n_pairs(db, nullptr);
  void *d_vals = nullptr;
  st = scratch(ctx, kSlotOut, std::max<int64_t>(pairs, 1) * 4, &d_vals);
  if (st != SK_OK) return st;
  if (pairs > 0) {
    st = dense_to_device(ctx, db, nullptr, random, kOutColumn, dist_col, d_vals);
    if (st != SK_OK) return st;
  }
  return threshold_device(ctx, static_cast<float *>(d_vals), db->n, 1, 0, cutoff, out);
}

int64_t sk_sparse_size(const sk_sparse *sp) { return sp ? static_cast<int64_t>(sp->d.size()) : 0; }

sk_status sk_sparse_copy(const sk_sparse *sp, int64_t *i_out, int64_t *j_out, float *d_out) {
  if (!sp) return SK_EINVAL;
  if (i_out) std::copy(sp->i.begin(), sp->i.end(), i_out);
  if (j_out) std::copy(sp->j.begin(), sp->j.end(), j_out);
  if (d_out) std::copy(sp->d.begin(), sp->d.end(), d_out);
  return SK_OK;
}

sk_status sk_sparse_destroy(sk_sparse *sp) {
  if (!sp) return SK_EINVAL;
  delete sp;
  return SK_OK;
}

// ------------------------------------------------------------ long / square

sk_status sk_long_to_square(sk_ctx *ctx, const float *rr, int64_t n_rr, const float *qr,
                            const float *qq, int64_t n_qq, float *square) {
  SK_GUARD(ctx);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (n_rr < 0 || n_qq < 0 || (n_qq > 0 && !qr)) return fail(ctx, SK_EINVAL, "bad long-form shape");
  const int64_t n = n_rr + n_qq;
  if (n == 0) return SK_OK;
  const int64_t n_rr_long = n_rr * (n_rr - 1) / 2, n_qq_long = n_qq * (n_qq - 1) / 2;
  const int64_t n_qr = n_rr * n_qq;
  void *d = nullptr;
  const size_t bytes = (n_rr_long + n_qr + n_qq_long + n * n) * 4;
  st = scratch(ctx, kSlotOut, std::max<size_t>(bytes, 16), &d);
  if (st != SK_OK) return st;
  float *drr = static_cast<float *>(d), *dqr = drr + n_rr_long, *dqq = dqr + n_qr, *dsq = dqq + n_qq_long;
  cudaError_t e = cudaSuccess;
  if (n_rr_long) e = cudaMemcpyAsync(drr, rr, n_rr_long * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && n_qr) e = cudaMemcpyAsync(dqr, qr, n_qr * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && n_qq_long && qq) e = cudaMemcpyAsync(dqq, qq, n_qq_long * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = launch_long_to_square(drr, n_rr, dqr, dqq, n_qq, dsq, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(square, dsq, n * n * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "long_to_square");
  return finish_call(ctx);
}

sk_status sk_square_to_long(sk_ctx *ctx, const float *square, int64_t n, float *long_out) {
  SK_GUARD(ctx);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (n < 0) return fail(ctx, SK_EINVAL, "square_to_long input must be a square matrix");
  if (n < 2) return SK_OK;
  const int64_t n_long = n * (n - 1) / 2;
  void *d = nullptr;
  st = scratch(ctx, kSlotOut, (n * n + n_long) * 4, &d);
  if (st != SK_OK) return st;
  float *dsq = static_cast<float *>(d), *dl = dsq + n * n;
  cudaError_t e = cudaMemcpyAsync(dsq, square, n * n * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = launch_square_to_long(dsq, n, dl, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(long_out, dl, n_long * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "square_to_long");
  return finish_call(ctx);
}

// ---------------------------------------------------------------- synthetic

sk_status sk_synth_host(const int32_t *parent, const uint32_t *thresh, int64_t n_samples,
                        int32_t n_kmers, int32_t sketchsize64, uint64_t seed, int32_t threads,
                        uint64_t *words) {
  if (!parent || !thresh || !words || n_samples < 0 || n_kmers < 1 || sketchsize64 < 1)
    return SK_EINVAL;
  for (int64_t s = 0; s < n_samples; ++s)
    if (parent[s] >= s) return SK_EINVAL;  // parents precede children
  const int nt = std::max(1, threads);
  auto work = [&](int tid) {
    for (int64_t s = tid; s < n_samples; s += nt) {
      for (int k = 0; k < n_kmers; ++k) {
        for (int b = 0; b < sketchsize64; ++b) {
          uint64_t w[kBbits] = {0};
          for (int i = 0; i < 64; ++i) {
            const uint32_t v = synth_bin(parent, thresh, n_kmers, s, k, b * 64u + i, seed);
            for (int p = 0; p < kBbits; ++p) w[p] |= static_cast<uint64_t>((v >> p) & 1u) << i;
          }
          uint64_t *o = words + ((s * n_kmers + k) * static_cast<int64_t>(sketchsize64) + b) * kBbits;
          for (int p = 0; p < kBbits; ++p) o[p] = w[p];
        }
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto &t : pool) t.join();
  return SK_OK;
}

sk_status sk_synth_device(sk_ctx *ctx, const int32_t *parent, const uint32_t *thresh, int64_t n_samples,
                          int32_t n_kmers, int32_t sketchsize64, uint64_t seed, uint64_t *d_words) {
  SK_GUARD(ctx);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (!parent || !thresh || !d_words || n_samples < 1 || n_kmers < 1 || sketchsize64 < 1)
    return fail(ctx, SK_EINVAL, "bad synthetic generator arguments");
  for (int64_t s = 0; s < n_samples; ++s)
    if (parent[s] >= s) return fail(ctx, SK_EINVAL, "parents must precede their children");
  int32_t *d_parent = nullptr;
  uint32_t *d_thresh = nullptr;
  cudaError_t e = cudaMalloc(&d_parent, n_samples * 4);
  if (e == cudaSuccess) e = cudaMalloc(&d_thresh, n_samples * n_kmers * 4);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_parent, parent, n_samples * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_thresh, thresh, n_samples * n_kmers * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = launch_synth(d_parent, d_thresh, n_samples, n_kmers, sketchsize64, seed, d_words, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (d_parent) cudaFree(d_parent);
  if (d_thresh) cudaFree(d_thresh);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "synthetic sketches");
  return SK_OK;
}

}  // extern "C"
