// query_db.cu -- host sketches in, host distances out, with the upload
// overlapped with the distance kernel.
//
// The reference's query_db_cuda (src/gpu/gpu_api.cpp:352-494) flattens every
// sketch on the host, copies them all, launches, waits, and copies the result
// back, one step after another.  Here the reference-layout words go up in
// sample chunks on the context's copy stream, double-buffered through a
// device staging area; each chunk is packed on a high-priority stream as soon
// as it lands, and the tiles whose samples have all arrived run as one
// persistent launch while the next chunk is in flight.
//
//   self:  the chunks go up from the last samples down: tile (ti, tj) reads
//          samples from ti QT on, so it runs after the chunk holding ti QT,
//          and that chunk's launch writes every pair of the chunk's rows.  With
//          a pinned destination those rows (one contiguous range of the long
//          form) are copied back on their own stream while lower chunks
//          compute.
//   query: the query samples go up first, then the references in chunks;
//          tile (ti, tj) runs after the reference chunk holding (tj+1) RT - 1.
//
// Each chunk's work list gets its own tail split (small early chunks are cut
// along k to fill the GPU) and its own control block.  Launches alternate
// between two compute streams with a count scratch each, so one launch's tail
// wave is filled by the next launch's CTAs.  The packed arrays, staging area
// and output staging are context scratch, so a repeated call allocates
// nothing.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "sk_runtime.h"

using namespace sk;

namespace {

constexpr int64_t kChunkAlign = 256;   // samples: a multiple of every tile side and of the padding
constexpr int64_t kMinChunk = 512;     // samples per chunk at least (the copy must be worth a launch)
constexpr int64_t kMaxChunks = 8;

// Samples per chunk for n samples: about n / 8, at least 512, 256-aligned.
int64_t chunk_samples(int64_t n) {
  const int64_t c = std::clamp<int64_t>((n + kMinChunk - 1) / kMinChunk, 1, kMaxChunks);
  const int64_t per = (n + c - 1) / c;
  return std::max<int64_t>(kChunkAlign, (per + kChunkAlign - 1) / kChunkAlign * kChunkAlign);
}

// The second compute stream, the high-priority pack stream and the join event.
sk_status ensure_compute_streams(sk_ctx *ctx) {
  cudaError_t e = cudaSuccess;
  if (!ctx->stream_b) e = cudaStreamCreateWithFlags(&ctx->stream_b, cudaStreamNonBlocking);
  if (e == cudaSuccess && !ctx->pack_stream) {
    int least = 0, greatest = 0;
    e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess)
      e = cudaStreamCreateWithPriority(&ctx->pack_stream, cudaStreamNonBlocking, greatest);
  }
  if (e == cudaSuccess && !ctx->ev_join) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
  if (e == cudaSuccess && !ctx->d2h_stream)
    e = cudaStreamCreateWithFlags(&ctx->d2h_stream, cudaStreamNonBlocking);
  return e == cudaSuccess ? SK_OK : cuda_fail(ctx, e, "compute stream setup");
}

// One host-to-device chunk.
struct Unit {
  sk_db *db;
  const uint64_t *host;   // first word of the chunk
  int64_t s0, n;          // first sample and sample count
  int chunk;              // reference chunk whose tiles become runnable, or -1
};

// The databases of one call, released after both streams are idle.
struct CallDbs {
  sk_ctx *ctx;
  sk_db *ref = nullptr, *query = nullptr;
  ~CallDbs() {
    for (cudaStream_t st : {ctx->copy_stream, ctx->pack_stream, ctx->stream_b, ctx->d2h_stream})
      if (st) cudaStreamSynchronize(st);
    cudaStreamSynchronize(ctx->stream);
    if (ref) db_free(ref);
    if (query) db_free(query);
  }
};

sk_status make_side(sk_ctx *ctx, const sk_host_sketches *h, const int32_t *kmers, int32_t K,
                    int32_t s64, int32_t bbits, int slot, sk_db **out) {
  if (h->n < 0) return fail(ctx, SK_EINVAL, "negative sample count");
  if (h->n > 0 && !h->words) return fail(ctx, SK_EINVAL, "null sketch words");
  sk_status st = db_alloc(ctx, h->n, kmers, K, s64, bbits, out, slot);
  if (st != SK_OK) return st;
  if (h->cluster || h->seq_len) return sk_db_set_sample_info(*out, h->cluster, h->seq_len);
  return SK_OK;
}

}  // namespace

extern "C" sk_status sk_query_db(sk_ctx *ctx, const sk_host_sketches *ref,
                                 const sk_host_sketches *query, const int32_t *kmers,
                                 int32_t n_kmers, int32_t sketchsize64, int32_t bbits,
                                 const sk_random *random, int32_t out_mode, void *out) {
  return sk_query_db_ready(ctx, ref, query, kmers, n_kmers, sketchsize64, bbits, random, out_mode,
                           out, nullptr, nullptr);
}

extern "C" sk_status sk_query_db_ready(sk_ctx *ctx, const sk_host_sketches *ref,
                                       const sk_host_sketches *query, const int32_t *kmers,
                                       int32_t n_kmers, int32_t sketchsize64, int32_t bbits,
                                       const sk_random *random, int32_t out_mode, void *out,
                                       sk_words_ready_fn ready, void *user) {
  if (!ctx) return SK_EINVAL;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  DeviceGuard dev(ctx->device);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (!ref) return fail(ctx, SK_EINVAL, "null reference sketches");
  if (ref->n < 1 || (query && query->n < 1))
    return fail(ctx, SK_EINVAL, "Query with empty ref or query list!");
  if (out_mode != kOutCoreAcc && out_mode != kOutJaccard && out_mode != kOutCounts)
    return fail(ctx, SK_EINVAL, "Unknown output mode %d", out_mode);
  st = ensure_copy_stream(ctx);
  if (st == SK_OK) st = ensure_compute_streams(ctx);
  if (st != SK_OK) return st;

  CallDbs dbs{ctx};
  st = make_side(ctx, ref, kmers, n_kmers, sketchsize64, bbits, kSlotPackedRef, &dbs.ref);
  if (st == SK_OK && query)
    st = make_side(ctx, query, kmers, n_kmers, sketchsize64, bbits, kSlotPackedQuery, &dbs.query);
  if (st != SK_OK) return st;
  const int64_t pairs = n_pairs(dbs.ref, dbs.query);
  if (pairs > 0 && !out) return fail(ctx, SK_EINVAL, "null output buffer");
  if (pairs == 0) return finish_call(ctx);
  const size_t out_sz = out_bytes(out_mode, pairs, n_kmers);
  // an output above the device memory allowed for it is computed in row
  // blocks after the upload (dense_blocked_to_host); the upload still streams
  const size_t budget = dense_budget(ctx);
  const bool blocked = out_sz > budget;
  void *d_out = nullptr;
  if (!blocked) {
    st = scratch(ctx, kSlotOut, out_sz, &d_out);
    if (st != SK_OK) return st;
  }

  JobParams jp;
  const TileConfig *cfg = nullptr;
  st = build_job(ctx, dbs.ref, dbs.query, random, out_mode, 0, d_out, &cfg, &jp);
  if (st == SK_OK) st = attach_count_tables(ctx, &jp);
  if (st != SK_OK) return st;
  const int grid = resident_grid(ctx, *cfg);
  if (grid < 1) return fail(ctx, SK_ECUDA, "Tile configuration %d does not fit the device", cfg->id);

  // ---- work lists, one per reference chunk
  const int64_t n_ref = dbs.ref->n;
  const int64_t cs = chunk_samples(n_ref);
  const int n_chunks = static_cast<int>((n_ref + cs - 1) / cs);
  std::vector<std::vector<int64_t>> bucket(n_chunks);
  const bool reverse = jp.self && !blocked;
  bool pinned_out = false;
  {
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, out) == cudaSuccess) pinned_out = pa.type == cudaMemoryTypeHost;
    else cudaGetLastError();   // not a pointer CUDA knows: pageable
  }
  const bool stream_out = reverse && pinned_out;
  {
    int64_t tile = 0;
    const int64_t m = jp.tile_rows / jp.tile_cols;
    for (int64_t ti = 0; ti < jp.n_row_tiles; ++ti) {
      const int64_t tj0 = jp.self ? ti * m : 0;
      for (int64_t tj = tj0; tj < jp.n_col_tiles; ++tj, ++tile) {
        const int64_t last_col = std::min<int64_t>((tj + 1) * jp.tile_cols, n_ref) - 1;
        const int64_t last_row = jp.self ? std::min<int64_t>((ti + 1) * jp.tile_rows, n_ref) - 1 : 0;
        bucket[reverse ? (ti * jp.tile_rows) / cs : std::max(last_col, last_row) / cs].push_back(tile);
      }
    }
  }
  std::vector<WorkItem> items;
  const std::vector<JobParams> job_list{jp};
  std::vector<size_t> start(n_chunks), count(n_chunks);
  std::vector<int32_t> splits(n_chunks);
  int32_t max_splits = 0;
  for (int c = 0; c < n_chunks; ++c) {
    start[c] = items.size();
    for (int64_t t : bucket[c])
      items.push_back(WorkItem{t, 0, 0, static_cast<int16_t>(jp.n_kmers), -1, 1});
    split_tail(items, start[c], grid, &splits[c], &job_list);
    count[c] = items.size() - start[c];
    max_splits = std::max(max_splits, splits[c]);
  }

  // ---- device buffers: job, all items, one control block per chunk
  const size_t items_off = (sizeof(JobParams) + 255) & ~static_cast<size_t>(255);
  const size_t ctrl_off = (items_off + items.size() * sizeof(WorkItem) + 255) & ~static_cast<size_t>(255);
  std::vector<size_t> ctrl_at(n_chunks);
  size_t meta_bytes = ctrl_off;
  for (int c = 0; c < n_chunks; ++c) {
    ctrl_at[c] = meta_bytes;
    meta_bytes += (8 + static_cast<size_t>(splits[c]) * cfg->threads * 4 + 255) & ~static_cast<size_t>(255);
  }
  const int32_t k_slots = items_slots(items, job_slots(jp));
  const size_t slot = count_slot_bytes(*cfg, k_slots);
  const int64_t wps = static_cast<int64_t>(n_kmers) * sketchsize64 * bbits;   // words per sample
  void *meta = nullptr, *staging = nullptr, *cta[2] = {}, *split[2] = {};
  const size_t split_bytes = std::max<size_t>(static_cast<size_t>(max_splits) * slot, 16);
  st = scratch(ctx, kSlotLaunchMeta, meta_bytes, &meta);
  if (st == SK_OK) st = scratch(ctx, kSlotCounts, static_cast<size_t>(grid) * slot, &cta[0]);
  if (st == SK_OK) st = scratch(ctx, kSlotCountsB, static_cast<size_t>(grid) * slot, &cta[1]);
  if (st == SK_OK) st = scratch(ctx, kSlotSplitCounts, split_bytes, &split[0]);
  if (st == SK_OK) st = scratch(ctx, kSlotSplitCountsB, split_bytes, &split[1]);
  if (st == SK_OK) st = scratch(ctx, kSlotStaging, static_cast<size_t>(2 * cs * wps) * 8, &staging);
  if (st != SK_OK) return st;
  char *m = static_cast<char *>(meta);
  cudaError_t e = cudaMemcpyAsync(m, &jp, sizeof(jp), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m + items_off, items.data(), items.size() * sizeof(WorkItem),
                        cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(m + ctrl_off, 0, meta_bytes - ctrl_off, ctx->stream);
  // the second compute stream starts after the status reset and the work list
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_join, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream_b, ctx->ev_join, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "work list upload");
  LaunchParams base{};
  base.jobs = reinterpret_cast<const JobParams *>(m);
  base.k_slots = k_slots;
  base.wide = needs_wide(jp) ? 1 : 0;
  base.status = ctx->status_dev;
  base.cancel = ctx->cancel_dev;
  const WorkItem *d_items = reinterpret_cast<const WorkItem *>(m + items_off);

  // ---- upload units: the query side whole (in chunk-sized pieces), then the
  // reference chunk by chunk
  std::vector<Unit> units;
  if (dbs.query)
    for (int64_t s0 = 0; s0 < dbs.query->n; s0 += cs)
      units.push_back(Unit{dbs.query, query->words + s0 * wps, s0, std::min(cs, dbs.query->n - s0), -1});
  for (int k = 0; k < n_chunks; ++k) {
    const int c = reverse ? n_chunks - 1 - k : k;
    const int64_t s0 = c * cs;
    units.push_back(Unit{dbs.ref, ref->words + s0 * wps, s0, std::min(cs, n_ref - s0), c});
  }
  while (ctx->ev_out.size() < static_cast<size_t>(n_chunks)) {
    cudaEvent_t ev = nullptr;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "chunk events");
    ctx->ev_out.push_back(ev);
  }
  const size_t elem = out_bytes(out_mode, 1, n_kmers);
  auto first_row = [&](int64_t i) { return n_ref * i - i * (i + 1) / 2; };   // rows of sample i start
  while (ctx->ev_chunk.size() < units.size()) {
    cudaEvent_t ev = nullptr;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "chunk events");
    ctx->ev_chunk.push_back(ev);
  }
  // copy stream: H2D of unit i into staging buffer i & 1 (once unit i - 2 is
  // packed); pack stream (high priority, so its CTAs take SMs first): pack unit
  // i; compute streams, alternating: the tiles chunk c completes, after its
  // pack.  Chunk launches on the two streams overlap, so one launch's tail
  // wave is filled by the next launch's CTAs; each stream has its own count
  // scratch and every launch its own control block.
  uint64_t *stage[2] = {static_cast<uint64_t *>(staging), static_cast<uint64_t *>(staging) + cs * wps};
  cudaStream_t compute[2] = {ctx->stream, ctx->stream_b};
  int launches = 0;
  for (size_t i = 0; i < units.size() && e == cudaSuccess; ++i) {
    const Unit &u = units[i];
    const int b = static_cast<int>(i & 1);
    if (ready && ready(user, u.db == dbs.query ? 1 : 0, u.s0, u.n) != 0)
      return fail(ctx, SK_ETIMEDOUT, "sketch words of samples %lld..%lld never became ready",
                  static_cast<long long>(u.s0), static_cast<long long>(u.s0 + u.n - 1));
    if (i >= 2) e = cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_free[b], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(stage[b], u.host, static_cast<size_t>(u.n * wps) * 8, cudaMemcpyHostToDevice,
                          ctx->copy_stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_ready[b], ctx->copy_stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->pack_stream, ctx->ev_ready[b], 0);
    const int32_t g0 = static_cast<int32_t>(u.s0 / kGranule);
    const bool last_of_db = u.s0 + u.n == u.db->n;
    const int32_t ng = last_of_db ? u.db->ng - g0 : static_cast<int32_t>(u.n / kGranule);
    if (e == cudaSuccess)
      e = launch_pack_range(stage[b], u.n, n_kmers, sketchsize64, ng, g0, u.db->ng, u.db->packed,
                            ctx->pack_stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_free[b], ctx->pack_stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_chunk[i], ctx->pack_stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "sketch upload");
    if (!blocked && u.chunk >= 0 && count[u.chunk] > 0) {
      const int w = launches++ & 1;
      LaunchParams lp = base;
      lp.cta_scratch = static_cast<uint16_t *>(cta[w]);
      lp.split_scratch = static_cast<uint16_t *>(split[w]);
      lp.items = d_items + start[u.chunk];
      lp.n_items = static_cast<int64_t>(count[u.chunk]);
      lp.item_counter = reinterpret_cast<unsigned long long *>(m + ctrl_at[u.chunk]);
      lp.split_done = reinterpret_cast<unsigned int *>(m + ctrl_at[u.chunk] + 8);
      const int g = static_cast<int>(std::min<int64_t>(grid, lp.n_items));
      e = cudaStreamWaitEvent(compute[w], ctx->ev_chunk[i], 0);   // packs complete in unit order
      if (e == cudaSuccess) e = cfg->launch(lp, g, compute[w]);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "distance kernel launch");
      if (stream_out) {   // this chunk's rows are final: copy them back now
        const int64_t i0 = u.chunk * cs, i1 = std::min<int64_t>((u.chunk + 1) * cs, n_ref - 1);
        if (i1 > i0) {
          const int64_t r0 = first_row(i0), r1 = first_row(i1);
          e = cudaEventRecord(ctx->ev_out[u.chunk], compute[w]);
          if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->d2h_stream, ctx->ev_out[u.chunk], 0);
          if (e == cudaSuccess)
            e = cudaMemcpyAsync(static_cast<char *>(out) + r0 * elem,
                                static_cast<char *>(d_out) + r0 * elem, (r1 - r0) * elem,
                                cudaMemcpyDeviceToHost, ctx->d2h_stream);
          if (e != cudaSuccess) return cuda_fail(ctx, e, "result copy");
        }
      }
    }
  }
  // join: the context stream waits for the last pack and the second stream
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_chunk[units.size() - 1], 0);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_join, ctx->stream_b);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "stream join");
  if (blocked) {
    st = dense_blocked_to_host(ctx, dbs.ref, dbs.query, random, out_mode, out, budget);
    return st == SK_OK ? finish_call(ctx) : st;
  }
  if (stream_out) {   // the rows went back chunk by chunk: wait for the last copies
    e = cudaEventRecord(ctx->ev_join, ctx->d2h_stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "result copy");
    return finish_call(ctx);
  }
  e = cudaMemcpyAsync(out, d_out, out_sz, cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "result copy");
  return finish_call(ctx);
}

extern "C" {

sk_status sk_host_alloc(int64_t bytes, void **out) {
  if (!out || bytes < 0) return SK_EINVAL;
  *out = nullptr;
  if (bytes == 0) return SK_OK;
  const cudaError_t e = cudaHostAlloc(out, static_cast<size_t>(bytes), cudaHostAllocPortable);
  if (e != cudaSuccess) {
    *out = nullptr;
    return SK_ENOMEM;
  }
  return SK_OK;
}

sk_status sk_host_free(void *ptr) {
  if (!ptr) return SK_OK;
  return cudaFreeHost(ptr) == cudaSuccess ? SK_OK : SK_ECUDA;
}

}  // extern "C"
