// serve.cu -- a query server over a reference database resident in HBM.
//
// Requests (a batch of query sketches each) arrive at any time from any host
// thread.  A scheduler thread packs waiting queries into slices and runs the
// slices on `slots`: each slot owns a context (its own stream and kernel
// scratch), a packed query buffer, a distance column for one slice against
// every reference and the kNN result buffers, all allocated once at start-up,
// so admission is by free slot, i.e. by free HBM, and the server's footprint
// is fixed (slots x slot bytes + the reference; `device_bytes` caps it).
// Slices run on different streams and overlap on the device: a slot's
// persistent kernel takes SMs as another slot's kernel releases them.
//
// Continuous batching.  A slice is a list of segments, each a run of one
// request's queries; the slice's queries go up, are packed and are scored as
// one query database in one launch, and each segment's results go back to its
// request.  Queries that arrive while the device is busy therefore share the
// next launch and its query tiles instead of each paying for a whole tile of
// their own.  Every query's result depends only on that query (its sketch,
// cluster id and length) and the references, so a request gets bit-identical
// results alone or in any mix.
//
// Scheduling.  The distance kernel is persistent and fills every SM, so
// slices queued on several streams run one after another; what decides a
// small request's latency is how many slices the block scheduler starts
// before its own.  So:
//   * free slots go to the request with the fewest queries left (shortest
//     remaining work first), FIFO among equals; a request older than
//     kStarveSeconds goes ahead of every younger one, so a stream of small
//     requests cannot hold a large one back for good;
//   * requests of at most slice_queries queries (small) run whole in one
//     slice on a high-priority stream, packed with other small requests in
//     that order while they fit: their kernels start as soon as the slice on
//     the SMs ends, ahead of slices of larger requests already queued;
//   * slices of larger requests (large_slice_queries queries, the tail of one
//     request continued by the head of the next) hold at most half the slots
//     (at least one), so a small request finds a slot free and waits at most
//     for the slice already running, and the device still always has a large
//     slice queued behind the running one;
//   * rows left free in a slice's last query tile are filled with queries of
//     larger requests: the kernel computes whole tiles anyway.
//
// Per slice: the query words uploaded straight from a request's page-locked
// buffer, or staged through the slot's pinned buffer when the caller's is
// pageable; cluster ids and lengths; H2D, pack, the distance kernel (core or accessory column vs all
// references, optionally the full core/accessory rows), per-query top-kNN,
// D2H of the kNN lists (and rows).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "sk_runtime.h"

using namespace sk;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  const uint64_t *words = nullptr;   // caller's host buffer, kept alive until done
  bool pinned = false;               // page-locked: uploaded directly, not staged
  int64_t n = 0;
  std::vector<uint16_t> cluster;     // [n] random-match cluster per query
  std::vector<uint64_t> seq_len;     // [n] sequence length per query
  int64_t dispatched = 0;            // queries handed to slots
  int64_t completed = 0;             // queries finished
  int inflight = 0;                  // slices on the device
  bool failed = false;
  std::string error;
  std::vector<int64_t> knn_idx;      // [n][kNN]
  std::vector<float> knn_dist;
  std::vector<float> rows;           // [n][n_ref][2] when dense output is kept
  Clock::time_point t_submit, t_done;
  bool done = false;
};

// A run of one request's queries inside a slice: queries q0 .. q0+nq-1 of
// the request are slice rows row0 .. row0+nq-1.
struct Segment {
  std::shared_ptr<Request> req;
  int64_t q0 = 0, nq = 0, row0 = 0;
};

struct Slot {
  sk_ctx *ctx = nullptr;
  sk_db qdb;                         // packed query buffer (pre-allocated)
  uint64_t *d_words = nullptr;       // staging of the reference-layout words
  uint64_t *h_words = nullptr;       // pinned host staging
  uint16_t *h_cluster = nullptr;     // pinned cluster ids of the slice's queries
  float *d_col = nullptr;            // [slice][n_ref] distance column
  float *d_rows = nullptr;           // [slice][n_ref][2] core/accessory (optional)
  int64_t *d_knn = nullptr;
  float *d_knn_d = nullptr;
  int64_t *h_knn = nullptr;          // pinned results
  float *h_knn_d = nullptr;
  float *h_rows = nullptr;
  cudaEvent_t done_ev = nullptr;
  cudaStream_t lo_stream = nullptr;  // the slot context's own stream
  cudaStream_t hi_stream = nullptr;  // greatest priority, for slices of small requests
  std::vector<Segment> segs;         // the running slice
  int64_t nq = 0;                    // queries in the running slice
  bool busy = false;
  bool high = false;                 // the running slice is on hi_stream
};

// A request waiting longer than this goes ahead of every younger request.
constexpr double kStarveSeconds = 2.0;

}  // namespace

struct sk_server {
  sk_ctx *ctx = nullptr;             // the reference database's context
  const sk_db *ref = nullptr;
  const sk_random *random = nullptr;
  sk_server_params params{};
  size_t words_per_sample = 0;
  int64_t slot_bytes = 0;            // device bytes one slot holds
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv;        // wakes the scheduler
  std::condition_variable done_cv;   // wakes waiters
  std::deque<std::shared_ptr<Request>> pending;   // not fully dispatched
  std::map<int64_t, std::shared_ptr<Request>> all;
  int64_t next_id = 1;
  bool stop = false;
  std::thread worker;
  // statistics
  int64_t pairs_done = 0;
  int64_t slices = 0, slices_shared = 0;
  Clock::time_point t_start;
};

namespace {

void free_slot(Slot &s) {
  if (s.ctx && s.lo_stream) s.ctx->stream = s.lo_stream;   // the context destroys its own
  if (s.hi_stream) cudaStreamDestroy(s.hi_stream);
  if (s.done_ev) cudaEventDestroy(s.done_ev);
  if (s.d_words) cudaFree(s.d_words);
  if (s.h_words) cudaFreeHost(s.h_words);
  if (s.h_cluster) cudaFreeHost(s.h_cluster);
  if (s.d_col) cudaFree(s.d_col);
  if (s.d_rows) cudaFree(s.d_rows);
  if (s.d_knn) cudaFree(s.d_knn);
  if (s.h_knn) cudaFreeHost(s.h_knn);
  if (s.h_rows) cudaFreeHost(s.h_rows);
  if (s.qdb.packed) cudaFree(s.qdb.packed);
  if (s.qdb.cluster) cudaFree(s.qdb.cluster);
  if (s.qdb.jv) cudaFree(s.qdb.jv);
  if (s.ctx) sk_ctx_destroy(s.ctx);
  s = Slot{};
}

// Device bytes of one slot's own buffers (kernel scratch comes on top and is
// measured when it is reserved).
int64_t slot_buffer_bytes(const sk_db *ref, const sk_server_params &p, size_t words_per_sample) {
  const int64_t sq = p.slice_queries;
  const int64_t npad = ((sq + kSamplePad - 1) / kSamplePad) * kSamplePad;
  int64_t b = static_cast<int64_t>(ref->K) * 2 * ref->s64 * (npad / kGranule) * kStripeWords * 4;
  b += npad * 2;                                          // cluster ids
  b += static_cast<int64_t>(ref->K) * npad * 8;           // equal-base factors
  b += sq * static_cast<int64_t>(words_per_sample) * 8;   // word staging
  b += sq * ref->n * 4;                                   // distance column
  if (p.keep_rows) b += sq * ref->n * 8;
  if (p.kNN > 0) b += sq * p.kNN * 12;
  return b;
}

// Reserves, at start-up, the kernel scratch of the largest slice under every
// tile shape a slice can take (the default shape and the 64-row one of small
// batches).  Growing a scratch buffer mid-request would free the old one, and
// cudaFree waits for the whole device: every slot's work would stall behind
// it.  build_job on a full-size slice also creates the lazily built
// per-query random-match factors here.  Adds the scratch bytes to *bytes.
sk_status reserve_slice_scratch(sk_server *sv, Slot &s, int64_t *bytes) {
  sk_ctx *ctx = s.ctx;
  const sk_db *ref = sv->ref;
  const int64_t sq = sv->params.slice_queries;
  s.qdb.n = sq;
  s.qdb.jv_rc = -1;
  s.qdb.seq_len.assign(sq, 0);
  JobParams jp;
  const TileConfig *cfg = nullptr;
  sk_status st = build_job(ctx, ref, &s.qdb, sv->random, kOutColumn, sv->params.dist_col,
                           s.d_col, &cfg, &jp);
  // the slices' Jaccard tables are built now, not on the first request
  if (st == SK_OK) st = attach_count_tables(ctx, &jp);
  if (st != SK_OK) return st;
  size_t meta = 0, cta = 16, split = 16;
  for (const TileConfig *c : {choose_config(ctx, ref->K, ref->s64), tile_config(kSmallQueryConfig)}) {
    if (!c || c->max_kmers < ref->K) continue;
    const int grid = resident_grid(ctx, *c);
    if (grid < 1) continue;
    const int64_t tiles = ((sq + c->tile_rows - 1) / c->tile_rows) *
                          ((ref->n + c->tile_cols - 1) / c->tile_cols);
    // the tail tiles (fewer than the grid) may each be cut into K parts and
    // each part into block ranges, every range its own count slot
    const int32_t q = tail_block_parts(jp);
    const int64_t items = tiles + static_cast<int64_t>(grid) * ref->K * q;
    meta = std::max(meta, meta_layout(1, static_cast<size_t>(items), grid, c->threads).bytes);
    const size_t slot = count_slot_bytes(*c, std::max(job_slots(jp), ref->K * q));
    cta = std::max(cta, static_cast<size_t>(grid) * slot);
    split = std::max(split, static_cast<size_t>(grid) * slot);
  }
  void *p = nullptr;
  st = scratch(ctx, kSlotLaunchMeta, meta, &p);
  if (st == SK_OK) st = scratch(ctx, kSlotCounts, cta, &p);
  if (st == SK_OK) st = scratch(ctx, kSlotSplitCounts, split, &p);
  *bytes += static_cast<int64_t>(meta + cta + split);
  return st;
}

// Queues one slice on its slot's stream.  Called by the scheduler thread only.
sk_status start_slice(sk_server *sv, Slot &s) {
  sk_ctx *ctx = s.ctx;
  const sk_db *ref = sv->ref;
  const size_t wps = sv->words_per_sample;
  DeviceGuard g(ctx->device);
  ctx->stream = s.high ? s.hi_stream : s.lo_stream;
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  // the query database of this slice: same packed buffer, new samples, and
  // every query's cluster id and length set again (nothing is kept from the
  // slot's previous slice)
  s.qdb.n = s.nq;
  s.qdb.jv_rc = -1;   // equal-base factors depend on the samples
  s.qdb.seq_len.resize(s.nq);
  cudaError_t e = cudaSuccess;
  bool staged = false;
  for (const Segment &seg : s.segs) {
    const Request &r = *seg.req;
    const size_t bytes = static_cast<size_t>(seg.nq) * wps * 8;
    if (r.pinned) {   // straight from the caller's page-locked buffer
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(s.d_words + seg.row0 * wps, r.words + seg.q0 * wps, bytes,
                            cudaMemcpyHostToDevice, ctx->stream);
    } else {
      std::memcpy(s.h_words + seg.row0 * wps, r.words + seg.q0 * wps, bytes);
      staged = true;
    }
    std::copy(r.cluster.begin() + seg.q0, r.cluster.begin() + seg.q0 + seg.nq,
              s.h_cluster + seg.row0);
    std::copy(r.seq_len.begin() + seg.q0, r.seq_len.begin() + seg.q0 + seg.nq,
              s.qdb.seq_len.begin() + seg.row0);
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.qdb.cluster, s.h_cluster, s.nq * 2, cudaMemcpyHostToDevice, ctx->stream);
  // staged segments go up in one copy per contiguous run of rows
  for (size_t a = 0; staged && e == cudaSuccess && a < s.segs.size();) {
    if (s.segs[a].req->pinned) {
      ++a;
      continue;
    }
    size_t b = a + 1;
    while (b < s.segs.size() && !s.segs[b].req->pinned) ++b;
    const int64_t r0 = s.segs[a].row0, r1 = s.segs[b - 1].row0 + s.segs[b - 1].nq;
    e = cudaMemcpyAsync(s.d_words + r0 * wps, s.h_words + r0 * wps,
                        static_cast<size_t>(r1 - r0) * wps * 8, cudaMemcpyHostToDevice,
                        ctx->stream);
    a = b;
  }
  if (e == cudaSuccess)
    e = launch_pack(s.d_words, s.nq, ref->K, ref->s64, s.qdb.ng, s.qdb.packed, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "query upload");
  const int col = sv->params.dist_col;
  if (sv->params.keep_rows) {
    st = dense_to_device(ctx, ref, &s.qdb, sv->random, kOutCoreAcc, 0, s.d_rows);
    if (st != SK_OK) return st;
    e = cudaMemcpyAsync(s.h_rows, s.d_rows, static_cast<size_t>(s.nq) * ref->n * 8,
                        cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "row copy");
  }
  st = dense_to_device(ctx, ref, &s.qdb, sv->random, kOutColumn, col, s.d_col);
  if (st != SK_OK) return st;
  const int knn = sv->params.kNN;
  if (knn > 0) {
    e = launch_knn_rows(s.d_col, s.nq, ref->n, knn, -1, 0, s.d_knn, s.d_knn_d, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s.h_knn, s.d_knn, static_cast<size_t>(s.nq) * knn * 8,
                          cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s.h_knn_d, s.d_knn_d, static_cast<size_t>(s.nq) * knn * 4,
                          cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "kNN");
  }
  e = cudaEventRecord(s.done_ev, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "event");
  return SK_OK;
}

void finish_slice(sk_server *sv, Slot &s) {
  const int knn = sv->params.kNN;
  const int64_t n_ref = sv->ref->n;
  DevStatus dst{};
  {
    DeviceGuard g(s.ctx->device);
    cudaMemcpy(&dst, s.ctx->status_dev, sizeof(dst), cudaMemcpyDeviceToHost);
  }
  for (const Segment &seg : s.segs) {
    Request &r = *seg.req;
    if (dst.error) {
      r.failed = true;
      r.error = (dst.error & 2u) ? "cancelled" : "device-side error";
    }
    if (knn > 0) {
      std::memcpy(r.knn_idx.data() + seg.q0 * knn, s.h_knn + seg.row0 * knn,
                  static_cast<size_t>(seg.nq) * knn * 8);
      std::memcpy(r.knn_dist.data() + seg.q0 * knn, s.h_knn_d + seg.row0 * knn,
                  static_cast<size_t>(seg.nq) * knn * 4);
    }
    if (sv->params.keep_rows)
      std::memcpy(r.rows.data() + seg.q0 * n_ref * 2, s.h_rows + seg.row0 * n_ref * 2,
                  static_cast<size_t>(seg.nq) * n_ref * 8);
    r.completed += seg.nq;
    r.inflight -= 1;
    if (r.completed == r.n) {
      r.done = true;
      r.t_done = Clock::now();
    }
  }
  sv->pairs_done += s.nq * n_ref;
  s.segs.clear();
  s.nq = 0;
  s.busy = false;
}

// Admission order: a request waiting longer than kStarveSeconds first (FIFO
// among those), then the fewest queries left, then FIFO.
bool goes_before(const Request &a, const Request &b, Clock::time_point now) {
  const bool sa = std::chrono::duration<double>(now - a.t_submit).count() > kStarveSeconds;
  const bool sb = std::chrono::duration<double>(now - b.t_submit).count() > kStarveSeconds;
  if (sa != sb) return sa;
  if (!sa) {
    const int64_t ra = a.n - a.dispatched, rb = b.n - b.dispatched;
    if (ra != rb) return ra < rb;
  }
  return a.id < b.id;
}

// Appends up to `room` queries of request r (from its next undispatched one)
// to the slot's slice.  Returns the number taken.
int64_t take(Slot &s, const std::shared_ptr<Request> &r, int64_t room) {
  const int64_t nq = std::min(room, r->n - r->dispatched);
  if (nq <= 0) return 0;
  s.segs.push_back(Segment{r, r->dispatched, nq, s.nq});
  r->dispatched += nq;
  r->inflight += 1;
  s.nq += nq;
  return nq;
}

// Rows of the query tile(s) a slice of nq queries occupies: the 64-row tile
// of at most 64 queries, else 128-row tiles (build_job's choice).
int64_t tile_rows_for(int64_t nq) { return nq <= 64 ? 64 : ((nq + 127) / 128) * 128; }

// Fills a free slot with the next slice, or leaves it empty when nothing may
// start now.  `order` is the pending requests in admission order.
void compose_slice(sk_server *sv, Slot &s, const std::vector<std::shared_ptr<Request>> &order,
                   int large_busy, int large_cap) {
  const int64_t sq = sv->params.slice_queries;
  auto small = [&](const Request &r) { return r.n <= sq && r.dispatched == 0; };
  auto open = [](const Request &r) { return r.dispatched < r.n; };
  std::shared_ptr<Request> first;
  for (const auto &r : order) {
    if (!open(*r)) continue;
    if (small(*r) || large_busy < large_cap) {
      first = r;
      break;
    }
  }
  if (!first) return;
  s.segs.clear();
  s.nq = 0;
  if (small(*first)) {
    // whole small requests, in admission order, while they fit
    s.high = true;
    for (const auto &r : order)
      if (small(*r) && s.nq + r->n <= sq) take(s, r, r->n);
  } else {
    // large_slice_queries queries of the large requests, in admission order
    s.high = false;
    const int64_t cap = sv->params.large_slice_queries;
    for (const auto &r : order) {
      if (s.nq >= cap) break;
      if (open(*r) && !small(*r)) take(s, r, cap - s.nq);
    }
  }
  // free rows of the last query tile: queries of large requests ride along
  const int64_t fill = std::min(tile_rows_for(s.nq), sq);
  for (const auto &r : order) {
    if (s.nq >= fill) break;
    if (open(*r) && !small(*r)) take(s, r, fill - s.nq);
  }
}

void scheduler(sk_server *sv) {
  std::unique_lock<std::mutex> lock(sv->mu);
  const int large_cap = std::max<int>(1, static_cast<int>(sv->slots.size()) / 2);
  std::vector<std::shared_ptr<Request>> order;
  while (true) {
    bool progressed = false;
    // completions
    for (Slot &s : sv->slots) {
      if (!s.busy) continue;
      cudaError_t q;
      {
        DeviceGuard g(s.ctx->device);
        q = cudaEventQuery(s.done_ev);
      }
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) {
        for (Segment &seg : s.segs) {
          seg.req->failed = true;
          seg.req->error = cudaGetErrorString(q);
        }
      }
      finish_slice(sv, s);
      progressed = true;
    }
    if (progressed) sv->done_cv.notify_all();
    // admissions
    for (Slot &s : sv->slots) {
      if (s.busy || sv->pending.empty()) continue;
      int large_busy = 0;
      for (const Slot &o : sv->slots) large_busy += (o.busy && !o.high) ? 1 : 0;
      const auto now = Clock::now();
      order.assign(sv->pending.begin(), sv->pending.end());
      std::stable_sort(order.begin(), order.end(),
                       [now](const std::shared_ptr<Request> &a, const std::shared_ptr<Request> &b) {
                         return goes_before(*a, *b, now);
                       });
      compose_slice(sv, s, order, large_busy, large_cap);
      if (s.nq == 0) break;
      s.busy = true;
      sv->slices += 1;
      sv->slices_shared += s.segs.size() > 1 ? 1 : 0;
      sk_status st = start_slice(sv, s);
      if (st != SK_OK) {
        for (Segment &seg : s.segs) {
          seg.req->failed = true;
          seg.req->error = sk_last_error(s.ctx);
        }
        // the slice still completes through its event (recorded or not)
        DeviceGuard g(s.ctx->device);
        cudaEventRecord(s.done_ev, s.ctx->stream);
      }
      progressed = true;
    }
    // drop fully dispatched requests from the pending list
    sv->pending.erase(std::remove_if(sv->pending.begin(), sv->pending.end(),
                                     [](const std::shared_ptr<Request> &r) {
                                       return r->dispatched >= r->n;
                                     }),
                      sv->pending.end());
    bool any_busy = false;
    for (Slot &s : sv->slots) any_busy |= s.busy;
    if (sv->stop && !any_busy && sv->pending.empty()) break;
    if (!progressed) {
      if (any_busy)
        sv->cv.wait_for(lock, std::chrono::microseconds(100));
      else
        sv->cv.wait_for(lock, std::chrono::milliseconds(50));
    }
  }
}

// One slot: its context and streams, buffers, and reserved kernel scratch.
// Adds the device bytes it holds to *bytes.
sk_status make_slot(sk_server *sv, sk_ctx *ctx, Slot &s, int64_t *bytes) {
  const sk_db *ref = sv->ref;
  const sk_server_params &p = sv->params;
  const int64_t sq = p.slice_queries;
  const int64_t npad = ((sq + kSamplePad - 1) / kSamplePad) * kSamplePad;
  sk_status st = sk_ctx_create(ctx->device, &s.ctx);
  if (st != SK_OK) return st;
  s.lo_stream = s.ctx->stream;
  {
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess)
      e = cudaStreamCreateWithPriority(&s.hi_stream, cudaStreamNonBlocking, greatest);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "server stream");
  }
  s.ctx->tile_cfg = ctx->tile_cfg;
  s.ctx->tuning = ctx->tuning;
  s.ctx->semantics = ctx->semantics;   // fixed for the server's lifetime
  s.qdb.ctx = s.ctx;
  s.qdb.K = ref->K;
  s.qdb.s64 = ref->s64;
  s.qdb.bbits = ref->bbits;
  s.qdb.kmers = ref->kmers;
  s.qdb.ng = static_cast<int32_t>(npad / kGranule);
  const size_t wps = sv->words_per_sample;
  cudaError_t e = cudaMalloc(&s.qdb.packed, static_cast<size_t>(ref->K) * 2 * ref->s64 *
                                                s.qdb.ng * kStripeWords * 4);
  if (e == cudaSuccess) e = cudaMalloc(&s.qdb.cluster, npad * 2);
  if (e == cudaSuccess) e = cudaMemset(s.qdb.cluster, 0, npad * 2);
  if (e == cudaSuccess) e = cudaMalloc(&s.d_words, sq * wps * 8);
  if (e == cudaSuccess)
    e = cudaHostAlloc(reinterpret_cast<void **>(&s.h_words), sq * wps * 8, cudaHostAllocDefault);
  if (e == cudaSuccess)
    e = cudaHostAlloc(reinterpret_cast<void **>(&s.h_cluster), sq * 2, cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaMalloc(&s.d_col, sq * ref->n * 4);
  if (e == cudaSuccess && p.keep_rows) e = cudaMalloc(&s.d_rows, sq * ref->n * 8);
  if (e == cudaSuccess && p.keep_rows)
    e = cudaHostAlloc(reinterpret_cast<void **>(&s.h_rows), sq * ref->n * 8, cudaHostAllocDefault);
  if (e == cudaSuccess && p.kNN > 0) e = cudaMalloc(&s.d_knn, sq * p.kNN * 12);
  if (e == cudaSuccess && p.kNN > 0)
    e = cudaHostAlloc(reinterpret_cast<void **>(&s.h_knn), sq * p.kNN * 12, cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done_ev, cudaEventDisableTiming);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "server slot allocation");
  if (p.kNN > 0) {
    s.d_knn_d = reinterpret_cast<float *>(s.d_knn + sq * p.kNN);
    s.h_knn_d = reinterpret_cast<float *>(s.h_knn + sq * p.kNN);
  }
  *bytes += slot_buffer_bytes(ref, p, wps);
  st = reserve_slice_scratch(sv, s, bytes);
  if (st != SK_OK) return fail(ctx, st, "server slot scratch: %s", sk_last_error(s.ctx));
  return SK_OK;
}

}  // namespace

extern "C" {

sk_status sk_server_create(sk_ctx *ctx, const sk_db *ref, const sk_random *random,
                           const sk_server_params *params, sk_server **out) {
  if (!ctx) return SK_EINVAL;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  DeviceGuard g(ctx->device);
  ctx->err.clear();
  if (!out || !ref || !params) return fail(ctx, SK_EINVAL, "null argument");
  *out = nullptr;
  if (ref->n < 1) return fail(ctx, SK_EINVAL, "Query with empty ref or query list!");
  const sk_server_params &p = *params;
  if (p.slots < 1 || p.slots > 16 || p.slice_queries < 1 || p.slice_queries > 65536 ||
      p.large_slice_queries < 0 || p.large_slice_queries > p.slice_queries ||
      p.kNN < 0 || p.kNN > ref->n || (p.dist_col != 0 && p.dist_col != 1) ||
      p.device_bytes < 0)
    return fail(ctx, SK_EINVAL, "bad server parameters");
  if (random && random->kmers != ref->kmers)
    return fail(ctx, SK_EMISMATCH, "Random match table k-mer lengths differ from the sketches");
  if (random && random->mode == kRandEqualBase) {
    sk_status st = ensure_jv(ctx, const_cast<sk_db *>(ref), random->use_rc);   // before threads
    if (st != SK_OK) return st;
  }
  sk_server *sv = new sk_server();
  sv->ctx = ctx;
  sv->ref = ref;
  sv->random = random;
  sv->params = p;
  if (sv->params.large_slice_queries == 0) sv->params.large_slice_queries = p.slice_queries;
  sv->words_per_sample = static_cast<size_t>(ref->K) * ref->s64 * kBbits;
  // Slots are made one at a time; under a budget, the first slot's measured
  // bytes decide how many fit.
  sk_status st = SK_OK;
  int target = p.slots;
  for (int i = 0; i < target; ++i) {
    sv->slots.emplace_back();
    int64_t bytes = 0;
    st = make_slot(sv, ctx, sv->slots.back(), &bytes);
    if (st != SK_OK) break;
    if (i == 0) {
      sv->slot_bytes = bytes;
      if (p.device_bytes > 0) {
        if (p.device_bytes < bytes) {
          st = fail(ctx, SK_ENOMEM, "server budget of %lld bytes is below one slot (%lld bytes)",
                    static_cast<long long>(p.device_bytes), static_cast<long long>(bytes));
          break;
        }
        target = static_cast<int>(std::min<int64_t>(p.slots, p.device_bytes / bytes));
      }
    }
  }
  if (st != SK_OK) {
    for (Slot &s : sv->slots) free_slot(s);
    delete sv;
    return st;
  }
  ctx_retain(ctx);
  sv->t_start = Clock::now();
  sv->worker = std::thread(scheduler, sv);
  *out = sv;
  return SK_OK;
}

sk_status sk_server_submit(sk_server *sv, const uint64_t *query_words, int64_t n_queries,
                           const uint16_t *cluster, const uint64_t *seq_len,
                           const double *base_freq, int64_t *ticket) {
  if (!sv || !ticket || n_queries < 1 || !query_words) return SK_EINVAL;
  auto r = std::make_shared<Request>();
  r->words = query_words;
  r->n = n_queries;
  {
    DeviceGuard g(sv->ctx->device);   // the query runs on the server's device, not device 0
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, query_words) == cudaSuccess)
      r->pinned = attr.type == cudaMemoryTypeHost;
    cudaGetLastError();   // a pageable pointer is not an error worth keeping
  }
  if (cluster) {
    r->cluster.assign(cluster, cluster + n_queries);
    // an id beyond the random-match table would index past it on the device
    const sk_random *rnd = sv->random;
    if (rnd && rnd->mode == kRandTable &&
        *std::max_element(r->cluster.begin(), r->cluster.end()) >= rnd->n_clusters)
      return SK_EINVAL;
  } else {
    r->cluster.assign(n_queries, 0);
    const sk_random *rnd = sv->random;
    if (base_freq && rnd && rnd->mode == kRandTable && !rnd->centroids.empty()) {
      const sk_status st = sk_closest_cluster(rnd->centroids.data(), rnd->n_clusters, rnd->use_rc,
                                              base_freq, n_queries, r->cluster.data());
      if (st != SK_OK) return st;
    }
  }
  if (seq_len) r->seq_len.assign(seq_len, seq_len + n_queries);
  else r->seq_len.assign(n_queries, 0);
  if (sv->params.kNN > 0) {
    r->knn_idx.assign(static_cast<size_t>(n_queries) * sv->params.kNN, -1);
    r->knn_dist.assign(static_cast<size_t>(n_queries) * sv->params.kNN, 0.0f);
  }
  if (sv->params.keep_rows) r->rows.assign(static_cast<size_t>(n_queries) * sv->ref->n * 2, 0.0f);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    if (sv->stop) return SK_EINVAL;
    r->id = sv->next_id++;
    sv->pending.push_back(r);
    sv->all[r->id] = r;
  }
  sv->cv.notify_one();
  *ticket = r->id;
  return SK_OK;
}

sk_status sk_server_wait(sk_server *sv, int64_t ticket, double timeout_s) {
  if (!sv) return SK_EINVAL;
  std::unique_lock<std::mutex> lock(sv->mu);
  auto it = sv->all.find(ticket);
  if (it == sv->all.end()) return SK_EINVAL;
  std::shared_ptr<Request> r = it->second;
  const auto deadline = Clock::now() + std::chrono::duration<double>(timeout_s);
  while (!r->done) {
    if (sv->done_cv.wait_until(lock, deadline) == std::cv_status::timeout && !r->done)
      return SK_ETIMEDOUT;
  }
  return r->failed ? SK_EKERNEL : SK_OK;
}

sk_status sk_server_result(sk_server *sv, int64_t ticket, int64_t *knn_idx, float *knn_dist,
                           float *rows, double *latency_s) {
  if (!sv) return SK_EINVAL;
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->all.find(ticket);
  if (it == sv->all.end()) return SK_EINVAL;
  Request &r = *it->second;
  if (!r.done) return SK_EINVAL;
  if (knn_idx) std::copy(r.knn_idx.begin(), r.knn_idx.end(), knn_idx);
  if (knn_dist) std::copy(r.knn_dist.begin(), r.knn_dist.end(), knn_dist);
  if (rows) std::copy(r.rows.begin(), r.rows.end(), rows);
  if (latency_s) *latency_s = std::chrono::duration<double>(r.t_done - r.t_submit).count();
  return r.failed ? SK_EKERNEL : SK_OK;
}

sk_status sk_server_release(sk_server *sv, int64_t ticket) {
  if (!sv) return SK_EINVAL;
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->all.find(ticket);
  if (it == sv->all.end() || !it->second->done) return SK_EINVAL;
  sv->all.erase(it);
  return SK_OK;
}

sk_status sk_server_stats(sk_server *sv, int64_t *pairs_done, double *uptime_s,
                          int64_t *queued_queries) {
  if (!sv) return SK_EINVAL;
  std::lock_guard<std::mutex> lock(sv->mu);
  if (pairs_done) *pairs_done = sv->pairs_done;
  if (uptime_s) *uptime_s = std::chrono::duration<double>(Clock::now() - sv->t_start).count();
  if (queued_queries) {
    int64_t q = 0;
    for (auto &r : sv->pending) q += r->n - r->dispatched;
    *queued_queries = q;
  }
  return SK_OK;
}

sk_status sk_server_info(sk_server *sv, int32_t *slots, int64_t *slot_bytes, int64_t *slices,
                         int64_t *slices_shared) {
  if (!sv) return SK_EINVAL;
  std::lock_guard<std::mutex> lock(sv->mu);
  if (slots) *slots = static_cast<int32_t>(sv->slots.size());
  if (slot_bytes) *slot_bytes = sv->slot_bytes;
  if (slices) *slices = sv->slices;
  if (slices_shared) *slices_shared = sv->slices_shared;
  return SK_OK;
}

sk_status sk_server_destroy(sk_server *sv) {
  if (!sv) return SK_EINVAL;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->stop = true;
  }
  sv->cv.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  for (Slot &s : sv->slots) {
    DeviceGuard g(s.ctx ? s.ctx->device : 0);
    free_slot(s);
  }
  sk_ctx *ctx = sv->ctx;
  delete sv;
  ctx_release(ctx);
  return SK_OK;
}

}  // extern "C"
