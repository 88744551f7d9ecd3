// serve.cu -- a query server over a reference database resident in HBM.
//
// Requests (a batch of query sketches each) arrive at any time from any host
// thread.  A scheduler thread cuts every request into slices of at most
// `slice_queries` queries and runs slices on `slots`: each slot owns a
// context (its own stream and kernel scratch), a packed query buffer, a
// distance column for the slice against every reference and the kNN result
// buffers, all allocated once at start-up, so admission is by free slot and
// the server's HBM footprint is fixed (slots x slot bytes + the reference).
// Slices of different requests run on different streams and overlap on the
// device: a slot's persistent kernel takes SMs as another slot's kernel
// releases them.
//
// Scheduling.  The distance kernel is persistent and fills every SM, so
// slices queued on several streams run one after another; what decides a
// small request's latency is how many slices the block scheduler starts
// before its own.  So:
//   * free slots go to the request with the fewest queries left (shortest
//     remaining work first), FIFO among equals; a request older than
//     kStarveSeconds goes ahead of every younger one, so a stream of small
//     requests cannot hold a large one back for good;
//   * a request that fits in one slice runs on a high-priority stream: its
//     kernels start as soon as the slice on the SMs ends, ahead of slices of
//     larger requests already queued;
//   * slices of requests larger than one slice hold at most half the slots
//     (at least one), so a request of one slice finds a slot free and waits
//     at most for the slice already running, and the device still always has
//     a large slice queued behind the running one.
//
// Per slice: pinned staging copy of the query words, H2D, pack, the distance
// kernel (core or accessory column vs all references, optionally the full
// core/accessory rows), per-query top-kNN, D2H of the kNN lists (and rows).
// Results of each query depend only on that query and the references, so a
// request gets bit-identical results alone or in any mix.
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
  int64_t n = 0;
  std::vector<uint16_t> cluster;
  std::vector<uint64_t> seq_len;
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

struct Slot {
  sk_ctx *ctx = nullptr;
  sk_db qdb;                         // packed query buffer (pre-allocated)
  uint64_t *d_words = nullptr;       // staging of the reference-layout words
  uint64_t *h_words = nullptr;       // pinned host staging
  float *d_col = nullptr;            // [slice][n_ref] distance column
  float *d_rows = nullptr;           // [slice][n_ref][2] core/accessory (optional)
  int64_t *d_knn = nullptr;
  float *d_knn_d = nullptr;
  int64_t *h_knn = nullptr;          // pinned results
  float *h_knn_d = nullptr;
  float *h_rows = nullptr;
  cudaEvent_t done_ev = nullptr;
  cudaStream_t lo_stream = nullptr;  // the slot context's own stream
  cudaStream_t hi_stream = nullptr;  // greatest priority, for one-slice requests
  std::shared_ptr<Request> req;
  int64_t q0 = 0, nq = 0;
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
  double busy_s = 0;
  Clock::time_point t_start;
  std::string fatal;
};

namespace {

void free_slot(Slot &s) {
  if (s.ctx && s.lo_stream) s.ctx->stream = s.lo_stream;   // the context destroys its own
  if (s.hi_stream) cudaStreamDestroy(s.hi_stream);
  if (s.done_ev) cudaEventDestroy(s.done_ev);
  if (s.d_words) cudaFree(s.d_words);
  if (s.h_words) cudaFreeHost(s.h_words);
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

// Reserves, at start-up, the kernel scratch of the largest slice under every
// tile shape a slice can take (the default shape and the 64-row one of small
// batches).  Growing a scratch buffer mid-request would free the old one, and
// cudaFree waits for the whole device: every slot's work would stall behind
// it.  build_job on a full-size slice also creates the lazily built
// per-query random-match factors here.
sk_status reserve_slice_scratch(sk_server *sv, Slot &s) {
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
  if (st != SK_OK) return st;
  size_t meta = 0, cta = 16, split = 16;
  for (const TileConfig *c : {choose_config(ctx, ref->K, ref->s64), tile_config(kSmallQueryConfig)}) {
    if (!c || c->max_kmers < ref->K) continue;
    const int grid = resident_grid(ctx, *c);
    if (grid < 1) continue;
    const int64_t tiles = ((sq + c->tile_rows - 1) / c->tile_rows) *
                          ((ref->n + c->tile_cols - 1) / c->tile_cols);
    // the tail tiles (fewer than the grid) may each be cut into K parts
    const int64_t items = tiles + static_cast<int64_t>(grid) * ref->K;
    meta = std::max(meta, meta_layout(1, static_cast<size_t>(items), grid, c->threads).bytes);
    const size_t slot = count_slot_bytes(*c, ref->K);
    cta = std::max(cta, static_cast<size_t>(grid) * slot);
    split = std::max(split, static_cast<size_t>(grid) * slot);
  }
  void *p = nullptr;
  st = scratch(ctx, kSlotLaunchMeta, meta, &p);
  if (st == SK_OK) st = scratch(ctx, kSlotCounts, cta, &p);
  if (st == SK_OK) st = scratch(ctx, kSlotSplitCounts, split, &p);
  return st;
}

// Queues one slice on its slot's stream.  Called by the scheduler thread only.
sk_status start_slice(sk_server *sv, Slot &s) {
  sk_ctx *ctx = s.ctx;
  const sk_db *ref = sv->ref;
  const size_t wps = sv->words_per_sample;
  Request &r = *s.req;
  DeviceGuard g(ctx->device);
  ctx->stream = s.high ? s.hi_stream : s.lo_stream;
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  std::memcpy(s.h_words, r.words + s.q0 * wps, static_cast<size_t>(s.nq) * wps * 8);
  // the query database of this slice: same packed buffer, new samples
  s.qdb.n = s.nq;
  s.qdb.jv_rc = -1;   // equal-base factors depend on the samples
  if (!r.cluster.empty()) {
    cudaError_t e = cudaMemcpyAsync(s.qdb.cluster, r.cluster.data() + s.q0, s.nq * 2,
                                    cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "query clusters");
  }
  if (!r.seq_len.empty())
    s.qdb.seq_len.assign(r.seq_len.begin() + s.q0, r.seq_len.begin() + s.q0 + s.nq);
  else
    s.qdb.seq_len.assign(s.nq, 0);
  cudaError_t e = cudaMemcpyAsync(s.d_words, s.h_words, static_cast<size_t>(s.nq) * wps * 8,
                                  cudaMemcpyHostToDevice, ctx->stream);
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
  Request &r = *s.req;
  const int knn = sv->params.kNN;
  DevStatus dst{};
  {
    DeviceGuard g(s.ctx->device);
    cudaMemcpy(&dst, s.ctx->status_dev, sizeof(dst), cudaMemcpyDeviceToHost);
  }
  if (dst.error) {
    r.failed = true;
    r.error = (dst.error & 2u) ? "cancelled" : "device-side error";
  }
  if (knn > 0) {
    std::memcpy(r.knn_idx.data() + s.q0 * knn, s.h_knn, static_cast<size_t>(s.nq) * knn * 8);
    std::memcpy(r.knn_dist.data() + s.q0 * knn, s.h_knn_d, static_cast<size_t>(s.nq) * knn * 4);
  }
  if (sv->params.keep_rows)
    std::memcpy(r.rows.data() + s.q0 * sv->ref->n * 2, s.h_rows,
                static_cast<size_t>(s.nq) * sv->ref->n * 8);
  r.completed += s.nq;
  r.inflight -= 1;
  sv->pairs_done += s.nq * sv->ref->n;
  if (r.completed == r.n) {
    r.done = true;
    r.t_done = Clock::now();
  }
  s.req.reset();
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

void scheduler(sk_server *sv) {
  std::unique_lock<std::mutex> lock(sv->mu);
  const int64_t sq = sv->params.slice_queries;
  const int large_cap = std::max<int>(1, static_cast<int>(sv->slots.size()) / 2);
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
        s.req->failed = true;
        s.req->error = cudaGetErrorString(q);
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
      std::shared_ptr<Request> pick;
      for (auto &cand : sv->pending) {
        if (cand->dispatched >= cand->n) continue;
        if (cand->n > sq && large_busy >= large_cap) continue;
        if (!pick || goes_before(*cand, *pick, now)) pick = cand;
      }
      if (!pick) break;
      s.req = pick;
      s.high = pick->n <= sq;
      s.q0 = pick->dispatched;
      s.nq = std::min<int64_t>(s.high ? sq : sv->params.large_slice_queries,
                               pick->n - pick->dispatched);
      pick->dispatched += s.nq;
      pick->inflight += 1;
      s.busy = true;
      sk_status st = start_slice(sv, s);
      if (st != SK_OK) {
        pick->failed = true;
        pick->error = sk_last_error(s.ctx);
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
      p.kNN < 0 || p.kNN > 800 || p.kNN > ref->n || (p.dist_col != 0 && p.dist_col != 1))
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
  sv->slots.resize(p.slots);
  const int64_t sq = p.slice_queries;
  const int64_t npad = ((sq + kSamplePad - 1) / kSamplePad) * kSamplePad;
  sk_status st = SK_OK;
  for (Slot &s : sv->slots) {
    st = sk_ctx_create(ctx->device, &s.ctx);
    if (st != SK_OK) break;
    s.lo_stream = s.ctx->stream;
    {
      int least = 0, greatest = 0;
      cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
      if (e == cudaSuccess)
        e = cudaStreamCreateWithPriority(&s.hi_stream, cudaStreamNonBlocking, greatest);
      if (e != cudaSuccess) {
        st = cuda_fail(ctx, e, "server stream");
        break;
      }
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
    cudaError_t e = cudaMalloc(&s.qdb.packed, static_cast<size_t>(ref->K) * 2 * ref->s64 *
                                                  s.qdb.ng * kStripeWords * 4);
    if (e == cudaSuccess) e = cudaMalloc(&s.qdb.cluster, npad * 2);
    if (e == cudaSuccess) e = cudaMemset(s.qdb.cluster, 0, npad * 2);
    if (e == cudaSuccess) e = cudaMalloc(&s.d_words, sq * sv->words_per_sample * 8);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void **>(&s.h_words),
                                            sq * sv->words_per_sample * 8, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc(&s.d_col, sq * ref->n * 4);
    if (e == cudaSuccess && p.keep_rows) e = cudaMalloc(&s.d_rows, sq * ref->n * 8);
    if (e == cudaSuccess && p.keep_rows)
      e = cudaHostAlloc(reinterpret_cast<void **>(&s.h_rows), sq * ref->n * 8, cudaHostAllocDefault);
    if (e == cudaSuccess && p.kNN > 0) e = cudaMalloc(&s.d_knn, sq * p.kNN * 12);
    if (e == cudaSuccess && p.kNN > 0)
      e = cudaHostAlloc(reinterpret_cast<void **>(&s.h_knn), sq * p.kNN * 12, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done_ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      st = cuda_fail(ctx, e, "server slot allocation");
      break;
    }
    if (p.kNN > 0) {
      s.d_knn_d = reinterpret_cast<float *>(s.d_knn + sq * p.kNN);
      s.h_knn_d = reinterpret_cast<float *>(s.h_knn + sq * p.kNN);
    }
    st = reserve_slice_scratch(sv, s);
    if (st != SK_OK) {
      fail(ctx, st, "server slot scratch: %s", sk_last_error(s.ctx));
      break;
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
                           const uint16_t *cluster, const uint64_t *seq_len, int64_t *ticket) {
  if (!sv || !ticket || n_queries < 1 || !query_words) return SK_EINVAL;
  auto r = std::make_shared<Request>();
  r->words = query_words;
  r->n = n_queries;
  if (cluster) r->cluster.assign(cluster, cluster + n_queries);
  if (seq_len) r->seq_len.assign(seq_len, seq_len + n_queries);
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
