// pp_sketchlib_module.cpp -- the drop-in pybind11 module.
//
// Mirrors the distance entry points of the reference module
// (src/sketchlib_bindings.cpp:238-312): same function names, keyword
// arguments, defaults, return types and error messages, with every distance
// computed by the B200 library through its C ABI (include/sketchlib_b200.h).
// Sketch databases are read with the built-in HDF5 reader (host_h5.cpp), so no
// libhdf5 is needed.
//
// Differences from the reference, by design:
//   * there is no CPU distance path: use_gpu is accepted and ignored, all work
//     runs on device_id;
//   * Jaccard output and kNN on Jaccard run on the GPU (the reference GPU path
//     refuses both, sketchlib_bindings.cpp:98-101, 144-147);
//   * fewer than two k-mer lengths with core/accessory output raises instead
//     of exiting the process (linear_regression.cpp:51-58);
//   * constructDatabase sketches on the GPU (sk_sketch) and writes the
//     database with the built-in HDF5 writer (host_h5_write.cpp); it computes
//     no Monte Carlo random-match table (calc_random only prints a note), and
//     a read filter (min_count) counts k-mers exactly.  addRandom raises
//     NotImplementedError.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include <algorithm>
#include <array>
#include <cstdio>
#include <iostream>
#include <sys/stat.h>

#include "host_db.h"
#include "host_h5.h"
#include "host_h5_write.h"
#include "host_seqio.h"
#include "sketchlib_b200.h"

namespace py = pybind11;

using sparse_coo = std::tuple<std::vector<long>, std::vector<long>, std::vector<float>>;
using FloatArray = py::array_t<float, py::array::c_style | py::array::forcecast>;

namespace {

// ------------------------------------------------------------- C ABI glue

std::mutex g_ctx_mu;
std::map<int, sk_ctx *> g_ctx;

sk_ctx *context(int device_id) {
  std::lock_guard<std::mutex> lock(g_ctx_mu);
  auto it = g_ctx.find(device_id);
  if (it != g_ctx.end()) return it->second;
  sk_ctx *ctx = nullptr;
  if (sk_ctx_create(device_id, &ctx) != SK_OK)
    throw std::runtime_error("Unable to open CUDA device " + std::to_string(device_id));
  g_ctx[device_id] = ctx;
  return ctx;
}

void check(sk_ctx *ctx, sk_status st) {
  if (st != SK_OK) throw std::runtime_error(sk_last_error(ctx));
}

// Runs a library call with the GIL released, polling for Ctrl-C like the
// reference's progress loop (src/gpu/dist.cu:351-370): an interrupt cancels
// the running kernels (sk_cancel) and raises KeyboardInterrupt here.
// The wait wakes as soon as the call returns (a 20 ms sleep between polls
// added 10 ms to a call on average).
template <class F>
void run_gpu(sk_ctx *ctx, F &&fn) {
  std::mutex mu;
  std::condition_variable cv;
  bool done = false;
  sk_status st = SK_OK;
  {
    py::gil_scoped_release release;
    std::thread worker([&] {
      const sk_status s = fn();
      std::lock_guard<std::mutex> lock(mu);
      st = s;
      done = true;
      cv.notify_all();
    });
    bool interrupted = false;
    for (;;) {
      {
        std::unique_lock<std::mutex> lock(mu);
        if (cv.wait_for(lock, std::chrono::milliseconds(20), [&] { return done; })) break;
      }
      if (!interrupted) {
        py::gil_scoped_acquire acquire;
        if (PyErr_CheckSignals() != 0) {
          interrupted = true;
          sk_cancel(ctx);
        }
      }
    }
    worker.join();
    if (interrupted) {
      py::gil_scoped_acquire acquire;
      throw py::error_already_set();
    }
  }
  check(ctx, st);
}

struct DbHandle {
  sk_db *h = nullptr;
  DbHandle() = default;
  DbHandle(const DbHandle &) = delete;
  ~DbHandle() {
    if (h) sk_db_destroy(h);
  }
};

struct RandomHandle {
  sk_random *h = nullptr;
  RandomHandle() = default;
  RandomHandle(const RandomHandle &) = delete;
  ~RandomHandle() {
    if (h) sk_random_destroy(h);
  }
};

// Page-locked staging for the sketch words of queryDatabase, kept between
// calls and grown when a call needs more: the upload runs at the pinned copy
// rate, and no call pays first-touch page faults on a fresh buffer of the
// whole database.  Calls hold the lock while they use it.
struct PinnedStage {
  std::mutex mu;
  void *ptr = nullptr;
  size_t bytes = 0;
  uint64_t *words(size_t n_words) {
    const size_t need = n_words * sizeof(uint64_t);
    if (need > bytes) {
      if (ptr) sk_host_free(ptr);
      ptr = nullptr;
      bytes = 0;
      if (sk_host_alloc(static_cast<int64_t>(need), &ptr) != SK_OK)
        throw std::runtime_error("Unable to allocate page-locked host memory for the sketches");
      bytes = need;
    }
    return static_cast<uint64_t *>(ptr);
  }
};
PinnedStage g_stage;       // sketch words
PinnedStage g_out_stage;   // distances (their rows come back while later rows compute)

// Copies a call's sketch words into the page-locked stage on background
// threads while sk_query_db_ready runs, in blocks of kBlock samples and in
// the order the upload asks for them (all-vs-all from the last samples down;
// otherwise the queries, then the references from the first up); the call's
// ready callback waits for the blocks of the chunk it is about to copy.
class Prefetch {
 public:
  struct Side {
    const skhost::SketchReader *reader = nullptr;
    uint64_t *dst = nullptr;
    size_t n = 0;
  };

  Prefetch(Side ref, Side query, bool self, int threads) {
    sides_[0] = ref;
    sides_[1] = query;
    for (int s = 0; s < 2; ++s) {
      const size_t blocks = (sides_[s].n + kBlock - 1) / kBlock;
      done_[s].reset(new std::atomic<uint8_t>[blocks == 0 ? 1 : blocks]);
      for (size_t b = 0; b < blocks; ++b) done_[s][b] = 0;
    }
    const size_t rb = (ref.n + kBlock - 1) / kBlock, qb = (query.n + kBlock - 1) / kBlock;
    if (self) {
      for (size_t b = rb; b-- > 0;) order_.emplace_back(0, b);
    } else {
      for (size_t b = 0; b < qb; ++b) order_.emplace_back(1, b);
      for (size_t b = 0; b < rb; ++b) order_.emplace_back(0, b);
    }
    const int nt = std::max(1, std::min<int>(threads, static_cast<int>(order_.size())));
    for (int t = 0; t < nt; ++t) pool_.emplace_back([this] { work(); });
  }

  ~Prefetch() { join(); }

  // sk_words_ready_fn: 0 once samples [s0, s0 + n) of `side` are copied
  static int ready(void *user, int32_t side, int64_t s0, int64_t n) {
    Prefetch *p = static_cast<Prefetch *>(user);
    if (side < 0 || side > 1 || n <= 0) return 1;
    const size_t b0 = static_cast<size_t>(s0) / kBlock, b1 = static_cast<size_t>(s0 + n - 1) / kBlock;
    std::unique_lock<std::mutex> lock(p->mu_);
    const bool ok = p->cv_.wait_for(lock, std::chrono::seconds(300), [&] {
      if (p->failed_) return true;
      for (size_t b = b0; b <= b1; ++b)
        if (!p->done_[side][b]) return false;
      return true;
    });
    return ok && !p->failed_ ? 0 : 1;
  }

  // waits for the copies; rethrows the first error of a copy thread
  void finish() {
    join();
    if (err_) std::rethrow_exception(err_);
  }

 private:
  static constexpr size_t kBlock = 32;

  void work() {
    for (;;) {
      const size_t i = next_.fetch_add(1);
      if (i >= order_.size() || failed_) return;
      const int s = order_[i].first;
      const size_t b = order_[i].second;
      try {
        const size_t s0 = b * kBlock, s1 = std::min(sides_[s].n, s0 + kBlock);
        sides_[s].reader->copy(s0, s1, sides_[s].dst);
      } catch (...) {
        std::lock_guard<std::mutex> lock(mu_);
        if (!err_) err_ = std::current_exception();
        failed_ = true;
        cv_.notify_all();
        return;
      }
      std::lock_guard<std::mutex> lock(mu_);
      done_[s][b] = 1;
      cv_.notify_all();
    }
  }

  void join() {
    for (auto &t : pool_)
      if (t.joinable()) t.join();
  }

  Side sides_[2];
  std::vector<std::pair<int, size_t>> order_;
  std::unique_ptr<std::atomic<uint8_t>[]> done_[2];
  std::atomic<size_t> next_{0};
  std::atomic<bool> failed_{false};
  std::mutex mu_;
  std::condition_variable cv_;
  std::exception_ptr err_;
  std::vector<std::thread> pool_;
};

// Copies n floats on up to `threads` threads (the result rows from the
// page-locked stage into the numpy array, whose pages fault in on first touch).
void parallel_copy(float *dst, const float *src, size_t n, int threads) {
  if (n == 0) return;
  const size_t per = std::max<size_t>(1 << 20, (n + threads - 1) / threads);
  std::vector<std::thread> pool;
  for (size_t s0 = per; s0 < n; s0 += per)
    pool.emplace_back([=] { std::memcpy(dst + s0, src + s0, std::min(per, n - s0) * sizeof(float)); });
  std::memcpy(dst, src, std::min(per, n) * sizeof(float));
  for (auto &t : pool) t.join();
}

int loader_threads() {
  const unsigned hw = std::thread::hardware_concurrency();
  return static_cast<int>(std::min(16u, std::max(1u, hw)));
}

void upload(sk_ctx *ctx, const skhost::SketchSet &s, const std::vector<uint16_t> &clusters,
            DbHandle &db) {
  check(ctx, sk_db_create(ctx, s.words.data(), static_cast<int64_t>(s.size()), s.kmers.data(),
                          static_cast<int32_t>(s.kmers.size()), s.sketchsize64, s.bbits, &db.h));
  check(ctx, sk_db_set_sample_info(db.h, clusters.data(), s.seq_len.data()));
}

// The reference path a call reproduces: "cpu" (query_db + fit_slope, the
// default) or "gpu" (the reference GPU kernel, bit for bit).  An extra keyword
// beside the reference's own arguments; set on the shared context for the
// call only.
int parse_semantics(const std::string &s) {
  if (s == "cpu") return SK_SEMANTICS_REFERENCE_CPU;
  if (s == "gpu") return SK_SEMANTICS_REFERENCE_GPU;
  throw py::value_error("semantics must be 'cpu' or 'gpu'");
}

struct SemanticsScope {
  sk_ctx *ctx;
  SemanticsScope(sk_ctx *c, int sem) : ctx(c) { check(ctx, sk_ctx_set_semantics(ctx, sem)); }
  ~SemanticsScope() { sk_ctx_set_semantics(ctx, SK_SEMANTICS_REFERENCE_CPU); }
};

void make_random(sk_ctx *ctx, const skhost::RandomModel &r, const std::vector<int32_t> &kmers,
                 RandomHandle &out, bool gpu_rule) {
  int mode = SK_RANDOM_NONE;
  std::vector<float> table;
  if (r.mode == 1) mode = SK_RANDOM_EQUAL_BASE;
  if (r.mode == 2) {
    mode = SK_RANDOM_TABLE;
    table = r.flat_table(kmers, gpu_rule);
  }
  check(ctx, sk_random_create(ctx, mode, r.use_rc ? 1 : 0, kmers.data(),
                              static_cast<int32_t>(kmers.size()), r.n_clusters,
                              table.empty() ? nullptr : table.data(), &out.h));
}

skhost::RandomModel random_for(const std::string &db_name, bool random_correct) {
  if (!random_correct) {
    skhost::RandomModel none;
    none.mode = 0;
    return none;
  }
  // Reference::rc() is true for sketches loaded from a database
  return skhost::get_random(db_name, true);
}

std::vector<int32_t> to_kmers(const std::vector<size_t> &klist) {
  return std::vector<int32_t>(klist.begin(), klist.end());
}

void check_min_k(const skhost::RandomModel &r, const std::vector<int32_t> &kmers) {
  if (!kmers.empty() && static_cast<size_t>(kmers[0]) < r.min_supported_k())
    throw std::runtime_error(
        "Smallest k-mer has no signal above random chance; increase minimum k-mer length");
}

// ------------------------------------------------------------ entry points

py::array_t<float> queryDatabase(const std::string &ref_db_name, const std::string &query_db_name,
                                 const std::vector<std::string> &ref_names,
                                 const std::vector<std::string> &query_names,
                                 std::vector<size_t> kmer_lengths, const bool random_correct,
                                 const bool jaccard, const size_t num_threads, const bool use_gpu,
                                 const int device_id, const std::string &semantics) {
  (void)num_threads;
  (void)use_gpu;
  const int sem = parse_semantics(semantics);
  if (ref_names.empty() || query_names.empty())
    throw std::runtime_error("Query with empty ref or query list!");
  if (!jaccard && kmer_lengths.size() < 2)
    throw std::runtime_error("Core and accessory distances need at least two k-mer lengths");
  const std::vector<int32_t> kmers = to_kmers(kmer_lengths);
  const bool self = ref_db_name == query_db_name && ref_names == query_names;
  // the sketch words go straight from the mapped files into pinned staging
  std::lock_guard<std::mutex> stage_lock(g_stage.mu);
  std::lock_guard<std::mutex> out_lock(g_out_stage.mu);
  const size_t w_ref = static_cast<size_t>(skhost::sketch_words_per_k(ref_db_name, ref_names[0]));
  const size_t w_query =
      self ? 0 : static_cast<size_t>(skhost::sketch_words_per_k(query_db_name, query_names[0]));
  const size_t ref_words = ref_names.size() * kmers.size() * w_ref;
  const size_t query_words = self ? 0 : query_names.size() * kmers.size() * w_query;
  uint64_t *stage = g_stage.words(ref_words + query_words);
  // attributes and checks of every sample first; the words follow on
  // background threads while the upload runs (Prefetch below)
  skhost::SketchSet ref, query;
  const skhost::SketchReader ref_reader(ref_db_name, ref_names, kmers, ref, loader_threads());
  std::unique_ptr<skhost::SketchReader> query_reader;
  if (!self) {
    query_reader.reset(
        new skhost::SketchReader(query_db_name, query_names, kmers, query, loader_threads()));
    // checkSketchParamsMatch (src/gpu/gpu_api.cpp:170-185)
    if (query.bbits != ref.bbits) throw std::runtime_error("Mismatching bbits in sketches");
    if (query.sketchsize64 != ref.sketchsize64)
      throw std::runtime_error("Mismatching sketchsize64 in sketches");
  }
  skhost::RandomModel random = random_for(ref_db_name, random_correct);
  check_min_k(random, kmers);

  sk_ctx *ctx = context(device_id);
  SemanticsScope scope(ctx, sem);
  RandomHandle rnd;
  make_random(ctx, random, kmers, rnd, sem == SK_SEMANTICS_REFERENCE_GPU);
  // one sk_query_db call: the sketch upload overlaps the distance kernel
  const std::vector<uint16_t> ref_cl = random.lookup(ref, false);
  const std::vector<uint16_t> query_cl = self ? std::vector<uint16_t>() : random.lookup(query, true);
  const sk_host_sketches r{stage, static_cast<int64_t>(ref.size()), ref_cl.data(),
                           ref.seq_len.data()};
  const sk_host_sketches q{self ? nullptr : stage + ref_words,
                           self ? 0 : static_cast<int64_t>(query.size()),
                           self ? nullptr : query_cl.data(), self ? nullptr : query.seq_len.data()};
  const int64_t n_ref = static_cast<int64_t>(ref.size());
  const int64_t rows = self ? n_ref * (n_ref - 1) / 2 : static_cast<int64_t>(query.size()) * n_ref;
  const int64_t cols = jaccard ? static_cast<int64_t>(kmers.size()) : 2;
  py::array_t<float> out({rows, cols});
  const size_t n_out = static_cast<size_t>(rows) * static_cast<size_t>(cols);
  float *staged = reinterpret_cast<float *>(g_out_stage.words((n_out + 1) / 2));
  {
    Prefetch prefetch({&ref_reader, stage, ref.size()},
                      {query_reader.get(), stage + ref_words, self ? 0 : query.size()}, self,
                      loader_threads());
    try {
      run_gpu(ctx, [&] {
        return sk_query_db_ready(ctx, &r, self ? nullptr : &q, kmers.data(),
                                 static_cast<int32_t>(kmers.size()), ref.sketchsize64, ref.bbits,
                                 rnd.h, jaccard ? SK_OUT_JACCARD : SK_OUT_CORE_ACC, staged,
                                 &Prefetch::ready, &prefetch);
      });
    } catch (...) {
      prefetch.finish();   // a failed read explains a failed call best
      throw;
    }
    prefetch.finish();
  }
  parallel_copy(out.mutable_data(), staged, n_out, loader_threads());
  return out;
}

sparse_coo to_coo(const std::vector<int64_t> &i, const std::vector<int64_t> &j,
                  const std::vector<float> &d) {
  return sparse_coo(std::vector<long>(i.begin(), i.end()), std::vector<long>(j.begin(), j.end()), d);
}

sparse_coo querySelfSparse(const std::string &ref_db_name, const std::vector<std::string> &ref_names,
                           std::vector<size_t> kmer_lengths, const bool random_correct,
                           const bool jaccard, const unsigned long int kNN, const float dist_cutoff,
                           const size_t dist_col, const size_t num_threads, const bool use_gpu,
                           const int device_id, const std::string &semantics) {
  (void)num_threads;
  (void)use_gpu;
  const int sem = parse_semantics(semantics);
  if (ref_names.empty()) throw std::runtime_error("Query with empty ref or query list!");
  const std::vector<int32_t> kmers = to_kmers(kmer_lengths);
  skhost::SketchSet ref = skhost::load_sketches(ref_db_name, ref_names, kmers);
  skhost::RandomModel random = random_for(ref_db_name, random_correct);
  check_min_k(random, kmers);
  sk_ctx *ctx = context(device_id);
  SemanticsScope scope(ctx, sem);
  DbHandle db;
  upload(ctx, ref, random.lookup(ref, false), db);
  RandomHandle rnd;
  make_random(ctx, random, kmers, rnd, sem == SK_SEMANTICS_REFERENCE_GPU);

  std::vector<int64_t> i, j;
  std::vector<float> d;
  if (dist_cutoff > 0) {
    // dense core/accessory -> square -> threshold (sketchlib_bindings.cpp:159-169),
    // here without leaving the device
    if (dist_col > 1) throw std::runtime_error("dist_col out of range");
    if (kmers.size() < 2)
      throw std::runtime_error("Core and accessory distances need at least two k-mer lengths");
    sk_sparse *sp = nullptr;
    run_gpu(ctx, [&] {
      return sk_dists_threshold(ctx, db.h, rnd.h, static_cast<int32_t>(dist_col), dist_cutoff, &sp);
    });
    const int64_t m = sk_sparse_size(sp);
    i.resize(m);
    j.resize(m);
    d.resize(m);
    sk_sparse_copy(sp, i.data(), j.data(), d.data());
    sk_sparse_destroy(sp);
  } else {
    if (!jaccard && kmers.size() < 2)
      throw std::runtime_error("Core and accessory distances need at least two k-mer lengths");
    const int64_t n = static_cast<int64_t>(ref.size());
    const int64_t m = n * static_cast<int64_t>(kNN);
    i.resize(m);
    j.resize(m);
    d.resize(m);
    run_gpu(ctx, [&] {
      return sk_dists_knn(ctx, db.h, rnd.h, static_cast<int32_t>(kNN),
                          static_cast<int32_t>(dist_col), jaccard ? 1 : 0, i.data(), j.data(),
                          d.data());
    });
  }
  return to_coo(i, j, d);
}

double jaccardDist(const std::string &db_name, const std::string &sample1,
                   const std::string &sample2, const size_t kmer_size, bool random_correct) {
  const std::vector<int32_t> kmers{static_cast<int32_t>(kmer_size)};
  skhost::SketchSet s = skhost::load_sketches(db_name, {sample1, sample2}, kmers);
  skhost::RandomModel random = random_for(db_name, random_correct);
  sk_ctx *ctx = context(0);
  DbHandle db;
  upload(ctx, s, random.lookup(s, false), db);
  uint32_t count = 0;
  run_gpu(ctx, [&] { return sk_dists_dense(ctx, db.h, nullptr, nullptr, SK_OUT_COUNTS, &count, 0); });
  // Reference::jaccard_dist (src/reference.cpp:86-103) on the device's count
  double r = 0.0;
  if (random.mode == 1) {
    const double mc = std::ldexp(1.0, (static_cast<int>(kmer_size) - 1) * 2 + (random.use_rc ? 1 : 0));
    const double j1 = 1 - std::pow(1 - (double)1 / mc, (double)s.seq_len[0]);
    const double j2 = 1 - std::pow(1 - (double)1 / mc, (double)s.seq_len[1]);
    if (j1 > 0 && j2 > 0) r = (j1 * j2) / (j1 + j2 - j1 * j2);
  } else if (random.mode == 2) {
    const auto cl = random.lookup(s, false);
    const auto table = random.flat_table(kmers);
    r = table[static_cast<size_t>(cl[0]) * random.n_clusters + cl[1]];
  }
  const double obs = count / (double)(64 * static_cast<uint64_t>(s.sketchsize64));
  const double diff = obs > r ? obs - r : 0;
  return diff * 1 / (1 - r);
}

int64_t rows_to_samples(int64_t rows) {
  return static_cast<int64_t>(0.5 * (1 + std::sqrt(1 + 8 * static_cast<double>(rows))));
}

py::array_t<float> long_to_square_impl(const FloatArray &rr, const FloatArray *qr,
                                       const FloatArray *qq) {
  const int64_t n_rr = rows_to_samples(rr.size());
  int64_t n_qq = 0;
  if (qr && qr->size() > 0) {
    n_qq = rows_to_samples(qq ? qq->size() : 0);
    if (n_qq < 1) n_qq = 1;
    if (qr->size() != n_rr * n_qq)
      throw std::runtime_error("Shape of reference, query and ref vs query matrices mismatches");
  }
  const int64_t n = n_rr + n_qq;
  py::array_t<float> out({n, n});
  sk_ctx *ctx = context(0);
  const float *qr_p = (qr && qr->size() > 0) ? qr->data() : nullptr;
  const float *qq_p = (qq && qq->size() > 0) ? qq->data() : nullptr;
  float *dst = out.mutable_data();
  run_gpu(ctx, [&] { return sk_long_to_square(ctx, rr.data(), n_rr, qr_p, qq_p, n_qq, dst); });
  return out;
}

py::array_t<float> longToSquare(const FloatArray &distVec, const unsigned int num_threads) {
  (void)num_threads;
  return long_to_square_impl(distVec, nullptr, nullptr);
}

py::array_t<float> longToSquareMulti(const FloatArray &distVec, const FloatArray &qr,
                                     const FloatArray &qq, const unsigned int num_threads) {
  (void)num_threads;
  return long_to_square_impl(distVec, &qr, &qq);
}

py::array_t<float> squareToLong(const FloatArray &distMat, const unsigned int num_threads) {
  (void)num_threads;
  if (distMat.ndim() != 2 || distMat.shape(0) != distMat.shape(1))
    throw std::runtime_error("square_to_long input must be a square matrix");
  const int64_t n = distMat.shape(0);
  py::array_t<float> out(n * (n - 1) / 2);
  sk_ctx *ctx = context(0);
  float *dst = out.mutable_data();
  run_gpu(ctx, [&] { return sk_square_to_long(ctx, distMat.data(), n, dst); });
  return out;
}

sparse_coo sparsifyDistsByThreshold(const FloatArray &denseDists, const float distCutoff,
                                    const size_t num_threads) {
  (void)num_threads;
  if (distCutoff < 0) throw std::runtime_error("Distance threshold must be at least 0");
  if (denseDists.ndim() != 2 || denseDists.shape(0) != denseDists.shape(1))
    throw std::runtime_error("sparsifyDistsByThreshold needs a square distance matrix");
  const int64_t n = denseDists.shape(0);
  std::vector<float> lf(static_cast<size_t>(n * (n - 1) / 2));
  sk_ctx *ctx = context(0);
  run_gpu(ctx, [&] { return sk_square_to_long(ctx, denseDists.data(), n, lf.data()); });
  sk_sparse *sp = nullptr;
  run_gpu(ctx, [&] { return sk_sparse_threshold(ctx, lf.data(), n, 1, 0, distCutoff, &sp); });
  const int64_t m = sk_sparse_size(sp);
  std::vector<int64_t> i(m), j(m);
  std::vector<float> d(m);
  sk_sparse_copy(sp, i.data(), j.data(), d.data());
  sk_sparse_destroy(sp);
  return to_coo(i, j, d);
}

sparse_coo sparsifyDists(const FloatArray &, const float, const int, const size_t) {
  throw std::runtime_error(
      "pp_sketchlib.sparsifyDists was deprecated in v2.0.1\n"
      "Downgrade to v2.0.0, or update the calling package");
}

// What constructDatabase stores per sample besides the sketch words.
struct SampleInfo {
  std::string name;
  uint64_t length = 0, missing = 0;
  bool reads = false, densified = false;
  std::array<double, 4> bases{};
};

// Writes sketches [n][K][s64 * 14] in the reference's database layout
// (src/database/database.cpp:40-96, 235-258): /sketches with codon_phased and
// reverse_complement, one group per sample with its attributes and one
// uint64 dataset per k.  The sketch_version string is left out (the
// reference reads it only when present).
void save_sketch_db(const std::string &path, const std::vector<SampleInfo> &info,
                    const std::vector<uint64_t> &words, const std::vector<int32_t> &kmers, int s64,
                    bool use_rc, bool codon_phased) {
  const size_t K = kmers.size(), W = static_cast<size_t>(s64) * 14;
  h5w::Group root, sk;
  sk.name = "sketches";
  sk.attrs = {h5w::Attr::u8("codon_phased", codon_phased ? 1 : 0),
              h5w::Attr::u8("reverse_complement", use_rc ? 1 : 0)};
  for (size_t i = 0; i < info.size(); ++i) {
    h5w::Group g;
    g.name = info[i].name;
    g.attrs = {h5w::Attr::u64("sketchsize64", static_cast<uint64_t>(s64)),
               h5w::Attr::u64("bbits", 14),
               h5w::Attr::u64("length", info[i].length),
               h5w::Attr::u64("missing_bases", info[i].missing),
               h5w::Attr::u8("reads", info[i].reads ? 1 : 0),
               h5w::Attr::f64_vec("base_freq", std::vector<double>(info[i].bases.begin(), info[i].bases.end())),
               h5w::Attr::i32_vec("kmers", kmers)};
    for (size_t k = 0; k < K; ++k) {
      h5w::Dataset d;
      d.name = std::to_string(kmers[k]);
      d.data = words.data() + (i * K + k) * W;
      d.count = W;
      d.attrs = {h5w::Attr::i32("kmer-size", kmers[k])};
      g.datasets.push_back(std::move(d));
    }
    sk.groups.push_back(std::move(g));
  }
  root.groups.push_back(std::move(sk));
  h5w::write_file(path, root);
}

bool file_exists(const std::string &path) {
  struct stat st {};
  return stat(path.c_str(), &st) == 0;
}

// constructDatabase (src/sketchlib_bindings.cpp:47-87, src/api.cpp:39-135):
// reads each sample's files as the reference's SeqBuf does, sketches every
// sample on the GPU (sk_sketch) and writes the database.  An existing
// database that already holds every sample at these k-mer lengths is kept,
// as the reference keeps it.  Read sets (FASTQ input) with min_count > 0 are
// filtered by exact k-mer counts (the reference's `exact = true`).
void constructDatabase(const std::string &db_name, const std::vector<std::string> &names,
                       const std::vector<std::vector<std::string>> &files,
                       std::vector<size_t> kmer_lengths, const size_t sketch_size,
                       const bool codon_phased, const bool calc_random, const bool use_rc,
                       size_t min_count, const bool exact, const size_t num_threads,
                       const bool /*use_gpu*/, const int device_id) {
  if (names.size() != files.size()) throw std::runtime_error("Sample names and file lists differ in length");
  for (const std::string &nm : names)   // HDF5 link names: no path separator, not empty
    if (nm.empty() || nm.find('/') != std::string::npos || nm == "." || nm == "..")
      throw std::runtime_error("Sample name '" + nm + "' cannot name a database group");
  if (kmer_lengths.empty()) throw std::runtime_error("No k-mer lengths given");
  const std::string path = db_name + ".h5";
  std::vector<int32_t> kmers = to_kmers(kmer_lengths);
  std::sort(kmers.begin(), kmers.end());
  if (file_exists(path)) {
    try {
      skhost::load_sketches(db_name, names, kmers);
      return;   // every sample is already sketched
    } catch (const std::exception &) {
    }
  }
  const size_t min_len = kmer_lengths.back();   // SeqBuf(files, kmer_lengths.back())
  const size_t n = names.size();
  if (min_count > 0 && !exact)
    std::cerr << "NOTE: min_count uses exact k-mer counts on the GPU (the count-min "
                 "approximation of the CPU sketcher is not reproduced)" << std::endl;
  if (min_count > 255) min_count = 255;
  const int s64 = static_cast<int>(sketch_size);
  const size_t K = kmers.size(), W = static_cast<size_t>(s64) * 14;
  std::vector<uint64_t> words(n * K * W);
  std::vector<SampleInfo> info(n);
  sk_ctx *ctx = context(device_id);
  // samples are read (num_threads at a time) and sketched in chunks of about
  // kChunkBases bases, so only one chunk's sequences are held at once
  constexpr uint64_t kChunkBases = 2ULL << 30;
  size_t start = 0;
  while (start < n) {
    std::vector<skhost::SampleSeqs> seqs;
    size_t end = start;
    {
      py::gil_scoped_release release;
      std::mutex mu;
      size_t next = start;
      uint64_t held = 0;
      std::vector<std::pair<size_t, skhost::SampleSeqs>> done;
      std::vector<std::string> errors;
      auto work = [&] {
        for (;;) {
          size_t i;
          {
            std::lock_guard<std::mutex> g(mu);
            if (next >= n || (held >= kChunkBases && next > start)) return;
            i = next++;
          }
          skhost::SampleSeqs got;
          std::string err;
          try {
            got = skhost::read_sample(files[i], min_len);
            if (got.seqs.empty()) err = names[i] + " contains no sequence";
          } catch (const std::exception &e) {
            err = e.what();
          }
          std::lock_guard<std::mutex> g(mu);
          held += got.total;
          if (!err.empty()) errors.push_back(err);
          done.emplace_back(i, std::move(got));
        }
      };
      std::vector<std::thread> pool;
      for (size_t t = 1; t < std::max<size_t>(1, num_threads); ++t) pool.emplace_back(work);
      work();
      for (auto &t : pool) t.join();
      if (!errors.empty()) throw std::runtime_error(errors.front());
      end = next;
      seqs.resize(end - start);
      for (auto &d : done) seqs[d.first - start] = std::move(d.second);
    }
    for (int pass = 0; pass < 2; ++pass) {   // assemblies, then read sets
      std::vector<size_t> idx;
      for (size_t i = start; i < end; ++i)
        if (seqs[i - start].reads == (pass == 1)) idx.push_back(i);
      if (idx.empty()) continue;
      std::string bases;
      std::vector<int64_t> off{0}, first{0};
      for (size_t i : idx) {
        for (const std::string &q : seqs[i - start].seqs) {
          bases += q;
          off.push_back(static_cast<int64_t>(bases.size()));
        }
        first.push_back(static_cast<int64_t>(off.size() - 1));
      }
      std::vector<uint64_t> w(idx.size() * K * W);
      std::vector<double> inv(idx.size() * K);
      std::vector<uint8_t> dens(idx.size());
      const int32_t mc = pass == 1 ? static_cast<int32_t>(min_count) : 0;
      run_gpu(ctx, [&] {
        return sk_sketch(ctx, bases.data(), off.data(), first.data(), static_cast<int64_t>(idx.size()),
                         kmers.data(), static_cast<int32_t>(K), s64, use_rc ? 1 : 0,
                         codon_phased ? 1 : 0, mc, w.data(), inv.data(), dens.data());
      });
      for (size_t j = 0; j < idx.size(); ++j) {
        const size_t i = idx[j];
        const skhost::SampleSeqs &sq = seqs[i - start];
        std::copy(w.begin() + j * K * W, w.begin() + (j + 1) * K * W, words.begin() + i * K * W);
        SampleInfo &si = info[i];
        si.name = names[i];
        si.reads = sq.reads;
        si.missing = sq.missing_bases;
        si.densified = dens[j] != 0;
        std::copy(sq.base_freq, sq.base_freq + 4, si.bases.begin());
        if (si.reads) {   // 1/N ~ E(minhash) over the k-mer lengths (src/reference.cpp:47-54)
          double sum = 0;
          for (size_t k = 0; k < K; ++k) sum += inv[j * K + k];
          si.length = static_cast<uint64_t>(static_cast<double>(K) / sum);
        } else {
          si.length = sq.total;
        }
      }
    }
    start = end;
  }
  std::cerr << "Writing sketches to file" << std::endl;
  save_sketch_db(path, info, words, kmers, s64, use_rc, codon_phased);
  for (const SampleInfo &si : info)
    if (si.densified) std::cerr << "NOTE: " << si.name << " required densification" << std::endl;
  if (calc_random) {
    if (n >= 3)   // default_n_clusters (src/random/random_match.hpp)
      std::cerr << "NOTE: random match chances were not calculated (the Monte Carlo random "
                   "genomes are not part of this library); queries use the equal-base "
                   "random-match formula" << std::endl;
    else
      std::cerr << "Too few input genomes to calculate random match chances" << std::endl;
  }
}

// Test hook: the SeqBuf view of one sample's files.
py::dict read_sequences(const std::vector<std::string> &files, size_t min_len) {
  skhost::SampleSeqs s = skhost::read_sample(files, min_len);
  py::dict d;
  d["seqs"] = s.seqs;
  d["reads"] = s.reads;
  d["missing_bases"] = s.missing_bases;
  d["total"] = s.total;
  d["base_freq"] = std::vector<double>(s.base_freq, s.base_freq + 4);
  d["max_length"] = s.max_length;
  return d;
}

// Test hook: writes a database from sketch words (save_sketch_db).
void save_sketch_db_py(const std::string &db_name, const std::vector<std::string> &names,
                       py::array_t<uint64_t, py::array::c_style | py::array::forcecast> words,
                       std::vector<size_t> kmer_lengths, int sketchsize64,
                       std::vector<uint64_t> lengths, bool use_rc) {
  const std::vector<int32_t> kmers = to_kmers(kmer_lengths);
  const size_t need = names.size() * kmers.size() * static_cast<size_t>(sketchsize64) * 14;
  if (static_cast<size_t>(words.size()) != need) throw std::runtime_error("words have the wrong size");
  std::vector<SampleInfo> info(names.size());
  for (size_t i = 0; i < names.size(); ++i) {
    info[i].name = names[i];
    info[i].length = i < lengths.size() ? lengths[i] : 0;
    info[i].bases = {0.25, 0.25, 0.25, 0.25};
  }
  std::vector<uint64_t> w(words.data(), words.data() + need);
  save_sketch_db(db_name + ".h5", info, w, kmers, sketchsize64, use_rc, false);
}

void not_in_path(const char *what) {
  const std::string msg = std::string(what) +
                          " computes random-match chances from Monte Carlo random genomes, "
                          "which this library does not build (use the reference pp-sketchlib)";
  PyErr_SetString(PyExc_NotImplementedError, msg.c_str());
  throw py::error_already_set();
}

py::dict load_sketch_db(const std::string &db_name, std::vector<std::string> names,
                        std::vector<size_t> kmer_lengths, int threads) {
  if (names.empty()) names = skhost::list_samples(db_name);
  if (names.empty()) throw std::runtime_error("Database " + db_name + " holds no sketches");
  const std::vector<int32_t> kmers = to_kmers(kmer_lengths);
  skhost::SketchSet s;
  const py::ssize_t W = static_cast<py::ssize_t>(skhost::sketch_words_per_k(db_name, names[0]));
  py::array_t<uint64_t> words({static_cast<py::ssize_t>(names.size()),
                               static_cast<py::ssize_t>(kmers.size()), W});
  // the same multi-threaded read queryDatabase uses, into the numpy array
  skhost::load_sketches_into(db_name, names, kmers, s, words.mutable_data(), threads);
  py::dict d;
  d["names"] = s.names;
  d["kmers"] = s.kmers;
  d["sketchsize64"] = s.sketchsize64;
  d["bbits"] = s.bbits;
  d["words"] = words;
  d["length"] = s.seq_len;
  d["base_freq"] = s.bases;
  return d;
}

py::dict load_random_model(const std::string &db_name) {
  skhost::RandomModel r = skhost::get_random(db_name, true);
  py::dict d;
  d["mode"] = r.mode;
  d["use_rc"] = r.use_rc;
  d["k_min"] = r.min_k;
  d["k_max"] = r.max_k;
  d["n_clusters"] = r.n_clusters;
  d["cluster_table"] = r.cluster_table;
  d["matches"] = r.matches;
  d["centroids"] = r.centroids;
  d["min_supported_k"] = r.min_supported_k();
  return d;
}

}  // namespace

PYBIND11_MODULE(_pp_sketchlib, m) {
  m.doc() = "B200 core/accessory distances, drop-in for pp_sketchlib's distance functions";

  m.def("queryDatabase", &queryDatabase, "Find distances between sketches; return all distances",
        py::arg("ref_db_name"), py::arg("query_db_name"), py::arg("rList"), py::arg("qList"),
        py::arg("klist"), py::arg("random_correct") = true, py::arg("jaccard") = false,
        py::arg("num_threads") = 1, py::arg("use_gpu") = false, py::arg("device_id") = 0,
        py::arg("semantics") = "cpu");

  m.def("querySelfSparse", &querySelfSparse,
        "Find self-self distances between sketches; return a sparse matrix",
        py::arg("ref_db_name"), py::arg("rList"), py::arg("klist"),
        py::arg("random_correct") = true, py::arg("jaccard") = false, py::arg("kNN") = 0,
        py::arg("dist_cutoff") = 0.0f, py::arg("dist_col") = 0, py::arg("num_threads") = 1,
        py::arg("use_gpu") = false, py::arg("device_id") = 0, py::arg("semantics") = "cpu");

  m.def("jaccardDist", &jaccardDist, "Calculate a raw Jaccard distance", py::arg("db_name"),
        py::arg("ref_name"), py::arg("query_name"), py::arg("kmer_length"),
        py::arg("random_correct") = false);

  m.def("squareToLong", &squareToLong, "Convert dense square matrices to long form",
        py::arg("distMat"), py::arg("num_threads") = 1);
  m.def("longToSquare", &longToSquare, "Convert dense long form distance matrices to square form",
        py::arg("distVec"), py::arg("num_threads") = 1);
  m.def("longToSquareMulti", &longToSquareMulti,
        "Convert dense long form distance matrices to square form (in three blocks)",
        py::arg("distVec"), py::arg("query_ref_distVec"), py::arg("query_query_distVec"),
        py::arg("num_threads") = 1);
  m.def("sparsifyDistsByThreshold", &sparsifyDistsByThreshold,
        "Transform all distances into a sparse matrix", py::arg("distMat"),
        py::arg("distCutoff") = 0, py::arg("num_threads") = 1);
  m.def("sparsifyDists", &sparsifyDists, "Transform all distances into a sparse matrix",
        py::arg("distMat"), py::arg("distCutoff") = 0, py::arg("kNN") = 0,
        py::arg("num_threads") = 1);

  m.def("constructDatabase", &constructDatabase, "Create and save sketches", py::arg("db_name"),
        py::arg("samples"), py::arg("files"), py::arg("klist"), py::arg("sketch_size"),
        py::arg("codon_phased") = false, py::arg("calc_random") = true, py::arg("use_rc") = true,
        py::arg("min_count") = 0, py::arg("exact") = false, py::arg("num_threads") = 1,
        py::arg("use_gpu") = false, py::arg("device_id") = 0);
  m.def("addRandom", [](py::args, py::kwargs) { not_in_path("addRandom"); });

  // not in the reference module: the sequence reader and database writer
  // behind constructDatabase (tests)
  m.def("_read_sequences", &read_sequences, py::arg("files"), py::arg("min_len"));
  m.def("_save_sketch_db", &save_sketch_db_py, py::arg("db_name"), py::arg("names"),
        py::arg("words"), py::arg("klist"), py::arg("sketchsize64"),
        py::arg("lengths") = std::vector<uint64_t>{}, py::arg("use_rc") = true);

  // not in the reference module: reads a database's sketches (tests, tools)
  m.def("_load_sketch_db", &load_sketch_db, py::arg("db_name"),
        py::arg("names") = std::vector<std::string>{}, py::arg("klist"), py::arg("threads") = 1);

  m.def("_load_random", &load_random_model, py::arg("db_name"));

  m.attr("version") = "2.1.5+b200";
  m.attr("sketchVersion") = "b200";

  py::register_exception<h5::Error>(m, "HDF5Exception", PyExc_RuntimeError);
}
