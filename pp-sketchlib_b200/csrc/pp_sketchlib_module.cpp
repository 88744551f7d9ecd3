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
//   * sketch creation (constructDatabase, addRandom) is outside this path and
//     raises NotImplementedError.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <atomic>
#include <chrono>
#include <cmath>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "host_db.h"
#include "host_h5.h"
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
template <class F>
void run_gpu(sk_ctx *ctx, F &&fn) {
  std::atomic<bool> done{false};
  sk_status st = SK_OK;
  {
    py::gil_scoped_release release;
    std::thread worker([&] {
      st = fn();
      done = true;
    });
    bool interrupted = false;
    while (!done) {
      std::this_thread::sleep_for(std::chrono::milliseconds(20));
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
  skhost::SketchSet ref = skhost::load_sketches(ref_db_name, ref_names, kmers);
  const bool self = ref_db_name == query_db_name && ref_names == query_names;
  skhost::SketchSet query;
  if (!self) {
    query = skhost::load_sketches(query_db_name, query_names, kmers);
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
  const sk_host_sketches r{ref.words.data(), static_cast<int64_t>(ref.size()), ref_cl.data(),
                           ref.seq_len.data()};
  const sk_host_sketches q{self ? nullptr : query.words.data(),
                           self ? 0 : static_cast<int64_t>(query.size()),
                           self ? nullptr : query_cl.data(), self ? nullptr : query.seq_len.data()};
  const int64_t n_ref = static_cast<int64_t>(ref.size());
  const int64_t rows = self ? n_ref * (n_ref - 1) / 2 : static_cast<int64_t>(query.size()) * n_ref;
  const int64_t cols = jaccard ? static_cast<int64_t>(kmers.size()) : 2;
  py::array_t<float> out({rows, cols});
  float *dst = out.mutable_data();
  run_gpu(ctx, [&] {
    return sk_query_db(ctx, &r, self ? nullptr : &q, kmers.data(),
                       static_cast<int32_t>(kmers.size()), ref.sketchsize64, ref.bbits, rnd.h,
                       jaccard ? SK_OUT_JACCARD : SK_OUT_CORE_ACC, dst);
  });
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

void not_in_path(const char *what) {
  const std::string msg = std::string(what) +
                          " creates sketches; sketching is not part of this library's GPU "
                          "distance path (use the reference pp-sketchlib to build databases)";
  PyErr_SetString(PyExc_NotImplementedError, msg.c_str());
  throw py::error_already_set();
}

py::dict load_sketch_db(const std::string &db_name, std::vector<std::string> names,
                        std::vector<size_t> kmer_lengths) {
  if (names.empty()) names = skhost::list_samples(db_name);
  skhost::SketchSet s = skhost::load_sketches(db_name, names, to_kmers(kmer_lengths));
  py::dict d;
  const py::ssize_t W = static_cast<py::ssize_t>(s.sketchsize64) * s.bbits;
  py::array_t<uint64_t> words({static_cast<py::ssize_t>(s.size()),
                               static_cast<py::ssize_t>(s.kmers.size()), W});
  std::copy(s.words.begin(), s.words.end(), words.mutable_data());
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

  m.def("constructDatabase", [](py::args, py::kwargs) { not_in_path("constructDatabase"); });
  m.def("addRandom", [](py::args, py::kwargs) { not_in_path("addRandom"); });

  // not in the reference module: reads a database's sketches (tests, tools)
  m.def("_load_sketch_db", &load_sketch_db, py::arg("db_name"),
        py::arg("names") = std::vector<std::string>{}, py::arg("klist"));

  m.def("_load_random", &load_random_model, py::arg("db_name"));

  m.attr("version") = "2.1.5+b200";
  m.attr("sketchVersion") = "b200";

  py::register_exception<h5::Error>(m, "HDF5Exception", PyExc_RuntimeError);
}
