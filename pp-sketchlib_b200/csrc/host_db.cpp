// host_db.cpp -- see host_db.h.
#include "host_db.h"
#include "sketchlib_b200.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <thread>

#include "host_h5.h"

namespace skhost {
namespace {

constexpr uint64_t kDefaultLength = 3000000;  // DEFAULT_LENGTH, database.hpp:22

std::string h5_path(const std::string &db_name) {
  // the reference appends ".h5" to the database prefix (api.cpp:458)
  return db_name + ".h5";
}

std::string join(const std::vector<int32_t> &v) {
  std::ostringstream o;
  for (int32_t x : v) o << x << ",";
  return o.str();
}

}  // namespace

std::vector<std::string> list_samples(const std::string &db_name) {
  h5::File f(h5_path(db_name));
  return f.list(f.open("/sketches"));
}

int64_t sketch_words_per_k(const std::string &db_name, const std::string &first_name) {
  h5::File f(h5_path(db_name));
  const h5::Object sketches = f.open("/sketches");
  const auto samples = f.members(sketches);
  const auto it = samples.find(first_name);
  if (it == samples.end())
    throw h5::Error("Missing sketch: Object /sketches/" + first_name + " does not exist in " +
                    f.path());
  const h5::Object g = f.object_at(it->second);
  return f.attr_ints(g, "sketchsize64").at(0) * f.attr_ints(g, "bbits").at(0);
}

struct SketchReader::Impl {
  h5::File f;
  std::vector<h5::Object> ds;   // [n][K] the samples' datasets
  size_t K = 0, W = 0;
  explicit Impl(const std::string &path) : f(path) {}
};

SketchReader::SketchReader(const std::string &db_name, const std::vector<std::string> &names,
                           const std::vector<int32_t> &kmers, SketchSet &out, int threads)
    : impl_(new Impl(h5_path(db_name))) {
  h5::File &f = impl_->f;
  out.names = names;
  out.kmers = kmers;
  out.words.clear();
  const size_t n = names.size();
  const size_t K = kmers.size();
  impl_->K = K;
  impl_->ds.resize(n * K);
  out.seq_len.assign(n, 0);
  out.bases.assign(n, {});
  std::vector<uint8_t> reads(n, 0);
  // one walk of /sketches for every sample, one of each sample's group for its k
  const h5::Object sketches = f.open("/sketches");
  const auto samples = f.members(sketches);
  std::vector<int32_t> req(kmers);
  std::sort(req.begin(), req.end());
  int32_t s64_0 = 0, bbits_0 = 0;
  size_t W = 0;
  // the first sample fixes sketchsize64 and bbits (every other must match)
  auto sample = [&](size_t i) {
    const auto it = samples.find(names[i]);
    if (it == samples.end())
      throw h5::Error("Missing sketch: Object /sketches/" + names[i] + " does not exist in " +
                      f.path());
    const h5::Object g = f.object_at(it->second);
    std::vector<int64_t> have = f.attr_ints(g, "kmers");
    const int32_t s64 = static_cast<int32_t>(f.attr_ints(g, "sketchsize64").at(0));
    const int32_t bbits = static_cast<int32_t>(f.attr_ints(g, "bbits").at(0));
    if (i == 0) {
      s64_0 = s64;
      bbits_0 = bbits;
      W = static_cast<size_t>(s64) * bbits;
    } else if (s64 != s64_0) {
      throw std::runtime_error("Mismatching sketchsize64 in sketches");
    } else if (bbits != bbits_0) {
      throw std::runtime_error("Mismatching bbits in sketches");
    }
    // every requested k must be present (api.cpp:464-489)
    std::vector<int32_t> have32(have.begin(), have.end());
    std::sort(have32.begin(), have32.end());
    for (int32_t k : kmers) {
      if (!std::binary_search(have32.begin(), have32.end(), k))
        throw std::runtime_error("Mismatched data: k-mer lengths in old database (" + join(have32) +
                                 ") do not match those requested (" + join(req) + ")");
    }
    out.seq_len[i] = h5::File::has_attr(g, "length")
                         ? static_cast<uint64_t>(f.attr_ints(g, "length").at(0))
                         : kDefaultLength;
    out.bases[i] = h5::File::has_attr(g, "base_freq") ? f.attr_doubles(g, "base_freq")
                                                      : std::vector<double>{0.25, 0.25, 0.25, 0.25};
    if (h5::File::has_attr(g, "reads")) reads[i] = f.attr_ints(g, "reads").at(0) != 0;
    const auto ks = f.members(g);
    for (size_t ki = 0; ki < K; ++ki) {
      const auto kt = ks.find(std::to_string(kmers[ki]));
      if (kt == ks.end())
        throw h5::Error("Object /sketches/" + names[i] + "/" + std::to_string(kmers[ki]) +
                        " does not exist in " + f.path());
      h5::Object ds = f.object_at(kt->second);
      if (ds.space.count() != W)
        throw std::runtime_error("Sketch " + names[i] + " at k = " + std::to_string(kmers[ki]) +
                                 " has the wrong number of words");
      impl_->ds[i * K + ki] = std::move(ds);
    }
  };
  if (n == 0) return;
  sample(0);
  const int nt = std::max(1, std::min<int>(threads, static_cast<int>(n)));
  std::vector<std::exception_ptr> errs(nt);
  auto work = [&](int t) {
    try {
      for (size_t i = 1 + t; i < n; i += nt) sample(i);
    } catch (...) {
      errs[t] = std::current_exception();
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto &th : pool) th.join();
  for (auto &e : errs)
    if (e) std::rethrow_exception(e);
  impl_->W = W;
  out.sketchsize64 = s64_0;
  out.bbits = bbits_0;
  out.reads = std::any_of(reads.begin(), reads.end(), [](uint8_t r) { return r != 0; });
}

SketchReader::~SketchReader() = default;

size_t SketchReader::words_per_sample() const { return impl_->K * impl_->W; }

void SketchReader::copy(size_t s0, size_t s1, uint64_t *dst) const {
  const size_t K = impl_->K, W = impl_->W;
  for (size_t i = s0; i < s1; ++i)
    for (size_t ki = 0; ki < K; ++ki)
      impl_->f.read_u64(impl_->ds[i * K + ki], dst + (i * K + ki) * W);
}

void load_sketches_into(const std::string &db_name, const std::vector<std::string> &names,
                        const std::vector<int32_t> &kmers, SketchSet &out, uint64_t *dst,
                        int threads) {
  const SketchReader reader(db_name, names, kmers, out, threads);
  const size_t n = names.size();
  if (n == 0) return;
  const int nt = std::max(1, std::min<int>(threads, static_cast<int>(n)));
  std::vector<std::exception_ptr> errs(nt);
  auto work = [&](int t) {
    try {
      for (size_t i = t; i < n; i += nt) reader.copy(i, i + 1, dst);
    } catch (...) {
      errs[t] = std::current_exception();
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto &th : pool) th.join();
  for (auto &e : errs)
    if (e) std::rethrow_exception(e);
}

SketchSet load_sketches(const std::string &db_name, const std::vector<std::string> &names,
                        const std::vector<int32_t> &kmers) {
  SketchSet out;
  if (names.empty()) {
    out.kmers = kmers;
    return out;
  }
  const int64_t W = sketch_words_per_k(db_name, names[0]);
  std::vector<uint64_t> words(names.size() * kmers.size() * static_cast<size_t>(W));
  load_sketches_into(db_name, names, kmers, out, words.data(), 1);
  out.words = std::move(words);
  return out;
}

uint16_t RandomModel::closest_cluster(const std::vector<double> &bases_in, bool rc) const {
  if (mode != 2 || n_clusters == 0) return 0;
  uint16_t id = 0;
  sk_closest_cluster(centroids.data(), n_clusters, rc ? 1 : 0, bases_in.data(), 1, &id);
  return id;
}

std::vector<uint16_t> RandomModel::lookup(const SketchSet &s, bool queries_by_centroid) const {
  std::vector<uint16_t> ids(s.size(), 0);
  if (mode != 2) return ids;
  for (size_t i = 0; i < s.size(); ++i) {
    auto it = cluster_table.find(s.names[i]);
    if (!queries_by_centroid && it != cluster_table.end()) {
      ids[i] = it->second;
    } else {
      ids[i] = closest_cluster(s.bases[i], true);  // loaded references have rc() == true
    }
  }
  return ids;
}

std::vector<float> RandomModel::flat_table(const std::vector<int32_t> &kmers, bool gpu_rule) const {
  const size_t C = static_cast<size_t>(std::max(1, n_clusters));
  std::vector<float> t(kmers.size() * C * C, 0.0f);
  if (mode != 2) return t;
  for (size_t ki = 0; ki < kmers.size(); ++ki) {
    const int64_t k = kmers[ki];
    // CPU path: strict < (random_match.cpp:191); GPU path: <= (random_match.cpp:300)
    if (gpu_rule ? k > static_cast<int64_t>(max_k) : k >= static_cast<int64_t>(max_k)) continue;
    auto it = matches.find(k);
    if (it == matches.end())
      throw std::runtime_error("Trying to choose a k-mer length below the minimum allowed\n");
    std::copy(it->second.begin(), it->second.end(), t.begin() + ki * C * C);
  }
  return t;
}

size_t RandomModel::min_supported_k() const {
  size_t min_k_signal = min_k;
  if (mode == 2) {
    for (size_t k = min_k; k < max_k; ++k) {
      auto it = matches.find(static_cast<int64_t>(k));
      if (it == matches.end()) continue;
      const double mean =
          std::accumulate(it->second.begin(), it->second.end(), 0.0) / it->second.size();
      if (mean < 1) {
        min_k_signal = k;
        break;
      }
    }
  }
  return min_k_signal;
}

RandomModel get_random(const std::string &db_name, bool use_rc_default) {
  RandomModel r;
  r.mode = 1;
  r.use_rc = use_rc_default;
  r.min_k = 0;
  r.max_k = 101;
  h5::File f(h5_path(db_name));
  if (!f.exists("/random")) return r;
  h5::Object g = f.open("/random");
  r.mode = 2;
  r.min_k = static_cast<unsigned>(f.attr_ints(g, "k_min").at(0));
  r.max_k = static_cast<unsigned>(f.attr_ints(g, "k_max").at(0));
  r.use_rc = f.attr_ints(g, "use_rc").at(0) != 0;
  const auto names = f.read_strings(f.open("/random/table_keys"));
  const auto ids = f.read_ints(f.open("/random/table_values"));
  for (size_t i = 0; i < names.size() && i < ids.size(); ++i)
    r.cluster_table[names[i]] = static_cast<uint16_t>(ids[i]);
  const auto keys = f.read_ints(f.open("/random/matches_keys"));
  h5::Object mv = f.open("/random/matches_values");
  const auto values = f.read_doubles(mv);
  const auto dims = f.attr_ints(mv, "dims");
  const size_t C = static_cast<size_t>(dims.at(0));
  if (dims.at(1) != dims.at(0)) throw std::runtime_error("random match matrices are not square");
  r.n_clusters = static_cast<int>(C);
  for (size_t i = 0; i < keys.size(); ++i) {
    if ((i + 1) * C * C > values.size()) throw std::runtime_error("truncated random match table");
    r.matches[keys[i]] = std::vector<float>(values.begin() + i * C * C, values.begin() + (i + 1) * C * C);
  }
  h5::Object cen = f.open("/random/centroids");
  const auto cvals = f.read_doubles(cen);
  r.centroids.assign(cvals.begin(), cvals.end());
  return r;
}

}  // namespace skhost
