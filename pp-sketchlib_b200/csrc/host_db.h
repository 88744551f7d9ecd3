// host_db.h -- reads pp-sketchlib sketch databases (<name>.h5) into the flat
// word layout of the C ABI, plus the random-match model stored beside them.
//
// Database layout (src/database/database.cpp:48-112, 195-227):
//   /sketches                      attrs sketch_version, codon_phased, reverse_complement
//   /sketches/<sample>             attrs kmers (int[]), sketchsize64, bbits, length,
//                                  missing_bases, reads, base_freq (double[4])
//   /sketches/<sample>/<k>         uint64[sketchsize64 * bbits]
//   /random                        attrs k_min, k_max, use_rc
//   /random/table_keys|_values     sample name -> cluster id (uint16)
//   /random/matches_keys|_values   k -> C x C float matrix (attr dims = [C, C, n_k])
//   /random/centroids              C x 4 float (attr dims), base composition centroids
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace skhost {

struct SketchSet {
  std::vector<std::string> names;
  std::vector<int32_t> kmers;           // in the order requested
  int32_t sketchsize64 = 0, bbits = 0;
  std::vector<uint64_t> words;          // [n][K][sketchsize64 * bbits]
  std::vector<uint64_t> seq_len;        // Reference::seq_length
  std::vector<std::vector<double>> bases;  // A, C, G, T frequencies
  bool reads = false;
  size_t size() const { return names.size(); }
};

// load_sketches (src/api.cpp:436-516): the named samples' sketches at the
// requested k-mer lengths.  Throws std::runtime_error with the reference's
// messages when a sample or k-mer length is missing.
// The same into a caller's buffer of names.size() * kmers.size() * W words
// (W = sketchsize64 * bbits, found in the file: `words_per_sample_k` gives it
// before the buffer is sized): out.words stays empty.  Samples are read on up
// to `threads` threads straight from the mapped file.
int64_t sketch_words_per_k(const std::string &db_name, const std::string &first_name);

// The same read in two passes.  The constructor reads every sample's
// attributes and finds its datasets (all of the checks above, on up to
// `threads` threads) and fills everything of `out` but the words; copy()
// then moves the words of samples [s0, s1) into dst ([n][K][W], the layout
// of load_sketches_into), straight from the mapped file, from any thread and
// in any order -- so a caller can hand the words to the device while later
// samples are still being read.
class SketchReader {
 public:
  SketchReader(const std::string &db_name, const std::vector<std::string> &names,
               const std::vector<int32_t> &kmers, SketchSet &out, int threads);
  ~SketchReader();
  SketchReader(const SketchReader &) = delete;
  SketchReader &operator=(const SketchReader &) = delete;
  void copy(size_t s0, size_t s1, uint64_t *dst) const;
  size_t words_per_sample() const;   // K * W

 private:
  struct Impl;
  std::unique_ptr<Impl> impl_;
};
void load_sketches_into(const std::string &db_name, const std::vector<std::string> &names,
                        const std::vector<int32_t> &kmers, SketchSet &out, uint64_t *dst,
                        int threads);
SketchSet load_sketches(const std::string &db_name, const std::vector<std::string> &names,
                        const std::vector<int32_t> &kmers);

// All sample names in a database, in the file's (sorted) order.
std::vector<std::string> list_samples(const std::string &db_name);

// RandomMC as loaded by Database::load_random (database.cpp:195-227).
struct RandomModel {
  int mode = 0;                 // 0 NoAdjust, 1 EqualBase, 2 MonteCarlo
  bool use_rc = true;
  unsigned min_k = 0, max_k = 101;
  std::map<std::string, uint16_t> cluster_table;
  std::map<int64_t, std::vector<float>> matches;   // k -> C*C row-major
  int n_clusters = 0;
  std::vector<float> centroids;                   // C x 4 row-major

  // closest_cluster (random_match.cpp:222-229, nearest_neighbour :339-348)
  uint16_t closest_cluster(const std::vector<double> &bases, bool rc) const;
  // cluster ids for samples: table entry, else nearest centroid
  std::vector<uint16_t> lookup(const SketchSet &s, bool queries_by_centroid) const;
  // [K][C][C] table with zeros for k >= max_k (random_match.cpp:191)
  // [K][C][C] table for the given k-mer lengths; k at or beyond max_k gives 0
  // (CPU path, strict <) or copies the table up to max_k inclusive (GPU path,
  // flattened_random's <=).
  std::vector<float> flat_table(const std::vector<int32_t> &kmers, bool gpu_rule = false) const;
  // min_supported_k (random_match.cpp:165-182)
  size_t min_supported_k() const;
};

// get_random (src/api.cpp:531-535): MonteCarlo when the database holds
// /random, else EqualBase (use_rc_default); random_correct = false gives NoAdjust.
RandomModel get_random(const std::string &db_name, bool use_rc_default);

}  // namespace skhost
