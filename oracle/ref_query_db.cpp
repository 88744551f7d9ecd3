// ref_query_db.cpp -- the reference's CPU distance loop around the
// reference's own compiled calc_intersize.
//
// TEST INFRASTRUCTURE ONLY: the timed CPU baseline of bench.py and a second
// checker for the oracle.  Built by oracle/Makefile together with
// src/dist/dist.cpp compiled from the reference sources (the function where
// the reference CPU path spends its time); the surrounding Reference::jaccard_dist,
// observed_excess and float fit_slope arithmetic are the restatements of
// sk_oracle.c, so this library needs neither Eigen nor HDF5.
//
// The loop is query_db's all-vs-all branch (src/api.cpp:195-221): OpenMP
// `schedule(dynamic, 5)` over rows i, columns j > i, core/accessory per pair.
// Sketches are held per sample and k-mer length as std::vector<uint64_t>, the
// container Reference::get_sketch hands to calc_intersize.
#include <cstdint>
#include <vector>

#include "dist/dist.hpp"  // calc_intersize, from the reference sources

extern "C" {
void sko_fit_slope_f32(const float *J, const int *kmers, int K, int s64, float *core, float *acc);
double sko_jaccard(uint32_t intersize, int s64, double random_jaccard);
}

namespace {
int64_t condensed(int64_t i, int64_t j, int64_t n) { return n * i - ((i * (i + 1)) >> 1) + j - 1 - i; }
}  // namespace

extern "C" {

// Number of words of one (sample, k) sketch.
void *ref_sketches_create(const uint64_t *words, int64_t n, int K, int s64, int bbits) {
  auto *sk = new std::vector<std::vector<std::vector<uint64_t>>>(n);
  const int64_t W = static_cast<int64_t>(s64) * bbits;
  for (int64_t s = 0; s < n; ++s) {
    (*sk)[s].resize(K);
    for (int k = 0; k < K; ++k)
      (*sk)[s][k].assign(words + (s * K + k) * W, words + (s * K + k + 1) * W);
  }
  return sk;
}

void ref_sketches_destroy(void *h) { delete static_cast<std::vector<std::vector<std::vector<uint64_t>>> *>(h); }

// All-vs-all core/accessory for rows [row_begin, row_end) of n samples, no
// random-match correction (random_correct = False).  out: float (pairs, 2) in
// long-form order over the full matrix; only the rows asked for are written.
// Returns the number of pairs computed.
int64_t ref_query_db_self(void *h, int64_t n, int K, const int *kmers, int s64, int bbits,
                          int64_t row_begin, int64_t row_end, float *out, int threads) {
  const auto &sk = *static_cast<std::vector<std::vector<std::vector<uint64_t>>> *>(h);
  int64_t done = 0;
#pragma omp parallel for schedule(dynamic, 5) num_threads(threads) reduction(+ : done)
  for (int64_t i = row_begin; i < row_end; i++) {
    float J[128];
    for (int64_t j = i + 1; j < n; j++) {
      for (int k = 0; k < K; k++) {
        const size_t inter = calc_intersize(&sk[i][k], &sk[j][k], s64, bbits);
        J[k] = static_cast<float>(sko_jaccard(static_cast<uint32_t>(inter), s64, 0.0));
      }
      float core, acc;
      sko_fit_slope_f32(J, kmers, K, s64, &core, &acc);
      const int64_t pos = condensed(i, j, n);
      out[pos * 2] = core;
      out[pos * 2 + 1] = acc;
      ++done;
    }
  }
  return done;
}

// calc_intersize of one pair, for checking the oracle's restatement.
uint32_t ref_intersize(const uint64_t *a, const uint64_t *b, int s64, int bbits) {
  std::vector<uint64_t> va(a, a + static_cast<int64_t>(s64) * bbits);
  std::vector<uint64_t> vb(b, b + static_cast<int64_t>(s64) * bbits);
  return static_cast<uint32_t>(calc_intersize(&va, &vb, s64, bbits));
}

}  // extern "C"
