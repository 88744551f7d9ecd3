/*
 * sk_oracle.c -- CPU restatement of pp-sketchlib's distance path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against (and the CPU baseline bench.py times); the product library never
 * links, loads or calls it.
 *
 * Every function restates one piece of the reference (paths within
 * bacpop/pp-sketchlib):
 *   sko_intersize      calc_intersize            src/dist/dist.cpp:50-78
 *   sko_csrs           csrs                      src/random/random_match.cpp:318-336
 *   sko_jaccard        Reference::jaccard_dist   src/reference.cpp:86-96
 *                      observed_excess           src/dist/dist.hpp:14-24
 *   sko_fit_slope_f64  fit_slope (semantics)     src/dist/linear_regression.cpp:16-60
 *   sko_fit_slope_f32  fit_slope (float LDLT arithmetic of Eigen's pivoted LDLT)
 *   sko_dists          query_db loops            src/api.cpp:195-283
 *   sko_dists_multi    the same, every float output of one pass
 *   sko_knn_self       query_db_sparse           src/api.cpp:332-432
 *   sko_sparsify       sparsify_dists_by_threshold src/dist/matrix_ops.cpp:38-69
 *   sko_long_to_square long_to_square            src/dist/matrix_ops.cpp:71-126
 *   sko_square_to_long square_to_long            src/dist/matrix_ops.cpp:130-150
 *   sko_closest_cluster closest_cluster / nearest_neighbour
 *                                                src/random/random_match.cpp:222-227, 338-359
 *   sko_sketch         sketch (one sample, one k) src/sketch/sketch.cpp:120-168
 *                      stHashIterator / NTMC64   src/sketch/stHashIterator.hpp:63-120,
 *                                                src/sketch/nthash.hpp:57-126, 341-372
 *                      binsign, fillusigs, densifybin, univhash, inverse_minhash
 *                                                src/sketch/sketch.cpp:63-118
 *
 * Pinning: the golden vectors of the reference's own regression test
 * (test/ppsketch_ref*.npy, checked by test/test-dists.py) pin the Jaccard,
 * random-correction and fit semantics; tests/test_oracle_golden.py holds the
 * checks.  Built with -ffp-contract=off so no multiply-add is fused.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------- intersection */

/* Number of the 64*s64 bins whose bbits-bit values are equal in both sketches.
 * The reference returns raw samebits in both of its branches: observed_excess
 * with expected 0 is samebits * max / max. */
uint32_t sko_intersize(const uint64_t *s1, const uint64_t *s2, int s64, int bbits) {
  uint64_t samebits = 0;
  for (int i = 0; i < s64; i++) {
    uint64_t bits = ~(uint64_t)0;
    for (int j = 0; j < bbits; j++) bits &= ~(s1[i * bbits + j] ^ s2[i * bbits + j]);
    samebits += (uint64_t)__builtin_popcountll(bits);
  }
  return (uint32_t)samebits;
}

/* ----------------------------------------------------------- random match */

double sko_csrs(int k, int use_rc, uint64_t l1, uint64_t l2) {
  double random_chance = 0;
  const double match_chance = ldexp(1.0, (k - 1) * 2 + (use_rc ? 1 : 0));
  const double j1 = 1 - pow(1 - (double)1 / match_chance, (double)l1);
  const double j2 = 1 - pow(1 - (double)1 / match_chance, (double)l2);
  if (j1 > 0 && j2 > 0) random_chance = (j1 * j2) / (j1 + j2 - j1 * j2);
  return random_chance;
}

typedef struct {
  int mode;               /* 0 none, 1 equal base, 2 table */
  int use_rc;
  int n_clusters;
  const float *table;     /* [K][C][C] */
  const uint16_t *cl_rows, *cl_cols;
  const uint64_t *len_rows, *len_cols;
} sko_random;

/* Self: rows are "this" (r1 = i); query mode: rows are queries and the table
 * is indexed [k][cluster(ref = col)][cluster(query = row)] (src/api.cpp:264-266). */
static double random_for(const sko_random *r, int self, int k_idx, int kmer, int64_t i,
                         int64_t j) {
  if (!r || r->mode == 0) return 0.0;
  if (r->mode == 1) {
    const uint64_t li = r->len_rows ? r->len_rows[i] : 0, lj = r->len_cols ? r->len_cols[j] : 0;
    return self ? sko_csrs(kmer, r->use_rc, li, lj) : sko_csrs(kmer, r->use_rc, lj, li);
  }
  const int C = r->n_clusters;
  const int ci = r->cl_rows ? r->cl_rows[i] : 0, cj = r->cl_cols ? r->cl_cols[j] : 0;
  const int a = self ? ci : cj, b = self ? cj : ci;
  return (double)r->table[(int64_t)k_idx * C * C + a * C + b];
}

/* Reference::jaccard_dist + observed_excess(obs, r, 1), as a double. */
double sko_jaccard(uint32_t intersize, int s64, double random_jaccard) {
  const double jaccard_obs = intersize / (double)(64 * (uint64_t)s64);
  const double diff = jaccard_obs > random_jaccard ? jaccard_obs - random_jaccard : 0;
  return diff * 1 / (1 - random_jaccard);
}

/* ------------------------------------------------------------ regression */

/* Range of the fit: first..last index with J > tolerance (the reference's
 * `valid` vector).  Returns the range length, 0 when no J passes. */
static int fit_range(const float *J, int K, int s64, int *first) {
  const double tolerance = 5.0 / (s64 * 64);
  int f = -1, l = -1;
  for (int i = 0; i < K; i++) {
    if (J[i] > tolerance) {
      if (f < 0) f = i;
      l = i;
    }
  }
  *first = f;
  return f < 0 ? 0 : l - f + 1;
}

/* Exact-arithmetic semantics of fit_slope: least squares of log J on k over
 * the range in double,
 *   xm = sum x / n, ym = sum y / n,
 *   slope = sum (x - xm) y / sum (x - xm)^2, intercept = ym - slope xm.
 * Fewer than 2 points in the range gives (0, 0) (the reference CPU calls
 * exit(1) there, its GPU writes 0, 0); so does a zero J strictly inside the
 * range (first and last are above tolerance by construction). */
void sko_fit_slope_f64(const float *J, const int *kmers, int K, int s64, float *core, float *acc) {
  int f;
  const int n = fit_range(J, K, s64, &f);
  *core = 0.0f;
  *acc = 0.0f;
  if (n < 2) return;
  /* a zero J inside the range has no logarithm; Eigen's float LDLT solve
   * (the arithmetic of sko_fit_slope_f32) turns the -inf into NaN slopes,
   * which fit_slope reports as (0, 0) */
  for (int i = f + 1; i < f + n - 1; i++)
    if (J[i] <= 0.0f) return;
  double sx = 0.0;
  for (int i = f; i < f + n; i++) sx = sx + (double)kmers[i];
  const double xm = sx / n;
  double sy = 0.0, sxx = 0.0, sxy = 0.0;
  for (int i = f; i < f + n; i++) {
    const double y = log((double)J[i]);
    const double dx = (double)kmers[i] - xm;
    sy = sy + y;
    sxx = sxx + dx * dx;
    sxy = sxy + dx * y;
  }
  const double ym = sy / n;
  const double slope = sxy / sxx;
  const double icpt = ym - slope * xm;
  if (slope < 0.0) *core = (float)(1.0 - exp(slope));
  if (icpt < 0.0) *acc = (float)(1.0 - exp(icpt));
}

/* The reference's float arithmetic: normal equations X'X b = X'y with
 * X = [1, k] solved by Eigen's pivoted LDLT in float.  The larger diagonal
 * (sum k^2) is pivoted first, so with c = sum k^2, b = sum k, a = n:
 *   l = b / c, d1 = a - l * (c * l),
 *   z0 = sum k*y, z1 = sum y - l * z0, z0 /= c, z1 /= d1, z0 -= l * z1,
 *   slope = z0, intercept = z1; then 1 - expf() of each when negative. */
void sko_fit_slope_f32(const float *J, const int *kmers, int K, int s64, float *core, float *acc) {
  int f;
  const int n = fit_range(J, K, s64, &f);
  *core = 0.0f;
  *acc = 0.0f;
  if (n < 2) return;
  float a = (float)n, b = 0.0f, c = 0.0f, sy = 0.0f, sxy = 0.0f;
  for (int i = f; i < f + n; i++) {
    const float x = (float)kmers[i], y = logf(J[i]);
    b = b + x;
    c = c + x * x;
    sy = sy + y;
    sxy = sxy + x * y;
  }
  const float l = b / c;
  const float d1 = a - l * (c * l);
  float z0 = sxy;
  float z1 = sy - l * z0;
  z0 = z0 / c;
  z1 = (fabsf(d1) > 1.17549435e-38f) ? z1 / d1 : 0.0f;
  z0 = z0 - l * z1;
  if (z0 < 0.0f) *core = 1.0f - expf(z0);
  if (z1 < 0.0f) *acc = 1.0f - expf(z1);
}

/* --------------------------------------------------------------- dists */

static int64_t condensed(int64_t i, int64_t j, int64_t n) {
  return n * i - ((i * (i + 1)) >> 1) + j - 1 - i;
}

/* Dense distances, rows x cols, in the reference's long-form order.
 * Sketches in the reference word layout [n][K][s64 * bbits].
 * out_mode 0: float (pairs, 2) core/acc; 1: float (pairs, K) Jaccard;
 *          2: uint32 (pairs, K) intersection counts.
 * regress 0: sko_fit_slope_f64, 1: sko_fit_slope_f32. */
void sko_dists(const uint64_t *rows, int64_t n_rows, const uint64_t *cols, int64_t n_cols, int self,
               int K, const int *kmers, int s64, int bbits, const sko_random *random, int out_mode,
               int regress, void *out, int threads) {
  const int64_t W = (int64_t)s64 * bbits;
  const int64_t outer = self ? n_cols : n_rows;
#ifdef _OPENMP
  if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 5) num_threads(threads)
#endif
  for (int64_t i = 0; i < outer; i++) {
    float J[128];
    const int64_t j0 = self ? i + 1 : 0;
    for (int64_t j = j0; j < n_cols; j++) {
      const int64_t pos = self ? condensed(i, j, n_cols) : i * n_cols + j;
      const uint64_t *si = (self ? cols : rows) + i * K * W;
      const uint64_t *sj = cols + j * K * W;
      for (int k = 0; k < K; k++) {
        const uint32_t c = sko_intersize(si + k * W, sj + k * W, s64, bbits);
        if (out_mode == 2) {
          ((uint32_t *)out)[pos * K + k] = c;
          continue;
        }
        J[k] = (float)sko_jaccard(c, s64, random_for(random, self, k, kmers[k], i, j));
      }
      if (out_mode == 1) {
        memcpy((float *)out + pos * K, J, sizeof(float) * K);
      } else if (out_mode == 0) {
        float core, acc;
        if (regress) sko_fit_slope_f32(J, kmers, K, s64, &core, &acc);
        else sko_fit_slope_f64(J, kmers, K, s64, &core, &acc);
        ((float *)out)[pos * 2] = core;
        ((float *)out)[pos * 2 + 1] = acc;
      }
    }
  }
}

/* The query_db loops for rows [row_begin, row_end) with every float output of
 * one intersection pass: the Jaccards (pairs, K), the double fit and the
 * float-LDLT fit (pairs, 2); any output may be NULL.  Outputs hold only the
 * rows asked for, in long-form order starting at the first pair of
 * row_begin (self: condensed(row_begin, row_begin + 1); query:
 * row_begin * n_cols).  Returns the pairs computed. */
int64_t sko_dists_multi(const uint64_t *rows, int64_t n_rows, const uint64_t *cols, int64_t n_cols,
                        int self, int K, const int *kmers, int s64, int bbits,
                        const sko_random *random, int64_t row_begin, int64_t row_end, float *jac,
                        float *fit64, float *fit32, int threads) {
  const int64_t W = (int64_t)s64 * bbits;
  const int64_t base = self ? (row_begin < n_cols - 1 ? condensed(row_begin, row_begin + 1, n_cols) : 0)
                            : row_begin * n_cols;
  int64_t done = 0;
#ifdef _OPENMP
  if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 5) num_threads(threads) reduction(+ : done)
#endif
  for (int64_t i = row_begin; i < row_end; i++) {
    float J[128];
    const int64_t j0 = self ? i + 1 : 0;
    const uint64_t *si = (self ? cols : rows) + i * K * W;
    for (int64_t j = j0; j < n_cols; j++) {
      const int64_t pos = (self ? condensed(i, j, n_cols) : i * n_cols + j) - base;
      const uint64_t *sj = cols + j * K * W;
      for (int k = 0; k < K; k++)
        J[k] = (float)sko_jaccard(sko_intersize(si + k * W, sj + k * W, s64, bbits), s64,
                                  random_for(random, self, k, kmers[k], i, j));
      if (jac) memcpy(jac + pos * K, J, sizeof(float) * K);
      if (fit64) sko_fit_slope_f64(J, kmers, K, s64, &fit64[pos * 2], &fit64[pos * 2 + 1]);
      if (fit32) sko_fit_slope_f32(J, kmers, K, s64, &fit32[pos * 2], &fit32[pos * 2 + 1]);
      done++;
    }
  }
  return done;
}

/* All-vs-all core/accessory (double fit) for rows [row_begin, row_end) only;
 * out is the full (n(n-1)/2, 2) long form.  Returns the pairs computed. */
int64_t sko_dists_self_rows(const uint64_t *words, int64_t n, int K, const int *kmers, int s64,
                            int bbits, int64_t row_begin, int64_t row_end, float *out,
                            int threads) {
  const int64_t W = (int64_t)s64 * bbits;
  int64_t done = 0;
#ifdef _OPENMP
  if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 5) num_threads(threads) reduction(+ : done)
#endif
  for (int64_t i = row_begin; i < row_end; i++) {
    float J[128];
    for (int64_t j = i + 1; j < n; j++) {
      for (int k = 0; k < K; k++)
        J[k] = (float)sko_jaccard(sko_intersize(words + (i * K + k) * W, words + (j * K + k) * W,
                                                s64, bbits), s64, 0.0);
      const int64_t pos = condensed(i, j, n);
      sko_fit_slope_f64(J, kmers, K, s64, &out[pos * 2], &out[pos * 2 + 1]);
      done++;
    }
  }
  return done;
}

/* ------------------------------------------------------------------ kNN */

/* Self kNN from a dense long-form matrix (pairs, n_cols), column `col`:
 * per row the kNN smallest d(i, j), j != i, with self as +inf; ascending by
 * (d, j).  jaccard != 0 ranks 1 - J and reports 1 - (1 - J) as the reference
 * does (src/api.cpp:370-371, 424-429). */
void sko_knn_self(const float *long_form, int64_t n, int n_cols, int col, int jaccard, int knn,
                  int64_t *i_out, int64_t *j_out, float *d_out) {
  float *key = (float *)malloc(sizeof(float) * (size_t)knn);
  int64_t *idx = (int64_t *)malloc(sizeof(int64_t) * (size_t)knn);
  for (int64_t i = 0; i < n; i++) {
    int count = 0;
    for (int64_t j = 0; j < n; j++) {
      float d;
      if (j == i) {
        d = INFINITY;
      } else {
        const int64_t a = j < i ? j : i, b = j < i ? i : j;
        d = long_form[condensed(a, b, n) * n_cols + col];
        if (jaccard) d = 1.0f - d;
      }
      if (count < knn || d < key[knn - 1]) {
        int pos = count < knn ? count++ : knn - 1;
        while (pos > 0 && key[pos - 1] > d) {
          key[pos] = key[pos - 1];
          idx[pos] = idx[pos - 1];
          pos--;
        }
        key[pos] = d;
        idx[pos] = j;
      }
    }
    for (int e = 0; e < knn; e++) {
      i_out[i * knn + e] = i;
      j_out[i * knn + e] = idx[e];
      d_out[i * knn + e] = jaccard ? 1.0f - key[e] : key[e];
    }
  }
  free(key);
  free(idx);
}

/* ----------------------------------------------------- matrix transforms */

/* Upper-triangle entries of the square form with value < cutoff, row-major.
 * Returns the count; outputs may be NULL to count only. */
int64_t sko_sparsify(const float *long_form, int64_t n, int n_cols, int col, float cutoff,
                     int64_t *i_out, int64_t *j_out, float *d_out) {
  int64_t m = 0;
  for (int64_t i = 0; i < n; i++) {
    for (int64_t j = i + 1; j < n; j++) {
      const float v = long_form[condensed(i, j, n) * n_cols + col];
      if (v < cutoff) {
        if (i_out) {
          i_out[m] = i;
          j_out[m] = j;
          d_out[m] = v;
        }
        m++;
      }
    }
  }
  return m;
}

void sko_long_to_square(const float *rr, int64_t n_rr, const float *qr, const float *qq,
                        int64_t n_qq, float *square) {
  const int64_t n = n_rr + n_qq;
  for (int64_t i = 0; i < n; i++) square[i * n + i] = 0.0f;
  for (int64_t i = 0; i < n_rr; i++)
    for (int64_t j = i + 1; j < n_rr; j++)
      square[i * n + j] = square[j * n + i] = rr[condensed(i, j, n_rr)];
  for (int64_t i = 0; i < n_qq; i++)
    for (int64_t j = i + 1; j < n_qq; j++)
      square[(i + n_rr) * n + j + n_rr] = square[(j + n_rr) * n + i + n_rr] =
          qq[condensed(i, j, n_qq)];
  for (int64_t d = 0; d < n_rr * n_qq; d++) {
    const int64_t i = d % n_rr, j = d / n_rr + n_rr;
    square[i * n + j] = square[j * n + i] = qr[d];
  }
}

void sko_square_to_long(const float *square, int64_t n, float *long_out) {
  for (int64_t i = 0; i < n; i++)
    for (int64_t j = i + 1; j < n; j++) long_out[condensed(i, j, n)] = square[i * n + j];
}

/* ------------------------------------------------- query cluster lookup */

/* Cluster of a query missing from the Monte Carlo model's table
 * (RandomMC::lookup_array -> closest_cluster -> nearest_neighbour,
 * src/random/random_match.cpp:254-273, 222-227, 351-359; apply_rc :338-349):
 * with use_rc the A/T and C/G frequencies are averaged; the composition is
 * cast to float and the centroid [C][4] with the smallest squared distance,
 * summed over A, C, G, T in order, is taken, the first on a tie; 0 without
 * clusters. */
void sko_closest_cluster(const float *centroids, int n_clusters, int use_rc,
                         const double *base_freq, int64_t n, uint16_t *out) {
  for (int64_t i = 0; i < n; i++) {
    double b[4] = {base_freq[4 * i], base_freq[4 * i + 1], base_freq[4 * i + 2],
                   base_freq[4 * i + 3]};
    if (use_rc) {
      b[0] = 0.5 * (b[0] + b[3]);
      b[1] = 0.5 * (b[1] + b[2]);
      b[2] = b[1];
      b[3] = b[0];
    }
    int best = 0;
    float best_d = INFINITY;
    for (int c = 0; c < n_clusters; c++) {
      float d = 0.0f;
      for (int j = 0; j < 4; j++) {
        const float diff = centroids[c * 4 + j] - (float)b[j];
        d += diff * diff;
      }
      if (d < best_d) {
        best_d = d;
        best = c;
      }
    }
    out[i] = (uint16_t)best;
  }
}

/* ------------------------------------------------------ synthetic inputs */

/* The seeded bin-level tree generator of the benchmarks, restated so the
 * timed reference arm can build its inputs without the library under test.
 * Sample s at k-mer index k, bin `bin`: h = splitmix64 finaliser of
 *   seed ^ s * 0x9E3779B97F4A7C15 ^ ((k << 32 | bin) * 0xC2B2AE3D27D4EB4F);
 * a root, or a sample whose (h >> 32) < thresh[s][k], takes the 14-bit value
 * h & 0x3FFF, every other sample its parent's value.  Samples are filled
 * level by level (parents first), a bin being inherited by copying its bit
 * from the parent's plane words; the result is the reference word layout
 * [n][K][s64][bbits] (src/sketch/sketch.cpp:82-92).  Returns -1 when a
 * parent does not precede its child. */
static uint64_t sko_mix(uint64_t x) {
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ULL;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBULL;
  x ^= x >> 31;
  return x;
}

int sko_synth_words(const int32_t *parent, const uint32_t *thresh, int64_t n, int K, int s64,
                    uint64_t seed, uint64_t *words, int threads) {
  const int bbits = 14;
  int32_t *depth = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
  int32_t max_depth = 0;
  for (int64_t s = 0; s < n; s++) {
    if (parent[s] >= s) {
      free(depth);
      return -1;
    }
    depth[s] = parent[s] < 0 ? 0 : depth[parent[s]] + 1;
    if (depth[s] > max_depth) max_depth = depth[s];
  }
  const int64_t W = (int64_t)s64 * bbits;
  for (int32_t level = 0; level <= max_depth; level++) {
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
    for (int64_t s = 0; s < n; s++) {
      if (depth[s] != level) continue;
      const int32_t par = parent[s];
      for (int k = 0; k < K; k++) {
        const uint32_t th = thresh[s * K + k];
        uint64_t *o = words + (s * K + k) * W;
        const uint64_t *po = par < 0 ? NULL : words + ((int64_t)par * K + k) * W;
        for (int b = 0; b < s64; b++) {
          uint64_t w[14] = {0}, fresh = 0;
          for (int i = 0; i < 64; i++) {
            const uint64_t bin = (uint64_t)b * 64u + (uint64_t)i;
            const uint64_t h = sko_mix(seed ^ ((uint64_t)s * 0x9E3779B97F4A7C15ULL) ^
                                       ((((uint64_t)k << 32) | bin) * 0xC2B2AE3D27D4EB4FULL));
            if (par < 0 || (uint32_t)(h >> 32) < th) {
              const uint32_t v = (uint32_t)h & 0x3FFFu;
              fresh |= 1ULL << i;
              for (int p = 0; p < bbits; p++) w[p] |= (uint64_t)((v >> p) & 1u) << i;
            }
          }
          for (int p = 0; p < bbits; p++)
            o[b * bbits + p] = po ? (po[b * bbits + p] & ~fresh) | w[p] : w[p];
        }
      }
    }
  }
  free(depth);
  return 0;
}

/* -------------------------------------------------------------- sketching */

/* ntHash (Mohamadi et al., Bioinformatics 2016) as the reference uses it:
 * 64-bit per-base seeds (src/sketch/nthash_tables.hpp:25-29), combined with a
 * "split rotation" that rotates the low 33 bits and the high 31 bits of the
 * hash independently (nthash.hpp:17-55).  Forward hash of b_0..b_{k-1}:
 * XOR_i srol^(k-1-i)(seed[b_i]); reverse: XOR_i srol^i(seed[comp(b_i)]);
 * canonical: the smaller of the two (nthash.hpp:103-118). */
static const uint64_t kNtSeed[4] = {0x3c8bfbb395c60474ULL, 0x3193c18562a02b4cULL,
                                    0x20323ed082572324ULL, 0x295549f54be24456ULL};
#define SKO_LO33 0x1FFFFFFFFULL
#define SKO_SIGN_MOD ((1ULL << 61) - 1ULL)

static uint64_t sko_srol(uint64_t v, unsigned n) {
  const uint64_t lo = v & SKO_LO33, hi = v >> 33;
  const unsigned a = n % 33, b = n % 31;
  const uint64_t lo2 = a ? (((lo << a) | (lo >> (33 - a))) & SKO_LO33) : lo;
  const uint64_t hi2 = b ? (((hi << b) | (hi >> (31 - b))) & 0x7FFFFFFFULL) : hi;
  return (hi2 << 33) | lo2;
}

static uint64_t sko_sror1(uint64_t v) {
  const uint64_t lo = v & SKO_LO33, hi = v >> 33;
  const uint64_t lo2 = ((lo >> 1) | (lo << 32)) & SKO_LO33;
  const uint64_t hi2 = ((hi >> 1) | (hi << 30)) & 0x7FFFFFFFULL;
  return (hi2 << 33) | lo2;
}

/* 0..3 for A, C, G, T (U counts as T), either case; -1 for anything else,
 * which the reference's seed table maps to the zero seed and skips. */
static int sko_base(unsigned char c) {
  switch (c) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': case 'U': case 'u': return 3;
    default: return -1;
  }
}

static uint64_t sko_univhash(uint64_t s, uint64_t t) {
  const uint64_t x = 1009ULL * s + (1000ULL * 1000ULL + 3ULL) * t;
  return (48271ULL * x + 11ULL) % ((1ULL << 31) - 1ULL);
}

/* Sketch of one sample at one k: the sequences seq_off[first..last) (each
 * sequence i is bases[seq_off[i], seq_off[i+1])), every window of k valid
 * bases inside one sequence hashed, the hash reduced mod 2^61-1 and kept as
 * its bin's minimum; then the empty bins are filled in order by the
 * reference's probe sequence and the low bbits bits of each bin value are
 * written as bit planes, 64 bins per word.  Returns the densify result
 * (0 no empty bin, 1 filled, -1 all empty); *inv_minhash is bin 0's value
 * over 2^61-1 before filling. */
static int sko_cmp_u64(const void *a, const void *b) {
  const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : x > y;
}

static void sko_binsign(uint64_t *signs, uint64_t h, uint64_t binsize) {
  const uint64_t sign = h % SKO_SIGN_MOD;
  const uint64_t bin = sign / binsize;
  if (sign < signs[bin]) signs[bin] = sign;
}

/* min_count > 0: only hashes that occur at least min_count times in the
 * sample enter the bins -- the reference's exact counter (HashCounter,
 * src/sketch/countmin.cpp:55-72, counting full 64-bit hash values; its uint8
 * saturation at 255 never changes the answer for min_count <= 255). */
/* Codon-phased spaced-seed hash of the window at s (generate_seeds,
 * src/sketch/sketch.cpp:30-61: k kept positions 0, 3, ..., 3(k-1) of a
 * window of 3k-2 bases; NTMSMC64 / NTMSM64, src/sketch/nthash.hpp:553-722:
 * the dense hash with the masked positions' terms XORed out, i.e. the XOR of
 * the kept positions' terms).  Every base of the window must be valid. */
static uint64_t sko_phased_hash(const unsigned char *s, int k, int use_rc) {
  const int kw = 3 * k - 2;
  uint64_t fs = 0, rs = 0;
  for (int m = 0; m < k; m++) {
    const int i = 3 * m, c = sko_base(s[i]);
    fs ^= sko_srol(kNtSeed[c], (unsigned)(kw - 1 - i));
    rs ^= sko_srol(kNtSeed[3 - c], (unsigned)i);
  }
  return (use_rc && rs < fs) ? rs : fs;
}

int sko_sketch(const char *bases, const int64_t *seq_off, int64_t first, int64_t last, int k,
               int s64, int bbits, int use_rc, int codon_phased, int min_count, uint64_t *signs,
               uint64_t *words, double *inv_minhash) {
  const uint64_t nbins = (uint64_t)s64 * 64;
  const uint64_t binsize = (SKO_SIGN_MOD + nbins - 1) / nbins;
  uint64_t rk[4];
  uint64_t *hashes = NULL;
  int64_t n_hashes = 0;
  if (min_count > 0) hashes = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(seq_off[last] - seq_off[first] + 1));
  for (int c = 0; c < 4; c++) rk[c] = sko_srol(kNtSeed[c], (unsigned)k);
  for (uint64_t b = 0; b < nbins; b++) signs[b] = UINT64_MAX;
  for (int64_t sq = first; sq < last && codon_phased; sq++) {   /* spaced seeds */
    const unsigned char *s = (const unsigned char *)bases + seq_off[sq];
    const int64_t len = seq_off[sq + 1] - seq_off[sq], kw = 3 * (int64_t)k - 2;
    int64_t run = 0;
    for (int64_t p = 0; p < len; p++) {
      run = sko_base(s[p]) < 0 ? 0 : run + 1;
      if (run >= kw) {
        const uint64_t h = sko_phased_hash(s + p - kw + 1, k, use_rc);
        if (hashes) hashes[n_hashes++] = h;
        else sko_binsign(signs, h, binsize);
      }
    }
  }
  for (int64_t sq = first; sq < last && !codon_phased; sq++) {
    const unsigned char *s = (const unsigned char *)bases + seq_off[sq];
    const int64_t len = seq_off[sq + 1] - seq_off[sq];
    uint64_t fh = 0, rh = 0;
    int64_t run = 0;
    for (int64_t p = 0; p < len; p++) {
      const int c = sko_base(s[p]);
      if (c < 0) {  /* restart after a non-base, as stHashIterator::init does */
        run = 0;
        fh = rh = 0;
        continue;
      }
      /* roll in base p; roll out base p-k once the window is full */
      uint64_t f = sko_srol(fh, 1) ^ kNtSeed[c];
      uint64_t r = rh ^ rk[3 - c];
      if (run >= k) {
        const int o = sko_base(s[p - k]);
        f ^= rk[o];
        r ^= kNtSeed[3 - o];
      }
      fh = f;
      rh = sko_sror1(r);
      if (run < k) run++;
      if (run >= k) {
        const uint64_t h = (use_rc && rh < fh) ? rh : fh;
        if (hashes) hashes[n_hashes++] = h;
        else sko_binsign(signs, h, binsize);
      }
    }
  }
  if (hashes) {
    qsort(hashes, (size_t)n_hashes, sizeof(uint64_t), sko_cmp_u64);
    for (int64_t i = 0; i < n_hashes;) {
      int64_t j = i;
      while (j < n_hashes && hashes[j] == hashes[i]) j++;
      if (j - i >= min_count) sko_binsign(signs, hashes[i], binsize);
      i = j;
    }
    free(hashes);
  }
  if (inv_minhash) *inv_minhash = (double)signs[0] / (double)SKO_SIGN_MOD;
  uint64_t mn = UINT64_MAX, mx = 0;
  for (uint64_t b = 0; b < nbins; b++) {
    if (signs[b] < mn) mn = signs[b];
    if (signs[b] > mx) mx = signs[b];
  }
  int densified = 0;
  if (mx == UINT64_MAX) {
    if (mn == UINT64_MAX) {
      densified = -1;
    } else {
      for (uint64_t i = 0; i < nbins; i++) {
        uint64_t j = i, attempt = 0;
        while (signs[j] == UINT64_MAX) j = sko_univhash(i, attempt++) % nbins;
        signs[i] = signs[j];
      }
      densified = 1;
    }
  }
  memset(words, 0, sizeof(uint64_t) * (size_t)s64 * (size_t)bbits);
  for (uint64_t b = 0; b < nbins; b++)
    for (int i = 0; i < bbits; i++)
      words[(b / 64) * (uint64_t)bbits + (uint64_t)i] |= ((signs[b] >> i) & 1ULL) << (b % 64);
  return densified;
}

/* sko_sketch over n samples (sample s owns sequences sample_seqs[s] ..
 * sample_seqs[s+1]) and K k-mer lengths: words [n][K][s64*bbits],
 * inv_minhash [n][K], densified [n] (any k with a nonzero densify result). */
void sko_sketch_samples(const char *bases, const int64_t *seq_off, const int64_t *sample_seqs,
                        int64_t n, const int *kmers, int K, int s64, int bbits, int use_rc,
                        int codon_phased, int min_count, uint64_t *words, double *inv_minhash,
                        uint8_t *densified, int threads) {
  const int64_t W = (int64_t)s64 * bbits;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
  for (int64_t s = 0; s < n; s++) {
    uint64_t *signs = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)s64 * 64);
    uint8_t any = 0;
    for (int k = 0; k < K; k++) {
      const int d = sko_sketch(bases, seq_off, sample_seqs[s], sample_seqs[s + 1], kmers[k], s64,
                               bbits, use_rc, codon_phased, min_count, signs,
                               words + (s * K + k) * W,
                               inv_minhash ? inv_minhash + s * K + k : NULL);
      if (d != 0) any = 1;
    }
    if (densified) densified[s] = any;
    free(signs);
  }
}
