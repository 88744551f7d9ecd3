// ref_gpu_dists.cu -- launches the reference's own GPU distance kernel.
//
// Same-GPU comparison and test infrastructure only.  oracle/Makefile compiles the
// reference's src/gpu/dist.cu for sm_100a from its own tree (with the
// stand-in header in oracle/ref_gpu_stub/) and links it with this file into
// oracle/_ref/libref_gpu.so.  This file reproduces what the reference's host
// driver does around the kernel for an all-vs-all or query-vs-reference call:
//
//   * flatten_by_samples (src/gpu/gpu_api.cpp:269-305) for the references:
//     uint64 words laid out [K][W][warpPad(N)] -- sample index fastest, bins
//     padded to a multiple of 32 samples; bin_stride = warpPad(N),
//     kmer_stride = bin_stride * W, sample_stride = 1;
//   * flatten_by_bins (src/gpu/gpu_api.cpp:232-265) for the queries:
//     [N][K][warpPad(W)]; bin_stride = 1, kmer_stride = warpPad(W),
//     sample_stride = K * kmer_stride;
//   * DeviceMemory (src/gpu/device_memory.cu:6-61): sketches, random table,
//     cluster lookup, k-mer list and the [core(n) | acc(n)] output on device;
//   * dispatchDists (src/gpu/dist.cu:408-470): L1-preferring cache config,
//     block shape from the reference's getBlockSize (src/gpu/dist.cu:327-347),
//     dynamic shared memory = sketchsize64 * bbits * 8 bytes, use_shared when
//     that fits the 48 KB default, dist_col = -1, max_diagonal = false;
//   * query_db_cuda's reshape (src/gpu/gpu_api.cpp:477-493) of the column-major
//     result into row-major (n_pairs, 2).
//
// The random-match table is either K floats with strides {1, 0, 0}
// (NoAdjust as zeros, EqualBase as one chance per k) or [K][C][C] with strides
// {C*C, C, 1} indexed by the reference and query cluster lookups
// (RandomMC::flattened_random, src/random/random_match.cpp:278-310).  The
// progress words live in device memory and the kill flag stays false.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <stdexcept>
#include <tuple>
#include <vector>

#include "gpu/cuda.cuh"            // progress_ptrs (reference header)
#include "gpu/device_memory.cuh"   // SketchStrides, RandomStrides (reference header)

// Defined in the reference's src/gpu/dist.cu.
__global__ void calculate_dists(const bool self, const uint64_t *ref, const long ref_n,
                                const uint64_t *query, const long query_n, const int *kmers,
                                const int kmer_n, float *dists, const long long dist_n,
                                const float *random_table, const uint16_t *ref_idx_lookup,
                                const uint16_t *query_idx_lookup, const SketchStrides ref_strides,
                                const SketchStrides query_strides,
                                const RandomStrides random_strides, progress_ptrs progress,
                                const bool use_shared, const int dist_col,
                                const bool max_diagonal);
std::tuple<size_t, size_t> getBlockSize(const size_t ref_samples, const size_t query_samples,
                                        const size_t dist_rows, const bool self);

// dist.cu's dispatchDists refers to DeviceMemory, whose definition needs the
// reference's full host build; the harness allocates its own buffers and never
// calls dispatchDists, so these bodies only satisfy the linker.
DeviceMemory::DeviceMemory(SketchStrides &, SketchStrides &, std::vector<Reference> &,
                           std::vector<Reference> &, const SketchSlice &, const FlatRandom &,
                           const std::vector<uint16_t> &, const std::vector<uint16_t> &,
                           const std::vector<size_t> &, long long, const bool, const int) {
  throw std::runtime_error("DeviceMemory is not built in the kernel harness");
}
DeviceMemory::~DeviceMemory() {}
std::vector<float> DeviceMemory::read_dists() {
  throw std::runtime_error("DeviceMemory is not built in the kernel harness");
}

namespace {

struct Buffers {
  void *p[9] = {};
  ~Buffers() {
    for (void *q : p)
      if (q) cudaFree(q);
  }
};

int report(char *err, int errlen, const char *what, cudaError_t e) {
  if (err && errlen > 0)
    std::snprintf(err, static_cast<size_t>(errlen), "%s: %s", what, cudaGetErrorString(e));
  return 1;
}

}  // namespace

extern "C" {

// Distances with the reference kernel.
//   ref_words    host [n_ref][K][sketchsize64 * bbits] uint64, the reference layout
//   query_words  host [n_query][K][...] or null for all-vs-all of ref_words
//   table        host float: [K] (n_clusters = 0) or [K][C][C] (n_clusters = C),
//                or null (NoAdjust)
//   ref_lookup / query_lookup  host uint16 cluster ids (n_clusters > 0)
//   out          host [n_pairs][2] float32 (core, accessory), or null
//   ms           per timed launch, mean (CUDA events on the launch stream)
// Requires n_pairs >= 1000: the kernel's progress update divides the pair index
// by n_pairs / 1000.  Returns 0, or 1 with a message in err.
int refgpu_dists(const uint64_t *ref_words, int64_t n_ref, const uint64_t *query_words,
                 int64_t n_query, const int32_t *kmers, int K, int sketchsize64, int bbits,
                 const float *table, int n_clusters, const uint16_t *ref_lookup,
                 const uint16_t *query_lookup, int warmup, int launches, float *out, double *ms,
                 char *err, int errlen) {
  const bool self = query_words == nullptr;
  const int64_t n_q = self ? n_ref : n_query;
  const long long n_pairs = self ? static_cast<long long>(n_ref) * (n_ref - 1) / 2
                                 : static_cast<long long>(n_ref) * n_query;
  if (n_pairs < 1000 || K < 1 || launches < 0 || warmup < 0 || n_clusters < 0 ||
      (n_clusters > 0 && (!table || !ref_lookup || (!self && !query_lookup)))) {
    if (err && errlen > 0)
      std::snprintf(err, static_cast<size_t>(errlen),
                    "need >= 1000 pairs, K >= 1 and lookups for a clustered table");
    return 1;
  }
  const size_t W = static_cast<size_t>(sketchsize64) * bbits;
  auto warp_pad = [](size_t x) { return (x + 31) / 32 * 32; };
  SketchStrides rs_{};
  rs_.sample_stride = 1;
  rs_.bin_stride = warp_pad(static_cast<size_t>(n_ref));
  rs_.kmer_stride = rs_.bin_stride * W;
  rs_.sketchsize64 = static_cast<size_t>(sketchsize64);
  rs_.bbits = static_cast<size_t>(bbits);
  std::vector<uint64_t> flat_ref(rs_.kmer_stride * K, 0);
  for (int k = 0; k < K; ++k)
    for (size_t b = 0; b < W; ++b) {
      uint64_t *dst = flat_ref.data() + k * rs_.kmer_stride + b * rs_.bin_stride;
      for (int64_t i = 0; i < n_ref; ++i) dst[i] = ref_words[(static_cast<size_t>(i) * K + k) * W + b];
    }
  SketchStrides qs_ = rs_;
  std::vector<uint64_t> flat_q;
  if (!self) {
    qs_.bin_stride = 1;
    qs_.kmer_stride = warp_pad(W);
    qs_.sample_stride = qs_.kmer_stride * K;
    flat_q.assign(qs_.sample_stride * n_query, 0);
    for (int64_t i = 0; i < n_query; ++i)
      for (int k = 0; k < K; ++k)
        std::memcpy(flat_q.data() + i * qs_.sample_stride + k * qs_.kmer_stride,
                    query_words + (static_cast<size_t>(i) * K + k) * W, W * 8);
  }
  const size_t C = static_cast<size_t>(n_clusters);
  std::vector<float> tab = n_clusters > 0 ? std::vector<float>(table, table + K * C * C)
                                          : std::vector<float>(K, 0.0f);
  if (n_clusters == 0 && table)
    for (int k = 0; k < K; ++k) tab[k] = table[k];
  const RandomStrides rstr = n_clusters > 0 ? RandomStrides{C * C, C, 1} : RandomStrides{1, 0, 0};
  std::vector<uint16_t> rl(n_ref, 0), ql(n_q, 0);
  if (n_clusters > 0) {
    std::copy(ref_lookup, ref_lookup + n_ref, rl.begin());
    if (!self) std::copy(query_lookup, query_lookup + n_query, ql.begin());
  }
  std::vector<int> km(kmers, kmers + K);

  Buffers buf;
  uint64_t *d_ref = nullptr, *d_query = nullptr;
  float *d_table = nullptr, *d_dists = nullptr;
  uint16_t *d_rl = nullptr, *d_ql = nullptr;
  int *d_kmers = nullptr, *d_done = nullptr;
  bool *d_kill = nullptr;
  cudaError_t e;
#define REFGPU_TRY(call, what)                     \
  if ((e = (call)) != cudaSuccess) return report(err, errlen, what, e)
#define REFGPU_ALLOC(ptr, bytes, slot, what)       \
  REFGPU_TRY(cudaMalloc(&ptr, bytes), what);       \
  buf.p[slot] = ptr
  REFGPU_ALLOC(d_ref, flat_ref.size() * 8, 0, "cudaMalloc sketches");
  if (!self) {
    REFGPU_ALLOC(d_query, flat_q.size() * 8, 1, "cudaMalloc queries");
  }
  REFGPU_ALLOC(d_table, tab.size() * sizeof(float), 2, "cudaMalloc table");
  REFGPU_ALLOC(d_rl, rl.size() * sizeof(uint16_t), 3, "cudaMalloc lookup");
  if (!self) {
    REFGPU_ALLOC(d_ql, ql.size() * sizeof(uint16_t), 4, "cudaMalloc lookup");
  }
  REFGPU_ALLOC(d_kmers, K * sizeof(int), 5, "cudaMalloc kmers");
  REFGPU_ALLOC(d_dists, 2 * n_pairs * sizeof(float), 6, "cudaMalloc dists");
  REFGPU_ALLOC(d_done, sizeof(int), 7, "cudaMalloc progress");
  REFGPU_ALLOC(d_kill, sizeof(bool), 8, "cudaMalloc kill flag");
  REFGPU_TRY(cudaMemcpy(d_ref, flat_ref.data(), flat_ref.size() * 8, cudaMemcpyHostToDevice), "copy sketches");
  if (!self)
    REFGPU_TRY(cudaMemcpy(d_query, flat_q.data(), flat_q.size() * 8, cudaMemcpyHostToDevice), "copy queries");
  REFGPU_TRY(cudaMemcpy(d_table, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice), "copy table");
  REFGPU_TRY(cudaMemcpy(d_rl, rl.data(), rl.size() * sizeof(uint16_t), cudaMemcpyHostToDevice), "copy lookup");
  if (!self)
    REFGPU_TRY(cudaMemcpy(d_ql, ql.data(), ql.size() * sizeof(uint16_t), cudaMemcpyHostToDevice), "copy lookup");
  REFGPU_TRY(cudaMemcpy(d_kmers, km.data(), K * sizeof(int), cudaMemcpyHostToDevice), "copy kmers");
  REFGPU_TRY(cudaMemset(d_dists, 0, 2 * n_pairs * sizeof(float)), "memset dists");
  REFGPU_TRY(cudaMemset(d_done, 0, sizeof(int)), "memset progress");
  REFGPU_TRY(cudaMemset(d_kill, 0, sizeof(bool)), "memset kill flag");
  REFGPU_TRY(cudaFuncSetCacheConfig(calculate_dists, cudaFuncCachePreferL1), "cache config");

  size_t block_size = 0, block_count = 0;
  std::tie(block_size, block_count) = getBlockSize(static_cast<size_t>(n_ref),
                                                   static_cast<size_t>(n_q), n_pairs, self);
  const size_t shared = W * sizeof(uint64_t);
  const bool use_shared = shared <= 48 * 1024;
  progress_ptrs prog{d_done, d_kill};
  const uint64_t *d_qw = self ? d_ref : d_query;
  const uint16_t *d_qlk = self ? d_rl : d_ql;

  cudaEvent_t t0, t1;
  REFGPU_TRY(cudaEventCreate(&t0), "event");
  REFGPU_TRY(cudaEventCreate(&t1), "event");
  double total = 0.0;
  for (int it = 0; it < warmup + launches; ++it) {
    REFGPU_TRY(cudaEventRecord(t0, 0), "event record");
    calculate_dists<<<static_cast<unsigned>(block_count), static_cast<unsigned>(block_size),
                      use_shared ? shared : 0>>>(
        self, d_ref, static_cast<long>(n_ref), d_qw, static_cast<long>(n_q), d_kmers, K, d_dists,
        n_pairs, d_table, d_rl, d_qlk, rs_, self ? rs_ : qs_, rstr, prog, use_shared, -1, false);
    REFGPU_TRY(cudaGetLastError(), "calculate_dists launch");
    REFGPU_TRY(cudaEventRecord(t1, 0), "event record");
    REFGPU_TRY(cudaEventSynchronize(t1), "calculate_dists");
    float t = 0.0f;
    REFGPU_TRY(cudaEventElapsedTime(&t, t0, t1), "event time");
    if (it >= warmup) total += t;
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (ms) *ms = launches ? total / launches : 0.0;
  if (out) {
    std::vector<float> colmajor(2 * n_pairs);
    REFGPU_TRY(cudaMemcpy(colmajor.data(), d_dists, colmajor.size() * sizeof(float),
                          cudaMemcpyDeviceToHost),
               "copy dists");
    for (long long p = 0; p < n_pairs; ++p) {
      out[2 * p] = colmajor[p];
      out[2 * p + 1] = colmajor[p + n_pairs];
    }
  }
#undef REFGPU_ALLOC
#undef REFGPU_TRY
  return 0;
}

// All-vs-all with a per-k table (null = NoAdjust); kept for the bench.
int refgpu_self_dists(const uint64_t *words, int64_t n, const int32_t *kmers, int K,
                      int sketchsize64, int bbits, const float *random_k, int warmup,
                      int launches, float *out, double *ms, char *err, int errlen) {
  return refgpu_dists(words, n, nullptr, 0, kmers, K, sketchsize64, bbits, random_k, 0, nullptr,
                      nullptr, warmup, launches, out, ms, err, errlen);
}

}  // extern "C"
