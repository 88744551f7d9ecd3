// ref_gpu_dists.cu -- launches the reference's own GPU distance kernel.
//
// BASELINE / TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles the
// reference's src/gpu/dist.cu for sm_100a from its own tree (with the
// stand-in header in oracle/ref_gpu_stub/) and links it with this file into
// oracle/_ref/libref_gpu.so.  This file reproduces what the reference's host
// driver does around the kernel for a self (all-vs-all) query:
//
//   * flatten_by_samples (src/gpu/gpu_api.cpp:253-287): uint64 words laid out
//     [K][W][warpPad(N)] -- sample index fastest, bins padded to a multiple of
//     32 samples; bin_stride = warpPad(N), kmer_stride = bin_stride * W,
//     sample_stride = 1;
//   * DeviceMemory (src/gpu/device_memory.cu:6-61): sketches, random table,
//     cluster lookup, k-mer list and the [core(n) | acc(n)] output on device;
//   * dispatchDists (src/gpu/dist.cu:408-470): L1-preferring cache config,
//     block shape from the reference's getBlockSize (src/gpu/dist.cu:327-347),
//     dynamic shared memory = sketchsize64 * bbits * 8 bytes, use_shared when
//     that fits the 48 KB default, dist_col = -1, max_diagonal = false;
//   * query_db_cuda's reshape (src/gpu/gpu_api.cpp:477-493) of the column-major
//     result into row-major (n_pairs, 2).
//
// The random-match table is K floats with strides {1, 0, 0} (one cluster),
// which covers NoAdjust (all zero) and a single-cluster table.  The progress
// words live in device memory and the kill flag stays false.
#include <cstdint>
#include <cstdio>
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
  void *p[7] = {};
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

// All-vs-all distances of n samples with the reference kernel.
//   words     host [n][K][sketchsize64 * bbits] uint64, the reference layout
//   random_k  host [K] random-match chance per k (null = NoAdjust)
//   out       host [n(n-1)/2][2] float32 (core, accessory), or null
//   ms        per timed launch, mean (CUDA events on the launch stream)
// Requires n(n-1)/2 >= 1000: the kernel's progress update divides the pair
// index by n_pairs / 1000.  Returns 0, or 1 with a message in err.
int refgpu_self_dists(const uint64_t *words, int64_t n, const int32_t *kmers, int K,
                      int sketchsize64, int bbits, const float *random_k, int warmup,
                      int launches, float *out, double *ms, char *err, int errlen) {
  const long long n_pairs = static_cast<long long>(n) * (n - 1) / 2;
  if (n_pairs < 1000 || K < 1 || launches < 0 || warmup < 0) {
    if (err && errlen > 0)
      std::snprintf(err, static_cast<size_t>(errlen), "need >= 1000 pairs and K >= 1");
    return 1;
  }
  const size_t W = static_cast<size_t>(sketchsize64) * bbits;
  const size_t pad = (static_cast<size_t>(n) + 31) / 32 * 32;
  SketchStrides s{};
  s.sample_stride = 1;
  s.bin_stride = pad;
  s.kmer_stride = pad * W;
  s.sketchsize64 = static_cast<size_t>(sketchsize64);
  s.bbits = static_cast<size_t>(bbits);
  std::vector<uint64_t> flat(s.kmer_stride * K, 0);
  for (int k = 0; k < K; ++k)
    for (size_t b = 0; b < W; ++b) {
      uint64_t *dst = flat.data() + k * s.kmer_stride + b * s.bin_stride;
      for (int64_t i = 0; i < n; ++i) dst[i] = words[(static_cast<size_t>(i) * K + k) * W + b];
    }
  std::vector<float> table(K, 0.0f);
  if (random_k)
    for (int k = 0; k < K; ++k) table[k] = random_k[k];
  const RandomStrides rs{1, 0, 0};
  std::vector<int> km(kmers, kmers + K);

  Buffers buf;
  uint64_t *d_ref = nullptr;
  float *d_table = nullptr, *d_dists = nullptr;
  uint16_t *d_lookup = nullptr;
  int *d_kmers = nullptr, *d_done = nullptr;
  bool *d_kill = nullptr;
  cudaError_t e;
#define REFGPU_TRY(call, what)                     \
  if ((e = (call)) != cudaSuccess) return report(err, errlen, what, e)
  REFGPU_TRY(cudaMalloc(&d_ref, flat.size() * 8), "cudaMalloc sketches");
  buf.p[0] = d_ref;
  REFGPU_TRY(cudaMalloc(&d_table, K * sizeof(float)), "cudaMalloc table");
  buf.p[1] = d_table;
  REFGPU_TRY(cudaMalloc(&d_lookup, n * sizeof(uint16_t)), "cudaMalloc lookup");
  buf.p[2] = d_lookup;
  REFGPU_TRY(cudaMalloc(&d_kmers, K * sizeof(int)), "cudaMalloc kmers");
  buf.p[3] = d_kmers;
  REFGPU_TRY(cudaMalloc(&d_dists, 2 * n_pairs * sizeof(float)), "cudaMalloc dists");
  buf.p[4] = d_dists;
  REFGPU_TRY(cudaMalloc(&d_done, sizeof(int)), "cudaMalloc progress");
  buf.p[5] = d_done;
  REFGPU_TRY(cudaMalloc(&d_kill, sizeof(bool)), "cudaMalloc kill flag");
  buf.p[6] = d_kill;
  REFGPU_TRY(cudaMemcpy(d_ref, flat.data(), flat.size() * 8, cudaMemcpyHostToDevice), "copy sketches");
  REFGPU_TRY(cudaMemcpy(d_table, table.data(), K * sizeof(float), cudaMemcpyHostToDevice), "copy table");
  REFGPU_TRY(cudaMemset(d_lookup, 0, n * sizeof(uint16_t)), "memset lookup");
  REFGPU_TRY(cudaMemcpy(d_kmers, km.data(), K * sizeof(int), cudaMemcpyHostToDevice), "copy kmers");
  REFGPU_TRY(cudaMemset(d_dists, 0, 2 * n_pairs * sizeof(float)), "memset dists");
  REFGPU_TRY(cudaMemset(d_done, 0, sizeof(int)), "memset progress");
  REFGPU_TRY(cudaMemset(d_kill, 0, sizeof(bool)), "memset kill flag");
  REFGPU_TRY(cudaFuncSetCacheConfig(calculate_dists, cudaFuncCachePreferL1), "cache config");

  size_t block_size = 0, block_count = 0;
  std::tie(block_size, block_count) =
      getBlockSize(static_cast<size_t>(n), static_cast<size_t>(n), n_pairs, true);
  const size_t shared = W * sizeof(uint64_t);
  const bool use_shared = shared <= 48 * 1024;
  progress_ptrs prog{d_done, d_kill};

  cudaEvent_t t0, t1;
  REFGPU_TRY(cudaEventCreate(&t0), "event");
  REFGPU_TRY(cudaEventCreate(&t1), "event");
  double total = 0.0;
  for (int it = 0; it < warmup + launches; ++it) {
    REFGPU_TRY(cudaEventRecord(t0, 0), "event record");
    calculate_dists<<<static_cast<unsigned>(block_count), static_cast<unsigned>(block_size),
                      use_shared ? shared : 0>>>(
        true, d_ref, static_cast<long>(n), d_ref, static_cast<long>(n), d_kmers, K, d_dists,
        n_pairs, d_table, d_lookup, d_lookup, s, s, rs, prog, use_shared, -1, false);
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
#undef REFGPU_TRY
  return 0;
}

}  // extern "C"
