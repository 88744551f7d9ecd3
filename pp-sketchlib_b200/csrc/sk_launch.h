// sk_launch.h -- host-side declarations of the kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "sk_common.h"

namespace sk {

// One compiled instance of the tiled distance kernel.
struct TileConfig {
  int id;
  int tile_rows, tile_cols;      // CTA tile (rows x cols of pairs)
  int thread_rows, thread_cols;  // per-thread register block
  int max_kmers;                 // largest K the instance handles
  int stages;                    // pipeline depth
  int threads;
  int smem_bytes;
  cudaError_t (*launch)(const LaunchParams &, int grid, cudaStream_t);
  int (*blocks_per_sm)();        // resident CTAs per SM at this shape's shared memory
};

int tile_config_count();
const TileConfig *tile_config(int id);
// The 64 x 64 shape (8 x 4 pairs per thread, three CTAs per SM) used for
// query batches of at most 64 samples.
constexpr int kSmallQueryConfig = 6;
// Bytes of count scratch per slot (one per CTA, one per split tile).
inline size_t count_slot_bytes(const TileConfig &cfg, int k_slots) {
  return static_cast<size_t>(k_slots) * cfg.tile_rows * cfg.tile_cols * 2;
}


// aux_kernels.cu
cudaError_t launch_pack(const uint64_t *words, int64_t n, int32_t n_kmers, int32_t s64,
                        int32_t ng, uint32_t *packed, cudaStream_t stream);
// Packs n samples (reference layout at `words`) into granules g0 .. g0+ng-1 of
// a packed array of ng_total granules.
cudaError_t launch_pack_range(const uint64_t *words, int64_t n, int32_t n_kmers, int32_t s64,
                              int32_t ng, int32_t g0, int32_t ng_total, uint32_t *packed,
                              cudaStream_t stream);
cudaError_t launch_unpack(const uint32_t *packed, int64_t n, int32_t n_kmers, int32_t s64,
                          int32_t ng, uint64_t *words, cudaStream_t stream);
cudaError_t launch_synth(const int32_t *parent, const uint32_t *thresh, int64_t n,
                         int32_t n_kmers, int32_t s64, uint64_t seed, uint64_t *words,
                         cudaStream_t stream);
// kNN lists of at most kKnnListMax entries are kept per lane in shared memory
// (the condensed self column and dense rows); longer ones only over dense
// rows, by radix select and a bitonic sort per row.
constexpr int kKnnListMax = 800;
cudaError_t launch_knn_self(const float *col_vals, int64_t n, int32_t knn, int32_t jaccard,
                            int64_t *j_out, float *d_out, cudaStream_t stream);
cudaError_t launch_knn_rows(const float *vals, int64_t n_rows, int64_t n_cols, int32_t knn,
                            int64_t diag0, int32_t jaccard, int64_t *j_out, float *d_out,
                            cudaStream_t stream);
// Jaccard / log-Jaccard by intersection count 0 .. n-1 for jobs without
// random-match correction (JobParams::jtab / ltab).
cudaError_t launch_count_tables(double union_bits, int64_t n, float *jtab, double *ltab,
                                cudaStream_t stream);
cudaError_t launch_threshold_count(const float *vals, int64_t n, int32_t stride, int32_t col,
                                   float cutoff, int64_t *row_counts, cudaStream_t stream);
cudaError_t launch_threshold_fill(const float *vals, int64_t n, int32_t stride, int32_t col,
                                  float cutoff, const int64_t *row_offsets, int64_t *i_out,
                                  int64_t *j_out, float *d_out, cudaStream_t stream);
cudaError_t exclusive_scan_i64(const int64_t *in, int64_t *out, int64_t n, void *tmp,
                               size_t *tmp_bytes, cudaStream_t stream);
cudaError_t launch_long_to_square(const float *rr, int64_t n_rr, const float *qr,
                                  const float *qq, int64_t n_qq, float *square,
                                  cudaStream_t stream);
cudaError_t launch_square_to_long(const float *square, int64_t n, float *long_out,
                                  cudaStream_t stream);

}  // namespace sk
