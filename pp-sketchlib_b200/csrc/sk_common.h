// sk_common.h -- types shared by the host runtime and the device kernels.
//
// Packed device layout of a sketch database ("stripes"):
//   uint32 words[n_kmers][nb][n_granules][kBbits][kGranule]
// with nb = 2 * sketchsize64 32-bin blocks, kGranule = 64 samples per granule.
// Element (k, b, g, plane, lane) is bit-plane `plane` of bins 32*b .. 32*b+31 of
// sample g*64+lane at k-mer index k: the low (b even) or high (b odd) half of
// reference word (b/2)*bbits + plane (src/sketch/sketch.cpp:82-92).  One
// (k, b, g) stripe is 14*64*4 = 3584 contiguous bytes, so a tile of samples for
// one block is a single bulk copy, and the 64 samples of a plane are one
// 256-byte row read with 128-bit shared-memory loads.
#pragma once

#include <cstddef>
#include <cstdint>

namespace sk {

constexpr int kBbits = 14;              // def_bbits (src/reference.hpp:18)
constexpr int kGranule = 64;            // samples per packed granule
constexpr int kStripeWords = kBbits * kGranule;       // 896 uint32
constexpr int kStripeBytes = kStripeWords * 4;        // 3584 bytes
constexpr int kSamplePad = 256;         // databases are padded to this many samples
constexpr int kMaxKmers = 128;          // k-mer lengths per database
constexpr int kNarrowKmers = 32;        // k-mer lengths the narrow kernel instance finishes
constexpr int kMaxKmerLength = 255;     // longest k (the sketcher's limit)
constexpr int kMaxSketch64 = 1 << 16;   // sketchsize64 accepted (4.2 M bins per k)
// 32-bin blocks of one k whose bin matches fit a uint16 tile counter
// (2046 * 32 = 65,472): a k with more blocks is counted in chunks of this
// many blocks, each in its own count slot, summed by the epilogue.
constexpr int kMaxChunkBlocks = 2046;

// Output modes (public values in sketchlib_b200.h) plus internal single-column modes.
enum OutMode : int {
  kOutCoreAcc = 0,   // float2 per pair
  kOutJaccard = 1,   // float[K] per pair
  kOutCounts = 2,    // uint32[K] per pair
  kOutColumn = 3     // float per pair: core (col 0) / accessory (col 1)
};
enum RandMode : int { kRandNone = 0, kRandEqualBase = 1, kRandTable = 2 };
enum Semantics : int { kSemRefCpu = 0, kSemRefGpu = 1 };

// Device-side status word of a context.  error != 0 makes the host call fail.
struct DevStatus {
  unsigned int error;      // bit 0: bounded wait timed out, bit 1: cancelled
  unsigned int where;      // last site that raised an error
  unsigned long long tiles_done;
};

// Everything one distance launch (one job) needs.  Rows are the "this"/query
// side of a pair, columns the reference side; for all-vs-all both are the
// same database and only pairs with col > row are produced.
struct JobParams {
  const uint32_t *row_words;   // packed stripes of the row database
  const uint32_t *col_words;   // packed stripes of the column database
  int64_t n_rows, n_cols;      // real sample counts
  int32_t ng_rows, ng_cols;    // granules in each packed array
  int32_t n_kmers;             // K
  int32_t nb;                  // 2 * sketchsize64
  int32_t nchunk;              // count slots per k: ceil(nb / kMaxChunkBlocks)
  int32_t chunk_nb;            // blocks per count slot (even; the last may hold fewer)
  int32_t self;                // 1: all-vs-all upper triangle
  int32_t out_mode;            // OutMode
  int32_t out_col;             // column for kOutColumn
  int32_t tile_rows, tile_cols;  // CTA tile (must match the kernel instance)
  int64_t n_tiles;
  int32_t n_row_tiles, n_col_tiles;
  void *out;                   // device output
  int64_t out_row0;            // long-form row held by out[0] (0 unless the output is blocked)
  double tol;                  // 5 / (64 * s64) (src/dist/linear_regression.cpp:22)
  double union_bits;           // 64 * s64 (src/reference.cpp:91)
  // Jobs without random-match correction: the Jaccard and its logarithm by
  // intersection count 0 .. union_bits, shared by every pair of the sketch
  // width (null: the epilogue computes them per pair)
  const float *jtab;
  const double *ltab;
  // random-match correction
  int32_t rmode;
  const float *rtable;         // kRandTable: [K][C][C]
  int32_t rs_k, rs_row, rs_col;  // strides into rtable for (k, row cluster, col cluster)
  const uint16_t *cl_rows, *cl_cols;   // per-sample cluster ids (may be null)
  const double *jv_rows, *jv_cols;     // kRandEqualBase: [K][n_pad] 1-(1-4^-k')^len
  int64_t jv_rows_ld, jv_cols_ld;      // leading dimension (padded samples)
  int32_t kmers[kMaxKmers];
  uint32_t one;                // 1 (a run-time operand for the count multiply-adds)
  int32_t semantics;           // Semantics: which reference path the fit follows
  // Rows that are a block of the column database itself (blocked self kNN):
  // row r is sample row_base + r, and a random-table lookup orders the pair's
  // clusters by sample index as the all-vs-all path does.
  int32_t self_view;
  int64_t row_base;
};

// Count slots one job's tile needs: one per (k, chunk of blocks).
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int32_t job_slots(const JobParams &jp) { return jp.n_kmers * jp.nchunk; }

// Jobs the wide kernel instance must run: more k-mer lengths than the narrow
// instance finishes, or sketches counted in chunks.
#if defined(__CUDACC__)
__host__ __device__
#endif
inline bool needs_wide(const JobParams &jp) { return jp.n_kmers > kNarrowKmers || jp.nchunk > 1; }

// One unit of work of the persistent distance kernel: k-mer indices
// [k0, k1) of one tile of one job.  A tile whose k range is cut into several
// items (the last wave's tiles, to even out the tail) shares a split slot; the
// item that finishes last runs the tile's epilogue.
struct WorkItem {
  int64_t tile;     // tile index within the job
  int32_t job;
  int16_t k0, k1;
  int32_t split;    // split slot, -1 for a whole tile
  int32_t nparts;   // items sharing the split slot
  int32_t b0, b1;   // 32-bin blocks [b0, b1) of each k; b1 == 0: all of them
  int16_t bpart, nbpart;  // block range index, ranges per k (0: one)
  int32_t pad;
};

// Everything one launch needs: the job table, the work list and the scratch.
struct LaunchParams {
  const JobParams *jobs;
  const WorkItem *items;
  int64_t n_items;
  unsigned long long *item_counter;   // zeroed before each launch
  unsigned int *split_done;           // [n_splits][threads], zeroed before each launch
  uint16_t *cta_scratch;              // [grid][k_slots][threads][pairs per thread]
  uint16_t *split_scratch;            // [n_splits][k_slots][threads][pairs per thread]
  int32_t k_slots;                    // largest K x nchunk over the jobs
  int32_t wide;                       // 1: some job needs the wide kernel instance
  DevStatus *status;
  const volatile int *cancel;
};

// splitmix64 finaliser: the counter-based hash of the synthetic generator.
// Identical on host and device (pure integer arithmetic).
#if defined(__CUDACC__)
__host__ __device__
#endif
inline uint64_t synth_mix(uint64_t x) {
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ULL;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBULL;
  x ^= x >> 31;
  return x;
}

// 14-bit bin value of sample s at k-mer index k, bin `bin`.  A sample copies
// its parent's bin unless the hash's high word falls below thresh[s][k]
// (probability 1-(1-c)^k(1-a) for its branch), in which case it draws a fresh
// uniform value; roots always draw.  Walking up the lineage makes every bin
// independent of the order samples are generated in.
#if defined(__CUDACC__)
__host__ __device__
#endif
inline uint32_t synth_bin(const int32_t *parent, const uint32_t *thresh,
                          int32_t n_kmers, int64_t s, int32_t k, uint32_t bin,
                          uint64_t seed) {
  int64_t node = s;
  for (;;) {
    uint64_t h = synth_mix(seed ^ (static_cast<uint64_t>(node) * 0x9E3779B97F4A7C15ULL) ^
                           ((static_cast<uint64_t>(k) << 32 | bin) * 0xC2B2AE3D27D4EB4FULL));
    int32_t par = parent[node];
    if (par < 0 || static_cast<uint32_t>(h >> 32) < thresh[node * n_kmers + k]) {
      return static_cast<uint32_t>(h) & ((1u << kBbits) - 1u);
    }
    node = par;
  }
}

}  // namespace sk
