// sk_runtime.h -- host-side state behind the opaque C ABI handles.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "sk_common.h"
#include "sk_launch.h"
#include "sketchlib_b200.h"

struct Scratch {
  void *ptr = nullptr;
  size_t bytes = 0;
};

// Context scratch slots (each a growable device buffer).
enum ScratchSlot : int {
  kSlotCounts = 0,        // per-CTA tile counts of the distance kernel
  kSlotOut = 1,           // dense result staging
  kSlotResult = 2,        // kNN / threshold results
  kSlotTemp = 3,          // temporaries (scan storage, unpacking, probes)
  kSlotSplitCounts = 4,   // counts of tiles split along k
  kSlotLaunchMeta = 5,    // job table, work list, control block
  kSlotStaging = 6,       // sketch words in the reference layout on their way in
  kSlotPackedRef = 7,     // packed arrays of the databases of one sk_query_db call
  kSlotPackedQuery = 8,
  kSlotCountsB = 9,       // count scratch of launches on the second compute stream
  kSlotSplitCountsB = 10,
  kSlotSketchCodes = 11,  // bases of one sketching batch, rewritten as base codes
  kSlotSketchSeqs = 12,   // sequence offsets of the batch
  kSlotSketchItems = 13,  // sketching work items
  kSlotSketchTables = 14, // rolling-hash tables per k
  kSlotSketchBins = 15,   // bin minima per (sample, k)
  kSlotSketchWords = 16,  // finished sketches, inverse minhashes, densify flags
  kSlotSketchTable = 17,  // k-mer count table of read sets
  kSlotCount = 18
};

struct sk_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  cudaStream_t copy_stream = nullptr;   // copies overlapped with kernels (created on first use)
  cudaEvent_t ev_ready[2] = {};         // double buffer b holds data
  cudaEvent_t ev_free[2] = {};          // double buffer b may be overwritten
  cudaStream_t stream_b = nullptr;      // second compute stream (chunk launches alternate)
  cudaStream_t pack_stream = nullptr;   // high-priority stream for packing uploaded chunks
  std::vector<cudaEvent_t> ev_chunk;    // chunk c packed
  cudaStream_t d2h_stream = nullptr;    // result rows copied back while later chunks compute
  std::vector<cudaEvent_t> ev_out;      // chunk c's output rows written
  cudaEvent_t ev_join = nullptr;        // second compute stream done
  int64_t mem_limit = 0;                // bytes a dense call may stage output in (0 = free memory)
  int sm_count = 0;
  std::string err;
  int *cancel_host = nullptr;   // mapped pinned word polled by the kernels
  int *cancel_dev = nullptr;
  sk::DevStatus *status_dev = nullptr;
  unsigned long long last_tiles = 0;
  int tile_cfg = 0;                               // forced tile shape (0 = automatic)
  int semantics = 0;                              // sk::Semantics of later calls
  std::map<std::pair<int, int>, int> tuning;      // (K, s64) -> shape id
  Scratch scratch[kSlotCount];                    // reusable device buffers
  void *noalloc_scratch = nullptr;                // device address of the static no-alloc buffer
  // Jaccard / log-Jaccard tables by count of uncorrected jobs, per union size
  // (64 * sketchsize64); allocated on first use, freed with the context
  std::map<int64_t, std::pair<float *, double *>> count_tables;
  std::mutex count_tables_mu;
  std::recursive_mutex mu;
  // Databases and random models keep their context alive: sk_ctx_destroy only
  // marks it, the last dependent handle to go frees it.
  int refs = 1;
  bool destroyed = false;
};

struct sk_db {
  sk_ctx *ctx = nullptr;
  int64_t n = 0;
  int32_t K = 0, s64 = 0, bbits = 0;
  std::vector<int32_t> kmers;
  int32_t ng = 0;                 // granules in the packed array (padded samples / 64)
  uint32_t *packed = nullptr;     // [K][2*s64][ng][14][64]
  bool own_packed = true;         // false: the array is context scratch
  uint16_t *cluster = nullptr;    // [ng*64] random-match cluster ids
  int32_t max_cluster = 0;        // the largest of them
  std::vector<uint64_t> seq_len;  // per-sample sequence lengths
  double *jv = nullptr;           // [K][ng*64] equal-base factors
  int jv_rc = -1;
  float *jgpu = nullptr;          // [K] equal-base chances of the reference GPU path
  int jgpu_rc = -1;
};

struct sk_random {
  sk_ctx *ctx = nullptr;
  int mode = 0;
  int use_rc = 1;
  std::vector<int32_t> kmers;
  int n_clusters = 0;
  float *table = nullptr;         // [K][C][C]
  std::vector<float> centroids;   // [C][4] base-composition centroids (may be empty)
};

struct sk_sparse {
  std::vector<int64_t> i, j;
  std::vector<float> d;
};

namespace sk {

// A launch of the persistent distance kernel: tile shape, grid and work list.
struct Plan {
  const TileConfig *cfg = nullptr;
  int grid = 0;
  std::vector<WorkItem> items;
  int32_t n_splits = 0;
  int32_t k_slots = 1;
};

// Byte layout of a launch's meta buffer: job table at 0, then the work list
// and the control block (queue counter, split arrival counters), 256-aligned.
struct MetaLayout {
  size_t items_off = 0, ctrl_off = 0, ctrl_bytes = 0, bytes = 0;
};
MetaLayout meta_layout(size_t n_jobs, size_t n_items, int32_t n_splits, int threads);

struct LaunchBuffers {
  void *meta = nullptr, *cta = nullptr, *split = nullptr;
  void *ctrl = nullptr;
  size_t ctrl_bytes = 0;
  LaunchParams lp{};
};

class DeviceGuard {
 public:
  explicit DeviceGuard(int dev);
  ~DeviceGuard();
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;

 private:
  int prev_ = 0;
};

sk_status fail(sk_ctx *ctx, sk_status st, const char *fmt, ...);
void ctx_retain(sk_ctx *ctx);
void ctx_release(sk_ctx *ctx);
sk_status cuda_fail(sk_ctx *ctx, cudaError_t e, const char *what);
sk_status scratch(sk_ctx *ctx, int slot, size_t bytes, void **out);
sk_status begin_call(sk_ctx *ctx);
sk_status finish_call(sk_ctx *ctx);
const TileConfig *choose_config(sk_ctx *ctx, int K, int s64);
void plan_tiles(JobParams &jp, const TileConfig &cfg);
sk_status build_job(sk_ctx *ctx, const sk_db *ref, const sk_db *query, const sk_random *random,
                    int out_mode, int out_col, void *d_out, const TileConfig **cfg_out,
                    JobParams *jp);
sk_status launch_job(sk_ctx *ctx, const JobParams &jp, const TileConfig &cfg);
// Points a job without random-match correction at the context's Jaccard /
// log-Jaccard tables by count for its union size, built on first use (one
// allocation and a small kernel, then a wait on the context stream); alloc
// false: only tables that already exist are used.  Corrected jobs, the
// reference GPU semantics, count output and sketches counted in chunks are
// left as they are (their epilogue computes per pair): per-entry tables for
// a Monte Carlo table measured no faster (20.69 against 20.71 ms at 4,096
// samples).
sk_status attach_count_tables(sk_ctx *ctx, JobParams *jp, bool alloc = true);
void plan_items(const std::vector<JobParams> &jobs, int grid, Plan &plan);
void split_tail(std::vector<WorkItem> &items, size_t begin, int grid, int32_t *n_splits,
                const std::vector<JobParams> *jobs = nullptr);
int32_t items_slots(const std::vector<WorkItem> &items, int32_t base);
int32_t tail_block_parts(const JobParams &jp);
sk_status db_alloc(sk_ctx *ctx, int64_t n, const int32_t *kmers, int32_t K, int32_t s64,
                   int32_t bbits, sk_db **out, int packed_slot = -1);
void db_free(sk_db *db);
sk_status make_plan(sk_ctx *ctx, const std::vector<JobParams> &jobs, const TileConfig &cfg,
                    Plan &plan);
sk_status upload_plan(sk_ctx *ctx, const std::vector<JobParams> &jobs, Plan &plan,
                      LaunchBuffers &buf, bool owned);
sk_status enqueue_plan(sk_ctx *ctx, const Plan &plan, const LaunchBuffers &buf);
int resident_grid(sk_ctx *ctx, const TileConfig &cfg);
sk_status dense_to_device(sk_ctx *ctx, const sk_db *ref, const sk_db *query,
                          const sk_random *random, int out_mode, int out_col, void *d_out);
int64_t n_pairs(const sk_db *ref, const sk_db *query);
sk_status ensure_jv(sk_ctx *ctx, sk_db *db, int use_rc);
std::vector<double> equal_base_factors(const sk_db *db, int use_rc);
std::vector<float> equal_base_gpu(const sk_db *db, int use_rc);
sk_status ensure_copy_stream(sk_ctx *ctx);
size_t dense_budget(sk_ctx *ctx);
sk_status dense_blocked_to_host(sk_ctx *ctx, const sk_db *ref, const sk_db *query,
                                const sk_random *random, int out_mode, void *out, size_t budget);
size_t out_bytes(int out_mode, int64_t pairs, int K);

}  // namespace sk
