/*
 * sketchlib_b200.h -- C ABI of the B200 core/accessory distance library.
 *
 * This is the drop-in boundary for pp-sketchlib's GPU distance path.  Every
 * entry point takes plain pointers and sizes; nothing here names a CUDA,
 * torch or C++ type, so the library can be bound from C, ctypes, cgo or a
 * pybind11 module alike.  No entry point throws: each returns an sk_status and
 * leaves a message readable through sk_last_error().
 *
 * Sketch words are passed in the reference's own word layout: for sample s and
 * k-mer index ki, sketchsize64 * bbits uint64 words, where word
 * (blk * bbits + plane) holds bit `plane` of the 64 bins 64*blk .. 64*blk+63
 * (bin i of the block is bit i of the word).  The host buffer is
 * [n_samples][n_kmers][sketchsize64 * bbits], which is what
 * Reference::get_sketch (src/reference.cpp:143-150) hands out per k, laid end to
 * end per sample; src/sketch/sketch.cpp:82-92 (fillusigs) writes this layout.
 *
 * Reference interfaces replaced (paths are within bacpop/pp-sketchlib):
 *   sk_db_create            <- flatten_by_bins / flatten_by_samples + DeviceMemory
 *                              (src/gpu/gpu_api.cpp:232-305, src/gpu/device_memory.cu:7-65)
 *   sk_random_create        <- RandomMC::flattened_random / lookup_array / csrs
 *                              (src/random/random_match.cpp:254-310, 318-336)
 *   sk_closest_cluster      <- RandomMC::closest_cluster / nearest_neighbour / apply_rc
 *                              (src/random/random_match.cpp:222-227, 338-360)
 *   sk_dists_dense          <- query_db_cuda / dispatchDists / calculate_dists
 *                              (src/gpu/gpu_api.cpp:352-494, src/gpu/dist.cu:164-317, 408-489)
 *                              and, for SK_OUT_JACCARD, the CPU-only jaccard branch of
 *                              query_db (src/api.cpp:206-211, 256-260)
 *   sk_query_db             <- query_db_cuda as one host-in / host-out call
 *                              (src/gpu/gpu_api.cpp:352-494)
 *   sk_dists_knn            <- query_db_sparse_cuda / sparseDists
 *                              (src/gpu/gpu_api.cpp:496-531, src/gpu/dist.cu:495-791) and
 *                              query_db_sparse (src/api.cpp:332-432)
 *   sk_sparse_threshold     <- sparsify_dists_by_threshold (src/dist/matrix_ops.cpp:38-69)
 *   sk_long_to_square       <- long_to_square (src/dist/matrix_ops.cpp:71-126)
 *   sk_square_to_long       <- square_to_long (src/dist/matrix_ops.cpp:130-150)
 *   sk_cancel               <- progress_atomics::set_kill (src/gpu/cuda.cuh:41-87),
 *                              without the reference's __trap()
 *   sk_sketch               <- sketch() per sample and k (src/sketch/sketch.cpp:120-168)
 *                              and its GPU counterpart sketch_gpu / get_signs
 *                              (src/sketch/sketch.cpp:170-205, src/gpu/sketch.cu:404-470)
 */
#ifndef SKETCHLIB_B200_H
#define SKETCHLIB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SK_ABI_VERSION 1

typedef enum sk_status {
  SK_OK = 0,
  SK_EINVAL = 1,      /* bad argument; the reference throws std::runtime_error */
  SK_ENOMEM = 2,      /* device or pinned-host allocation failed */
  SK_ECUDA = 3,       /* CUDA runtime error (the reference's CUDA_CALL throw) */
  SK_EMISMATCH = 4,   /* bbits / sketchsize64 / k-mer lists differ between sketches */
  SK_ECANCELLED = 5,  /* sk_cancel() was observed by the running kernels */
  SK_ETIMEDOUT = 6,   /* a bounded wait (host or device) ran out */
  SK_ENOTSUP = 7,     /* a parameter value this build does not implement */
  SK_EKERNEL = 8,     /* a kernel raised its device-side error flag */
  SK_ERANGE = 9       /* a size beyond a stated maximum */
} sk_status;

typedef struct sk_ctx sk_ctx;       /* one device + one stream + error state */
typedef struct sk_db sk_db;         /* sketches resident in HBM, packed layout */
typedef struct sk_random sk_random; /* random-match correction model */
typedef struct sk_sparse sk_sparse; /* variable-length sparse (i, j, d) result */

/* Random-match correction modes (RandomType, src/random/random_match.hpp:25). */
enum {
  SK_RANDOM_NONE = 0,       /* RandomType::NoAdjust: r = 0 */
  SK_RANDOM_EQUAL_BASE = 1, /* RandomType::EqualBase: r = csrs(k, use_rc, len_a, len_b) */
  SK_RANDOM_TABLE = 2       /* RandomType::MonteCarlo: r = table[k][cluster_ref][cluster_query] */
};

/* Dense output modes. */
enum {
  SK_OUT_CORE_ACC = 0, /* float32 (n_pairs, 2) row-major: core, accessory */
  SK_OUT_JACCARD = 1,  /* float32 (n_pairs, n_kmers) row-major: corrected Jaccard */
  SK_OUT_COUNTS = 2    /* uint32 (n_pairs, n_kmers) row-major: raw intersection counts */
};

/* Which of the reference's two distance paths the core/accessory output
 * reproduces (the reference's CPU and GPU paths disagree, see
 * sk_ctx_set_semantics). */
enum {
  SK_SEMANTICS_REFERENCE_CPU = 0, /* query_db + fit_slope (default) */
  SK_SEMANTICS_REFERENCE_GPU = 1  /* calculate_dists, bit for bit */
};

/* ---- library / context ------------------------------------------------- */

int32_t sk_abi_version(void);

/* Binds a context to device_id (cudaSetDevice, src/gpu/dist.cu:373-384) and
 * creates its own non-blocking stream. */
sk_status sk_ctx_create(int32_t device_id, sk_ctx **out);
/* Releases the caller's handle.  Databases and random models created on the
 * context keep it alive; its device resources go with the last of them. */
sk_status sk_ctx_destroy(sk_ctx *ctx);
/* Last error message of this context ("" if none).  Valid until the next call. */
const char *sk_last_error(const sk_ctx *ctx);
/* Runs all of this context's work on `stream` (a cudaStream_t) instead of its own. */
sk_status sk_ctx_set_stream(sk_ctx *ctx, void *stream);
/* Asks running kernels of this context to stop at their next tile boundary;
 * the interrupted call returns SK_ECANCELLED.  Cleared when a call starts. */
sk_status sk_cancel(sk_ctx *ctx);
sk_status sk_device_info(sk_ctx *ctx, int64_t *mem_free, int64_t *mem_total,
                         int32_t *sm_count);
/* Waits for all work queued on the context's stream (calls made with
 * out_on_device = 1 return before their kernels finish) and reports any
 * device-side error or cancellation they raised. */
sk_status sk_ctx_synchronize(sk_ctx *ctx);
/* Chooses the dense kernel's tile shape (0 = automatic, from the tuning table
 * or the built-in default; >0 = a shape id from sk_tile_config_count()). */
sk_status sk_ctx_set_tile_config(sk_ctx *ctx, int32_t config_id);
/* Selects the arithmetic of the core/accessory fit for this context's later
 * calls.  SK_SEMANTICS_REFERENCE_CPU (default): the reference CPU path
 * (src/api.cpp:195-283, src/dist/linear_regression.cpp:16-60): Jaccard in
 * double, fit over the k range from the first to the last Jaccard above
 * 5 / (64 * sketchsize64), least squares in double, random table read as
 * [k][cluster of row i][cluster of column j] for all-vs-all and 0 from k = max_k
 * on (the table passed in decides that).  SK_SEMANTICS_REFERENCE_GPU: the
 * reference GPU kernel's float arithmetic (calculate_dists, src/gpu/dist.cu:
 * 164-317): Jaccard count / (64 * sketchsize64) rounded up, float
 * observed_excess, the fit stops at the first k below tolerance, running
 * float sums, correlation-form slope with round-up intrinsics, __logf /
 * __expf; random table read as [k][cluster of the column (reference)
 * sample][cluster of the row (query) sample]; SK_RANDOM_EQUAL_BASE uses the
 * first reference sample's length for every pair (src/gpu/gpu_api.cpp:402-403).
 * Jaccard and count outputs are the same under both. */
sk_status sk_ctx_set_semantics(sk_ctx *ctx, int32_t semantics);
/* Device memory, in bytes, a dense call returning to the host may use for its
 * output (0 = the free memory less 2 GiB, the default).  A larger output is
 * computed in blocks of rows that are copied back while the next block
 * computes, as the reference splits an all-vs-all that exceeds device memory
 * into chunks (query_db_cuda, src/gpu/gpu_api.cpp:357-389); query-vs-reference
 * outputs are blocked the same way (the reference refuses them).  The same
 * limit bounds sk_sketch's k-mer counting for read sets: a quarter of it
 * (default: a quarter of the free memory less 2 GiB) holds a sample's hashes
 * grouped by range (8 bytes per base); a sample larger than that is counted
 * in a global table, in passes over bin ranges when the table would exceed
 * the quarter. */
sk_status sk_ctx_set_memory_limit(sk_ctx *ctx, int64_t bytes);
int32_t sk_tile_config_count(void);
/* Describes shape `config_id`: rows x cols of the CTA tile and per-thread block. */
sk_status sk_tile_config_info(int32_t config_id, int32_t *tile_rows,
                              int32_t *tile_cols, int32_t *thread_rows,
                              int32_t *thread_cols, int32_t *max_kmers);
/* Loads a tuning table written by the autotuner: lines "n_kmers sketchsize64 config_id". */
sk_status sk_ctx_load_tuning(sk_ctx *ctx, const char *path);

/* ---- sketch databases --------------------------------------------------- */

/* Uploads sketches from HOST memory in the reference word layout (see top of
 * file) and packs them on the device.  kmers: the n_kmers k-mer lengths, in
 * the order the words are stored (ascending in the reference).  bbits must
 * be 14 (def_bbits, src/reference.hpp:18). */
sk_status sk_db_create(sk_ctx *ctx, const uint64_t *words, int64_t n_samples,
                       const int32_t *kmers, int32_t n_kmers,
                       int32_t sketchsize64, int32_t bbits, sk_db **out);
/* Same, with `d_words` already in this context's device memory. */
sk_status sk_db_create_device(sk_ctx *ctx, const uint64_t *d_words,
                              int64_t n_samples, const int32_t *kmers,
                              int32_t n_kmers, int32_t sketchsize64,
                              int32_t bbits, sk_db **out);
sk_status sk_db_destroy(sk_db *db);
sk_status sk_db_info(const sk_db *db, int64_t *n_samples, int32_t *n_kmers,
                     int32_t *sketchsize64, int32_t *bbits);
/* Per-sample random-match inputs: cluster ids (RandomMC::lookup_array,
 * src/random/random_match.cpp:254-273) and sequence lengths
 * (Reference::seq_length).  Either may be NULL (all zero). */
sk_status sk_db_set_sample_info(sk_db *db, const uint16_t *cluster,
                                const uint64_t *seq_len);
/* Copies the packed device layout back out in the reference word layout
 * (host buffer of n_samples * n_kmers * sketchsize64 * bbits words). */
sk_status sk_db_download(sk_ctx *ctx, const sk_db *db, uint64_t *words);

/* ---- random-match model ------------------------------------------------- */

/* mode SK_RANDOM_TABLE: `table` is float [n_kmers][n_clusters][n_clusters],
 *   indexed [k][cluster of the reference-side sample][cluster of the
 *   query-side sample] (RandomMC::random_match, random_match.cpp:185-206); the
 *   caller writes 0 for k >= max_k as the reference CPU path does.
 * mode SK_RANDOM_EQUAL_BASE: per-pair csrs(k, use_rc, len_a, len_b)
 *   (random_match.cpp:318-336) from the databases' seq_len.
 * mode SK_RANDOM_NONE: no correction.  `kmers` must equal the databases'. */
sk_status sk_random_create(sk_ctx *ctx, int32_t mode, int32_t use_rc,
                           const int32_t *kmers, int32_t n_kmers,
                           int32_t n_clusters, const float *table,
                           sk_random **out);
sk_status sk_random_destroy(sk_random *random);

/* Random-match cluster of each of n samples from its base composition, for
 * queries that are not in the model's cluster table (RandomMC::closest_cluster
 * / nearest_neighbour / apply_rc, src/random/random_match.cpp:222-227,
 * 338-360): with use_rc the A/T and C/G frequencies are averaged, then the
 * nearest of the n_clusters centroids [C][4] (A, C, G, T) by squared distance in
 * float is chosen, the first on a tie (the reference sums the four squares in
 * Eigen's order, so centroids equidistant within float rounding may resolve
 * differently).  base_freq is [n][4] in A, C, G, T order.  Host-only: no
 * context or device.  Feeds `cluster` of sk_db_set_sample_info and
 * sk_server_submit. */
sk_status sk_closest_cluster(const float *centroids, int32_t n_clusters, int32_t use_rc,
                             const double *base_freq, int64_t n, uint16_t *cluster_out);
/* Gives a table model its base-composition centroids [n_clusters][4] (the
 * /random/centroids of a database, Database::load_random,
 * src/database/database.cpp:195-227), from which the query server assigns
 * clusters with sk_closest_cluster under the model's use_rc. */
sk_status sk_random_set_centroids(sk_random *random, const float *centroids,
                                  int32_t n_clusters);

/* ---- dense distances ---------------------------------------------------- */

/* Number of output rows: n*(n-1)/2 when query is NULL (all-vs-all of `ref`),
 * else n_query * n_ref.  Row order follows square_to_condensed
 * (src/dist/matrix_idx.hpp:46-50) for self, q * n_ref + r for query mode
 * (src/api.cpp:251). */
int64_t sk_dists_rows(const sk_db *ref, const sk_db *query);

/* All-vs-all (query == NULL) or query-vs-reference distances.
 * out: host pointer (out_on_device = 0: the call copies the result back and
 * returns after it is complete) or device pointer (out_on_device = 1: the
 * call returns once the kernels are queued on the context's stream).
 * random may be NULL (no correction). */
sk_status sk_dists_dense(sk_ctx *ctx, const sk_db *ref, const sk_db *query,
                         const sk_random *random, int32_t out_mode, void *out,
                         int32_t out_on_device);

/* Host sketches of one side of a query_db call. */
typedef struct sk_host_sketches {
  const uint64_t *words;     /* [n][n_kmers][sketchsize64 * bbits], reference layout */
  int64_t n;                 /* samples */
  const uint16_t *cluster;   /* [n] random-match cluster ids, or NULL */
  const uint64_t *seq_len;   /* [n] sequence lengths, or NULL */
} sk_host_sketches;

/* Host sketches in, host distances out, in one call: the shape of
 * query_db_cuda (src/gpu/gpu_api.cpp:352-494, what queryDatabase(use_gpu=True)
 * runs).  query == NULL: all-vs-all of ref.  The sketch words go up in sample
 * chunks on a second stream; each chunk is packed as it lands and the tiles
 * whose samples have all arrived are computed while the next chunk is in
 * flight, so the host-to-device copy overlaps the distance kernel.  `out` is a
 * host buffer of sk_dists_rows-equivalent rows (n(n-1)/2 or n_query * n_ref)
 * in the layout of out_mode; results are identical to sk_db_create +
 * sk_dists_dense.  Pinned host buffers give the full copy rate; pageable ones
 * work. */
sk_status sk_query_db(sk_ctx *ctx, const sk_host_sketches *ref,
                      const sk_host_sketches *query, const int32_t *kmers,
                      int32_t n_kmers, int32_t sketchsize64, int32_t bbits,
                      const sk_random *random, int32_t out_mode, void *out);

/* sk_query_db for a caller still filling the sketch words (reading them from
 * a file, say) while the call runs: before the call copies samples
 * [s0, s0 + n) of one side (side 0 = ref, 1 = query) it calls
 * ready(user, side, s0, n) on the calling thread, which returns 0 once those
 * words are in place, or nonzero to abandon the call (SK_ETIMEDOUT).  The
 * sample counts, cluster ids and sequence lengths must be complete when the
 * call starts.  Chunks are requested in upload order: an all-vs-all whose
 * output fits the device from the last samples down, otherwise the queries
 * first, then the references from the first up.  No reference counterpart: query_db_cuda
 * starts after every sketch is loaded (src/api.cpp:140-291). */
typedef int (*sk_words_ready_fn)(void *user, int32_t side, int64_t s0, int64_t n);
sk_status sk_query_db_ready(sk_ctx *ctx, const sk_host_sketches *ref,
                            const sk_host_sketches *query, const int32_t *kmers,
                            int32_t n_kmers, int32_t sketchsize64, int32_t bbits,
                            const sk_random *random, int32_t out_mode, void *out,
                            sk_words_ready_fn ready, void *user);

/* Page-locked host memory (cudaHostAlloc, portable) for the sketch words a
 * host program hands to sk_query_db, and its release.  No reference
 * counterpart: query_db_cuda copies from pageable vectors
 * (src/gpu/gpu_api.cpp:232-305), which both halves the copy rate and costs a
 * first-touch page fault per 4 KiB of every freshly allocated buffer; a
 * caller that keeps one such buffer across calls pays neither. */
sk_status sk_host_alloc(int64_t bytes, void **out);
sk_status sk_host_free(void *ptr);

/* Self kNN (querySelfSparse with kNN > 0, src/sketchlib_bindings.cpp:136-187):
 * for every sample i, the kNN smallest distances d(i, j), j != i, of column
 * dist_col (0 = core, 1 = accessory; jaccard != 0 sorts on 1 - J at k-mer
 * index dist_col and reports J).  Outputs have n_samples * kNN entries,
 * ascending per row, ties broken by the smaller j.  Host pointers. */
sk_status sk_dists_knn(sk_ctx *ctx, const sk_db *db, const sk_random *random,
                       int32_t kNN, int32_t dist_col, int32_t jaccard,
                       int64_t *i_out, int64_t *j_out, float *d_out);

/* Query kNN: for each query q, the kNN smallest column-dist_col distances to
 * the references (query-vs-reference rows), ascending, ties by smaller r. */
sk_status sk_query_knn(sk_ctx *ctx, const sk_db *ref, const sk_db *query,
                       const sk_random *random, int32_t kNN, int32_t dist_col,
                       int64_t *r_out, float *d_out);

/* ---- dense distances without device allocation ---------------------------- */

/* Bytes of the static device buffer behind sk_dists_dense_noalloc. */
#define SK_NOALLOC_SCRATCH_BYTES (64u << 20)

/* No counterpart in the reference.  Dense distances (as sk_dists_dense with
 * out_on_device = 1) for callers that cannot allocate device memory at call
 * time: services whose device memory is partitioned once at start-up, and
 * hosts that share the device with an allocator they do not control.  The call
 * makes no cudaMalloc, cudaFree or other allocating call: the kernel's scratch
 * (job descriptor, work list, queue counter, per-CTA count slots, equal-base
 * random-match factors) lives in one static device array of
 * SK_NOALLOC_SCRATCH_BYTES, which every GPU that loads this library holds
 * until the process exits.  The databases (created earlier) are the inputs and
 * `d_out` (caller-allocated device memory, sk_dists_rows(ref, query) rows) the
 * output.  A job whose work list and one count slot do not fit the buffer is
 * rejected with SK_ERANGE; when the count slots of all resident CTAs do not
 * fit, fewer CTAs run.  The first call on each context looks up the buffer's
 * device address (cudaGetSymbolAddress, with the context's device current)
 * and keeps it on the context, so that first call should come before any
 * stream capture; a context created after a device reset looks it up again.
 * Its small uploads (job descriptor, work list, equal-base factors) are
 * copied from host memory owned by the call.  Every call shares the buffer and leaves its contents behind (the
 * work counter is cleared by each call): calls that overlap on the GPU, from
 * different contexts or streams of one device, race; calls queued on one
 * stream do not.  Returns once the work is queued on the context's stream;
 * sk_ctx_synchronize() waits and reports device-side errors. */
sk_status sk_dists_dense_noalloc(sk_ctx *ctx, const sk_db *ref, const sk_db *query,
                                 const sk_random *random, int32_t out_mode, void *d_out);

/* ---- batched persistent launch ------------------------------------------- */

/* One distance job of a batch: all-vs-all of `ref` (query NULL) or query vs
 * ref, written to `out` in DEVICE memory (sk_dists_rows(ref, query) rows of
 * the out_mode's width).  Jobs of one batch may differ in sample counts, k-mer
 * sets and sketch widths. */
typedef struct sk_job {
  const sk_db *ref;
  const sk_db *query;
  const sk_random *random;
  int32_t out_mode;
  void *out;
} sk_job;

typedef struct sk_batch sk_batch;

enum { SK_BATCH_AUTOTUNE = 1 /* time every tile shape on this batch, keep the fastest */ };

/* Plans all jobs as one work list for one persistent kernel launch (longest
 * tiles first, the last wave split along k), and captures the launch in a
 * CUDA graph on the context's stream.  The databases, random models and
 * output buffers must outlive the batch.  No reference counterpart: the
 * reference runs one dispatchDists per job (src/gpu/dist.cu:408-489). */
sk_status sk_batch_create(sk_ctx *ctx, const sk_job *jobs, int32_t n_jobs, int32_t flags,
                          sk_batch **out);
/* Replays the graph and waits for it. */
sk_status sk_batch_run(sk_batch *batch);
/* Replays the graph and returns; sk_ctx_synchronize() waits. */
sk_status sk_batch_launch(sk_batch *batch);
sk_status sk_batch_info(const sk_batch *batch, int32_t *tile_config, int32_t *grid,
                        int64_t *n_items, int64_t *n_pairs);
sk_status sk_batch_destroy(sk_batch *batch);

/* Autotuner: times every tile shape on one job (out_mode core/accessory into
 * scratch), records the fastest for the job's (n_kmers, sketchsize64) class in
 * the context's tuning table and returns it. */
sk_status sk_autotune(sk_ctx *ctx, const sk_db *ref, const sk_db *query,
                      const sk_random *random, int32_t repeats, int32_t *best_config);
/* Writes the context's tuning table ("n_kmers sketchsize64 config_id" lines)
 * for sk_ctx_load_tuning. */
sk_status sk_ctx_save_tuning(sk_ctx *ctx, const char *path);

/* ---- query server: resident references, continuous batching --------------- */

typedef struct sk_server sk_server;

typedef struct sk_server_params {
  int32_t slots;          /* slices on the device at once (one stream each), 1..16 */
  int32_t slice_queries;  /* largest number of queries per slice; a request of at
                             most this many runs as one slice at high priority */
  int32_t kNN;            /* nearest references returned per query, 0..n_refs */
  int32_t dist_col;       /* distance the kNN ranks by: 0 core, 1 accessory */
  int32_t keep_rows;      /* 1: also return each query's core/accessory row */
  int32_t large_slice_queries;  /* slice size for larger requests, 1..slice_queries
                                   (0: slice_queries); smaller slices shorten the wait
                                   of a one-slice request behind a large one */
  int64_t device_bytes;   /* HBM the slots may take (0: no budget, `slots` slots).
                             With a budget the server makes as many slots as fit in
                             it, at most `slots`; a budget below one slot is
                             refused with SK_ENOMEM (sk_server_info reports the
                             bytes one slot holds) */
} sk_server_params;

/* Starts a server over `ref` (kept resident; it must outlive the server).
 * Every slot's buffers and kernel scratch are allocated here, so the HBM
 * footprint is fixed (slots x slot bytes, bounded by device_bytes) and
 * queries are admitted onto the device as slots, i.e. their memory, free up.
 * A slot runs one slice: up to slice_queries queries, which may come from
 * several requests.  Free slots go to the request with the fewest queries left
 * (a request waiting over 2 s first); whole requests of at most slice_queries
 * queries are packed together into one slice on a high-priority stream, and
 * slices of larger requests (large_slice_queries each, the tail of one request
 * packed with the head of the next) hold at most half the slots.  Free rows
 * of a slice's last query tile are filled with queries of larger requests.
 * The context's tile shape, tuning and semantics at this moment apply to
 * every request.  No reference counterpart: the reference answers one
 * query_db_cuda call at a time (src/gpu/gpu_api.cpp:352). */
sk_status sk_server_create(sk_ctx *ctx, const sk_db *ref, const sk_random *random,
                           const sk_server_params *params, sk_server **out);
/* Queues a request: n_queries sketches in the reference word layout (host
 * memory that must stay valid until the request is done), and optional
 * per-query random-match inputs: cluster ids, sequence lengths and base
 * compositions base_freq [n][4] (A, C, G, T).  Under a table random model
 * with centroids (sk_random_set_centroids), queries without cluster ids get
 * the nearest centroid of their base composition, as the reference assigns
 * queries missing from its cluster table (RandomMC::lookup_array /
 * closest_cluster, src/random/random_match.cpp:222-227, 254-273).  Queries
 * with neither get cluster 0 and length 0, as sk_db_set_sample_info with
 * NULL.  Query words in page-locked memory (sk_host_alloc, cudaHostAlloc)
 * go to the device directly; pageable ones are staged by the server first.
 * Thread-safe. */
sk_status sk_server_submit(sk_server *server, const uint64_t *query_words, int64_t n_queries,
                           const uint16_t *cluster, const uint64_t *seq_len,
                           const double *base_freq, int64_t *ticket);
/* Waits for a request (bounded by timeout_s; SK_ETIMEDOUT when it runs out). */
sk_status sk_server_wait(sk_server *server, int64_t ticket, double timeout_s);
/* Copies a finished request's results: knn_idx / knn_dist [n_queries][kNN]
 * (ascending, ties by smaller reference index), rows [n_queries][n_ref][2]
 * when keep_rows; latency_s from submit to completion.  NULL skips a field. */
sk_status sk_server_result(sk_server *server, int64_t ticket, int64_t *knn_idx, float *knn_dist,
                           float *rows, double *latency_s);
/* Forgets a finished request. */
sk_status sk_server_release(sk_server *server, int64_t ticket);
sk_status sk_server_stats(sk_server *server, int64_t *pairs_done, double *uptime_s,
                          int64_t *queued_queries);
/* Slots the server made, HBM one slot holds, and slices run so far with the
 * number of requests they carried (slices_shared: slices holding queries of
 * more than one request). */
sk_status sk_server_info(sk_server *server, int32_t *slots, int64_t *slot_bytes,
                         int64_t *slices, int64_t *slices_shared);
/* Finishes the queued work, stops the scheduler thread and frees the slots. */
sk_status sk_server_destroy(sk_server *server);

/* ---- sparse / matrix transforms (device kernels over long-form data) ---- */

/* Entries (i, j > i) of the square form of a long-form column with value
 * < cutoff, row-major (src/dist/matrix_ops.cpp:38-69).  long_form: float
 * (n_pairs, n_cols) row-major, host memory. */
sk_status sk_sparse_threshold(sk_ctx *ctx, const float *long_form,
                              int64_t n_samples, int32_t n_cols, int32_t col,
                              float cutoff, sk_sparse **out);
/* Threshold sparsification straight from sketches: dense distances stay on
 * the device and only the sparse entries come back. */
sk_status sk_dists_threshold(sk_ctx *ctx, const sk_db *db,
                             const sk_random *random, int32_t dist_col,
                             float cutoff, sk_sparse **out);
int64_t sk_sparse_size(const sk_sparse *sp);
sk_status sk_sparse_copy(const sk_sparse *sp, int64_t *i_out, int64_t *j_out,
                         float *d_out);
sk_status sk_sparse_destroy(sk_sparse *sp);

/* long_to_square (matrix_ops.cpp:71-126): rr has n_rr*(n_rr-1)/2 values,
 * qr n_rr*n_qq (ref index fastest) and qq n_qq*(n_qq-1)/2; qr/qq may be NULL
 * with n_qq = 0.  square: float (n_rr+n_qq)^2 row-major.  Host pointers. */
sk_status sk_long_to_square(sk_ctx *ctx, const float *rr, int64_t n_rr,
                            const float *qr, const float *qq, int64_t n_qq,
                            float *square);
/* square_to_long (matrix_ops.cpp:130-150): upper triangle of an n x n
 * row-major matrix into n*(n-1)/2 values.  Host pointers. */
sk_status sk_square_to_long(sk_ctx *ctx, const float *square, int64_t n,
                            float *long_out);

/* ---- synthetic sketches (seeded generators for tests and benchmarks) ---- */

/* Bin-level tree generator.  parent[s] < s (or -1 for a root); thresh[s][k]
 * is the probability, scaled by 2^32, that sample s resamples a bin at
 * k-mer index k instead of inheriting it from its parent.  Writes the
 * reference word layout.  _host runs on the CPU (threads), _device writes a
 * device buffer; both produce identical words. */
sk_status sk_synth_host(const int32_t *parent, const uint32_t *thresh,
                        int64_t n_samples, int32_t n_kmers,
                        int32_t sketchsize64, uint64_t seed, int32_t threads,
                        uint64_t *words);
sk_status sk_synth_device(sk_ctx *ctx, const int32_t *parent,
                          const uint32_t *thresh, int64_t n_samples,
                          int32_t n_kmers, int32_t sketchsize64, uint64_t seed,
                          uint64_t *d_words);

/* ---- sketching -------------------------------------------------------------- */

/* MinHash sketches of sequences, the words every distance entry point takes.
 * The sequences of all samples lie back to back in `bases` (host memory):
 * sequence i is bases[seq_offsets[i], seq_offsets[i+1]), and sample s owns
 * sequences sample_seqs[s] .. sample_seqs[s+1]-1 (at least one; the reference
 * throws "... contains no sequence").  Each sample is sketched as the
 * reference's sketch() does for every k of `kmers` (each k >= 3, "Minimum k
 * must be 3 or higher"): every window of k bases A, C, G, T/U (either case)
 * inside one sequence is hashed with ntHash (canonical when use_rc = 1), the
 * hash mod 2^61-1 is kept as the minimum of its bin among 64 * sketchsize64,
 * empty bins are filled by the reference's probe sequence, and the low 14 bits
 * of each bin are written as bit planes.  Sequences go in as given; the
 * reference's file reader upper-cases them and drops those shorter than the
 * largest k (SeqBuf, src/sketch/seqio.cpp:55-100), which callers reproduce by
 * what they pass.  Bytes other than the ten base letters count as non-bases
 * (the reference's seed table also takes the control bytes 1, 3, 4, 5 and 7
 * as bases; sequence text never holds them).
 *
 * min_count > 0 (read sets, 1..255) keeps only k-mers seen at least min_count
 * times in the sample: the reference's exact counter (`exact = true`,
 * HashCounter, src/sketch/countmin.cpp:55-72).  The reference's default
 * count-min filter is an approximation whose answer depends on read order
 * (and, in its GPU sketcher, on a data race); it is not reproduced.
 *
 * codon_phased = 1 uses the reference's codon-phased spaced seeds
 * (generate_seeds, src/sketch/sketch.cpp:30-61): for each k a window of 3k-2
 * bases of which positions 0, 3, ..., 3(k-1) are hashed, every base of the
 * window valid (the reference's GPU sketcher refuses these seeds).
 *
 * Outputs (host): words [n_samples][n_kmers][sketchsize64 * 14] in the
 * reference layout; inv_minhash [n_samples][n_kmers] (bin 0's value over
 * 2^61-1 before densifying, whose per-sample sum gives the reference's read-set
 * size estimate K / sum) or NULL; densified [n_samples] (any k had empty bins)
 * or NULL. */
sk_status sk_sketch(sk_ctx *ctx, const char *bases, const int64_t *seq_offsets,
                    const int64_t *sample_seqs, int64_t n_samples, const int32_t *kmers,
                    int32_t n_kmers, int32_t sketchsize64, int32_t use_rc, int32_t codon_phased,
                    int32_t min_count, uint64_t *words, double *inv_minhash, uint8_t *densified);

/* sk_sketch with the bases already in device memory (d_bases, not modified)
 * and device outputs: d_words [n_samples][n_kmers][sketchsize64 * 14],
 * d_inv_minhash [n_samples][n_kmers] or NULL, d_densified [n_samples] or NULL.
 * seq_offsets and sample_seqs stay host arrays (the work is planned on the
 * host).  For sequences produced on the GPU, and to sketch straight into
 * memory that sk_db_create_device packs. */
sk_status sk_sketch_device(sk_ctx *ctx, const char *d_bases, const int64_t *seq_offsets,
                           const int64_t *sample_seqs, int64_t n_samples, const int32_t *kmers,
                           int32_t n_kmers, int32_t sketchsize64, int32_t use_rc,
                           int32_t codon_phased, int32_t min_count, uint64_t *d_words,
                           double *d_inv_minhash, uint8_t *d_densified);

/* ---- measurement ---------------------------------------------------------- */

/* Measured integer-ALU peaks of the context's device, in operations per
 * second: 32-bit LOP3 (the distance kernel's bound) and POPC.  Each is one
 * ~20 ms saturating kernel on the context's stream. */
sk_status sk_probe_alu_peak(sk_ctx *ctx, double *lop3_per_s, double *popc_per_s);
/* Checks the device-side bounded wait on this context: one CTA waits on a
 * barrier that nothing completes, gives up after limit_ms (1..10000) and
 * reports it, so the call returns SK_ETIMEDOUT ("A device-side bounded wait
 * timed out") and the context stays usable.  Every wait in this library's
 * kernels uses the same bounded wait (a 2 s limit in the distance kernel). */
sk_status sk_probe_wait_limit(sk_ctx *ctx, int32_t limit_ms);

#ifdef __cplusplus
}
#endif

#endif /* SKETCHLIB_B200_H */
