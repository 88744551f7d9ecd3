// noalloc.cu -- dense distances with no device allocation.
//
// Some callers cannot allocate device memory when they compute distances: a
// service whose device memory is carved up once at start-up and must not
// grow, or a host program that links this library next to an allocator it
// does not control.  For them
// sk_dists_dense_noalloc runs the same persistent distance kernel as
// sk_dists_dense, but every byte the kernel needs beyond its inputs (the
// databases) and its output (the caller's device buffer) comes from one
// file-scope static device array of SK_NOALLOC_SCRATCH_BYTES: the job
// descriptor, the work list, the queue counter, the per-CTA count scratch and
// the equal-base random-match factors.  Every GPU that loads the library holds
// that array until the process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "sk_runtime.h"

using namespace sk;

namespace {

constexpr size_t kNoAllocBytes = static_cast<size_t>(SK_NOALLOC_SCRATCH_BYTES);

// The scratch.  Host code must not use this name as an address (on the host it
// is only a stand-in); its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Looks up the array's device address on the context's first call, with the
// context's device current (the caller's DeviceGuard has made it current),
// and keeps it on the context: a context made after a device reset looks it
// up again instead of reusing an address from before the reset.
sk_status scratch_address(sk_ctx *ctx, unsigned char **out) {
  if (!ctx->noalloc_scratch) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress of the no-alloc scratch");
    ctx->noalloc_scratch = p;
  }
  *out = static_cast<unsigned char *>(ctx->noalloc_scratch);
  return SK_OK;
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

}  // namespace

extern "C" sk_status sk_dists_dense_noalloc(sk_ctx *ctx, const sk_db *ref, const sk_db *query,
                                            const sk_random *random, int32_t out_mode,
                                            void *d_out) {
  if (!ctx) return SK_EINVAL;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  DeviceGuard dev_guard(ctx->device);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  if (out_mode != SK_OUT_CORE_ACC && out_mode != SK_OUT_JACCARD && out_mode != SK_OUT_COUNTS)
    return fail(ctx, SK_EINVAL, "Unknown output mode %d", out_mode);
  if (!ref) return fail(ctx, SK_EINVAL, "No reference database");
  if (n_pairs(ref, query) > 0 && !d_out) return fail(ctx, SK_EINVAL, "null output buffer");

  // The job, built without the random model: the existing builder would
  // allocate the equal-base factors on the databases; here they go into the
  // static array instead, and the table model needs no device memory of its own.
  JobParams jp;
  const TileConfig *cfg = nullptr;
  st = build_job(ctx, ref, query, nullptr, out_mode, 0, d_out, &cfg, &jp);
  if (st != SK_OK) return st;
  if (random && random->kmers != ref->kmers)
    return fail(ctx, SK_EMISMATCH, "Random match table k-mer lengths differ from the sketches");
  if (jp.n_tiles == 0) return SK_OK;
  const sk_db *rows = query ? query : ref;

  // Layout of the static array for this call.
  std::vector<double> jv_rows, jv_cols;
  std::vector<float> jgpu;   // equal-base chances of the reference GPU path
  if (random && random->mode == kRandEqualBase && jp.semantics == kSemRefGpu) {
    jgpu = equal_base_gpu(ref, random->use_rc);
  } else if (random && random->mode == kRandEqualBase) {
    jv_cols = equal_base_factors(ref, random->use_rc);
    if (query) jv_rows = equal_base_factors(rows, random->use_rc);
  }
  int grid = resident_grid(ctx, *cfg);
  if (grid < 1) return fail(ctx, SK_ECUDA, "Tile configuration %d does not fit the device", cfg->id);
  if (grid > jp.n_tiles) grid = static_cast<int>(jp.n_tiles);
  std::vector<WorkItem> items(static_cast<size_t>(jp.n_tiles));
  for (int64_t t = 0; t < jp.n_tiles; ++t)
    items[t] = WorkItem{t, 0, 0, static_cast<int16_t>(jp.n_kmers), -1, 1};
  const size_t off_job = 0;
  const size_t off_items = align256(off_job + sizeof(JobParams));
  const size_t off_ctrl = align256(off_items + items.size() * sizeof(WorkItem));
  const size_t off_jv_cols = align256(off_ctrl + 8);
  const size_t off_jv_rows = align256(off_jv_cols + jv_cols.size() * sizeof(double));
  const size_t off_jgpu = align256(off_jv_rows + jv_rows.size() * sizeof(double));
  const size_t off_counts = align256(off_jgpu + jgpu.size() * sizeof(float));
  const size_t slot = count_slot_bytes(*cfg, job_slots(jp));
  const size_t fixed = off_counts;
  if (fixed + slot > kNoAllocBytes)
    return fail(ctx, SK_ERANGE,
                "No-alloc distances need %zu bytes of scratch for this job (work list %zu, one "
                "count slot %zu), above the %zu-byte static buffer; use sk_dists_dense",
                fixed + slot, items.size() * sizeof(WorkItem), slot, kNoAllocBytes);
  // fewer resident CTAs if the count slots of all of them do not fit
  grid = static_cast<int>(std::min<size_t>(grid, (kNoAllocBytes - fixed) / slot));

  unsigned char *base = nullptr;
  st = scratch_address(ctx, &base);
  if (st != SK_OK) return st;
  if (!jv_cols.empty()) {
    jp.rmode = kRandEqualBase;
    jp.jv_cols = reinterpret_cast<const double *>(base + off_jv_cols);
    jp.jv_rows = query ? reinterpret_cast<const double *>(base + off_jv_rows) : jp.jv_cols;
    jp.jv_cols_ld = static_cast<int64_t>(ref->ng) * kGranule;
    jp.jv_rows_ld = static_cast<int64_t>(rows->ng) * kGranule;
  } else if (!jgpu.empty()) {
    jp.rmode = kRandTable;
    jp.rtable = reinterpret_cast<const float *>(base + off_jgpu);
    jp.rs_k = 1;
    jp.rs_row = jp.rs_col = 0;
  } else if (random && random->mode == kRandTable) {
    const int C = random->n_clusters;
    const bool col_major = query || jp.semantics == kSemRefGpu;
    jp.rmode = kRandTable;
    jp.rtable = random->table;
    jp.rs_k = C * C;
    jp.rs_row = col_major ? 1 : C;
    jp.rs_col = col_major ? C : 1;
    jp.cl_rows = rows->cluster;
    jp.cl_cols = ref->cluster;
  }

  // Uploads (pageable host sources: each copy is staged before it returns).
  cudaError_t e = cudaMemcpyAsync(base + off_job, &jp, sizeof(JobParams), cudaMemcpyHostToDevice,
                                  ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + off_items, items.data(), items.size() * sizeof(WorkItem),
                        cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && !jv_cols.empty())
    e = cudaMemcpyAsync(base + off_jv_cols, jv_cols.data(), jv_cols.size() * sizeof(double),
                        cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && !jgpu.empty())
    e = cudaMemcpyAsync(base + off_jgpu, jgpu.data(), jgpu.size() * sizeof(float),
                        cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && !jv_rows.empty())
    e = cudaMemcpyAsync(base + off_jv_rows, jv_rows.data(), jv_rows.size() * sizeof(double),
                        cudaMemcpyHostToDevice, ctx->stream);
  // the queue counter must start at zero; everything else is written before it is read
  if (e == cudaSuccess) e = cudaMemsetAsync(base + off_ctrl, 0, 8, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "no-alloc upload");

  LaunchParams lp{};
  lp.jobs = reinterpret_cast<const JobParams *>(base + off_job);
  lp.items = reinterpret_cast<const WorkItem *>(base + off_items);
  lp.n_items = static_cast<int64_t>(items.size());
  lp.item_counter = reinterpret_cast<unsigned long long *>(base + off_ctrl);
  lp.split_done = nullptr;       // no tile is split here
  lp.cta_scratch = reinterpret_cast<uint16_t *>(base + off_counts);
  lp.split_scratch = nullptr;
  lp.k_slots = job_slots(jp);
  lp.wide = needs_wide(jp) ? 1 : 0;
  lp.status = ctx->status_dev;
  lp.cancel = ctx->cancel_dev;
  e = cfg->launch(lp, grid, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "no-alloc distance kernel launch");
  return SK_OK;
}
