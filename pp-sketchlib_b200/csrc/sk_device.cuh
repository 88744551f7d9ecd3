// sk_device.cuh -- device helpers shared by the distance kernels: bulk-copy /
// mbarrier wrappers with bounded waits, the bit-plane intersect primitive, the
// triangular tile map and the per-pair epilogue (random-match correction,
// k-range truncation and the log-linear fit).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "sk_common.h"

namespace sk {

// ---------------------------------------------------------------- PTX wrappers

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// One bulk (TMA engine) copy global -> shared, completing on `bar`.
// dst, src and bytes must be multiples of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for phase `parity` of `bar` for at most `limit_ns`.  Returns false on
// timeout; the caller records the error and unwinds instead of spinning on.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

// acc & ~(a ^ b): one 3-input LOP3 per 32 bins per bit plane.
__device__ __forceinline__ uint32_t lop_eq_and(uint32_t acc, uint32_t a, uint32_t b) {
  uint32_t d;
  asm("lop3.b32 %0, %1, %2, %3, 0x82;" : "=r"(d) : "r"(a), "r"(b), "r"(acc));
  return d;
}
// ~(a ^ b): the first plane of a block.
__device__ __forceinline__ uint32_t lop_eq(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("lop3.b32 %0, %1, %2, %1, 0xC3;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}

// d = a * b + c on 32-bit integers (an IMAD: FMA pipe).
__device__ __forceinline__ uint32_t mad_u32(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// ------------------------------------------------------------------ tile map

// All-vs-all: row tile ti (rows ti*tr .. ti*tr+tr-1) needs column tiles
// tj >= ti*m (m = tile_rows / tile_cols), the first one holding a column
// greater than the tile's first row.  Tiles are numbered row-tile-major.
__device__ __forceinline__ int64_t tri_tiles_before(int64_t ti, int64_t n_col_tiles, int64_t m) {
  return ti * n_col_tiles - m * ti * (ti - 1) / 2;
}

__device__ __forceinline__ void tile_coords(const JobParams &p, int64_t tile, int32_t &ti,
                                            int32_t &tj) {
  if (p.self) {
    const int64_t m = p.tile_rows / p.tile_cols;
    int64_t lo = 0, hi = p.n_row_tiles - 1;
    while (lo < hi) {  // largest ti with tiles_before(ti) <= tile
      const int64_t mid = (lo + hi + 1) >> 1;
      if (tri_tiles_before(mid, p.n_col_tiles, m) <= tile) lo = mid; else hi = mid - 1;
    }
    ti = static_cast<int32_t>(lo);
    tj = static_cast<int32_t>(lo * m + (tile - tri_tiles_before(lo, p.n_col_tiles, m)));
  } else {
    ti = static_cast<int32_t>(tile / p.n_col_tiles);
    tj = static_cast<int32_t>(tile % p.n_col_tiles);
  }
}

// -------------------------------------------------------------- pair epilogue

// Intersection count of k-mer index k: its count slot, or (CHUNKED) the sum
// of its chunks' slots when the sketch is wider than one uint16 counter holds
// (counts[(k * nchunk + c) * stride]).
template <bool CHUNKED>
__device__ __forceinline__ uint32_t pair_count(const JobParams &p, const uint16_t *counts,
                                               int stride, int k) {
  if (!CHUNKED) return counts[k * stride];
  uint32_t c = 0;
  for (int q = 0; q < p.nchunk; ++q) c += counts[(k * p.nchunk + q) * stride];
  return c;
}

// Loop bound over the k-mer lengths of a per-pair array of KMAX entries: the
// constant KMAX (loops unroll, arrays stay in registers) for the narrow
// instance's arrays, the job's K (loops stay loops) for the wide one.
template <int KMAX>
__device__ __forceinline__ int k_bound(const JobParams &p) {
  return KMAX <= kNarrowKmers ? KMAX : p.n_kmers;
}

// Entry of the Monte Carlo table for (row gi, col gj) at k-mer index k.
__device__ __forceinline__ int64_t random_table_index(const JobParams &p, int k, int64_t gi,
                                                      int64_t gj) {
  int cr = p.cl_rows ? p.cl_rows[gi] : 0;
  int cc = p.cl_cols ? p.cl_cols[gj] : 0;
  if (p.self_view && p.row_base + gi > gj) {   // the all-vs-all path sees (gj, row)
    const int t = cr;
    cr = cc;
    cc = t;
  }
  return static_cast<int64_t>(k) * p.rs_k + cr * p.rs_row + cc * p.rs_col;
}

// Random match chance for (row gi, col gj) at k-mer index k
// (RandomMC::random_match, src/random/random_match.cpp:185-206; csrs :318-336).
__device__ __forceinline__ double random_match(const JobParams &p, int k, int64_t gi, int64_t gj) {
  if (p.rmode == kRandTable) return static_cast<double>(p.rtable[random_table_index(p, k, gi, gj)]);
  if (p.rmode == kRandEqualBase) {
    const double j1 = p.jv_rows[k * p.jv_rows_ld + gi];
    const double j2 = p.jv_cols[k * p.jv_cols_ld + gj];
    if (j1 > 0.0 && j2 > 0.0) {
      const double num = __dmul_rn(j1, j2);
      return __ddiv_rn(num, __dsub_rn(__dadd_rn(j1, j2), num));
    }
  }
  return 0.0;
}

// Random-corrected Jaccard as the float the reference regresses on:
// J = max(obs - r, 0) / (1 - r), obs = count / (64 * s64) in double
// (Reference::jaccard_dist, src/reference.cpp:86-96; observed_excess,
// src/dist/dist.hpp:19-24), then narrowed to float (regress_kmers,
// src/dist/linear_regression.cpp:66-69).
__device__ __forceinline__ float corrected_jaccard(uint32_t count, double union_bits, double r) {
  const double obs = __ddiv_rn(static_cast<double>(count), union_bits);
  const double diff = obs > r ? __dsub_rn(obs, r) : 0.0;
  return __double2float_rn(__ddiv_rn(diff, __dsub_rn(1.0, r)));
}

// Log-linear fit log J_k = log(1-acc) + k log(1-core) over the contiguous
// k-range from the first to the last J above tolerance (fit_slope,
// src/dist/linear_regression.cpp:16-60).  Fewer than 2 points in the range
// gives (0, 0), the reference GPU's result (src/gpu/dist.cu:95-97); the
// reference CPU exits the process there; a zero J strictly inside the range
// gives (0, 0) too.  Least squares in double:
//   xm = sum x / n, ym = sum y / n,
//   slope = sum (x - xm) y / sum (x - xm)^2, intercept = ym - slope xm,
// without fused multiply-adds, in the same operation order as the oracle.
template <int KMAX, bool CHUNKED>
__device__ __forceinline__ float2 fit_core_acc(const float (&jf)[KMAX], const JobParams &p,
                                               const uint16_t *counts, int stride) {
  int first = -1, last = -1;
#pragma unroll
  for (int k = 0; k < k_bound<KMAX>(p); ++k) {
    if (k < p.n_kmers && static_cast<double>(jf[k]) > p.tol) {
      if (first < 0) first = k;
      last = k;
    }
  }
  float2 res = make_float2(0.0f, 0.0f);
  if (first < 0 || last - first + 1 < 2) return res;
  // A zero Jaccard inside the range has no logarithm: the reference's float
  // solve turns it into NaN slopes, i.e. (0, 0).
  bool zero_inside = false;
#pragma unroll
  for (int k = 0; k < k_bound<KMAX>(p); ++k)
    if (k > first && k < last && jf[k] <= 0.0f) zero_inside = true;
  if (zero_inside) return res;
  const double n = static_cast<double>(last - first + 1);
  double sx = 0.0;
#pragma unroll
  for (int k = 0; k < k_bound<KMAX>(p); ++k)
    if (k >= first && k <= last) sx = __dadd_rn(sx, static_cast<double>(p.kmers[k]));
  const double xm = __ddiv_rn(sx, n);
  double sy = 0.0, sxx = 0.0, sxy = 0.0;
#pragma unroll
  for (int k = 0; k < k_bound<KMAX>(p); ++k) {
    if (k >= first && k <= last) {
      const double y = p.ltab ? p.ltab[pair_count<CHUNKED>(p, counts, stride, k)]
                              : log(static_cast<double>(jf[k]));
      const double dx = __dsub_rn(static_cast<double>(p.kmers[k]), xm);
      sy = __dadd_rn(sy, y);
      sxx = __dadd_rn(sxx, __dmul_rn(dx, dx));
      sxy = __dadd_rn(sxy, __dmul_rn(dx, y));
    }
  }
  const double ym = __ddiv_rn(sy, n);
  const double slope = __ddiv_rn(sxy, sxx);
  const double icpt = __dsub_rn(ym, __dmul_rn(slope, xm));
  if (slope < 0.0) res.x = __double2float_rn(__dsub_rn(1.0, exp(slope)));
  if (icpt < 0.0) res.y = __double2float_rn(__dsub_rn(1.0, exp(icpt)));
  return res;
}

// The reference GPU kernel's per-pair arithmetic, for
// SK_SEMANTICS_REFERENCE_GPU (calculate_dists, src/gpu/dist.cu:199-289, with
// jaccard_dist :57-84, observed_excess :46-54, simple_linear_regression
// :89-129; no fast-math in the reference's CUDA flags, so `/` is the IEEE
// division and nvcc fuses `sum += k * y` and `sum += y * y` into FMAs):
//   J = count / (64 s64) rounded up, J' = max(J - r, 0) / (1 - r) in float;
//   the fit takes k in order until the first J' below 5 / (64 s64) (fast
//   division), summing x = k, y = __logf(J'), x y, x^2, y^2 in float;
//   fewer than 2 points gives (0, 0); slope = r_xy * sd_y / sd_x from the
//   correlation coefficient with round-up intrinsics, intercept =
//   ybar - slope xbar (round-up FMA); core / accessory = 1 - __expf(.) when
//   negative.  A pair whose Jaccards are all equal has sd_y = 0, r_xy = 0 / 0
//   and so (0, 0), as in the reference kernel.
template <bool CHUNKED>
__device__ __forceinline__ float2 refgpu_core_acc(const JobParams &p, int64_t gi, int64_t gj,
                                                  const uint16_t *counts, int stride) {
  const int bins = static_cast<int>(p.union_bits);
  const float unionf = static_cast<float>(bins);
  const float tol = __fdividef(5.0f, __int2float_rz(bins));
  int used = 0;
  float xsum = 0.0f, ysum = 0.0f, xysum = 0.0f, xsq = 0.0f, ysq = 0.0f;
  bool stop = false;
  for (int k = 0; k < p.n_kmers; ++k) {
    const float obs = __fdiv_ru(static_cast<float>(pair_count<CHUNKED>(p, counts, stride, k)), unionf);
    const float r = static_cast<float>(random_match(p, k, gi, gj));
    const float diff = obs > r ? __fsub_rn(obs, r) : 0.0f;
    const float jac = __fdiv_rn(diff, __fsub_rn(1.0f, r));
    if (jac < tol) {
      stop = true;
    } else if (!stop) {
      const float y = __logf(jac);
      const int km = p.kmers[k];
      ++used;
      xsum = __fadd_rn(xsum, static_cast<float>(km));
      ysum = __fadd_rn(ysum, y);
      xysum = __fmaf_rn(static_cast<float>(km), y, xysum);
      xsq = __fadd_rn(xsq, static_cast<float>(km * km));
      ysq = __fmaf_rn(y, y, ysq);
    }
  }
  float2 res = make_float2(0.0f, 0.0f);
  if (used < 2) return res;
  const float n = static_cast<float>(used);
  const float xbar = __fdiv_rn(xsum, n);
  const float ybar = __fdiv_rn(ysum, n);
  const float x_diff = __fsub_rn(xsq, __fdiv_rn(__fmul_ru(xsum, xsum), n));
  const float y_diff = __fsub_rn(ysq, __fdiv_rn(__fmul_ru(ysum, ysum), n));
  const float sd_x = __fsqrt_ru(__fdiv_rn(x_diff, n));
  const float sd_y = __fsqrt_ru(__fdiv_rn(y_diff, n));
  const float r_xy = __fdiv_ru(__fsub_rn(xysum, __fdiv_rn(__fmul_ru(xsum, ysum), n)),
                               __fsqrt_ru(__fmul_rn(x_diff, y_diff)));
  const float beta = __fmul_ru(r_xy, __fdiv_ru(sd_y, sd_x));
  const float alpha = __fmaf_ru(-beta, xbar, ybar);
  if (beta < 0.0f) res.x = __fsub_rn(1.0f, __expf(beta));
  if (alpha < 0.0f) res.y = __fsub_rn(1.0f, __expf(alpha));
  return res;
}

// Long-form row of pair (gi, gj): square_to_condensed (src/dist/matrix_idx.hpp:46-50)
// for all-vs-all, gi * n_cols + gj for query-vs-reference (src/api.cpp:251),
// relative to the first row held by the output buffer.
__device__ __forceinline__ int64_t pair_row(const JobParams &p, int64_t gi, int64_t gj) {
  if (p.self) return p.n_rows * gi - ((gi * (gi + 1)) >> 1) + gj - 1 - gi - p.out_row0;
  return gi * p.n_cols + gj - p.out_row0;
}

// Finishes one pair from its K intersection counts (counts[k * stride]) and
// writes its long-form row.
template <int KMAX, bool CHUNKED>
__device__ __forceinline__ void finish_pair(const JobParams &p, int64_t gi, int64_t gj,
                                            const uint16_t *counts, int stride) {
  const int64_t row = pair_row(p, gi, gj);
  const int K = p.n_kmers;
  if (p.out_mode == kOutCounts) {
    uint32_t *o = static_cast<uint32_t *>(p.out) + row * K;
    for (int k = 0; k < K; ++k) o[k] = pair_count<CHUNKED>(p, counts, stride, k);
    return;
  }
  if (p.semantics == kSemRefGpu &&
      (p.out_mode == kOutCoreAcc || (p.out_mode == kOutColumn && p.out_col < 2))) {
    const float2 ca = refgpu_core_acc<CHUNKED>(p, gi, gj, counts, stride);
    if (p.out_mode == kOutCoreAcc) static_cast<float2 *>(p.out)[row] = ca;
    else static_cast<float *>(p.out)[row] = p.out_col == 0 ? ca.x : ca.y;
    return;
  }
  float jf[KMAX];
#pragma unroll
  for (int k = 0; k < k_bound<KMAX>(p); ++k) {
    jf[k] = 0.0f;
    if (k < K) {
      const uint32_t c = pair_count<CHUNKED>(p, counts, stride, k);
      jf[k] = p.jtab ? p.jtab[c] : corrected_jaccard(c, p.union_bits, random_match(p, k, gi, gj));
    }
  }
  if (p.out_mode == kOutJaccard) {
    float *o = static_cast<float *>(p.out) + row * K;
#pragma unroll
    for (int k = 0; k < k_bound<KMAX>(p); ++k)
      if (k < K) o[k] = jf[k];
    return;
  }
  if (p.out_mode == kOutColumn && p.out_col >= 2) {  // Jaccard at k index out_col - 2
    float v = 0.0f;
#pragma unroll
    for (int k = 0; k < k_bound<KMAX>(p); ++k)
      if (k == p.out_col - 2) v = jf[k];
    static_cast<float *>(p.out)[row] = v;
    return;
  }
  const float2 ca = fit_core_acc<KMAX, CHUNKED>(jf, p, counts, stride);
  if (p.out_mode == kOutCoreAcc) {
    static_cast<float2 *>(p.out)[row] = ca;
  } else {
    static_cast<float *>(p.out)[row] = p.out_col == 0 ? ca.x : ca.y;
  }
}

// Dispatches on the number of k-mer lengths so the per-pair arrays stay in
// registers for the common K <= 8 and K <= 16 cases.  The narrow kernel
// instance finishes up to kNarrowKmers k-mer lengths with unrolled arrays;
// the wide one finishes wider k sets, and sketches counted in chunks, with
// loops over arrays in local memory.
template <bool WIDE>
__device__ __forceinline__ void finish_pair_any(const JobParams &p, int64_t gi, int64_t gj,
                                                const uint16_t *counts, int stride) {
  if constexpr (WIDE) {
    if (p.nchunk == 1 && p.n_kmers <= 8) finish_pair<8, false>(p, gi, gj, counts, stride);
    else if (p.nchunk == 1 && p.n_kmers <= 16) finish_pair<16, false>(p, gi, gj, counts, stride);
    else finish_pair<kMaxKmers, true>(p, gi, gj, counts, stride);
  } else {
    if (p.n_kmers <= 8) finish_pair<8, false>(p, gi, gj, counts, stride);
    else if (p.n_kmers <= 16) finish_pair<16, false>(p, gi, gj, counts, stride);
    else finish_pair<kNarrowKmers, false>(p, gi, gj, counts, stride);
  }
}

}  // namespace sk
