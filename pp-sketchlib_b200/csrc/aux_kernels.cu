// aux_kernels.cu -- the kernels around the distance kernel: packing sketches
// into device stripes, the synthetic sketch generator, kNN selection,
// threshold sparsification and long <-> square conversion.  All are
// memory-bound; each keeps its global accesses coalesced along the
// contiguous dimension of the long-form / stripe layouts.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <cfloat>
#include <cstdint>

#include "sk_common.h"
#include "sk_device.cuh"
#include "sk_launch.h"

namespace sk {

namespace {

constexpr int kThreads = 256;

inline int grid_for(int64_t work, int per_block, int cap = 148 * 32) {
  int64_t g = (work + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return static_cast<int>(g);
}

__device__ __forceinline__ int64_t condensed(int64_t i, int64_t j, int64_t n) {
  return n * i - ((i * (i + 1)) >> 1) + j - 1 - i;
}

// ------------------------------------------------------------------- packing

// One CTA per (k, granule of 64 samples, group of up to kPackBlocks 64-bin
// blocks): each sample's words for the group are kPackBlocks * 14 contiguous
// uint64 in the reference layout, read with consecutive threads on
// consecutive words into a shared tile, then written out as the group's
// 2 * kPackBlocks stripes (3584 contiguous bytes each).  `words` holds n
// samples that become granules g0 .. g0 + ng - 1 of an array of ng_total
// granules (samples past n are written as zeros).
constexpr int kPackBlocks = 4;
constexpr int kPackRow = kPackBlocks * kBbits + 1;   // tile row stride in uint64 (odd: fewer bank conflicts)

__global__ void pack_kernel(const uint64_t *__restrict__ words, int64_t n, int n_kmers, int s64,
                            int ng, int g0, int ng_total, uint32_t *__restrict__ packed) {
  __shared__ uint64_t tile[kGranule * kPackRow];
  const bool vec = (reinterpret_cast<uintptr_t>(words) & 15) == 0;   // rows are 112-byte multiples
  const int groups = (s64 + kPackBlocks - 1) / kPackBlocks;
  const int64_t n_items = static_cast<int64_t>(n_kmers) * ng * groups;
  const int nb = 2 * s64;
  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int grp = static_cast<int>(item % groups);
    const int64_t rest = item / groups;
    const int g = static_cast<int>(rest % ng);
    const int k = static_cast<int>(rest / ng);
    const int b0 = grp * kPackBlocks;
    const int nblk = min(kPackBlocks, s64 - b0);
    const int row_words = nblk * kBbits;
    if (nblk == kPackBlocks && vec) {
      // full group, 16-byte aligned rows: every 128-bit load in flight at once
      constexpr int kRowVec = kPackBlocks * kBbits / 2;            // uint4 per sample row
      constexpr int kPerThread = kGranule * kRowVec / kThreads;     // 7
      static_assert(kGranule * kRowVec % kThreads == 0, "whole loads per thread");
      uint4 v[kPerThread];
#pragma unroll
      for (int r = 0; r < kPerThread; ++r) {
        const int e = threadIdx.x + r * kThreads;
        const int lane = e / kRowVec, q = e % kRowVec;
        const int64_t smp = static_cast<int64_t>(g) * kGranule + lane;
        v[r] = smp < n ? reinterpret_cast<const uint4 *>(
                             words + ((smp * n_kmers + k) * s64 + b0) * kBbits)[q]
                       : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (int r = 0; r < kPerThread; ++r) {
        const int e = threadIdx.x + r * kThreads;
        const int lane = e / kRowVec, q = e % kRowVec;
        tile[lane * kPackRow + 2 * q] = (static_cast<uint64_t>(v[r].y) << 32) | v[r].x;
        tile[lane * kPackRow + 2 * q + 1] = (static_cast<uint64_t>(v[r].w) << 32) | v[r].z;
      }
    } else {
      for (int e = threadIdx.x; e < kGranule * row_words; e += blockDim.x) {
        const int lane = e / row_words, w = e % row_words;
        const int64_t smp = static_cast<int64_t>(g) * kGranule + lane;
        tile[lane * kPackRow + w] =
            smp < n ? words[((smp * n_kmers + k) * s64 + b0) * kBbits + w] : 0ull;
      }
    }
    __syncthreads();
    // four consecutive samples of one plane per 128-bit store
    constexpr int kStripeVec = kStripeWords / 4;
    for (int e = threadIdx.x; e < 2 * nblk * kStripeVec; e += blockDim.x) {
      const int stripe = e / kStripeVec, w = (e % kStripeVec) * 4;
      const int b = stripe >> 1, h = stripe & 1;
      const int plane = w / kGranule, lane = w % kGranule;
      const uint64_t *t = tile + lane * kPackRow + b * kBbits + plane;
      const int sh = h ? 32 : 0;
      const uint4 o = make_uint4(static_cast<uint32_t>(t[0] >> sh),
                                 static_cast<uint32_t>(t[kPackRow] >> sh),
                                 static_cast<uint32_t>(t[2 * kPackRow] >> sh),
                                 static_cast<uint32_t>(t[3 * kPackRow] >> sh));
      const int64_t blk = static_cast<int64_t>(k) * nb + 2 * (b0 + b) + h;
      reinterpret_cast<uint4 *>(packed + (blk * ng_total + g0 + g) * kStripeWords)[w / 4] = o;
    }
    __syncthreads();
  }
}

__global__ void unpack_kernel(const uint32_t *__restrict__ packed, int64_t n, int n_kmers,
                              int s64, int ng, uint64_t *__restrict__ words) {
  const int64_t total = n * n_kmers * s64 * kBbits;
  const int nb = 2 * s64;
  for (int64_t o = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; o < total;
       o += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int plane = static_cast<int>(o % kBbits);
    int64_t r = o / kBbits;
    const int b64 = static_cast<int>(r % s64);
    r /= s64;
    const int k = static_cast<int>(r % n_kmers);
    const int64_t s = r / n_kmers;
    const int64_t g = s / kGranule, lane = s % kGranule;
    const int64_t base = ((static_cast<int64_t>(k) * nb + 2 * b64) * ng + g) * kStripeWords +
                         plane * kGranule + lane;
    const uint64_t lo = packed[base];
    const uint64_t hi = packed[base + static_cast<int64_t>(ng) * kStripeWords];
    words[o] = lo | (hi << 32);
  }
}

// ----------------------------------------------------------------- synthetic

// One warp per (sample, k, 64-bin block): each lane draws bins lane and
// lane+32, the 14 bit planes are gathered with ballots into reference words.
__global__ void synth_kernel(const int32_t *__restrict__ parent, const uint32_t *__restrict__ thresh,
                             int64_t n, int n_kmers, int s64, uint64_t seed,
                             uint64_t *__restrict__ words) {
  const int lane = threadIdx.x & 31;
  const int64_t warps_total = n * n_kmers * s64;
  const int64_t warp0 = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
  const int64_t wstride = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t w = warp0; w < warps_total; w += wstride) {
    const int b64 = static_cast<int>(w % s64);
    const int64_t rest = w / s64;
    const int k = static_cast<int>(rest % n_kmers);
    const int64_t s = rest / n_kmers;
    const uint32_t bin = static_cast<uint32_t>(b64) * 64u + lane;
    const uint32_t vlo = synth_bin(parent, thresh, n_kmers, s, k, bin, seed);
    const uint32_t vhi = synth_bin(parent, thresh, n_kmers, s, k, bin + 32u, seed);
    uint64_t mine = 0;
#pragma unroll
    for (int p = 0; p < kBbits; ++p) {
      const uint32_t lo = __ballot_sync(0xffffffffu, (vlo >> p) & 1u);
      const uint32_t hi = __ballot_sync(0xffffffffu, (vhi >> p) & 1u);
      if (lane == p) mine = static_cast<uint64_t>(lo) | (static_cast<uint64_t>(hi) << 32);
    }
    if (lane < kBbits) words[w * kBbits + lane] = mine;
  }
}

// ----------------------------------------------------------------------- kNN

// Self kNN over a condensed single column: lane = row i of a 32-row block.
// Each lane keeps its kNN best (key, j) in shared memory, sorted ascending;
// j is visited in increasing order, so equal keys keep the smaller j first.
// Keys are the distances, or 1 - J for Jaccard (src/api.cpp:370-371).
__global__ void knn_self_kernel(const float *__restrict__ vals, int64_t n, int knn, int jaccard,
                                int64_t *__restrict__ j_out, float *__restrict__ d_out) {
  extern __shared__ unsigned char smem[];
  float *key = reinterpret_cast<float *>(smem);
  int32_t *idx = reinterpret_cast<int32_t *>(key + 32 * knn);
  const int lane = threadIdx.x;
  const int64_t i = static_cast<int64_t>(blockIdx.x) * 32 + lane;
  const bool active = i < n;
  int count = 0;
  float worst = FLT_MAX;
  for (int64_t j = 0; j < n; ++j) {
    if (!active) break;
    float d;
    if (j == i) {
      d = INFINITY;  // the diagonal (src/api.cpp:365)
    } else {
      const int64_t a = j < i ? j : i, b = j < i ? i : j;
      d = vals[condensed(a, b, n)];
      if (jaccard) d = 1.0f - d;
    }
    if (count < knn || d < worst) {
      int pos = count < knn ? count++ : knn - 1;
      while (pos > 0 && key[(pos - 1) * 32 + lane] > d) {
        key[pos * 32 + lane] = key[(pos - 1) * 32 + lane];
        idx[pos * 32 + lane] = idx[(pos - 1) * 32 + lane];
        --pos;
      }
      key[pos * 32 + lane] = d;
      idx[pos * 32 + lane] = static_cast<int32_t>(j);
      worst = key[(count - 1) * 32 + lane];
    }
  }
  if (active) {
    for (int e = 0; e < knn; ++e) {
      const float k = key[e * 32 + lane];
      j_out[i * knn + e] = idx[e * 32 + lane];
      d_out[i * knn + e] = jaccard ? 1.0f - k : k;
    }
  }
}

// Row kNN over a dense (n_rows, n_cols) column: one warp per row, lanes take
// every 32nd column, then lane 0 merges the 32 sorted lists by (key, col).
// diag0 >= 0: row r is sample diag0 + r of the column set, whose own column
// counts as +inf (as in knn_self_kernel); jaccard: keys are 1 - J.
__global__ void knn_rows_kernel(const float *__restrict__ vals, int64_t n_rows, int64_t n_cols,
                                int knn, int64_t diag0, int jaccard, int64_t *__restrict__ j_out,
                                float *__restrict__ d_out) {
  extern __shared__ unsigned char smem[];
  float *key = reinterpret_cast<float *>(smem);
  int32_t *idx = reinterpret_cast<int32_t *>(key + 32 * knn);
  __shared__ int counts[32];
  const int lane = threadIdx.x;
  for (int64_t row = blockIdx.x; row < n_rows; row += gridDim.x) {
    const float *v = vals + row * n_cols;
    int count = 0;
    float worst = FLT_MAX;
    for (int64_t c = lane; c < n_cols; c += 32) {
      float d;
      if (diag0 >= 0 && c == diag0 + row) {
        d = INFINITY;
      } else {
        d = v[c];
        if (jaccard) d = 1.0f - d;
      }
      if (count < knn || d < worst) {
        int pos = count < knn ? count++ : knn - 1;
        while (pos > 0 && key[(pos - 1) * 32 + lane] > d) {
          key[pos * 32 + lane] = key[(pos - 1) * 32 + lane];
          idx[pos * 32 + lane] = idx[(pos - 1) * 32 + lane];
          --pos;
        }
        key[pos * 32 + lane] = d;
        idx[pos * 32 + lane] = static_cast<int32_t>(c);
        worst = key[(count - 1) * 32 + lane];
      }
    }
    counts[lane] = count;
    __syncwarp();
    if (lane == 0) {
      int head[32];
      for (int l = 0; l < 32; ++l) head[l] = 0;
      for (int e = 0; e < knn; ++e) {
        int best = -1;
        float bk = 0.0f;
        int32_t bj = 0;
        for (int l = 0; l < 32; ++l) {
          if (head[l] >= counts[l]) continue;
          const float k = key[head[l] * 32 + l];
          const int32_t j = idx[head[l] * 32 + l];
          if (best < 0 || k < bk || (k == bk && j < bj)) { best = l; bk = k; bj = j; }
        }
        if (best < 0) { j_out[row * knn + e] = -1; d_out[row * knn + e] = INFINITY; continue; }
        ++head[best];
        j_out[row * knn + e] = bj;
        d_out[row * knn + e] = jaccard ? 1.0f - bk : bk;
      }
    }
    __syncwarp();
  }
}

// Row kNN for any kNN up to the row length (the kernels above keep kNN lists
// per lane in shared memory, up to kKnnListMax entries).  One CTA per row, in four steps:
//  1. radix select over the 32-bit order-preserving image of the key (four
//     8-bit digits, most significant first; a 256-bin shared histogram per
//     pass over the row) finds the bucket [lo, hi] of keys that holds the
//     kNN-th smallest, and how many of its entries (need) are taken;
//  2. one more pass gathers every entry below lo, and the first `need`
//     entries of the bucket in column order (a CTA-wide ordered scan), as
//     64-bit (key image << 32 | column) words: unique, so their order is the
//     (key, column) order of the per-lane lists above;
//  3. a bitonic network with every comparator ascending sorts the kNN words;
//     positions past kNN act as +inf and are never touched, so the list
//     needs no padding.  It sorts in shared memory, or in the row's own
//     output slots (j_out, 8 bytes per entry) when the list is larger than
//     kKnnSmemList;
//  4. the words become (column, key) outputs.
// Keys are the distances (1 - J for Jaccard), the row's own column (diag0 >=
// 0) +inf, -0 read as +0.
constexpr int kKnnSelectThreads = 512;
constexpr int kKnnSmemList = 12288;   // 96 KiB of 64-bit words

__device__ __forceinline__ uint32_t key_image(float f) {
  if (f == 0.0f) f = 0.0f;
  const uint32_t b = __float_as_uint(f);
  return b ^ ((b >> 31) ? 0xFFFFFFFFu : 0x80000000u);
}

__device__ __forceinline__ float image_key(uint32_t u) {
  return __uint_as_float(u ^ ((u >> 31) ? 0x80000000u : 0xFFFFFFFFu));
}

__global__ void __launch_bounds__(kKnnSelectThreads)
knn_select_kernel(const float *__restrict__ vals, int64_t n_rows, int64_t n_cols, int knn,
                  int64_t diag0, int jaccard, int64_t *__restrict__ j_out,
                  float *__restrict__ d_out) {
  extern __shared__ unsigned long long sel_list[];
  __shared__ unsigned int hist[256];
  __shared__ unsigned int warp_tot[kKnnSelectThreads / 32];
  __shared__ unsigned int s_digit, s_before, s_bucket, s_less;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = kKnnSelectThreads / 32;
  for (int64_t row = blockIdx.x; row < n_rows; row += gridDim.x) {
    const float *v = vals + row * n_cols;
    const int64_t own = diag0 >= 0 ? diag0 + row : -1;
    auto image = [&](int64_t c) -> uint32_t {
      float d = c == own ? INFINITY : v[c];
      if (jaccard && c != own) d = 1.0f - d;
      return key_image(d);
    };

    // 1. the bucket of the kNN-th smallest key
    uint32_t prefix = 0, mask = 0;
    unsigned int rank = static_cast<unsigned int>(knn);
    for (int shift = 24; shift >= 0; shift -= 8) {
      for (int i = tid; i < 256; i += kKnnSelectThreads) hist[i] = 0;
      __syncthreads();
      for (int64_t c = tid; c < n_cols; c += kKnnSelectThreads) {
        const uint32_t u = image(c);
        if ((u & mask) == prefix) atomicAdd(&hist[(u >> shift) & 255u], 1u);
      }
      __syncthreads();
      if (warp == 0) {
        unsigned int h[8], sum = 0;
#pragma unroll
        for (int b = 0; b < 8; ++b) sum += (h[b] = hist[8 * lane + b]);
        unsigned int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const unsigned int t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        const unsigned int hit = __ballot_sync(0xffffffffu, incl >= rank);
        if (lane == __ffs(hit) - 1) {
          unsigned int cum = incl - sum;
          for (int b = 0; b < 8; ++b) {
            if (cum + h[b] >= rank) {
              s_digit = 8 * lane + b;
              s_before = cum;
              s_bucket = h[b];
              break;
            }
            cum += h[b];
          }
        }
      }
      __syncthreads();
      prefix |= s_digit << shift;
      mask |= 255u << shift;
      rank -= s_before;
      const bool whole = s_bucket == rank;   // every entry of the bucket is taken
      __syncthreads();
      if (whole) break;
    }
    const uint32_t lo = prefix, hi = prefix | ~mask;
    const unsigned int need = rank;

    // 2. gather: below the bucket in any order, the bucket in column order
    unsigned long long *list =
        knn <= kKnnSmemList ? sel_list : reinterpret_cast<unsigned long long *>(j_out + row * knn);
    if (tid == 0) s_less = 0;
    __syncthreads();
    const unsigned int n_less = static_cast<unsigned int>(knn) - need;
    unsigned int taken = 0;   // bucket entries taken so far (CTA-uniform)
    unsigned int less = 0;    // entries below the bucket gathered so far (CTA-uniform)
    for (int64_t c0 = 0; c0 < n_cols && (taken < need || less < n_less); c0 += kKnnSelectThreads) {
      const int64_t c = c0 + tid;
      const uint32_t u = c < n_cols ? image(c) : 0xFFFFFFFFu;
      const bool in = c < n_cols && u >= lo && u <= hi;
      if (c < n_cols && u < lo) {
        const unsigned int slot = atomicAdd(&s_less, 1u);
        list[slot] = (static_cast<unsigned long long>(u) << 32) | static_cast<uint32_t>(c);
      }
      const unsigned int bal = __ballot_sync(0xffffffffu, in);
      if (lane == 0) warp_tot[warp] = __popc(bal);
      __syncthreads();
      unsigned int before = 0, total = 0;
      for (int w = 0; w < NW; ++w) {
        const unsigned int t = warp_tot[w];
        if (w < warp) before += t;
        total += t;
      }
      const unsigned int r = taken + before + __popc(bal & ((1u << lane) - 1u));
      if (in && r < need)
        list[n_less + r] = (static_cast<unsigned long long>(u) << 32) | static_cast<uint32_t>(c);
      taken += total;
      less = s_less;   // read between the two barriers: no thread adds to it here
      __syncthreads();
    }

    // 3. sort the kNN words ascending (positions >= knn are +inf)
    int P = 1;
    while (P < knn) P <<= 1;
    for (int k = 2; k <= P; k <<= 1) {
      for (int h = k >> 1; h >= 1; h >>= 1) {
        for (int t = tid; t < P / 2; t += kKnnSelectThreads) {
          const int i = (t / h) * 2 * h + (t % h);
          const int j = h == (k >> 1) ? (i ^ (k - 1)) : i + h;   // mirror, then half-cleaners
          if (j < knn) {
            const unsigned long long a = list[i], b = list[j];
            if (b < a) {
              list[i] = b;
              list[j] = a;
            }
          }
        }
        __syncthreads();
      }
    }

    // 4. outputs
    for (int e = tid; e < knn; e += kKnnSelectThreads) {
      const unsigned long long w = list[e];
      const float key = image_key(static_cast<uint32_t>(w >> 32));
      j_out[row * knn + e] = static_cast<int64_t>(w & 0xFFFFFFFFull);
      d_out[row * knn + e] = jaccard ? 1.0f - key : key;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ count tables

// Jaccard (no random-match correction) and its logarithm for every count
// 0 .. n-1 of a union of `union_bits` bins, by the epilogue's own functions,
// so a table entry is bit-identical to the per-pair computation it replaces.
__global__ void count_table_kernel(double union_bits, int64_t n, float *__restrict__ jtab,
                                   double *__restrict__ ltab) {
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < n;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float j = corrected_jaccard(static_cast<uint32_t>(c), union_bits, 0.0);
    jtab[c] = j;
    ltab[c] = log(static_cast<double>(j));
  }
}

// ---------------------------------------------------------- threshold sparse

// Row i of the square form above the diagonal is condensed entries
// [condensed(i, i+1), +n-i-1): contiguous, read by one warp per row.
__global__ void threshold_count_kernel(const float *__restrict__ vals, int64_t n, int stride,
                                       int col, float cutoff, int64_t *__restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t warp0 = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
  const int64_t wstride = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = warp0; i < n; i += wstride) {
    const int64_t base = i + 1 < n ? condensed(i, i + 1, n) : 0;
    const int64_t len = n - i - 1;
    int64_t c = 0;
    for (int64_t e0 = 0; e0 < len; e0 += 32) {
      const int64_t e = e0 + lane;
      const bool hit = e < len && vals[(base + e) * stride + col] < cutoff;
      c += __popc(__ballot_sync(0xffffffffu, hit));
    }
    if (lane == 0) counts[i] = c;
  }
}

__global__ void threshold_fill_kernel(const float *__restrict__ vals, int64_t n, int stride,
                                      int col, float cutoff, const int64_t *__restrict__ offsets,
                                      int64_t *__restrict__ i_out, int64_t *__restrict__ j_out,
                                      float *__restrict__ d_out) {
  const int lane = threadIdx.x & 31;
  const int64_t warp0 = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
  const int64_t wstride = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = warp0; i < n; i += wstride) {
    const int64_t base = i + 1 < n ? condensed(i, i + 1, n) : 0;
    const int64_t len = n - i - 1;
    int64_t out = offsets[i];
    for (int64_t e0 = 0; e0 < len; e0 += 32) {
      const int64_t e = e0 + lane;
      float v = 0.0f;
      const bool hit = e < len && (v = vals[(base + e) * stride + col]) < cutoff;
      const uint32_t mask = __ballot_sync(0xffffffffu, hit);
      if (hit) {
        const int64_t o = out + __popc(mask & ((1u << lane) - 1u));
        i_out[o] = i;
        j_out[o] = i + 1 + e;
        d_out[o] = v;
      }
      out += __popc(mask);
    }
  }
}

// ------------------------------------------------------- long <-> square

__global__ void long_to_square_kernel(const float *__restrict__ rr, int64_t n_rr,
                                      const float *__restrict__ qr, const float *__restrict__ qq,
                                      int64_t n_qq, float *__restrict__ square) {
  const int64_t n = n_rr + n_qq;
  const int64_t total = n * n;
  for (int64_t o = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; o < total;
       o += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = o / n, j = o % n;
    float v = 0.0f;
    if (i != j) {
      const int64_t a = i < j ? i : j, b = i < j ? j : i;
      if (b < n_rr) {
        v = rr[condensed(a, b, n_rr)];
      } else if (a >= n_rr) {
        v = qq[condensed(a - n_rr, b - n_rr, n_qq)];
      } else {
        v = qr[(b - n_rr) * n_rr + a];  // ref index fastest (src/dist/matrix_ops.cpp:115-123)
      }
    }
    square[o] = v;
  }
}

__global__ void square_to_long_kernel(const float *__restrict__ square, int64_t n,
                                      float *__restrict__ long_out) {
  for (int64_t i = blockIdx.x; i < n - 1; i += gridDim.x) {
    const int64_t base = condensed(i, i + 1, n);
    for (int64_t j = i + 1 + threadIdx.x; j < n; j += blockDim.x) {
      long_out[base + (j - i - 1)] = square[i * n + j];
    }
  }
}

}  // namespace

cudaError_t launch_pack(const uint64_t *words, int64_t n, int32_t n_kmers, int32_t s64, int32_t ng,
                        uint32_t *packed, cudaStream_t stream) {
  return launch_pack_range(words, n, n_kmers, s64, ng, 0, ng, packed, stream);
}

cudaError_t launch_pack_range(const uint64_t *words, int64_t n, int32_t n_kmers, int32_t s64,
                              int32_t ng, int32_t g0, int32_t ng_total, uint32_t *packed,
                              cudaStream_t stream) {
  const int64_t items = static_cast<int64_t>(n_kmers) * ng * ((s64 + kPackBlocks - 1) / kPackBlocks);
  if (items == 0) return cudaSuccess;
  pack_kernel<<<grid_for(items, 1, 148 * 64), kThreads, 0, stream>>>(words, n, n_kmers, s64, ng,
                                                                     g0, ng_total, packed);
  return cudaGetLastError();
}

cudaError_t launch_unpack(const uint32_t *packed, int64_t n, int32_t n_kmers, int32_t s64,
                          int32_t ng, uint64_t *words, cudaStream_t stream) {
  const int64_t total = n * n_kmers * s64 * kBbits;
  unpack_kernel<<<grid_for(total, kThreads), kThreads, 0, stream>>>(packed, n, n_kmers, s64, ng,
                                                                    words);
  return cudaGetLastError();
}

cudaError_t launch_synth(const int32_t *parent, const uint32_t *thresh, int64_t n,
                         int32_t n_kmers, int32_t s64, uint64_t seed, uint64_t *words,
                         cudaStream_t stream) {
  const int64_t warps = n * n_kmers * s64;
  synth_kernel<<<grid_for(warps, kThreads / 32, 148 * 64), kThreads, 0, stream>>>(
      parent, thresh, n, n_kmers, s64, seed, words);
  return cudaGetLastError();
}

cudaError_t launch_knn_self(const float *col_vals, int64_t n, int32_t knn, int32_t jaccard,
                            int64_t *j_out, float *d_out, cudaStream_t stream) {
  if (knn > kKnnListMax || knn > n) return cudaErrorInvalidValue;
  const int smem = 32 * knn * 8;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(knn_self_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
  }
  const int blocks = static_cast<int>((n + 31) / 32);
  knn_self_kernel<<<blocks, 32, smem, stream>>>(col_vals, n, knn, jaccard, j_out, d_out);
  return cudaGetLastError();
}

cudaError_t launch_knn_rows(const float *vals, int64_t n_rows, int64_t n_cols, int32_t knn,
                            int64_t diag0, int32_t jaccard, int64_t *j_out, float *d_out,
                            cudaStream_t stream) {
  if (knn > n_cols) return cudaErrorInvalidValue;
  if (knn > kKnnListMax) {
    const int smem = knn <= kKnnSmemList ? knn * 8 : 0;
    if (smem > 48 * 1024) {
      const cudaError_t attr = cudaFuncSetAttribute(
          knn_select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kKnnSmemList * 8);
      if (attr != cudaSuccess) return attr;
    }
    const int blocks = static_cast<int>(n_rows < 148 * 4 ? n_rows : 148 * 4);
    knn_select_kernel<<<blocks > 0 ? blocks : 1, kKnnSelectThreads, smem, stream>>>(
        vals, n_rows, n_cols, knn, diag0, jaccard, j_out, d_out);
    return cudaGetLastError();
  }
  const int smem = 32 * knn * 8;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(knn_rows_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
  }
  const int blocks = static_cast<int>(n_rows < 148 * 64 ? n_rows : 148 * 64);
  knn_rows_kernel<<<blocks > 0 ? blocks : 1, 32, smem, stream>>>(vals, n_rows, n_cols, knn, diag0,
                                                                 jaccard, j_out, d_out);
  return cudaGetLastError();
}

cudaError_t launch_count_tables(double union_bits, int64_t n, float *jtab, double *ltab,
                                cudaStream_t stream) {
  count_table_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(union_bits, n, jtab, ltab);
  return cudaGetLastError();
}

cudaError_t launch_threshold_count(const float *vals, int64_t n, int32_t stride, int32_t col,
                                   float cutoff, int64_t *row_counts, cudaStream_t stream) {
  threshold_count_kernel<<<grid_for(n, kThreads / 32), kThreads, 0, stream>>>(
      vals, n, stride, col, cutoff, row_counts);
  return cudaGetLastError();
}

cudaError_t launch_threshold_fill(const float *vals, int64_t n, int32_t stride, int32_t col,
                                  float cutoff, const int64_t *row_offsets, int64_t *i_out,
                                  int64_t *j_out, float *d_out, cudaStream_t stream) {
  threshold_fill_kernel<<<grid_for(n, kThreads / 32), kThreads, 0, stream>>>(
      vals, n, stride, col, cutoff, row_offsets, i_out, j_out, d_out);
  return cudaGetLastError();
}

cudaError_t exclusive_scan_i64(const int64_t *in, int64_t *out, int64_t n, void *tmp,
                               size_t *tmp_bytes, cudaStream_t stream) {
  return cub::DeviceScan::ExclusiveSum(tmp, *tmp_bytes, in, out, n, stream);
}

cudaError_t launch_long_to_square(const float *rr, int64_t n_rr, const float *qr, const float *qq,
                                  int64_t n_qq, float *square, cudaStream_t stream) {
  const int64_t n = n_rr + n_qq;
  long_to_square_kernel<<<grid_for(n * n, kThreads), kThreads, 0, stream>>>(rr, n_rr, qr, qq,
                                                                           n_qq, square);
  return cudaGetLastError();
}

cudaError_t launch_square_to_long(const float *square, int64_t n, float *long_out,
                                  cudaStream_t stream) {
  if (n < 2) return cudaSuccess;
  square_to_long_kernel<<<grid_for(n, 1), kThreads, 0, stream>>>(square, n, long_out);
  return cudaGetLastError();
}

}  // namespace sk
