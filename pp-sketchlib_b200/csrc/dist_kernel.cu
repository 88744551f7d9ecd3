// dist_kernel.cu -- the fused bit-sliced MinHash distance kernel for sm_100a.
//
// One persistent CTA per SM walks its share of (row tile x column tile) work
// items.  For every k-mer length and every 32-bin block it stages the 14 bit
// planes of its row and column samples into shared memory with bulk copies
// (TMA engine, one copy per 64-sample stripe, mbarrier completion), and each
// thread intersects a TQ x TR register block of pairs:
//     acc = AND over planes of ~(row_word ^ col_word)   (one LOP3 per plane)
//     count += popc(acc)
// which is calc_intersize (src/dist/dist.cpp:50-78) for 32 bins at a time.
// Per-k counts of the tile go to shared memory as uint16; once all k are done
// the CTA turns each pair's counts into random-corrected Jaccards and the
// log-linear core/accessory fit and writes the long-form row directly.
//
// Replaces calculate_dists (src/gpu/dist.cu:164-317): one thread per pair with
// strided 8-byte global loads there; register-blocked tiles over staged
// stripes here.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "sk_device.cuh"
#include "sk_launch.h"

namespace sk {

constexpr int kBlocksPerStage = 2;   // 32-bin blocks per pipeline stage
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s bounded waits

template <int QT, int RT, int TQ, int TR, int STAGES>
struct TileShape {
  static constexpr int kThreads = (QT / TQ) * (RT / TR);
  static constexpr int kPairsPerThread = TQ * TR;
  static constexpr int kQG = QT / kGranule;
  static constexpr int kRG = RT / kGranule;
  static constexpr int kStageQWords = kBlocksPerStage * kQG * kStripeWords;
  static constexpr int kStageRWords = kBlocksPerStage * kRG * kStripeWords;
  static constexpr int kStageBytes = (kStageQWords + kStageRWords) * 4;
  static constexpr int kSmemBytes = STAGES * kStageBytes;
  static_assert(QT % kGranule == 0 && RT % kGranule == 0, "tiles are whole granules");
  static_assert(kGranule % TQ == 0 && kGranule % TR == 0, "thread blocks stay in a granule");
  static_assert(TQ % 4 == 0 && TR % 4 == 0, "128-bit shared loads");
  static_assert(kPairsPerThread % 8 == 0, "counts are stored as 16-byte groups");
  static_assert(QT % RT == 0, "triangular map needs tile_rows multiple of tile_cols");
};

// Per-k counts of a thread's TQ x TR pairs are parked in `scratch` (this CTA's
// slot: [K][threads][TQ*TR] uint16, written and read back by the same thread,
// so no barrier is needed; 38 MB for 296 CTAs at K = 8, resident in L2).  The
// thread then finishes its own pairs, so a tile needs no CTA-wide epilogue.
template <int QT, int RT, int TQ, int TR, int STAGES, int MINB>
__global__ void __launch_bounds__((QT / TQ) * (RT / TR), MINB)
    dist_tiles_kernel(const JobParams p, uint16_t *__restrict__ scratch, DevStatus *status,
                      const volatile int *cancel) {
  using S = TileShape<QT, RT, TQ, TR, STAGES>;
  constexpr int NT = S::kThreads;
  constexpr int PT = S::kPairsPerThread;
  constexpr int TCOLS = RT / TR;

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t *sq = reinterpret_cast<uint32_t *>(smem);
  uint32_t *sr = sq + STAGES * S::kStageQWords;
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ int s_abort;

  const int tid = threadIdx.x;
  const int tq = tid / TCOLS;
  const int tr = tid % TCOLS;
  const int row0 = tq * TQ;   // first tile row of this thread
  const int col0 = tr * TR;   // first tile column of this thread

  if (blockIdx.x >= p.n_tiles) return;
  const int64_t my_tiles = (p.n_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
  const int64_t steps_per_k = p.nb / kBlocksPerStage;
  const int64_t spt = steps_per_k * p.n_kmers;
  const int64_t total = my_tiles * spt;
  uint16_t *my_counts = scratch + (static_cast<int64_t>(blockIdx.x) * p.n_kmers * NT + tid) * PT;
  const int64_t k_stride = static_cast<int64_t>(NT) * PT;   // uint16 between k slots

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&full_bar[s], 1);
    fence_mbar_init();
    s_abort = 0;
  }
  __syncthreads();

  // Producer (thread 0): stage step u into buffer u % STAGES.
  int64_t next_issue = 0;
  auto issue = [&](int64_t u) {
    const int64_t tile_iter = u / spt;
    const int64_t local = u - tile_iter * spt;
    const int64_t kidx = local / steps_per_k;
    const int64_t b0 = (local - kidx * steps_per_k) * kBlocksPerStage;
    int32_t ti, tj;
    tile_coords(p, blockIdx.x + tile_iter * gridDim.x, ti, tj);
    const int s = static_cast<int>(u % STAGES);
    mbar_arrive_expect_tx(&full_bar[s], S::kStageBytes);
#pragma unroll
    for (int b = 0; b < kBlocksPerStage; ++b) {
      const int64_t blk = kidx * p.nb + b0 + b;
      const uint32_t *src_q =
          p.row_words + ((blk * p.ng_rows) + static_cast<int64_t>(ti) * S::kQG) * kStripeWords;
      const uint32_t *src_r =
          p.col_words + ((blk * p.ng_cols) + static_cast<int64_t>(tj) * S::kRG) * kStripeWords;
      bulk_g2s(sq + (s * kBlocksPerStage + b) * S::kQG * kStripeWords, src_q,
               S::kQG * kStripeBytes, &full_bar[s]);
      bulk_g2s(sr + (s * kBlocksPerStage + b) * S::kRG * kStripeWords, src_r,
               S::kRG * kStripeBytes, &full_bar[s]);
    }
  };
  if (tid == 0) {
    while (next_issue < total && next_issue < STAGES) issue(next_issue++);
  }

  // 1 at run time: makes the count accumulation a multiply-add, which runs on
  // the otherwise idle FMA pipe instead of taking ALU slots from the LOP3s.
  const uint32_t one = p.one;
  uint32_t cnt[TQ][TR];
#pragma unroll
  for (int i = 0; i < TQ; ++i)
#pragma unroll
    for (int j = 0; j < TR; ++j) cnt[i][j] = 0;

  int64_t t = 0;
  for (; t < total; ++t) {
    const int s = static_cast<int>(t % STAGES);
    const uint32_t parity = static_cast<uint32_t>((t / STAGES) & 1);
    const bool ok = mbar_wait_bounded(&full_bar[s], parity, kWaitLimitNs);
    if (!ok) {
      s_abort = 1;
      atomicOr(&status->error, 1u);
      status->where = 1;
    } else {
#pragma unroll
      for (int b = 0; b < kBlocksPerStage; ++b) {
        const uint32_t *qb = sq + (s * kBlocksPerStage + b) * S::kQG * kStripeWords +
                             (row0 / kGranule) * kStripeWords + (row0 % kGranule);
        const uint32_t *rb = sr + (s * kBlocksPerStage + b) * S::kRG * kStripeWords +
                             (col0 / kGranule) * kStripeWords + (col0 % kGranule);
        uint32_t acc[TQ][TR];
#pragma unroll
        for (int pl = 0; pl < kBbits; ++pl) {
          uint32_t qv[TQ], rv[TR];
#pragma unroll
          for (int i = 0; i < TQ; i += 4) {
            const uint4 v = *reinterpret_cast<const uint4 *>(qb + pl * kGranule + i);
            qv[i] = v.x; qv[i + 1] = v.y; qv[i + 2] = v.z; qv[i + 3] = v.w;
          }
#pragma unroll
          for (int j = 0; j < TR; j += 4) {
            const uint4 v = *reinterpret_cast<const uint4 *>(rb + pl * kGranule + j);
            rv[j] = v.x; rv[j + 1] = v.y; rv[j + 2] = v.z; rv[j + 3] = v.w;
          }
#pragma unroll
          for (int i = 0; i < TQ; ++i)
#pragma unroll
            for (int j = 0; j < TR; ++j)
              acc[i][j] = pl == 0 ? lop_eq(qv[i], rv[j]) : lop_eq_and(acc[i][j], qv[i], rv[j]);
        }
#pragma unroll
        for (int i = 0; i < TQ; ++i)
#pragma unroll
          for (int j = 0; j < TR; ++j) cnt[i][j] = mad_u32(__popc(acc[i][j]), one, cnt[i][j]);
      }
    }
    __syncthreads();  // stage s fully read by every warp
    if (s_abort) break;
    if (tid == 0 && next_issue < total) issue(next_issue++);

    const int64_t local = t % spt;
    const int64_t kidx = local / steps_per_k;
    if (local - kidx * steps_per_k == steps_per_k - 1) {
      // all blocks of k-mer index kidx done: park this thread's counts
      uint4 *dst = reinterpret_cast<uint4 *>(my_counts + kidx * k_stride);
#pragma unroll
      for (int w = 0; w < PT / 8; ++w) {
        uint32_t packed[4];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int q0 = w * 8 + 2 * h, q1 = q0 + 1;
          packed[h] = cnt[q0 / TR][q0 % TR] | (cnt[q1 / TR][q1 % TR] << 16);
        }
        dst[w] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
      }
#pragma unroll
      for (int i = 0; i < TQ; ++i)
#pragma unroll
        for (int j = 0; j < TR; ++j) cnt[i][j] = 0;

      if (kidx == p.n_kmers - 1) {
        // tile complete: this thread finishes its own TQ x TR pairs
        int32_t ti, tj;
        tile_coords(p, blockIdx.x + (t / spt) * gridDim.x, ti, tj);
        const int64_t gi0 = static_cast<int64_t>(ti) * QT + row0;
        const int64_t gj0 = static_cast<int64_t>(tj) * RT + col0;
#pragma unroll 1
        for (int q = 0; q < PT; ++q) {
          const int64_t gi = gi0 + q / TR;
          const int64_t gj = gj0 + q % TR;
          const bool valid = p.self ? (gj > gi && gj < p.n_cols) : (gi < p.n_rows && gj < p.n_cols);
          if (valid) finish_pair_any(p, gi, gj, my_counts + q, static_cast<int>(k_stride));
        }
        if (tid == 0) {
          atomicAdd(&status->tiles_done, 1ull);
          if (cancel != nullptr && *cancel != 0) {
            s_abort = 1;   // seen by every thread after the next step's barrier
            atomicOr(&status->error, 2u);
          }
        }
      }
    }
  }

  if (tid == 0 && t < total) {
    // unwinding early: let the copies already in flight land before exit
    for (int64_t u = t; u < next_issue; ++u)
      (void)mbar_wait_bounded(&full_bar[u % STAGES], static_cast<uint32_t>((u / STAGES) & 1),
                              kWaitLimitNs);
  }
}

// ------------------------------------------------------------ config registry

namespace {

template <int QT, int RT, int TQ, int TR, int STAGES, int MINB>
cudaError_t launch_cfg(const JobParams &p, uint16_t *scratch, DevStatus *status,
                       const volatile int *cancel, int grid, cudaStream_t stream) {
  using S = TileShape<QT, RT, TQ, TR, STAGES>;
  auto kern = dist_tiles_kernel<QT, RT, TQ, TR, STAGES, MINB>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         S::kSmemBytes);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  kern<<<grid, S::kThreads, S::kSmemBytes, stream>>>(p, scratch, status, cancel);
  return cudaGetLastError();
}

template <int QT, int RT, int TQ, int TR, int STAGES, int MINB>
int occupancy_cfg() {
  using S = TileShape<QT, RT, TQ, TR, STAGES>;
  auto kern = dist_tiles_kernel<QT, RT, TQ, TR, STAGES, MINB>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kSmemBytes) !=
      cudaSuccess)
    return 0;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, S::kThreads, S::kSmemBytes) !=
      cudaSuccess)
    return 0;
  return blocks;
}

template <int QT, int RT, int TQ, int TR, int STAGES, int MINB>
constexpr TileConfig make_cfg(int id) {
  return TileConfig{id,
                    QT,
                    RT,
                    TQ,
                    TR,
                    kMaxKmers,
                    STAGES,
                    TileShape<QT, RT, TQ, TR, STAGES>::kThreads,
                    TileShape<QT, RT, TQ, TR, STAGES>::kSmemBytes,
                    &launch_cfg<QT, RT, TQ, TR, STAGES, MINB>,
                    &occupancy_cfg<QT, RT, TQ, TR, STAGES, MINB>};
}

const TileConfig kConfigs[] = {
    make_cfg<128, 64, 8, 4, 3, 2>(1),   // default: 2 CTAs x 8 warps per SM
    make_cfg<64, 64, 4, 4, 3, 2>(2),    // small tiles, 16 pairs per thread
    make_cfg<128, 128, 8, 8, 3, 1>(3),  // large tiles, 64 pairs per thread, 1 CTA per SM
    make_cfg<64, 64, 8, 4, 4, 3>(4),    // 128 threads, 3 CTAs per SM
    make_cfg<128, 64, 4, 8, 3, 2>(5),   // transposed thread block
    make_cfg<128, 128, 8, 4, 3, 1>(6),  // 512 threads, 16 warps in one CTA
};

}  // namespace

int tile_config_count() { return static_cast<int>(sizeof(kConfigs) / sizeof(kConfigs[0])); }

const TileConfig *tile_config(int id) {
  for (const TileConfig &c : kConfigs)
    if (c.id == id) return &c;
  return nullptr;
}

}  // namespace sk
