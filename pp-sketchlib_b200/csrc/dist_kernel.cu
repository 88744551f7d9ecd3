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

template <int QT, int RT, int TQ, int TR, int KMAX, int STAGES>
struct TileShape {
  static constexpr int kThreads = (QT / TQ) * (RT / TR);
  static constexpr int kQG = QT / kGranule;
  static constexpr int kRG = RT / kGranule;
  static constexpr int kStageQWords = kBlocksPerStage * kQG * kStripeWords;
  static constexpr int kStageRWords = kBlocksPerStage * kRG * kStripeWords;
  static constexpr int kStageBytes = (kStageQWords + kStageRWords) * 4;
  static constexpr int kCountBytes = KMAX * QT * RT * 2;
  static constexpr int kSmemBytes = STAGES * kStageBytes + kCountBytes;
  static_assert(QT % kGranule == 0 && RT % kGranule == 0, "tiles are whole granules");
  static_assert(kGranule % TQ == 0 && kGranule % TR == 0, "thread blocks stay in a granule");
  static_assert(TQ % 4 == 0 && TR % 4 == 0, "128-bit shared loads");
  static_assert(QT % RT == 0, "triangular map needs tile_rows multiple of tile_cols");
};

template <int QT, int RT, int TQ, int TR, int KMAX, int STAGES>
__global__ void __launch_bounds__((QT / TQ) * (RT / TR), 1)
    dist_tiles_kernel(const JobParams p, DevStatus *status, const volatile int *cancel) {
  using S = TileShape<QT, RT, TQ, TR, KMAX, STAGES>;
  constexpr int NT = S::kThreads;
  constexpr int TCOLS = RT / TR;

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t *sq = reinterpret_cast<uint32_t *>(smem);
  uint32_t *sr = sq + STAGES * S::kStageQWords;
  uint16_t *scnt = reinterpret_cast<uint16_t *>(sr + STAGES * S::kStageRWords);
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
          for (int j = 0; j < TR; ++j) cnt[i][j] += __popc(acc[i][j]);
      }
    }

    const int64_t local = t % spt;
    const int64_t kidx = local / steps_per_k;
    if (local - kidx * steps_per_k == steps_per_k - 1) {
      // all blocks of k-mer index kidx done: park the counts in shared memory
      uint16_t *dst = scnt + kidx * (QT * RT);
#pragma unroll
      for (int i = 0; i < TQ; ++i)
#pragma unroll
        for (int j = 0; j < TR; ++j) {
          dst[(row0 + i) * RT + col0 + j] = static_cast<uint16_t>(cnt[i][j]);
          cnt[i][j] = 0;
        }
    }
    __syncthreads();  // stage s fully read; counts of kidx visible
    if (s_abort) break;
    if (tid == 0 && next_issue < total) issue(next_issue++);

    if (local == spt - 1) {
      // tile complete: epilogue over all pairs of the tile
      int32_t ti, tj;
      tile_coords(p, blockIdx.x + (t / spt) * gridDim.x, ti, tj);
      const int64_t gi0 = static_cast<int64_t>(ti) * QT;
      const int64_t gj0 = static_cast<int64_t>(tj) * RT;
      for (int pidx = tid; pidx < QT * RT; pidx += NT) {
        const int64_t gi = gi0 + pidx / RT;
        const int64_t gj = gj0 + pidx % RT;
        const bool valid = p.self ? (gj > gi && gj < p.n_cols) : (gi < p.n_rows && gj < p.n_cols);
        if (valid) finish_pair<KMAX>(p, gi, gj, scnt + pidx, QT * RT);
      }
      if (tid == 0) {
        atomicAdd(&status->tiles_done, 1ull);
        if (cancel != nullptr && *cancel != 0) {
          s_abort = 1;
          atomicOr(&status->error, 2u);
        }
      }
      __syncthreads();  // counts consumed before the next tile overwrites them
      if (s_abort) break;
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

template <int QT, int RT, int TQ, int TR, int KMAX, int STAGES>
cudaError_t launch_cfg(const JobParams &p, DevStatus *status, const volatile int *cancel,
                       int grid, cudaStream_t stream) {
  using S = TileShape<QT, RT, TQ, TR, KMAX, STAGES>;
  auto kern = dist_tiles_kernel<QT, RT, TQ, TR, KMAX, STAGES>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         S::kSmemBytes);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  kern<<<grid, S::kThreads, S::kSmemBytes, stream>>>(p, status, cancel);
  return cudaGetLastError();
}

template <int QT, int RT, int TQ, int TR, int KMAX, int STAGES>
int occupancy_cfg() {
  using S = TileShape<QT, RT, TQ, TR, KMAX, STAGES>;
  auto kern = dist_tiles_kernel<QT, RT, TQ, TR, KMAX, STAGES>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kSmemBytes) !=
      cudaSuccess)
    return 0;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, S::kThreads, S::kSmemBytes) !=
      cudaSuccess)
    return 0;
  return blocks;
}

template <int QT, int RT, int TQ, int TR, int KMAX, int STAGES>
constexpr TileConfig make_cfg(int id) {
  return TileConfig{id,
                    QT,
                    RT,
                    TQ,
                    TR,
                    KMAX,
                    STAGES,
                    TileShape<QT, RT, TQ, TR, KMAX, STAGES>::kThreads,
                    TileShape<QT, RT, TQ, TR, KMAX, STAGES>::kSmemBytes,
                    &launch_cfg<QT, RT, TQ, TR, KMAX, STAGES>,
                    &occupancy_cfg<QT, RT, TQ, TR, KMAX, STAGES>};
}

const TileConfig kConfigs[] = {
    make_cfg<128, 64, 8, 4, 8, 3>(1),   // default for K <= 8
    make_cfg<64, 64, 4, 4, 16, 3>(2),   // K <= 16
    make_cfg<128, 128, 8, 8, 4, 3>(3),  // K <= 4, largest tile
    make_cfg<64, 64, 8, 4, 16, 3>(4),   // K <= 16, 128 threads
    make_cfg<128, 64, 4, 8, 8, 3>(5),   // K <= 8, transposed thread block
    make_cfg<64, 64, 4, 4, 8, 4>(6),    // K <= 8, small tiles for small problems
};

}  // namespace

int tile_config_count() { return static_cast<int>(sizeof(kConfigs) / sizeof(kConfigs[0])); }

const TileConfig *tile_config(int id) {
  for (const TileConfig &c : kConfigs)
    if (c.id == id) return &c;
  return nullptr;
}

}  // namespace sk
