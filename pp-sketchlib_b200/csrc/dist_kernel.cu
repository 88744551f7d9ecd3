// dist_kernel.cu -- the fused bit-sliced MinHash distance kernel for sm_100a.
//
// A persistent kernel: every CTA pulls work items (job, tile, k range) from a
// device queue, so one launch can serve one all-vs-all, one query batch or a
// whole batch of unrelated databases of different sizes, k sets and sketch
// widths.  Thread 0 is the producer: for every 2-block step of its current
// item it stages the 14 bit planes of the tile's row and column samples into
// shared memory with bulk copies (TMA engine, one copy per 64-sample stripe,
// mbarrier completion) and records the step in a per-stage descriptor.  All
// warps consume: each thread intersects a TQ x TR register block of pairs
//     acc = AND over planes of ~(row_word ^ col_word)   (one LOP3 per plane)
//     count += popc(acc)                                 (POPC + IMAD)
// which is calc_intersize (src/dist/dist.cpp:50-78) for 32 bins at a time,
// releases the stage with a per-stage named barrier (only the step's refill
// warp, rotating over the SM's sub-partitions, waits on it and issues the
// next copies), parks its per-k counts in L2-resident scratch, and
// after an item's last k turns its own pairs into random-corrected Jaccards
// and the log-linear core/accessory fit, written straight to the long form.
//
// Replaces calculate_dists (src/gpu/dist.cu:164-317): one thread per pair with
// strided 8-byte global loads there; register-blocked tiles over staged
// stripes here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "sk_device.cuh"
#include "sk_launch.h"

namespace sk {

constexpr int kBlocksPerStage = 2;   // 32-bin blocks per pipeline stage
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s bounded waits

// Per-stage step descriptor written by the producer before it arms the stage.
struct StepMeta {
  int32_t job;
  int32_t ti, tj;     // tile coordinates within the job
  int32_t kidx;       // count slot of this step: k-mer index x nchunk + chunk
  int32_t flags;      // kStepEnd / kStepLastOfK (last step of a count slot) / kStepLastOfItem
  int32_t split;      // split slot of the item, -1 for whole tiles
  int32_t nparts;
  int32_t nbpart;     // block ranges per k of the item's tile (count slots per k)
};
constexpr int32_t kStepEnd = 1, kStepLastOfK = 2, kStepLastOfItem = 4;

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
  static_assert(STAGES >= 2 && STAGES <= 8, "one named barrier (ids 1..8) per stage");
  static_assert(kThreads % 32 == 0, "whole warps");
};

// Per-stage named barriers 1..STAGES with literal ids (the hardware reserves
// only the ids a kernel names, so each instance names only its own).
template <int NT, int STAGES>
__device__ __forceinline__ void stage_sync(int s) {
  switch (s) {
    case 0: asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory"); break;
    case 1: if constexpr (STAGES > 1) asm volatile("bar.sync 2, %0;" ::"n"(NT) : "memory"); break;
    case 2: if constexpr (STAGES > 2) asm volatile("bar.sync 3, %0;" ::"n"(NT) : "memory"); break;
    case 3: if constexpr (STAGES > 3) asm volatile("bar.sync 4, %0;" ::"n"(NT) : "memory"); break;
    case 4: if constexpr (STAGES > 4) asm volatile("bar.sync 5, %0;" ::"n"(NT) : "memory"); break;
    case 5: if constexpr (STAGES > 5) asm volatile("bar.sync 6, %0;" ::"n"(NT) : "memory"); break;
    case 6: if constexpr (STAGES > 6) asm volatile("bar.sync 7, %0;" ::"n"(NT) : "memory"); break;
    case 7: if constexpr (STAGES > 7) asm volatile("bar.sync 8, %0;" ::"n"(NT) : "memory"); break;
  }
}
template <int NT, int STAGES>
__device__ __forceinline__ void stage_arrive(int s) {
  switch (s) {
    case 0: asm volatile("bar.arrive 1, %0;" ::"n"(NT) : "memory"); break;
    case 1: if constexpr (STAGES > 1) asm volatile("bar.arrive 2, %0;" ::"n"(NT) : "memory"); break;
    case 2: if constexpr (STAGES > 2) asm volatile("bar.arrive 3, %0;" ::"n"(NT) : "memory"); break;
    case 3: if constexpr (STAGES > 3) asm volatile("bar.arrive 4, %0;" ::"n"(NT) : "memory"); break;
    case 4: if constexpr (STAGES > 4) asm volatile("bar.arrive 5, %0;" ::"n"(NT) : "memory"); break;
    case 5: if constexpr (STAGES > 5) asm volatile("bar.arrive 6, %0;" ::"n"(NT) : "memory"); break;
    case 6: if constexpr (STAGES > 6) asm volatile("bar.arrive 7, %0;" ::"n"(NT) : "memory"); break;
    case 7: if constexpr (STAGES > 7) asm volatile("bar.arrive 8, %0;" ::"n"(NT) : "memory"); break;
  }
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Count scratch layout (per CTA slot, and per split slot): [k][threads][pairs
// per thread] uint16; a thread writes and reads back only its own entries.
// ROT: the refill duty (wait for every warp on the stage barrier, then issue
// the next copies) moves round-robin over warps 0..ROT-1, one per SM
// sub-partition for ROT = 4, so no scheduler carries all of it.
// WIDE: the instance for jobs with more than kNarrowKmers k-mer lengths or
// sketches counted in chunks (one count slot per chunk of kMaxChunkBlocks
// blocks); the narrow instance keeps one slot per k and the unrolled
// epilogues, whose code size the hot loop is sensitive to.
template <int QT, int RT, int TQ, int TR, int STAGES, int MINB, int ROT, bool WIDE>
__global__ void __launch_bounds__((QT / TQ) * (RT / TR), MINB)
    dist_items_kernel(const LaunchParams lp) {
  using S = TileShape<QT, RT, TQ, TR, STAGES>;
  constexpr int NT = S::kThreads;
  constexpr int PT = S::kPairsPerThread;
  static_assert(ROT >= 1 && ROT <= NT / 32, "refill warps must exist");
  constexpr int TCOLS = RT / TR;

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t *sq = reinterpret_cast<uint32_t *>(smem);
  uint32_t *sr = sq + STAGES * S::kStageQWords;
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ StepMeta meta[STAGES];
  __shared__ int s_abort;

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int tq = tid / TCOLS;
  const int tr = tid % TCOLS;
  const int row0 = tq * TQ;   // first tile row of this thread
  const int col0 = tr * TR;   // first tile column of this thread
  const int64_t slot_k_stride = static_cast<int64_t>(NT) * PT;      // uint16 between k slots
  const int64_t slot_size = slot_k_stride * lp.k_slots;
  uint16_t *my_counts = lp.cta_scratch + blockIdx.x * slot_size + static_cast<int64_t>(tid) * PT;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&full_bar[s], 1);
    fence_mbar_init();
    s_abort = 0;
  }
  __syncthreads();

  // ---------------------------------------------------------------- producer
  // (thread 0 only)  Its state lives in shared memory so the consumer loop
  // keeps its registers for the pair block.
  struct Producer {
    const uint32_t *rows, *cols;
    int32_t done, have, job, ti, tj, k, k1, split, nparts, b0, nb, ngr, ngc;
    int32_t slot, slot_end, chunk_nb;   // count slot of the step, its last block + 1
    int32_t bstart, bend, bpart, nbpart;  // the item's block range of each k
  };
  __shared__ Producer ps;
  if (tid == 0) {
    ps.done = 0;
    ps.have = 0;
  }

  // fills stage s with the next step of the stream (called in step order)
  auto produce = [&](int s) {
    if (ps.done) return;
    if (s_abort != 0) {   // a consumer timed out: end the stream now
      meta[s].flags = kStepEnd;
      mbar_arrive(&full_bar[s]);
      ps.done = 1;
      return;
    }
    if (!ps.have) {
      const bool cancelled = lp.cancel != nullptr && *lp.cancel != 0;
      if (cancelled) atomicOr(&lp.status->error, 2u);
      const unsigned long long idx = cancelled ? ~0ull : atomicAdd(lp.item_counter, 1ull);
      if (idx >= static_cast<unsigned long long>(lp.n_items)) {
        meta[s].flags = kStepEnd;
        mbar_arrive(&full_bar[s]);   // completes the phase without data
        ps.done = 1;
        return;
      }
      const WorkItem it = lp.items[idx];
      const JobParams &jp = lp.jobs[it.job];
      ps.job = it.job;
      int32_t ti, tj;
      tile_coords(jp, it.tile, ti, tj);
      ps.ti = ti;
      ps.tj = tj;
      ps.k = it.k0;
      ps.k1 = it.k1;
      ps.split = it.split;
      ps.nparts = it.nparts;
      ps.nb = jp.nb;
      ps.bstart = it.b1 ? it.b0 : 0;
      ps.bend = it.b1 ? it.b1 : jp.nb;
      ps.bpart = it.bpart;
      ps.nbpart = it.nbpart > 1 ? it.nbpart : 1;
      ps.b0 = WIDE ? 0 : ps.bstart;
      ps.rows = jp.row_words;
      ps.cols = jp.col_words;
      ps.ngr = jp.ng_rows;
      ps.ngc = jp.ng_cols;
      if constexpr (WIDE) {
        ps.slot = it.k0 * jp.nchunk;
        ps.chunk_nb = jp.chunk_nb;
        ps.slot_end = jp.chunk_nb;   // chunk_nb == nb when one slot holds a whole k
      }
      ps.have = 1;
      atomicAdd(&lp.status->tiles_done, 1ull);
    }
    // slot ends fall on step boundaries (chunk_nb and nb are even)
    const bool last_of_slot = WIDE ? ps.b0 + kBlocksPerStage >= ps.slot_end
                                   : ps.b0 + kBlocksPerStage >= ps.bend;
    const bool last_of_k = WIDE ? last_of_slot && ps.slot_end >= ps.nb : last_of_slot;
    const bool last_of_item = last_of_k && ps.k + 1 >= ps.k1;
    StepMeta &m = meta[s];
    m.job = ps.job;
    m.ti = ps.ti;
    m.tj = ps.tj;
    m.kidx = WIDE ? ps.slot : ps.k * ps.nbpart + ps.bpart;
    m.nbpart = WIDE ? 1 : ps.nbpart;
    m.flags = (last_of_slot ? kStepLastOfK : 0) | (last_of_item ? kStepLastOfItem : 0);
    m.split = ps.split;
    m.nparts = ps.nparts;
    mbar_arrive_expect_tx(&full_bar[s], S::kStageBytes);
#pragma unroll
    for (int b = 0; b < kBlocksPerStage; ++b) {
      const int64_t blk = static_cast<int64_t>(ps.k) * ps.nb + ps.b0 + b;
      const uint32_t *src_q =
          ps.rows + ((blk * ps.ngr) + static_cast<int64_t>(ps.ti) * S::kQG) * kStripeWords;
      const uint32_t *src_r =
          ps.cols + ((blk * ps.ngc) + static_cast<int64_t>(ps.tj) * S::kRG) * kStripeWords;
      bulk_g2s(sq + (s * kBlocksPerStage + b) * S::kQG * kStripeWords, src_q,
               S::kQG * kStripeBytes, &full_bar[s]);
      bulk_g2s(sr + (s * kBlocksPerStage + b) * S::kRG * kStripeWords, src_r,
               S::kRG * kStripeBytes, &full_bar[s]);
    }
    ps.b0 += kBlocksPerStage;
    if constexpr (WIDE) {
      if (last_of_slot) {
        ++ps.slot;
        if (last_of_k) {
          ps.b0 = 0;
          ++ps.k;
          ps.slot_end = ps.chunk_nb;
          if (last_of_item) ps.have = 0;
        } else {
          ps.slot_end = min(ps.slot_end + ps.chunk_nb, ps.nb);
        }
      }
    } else if (last_of_k) {
      ps.b0 = ps.bstart;
      ++ps.k;
      if (last_of_item) ps.have = 0;
    }
  };

  if (tid == 0) {
    for (int u = 0; u < STAGES; ++u) produce(u);
  }

  // ---------------------------------------------------------------- consumers
  // Counts of one k for columns 2c and 2c + 1 share a register (low / high
  // 16 bits): at most 64 * sketchsize64 <= 65,472 per k, so the low half never
  // carries.  `one` is 1 at run time, which keeps the count multiply-adds on
  // the FMA pipe and the ALU free for the LOP3s.
  const uint32_t one = lp.jobs[0].one;
  const uint32_t hi_one = one << 16;
  uint32_t cnt[TQ][TR / 2];
#pragma unroll
  for (int i = 0; i < TQ; ++i)
#pragma unroll
    for (int j = 0; j < TR / 2; ++j) cnt[i][j] = 0;

  int s = 0;              // stage of step t
  uint32_t parity = 0;    // phase parity of step t on that stage
  for (uint32_t t = 0;; ++t) {
    StepMeta m;
    if (mbar_wait_bounded(&full_bar[s], parity, kWaitLimitNs)) {
      m = meta[s];
      if (m.flags & kStepEnd) break;
    } else {
      // a stage never landed: record it and keep to the protocol without
      // computing; the producer ends the stream at its next step, so every
      // warp still arrives at every stage barrier and the loop ends
      s_abort = 1;
      atomicOr(&lp.status->error, 1u);
      lp.status->where = 1;
      m.flags = 0;
      m.split = -1;
    }

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
        // column words before row words: measured 0.3% faster than the reverse
#pragma unroll
        for (int j = 0; j < TR; j += 4) {
          const uint4 v = *reinterpret_cast<const uint4 *>(rb + pl * kGranule + j);
          rv[j] = v.x; rv[j + 1] = v.y; rv[j + 2] = v.z; rv[j + 3] = v.w;
        }
#pragma unroll
        for (int i = 0; i < TQ; i += 4) {
          const uint4 v = *reinterpret_cast<const uint4 *>(qb + pl * kGranule + i);
          qv[i] = v.x; qv[i + 1] = v.y; qv[i + 2] = v.z; qv[i + 3] = v.w;
        }
        // column-major issue order: measured 0.5% faster than row-major
#pragma unroll
        for (int j = 0; j < TR; ++j)
#pragma unroll
          for (int i = 0; i < TQ; ++i)
            acc[i][j] = pl == 0 ? lop_eq(qv[i], rv[j]) : lop_eq_and(acc[i][j], qv[i], rv[j]);
      }
#pragma unroll
      for (int i = 0; i < TQ; ++i)
#pragma unroll
        for (int j = 0; j < TR / 2; ++j)
          cnt[i][j] = mad_u32(__popc(acc[i][2 * j + 1]), hi_one,
                              mad_u32(__popc(acc[i][2 * j]), one, cnt[i][j]));
    }

    // release the stage: the refill warp of this step waits for every warp
    // and refills it with step t + STAGES; the others only arrive and run
    // ahead into the stages already armed.  A warp arrives at barrier s for
    // step t + STAGES only after that refill armed it, so barrier
    // generations never mix, and the producer state written by one refill
    // is published to the next refill warp by the barrier itself.
    const int refill_warp = ROT > 1 ? static_cast<int>(t % ROT) : 0;
    if (warp == refill_warp) {
      stage_sync<NT, STAGES>(s);
      if (lane == 0) produce(s);
    } else {
      stage_arrive<NT, STAGES>(s);
    }
    if (++s == STAGES) {
      s = 0;
      parity ^= 1u;
    }

    if (m.flags & kStepLastOfK) {
      // counts of count slot m.kidx done: park them (own slot or split slot)
      uint16_t *base = m.split >= 0
                           ? lp.split_scratch + m.split * slot_size + static_cast<int64_t>(tid) * PT
                           : my_counts;
      // pair q = i * TR + j is uint16 q of the slot: word q / 2 = cnt[i][j / 2]
      uint4 *dst = reinterpret_cast<uint4 *>(base + m.kidx * slot_k_stride);
      constexpr int CW = TR / 2;
#pragma unroll
      for (int w = 0; w < PT / 8; ++w)
        dst[w] = make_uint4(cnt[(4 * w) / CW][(4 * w) % CW], cnt[(4 * w + 1) / CW][(4 * w + 1) % CW],
                            cnt[(4 * w + 2) / CW][(4 * w + 2) % CW],
                            cnt[(4 * w + 3) / CW][(4 * w + 3) % CW]);
#pragma unroll
      for (int i = 0; i < TQ; ++i)
#pragma unroll
        for (int j = 0; j < TR / 2; ++j) cnt[i][j] = 0;
    }

    if (m.flags & kStepLastOfItem) {
      const JobParams &jp = lp.jobs[m.job];
      bool finish = true;
      if (m.split >= 0) {
        // Split tile: every thread owns its pairs' counts, so each thread
        // counts its own arrivals; the thread of the last part to arrive
        // gathers all k from the split slot and finishes those pairs.  No
        // CTA-wide barrier, so a stage that timed out cannot strand a warp.
        __threadfence();
        const unsigned int prev =
            atomicAdd(&lp.split_done[static_cast<int64_t>(m.split) * NT + tid], 1u);
        finish = prev + 1 == static_cast<unsigned int>(m.nparts);
        if (finish) {
          __threadfence();
          const uint4 *src = reinterpret_cast<const uint4 *>(
              lp.split_scratch + m.split * slot_size + static_cast<int64_t>(tid) * PT);
          if (WIDE || m.nbpart == 1) {
            const int slots = WIDE ? job_slots(jp) : jp.n_kmers;
            for (int k = 0; k < slots; ++k)
#pragma unroll
              for (int w = 0; w < PT / 8; ++w)
                reinterpret_cast<uint4 *>(my_counts + k * slot_k_stride)[w] =
                    __ldcg(src + k * (slot_k_stride / 8) + w);
          } else {
            // block ranges of one k: partial counts add up (two 16-bit
            // counts per word never carry: their sums fit 16 bits)
            for (int k = 0; k < jp.n_kmers; ++k)
#pragma unroll
              for (int w = 0; w < PT / 8; ++w) {
                uint4 acc = __ldcg(src + (k * m.nbpart) * (slot_k_stride / 8) + w);
                for (int p = 1; p < m.nbpart; ++p) {
                  const uint4 v = __ldcg(src + (k * m.nbpart + p) * (slot_k_stride / 8) + w);
                  acc.x += v.x; acc.y += v.y; acc.z += v.z; acc.w += v.w;
                }
                reinterpret_cast<uint4 *>(my_counts + k * slot_k_stride)[w] = acc;
              }
          }
        }
      }
      if (finish) {
        const int64_t gi0 = static_cast<int64_t>(m.ti) * QT + row0;
        const int64_t gj0 = static_cast<int64_t>(m.tj) * RT + col0;
#pragma unroll 1
        for (int q = 0; q < PT; ++q) {
          const int64_t gi = gi0 + q / TR;
          const int64_t gj = gj0 + q % TR;
          const bool valid =
              jp.self ? (gj > gi && gj < jp.n_cols) : (gi < jp.n_rows && gj < jp.n_cols);
          if (valid)
            finish_pair_any<WIDE>(jp, gi, gj, my_counts + q, static_cast<int>(slot_k_stride));
        }
      }
    }
  }
}

// ------------------------------------------------------------ config registry

namespace {

// Raises the instance's dynamic shared memory limit once (before any launch,
// so never inside a stream capture).
template <int QT, int RT, int TQ, int TR, int STAGES, int MINB, int ROT, bool WIDE>
cudaError_t ensure_smem_attr() {
  using S = TileShape<QT, RT, TQ, TR, STAGES>;
  static cudaError_t status = cudaFuncSetAttribute(
      dist_items_kernel<QT, RT, TQ, TR, STAGES, MINB, ROT, WIDE>,
      cudaFuncAttributeMaxDynamicSharedMemorySize, S::kSmemBytes);
  return status;
}

template <int QT, int RT, int TQ, int TR, int STAGES, int MINB, int ROT>
cudaError_t launch_cfg(const LaunchParams &lp, int grid, cudaStream_t stream) {
  using S = TileShape<QT, RT, TQ, TR, STAGES>;
  if (lp.wide) {
    cudaError_t e = ensure_smem_attr<QT, RT, TQ, TR, STAGES, MINB, ROT, true>();
    if (e != cudaSuccess) return e;
    dist_items_kernel<QT, RT, TQ, TR, STAGES, MINB, ROT, true>
        <<<grid, S::kThreads, S::kSmemBytes, stream>>>(lp);
  } else {
    cudaError_t e = ensure_smem_attr<QT, RT, TQ, TR, STAGES, MINB, ROT, false>();
    if (e != cudaSuccess) return e;
    dist_items_kernel<QT, RT, TQ, TR, STAGES, MINB, ROT, false>
        <<<grid, S::kThreads, S::kSmemBytes, stream>>>(lp);
  }
  return cudaGetLastError();
}

template <int QT, int RT, int TQ, int TR, int STAGES, int MINB, int ROT, bool WIDE>
int occupancy_one() {
  using S = TileShape<QT, RT, TQ, TR, STAGES>;
  if (ensure_smem_attr<QT, RT, TQ, TR, STAGES, MINB, ROT, WIDE>() != cudaSuccess) return 0;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &blocks, dist_items_kernel<QT, RT, TQ, TR, STAGES, MINB, ROT, WIDE>, S::kThreads,
          S::kSmemBytes) != cudaSuccess)
    return 0;
  return blocks;
}

// Resident CTAs per SM of both instances (a grid sized by it suits either).
template <int QT, int RT, int TQ, int TR, int STAGES, int MINB, int ROT>
int occupancy_cfg() {
  return std::min(occupancy_one<QT, RT, TQ, TR, STAGES, MINB, ROT, false>(),
                  occupancy_one<QT, RT, TQ, TR, STAGES, MINB, ROT, true>());
}

template <int QT, int RT, int TQ, int TR, int STAGES, int MINB, int ROT = 1>
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
                    &launch_cfg<QT, RT, TQ, TR, STAGES, MINB, ROT>,
                    &occupancy_cfg<QT, RT, TQ, TR, STAGES, MINB, ROT>};
}

const TileConfig kConfigs[] = {
    make_cfg<128, 128, 8, 4, 4, 1, 4>(1),  // default: 512 threads, 16 warps, one CTA per SM
    make_cfg<128, 64, 8, 4, 4, 2>(2),   // 256 threads, two CTAs per SM
    make_cfg<64, 64, 4, 4, 4, 2>(3),    // small tiles, 16 pairs per thread
    make_cfg<128, 128, 8, 8, 4, 1>(4),  // 256 threads, 64 pairs per thread
    make_cfg<128, 64, 4, 8, 4, 2>(5),   // transposed thread block
    make_cfg<64, 64, 8, 4, 4, 3>(6),    // 128 threads, three CTAs per SM
};

}  // namespace

int tile_config_count() { return static_cast<int>(sizeof(kConfigs) / sizeof(kConfigs[0])); }

const TileConfig *tile_config(int id) {
  for (const TileConfig &c : kConfigs)
    if (c.id == id) return &c;
  return nullptr;
}

}  // namespace sk
