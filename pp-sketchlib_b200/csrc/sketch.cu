// sketch.cu -- MinHash sketches of sequences on the device: the producer of
// the distance path's input.
//
// The reference sketches on the CPU, one sample and one k at a time
// (sketch(), src/sketch/sketch.cpp:120-168): ntHash rolls along each sequence
// (stHashIterator, src/sketch/stHashIterator.hpp:63-120), each canonical hash
// mod 2^61-1 keeps its bin's minimum (binsign, :69-73), empty bins are filled
// from a probe sequence (densifybin, :93-118) and the low 14 bits of every
// bin become bit planes, 64 bins per word (fillusigs, :82-91).  Here:
//
//   codes      the bases go up as they are (or are read where they lie in
//              device memory) and become one byte per base: 0..3 for A, C, G,
//              T/U in either case, 4 for any other byte, plus kCodeStart on
//              the first base of each sequence.
//   hashing    a work item is (sample, k, range of window starts).  Its CTA
//              keeps the item's bin minima in shared memory; each thread rolls
//              the forward and reverse hashes over its share of the range.  A
//              non-base contributes zero to both hashes, so the roll never
//              restarts: a window is emitted once the bases since the last
//              non-base or sequence start number k, and the hash then equals
//              the reference's freshly initialised one.  The CTA folds its
//              minima into the sample's bins with atomicMin.
//   finishing  one CTA per (sample, k) records bin 0 (inverse_minhash), fills
//              empty bins in the reference's order and writes the bit planes
//              with warp ballots.
//   phased     codon-phased spaced seeds (k bases at positions 0, 3, ...,
//              3(k-1) of a 3k-2 window) are a rolling hash along each of the
//              three phase subsequences: three states rotate, each stepping
//              by a split rotation of three with the base 3k back leaving.
//   counting   with min_count > 0 (read sets), hashes are counted in a device
//              hash table and the insertion that brings a hash's count to
//              min_count enters it in its bin: the reference's exact counter
//              (HashCounter, src/sketch/countmin.cpp:55-72, `exact = true`),
//              whose answer does not depend on read order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "sk_runtime.h"

namespace sk {
namespace {

constexpr uint64_t kSignMod = (1ULL << 61) - 1;   // SIGN_MOD (src/sketch/sketch.cpp:23)
constexpr uint64_t kLo33 = 0x1FFFFFFFFULL;
constexpr uint8_t kCodeInvalid = 4;
constexpr uint8_t kCodeStart = 8;
constexpr int kSketchThreads = 512;
constexpr int kPerThread = 512;                    // window starts per thread, at most
constexpr int64_t kItemWindows = static_cast<int64_t>(kSketchThreads) * kPerThread;
constexpr int kFinishThreads = 512;
constexpr int kMinK = 3;                           // generate_seeds (src/sketch/sketch.cpp:33-40)
constexpr int kMaxK = kMaxKmerLength;
constexpr unsigned long long kEmptyKey = ~0ULL;
// Invalid codes before and after a batch's bases: the roll reads up to
// 16 * ceil(k_out / 16) bytes before a range and its window length + 31
// bytes after it (k_out and the window length are 3k and 3k - 2 for
// codon-phased seeds, k <= 255).
constexpr int64_t kCodePad = 1024;
constexpr unsigned kErrDensify = 4u;               // DevStatus.error bits of the sketcher
constexpr unsigned kErrTable = 8u;

// ntHash per-base seeds for A, C, G, T (ntHash, Mohamadi et al. 2016; the
// values of the reference's src/sketch/nthash_tables.hpp:25-29).
constexpr uint64_t kNtSeed[4] = {0x3c8bfbb395c60474ULL, 0x3193c18562a02b4cULL,
                                 0x20323ed082572324ULL, 0x295549f54be24456ULL};

// ntHash's split rotation: the low 33 bits and the high 31 bits of the hash
// rotate independently (src/sketch/nthash.hpp:17-55); used on the host to
// build the rolling tables.
__host__ __device__ __forceinline__ uint64_t srol1(uint64_t v) {
  const uint64_t lo = v & kLo33, hi = v & ~kLo33;
  return (((lo << 1) | (lo >> 32)) & kLo33) | ((hi << 1) & ~kLo33) | ((hi >> 30) & (1ULL << 33));
}

// The same rotations on the two 32-bit halves of the hash: low word L holds
// bits 0..31, high word H bit 0 is bit 32 (the top of the 33-bit part) and
// bits 1..31 the 31-bit part.
__device__ __forceinline__ uint64_t srol1_w(uint64_t v) {
  const uint32_t L = static_cast<uint32_t>(v), H = static_cast<uint32_t>(v >> 32);
  const uint32_t lo = __funnelshift_l(H << 31, L, 1);     // L << 1 | bit 32
  const uint32_t f = __funnelshift_l(L, H, 1);            // H << 1 | bit 31
  const uint32_t hi = (f & ~2u) | ((H >> 30) & 2u);        // bit 33 <- bit 63
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

__device__ __forceinline__ uint64_t sror1_w(uint64_t v) {
  const uint32_t L = static_cast<uint32_t>(v), H = static_cast<uint32_t>(v >> 32);
  const uint32_t lo = __funnelshift_r(L, H, 1);           // L >> 1 | bit 32 << 31
  const uint32_t t = __funnelshift_r(H, H, 1);
  const uint32_t hi = (t & 0x7FFFFFFEu) | (L & 1u) | ((H & 2u) << 30);   // bit 32 <- bit 0, bit 63 <- bit 33
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

// Split rotation by three positions (one step of a codon phase).
__device__ __forceinline__ uint64_t srol3(uint64_t v) {
  const uint64_t lo = v & kLo33, hi = v >> 33;
  return ((((hi << 3) | (hi >> 28)) & 0x7FFFFFFFULL) << 33) | (((lo << 3) | (lo >> 30)) & kLo33);
}

__device__ __forceinline__ uint64_t sror3(uint64_t v) {
  const uint64_t lo = v & kLo33, hi = v >> 33;
  return ((((hi >> 3) | (hi << 28)) & 0x7FFFFFFFULL) << 33) | (((lo >> 3) | (lo << 30)) & kLo33);
}

uint64_t srol_n(uint64_t v, unsigned n) {
  for (unsigned i = 0; i < n % (33ULL * 31ULL); ++i) v = srol1(v);
  return v;
}

struct SketchItem {
  int64_t begin, end;     // window starts, offsets into the code buffer
  int32_t row;            // sample * K + k index (bins row)
  int32_t k;
  int32_t tab;            // k index (table row)
  int32_t per;            // window starts per thread (a multiple of 16, at most kPerThread)
};

// Rolling table of one k, indexed by (entering base | leaving base << 3):
// the XOR of seed[in] and srol^n(seed[out]) for the forward hash and of
// srol^n(seed[3-in]) and seed[3-out] for the reverse one, n = k (dense
// seeds) or 3k (codon-phased seeds: the hash of one phase's subsequence
// rolls three positions per step); a code of 4 (not a base) contributes
// zero.
struct RollTable {
  ulonglong2 v[64];
};

RollTable make_table(int k, bool phased) {
  const unsigned n = static_cast<unsigned>(phased ? 3 * k : k);
  uint64_t fin[8] = {}, rin[8] = {}, fout[8] = {}, rout[8] = {};
  for (int c = 0; c < 4; ++c) {
    fin[c] = kNtSeed[c];
    rin[c] = srol_n(kNtSeed[3 - c], n);
    fout[c] = srol_n(kNtSeed[c], n);
    rout[c] = kNtSeed[3 - c];
  }
  RollTable t{};
  for (int ci = 0; ci < 8; ++ci)
    for (int co = 0; co < 8; ++co)
      t.v[ci | (co << 3)] = make_ulonglong2(fin[ci] ^ fout[co], rin[ci] ^ rout[co]);
  return t;
}

__device__ __forceinline__ uint64_t mod_sign(uint64_t h) {
  const uint64_t r = (h & kSignMod) + (h >> 61);
  return r >= kSignMod ? r - kSignMod : r;
}

// sign / binsize exactly: magic = floor((2^64-1) / binsize) under-estimates
// the quotient by less than one for sign < 2^61 (by under sign / 2^64 <= 1/8).
// magic < 2^32 (the host refuses wider: it is about 8 x the bin count), so
// the high half of sign * magic is (hi(sign) * magic + umulhi(lo(sign),
// magic)) >> 32, two multiplies; the quotient is below the bin count and
// q * hi(binsize) below 2^29, so q * binsize needs two more.
__device__ __forceinline__ uint32_t bin_of(uint64_t sign, uint64_t binsize, uint64_t magic) {
  const uint32_t m = static_cast<uint32_t>(magic);
  const uint32_t s_lo = static_cast<uint32_t>(sign), s_hi = static_cast<uint32_t>(sign >> 32);
  const uint64_t t = static_cast<uint64_t>(s_hi) * m + __umulhi(s_lo, m);
  uint32_t q = static_cast<uint32_t>(t >> 32);
  const uint64_t qb = static_cast<uint64_t>(q) * static_cast<uint32_t>(binsize) +
                      (static_cast<uint64_t>(q * static_cast<uint32_t>(binsize >> 32)) << 32);
  if (sign - qb >= binsize) ++q;
  return q;
}

__device__ __forceinline__ uint8_t base_code(uint8_t c) {
  const uint8_t l = c | 0x20;   // letters to lower case
  return l == 'a' ? 0 : l == 'c' ? 1 : l == 'g' ? 2 : (l == 't' || l == 'u') ? 3 : kCodeInvalid;
}

// Base codes of n bytes, src -> dst (the same buffer when converting in place).
__global__ void codes_kernel(const uint8_t *src, uint8_t *dst, int64_t n) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t first = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  int64_t done = 0;
  if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
    const int64_t nv = n / 16;
    const uint4 *vs = reinterpret_cast<const uint4 *>(src);
    uint4 *vd = reinterpret_cast<uint4 *>(dst);
    for (int64_t i = first; i < nv; i += stride) {
      const uint4 x = vs[i];
      uint32_t w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        uint32_t o = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) o |= static_cast<uint32_t>(base_code((w[j] >> (8 * b)) & 0xFF)) << (8 * b);
        w[j] = o;
      }
      vd[i] = make_uint4(w[0], w[1], w[2], w[3]);
    }
    done = nv * 16;
  }
  for (int64_t i = done + first; i < n; i += stride) dst[i] = base_code(src[i]);
}

// Flags the first base of sequences 0 .. n_seqs-1; seq_off[i] - base is the
// sequence's offset in the code buffer.
__global__ void mark_starts_kernel(uint8_t *__restrict__ codes, const int64_t *__restrict__ seq_off,
                                   int64_t n_seqs, int64_t base) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n_seqs; i += stride) {
    const int64_t a = seq_off[i] - base, b = seq_off[i + 1] - base;
    if (b > a) codes[a] |= kCodeStart;
  }
}

// Per-sample densify flags from the per-(sample, k) densify results.
__global__ void densified_kernel(const int8_t *__restrict__ rows, int64_t n, int K,
                                 uint8_t *__restrict__ out) {
  const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (s >= n) return;
  uint8_t any = 0;
  for (int k = 0; k < K; ++k) any |= rows[s * K + k] != 0;
  out[s] = any;
}

// An emitter with a kBatch member takes the hashes of kBatch steps at a time
// (put, then flush): its table probes can then be issued together.
template <typename T, typename = void>
struct is_batched : std::false_type {};
template <typename T>
struct is_batched<T, std::void_t<decltype(T::kBatch)>> : std::true_type {};

// Rolling state: forward and reverse hashes (three of each, one per codon
// phase, for spaced seeds), the count of bases since the last break, and the
// loaded chunks.
struct RollState {
  uint64_t f[3], r[3];
  int run;
  uint4 oa, ob, in;
};

// Sixteen roll steps over one aligned chunk of codes.  `in` holds the bases
// entering at relative positions p0 .. p0+15; the bases leaving (k_out
// earlier) are bytes d .. d+15 of the 32-byte pair (oa, ob), d = (-k_out)
// mod 16, picked with a uniform word select and funnel shift.  kMask: the
// chunk lies within the first k_out positions, where a leaving position
// before the range start contributes nothing.  kRange: some windows ending in
// the chunk start outside [lo, hi).  kRc: canonical hashes (the reverse
// strand is rolled too).  kPhased: codon-phased spaced seeds -- the state of
// the current base's phase takes the step (rotation by three, k_out = 3k)
// and the three states rotate; windows are k_win = 3k - 2 bases.
template <bool kMask, bool kRange, bool kRc, bool kPhased, typename Emit>
__device__ __forceinline__ void roll_chunk(int D, int sh, int p0, int k_out, int k_win, int lo, int hi,
                                           const RollTable &t, RollState &st, Emit &emit) {
  const uint32_t X[8] = {st.oa.x, st.oa.y, st.oa.z, st.oa.w, st.ob.x, st.ob.y, st.ob.z, st.ob.w};
  uint32_t Y[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) Y[m] = D == 0 ? X[m] : D == 1 ? X[m + 1] : D == 2 ? X[m + 2] : X[m + 3];
  uint32_t O[4];
#pragma unroll
  for (int w = 0; w < 4; ++w) O[w] = __funnelshift_r(Y[w], Y[w + 1], sh);
  const uint32_t I[4] = {st.in.x, st.in.y, st.in.z, st.in.w};
  uint32_t IX[4];   // table indices of the 16 steps, four per word
#pragma unroll
  for (int w = 0; w < 4; ++w) IX[w] = (I[w] & 0x07070707u) | ((O[w] & 0x07070707u) << 3);
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const uint32_t ci = (I[i >> 2] >> (8 * (i & 3))) & 0xFF;
    uint32_t idx = (IX[i >> 2] >> (8 * (i & 3))) & 0x3F;
    const int p = p0 + i;
    if (kMask && p < k_out) idx = (idx & 7) | (kCodeInvalid << 3);
    const ulonglong2 v = t.v[idx];
    uint64_t hf, hr = 0;
    if (!kPhased) {
      st.f[0] = hf = srol1_w(st.f[0]) ^ v.x;
      if (kRc) st.r[0] = hr = sror1_w(st.r[0] ^ v.y);
    } else {
      hf = srol3(st.f[0]) ^ v.x;
      st.f[0] = st.f[1];
      st.f[1] = st.f[2];
      st.f[2] = hf;
      if (kRc) {
        hr = sror3(st.r[0] ^ v.y);
        st.r[0] = st.r[1];
        st.r[1] = st.r[2];
        st.r[2] = hr;
      }
    }
    st.run = (ci & 7) == kCodeInvalid ? 0 : ((ci & kCodeStart) ? 1 : min(st.run + 1, k_win));
    const int w = p - k_win + 1;   // start of the window ending at p
    const bool valid = st.run >= k_win && (!kRange || (w >= lo && w < hi));
    if constexpr (is_batched<Emit>::value) {
      emit.put(i % Emit::kBatch, kRc && hr < hf ? hr : hf, valid);
      if (i % Emit::kBatch == Emit::kBatch - 1) emit.flush();
    } else {
      if (valid) emit(kRc && hr < hf ? hr : hf);
    }
  }
}

// Chunks j0 .. j1-1 of a range, each chunk's loads issued one chunk ahead.
template <bool kMask, bool kRange, bool kRc, bool kPhased, typename Emit>
__device__ __forceinline__ void roll_span(const uint4 *base, int j0, int j1, int c, int D, int sh,
                                          int k_out, int k_win, int lo, int hi, const RollTable &t,
                                          RollState &st, Emit &emit) {
  for (int j = j0; j < j1; ++j) {
    const uint4 in_n = base[j + 1], ob_n = base[j + 2 - c];
    roll_chunk<kMask, kRange, kRc, kPhased>(D, sh, 16 * j, k_out, k_win, lo, hi, t, st, emit);
    st.oa = st.ob;
    st.ob = ob_n;
    st.in = in_n;
  }
}

// Calls emit(hash) for every window of k bases (3k - 2 for codon-phased
// seeds) inside one sequence whose start lies in [s, e).  Rolls from s
// rounded down to 16 with a zero state (a non-base contributes zero, so the
// state after k_out positions is the window's hash whatever came before);
// reads the 16-byte chunks of codes from 16 * c bytes before that through
// e + k_win + 31 (the code buffer's pads cover both).  Chunks whose windows
// all start inside [s, e) skip the range test.
template <bool kRc, bool kPhased, typename Emit>
__device__ __forceinline__ void roll_windows(const uint8_t *__restrict__ codes, int64_t s, int64_t e,
                                             int k, const RollTable &t, Emit emit) {
  const int k_out = kPhased ? 3 * k : k, k_win = kPhased ? 3 * k - 2 : k;
  const int64_t s0 = s & ~static_cast<int64_t>(15);
  const int lo = static_cast<int>(s - s0), hi = static_cast<int>(e - s0);
  const int n_chunks = (hi + k_win - 1 + 15) >> 4;
  const int d = (-k_out) & 15, D = d >> 2, sh = 8 * (d & 3);
  const int c = (k_out + d) >> 4;        // the leaving bytes start in chunk j - c
  const uint4 *base = reinterpret_cast<const uint4 *>(codes + s0);
  RollState st{{0, 0, 0}, {0, 0, 0}, 0, base[-c], base[1 - c], base[0]};
  const int masked = min(n_chunks, c);
  // chunk j ends windows starting at 16j - k_win + 1 .. 16j + 16 - k_win
  const int inner0 = max(masked, (lo + k_win - 1 + 15) >> 4);
  const int inner1 = max(inner0, min(n_chunks, (hi + k_win - 1) >> 4));
  roll_span<true, true, kRc, kPhased>(base, 0, masked, c, D, sh, k_out, k_win, lo, hi, t, st, emit);
  roll_span<false, true, kRc, kPhased>(base, masked, inner0, c, D, sh, k_out, k_win, lo, hi, t, st, emit);
  roll_span<false, false, kRc, kPhased>(base, inner0, inner1, c, D, sh, k_out, k_win, lo, hi, t, st, emit);
  roll_span<false, true, kRc, kPhased>(base, inner1, n_chunks, c, D, sh, k_out, k_win, lo, hi, t, st, emit);
}

// One slot of the k-mer count table: key and count share a 16-byte slot, so
// an insertion touches one memory sector.
struct __align__(16) TableSlot {
  unsigned long long key;
  unsigned int count;
  unsigned int pad;
};

__global__ void table_clear_kernel(TableSlot *__restrict__ t, uint64_t n, unsigned int *max_key_count) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
    reinterpret_cast<uint4 *>(t)[i] = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u);
  if (blockIdx.x == 0 && threadIdx.x == 0) *max_key_count = 0;
}

struct SketchArgs {
  const uint8_t *codes;
  const SketchItem *items;
  const RollTable *tables;
  unsigned long long *signs;     // [rows][nbins]
  int nbins;
  int use_rc;
  uint64_t binsize, magic;
  // counting mode
  struct TableSlot *table;       // hash-count table (key kEmptyKey = free)
  uint64_t table_mask;
  unsigned int *max_key_count;   // occurrences of the one hash equal to kEmptyKey
  uint32_t bin_lo, bin_hi;       // bins this pass counts
  unsigned int min_count;        // a hash enters its bin when its count reaches this
  DevStatus *status;
};

// Bin minima of one item; kShared keeps them in shared memory (nbins * 8
// bytes of dynamic shared memory), else the CTA updates the global row.
template <bool kShared, bool kRc, bool kPhased>
__global__ void __launch_bounds__(kSketchThreads, 1)
sketch_kernel(SketchArgs a) {
  extern __shared__ unsigned long long sh_bins[];
  __shared__ RollTable tab;
  const SketchItem it = a.items[blockIdx.x];
  unsigned long long *row = a.signs + static_cast<int64_t>(it.row) * a.nbins;
  unsigned long long *bins = kShared ? sh_bins : row;
  if (kShared)
    for (int i = threadIdx.x; i < a.nbins; i += kSketchThreads) sh_bins[i] = kEmptyKey;
  if (threadIdx.x < 64) {
    const ulonglong2 *src = reinterpret_cast<const ulonglong2 *>(a.tables + it.tab);
    reinterpret_cast<ulonglong2 *>(&tab)[threadIdx.x] = src[threadIdx.x];
  }
  __syncthreads();
  const int64_t s = it.begin + static_cast<int64_t>(threadIdx.x) * it.per;
  const int64_t e = min(s + it.per, it.end);
  if (s < e) {
    const uint64_t binsize = a.binsize, magic = a.magic;
    roll_windows<kRc, kPhased>(a.codes, s, e, it.k, tab, [&](uint64_t h) {
      const uint64_t sign = mod_sign(h);
      const uint32_t q = bin_of(sign, binsize, magic);
      if (sign < bins[q]) atomicMin(bins + q, static_cast<unsigned long long>(sign));
    });
  }
  if (kShared) {
    __syncthreads();
    for (int i = threadIdx.x; i < a.nbins; i += kSketchThreads) {
      const unsigned long long v = sh_bins[i];
      if (v < row[i]) atomicMin(row + i, v);
    }
  }
}

__device__ __forceinline__ uint64_t table_slot(uint64_t h, uint64_t mask) {
  h ^= h >> 33;
  h *= 0xff51afd7ed558ccdULL;
  h ^= h >> 33;
  return h & mask;
}

// The counting pass's emitter: 8 hashes at a time, their first table slots
// loaded together so that 8 independent memory requests per thread are in
// flight, then each insertion resolved (probe, compare-and-swap, count).  The
// insertion that brings a hash's count to min_count puts it in its bin (the
// reference's counter adds a k-mer at the occurrence whose count reaches
// min_count, src/sketch/sketch.cpp:143-148).
struct CountBatch {
  static constexpr int kBatch = 8;
  const SketchArgs &a;
  unsigned long long *row;
  uint64_t h[kBatch];
  bool v[kBatch];

  __device__ __forceinline__ void put(int i, uint64_t hash, bool valid) {
    h[i] = hash;
    v[i] = valid;
  }

  __device__ __forceinline__ void insert(uint64_t hh, uint64_t slot, unsigned long long cur) {
    unsigned int old = 0;
    if (hh == kEmptyKey) {
      old = atomicAdd(a.max_key_count, 1u);
    } else {
      uint64_t probe = 0;
      for (; probe <= a.table_mask; ++probe) {
        TableSlot *t = a.table + slot;
        if (probe > 0) cur = t->key;
        if (cur == kEmptyKey) {
          cur = atomicCAS(&t->key, kEmptyKey, static_cast<unsigned long long>(hh));
          if (cur == kEmptyKey) cur = hh;
        }
        if (cur == hh) {
          old = atomicAdd(&t->count, 1u);
          break;
        }
        slot = (slot + 1) & a.table_mask;
      }
      if (probe > a.table_mask) {
        atomicOr(&a.status->error, kErrTable);   // table full (sized at twice the windows: not reached)
        return;
      }
    }
    if (old + 1 == a.min_count) {
      const uint64_t sign = mod_sign(hh);
      const uint32_t q = bin_of(sign, a.binsize, a.magic);
      if (sign < row[q]) atomicMin(row + q, static_cast<unsigned long long>(sign));
    }
  }

  __device__ __forceinline__ void flush() {
    uint64_t slot[kBatch];
    unsigned long long cur[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      if (v[j]) {   // the pass's bin range
        const uint32_t q = bin_of(mod_sign(h[j]), a.binsize, a.magic);
        v[j] = q >= a.bin_lo && q < a.bin_hi;
      }
      slot[j] = table_slot(h[j], a.table_mask);
    }
#pragma unroll
    for (int j = 0; j < kBatch; ++j) cur[j] = v[j] && h[j] != kEmptyKey ? a.table[slot[j]].key : kEmptyKey;
#pragma unroll
    for (int j = 0; j < kBatch; ++j)
      if (v[j]) insert(h[j], slot[j], cur[j]);
  }
};

// Counting pass: every hash whose bin lies in [bin_lo, bin_hi) is counted.
template <bool kRc, bool kPhased>
__global__ void __launch_bounds__(kSketchThreads, 1)
count_kernel(SketchArgs a) {
  __shared__ RollTable tab;
  const SketchItem it = a.items[blockIdx.x];
  if (threadIdx.x < 64) {
    const ulonglong2 *src = reinterpret_cast<const ulonglong2 *>(a.tables + it.tab);
    reinterpret_cast<ulonglong2 *>(&tab)[threadIdx.x] = src[threadIdx.x];
  }
  __syncthreads();
  const int64_t s = it.begin + static_cast<int64_t>(threadIdx.x) * it.per;
  const int64_t e = min(s + it.per, it.end);
  if (s >= e) return;
  CountBatch emit{a, a.signs + static_cast<int64_t>(it.row) * a.nbins, {}, {}};
  roll_windows<kRc, kPhased>(a.codes, s, e, it.k, tab, emit);
}

// ---- partitioned exact counting
//
// The hashes of one (sample, k) are grouped by the top log2p bits of their
// 61-bit sign (a contiguous range of bins per group) in two rolls over the
// windows: the first counts each group, the second reserves each CTA's range
// of every group and writes the hashes there.  Then one CTA per group counts
// its hashes in a shared-memory table; the occurrence that brings a hash's
// count to min_count puts it in its bin, as in the table pass above.  Every
// occurrence of a hash lands in the same group, so the counts are exact and
// the result does not depend on the order of the writes.
struct PartArgs {
  unsigned int *cta_count;      // [items][P] hashes per group of each CTA (count roll)
  unsigned int *count;          // [P] hashes per group
  unsigned int *cursor;         // [P] next free position of each group
  unsigned int *start;          // [P + 1] first position of each group
  unsigned long long *hashes;   // the hashes, grouped
  int log2p;                    // P = 2^log2p groups
  int table_slots;              // slots of one group's counting table (a power of two)
};

// The scatter roll's emitter: 8 hashes at a time, their ranks in their
// groups taken by 8 independent shared-memory atomics before the 8 stores, so
// no store waits on its own atomic alone.
struct ScatterBatch {
  static constexpr int kBatch = 8;
  unsigned int *rank;           // [P] next position of each group for this CTA
  unsigned long long *out;
  int shift;
  uint64_t h[kBatch];
  bool v[kBatch];

  __device__ __forceinline__ void put(int i, uint64_t hash, bool valid) {
    h[i] = hash;
    v[i] = valid;
  }
  __device__ __forceinline__ void flush() {
    unsigned int pos[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; ++j)
      if (v[j]) pos[j] = atomicAdd(rank + (mod_sign(h[j]) >> shift), 1u);
#pragma unroll
    for (int j = 0; j < kBatch; ++j)
      if (v[j]) out[pos[j]] = h[j];
  }
};

// kScatter false: the count roll, per-group counts of the CTA (kept) and of
// the sample; true: the scatter roll, the hashes into their groups (the
// cursors start at the groups' first positions), each CTA reserving its
// ranges from the counts its item's count roll kept.
template <bool kRc, bool kPhased, bool kScatter>
__global__ void __launch_bounds__(kSketchThreads, 1)
part_kernel(SketchArgs a, PartArgs pa) {
  extern __shared__ unsigned int sh_part[];   // [P]
  __shared__ RollTable tab;
  const SketchItem it = a.items[blockIdx.x];
  const int P = 1 << pa.log2p;
  const int shift = 61 - pa.log2p;
  unsigned int *mine = pa.cta_count + static_cast<int64_t>(blockIdx.x) * P;
  if (threadIdx.x < 64) {
    const ulonglong2 *src = reinterpret_cast<const ulonglong2 *>(a.tables + it.tab);
    reinterpret_cast<ulonglong2 *>(&tab)[threadIdx.x] = src[threadIdx.x];
  }
  const int64_t s = it.begin + static_cast<int64_t>(threadIdx.x) * it.per;
  const int64_t e = min(s + it.per, it.end);
  if constexpr (!kScatter) {
    for (int i = threadIdx.x; i < P; i += kSketchThreads) sh_part[i] = 0;
    __syncthreads();
    if (s < e)
      roll_windows<kRc, kPhased>(a.codes, s, e, it.k, tab, [&](uint64_t h) {
        atomicAdd(&sh_part[mod_sign(h) >> shift], 1u);
      });
    __syncthreads();
    for (int i = threadIdx.x; i < P; i += kSketchThreads) {
      const unsigned int n = sh_part[i];
      mine[i] = n;
      if (n) atomicAdd(pa.count + i, n);
    }
  } else {
    for (int i = threadIdx.x; i < P; i += kSketchThreads) {
      const unsigned int n = mine[i];
      sh_part[i] = n ? atomicAdd(pa.cursor + i, n) : 0u;
    }
    __syncthreads();
    if (s < e) {
      ScatterBatch emit{sh_part, pa.hashes, shift, {}, {}};
      roll_windows<kRc, kPhased>(a.codes, s, e, it.k, tab, emit);
    }
  }
}

// Exclusive prefix sum of the group counts (one CTA of kScanThreads): the
// groups' first positions, also the scatter's starting cursors.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) part_scan_kernel(PartArgs pa) {
  __shared__ unsigned int warp_sums[kScanThreads / 32];
  const int P = 1 << pa.log2p;
  const int per = (P + kScanThreads - 1) / kScanThreads;
  const int i0 = min(P, threadIdx.x * per), i1 = min(P, i0 + per);
  unsigned int sum = 0;
  for (int i = i0; i < i1; ++i) sum += pa.count[i];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned int incl = sum;
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned int v = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += v;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    unsigned int w = warp_sums[lane];
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned int v = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += v;
    }
    warp_sums[lane] = w;   // inclusive sums of the warps
  }
  __syncthreads();
  unsigned int run = incl - sum + (warp > 0 ? warp_sums[warp - 1] : 0u);
  for (int i = i0; i < i1; ++i) {
    pa.start[i] = run;
    pa.cursor[i] = run;
    run += pa.count[i];
  }
  if (threadIdx.x == kScanThreads - 1) pa.start[P] = run;
}

// One CTA per group: the group's hashes counted in a shared-memory table of
// table_slots keys and counts.
constexpr int kPartCountThreads = 512;
__global__ void __launch_bounds__(kPartCountThreads)
part_count_kernel(SketchArgs a, PartArgs pa, unsigned long long *__restrict__ row) {
  extern __shared__ unsigned long long sh_keys[];   // [C] keys, then [C] counts
  __shared__ unsigned int empty_count;               // occurrences of the hash equal to kEmptyKey
  const int C = pa.table_slots;
  unsigned int *sh_counts = reinterpret_cast<unsigned int *>(sh_keys + C);
  for (int i = threadIdx.x; i < C; i += kPartCountThreads) {
    sh_keys[i] = kEmptyKey;
    sh_counts[i] = 0;
  }
  if (threadIdx.x == 0) empty_count = 0;
  __syncthreads();
  const unsigned int b0 = pa.start[blockIdx.x], b1 = pa.start[blockIdx.x + 1];
  unsigned long long next = b0 + threadIdx.x < b1 ? pa.hashes[b0 + threadIdx.x] : 0ULL;
  for (unsigned int i = b0 + threadIdx.x; i < b1; i += kPartCountThreads) {
    const unsigned long long h = next;   // this hash; the next one loads meanwhile
    if (i + kPartCountThreads < b1) next = pa.hashes[i + kPartCountThreads];
    unsigned int old;
    if (h == kEmptyKey) {
      old = atomicAdd(&empty_count, 1u);
    } else {
      uint32_t slot = static_cast<uint32_t>(table_slot(h, static_cast<uint64_t>(C - 1)));
      int probe = 0;
      for (; probe < C; ++probe) {
        unsigned long long cur = *reinterpret_cast<volatile unsigned long long *>(sh_keys + slot);
        if (cur == kEmptyKey) {
          cur = atomicCAS(sh_keys + slot, kEmptyKey, h);
          if (cur == kEmptyKey) cur = h;
        }
        if (cur == h) break;
        slot = (slot + 1) & static_cast<uint32_t>(C - 1);
      }
      if (probe == C) {   // more distinct hashes than slots (1.5 per base of the group: not reached)
        atomicOr(&a.status->error, kErrTable);
        continue;
      }
      old = atomicAdd(sh_counts + slot, 1u);
    }
    if (old + 1 == a.min_count) {
      const uint64_t sign = mod_sign(h);
      const uint32_t q = bin_of(sign, a.binsize, a.magic);
      if (sign < row[q]) atomicMin(row + q, static_cast<unsigned long long>(sign));
    }
  }
}

__device__ __forceinline__ uint64_t univhash(uint64_t s, uint64_t t) {
  const uint64_t x = 1009ULL * s + (1000ULL * 1000ULL + 3ULL) * t;
  return (48271ULL * x + 11ULL) % ((1ULL << 31) - 1ULL);
}

// One CTA per bins row: inverse minhash, densify, bit planes.
__global__ void __launch_bounds__(kFinishThreads)
finish_kernel(unsigned long long *__restrict__ signs, int nbins, int s64, uint64_t *__restrict__ words,
              double *__restrict__ inv_minhash, int8_t *__restrict__ densified, DevStatus *status) {
  unsigned long long *row = signs + static_cast<int64_t>(blockIdx.x) * nbins;
  __shared__ unsigned long long smin, smax;
  if (threadIdx.x == 0) {
    smin = kEmptyKey;
    smax = 0;
    inv_minhash[blockIdx.x] = static_cast<double>(row[0]) / static_cast<double>(kSignMod);
  }
  __syncthreads();
  unsigned long long mn = kEmptyKey, mx = 0;
  for (int i = threadIdx.x; i < nbins; i += kFinishThreads) {
    const unsigned long long v = row[i];
    mn = min(mn, v);
    mx = max(mx, v);
  }
  atomicMin(&smin, mn);
  atomicMax(&smax, mx);
  __syncthreads();
  const bool some_empty = smax == kEmptyKey, all_empty = smin == kEmptyKey;
  if (threadIdx.x == 0) densified[blockIdx.x] = some_empty ? (all_empty ? -1 : 1) : 0;
  if (some_empty && !all_empty && threadIdx.x < 32) {
    // empty bins in increasing order, each from the first filled bin of its
    // probe sequence (bins filled earlier in the loop count as filled)
    const unsigned lane = threadIdx.x;
    for (int base = 0; base < nbins; base += 32) {
      const int i0 = base + static_cast<int>(lane);
      unsigned m = __ballot_sync(0xffffffffu, i0 < nbins && row[i0] == kEmptyKey);
      while (m) {
        const int i = base + __ffs(m) - 1;
        m &= m - 1;
        uint64_t j = static_cast<uint64_t>(i), attempt = 0;
        unsigned long long v = kEmptyKey;
        while ((v = row[j]) == kEmptyKey) {
          if (attempt > (1ULL << 24)) {
            if (lane == 0) atomicOr(&status->error, kErrDensify);
            break;
          }
          j = univhash(static_cast<uint64_t>(i), attempt++) % static_cast<uint64_t>(nbins);
        }
        __syncwarp();
        if (lane == 0) row[i] = v;
        __syncwarp();
      }
    }
  }
  __syncthreads();
  // bit planes: word (block b, plane p) holds bit p of bins 64b .. 64b+63
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  uint64_t *out = words + static_cast<int64_t>(blockIdx.x) * s64 * kBbits;
  for (int b = warp; b < s64; b += kFinishThreads / 32) {
    const unsigned long long v0 = row[64 * b + lane], v1 = row[64 * b + 32 + lane];
    uint64_t mine = 0;
#pragma unroll
    for (int p = 0; p < kBbits; ++p) {
      const unsigned lo = __ballot_sync(0xffffffffu, (v0 >> p) & 1ULL);
      const unsigned hi = __ballot_sync(0xffffffffu, (v1 >> p) & 1ULL);
      if (lane == p) mine = (static_cast<uint64_t>(hi) << 32) | lo;
    }
    if (lane < kBbits) out[static_cast<int64_t>(b) * kBbits + lane] = mine;
  }
}

int max_dyn_smem(int device) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  return v;
}

// Largest bins row kept in shared memory.
bool bins_fit_shared(int device, int nbins) {
  return static_cast<int64_t>(nbins) * 8 + static_cast<int64_t>(sizeof(RollTable)) + 1024 <=
         max_dyn_smem(device);
}

struct Batch {
  int64_t s0, s1;          // samples
  int64_t q0, q1;          // sequences
  int64_t b0, b1;          // bytes (offsets in the caller's buffer)
};

constexpr int64_t kBatchBytes = 1LL << 30;         // bases per batch
constexpr int64_t kBatchBins = 1LL << 30;          // bytes of bins rows per batch

}  // namespace
}  // namespace sk

using namespace sk;

namespace {

struct SketchCall {
  sk_ctx *ctx;
  const char *bases;               // host or (device_in) device
  bool device_in = false;
  const int64_t *seq_off;
  const int64_t *sample_seqs;
  int64_t n;
  std::vector<int32_t> kmers;
  int s64, use_rc, codon_phased, min_count;
  int nbins;
  uint64_t binsize, magic;
  // device buffers (context scratch unless the caller gave them)
  uint8_t *d_codes = nullptr;
  int64_t *d_seq_off = nullptr;
  RollTable *d_tables = nullptr;
  unsigned long long *d_signs = nullptr;
  uint64_t *d_words = nullptr;
  double *d_inv = nullptr;
  int8_t *d_dens = nullptr;
};

sk_status check_inputs(sk_ctx *ctx, const char *bases, const int64_t *seq_off,
                       const int64_t *sample_seqs, int64_t n, const int32_t *kmers, int32_t K,
                       int32_t s64, int32_t use_rc, int32_t codon_phased, int32_t min_count) {
  if (n < 0) return fail(ctx, SK_EINVAL, "negative sample count");
  if (n == 0) return SK_OK;
  if (!seq_off || !sample_seqs || !kmers) return fail(ctx, SK_EINVAL, "null argument");
  if (K < 1 || K > kMaxKmers) return fail(ctx, SK_ERANGE, "n_kmers %d outside [1, %d]", K, kMaxKmers);
  for (int k = 0; k < K; ++k) {
    if (kmers[k] < kMinK) return fail(ctx, SK_EINVAL, "Minimum k must be 3 or higher");
    if (kmers[k] > kMaxK) return fail(ctx, SK_EINVAL, "k-mer length %d above %d", kmers[k], kMaxK);
  }
  if (s64 < 1 || s64 > kMaxSketch64)
    return fail(ctx, SK_ERANGE, "sketchsize64 %d outside [1, %d]", s64, kMaxSketch64);
  if (use_rc != 0 && use_rc != 1) return fail(ctx, SK_EINVAL, "use_rc must be 0 or 1");
  if (codon_phased != 0 && codon_phased != 1) return fail(ctx, SK_EINVAL, "codon_phased must be 0 or 1");
  if (min_count < 0 || min_count > 255) return fail(ctx, SK_EINVAL, "min_count %d outside [0, 255]", min_count);
  if (sample_seqs[0] < 0) return fail(ctx, SK_EINVAL, "negative sequence index");
  for (int64_t s = 0; s < n; ++s)
    if (sample_seqs[s + 1] <= sample_seqs[s])
      return fail(ctx, SK_EINVAL, "sample %lld contains no sequence", static_cast<long long>(s));
  for (int64_t q = sample_seqs[0]; q < sample_seqs[n]; ++q)
    if (seq_off[q + 1] < seq_off[q])
      return fail(ctx, SK_EINVAL, "sequence offsets decrease at %lld", static_cast<long long>(q));
  if (seq_off[sample_seqs[n]] > seq_off[sample_seqs[0]] && !bases)
    return fail(ctx, SK_EINVAL, "null bases");
  return SK_OK;
}

// Samples [s0, s1): their sequences [q0, q1) and bytes [b0, b1) of the caller's buffer.
Batch span(const SketchCall &c, int64_t s0, int64_t s1) {
  Batch b{};
  b.s0 = s0;
  b.s1 = s1;
  b.q0 = c.sample_seqs[s0];
  b.q1 = c.sample_seqs[s1];
  b.b0 = c.seq_off[b.q0];
  b.b1 = c.seq_off[b.q1];
  return b;
}

std::vector<Batch> make_batches(const SketchCall &c) {
  std::vector<Batch> out;
  const int64_t row_bytes = static_cast<int64_t>(c.kmers.size()) * c.nbins * 8;
  int64_t s = 0;
  while (s < c.n) {
    const int64_t b0 = c.seq_off[c.sample_seqs[s]];
    int64_t e = s + 1;
    while (e < c.n && c.seq_off[c.sample_seqs[e + 1]] - b0 <= kBatchBytes &&
           (e + 1 - s) * row_bytes <= kBatchBins)
      ++e;
    out.push_back(span(c, s, e));
    s = e;
  }
  return out;
}

// Upload pieces of a batch: whole samples, about bytes / kUploadChunks each
// and at least kMinUploadBytes.
constexpr int kUploadChunks = 8;
constexpr int64_t kMinUploadBytes = 8LL << 20;

std::vector<Batch> upload_chunks(const SketchCall &c, const Batch &b) {
  std::vector<Batch> out;
  const int64_t target = std::max<int64_t>(kMinUploadBytes, (b.b1 - b.b0 + kUploadChunks - 1) / kUploadChunks);
  int64_t s = b.s0;
  while (s < b.s1) {
    int64_t e = s + 1;
    while (e < b.s1 && c.seq_off[c.sample_seqs[e]] - c.seq_off[c.sample_seqs[s]] < target) ++e;
    out.push_back(span(c, s, e));
    s = e;
  }
  return out;
}

// Work items of samples [s0, s1) of batch b (code offsets relative to b.b0):
// window starts of each sample in equal pieces of at most kItemWindows (so
// the threads of every item get the same share), every k of a piece adjacent
// (they read the same bases).  Windows end inside their sample, so a sample's
// items read no other sample's codes that they depend on.
void make_items(const SketchCall &c, const Batch &b, int64_t s0, int64_t s1, int k_only,
                std::vector<SketchItem> &items, int64_t max_windows = kItemWindows) {
  const int K = static_cast<int>(c.kmers.size());
  for (int64_t s = s0; s < s1; ++s) {
    const int64_t a = c.seq_off[c.sample_seqs[s]] - b.b0, e = c.seq_off[c.sample_seqs[s + 1]] - b.b0;
    const int64_t pieces = std::max<int64_t>(1, (e - a + max_windows - 1) / max_windows);
    const int64_t piece = (e - a + pieces - 1) / pieces;
    const int32_t per = static_cast<int32_t>(
        std::max<int64_t>(16, ((piece + kSketchThreads - 1) / kSketchThreads + 15) / 16 * 16));
    const int64_t step = static_cast<int64_t>(per) * kSketchThreads;
    for (int64_t p = a; p < e; p += step)
      for (int k = 0; k < K; ++k) {
        if (k_only >= 0 && k != k_only) continue;
        SketchItem it{};
        it.begin = p;
        it.per = per;
        const int64_t window = c.codon_phased ? 3 * static_cast<int64_t>(c.kmers[k]) - 2 : c.kmers[k];
        it.end = std::min(p + step, e - window + 1);
        if (it.end <= it.begin) continue;
        it.row = static_cast<int32_t>((s - b.s0) * K + k);
        it.k = c.kmers[k];
        it.tab = k;
        items.push_back(it);
      }
  }
}

sk_status upload(sk_ctx *ctx, void *dst, const void *src, size_t bytes) {
  if (!bytes) return SK_OK;
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
  return e == cudaSuccess ? SK_OK : cuda_fail(ctx, e, "sketch upload");
}

sk_status launch_hash(sk_ctx *ctx, const SketchCall &c, SketchArgs args, const SketchItem *d_items,
                      size_t n_items, cudaStream_t stream) {
  if (n_items == 0) return SK_OK;
  args.items = d_items;
  const bool shared = bins_fit_shared(ctx->device, c.nbins);
  const size_t smem = shared ? static_cast<size_t>(c.nbins) * 8 : 0;
  cudaError_t e = cudaSuccess;
  const unsigned grid = static_cast<unsigned>(n_items);
  if (shared) {
    auto kern = c.codon_phased ? (c.use_rc ? sketch_kernel<true, true, true> : sketch_kernel<true, false, true>)
                               : (c.use_rc ? sketch_kernel<true, true, false> : sketch_kernel<true, false, false>);
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e == cudaSuccess) kern<<<grid, kSketchThreads, smem, stream>>>(args);
  } else {
    auto kern = c.codon_phased ? (c.use_rc ? sketch_kernel<false, true, true> : sketch_kernel<false, false, true>)
                               : (c.use_rc ? sketch_kernel<false, true, false> : sketch_kernel<false, false, false>);
    kern<<<grid, kSketchThreads, 0, stream>>>(args);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? SK_OK : cuda_fail(ctx, e, "sketch kernel");
}

// Codes of bytes [a, b) of the caller's buffer (offsets relative to the
// batch) and start flags of sequences [q0, q1), on `stream`.
sk_status make_codes(SketchCall &c, const Batch &batch, const Batch &part, cudaStream_t stream) {
  sk_ctx *ctx = c.ctx;
  const int64_t bytes = part.b1 - part.b0;
  uint8_t *dst = c.d_codes + (part.b0 - batch.b0);
  const uint8_t *src = c.device_in ? reinterpret_cast<const uint8_t *>(c.bases) + part.b0 : dst;
  const unsigned g = static_cast<unsigned>(
      std::max<int64_t>(1, std::min<int64_t>(ctx->sm_count * 8, (bytes / 16 + 255) / 256)));
  if (bytes > 0) codes_kernel<<<g, 256, 0, stream>>>(src, dst, bytes);
  const int64_t n_seqs = part.q1 - part.q0;
  if (n_seqs > 0)
    mark_starts_kernel<<<static_cast<unsigned>(std::min<int64_t>(ctx->sm_count * 8, (n_seqs + 255) / 256)),
                         256, 0, stream>>>(c.d_codes, c.d_seq_off + (part.q0 - batch.q0), n_seqs,
                                                batch.b0);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SK_OK : cuda_fail(ctx, e, "sketch codes");
}

uint64_t next_pow2(uint64_t v) {
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

// Groups of the partitioned count: at most kPartHashes bases per group (while
// there are at most 2^kMaxLog2Parts groups), tables of 2048..kMaxPartSlots
// slots (1.5 times the bases of a group, the hashes' upper bound).
constexpr int64_t kPartHashes = 4096;
constexpr int kMaxLog2Parts = 15;
constexpr int kMaxPartSlots = 16384;

// The exact count of one (sample, k) by groups of hashes (part_kernel,
// part_scan_kernel, part_count_kernel), in items of at most per_item window
// starts; pa's buffers hold the sample's hashes and its groups.
sk_status count_partitioned(SketchCall &c, const Batch &b, SketchArgs &args, std::vector<SketchItem> &items,
                            int64_t s, int k, int64_t per_item, const PartArgs &pa) {
  sk_ctx *ctx = c.ctx;
  const int K = static_cast<int>(c.kmers.size());
  items.clear();
  make_items(c, b, s, s + 1, k, items, per_item);
  if (items.empty()) return SK_OK;
  void *p = nullptr;
  sk_status st = scratch(ctx, kSlotSketchItems, items.size() * sizeof(SketchItem), &p);
  if (st == SK_OK) st = upload(ctx, p, items.data(), items.size() * sizeof(SketchItem));
  if (st != SK_OK) return st;
  args.items = static_cast<SketchItem *>(p);
  const int P = 1 << pa.log2p;
  const size_t part_smem = static_cast<size_t>(P) * 4;
  const size_t table_smem = static_cast<size_t>(pa.table_slots) * 12;
  auto hist = c.codon_phased ? (c.use_rc ? part_kernel<true, true, false> : part_kernel<false, true, false>)
                             : (c.use_rc ? part_kernel<true, false, false> : part_kernel<false, false, false>);
  auto scat = c.codon_phased ? (c.use_rc ? part_kernel<true, true, true> : part_kernel<false, true, true>)
                             : (c.use_rc ? part_kernel<true, false, true> : part_kernel<false, false, true>);
  cudaError_t e = cudaFuncSetAttribute(hist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(part_smem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(scat, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(part_smem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(part_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(table_smem));
  if (e == cudaSuccess) e = cudaMemsetAsync(pa.count, 0, part_smem, ctx->stream);
  const unsigned grid = static_cast<unsigned>(items.size());
  if (e == cudaSuccess) {
    hist<<<grid, kSketchThreads, part_smem, ctx->stream>>>(args, pa);
    part_scan_kernel<<<1, kScanThreads, 0, ctx->stream>>>(pa);
    scat<<<grid, kSketchThreads, part_smem, ctx->stream>>>(args, pa);
    unsigned long long *row = args.signs + ((s - b.s0) * K + k) * static_cast<int64_t>(c.nbins);
    part_count_kernel<<<static_cast<unsigned>(P), kPartCountThreads, table_smem, ctx->stream>>>(args, pa, row);
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? SK_OK : cuda_fail(ctx, e, "sketch counting");
}

// Bins rows of one batch with the exact count filter, a hash entering its bin
// when its count reaches min_count.  Per sample and k the hashes are counted
// by groups (count_partitioned) when the sample's hash buffer fits the table
// budget and its groups fit shared memory; otherwise in a global table of
// twice the sample's windows (in bin-range passes when that exceeds the
// budget).  The table pass's items are an eighth of the hashing ones (no
// per-CTA bins to amortise; more CTAs in flight hide the table's memory
// latency).
constexpr int64_t kCountItemWindows = kItemWindows / 8;

sk_status count_batch(SketchCall &c, const Batch &b, SketchArgs &args, std::vector<SketchItem> &items) {
  sk_ctx *ctx = c.ctx;
  const int K = static_cast<int>(c.kmers.size());
  // bytes of table per pass: a quarter of the context's memory limit when one
  // is set, else a quarter of the free device memory less 2 GiB (at least 1 GiB)
  uint64_t kTableBudget = 0;
  if (ctx->mem_limit > 0) {
    kTableBudget = std::max<uint64_t>(1ULL << 16, static_cast<uint64_t>(ctx->mem_limit) / 4);
  } else {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
    kTableBudget = std::max<uint64_t>(1ULL << 30, free_b > (2ULL << 30) ? (free_b - (2ULL << 30)) / 4 : 0);
  }
  args.min_count = static_cast<unsigned int>(c.min_count);
  for (int64_t s = b.s0; s < b.s1; ++s) {
    const int64_t windows = c.seq_off[c.sample_seqs[s + 1]] - c.seq_off[c.sample_seqs[s]];
    if (windows <= 0) continue;
    int log2p = 0;
    while (log2p < kMaxLog2Parts && (kPartHashes << log2p) < windows) ++log2p;
    const int64_t per_part = (windows + (int64_t(1) << log2p) - 1) >> log2p;
    // 1.5 slots per base of a group: the distinct hashes (at most the
    // bases) fill at most two thirds of a table
    const int part_slots =
        static_cast<int>(std::max<uint64_t>(2048, next_pow2(static_cast<uint64_t>(per_part) * 3 / 2)));
    // items of the grouped count: two per SM, at least 4 P windows each
    const int64_t per_item = std::min<int64_t>(
        kItemWindows, std::max<int64_t>(int64_t(4) << log2p, (windows + 2 * ctx->sm_count - 1) / (2 * ctx->sm_count)));
    const int64_t max_items = (windows + per_item - 1) / per_item + 1;   // items of one k
    const uint64_t part_bytes = static_cast<uint64_t>(windows) * 8 + ((uint64_t(3) << log2p) + 1) * 4 +
                                (static_cast<uint64_t>(max_items) << log2p) * 4 + 256;
    if (part_slots <= kMaxPartSlots && windows < (int64_t(1) << 32) && part_bytes <= kTableBudget) {
      void *tk = nullptr;
      sk_status st = scratch(ctx, kSlotSketchTable, part_bytes, &tk);
      if (st != SK_OK) return st;
      PartArgs pa{};
      pa.hashes = static_cast<unsigned long long *>(tk);
      pa.count = reinterpret_cast<unsigned int *>(pa.hashes + windows);
      pa.cursor = pa.count + (1 << log2p);
      pa.start = pa.cursor + (1 << log2p);
      pa.cta_count = pa.start + (1 << log2p) + 1;
      pa.log2p = log2p;
      pa.table_slots = part_slots;
      for (int k = 0; k < K; ++k) {
        st = count_partitioned(c, b, args, items, s, k, per_item, pa);
        if (st != SK_OK) return st;
      }
      continue;
    }
    const uint64_t want = next_pow2(static_cast<uint64_t>(windows) * 2);
    const uint64_t passes = std::max<uint64_t>(1, (want * sizeof(TableSlot) + kTableBudget - 1) / kTableBudget);
    const uint64_t slots = std::max<uint64_t>(1024, next_pow2((want + passes - 1) / passes));
    void *tk = nullptr;
    sk_status st = scratch(ctx, kSlotSketchTable, slots * sizeof(TableSlot) + 16, &tk);
    if (st != SK_OK) return st;
    args.table = static_cast<TableSlot *>(tk);
    args.max_key_count = reinterpret_cast<unsigned int *>(static_cast<char *>(tk) + slots * sizeof(TableSlot));
    args.table_mask = slots - 1;
    args.min_count = static_cast<unsigned int>(c.min_count);
    for (int k = 0; k < K; ++k) {
      items.clear();
      make_items(c, b, s, s + 1, k, items, kCountItemWindows);
      if (items.empty()) continue;
      void *p = nullptr;
      st = scratch(ctx, kSlotSketchItems, items.size() * sizeof(SketchItem), &p);
      if (st == SK_OK) st = upload(ctx, p, items.data(), items.size() * sizeof(SketchItem));
      if (st != SK_OK) return st;
      args.items = static_cast<SketchItem *>(p);
      for (uint64_t pass = 0; pass < passes; ++pass) {
        args.bin_lo = static_cast<uint32_t>(c.nbins * pass / passes);
        args.bin_hi = static_cast<uint32_t>(c.nbins * (pass + 1) / passes);
        table_clear_kernel<<<static_cast<unsigned>(std::min<uint64_t>(4096, (slots + 255) / 256)), 256, 0,
                             ctx->stream>>>(args.table, slots, args.max_key_count);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) {
          auto kern = c.codon_phased ? (c.use_rc ? count_kernel<true, true> : count_kernel<false, true>)
                                     : (c.use_rc ? count_kernel<true, false> : count_kernel<false, false>);
          kern<<<static_cast<unsigned>(items.size()), kSketchThreads, 0, ctx->stream>>>(args);
          e = cudaGetLastError();
        }
        if (e != cudaSuccess) return cuda_fail(ctx, e, "sketch counting");
      }
    }
  }
  return SK_OK;
}

// Bins rows of one batch without a count filter.  Host bases go up in sample
// chunks on the copy stream; each chunk's codes and items run as soon as it
// has landed, while later chunks copy, on two compute streams in turn (so
// one chunk's last wave is filled by the next chunk's CTAs; chunks touch
// disjoint bins rows and codes, and no emitted window reads another chunk's
// bytes).
sk_status hash_batch(SketchCall &c, const Batch &b, SketchArgs &args, std::vector<SketchItem> &items) {
  sk_ctx *ctx = c.ctx;
  const std::vector<Batch> parts = c.device_in ? std::vector<Batch>{b} : upload_chunks(c, b);
  std::vector<size_t> first(parts.size() + 1, 0);
  items.clear();
  for (size_t i = 0; i < parts.size(); ++i) {
    make_items(c, b, parts[i].s0, parts[i].s1, -1, items);
    first[i + 1] = items.size();
  }
  void *p = nullptr;
  sk_status st = SK_OK;
  if (!items.empty()) {
    st = scratch(ctx, kSlotSketchItems, items.size() * sizeof(SketchItem), &p);
    if (st == SK_OK) st = upload(ctx, p, items.data(), items.size() * sizeof(SketchItem));
    if (st != SK_OK) return st;
  }
  const SketchItem *d_items = static_cast<const SketchItem *>(p);
  if (c.device_in) {
    st = make_codes(c, b, b, ctx->stream);
    return st == SK_OK ? launch_hash(ctx, c, args, d_items, items.size(), ctx->stream) : st;
  }
  st = ensure_copy_stream(ctx);
  if (st != SK_OK) return st;
  cudaError_t e = cudaSuccess;
  if (!ctx->stream_b) e = cudaStreamCreateWithFlags(&ctx->stream_b, cudaStreamNonBlocking);
  if (e == cudaSuccess && !ctx->ev_join) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
  while (e == cudaSuccess && ctx->ev_chunk.size() < parts.size()) {
    cudaEvent_t ev = nullptr;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) ctx->ev_chunk.push_back(ev);
  }
  // the copies start after the buffers' set-up on the context's stream
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_chunk[0], ctx->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_chunk[0], 0);
  for (size_t i = 0; i < parts.size() && e == cudaSuccess; ++i) {
    const int64_t bytes = parts[i].b1 - parts[i].b0;
    if (bytes > 0)
      e = cudaMemcpyAsync(c.d_codes + (parts[i].b0 - b.b0), c.bases + parts[i].b0, static_cast<size_t>(bytes),
                          cudaMemcpyHostToDevice, ctx->copy_stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_chunk[i], ctx->copy_stream);
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "sketch upload");
  cudaStream_t compute[2] = {ctx->stream, ctx->stream_b};
  for (size_t i = 0; i < parts.size(); ++i) {
    cudaStream_t s = compute[i & 1];
    e = cudaStreamWaitEvent(s, ctx->ev_chunk[i], 0);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "sketch upload");
    st = make_codes(c, b, parts[i], s);
    if (st == SK_OK) st = launch_hash(ctx, c, args, d_items + first[i], first[i + 1] - first[i], s);
    if (st != SK_OK) return st;
  }
  // the context's stream (finishing, copies back) waits for the second one
  e = cudaEventRecord(ctx->ev_join, ctx->stream_b);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0);
  return e == cudaSuccess ? SK_OK : cuda_fail(ctx, e, "stream join");
}

// Sketches the samples of one batch into d_words / d_inv / d_dens (rows of the
// batch's samples) on the context's stream.
sk_status sketch_batch(SketchCall &c, const Batch &b, std::vector<SketchItem> &items) {
  sk_ctx *ctx = c.ctx;
  const int K = static_cast<int>(c.kmers.size());
  const int64_t rows = (b.s1 - b.s0) * K;
  const int64_t bytes = b.b1 - b.b0;
  const int64_t n_seqs = b.q1 - b.q0;
  void *p = nullptr;
  sk_status st = scratch(ctx, kSlotSketchCodes, static_cast<size_t>(bytes + 2 * kCodePad), &p);
  if (st != SK_OK) return st;
  c.d_codes = static_cast<uint8_t *>(p) + kCodePad;
  st = scratch(ctx, kSlotSketchSeqs, static_cast<size_t>(n_seqs + 1) * 8, &p);
  if (st != SK_OK) return st;
  c.d_seq_off = static_cast<int64_t *>(p);
  st = scratch(ctx, kSlotSketchBins, static_cast<size_t>(rows) * c.nbins * 8, &p);
  if (st != SK_OK) return st;
  c.d_signs = static_cast<unsigned long long *>(p);
  cudaError_t e = cudaMemsetAsync(c.d_codes - kCodePad, kCodeInvalid, kCodePad, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.d_codes + bytes, kCodeInvalid, kCodePad, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.d_signs, 0xFF, static_cast<size_t>(rows) * c.nbins * 8, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "sketch buffers");
  st = upload(ctx, c.d_seq_off, c.seq_off + b.q0, static_cast<size_t>(n_seqs + 1) * 8);
  if (st != SK_OK) return st;
  SketchArgs args{};
  args.codes = c.d_codes;
  args.tables = c.d_tables;
  args.signs = c.d_signs;
  args.nbins = c.nbins;
  args.use_rc = c.use_rc;
  args.binsize = c.binsize;
  args.magic = c.magic;
  args.status = ctx->status_dev;
  if (c.min_count > 0) {
    if (!c.device_in) st = upload(ctx, c.d_codes, c.bases + b.b0, static_cast<size_t>(bytes));
    if (st == SK_OK) st = make_codes(c, b, b, ctx->stream);
    if (st == SK_OK) st = count_batch(c, b, args, items);
  } else {
    st = hash_batch(c, b, args, items);
  }
  if (st != SK_OK) return st;
  finish_kernel<<<static_cast<unsigned>(rows), kFinishThreads, 0, ctx->stream>>>(
      c.d_signs, c.nbins, c.s64, c.d_words + b.s0 * K * static_cast<int64_t>(c.s64) * kBbits,
      c.d_inv + b.s0 * K, c.d_dens + b.s0 * K, ctx->status_dev);
  e = cudaGetLastError();
  return e == cudaSuccess ? SK_OK : cuda_fail(ctx, e, "sketch finish");
}

// Everything up to device-resident words / inverse minhashes / densify flags
// of all samples.
sk_status sketch_to_device(SketchCall &c) {
  sk_ctx *ctx = c.ctx;
  const int K = static_cast<int>(c.kmers.size());
  std::vector<RollTable> tables(K);
  for (int k = 0; k < K; ++k) tables[k] = make_table(c.kmers[k], c.codon_phased != 0);
  void *p = nullptr;
  sk_status st = scratch(ctx, kSlotSketchTables, tables.size() * sizeof(RollTable), &p);
  if (st == SK_OK) st = upload(ctx, p, tables.data(), tables.size() * sizeof(RollTable));
  if (st != SK_OK) return st;
  c.d_tables = static_cast<RollTable *>(p);
  std::vector<SketchItem> items;
  const std::vector<Batch> batches = make_batches(c);
  for (size_t i = 0; i < batches.size(); ++i) {
    st = sketch_batch(c, batches[i], items);
    if (st != SK_OK) return st;
    if (i + 1 < batches.size()) {   // the next batch reuses the scratch buffers
      cudaError_t e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "sketch batch");
    }
  }
  return SK_OK;
}

// After a failed call: waits for the copy and second compute streams, so no
// copy still reads the caller's host buffer once the call has returned.
sk_status drain(sk_ctx *ctx, sk_status st) {
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  if (ctx->stream_b) cudaStreamSynchronize(ctx->stream_b);
  cudaStreamSynchronize(ctx->stream);
  return st;
}

// Call set-up; d_words / d_inv given by the caller are written directly,
// else they are context scratch.
sk_status setup_call(SketchCall &c, sk_ctx *ctx, const char *bases, bool device_in,
                     const int64_t *seq_offsets, const int64_t *sample_seqs, int64_t n,
                     const int32_t *kmers, int32_t K, int32_t s64, int32_t use_rc,
                     int32_t codon_phased, int32_t min_count, uint64_t *d_words, double *d_inv) {
  c.ctx = ctx;
  c.bases = bases;
  c.device_in = device_in;
  c.seq_off = seq_offsets;
  c.sample_seqs = sample_seqs;
  c.n = n;
  c.kmers.assign(kmers, kmers + K);
  c.s64 = s64;
  c.use_rc = use_rc;
  c.codon_phased = codon_phased;
  c.min_count = min_count;
  c.nbins = s64 * 64;
  c.binsize = (kSignMod + static_cast<uint64_t>(c.nbins) - 1) / static_cast<uint64_t>(c.nbins);
  c.magic = ~0ULL / c.binsize;
  if (c.magic >> 32) return fail(ctx, SK_ERANGE, "bin divisor out of range");   // about 8 x nbins
  const size_t words = static_cast<size_t>(n) * K * s64 * kBbits;
  const size_t rows = static_cast<size_t>(n) * K;
  const size_t bytes = (d_words ? 0 : words * 8) + (d_inv ? 0 : rows * 8) + rows + 16;
  void *p = nullptr;
  sk_status st = scratch(ctx, kSlotSketchWords, bytes, &p);
  if (st != SK_OK) return st;
  char *q = static_cast<char *>(p);
  c.d_words = d_words ? d_words : reinterpret_cast<uint64_t *>(q);
  if (!d_words) q += words * 8;
  c.d_inv = d_inv ? d_inv : reinterpret_cast<double *>(q);
  if (!d_inv) q += rows * 8;
  c.d_dens = reinterpret_cast<int8_t *>(q);
  return SK_OK;
}

}  // namespace

extern "C" {

sk_status sk_sketch(sk_ctx *ctx, const char *bases, const int64_t *seq_offsets,
                    const int64_t *sample_seqs, int64_t n_samples, const int32_t *kmers,
                    int32_t n_kmers, int32_t sketchsize64, int32_t use_rc, int32_t codon_phased,
                    int32_t min_count, uint64_t *words, double *inv_minhash, uint8_t *densified) {
  if (!ctx) return SK_EINVAL;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  DeviceGuard dev(ctx->device);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  st = check_inputs(ctx, bases, seq_offsets, sample_seqs, n_samples, kmers, n_kmers, sketchsize64,
                    use_rc, codon_phased, min_count);
  if (st != SK_OK || n_samples == 0) return st;
  if (!words) return fail(ctx, SK_EINVAL, "null output words");
  SketchCall c{};
  st = setup_call(c, ctx, bases, false, seq_offsets, sample_seqs, n_samples, kmers, n_kmers,
                  sketchsize64, use_rc, codon_phased, min_count, nullptr, nullptr);
  if (st == SK_OK) st = sketch_to_device(c);
  if (st != SK_OK) return drain(ctx, st);
  const size_t n_words = static_cast<size_t>(n_samples) * n_kmers * sketchsize64 * kBbits;
  const size_t rows = static_cast<size_t>(n_samples) * n_kmers;
  std::vector<int8_t> dens(rows);
  cudaError_t e = cudaMemcpyAsync(words, c.d_words, n_words * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && inv_minhash)
    e = cudaMemcpyAsync(inv_minhash, c.d_inv, rows * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dens.data(), c.d_dens, rows, cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return drain(ctx, cuda_fail(ctx, e, "sketch download"));
  st = finish_call(ctx);
  if (st != SK_OK) return st;
  if (densified)
    for (int64_t s = 0; s < n_samples; ++s) {
      uint8_t any = 0;
      for (int k = 0; k < n_kmers; ++k) any |= dens[s * n_kmers + k] != 0;
      densified[s] = any;
    }
  return SK_OK;
}

sk_status sk_sketch_device(sk_ctx *ctx, const char *d_bases, const int64_t *seq_offsets,
                           const int64_t *sample_seqs, int64_t n_samples, const int32_t *kmers,
                           int32_t n_kmers, int32_t sketchsize64, int32_t use_rc,
                           int32_t codon_phased, int32_t min_count, uint64_t *d_words,
                           double *d_inv_minhash, uint8_t *d_densified) {
  if (!ctx) return SK_EINVAL;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  DeviceGuard dev(ctx->device);
  sk_status st = begin_call(ctx);
  if (st != SK_OK) return st;
  st = check_inputs(ctx, d_bases, seq_offsets, sample_seqs, n_samples, kmers, n_kmers, sketchsize64,
                    use_rc, codon_phased, min_count);
  if (st != SK_OK || n_samples == 0) return st;
  if (!d_words) return fail(ctx, SK_EINVAL, "null output words");
  SketchCall c{};
  st = setup_call(c, ctx, d_bases, true, seq_offsets, sample_seqs, n_samples, kmers, n_kmers,
                  sketchsize64, use_rc, codon_phased, min_count, d_words, d_inv_minhash);
  if (st == SK_OK) st = sketch_to_device(c);
  if (st != SK_OK) return drain(ctx, st);
  if (d_densified) {
    densified_kernel<<<static_cast<unsigned>((n_samples + 255) / 256), 256, 0, ctx->stream>>>(
        c.d_dens, n_samples, n_kmers, d_densified);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "densify flags");
  }
  return finish_call(ctx);
}

}  // extern "C"
