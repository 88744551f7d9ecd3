// ref_sketch.cpp -- synthetic genomes sketched by the reference's own sketcher.
//
// TEST INFRASTRUCTURE ONLY.  Builds the inputs of the CPU-runnable parity
// case: 64 genomes of 2.5 Mb derived from one seeded root, sketched with the
// reference's sketch() (src/sketch/sketch.cpp:120-168, compiled from the
// reference sources by oracle/Makefile with -DWEB_SKETCH, which leaves out
// the GPU headers).  The sketches then go through the CUDA path and the
// oracle like any other database.
//
// Genome model: i.i.d. bases at GC 0.38 (A = T = 0.31, C = G = 0.19) for the
// root; genome i > 0 copies a uniformly chosen earlier genome, then mutates a
// fraction c ~ U(0, 0.004) of positions to another base (core SNPs) and
// replaces a fraction a ~ U(0, 0.03) of the sequence with fresh random 5 kb
// segments (accessory).  Over the ~8 branches between two genomes of the
// random recursive tree, pairs span about 0-3% core and 0-20% accessory
// divergence.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "sketch/sketch.hpp"   // from the reference sources

namespace {

struct Rng {  // splitmix64
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  char base() {
    const double u = uniform();
    return u < 0.31 ? 'A' : u < 0.50 ? 'C' : u < 0.69 ? 'G' : 'T';
  }
};

}  // namespace

extern "C" {

// Writes n genomes of `length` bases to out (n * length chars, no separators).
void ref_make_genomes(int n, int64_t length, uint64_t seed, char *out) {
  Rng rng{seed};
  for (int64_t p = 0; p < length; ++p) out[p] = rng.base();
  for (int g = 1; g < n; ++g) {
    const int parent = static_cast<int>(rng.next() % static_cast<uint64_t>(g));
    char *dst = out + static_cast<int64_t>(g) * length;
    std::memcpy(dst, out + static_cast<int64_t>(parent) * length, length);
    const double c = 0.004 * rng.uniform();
    const double a = 0.03 * rng.uniform();
    const int64_t snps = static_cast<int64_t>(c * length);
    for (int64_t s = 0; s < snps; ++s) {
      const int64_t p = static_cast<int64_t>(rng.next() % static_cast<uint64_t>(length));
      char b;
      do {
        b = rng.base();
      } while (b == dst[p]);
      dst[p] = b;
    }
    const int64_t seg = 5000;
    const int64_t segments = static_cast<int64_t>(a * length / seg);
    for (int64_t s = 0; s < segments; ++s) {
      const int64_t p = static_cast<int64_t>(rng.next() % static_cast<uint64_t>(length - seg));
      for (int64_t q = 0; q < seg; ++q) dst[p + q] = rng.base();
    }
  }
}

// Sketches n genomes of `length` bases with the reference's sketch() at the
// given k-mer lengths: out [n][K][sketchsize64 * 14] in the reference word
// layout.  Returns the number of genomes that came out densified.
int ref_sketch_genomes(const char *seqs, int n, int64_t length, const int32_t *kmers, int K,
                       int sketchsize64, int use_rc, int threads, uint64_t *out) {
  std::vector<size_t> kl(kmers, kmers + K);
  const KmerSeeds seeds = generate_seeds(kl, false);
  const int64_t W = static_cast<int64_t>(sketchsize64) * 14;
  int densified = 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads) reduction(+ : densified)
  for (int g = 0; g < n; ++g) {
    SeqBuf buf(std::vector<std::string>{std::string(seqs + static_cast<int64_t>(g) * length, length)});
    bool any = false;
    for (int k = 0; k < K; ++k) {
      auto res = sketch(buf, static_cast<uint64_t>(sketchsize64), seeds.at(kl[k]), 14, false,
                        use_rc != 0, 0, false);
      const std::vector<uint64_t> &usigs = std::get<0>(res);
      std::memcpy(out + (static_cast<int64_t>(g) * K + k) * W, usigs.data(), W * 8);
      any = any || std::get<2>(res);
    }
    densified += any ? 1 : 0;
  }
  return densified;
}

// Sketches n samples given as sequences with the reference's sketch():
// sample s owns sequences sample_seqs[s] .. sample_seqs[s+1], sequence i is
// bases[seq_off[i], seq_off[i+1]).  Outputs words [n][K][sketchsize64 * 14],
// inv_minhash [n][K] (bin 0 over 2^61-1 before densifying) and densified [n]
// (any k densified).  The sequences go in as given (no case change, no length
// filter): the reference's SeqBuf(std::vector<std::string>) constructor.
// codon_phased selects the reference's spaced seeds (generate_seeds).
void ref_sketch_seqs(const char *bases, const int64_t *seq_off, const int64_t *sample_seqs, int n,
                     const int32_t *kmers, int K, int sketchsize64, int use_rc, int codon_phased,
                     int threads, uint64_t *out, double *inv_minhash, uint8_t *densified) {
  std::vector<size_t> kl(kmers, kmers + K);
  const KmerSeeds seeds = generate_seeds(kl, codon_phased != 0);
  const int64_t W = static_cast<int64_t>(sketchsize64) * 14;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
  for (int s = 0; s < n; ++s) {
    std::vector<std::string> seqs;
    for (int64_t q = sample_seqs[s]; q < sample_seqs[s + 1]; ++q)
      seqs.emplace_back(bases + seq_off[q], static_cast<size_t>(seq_off[q + 1] - seq_off[q]));
    SeqBuf buf(seqs);
    bool any = false;
    for (int k = 0; k < K; ++k) {
      auto res = sketch(buf, static_cast<uint64_t>(sketchsize64), seeds.at(kl[k]), 14,
                        codon_phased != 0, use_rc != 0, 0, false);
      std::memcpy(out + (static_cast<int64_t>(s) * K + k) * W, std::get<0>(res).data(), W * 8);
      inv_minhash[static_cast<int64_t>(s) * K + k] = std::get<1>(res);
      any = any || std::get<2>(res);
    }
    densified[s] = any ? 1 : 0;
  }
}

// Sketches one sample read from sequence files the way constructDatabase does
// (src/api.cpp:87-89): SeqBuf(files, largest k) -- upper-cased, sequences
// shorter than the largest k dropped, FASTQ input marks a read set -- then
// sketch() at each k with the given min_count and exact flag.  Outputs as
// ref_sketch_seqs for one sample; returns 1 if the input was a read set.
int ref_sketch_file(const char *path, const int32_t *kmers, int K, int sketchsize64, int use_rc,
                    int min_count, int exact, uint64_t *out, double *inv_minhash,
                    uint8_t *densified) {
  std::vector<size_t> kl(kmers, kmers + K);
  const KmerSeeds seeds = generate_seeds(kl, false);
  const int64_t W = static_cast<int64_t>(sketchsize64) * 14;
  SeqBuf buf(std::vector<std::string>{std::string(path)}, *std::max_element(kl.begin(), kl.end()));
  bool any = false;
  for (int k = 0; k < K; ++k) {
    auto res = sketch(buf, static_cast<uint64_t>(sketchsize64), seeds.at(kl[k]), 14, false,
                      use_rc != 0, static_cast<uint8_t>(min_count), exact != 0);
    std::memcpy(out + k * W, std::get<0>(res).data(), W * 8);
    inv_minhash[k] = std::get<1>(res);
    any = any || std::get<2>(res);
  }
  *densified = any ? 1 : 0;
  return buf.is_reads() ? 1 : 0;
}

// What the reference's SeqBuf(files, kmer_len) keeps of one file
// (src/sketch/seqio.cpp:55-100): the kept sequences back to back in `bases`
// (capacity cap bytes) with their offsets in `off` (capacity cap_seqs + 1),
// and info = {n_seqs, total bases, N count, reads, max_length}, freq = base
// composition A, C, G, T.  Returns 0, or -1 when a capacity is too small.
int ref_seqbuf(const char *path, int kmer_len, char *bases, int64_t cap, int64_t *off,
               int64_t cap_seqs, int64_t *info, double *freq) {
  SeqBuf buf(std::vector<std::string>{std::string(path)}, static_cast<size_t>(kmer_len));
  int64_t n = 0, used = 0;
  off[0] = 0;
  while (buf.nseqs() > 0 && !buf.eof()) {
    const std::string &q = *buf.getseq();
    if (n >= cap_seqs || used + static_cast<int64_t>(q.size()) > cap) return -1;
    std::memcpy(bases + used, q.data(), q.size());
    used += static_cast<int64_t>(q.size());
    off[++n] = used;
    buf.move_next_seq();
  }
  const BaseComp<double> c = buf.get_composition();
  info[0] = n;
  info[1] = static_cast<int64_t>(c.total);
  info[2] = static_cast<int64_t>(buf.missing_bases());
  info[3] = buf.is_reads() ? 1 : 0;
  info[4] = static_cast<int64_t>(buf.max_length());
  freq[0] = c.a;
  freq[1] = c.c;
  freq[2] = c.g;
  freq[3] = c.t;
  return 0;
}

}  // extern "C"
