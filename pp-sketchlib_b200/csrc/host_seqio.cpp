// host_seqio.cpp -- FASTA/FASTQ reading for constructDatabase (see
// host_seqio.h).  A buffered byte reader over zlib's gzread, which also reads
// uncompressed files, and a record parser with the reference reader's rules.
#include "host_seqio.h"

#include <zlib.h>

#include <stdexcept>

namespace skhost {
namespace {

constexpr uint64_t kCompositionSample = 1000000;   // max_composition_sample (src/sketch/seqio.cpp:24)

class Reader {
 public:
  explicit Reader(const std::string &path) : f_(gzopen(path.c_str(), "rb")) {
    if (!f_) throw std::runtime_error("Could not open " + path);
    gzbuffer(f_, 1 << 20);
  }
  ~Reader() {
    if (f_) gzclose(f_);
  }
  Reader(const Reader &) = delete;
  Reader &operator=(const Reader &) = delete;

  int get() {
    if (pos_ == len_) {
      const int n = gzread(f_, buf_.data(), static_cast<unsigned>(buf_.size()));
      if (n <= 0) return -1;
      len_ = static_cast<size_t>(n);
      pos_ = 0;
    }
    return static_cast<unsigned char>(buf_[pos_++]);
  }
  // Appends the rest of the line (without '\n') to s; returns the byte that
  // ended it ('\n' or -1).
  int rest_of_line(std::string &s) {
    int c;
    while ((c = get()) != -1 && c != '\n') s.push_back(static_cast<char>(c));
    return c;
  }

 private:
  gzFile f_;
  std::vector<char> buf_ = std::vector<char>(1 << 20);
  size_t len_ = 0, pos_ = 0;
};

void strip_cr(std::string &s) {
  if (s.size() > 1 && s.back() == '\r') s.pop_back();
}

// One record: returns false at end of file or on a truncated quality string.
bool next_record(Reader &r, int &pending, std::string &seq, bool &has_qual) {
  int c = pending;
  if (c == 0) {
    while ((c = r.get()) != -1 && c != '>' && c != '@') {
    }
    if (c == -1) return false;
  }
  pending = 0;
  seq.clear();
  has_qual = false;
  // header: name up to white space, then the rest of the line
  while ((c = r.get()) != -1 && c != '\n') {
  }
  if (c == -1) return false;
  while ((c = r.get()) != -1 && c != '>' && c != '+' && c != '@') {
    if (c == '\n') continue;
    seq.push_back(static_cast<char>(c));
    r.rest_of_line(seq);
    strip_cr(seq);
  }
  if (c == '>' || c == '@') pending = c;
  if (c != '+') return true;
  while ((c = r.get()) != -1 && c != '\n') {
  }
  if (c == -1) return false;
  std::string qual;
  while (qual.size() < seq.size()) {
    const int e = r.rest_of_line(qual);
    strip_cr(qual);
    if (e == -1) break;
  }
  if (qual.size() != seq.size()) return false;
  has_qual = !qual.empty();
  return true;
}

}  // namespace

SampleSeqs read_sample(const std::vector<std::string> &files, size_t min_len) {
  SampleSeqs out;
  uint64_t counts[4] = {0, 0, 0, 0};
  for (const std::string &path : files) {
    Reader r(path);
    int pending = 0;
    std::string seq;
    bool has_qual = false;
    while (next_record(r, pending, seq, has_qual)) {
      if (seq.size() > out.max_length) out.max_length = seq.size();
      if (seq.size() >= min_len) {
        for (char &ch : seq) {
          if (ch >= 'a' && ch <= 'z') ch = static_cast<char>(ch ^ 0x20);
          ++out.total;
          if (out.total < kCompositionSample) {
            switch (ch) {
              case 'A': ++counts[0]; break;
              case 'C': ++counts[1]; break;
              case 'G': ++counts[2]; break;
              case 'T': case 'U': ++counts[3]; break;
              default: break;
            }
          }
          if (ch == 'N') ++out.missing_bases;
        }
        out.seqs.push_back(std::move(seq));
        seq = std::string();
      }
      if (has_qual) out.reads = true;
    }
  }
  // one reciprocal, four products: what the reference's Release build
  // (-ffast-math) computes for its four divisions by the same total
  const double inv = 1.0 / static_cast<double>(out.total < kCompositionSample ? out.total : kCompositionSample);
  for (int b = 0; b < 4; ++b) out.base_freq[b] = static_cast<double>(counts[b]) * inv;
  return out;
}

}  // namespace skhost
