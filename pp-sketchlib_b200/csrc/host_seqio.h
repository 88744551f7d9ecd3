// host_seqio.h -- FASTA/FASTQ reading for the drop-in module's
// constructDatabase: what the reference's SeqBuf keeps of a sample's files
// (src/sketch/seqio.cpp:55-100), ready for sk_sketch.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace skhost {

struct SampleSeqs {
  std::vector<std::string> seqs;   // kept sequences, upper case
  bool reads = false;              // any record carried a quality string
  uint64_t missing_bases = 0;      // 'N' bases in the kept sequences
  uint64_t total = 0;              // bases in the kept sequences
  double base_freq[4] = {0, 0, 0, 0};   // A, C, G, T(+U) over the first 10^6 bases
  size_t max_length = 0;           // longest record, kept or not
};

// Reads every FASTA/FASTQ file (plain or gzip) of one sample.  Records are
// parsed as the reference's kseq reader does: a header starts with '>' or
// '@', sequence lines run to the next line starting with '>', '@' or '+',
// empty lines are skipped and a trailing '\r' is dropped; a '+' line starts
// the quality string, read until it is as long as the sequence (a record
// whose quality string ends short stops reading that file).  Sequences of at
// least min_len bases are kept, upper-cased; composition counts A, C, G, T/U
// among the first 999,999 kept bases over min(total, 10^6).  Throws
// std::runtime_error when a file cannot be opened.
SampleSeqs read_sample(const std::vector<std::string> &files, size_t min_len);

}  // namespace skhost
