// rows_check.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Reads a ROWS-mode file with the library's reader (kgio::RowsReader,
// supergwas_b200/csrc/kgwas_io.cpp) in batches of max_rows rows, as the kgwas
// program does, and hands back the packed rows, the k-mers (one per line) and
// the reader's count of non-empty lines.
#include <cstring>
#include <string>
#include <vector>

#include "../../supergwas_b200/csrc/kgwas_io.hpp"

extern "C" long rows_parse(const char* path, const int* idxs, int n, int threads, unsigned long max_rows,
                           uint64_t* packed_out, unsigned long packed_cap, char* kmers_out,
                           unsigned long kmers_cap, unsigned long* lines_out, unsigned long* batches_out) {
  std::vector<int> ix(idxs, idxs + n);
  kgio::RowsReader rr(path, threads);
  std::vector<std::string> kmers;
  std::vector<uint64_t> packed;
  unsigned long batches = 0, total = 0;
  std::string joined;
  std::vector<uint64_t> all;
  for (;;) {
    kmers.clear();
    packed.clear();
    const size_t got = rr.read(max_rows, ix, kmers, packed);
    if (got == 0) break;
    if (got > max_rows) return -2;
    ++batches;
    total += got;
    for (auto& k : kmers) joined += k + "\n";
    all.insert(all.end(), packed.begin(), packed.end());
  }
  if (all.size() > packed_cap || joined.size() + 1 > kmers_cap) return -1;
  std::memcpy(packed_out, all.data(), all.size() * 8);
  std::memcpy(kmers_out, joined.c_str(), joined.size() + 1);
  *lines_out = rr.lines;
  *batches_out = batches;
  return (long)total;
}
