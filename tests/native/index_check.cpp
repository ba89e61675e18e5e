// index_check.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Feeds the rows of a kgwas output file to the library's index writer
// (kgio::write_index, supergwas_b200/csrc/kgwas_io.cpp) the way kgwas
// --index-out / --index-2d-out do, so that the CPU test suite can compare its
// files with the reference build_index's.  Rows are "kmer<TAB>effect<TAB>p"
// (.tsv) or "kmer<TAB>bits<TAB>effect<TAB>p" (.2d.tsv); k is the first row's
// k-mer length and rows of another length are left out.
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "../../supergwas_b200/csrc/kgwas_io.hpp"

extern "C" int index_from_tsv(const char* tsv, const char* dir, unsigned M) {
  std::ifstream in(tsv);
  if (!in) return -1;
  std::vector<kgio::IndexRow> rows;
  std::string line;
  uint32_t K = 0;
  while (std::getline(in, line)) {
    if (line.empty()) continue;
    const size_t t1 = line.find('\t');
    const size_t t2 = t1 == std::string::npos ? t1 : line.find('\t', t1 + 1);
    if (t2 == std::string::npos) return -2;
    const size_t t3 = line.find('\t', t2 + 1);
    const std::string kmer = line.substr(0, t1);
    if (!K) K = (uint32_t)kmer.size();
    kgio::IndexRow r;
    if (kmer.size() != K || !kgio::canonical_kmer(kmer, r.key)) continue;
    r.k = K;
    size_t e = t1 + 1, p = t2 + 1;
    if (t3 != std::string::npos) {
      r.bits = line.substr(t1 + 1, t2 - t1 - 1);
      e = t2 + 1;
      p = t3 + 1;
    }
    r.effect = std::strtod(line.c_str() + e, nullptr);
    r.pval = std::strtod(line.c_str() + p, nullptr);
    rows.push_back(std::move(r));
  }
  return kgio::write_index(dir, K, M, rows) ? 0 : -3;
}
