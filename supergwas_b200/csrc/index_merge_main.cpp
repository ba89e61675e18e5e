// index_merge_main.cpp -- bin/kgwas_index_merge: joins the sharded k-mer
// indexes that `kgwas --index-out` / `--index-2d-out` wrote per batch into the
// index that the reference's build_index makes of all the batches' files
// (src/build_index.cpp:29-273; build_index.sh over the .tsv files,
// build_index_2d.sh over the .2d.tsv files):
//
//   kgwas_index_merge OUT_DIR IN_DIR [IN_DIR ...] [--shards M]
//
// The records are binary already, so no text is parsed: every input's rows are
// read, re-sharded by (canonical encoding & (M - 1)), sorted by encoding and
// written with their Bloom filters.  M defaults to the first input's.  Where
// several inputs hold the same canonical k-mer the first input given wins;
// build_index keeps one of them with no rule (an unstable sort over files
// loaded in parallel).
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "kgwas_io.hpp"

using kgio::die;

int main(int argc, char** argv) {
  std::vector<std::string> pos;
  uint32_t M = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--shards" && i + 1 < argc) M = (uint32_t)std::stoul(argv[++i]);
    else pos.push_back(a);
  }
  if (pos.size() < 2) {
    std::cerr << "Usage:\n  " << argv[0] << " <out_dir> <index_dir> [<index_dir> ...] [--shards M]\n";
    return 1;
  }
  kgio::Timer t;
  std::vector<kgio::IndexRow> rows;
  uint32_t K = 0;
  for (size_t i = 1; i < pos.size(); ++i) {
    uint32_t k = 0, m = 0;
    const size_t before = rows.size();
    if (!kgio::read_index_rows(pos[i], k, m, rows)) die("Failed to read index " + pos[i]);
    if (K && k != K) die("K mismatch: " + pos[i] + " has K=" + std::to_string(k) + ", expected " + std::to_string(K));
    K = k;
    if (!M) M = m;
    std::cerr << "[INFO] " << pos[i] << ": " << rows.size() - before << " records (K=" << k << ", M=" << m << ")\n";
  }
  if (M == 0 || (M & (M - 1)) != 0) die("--shards must be a power of 2, got " + std::to_string(M));
  const size_t n_in = rows.size();
  if (!kgio::write_index(pos[0], K, M, rows)) die("Failed to write index " + pos[0]);
  std::cerr << "[INFO] merged " << n_in << " records into a " << M << "-shard index at " << pos[0] << " in "
            << t.sec() << " s\n";
  return 0;
}
