// kgwas_io.hpp -- file readers of the kgwas program.
//
// Same inputs, checks and [ERROR] messages as the reference's readers
// (src/kgwas_utils.hpp), but the column matrix is packed straight into
// k-mer-major bit rows (1 bit per sample) instead of an n x N float matrix.
#pragma once
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

namespace kgio {

[[noreturn]] void die(const std::string& m);   // "[ERROR] m", exit(1)
void warn(const std::string& m);               // "[WARN] m"
// Thread counts from the environment (LOAD_THREADS, BLAS_THREADS,
// EMIT_THREADS; src/kgwas_utils.hpp:43-47): the leading integer, at least 1,
// else `fallback`.
int env_int(const char* name, int fallback);

struct Timer {
  double t0;
  Timer();
  double sec() const;
};

// samples.txt (src/kgwas_utils.hpp:51-61): one id per line, empty lines
// skipped, one trailing '\r' dropped.  "[ERROR] open: file" when unreadable.
std::vector<std::string> read_sample_ids(const std::string& file);

// The overlap of the sample list with a phenotype file of whitespace-
// separated "id value" pairs (src/kgwas_utils.hpp:63-70, 285-314): the
// positions in the sample list whose id has a value, in list order, and
// their values (the last pair of an id wins).  No emptiness checks.
struct Overlap {
  std::vector<int> idxs;                        // positions in samples.txt
  std::vector<std::string> samples;
  std::vector<double> y;
};
Overlap match_phenotypes(const std::vector<std::string>& ids, const std::string& pheno_file);
// COLS mode: read_sample_ids + match_phenotypes with the "samples empty" and
// "no phenotype overlap" checks and the [INFO] line.
Overlap build_overlap(const std::string& samples_file, const std::string& pheno_file);

// U.bin (src/compute_structure_all.cpp:80-88): int32 n, int32 k, then n*k
// FP64 column-major.  read_ubin_file only parses; the modes word their own
// errors (COLS: load_ubin, src/kgwas_utils.hpp:129-157; ROWS:
// src/kgwas.cpp:372-381).
struct UbinFile {
  enum Status { kOk, kNoFile, kShortHeader, kShortBody } status = kNoFile;
  int n = 0, k = 0;           // header fields that were present (0 otherwise)
  size_t header_bytes = 0;
  std::vector<double> U;      // the values present: n*k when the body is complete
};
UbinFile read_ubin_file(const std::string& path);
struct UData {
  std::vector<double> U;                        // n x k column-major
  int n = 0, k = 0;
};
UData load_ubin(const std::string& path, int n);

size_t infer_N_from_bits(const std::string& bits_dir, int first_idx);   // src/kgwas_utils.hpp:317-332
std::vector<std::string> load_kmers(const std::string& path, size_t N);  // src/kgwas_utils.hpp:93-127

inline uint32_t words_per_kmer(int n) {
  uint32_t w = (uint32_t)((n + 63) / 64);
  return w + (w & 1u);
}

// src/kgwas_utils.hpp:225-282: column k of the overlap is bits/col_%06d of
// idxs[k] (.txt preferred over .txt.gz); row i is byte i & 1.  Writes
// N x words_per_kmer(n) packed words into `out` (caller-allocated).
void load_matrix_packed(const std::string& bits_dir, const std::vector<int>& idxs, size_t N, int threads,
                        uint64_t* out);

// ROWS-mode input (src/kgwas.cpp:435-459): "kmer<TAB or SPACE>bitstring" lines,
// x_j = (bits[idxs[j]] == '1').  Appends to kmers/packed.
// Lines are parsed in parallel (`threads` host threads) from large blocks of
// the file; the rows come back in file order.
struct RowsReader {
  explicit RowsReader(const std::string& path, int threads = 1);
  ~RowsReader();
  // Reads up to max_rows rows; returns the number read (0 at end).
  size_t read(size_t max_rows, const std::vector<int>& idxs, std::vector<std::string>& kmers,
              std::vector<uint64_t>& packed);
  size_t lines = 0;   // non-empty lines seen (the reference's line_count)
 private:
  void* gz = nullptr;
  const char* map = nullptr;  // a plain file, mapped whole
  size_t map_sz = 0;
  int threads = 1;
  std::vector<char> buf;  // gz: inflated bytes [beg, end) not yet parsed
  size_t beg = 0, end = 0;
  bool eof = false;
  const char* data() const { return map ? map : buf.data(); }
  void fill();
};

// Sharded k-mer index with bitstrings (the input of the 2-D pair test):
// INDEX_DIR/index.meta ("K=", "M=", "N=" lines) and, per shard s < M,
// shard_%03u.umap (magic "UMAPd4\0\0", uint32 K, uint64 N, N records of a
// 16-byte 2-bit-encoded canonical k-mer + FP64 effect + FP64 p) and
// shard_%03u.bits (uint64 N, then per record uint32 length + bitstring).
// Follows load_X_from_index (src/kgwas_2d.cpp:80-153) and read_index_meta /
// load_shard (src/map_utils.hpp:319-479): the k-mers that carry a bitstring,
// sorted by their encoding, decoded to A/C/G/T.  Failures print the
// reference's [ERROR] lines and exit(1).
struct IndexBits {
  uint32_t K = 0;
  std::vector<std::string> kmers;
  std::vector<std::string> bits;
};
IndexBits load_index_bits(const std::string& dir, int threads);

// Writing the same sharded index (the input of the 2-D test) straight from
// emitted rows, without the text pass of the reference's build_index
// (src/build_index.cpp:29-273): a k-mer is stored under its canonical 2-bit
// encoding (the smaller of the k-mer and its reverse complement, A/C/G/T =
// 0/1/2/3, first base most significant) in shard (encoding & (M - 1)); each
// shard is sorted by encoding, duplicates keep one entry, and gets its .umap,
// .bits (when any entry has a bitstring) and a 2-hash Bloom filter (.bloom,
// 10 bits per entry rounded up to a power of two, SplitMix64 finaliser).
struct IndexRow {
  unsigned __int128 key = 0;  // canonical encoding
  uint32_t k = 0;             // k-mer length
  double effect = 0, pval = 0;
  std::string bits;
};
// Canonical encoding of a k-mer; false if it holds a base other than ACGT/acgt
// or is longer than 64.
bool canonical_kmer(const std::string& kmer, unsigned __int128& key);
// Writes index.meta and shard_%03u.{umap,bits,bloom}, s < M (M a power of 2);
// returns false (with an [ERROR] line) when a file cannot be written.
bool write_index(const std::string& dir, uint32_t K, uint32_t M, std::vector<IndexRow>& rows);
// Appends every record of an index written as above, shard by shard in file
// order, with its bitstring (empty where the shard has no .bits); sets K and M
// from index.meta.  false (with an [ERROR] line) on a missing or malformed file.
bool read_index_rows(const std::string& dir, uint32_t& K, uint32_t& M, std::vector<IndexRow>& rows);

}  // namespace kgio
