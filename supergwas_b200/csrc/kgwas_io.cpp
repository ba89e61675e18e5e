// kgwas_io.cpp -- see kgwas_io.hpp.
#include "kgwas_io.hpp"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <climits>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <memory>
#include <mutex>
#include <sstream>

#include <omp.h>

namespace kgio {

// One [ERROR] line even when several threads fail at once, and no exit-time
// teardown while another thread may be inside the CUDA runtime (the programs
// set up the GPU on a thread of their own while they read their inputs).
void die(const std::string& m) {
  static std::mutex mu;
  mu.lock();
  std::cerr << "[ERROR] " << m << "\n";
  std::cerr.flush();
  std::fflush(stdout);
  std::_Exit(1);
}

void warn(const std::string& m) { std::cerr << "[WARN] " << m << "\n"; }

// A thread count from the environment: the leading integer of the value
// (after blanks, with an optional sign; trailing text ignored), at least 1;
// `fallback` when the variable is unset or empty, has no leading integer or
// leaves the int range.
int env_int(const char* name, int fallback) {
  const char* text = std::getenv(name);
  if (text == nullptr || text[0] == '\0') return fallback;
  errno = 0;
  char* stop = nullptr;
  const long v = std::strtol(text, &stop, 10);
  if (stop == text || errno == ERANGE || v < INT_MIN || v > INT_MAX) return fallback;
  return v < 1 ? 1 : (int)v;
}

static double now_s() {
  using clk = std::chrono::steady_clock;
  return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}
Timer::Timer() : t0(now_s()) {}
double Timer::sec() const { return now_s() - t0; }

// ------------------------------------------------------------ input sources
namespace {

// A regular file mapped read-only for the lifetime of the object.  open()
// reports which step failed; files shorter than `min_size` are not mapped.
class MappedFile {
 public:
  enum Status { kOk, kEmpty, kTooShort, kNotRegular, kOpenFailed, kStatFailed, kMapFailed };
  MappedFile() = default;
  MappedFile(const MappedFile&) = delete;
  MappedFile& operator=(const MappedFile&) = delete;
  MappedFile(MappedFile&& o) noexcept { swap(o); }
  MappedFile& operator=(MappedFile&& o) noexcept {
    swap(o);
    return *this;
  }
  ~MappedFile() {
    if (base_) munmap(base_, size_);
  }

  Status open(const std::string& path, size_t min_size = 1) {
    const int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) return kOpenFailed;
    struct stat info {};
    Status s = kOk;
    if (fstat(fd, &info) != 0) s = kStatFailed;
    else if (!S_ISREG(info.st_mode)) s = kNotRegular;
    else {
      size_ = (size_t)info.st_size;
      if (size_ == 0) s = kEmpty;
      else if (size_ < min_size) s = kTooShort;
      else {
        void* p = mmap(nullptr, size_, PROT_READ, MAP_PRIVATE, fd, 0);
        if (p == MAP_FAILED) s = kMapFailed;
        else {
          base_ = p;
          madvise(p, size_, MADV_SEQUENTIAL);
        }
      }
    }
    ::close(fd);
    return s;
  }
  const unsigned char* bytes() const { return static_cast<const unsigned char*>(base_); }
  size_t size() const { return size_; }

 private:
  void swap(MappedFile& o) noexcept {
    std::swap(base_, o.base_);
    std::swap(size_, o.size_);
  }
  void* base_ = nullptr;
  size_t size_ = 0;
};

// A gzip stream read through zlib's gz interface with a 1 MB buffer.
class GzSource {
 public:
  explicit GzSource(const std::string& path) : f_(gzopen(path.c_str(), "rb")) {
    if (f_) gzbuffer(f_, 1u << 20);
  }
  GzSource(const GzSource&) = delete;
  GzSource& operator=(const GzSource&) = delete;
  ~GzSource() {
    if (f_) gzclose(f_);
  }
  bool ok() const { return f_ != nullptr; }
  // Up to `len` inflated bytes (fewer only at the end of the stream); -1 when
  // zlib reports an error (see error()).
  long long fill(void* dst, size_t len) {
    size_t have = 0;
    while (have < len) {
      const unsigned ask = (unsigned)std::min<size_t>(len - have, (size_t)1 << 30);
      const int r = gzread(f_, static_cast<unsigned char*>(dst) + have, ask);
      if (r < 0) return -1;
      if (r == 0) break;
      have += (size_t)r;
    }
    return (long long)have;
  }
  // zlib's state after a short or failed fill: its message and code.
  std::string error(int* code = nullptr) const {
    int c = Z_OK;
    const char* m = gzerror(f_, &c);
    if (code) *code = c;
    return m ? m : "";
  }

 private:
  gzFile f_;
};

// Whole file as bytes; false when it cannot be opened.
bool slurp(const std::string& path, std::string& out) {
  std::FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  out.clear();
  char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) out.append(chunk, got);
  std::fclose(f);
  return true;
}

// Calls fn(begin, length) for each '\n'-terminated line of [p, p + len) and
// for a last line without '\n' when it is not empty (std::getline's lines).
template <class Fn>
void for_each_line(const char* p, size_t len, Fn&& fn) {
  const char* end = p + len;
  while (p < end) {
    const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
    const char* stop = nl ? nl : end;
    fn(p, (size_t)(stop - p));
    if (!nl) break;
    p = nl + 1;
  }
}

bool is_regular(const std::string& p) {
  struct stat info {};
  return ::stat(p.c_str(), &info) == 0 && S_ISREG(info.st_mode);
}

// Where the column of one sample lives: bits/col_%06d.txt, else the same
// name with .gz (src/kgwas_utils.hpp:238-240).
struct ColumnFile {
  std::string plain, gz;
  enum Kind { kPlain, kGz, kMissing } kind;
};
ColumnFile locate_column(const std::string& bits_dir, int sample_pos) {
  char name[48];
  std::snprintf(name, sizeof(name), "/col_%06d.txt", sample_pos);
  ColumnFile c;
  c.plain = bits_dir + name;
  c.gz = c.plain + ".gz";
  c.kind = is_regular(c.plain) ? ColumnFile::kPlain : is_regular(c.gz) ? ColumnFile::kGz : ColumnFile::kMissing;
  return c;
}
[[noreturn]] void die_missing(const ColumnFile& c) { die("missing column: " + c.plain + " (and " + c.gz + ")"); }

// Length of the first line of a column file: the bytes before the first
// '\n', or the whole file when it has none.
size_t first_line_plain(const std::string& path) {
  MappedFile f;
  switch (f.open(path)) {
    case MappedFile::kOpenFailed: die("open: " + path);
    case MappedFile::kStatFailed: die("fstat: " + path);
    case MappedFile::kEmpty: die("empty: " + path);
    case MappedFile::kMapFailed:
    case MappedFile::kNotRegular:
    case MappedFile::kTooShort: die("mmap: " + path);
    case MappedFile::kOk: break;
  }
  const void* nl = std::memchr(f.bytes(), '\n', f.size());
  const size_t len = nl ? (size_t)(static_cast<const unsigned char*>(nl) - f.bytes()) : f.size();
  if (len == 0) die("no bytes before newline: " + path);
  return len;
}

size_t first_line_gz(const std::string& path) {
  GzSource z(path);
  if (!z.ok()) die("gzopen: " + path);
  std::vector<unsigned char> block((size_t)1 << 20);
  size_t before = 0;  // bytes of the first line in earlier blocks
  for (;;) {
    const long long got = z.fill(block.data(), block.size());
    if (got < 0) die("gzread error: " + z.error());
    const void* nl = std::memchr(block.data(), '\n', (size_t)got);
    if (nl) return before + (size_t)(static_cast<const unsigned char*>(nl) - block.data());
    before += (size_t)got;
    if ((size_t)got < block.size()) break;  // end of stream
  }
  if (before == 0) die("empty gz column: " + path);
  return before;
}

// One sample's column of N bytes: a mapping of the plain file, or the first
// N inflated bytes of the .gz file, which must end there or with '\n'.
struct ColumnBytes {
  MappedFile map;
  std::unique_ptr<unsigned char[]> inflated;
  const unsigned char* p = nullptr;
};

void open_column(const ColumnFile& c, size_t N, ColumnBytes& out) {
  if (c.kind == ColumnFile::kMissing) die_missing(c);
  if (c.kind == ColumnFile::kPlain) {
    switch (out.map.open(c.plain, N)) {
      case MappedFile::kOpenFailed: die("open: " + c.plain);
      case MappedFile::kStatFailed: die("fstat: " + c.plain);
      case MappedFile::kEmpty:
      case MappedFile::kTooShort:
        die("short column: " + c.plain + " (size " + std::to_string(out.map.size()) + " < N " + std::to_string(N) +
            ")");
      case MappedFile::kNotRegular:
      case MappedFile::kMapFailed: die("mmap: " + c.plain);
      case MappedFile::kOk: break;
    }
    out.p = out.map.bytes();
    return;
  }
  GzSource z(c.gz);
  if (!z.ok()) die("gzopen: " + c.gz);
  out.inflated.reset(new unsigned char[N + 1]);
  const long long got = z.fill(out.inflated.get(), N);
  if (got < 0 || (size_t)got < N) {
    int code = Z_OK;
    const std::string msg = z.error(&code);
    if (got >= 0 && code == Z_STREAM_END)
      die("short gz column: " + c.gz + " (got " + std::to_string(got) + " < N " + std::to_string(N) + ")");
    die("gzread error: " + msg);
  }
  // one byte past the column may only be the line end
  if (z.fill(out.inflated.get() + N, 1) == 1 && out.inflated[N] != '\n')
    die("gz column longer than expected (N+ extra non-newline): " + c.gz);
  out.p = out.inflated.get();
}

}  // namespace

// ---------------------------------------------------- samples and phenotype
std::vector<std::string> read_sample_ids(const std::string& file) {
  std::string text;
  if (!slurp(file, text)) die("open: " + file);
  std::vector<std::string> ids;
  for_each_line(text.data(), text.size(), [&](const char* p, size_t len) {
    if (len == 0) return;                   // empty lines are skipped ...
    if (p[len - 1] == '\r') --len;          // ... before one '\r' is dropped
    ids.emplace_back(p, len);
  });
  return ids;
}

// The phenotype file is a sequence of whitespace-separated (id, value) pairs
// read with formatted stream extraction, up to the first pair that does not
// parse; a later pair for the same id replaces an earlier one.  Each value
// goes to every position of its id in the sample list.
Overlap match_phenotypes(const std::vector<std::string>& ids, const std::string& pheno_file) {
  std::unordered_map<std::string, std::vector<int>> positions;
  positions.reserve(ids.size());
  for (int j = 0; j < (int)ids.size(); ++j) positions[ids[j]].push_back(j);
  std::string text;
  if (!slurp(pheno_file, text)) die("open: " + pheno_file);
  std::vector<double> value(ids.size(), 0.0);
  std::vector<char> seen(ids.size(), 0);
  std::istringstream pairs(std::move(text));
  std::string id;
  double v = 0.0;
  while (pairs >> id >> v) {
    const auto hit = positions.find(id);
    if (hit == positions.end()) continue;
    for (int j : hit->second) {
      value[j] = v;
      seen[j] = 1;
    }
  }
  Overlap ov;
  for (int j = 0; j < (int)ids.size(); ++j)
    if (seen[j]) {
      ov.idxs.push_back(j);
      ov.y.push_back(value[j]);
    }
  ov.samples = ids;
  return ov;
}

Overlap build_overlap(const std::string& samples_file, const std::string& pheno_file) {
  Timer t;
  const std::vector<std::string> ids = read_sample_ids(samples_file);
  if (ids.empty()) die("samples empty");
  Overlap ov = match_phenotypes(ids, pheno_file);
  if (ov.idxs.empty()) die("no phenotype overlap");
  std::cerr << "[INFO] n=" << ov.y.size() << " (overlap)  (" << t.sec() << " s)\n";
  return ov;
}

// -------------------------------------------------------------------- U.bin
UbinFile read_ubin_file(const std::string& path) {
  UbinFile u;
  std::string bytes;
  if (!slurp(path, bytes)) {
    u.status = UbinFile::kNoFile;
    return u;
  }
  int32_t head[2] = {0, 0};
  std::memcpy(head, bytes.data(), std::min<size_t>(bytes.size(), sizeof(head)));
  u.n = head[0];
  u.k = head[1];
  u.header_bytes = std::min<size_t>(bytes.size(), sizeof(head));
  if (u.header_bytes < sizeof(head)) {
    u.status = UbinFile::kShortHeader;
    return u;
  }
  const size_t body = bytes.size() - sizeof(head);
  if (u.n < 0 || u.k < 0) {
    u.status = UbinFile::kShortBody;
    return u;
  }
  const size_t want = (size_t)u.n * (size_t)u.k;
  const size_t have = std::min(want, body / sizeof(double));
  u.U.resize(have);
  if (have) std::memcpy(u.U.data(), bytes.data() + sizeof(head), have * sizeof(double));
  u.status = have == want ? UbinFile::kOk : UbinFile::kShortBody;
  return u;
}

UData load_ubin(const std::string& path, int n) {
  Timer t;
  UbinFile f = read_ubin_file(path);
  if (f.status == UbinFile::kNoFile) die("open: " + path);
  if (f.status == UbinFile::kShortHeader) die("short U.bin header");
  if (f.n != n) die("U.bin n mismatch: file n=" + std::to_string(f.n) + " vs overlap n=" + std::to_string(n));
  if (f.status != UbinFile::kOk) die("short U.bin body");
  UData ud;
  ud.n = n;
  ud.k = f.k;
  ud.U = std::move(f.U);
  std::cerr << "[INFO] loaded U (n=" << n << ", r=" << ud.k << ")  (" << t.sec() << " s)\n";
  return ud;
}

// ---------------------------------------------------------- batch directory
size_t infer_N_from_bits(const std::string& bits_dir, int first_idx) {
  Timer t;
  const ColumnFile c = locate_column(bits_dir, first_idx);
  if (c.kind == ColumnFile::kMissing) die_missing(c);
  const bool plain = c.kind == ColumnFile::kPlain;
  const size_t N = plain ? first_line_plain(c.plain) : first_line_gz(c.gz);
  if (N == 0) die("N=0");
  std::cerr << "[INFO] inferred N=" << N << " rows  (" << t.sec() << " s)"
            << (plain ? " [from .txt]" : " [from .txt.gz]") << "\n";
  return N;
}

std::vector<std::string> load_kmers(const std::string& path, size_t N) {
  std::vector<std::string> kmers;
  kmers.reserve(N);
  const bool gz = path.size() >= 3 && path.compare(path.size() - 3, 3, ".gz") == 0;
  if (gz) {
    GzSource z(path);
    if (!z.ok()) die("gzopen: " + path);
    // inflated in 4 MB blocks and split at '\n'; only '\n'-terminated lines
    // count (an unterminated last line is not a k-mer), as with gzgets
    std::vector<char> buf((size_t)4 << 20);
    std::string part;  // a line that continues in the next block
    while (kmers.size() < N) {
      const long long r = z.fill(buf.data(), buf.size());
      if (r <= 0) {
        int code = Z_OK;
        const std::string msg = z.error(&code);
        if (r < 0 || (code != Z_OK && code != Z_STREAM_END)) die("gzgets error: " + msg);
        break;
      }
      const char* p = buf.data();
      const char* e = p + r;
      while (p < e && kmers.size() < N) {
        const char* nl = (const char*)std::memchr(p, '\n', (size_t)(e - p));
        if (!nl) {
          part.append(p, (size_t)(e - p));
          break;
        }
        if (part.empty()) {
          kmers.emplace_back(p, (size_t)(nl - p));
        } else {
          part.append(p, (size_t)(nl - p));
          kmers.push_back(std::move(part));
          part.clear();
        }
        p = nl + 1;
      }
    }
  } else {
    // plain: std::getline's lines (a last line without '\n' counts), one
    // trailing '\r' dropped, empty lines kept
    MappedFile f;
    const MappedFile::Status s = f.open(path);
    if (s == MappedFile::kOpenFailed) die("open: " + path);
    if (s == MappedFile::kOk) {
      const char* text = reinterpret_cast<const char*>(f.bytes());
      for_each_line(text, f.size(), [&](const char* p, size_t len) {
        if (kmers.size() >= N) return;
        if (len && p[len - 1] == '\r') --len;
        kmers.emplace_back(p, len);
      });
    }
  }
  if (kmers.size() != N)
    die("kmers lines != N (got " + std::to_string(kmers.size()) + ", expected " + std::to_string(N) + ")");
  return kmers;
}

void load_matrix_packed(const std::string& bits_dir, const std::vector<int>& idxs, size_t N, int threads,
                        uint64_t* out) {
  Timer t;
  const int n = (int)idxs.size();
  const uint32_t W = words_per_kmer(n);
  std::vector<ColumnBytes> cols(n);
  std::atomic<int> done{0};
  omp_set_num_threads(std::max(1, threads));
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < n; ++k) {
    open_column(locate_column(bits_dir, idxs[k]), N, cols[k]);
    const int d = ++done;
    if ((d % 8) == 0) {
#pragma omp critical
      std::cerr << "\r[LOAD] " << d << "/" << n << std::flush;
    }
  }
  // Transpose 64 sample columns at a time into one word column: 8 k-mers x 8
  // samples per step, each sample's 8 bytes read as one word whose low bits
  // (the '0'/'1' parity) land in 8 bits of one byte per k-mer.
  const size_t BLK = 8192;
  const size_t nblk = (N + BLK - 1) / BLK;
#pragma omp parallel
  {
    std::vector<uint64_t> acc(BLK);
#pragma omp for schedule(static)
    for (size_t b = 0; b < nblk; ++b) {
      const size_t j0 = b * BLK, len = std::min(BLK, N - j0);
      for (uint32_t wc = 0; wc < W; ++wc) {
        std::fill(acc.begin(), acc.begin() + len, 0ull);
        uint8_t* ab = reinterpret_cast<uint8_t*>(acc.data());  // byte q of a word: samples 8q..8q+7 (little-endian)
        const size_t len8 = len & ~(size_t)7;
        for (int q = 0; q < 8; ++q) {
          const int s0 = (int)wc * 64 + q * 8;
          if (s0 >= n) break;
          const int ns = n - s0 < 8 ? n - s0 : 8;
          const unsigned char* src[8];
          for (int t = 0; t < 8; ++t) src[t] = cols[s0 + (t < ns ? t : 0)].p + j0;
          for (size_t jj = 0; jj < len8; jj += 8) {
            uint64_t w = 0;  // byte b: bit t = sample s0 + t of k-mer j0 + jj + b
            for (int t = 0; t < ns; ++t) {
              uint64_t v;
              std::memcpy(&v, src[t] + jj, 8);
              w |= (v & 0x0101010101010101ull) << t;
            }
            for (int b = 0; b < 8; ++b) ab[(jj + b) * 8 + q] = (uint8_t)(w >> (8 * b));
          }
          for (size_t jj = len8; jj < len; ++jj) {
            uint8_t w = 0;
            for (int t = 0; t < ns; ++t) w |= (uint8_t)((src[t][jj] & 1u) << t);
            ab[jj * 8 + q] = w;
          }
        }
        for (size_t jj = 0; jj < len; ++jj) out[(j0 + jj) * W + wc] = acc[jj];
      }
    }
  }
  std::cerr << "\r[LOAD] " << n << "/" << n << "  (" << t.sec() << " s, LOAD_THREADS=" << threads << ")\n";
}

// ------------------------------------------------------------ ROWS reader
RowsReader::RowsReader(const std::string& path, int nthreads) : threads(std::max(1, nthreads)) {
  const bool gzm = path.size() >= 3 && path.compare(path.size() - 3, 3, ".gz") == 0;
  if (gzm) {
    gzFile f = gzopen(path.c_str(), "rb");
    if (!f) die("Cannot open gz file: " + path);
    gzbuffer(f, 1u << 20);
    gz = f;
    buf.resize((size_t)64 << 20);
  } else {
    const int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) die("Cannot open kmer file: " + path);
    struct stat st {};
    if (fstat(fd, &st) != 0) {
      ::close(fd);
      die("Cannot open kmer file: " + path);
    }
    map_sz = (size_t)st.st_size;
    if (map_sz > 0) {
      void* p = mmap(nullptr, map_sz, PROT_READ, MAP_PRIVATE, fd, 0);
      if (p == MAP_FAILED) {
        ::close(fd);
        die("mmap: " + path);
      }
      madvise(p, map_sz, MADV_SEQUENTIAL);
      map = (const char*)p;
    }
    ::close(fd);
    end = map_sz;
    eof = true;
  }
}

RowsReader::~RowsReader() {
  if (gz) gzclose((gzFile)gz);
  if (map) munmap((void*)map, map_sz);
}

// gz input: appends inflated bytes after [beg, end), moving the unparsed rest
// to the front first and growing the buffer when one line fills it; sets eof
// at the end of the stream.
void RowsReader::fill() {
  if (map) return;
  if (beg > 0) {
    std::memmove(buf.data(), buf.data() + beg, end - beg);
    end -= beg;
    beg = 0;
  }
  if (end == buf.size()) buf.resize(2 * buf.size());
  const int r = gzread((gzFile)gz, buf.data() + end, (unsigned)std::min<size_t>(buf.size() - end, 1u << 30));
  if (r < 0) {
    int err = 0;
    const char* msg = gzerror((gzFile)gz, &err);
    die(std::string("gzread error: ") + (msg ? msg : ""));
  }
  if (r == 0) eof = true;
  end += (size_t)r;
}

// src/kgwas.cpp:435-459.  Lines as the reference reads them: std::getline for
// plain input (a '\r' stays in the line), gzgets for gz input with one '\r'
// before '\n' dropped (:318-341); empty lines skipped; the k-mer ends at the
// first tab, else the first space, else the line is skipped; overlap sample j
// is character idxs[j] of the bitstring (one past its end reads '\0').
size_t RowsReader::read(size_t max_rows, const std::vector<int>& idxs, std::vector<std::string>& kmers,
                        std::vector<uint64_t>& packed) {
  const int n = (int)idxs.size();
  const uint32_t W = words_per_kmer(n);
  size_t got = 0;
  std::vector<size_t> ls, le;  // line spans [ls, le) of this round
  std::vector<size_t> sep;     // separator position (or SIZE_MAX: no row)
  std::vector<size_t> slot;    // output row of each line
  // the overlap positions as maximal runs of consecutive positions
  struct IdxRun {
    int j0;
    size_t p0;
    int len;
  };
  std::vector<IdxRun> runs;
  size_t max_pos = 0;
  for (int j = 0; j < n; ++j) {
    const size_t pos = (size_t)idxs[j];
    max_pos = std::max(max_pos, pos);
    if (!runs.empty() && runs.back().p0 + (size_t)runs.back().len == pos) ++runs.back().len;
    else runs.push_back({j, pos, 1});
  }
  while (got < max_rows) {
    ls.clear();
    le.clear();
    const size_t want = max_rows - got;
    const char* B0 = data();
    // line ends in a window of up to 256 MB, found by the threads in equal
    // pieces and kept in file order
    const size_t win = std::min(end - beg, (size_t)256 << 20);
    const unsigned nt = win >= ((size_t)4 << 20) ? (unsigned)threads : 1u;
    std::vector<std::vector<size_t>> nls(nt);
#pragma omp parallel for num_threads(nt) schedule(static, 1)
    for (int t = 0; t < (int)nt; ++t) {
      const size_t a = beg + win * (size_t)t / nt, b = beg + win * (size_t)(t + 1) / nt;
      for (size_t q = a; q < b;) {
        const char* nl = (const char*)std::memchr(B0 + q, '\n', b - q);
        if (!nl) break;
        nls[t].push_back((size_t)(nl - B0));
        q = nls[t].back() + 1;
      }
    }
    size_t p = beg;
    for (unsigned t = 0; t < nt && ls.size() < want; ++t)
      for (size_t e : nls[t]) {
        if (ls.size() >= want) break;
        ls.push_back(p);
        le.push_back(e);
        p = e + 1;
      }
    if (ls.empty() && win < end - beg) {  // a line longer than the window
      const char* nl = (const char*)std::memchr(B0 + beg, '\n', end - beg);
      if (nl) {
        ls.push_back(beg);
        le.push_back((size_t)(nl - B0));
        p = le.back() + 1;
      }
    }
    if (ls.empty()) {
      if (!eof) {
        fill();
        continue;
      }
      if (beg == end) break;
      ls.push_back(beg);  // a last line without '\n'
      le.push_back(end);
      p = end;
    }
    beg = p;
    const size_t L = ls.size();
    sep.assign(L, SIZE_MAX);
    slot.assign(L, 0);
    const char* B = data();
    // pass 1: which lines are rows, and where their k-mers end
    size_t nonempty = 0;
#pragma omp parallel for num_threads(threads) schedule(static) reduction(+ : nonempty)
    for (int64_t t = 0; t < (int64_t)L; ++t) {
      size_t e = le[t];
      if (gz && e > ls[t] && B[e - 1] == '\r') le[t] = --e;
      if (e == ls[t]) continue;
      ++nonempty;
      const char* a = B + ls[t];
      const void* tb = std::memchr(a, '\t', e - ls[t]);
      if (!tb) tb = std::memchr(a, ' ', e - ls[t]);
      if (tb) sep[t] = (size_t)((const char*)tb - B);
    }
    lines += nonempty;
    size_t rows = 0;
    for (size_t t = 0; t < L; ++t) {
      slot[t] = rows;
      rows += sep[t] != SIZE_MAX ? 1 : 0;
    }
    const size_t k0 = kmers.size(), p0 = packed.size();
    kmers.resize(k0 + rows);
    packed.resize(p0 + rows * W, 0ull);
    // pass 2: pack the rows; the first row (in file order) whose bitstring is
    // too short is the error.  Runs of consecutive positions go 8 samples at
    // a time: the 8 characters as one word, an exact per-byte test for '1'
    // (xor, then a zero-byte test without borrows between bytes) and one
    // multiply that gathers the 8 flags into one byte in sample order.
    std::atomic<size_t> bad{SIZE_MAX};
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t t = 0; t < (int64_t)L; ++t) {
      if (sep[t] == SIZE_MAX) continue;
      const char* bits = B + sep[t] + 1;
      const size_t nb = le[t] - (sep[t] + 1);
      uint64_t* row = packed.data() + p0 + slot[t] * W;
      bool ok = max_pos <= nb;  // one past the end reads '\0'
      for (size_t gi = 0; ok && gi < runs.size(); ++gi) {
        const IdxRun& g = runs[gi];
        int k = 0;
        for (; k + 8 <= g.len && g.p0 + (size_t)k + 8 <= nb; k += 8) {
          uint64_t v;
          std::memcpy(&v, bits + g.p0 + k, 8);
          const uint64_t x = v ^ 0x3131313131313131ull;  // zero bytes where '1'
          const uint64_t z = ~(((x & 0x7F7F7F7F7F7F7F7Full) + 0x7F7F7F7F7F7F7F7Full) | x | 0x7F7F7F7F7F7F7F7Full);
          const uint64_t f = (((z >> 7) & 0x0101010101010101ull) * 0x0102040810204080ull) >> 56;
          const int j = g.j0 + k;
          row[j >> 6] |= f << (j & 63);
          if ((j & 63) > 56) row[(j >> 6) + 1] |= f >> (64 - (j & 63));
        }
        for (; k < g.len; ++k) {
          const size_t pos = g.p0 + (size_t)k;
          const int j = g.j0 + k;
          if (pos < nb && bits[pos] == '1') row[j >> 6] |= 1ull << (j & 63);
        }
      }
      if (!ok) {
        size_t cur = bad.load();
        while ((size_t)t < cur && !bad.compare_exchange_weak(cur, (size_t)t)) {
        }
        continue;
      }
      kmers[k0 + slot[t]].assign(B + ls[t], sep[t] - ls[t]);
    }
    if (bad.load() != SIZE_MAX) {
      const size_t t = bad.load();
      die("bitstring shorter than the samples list in row: " + std::string(B + ls[t], sep[t] - ls[t]));
    }
    got += rows;
  }
  return got;
}

// ------------------------------------------------ sharded index (2-D input)

namespace {

using Key = unsigned __int128;

bool read_meta(const std::string& dir, uint32_t& K, uint32_t& M, uint64_t& N) {
  std::ifstream in(dir + "/index.meta");
  if (!in) {
    std::cerr << "[ERROR] cannot read index.meta in " << dir << "\n";
    return false;
  }
  std::string line;
  K = 0;
  M = 0;
  N = 0;
  while (std::getline(in, line)) {
    if (line.compare(0, 2, "K=") == 0) K = (uint32_t)std::stoul(line.substr(2));
    else if (line.compare(0, 2, "M=") == 0) M = (uint32_t)std::stoul(line.substr(2));
    else if (line.compare(0, 2, "N=") == 0) N = std::stoull(line.substr(2));
  }
  if (K == 0 || M == 0) {
    std::cerr << "[ERROR] invalid index.meta (K=" << K << " M=" << M << ")\n";
    return false;
  }
  return true;
}

bool slurp(const std::string& path, std::vector<char>& buf, const char* what) {
  std::ifstream in(path, std::ios::binary);
  if (!in) {
    std::cerr << "[ERROR] cannot open " << path << "\n";
    return false;
  }
  in.seekg(0, std::ios::end);
  buf.resize((size_t)in.tellg());
  in.seekg(0, std::ios::beg);
  in.read(buf.data(), (std::streamsize)buf.size());
  if (!in) {
    std::cerr << "[ERROR] short read: " << path << "\n";
    return false;
  }
  (void)what;
  return true;
}

// One shard: the keys of its .umap (first record of a key kept) and, from
// its .bits, the last non-empty bitstring recorded for each key.
bool load_shard_bits(const std::string& dir, uint32_t sid, uint32_t K, std::vector<std::pair<Key, std::string>>& out) {
  char fname[32];
  std::snprintf(fname, sizeof(fname), "shard_%03u", sid);
  const std::string umap = dir + "/" + fname + ".umap", bitsp = dir + "/" + fname + ".bits";
  std::vector<char> buf;
  if (!slurp(umap, buf, "umap")) return false;
  if (buf.size() < 20) {
    std::cerr << "[ERROR] file too small: " << umap << "\n";
    return false;
  }
  static const char MAGIC[8] = {'U', 'M', 'A', 'P', 'd', '4', '\0', '\0'};
  if (std::memcmp(buf.data(), MAGIC, 8) != 0) {
    std::cerr << "[ERROR] bad magic in " << umap << "\n";
    return false;
  }
  uint32_t k;
  uint64_t n;
  std::memcpy(&k, buf.data() + 8, 4);
  std::memcpy(&n, buf.data() + 12, 8);
  if (K && k != K) {
    std::cerr << "[ERROR] K mismatch in " << umap << ": got " << k << " expected " << K << "\n";
    return false;
  }
  if (buf.size() < 20 + (size_t)n * 32) {
    std::cerr << "[ERROR] short read: " << umap << "\n";
    return false;
  }
  std::unordered_map<uint64_t, std::vector<size_t>> seen;  // hash of key -> slots
  std::vector<Key> keys;
  std::vector<std::string> bits;
  auto hkey = [](Key x) { return (uint64_t)x ^ (uint64_t)(x >> 64) * 0x9E3779B97F4A7C15ull; };
  auto find = [&](Key x) -> long {
    auto it = seen.find(hkey(x));
    if (it == seen.end()) return -1;
    for (size_t s : it->second)
      if (keys[s] == x) return (long)s;
    return -1;
  };
  std::vector<Key> rec((size_t)n);
  for (uint64_t i = 0; i < n; ++i) {
    Key x;
    std::memcpy(&x, buf.data() + 20 + i * 32, 16);
    rec[i] = x;
    if (find(x) < 0) {
      seen[hkey(x)].push_back(keys.size());
      keys.push_back(x);
      bits.emplace_back();
    }
  }
  std::vector<char> bb;
  if (!slurp(bitsp, bb, "bits")) return false;
  if (bb.size() < 8) {
    std::cerr << "[ERROR] short read: " << bitsp << "\n";
    return false;
  }
  uint64_t bn;
  std::memcpy(&bn, bb.data(), 8);
  if (bn != n) {
    std::cerr << "[ERROR] .bits N=" << bn << " != .umap N=" << n << "\n";
    return false;
  }
  size_t off = 8;
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t blen = 0;
    if (off + 4 > bb.size()) return false;
    std::memcpy(&blen, bb.data() + off, 4);
    off += 4;
    if (blen > 0) {
      if (off + blen > bb.size()) return false;
      const long s = find(rec[i]);
      if (s >= 0) bits[(size_t)s].assign(bb.data() + off, blen);
    }
    off += blen;
  }
  for (size_t s = 0; s < keys.size(); ++s)
    if (!bits[s].empty()) out.emplace_back(keys[s], std::move(bits[s]));
  return true;
}

}  // namespace

IndexBits load_index_bits(const std::string& dir, int threads) {
  Timer t;
  struct stat st;
  if (stat(dir.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) die("Index path is not a directory: " + dir);
  uint32_t K = 0, M = 0;
  uint64_t N = 0;
  if (!read_meta(dir, K, M, N)) die("Failed to read index meta from " + dir);
  std::vector<std::vector<std::pair<Key, std::string>>> shards(M);
  std::atomic<bool> ok{true};
#pragma omp parallel for schedule(dynamic, 1) num_threads(std::max(1, threads))
  for (int64_t s = 0; s < (int64_t)M; ++s)
    if (!load_shard_bits(dir, (uint32_t)s, K, shards[(size_t)s])) ok = false;
  if (!ok) die("Failed to load index shards");
  std::vector<std::pair<Key, std::string>> all;
  for (auto& v : shards)
    for (auto& e : v) all.push_back(std::move(e));
  std::cerr << "[INFO] Loaded index: " << all.size() << " kmers with bitstrings (" << M << " shards, K=" << K
            << ") in " << t.sec() << " s\n";
  std::sort(all.begin(), all.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  if (all.empty()) die("No k-mers with bitstrings in index");
  IndexBits out;
  out.K = K;
  out.kmers.resize(all.size());
  out.bits.resize(all.size());
  static const char DEC[4] = {'A', 'C', 'G', 'T'};
  for (size_t i = 0; i < all.size(); ++i) {
    std::string& s = out.kmers[i];
    s.resize(K);
    Key e = all[i].first;
    for (uint32_t c = K; c > 0; --c) {
      s[c - 1] = DEC[(unsigned)(e & 3u)];
      e >>= 2;
    }
    out.bits[i] = std::move(all[i].second);
  }
  return out;
}

// ------------------------------------------------- sharded index (writer)

bool canonical_kmer(const std::string& kmer, unsigned __int128& key) {
  const size_t K = kmer.size();
  if (K == 0 || K > 64) return false;
  unsigned __int128 f = 0, r = 0;
  for (size_t i = 0; i < K; ++i) {
    int b;
    switch (kmer[i]) {
      case 'A': case 'a': b = 0; break;
      case 'C': case 'c': b = 1; break;
      case 'G': case 'g': b = 2; break;
      case 'T': case 't': b = 3; break;
      default: return false;
    }
    f = (f << 2) | (unsigned)b;
    r |= (unsigned __int128)(3 - b) << (2 * i);  // complement, read backwards
  }
  key = f < r ? f : r;
  return true;
}

namespace {

uint64_t splitmix_final(uint64_t x) {  // finaliser of SplitMix64 (Steele, Lea, Flood 2014)
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebULL;
  x ^= x >> 31;
  return x;
}

template <class T>
void put(std::string& b, const T& v) {
  b.append(reinterpret_cast<const char*>(&v), sizeof(T));
}

bool write_file(const std::string& path, const std::string& data) {
  std::ofstream out(path, std::ios::binary);
  if (!out) return false;
  out.write(data.data(), (std::streamsize)data.size());
  return (bool)out;
}

}  // namespace

bool write_index(const std::string& dir, uint32_t K, uint32_t M, std::vector<IndexRow>& rows) {
  std::error_code ec;
  std::filesystem::create_directories(dir, ec);
  std::vector<std::vector<IndexRow>> sh(M);
  for (auto& r : rows) sh[(size_t)((uint64_t)r.key & (M - 1))].push_back(std::move(r));
  static const char MAGIC[8] = {'U', 'M', 'A', 'P', 'd', '4', '\0', '\0'};
  // shards are independent: sorted, deduplicated and written in parallel
  auto write_shard = [&](uint32_t s) -> bool {
    auto& v = sh[s];
    std::stable_sort(v.begin(), v.end(), [](const IndexRow& a, const IndexRow& b) { return a.key < b.key; });
    v.erase(std::unique(v.begin(), v.end(), [](const IndexRow& a, const IndexRow& b) { return a.key == b.key; }),
            v.end());
    char fname[32];
    std::snprintf(fname, sizeof(fname), "shard_%03u", s);
    const std::string stem = dir + "/" + fname;
    std::string u;
    u.append(MAGIC, 8);
    put(u, K);
    put(u, (uint64_t)v.size());
    bool any_bits = false;
    for (const auto& r : v) {
      put(u, r.key);
      put(u, r.effect);
      put(u, r.pval);
      any_bits = any_bits || !r.bits.empty();
    }
    if (!write_file(stem + ".umap", u)) {
      std::cerr << "[ERROR] cannot write " << stem << ".umap\n";
      return false;
    }
    if (any_bits) {
      std::string b;
      put(b, (uint64_t)v.size());
      for (const auto& r : v) {
        put(b, (uint32_t)r.bits.size());
        b += r.bits;
      }
      if (!write_file(stem + ".bits", b)) {
        std::cerr << "[ERROR] cannot write " << stem << ".bits\n";
        return false;
      }
    }
    // Bloom filter: m = 10 bits per entry rounded up to a power of two (64
    // for an empty shard), two bit positions per key
    uint64_t target = (uint64_t)v.size() * 10, m = 1;
    if (target == 0) target = 64;
    while (m < target) m <<= 1;
    std::vector<uint64_t> words((m + 63) / 64, 0);
    for (const auto& r : v) {
      const uint64_t h1 = splitmix_final((uint64_t)r.key ^ (uint64_t)(r.key >> 64));
      const uint64_t h2 = splitmix_final(h1);
      const uint64_t i1 = h1 & (m - 1), i2 = h2 & (m - 1);
      words[i1 >> 6] |= 1ull << (i1 & 63);
      words[i2 >> 6] |= 1ull << (i2 & 63);
    }
    std::string bl;
    put(bl, m);
    put(bl, (uint64_t)words.size());
    bl.append(reinterpret_cast<const char*>(words.data()), words.size() * 8);
    if (!write_file(stem + ".bloom", bl)) {
      std::cerr << "[ERROR] cannot write " << stem << ".bloom\n";
      return false;
    }
    return true;
  };
  std::atomic<bool> ok{true};
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t s = 0; s < (int64_t)M; ++s)
    if (!write_shard((uint32_t)s)) ok = false;
  if (!ok) return false;
  uint64_t total = 0;
  for (const auto& v : sh) total += v.size();
  std::ostringstream meta;
  meta << "K=" << K << "\nM=" << M << "\nN=" << total << "\n";
  if (!write_file(dir + "/index.meta", meta.str())) {
    std::cerr << "[ERROR] cannot write index.meta in " << dir << "\n";
    return false;
  }
  return true;
}

bool read_index_rows(const std::string& dir, uint32_t& K, uint32_t& M, std::vector<IndexRow>& rows) {
  uint64_t N = 0;
  if (!read_meta(dir, K, M, N)) return false;
  static const char MAGIC[8] = {'U', 'M', 'A', 'P', 'd', '4', '\0', '\0'};
  for (uint32_t s = 0; s < M; ++s) {
    char fname[32];
    std::snprintf(fname, sizeof(fname), "shard_%03u", s);
    const std::string umap = dir + "/" + fname + ".umap", bitsp = dir + "/" + fname + ".bits";
    std::vector<char> buf;
    if (!slurp(umap, buf, "umap")) return false;
    uint32_t k = 0;
    uint64_t n = 0;
    if (buf.size() < 20 || std::memcmp(buf.data(), MAGIC, 8) != 0) {
      std::cerr << "[ERROR] bad magic in " << umap << "\n";
      return false;
    }
    std::memcpy(&k, buf.data() + 8, 4);
    std::memcpy(&n, buf.data() + 12, 8);
    if (k != K) {
      std::cerr << "[ERROR] K mismatch in " << umap << ": got " << k << " expected " << K << "\n";
      return false;
    }
    if (buf.size() < 20 + (size_t)n * 32) {
      std::cerr << "[ERROR] short read: " << umap << "\n";
      return false;
    }
    const size_t r0 = rows.size();
    rows.resize(r0 + (size_t)n);
    for (uint64_t i = 0; i < n; ++i) {
      IndexRow& r = rows[r0 + (size_t)i];
      const char* p = buf.data() + 20 + i * 32;
      std::memcpy(&r.key, p, 16);
      std::memcpy(&r.effect, p + 16, 8);
      std::memcpy(&r.pval, p + 24, 8);
      r.k = K;
    }
    struct stat st;
    if (stat(bitsp.c_str(), &st) != 0) continue;  // a shard without bitstrings has no .bits
    std::vector<char> bb;
    uint64_t bn = 0;
    if (!slurp(bitsp, bb, "bits")) return false;
    if (bb.size() >= 8) std::memcpy(&bn, bb.data(), 8);
    if (bb.size() < 8 || bn != n) {
      std::cerr << "[ERROR] .bits N=" << bn << " != .umap N=" << n << " in " << bitsp << "\n";
      return false;
    }
    size_t off = 8;
    for (uint64_t i = 0; i < n; ++i) {
      uint32_t blen = 0;
      if (off + 4 > bb.size()) return false;
      std::memcpy(&blen, bb.data() + off, 4);
      off += 4;
      if (off + blen > bb.size()) {
        std::cerr << "[ERROR] short read: " << bitsp << "\n";
        return false;
      }
      rows[r0 + (size_t)i].bits.assign(bb.data() + off, blen);
      off += blen;
    }
  }
  return true;
}

}  // namespace kgio
