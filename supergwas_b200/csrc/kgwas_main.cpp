// kgwas_main.cpp -- drop-in replacement of the reference's `kgwas` program
// (src/kgwas.cpp) with the association arithmetic on a B200.
//
//   kgwas samples.txt phenotype.txt INPUT U.bin output.tsv [log10_thresh]
//         [--mode cols|rows] [--log10-thresh-2d X]
//
// Same arguments, environment variables (LOAD_THREADS, BLAS_THREADS,
// EMIT_THREADS, CORR_THRESHOLD, LOG10_THRESH_2D_INPUT), readers, output rows
// (.tsv, .2d.tsv, .count) and [ERROR] messages.  Added variables, which the
// reference ignores:
//   KGWAS_PRECISION  split (default: tcgen05 int8 limbs) | fp64 (CUDA cores)
//   KGWAS_DEVICE     CUDA device ordinal (default 0)
//   --index-out DIR     also write the .tsv rows as the sharded k-mer index
//                       that the reference's build_index makes of the .tsv
//                       file (--index-shards M, default 16)
//   --index-2d-out DIR  the same for the .2d rows (the .2d.tsv file; 4 shards
//                       by default, as build_index_2d.sh), the input of kgwas_2d
//                       (bin/kgwas_index_merge joins the indexes of batches)
//   KGWAS_ROWS_BATCH rows per batch in ROWS mode (default 4194304); the next
//                    batch is read while the current one is tested
//   KGWAS_KBITS      1: keep the packed rows of the batch in a sidecar file
//                    <batch>/kgwas_<N>_<n>_<hash>.kbits (hash of the overlap
//                    sample positions) and reuse it instead of re-reading the
//                    n ASCII/gz column files
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <memory>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/kgwas_cuda.h"
#include "cli.hpp"
#include "kgwas_io.hpp"

using kgio::die;
using std::string;
using std::vector;

struct Config {                      // src/kgwas.cpp:26-35
  string samples_file, pheno_file, input_path, U_file, out_file;
  double log10_thresh = 6.0;
  double log10_thresh_2d = 15.0;
  double corr_threshold = 0.2;
  int LOAD_THREADS = 24;
  int BLAS_THREADS = 112;
  int EMIT_THREADS = 112;
  string mode;
  int precision = KG_PREC_SPLIT_I8;
  int device = 0;
  string index_out;     // --index-out DIR: the .tsv rows as a sharded index (build_index's output)
  string index_2d_out;  // --index-2d-out DIR: the .2d rows as a sharded index
  uint32_t index_shards = 16;    // build_index.sh's default
  uint32_t index_2d_shards = 4;  // build_index_2d.sh's
};

static void print_usage(const char* prog) {
  std::cerr << "Usage: " << prog
            << " samples.txt phenotype.txt INPUT U.bin output.tsv [log10_thresh] [--mode cols|rows]\n"
            << "\n"
            << "  INPUT: directory (batch with bits/ + kmers.txt.gz) for COLS mode,\n"
            << "         or a .tsv[.gz] file for ROWS mode.\n"
            << "  Auto-detects mode from INPUT type unless --mode is specified.\n"
            << "\n"
            << "  Index outputs: --index-out DIR [--index-shards M] (the .tsv rows),\n"
            << "                 --index-2d-out DIR [--index-2d-shards M] (the .2d rows)\n"
            << "\n"
            << "  Env: LOAD_THREADS, BLAS_THREADS, EMIT_THREADS, CORR_THRESHOLD, BATCH_SIZE,\n"
            << "       KGWAS_PRECISION (split|fp64), KGWAS_DEVICE\n";
}

// The command line of src/kgwas.cpp:67-126 as a table: five leading paths,
// then options and -log10 thresholds (a later threshold replaces an earlier
// one; a word that is no number is an error).
static Config parse_args(int argc, char** argv) {
  Config cfg;
  kgcli::Grammar g;
  g.required = 5;
  g.usage = print_usage;
  g.options = {
      {"--mode", [&](const string& v) { cfg.mode = v; }},
      {"--log10-thresh-2d", [&](const string& v) { cfg.log10_thresh_2d = std::stod(v); }},
      {"--index-out", [&](const string& v) { cfg.index_out = v; }},
      {"--index-shards", [&](const string& v) { cfg.index_shards = (uint32_t)std::stoul(v); }},
      {"--index-2d-out", [&](const string& v) { cfg.index_2d_out = v; }},
      {"--index-2d-shards", [&](const string& v) { cfg.index_2d_shards = (uint32_t)std::stoul(v); }},
  };
  g.other = [&](const string& w) {
    double t = 0.0;
    try {
      t = std::stod(w);
    } catch (...) {
      die("invalid argument: " + w);
    }
    if (t < 0.0) die("threshold must be >= 0");
    cfg.log10_thresh = t;
  };
  const vector<string> lead = kgcli::parse(argc, argv, g);
  cfg.samples_file = lead[0];
  cfg.pheno_file = lead[1];
  cfg.input_path = lead[2];
  cfg.U_file = lead[3];
  cfg.out_file = lead[4];
  cfg.LOAD_THREADS = kgio::env_int("LOAD_THREADS", cfg.LOAD_THREADS);
  cfg.BLAS_THREADS = kgio::env_int("BLAS_THREADS", cfg.BLAS_THREADS);
  cfg.EMIT_THREADS = kgio::env_int("EMIT_THREADS", cfg.EMIT_THREADS);
  if (const char* v = std::getenv("CORR_THRESHOLD")) cfg.corr_threshold = std::stod(v);
  if (const char* v = std::getenv("LOG10_THRESH_2D_INPUT")) cfg.log10_thresh_2d = std::stod(v);
  if (const char* v = std::getenv("KGWAS_PRECISION")) {
    const string p = v;
    if (p == "fp64") cfg.precision = KG_PREC_FP64;
    else if (p == "split" || p.empty()) cfg.precision = KG_PREC_SPLIT_I8;
    else die("KGWAS_PRECISION must be 'split' or 'fp64', got: " + p);
  }
  if (const char* v = std::getenv("KGWAS_DEVICE")) cfg.device = std::atoi(v);
  if (cfg.mode.empty()) {  // a directory is a COLS batch, anything else a ROWS file
    struct stat info {};
    if (::stat(cfg.input_path.c_str(), &info) != 0) die("cannot stat INPUT: " + cfg.input_path);
    cfg.mode = S_ISDIR(info.st_mode) ? "cols" : "rows";
    std::cerr << "[INFO] auto-detected mode: " << cfg.mode << "\n";
  }
  if (cfg.mode != "cols" && cfg.mode != "rows") die("--mode must be 'cols' or 'rows', got: " + cfg.mode);
  auto pow2 = [](uint32_t m) { return m != 0 && (m & (m - 1)) == 0; };
  if (!pow2(cfg.index_shards)) die("--index-shards must be a power of 2, got " + std::to_string(cfg.index_shards));
  if (!pow2(cfg.index_2d_shards))
    die("--index-2d-shards must be a power of 2, got " + std::to_string(cfg.index_2d_shards));
  if (!cfg.index_2d_out.empty() && !(cfg.log10_thresh_2d > 0.0))
    die("--index-2d-out needs the .2d rows (--log10-thresh-2d > 0)");
  return cfg;
}

// ------------------------------------------------------------- GPU context
// The context is created on a thread of its own (start) while the program
// reads its inputs; open() waits for it and reports a failure at the point
// where the reference would meet it, after the inputs.
struct Gpu {
  kg_ctx* ctx = nullptr;
  std::thread th;
  int rc = KG_OK;
  ~Gpu() {
    if (th.joinable()) th.join();
    kg_destroy(ctx);
  }
  void check(int rc_, const char* what) {
    if (rc_ != KG_OK) die(string("GPU ") + what + " failed (code " + std::to_string(rc_) + "): " + kg_last_error(ctx));
  }
  void start(const Config& cfg) {
    kg_opts o;
    kg_default_opts(&o);
    o.device = cfg.device;
    o.precision = cfg.precision;
    o.corr_threshold = cfg.corr_threshold;
    o.log10_thresh = cfg.log10_thresh;
    th = std::thread([this, o] { rc = kg_create(&ctx, &o); });
  }
  // Once the batch's shape is known: the host pipeline's buffers, allocated
  // on the same thread after the context (while the inputs are still read).
  void reserve(uint64_t n_kmers, uint32_t words_per_kmer) {
    std::thread prev = std::move(th);
    th = std::thread([this, n_kmers, words_per_kmer, p = std::move(prev)]() mutable {
      if (p.joinable()) p.join();
      if (rc == KG_OK && ctx) kg_reserve_host(ctx, n_kmers, words_per_kmer);  // kg_run_host retries on failure
    });
  }
  // The program is about to end with every output written: the context is
  // left to the driver, which frees a process's device resources when it
  // exits (unpinning the staging buffers one by one alone takes a visible
  // part of a batch's run).
  void leave() {
    if (th.joinable()) th.join();
    ctx = nullptr;
  }
  void open(const Config& cfg) {
    if (!th.joinable() && !ctx) start(cfg);
    if (th.joinable()) th.join();
    if (rc != KG_OK) die("GPU context creation failed (code " + std::to_string(rc) + ") on device " +
                         std::to_string(cfg.device));
  }
};

// Host buffer for the packed matrix.  Pageable: no CUDA call is needed before
// the inputs are read, and kg_run_host stages pageable rows through its own
// pinned buffers (where it also finds runs of equal rows).
struct HostWords {
  uint64_t* p = nullptr;
  std::unique_ptr<uint64_t[]> v;
  void alloc(size_t words) {
    v.reset(new uint64_t[words ? words : 1]);  // every word is written by the reader
    p = v.get();
  }
};

// The .2d.tsv path: ".2d" goes in front of the last '.' of the output path
// (wherever that dot is), or at the end when there is none
// (src/kgwas.cpp:273-278).
static string path_2d(const string& out_file) {
  string p = out_file;
  const size_t dot = p.rfind('.');
  p.insert(dot == string::npos ? p.size() : dot, ".2d");
  return p;
}

// The .count file (src/kgwas.cpp:291-304): "<label>\t<tested>\n" in
// out_file + ".count", the label being the output file's name without its
// directory ('/' or '\\') and without its last extension.  Nothing is written
// when the file cannot be created.
static void write_count(const string& out_file, uint64_t n_tested) {
  const size_t name_at = out_file.find_last_of("/\\");
  string label = name_at == string::npos ? out_file : out_file.substr(name_at + 1);
  const size_t ext = label.find_last_of('.');
  if (ext != string::npos) label.erase(ext);
  const string path = out_file + ".count";
  std::FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return;
  std::fprintf(f, "%s\t%llu\n", label.c_str(), (unsigned long long)n_tested);
  std::fclose(f);
  std::cerr << "[INFO] Count written to " << path << "\n";
}

// Text of the emitted rows (src/kgwas.cpp:239-259): default ostream float
// formatting (6 significant digits), k-mer order.  With index1/index2 the rows
// are also kept for the index writer, with the values as printed (build_index
// reads them back with strtod, src/build_index.cpp:89-90).
static void format_range(const kg_result& r, uint64_t h0, uint64_t h1, const vector<string>& kmers,
                         const uint64_t* packed, uint32_t W, int n, bool do_2d, double p_thresh_2d, string& one,
                         string& two, vector<kgio::IndexRow>* index1, vector<kgio::IndexRow>* index2) {
  std::ostringstream o1, o2, ev, pv;
  o1.setf(std::ios::fmtflags(0), std::ios::floatfield);
  o2.setf(std::ios::fmtflags(0), std::ios::floatfield);
  string bits(n, '0');
  for (uint64_t h = h0; h < h1; ++h) {
    const kg_hit& x = r.hits[h];
    const string& km = kmers[x.kmer];
    const bool is2 = do_2d && x.pval <= p_thresh_2d;
    if (is2) {
      const uint64_t* row = packed + (size_t)x.kmer * W;
      for (int i = 0; i < n; ++i) bits[i] = ((row[i >> 6] >> (i & 63)) & 1u) ? '1' : '0';
    }
    kgio::IndexRow ir;
    if (!index1 && !(is2 && index2)) {
      o1 << km << '\t' << x.effect << '\t' << x.pval << '\n';
      if (is2) o2 << km << '\t' << bits << '\t' << x.effect << '\t' << x.pval << '\n';
      continue;
    }
    // the values printed once (same stream formatting), then read back as
    // build_index reads them
    ev.str("");
    pv.str("");
    ev << x.effect;
    pv << x.pval;
    const string e = ev.str(), q = pv.str();
    o1 << km << '\t' << e << '\t' << q << '\n';
    if (is2) o2 << km << '\t' << bits << '\t' << e << '\t' << q << '\n';
    if (!kgio::canonical_kmer(km, ir.key)) continue;  // a base other than ACGT: build_index skips the row
    ir.effect = std::strtod(e.c_str(), nullptr);
    ir.pval = std::strtod(q.c_str(), nullptr);
    ir.k = (uint32_t)km.size();
    if (is2 && index2) {
      kgio::IndexRow r2 = ir;
      r2.bits = bits;
      index2->push_back(std::move(r2));
    }
    if (index1) index1->push_back(std::move(ir));
  }
  one = o1.str();
  two = o2.str();
}

// The hits in `threads` contiguous slices (EMIT_THREADS, src/kgwas.cpp:227-259),
// each formatted on its own thread and joined in order: the same bytes as one
// pass.  The index rows are appended to index1 / index2 in row order.
static void format_hits(const kg_result& r, const vector<string>& kmers, const uint64_t* packed, uint32_t W,
                        int n, bool do_2d, double p_thresh_2d, string& one, string& two, int threads,
                        vector<kgio::IndexRow>* index1 = nullptr, vector<kgio::IndexRow>* index2 = nullptr) {
  const uint64_t H = r.n_hits;
  const int T = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)std::max(1, threads), H / 256));
  vector<string> ones(T), twos(T);
  vector<vector<kgio::IndexRow>> i1(T), i2(T);
#pragma omp parallel for num_threads(T) schedule(static, 1)
  for (int t = 0; t < T; ++t)
    format_range(r, H * t / T, H * (t + 1) / T, kmers, packed, W, n, do_2d, p_thresh_2d, ones[t], twos[t],
                 index1 ? &i1[t] : nullptr, index2 ? &i2[t] : nullptr);
  size_t b1 = 0, b2 = 0;
  for (int t = 0; t < T; ++t) {
    b1 += ones[t].size();
    b2 += twos[t].size();
  }
  one.clear();
  two.clear();
  one.reserve(b1);
  two.reserve(b2);
  for (int t = 0; t < T; ++t) {
    one += ones[t];
    two += twos[t];
    if (index1) index1->insert(index1->end(), std::make_move_iterator(i1[t].begin()), std::make_move_iterator(i1[t].end()));
    if (index2) index2->insert(index2->end(), std::make_move_iterator(i2[t].begin()), std::make_move_iterator(i2[t].end()));
  }
}

// Writes one index (build_index on this run's .tsv or .2d.tsv file): k from
// the first row, rows of another length left out (src/build_index.cpp:73-75,
// 153-156).  Without rows, k is the first k-mer's length and every shard is
// empty (build_index instead stops with "Could not infer k-mer length").
static void write_index_out(const string& dir, uint32_t M, const char* what, const vector<string>& kmers,
                            vector<kgio::IndexRow>& rows) {
  if (dir.empty()) return;
  const uint32_t K = !rows.empty() ? rows[0].k : kmers.empty() ? 0u : (uint32_t)kmers[0].size();
  rows.erase(std::remove_if(rows.begin(), rows.end(), [K](const kgio::IndexRow& r) { return r.k != K; }),
             rows.end());
  const size_t n_rows = rows.size();
  if (!kgio::write_index(dir, K, M, rows)) die("Failed to write index " + dir);
  std::cerr << "[INFO] wrote " << n_rows << " " << what << " rows as a " << M << "-shard index to " << dir << "\n";
}

static void write_indexes(const Config& cfg, const vector<string>& kmers, vector<kgio::IndexRow>& rows1,
                          vector<kgio::IndexRow>& rows2) {
  write_index_out(cfg.index_out, cfg.index_shards, ".tsv", kmers, rows1);
  write_index_out(cfg.index_2d_out, cfg.index_2d_shards, ".2d", kmers, rows2);
}

// ---------------------------------------------------------- .kbits cache
// 64-byte header: "KGWASKB1", N, n, words_per_kmer, FNV-1a of the overlap
// positions; then N * words_per_kmer little-endian uint64 words.
struct KbitsHeader {
  char magic[8];
  uint64_t N;
  uint32_t n, wpk;
  uint64_t idx_hash;
  char pad[32];
};
static_assert(sizeof(KbitsHeader) == 64, "kbits header");

static uint64_t fnv1a(const vector<int>& v) {
  uint64_t h = 1469598103934665603ull;
  for (int x : v)
    for (int b = 0; b < 4; ++b) {
      h ^= (uint64_t)((x >> (8 * b)) & 0xff);
      h *= 1099511628211ull;
    }
  return h;
}

static string kbits_path(const string& batch, size_t N, int n, uint64_t h) {
  char buf[96];
  std::snprintf(buf, sizeof(buf), "/kgwas_%zu_%d_%016llx.kbits", N, n, (unsigned long long)h);
  return batch + buf;
}

static bool kbits_read(const string& path, size_t N, int n, uint32_t W, uint64_t h, uint64_t* out) {
  std::ifstream in(path, std::ios::binary);
  if (!in) return false;
  KbitsHeader hd{};
  in.read((char*)&hd, sizeof(hd));
  if (!in || std::memcmp(hd.magic, "KGWASKB1", 8) != 0 || hd.N != N || hd.n != (uint32_t)n || hd.wpk != W ||
      hd.idx_hash != h)
    return false;
  in.read((char*)out, (std::streamsize)(N * W * 8));
  return (bool)in;
}

static void kbits_write(const string& path, size_t N, int n, uint32_t W, uint64_t h, const uint64_t* x) {
  const string tmp = path + ".tmp." + std::to_string(::getpid());
  std::ofstream out(tmp, std::ios::binary);
  if (!out) return;
  KbitsHeader hd{};
  std::memcpy(hd.magic, "KGWASKB1", 8);
  hd.N = N;
  hd.n = (uint32_t)n;
  hd.wpk = W;
  hd.idx_hash = h;
  out.write((const char*)&hd, sizeof(hd));
  out.write((const char*)x, (std::streamsize)(N * W * 8));
  out.close();
  if (out) std::rename(tmp.c_str(), path.c_str());
  else std::remove(tmp.c_str());
}

static void run_cols(const Config& cfg) {  // src/kgwas.cpp:168-307
  kgio::Timer tall;
  Gpu g;
  g.start(cfg);
  kgio::Overlap ov = kgio::build_overlap(cfg.samples_file, cfg.pheno_file);
  const int n = (int)ov.y.size();
  kgio::UData ud = kgio::load_ubin(cfg.U_file, n);
  const string bits_dir = cfg.input_path + "/bits";
  const string kmers_gz = cfg.input_path + "/kmers.txt.gz";
  const size_t N = kgio::infer_N_from_bits(bits_dir, ov.idxs.front());
  // the k-mer strings are read beside the columns
  vector<string> kmers;
  std::thread kt([&] { kmers = kgio::load_kmers(kmers_gz, N); });
  const uint32_t W = kgio::words_per_kmer(n);
  if (N > 0) g.reserve(N, W);
  HostWords X;
  X.alloc((size_t)N * W);
  const char* kb = std::getenv("KGWAS_KBITS");
  const bool use_kbits = kb && std::string(kb) == "1";
  const uint64_t h = fnv1a(ov.idxs);
  const string kpath = kbits_path(cfg.input_path, N, n, h);
  if (use_kbits && kbits_read(kpath, N, n, W, h, X.p)) {
    std::cerr << "[INFO] packed rows from " << kpath << "\n";
  } else {
    kgio::load_matrix_packed(bits_dir, ov.idxs, N, cfg.LOAD_THREADS, X.p);
    if (use_kbits) kbits_write(kpath, N, n, W, h, X.p);
  }
  kt.join();
  std::cerr << "[TIME] inputs read " << tall.sec() << " s\n";

  g.open(cfg);
  std::cerr << "[TIME] GPU context ready " << tall.sec() << " s\n";
  kgio::Timer tg;
  double yyM = 0;
  g.check(kg_set_structure(g.ctx, ud.U.data(), n, ud.k, ov.y.data(), &yyM), "set_structure");
  if (!(yyM > 1e-12)) kgio::warn("yyM ~ 0");
  kg_result res{};
  g.check(kg_run_host(g.ctx, X.p, N, W, &res, nullptr), "run");
  std::cerr << "[INFO] CORR_THRESHOLD=" << cfg.corr_threshold << "  total kmers: " << N
            << ", passed correlation filter: " << res.n_tested << "\n";
  std::cerr << "[INFO] GPU association test (" << tg.sec() << " s, "
            << (cfg.precision == KG_PREC_FP64 ? "fp64" : "split-precision int8 tcgen05") << ")\n";
  std::cerr << "[TIME] GPU test done " << tall.sec() << " s\n";

  kgio::Timer te;
  const bool do_2d = (cfg.log10_thresh_2d > 0.0);
  const double p_thresh_2d = do_2d ? std::pow(10.0, -cfg.log10_thresh_2d) : 0.0;
  string one, two;
  vector<kgio::IndexRow> index1, index2;
  format_hits(res, kmers, X.p, W, n, do_2d, p_thresh_2d, one, two, cfg.EMIT_THREADS,
              cfg.index_out.empty() ? nullptr : &index1,
              cfg.index_2d_out.empty() ? nullptr : &index2);
  {
    std::ofstream out(cfg.out_file, std::ios::binary);
    if (!out) die("open out: " + cfg.out_file);
    out.write(one.data(), (std::streamsize)one.size());
    out.close();
    if (!out) die("write out failed");
  }
  std::cerr << "[INFO] wrote 1D hits at -log10(p) >= " << cfg.log10_thresh << " (" << te.sec()
            << " s, EMIT_THREADS=" << cfg.EMIT_THREADS << ")\n";
  if (do_2d) {
    const string p2 = path_2d(cfg.out_file);
    std::ofstream out2d(p2, std::ios::binary);
    if (!out2d) die("open 2D out: " + p2);
    out2d.write(two.data(), (std::streamsize)two.size());
    out2d.close();
    if (!out2d) die("write 2D out failed");
    std::cerr << "[INFO] wrote 2D hits at -log10(p) >= " << cfg.log10_thresh_2d << " to " << p2 << "\n";
  }
  write_indexes(cfg, kmers, index1, index2);
  write_count(cfg.out_file, res.n_tested);
  std::cerr << "[TIME] total " << tall.sec() << " s\n";
  g.leave();
}

static void run_rows(const Config& cfg) {  // src/kgwas.cpp:343-522
  kgio::Timer tall;
  Gpu g;
  g.start(cfg);
  // ROWS mode words its input errors differently from COLS mode
  // (src/kgwas.cpp:349-381): no check for an empty sample list, and U.bin is
  // only checked for its row count.
  const kgio::Overlap ov = kgio::match_phenotypes(kgio::read_sample_ids(cfg.samples_file), cfg.pheno_file);
  const vector<int>& idxs = ov.idxs;
  const vector<double>& y = ov.y;
  const int n = (int)idxs.size();
  if (n == 0) die("No overlapping genomes in phenotype.");
  const kgio::UbinFile uf = kgio::read_ubin_file(cfg.U_file);
  if (uf.status == kgio::UbinFile::kNoFile) die("Cannot open " + cfg.U_file);
  if (uf.n != n)
    die("U.bin row count (" + std::to_string(uf.n) + ") does not match phenotype size (" + std::to_string(n) + ")");
  if (uf.k < 0) die("Cannot open " + cfg.U_file);
  const int r = uf.k;
  vector<double> U((size_t)n * r, 0.0);  // a short body leaves zeros
  std::copy(uf.U.begin(), uf.U.begin() + std::min(uf.U.size(), U.size()), U.begin());
  std::cerr << "[INFO] CORR_THRESHOLD=" << cfg.corr_threshold << "\n";

  kgio::RowsReader rr(cfg.input_path, cfg.LOAD_THREADS);
  std::ofstream out(cfg.out_file);
  if (!out) die("Cannot open output: " + cfg.out_file);
  const bool do_2d = (cfg.log10_thresh_2d > 0.0);
  const double p_thresh_2d = do_2d ? std::pow(10.0, -cfg.log10_thresh_2d) : 0.0;
  std::ofstream out2d;
  string p2;
  if (do_2d) {
    p2 = path_2d(cfg.out_file);
    out2d.open(p2);
    if (!out2d) die("Cannot open 2D output: " + p2);
  }
  const uint32_t W = kgio::words_per_kmer(n);
  uint64_t passed = 0;
  size_t BATCH = (size_t)1 << 22;
  if (const char* v = std::getenv("KGWAS_ROWS_BATCH")) BATCH = (size_t)std::max(1L, std::atol(v));
  g.reserve(BATCH, W);  // while the first batch is read
  struct Batch {
    vector<string> kmers;
    vector<uint64_t> packed;
    size_t got = 0;
  } cur, nxt;
  auto read_into = [&](Batch& b) {
    b.kmers.clear();
    b.packed.clear();
    b.got = rr.read(BATCH, idxs, b.kmers, b.packed);
  };
  vector<kgio::IndexRow> index1, index2;
  string first_kmer;
  double t_read = 0, t_gpu = 0;
  // the first batch is read while the GPU context is set up, and each next
  // batch while the current one is tested and written
  kgio::Timer tr;
  read_into(cur);
  t_read += tr.sec();
  g.open(cfg);
  double yyM = 0;
  g.check(kg_set_structure(g.ctx, U.data(), n, r, y.data(), &yyM), "set_structure");
  if (!(yyM > 1e-12)) std::cerr << "[WARN] yyM ~ 0. Tests unstable.\n";
  while (cur.got > 0) {
    double t_next = 0;
    std::thread rd([&] {
      kgio::Timer t;
      read_into(nxt);
      t_next = t.sec();
    });
    kg_result res{};
    kgio::Timer tg;
    g.check(kg_run_host(g.ctx, cur.packed.data(), cur.got, W, &res, nullptr), "run");
    t_gpu += tg.sec();
    passed += res.n_tested;
    string one, two;
    format_hits(res, cur.kmers, cur.packed.data(), W, n, do_2d, p_thresh_2d, one, two, cfg.EMIT_THREADS,
                cfg.index_out.empty() ? nullptr : &index1, cfg.index_2d_out.empty() ? nullptr : &index2);
    if (first_kmer.empty() && !cur.kmers.empty()) first_kmer = cur.kmers[0];
    out.write(one.data(), (std::streamsize)one.size());
    if (do_2d) out2d.write(two.data(), (std::streamsize)two.size());
    rd.join();
    t_read += t_next;
    std::swap(cur, nxt);
  }
  std::cerr << "[INFO] Total kmers: " << rr.lines << ", passed correlation filter: " << passed << "\n";
  if (do_2d) {
    out2d.close();
    std::cerr << "[INFO] 2D hits written to " << p2 << "\n";
  }
  out.close();
  write_indexes(cfg, vector<string>{first_kmer}, index1, index2);
  write_count(cfg.out_file, passed);
  std::cerr << "[TIME] rows read " << t_read << " s, GPU tests " << t_gpu << " s\n";
  std::cerr << "[TIME] End-to-end " << tall.sec() << "s\n";
  g.leave();
}

int main(int argc, char** argv) {
  // Host-pipeline chunks of 64 MB unless the user chose a size: the staging
  // buffers are page-locked while the inputs are read and released at exit,
  // and 2 x 64 MB take a fraction of the time of the library's default
  // 2 x 512 MB (measured on a 4M-k-mer batch: 0.95 s against 1.26 s for the
  // whole run); rows read from files do not need larger copies.
  setenv("KG_CHUNK_MB", "64", 0);
  Config cfg = parse_args(argc, argv);
  if (cfg.mode == "cols") run_cols(cfg);
  else run_rows(cfg);
  // every output file is closed; the device context goes with the process
  // (see Gpu::leave) instead of through the runtime's exit handlers
  std::cout.flush();
  std::cerr.flush();
  std::fflush(nullptr);
  std::_Exit(0);
}
