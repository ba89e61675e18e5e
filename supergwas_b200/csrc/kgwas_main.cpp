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
//   KGWAS_KBITS      1: keep the packed rows of the batch in a sidecar file
//                    <batch>/kgwas_<N>_<n>_<hash>.kbits (hash of the overlap
//                    sample positions) and reuse it instead of re-reading the
//                    n ASCII/gz column files
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/kgwas_cuda.h"
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
};

static Config parse_args(int argc, char** argv) {  // src/kgwas.cpp:67-126
  if (argc < 6) {
    std::cerr << "Usage: " << argv[0]
              << " samples.txt phenotype.txt INPUT U.bin output.tsv [log10_thresh] [--mode cols|rows]\n"
              << "\n"
              << "  INPUT: directory (batch with bits/ + kmers.txt.gz) for COLS mode,\n"
              << "         or a .tsv[.gz] file for ROWS mode.\n"
              << "  Auto-detects mode from INPUT type unless --mode is specified.\n"
              << "\n"
              << "  Env: LOAD_THREADS, BLAS_THREADS, EMIT_THREADS, CORR_THRESHOLD, BATCH_SIZE,\n"
              << "       KGWAS_PRECISION (split|fp64), KGWAS_DEVICE\n";
    std::exit(1);
  }
  Config cfg;
  cfg.samples_file = argv[1];
  cfg.pheno_file = argv[2];
  cfg.input_path = argv[3];
  cfg.U_file = argv[4];
  cfg.out_file = argv[5];
  for (int i = 6; i < argc; ++i) {
    string a = argv[i];
    if (a == "--mode" && i + 1 < argc) {
      cfg.mode = argv[++i];
    } else if (a == "--log10-thresh-2d" && i + 1 < argc) {
      cfg.log10_thresh_2d = std::stod(argv[++i]);
    } else {
      try {
        cfg.log10_thresh = std::stod(a);
      } catch (...) {
        die("invalid argument: " + a);
      }
      if (cfg.log10_thresh < 0.0) die("threshold must be >= 0");
    }
  }
  cfg.LOAD_THREADS = kgio::env_int("LOAD_THREADS", cfg.LOAD_THREADS);
  cfg.BLAS_THREADS = kgio::env_int("BLAS_THREADS", cfg.BLAS_THREADS);
  cfg.EMIT_THREADS = kgio::env_int("EMIT_THREADS", cfg.EMIT_THREADS);
  if (const char* v = std::getenv("CORR_THRESHOLD")) cfg.corr_threshold = std::stod(v);
  if (const char* v = std::getenv("LOG10_THRESH_2D_INPUT")) cfg.log10_thresh_2d = std::stod(v);
  if (const char* v = std::getenv("KGWAS_PRECISION")) {
    string p = v;
    if (p == "fp64") cfg.precision = KG_PREC_FP64;
    else if (p == "split" || p.empty()) cfg.precision = KG_PREC_SPLIT_I8;
    else die("KGWAS_PRECISION must be 'split' or 'fp64', got: " + p);
  }
  if (const char* v = std::getenv("KGWAS_DEVICE")) cfg.device = std::atoi(v);
  if (cfg.mode.empty()) {
    struct stat st {};
    if (::stat(cfg.input_path.c_str(), &st) != 0) die("cannot stat INPUT: " + cfg.input_path);
    cfg.mode = S_ISDIR(st.st_mode) ? "cols" : "rows";
    std::cerr << "[INFO] auto-detected mode: " << cfg.mode << "\n";
  }
  if (cfg.mode != "cols" && cfg.mode != "rows") die("--mode must be 'cols' or 'rows', got: " + cfg.mode);
  return cfg;
}

// ------------------------------------------------------------- GPU context
struct Gpu {
  kg_ctx* ctx = nullptr;
  ~Gpu() { kg_destroy(ctx); }
  void check(int rc, const char* what) {
    if (rc != KG_OK) die(string("GPU ") + what + " failed (code " + std::to_string(rc) + "): " + kg_last_error(ctx));
  }
  void open(const Config& cfg) {
    kg_opts o;
    kg_default_opts(&o);
    o.device = cfg.device;
    o.precision = cfg.precision;
    o.corr_threshold = cfg.corr_threshold;
    o.log10_thresh = cfg.log10_thresh;
    const int rc = kg_create(&ctx, &o);
    if (rc != KG_OK) die("GPU context creation failed (code " + std::to_string(rc) + ") on device " +
                         std::to_string(cfg.device));
  }
};

// Pinned host buffer for the packed matrix (pageable fallback).
struct HostWords {
  uint64_t* p = nullptr;
  bool pinned = false;
  vector<uint64_t> v;
  void alloc(size_t words) {
    p = (uint64_t*)kg_host_alloc(words * 8);
    pinned = p != nullptr;
    if (!p) {
      v.assign(words, 0);
      p = v.data();
    }
  }
  ~HostWords() {
    if (pinned) kg_host_free(p);
  }
};

static string path_2d(const string& out_file) {  // src/kgwas.cpp:273-278
  string p = out_file;
  size_t dot = p.rfind('.');
  if (dot != string::npos) return p.substr(0, dot) + ".2d" + p.substr(dot);
  return p + ".2d";
}

static void write_count(const string& out_file, uint64_t n_tested) {  // src/kgwas.cpp:291-304
  std::string countfile = out_file + ".count";
  std::string shardname = out_file;
  size_t lastslash = shardname.find_last_of("/\\");
  if (lastslash != std::string::npos) shardname = shardname.substr(lastslash + 1);
  size_t lastdot = shardname.find_last_of('.');
  if (lastdot != std::string::npos) shardname = shardname.substr(0, lastdot);
  std::ofstream countout(countfile);
  if (countout.is_open()) {
    countout << shardname << "\t" << n_tested << "\n";
    std::cerr << "[INFO] Count written to " << countfile << "\n";
  }
}

// Text of the emitted rows (src/kgwas.cpp:239-259): default ostream float
// formatting (6 significant digits), k-mer order.
static void format_hits(const kg_result& r, const vector<string>& kmers, const uint64_t* packed, uint32_t W,
                        int n, bool do_2d, double p_thresh_2d, string& one, string& two) {
  std::ostringstream o1, o2;
  o1.setf(std::ios::fmtflags(0), std::ios::floatfield);
  o2.setf(std::ios::fmtflags(0), std::ios::floatfield);
  string bits(n, '0');
  for (uint64_t h = 0; h < r.n_hits; ++h) {
    const kg_hit& x = r.hits[h];
    o1 << kmers[x.kmer] << '\t' << x.effect << '\t' << x.pval << '\n';
    if (do_2d && x.pval <= p_thresh_2d) {
      const uint64_t* row = packed + (size_t)x.kmer * W;
      for (int i = 0; i < n; ++i) bits[i] = ((row[i >> 6] >> (i & 63)) & 1u) ? '1' : '0';
      o2 << kmers[x.kmer] << '\t' << bits << '\t' << x.effect << '\t' << x.pval << '\n';
    }
  }
  one = o1.str();
  two = o2.str();
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
  kgio::Overlap ov = kgio::build_overlap(cfg.samples_file, cfg.pheno_file);
  const int n = (int)ov.y.size();
  kgio::UData ud = kgio::load_ubin(cfg.U_file, n);
  const string bits_dir = cfg.input_path + "/bits";
  const string kmers_gz = cfg.input_path + "/kmers.txt.gz";
  const size_t N = kgio::infer_N_from_bits(bits_dir, ov.idxs.front());
  vector<string> kmers = kgio::load_kmers(kmers_gz, N);
  const uint32_t W = kgio::words_per_kmer(n);
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

  Gpu g;
  g.open(cfg);
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

  kgio::Timer te;
  const bool do_2d = (cfg.log10_thresh_2d > 0.0);
  const double p_thresh_2d = do_2d ? std::pow(10.0, -cfg.log10_thresh_2d) : 0.0;
  string one, two;
  format_hits(res, kmers, X.p, W, n, do_2d, p_thresh_2d, one, two);
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
  write_count(cfg.out_file, res.n_tested);
  std::cerr << "[TIME] total " << tall.sec() << " s\n";
}

static void run_rows(const Config& cfg) {  // src/kgwas.cpp:343-522
  kgio::Timer tall;
  const auto all_ids = kgio::load_lines(cfg.samples_file);
  const auto pheno = kgio::load_pheno(cfg.pheno_file);
  vector<int> idxs;
  vector<double> y;
  for (int i = 0; i < (int)all_ids.size(); ++i) {
    auto it = pheno.find(all_ids[i]);
    if (it != pheno.end()) {
      idxs.push_back(i);
      y.push_back(it->second);
    }
  }
  const int n = (int)idxs.size();
  if (n == 0) die("No overlapping genomes in phenotype.");
  std::ifstream uin(cfg.U_file, std::ios::binary);
  if (!uin) die("Cannot open " + cfg.U_file);
  int n_u = 0, r = 0;
  uin.read((char*)&n_u, sizeof(int));
  uin.read((char*)&r, sizeof(int));
  if (n_u != n)
    die("U.bin row count (" + std::to_string(n_u) + ") does not match phenotype size (" + std::to_string(n) + ")");
  if (r < 0) die("Cannot open " + cfg.U_file);
  vector<double> U((size_t)n * r, 0.0);
  uin.read((char*)U.data(), (std::streamsize)(sizeof(double) * (size_t)n * r));
  std::cerr << "[INFO] CORR_THRESHOLD=" << cfg.corr_threshold << "\n";

  kgio::RowsReader rr(cfg.input_path);
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
  Gpu g;
  g.open(cfg);
  double yyM = 0;
  g.check(kg_set_structure(g.ctx, U.data(), n, r, y.data(), &yyM), "set_structure");
  if (!(yyM > 1e-12)) std::cerr << "[WARN] yyM ~ 0. Tests unstable.\n";
  const uint32_t W = kgio::words_per_kmer(n);
  uint64_t passed = 0;
  const size_t BATCH = (size_t)1 << 22;
  vector<string> kmers;
  vector<uint64_t> packed;
  for (;;) {
    kmers.clear();
    packed.clear();
    const size_t got = rr.read(BATCH, idxs, kmers, packed);
    if (got == 0) break;
    kg_result res{};
    g.check(kg_run_host(g.ctx, packed.data(), got, W, &res, nullptr), "run");
    passed += res.n_tested;
    string one, two;
    format_hits(res, kmers, packed.data(), W, n, do_2d, p_thresh_2d, one, two);
    out.write(one.data(), (std::streamsize)one.size());
    if (do_2d) out2d.write(two.data(), (std::streamsize)two.size());
  }
  std::cerr << "[INFO] Total kmers: " << rr.lines << ", passed correlation filter: " << passed << "\n";
  if (do_2d) {
    out2d.close();
    std::cerr << "[INFO] 2D hits written to " << p2 << "\n";
  }
  out.close();
  write_count(cfg.out_file, passed);
  std::cerr << "[TIME] End-to-end " << tall.sec() << "s\n";
}

int main(int argc, char** argv) {
  Config cfg = parse_args(argc, argv);
  if (cfg.mode == "cols") run_cols(cfg);
  else run_rows(cfg);
  return 0;
}
