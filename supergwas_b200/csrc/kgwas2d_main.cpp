// kgwas2d_main.cpp -- drop-in replacement of the reference's `kgwas_2d`
// program (src/kgwas_2d.cpp) with the pair arithmetic on a B200.
//
//   kgwas_2d samples.txt phenotype.txt U2D.bin INDEX_DIR out_prefix
//            [log10_thresh] [--emit-threads N] [--out-chunk N]
//            [--task-id T] [--num-tasks K]
//
// Same arguments, environment variables (BLAS_THREADS, EMIT_THREADS), index
// reader, outputs (out_prefix[.part_T].tsv with "i<TAB>j<TAB>effect<TAB>p"
// rows sorted by (i, j); out_prefix.kmers from task 0) and [ERROR] messages.
// Added variable, which the reference ignores: KGWAS_DEVICE (CUDA device).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/kgwas_cuda.h"
#include "cli.hpp"
#include "kgwas_io.hpp"

using kgio::die;
using std::string;
using std::vector;

struct Config {  // src/kgwas_2d.cpp:24-35
  string samples_file, pheno_file, U_file, index_dir, out_prefix;
  double log10_thresh = 6.0;
  int BLAS_THREADS = 112;
  int EMIT_THREADS = 112;
  int OUT_CHUNK = 1000;
  int task_id = 0;
  int num_tasks = 1;
  int device = 0;
};

static void print_usage(const char* prog) {
  std::cerr << "Usage: " << prog << " samples.txt phenotype.txt U2D.bin INDEX_DIR out_prefix"
            << " [log10_thresh] [--emit-threads N] [--out-chunk N]\n"
            << "\nOutputs:\n"
            << "  out_prefix.tsv   — idx_a, idx_b, effect, pvalue\n"
            << "  out_prefix.kmers — one k-mer sequence per line (line# = index)\n";
}

// The command line of src/kgwas_2d.cpp:44-76 as a table: five leading paths,
// a -log10 threshold when the next word does not start with '-', then
// integer options; other words are ignored.  Malformed numbers end the
// program with an uncaught exception, as in the reference.
static Config parse_args(int argc, char** argv) {
  Config cfg;
  kgcli::Grammar g;
  g.required = 5;
  g.usage = print_usage;
  g.leading_accept = [](const string& w) { return w.empty() || w[0] != '-'; };
  g.leading_take = [&](const string& w) { cfg.log10_thresh = std::stod(w); };
  g.options = {
      {"--emit-threads", [&](const string& v) { cfg.EMIT_THREADS = std::stoi(v); }},
      {"--out-chunk", [&](const string& v) { cfg.OUT_CHUNK = std::stoi(v); }},
      {"--task-id", [&](const string& v) { cfg.task_id = std::stoi(v); }},
      {"--num-tasks", [&](const string& v) { cfg.num_tasks = std::stoi(v); }},
  };
  const vector<string> lead = kgcli::parse(argc, argv, g);
  cfg.samples_file = lead[0];
  cfg.pheno_file = lead[1];
  cfg.U_file = lead[2];
  cfg.index_dir = lead[3];
  cfg.out_prefix = lead[4];
  cfg.BLAS_THREADS = kgio::env_int("BLAS_THREADS", cfg.BLAS_THREADS);
  cfg.EMIT_THREADS = kgio::env_int("EMIT_THREADS", cfg.EMIT_THREADS);
  if (const char* v = std::getenv("KGWAS_DEVICE")) cfg.device = std::atoi(v);
  return cfg;
}

// The context is created on a thread of its own while the index is read;
// a failure is reported where the reference would meet it, after the inputs.
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
  void start(const kg_opts& o) {
    th = std::thread([this, o] { rc = kg_create(&ctx, &o); });
  }
  void wait(int device) {
    if (th.joinable()) th.join();
    if (rc != KG_OK) die("GPU context creation failed (code " + std::to_string(rc) + ") on device " +
                         std::to_string(device));
  }
};

int main(int argc, char** argv) {
  const Config cfg = parse_args(argc, argv);
  kgio::Timer tall;
  Gpu g;
  {
    kg_opts o;
    kg_default_opts(&o);
    o.device = cfg.device;
    o.log10_thresh = cfg.log10_thresh;
    g.start(o);
  }
  const kgio::Overlap ov = kgio::build_overlap(cfg.samples_file, cfg.pheno_file);
  const int n = (int)ov.y.size();
  const kgio::UData ud = kgio::load_ubin(cfg.U_file, n);

  // load_X_from_index (src/kgwas_2d.cpp:80-207): k-mers with bitstrings, in
  // encoding order; a bitstring of length n is in overlap order, a longer one
  // (beyond the largest overlap position) in samples order; others are dropped.
  kgio::Timer tx;
  kgio::IndexBits ix = kgio::load_index_bits(cfg.index_dir, std::max(1, cfg.BLAS_THREADS));
  std::cerr << "[INFO] " << ix.kmers.size() << " k-mers with bitstrings\n";
  const int maxidx = ov.idxs.empty() ? -1 : *std::max_element(ov.idxs.begin(), ov.idxs.end());
  const uint32_t wpk = kgio::words_per_kmer(n);
  vector<uint64_t> X;
  X.reserve(ix.kmers.size() * wpk);
  vector<string> seqs;
  seqs.reserve(ix.kmers.size());
  for (size_t j = 0; j < ix.kmers.size(); ++j) {
    const string& b = ix.bits[j];
    const long B = (long)b.size();
    const bool direct = B == n;
    if (!direct && !(maxidx >= 0 && B > maxidx)) continue;
    const size_t r0 = X.size();
    X.resize(r0 + wpk, 0);
    for (int i = 0; i < n; ++i) {
      const char ch = direct ? b[(size_t)i] : b[(size_t)ov.idxs[(size_t)i]];
      if (ch == '1') X[r0 + (size_t)(i >> 6)] |= 1ull << (i & 63);
    }
    seqs.push_back(std::move(ix.kmers[j]));
  }
  const int64_t N = (int64_t)seqs.size();
  if (N <= 0) die("No valid k-mers after bitstring parsing");
  std::cerr << "[INFO] Built X from index (N=" << N << ", n=" << n << ", " << tx.sec() << " s)\n";

  // emit_pairs_self's column check (src/kgwas_2d.cpp:240), made before the
  // GPU is touched so that the failure needs no device
  if (N < 2) die("emit_pairs_self: need at least 2 columns");
  // build_stats2d_self + emit_pairs_self (src/kgwas_2d.cpp:210-392) on the GPU
  g.wait(cfg.device);
  double yyM = 0;
  g.check(kg_set_structure(g.ctx, ud.U.data(), n, ud.k, ov.y.data(), &yyM), "set_structure");
  if (!(yyM > 1e-12)) kgio::warn("yyM ~ 0");
  const int64_t rows_per_task = (N + cfg.num_tasks - 1) / cfg.num_tasks;
  const int64_t row_start = (int64_t)cfg.task_id * rows_per_task;
  const int64_t row_end = std::min(row_start + rows_per_task, N);
  if (row_start >= N) {
    std::cerr << "[INFO] task " << cfg.task_id << ": no rows to process\n";
    std::cerr << "[TIME] total " << tall.sec() << " s\n";
    return 0;
  }
  kgio::Timer te;
  kg_pair_result res;
  g.check(kg_pairs_run_host(g.ctx, X.data(), (uint64_t)N, wpk, (uint64_t)row_start, (uint64_t)row_end, &res),
          "pair test");
  std::cerr << "[INFO] found " << res.n_pairs << " passing pairs in " << te.sec() << " s ("
            << res.n_evaluated << " pairs evaluated on the GPU)\n";

  // outputs (src/kgwas_2d.cpp:350-389)
  {
    kgio::Timer tw;
    string pairs_path = cfg.out_prefix;
    if (cfg.num_tasks > 1) pairs_path += ".part_" + std::to_string(cfg.task_id);
    pairs_path += ".tsv";
    std::ofstream out(pairs_path, std::ios::binary);
    if (!out) die("open out: " + pairs_path);
    std::ostringstream oss;
    for (uint64_t h = 0; h < res.n_pairs; ++h) {
      const kg_pair& p = res.pairs[h];
      oss << p.a << '\t' << p.b << '\t' << std::setprecision(9) << std::defaultfloat << p.effect << '\t'
          << std::setprecision(9) << std::scientific << p.pval << '\n';
    }
    const string buf = std::move(oss).str();
    out.write(buf.data(), (std::streamsize)buf.size());
    out.close();
    if (!out) die("write out failed");
    std::cerr << "[INFO] wrote " << res.n_pairs << " pairs to " << pairs_path << " in " << tw.sec() << " s\n";
  }
  if (cfg.task_id == 0) {
    kgio::Timer tw;
    const string kmers_path = cfg.out_prefix + ".kmers";
    std::ofstream out(kmers_path);
    if (!out) die("open out: " + kmers_path);
    for (const auto& s : seqs) out << s << '\n';
    out.close();
    std::cerr << "[INFO] wrote " << seqs.size() << " k-mers to " << kmers_path << " in " << tw.sec() << " s\n";
  }
  std::cerr << "[TIME] total " << tall.sec() << " s\n";
  return 0;
}
