// ctx.hpp -- the context behind the C ABI (private to the library).
#pragma once
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kgwas_cuda.h"
#include "kernels.hpp"
#include "prep.hpp"

namespace kgctx {

constexpr int NBUF = 2;  // host-run chunk buffers in flight

template <class T>
inline void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

// Smallest r2 that can still give p = erfc(sqrt(T/2)) <= p_thresh with
// T = n log(1/(1-r2)) (src/kgwas.cpp:51-52), lowered by a relative margin of
// 1e-9 so that k-mers below it are certainly not emitted.  -1 when every
// tested k-mer may be emitted.
inline double r2_candidate(double p_thresh, int n) {
  if (!(p_thresh < 1.0)) return -1.0;
  if (p_thresh <= 0.0) return 2.0;
  double lo = 0.0, hi = 1.0;
  while (std::erfc(std::sqrt(0.5 * hi)) > p_thresh && hi < 1e7) hi *= 2;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (std::erfc(std::sqrt(0.5 * mid)) > p_thresh) lo = mid; else hi = mid;
  }
  const double r2 = -std::expm1(-lo / (double)n);
  return r2 * (1.0 - 1e-9);
}

// Epilogue constants of one prepared phenotype.
inline void fill_epi(kg::EpiParams& P, const kg::Prepared& p, const kg_opts& o, bool refine) {
  std::memset(&P, 0, sizeof(P));
  P.n = p.n;
  P.k = p.k;
  P.b = p.b;
  P.kappa = p.kappa;
  P.yyM = p.yyM;
  P.ynorm = p.ynorm;
  P.corr_thr = o.corr_threshold;
  P.p_thresh = std::pow(10.0, -o.log10_thresh);
  P.r2_cand = r2_candidate(P.p_thresh, p.n);
  P.thr2_ynorm2 = o.corr_threshold * o.corr_threshold * p.ynorm * p.ynorm;
  for (int j = 0; j < p.k; ++j) {
    P.a[j] = p.a[j];
    P.g[j] = p.g[j];
  }
  if (refine) {
    P.refine = 1;
    P.r2_ref = -std::expm1(-kg::REFINE_CHISQ / (double)p.n);
  }
}

// State of the many-phenotype path.
struct Multi {
  int np = 0, n_row = 0, NP = 0, G = 0, kpad = 0, cm = 0, nsteps = 0;
  int PPG = 1;          // phenotypes per group (one MMA of NP * PPG columns)
  bool stationary = false;  // the group image fits in shared memory: kernel_mpb.cu
  bool pair_ok = false;     // kernel_mpb2.cu can run these phenotypes (PPG = 1 images)
  int kern = 0;             // chosen kernel: 0 image streamed (mp), 1 image resident (mpb), 2 SM pair (mpb2)
  int bt_scale = 2;         // tile-iterations per L2 block: the 48 MB rule times bt_scale / 2
  int8_t* dB = nullptr;
  kg::MPheno* dPh = nullptr;
  double* dV = nullptr;
  double* dT = nullptr;  // byte tables of V (refinement), one block per phenotype
  size_t vstride = 0;
  unsigned long long* dCounters = nullptr;
  unsigned long long* dTested = nullptr;
  size_t tested_cap = 0;
  kg_phit* dHits = nullptr;
  unsigned long long hit_cap = 0;
  unsigned long long* dShard = nullptr;
  int shard_cap = 0;
  int n_shards = 1;
  std::vector<unsigned long long> shard_host;
  std::vector<kg_phit> hits;
  std::vector<uint64_t> tested;
  unsigned long long counters[4] = {0, 0, 0, 0};
  // launch shape chosen by the autotuner: x tiles resident, B ring stages
  int xs = 1, nb = 4;
  int bt = 0;  // B-stationary kernel: tile-iterations per L2 block of the last launch
  bool tuned = false;
  int tuned_nbox = -1;
  // pending device launch and its captured graph
  bool pending = false;
  const uint64_t* pend_x = nullptr;
  uint64_t pend_m = 0;
  uint32_t pend_wpk = 0;
  cudaStream_t pend_stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  const uint64_t* g_x = nullptr;
  uint64_t g_m = 0;
  uint32_t g_wpk = 0;
  cudaStream_t g_stream = nullptr;
  int g_seen = 0;
};

}  // namespace kgctx

struct kg_ctx {
  kg_opts opts{};
  int num_sms = 0;
  cudaStream_t stream = nullptr, copy_stream = nullptr;
  std::string err;
  bool have_structure = false;
  int n_row = 0;  // samples per packed row
  kg::Prepared prep;
  kg::LimbCols limbs;
  kg::EpiParams P{};
  kg::LimbMap LM{};
  // structure on the device
  double* dV = nullptr;
  double* dT = nullptr;      // byte tables of V for the split form's FP64 refinement
  int cm = 0, nsteps = 0;
  int8_t* dB = nullptr;      // B image of the smem-A kernel
  int8_t* dBts = nullptr;    // B image of the TMEM-A kernel
  int nchunk = 0;
  // outputs on the device
  unsigned long long* dCounters = nullptr;
  kg_hit* dHits = nullptr;
  unsigned long long hit_cap = 0;
  unsigned long long* dCand = nullptr;  // FP64 refinement candidates (split form)
  unsigned long long cand_cap = 0;
  uint8_t* dTested = nullptr;
  double* dStat[7] = {};
  size_t stat_cap = 0;
  // host result
  std::vector<kg_hit> hits;
  unsigned long long counters[3] = {0, 0, 0};
  // pending device launch
  bool pending = false;
  const uint64_t* pend_x = nullptr;
  uint64_t pend_m = 0;
  uint32_t pend_wpk = 0;
  bool pend_stats = false;
  cudaStream_t pend_stream = nullptr;
  int launches = 0;
  const char* last_kernel = "";
  // bounded device waits: pipeline wait limit (0: the default) and the
  // one-launch stall of the row producer that the failure tests use
  unsigned long long wait_ns = 0;
  unsigned long long stall_once = 0;
  // host-run buffers
  uint64_t* dChunk[kgctx::NBUF] = {};
  void* hStage[kgctx::NBUF] = {};
  size_t chunk_bytes = 0;
  cudaEvent_t ev_h2d[kgctx::NBUF] = {}, ev_k[kgctx::NBUF] = {};
  // runs of equal adjacent rows (kg_run_host): first row and length of each
  // run; the device copy of the lengths weighs the tested count
  std::vector<uint64_t> run_first;
  std::vector<uint32_t> run_len;
  uint32_t* dWeight = nullptr;
  size_t weight_cap = 0;
  uint32_t* hWeight[kgctx::NBUF] = {};  // pinned staging of one chunk's run lengths
  size_t hweight_cap = 0;
  const uint32_t* cur_weight = nullptr;  // set while a deduplicated run is in flight
  uint64_t unique_rows = 0;              // rows the last kg_run_host tested (0: no deduplication)
  // many phenotypes
  kgctx::Multi mp;
  // 2-D pair test
  uint64_t* dPX = nullptr;        // packed rows on the device
  size_t px_bytes = 0;
  kg_pair* dPairs = nullptr;
  unsigned long long pair_cap = 0;
  unsigned long long* dUnitOff = nullptr;
  size_t unit_cap = 0;
  std::vector<kg_pair> pairs;

  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
  int cuda_fail(cudaError_t e, const char* what) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return KG_ERR_CUDA;
  }
};

#define KG_CUDA(call, what)                                    \
  do {                                                         \
    cudaError_t e__ = (call);                                  \
    if (e__ != cudaSuccess) return ctx->cuda_fail(e__, what);  \
  } while (0)

namespace kgctx {
void free_multi(kg_ctx* ctx);  // capi_multi.cpp
}  // namespace kgctx

namespace kgctx {

// Runs of equal adjacent host rows.  Real batches are sorted by bit pattern
// (src/convert_matrix.cpp:366-368), so equal rows sit next to each other; an
// equal row has equal statistics, so one row per run is tested and counts as
// many tested k-mers as the run has rows.
//
// use_runs: whether to test one row per run.  Finding the runs reads every
// row on the host, which pays only where the rows are copied through the host
// anyway (pageable memory): there, at least 10 % of 4096 sampled adjacent
// pairs must be equal.  KG_DEDUP=0 never, KG_DEDUP=1 always (pinned too).
bool use_runs(const uint64_t* x, uint64_t m, uint32_t wpk, bool pageable);
inline bool rows_equal(const uint64_t* a, const uint64_t* b, uint32_t wpk) {
  uint64_t d = 0;
  for (uint32_t w = 0; w < wpk; ++w) d |= a[w] ^ b[w];
  return d == 0;
}
// A slice of a staging buffer: `rows` rows from row `stage_row` on.
struct StageSeg {
  uint64_t stage_row, rows;
};
// Rows [s0, s0 + cnt) of x in one pass: a row starts a run when it is the
// first of the range, differs from its predecessor or is in `bounds`
// (ascending row indices).  Host threads copy the first row of each run into
// their own slices of dst (listed in segs, in row order), the runs' first rows
// and lengths are appended to first / len; returns the number of runs.
uint64_t scan_gather(const uint64_t* x, uint64_t s0, uint64_t cnt, uint32_t wpk, void* dst,
                     const std::vector<unsigned long long>& bounds, std::vector<uint64_t>& first,
                     std::vector<uint32_t>& len, std::vector<StageSeg>& segs);
// All runs of x at once (kg_run_multi_host): fills ctx->run_first / run_len
// and returns true when use_runs holds and the runs save at least 10 % of the
// rows; `bounds` (shard starts) also start runs.
bool find_runs(kg_ctx* ctx, const uint64_t* x, uint64_t m, uint32_t wpk, const std::vector<unsigned long long>& bounds,
               bool pageable);
bool is_pinned(const void* p);
// Copies the run lengths to the device and makes them the tested-count
// weights of the following launches (ctx->cur_weight).
int upload_run_lengths(kg_ctx* ctx, cudaStream_t st);
// Host copies in up to 8 threads (for 64 MB or more).
void par_memcpy(void* dst, const void* src, size_t bytes);
// Gathers rows sel[0..cnt) of x into dst (row bytes each).
void par_gather(void* dst, const uint64_t* x, const uint64_t* sel, uint64_t cnt, size_t row);
// Repeats each hit of a distinct row for every row of its run, in row order.
void expand_runs(const kg_ctx* ctx, std::vector<kg_hit>& hits);
void expand_runs(const kg_ctx* ctx, std::vector<kg_phit>& hits);

}  // namespace kgctx

