// capi_pairs.cpp -- kg_pairs_run_host, the 2-D pair test of include/kgwas_cuda.h.
//
// Replaces build_stats2d_self + emit_pairs_self (src/kgwas_2d.cpp:210-392):
// the packed rows go to the device once; pairs (i, j), i < j, i in the row
// range, are scheduled as units of one 128-row j-block and up to `ic`
// consecutive i (kernel_pairs.cu); pairs whose split-form chi-square reaches
// the refinement threshold are recomputed in FP64 and the rows with
// p <= 10^-log10_thresh come back sorted by (i, j) (:333-345).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kgwas_cuda.h"
#include "kernels.hpp"
#include "prep.hpp"
#include "ctx.hpp"

using namespace kgctx;

namespace {

int ensure_pairs(kg_ctx* ctx, unsigned long long cap) {
  if (ctx->pair_cap >= cap && ctx->dPairs) return KG_OK;
  dfree(ctx->dPairs);
  ctx->pair_cap = 0;
  KG_CUDA(cudaMalloc((void**)&ctx->dPairs, cap * sizeof(kg_pair)), "cudaMalloc(pairs)");
  ctx->pair_cap = cap;
  return KG_OK;
}

int ensure_pair_cand(kg_ctx* ctx, unsigned long long cap) {
  if (ctx->cand_cap >= cap && ctx->dCand) return KG_OK;
  dfree(ctx->dCand);
  ctx->cand_cap = 0;
  KG_CUDA(cudaMalloc((void**)&ctx->dCand, cap * sizeof(unsigned long long)), "cudaMalloc(candidates)");
  ctx->cand_cap = cap;
  return KG_OK;
}

// Sorts the emitted pairs by (a, b).  a lies in the task's row range
// [row_start, row_end): a counting sort on a, then each row's few pairs
// sorted by b.  The scatter is bound by cache misses, so host threads each
// take a block of rows with about the same number of pairs, scatter the pairs
// of their rows and sort those rows.  A range much wider than the number of
// pairs falls back to a comparison sort.
void sort_pairs(std::vector<kg_pair>& v, uint64_t row_start, uint64_t row_end) {
  auto less = [](const kg_pair& x, const kg_pair& y) { return x.a != y.a ? x.a < y.a : x.b < y.b; };
  const size_t n = v.size();
  if (n < 2) return;
  const uint64_t R = row_end > row_start ? row_end - row_start : 0;
  bool in_range = R <= 8 * (uint64_t)n + 4096;
  for (size_t k = 0; k < n && in_range; ++k) in_range = v[k].a >= row_start && v[k].a < row_end;
  if (!in_range) {
    std::sort(v.begin(), v.end(), less);
    return;
  }
  std::vector<uint32_t> pos((size_t)R + 1, 0);  // pos[r]: first slot of row r
  for (const kg_pair& p : v) ++pos[(size_t)(p.a - row_start) + 1];
  for (size_t r = 0; r < R; ++r) pos[r + 1] += pos[r];
  std::vector<kg_pair> out(n);
  unsigned nt = std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency()));
  if (n < 20000) nt = 1;
  // row blocks [rb[t], rb[t+1]) with about n / nt pairs each
  std::vector<size_t> rb(nt + 1, (size_t)R);
  rb[0] = 0;
  for (unsigned t = 1; t < nt; ++t)
    rb[t] = (size_t)(std::lower_bound(pos.begin(), pos.end(), (uint32_t)(n * t / nt)) - pos.begin());
  for (unsigned t = 1; t < nt; ++t) rb[t] = std::min(std::max(rb[t], rb[t - 1]), (size_t)R);
  auto work = [&](unsigned t) {
    const size_t r0 = rb[t], r1 = rb[t + 1];
    if (r0 >= r1) return;
    std::vector<uint32_t> next(pos.begin() + (long)r0, pos.begin() + (long)r1);
    for (const kg_pair& p : v) {
      const size_t r = (size_t)(p.a - row_start);
      if (r >= r0 && r < r1) out[next[r - r0]++] = p;  // stable within a row
    }
    for (size_t r = r0; r < r1; ++r) {
      const size_t b0 = pos[r], b1 = pos[r + 1];
      if (b1 - b0 <= 1) continue;
      if (b1 - b0 <= 16) {
        for (size_t k = b0 + 1; k < b1; ++k)  // insertion sort by b
          for (size_t m = k; m > b0 && out[m].b < out[m - 1].b; --m) std::swap(out[m], out[m - 1]);
      } else {
        std::sort(out.begin() + (long)b0, out.begin() + (long)b1, less);
      }
    }
  };
  if (nt == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) th.emplace_back(work, t);
    for (auto& t : th) t.join();
  }
  v.swap(out);
}

}  // namespace

extern "C" {

int kg_pairs_run_host(kg_ctx* ctx, const uint64_t* xbits, uint64_t n_kmers, uint32_t wpk, uint64_t row_start,
                      uint64_t row_end, kg_pair_result* res) {
  if (!ctx) return KG_ERR_INVALID;
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");
  if (!ctx->have_structure) return ctx->fail(KG_ERR_STATE, "kg_set_structure has not succeeded");
  if (ctx->opts.precision != KG_PREC_SPLIT_I8)
    return ctx->fail(KG_ERR_UNSUPPORTED, "the pair test runs in split precision");
  if (n_kmers > 0 && !xbits) return ctx->fail(KG_ERR_INVALID, "xbits is NULL");
  if (wpk == 0 || (wpk & 1u)) return ctx->fail(KG_ERR_INVALID, "words_per_kmer must be even and > 0");
  if ((uint64_t)wpk * 64 < (uint64_t)ctx->n_row) return ctx->fail(KG_ERR_INVALID, "words_per_kmer*64 < samples per row");
  if (n_kmers >= (1ull << 32)) return ctx->fail(KG_ERR_UNSUPPORTED, "more than 2^32 - 1 k-mers");
  if (row_end > n_kmers) row_end = n_kmers;
  ctx->pairs.clear();
  ctx->launches = 0;
  if (res) {
    res->n_kmers = n_kmers;
    res->n_evaluated = 0;
    res->n_pairs = 0;
    res->pairs = nullptr;
  }
  if (row_start >= row_end || n_kmers < 2) return KG_OK;
  // rows of at least 128 bytes (one TMA box row); narrower rows are padded
  const uint32_t wd = std::max<uint32_t>(wpk, 16);
  const int N = ctx->limbs.N;
  if (!kg::pairs_supported(N, ctx->opts.limbs_u, ctx->opts.limbs_y, ctx->limbs.Kpad, (int)wd))
    return ctx->fail(KG_ERR_UNSUPPORTED, "structure or row width outside the pair kernel's range");
  const size_t bytes = (size_t)n_kmers * wd * 8;
  if (ctx->px_bytes < bytes) {
    dfree(ctx->dPX);
    ctx->px_bytes = 0;
    KG_CUDA(cudaMalloc((void**)&ctx->dPX, bytes), "cudaMalloc(rows)");
    ctx->px_bytes = bytes;
  }
  cudaStream_t st = ctx->stream;
  if (wd == wpk) {
    KG_CUDA(cudaMemcpyAsync(ctx->dPX, xbits, bytes, cudaMemcpyHostToDevice, st), "H2D");
  } else {
    std::vector<uint64_t> padded((size_t)n_kmers * wd, 0);
    for (uint64_t r = 0; r < n_kmers; ++r)
      std::memcpy(&padded[(size_t)r * wd], xbits + (size_t)r * wpk, (size_t)wpk * 8);
    KG_CUDA(cudaMemcpyAsync(ctx->dPX, padded.data(), bytes, cudaMemcpyHostToDevice, st), "H2D");
    KG_CUDA(cudaStreamSynchronize(st), "H2D");
  }
  // schedule: j-block jb covers j in [128 jb, 128 jb + 128); its i range is
  // [row_start, min(row_end, last j of the block)), cut into units of ic
  unsigned long long ic = 32;
  if (const char* v = std::getenv("KG_PAIR_IC")) ic = (unsigned long long)std::max(1, std::atoi(v));
  const int njb = (int)((n_kmers + 127) / 128);
  std::vector<unsigned long long> off((size_t)njb + 1, 0);
  for (int jb = 0; jb < njb; ++jb) {
    const unsigned long long jend = std::min<unsigned long long>(128ull * (jb + 1), n_kmers);
    const unsigned long long ihi = std::min<unsigned long long>(row_end, jend - 1);
    const unsigned long long units = ihi > row_start ? (ihi - row_start + ic - 1) / ic : 0;
    off[(size_t)jb + 1] = off[(size_t)jb] + units;
  }
  if (ctx->unit_cap < off.size()) {
    dfree(ctx->dUnitOff);
    ctx->unit_cap = 0;
    KG_CUDA(cudaMalloc((void**)&ctx->dUnitOff, off.size() * sizeof(unsigned long long)), "cudaMalloc(schedule)");
    ctx->unit_cap = off.size();
  }
  KG_CUDA(cudaMemcpyAsync(ctx->dUnitOff, off.data(), off.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                          st),
          "copy schedule");
  KG_CUDA(cudaStreamSynchronize(st), "copy schedule");
  kg::PairSched S{ctx->dUnitOff, njb, off.back(), n_kmers, row_start, row_end, ic};
  int rc;
  if ((rc = ensure_pairs(ctx, std::max<unsigned long long>(ctx->pair_cap, 1ull << 16)))) return rc;
  if ((rc = ensure_pair_cand(ctx, std::max<unsigned long long>(ctx->cand_cap, 1ull << 20)))) return rc;
  unsigned long long cnt[4] = {0, 0, 0, 0};
  for (int attempt = 0; attempt < 8; ++attempt) {
    kg::DevOutPairs O{ctx->dCounters, ctx->dPairs, ctx->pair_cap, ctx->dCand, ctx->cand_cap, ctx->wait_ns};
    KG_CUDA(cudaMemsetAsync(ctx->dCounters, 0, 4 * sizeof(unsigned long long), st), "memset");
    kg::LaunchPairs L{ctx->dPX, (int)wd, ctx->limbs.Kpad, ctx->prep.drop0 && ctx->P.k > 0, S, ctx->dBts, &ctx->P,
                      &ctx->LM, &O, ctx->num_sms};
    cudaError_t e = kg::launch_pairs(L, st);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "pair kernel launch");
    kg::LaunchPairRefine R{ctx->dPX, (int)wd, ctx->dT, ctx->nsteps * 128, ctx->cm, &ctx->P, &O, ctx->num_sms};
    e = kg::launch_pair_refine(R, st);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "pair refinement launch");
    ctx->launches = 2;
    KG_CUDA(cudaMemcpyAsync(cnt, ctx->dCounters, sizeof(cnt), cudaMemcpyDeviceToHost, st), "copy counters");
    KG_CUDA(cudaStreamSynchronize(st), "pair kernels");
    if (cnt[2] & ~(unsigned long long)(kg::ERR_HIT_OVERFLOW | kg::ERR_CAND_OVERFLOW))
      return ctx->fail(KG_ERR_TIMEOUT, "a bounded device-side wait gave up (error bits " + std::to_string(cnt[2]) + ")");
    if (!(cnt[2] & (kg::ERR_HIT_OVERFLOW | kg::ERR_CAND_OVERFLOW))) break;
    if ((cnt[2] & kg::ERR_CAND_OVERFLOW) && (rc = ensure_pair_cand(ctx, std::max(cnt[3], 4 * ctx->cand_cap))))
      return rc;
    if ((cnt[2] & kg::ERR_HIT_OVERFLOW) && (rc = ensure_pairs(ctx, std::max(cnt[1] + (1ull << 16), 2 * ctx->pair_cap))))
      return rc;
    if (attempt == 7) return ctx->fail(KG_ERR_NOMEM, "pair or candidate buffer still too small");
  }
  ctx->pairs.resize(cnt[1]);
  if (cnt[1])
    KG_CUDA(cudaMemcpy(ctx->pairs.data(), ctx->dPairs, cnt[1] * sizeof(kg_pair), cudaMemcpyDeviceToHost),
            "copy pairs");
  sort_pairs(ctx->pairs, row_start, row_end);
  if (res) {
    res->n_evaluated = cnt[0];
    res->n_pairs = cnt[1];
    res->pairs = ctx->pairs.data();
  }
  return KG_OK;
}

}  // extern "C"
