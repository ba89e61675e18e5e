// capi.cpp -- the C ABI of include/kgwas_cuda.h.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kgwas_cuda.h"
#include "kernels.hpp"
#include "prep.hpp"

#define KG_VERSION "kgwas-b200 0.1.0"

#include "ctx.hpp"

using namespace kgctx;

extern "C" {

const char* kg_version(void) { return KG_VERSION; }

void kg_default_opts(kg_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->device = 0;
  o->precision = KG_PREC_SPLIT_I8;
  o->corr_threshold = 0.2;
  o->log10_thresh = 6.0;
  o->limbs_u = 3;
  o->limbs_y = 5;
}

int kg_create(kg_ctx** out, const kg_opts* opts) {
  if (!out) return KG_ERR_INVALID;
  *out = nullptr;
  kg_ctx* ctx = new (std::nothrow) kg_ctx();
  if (!ctx) return KG_ERR_NOMEM;
  if (opts) ctx->opts = *opts; else kg_default_opts(&ctx->opts);
  if (ctx->opts.limbs_u == 0) ctx->opts.limbs_u = 3;
  if (ctx->opts.limbs_y == 0) ctx->opts.limbs_y = 5;
  if (ctx->opts.precision != KG_PREC_SPLIT_I8 && ctx->opts.precision != KG_PREC_FP64) {
    delete ctx;
    return KG_ERR_INVALID;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ctx->opts.device < 0 || ctx->opts.device >= ndev) {
    delete ctx;
    return KG_ERR_CUDA;
  }
  if (cudaSetDevice(ctx->opts.device) != cudaSuccess ||
      cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->opts.device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc((void**)&ctx->dCounters, 4 * sizeof(unsigned long long)) != cudaSuccess) {
    kg_destroy(ctx);
    return KG_ERR_CUDA;
  }
  if (ctx->opts.precision == KG_PREC_SPLIT_I8) {
    int cc_major = 0, cc_minor = 0;
    cudaDeviceGetAttribute(&cc_major, cudaDevAttrComputeCapabilityMajor, ctx->opts.device);
    cudaDeviceGetAttribute(&cc_minor, cudaDevAttrComputeCapabilityMinor, ctx->opts.device);
    if (cc_major != 10 || cc_minor != 0) {
      kg_destroy(ctx);
      return KG_ERR_UNSUPPORTED;
    }
  }
  for (int b = 0; b < NBUF; ++b) {
    if (cudaEventCreateWithFlags(&ctx->ev_h2d[b], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_k[b], cudaEventDisableTiming) != cudaSuccess) {
      kg_destroy(ctx);
      return KG_ERR_CUDA;
    }
  }
  *out = ctx;
  return KG_OK;
}

void kg_destroy(kg_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->opts.device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  dfree(ctx->dV);
  dfree(ctx->dT);
  dfree(ctx->dB);
  dfree(ctx->dBts);
  dfree(ctx->dCounters);
  dfree(ctx->dHits);
  dfree(ctx->dCand);
  dfree(ctx->dTested);
  dfree(ctx->dPX);
  dfree(ctx->dPairs);
  dfree(ctx->dUnitOff);
  dfree(ctx->dWeight);
  for (auto& p : ctx->dStat) dfree(p);
  for (int b = 0; b < NBUF; ++b) {
    dfree(ctx->dChunk[b]);
    if (ctx->hStage[b]) cudaFreeHost(ctx->hStage[b]);
    if (ctx->hWeight[b]) cudaFreeHost(ctx->hWeight[b]);
    if (ctx->ev_h2d[b]) cudaEventDestroy(ctx->ev_h2d[b]);
    if (ctx->ev_k[b]) cudaEventDestroy(ctx->ev_k[b]);
  }
  kgctx::free_multi(ctx);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  delete ctx;
}

const char* kg_last_error(const kg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int kg_last_launch_count(const kg_ctx* ctx) { return ctx ? ctx->launches : 0; }

const char* kg_last_kernel(const kg_ctx* ctx) { return ctx ? ctx->last_kernel : ""; }

int kg_set_wait_limit(kg_ctx* ctx, uint64_t wait_ns) {
  if (!ctx) return KG_ERR_INVALID;
  ctx->wait_ns = wait_ns;
  return KG_OK;
}

int kg_inject_stall(kg_ctx* ctx, uint64_t stop_after_loads) {
  if (!ctx) return KG_ERR_INVALID;
  ctx->stall_once = stop_after_loads;
  return KG_OK;
}

int kg_set_structure_ex(kg_ctx* ctx, const double* U, int n, int k, const double* y, const int32_t* sample_pos,
                        int n_row_samples, double* yyM_out) {
  if (!ctx) return KG_ERR_INVALID;
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");
  ctx->have_structure = false;
  const int n_row = sample_pos ? n_row_samples : n;
  if (sample_pos) {
    if (n_row_samples < n) return ctx->fail(KG_ERR_INVALID, "n_row_samples < n");
    std::vector<char> seen((size_t)n_row_samples, 0);
    for (int i = 0; i < n; ++i) {
      if (sample_pos[i] < 0 || sample_pos[i] >= n_row_samples)
        return ctx->fail(KG_ERR_INVALID, "sample_pos out of range");
      if (seen[sample_pos[i]]++) return ctx->fail(KG_ERR_INVALID, "sample_pos has a repeated position");
    }
  }
  std::string e = kg::prepare(U, n, k, y, ctx->prep);
  if (!e.empty()) return ctx->fail(KG_ERR_INVALID, e);
  const kg::Prepared& p = ctx->prep;
  kg::EpiParams& P = ctx->P;
  std::memset(&P, 0, sizeof(P));
  P.n = n;
  P.k = k;
  P.b = p.b;
  P.kappa = p.kappa;
  P.yyM = p.yyM;
  P.ynorm = p.ynorm;
  P.corr_thr = ctx->opts.corr_threshold;
  P.p_thresh = std::pow(10.0, -ctx->opts.log10_thresh);
  P.r2_cand = r2_candidate(P.p_thresh, n);
  P.thr2_ynorm2 = ctx->opts.corr_threshold * ctx->opts.corr_threshold * p.ynorm * p.ynorm;
  for (int j = 0; j < k; ++j) {
    P.a[j] = p.a[j];
    P.g[j] = p.g[j];
  }
  if (yyM_out) *yyM_out = p.yyM;
  ctx->n_row = n_row;
  // FP64 columns [count, d_0 .. d_{k-1}, d_y], rows = packed-row sample
  // positions: the FP64 form's operand, and the split form's refinement operand
  {
    const int C = k + 2;
    ctx->cm = kg::fp64_cm(C);
    if (ctx->cm < 0) return ctx->fail(KG_ERR_UNSUPPORTED, "too many U.bin columns for the FP64 form");
    ctx->nsteps = kg::fp64_steps(n_row);
    std::vector<double> V((size_t)ctx->nsteps * 128 * ctx->cm, 0.0);
    for (int i = 0; i < n; ++i) {
      const size_t r = (size_t)(sample_pos ? sample_pos[i] : i) * ctx->cm;
      V[r] = 1.0;
      for (int j = 0; j <= k; ++j) V[r + 1 + j] = p.d[(size_t)j * n + i];
    }
    dfree(ctx->dV);
    KG_CUDA(cudaMalloc((void**)&ctx->dV, V.size() * sizeof(double)), "cudaMalloc(V)");
    KG_CUDA(cudaMemcpy(ctx->dV, V.data(), V.size() * sizeof(double), cudaMemcpyHostToDevice), "copy V");
  }
  if (ctx->opts.precision == KG_PREC_SPLIT_I8) {
    // byte tables of V for the FP64 refinement of high-chi-square k-mers
    const int vrows = ctx->nsteps * 128;
    dfree(ctx->dT);
    KG_CUDA(cudaMalloc((void**)&ctx->dT, kg::refine_table_len(vrows, ctx->cm) * sizeof(double)),
            "cudaMalloc(refinement tables)");
    kg::LaunchTable LT{ctx->dV, vrows, ctx->cm, (unsigned long long)vrows * ctx->cm, 1, ctx->dT};
    KG_CUDA(kg::launch_refine_table(LT, ctx->stream), "refinement tables");
    KG_CUDA(cudaStreamSynchronize(ctx->stream), "refinement tables");
    P.refine = 1;
    P.r2_ref = -std::expm1(-kg::REFINE_CHISQ / (double)n);
    e = kg::make_limbs(p, sample_pos, n_row, ctx->opts.limbs_u, ctx->opts.limbs_y, kg::tc_kc(), ctx->limbs);
    if (!e.empty()) return ctx->fail(KG_ERR_UNSUPPORTED, e);
    if (!kg::tc_supported_n(ctx->limbs.N))
      return ctx->fail(KG_ERR_UNSUPPORTED, "contraction width N=" + std::to_string(ctx->limbs.N) +
                                               " not supported by the tensor-core kernel");
    std::vector<int8_t> img;
    kg::make_b_image(ctx->limbs, kg::tc_kc(), img);
    ctx->nchunk = ctx->limbs.Kpad / kg::tc_kc();
    kg::LimbMap& LM = ctx->LM;
    std::memset(&LM, 0, sizeof(LM));
    LM.N = ctx->limbs.N;
    LM.count_col = ctx->limbs.count_col;
    for (int j = 0; j <= k; ++j) {
      LM.first[j] = ctx->limbs.first[j];
      LM.nl[j] = ctx->limbs.nl[j];
      LM.scale[j] = ctx->limbs.scale[j];
    }
    kg::set_limb_consts(LM);
    dfree(ctx->dB);
    KG_CUDA(cudaMalloc((void**)&ctx->dB, img.size()), "cudaMalloc(B)");
    KG_CUDA(cudaMemcpy(ctx->dB, img.data(), img.size(), cudaMemcpyHostToDevice), "copy B");
    kg::make_b_image_ts(ctx->limbs, img);
    dfree(ctx->dBts);
    KG_CUDA(cudaMalloc((void**)&ctx->dBts, img.size()), "cudaMalloc(B)");
    KG_CUDA(cudaMemcpy(ctx->dBts, img.data(), img.size(), cudaMemcpyHostToDevice), "copy B");
  }
  ctx->have_structure = true;
  return KG_OK;
}

int kg_set_structure(kg_ctx* ctx, const double* U, int n, int k, const double* y, double* yyM_out) {
  return kg_set_structure_ex(ctx, U, n, k, y, nullptr, n, yyM_out);
}

}  // extern "C"

namespace kgctx {

// Copy in up to 8 host threads (copies of 64 MB or more).
void par_memcpy(void* dst, const void* src, size_t bytes) {
  const size_t kMin = (size_t)64 << 20;
  unsigned nt = std::min<unsigned>(8, std::max(1u, std::thread::hardware_concurrency()));
  if (bytes < kMin || nt == 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  std::vector<std::thread> th;
  const size_t per = (bytes + nt - 1) / nt;
  for (unsigned t = 0; t < nt; ++t) {
    const size_t a = t * per, b = std::min(bytes, a + per);
    if (a >= b) break;
    th.emplace_back([=] { std::memcpy((char*)dst + a, (const char*)src + a, b - a); });
  }
  for (auto& t : th) t.join();
}

// Gathers rows sel[0..cnt) of x into dst (row bytes each), in parallel for
// large copies.
void par_gather(void* dst, const uint64_t* x, const uint64_t* sel, uint64_t cnt, size_t row) {
  auto body = [=](uint64_t a, uint64_t b) {
    for (uint64_t u = a; u < b; ++u) std::memcpy((char*)dst + u * row, (const char*)x + sel[u] * row, row);
  };
  const size_t kMin = (size_t)64 << 20;
  unsigned nt = std::min<unsigned>(8, std::max(1u, std::thread::hardware_concurrency()));
  if (cnt * row < kMin || nt == 1) {
    body(0, cnt);
    return;
  }
  std::vector<std::thread> th;
  const uint64_t per = (cnt + nt - 1) / nt;
  for (unsigned t = 0; t < nt; ++t) {
    const uint64_t a = t * per, b = std::min<uint64_t>(cnt, a + per);
    if (a >= b) break;
    th.emplace_back(body, a, b);
  }
  for (auto& t : th) t.join();
}

bool is_pinned(const void* p) {
  cudaPointerAttributes attr{};
  const bool pinned = cudaPointerGetAttributes(&attr, p) == cudaSuccess &&
                      (attr.type == cudaMemoryTypeHost || attr.type == cudaMemoryTypeManaged);
  cudaGetLastError();
  return pinned;
}

bool use_runs(const uint64_t* x, uint64_t m, uint32_t wpk, bool pageable) {
  const char* v = std::getenv("KG_DEDUP");
  if ((v && std::string(v) == "0") || m < 2 || m >= (1ull << 32)) return false;
  if (v && std::string(v) == "1") return true;
  if (!pageable || m < 4096) return false;
  int dups = 0;
  for (int i = 0; i < 4096; ++i) {
    const uint64_t j = 1 + (uint64_t)i * (m - 1) / 4096;
    dups += rows_equal(x + j * wpk, x + (j - 1) * wpk, wpk) ? 1 : 0;
  }
  return dups * 10 >= 4096;
}

uint64_t scan_gather(const uint64_t* x, uint64_t s0, uint64_t cnt, uint32_t wpk, void* dst,
                     const std::vector<unsigned long long>& bounds, std::vector<uint64_t>& first,
                     std::vector<uint32_t>& len, std::vector<StageSeg>& segs) {
  const size_t row = (size_t)wpk * 8;
  unsigned nt = std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency()));
  if (cnt < (1u << 16)) nt = 1;
  std::vector<std::vector<uint64_t>> st(nt);
  // one pass: thread t scans rows [a, b) and copies each run's first row to
  // its own slice of dst (rows a - s0 onwards)
  auto scan = [&](unsigned t) {
    const uint64_t a = s0 + cnt * t / nt, b = s0 + cnt * (t + 1) / nt;
    auto bd = std::lower_bound(bounds.begin(), bounds.end(), (unsigned long long)a);
    char* out = (char*)dst + (a - s0) * row;
    std::vector<uint64_t>& v = st[t];
    v.reserve((b - a) / 2 + 16);
    for (uint64_t i = a; i < b; ++i) {
      bool start = i == s0 || !rows_equal(x + i * wpk, x + (i - 1) * wpk, wpk);
      while (bd != bounds.end() && *bd < i) ++bd;
      if (bd != bounds.end() && *bd == i) start = true;
      if (start) {
        std::memcpy(out, x + i * wpk, row);
        out += row;
        v.push_back(i);
      }
    }
  };
  if (nt == 1) {
    scan(0);
  } else {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) th.emplace_back(scan, t);
    for (auto& t : th) t.join();
  }
  const size_t base = first.size();
  segs.clear();
  for (unsigned t = 0; t < nt; ++t) {
    if (!st[t].empty()) segs.push_back({cnt * t / nt, (uint64_t)st[t].size()});
    first.insert(first.end(), st[t].begin(), st[t].end());
  }
  const uint64_t nu = first.size() - base;
  len.resize(base + nu);
  for (uint64_t u = 0; u < nu; ++u)
    len[base + u] = (uint32_t)((u + 1 < nu ? first[base + u + 1] : s0 + cnt) - first[base + u]);
  return nu;
}

bool find_runs(kg_ctx* ctx, const uint64_t* x, uint64_t m, uint32_t wpk, const std::vector<unsigned long long>& bounds,
               bool pageable) {
  if (!use_runs(x, m, wpk, pageable)) return false;
  const char* v = std::getenv("KG_DEDUP");
  const bool force = v && std::string(v) == "1";
  auto same = [&](uint64_t i) { return rows_equal(x + i * wpk, x + (i - 1) * wpk, wpk); };
  unsigned nt = std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency()));
  if (m < (1u << 16)) nt = 1;
  std::vector<std::vector<uint64_t>> starts(nt);
  auto scan = [&](unsigned t) {
    const uint64_t a = m * t / nt, b = m * (t + 1) / nt;
    // the bounds (shard starts) also start runs
    auto bd = std::lower_bound(bounds.begin(), bounds.end(), (unsigned long long)a);
    for (uint64_t i = a; i < b; ++i) {
      bool start = i == 0 || !same(i);
      while (bd != bounds.end() && *bd < i) ++bd;
      if (bd != bounds.end() && *bd == i) start = true;
      if (start) starts[t].push_back(i);
    }
  };
  if (nt == 1) {
    scan(0);
  } else {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) th.emplace_back(scan, t);
    for (auto& t : th) t.join();
  }
  size_t nu = 0;
  for (auto& s : starts) nu += s.size();
  if (force ? nu == m : nu * 10 > m * 9) return false;
  ctx->run_first.clear();
  ctx->run_first.reserve(nu);
  for (auto& s : starts) ctx->run_first.insert(ctx->run_first.end(), s.begin(), s.end());
  ctx->run_len.resize(nu);
  for (size_t u = 0; u < nu; ++u)
    ctx->run_len[u] = (uint32_t)((u + 1 < nu ? ctx->run_first[u + 1] : m) - ctx->run_first[u]);
  return true;
}

int upload_run_lengths(kg_ctx* ctx, cudaStream_t st) {
  const size_t nu = ctx->run_len.size();
  if (ctx->weight_cap < nu) {
    dfree(ctx->dWeight);
    ctx->weight_cap = 0;
    KG_CUDA(cudaMalloc((void**)&ctx->dWeight, nu * sizeof(uint32_t)), "cudaMalloc(run lengths)");
    ctx->weight_cap = nu;
  }
  KG_CUDA(cudaMemcpyAsync(ctx->dWeight, ctx->run_len.data(), nu * sizeof(uint32_t), cudaMemcpyHostToDevice, st),
          "copy run lengths");
  ctx->cur_weight = ctx->dWeight;
  ctx->unique_rows = nu;
  return KG_OK;
}

void expand_runs(const kg_ctx* ctx, std::vector<kg_hit>& hits) {
  std::vector<kg_hit> all;
  for (const kg_hit& h : hits) {
    const uint64_t f = ctx->run_first[h.kmer], e = f + ctx->run_len[h.kmer];
    for (uint64_t i = f; i < e; ++i) {
      all.push_back(h);
      all.back().kmer = i;
    }
  }
  hits.swap(all);
}

void expand_runs(const kg_ctx* ctx, std::vector<kg_phit>& hits) {
  std::vector<kg_phit> all;
  for (const kg_phit& h : hits) {
    const uint64_t f = ctx->run_first[h.kmer], e = f + ctx->run_len[h.kmer];
    for (uint64_t i = f; i < e; ++i) {
      all.push_back(h);
      all.back().kmer = i;
    }
  }
  hits.swap(all);
}

}  // namespace kgctx

namespace {

int ensure_hits(kg_ctx* ctx, unsigned long long cap) {
  if (ctx->hit_cap >= cap && ctx->dHits) return KG_OK;
  dfree(ctx->dHits);
  ctx->hit_cap = 0;
  KG_CUDA(cudaMalloc((void**)&ctx->dHits, cap * sizeof(kg_hit)), "cudaMalloc(hits)");
  ctx->hit_cap = cap;
  return KG_OK;
}

int ensure_cand(kg_ctx* ctx, unsigned long long cap) {
  if (ctx->cand_cap >= cap && ctx->dCand) return KG_OK;
  dfree(ctx->dCand);
  ctx->cand_cap = 0;
  KG_CUDA(cudaMalloc((void**)&ctx->dCand, cap * sizeof(unsigned long long)), "cudaMalloc(candidates)");
  ctx->cand_cap = cap;
  return KG_OK;
}

int ensure_stats(kg_ctx* ctx, size_t m) {
  if (ctx->stat_cap >= m && ctx->dTested) return KG_OK;
  dfree(ctx->dTested);
  dfree(ctx->dPX);
  dfree(ctx->dPairs);
  dfree(ctx->dUnitOff);
  for (auto& p : ctx->dStat) dfree(p);
  ctx->stat_cap = 0;
  KG_CUDA(cudaMalloc((void**)&ctx->dTested, std::max<size_t>(m, 1)), "cudaMalloc(stats)");
  for (auto& p : ctx->dStat) KG_CUDA(cudaMalloc((void**)&p, std::max<size_t>(m, 1) * sizeof(double)), "cudaMalloc(stats)");
  ctx->stat_cap = m;
  return KG_OK;
}

int check_shape(kg_ctx* ctx, const void* x, uint64_t m, uint32_t wpk) {
  if (!ctx->have_structure) return ctx->fail(KG_ERR_STATE, "kg_set_structure has not succeeded");
  if (m > 0 && !x) return ctx->fail(KG_ERR_INVALID, "xbits is NULL");
  if (wpk == 0 || (wpk & 1u)) return ctx->fail(KG_ERR_INVALID, "words_per_kmer must be even and > 0");
  if ((uint64_t)wpk * 64 < (uint64_t)ctx->n_row)
    return ctx->fail(KG_ERR_INVALID, "words_per_kmer*64 < samples per row");
  return KG_OK;
}

int launch_one(kg_ctx* ctx, const uint64_t* dx, uint64_t m, uint32_t wpk, uint64_t offset, bool stats,
               cudaStream_t st) {
  if (m == 0) return KG_OK;
  kg::DevOut O{};
  O.counters = ctx->dCounters;
  O.hits = ctx->dHits;
  O.hit_cap = ctx->hit_cap;
  O.kmer_offset = offset;
  O.cand = ctx->dCand;
  O.cand_cap = ctx->cand_cap;
  O.weight = ctx->cur_weight;
  O.wait_ns = ctx->wait_ns;
  O.stall_loads = ctx->stall_once;
  ctx->stall_once = 0;
  if (stats) {
    O.tested = ctx->dTested;
    O.chisq = ctx->dStat[0];
    O.pval = ctx->dStat[1];
    O.effect = ctx->dStat[2];
    O.mlog10p = ctx->dStat[3];
    O.xxM = ctx->dStat[4];
    O.xyM = ctx->dStat[5];
    O.cor = ctx->dStat[6];
  }
  cudaError_t e;
  if (ctx->opts.precision == KG_PREC_FP64) {
    kg::LaunchFp64 L{dx, m, (int)wpk, ctx->dV, ctx->nsteps, ctx->cm, &ctx->P, &O, ctx->num_sms};
    e = kg::launch_fp64(L, st);
    ctx->last_kernel = "fp64";
  } else {
    // refinement candidates of this launch start from zero
    KG_CUDA(cudaMemsetAsync(ctx->dCounters + 3, 0, sizeof(unsigned long long), st), "memset");
    const char* force = std::getenv("KG_KERNEL");
    const bool want_ss = force && std::string(force) == "ss";
    const bool ts_ok = kg::ts_supported(ctx->limbs.N, ctx->opts.limbs_u, ctx->opts.limbs_y, ctx->limbs.Kpad,
                                        (int)wpk) &&
                       ((uintptr_t)dx % 16) == 0;
    if (force && std::string(force) == "ts" && !ts_ok)
      return ctx->fail(KG_ERR_UNSUPPORTED, "KG_KERNEL=ts: shape not supported by the TMEM-A kernel");
    if (ts_ok && !want_ss) {
      kg::LaunchTs L{dx, m, (int)wpk, ctx->limbs.Kpad, ctx->prep.drop0 && ctx->P.k > 0, ctx->dBts, &ctx->P,
                     &ctx->LM, &O, ctx->num_sms};
      e = kg::launch_ts(L, st);
      ctx->last_kernel = "ts";
    } else {
      kg::LaunchTc L{dx, m, (int)wpk, ctx->nchunk, ctx->dB, &ctx->P, &ctx->LM, &O, ctx->num_sms};
      e = kg::launch_tc(L, st);
      ctx->last_kernel = "ss";
    }
  }
  if (e != cudaSuccess) return ctx->cuda_fail(e, "kernel launch");
  ++ctx->launches;
  if (ctx->P.refine) {
    kg::LaunchFp64 R{dx, m, (int)wpk, ctx->dV, ctx->nsteps, ctx->cm, &ctx->P, &O, ctx->num_sms, ctx->dT};
    e = kg::launch_refine(R, st);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "refinement launch");
    ++ctx->launches;
  }
  return KG_OK;
}

int collect(kg_ctx* ctx, uint64_t m, kg_result* res, kg_stats* st, bool stats_on_device) {
  if (ctx->counters[2] & ~(unsigned long long)(kg::ERR_HIT_OVERFLOW | kg::ERR_CAND_OVERFLOW))
    return ctx->fail(KG_ERR_TIMEOUT, "a bounded device-side wait gave up (error bits " +
                                         std::to_string(ctx->counters[2]) + ")");
  const unsigned long long nh = ctx->counters[1];
  ctx->hits.resize(nh);
  if (nh) {
    KG_CUDA(cudaMemcpy(ctx->hits.data(), ctx->dHits, nh * sizeof(kg_hit), cudaMemcpyDeviceToHost), "copy hits");
    std::sort(ctx->hits.begin(), ctx->hits.end(), [](const kg_hit& a, const kg_hit& b) { return a.kmer < b.kmer; });
  }
  if (st && stats_on_device && m) {
    if (st->tested) KG_CUDA(cudaMemcpy(st->tested, ctx->dTested, m, cudaMemcpyDeviceToHost), "copy stats");
    double* outs[7] = {st->chisq, st->pval, st->effect, st->mlog10p, st->xxM, st->xyM, st->cor};
    for (int i = 0; i < 7; ++i)
      if (outs[i]) KG_CUDA(cudaMemcpy(outs[i], ctx->dStat[i], m * sizeof(double), cudaMemcpyDeviceToHost), "copy stats");
  }
  if (res) {
    res->n_kmers = m;
    res->n_tested = ctx->counters[0];
    res->n_hits = nh;
    res->hits = ctx->hits.data();
  }
  return KG_OK;
}

bool want_stats(const kg_stats* st) {
  return st && (st->tested || st->chisq || st->pval || st->effect || st->mlog10p || st->xxM || st->xyM || st->cor);
}


// One pass of the rows through the chunked host-to-device pipeline.  With
// `runs`, each chunk is scanned for runs of equal rows while it is staged and
// only the first row of each run is copied and tested, weighted by its run's
// length (ctx->run_first / run_len / unique_rows describe the runs).
// Rows per chunk of the host pipeline for m rows of wpk words: 512 MB of
// rows (KG_CHUNK_MB), at most m.
uint64_t host_chunk_rows(uint64_t m, uint32_t wpk) {
  const size_t row = (size_t)wpk * 8;
  size_t want = (size_t)512 << 20;
  if (const char* v = std::getenv("KG_CHUNK_MB")) want = (size_t)std::max(1, std::atoi(v)) << 20;
  uint64_t per = std::max<uint64_t>(1, want / row);
  return per > m ? m : per;
}

// The device chunks (and, with `staging`, the pinned staging buffers) of the
// host pipeline, at least `bytes` each; kept for later calls.
int ensure_chunks(kg_ctx* ctx, size_t bytes, bool staging) {
  if (ctx->chunk_bytes < bytes) {
    for (int b = 0; b < NBUF; ++b) {
      dfree(ctx->dChunk[b]);
      if (ctx->hStage[b]) cudaFreeHost(ctx->hStage[b]);
      ctx->hStage[b] = nullptr;
    }
    ctx->chunk_bytes = 0;
    for (int b = 0; b < NBUF; ++b) KG_CUDA(cudaMalloc((void**)&ctx->dChunk[b], bytes), "cudaMalloc(chunk)");
    ctx->chunk_bytes = bytes;
  }
  if (staging)
    for (int b = 0; b < NBUF; ++b)
      if (!ctx->hStage[b]) KG_CUDA(cudaHostAlloc(&ctx->hStage[b], ctx->chunk_bytes, cudaHostAllocDefault), "cudaHostAlloc");
  return KG_OK;
}

int run_host_once(kg_ctx* ctx, const uint64_t* xbits, uint64_t m, uint32_t wpk, bool stats, bool runs) {
  const size_t row = (size_t)wpk * 8;
  const uint64_t per = host_chunk_rows(m, wpk);
  const size_t bytes = (size_t)per * row;
  const bool pinned = !runs && is_pinned(xbits);
  if (int rc = ensure_chunks(ctx, bytes, !pinned)) return rc;
  if (runs) {
    ctx->run_first.clear();
    ctx->run_len.clear();
    if (ctx->weight_cap < m) {
      dfree(ctx->dWeight);
      ctx->weight_cap = 0;
      KG_CUDA(cudaMalloc((void**)&ctx->dWeight, m * sizeof(uint32_t)), "cudaMalloc(run lengths)");
      ctx->weight_cap = m;
    }
    if (ctx->hweight_cap < per) {
      for (int b = 0; b < NBUF; ++b) {
        if (ctx->hWeight[b]) cudaFreeHost(ctx->hWeight[b]);
        ctx->hWeight[b] = nullptr;
      }
      ctx->hweight_cap = 0;
      for (int b = 0; b < NBUF; ++b)
        KG_CUDA(cudaHostAlloc((void**)&ctx->hWeight[b], per * sizeof(uint32_t), cudaHostAllocDefault), "cudaHostAlloc");
      ctx->hweight_cap = per;
    }
    ctx->cur_weight = ctx->dWeight;
  }
  KG_CUDA(cudaMemsetAsync(ctx->dCounters, 0, 4 * sizeof(unsigned long long), ctx->stream), "memset");
  const uint64_t nch = (m + per - 1) / per;
  uint64_t u0 = 0;  // runs before this chunk
  std::vector<StageSeg> segs;
  for (uint64_t i = 0; i < nch; ++i) {
    const int b = (int)(i % NBUF);
    const uint64_t s = i * per, cnt = std::min<uint64_t>(per, m - s);
    const size_t nb = (size_t)cnt * row;
    uint64_t rows = cnt, offset = s;
    const char* src = (const char*)xbits + (size_t)s * row;
    if (i >= (uint64_t)NBUF) {
      // buffer b was last read by chunk i-NBUF's copy and kernel
      KG_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_k[b], 0), "wait");
      if (!pinned) KG_CUDA(cudaEventSynchronize(ctx->ev_h2d[b]), "sync");
    }
    if (runs) {
      rows = scan_gather(xbits, s, cnt, wpk, ctx->hStage[b], {}, ctx->run_first, ctx->run_len, segs);
      std::memcpy(ctx->hWeight[b], ctx->run_len.data() + u0, rows * sizeof(uint32_t));
      KG_CUDA(cudaMemcpyAsync(ctx->dWeight + u0, ctx->hWeight[b], rows * sizeof(uint32_t), cudaMemcpyHostToDevice,
                              ctx->copy_stream),
              "H2D");
      // the threads' slices of the staging buffer, back to back on the device
      uint64_t d = 0;
      for (const StageSeg& g : segs) {
        KG_CUDA(cudaMemcpyAsync((char*)ctx->dChunk[b] + d * row, (const char*)ctx->hStage[b] + g.stage_row * row,
                                g.rows * row, cudaMemcpyHostToDevice, ctx->copy_stream),
                "H2D");
        d += g.rows;
      }
      offset = u0;
      u0 += rows;
    } else {
      if (!pinned) {
        par_memcpy(ctx->hStage[b], src, nb);
        src = (const char*)ctx->hStage[b];
      }
      KG_CUDA(cudaMemcpyAsync(ctx->dChunk[b], src, nb, cudaMemcpyHostToDevice, ctx->copy_stream), "H2D");
    }
    KG_CUDA(cudaEventRecord(ctx->ev_h2d[b], ctx->copy_stream), "record");
    KG_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev_h2d[b], 0), "wait");
    int rc = launch_one(ctx, ctx->dChunk[b], rows, wpk, offset, stats, ctx->stream);
    if (rc) return rc;
    KG_CUDA(cudaEventRecord(ctx->ev_k[b], ctx->stream), "record");
  }
  if (runs) ctx->unique_rows = u0;
  KG_CUDA(cudaMemcpyAsync(ctx->counters, ctx->dCounters, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          ctx->stream),
          "copy counters");
  KG_CUDA(cudaStreamSynchronize(ctx->stream), "kernel");
  return KG_OK;
}

}  // namespace

extern "C" {

int kg_run_host(kg_ctx* ctx, const uint64_t* xbits, uint64_t m, uint32_t wpk, kg_result* res, kg_stats* st) {
  if (!ctx) return KG_ERR_INVALID;
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");
  int rc = check_shape(ctx, xbits, m, wpk);
  if (rc) return rc;
  ctx->pending = false;
  ctx->launches = 0;
  ctx->unique_rows = 0;
  const bool stats = want_stats(st);
  if (stats && (rc = ensure_stats(ctx, m))) return rc;
  if ((rc = ensure_hits(ctx, std::max<unsigned long long>(ctx->hit_cap, 1ull << 16)))) return rc;
  if ((rc = ensure_cand(ctx, std::max<unsigned long long>(ctx->cand_cap, 1ull << 20)))) return rc;
  std::memset(ctx->counters, 0, sizeof(ctx->counters));
  // per-k-mer outputs are kept for every row, so runs are only used without them
  const bool runs = !stats && use_runs(xbits, m, wpk, !is_pinned(xbits));
  struct Reset {
    kg_ctx* c;
    ~Reset() { c->cur_weight = nullptr; }
  } reset{ctx};
  if (m) {
    if ((rc = run_host_once(ctx, xbits, m, wpk, stats, runs))) return rc;
    for (int retry = 0; retry < 8 && (ctx->counters[2] & (kg::ERR_HIT_OVERFLOW | kg::ERR_CAND_OVERFLOW)); ++retry) {
      if ((ctx->counters[2] & kg::ERR_HIT_OVERFLOW) && (rc = ensure_hits(ctx, ctx->counters[1]))) return rc;
      if ((ctx->counters[2] & kg::ERR_CAND_OVERFLOW) && (rc = ensure_cand(ctx, 4 * ctx->cand_cap))) return rc;
      if ((rc = run_host_once(ctx, xbits, m, wpk, stats, runs))) return rc;
    }
  }
  const uint64_t mt = runs ? ctx->unique_rows : m;  // rows tested on the device
  if ((rc = collect(ctx, mt, res, st, stats))) return rc;
  if (runs) {
    // every row of a run gets its run's row, in row order
    expand_runs(ctx, ctx->hits);
    if (res) {
      res->n_kmers = m;
      res->n_hits = ctx->hits.size();
      res->hits = ctx->hits.data();
    }
  }
  return KG_OK;
}

uint64_t kg_last_unique_rows(const kg_ctx* ctx) { return ctx ? ctx->unique_rows : 0; }

int kg_launch_device(kg_ctx* ctx, const uint64_t* d_x, uint64_t m, uint32_t wpk, void* stream) {
  if (!ctx) return KG_ERR_INVALID;
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");
  int rc = check_shape(ctx, d_x, m, wpk);
  if (rc) return rc;
  if ((rc = ensure_hits(ctx, std::max<unsigned long long>(ctx->hit_cap, 1ull << 16)))) return rc;
  if ((rc = ensure_cand(ctx, std::max<unsigned long long>(ctx->cand_cap, 1ull << 20)))) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  ctx->launches = 0;
  KG_CUDA(cudaMemsetAsync(ctx->dCounters, 0, 4 * sizeof(unsigned long long), st), "memset");
  if ((rc = launch_one(ctx, d_x, m, wpk, 0, ctx->pend_stats, st))) return rc;
  ctx->pending = true;
  ctx->pend_x = d_x;
  ctx->pend_m = m;
  ctx->pend_wpk = wpk;
  ctx->pend_stream = st;
  return KG_OK;
}

}  // extern "C"

// Per-k-mer statistics for device launches are switched on by this
// internal entry (used by kg_fetch's caller through kg_launch_device_stats).
extern "C" int kg_launch_device_stats(kg_ctx* ctx, const uint64_t* d_x, uint64_t m, uint32_t wpk, void* stream) {
  if (!ctx) return KG_ERR_INVALID;
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");  // the statistics buffers live on the context's GPU
  int rc = ensure_stats(ctx, m);
  if (rc) return rc;
  ctx->pend_stats = true;
  rc = kg_launch_device(ctx, d_x, m, wpk, stream);
  if (rc) ctx->pend_stats = false;
  return rc;
}

extern "C" int kg_reserve_host(kg_ctx* ctx, uint64_t m, uint32_t wpk) {
  if (!ctx) return KG_ERR_INVALID;
  if (m == 0 || wpk == 0) return ctx->fail(KG_ERR_INVALID, "kg_reserve_host: empty batch");
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");
  return ensure_chunks(ctx, (size_t)host_chunk_rows(m, wpk) * wpk * 8, true);
}

extern "C" void* kg_host_alloc(size_t bytes) {
  void* p = nullptr;
  // portable: page-locked for every GPU's context, whichever device is current
  if (cudaHostAlloc(&p, bytes ? bytes : 1, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

extern "C" void kg_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

extern "C" int kg_fetch(kg_ctx* ctx, kg_result* res, kg_stats* st) {
  if (!ctx) return KG_ERR_INVALID;
  if (!ctx->pending) return ctx->fail(KG_ERR_STATE, "kg_fetch without a pending kg_launch_device");
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");
  ctx->pending = false;
  const bool stats = ctx->pend_stats;
  ctx->pend_stats = false;
  KG_CUDA(cudaMemcpyAsync(ctx->counters, ctx->dCounters, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          ctx->pend_stream),
          "copy counters");
  KG_CUDA(cudaStreamSynchronize(ctx->pend_stream), "kernel");
  for (int retry = 0; retry < 8 && (ctx->counters[2] & (kg::ERR_HIT_OVERFLOW | kg::ERR_CAND_OVERFLOW)); ++retry) {
    int rc = 0;
    if ((ctx->counters[2] & kg::ERR_HIT_OVERFLOW) && (rc = ensure_hits(ctx, ctx->counters[1]))) return rc;
    if ((ctx->counters[2] & kg::ERR_CAND_OVERFLOW) && (rc = ensure_cand(ctx, 4 * ctx->cand_cap))) return rc;
    KG_CUDA(cudaMemsetAsync(ctx->dCounters, 0, 4 * sizeof(unsigned long long), ctx->pend_stream), "memset");
    if ((rc = launch_one(ctx, ctx->pend_x, ctx->pend_m, ctx->pend_wpk, 0, stats, ctx->pend_stream))) return rc;
    KG_CUDA(cudaMemcpyAsync(ctx->counters, ctx->dCounters, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            ctx->pend_stream),
            "copy counters");
    KG_CUDA(cudaStreamSynchronize(ctx->pend_stream), "kernel");
  }
  return collect(ctx, ctx->pend_m, res, st, stats);
}
