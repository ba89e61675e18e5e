// capi_multi.cpp -- the many-phenotype entry points of include/kgwas_cuda.h.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.hpp"

using namespace kgctx;

namespace kgctx {

void free_multi(kg_ctx* ctx) {
  Multi& M = ctx->mp;
  if (M.graph) cudaGraphExecDestroy(M.graph);
  M.graph = nullptr;
  dfree(M.dB);
  dfree(M.dPh);
  dfree(M.dV);
  dfree(M.dT);
  dfree(M.dCounters);
  dfree(M.dTested);
  dfree(M.dHits);
  dfree(M.dShard);
  M.tested_cap = 0;
  M.hit_cap = 0;
  M.shard_cap = 0;
  M.np = 0;
}

}  // namespace kgctx

namespace {

void drop_graph(Multi& M) {
  if (M.graph) cudaGraphExecDestroy(M.graph);
  M.graph = nullptr;
  M.g_seen = 0;
}

// Resident x tiles and B ring stages that fit the shared memory.
void pick_shape(Multi& M, int nbox, int xs_pref, int nb_pref) {
  const size_t budget = 220 * 1024;
  const int N = M.PPG * M.NP;
  int xs = xs_pref, nb = nb_pref;
  while (xs > 1 && kg::mp_smem_bytes(nbox, xs, 2, N) > budget) --xs;
  while (nb > 2 && kg::mp_smem_bytes(nbox, xs, nb, N) > budget) --nb;
  M.xs = xs;
  M.nb = nb;
}

int ensure_multi_out(kg_ctx* ctx, int n_shards, unsigned long long hit_cap) {
  Multi& M = ctx->mp;
  const size_t need = (size_t)n_shards * M.np;
  if (M.tested_cap < need || !M.dTested) {
    dfree(M.dTested);
    M.tested_cap = 0;
    KG_CUDA(cudaMalloc((void**)&M.dTested, need * sizeof(unsigned long long)), "cudaMalloc(tested)");
    M.tested_cap = need;
    drop_graph(M);
  }
  if (M.hit_cap < hit_cap || !M.dHits) {
    dfree(M.dHits);
    M.hit_cap = 0;
    KG_CUDA(cudaMalloc((void**)&M.dHits, hit_cap * sizeof(kg_phit)), "cudaMalloc(hits)");
    M.hit_cap = hit_cap;
    drop_graph(M);
  }
  if (M.shard_cap < n_shards || !M.dShard) {
    dfree(M.dShard);
    M.shard_cap = 0;
    KG_CUDA(cudaMalloc((void**)&M.dShard, (size_t)std::max(n_shards, 1) * sizeof(unsigned long long)),
            "cudaMalloc(shards)");
    M.shard_cap = n_shards;
    drop_graph(M);
  }
  if (!M.dCounters) KG_CUDA(cudaMalloc((void**)&M.dCounters, 4 * sizeof(unsigned long long)), "cudaMalloc");
  return KG_OK;
}

int set_shards(kg_ctx* ctx, const uint64_t* shard_start, int n_shards, uint64_t m) {
  Multi& M = ctx->mp;
  std::vector<unsigned long long> s;
  if (!shard_start || n_shards <= 0) {
    s.assign(1, 0ull);
  } else {
    if (shard_start[0] != 0) return ctx->fail(KG_ERR_INVALID, "shard_start[0] must be 0");
    for (int i = 0; i < n_shards; ++i) {
      if (i && shard_start[i] < shard_start[i - 1]) return ctx->fail(KG_ERR_INVALID, "shard_start not ascending");
      if (shard_start[i] > m) return ctx->fail(KG_ERR_INVALID, "shard_start beyond n_kmers");
      s.push_back(shard_start[i]);
    }
  }
  if (s != M.shard_host) drop_graph(M);
  M.shard_host = s;
  M.n_shards = (int)s.size();
  return KG_OK;
}

kg::DevOutMP dev_out(kg_ctx* ctx, unsigned long long offset) {
  Multi& M = ctx->mp;
  kg::DevOutMP O;
  std::memset(&O, 0, sizeof(O));
  O.counters = M.dCounters;
  O.tested = M.dTested;
  O.hits = M.dHits;
  O.hit_cap = M.hit_cap;
  O.cand = ctx->dCand;
  O.cand_cap = ctx->cand_cap;
  O.shard_start = M.dShard;
  O.n_shards = M.n_shards;
  O.n_pheno = M.np;
  O.kmer_offset = offset;
  O.weight = ctx->cur_weight;
  O.wait_ns = ctx->wait_ns;
  return O;
}

// Enqueue: candidate reset, the phenotype-tile kernel and its FP64 refinement.
int enqueue_multi(kg_ctx* ctx, const uint64_t* dx, uint64_t m, uint32_t wpk, unsigned long long offset,
                  cudaStream_t st) {
  Multi& M = ctx->mp;
  if (m == 0) return KG_OK;
  kg::DevOutMP O = dev_out(ctx, offset);
  KG_CUDA(cudaMemsetAsync(M.dCounters + 3, 0, sizeof(unsigned long long), st), "memset");
  cudaError_t e;
  if (M.kern >= 1) {
    // tile-iterations per block: the block's packed rows (every CTA's) stay in L2
    // across the G passes; the autotuner scales the 48 MB rule by bt_scale / 2
    const unsigned long long tiles = (m + 127) / 128;
    const unsigned long long grid = std::min<unsigned long long>(tiles, (unsigned long long)ctx->num_sms);
    const unsigned long long tile_bytes = 128ull * wpk * 8;
    unsigned long long bt = (48ull << 20) * (unsigned long long)M.bt_scale / 2 /
                            std::max<unsigned long long>(1, grid * tile_bytes);
    if (const char* v = std::getenv("KG_MP_BT")) bt = (unsigned long long)std::max(1, std::atoi(v));
    bt = std::max<unsigned long long>(1, std::min<unsigned long long>(bt, 1024));
    M.bt = (int)bt;
    kg::LaunchMpb L{dx, m, (int)wpk, M.kpad, M.NP, M.PPG, M.G, (int)bt, M.dB, M.dPh, &O, ctx->num_sms};
    e = M.kern == 2 ? kg::launch_mpb2(L, st) : kg::launch_mpb(L, st);
  } else {
    kg::LaunchMp L{dx, m, (int)wpk, M.kpad, M.NP, M.PPG, M.G, M.xs, M.nb, 0, 0, M.dB, M.dPh, &O, ctx->num_sms};
    e = kg::launch_mp(L, st);
  }
  if (e != cudaSuccess) return ctx->cuda_fail(e, "multi-phenotype kernel launch");
  kg::LaunchMpRefine R{dx, (int)wpk, M.dV, M.nsteps * 128, M.cm, M.vstride, M.dPh, &O, ctx->num_sms, M.dT};
  e = kg::launch_mp_refine(R, st);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "refinement launch");
  ctx->launches += 2;
  return KG_OK;
}

int reset_outputs(kg_ctx* ctx, cudaStream_t st) {
  Multi& M = ctx->mp;
  KG_CUDA(cudaMemsetAsync(M.dCounters, 0, 4 * sizeof(unsigned long long), st), "memset");
  KG_CUDA(cudaMemsetAsync(M.dTested, 0, (size_t)M.n_shards * M.np * sizeof(unsigned long long), st), "memset");
  return KG_OK;
}

// Autotuner.  Times candidate launch shapes on a prefix of the rows (up to
// 148 x 256 x 48 k-mers, every phenotype) and keeps the fastest for this row
// width:
//   image resident in shared memory: the one-SM kernel (mpb, PPG phenotypes
//   per MMA) and, where one phenotype fills an MMA group, the SM-pair kernel
//   (mpb2, two phenotypes per M = 256 MMA), each with L2 blocks of 0.5x, 1x
//   and 2x the 48 MB rule;
//   image streamed from L2 (mp): resident x tiles x B ring stages.
// KG_MP_KERNEL=mp|mpb|mpb2 restricts the search to one kernel.
int autotune(kg_ctx* ctx, const uint64_t* dx, uint64_t m, uint32_t wpk, cudaStream_t st) {
  Multi& M = ctx->mp;
  const int nbox = ((int)wpk * 8 + 127) / 128;
  if (M.tuned && M.tuned_nbox == nbox) return KG_OK;
  struct Cand {
    int kern, xs, nb, bt_scale;
  };
  std::vector<Cand> cands;
  const char* only = std::getenv("KG_MP_KERNEL");
  auto allowed = [&](const char* k) { return !only || std::string(only) == k; };
  if (M.stationary && !(only && std::string(only) == "mp")) {
    for (int s : {2, 1, 4}) {
      if (allowed("mpb")) cands.push_back({1, 1, 4, s});
      if (M.pair_ok && allowed("mpb2")) cands.push_back({2, 1, 4, s});
    }
    if (cands.empty()) cands.push_back({1, 1, 4, 2});  // the requested kernel does not fit these phenotypes
  }
  if (cands.empty()) {
    if (const char* v = std::getenv("KG_MP_SHAPE")) {  // "xs,nb": fixed shape, no tuning
      int xs = 1, nb = 4;
      if (std::sscanf(v, "%d,%d", &xs, &nb) == 2) cands.push_back({0, std::max(1, std::min(2, xs)), std::max(2, std::min(8, nb)), 2});
    }
    if (cands.empty())
      for (const Cand& c : {Cand{0, 1, 4, 2}, Cand{0, 1, 8, 2}, Cand{0, 2, 4, 2}, Cand{0, 2, 8, 2}}) cands.push_back(c);
  }
  if (cands.size() == 1) {
    M.kern = cands[0].kern;
    M.bt_scale = cands[0].bt_scale;
    pick_shape(M, nbox, cands[0].xs, cands[0].nb);
    M.tuned = true;
    M.tuned_nbox = nbox;
    return KG_OK;
  }
  const uint64_t sample = std::min<uint64_t>(m, (uint64_t)ctx->num_sms * 256 * 48);
  cudaEvent_t a, b;
  KG_CUDA(cudaEventCreate(&a), "event");
  KG_CUDA(cudaEventCreate(&b), "event");
  float best = 1e30f;
  Cand win = cands[0];
  for (const Cand& c : cands) {
    M.kern = c.kern;
    M.bt_scale = c.bt_scale;
    pick_shape(M, nbox, c.xs, c.nb);
    if (c.kern == 0 && (M.xs != c.xs || M.nb != c.nb)) continue;  // does not fit
    int rc = reset_outputs(ctx, st);
    if (rc) return rc;
    if ((rc = enqueue_multi(ctx, dx, sample, wpk, 0, st))) return rc;  // warm
    KG_CUDA(cudaEventRecord(a, st), "event");
    if ((rc = enqueue_multi(ctx, dx, sample, wpk, 0, st))) return rc;
    KG_CUDA(cudaEventRecord(b, st), "event");
    KG_CUDA(cudaEventSynchronize(b), "autotune");
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best) {
      best = ms;
      win = c;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  M.kern = win.kern;
  M.bt_scale = win.bt_scale;
  pick_shape(M, nbox, win.xs, win.nb);
  M.tuned = true;
  M.tuned_nbox = nbox;
  return KG_OK;
}

int collect_multi(kg_ctx* ctx, uint64_t m, kg_multi_result* res) {
  Multi& M = ctx->mp;
  if (M.counters[2] & ~(unsigned long long)(kg::ERR_HIT_OVERFLOW | kg::ERR_CAND_OVERFLOW))
    return ctx->fail(KG_ERR_TIMEOUT, "a bounded device-side wait gave up");
  const unsigned long long nh = M.counters[1];
  M.hits.resize(nh);
  if (nh) KG_CUDA(cudaMemcpy(M.hits.data(), M.dHits, nh * sizeof(kg_phit), cudaMemcpyDeviceToHost), "copy hits");
  std::sort(M.hits.begin(), M.hits.end(), [](const kg_phit& a, const kg_phit& b) {
    return a.pheno != b.pheno ? a.pheno < b.pheno : a.kmer < b.kmer;
  });
  M.tested.resize((size_t)M.n_shards * M.np);
  KG_CUDA(cudaMemcpy(M.tested.data(), M.dTested, M.tested.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost),
          "copy counts");
  if (res) {
    res->n_kmers = m;
    res->n_pheno = M.np;
    res->n_shards = M.n_shards;
    res->n_tested = M.tested.data();
    res->n_hits = nh;
    res->hits = M.hits.data();
  }
  return KG_OK;
}

int check_multi(kg_ctx* ctx, const void* x, uint64_t m, uint32_t wpk) {
  Multi& M = ctx->mp;
  if (M.np <= 0) return ctx->fail(KG_ERR_STATE, "kg_set_phenotypes has not succeeded");
  if (m > 0 && !x) return ctx->fail(KG_ERR_INVALID, "xbits is NULL");
  if (wpk == 0 || (wpk & 1u)) return ctx->fail(KG_ERR_INVALID, "words_per_kmer must be even and > 0");
  if ((uint64_t)wpk * 64 < (uint64_t)M.n_row) return ctx->fail(KG_ERR_INVALID, "words_per_kmer*64 < samples per row");
  if (!kg::mp_supported(M.NP, M.PPG, (int)wpk))
    return ctx->fail(KG_ERR_UNSUPPORTED, "rows must be at least 128 bytes (pad words_per_kmer to 16)");
  if (m >= (1ull << 48)) return ctx->fail(KG_ERR_UNSUPPORTED, "more than 2^48 k-mers in one call");
  return KG_OK;
}

}  // namespace

extern "C" {

int kg_set_phenotypes(kg_ctx* ctx, const kg_pheno* ph, int np, int n_row) {
  if (!ctx) return KG_ERR_INVALID;
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");
  Multi& M = ctx->mp;
  free_multi(ctx);
  M.tuned = false;
  if (ctx->opts.precision != KG_PREC_SPLIT_I8)
    return ctx->fail(KG_ERR_UNSUPPORTED, "many-phenotype launches use the split-precision kernels");
  if (ctx->opts.limbs_u != 3 || ctx->opts.limbs_y != 5)
    return ctx->fail(KG_ERR_UNSUPPORTED, "many-phenotype launches use 3 U limbs and 5 y' limbs");
  if (!ph || np <= 0 || np > 65535) return ctx->fail(KG_ERR_INVALID, "n_pheno must be in [1, 65535]");
  if (n_row <= 0) return ctx->fail(KG_ERR_INVALID, "n_row_samples must be positive");
  std::vector<kg::Prepared> prep(np);
  std::vector<kg::LimbCols> limbs(np);
  int NP = 16;
  for (int p = 0; p < np; ++p) {
    const kg_pheno& q = ph[p];
    if (!q.sample_pos || q.n <= 0 || q.n > n_row) return ctx->fail(KG_ERR_INVALID, "phenotype " + std::to_string(p) + ": bad n or sample_pos");
    std::vector<char> seen((size_t)n_row, 0);
    for (int i = 0; i < q.n; ++i) {
      if (q.sample_pos[i] < 0 || q.sample_pos[i] >= n_row || seen[q.sample_pos[i]]++)
        return ctx->fail(KG_ERR_INVALID, "phenotype " + std::to_string(p) + ": sample_pos out of range or repeated");
    }
    std::string e = kg::prepare(q.U_colmajor, q.n, q.k, q.y, prep[p]);
    if (!e.empty()) return ctx->fail(KG_ERR_INVALID, "phenotype " + std::to_string(p) + ": " + e);
    e = kg::make_limbs(prep[p], q.sample_pos, n_row, 3, 5, 128, limbs[p]);
    if (!e.empty()) return ctx->fail(KG_ERR_UNSUPPORTED, "phenotype " + std::to_string(p) + ": " + e);
    NP = std::max(NP, limbs[p].N);
  }
  if (NP > 128) return ctx->fail(KG_ERR_UNSUPPORTED, "a phenotype needs more than 128 limb columns (r too large)");
  // Phenotypes per group: a power of two with NP * PPG <= 128.  The
  // B-stationary kernel needs the group image (kpad x NP*PPG) and the x ring
  // in shared memory: take the widest group that fits; if none does, the
  // streamed-B kernel runs the widest group.
  const int kpad = limbs[0].Kpad;
  int PPG = 1;
  while (PPG * 2 * NP <= 128) PPG *= 2;
  bool stationary = false;
  if (!std::getenv("KG_MP_STREAMED"))
    for (int q = PPG; q >= 1 && !stationary; q /= 2)
      if (kg::mpb_supported(NP, q, kpad, 16)) {
        PPG = q;
        stationary = true;
      }
  const int N = PPG * NP, G = (np + PPG - 1) / PPG;
  M.np = np;
  M.n_row = n_row;
  M.NP = NP;
  M.PPG = PPG;
  M.stationary = stationary;
  M.pair_ok = stationary && PPG == 1 && np >= 2 && kg::mpb2_supported(NP, kpad, 16);
  M.kern = stationary ? 1 : 0;
  M.G = G;
  M.kpad = kpad;
  // B image: group gi at gi*kpad*N in the make_b_image_ts layout (the
  // streamed-B kernel reads it 128 samples at a time), phenotype slot pp at
  // columns [pp*NP, pp*NP + its N).
  std::vector<int8_t> img((size_t)G * kpad * N, 0);
  for (int gi = 0; gi < G; ++gi) {
    std::vector<int8_t> gimg((size_t)kpad * N, 0);
    for (int pp = 0; pp < PPG && gi * PPG + pp < np; ++pp) {
      const int p = gi * PPG + pp;
      if (limbs[p].first[prep[p].k] != 1 || limbs[p].nl[prep[p].k] != 5 || limbs[p].Kpad != kpad)
        return ctx->fail(KG_ERR_INVALID, "unexpected limb layout");
      kg::put_b_image_ts(limbs[p], pp * NP, N, gimg);
    }
    std::copy(gimg.begin(), gimg.end(), img.begin() + (size_t)gi * kpad * N);
  }
  std::vector<kg::MPheno> mph(np);
  int cm = 8;
  for (int p = 0; p < np; ++p) {
    const int k = prep[p].k;
    if (k > 0 && kg::fp64_cm(k + 2) < 0) return ctx->fail(KG_ERR_UNSUPPORTED, "too many U.bin columns");
    cm = std::max(cm, kg::fp64_cm(k + 2));
    std::memset(&mph[p], 0, sizeof(kg::MPheno));
    fill_epi(mph[p].P, prep[p], ctx->opts, true);
    kg::LimbMap& LM = mph[p].LM;
    LM.N = limbs[p].N;
    LM.count_col = limbs[p].count_col;
    for (int j = 0; j <= k; ++j) {
      LM.first[j] = limbs[p].first[j];
      LM.nl[j] = limbs[p].nl[j];
      LM.scale[j] = limbs[p].scale[j];
    }
    kg::set_limb_consts(LM);
    mph[p].drop0 = (k > 0 && prep[p].drop0) ? 1 : 0;
  }
  // FP64 refinement operands: per phenotype, rows = packed-row sample positions,
  // columns [count, d_0 .. d_{k-1}, d_y]
  M.cm = cm;
  M.nsteps = kg::fp64_steps(n_row);
  M.vstride = (size_t)M.nsteps * 128 * cm;
  std::vector<double> V((size_t)np * M.vstride, 0.0);
  for (int p = 0; p < np; ++p) {
    const kg::Prepared& P = prep[p];
    for (int i = 0; i < P.n; ++i) {
      double* row = &V[(size_t)p * M.vstride + (size_t)ph[p].sample_pos[i] * cm];
      row[0] = 1.0;
      for (int j = 0; j <= P.k; ++j) row[1 + j] = P.d[(size_t)j * P.n + i];
    }
  }
  KG_CUDA(cudaMalloc((void**)&M.dB, img.size()), "cudaMalloc(B)");
  KG_CUDA(cudaMemcpy(M.dB, img.data(), img.size(), cudaMemcpyHostToDevice), "copy B");
  KG_CUDA(cudaMalloc((void**)&M.dPh, mph.size() * sizeof(kg::MPheno)), "cudaMalloc(phenotypes)");
  KG_CUDA(cudaMemcpy(M.dPh, mph.data(), mph.size() * sizeof(kg::MPheno), cudaMemcpyHostToDevice), "copy");
  KG_CUDA(cudaMalloc((void**)&M.dV, V.size() * sizeof(double)), "cudaMalloc(V)");
  KG_CUDA(cudaMemcpy(M.dV, V.data(), V.size() * sizeof(double), cudaMemcpyHostToDevice), "copy V");
  const int vrows = M.nsteps * 128;
  KG_CUDA(cudaMalloc((void**)&M.dT, kg::refine_table_len(vrows, cm) * np * sizeof(double)),
          "cudaMalloc(refinement tables)");
  kg::LaunchTable LT{M.dV, vrows, cm, (unsigned long long)M.vstride, np, M.dT};
  KG_CUDA(kg::launch_refine_table(LT, ctx->stream), "refinement tables");
  KG_CUDA(cudaStreamSynchronize(ctx->stream), "refinement tables");
  return KG_OK;
}

int kg_multi_shape(const kg_ctx* ctx, kg_tile_shape* out) {
  if (!ctx || !out) return KG_ERR_INVALID;
  const Multi& M = ctx->mp;
  if (M.np <= 0) return KG_ERR_STATE;
  out->kernel = M.kern == 2 ? 3 : M.kern == 1 ? 1 : 2;
  out->np = M.NP;
  out->ppg = M.kern == 2 ? 2 : M.PPG;
  out->groups = M.kern == 2 ? (M.G + 1) / 2 : M.G;
  out->kpad = M.kpad;
  out->bt = M.bt;
  out->xs = M.xs;
  out->nb = M.nb;
  return KG_OK;
}

int kg_launch_multi_device(kg_ctx* ctx, const uint64_t* dx, uint64_t m, uint32_t wpk, const uint64_t* shard_start,
                           int n_shards, void* stream) {
  if (!ctx) return KG_ERR_INVALID;
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");
  Multi& M = ctx->mp;
  int rc = check_multi(ctx, dx, m, wpk);
  if (rc) return rc;
  if ((rc = set_shards(ctx, shard_start, n_shards, m))) return rc;
  if ((rc = ensure_multi_out(ctx, M.n_shards, std::max<unsigned long long>(M.hit_cap, 1ull << 16)))) return rc;
  if (!ctx->dCand || ctx->cand_cap < (1ull << 20)) {
    dfree(ctx->dCand);
    KG_CUDA(cudaMalloc((void**)&ctx->dCand, (1ull << 20) * sizeof(unsigned long long)), "cudaMalloc(candidates)");
    ctx->cand_cap = 1ull << 20;
    drop_graph(M);
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  KG_CUDA(cudaMemcpyAsync(M.dShard, M.shard_host.data(), M.shard_host.size() * sizeof(unsigned long long),
                          cudaMemcpyHostToDevice, st),
          "copy shards");
  if ((rc = autotune(ctx, dx, m, wpk, st))) return rc;
  ctx->launches = 0;
  // Repeated launches with the same rows and stream replay one captured graph.
  const bool same = M.g_x == dx && M.g_m == m && M.g_wpk == wpk && M.g_stream == st;
  if (!same) {
    drop_graph(M);
    M.g_x = dx;
    M.g_m = m;
    M.g_wpk = wpk;
    M.g_stream = st;
  }
  if (M.graph) {
    KG_CUDA(cudaGraphLaunch(M.graph, st), "graph launch");
    ctx->launches = 2;
  } else if (same && M.g_seen >= 1 && !std::getenv("KG_NO_GRAPH")) {
    cudaGraph_t g = nullptr;
    KG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
    int r1 = reset_outputs(ctx, st);
    int r2 = r1 ? r1 : enqueue_multi(ctx, dx, m, wpk, 0, st);
    cudaError_t ec = cudaStreamEndCapture(st, &g);
    if (r2) {
      if (g) cudaGraphDestroy(g);
      return r2;
    }
    if (ec != cudaSuccess) return ctx->cuda_fail(ec, "capture");
    ec = cudaGraphInstantiate(&M.graph, g, 0);
    cudaGraphDestroy(g);
    if (ec != cudaSuccess) return ctx->cuda_fail(ec, "graph instantiate");
    KG_CUDA(cudaGraphLaunch(M.graph, st), "graph launch");
    ctx->launches = 2;
  } else {
    if ((rc = reset_outputs(ctx, st))) return rc;
    if ((rc = enqueue_multi(ctx, dx, m, wpk, 0, st))) return rc;
    M.g_seen++;
  }
  M.pending = true;
  M.pend_x = dx;
  M.pend_m = m;
  M.pend_wpk = wpk;
  M.pend_stream = st;
  return KG_OK;
}

int kg_fetch_multi(kg_ctx* ctx, kg_multi_result* res) {
  if (!ctx) return KG_ERR_INVALID;
  Multi& M = ctx->mp;
  if (!M.pending) return ctx->fail(KG_ERR_STATE, "kg_fetch_multi without a pending kg_launch_multi_device");
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");
  M.pending = false;
  KG_CUDA(cudaMemcpyAsync(M.counters, M.dCounters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          M.pend_stream),
          "copy counters");
  KG_CUDA(cudaStreamSynchronize(M.pend_stream), "kernel");
  for (int retry = 0; retry < 8 && (M.counters[2] & (kg::ERR_HIT_OVERFLOW | kg::ERR_CAND_OVERFLOW)); ++retry) {
    int rc = 0;
    if ((M.counters[2] & kg::ERR_HIT_OVERFLOW) && (rc = ensure_multi_out(ctx, M.n_shards, M.counters[1])))
      return rc;
    if (M.counters[2] & kg::ERR_CAND_OVERFLOW) {
      const unsigned long long cap = 4 * ctx->cand_cap;
      dfree(ctx->dCand);
      ctx->cand_cap = 0;
      KG_CUDA(cudaMalloc((void**)&ctx->dCand, cap * sizeof(unsigned long long)), "cudaMalloc(candidates)");
      ctx->cand_cap = cap;
    }
    drop_graph(M);
    if ((rc = reset_outputs(ctx, M.pend_stream))) return rc;
    if ((rc = enqueue_multi(ctx, M.pend_x, M.pend_m, M.pend_wpk, 0, M.pend_stream))) return rc;
    KG_CUDA(cudaMemcpyAsync(M.counters, M.dCounters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            M.pend_stream),
            "copy counters");
    KG_CUDA(cudaStreamSynchronize(M.pend_stream), "kernel");
  }
  return collect_multi(ctx, M.pend_m, res);
}

int kg_run_multi_host(kg_ctx* ctx, const uint64_t* xbits, uint64_t m, uint32_t wpk, const uint64_t* shard_start,
                      int n_shards, kg_multi_result* res) {
  if (!ctx) return KG_ERR_INVALID;
  KG_CUDA(cudaSetDevice(ctx->opts.device), "cudaSetDevice");
  Multi& M = ctx->mp;
  int rc = check_multi(ctx, xbits, m, wpk);
  if (rc) return rc;
  if ((rc = set_shards(ctx, shard_start, n_shards, m))) return rc;
  cudaStream_t st = ctx->stream;
  // runs of equal rows (as in kg_run_host); a shard start also starts a run,
  // so each tested row belongs to one shard
  ctx->unique_rows = 0;
  const bool dedup = find_runs(ctx, xbits, m, wpk, M.shard_host, !is_pinned(xbits));
  const uint64_t* sel = nullptr;
  const uint64_t m_all = m;
  if (dedup) {
    std::vector<uint64_t> us(M.shard_host.size());
    for (size_t i = 0; i < us.size(); ++i)
      us[i] = (uint64_t)(std::lower_bound(ctx->run_first.begin(), ctx->run_first.end(), M.shard_host[i]) -
                         ctx->run_first.begin());
    m = ctx->run_first.size();
    sel = ctx->run_first.data();
    if ((rc = set_shards(ctx, us.data(), (int)us.size(), m))) return rc;
    if ((rc = upload_run_lengths(ctx, st))) return rc;
  }
  struct Reset {
    kg_ctx* c;
    ~Reset() { c->cur_weight = nullptr; }
  } reset{ctx};
  if ((rc = ensure_multi_out(ctx, M.n_shards, std::max<unsigned long long>(M.hit_cap, 1ull << 16)))) return rc;
  if (!ctx->dCand || ctx->cand_cap < (1ull << 20)) {
    dfree(ctx->dCand);
    KG_CUDA(cudaMalloc((void**)&ctx->dCand, (1ull << 20) * sizeof(unsigned long long)), "cudaMalloc(candidates)");
    ctx->cand_cap = 1ull << 20;
  }
  KG_CUDA(cudaMemcpyAsync(M.dShard, M.shard_host.data(), M.shard_host.size() * sizeof(unsigned long long),
                          cudaMemcpyHostToDevice, st),
          "copy shards");
  ctx->launches = 0;
  for (int attempt = 0; attempt < 8; ++attempt) {
    if ((rc = reset_outputs(ctx, st))) return rc;
    // Chunks of the rows stream through two device buffers: the copy of
    // chunk i+1 (copy stream) overlaps the kernels of chunk i (compute stream).
    const size_t row = (size_t)wpk * 8;
    size_t want = (size_t)512 << 20;  // small chunks: less copy and compute left unoverlapped at the ends
    if (const char* v = std::getenv("KG_CHUNK_MB")) want = (size_t)std::max(1, std::atoi(v)) << 20;
    uint64_t per = std::max<uint64_t>(1, want / row);
    if (per > m) per = m;
    const size_t bytes = (size_t)per * row;
    cudaPointerAttributes attr{};
    const bool pinned = !sel && (m == 0 || (cudaPointerGetAttributes(&attr, xbits) == cudaSuccess &&
                                            (attr.type == cudaMemoryTypeHost || attr.type == cudaMemoryTypeManaged)));
    cudaGetLastError();
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
    if (!pinned)
      for (int b = 0; b < NBUF; ++b)
        if (!ctx->hStage[b])
          KG_CUDA(cudaHostAlloc(&ctx->hStage[b], ctx->chunk_bytes, cudaHostAllocDefault), "cudaHostAlloc");
    const uint64_t nch = m ? (m + per - 1) / per : 0;
    for (uint64_t i = 0; i < nch; ++i) {
      const int b = (int)(i % NBUF);
      const uint64_t s0 = i * per, cnt = std::min<uint64_t>(per, m - s0);
      const size_t nb = (size_t)cnt * row;
      const char* src = (const char*)xbits + (size_t)s0 * row;
      if (i >= (uint64_t)NBUF) {
        KG_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_k[b], 0), "wait");
        if (!pinned) KG_CUDA(cudaEventSynchronize(ctx->ev_h2d[b]), "sync");
      }
      if (sel) {
        par_gather(ctx->hStage[b], xbits, sel + s0, cnt, row);
        src = (const char*)ctx->hStage[b];
      } else if (!pinned) {
        par_memcpy(ctx->hStage[b], src, nb);
        src = (const char*)ctx->hStage[b];
      }
      KG_CUDA(cudaMemcpyAsync(ctx->dChunk[b], src, nb, cudaMemcpyHostToDevice, ctx->copy_stream), "H2D");
      KG_CUDA(cudaEventRecord(ctx->ev_h2d[b], ctx->copy_stream), "record");
      KG_CUDA(cudaStreamWaitEvent(st, ctx->ev_h2d[b], 0), "wait");
      if (i == 0 && (rc = autotune(ctx, ctx->dChunk[b], cnt, wpk, st))) return rc;
      if (i == 0 && (rc = reset_outputs(ctx, st))) return rc;  // the autotuner's trial launches wrote outputs
      if ((rc = enqueue_multi(ctx, ctx->dChunk[b], cnt, wpk, s0, st))) return rc;
      KG_CUDA(cudaEventRecord(ctx->ev_k[b], st), "record");
    }
    KG_CUDA(cudaMemcpyAsync(M.counters, M.dCounters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st),
            "copy counters");
    KG_CUDA(cudaStreamSynchronize(st), "kernel");
    if (!(M.counters[2] & (kg::ERR_HIT_OVERFLOW | kg::ERR_CAND_OVERFLOW))) break;
    if ((M.counters[2] & kg::ERR_HIT_OVERFLOW) && (rc = ensure_multi_out(ctx, M.n_shards, M.counters[1])))
      return rc;
    if (M.counters[2] & kg::ERR_CAND_OVERFLOW) {
      const unsigned long long cap = 4 * ctx->cand_cap;
      dfree(ctx->dCand);
      ctx->cand_cap = 0;
      KG_CUDA(cudaMalloc((void**)&ctx->dCand, cap * sizeof(unsigned long long)), "cudaMalloc(candidates)");
      ctx->cand_cap = cap;
    }
  }
  drop_graph(M);
  M.g_x = nullptr;
  if ((rc = collect_multi(ctx, m, res))) return rc;
  if (dedup) {
    expand_runs(ctx, M.hits);
    if (res) {
      res->n_kmers = m_all;
      res->n_hits = M.hits.size();
      res->hits = M.hits.data();
    }
  }
  return KG_OK;
}

}  // extern "C"
