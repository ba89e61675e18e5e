// kernel_mp.cu -- many phenotypes per k-mer tile (split precision).
//
// The reference tests one phenotype per process and re-reads the batch for
// each (HPC/kgwas/kgwas_cols.sh:22-65).  Here a persistent CTA per SM takes a
// 128-k-mer tile, keeps its packed rows resident in shared memory, and runs
// every phenotype over it:
//   warps 0-3   epilogue: per phenotype of the group, limb recombination and
//               the FP64 statistic (src/kgwas.cpp:44-56, 182-218); tested
//               counts per (shard, phenotype), hit and refinement records;
//   warps 4-11  unpack, two groups: 128 samples of the resident tile ->
//               int8 (0 / -128) -> one TMEM A stage (tcgen05.st);
//   warp 12     x producer: the tile's packed rows, one 2-D TMA load per
//               1024 samples (128-byte swizzle, no multicast);
//   warp 13     B producer: the int8 limbs of each phenotype group, one
//               128-sample x N chunk per bulk copy from L2 into a ring;
//   warp 14     MMA: tcgen05.mma kind::i8, A from TMEM, B from the ring,
//               into split-K TMEM accumulators (N = phenotypes per group x
//               slot width <= 128 columns).
// Group gi of a tile re-unpacks the tile (cheap: it is on chip) while the
// previous group's accumulator is drained by the epilogue.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "device.cuh"
#include "kernels.hpp"

namespace kg {

constexpr int MP_TM = 128;
constexpr int MP_KS = 128;
constexpr int MP_UG = 2;
constexpr int MP_LU = 3, MP_LY = 5;
constexpr int MP_WARP_UNPACK0 = 4, MP_WARP_XP = 4 + 4 * MP_UG, MP_WARP_BP = MP_WARP_XP + 1,
              MP_WARP_MMA = MP_WARP_BP + 1;
constexpr int MP_THREADS = 32 * (MP_WARP_MMA + 1);
constexpr uint32_t MP_BOXB = MP_TM * 128;  // one TMA box: 128 rows x 128 bytes
constexpr unsigned long long MP_KMER_MASK = (1ull << 48) - 1;

// TMEM: NA accumulator buffers x S split-K accumulators x N columns, then A stages.
__host__ __device__ constexpr int mp_a0(int N, int S, int NA) { return ((NA * S * N + 31) / 32) * 32; }
__host__ __device__ constexpr int mp_ast(int N, int S, int NA) {
  return (512 - mp_a0(N, S, NA)) / 32 > 16 ? 16 : (512 - mp_a0(N, S, NA)) / 32;
}

struct MpSmem {
  uint32_t x, b, bars, tmem, abort, total;
};
__host__ __device__ inline MpSmem mp_smem(int nbox, int xs, int nb, int N) {
  MpSmem L;
  L.x = 0;
  L.b = (uint32_t)xs * nbox * MP_BOXB;
  L.bars = L.b + (uint32_t)nb * 128 * N;
  L.tmem = L.bars + 8 * (2 * 2 + 2 * 8 + 2 * 16 + 4 + 1);
  L.abort = L.tmem + 8;
  L.total = L.abort + 8;
  return L;
}

template <int NP, int PPG>
__global__ void __launch_bounds__(MP_THREADS, 1)
    mp_kernel(const __grid_constant__ CUtensorMap tmap, unsigned long long m, int nbox, int nchunk, int G,
              int xs_slots, int nb, int S, int NA, const int8_t* __restrict__ Bimg, const MPheno* __restrict__ ph,
              const DevOutMP O) {
  constexpr int N = PPG * NP;
  static_assert(N <= 128, "phenotype group wider than one MMA");
  const int A0 = mp_a0(N, S, NA);
  const int AST = mp_ast(N, S, NA);
  constexpr uint32_t IDESC = idesc_i8(MP_TM, N);
  constexpr uint32_t BCH = 128u * N;  // bytes of one B chunk (128 samples x N)
  constexpr int KU_MAX = (NP - 1 - MP_LY) / MP_LU;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gbase = smem_raw + (base - raw);
  const MpSmem L = mp_smem(nbox, xs_slots, nb, N);
  const uint32_t sx = base + L.x, sb = base + L.b;
  const uint32_t x_full = base + L.bars, x_empty = x_full + 16;
  const uint32_t b_full = x_empty + 16, b_empty = b_full + 64;
  const uint32_t a_full = b_empty + 64, a_empty = a_full + 128;
  const uint32_t acc_full = a_empty + 128, acc_empty = acc_full + 16, drain = acc_empty + 16;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(gbase + L.tmem);
  volatile int* s_abort = reinterpret_cast<volatile int*>(gbase + L.abort);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t xslot = (uint32_t)nbox * MP_BOXB;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < xs_slots; ++s) {
      mbar_init(x_full + 8 * s, 1);
      mbar_init(x_empty + 8 * s, 4 * MP_UG);
    }
    for (int s = 0; s < nb; ++s) {
      mbar_init(b_full + 8 * s, 1);
      mbar_init(b_empty + 8 * s, 1);
    }
    for (int t = 0; t < AST; ++t) {
      mbar_init(a_full + 8 * t, 4);
      mbar_init(a_empty + 8 * t, 1);
    }
    for (int b = 0; b < NA; ++b) {
      mbar_init(acc_full + 8 * b, 1);
      mbar_init(acc_empty + 8 * b, 4);
    }
    mbar_init(drain, 1);
    *s_abort = 0;
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const unsigned long long lim = wait_limit(O.wait_ns);
  const unsigned long long ntiles = (m + MP_TM - 1) / MP_TM;

  if (warp == MP_WARP_XP) {
    // ---------------------------------------------------------- x producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(&tmap) : "memory");
      uint32_t last_use[2] = {0xffffffffu, 0xffffffffu};
      uint32_t it = 0;
      for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const uint32_t xs = it % xs_slots, u = it / xs_slots;
        if (u > 0 && !wait_or_abort(x_empty + 8 * xs, (u - 1) & 1, s_abort, O.counters, ERR_TIMEOUT_FULL, lim)) break;
        mbar_arrive_expect_tx(x_full + 8 * xs, xslot);
        for (int bx = 0; bx < nbox; ++bx)
          tma_load_2d(sx + xs * xslot + bx * MP_BOXB, &tmap, bx * 128, (int)(tile * MP_TM), x_full + 8 * xs);
        last_use[xs] = u;
      }
      for (int s = 0; s < xs_slots; ++s)
        if (last_use[s] != 0xffffffffu) mbar_wait(x_full + 8 * s, last_use[s] & 1, O.counters, ERR_TIMEOUT_FULL);
    }
  } else if (warp == MP_WARP_BP) {
    // ---------------------------------------------------------- B producer
    if (lane == 0) {
      uint32_t last_use[8];
      for (int s = 0; s < 8; ++s) last_use[s] = 0xffffffffu;
      uint32_t h = 0;
      bool ok = true;
      for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x)
        for (int gi = 0; gi < G && ok; ++gi)
          for (int kc = 0; kc < nchunk; ++kc, ++h) {
            const uint32_t s = h % nb, u = h / nb;
            if (u > 0 && !wait_or_abort(b_empty + 8 * s, (u - 1) & 1, s_abort, O.counters, ERR_TIMEOUT_FULL, lim)) {
              ok = false;
              break;
            }
            mbar_arrive_expect_tx(b_full + 8 * s, BCH);
            bulk_g2s(sb + s * BCH, Bimg + ((size_t)gi * nchunk + kc) * BCH, BCH, b_full + 8 * s);
            last_use[s] = u;
          }
      for (int s = 0; s < nb; ++s)
        if (last_use[s] != 0xffffffffu) mbar_wait(b_full + 8 * s, last_use[s] & 1, O.counters, ERR_TIMEOUT_FULL);
    }
  } else if (warp == MP_WARP_MMA) {
    // ----------------------------------------------------------------- MMA
    if (lane == 0) {
      uint32_t g = 0, h = 0, w = 0;
      bool ok = true;
      for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        for (int gi = 0; gi < G && ok; ++gi, ++w) {
          const uint32_t b = w % NA, v = w / NA;
          if (v > 0 && !wait_or_abort(acc_empty + 8 * b, (v - 1) & 1, s_abort, O.counters, ERR_TIMEOUT_MMA, lim)) {
            ok = false;
            break;
          }
          tc_fence_after();
          for (int kc = 0; kc < nchunk; ++kc, ++g, ++h) {
            const uint32_t t = g % AST, s = h % nb;
            if (!wait_or_abort(a_full + 8 * t, (g / AST) & 1, s_abort, O.counters, ERR_TIMEOUT_MMA, lim) ||
                !wait_or_abort(b_full + 8 * s, (h / nb) & 1, s_abort, O.counters, ERR_TIMEOUT_MMA, lim)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t d_t = tmem + (b * S + kc % S) * N;  // split-K accumulator of this stage
#pragma unroll
            for (int ks = 0; ks < MP_KS / 32; ++ks) {
              const uint64_t bd = sdesc_noswz(sb + s * BCH + ks * 2 * (N * 16), N * 16, 128);
              tc_mma_i8_ts(d_t, tmem + A0 + t * 32 + ks * 8, bd, IDESC, (kc >= S || ks != 0) ? 1u : 0u);
            }
            tc_commit(a_empty + 8 * t);
            tc_commit(b_empty + 8 * s);
          }
          if (ok) tc_commit(acc_full + 8 * b);
        }
      }
      tc_commit(drain);
      mbar_wait(drain, 0, O.counters, ERR_TIMEOUT_MMA);
    }
  } else if (warp >= MP_WARP_UNPACK0) {
    // -------------------------------------------------------------- unpack
    const int grp = (warp - MP_WARP_UNPACK0) >> 2;
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    uint32_t g = 0, it = 0;
    bool ok = true;
    for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++it) {
      const uint32_t xs = it % xs_slots;
      if (!__all_sync(0xffffffffu, wait_or_abort(x_full + 8 * xs, (it / xs_slots) & 1, s_abort, O.counters,
                                           ERR_TIMEOUT_FULL, lim)))
        break;
      const uint32_t tb = sx + xs * xslot;
      for (int gi = 0; gi < G && ok; ++gi) {
        for (int kc = 0; kc < nchunk; ++kc, ++g) {
          if ((int)(g % MP_UG) != grp) continue;
          const uint32_t t = g % AST, u = g / AST;
          if (u > 0 && !__all_sync(0xffffffffu, wait_or_abort(a_empty + 8 * t, (u - 1) & 1, s_abort, O.counters,
                                                         ERR_TIMEOUT_MMA, lim))) {
            ok = false;
            break;
          }
          const int bx = kc >> 3, c = kc & 7;
          uint4 v;
          asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];"
                       : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                       : "r"(tb + bx * MP_BOXB + r * 128 + ((c ^ (r & 7)) << 4)));
          const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
          uint32_t o[32];
          unpack_stage(w4, o);
          tc_st32(tmem + lane_base + A0 + t * 32, o);
          tc_wait_st();
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(a_full + 8 * t);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(x_empty + 8 * xs);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    const int nsplit = nchunk < S ? nchunk : S;
    uint32_t w = 0;
    bool ok = true;
    for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
      const unsigned long long local = tile * MP_TM + r;
      const bool valid = local < m;
      const unsigned long long gk = O.kmer_offset + local;
      const int shard = mp_shard(O, gk);
      const unsigned match = __match_any_sync(0xffffffffu, shard);
      const bool leader = lane == __ffs(match) - 1;
      for (int gi = 0; gi < G; ++gi, ++w) {
        const uint32_t b = w % NA, v = w / NA;
        if (!__all_sync(0xffffffffu, wait_or_abort(acc_full + 8 * b, v & 1, s_abort, O.counters, ERR_TIMEOUT_MMA, lim))) {
          ok = false;
          break;
        }
        tc_fence_after();
        for (int pp = 0; pp < PPG; ++pp) {
          const int p = gi * PPG + pp;
          if (p >= O.n_pheno) break;
          // this phenotype's slot of the accumulator: NP int32 columns
          // sum of the split-K partial accumulators of this slot
          uint32_t d[NP];
#pragma unroll
          for (int c16 = 0; c16 < NP / 16; ++c16) {
            uint32_t rr[16];
            tc_ld16(tmem + lane_base + b * S * N + pp * NP + c16 * 16, rr);
            tc_wait_ld();
#pragma unroll
            for (int e = 0; e < 16; ++e) d[c16 * 16 + e] = rr[e];
            for (int sp = 1; sp < nsplit; ++sp) {
              tc_ld16(tmem + lane_base + (b * S + sp) * N + pp * NP + c16 * 16, rr);
              tc_wait_ld();
#pragma unroll
              for (int e = 0; e < 16; ++e) d[c16 * 16 + e] += rr[e];
            }
          }
          const MPheno& ME = ph[p];
          const int k = ME.P.k;
          const int drop0 = ME.drop0;
          // Limb sums hold -128 * integer sums only after recombination (half
          // the samples enter as 64 x against the digits of -2 V): recombine
          // exactly in int64 first, as kernel_ts.cu does.
          const int c = (-(int)d[0]) >> 7;
          const double cd = i2d_exact(c);
          long long Vy = (long long)(int)d[MP_LY];
#pragma unroll
          for (int l = 1; l < MP_LY; ++l) Vy += (long long)(int)d[MP_LY - l] * (1ll << (8 * l));
          const double sy = ME.LM.scale[k];
          const double ey = fma(magic_raw((-Vy) >> 7), sy, -MAGIC_BIAS * sy);
          double ss = 0, gs = 0;
          if (drop0) {
            const double s0 = ME.P.a[0] * cd;
            ss = s0 * s0;
          }
#pragma unroll
          for (int jj = 0; jj < KU_MAX; ++jj) {
            const int j = jj + drop0;
            const int o = 1 + MP_LY + MP_LU * jj;
            long long Vb = (long long)(int)d[o + MP_LU - 1] + (long long)0x4338000000000000LL;
#pragma unroll
            for (int l = 1; l < MP_LU; ++l) Vb += (long long)(int)d[o + MP_LU - 1 - l] * (1ll << (8 * l));
            const double e = fma(__longlong_as_double(Vb), ME.LM.esc[j], ME.LM.eoff[j]);
            const double sj = fma(ME.P.a[j], cd, e);
            ss = fma(sj, sj, ss);
            gs = fma(ME.P.g[j], e, gs);
          }
          bool tested, hit, cand;
          double T, pv, effect;
          mp_eval(ME.P, valid, c, ss, gs, ey, tested, hit, cand, T, pv, effect);
          mp_emit(O, p, gk, shard, match, leader, tested, hit, cand, T, pv, effect);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acc_empty + 8 * b);
      }
    }
  }
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// FP64 recomputation of the candidates of a multi-phenotype launch: one
// warp per (k-mer, phenotype), the phenotype's byte tables at T + p*tstride
// (lanes own the FP64 columns, one table row per byte of the packed row).
template <int CM>
__global__ void __launch_bounds__(256) mp_refine_kernel(const uint64_t* __restrict__ x, int wpk, int nwords,
                                                        const double* __restrict__ T, unsigned long long tstride,
                                                        const MPheno* __restrict__ ph, const DevOutMP O) {
  const int lane = threadIdx.x & 31;
  const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x >> 5);
  unsigned long long ncand = O.counters[3];
  if (ncand > O.cand_cap) ncand = O.cand_cap;
  for (unsigned long long w = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < ncand;
       w += warps) {
    const unsigned long long ent = O.cand[w];
    const unsigned long long gk = ent & MP_KMER_MASK;
    const int p = (int)(ent >> 48);
    const EpiParams& P = ph[p].P;
    const uint64_t* row = x + (gk - O.kmer_offset) * (unsigned long long)wpk;
    double acc[(CM + 31) / 32];
    table_row_sums<CM>(row, nwords, T + (size_t)p * tstride, lane, acc);
    int c;
    double ss, ey;
    refine_reduce<CM>(P, acc, lane, c, ss, ey);
    if (lane == 0) {
      const double xxM = (double)c - ss, xyM = P.b * (double)c + ey;
      double effect = 0, Tq = 0, pv = 1;
      if (xxM > 1e-12 && P.yyM > 1e-12) {
        double r2 = (xyM * xyM) / (xxM * P.yyM);
        if (r2 < 0) r2 = 0;
        if (r2 >= 1) r2 = 1 - 1e-15;
        Tq = (double)P.n * log(1.0 / (1.0 - r2));
        pv = erfc(sqrt(0.5 * Tq));
        effect = xyM / (xxM * P.yyM);
      }
      if (pv <= P.p_thresh) {
        const unsigned long long slot = atomicAdd(O.counters + 1, 1ull);
        if (slot < O.hit_cap) {
          kg_phit h;
          h.kmer = gk;
          h.pheno = p;
          h.shard = mp_shard(O, gk);
          h.effect = effect;
          h.pval = pv;
          h.chisq = Tq;
          O.hits[slot] = h;
        } else {
          atomicOr(O.counters + 2, (unsigned long long)ERR_HIT_OVERFLOW);
        }
      }
    }
  }
}

// ------------------------------------------------------------------- host

static PFN_cuTensorMapEncodeTiled_v12000 mp_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

size_t mp_smem_bytes(int nbox, int xs, int nb, int N) { return mp_smem(nbox, xs, nb, N).total + 1024; }

bool mp_supported(int NP, int PPG, int wpk) {
  if (NP < 16 || NP > 128 || NP % 16 || PPG < 1 || NP * PPG > 128) return false;
  if (wpk * 8 < 128) return false;
  return mp_encode_fn() != nullptr;
}

template <int NP, int PPG>
static cudaError_t launch_mp_t(const LaunchMp& L, const CUtensorMap& tm, cudaStream_t st) {
  constexpr int N = PPG * NP;
  const int nbox = (L.wpk * 8 + 127) / 128;
  const size_t smem = mp_smem_bytes(nbox, L.xs, L.nb, N);
  cudaError_t e = cudaFuncSetAttribute(mp_kernel<NP, PPG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const unsigned long long tiles = (L.m + MP_TM - 1) / MP_TM;
  unsigned long long grid = (unsigned long long)L.num_sms;
  if (grid > tiles) grid = tiles;
  int S = L.splits, NA = L.nacc;
  if (S < 1 || NA < 1 || mp_ast(N, S, NA) < 4) {  // default: one chain, two accumulator buffers
    S = 1;
    NA = 2;
  }
  mp_kernel<NP, PPG><<<(unsigned)grid, MP_THREADS, smem, st>>>(tm, L.m, nbox, L.kpad / MP_KS, L.G, L.xs, L.nb, S,
                                                               NA, L.Bimg, L.ph, *L.O);
  return cudaGetLastError();
}

bool mp_tmap(const uint64_t* x, unsigned long long m, int wpk, CUtensorMap* tm) {
  auto enc = mp_encode_fn();
  if (!enc) return false;
  const cuuint64_t rowbytes = (cuuint64_t)wpk * 8;
  cuuint64_t gdim[2] = {rowbytes, (cuuint64_t)m};
  cuuint64_t gstride[1] = {rowbytes};
  cuuint32_t box[2] = {128, MP_TM};
  cuuint32_t estr[2] = {1, 1};
  return enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)x, gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_mp(const LaunchMp& L, cudaStream_t st) {
  CUtensorMap tm;
  if (!mp_tmap(L.x, L.m, L.wpk, &tm)) return cudaErrorInvalidValue;
#define KG_MP_CASE(NP_, PPG_) \
  if (L.NP == NP_ && L.PPG == PPG_) return launch_mp_t<NP_, PPG_>(L, tm, st);
  KG_MP_GROUPS(KG_MP_CASE)
#undef KG_MP_CASE
  return cudaErrorInvalidValue;
}

template <int CM>
static cudaError_t launch_mp_refine_t(const LaunchMpRefine& L, cudaStream_t st) {
  static int per_sm = 0;  // every warp of the grid resident at once (candidates are dealt round-robin)
  if (per_sm < 1 &&
      (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mp_refine_kernel<CM>, 256, 0) != cudaSuccess ||
       per_sm < 1))
    per_sm = 1;
  mp_refine_kernel<CM><<<(unsigned)(L.num_sms * per_sm), 256, 0, st>>>(
      L.x, L.wpk, L.vrows / 64, L.T, (unsigned long long)refine_table_len(L.vrows, L.cm), L.ph, *L.O);
  return cudaGetLastError();
}

cudaError_t launch_mp_refine(const LaunchMpRefine& L, cudaStream_t st) {
  if (!L.T) return cudaErrorInvalidValue;
  switch (L.cm) {
    case 8: return launch_mp_refine_t<8>(L, st);
    case 12: return launch_mp_refine_t<12>(L, st);
    case 16: return launch_mp_refine_t<16>(L, st);
    case 20: return launch_mp_refine_t<20>(L, st);
    case 24: return launch_mp_refine_t<24>(L, st);
    case 28: return launch_mp_refine_t<28>(L, st);
    case 36: return launch_mp_refine_t<36>(L, st);
    case 44: return launch_mp_refine_t<44>(L, st);
    case 52: return launch_mp_refine_t<52>(L, st);
    case 68: return launch_mp_refine_t<68>(L, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kg
