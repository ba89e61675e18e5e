// kernels.cu -- the association kernels.
//
//   fp64_kernel  : plain FP64 form on CUDA cores.  One thread per k-mer;
//                  the contraction columns (phenotyped-sample indicator, then
//                  the centred structure and phenotype columns) are staged
//                  through shared memory 128 samples at a time and every lane
//                  FMAs its own bits against the broadcast rows.
//   tc_ss_kernel : split-precision form on the 5th-generation tensor cores.
//                  x is unpacked exactly to int8 (0/1), the centred columns are
//                  int8 limbs, tcgen05.mma kind::i8 accumulates exactly in
//                  int32 TMEM, and the FP64 epilogue recombines the limbs.
//
// Both replace the reference's Pearson pre-filter (src/kgwas.cpp:182-218),
// compute_cols_stats (:138-166), compute_hit (:44-56) and the emit selection
// (:247-255); see prep.hpp for the algebra.
#include <cstdio>

#include "device.cuh"
#include "kernels.hpp"

namespace kg {

// ======================================================= FP64 CUDA-core form
constexpr int F64_TB = 128;   // k-mers (threads) per block
constexpr int F64_SCH = 128;  // samples staged per step

template <int CM>
__global__ void __launch_bounds__(F64_TB) fp64_kernel(const uint64_t* __restrict__ x, unsigned long long m,
                                                      int wpk, const double* __restrict__ V, int nsteps,
                                                      const __grid_constant__ EpiParams P, const DevOut O) {
  extern __shared__ __align__(16) double sV[];  // F64_SCH x CM
  const int tid = threadIdx.x;
  for (unsigned long long tile = blockIdx.x; tile * F64_TB < m; tile += gridDim.x) {
    const unsigned long long local = tile * F64_TB + tid;
    const bool valid = local < m;
    const uint64_t* row = x + (valid ? local : 0) * (unsigned long long)wpk;
    double acc[CM];
#pragma unroll
    for (int j = 0; j < CM; ++j) acc[j] = 0.0;
    for (int q = 0; q < nsteps; ++q) {
      __syncthreads();
      const double2* src = reinterpret_cast<const double2*>(V + (size_t)q * F64_SCH * CM);
      double2* dst = reinterpret_cast<double2*>(sV);
      for (int i = tid; i < F64_SCH * CM / 2; i += F64_TB) dst[i] = src[i];
      __syncthreads();
      uint64_t w[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int wi = 2 * q + h;
        w[h] = (valid && wi < wpk) ? __ldg(row + wi) : 0ull;
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint32_t lo = (uint32_t)w[h], hi = (uint32_t)(w[h] >> 32);
#pragma unroll 8
        for (int bb = 0; bb < 64; ++bb) {
          const uint32_t bit = ((bb < 32 ? lo >> bb : hi >> (bb - 32)) & 1u);
          const double xf = __hiloint2double((int)(bit * 0x3FF00000u), 0);  // 1.0 or 0.0
          const double* vr = sV + (h * 64 + bb) * CM;
#pragma unroll
          for (int j = 0; j < CM; ++j) acc[j] = fma(xf, vr[j], acc[j]);
        }
      }
    }
    // column 0 counts the phenotyped samples present (exact: integer sums)
    const int c = (int)acc[0];
    double ss = 0, gs = 0, ey = 0;
#pragma unroll
    for (int j = 1; j < CM; ++j) {
      if (j <= P.k) {
        const double s = P.a[j - 1] * (double)c + acc[j];
        ss += s * s;
        gs += P.g[j - 1] * acc[j];
      } else if (j == P.k + 1) {
        ey = acc[j];
      }
    }
    finish_kmer(P, O, local, valid, c, ss, gs, ey);
  }
}

template <int CM>
static cudaError_t launch_fp64_t(const LaunchFp64& L, cudaStream_t st) {
  const size_t smem = (size_t)F64_SCH * CM * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(fp64_kernel<CM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fp64_kernel<CM>, F64_TB, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  const unsigned long long tiles = (L.m + F64_TB - 1) / F64_TB;
  unsigned long long grid = (unsigned long long)L.num_sms * per_sm;
  if (grid > tiles) grid = tiles;
  if (grid < 1) grid = 1;
  fp64_kernel<CM><<<(unsigned)grid, F64_TB, smem, st>>>(L.x, L.m, L.wpk, L.V, L.nsteps, *L.P, *L.O);
  return cudaGetLastError();
}

int fp64_cm(int C) {
  static const int cms[] = {8, 12, 16, 20, 24, 28, 36, 44, 52, 68};
  for (int cm : cms)
    if (C <= cm) return cm;
  return -1;
}

int fp64_steps(int n) { return (n + F64_SCH - 1) / F64_SCH; }

cudaError_t launch_fp64(const LaunchFp64& L, cudaStream_t st) {
  switch (L.cm) {
    case 8: return launch_fp64_t<8>(L, st);
    case 12: return launch_fp64_t<12>(L, st);
    case 16: return launch_fp64_t<16>(L, st);
    case 20: return launch_fp64_t<20>(L, st);
    case 24: return launch_fp64_t<24>(L, st);
    case 28: return launch_fp64_t<28>(L, st);
    case 36: return launch_fp64_t<36>(L, st);
    case 44: return launch_fp64_t<44>(L, st);
    case 52: return launch_fp64_t<52>(L, st);
    case 68: return launch_fp64_t<68>(L, st);
    default: return cudaErrorInvalidValue;
  }
}

// ====================================================== FP64 refinement pass
// One warp per candidate k-mer (chi-square >= REFINE_CHISQ in the split form):
// the lanes own the FP64 contraction columns (same layout as the FP64 form)
// and sum them over the row's bytes from the byte tables, one coalesced
// table row per byte; lane 0 then evaluates compute_hit
// (src/kgwas.cpp:44-56) in FP64 and emits the row.
template <int CM>
__global__ void __launch_bounds__(256) refine_kernel(const uint64_t* __restrict__ x, int wpk, int nwords,
                                                     const double* __restrict__ T,
                                                     const __grid_constant__ EpiParams P, const DevOut O) {
  const int lane = threadIdx.x & 31;
  const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x >> 5);
  unsigned long long ncand = O.counters[3];
  if (ncand > O.cand_cap) ncand = O.cand_cap;
  for (unsigned long long w = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < ncand;
       w += warps) {
    const unsigned long long g = O.cand[w];
    const uint64_t* row = x + (g - O.kmer_offset) * (unsigned long long)wpk;
    double acc[(CM + 31) / 32];
    table_row_sums<CM>(row, nwords, T, lane, acc);
    int c;
    double ss, ey;
    refine_reduce<CM>(P, acc, lane, c, ss, ey);
    if (lane == 0) {
      const double xxM = (double)c - ss, xyM = P.b * (double)c + ey;
      double effect = 0, Tq = 0, p = 1;
      const double eps = 1e-12;
      if (xxM > eps && P.yyM > eps) {
        double r2 = (xyM * xyM) / (xxM * P.yyM);
        if (r2 < 0) r2 = 0;
        if (r2 >= 1) r2 = 1 - 1e-15;
        Tq = (double)P.n * log(1.0 / (1.0 - r2));
        p = erfc(sqrt(0.5 * Tq));
        effect = xyM / (xxM * P.yyM);
      }
      if (p <= P.p_thresh) {
        const unsigned long long slot = atomicAdd(O.counters + 1, 1ull);
        if (slot < O.hit_cap) {
          kg_hit h;
          h.kmer = g;
          h.effect = effect;
          h.pval = p;
          h.chisq = Tq;
          O.hits[slot] = h;
        } else {
          atomicOr(O.counters + 2, (unsigned long long)ERR_HIT_OVERFLOW);
        }
      }
      if (O.tested) {
        O.chisq[g] = Tq;
        O.pval[g] = p;
        O.effect[g] = effect;
        O.mlog10p[g] = mlog10_sf(Tq);
        O.xxM[g] = xxM;
        O.xyM[g] = xyM;
      }
    }
  }
}

template <int CM>
static cudaError_t launch_refine_t(const LaunchFp64& L, cudaStream_t st) {
  static int per_sm = 0;  // every warp of the grid resident at once (candidates are dealt round-robin)
  if (per_sm < 1 &&
      (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, refine_kernel<CM>, 256, 0) != cudaSuccess || per_sm < 1))
    per_sm = 1;
  const unsigned grid = (unsigned)(L.num_sms * per_sm);
  refine_kernel<CM><<<grid, 256, 0, st>>>(L.x, L.wpk, L.nsteps * F64_SCH / 64, L.T, *L.P, *L.O);
  return cudaGetLastError();
}

cudaError_t launch_refine(const LaunchFp64& L, cudaStream_t st) {
  if (!L.T) return cudaErrorInvalidValue;
  switch (L.cm) {
    case 8: return launch_refine_t<8>(L, st);
    case 12: return launch_refine_t<12>(L, st);
    case 16: return launch_refine_t<16>(L, st);
    case 20: return launch_refine_t<20>(L, st);
    case 24: return launch_refine_t<24>(L, st);
    case 28: return launch_refine_t<28>(L, st);
    case 36: return launch_refine_t<36>(L, st);
    case 44: return launch_refine_t<44>(L, st);
    case 52: return launch_refine_t<52>(L, st);
    case 68: return launch_refine_t<68>(L, st);
    default: return cudaErrorInvalidValue;
  }
}

// Byte tables: one thread per (block, group, byte value, column); the entry
// adds the group's set samples in ascending order.
__global__ void __launch_bounds__(256) refine_table_kernel(const double* __restrict__ V, int cm,
                                                           unsigned long long vstride, unsigned long long total,
                                                           unsigned long long per_block, double* __restrict__ T) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long blk = i / per_block;
    const unsigned long long r = i - blk * per_block;
    const int j = (int)(r % (unsigned)cm);
    const unsigned long long gb = r / (unsigned)cm;
    const unsigned b = (unsigned)(gb & 255u);
    const unsigned long long grp = gb >> 8;
    const double* v = V + blk * vstride + grp * 8ull * (unsigned)cm + j;
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if ((b >> t) & 1u) s += v[(size_t)t * cm];
    T[i] = s;
  }
}

size_t refine_table_len(int vrows, int cm) { return (size_t)(vrows / 8) * 256 * (size_t)cm; }

cudaError_t launch_refine_table(const LaunchTable& L, cudaStream_t st) {
  if (L.vrows % 128 || L.cm <= 0 || L.nblocks <= 0 || !L.V || !L.T) return cudaErrorInvalidValue;
  const unsigned long long tlen = refine_table_len(L.vrows, L.cm);
  const unsigned long long total = tlen * (unsigned long long)L.nblocks;
  unsigned long long blocks = (total + 255) / 256;
  if (blocks > 65535ull * 16) blocks = 65535ull * 16;
  refine_table_kernel<<<(unsigned)blocks, 256, 0, st>>>(L.V, L.cm, L.vstride, total, tlen, L.T);
  return cudaGetLastError();
}

// ============================================== tcgen05 kind::i8, A from SMEM
constexpr int TC_TM = 128;   // k-mers per tile (MMA M)
constexpr int TC_KC = 256;   // samples per K chunk
constexpr int TC_NST = 2;    // pipeline stages

__host__ __device__ constexpr int tmem_cols_for(int N) {
  return N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
}

__host__ __device__ constexpr size_t tc_ss_smem(int N) {
  return (size_t)TC_NST * TC_TM * TC_KC      // A stages
         + (size_t)TC_NST * TC_KC * N        // B stages
         + (size_t)TC_TM * (N + 1) * 4       // accumulator staging for the epilogue
         + 2 * TC_NST * 8 + 16;              // mbarriers + TMEM address
}

// 16 bits -> 16 bytes of 0/1 (sample order preserved).
__device__ __forceinline__ uint4 expand16(uint32_t b) {
  uint4 r;
  r.x = ((b & 0xFu) * 0x00204081u) & 0x01010101u;
  r.y = (((b >> 4) & 0xFu) * 0x00204081u) & 0x01010101u;
  r.z = (((b >> 8) & 0xFu) * 0x00204081u) & 0x01010101u;
  r.w = (((b >> 12) & 0xFu) * 0x00204081u) & 0x01010101u;
  return r;
}

template <int N>
__global__ void __launch_bounds__(TC_TM, 1)
    tc_ss_kernel(const uint64_t* __restrict__ x, unsigned long long m, int wpk, int nchunk,
                 const int8_t* __restrict__ Bimg, const __grid_constant__ EpiParams P,
                 const __grid_constant__ LimbMap LM, const DevOut O) {
  constexpr int TCOLS = tmem_cols_for(N);
  constexpr uint32_t A_BYTES = TC_TM * TC_KC;
  constexpr uint32_t B_BYTES = TC_KC * N;
  constexpr uint32_t IDESC = idesc_i8(TC_TM, N);
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sA = smem;
  uint8_t* sB = sA + TC_NST * A_BYTES;
  int32_t* sD = reinterpret_cast<int32_t*>(sB + TC_NST * B_BYTES);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sD + TC_TM * (N + 1));
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + 2 * TC_NST);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t full0 = smem_u32(bars), done0 = smem_u32(bars + TC_NST);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < TC_NST; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(done0 + 8 * s, 1);
    }
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  uint32_t q = 0;  // chunks issued by this CTA
  int abort = 0;
  for (unsigned long long tile = blockIdx.x; tile * TC_TM < m; tile += gridDim.x) {
    const unsigned long long local = tile * TC_TM + tid;
    const bool valid = local < m;
    const uint64_t* row = x + (valid ? local : 0) * (unsigned long long)wpk;
    for (int kc = 0; kc < nchunk; ++kc, ++q) {
      const uint32_t s = q % TC_NST, u = q / TC_NST;
      bool ok = true;
      if (q >= TC_NST) ok = mbar_wait(done0 + 8 * s, (u - 1) & 1, O.counters, ERR_TIMEOUT_MMA);
      uint8_t* a = sA + s * A_BYTES;
      if (tid == 0 && ok) {
        mbar_arrive_expect_tx(full0 + 8 * s, B_BYTES);
        bulk_g2s(smem_u32(sB + s * B_BYTES), Bimg + (size_t)kc * B_BYTES, B_BYTES, full0 + 8 * s);
      }
      uint64_t w[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int wi = kc * 4 + t;
        w[t] = (valid && wi < wpk) ? __ldg(row + wi) : 0ull;
      }
#pragma unroll
      for (int g = 0; g < 16; ++g) {
        const uint32_t bits = (uint32_t)(w[g >> 2] >> ((g & 3) * 16)) & 0xFFFFu;
        *reinterpret_cast<uint4*>(a + g * (TC_TM * 16) + tid * 16) = expand16(bits);
      }
      fence_proxy_async_smem();
      // The thread that issued the B copy waits for it here, so that no copy
      // is in flight if the block gives up below.
      if (tid == 0 && ok) ok = mbar_wait(full0 + 8 * s, u & 1, O.counters, ERR_TIMEOUT_FULL);
      abort = __syncthreads_or(abort | !ok);
      if (abort) break;
      if (tid == 0) {
        tc_fence_after();
        const uint32_t a_s = smem_u32(a), b_s = smem_u32(sB + s * B_BYTES);
#pragma unroll
        for (int ks = 0; ks < TC_KC / 32; ++ks) {
          const uint64_t ad = sdesc_noswz(a_s + ks * 2 * (TC_TM * 16), TC_TM * 16, 128);
          const uint64_t bd = sdesc_noswz(b_s + ks * 2 * (N * 16), N * 16, 128);
          tc_mma_i8_ss(tmem, ad, bd, IDESC, (kc | ks) != 0);
        }
        tc_commit(done0 + 8 * s);
      }
    }
    if (abort) break;
    const uint32_t sl = (q - 1) % TC_NST, ul = (q - 1) / TC_NST;
    const bool ok = mbar_wait(done0 + 8 * sl, ul & 1, O.counters, ERR_TIMEOUT_MMA);
    tc_fence_after();
    if (ok) {
#pragma unroll
      for (int c16 = 0; c16 < N / 16; ++c16) {
        uint32_t r[16];
        tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c16 * 16, r);
        tc_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) sD[tid * (N + 1) + c16 * 16 + i] = (int32_t)r[i];
      }
    }
    tc_fence_before();
    abort = __syncthreads_or(!ok);
    if (abort) break;
    const int32_t* d = sD + tid * (N + 1);
    const int c = d[LM.count_col];
    double ss = 0, gs = 0, ey = 0;
    for (int j = 0; j <= P.k; ++j) {
      long long v = 0;
      for (int l = 0; l < LM.nl[j]; ++l) v = v * 256 + (long long)d[LM.first[j] + l];
      const double e = (double)v * LM.scale[j];
      if (j < P.k) {
        const double sj = fma(P.a[j], (double)c, e);
        ss = fma(sj, sj, ss);
        gs = fma(P.g[j], e, gs);
      } else {
        ey = e;
      }
    }
    finish_kmer(P, O, local, valid, c, ss, gs, ey);
  }
  // Drain: every MMA this CTA issued has been committed to a done barrier;
  // wait (bounded) for the most recent one before releasing TMEM.
  __syncthreads();
  if (tid == 0 && q > 0) {
    const uint32_t sl = (q - 1) % TC_NST, ul = (q - 1) / TC_NST;
    mbar_wait(done0 + 8 * sl, ul & 1, O.counters, ERR_TIMEOUT_MMA);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
}

template <int N>
static cudaError_t launch_tc_ss_t(const LaunchTc& L, cudaStream_t st) {
  const size_t smem = tc_ss_smem(N);
  cudaError_t e = cudaFuncSetAttribute(tc_ss_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const unsigned long long tiles = (L.m + TC_TM - 1) / TC_TM;
  unsigned long long grid = (unsigned long long)L.num_sms;
  if (grid > tiles) grid = tiles;
  if (grid < 1) grid = 1;
  tc_ss_kernel<N><<<(unsigned)grid, TC_TM, smem, st>>>(L.x, L.m, L.wpk, L.nchunk, L.Bimg, *L.P, *L.LM, *L.O);
  return cudaGetLastError();
}

int tc_kc() { return TC_KC; }

bool tc_supported_n(int N) { return N == 16 || N == 32 || N == 48 || N == 64 || N == 80 || N == 96 || N == 112 || N == 128; }

cudaError_t launch_tc(const LaunchTc& L, cudaStream_t st) {
  switch (L.LM->N) {
    case 16: return launch_tc_ss_t<16>(L, st);
    case 32: return launch_tc_ss_t<32>(L, st);
    case 48: return launch_tc_ss_t<48>(L, st);
    case 64: return launch_tc_ss_t<64>(L, st);
    case 80: return launch_tc_ss_t<80>(L, st);
    case 96: return launch_tc_ss_t<96>(L, st);
    case 112: return launch_tc_ss_t<112>(L, st);
    case 128: return launch_tc_ss_t<128>(L, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kg
