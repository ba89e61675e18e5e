// kernel_ts.cu -- split-precision association kernel with the unpacked x
// operand held in tensor memory.
//
// One persistent CTA per SM, warp-specialised (448 threads):
//   warps 0-3   epilogue: tcgen05.ld of the int32 accumulators (one TMEM lane
//               = one k-mer), limb recombination, FP64 statistics,
//               warp-aggregated hit compaction;
//   warps 4-11  unpack, two groups of four (one warp per TMEM lane quarter),
//               the groups taking K stages in turn so that two stores to
//               tensor memory are in flight per lane quarter:
//               read 128 samples of a packed row from the TMA-filled shared
//               tile and write them as int8 (0 / -128) straight into a TMEM
//               A stage with tcgen05.st -- the unpacked operand never touches
//               shared memory;
//   warp 12     producer: one 2-D TMA load (128 rows x 128 bytes, 128-byte
//               swizzle, no multicast) per 1024 samples of a 128-k-mer tile;
//   warp 13     MMA: tcgen05.mma kind::i8, A from TMEM, B (the int8 limbs of
//               the centred structure and phenotype columns, resident in
//               shared memory for the whole launch) from a smem descriptor,
//               accumulating into one of two TMEM accumulators.
// Tile = 128 k-mers (M), K stage = 128 samples (32 TMEM columns), N = 16..128.
// TMEM (512 columns): NBUF accumulator buffers of S split-K accumulators of
// N columns each, then the A stages.  K stage kc accumulates into split
// kc % S, so S independent MMA chains are in flight instead of one serial
// chain of K/32 dependent accumulations; the epilogue adds the S int32
// partial sums (exact).
//
// The accumulators hold -128 * sum_i x_i * digit_l(i) for every limb l; the
// epilogue recombines the limbs exactly in int64, scales by 2^-s / 128, and
// evaluates the reference's statistic (src/kgwas.cpp:44-56, 182-218) in FP64.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdio>
#include <cstdlib>

#include "device.cuh"
#include "kernels.hpp"

namespace kg {

constexpr int TS_TM = 128;
constexpr int TS_KS = 128;         // samples per A stage
constexpr int TS_BOX = 1024;       // samples per TMA box (128 bytes)
constexpr int TS_XST = 4;          // packed boxes in flight
constexpr int TS_UG = 2;           // unpack groups
constexpr int TS_THREADS = 32 * (4 + 4 * TS_UG + 2);
constexpr int TS_LU = 3, TS_LY = 5;
constexpr uint32_t TS_XBYTES = TS_TM * 128;  // one box: 128 rows x 128 bytes
constexpr int TS_WARP_UNPACK0 = 4, TS_WARP_PROD = 4 + 4 * TS_UG, TS_WARP_MMA = TS_WARP_PROD + 1;

__host__ __device__ constexpr int ts_a0(int N, int S, int NB) { return ((NB * S * N + 31) / 32) * 32; }
__host__ __device__ constexpr int ts_ast(int N, int S, int NB) {
  return (512 - ts_a0(N, S, NB)) / 32 > 16 ? 16 : (512 - ts_a0(N, S, NB)) / 32;
}

struct TsSmem {  // offsets from the 1024-aligned base
  uint32_t x, b, bars, tmem, abort, total;
};
__host__ __device__ inline TsSmem ts_smem(int b_bytes) {
  TsSmem L;
  L.x = 0;
  L.b = TS_XST * TS_XBYTES;
  L.bars = L.b + ((b_bytes + 127) / 128) * 128;
  L.tmem = L.bars + 8 * (2 * TS_XST + 2 * 16 + 4 + 2);
  L.abort = L.tmem + 8;
  L.total = L.abort + 8;
  return L;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void* tmap, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(tmap), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tc_st32(uint32_t taddr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]),
      "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]),
      "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
}

// Bounded wait that also gives up when another role has aborted.
__device__ __forceinline__ bool ts_wait(uint32_t bar, uint32_t parity, volatile int* abort,
                                        unsigned long long* counters, unsigned code) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtimer_ns();
  for (;;) {
    if (mbar_try(bar, parity)) return true;
    if (*abort) return false;
    if (gtimer_ns() - t0 > WAIT_LIMIT_NS) {
      atomicOr(counters + 2, (unsigned long long)code);
      *abort = 1;
      return false;
    }
  }
}

template <int N, bool DROP0>
__global__ void __launch_bounds__(TS_THREADS, 1)
    ts_kernel(const __grid_constant__ CUtensorMap tmap, unsigned long long m, int nbox, int nchunk,
              const int8_t* __restrict__ Bimg, int b_bytes, int S, int NB, const __grid_constant__ EpiParams P,
              const __grid_constant__ LimbMap LM, const DevOut O) {
  const int A0 = ts_a0(N, S, NB);
  const int AST = ts_ast(N, S, NB);
  constexpr uint32_t IDESC = idesc_i8(TS_TM, N);
  constexpr int KU_MAX = (N - 1 - TS_LY) / TS_LU;  // U columns that fit in N
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gbase = smem_raw + (base - raw);
  const TsSmem L = ts_smem(b_bytes);
  const uint32_t sx = base + L.x, sb = base + L.b;
  const uint32_t x_full = base + L.bars, x_empty = x_full + 8 * TS_XST;
  const uint32_t a_full = x_empty + 8 * TS_XST, a_empty = a_full + 8 * 16;
  const uint32_t acc_full = a_empty + 8 * 16, acc_empty = acc_full + 16, b_full = acc_empty + 16;
  const uint32_t drain = b_full + 8;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(gbase + L.tmem);
  volatile int* s_abort = reinterpret_cast<volatile int*>(gbase + L.abort);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < TS_XST; ++s) {
      mbar_init(x_full + 8 * s, 1);
      mbar_init(x_empty + 8 * s, 4 * TS_UG);  // every unpack warp
    }
    for (int t = 0; t < AST; ++t) {
      mbar_init(a_full + 8 * t, 4);   // the 4 warps of one unpack group
      mbar_init(a_empty + 8 * t, 1);  // tcgen05.commit
    }
    for (int b = 0; b < NB; ++b) {
      mbar_init(acc_full + 8 * b, 1);
      mbar_init(acc_empty + 8 * b, 4);
    }
    mbar_init(b_full, 1);
    mbar_init(drain, 1);
    *s_abort = 0;
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const unsigned long long ntiles = (m + TS_TM - 1) / TS_TM;

  if (warp == TS_WARP_PROD) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(&tmap) : "memory");
      mbar_arrive_expect_tx(b_full, (uint32_t)b_bytes);
      for (int off = 0; off < b_bytes; off += 32768) {
        const int len = b_bytes - off < 32768 ? b_bytes - off : 32768;
        bulk_g2s(sb + off, Bimg + off, (uint32_t)len, b_full);
      }
      uint32_t h = 0;
      uint32_t last_use[TS_XST];
      for (int s = 0; s < TS_XST; ++s) last_use[s] = 0xffffffffu;
      bool ok = true;
      for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        for (int bx = 0; bx < nbox; ++bx, ++h) {
          const uint32_t s = h % TS_XST, u = h / TS_XST;
          if (u > 0 && !ts_wait(x_empty + 8 * s, (u - 1) & 1, s_abort, O.counters, ERR_TIMEOUT_FULL)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(x_full + 8 * s, TS_XBYTES);
          tma_load_2d(sx + s * TS_XBYTES, &tmap, bx * 128, (int)(tile * TS_TM), x_full + 8 * s);
          last_use[s] = u;
        }
      }
      // no copy may still be landing when the block exits
      mbar_wait(b_full, 0, O.counters, ERR_TIMEOUT_FULL);
      for (int s = 0; s < TS_XST; ++s)
        if (last_use[s] != 0xffffffffu) mbar_wait(x_full + 8 * s, last_use[s] & 1, O.counters, ERR_TIMEOUT_FULL);
    }
  } else if (warp == TS_WARP_MMA) {
    // ----------------------------------------------------------------- MMA
    if (lane == 0) {
      bool ok = ts_wait(b_full, 0, s_abort, O.counters, ERR_TIMEOUT_FULL);
      uint32_t g = 0, i = 0;
      for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++i) {
        const uint32_t b = i % NB, v = i / NB;
        if (v > 0 && !ts_wait(acc_empty + 8 * b, (v - 1) & 1, s_abort, O.counters, ERR_TIMEOUT_MMA)) {
          ok = false;
          break;
        }
        tc_fence_after();
        for (int kc = 0; kc < nchunk; ++kc, ++g) {
          const uint32_t t = g % AST, u = g / AST;
          if (!ts_wait(a_full + 8 * t, u & 1, s_abort, O.counters, ERR_TIMEOUT_MMA)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_t = tmem + (b * S + kc % S) * N;  // split-K accumulator of this stage
#pragma unroll
          for (int ks = 0; ks < TS_KS / 32; ++ks) {
            const uint32_t a_t = tmem + A0 + t * 32 + ks * 8;
            const uint64_t bd = sdesc_noswz(sb + ((kc * TS_KS + ks * 32) / 16) * (N * 16), N * 16, 128);
            tc_mma_i8_ts(d_t, a_t, bd, IDESC, (kc >= S || ks != 0) ? 1u : 0u);
          }
          tc_commit(a_empty + 8 * t);
        }
        if (!ok) break;
        tc_commit(acc_full + 8 * b);
      }
      // drain: wait (bounded) until every issued MMA has completed
      tc_commit(drain);
      mbar_wait(drain, 0, O.counters, ERR_TIMEOUT_MMA);
    }
  } else if (warp >= TS_WARP_UNPACK0) {
    // -------------------------------------------------------------- unpack
    const int grp = (warp - TS_WARP_UNPACK0) >> 2;  // 0 .. TS_UG-1
    const int q = warp & 3;                    // TMEM lane quarter
    const int r = q * 32 + lane;               // row of the tile = TMEM lane
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    uint32_t g = 0, h = 0;
    bool ok = true;
    for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
      for (int bx = 0; bx < nbox && ok; ++bx, ++h) {
        const uint32_t s = h % TS_XST;
        if (!__all_sync(0xffffffffu, ts_wait(x_full + 8 * s, (h / TS_XST) & 1, s_abort, O.counters,
                                            ERR_TIMEOUT_FULL))) {
          ok = false;
          break;
        }
        const int kc0 = bx * (TS_BOX / TS_KS);
        const int kc1 = kc0 + TS_BOX / TS_KS < nchunk ? kc0 + TS_BOX / TS_KS : nchunk;
        for (int kc = kc0; kc < kc1; ++kc, ++g) {
          if ((int)(g % TS_UG) != grp) continue;
          const uint32_t t = g % AST, u = g / AST;
          if (u > 0 && !__all_sync(0xffffffffu, ts_wait(a_empty + 8 * t, (u - 1) & 1, s_abort, O.counters,
                                                        ERR_TIMEOUT_MMA))) {
            ok = false;
            break;
          }
          // 16 bytes (128 samples) of row r; 128-byte swizzle: chunk c of row r sits at c ^ (r % 8)
          const int c = kc - kc0;
          uint4 v;
          asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];"
                       : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                       : "r"(sx + s * TS_XBYTES + r * 128 + ((c ^ (r & 7)) << 4)));
          const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
          uint32_t o[32];
          // byte t of column 8qq+j = bit 8t+j of word qq, moved to the byte's
          // sign bit (0 or -128); the shift is a multiply so that it issues on
          // the FMA pipe and the mask on the ALU pipe
#pragma unroll
          for (int qq = 0; qq < 4; ++qq)
#pragma unroll
            for (int j = 0; j < 8; ++j) o[qq * 8 + j] = (w4[qq] * (1u << (7 - j))) & 0x80808080u;
          tc_st32(tmem + lane_base + A0 + t * 32, o);
          tc_wait_st();
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(a_full + 8 * t);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(x_empty + 8 * s);
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    uint32_t i = 0;
    const int nsplit = nchunk < S ? nchunk : S;  // splits that received a stage
    for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
      const uint32_t b = i % NB, v = i / NB;
      if (!__all_sync(0xffffffffu, ts_wait(acc_full + 8 * b, v & 1, s_abort, O.counters, ERR_TIMEOUT_MMA))) break;
      tc_fence_after();
      // sum the split-K partial accumulators, 16 columns at a time; every
      // tcgen05.ld completes (wait::ld) before its registers are used
      uint32_t d[N];
#pragma unroll
      for (int c16 = 0; c16 < N / 16; ++c16) {
        uint32_t rr[16];
        tc_ld16(tmem + lane_base + b * S * N + c16 * 16, rr);
        tc_wait_ld();
#pragma unroll
        for (int e = 0; e < 16; ++e) d[c16 * 16 + e] = rr[e];
        for (int sp = 1; sp < nsplit; ++sp) {
          tc_ld16(tmem + lane_base + (b * S + sp) * N + c16 * 16, rr);
          tc_wait_ld();
#pragma unroll
          for (int e = 0; e < 16; ++e) d[c16 * 16 + e] += rr[e];
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty + 8 * b);
      const unsigned long long local = tile * TS_TM + r;
      const bool valid = local < m;
      // accumulators hold -128 * (integer limb sums): divide the 128 out in
      // integers (exact), then recombine the limbs in FP64 (exact: the value
      // stays below 2^53), so the result equals the smem-A kernel's bit for bit
      const int c = (-(int)d[0]) >> 7;
      double vy = (double)((-(int)d[1]) >> 7);
#pragma unroll
      for (int l = 1; l < TS_LY; ++l) vy = fma(vy, 256.0, (double)((-(int)d[1 + l]) >> 7));
      const double ey = vy * LM.scale[P.k];
      double ss = 0, gs = 0;
      if (DROP0) {
        const double s0 = P.a[0] * (double)c;
        ss = s0 * s0;
      }
#pragma unroll
      for (int jj = 0; jj < KU_MAX; ++jj) {
        const int j = jj + (DROP0 ? 1 : 0);
        if (j < P.k) {
          const int o = 1 + TS_LY + TS_LU * jj;
          double vj = (double)((-(int)d[o]) >> 7);
#pragma unroll
          for (int l = 1; l < TS_LU; ++l) vj = fma(vj, 256.0, (double)((-(int)d[o + l]) >> 7));
          const double e = vj * LM.scale[j];
          const double sj = fma(P.a[j], (double)c, e);
          ss = fma(sj, sj, ss);
          gs = fma(P.g[j], e, gs);
        }
      }
      if (O.tested) finish_kmer(P, O, local, valid, c, ss, gs, ey);
      else finish_kmer_fast(P, O, local, valid, c, ss, gs, ey);
    }
  }
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// ------------------------------------------------------------------- host

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

// Split-K accumulators and accumulator buffers for width N (KG_TS_SPLIT=
// "S,NB" overrides).
static void ts_shape(int N, int& S, int& NB) {
  // measured on the 200M-k-mer workload: one chain, two buffers is fastest
  S = 1;
  NB = 2;
  if (const char* v = std::getenv("KG_TS_SPLIT")) {
    int s = 0, b = 0;
    if (std::sscanf(v, "%d,%d", &s, &b) == 2 && s >= 1 && s <= 8 && b >= 1 && b <= 2 &&
        ts_ast(N, s, b) >= 4)
      S = s, NB = b;
  }
}

bool ts_supported(int N, int limbs_u, int limbs_y, int kpad, int wpk) {
  if (limbs_u != TS_LU || limbs_y != TS_LY) return false;
  if (N < 16 || N > 128 || N % 16) return false;
  int S, NB;
  ts_shape(N, S, NB);
  if (ts_ast(N, S, NB) < 4) return false;
  if ((size_t)kpad * N > 128 * 1024) return false;  // B stays resident in shared memory
  if (wpk * 8 < 128) return false;                   // one TMA box row is 128 bytes
  return encode_fn() != nullptr;
}

template <int N, bool D0>
static cudaError_t launch_ts_t(const LaunchTs& L, const CUtensorMap& tm, cudaStream_t st) {
  const int b_bytes = L.kpad * N;
  const size_t smem = ts_smem(b_bytes).total + 1024;
  cudaError_t e = cudaFuncSetAttribute(ts_kernel<N, D0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const unsigned long long tiles = (L.m + TS_TM - 1) / TS_TM;
  unsigned long long grid = (unsigned long long)L.num_sms;
  if (grid > tiles) grid = tiles;
  const int nbox = (L.wpk * 8 + 127) / 128;
  const int nchunk = L.kpad / TS_KS;
  int S, NB;
  ts_shape(N, S, NB);
  ts_kernel<N, D0><<<(unsigned)grid, TS_THREADS, smem, st>>>(tm, L.m, nbox, nchunk, L.Bimg, b_bytes, S, NB,
                                                             *L.P, *L.LM, *L.O);
  return cudaGetLastError();
}

cudaError_t launch_ts(const LaunchTs& L, cudaStream_t st) {
  auto enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  CUtensorMap tm;
  const cuuint64_t rowbytes = (cuuint64_t)L.wpk * 8;
  cuuint64_t gdim[2] = {rowbytes, (cuuint64_t)L.m};
  cuuint64_t gstride[1] = {rowbytes};
  cuuint32_t box[2] = {128, TS_TM};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)L.x, gdim, gstride, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  const bool d0 = L.drop0;
  switch (L.LM->N) {
#define KG_TS_CASE(NN) \
  case NN: return d0 ? launch_ts_t<NN, true>(L, tm, st) : launch_ts_t<NN, false>(L, tm, st);
    KG_TS_CASE(16)
    KG_TS_CASE(32)
    KG_TS_CASE(48)
    KG_TS_CASE(64)
    KG_TS_CASE(80)
    KG_TS_CASE(96)
    KG_TS_CASE(112)
    KG_TS_CASE(128)
#undef KG_TS_CASE
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kg
