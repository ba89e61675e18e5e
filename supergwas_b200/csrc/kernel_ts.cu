// kernel_ts.cu -- split-precision association kernel with the unpacked x
// operand held in tensor memory.
//
// One persistent CTA per SM, warp-specialised (576 threads; 448 for N > 80):
//   warps 0-7   epilogue, two groups of four (one warp per TMEM lane quarter),
//               group e owning accumulator buffer e, i.e. every other tile:
//               tcgen05.ld of the int32 accumulators (one TMEM lane = one
//               k-mer), exact limb recombination, FP64 statistics,
//               warp-aggregated hit compaction;
//   warps 8-15  unpack, two groups of four taking super-stages in turn (one
//               group for N > 80, so that the epilogue keeps its registers): read
//               128 samples of a packed row from the TMA-filled shared tile
//               and write them as int8 (0 / -128, or 0 / 64 against -2x the
//               B digits) straight into a TMEM A slot with tcgen05.st -- the
//               unpacked operand never touches shared memory;
//   warp 16     producer (12 for N > 80): one 2-D TMA load (128 rows x 128 bytes, 128-byte
//               swizzle, no multicast) per 1024 samples of a 128-k-mer tile;
//   warp 17     MMA (13 for N > 80): tcgen05.mma kind::i8, A from TMEM, B (the int8 limbs of
//               the centred structure and phenotype columns, resident in
//               shared memory for the whole launch) from a smem descriptor.
// Tile = 128 k-mers (M), N = 16..128 limb columns.
//
// The MMA-issuing thread is the critical path: on B200 a kind::i8 M=128
// N=64 K=32 MMA occupies the tensor pipe 32 cycles (16384 int8 ops per SM
// cycle), and every barrier test, commit or runtime division between MMAs
// adds its latency on top.  So the
// A operand moves in super-stages of 512 samples (4 sub-stages of 128
// samples = 128 TMEM columns = 16 MMAs) with one barrier wait and one
// commit each, and every ring index is a compile-time-bounded counter.
// TMEM (512 columns): two accumulators of N columns, then NSLOT super-slots.
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
constexpr int TS_KS = 128;         // samples per sub-stage (32 TMEM columns, 4 MMAs)
constexpr int TS_SUPER = 4;        // sub-stages per super-stage (one barrier, one commit)
constexpr int TS_BOX = 1024;       // samples per TMA box (128 bytes)
// Packed boxes in flight: as many as the shared memory left by the B image
// holds, up to TS_XST_MAX (chosen at launch).  HBM latency under this load is
// ~2 us, so 4 boxes (64 KB per SM) cap the row stream near 4.3 TB/s.
constexpr int TS_XST_MAX = 12;
// Unpack groups (taking super-stages in turn): two while the epilogue fits
// the register budget of 18 warps, one for wide N.
__host__ __device__ constexpr int ts_ug(int N) { return N <= 80 ? 2 : 1; }
__host__ __device__ constexpr int ts_threads(int N) { return 32 * (8 + 4 * ts_ug(N) + 2); }
constexpr int TS_LU = 3, TS_LY = 5;
constexpr uint32_t TS_XBYTES = TS_TM * 128;  // one box: 128 rows x 128 bytes
constexpr int TS_WARP_UNPACK0 = 8;  // then the unpack groups, the producer, the MMA warp
constexpr int TS_MAXSLOT = 3;

// Super-slots of 128 TMEM columns left after the two N-column accumulators.
__host__ __device__ constexpr int ts_nslot(int N) {
  return (512 - 2 * N) / 128 > TS_MAXSLOT ? TS_MAXSLOT : (512 - 2 * N) / 128;
}

struct TsSmem {  // offsets from the 1024-aligned base
  uint32_t x, b, bars, tmem, abort, total;
};
__host__ __device__ inline TsSmem ts_smem(int b_bytes, int xst) {
  TsSmem L;
  L.x = 0;
  L.b = xst * TS_XBYTES;
  L.bars = L.b + ((b_bytes + 127) / 128) * 128;
  L.tmem = L.bars + 8 * (2 * TS_XST_MAX + 2 * TS_MAXSLOT + 4 + 2);
  L.abort = L.tmem + 8;
  L.total = L.abort + 8;
  return L;
}

template <int N, bool DROP0, bool GATE>
__global__ void __launch_bounds__(ts_threads(N), 1)
    ts_kernel(const __grid_constant__ CUtensorMap tmap, unsigned long long m, int nbox, int nsub, int xst,
              const int8_t* __restrict__ Bimg, int b_bytes, const __grid_constant__ EpiParams P,
              const __grid_constant__ LimbMap LM, const DevOut O) {
  constexpr int UG = ts_ug(N);
  constexpr int TS_WARP_PROD = TS_WARP_UNPACK0 + 4 * UG, TS_WARP_MMA = TS_WARP_PROD + 1;
  constexpr int NSLOT = ts_nslot(N);
  constexpr int A0 = 512 - NSLOT * 128;  // first A column (>= 2N)
  static_assert(NSLOT >= 2 && A0 >= 2 * N, "TMEM budget");
  constexpr uint32_t IDESC = idesc_i8(TS_TM, N);
  constexpr int KU_MAX = (N - 1 - TS_LY) / TS_LU;  // U columns that fit in N
  constexpr uint32_t BSTEP = (2 * N * 16) >> 4;    // descriptor step of one K=32 MMA
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gbase = smem_raw + (base - raw);
  const TsSmem L = ts_smem(b_bytes, xst);
  const uint32_t sx = base + L.x, sb = base + L.b;
  const uint32_t x_full = base + L.bars, x_empty = x_full + 8 * TS_XST_MAX;
  const uint32_t a_full = x_empty + 8 * TS_XST_MAX, a_empty = a_full + 8 * TS_MAXSLOT;
  const uint32_t acc_full = a_empty + 8 * TS_MAXSLOT, acc_empty = acc_full + 16, b_full = acc_empty + 16;
  const uint32_t drain = b_full + 8;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(gbase + L.tmem);
  volatile int* s_abort = reinterpret_cast<volatile int*>(gbase + L.abort);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nsp = (nsub + TS_SUPER - 1) / TS_SUPER;  // super-stages per tile

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < xst; ++s) {
      mbar_init(x_full + 8 * s, 1);
      mbar_init(x_empty + 8 * s, 4 * UG);  // every unpack warp
    }
    for (int t = 0; t < NSLOT; ++t) {
      mbar_init(a_full + 8 * t, 4);   // the four warps of one unpack group
      mbar_init(a_empty + 8 * t, 1);  // tcgen05.commit
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full + 8 * b, 1);
      mbar_init(acc_empty + 8 * b, 4);  // the four warps of epilogue group b
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
  const unsigned long long lim = wait_limit(O.wait_ns);

  if (warp == TS_WARP_PROD) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(&tmap) : "memory");
      mbar_arrive_expect_tx(b_full, (uint32_t)b_bytes);
      for (int off = 0; off < b_bytes; off += 32768) {
        const int len = b_bytes - off < 32768 ? b_bytes - off : 32768;
        bulk_g2s(sb + off, Bimg + off, (uint32_t)len, b_full);
      }
      RingN xr(xst);
      uint32_t last_phase[TS_XST_MAX];
      bool issued[TS_XST_MAX];
      for (int s = 0; s < TS_XST_MAX; ++s) issued[s] = false, last_phase[s] = 0;
      bool ok = true;
      unsigned long long loads = 0;
      for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        for (int bx = 0; bx < nbox; ++bx, xr.next()) {
          if (xr.used && !wait_or_abort(x_empty + 8 * xr.slot, xr.phase ^ 1u, s_abort, O.counters, ERR_TIMEOUT_FULL, lim)) {
            ok = false;
            break;
          }
          if (O.stall_loads && loads++ == O.stall_loads) {  // test hook: stop feeding the pipeline
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(x_full + 8 * xr.slot, TS_XBYTES);
          tma_load_2d(sx + xr.slot * TS_XBYTES, &tmap, bx * 128, (int)(tile * TS_TM), x_full + 8 * xr.slot);
          issued[xr.slot] = true;
          last_phase[xr.slot] = xr.phase;
        }
      }
      // no copy may still be landing when the block exits
      mbar_wait(b_full, 0, O.counters, ERR_TIMEOUT_FULL);
      for (int s = 0; s < xst; ++s)
        if (issued[s]) mbar_wait(x_full + 8 * s, last_phase[s], O.counters, ERR_TIMEOUT_FULL);
    }
  } else if (warp == TS_WARP_MMA) {
    // ----------------------------------------------------------------- MMA
    // The whole warp runs the loop (warp-uniform control flow and operands);
    // one elected lane issues the MMAs and the commits that track them.
    const bool leader = elect_one();
    bool ok = __all_sync(0xffffffffu, wait_or_abort(b_full, 0, s_abort, O.counters, ERR_TIMEOUT_FULL, lim));
    const uint64_t bdesc0 = sdesc_noswz(sb, N * 16, 128);
    Ring<NSLOT> ar;
    uint32_t i = 0;
    for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++i) {
      const uint32_t b = i & 1u;
      if (i >= 2 && !__all_sync(0xffffffffu, wait_or_abort(acc_empty + 8 * b, ((i >> 1) - 1) & 1u, s_abort, O.counters,
                                                     ERR_TIMEOUT_MMA, lim))) {
        ok = false;
        break;
      }
      const uint32_t d_t = tmem + b * N;
      uint64_t bd = bdesc0;
      for (int sp = 0; sp < nsp; ++sp, ar.next()) {
        if (!__all_sync(0xffffffffu, wait_or_abort(a_full + 8 * ar.slot, ar.phase, s_abort, O.counters, ERR_TIMEOUT_MMA, lim))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const int nsub_here = nsub - sp * TS_SUPER < TS_SUPER ? nsub - sp * TS_SUPER : TS_SUPER;
        const uint32_t a_t = tmem + A0 + ar.slot * 128;
        if (leader) {
          if (nsub_here == TS_SUPER) {
            // full super-stage: 16 MMAs with compile-time operand offsets
#pragma unroll
            for (int k = 0; k < TS_SUPER * (TS_KS / 32); ++k)
              tc_mma_i8_ts(d_t, a_t + k * 8, bd + (uint64_t)(k * BSTEP), IDESC, (sp | k) ? 1u : 0u);
          } else {
            uint64_t bk = bd;
            for (int sub = 0; sub < nsub_here; ++sub) {
#pragma unroll
              for (int ks = 0; ks < TS_KS / 32; ++ks) {
                tc_mma_i8_ts(d_t, a_t + sub * 32 + ks * 8, bk, IDESC, (sp | sub | ks) ? 1u : 0u);
                bk += BSTEP;
              }
            }
          }
          tc_commit(a_empty + 8 * ar.slot);
        }
        __syncwarp();
        bd += (uint64_t)(TS_SUPER * (TS_KS / 32) * BSTEP);
      }
      if (!ok) break;
      if (leader) tc_commit(acc_full + 8 * b);
      __syncwarp();
    }
    // drain: wait (bounded) until every issued MMA has completed
    if (leader) {
      tc_commit(drain);
      mbar_wait(drain, 0, O.counters, ERR_TIMEOUT_MMA);
    }
    __syncwarp();
  } else if (warp >= TS_WARP_UNPACK0) {
    // -------------------------------------------------------------- unpack
    const int grp = (warp - TS_WARP_UNPACK0) >> 2;  // takes every other super-stage
    const int q = warp & 3;                         // TMEM lane quarter
    const int r = q * 32 + lane;                    // row of the tile = TMEM lane
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    RingN xr(xst);
    Ring<NSLOT> ar;
    uint32_t turn = 0;  // super-stage counter modulo UG
    bool ok = true;
    for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
      int kc = 0;  // sub-stage of the tile
      for (int bx = 0; bx < nbox && ok; ++bx, xr.next()) {
        // every unpack warp waits for every box, also one holding none of its
        // super-stages, so that its release below belongs to this fill
        if (!__all_sync(0xffffffffu, wait_or_abort(x_full + 8 * xr.slot, xr.phase, s_abort, O.counters,
                                            ERR_TIMEOUT_FULL, lim))) {
          ok = false;
          break;
        }
        const int kc1 = (bx + 1) * (TS_BOX / TS_KS) < nsub ? (bx + 1) * (TS_BOX / TS_KS) : nsub;
        // super-stages never straddle a box: a box holds two of them
        while (kc < kc1) {
          const int ke = kc + TS_SUPER < kc1 ? kc + TS_SUPER : kc1;
          if (UG > 1 && turn != (uint32_t)grp) {  // another group's super-stage
            kc = ke;
            ar.next();
            turn = turn + 1 == (uint32_t)UG ? 0u : turn + 1;
            continue;
          }
          if (ar.used && !__all_sync(0xffffffffu, wait_or_abort(a_empty + 8 * ar.slot, ar.phase ^ 1u, s_abort,
                                                          O.counters, ERR_TIMEOUT_MMA, lim))) {
            ok = false;
            break;
          }
          const uint32_t xrow = sx + xr.slot * TS_XBYTES + r * 128;
          const uint32_t a_t = tmem + lane_base + A0 + ar.slot * 128;
          const int c0 = kc - bx * (TS_BOX / TS_KS);
          // 16 bytes (128 samples) of row r per sub-stage; 128-byte swizzle:
          // chunk c of row r sits at c ^ (r % 8).  Column 8qq+jj of a stage =
          // word qq shifted left by 2*(jj/2), masked to bit 7 (jj even: byte t
          // holds sample 8t+7-jj as 0 / -128) or bit 6 (jj odd: 0 / 64; the B
          // image holds -2 V there), so one shift serves two columns.  The
          // shift is a multiply so that it issues on the FMA pipe and the
          // masks on the ALU pipe.
          if (ke - kc == TS_SUPER) {
            uint32_t w[TS_SUPER][4];
#pragma unroll
            for (int sub = 0; sub < TS_SUPER; ++sub)
              asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];"
                           : "=r"(w[sub][0]), "=r"(w[sub][1]), "=r"(w[sub][2]), "=r"(w[sub][3])
                           : "r"(xrow + (((c0 + sub) ^ (r & 7)) << 4)));
#pragma unroll
            for (int sub = 0; sub < TS_SUPER; ++sub) {
              uint32_t o[32];
              unpack_stage(w[sub], o);
              tc_st32(a_t + sub * 32, o);
            }
          } else {
            for (int sub = 0; sub < ke - kc; ++sub) {
              uint4 v;
              asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];"
                           : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                           : "r"(xrow + (((c0 + sub) ^ (r & 7)) << 4)));
              const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
              uint32_t o[32];
              unpack_stage(w4, o);
              tc_st32(a_t + sub * 32, o);
            }
          }
          kc = ke;
          tc_wait_st();
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(a_full + 8 * ar.slot);
          ar.next();
          if (UG > 1) turn = turn + 1 == (uint32_t)UG ? 0u : turn + 1;
        }
        if (!ok) break;
        // every unpack warp releases every box, whether or not it read from it
        __syncwarp();
        if (lane == 0) mbar_arrive(x_empty + 8 * xr.slot);
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int e = warp >> 2;  // group = accumulator buffer
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    uint32_t jt = 0;            // tiles taken by this group
    uint32_t tested_local = 0;  // k-mers this thread tested (lean path)
    for (unsigned long long tile = blockIdx.x + (unsigned long long)e * gridDim.x; tile < ntiles;
         tile += 2ull * gridDim.x, ++jt) {
      if (!__all_sync(0xffffffffu, wait_or_abort(acc_full + 8 * e, jt & 1u, s_abort, O.counters, ERR_TIMEOUT_MMA, lim))) break;
      tc_fence_after();
      // all N columns in flight at once, then one wait
      uint32_t d[N];
#pragma unroll
      for (int c16 = 0; c16 < N / 16; ++c16) tc_ld16p(tmem + lane_base + e * N + c16 * 16, d + c16 * 16);
      tc_wait_ld();
#pragma unroll
      for (int c16 = 0; c16 < N / 16; ++c16) reg_fence16(d + c16 * 16);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty + 8 * e);
      const unsigned long long local = tile * TS_TM + r;
      const bool valid = local < m;
      // accumulators hold -128 * (integer limb sums).  The limbs are
      // recombined exactly in int64 and turned into doubles with the
      // bias trick (integer add + one FMA, no conversion instructions):
      //   U column: V = sum_l 256^(L-1-l) d_l = -128 v, |V| < 2^41, and
      //   e = V * (-scale/128) = v * scale, exact (LimbMap esc/eoff);
      //   y':       |V| < 2^57, so v = -V >> 7 (exact) first.
      // The values equal those of the smem-A kernel bit for bit.
      // Each partial sum below is one 32 x 32 -> 64-bit multiply-add (the
      // limb sums are int32, |d| <= 2^24).
      const int c = (-(int)d[0]) >> 7;
      const double cd = i2d_exact(c);
      long long Vy = (long long)(int)d[1 + TS_LY - 1];
#pragma unroll
      for (int l = 1; l < TS_LY; ++l) Vy += (long long)(int)d[TS_LY - l] * (1ll << (8 * l));
      const double sy = LM.scale[P.k];
      const double ey = fma(magic_raw((-Vy) >> 7), sy, -MAGIC_BIAS * sy);
      double ss = 0, gs = 0;
      if (DROP0) {
        const double s0 = P.a[0] * cd;
        ss = s0 * s0;
      }
      // straight-line over every column slot that fits in N: slots past the
      // phenotype's k columns have zero limbs and a = g = 0, so they add
      // exact zeros
#pragma unroll
      for (int jj = 0; jj < KU_MAX; ++jj) {
        const int j = jj + (DROP0 ? 1 : 0);
        const int o = 1 + TS_LY + TS_LU * jj;
        // biased: 1.5 * 2^52 + V as a bit pattern, V = sum_l 256^(L-1-l) d_l
        long long Vb = (long long)(int)d[o + TS_LU - 1] + (long long)0x4338000000000000LL;
#pragma unroll
        for (int l = 1; l < TS_LU; ++l) Vb += (long long)(int)d[o + TS_LU - 1 - l] * (1ll << (8 * l));
        const double e = fma(__longlong_as_double(Vb), LM.esc[j], LM.eoff[j]);
        const double sj = fma(P.a[j], cd, e);
        ss = fma(sj, sj, ss);
        if (GATE) gs = fma(P.g[j], e, gs);  // only the Pearson gate reads gs
      }
      if (O.tested) finish_kmer(P, O, local, valid, c, ss, gs, ey);
      else finish_kmer_lean(P, O, local, valid, c, cd, ss, gs, ey, tested_local);
    }
    flush_tested(O, tested_local);
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

bool ts_supported(int N, int limbs_u, int limbs_y, int kpad, int wpk) {
  if (limbs_u != TS_LU || limbs_y != TS_LY) return false;
  if (N < 16 || N > 128 || N % 16) return false;
  if (ts_nslot(N) < 2) return false;
  if ((size_t)kpad * N > 128 * 1024) return false;  // B stays resident in shared memory
  if (wpk * 8 < 128) return false;                   // one TMA box row is 128 bytes
  return encode_fn() != nullptr;
}

// Boxes of the packed-row ring that fit next to the B image (at least 2).
static int ts_ring_depth(int b_bytes) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) optin = 0;
  int x = TS_XST_MAX;
  while (x > 2 && ts_smem(b_bytes, x).total + 1024 > (uint32_t)optin) --x;
  if (const char* v = std::getenv("KG_TS_XST")) {
    const int want = std::atoi(v);
    if (want >= 2 && want < x) x = want;
  }
  return x;
}

template <int N, bool D0, bool GATE>
static cudaError_t launch_ts_t(const LaunchTs& L, const CUtensorMap& tm, cudaStream_t st) {
  const int b_bytes = L.kpad * N;
  const int xst = ts_ring_depth(b_bytes);
  const size_t smem = ts_smem(b_bytes, xst).total + 1024;
  cudaError_t e =
      cudaFuncSetAttribute(ts_kernel<N, D0, GATE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const unsigned long long tiles = (L.m + TS_TM - 1) / TS_TM;
  unsigned long long grid = (unsigned long long)L.num_sms;
  if (grid > tiles) grid = tiles;
  const int nbox = (L.wpk * 8 + 127) / 128;
  const int nsub = L.kpad / TS_KS;
  ts_kernel<N, D0, GATE><<<(unsigned)grid, ts_threads(N), smem, st>>>(tm, L.m, nbox, nsub, xst, L.Bimg, b_bytes,
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
  // the per-k-mer statistics path (O.tested) evaluates the correlation too
  const bool gate = L.P->corr_thr > 0.0 || L.O->tested != nullptr;
  switch (L.LM->N) {
#define KG_TS_CASE(NN)                                                                       \
  case NN:                                                                                   \
    if (gate) return d0 ? launch_ts_t<NN, true, true>(L, tm, st) : launch_ts_t<NN, false, true>(L, tm, st); \
    return d0 ? launch_ts_t<NN, true, false>(L, tm, st) : launch_ts_t<NN, false, false>(L, tm, st);
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
