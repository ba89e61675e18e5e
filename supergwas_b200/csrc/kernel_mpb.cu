// kernel_mpb.cu -- many phenotypes per launch with the B operand resident in
// shared memory ("B-stationary").
//
// The reference runs one kgwas process per phenotype over the same batch
// (HPC/kgwas/kgwas_cols.sh:22-65), i.e. the statistic of src/kgwas.cpp:44-56,
// 132-218 once per (k-mer, phenotype).  Here one launch covers every
// phenotype.  Per phenotype group g (PPG phenotypes, N = PPG * NP int8 limb
// columns) the whole Kpad x N limb image is loaded into shared memory once
// and stays there while the CTA streams a block of its k-mer tiles through
// the TMEM-A pipeline of kernel_ts.cu; then the next group's image replaces
// it and the same tiles stream again.  A block is BT tile-iterations of every
// CTA, sized by the host so that its packed rows stay in L2 across the G
// passes.  Per (tile, phenotype) the CTA therefore reads 128 packed rows
// (16-32 KB, from L2 after the first pass) instead of the Kpad x N image
// (160 KB at n = 2000): the streamed-B kernel (kernel_mp.cu) is bound by
// that image traffic.
//
// Warps (15):
//   0-7     epilogue, two groups of four taking tile-visits in turn;
//   8-11    unpack: packed rows -> int8 A operand in TMEM, 512-sample
//           super-stages;
//   XP      x producer: 2-D TMA loads of the packed rows (no multicast);
//   BP      B producer: the group's image, one bulk copy per 32 KB, after
//           the previous pass's MMAs have drained;
//   MMA     tcgen05.mma kind::i8, A from TMEM, B from shared memory.
// Every wait is bounded (KG_ERR_TIMEOUT), as in kernel_ts.cu.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "device.cuh"
#include "kernels.hpp"

namespace kg {

constexpr int MB_TM = 128;
constexpr int MB_KS = 128;
constexpr int MB_SUPER = 4;
constexpr int MB_BOX = 1024;
constexpr int MB_XST = 4;
constexpr uint32_t MB_XBYTES = MB_TM * 128;
constexpr int MB_LU = 3, MB_LY = 5;
constexpr int MB_MAXSLOT = 3;
constexpr int MB_WARP_UNPACK0 = 8;

// One unpack group: per (tile, phenotype) the MMAs take Kpad/32 x N/2 cycles
// (2560 at n = 2000, N = 80), which one group's unpack of the tile keeps up
// with, and 15 warps leave 128 registers a thread for the epilogue.
__host__ __device__ constexpr int mb_ug(int) { return 1; }
// Epilogue chunks of accumulator columns: 48 = the count, 5 y' limbs and 14
// U columns of 3 limbs, so a chunk never splits a limb group.
constexpr int MB_CH = 48;
#define MB_NCH(NP_) (((NP_) + MB_CH - 1) / MB_CH)
__host__ __device__ constexpr int mb_threads(int N) { return 32 * (8 + 4 * mb_ug(N) + 3); }
__host__ __device__ constexpr int mb_nslot(int N) {
  return (512 - 2 * N) / 128 > MB_MAXSLOT ? MB_MAXSLOT : (512 - 2 * N) / 128;
}

struct MbSmem {
  uint32_t x, b, bars, tmem, abort, total;
};
__host__ __device__ inline MbSmem mb_smem(int b_bytes) {
  MbSmem L;
  L.x = 0;
  L.b = MB_XST * MB_XBYTES;
  L.bars = L.b + ((b_bytes + 127) / 128) * 128;
  L.tmem = L.bars + 8 * (2 * MB_XST + 2 * MB_MAXSLOT + 4 + 3);
  L.abort = L.tmem + 8;
  L.total = L.abort + 8;
  return L;
}

// Adds the per-lane tested counts of PPG phenotypes (group g) to their
// (shard, phenotype) counters: one atomic per distinct shard in the warp.
template <int PPG>
__device__ __forceinline__ void mb_flush(const DevOutMP& O, int g, int shard, uint32_t (&cnt)[PPG]) {
  const unsigned lane = threadIdx.x & 31u;
  unsigned left = __ballot_sync(0xffffffffu, shard >= 0);
  while (left) {
    const int ld = __ffs(left) - 1;
    const int s = __shfl_sync(0xffffffffu, shard, ld);
    const bool in = shard == s;
#pragma unroll
    for (int pp = 0; pp < PPG; ++pp) {
      const unsigned tot = __reduce_add_sync(0xffffffffu, in ? cnt[pp] : 0u);
      const int p = g * PPG + pp;
      if ((int)lane == ld && tot && p < O.n_pheno)
        atomicAdd(O.tested + (size_t)s * O.n_pheno + p, (unsigned long long)tot);
    }
    left &= ~__ballot_sync(0xffffffffu, in);
  }
#pragma unroll
  for (int pp = 0; pp < PPG; ++pp) cnt[pp] = 0;
}

template <int NP, int PPG>
__global__ void __launch_bounds__(mb_threads(NP * PPG), 1)
    mpb_kernel(const __grid_constant__ CUtensorMap tmap, unsigned long long m, int nbox, int nsub, int G, int BT,
               const int8_t* __restrict__ Bimg, int b_bytes, const MPheno* __restrict__ ph, const DevOutMP O) {
  constexpr int N = NP * PPG;
  static_assert(N <= 128 && N % 16 == 0, "group width");
  constexpr int UG = mb_ug(N);
  constexpr int WXP = MB_WARP_UNPACK0 + 4 * UG, WBP = WXP + 1, WMMA = WXP + 2;
  constexpr int NSLOT = mb_nslot(N);
  constexpr int A0 = 512 - NSLOT * 128;
  static_assert(NSLOT >= 2 && A0 >= 2 * N, "TMEM budget");
  constexpr uint32_t IDESC = idesc_i8(MB_TM, N);
  constexpr int KU_MAX = (NP - 1 - MB_LY) / MB_LU;
  constexpr uint32_t BSTEP = (2 * N * 16) >> 4;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gbase = smem_raw + (base - raw);
  const MbSmem L = mb_smem(b_bytes);
  const uint32_t sx = base + L.x, sb = base + L.b;
  const uint32_t x_full = base + L.bars, x_empty = x_full + 8 * MB_XST;
  const uint32_t a_full = x_empty + 8 * MB_XST, a_empty = a_full + 8 * MB_MAXSLOT;
  const uint32_t acc_full = a_empty + 8 * MB_MAXSLOT, acc_empty = acc_full + 16;
  const uint32_t b_full = acc_empty + 16, b_free = b_full + 8, drain = b_free + 8;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(gbase + L.tmem);
  volatile int* s_abort = reinterpret_cast<volatile int*>(gbase + L.abort);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nsp = (nsub + MB_SUPER - 1) / MB_SUPER;
  const unsigned long long ntiles = (m + MB_TM - 1) / MB_TM;
  // tile-iterations of this CTA: tiles blockIdx.x + i * gridDim.x
  const unsigned long long nt =
      ntiles > blockIdx.x ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0ull;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < MB_XST; ++s) {
      mbar_init(x_full + 8 * s, 1);
      mbar_init(x_empty + 8 * s, 4 * UG);
    }
    for (int t = 0; t < NSLOT; ++t) {
      mbar_init(a_full + 8 * t, 4);
      mbar_init(a_empty + 8 * t, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full + 8 * b, 1);
      mbar_init(acc_empty + 8 * b, 4);
    }
    mbar_init(b_full, 1);
    mbar_init(b_free, 1);
    mbar_init(drain, 1);
    *s_abort = 0;
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const unsigned long long lim = wait_limit(O.wait_ns);

  if (warp == WXP) {
    // ---------------------------------------------------------- x producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(&tmap) : "memory");
      Ring<MB_XST> xr;
      uint32_t last_phase[MB_XST];
      bool issued[MB_XST];
      for (int s = 0; s < MB_XST; ++s) issued[s] = false, last_phase[s] = 0;
      bool ok = true;
      for (unsigned long long i0 = 0; i0 < nt && ok; i0 += BT) {
        const unsigned long long i1 = i0 + BT < nt ? i0 + BT : nt;
        for (int g = 0; g < G && ok; ++g)
          for (unsigned long long i = i0; i < i1 && ok; ++i) {
            const unsigned long long tile = blockIdx.x + i * gridDim.x;
            for (int bx = 0; bx < nbox; ++bx, xr.next()) {
              if (xr.used &&
                  !wait_or_abort(x_empty + 8 * xr.slot, xr.phase ^ 1u, s_abort, O.counters, ERR_TIMEOUT_FULL, lim)) {
                ok = false;
                break;
              }
              mbar_arrive_expect_tx(x_full + 8 * xr.slot, MB_XBYTES);
              tma_load_2d(sx + xr.slot * MB_XBYTES, &tmap, bx * 128, (int)(tile * MB_TM), x_full + 8 * xr.slot);
              issued[xr.slot] = true;
              last_phase[xr.slot] = xr.phase;
            }
          }
      }
      for (int s = 0; s < MB_XST; ++s)
        if (issued[s]) mbar_wait(x_full + 8 * s, last_phase[s], O.counters, ERR_TIMEOUT_FULL);
    }
  } else if (warp == WBP) {
    // ---------------------------------------------------------- B producer
    if (lane == 0) {
      uint32_t pi = 0;
      bool ok = true;
      for (unsigned long long i0 = 0; i0 < nt && ok; i0 += BT)
        for (int g = 0; g < G && ok; ++g, ++pi) {
          // the previous pass's MMAs have read the resident image
          if (pi > 0 && !wait_or_abort(b_free, (pi - 1) & 1u, s_abort, O.counters, ERR_TIMEOUT_FULL, lim)) {
            ok = false;
            break;
          }
          const int8_t* src = Bimg + (size_t)g * b_bytes;
          mbar_arrive_expect_tx(b_full, (uint32_t)b_bytes);
          for (int off = 0; off < b_bytes; off += 32768) {
            const int len = b_bytes - off < 32768 ? b_bytes - off : 32768;
            bulk_g2s(sb + off, src + off, (uint32_t)len, b_full);
          }
        }
      // no copy may still be landing when the block exits
      if (pi > 0) mbar_wait(b_full, (pi - 1) & 1u, O.counters, ERR_TIMEOUT_FULL);
    }
  } else if (warp == WMMA) {
    // ----------------------------------------------------------------- MMA
    const bool leader = elect_one();
    const uint64_t bdesc0 = sdesc_noswz(sb, N * 16, 128);
    Ring<NSLOT> ar;
    uint32_t v = 0, pi = 0;  // tile-visits, passes
    bool ok = true;
    for (unsigned long long i0 = 0; i0 < nt && ok; i0 += BT) {
      const unsigned long long i1 = i0 + BT < nt ? i0 + BT : nt;
      for (int g = 0; g < G && ok; ++g, ++pi) {
        if (!__all_sync(0xffffffffu, wait_or_abort(b_full, pi & 1u, s_abort, O.counters, ERR_TIMEOUT_MMA, lim))) {
          ok = false;
          break;
        }
        for (unsigned long long i = i0; i < i1 && ok; ++i, ++v) {
          const uint32_t b = v & 1u;
          if (v >= 2 && !__all_sync(0xffffffffu, wait_or_abort(acc_empty + 8 * b, ((v >> 1) - 1) & 1u, s_abort,
                                                               O.counters, ERR_TIMEOUT_MMA, lim))) {
            ok = false;
            break;
          }
          const uint32_t d_t = tmem + b * N;
          uint64_t bd = bdesc0;
          for (int sp = 0; sp < nsp; ++sp, ar.next()) {
            if (!__all_sync(0xffffffffu,
                            wait_or_abort(a_full + 8 * ar.slot, ar.phase, s_abort, O.counters, ERR_TIMEOUT_MMA, lim))) {
              ok = false;
              break;
            }
            tc_fence_after();
            const int nsub_here = nsub - sp * MB_SUPER < MB_SUPER ? nsub - sp * MB_SUPER : MB_SUPER;
            const uint32_t a_t = tmem + A0 + ar.slot * 128;
            if (leader) {
              if (nsub_here == MB_SUPER) {
#pragma unroll
                for (int k = 0; k < MB_SUPER * (MB_KS / 32); ++k)
                  tc_mma_i8_ts(d_t, a_t + k * 8, bd + (uint64_t)(k * BSTEP), IDESC, (sp | k) ? 1u : 0u);
              } else {
                uint64_t bk = bd;
                for (int sub = 0; sub < nsub_here; ++sub) {
#pragma unroll
                  for (int ks = 0; ks < MB_KS / 32; ++ks) {
                    tc_mma_i8_ts(d_t, a_t + sub * 32 + ks * 8, bk, IDESC, (sp | sub | ks) ? 1u : 0u);
                    bk += BSTEP;
                  }
                }
              }
              tc_commit(a_empty + 8 * ar.slot);
            }
            __syncwarp();
            bd += (uint64_t)(MB_SUPER * (MB_KS / 32) * BSTEP);
          }
          if (!ok) break;
          if (leader) tc_commit(acc_full + 8 * b);
          __syncwarp();
        }
        // the resident image may be replaced once this pass's MMAs complete
        if (leader) tc_commit(b_free);
        __syncwarp();
      }
    }
    if (leader) {
      tc_commit(drain);
      mbar_wait(drain, 0, O.counters, ERR_TIMEOUT_MMA);
    }
    __syncwarp();
  } else if (warp >= MB_WARP_UNPACK0) {
    // -------------------------------------------------------------- unpack
    const int grp = (warp - MB_WARP_UNPACK0) >> 2;
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    Ring<MB_XST> xr;
    Ring<NSLOT> ar;
    uint32_t turn = 0;
    bool ok = true;
    for (unsigned long long i0 = 0; i0 < nt && ok; i0 += BT) {
      const unsigned long long i1 = i0 + BT < nt ? i0 + BT : nt;
      for (int g = 0; g < G && ok; ++g)
        for (unsigned long long i = i0; i < i1 && ok; ++i) {
          int kc = 0;
          for (int bx = 0; bx < nbox && ok; ++bx, xr.next()) {
            if (!__all_sync(0xffffffffu,
                            wait_or_abort(x_full + 8 * xr.slot, xr.phase, s_abort, O.counters, ERR_TIMEOUT_FULL, lim))) {
              ok = false;
              break;
            }
            const int kc1 = (bx + 1) * (MB_BOX / MB_KS) < nsub ? (bx + 1) * (MB_BOX / MB_KS) : nsub;
            while (kc < kc1) {
              const int ke = kc + MB_SUPER < kc1 ? kc + MB_SUPER : kc1;
              if (UG == 2 && turn != (uint32_t)grp) {
                kc = ke;
                ar.next();
                turn ^= 1u;
                continue;
              }
              if (ar.used && !__all_sync(0xffffffffu, wait_or_abort(a_empty + 8 * ar.slot, ar.phase ^ 1u, s_abort,
                                                                    O.counters, ERR_TIMEOUT_MMA, lim))) {
                ok = false;
                break;
              }
              const uint32_t xrow = sx + xr.slot * MB_XBYTES + r * 128;
              const uint32_t a_t = tmem + lane_base + A0 + ar.slot * 128;
              const int c0 = kc - bx * (MB_BOX / MB_KS);
              for (int sub = 0; sub < ke - kc; ++sub) {
                uint4 w;
                asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];"
                             : "=r"(w.x), "=r"(w.y), "=r"(w.z), "=r"(w.w)
                             : "r"(xrow + (((c0 + sub) ^ (r & 7)) << 4)));
                const uint32_t w4[4] = {w.x, w.y, w.z, w.w};
                uint32_t o[32];
                unpack_stage(w4, o);
                tc_st32(a_t + sub * 32, o);
              }
              kc = ke;
              tc_wait_st();
              tc_fence_before();
              __syncwarp();
              if (lane == 0) mbar_arrive(a_full + 8 * ar.slot);
              ar.next();
              if (UG == 2) turn ^= 1u;
            }
            if (!ok) break;
            __syncwarp();
            if (lane == 0) mbar_arrive(x_empty + 8 * xr.slot);
          }
        }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int e = warp >> 2;
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    uint32_t v = 0, jt = 0;
    bool ok = true;
    for (unsigned long long i0 = 0; i0 < nt && ok; i0 += BT) {
      const unsigned long long i1 = i0 + BT < nt ? i0 + BT : nt;
      for (int g = 0; g < G && ok; ++g) {
        uint32_t cnt[PPG];
#pragma unroll
        for (int pp = 0; pp < PPG; ++pp) cnt[pp] = 0;
        int cur = -1;  // shard of the counts in cnt
        for (unsigned long long i = i0; i < i1; ++i, ++v) {
          if ((v & 1u) != (uint32_t)e) continue;
          if (!__all_sync(0xffffffffu,
                          wait_or_abort(acc_full + 8 * e, jt & 1u, s_abort, O.counters, ERR_TIMEOUT_MMA, lim))) {
            ok = false;
            break;
          }
          ++jt;
          tc_fence_after();
          const unsigned long long tile = blockIdx.x + i * gridDim.x;
          const unsigned long long local = tile * MB_TM + r;
          const bool valid = local < m;
          const unsigned long long gk = O.kmer_offset + local;
          const int shard = mp_shard(O, gk);
          const uint32_t wt = O.weight && valid ? O.weight[gk] : 1u;  // rows this row stands for
          if (__any_sync(0xffffffffu, shard != cur)) {
            mb_flush<PPG>(O, g, cur, cnt);
            cur = shard;
          }
#pragma unroll
          for (int pp = 0; pp < PPG; ++pp) {
            const int p = g * PPG + pp;
            const bool live = p < O.n_pheno;  // warp-uniform
            const MPheno* ME = ph + (live ? p : 0);
            const EpiParams& P = ME->P;
            int c = 0;
            double cd = 0, ey = 0, ss = 0, gs = 0;
            int drop0 = 0;
            // The phenotype's NP accumulator columns, 48 at a time: column 0
            // is the count, 1-5 the y' limbs, then 3 limbs per U column, so
            // every 48-column chunk holds whole limb groups.  The buffer is
            // released after the group's last load.
#pragma unroll
            for (int ch = 0; ch < MB_NCH(NP); ++ch) {
              constexpr int CH = MB_CH;
              const int width = NP - ch * CH < CH ? NP - ch * CH : CH;
              uint32_t d[CH];
              if (live) {
#pragma unroll
                for (int c16 = 0; c16 < CH / 16; ++c16) {
                  if (c16 * 16 < width) {
                    uint32_t rr[16];
                    tc_ld16(tmem + lane_base + e * N + pp * NP + ch * CH + c16 * 16, rr);
                    tc_wait_ld();
#pragma unroll
                    for (int k = 0; k < 16; ++k) d[c16 * 16 + k] = rr[k];
                  }
                }
              }
              if (pp == PPG - 1 && ch == MB_NCH(NP) - 1) {
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(acc_empty + 8 * e);
              }
              if (!live) continue;
              if (ch == 0) {
                // limb sums hold -128 * integer sums (see kernel_ts.cu)
                c = (-(int)d[0]) >> 7;
                cd = i2d_exact(c);
                long long Vy = (long long)(int)d[MB_LY];
#pragma unroll
                for (int l = 1; l < MB_LY; ++l) Vy += (long long)(int)d[MB_LY - l] * (1ll << (8 * l));
                const double sy = ME->LM.scale[P.k];
                ey = fma(magic_raw((-Vy) >> 7), sy, -MAGIC_BIAS * sy);
                drop0 = ME->drop0;
                if (drop0) {
                  const double s0 = P.a[0] * cd;
                  ss = s0 * s0;
                }
              }
              // slots past the phenotype's k columns have zero limbs and zero
              // constants: they add exact zeros
#pragma unroll
              for (int jj = 0; jj < KU_MAX; ++jj) {
                const int o = 1 + MB_LY + MB_LU * jj;  // first limb column of slot jj
                if (o / CH != ch) continue;
                const int od = o - ch * CH;
                const int j = jj + drop0;
                long long Vb = (long long)(int)d[od + MB_LU - 1] + (long long)0x4338000000000000LL;
#pragma unroll
                for (int l = 1; l < MB_LU; ++l) Vb += (long long)(int)d[od + MB_LU - 1 - l] * (1ll << (8 * l));
                const double ej = fma(__longlong_as_double(Vb), ME->LM.esc[j], ME->LM.eoff[j]);
                const double sj = fma(P.a[j], cd, ej);
                ss = fma(sj, sj, ss);
                gs = fma(P.g[j], ej, gs);
              }
            }
            if (!live) continue;
            bool tested, hit, cand;
            double T, pv, effect;
            mp_eval(P, valid, c, ss, gs, ey, tested, hit, cand, T, pv, effect);
            cnt[pp] += tested ? wt : 0u;
            if (__any_sync(0xffffffffu, hit || cand)) mp_emit_rare(O, p, gk, shard, hit, cand, T, pv, effect);
          }
        }
        mb_flush<PPG>(O, g, cur, cnt);
      }
    }
  }
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// ------------------------------------------------------------------- host

size_t mpb_smem_bytes(int N, int kpad) { return mb_smem(kpad * N).total + 1024; }

bool mpb_supported(int NP, int PPG, int kpad, int wpk) {
  if (NP < 16 || NP > 128 || NP % 16 || PPG < 1 || NP * PPG > 128) return false;
  if (wpk * 8 < 128) return false;
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return false;
  return mpb_smem_bytes(NP * PPG, kpad) <= (size_t)optin;
}

template <int NP, int PPG>
static cudaError_t launch_mpb_t(const LaunchMpb& L, const CUtensorMap& tm, cudaStream_t st) {
  constexpr int N = NP * PPG;
  const int b_bytes = L.kpad * N;
  const size_t smem = mpb_smem_bytes(N, L.kpad);
  cudaError_t e = cudaFuncSetAttribute(mpb_kernel<NP, PPG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const unsigned long long tiles = (L.m + MB_TM - 1) / MB_TM;
  unsigned long long grid = (unsigned long long)L.num_sms;
  if (grid > tiles) grid = tiles;
  const int nbox = (L.wpk * 8 + 127) / 128;
  mpb_kernel<NP, PPG><<<(unsigned)grid, mb_threads(N), smem, st>>>(tm, L.m, nbox, L.kpad / MB_KS, L.G,
                                                                   L.bt > 0 ? L.bt : 1, L.Bimg, b_bytes, L.ph,
                                                                   *L.O);
  return cudaGetLastError();
}

cudaError_t launch_mpb(const LaunchMpb& L, cudaStream_t st) {
  if (L.m == 0) return cudaSuccess;
  CUtensorMap tm;
  if (!mp_tmap(L.x, L.m, L.wpk, &tm)) return cudaErrorInvalidValue;
#define KG_MPB_CASE(NP_, PPG_) \
  if (L.NP == NP_ && L.PPG == PPG_) return launch_mpb_t<NP_, PPG_>(L, tm, st);
  KG_MP_GROUPS(KG_MPB_CASE)
#undef KG_MPB_CASE
  return cudaErrorInvalidValue;
}

}  // namespace kg
