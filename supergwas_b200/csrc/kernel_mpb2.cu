// kernel_mpb2.cu -- many phenotypes per launch, two phenotypes per MMA on a
// pair of SMs (tcgen05 cta_group::2).
//
// The reference runs one kgwas process per phenotype over the same batch
// (HPC/kgwas/kgwas_cols.sh:22-65), i.e. the statistic of src/kgwas.cpp:44-56,
// 132-218 once per (k-mer, phenotype).  kernel_mpb.cu runs it for every
// phenotype in one launch with one phenotype's int8 limb image (Kpad x NP)
// resident in shared memory per MMA group, and unpacks every tile's packed
// rows into the int8 A operand once per phenotype: two phenotypes' images
// (Kpad x 160 = 320 KB at n = 2000, r = 20+1) do not fit one SM's shared
// memory.
//
// Here a cluster of two CTAs on two SMs issues M = 256 MMAs (cta_group::2):
// each CTA holds 128 k-mers of a 256-k-mer pair-tile as its A operand in
// tensor memory and ONE phenotype's limb image (Kpad x NP) in shared memory
// as its half of B, and each CTA's tensor memory receives the 2 x NP
// accumulator columns of both phenotypes for its own 128 k-mers.  Each tile
// is unpacked once per two phenotypes; the MMA time per (k-mer, phenotype) is
// the same as kernel_mpb.cu's (an M = 128 or 256 kind::i8 MMA issues N / 2
// cycles per SM at every N measured).
//
// Roles (15 warps per CTA, both CTAs):
//   0-7   epilogue, two groups of four taking pair-tile visits in turn: the
//         accumulators of both phenotypes for this CTA's 128 k-mers;
//   8-11  unpack: packed rows -> int8 A operand in this CTA's tensor memory,
//         256-sample stages (64 columns);
//   XP    row producer: 2-D TMA loads of this CTA's 128 rows (no multicast);
//   BP    image producer: this CTA's phenotype image, bulk copies;
//   MMA   (leader CTA only) tcgen05.mma.cta_group::2, commits multicast to
//         both CTAs' barriers.
// The leader's MMA waits for both CTAs' unpack warps (a_full, 8 arrivals:
// 4 local, 4 remote), both images (b_pair, 2 arrivals) and both epilogues
// (acc_empty, 8 arrivals).  Every wait is bounded; a CTA that gives up also
// raises its peer's abort flag, and both drain their own copies and the MMAs
// before the pair frees its tensor memory.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "device.cuh"
#include "kernels.hpp"

namespace kg {

constexpr int M2_TM = 128;                    // k-mers per CTA (rows of its half of M)
constexpr int M2_KS = 128;                    // samples per sub-stage (32 TMEM columns, 4 MMAs)
constexpr int M2_SUPER = 2;                   // sub-stages per stage (64 columns, 8 MMAs)
constexpr int M2_BOX = 1024;                  // samples per TMA box (128 bytes)
constexpr int M2_XST = 4;                     // row boxes in flight per CTA
constexpr uint32_t M2_XBYTES = M2_TM * 128;
constexpr int M2_LU = 3, M2_LY = 5;
constexpr int M2_MAXSLOT = 4;
constexpr int M2_CH = 48;                     // epilogue chunk (whole limb groups)
#define M2_NCH(NP_) (((NP_) + M2_CH - 1) / M2_CH)
constexpr int M2_THREADS = 32 * (8 + 4 + 3);
constexpr int M2_WXP = 12, M2_WBP = 13, M2_WMMA = 14;

__host__ __device__ constexpr int m2_nslot(int NP) {
  return (512 - 4 * NP) / 64 > M2_MAXSLOT ? M2_MAXSLOT : (512 - 4 * NP) / 64;
}

struct M2Smem {
  uint32_t x, b, bars, tmem, abort, total;
};
__host__ __device__ inline M2Smem m2_smem(int b_bytes) {
  M2Smem L;
  L.x = 0;
  L.b = M2_XST * M2_XBYTES;
  L.bars = L.b + ((b_bytes + 127) / 128) * 128;
  L.tmem = L.bars + 8 * (2 * M2_XST + 2 * M2_MAXSLOT + 4 + 4);
  L.abort = L.tmem + 8;
  L.total = L.abort + 8;
  return L;
}

__device__ __forceinline__ uint32_t cta_rank_in_cluster() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t peer_addr(uint32_t local, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}
// Arrive on an mbarrier of any CTA of the cluster.  What the arrivals hand
// over is tensor memory (A slots written with tcgen05.st and completed by
// tcgen05.wait::st; accumulators read with tcgen05.ld and completed by
// tcgen05.wait::ld) and the end of copies or MMAs, each ordered by a
// tcgen05 fence or an mbarrier transaction, so the default (CTA-scope)
// release of the arrive suffices: a cluster-scope release would add a
// memory barrier to every hand-over.
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ bool mbar_try_cluster(uint32_t bar, uint32_t parity) { return mbar_try_sleep(bar, parity); }
// Bounded wait (acquire at cluster scope) that also gives up when this CTA's
// abort flag is raised; on giving up it raises both CTAs' flags.
__device__ __forceinline__ bool pair_wait(uint32_t bar, uint32_t parity, volatile int* abort, uint32_t peer_abort,
                                          unsigned long long* counters, unsigned code, unsigned long long limit_ns) {
  if (mbar_try_cluster(bar, parity)) return true;
  const unsigned long long t0 = gtimer_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_cluster(bar, parity)) return true;
    if ((it & 15u) == 0) {
      if (*abort) return false;
      if (gtimer_ns() - t0 > limit_ns) {
        atomicOr(counters + 2, (unsigned long long)code);
        *abort = 1;
        asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(peer_abort), "r"(1u) : "memory");
        return false;
      }
    }
  }
}
__device__ __forceinline__ void tc_commit_pair(uint32_t bar) {  // to the barrier at `bar` in both CTAs
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(bar),
      "h"((unsigned short)3)
      : "memory");
}
__device__ __forceinline__ void tc_commit_pair_local(uint32_t bar) {  // to the leader's barrier only
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_mma_i8_pair(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                               uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], [%1], %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u)
      : "memory");
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Tested counts of the two phenotypes of group g, flushed per shard (as
// kernel_mpb.cu's mb_flush).
__device__ __forceinline__ void m2_flush(const DevOutMP& O, int g, int shard, uint32_t (&cnt)[2]) {
  const unsigned lane = threadIdx.x & 31u;
  unsigned left = __ballot_sync(0xffffffffu, shard >= 0);
  while (left) {
    const int ld = __ffs(left) - 1;
    const int s = __shfl_sync(0xffffffffu, shard, ld);
    const bool in = shard == s;
#pragma unroll
    for (int pp = 0; pp < 2; ++pp) {
      const unsigned tot = __reduce_add_sync(0xffffffffu, in ? cnt[pp] : 0u);
      const int p = 2 * g + pp;
      if ((int)lane == ld && tot && p < O.n_pheno)
        atomicAdd(O.tested + (size_t)s * O.n_pheno + p, (unsigned long long)tot);
    }
    left &= ~__ballot_sync(0xffffffffu, in);
  }
  cnt[0] = cnt[1] = 0;
}

template <int NP>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(M2_THREADS, 1)
    mpb2_kernel(const __grid_constant__ CUtensorMap tmap, unsigned long long m, int nbox, int nsub, int G, int BT,
                const int8_t* __restrict__ Bimg, int b_bytes, const MPheno* __restrict__ ph, const DevOutMP O) {
  constexpr int N = 2 * NP;
  static_assert(N % 32 == 0 && N <= 256, "pair MMA width");
  constexpr int NSLOT = m2_nslot(NP);
  constexpr int A0 = 512 - NSLOT * 64;
  static_assert(NSLOT >= 2 && A0 >= 2 * N, "TMEM budget");
  constexpr uint32_t IDESC = idesc_i8(2 * M2_TM, N);
  constexpr int KU_MAX = (NP - 1 - M2_LY) / M2_LU;
  constexpr uint32_t BSTEP = (2 * NP * 16) >> 4;  // one K = 32 step of this CTA's NP-column half
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gbase = smem_raw + (base - raw);
  const M2Smem L = m2_smem(b_bytes);
  const uint32_t sx = base + L.x, sb = base + L.b;
  const uint32_t x_full = base + L.bars, x_empty = x_full + 8 * M2_XST;
  const uint32_t a_full = x_empty + 8 * M2_XST, a_empty = a_full + 8 * M2_MAXSLOT;
  const uint32_t acc_full = a_empty + 8 * M2_MAXSLOT, acc_empty = acc_full + 16;
  const uint32_t b_full = acc_empty + 16, b_pair = b_full + 8, b_free = b_pair + 8, drain = b_free + 8;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(gbase + L.tmem);
  volatile int* s_abort = reinterpret_cast<volatile int*>(gbase + L.abort);
  const uint32_t rank = cta_rank_in_cluster();
  const bool lead = rank == 0;
  const uint32_t peer_abort = peer_addr(base + L.abort, rank ^ 1u);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nsp = (nsub + M2_SUPER - 1) / M2_SUPER;
  const unsigned long long lim = wait_limit(O.wait_ns);
  // pair-tiles of 256 k-mers; this pair visits pt = pair, pair + npairs, ...
  const unsigned long long pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const unsigned long long npt = (m + 2 * M2_TM - 1) / (2 * M2_TM);
  const unsigned long long nt = npt > pair ? (npt - pair + npairs - 1) / npairs : 0ull;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < M2_XST; ++s) {
      mbar_init(x_full + 8 * s, 1);
      mbar_init(x_empty + 8 * s, 4);
    }
    for (int t = 0; t < NSLOT; ++t) {
      mbar_init(a_full + 8 * t, 8);   // the unpack warps of both CTAs (leader's barrier)
      mbar_init(a_empty + 8 * t, 1);  // multicast commit
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full + 8 * b, 1);   // multicast commit
      mbar_init(acc_empty + 8 * b, 8);  // the epilogue group of both CTAs (leader's barrier)
    }
    mbar_init(b_full, 1);
    mbar_init(b_pair, 2);  // both images loaded (leader's barrier)
    mbar_init(b_free, 1);  // multicast commit
    mbar_init(drain, 1);
    *s_abort = 0;
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // barriers, flags and tensor memory of both CTAs are in place
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  if (warp == M2_WXP) {
    // ------------------------------------------------------- row producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(&tmap) : "memory");
      Ring<M2_XST> xr;
      uint32_t last_phase[M2_XST];
      bool issued[M2_XST];
      for (int s = 0; s < M2_XST; ++s) issued[s] = false, last_phase[s] = 0;
      bool ok = true;
      for (unsigned long long i0 = 0; i0 < nt && ok; i0 += BT) {
        const unsigned long long i1 = i0 + BT < nt ? i0 + BT : nt;
        for (int g = 0; g < G && ok; ++g)
          for (unsigned long long i = i0; i < i1 && ok; ++i) {
            const unsigned long long row = (pair + i * npairs) * (2 * M2_TM) + rank * M2_TM;
            for (int bx = 0; bx < nbox; ++bx, xr.next()) {
              if (xr.used && !wait_or_abort(x_empty + 8 * xr.slot, xr.phase ^ 1u, s_abort, O.counters,
                                            ERR_TIMEOUT_FULL, lim)) {
                ok = false;
                break;
              }
              mbar_arrive_expect_tx(x_full + 8 * xr.slot, M2_XBYTES);
              tma_load_2d(sx + xr.slot * M2_XBYTES, &tmap, bx * 128, (int)row, x_full + 8 * xr.slot);
              issued[xr.slot] = true;
              last_phase[xr.slot] = xr.phase;
            }
          }
      }
      for (int s = 0; s < M2_XST; ++s)
        if (issued[s]) mbar_wait(x_full + 8 * s, last_phase[s], O.counters, ERR_TIMEOUT_FULL);
    }
  } else if (warp == M2_WBP) {
    // ------------------------------------------------------ image producer
    if (lane == 0) {
      const uint32_t lead_pair = peer_addr(b_pair, 0u);
      uint32_t pi = 0;
      bool ok = true;
      for (unsigned long long i0 = 0; i0 < nt && ok; i0 += BT)
        for (int g = 0; g < G && ok; ++g, ++pi) {
          // the previous pass's MMAs have read both images
          if (pi > 0 &&
              !pair_wait(b_free, (pi - 1) & 1u, s_abort, peer_abort, O.counters, ERR_TIMEOUT_FULL, lim)) {
            ok = false;
            break;
          }
          // this CTA's phenotype of group g (an odd count leaves the last
          // group's second slot to a copy of the first, never reported)
          const int p = 2 * g + (int)rank < O.n_pheno ? 2 * g + (int)rank : 2 * g;
          const int8_t* src = Bimg + (size_t)p * b_bytes;
          mbar_arrive_expect_tx(b_full, (uint32_t)b_bytes);
          for (int off = 0; off < b_bytes; off += 32768) {
            const int len = b_bytes - off < 32768 ? b_bytes - off : 32768;
            bulk_g2s(sb + off, src + off, (uint32_t)len, b_full);
          }
          if (!mbar_wait(b_full, pi & 1u, O.counters, ERR_TIMEOUT_FULL)) {
            ok = false;
            break;
          }
          mbar_arrive_cluster(lead_pair);
        }
      // no copy may still be landing when the block exits
      if (pi > 0) mbar_wait(b_full, (pi - 1) & 1u, O.counters, ERR_TIMEOUT_FULL);
    }
  } else if (warp == M2_WMMA) {
    // ------------------------------------------------- MMA (leader only)
    if (lead) {
      const bool leader = elect_one();
      const uint64_t bdesc0 = sdesc_noswz(sb, NP * 16, 128);
      Ring<NSLOT> ar;
      uint32_t v = 0, pi = 0;
      bool ok = true;
      for (unsigned long long i0 = 0; i0 < nt && ok; i0 += BT) {
        const unsigned long long i1 = i0 + BT < nt ? i0 + BT : nt;
        for (int g = 0; g < G && ok; ++g, ++pi) {
          if (!__all_sync(0xffffffffu,
                          pair_wait(b_pair, pi & 1u, s_abort, peer_abort, O.counters, ERR_TIMEOUT_MMA, lim))) {
            ok = false;
            break;
          }
          for (unsigned long long i = i0; i < i1 && ok; ++i, ++v) {
            const uint32_t b = v & 1u;
            if (v >= 2 && !__all_sync(0xffffffffu, pair_wait(acc_empty + 8 * b, ((v >> 1) - 1) & 1u, s_abort,
                                                             peer_abort, O.counters, ERR_TIMEOUT_MMA, lim))) {
              ok = false;
              break;
            }
            const uint32_t d_t = tmem + b * N;
            uint64_t bd = bdesc0;
            for (int sp = 0; sp < nsp; ++sp, ar.next()) {
              if (!__all_sync(0xffffffffu, pair_wait(a_full + 8 * ar.slot, ar.phase, s_abort, peer_abort,
                                                     O.counters, ERR_TIMEOUT_MMA, lim))) {
                ok = false;
                break;
              }
              tc_fence_after();
              const int nsub_here = nsub - sp * M2_SUPER < M2_SUPER ? nsub - sp * M2_SUPER : M2_SUPER;
              const uint32_t a_t = tmem + A0 + ar.slot * 64;
              if (leader) {
                if (nsub_here == M2_SUPER) {
#pragma unroll
                  for (int k = 0; k < M2_SUPER * (M2_KS / 32); ++k)
                    tc_mma_i8_pair(d_t, a_t + k * 8, bd + (uint64_t)(k * BSTEP), IDESC, (sp | k) ? 1u : 0u);
                } else {
                  uint64_t bk = bd;
                  for (int sub = 0; sub < nsub_here; ++sub) {
#pragma unroll
                    for (int ks = 0; ks < M2_KS / 32; ++ks) {
                      tc_mma_i8_pair(d_t, a_t + sub * 32 + ks * 8, bk, IDESC, (sp | sub | ks) ? 1u : 0u);
                      bk += BSTEP;
                    }
                  }
                }
                tc_commit_pair(a_empty + 8 * ar.slot);
              }
              __syncwarp();
              bd += (uint64_t)(M2_SUPER * (M2_KS / 32) * BSTEP);
            }
            if (!ok) break;
            if (leader) tc_commit_pair(acc_full + 8 * b);
            __syncwarp();
          }
          // the images may be replaced once this pass's MMAs complete
          if (leader) tc_commit_pair(b_free);
          __syncwarp();
        }
      }
      if (leader) {
        tc_commit_pair_local(drain);
        mbar_wait(drain, 0, O.counters, ERR_TIMEOUT_MMA);
      }
      __syncwarp();
    }
  } else if (warp >= 8) {
    // -------------------------------------------------------------- unpack
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    const uint32_t lead_a_full = peer_addr(a_full, 0u);
    Ring<M2_XST> xr;
    Ring<NSLOT> ar;
    bool ok = true;
    for (unsigned long long i0 = 0; i0 < nt && ok; i0 += BT) {
      const unsigned long long i1 = i0 + BT < nt ? i0 + BT : nt;
      for (int g = 0; g < G && ok; ++g)
        for (unsigned long long i = i0; i < i1 && ok; ++i) {
          int kc = 0;
          for (int bx = 0; bx < nbox && ok; ++bx, xr.next()) {
            if (!__all_sync(0xffffffffu, wait_or_abort(x_full + 8 * xr.slot, xr.phase, s_abort, O.counters,
                                                       ERR_TIMEOUT_FULL, lim))) {
              ok = false;
              break;
            }
            const int kc1 = (bx + 1) * (M2_BOX / M2_KS) < nsub ? (bx + 1) * (M2_BOX / M2_KS) : nsub;
            while (kc < kc1) {
              const int ke = kc + M2_SUPER < kc1 ? kc + M2_SUPER : kc1;
              if (ar.used && !__all_sync(0xffffffffu, pair_wait(a_empty + 8 * ar.slot, ar.phase ^ 1u, s_abort,
                                                                peer_abort, O.counters, ERR_TIMEOUT_MMA, lim))) {
                ok = false;
                break;
              }
              const uint32_t xrow = sx + xr.slot * M2_XBYTES + r * 128;
              const uint32_t a_t = tmem + lane_base + A0 + ar.slot * 64;
              const int c0 = kc - bx * (M2_BOX / M2_KS);
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
              if (lane == 0) mbar_arrive_cluster(lead_a_full + 8 * ar.slot);
              ar.next();
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
    const uint32_t lead_acc_empty = peer_addr(acc_empty, 0u);
    uint32_t v = 0, jt = 0;
    bool ok = true;
    for (unsigned long long i0 = 0; i0 < nt && ok; i0 += BT) {
      const unsigned long long i1 = i0 + BT < nt ? i0 + BT : nt;
      for (int g = 0; g < G && ok; ++g) {
        uint32_t cnt[2] = {0, 0};
        int cur = -1;  // shard of the counts in cnt
        for (unsigned long long i = i0; i < i1; ++i, ++v) {
          if ((v & 1u) != (uint32_t)e) continue;
          if (!__all_sync(0xffffffffu, pair_wait(acc_full + 8 * e, jt & 1u, s_abort, peer_abort, O.counters,
                                                 ERR_TIMEOUT_MMA, lim))) {
            ok = false;
            break;
          }
          ++jt;
          tc_fence_after();
          const unsigned long long local = (pair + i * npairs) * (2 * M2_TM) + rank * M2_TM + r;
          const bool valid = local < m;
          const unsigned long long gk = O.kmer_offset + local;
          const int shard = mp_shard(O, valid ? gk : O.kmer_offset);
          const uint32_t wt = O.weight && valid ? O.weight[gk] : 1u;  // rows this row stands for
          if (__any_sync(0xffffffffu, shard != cur)) {
            m2_flush(O, g, cur, cnt);
            cur = shard;
          }
#pragma unroll
          for (int pp = 0; pp < 2; ++pp) {
            const int p = 2 * g + pp;
            const bool live = p < O.n_pheno;  // warp-uniform
            const MPheno* ME = ph + (live ? p : 0);
            const EpiParams& P = ME->P;
            int c = 0;
            double cd = 0, ey = 0, ss = 0, gs = 0;
            int drop0 = 0;
            // the phenotype's NP accumulator columns, 48 at a time (column 0
            // the count, 1-5 the y' limbs, then 3 limbs per U column: every
            // chunk holds whole limb groups); the accumulator is released
            // after the last load
#pragma unroll
            for (int ch = 0; ch < M2_NCH(NP); ++ch) {
              constexpr int CH = M2_CH;
              const int width = NP - ch * CH < CH ? NP - ch * CH : CH;
              uint32_t d[CH];
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
              if (pp == 1 && ch == M2_NCH(NP) - 1) {
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(lead_acc_empty + 8 * e);
              }
              if (!live) continue;
              if (ch == 0) {
                // limb sums hold -128 * integer sums (see kernel_ts.cu)
                c = (-(int)d[0]) >> 7;
                cd = i2d_exact(c);
                long long Vy = (long long)(int)d[M2_LY];
#pragma unroll
                for (int l = 1; l < M2_LY; ++l) Vy += (long long)(int)d[M2_LY - l] * (1ll << (8 * l));
                const double sy = ME->LM.scale[P.k];
                ey = fma(magic_raw((-Vy) >> 7), sy, -MAGIC_BIAS * sy);
                drop0 = ME->drop0;
                if (drop0) {
                  const double s0 = P.a[0] * cd;
                  ss = s0 * s0;
                }
              }
#pragma unroll
              for (int jj = 0; jj < KU_MAX; ++jj) {
                const int o = 1 + M2_LY + M2_LU * jj;  // first limb column of slot jj
                if (o / CH != ch) continue;
                const int od = o - ch * CH;
                const int j = jj + drop0;
                long long Vb = (long long)(int)d[od + M2_LU - 1] + (long long)0x4338000000000000LL;
#pragma unroll
                for (int l = 1; l < M2_LU; ++l) Vb += (long long)(int)d[od + M2_LU - 1 - l] * (1ll << (8 * l));
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
        m2_flush(O, g, cur, cnt);
      }
    }
  }
  // the pair's MMAs have drained (leader) and no copy is in flight (both);
  // neither CTA frees its tensor memory before the other is done with it
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// ------------------------------------------------------------------- host

size_t mpb2_smem_bytes(int NP, int kpad) { return m2_smem(kpad * NP).total + 1024; }

bool mpb2_supported(int NP, int kpad, int wpk) {
  if (NP != 48 && NP != 64 && NP != 80 && NP != 96) return false;
  if (wpk * 8 < 128) return false;
  int dev = 0, optin = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return false;
  return sms >= 2 && mpb2_smem_bytes(NP, kpad) <= (size_t)optin;
}

template <int NP>
static cudaError_t launch_mpb2_t(const LaunchMpb& L, const CUtensorMap& tm, cudaStream_t st) {
  const int b_bytes = L.kpad * NP;
  const size_t smem = mpb2_smem_bytes(NP, L.kpad);
  cudaError_t e = cudaFuncSetAttribute(mpb2_kernel<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // as many pairs as can be resident at once (a GPC with an odd number of
  // free SMs leaves one SM without a partner), else a second wave of pairs
  // would double the launch
  static int resident_of[64] = {};  // per device ordinal; 0: not looked up yet
  int dev = 0;
  cudaGetDevice(&dev);
  int& resident = resident_of[dev & 63];
  if (resident <= 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(L.num_sms & ~1));
    cfg.blockDim = dim3(M2_THREADS);
    cfg.dynamicSmemBytes = smem;
    int clusters = 0;
    resident = cudaOccupancyMaxActiveClusters(&clusters, (void*)mpb2_kernel<NP>, &cfg) == cudaSuccess && clusters > 0
                   ? clusters
                   : L.num_sms / 2;
    cudaGetLastError();
  }
  const unsigned long long npt = (L.m + 2 * M2_TM - 1) / (2 * M2_TM);
  unsigned long long pairs = (unsigned long long)std::min(L.num_sms / 2, resident);
  if (pairs > npt) pairs = npt;
  if (pairs < 1) pairs = 1;
  const int nbox = (L.wpk * 8 + 127) / 128;
  const int G = (L.G + 1) / 2;  // L.G phenotypes (one image each), two per MMA
  mpb2_kernel<NP><<<(unsigned)(2 * pairs), M2_THREADS, smem, st>>>(tm, L.m, nbox, L.kpad / M2_KS, G,
                                                                    L.bt > 0 ? L.bt : 1, L.Bimg, b_bytes, L.ph, *L.O);
  return cudaGetLastError();
}

cudaError_t launch_mpb2(const LaunchMpb& L, cudaStream_t st) {
  if (L.m == 0) return cudaSuccess;
  CUtensorMap tm;
  if (!mp_tmap(L.x, L.m, L.wpk, &tm)) return cudaErrorInvalidValue;
  switch (L.NP) {
    case 48: return launch_mpb2_t<48>(L, tm, st);
    case 64: return launch_mpb2_t<64>(L, tm, st);
    case 80: return launch_mpb2_t<80>(L, tm, st);
    case 96: return launch_mpb2_t<96>(L, tm, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kg
