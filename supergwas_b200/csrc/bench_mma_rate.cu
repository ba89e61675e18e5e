// bench_mma_rate.cu -- measurement kernels behind the rate figures of the
// association kernels (libkgwas_bench.so; run by `bench.py --workload
// mma-rate`, not part of the association library).
//
// kg_bench_mma_rate times back-to-back tcgen05.mma kind::i8 instructions
// (K = 32, accumulating) per SM:
//   kind 0: one CTA per SM, `issuers` warps (on different SM sub-partitions)
//           each issuing into its own accumulator;
//   kind 1: two CTAs per SM (256 tensor-memory columns each), one issuer each;
//   kind 2: a cluster of two CTAs issuing M = 256 MMAs (cta_group::2), B split
//           over the pair, accumulators in both SMs' tensor memory;
//   kind 3: kind 0 with one issuer while four other warps write tensor memory
//           with tcgen05.st.32x32b.x32 (the A-operand stores of the unpack);
//   kind 4: kind 0 with one issuer while four other warps read tensor memory
//           with tcgen05.ld.32x32b.x16 (the accumulator loads of the epilogue);
//   kind 5: as kind 3, the stores issued four at a time before one
//           tcgen05.wait::st (as the unpack warps issue them): the store rate;
//   kind 6: kind 5 without MMAs (the issuer warp idles);
//   kind 7: kind 0 with one issuer while four other warps read shared memory
//           (ld.shared.v4 of the B region, as the unpack warps read row boxes):
//           does shared-memory traffic slow the MMAs' B reads?
//   kind 8: kind 7 without MMAs.
//   kinds 9-12: one issuer walking the operands as the single-phenotype
//           kernel does (A across three 128-column slots from column 128, B
//           across 32 K-steps of the resident image for N <= 64), with a
//           tcgen05.commit every 16 MMAs (kind 9) or every 4 (kind 10) to a
//           barrier nobody waits on, or a ring of 3 (kind 11) or 2 (kind 12)
//           A slots: before the MMAs of a slot's next use the issuer waits for
//           the commit of its previous use, as the unpack warps do.  This
//           isolates the cost of commits and of the slot hand-off from the
//           work of the other roles.  Kinds 11 and 12 wait with mbar_wait
//           (try_wait without a suspend-time hint, the clock read after every
//           test); kinds 13-15 are kind 11 waiting by spinning on
//           mbarrier.test_wait (13), on try_wait with a suspend-time hint (14)
//           or on try_wait without one (15), the clock read every 1024 tests;
//           kind 16 spins on test_wait bounded by a count of tests (no clock
//           read), kind 17 on try_wait bounded by the SM cycle counter;
//           kind 18 waits for its own last commit before each use (no ring);
//           kind 19 is the ring of 3 with a helper warp that waits for the
//           commits and frees the slots, the issuer waiting for the frees.
//           kinds 20-22 issue each use as one unrolled block of 16 MMAs with
//           compile-time offsets after a tcgen05 fence, as the kernels do:
//           kind 20 with the ring of 3, kind 21 with a try_wait that succeeds
//           at once before each use, kind 22 with only the clock reads.
//           For the ring kinds the side fields give the issuer's waits and
//           their average cycles.
//   kinds 23-30 (mma_ring): one accumulator, A slots from column N, uses of
//           MPU unrolled MMAs: 23 one slot of 16 MMAs (each use waits for the
//           last: MMA time + commit latency), 24 one slot of 1 MMA, 25 commits
//           alone, 26 three slots of 16 with a helper warp's hop, 27 six slots
//           of 8, 28 seven slots of 8 (448 columns), 29 as 28 with the hop,
//           30 three slots of 16 without the hop, 31 as 30 and 32 as 23
//           without the tcgen05 fence after the wait (the probe writes no A,
//           so nothing needs ordering), 33 as 30 waiting on try_wait with a
//           suspend-time hint; 34-36 (rings of 3 x 16, 2 x 16, 6 x 8) wait
//           for the next use's slot after issuing a use's MMAs and before
//           committing them, so no wait lies between a commit and the next
//           MMA; 37-39 are kind 30 while the CTA's seven other warps wait on
//           a barrier that never completes (try_wait; with a suspend-time
//           hint; after a 128 ns sleep), as a kernel's other roles wait.
//           The side fields give cycles per use.
//   kinds 40-44 (mma_pipe, 576 threads, the issuer in warp 17): the ring of
//           3 x 16 as the single-phenotype kernel runs it, its features added
//           one at a time: 40 none, 41 two accumulators alternating by tile,
//           42 + the accumulator hand-off through an epilogue group, 43 the
//           slot hand-off through a group of four warps, 44 all of them;
//           45-48 are kind 44 with one thread waiting: at the top of each use
//           (45), with the accumulator one use earlier (46), in the middle of
//           the previous use's MMAs (47), or testing there and waiting after
//           the commits only if a test failed (48); 49, 50 are kind 43 (no
//           accumulator hand-off) waiting as 45 and 47; 51-54 are kinds 44
//           and 47 while eight other warps (two per sub-partition) do
//           integer work with 2 (51, 52) or 4 (53, 54) independent chains;
//           55-57: two issuers (warps 16, 17) taking alternate tiles, each
//           with its own accumulator, alone (55) and beside the busy warps
//           with 2 (56) or 4 (57) chains;
//   kinds 58-60 (mma_pipe2): two issuers with private rings, their own
//           slot and accumulator groups: 3 slots of 8 MMAs each (58), 2 of 8
//           (59), 1 of 16 (60); 61, 62: kinds 56 and 51 with the eight
//           busy warps running FP64 multiply-add chains.
// A comes from tensor memory (M = 128 rows, 32 bytes of K per MMA), B from
// shared memory.  Every wait is bounded (2 s); no TMA.
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device.cuh"

using namespace kg;

namespace {

constexpr int kIters = 4096;

__device__ __forceinline__ uint32_t sm_id() {
  uint32_t s;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(s));
  return s;
}

// Bounded wait of the ring kinds in one of three forms: WK 0 spins on
// mbarrier.test_wait, 1 on try_wait with a suspend-time hint, 2 on try_wait
// without one; the clock is read every 1024 tests.
template <int WK>
__device__ __forceinline__ bool probe_wait(uint32_t bar, uint32_t parity, unsigned long long* err) {
  if (WK == 3) {  // test_wait, bounded by a count of tests, no clock read
    for (uint32_t it = 0; it < (1u << 27); ++it)
      if (mbar_test(bar, parity)) return true;
    atomicOr(err + 2, 1ull);
    return false;
  }
  if (WK == 4) {  // try_wait, bounded by the SM cycle counter
    if (mbar_try(bar, parity)) return true;
    const long long c0 = clock64();
    for (uint32_t it = 1;; ++it) {
      if (mbar_try(bar, parity)) return true;
      if ((it & 15u) == 0 && clock64() - c0 > 4000000000ll) {
        atomicOr(err + 2, 1ull);
        return false;
      }
    }
  }
  const unsigned long long t0 = gtimer_ns();
  for (uint32_t it = 1;; ++it) {
    const bool ok = WK == 0 ? mbar_test(bar, parity) : WK == 1 ? mbar_try_sleep(bar, parity) : mbar_try(bar, parity);
    if (ok) return true;
    if ((it & 1023u) == 0 && gtimer_ns() - t0 > WAIT_LIMIT_NS) {
      atomicOr(err + 2, 1ull);
      return false;
    }
  }
}

// out per CTA: [0] cycles of the MMA stream(s) (sum over issuers), [1]
// tensor-memory transfers done by the side warps, [2] their cycles, [3] error bits
template <int N, int ISS, int COLS, int SIDE>
__global__ void __launch_bounds__(256, 512 / COLS) mma_single(unsigned long long* out, unsigned long long* errs) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* g = smem_raw + (base - raw);
  // B: KST K-steps of 32 x N bytes (32 for the walking kinds, as the kernel's image)
  constexpr int KST = (SIDE >= 7 && N <= 64) ? 32 : 8;
  const uint32_t sB = base, bars = base + KST * 32 * N;
  __shared__ uint32_t s_tmem;
  __shared__ unsigned long long s_mma[4];
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < KST * 32 * N / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(g)[i] = 0x01010101u * (i & 3);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int w = 0; w < 12; ++w) mbar_init(bars + 8 * w, 1);  // [0, ISS): issuers; 4..7: commits; 8..11: free slots
    mbar_fence_init();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  unsigned long long* err = errs + (size_t)blockIdx.x * 4;
  if (warp < ISS && SIDE != 4 && SIDE != 6) {
    const bool leader = elect_one();
    constexpr uint32_t IDESC = idesc_i8(128, N);
    const uint64_t bdesc0 = sdesc_noswz(sB, N * 16, 128);
    constexpr uint32_t BSTEP = (2 * N * 16) >> 4;
    const uint32_t d = tmem + warp * N;
    const uint32_t a = tmem + ISS * N;  // 32 columns of A after the accumulators
    __syncwarp();
    const unsigned long long t0 = clock64();
    if (leader && SIDE < 7) {
      for (int it = 0; it < kIters; ++it) {
        const int st = it & 7;
        tc_mma_i8_ts(d, a + (st & 3) * 8, bdesc0 + st * BSTEP, IDESC, it ? 1u : 0u);
      }
      tc_commit(bars + 8 * warp);
      mbar_wait(bars + 8 * warp, 0, err, 1);
    } else if (leader && SIDE >= 18) {
      // per use: [SIDE 18] wait (ring of 3) + fence + 16 unrolled MMAs with
      // compile-time offsets + commit; [19] no ring: a try_wait on a barrier
      // whose phase 0 is already complete before each use; [20] no ring: two
      // clock reads per use
      const uint32_t ring = bars + 8 * 4, done0 = bars + 8 * 11;
      if (SIDE == 19) {
        tc_commit(done0);  // completes phase 0 once the (no) prior MMAs are done
        mbar_wait(done0, 0, err, 1);
      }
      unsigned long long nwait = 0, wcyc = 0;
      for (int su = 0; su < kIters / 16; ++su) {
        const long long w0 = clock64();
        if (SIDE == 18 && su >= 3) mbar_wait(ring + 8 * (su % 3), ((su / 3) - 1) & 1, err, 1);
        if (SIDE == 19) mbar_try(done0, 0);
        wcyc += (unsigned long long)(clock64() - w0);
        ++nwait;
        tc_fence_after();
        const uint32_t a_t = tmem + 128 + (uint32_t)(su % 3) * 128;
        const uint64_t bd = bdesc0 + (uint64_t)(((su * 16) % KST) * BSTEP);
#pragma unroll
        for (int k = 0; k < 16; ++k)
          tc_mma_i8_ts(d, a_t + k * 8, bd + (uint64_t)(k * BSTEP), IDESC, (su | k) ? 1u : 0u);
        tc_commit(ring + 8 * (su % 3));
      }
      tc_commit(bars + 8 * warp);
      mbar_wait(bars + 8 * warp, 0, err, 1);
      atomicAdd(out + (size_t)blockIdx.x * 4 + 1, nwait);
      atomicAdd(out + (size_t)blockIdx.x * 4 + 2, wcyc);
    } else if (leader) {
      // 16 MMAs (512 samples) per slot use; A slot s at columns 128 + 128 s
      constexpr int P = SIDE == 8 ? 4 : 16;          // MMAs per commit
      // ring slots (0: no waits); SIDE 16 waits for its own last commit
      constexpr int NS = SIDE == 16 ? 1 : (SIDE == 9 || SIDE >= 11) ? 3 : SIDE == 10 ? 2 : 0;
      const uint32_t ring = bars + 8 * 4, freeb = bars + 8 * 8;
      unsigned long long nwait = 0, wcyc = 0;
      for (int it = 0; it < kIters; ++it) {
        const int su = it / 16;  // slot use
        if (NS && (it & 15) == 0 && su >= NS) {
          // SIDE 17: a helper warp waits for the commits and frees the slots
          const uint32_t rb = (SIDE == 17 ? freeb : ring) + 8 * (su % NS), rp = ((su / NS) - 1) & 1;
          const long long w0 = clock64();
          ++nwait;
          if (SIDE == 11) probe_wait<0>(rb, rp, err);
          else if (SIDE == 12) probe_wait<1>(rb, rp, err);
          else if (SIDE == 13) probe_wait<2>(rb, rp, err);
          else if (SIDE == 14) probe_wait<3>(rb, rp, err);
          else if (SIDE == 15) probe_wait<4>(rb, rp, err);
          else mbar_wait(rb, rp, err, 1);
          wcyc += (unsigned long long)(clock64() - w0);
        }
        const uint32_t a_t = tmem + 128 + (uint32_t)(su % 3) * 128 + (uint32_t)(it & 15) * 8;
        tc_mma_i8_ts(d, a_t, bdesc0 + (uint64_t)((it % KST) * BSTEP), IDESC, it ? 1u : 0u);
        if (NS && (it & 15) == 15) tc_commit(ring + 8 * (su % NS));
        else if (!NS && it % P == P - 1) tc_commit(ring);
      }
      tc_commit(bars + 8 * warp);
      mbar_wait(bars + 8 * warp, 0, err, 1);
      if (NS) {  // waits of the issuer: count and cycles
        atomicAdd(out + (size_t)blockIdx.x * 4 + 1, nwait);
        atomicAdd(out + (size_t)blockIdx.x * 4 + 2, wcyc);
      }
    }
    __syncwarp();
    if (leader) s_mma[warp] = clock64() - t0;
  } else if (SIDE == 17 && warp == 4) {
    // helper: waits for each use's commit in order and frees its slot
    if (elect_one()) {
      const uint32_t ring = bars + 8 * 4, freeb = bars + 8 * 8;
      for (int su = 0; su < kIters / 16; ++su) {
        if (!mbar_wait(ring + 8 * (su % 3), (su / 3) & 1, err, 1)) break;
        mbar_arrive(freeb + 8 * (su % 3));
      }
    }
    __syncwarp();
  } else if (SIDE && SIDE <= 6 && warp >= 4) {
    constexpr int SIDE_KIND = SIDE == 4 ? 3 : SIDE == 6 ? 5 : SIDE;  // 4, 6: kinds 3, 5 with no MMAs
    // side traffic on lane quarter (warp & 3), columns 256..287
    const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + 256;
    const unsigned long long t0 = clock64();
    unsigned long long n = 0;
    if (SIDE_KIND == 1) {
      uint32_t o[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) o[k] = (uint32_t)k * 0x01010101u;
      for (int it = 0; it < kIters / 2; ++it, ++n) {
        tc_st32(taddr, o);
        tc_wait_st();
      }
    } else if (SIDE_KIND == 3) {
      uint32_t o[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) o[k] = (uint32_t)k * 0x01010101u;
      for (int it = 0; it < kIters / 8; ++it, n += 4) {
#pragma unroll
        for (int q = 0; q < 4; ++q) tc_st32(taddr + 32 * q, o);  // columns 256..383
        tc_wait_st();
      }
    } else if (SIDE_KIND == 5) {
      // 16 bytes per lane per load, 512 B per warp, walking the B region
      uint32_t acc = 0;
      const uint32_t span = 8 * 32 * N;
      uint32_t off = (threadIdx.x & 127) * 16;
      for (int it = 0; it < kIters * 2; ++it, ++n) {
        uint32_t a0, a1, a2, a3;
        // volatile: the addresses repeat every 8 loads and nothing stores to
        // them, so plain loads could be merged by the compiler
        asm volatile("ld.volatile.shared.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(a0), "=r"(a1), "=r"(a2), "=r"(a3)
                     : "r"(sB + off));
        acc += a0 ^ a1 ^ a2 ^ a3;
        off += 2048;
        if (off >= span) off -= span;
      }
      if (acc == 0x12345678u) err[3] = acc;  // keeps the loads
    } else {
      uint32_t acc = 0;
      for (int it = 0; it < kIters; ++it, ++n) {
        uint32_t r[16];
        tc_ld16(taddr, r);
        tc_wait_ld();
        acc += r[0] ^ r[15];
      }
      if (acc == 0x12345678u) err[3] = acc;  // keeps the loads
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(out + (size_t)blockIdx.x * 4 + 1, n);
      atomicAdd(out + (size_t)blockIdx.x * 4 + 2, clock64() - t0);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (tid == 0) {
    unsigned long long s = 0;
    for (int w = 0; w < ISS; ++w) s += s_mma[w];
    out[(size_t)blockIdx.x * 4] = s;
    out[(size_t)blockIdx.x * 4 + 3] = err[2] | ((unsigned long long)sm_id() << 32);
  }
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(COLS) : "memory");
}

// Ring of NSL A slots of MPU MMAs each (A from column N, one accumulator at
// column 0), the uses issued as unrolled blocks with compile-time offsets.
// Before a slot's next use the issuer waits for the commit of its previous
// use (HOP = 0), or for a helper warp that waits for that commit and then
// arrives on a second barrier (HOP = 1: the hand-off through another role).
// MPU = 0: commits only (the round trip of a commit with no MMA behind it).
// out[0]: cycles of the issuer; [1] uses, [2] the same cycles (cycles per use).
template <int N, int NSL, int MPU, int HOP, int FENCE = 1, int ORDER = 0, int SPIN = 0>
__global__ void __launch_bounds__(256, 1) mma_ring(unsigned long long* out, unsigned long long* errs) {
  constexpr int KST = N <= 64 ? 32 : 8;
  constexpr int USES = MPU ? kIters / MPU : 256;
  static_assert(N > 64 || N + NSL * (MPU ? MPU : 1) * 8 <= 512, "TMEM columns");  // launched for N <= 64
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* g = smem_raw + (base - raw);
  const uint32_t sB = base, commitb = base + KST * 32 * N, freeb = commitb + 8 * 8, fin = freeb + 8 * 8;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_done;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < KST * 32 * N / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(g)[i] = 0x01010101u * (i & 3);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int w = 0; w < 18; ++w) mbar_init(commitb + 8 * w, 1);  // the last: never completed (spinners)
    mbar_fence_init();
    s_done = 0;
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  unsigned long long* err = errs + (size_t)blockIdx.x * 4;
  if (warp == 0) {
    const bool leader = elect_one();
    constexpr uint32_t IDESC = idesc_i8(128, N);
    const uint64_t bdesc0 = sdesc_noswz(sB, N * 16, 128);
    constexpr uint32_t BSTEP = (2 * N * 16) >> 4;
    __syncwarp();
    const unsigned long long t0 = clock64();
    if (leader) {
      unsigned long long wcyc = 0;
      for (int su = 0; su < USES; ++su) {
        const int slot = su % NSL;
        if (ORDER == 1) {
          // this use's slot was waited for before the last commit
          if (FENCE) tc_fence_after();
          const uint32_t a_t = tmem + N + (uint32_t)slot * (MPU * 8);
          const uint64_t bd = bdesc0 + (uint64_t)(((su * MPU) % KST) * BSTEP);
#pragma unroll
          for (int k = 0; k < MPU; ++k)
            tc_mma_i8_ts(tmem, a_t + k * 8, bd + (uint64_t)((k % KST) * BSTEP), IDESC, (su | k) ? 1u : 0u);
          const int nx = su + 1;
          if (nx < USES && nx >= NSL) mbar_wait(commitb + 8 * (nx % NSL), ((nx / NSL) - 1) & 1, err, 1);
          tc_commit(commitb + 8 * slot);
          continue;
        }
        if (su >= NSL) {
          const long long w0 = clock64();
          if (HOP == 2) {  // try_wait with a suspend-time hint
            const uint32_t rb = commitb + 8 * slot, rp = ((su / NSL) - 1) & 1;
            while (!mbar_try_sleep(rb, rp)) {
            }
          } else {
            mbar_wait((HOP ? freeb : commitb) + 8 * slot, ((su / NSL) - 1) & 1, err, 1);
          }
          wcyc += (unsigned long long)(clock64() - w0);
        }
        if (FENCE) tc_fence_after();
        if (MPU) {
          const uint32_t a_t = tmem + N + (uint32_t)slot * (MPU * 8);
          const uint64_t bd = bdesc0 + (uint64_t)(((su * MPU) % KST) * BSTEP);
#pragma unroll
          for (int k = 0; k < MPU; ++k)
            tc_mma_i8_ts(tmem, a_t + k * 8, bd + (uint64_t)((k % KST) * BSTEP), IDESC, (su | k) ? 1u : 0u);
        }
        tc_commit(commitb + 8 * slot);
      }
      tc_commit(fin);
      mbar_wait(fin, 0, err, 1);
      const unsigned long long tot = clock64() - t0;
      s_done = 1;
      out[(size_t)blockIdx.x * 4] = tot;
      out[(size_t)blockIdx.x * 4 + 1] = USES;
      out[(size_t)blockIdx.x * 4 + 2] = tot;
      (void)wcyc;
    }
    __syncwarp();
  } else if (SPIN && warp >= 1) {
    // warps waiting on a barrier that never completes, as the other roles of
    // a kernel wait for theirs: SPIN 1 try_wait, 2 try_wait with a
    // suspend-time hint, 3 try_wait after a 128 ns sleep; bounded by a count
    const uint32_t never = commitb + 8 * 17;
    for (uint32_t it = 0; it < (1u << 22) && !s_done; ++it) {
      if (SPIN == 3) __nanosleep(128);
      const bool r = SPIN == 2 ? mbar_try_sleep(never, 0) : mbar_try(never, 0);
      if (r) break;
    }
  } else if (HOP == 1 && warp == 1) {
    if (elect_one()) {
      for (int su = 0; su < USES; ++su) {
        if (!mbar_wait(commitb + 8 * (su % NSL), (su / NSL) & 1, err, 1)) break;
        mbar_arrive(freeb + 8 * (su % NSL));
      }
    }
    __syncwarp();
  }
  if (tid == 0) out[(size_t)blockIdx.x * 4 + 3] = err[2];
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// Timeline of one issuer (CTA 0) on a ring of NSL A slots of 16 MMAs, N = 64:
// per use, the clock when its wait began, when the wait returned and when
// its last MMA and commit had been issued.  tl: 3 * kIters / 16 values.
// FORM 0: the association kernels' MMA (disable-output-lane mask of four
// zero registers, predicate from a register); 1: no mask; 2: no mask and a
// constant accumulate predicate after the first MMA.
template <int FORM>
__device__ __forceinline__ void mma_form(uint32_t d, uint32_t a, uint64_t bd, uint32_t idesc, uint32_t acc) {
  if (FORM == 0) {
    tc_mma_i8_ts(d, a, bd, idesc, acc);
  } else if (FORM == 1 || acc == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a), "l"(bd), "r"(idesc), "r"(acc)
        : "memory");
  } else {
    asm volatile("tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, 1;" ::"r"(d), "r"(a), "l"(bd), "r"(idesc)
                 : "memory");
  }
}

template <int NSL, int FORM = 0, int MPU = 16>
__global__ void __launch_bounds__(128, 1) mma_ring_timeline(unsigned long long* tl, unsigned long long* errs) {
  constexpr int N = 64, KST = 32, USES = kIters / MPU;
  static_assert(MPU % 16 == 0 && NSL * MPU * 8 + 64 <= 512, "TMEM columns");
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* g = smem_raw + (base - raw);
  const uint32_t sB = base, commitb = base + KST * 32 * N, fin = commitb + 8 * 8;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < KST * 32 * N / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(g)[i] = 0x01010101u * (i & 3);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int w = 0; w < 9; ++w) mbar_init(commitb + 8 * w, 1);
    mbar_fence_init();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  unsigned long long* err = errs + (size_t)blockIdx.x * 4;
  if (warp == 0) {
    const bool leader = elect_one();
    constexpr uint32_t IDESC = idesc_i8(128, N);
    const uint64_t bdesc0 = sdesc_noswz(sB, N * 16, 128);
    constexpr uint32_t BSTEP = (2 * N * 16) >> 4;
    __syncwarp();
    if (leader) {
      const long long t0 = clock64();
      for (int su = 0; su < USES; ++su) {
        const int slot = su % NSL;
        const long long a = clock64();
        if (su >= NSL) mbar_wait(commitb + 8 * slot, ((su / NSL) - 1) & 1, err, 1);
        const long long b = clock64();
        tc_fence_after();
        const uint32_t a_t = tmem + N + (uint32_t)slot * (MPU * 8);
#pragma unroll
        for (int k = 0; k < MPU; ++k)
          mma_form<FORM>(tmem, a_t + k * 8, bdesc0 + (uint64_t)((k % KST) * BSTEP), IDESC, (su | k) ? 1u : 0u);
        tc_commit(commitb + 8 * slot);
        const long long c = clock64();
        if (blockIdx.x == 0) {
          tl[3 * su] = (unsigned long long)(a - t0);
          tl[3 * su + 1] = (unsigned long long)(b - t0);
          tl[3 * su + 2] = (unsigned long long)(c - t0);
        }
      }
      tc_commit(fin);
      mbar_wait(fin, 0, err, 1);
    }
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// The single-phenotype kernel's MMA pipeline rebuilt step by step (N = 64,
// three A slots of 16 MMAs, tiles of two slot uses): ACC2 alternates two
// accumulators tile by tile (the first MMA of a tile overwrites); ACCW adds
// the accumulator hand-off (a commit per tile that an "epilogue" group of
// four warps waits for, and its release that the issuer waits for before
// reusing the buffer); HOPW frees the A slots through a group of four warps
// (each waits for the commit, the slot counts four arrivals) that the issuer
// waits for, instead of waiting for the commit itself.  out[0]: the issuer's
// cycles; [1] uses, [2] the same cycles.
template <int ACC2, int ACCW, int HOPW, int MODE = 0, int BUSY = 0, int ISS2 = 0>
__global__ void __launch_bounds__(576, 1) mma_pipe(unsigned long long* out, unsigned long long* errs) {
  constexpr int N = 64, KST = 32, USES = kIters / 16, NSL = 3;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* g = smem_raw + (base - raw);
  const uint32_t sB = base, a_empty = base + KST * 32 * N, a_full = a_empty + 32, acc_full = a_full + 32,
                 acc_empty = acc_full + 16, fin = acc_empty + 16;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_stop;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < KST * 32 * N / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(g)[i] = 0x01010101u * (i & 3);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    s_stop = 0;
    for (int t = 0; t < NSL; ++t) mbar_init(a_empty + 8 * t, 1), mbar_init(a_full + 8 * t, 4);
    for (int t = 0; t < 2; ++t) mbar_init(acc_full + 8 * t, 1), mbar_init(acc_empty + 8 * t, 4);
    mbar_init(fin, 1);
    mbar_init(fin + 8, 1);
    mbar_fence_init();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  unsigned long long* err = errs + (size_t)blockIdx.x * 4;
  if (ISS2 && (warp == 16 || warp == 17)) {
    // two issuers on two sub-partitions, taking alternate tiles (issuer j:
    // tiles t with t % 2 == j, accumulator j); one thread each, waiting at
    // the top of each use
    const int j = warp - 16;
    const bool leader = elect_one();
    constexpr uint32_t IDESC = idesc_i8(128, N);
    const uint64_t bdesc0 = sdesc_noswz(sB, N * 16, 128);
    constexpr uint32_t BSTEP = (2 * N * 16) >> 4;
    __syncwarp();
    const unsigned long long t0 = clock64();
    if (leader) {
      for (int tile = j; tile < USES / 2; tile += 2) {
        if (tile >= 2) mbar_wait(acc_empty + 8 * j, ((tile >> 1) - 1) & 1, err, 1);
        for (int u = 0; u < 2; ++u) {
          const int su = 2 * tile + u, slot = su % NSL;
          if (su >= NSL) mbar_wait(a_full + 8 * slot, ((su / NSL) - 1) & 1, err, 1);
          tc_fence_after();
          const uint32_t a_t = tmem + 2 * N + (uint32_t)slot * 128;
          const uint32_t d_t = tmem + j * N;
          const uint64_t bd = bdesc0 + (uint64_t)(((su * 16) % KST) * BSTEP);
#pragma unroll
          for (int k = 0; k < 16; ++k)
            tc_mma_i8_ts(d_t, a_t + k * 8, bd + (uint64_t)(k * BSTEP), IDESC, (u | k) ? 1u : 0u);
          tc_commit(a_empty + 8 * slot);
        }
        tc_commit(acc_full + 8 * j);
      }
      tc_commit(fin + 8 * j);
      mbar_wait(fin + 8 * j, 0, err, 1);
      const unsigned long long tot = clock64() - t0;
      if (j == 1) s_stop = 1;
      atomicMax(out + (size_t)blockIdx.x * 4, tot);
      out[(size_t)blockIdx.x * 4 + 1] = USES;
      atomicMax(out + (size_t)blockIdx.x * 4 + 2, tot);
    }
    __syncwarp();
  } else if (!ISS2 && warp == 17) {
    // issuer (the kernel's MMA warp is warp 17)
    const bool leader = elect_one();
    constexpr uint32_t IDESC = idesc_i8(128, N);
    const uint64_t bdesc0 = sdesc_noswz(sB, N * 16, 128);
    constexpr uint32_t BSTEP = (2 * N * 16) >> 4;
    const unsigned long long t0 = clock64();
    const uint32_t slot_bar = HOPW ? a_full : a_empty;
    if (MODE >= 1 && leader) {
      // one thread: MODE 1 waits at the top of each use; 2 as 1 with a tile's
      // accumulator waited for one use earlier; 3 waits for what the next use
      // needs after 8 of this use's 16 MMAs; 4 only tests there
      // (mbarrier.test_wait) and waits after the commits if a test failed
      for (int su = 0; su < USES; ++su) {
        const int slot = su % NSL, tile = su >> 1, b = ACC2 ? (tile & 1) : 0;
        if (MODE == 1) {
          if (ACCW && (su & 1) == 0 && tile >= 2) mbar_wait(acc_empty + 8 * b, ((tile >> 1) - 1) & 1, err, 1);
          if (su >= NSL) mbar_wait(slot_bar + 8 * slot, ((su / NSL) - 1) & 1, err, 1);
        } else if (MODE == 2) {
          if (su >= NSL) mbar_wait(slot_bar + 8 * slot, ((su / NSL) - 1) & 1, err, 1);
          if (ACCW && (su & 1) == 1 && tile + 1 >= 2)
            mbar_wait(acc_empty + 8 * (b ^ 1), (((tile + 1) >> 1) - 1) & 1, err, 1);
        }
        tc_fence_after();
        const uint32_t a_t = tmem + 2 * N + (uint32_t)slot * 128;
        const uint32_t d_t = tmem + b * N;
        const uint64_t bd = bdesc0 + (uint64_t)(((su * 16) % KST) * BSTEP);
        const uint32_t first = ACC2 ? (su & 1) : su;
        const int nx = su + 1, nslot = nx % NSL, ntile = nx >> 1, nb = ACC2 ? (ntile & 1) : 0;
        const bool need_slot = nx < USES && nx >= NSL;
        const bool need_acc = ACCW && nx < USES && (nx & 1) == 0 && ntile >= 2;
        bool slot_ok = true, acc_ok = true;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          if (k == 8 && MODE == 3) {
            if (need_slot) mbar_wait(slot_bar + 8 * nslot, ((nx / NSL) - 1) & 1, err, 1);
            if (need_acc) mbar_wait(acc_empty + 8 * nb, ((ntile >> 1) - 1) & 1, err, 1);
          }
          if (k == 8 && MODE == 4) {
            if (need_slot) slot_ok = mbar_test(slot_bar + 8 * nslot, ((nx / NSL) - 1) & 1);
            if (need_acc) acc_ok = mbar_test(acc_empty + 8 * nb, ((ntile >> 1) - 1) & 1);
          }
          tc_mma_i8_ts(d_t, a_t + k * 8, bd + (uint64_t)(k * BSTEP), IDESC, (first | k) ? 1u : 0u);
        }
        tc_commit(a_empty + 8 * slot);
        if (ACCW && (su & 1) == 1) tc_commit(acc_full + 8 * b);
        if (MODE == 4) {
          if (need_slot && !slot_ok) mbar_wait(slot_bar + 8 * nslot, ((nx / NSL) - 1) & 1, err, 1);
          if (need_acc && !acc_ok) mbar_wait(acc_empty + 8 * nb, ((ntile >> 1) - 1) & 1, err, 1);
        }
      }
    }
    for (int su = 0; su < (MODE ? 0 : USES); ++su) {
      const int slot = su % NSL, tile = su >> 1, b = ACC2 ? (tile & 1) : 0;
      if (ACCW && (su & 1) == 0 && tile >= 2)
        __all_sync(0xffffffffu, mbar_wait(acc_empty + 8 * b, ((tile >> 1) - 1) & 1, err, 1));
      if (su >= NSL)
        __all_sync(0xffffffffu, mbar_wait((HOPW ? a_full : a_empty) + 8 * slot, ((su / NSL) - 1) & 1, err, 1));
      tc_fence_after();
      if (leader) {
        const uint32_t a_t = tmem + 2 * N + (uint32_t)slot * 128;
        const uint32_t d_t = tmem + b * N;
        const uint64_t bd = bdesc0 + (uint64_t)(((su * 16) % KST) * BSTEP);
        const uint32_t first = ACC2 ? (su & 1) : su;  // 0: the tile's first use overwrites
#pragma unroll
        for (int k = 0; k < 16; ++k)
          tc_mma_i8_ts(d_t, a_t + k * 8, bd + (uint64_t)(k * BSTEP), IDESC, (first | k) ? 1u : 0u);
        tc_commit(a_empty + 8 * slot);
        if (ACCW && (su & 1) == 1) tc_commit(acc_full + 8 * b);
      }
      __syncwarp();
    }
    if (leader) {
      tc_commit(fin);
      mbar_wait(fin, 0, err, 1);
      const unsigned long long tot = clock64() - t0;
      s_stop = 1;
      out[(size_t)blockIdx.x * 4] = tot;
      out[(size_t)blockIdx.x * 4 + 1] = USES;
      out[(size_t)blockIdx.x * 4 + 2] = tot;
    }
    __syncwarp();
  } else if (BUSY && ((warp >= 4 && warp < 8) || (warp >= 12 && warp < 16))) {
    // two warps per sub-partition doing integer work, as the unpack warps
    // do (BUSY independent shift-and-mask chains per thread), until the
    // issuer is done; bounded by a count
    // BUSY 8: FP64 multiply-add chains instead (four per thread), as the
    // epilogue's statistics
    uint32_t x[4] = {(uint32_t)tid, (uint32_t)tid * 3u, (uint32_t)tid * 5u, (uint32_t)tid * 7u};
    double f[4] = {1.0 + tid, 2.0 + tid, 3.0 + tid, 4.0 + tid};
    for (uint32_t it = 0; it < (1u << 24) && !s_stop; ++it) {
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        if (BUSY == 8) {
#pragma unroll
          for (int c = 0; c < 4; ++c) f[c] = fma(f[c], 0.999999, 1e-9);
        } else {
#pragma unroll
          for (int c = 0; c < (BUSY < 4 ? BUSY : 4); ++c) x[c] = ((x[c] * 4u) & 0x80808080u) ^ (x[c] + 0x9e3779b9u);
        }
      }
    }
    if ((x[0] ^ x[1] ^ x[2] ^ x[3]) == 0x12345678u || f[0] + f[1] + f[2] + f[3] == 1.5) err[3] = 1;  // keeps the work
  } else if (HOPW && warp >= 8 && warp < 12) {
    // "unpack" group: waits for each slot's commit, then marks it full (4 arrivals)
    for (int su = NSL; su < USES; ++su) {
      const int slot = su % NSL;
      if (!__all_sync(0xffffffffu, mbar_wait(a_empty + 8 * slot, ((su / NSL) - 1) & 1, err, 1))) break;
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(a_full + 8 * slot);
    }
  } else if (ACCW && warp < 4) {
    // "epilogue" group: takes every tile's accumulator (count 4 on release)
    for (int tile = 0; tile < USES / 2; ++tile) {
      const int b = ACC2 ? (tile & 1) : 0;
      if (!__all_sync(0xffffffffu, mbar_wait(acc_full + 8 * b, (ACC2 ? tile >> 1 : tile) & 1, err, 1))) break;
      tc_fence_after();
      uint32_t r[16];
      tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + b * N, r);
      tc_wait_ld();
      if (r[0] == 0x7fffffffu && r[15] == 0x7fffffffu) err[3] = 1;  // keeps the load
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty + 8 * b);
    }
  }
  if (tid == 0) out[(size_t)blockIdx.x * 4 + 3] = err[2];
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// Two issuers (warps 16, 17) with private rings: issuer j takes the tiles t
// with t % 2 == j (two uses of MPU MMAs... each tile is 32 MMAs in uses of
// MPU) into accumulator j, from its own ring of NS2 A slots of MPU * 8
// columns that its own group of four "unpack" warps frees (warps 8-11 for
// ring 0, 12-15 for ring 1; each waits for the slot's commit and arrives on
// its full barrier), and its own "epilogue" group (warps 4j..4j+3) releases
// its accumulator.  out[0]: the slower issuer's cycles.
template <int MPU, int NS2>
__global__ void __launch_bounds__(576, 1) mma_pipe2(unsigned long long* out, unsigned long long* errs) {
  constexpr int N = 64, KST = 32, USES_T = 32 / MPU;  // uses per tile
  constexpr int TILES = kIters / 32;
  static_assert(2 * N + 2 * NS2 * MPU * 8 <= 512, "TMEM columns");
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* g = smem_raw + (base - raw);
  // barriers: a_empty[2][NS2], a_full[2][NS2], acc_full[2], acc_empty[2], fin[2]
  const uint32_t sB = base, a_empty = base + KST * 32 * N, a_full = a_empty + 8 * 2 * NS2,
                 acc_full = a_full + 8 * 2 * NS2, acc_empty = acc_full + 16, fin = acc_empty + 16;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < KST * 32 * N / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(g)[i] = 0x01010101u * (i & 3);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int t = 0; t < 2 * NS2; ++t) mbar_init(a_empty + 8 * t, 1), mbar_init(a_full + 8 * t, 4);
    for (int t = 0; t < 2; ++t) mbar_init(acc_full + 8 * t, 1), mbar_init(acc_empty + 8 * t, 4), mbar_init(fin + 8 * t, 1);
    mbar_fence_init();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  unsigned long long* err = errs + (size_t)blockIdx.x * 4;
  if (warp == 16 || warp == 17) {
    const int j = warp - 16;
    const bool leader = elect_one();
    constexpr uint32_t IDESC = idesc_i8(128, N);
    const uint64_t bdesc0 = sdesc_noswz(sB, N * 16, 128);
    constexpr uint32_t BSTEP = (2 * N * 16) >> 4;
    __syncwarp();
    const unsigned long long t0 = clock64();
    if (leader) {
      int u = 0;  // use of this issuer's ring
      for (int tile = j; tile < TILES; tile += 2) {
        const int it = tile >> 1;  // this issuer's tile count
        if (it >= 1) mbar_wait(acc_empty + 8 * j, (it - 1) & 1, err, 1);
        for (int q = 0; q < USES_T; ++q, ++u) {
          const int slot = u % NS2;
          if (u >= NS2) mbar_wait(a_full + 8 * (j * NS2 + slot), ((u / NS2) - 1) & 1, err, 1);
          tc_fence_after();
          const uint32_t a_t = tmem + 2 * N + (uint32_t)(j * NS2 + slot) * (MPU * 8);
          const uint32_t d_t = tmem + j * N;
          const uint64_t bd = bdesc0 + (uint64_t)(((q * MPU) % KST) * BSTEP);
#pragma unroll
          for (int k = 0; k < MPU; ++k)
            tc_mma_i8_ts(d_t, a_t + k * 8, bd + (uint64_t)(k * BSTEP), IDESC, (q | k) ? 1u : 0u);
          tc_commit(a_empty + 8 * (j * NS2 + slot));
        }
        tc_commit(acc_full + 8 * j);
      }
      tc_commit(fin + 8 * j);
      mbar_wait(fin + 8 * j, 0, err, 1);
      const unsigned long long tot = clock64() - t0;
      atomicMax(out + (size_t)blockIdx.x * 4, tot);
      out[(size_t)blockIdx.x * 4 + 1] = TILES * USES_T;
      atomicMax(out + (size_t)blockIdx.x * 4 + 2, tot);
    }
    __syncwarp();
  } else if (warp >= 8 && warp < 16) {
    // ring j's "unpack" group: frees each slot use after its commit
    const int j = (warp - 8) >> 2;
    const int uses = (TILES / 2) * USES_T;
    for (int u = NS2; u < uses; ++u) {
      const int slot = u % NS2;
      if (!__all_sync(0xffffffffu, mbar_wait(a_empty + 8 * (j * NS2 + slot), ((u / NS2) - 1) & 1, err, 1))) break;
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(a_full + 8 * (j * NS2 + slot));
    }
  } else if (warp < 8) {
    // accumulator j's "epilogue" group
    const int j = warp >> 2;
    for (int it = 0; it < TILES / 2; ++it) {
      if (!__all_sync(0xffffffffu, mbar_wait(acc_full + 8 * j, it & 1, err, 1))) break;
      tc_fence_after();
      uint32_t r[16];
      tc_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + j * N, r);
      tc_wait_ld();
      if (r[0] == 0x7fffffffu && r[15] == 0x7fffffffu) err[3] = 1;  // keeps the load
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty + 8 * j);
    }
  }
  if (tid == 0) out[(size_t)blockIdx.x * 4 + 3] = err[2];
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <int N>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(128, 1)
    mma_pair(unsigned long long* out, unsigned long long* errs) {
  constexpr int NH = N / 2;  // B columns held by each CTA of the pair
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* g = smem_raw + (base - raw);
  const uint32_t sB = base, bar = base + 8 * 32 * NH;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t rank = cluster_rank();
  for (int i = tid; i < 8 * 32 * NH / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(g)[i] = 0x01010101u * (i & 3);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  cluster_sync();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  unsigned long long* err = errs + (size_t)blockIdx.x * 4;
  unsigned long long t0 = clock64();
  if (rank == 0 && warp == 0) {
    const bool leader = elect_one();
    constexpr uint32_t IDESC = idesc_i8(256, N);
    const uint64_t bdesc0 = sdesc_noswz(sB, NH * 16, 128);
    constexpr uint32_t BSTEP = (2 * NH * 16) >> 4;
    __syncwarp();
    t0 = clock64();
    if (leader) {
      for (int it = 0; it < kIters; ++it) {
        const int st = it & 7;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::i8 [%0], [%1], %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n\t}" ::"r"(
                tmem),
            "r"(tmem + 256 + (st & 3) * 8), "l"(bdesc0 + st * BSTEP), "r"(IDESC), "r"(it ? 1u : 0u), "r"(0u)
            : "memory");
      }
      asm volatile(
          "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
              bar),
          "h"((unsigned short)3)
          : "memory");
    }
    __syncwarp();
  }
  if (tid == 0) mbar_wait(bar, 0, err, 1);
  if (tid == 0) {
    out[(size_t)blockIdx.x * 4] = rank == 0 ? clock64() - t0 : 0ull;  // the leader's stream
    out[(size_t)blockIdx.x * 4 + 3] = err[2];
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

struct Result {
  double cycles_per_mma = 0, side_cycles_per_op = 0;
  unsigned long long err = 0;
  int ok = 0;
};

template <class K>
int launch_and_read(K kernel, int grid, int threads, int smem, int per_cta_streams, int side, Result& r) {
  unsigned long long *d = nullptr, *e = nullptr;
  if (cudaMalloc(&d, (size_t)grid * 4 * 8) != cudaSuccess) return 3;
  if (cudaMalloc(&e, (size_t)grid * 4 * 8) != cudaSuccess) {
    cudaFree(d);
    return 3;
  }
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  int rc = 0;
  for (int rep = 0; rep < 3 && rc == 0; ++rep) {
    cudaMemset(d, 0, (size_t)grid * 4 * 8);
    cudaMemset(e, 0, (size_t)grid * 4 * 8);
    kernel<<<grid, threads, smem>>>(d, e);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = 2;
  }
  if (rc == 0) {
    std::vector<unsigned long long> h((size_t)grid * 4);
    cudaMemcpy(h.data(), d, h.size() * 8, cudaMemcpyDeviceToHost);
    double mma = 0, side_ops = 0, side_cyc = 0;
    int ctas = 0;
    for (int b = 0; b < grid; ++b) {
      if (h[4 * b] == 0 && h[4 * b + 1] == 0) continue;  // pair kernels: the peer issues nothing
      mma += (double)h[4 * b];
      side_ops += (double)h[4 * b + 1];
      side_cyc += (double)h[4 * b + 2];
      r.err |= h[4 * b + 3] & 0xffffffffull;
      ++ctas;
    }
    r.cycles_per_mma = ctas && mma > 0 ? mma / ((double)ctas * per_cta_streams * kIters) : 0.0;
    r.side_cycles_per_op = side_ops > 0 ? side_cyc / side_ops : 0.0;
    r.ok = ctas > 0 && r.err == 0;
    (void)side;
  }
  cudaFree(d);
  cudaFree(e);
  return rc;
}

template <int N>
int run_kind(int kind, int issuers, int sms, Result& r) {
  switch (kind) {
    case 0:
      if (issuers == 1) return launch_and_read(mma_single<N, 1, 512, 0>, sms, 256, 150 * 1024, 1, 0, r);
      if (issuers == 2 && 2 * N + 32 <= 512) return launch_and_read(mma_single<N, 2, 512, 0>, sms, 256, 150 * 1024, 2, 0, r);
      if (issuers == 4 && 4 * N + 32 <= 512) return launch_and_read(mma_single<N, 4, 512, 0>, sms, 256, 150 * 1024, 4, 0, r);
      return 1;
    case 1:
      if (N > 224) return 1;
      return launch_and_read(mma_single<N, 1, 256, 0>, 2 * sms, 256, 100 * 1024, 1, 0, r);
    case 2:
      if (N % 32) return 1;
      return launch_and_read(mma_pair<N>, sms & ~1, 128, 150 * 1024, 1, 0, r);
    case 3:
      if (N + 32 > 256) return 1;  // the side warps use columns 256..287
      return launch_and_read(mma_single<N, 1, 512, 1>, sms, 256, 150 * 1024, 1, 1, r);
    case 4:
      if (N + 32 > 256) return 1;
      return launch_and_read(mma_single<N, 1, 512, 2>, sms, 256, 150 * 1024, 1, 2, r);
    case 5:
      if (N + 32 > 256) return 1;  // the side warps use columns 256..383
      return launch_and_read(mma_single<N, 1, 512, 3>, sms, 256, 150 * 1024, 1, 3, r);
    case 6:
      return launch_and_read(mma_single<N, 1, 512, 4>, sms, 256, 150 * 1024, 1, 4, r);
    case 7: return launch_and_read(mma_single<N, 1, 512, 5>, sms, 256, 150 * 1024, 1, 5, r);
    case 8: return launch_and_read(mma_single<N, 1, 512, 6>, sms, 256, 150 * 1024, 1, 6, r);
    // kinds 9-12: accumulator + three 128-column A slots from column 128
    case 9: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 7>, sms, 256, 150 * 1024, 1, 0, r);
    case 10: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 8>, sms, 256, 150 * 1024, 1, 0, r);
    case 11: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 9>, sms, 256, 150 * 1024, 1, 0, r);
    case 12: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 10>, sms, 256, 150 * 1024, 1, 0, r);
    case 13: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 11>, sms, 256, 150 * 1024, 1, 0, r);
    case 14: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 12>, sms, 256, 150 * 1024, 1, 0, r);
    case 15: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 13>, sms, 256, 150 * 1024, 1, 0, r);
    case 16: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 14>, sms, 256, 150 * 1024, 1, 0, r);
    case 17: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 15>, sms, 256, 150 * 1024, 1, 0, r);
    case 18: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 16>, sms, 256, 150 * 1024, 1, 0, r);
    case 19: return N > 128 ? 1 : launch_and_read(mma_single<N, 1, 512, 17>, sms, 256, 150 * 1024, 1, 0, r);
    case 20: return N > 64 ? 1 : launch_and_read(mma_single<N, 1, 512, 18>, sms, 256, 150 * 1024, 1, 0, r);
    case 21: return N > 64 ? 1 : launch_and_read(mma_single<N, 1, 512, 19>, sms, 256, 150 * 1024, 1, 0, r);
    case 22: return N > 64 ? 1 : launch_and_read(mma_single<N, 1, 512, 20>, sms, 256, 150 * 1024, 1, 0, r);
    case 23: return N > 64 ? 1 : launch_and_read(mma_ring<N, 1, 16, 0>, sms, 256, 150 * 1024, 1, 0, r);
    case 24: return N > 64 ? 1 : launch_and_read(mma_ring<N, 1, 1, 0>, sms, 256, 150 * 1024, 1, 0, r);
    case 25: return N > 64 ? 1 : launch_and_read(mma_ring<N, 1, 0, 0>, sms, 256, 150 * 1024, 1, 0, r);
    case 26: return N > 64 ? 1 : launch_and_read(mma_ring<N, 3, 16, 1>, sms, 256, 150 * 1024, 1, 0, r);
    case 27: return N > 64 ? 1 : launch_and_read(mma_ring<N, 6, 8, 0>, sms, 256, 150 * 1024, 1, 0, r);
    case 28: return N > 64 ? 1 : launch_and_read(mma_ring<N, 7, 8, 0>, sms, 256, 150 * 1024, 1, 0, r);
    case 29: return N > 64 ? 1 : launch_and_read(mma_ring<N, 7, 8, 1>, sms, 256, 150 * 1024, 1, 0, r);
    case 30: return N > 64 ? 1 : launch_and_read(mma_ring<N, 3, 16, 0>, sms, 256, 150 * 1024, 1, 0, r);
    case 31: return N > 64 ? 1 : launch_and_read(mma_ring<N, 3, 16, 0, 0>, sms, 256, 150 * 1024, 1, 0, r);
    case 32: return N > 64 ? 1 : launch_and_read(mma_ring<N, 1, 16, 0, 0>, sms, 256, 150 * 1024, 1, 0, r);
    case 33: return N > 64 ? 1 : launch_and_read(mma_ring<N, 3, 16, 2>, sms, 256, 150 * 1024, 1, 0, r);
    case 34: return N > 64 ? 1 : launch_and_read(mma_ring<N, 3, 16, 0, 1, 1>, sms, 256, 150 * 1024, 1, 0, r);
    case 35: return N > 64 ? 1 : launch_and_read(mma_ring<N, 2, 16, 0, 1, 1>, sms, 256, 150 * 1024, 1, 0, r);
    case 36: return N > 64 ? 1 : launch_and_read(mma_ring<N, 6, 8, 0, 1, 1>, sms, 256, 150 * 1024, 1, 0, r);
    case 37: return N > 64 ? 1 : launch_and_read(mma_ring<N, 3, 16, 0, 1, 0, 1>, sms, 256, 150 * 1024, 1, 0, r);
    case 38: return N > 64 ? 1 : launch_and_read(mma_ring<N, 3, 16, 0, 1, 0, 2>, sms, 256, 150 * 1024, 1, 0, r);
    case 39: return N > 64 ? 1 : launch_and_read(mma_ring<N, 3, 16, 0, 1, 0, 3>, sms, 256, 150 * 1024, 1, 0, r);
    case 40: return N != 64 ? 1 : launch_and_read(mma_pipe<0, 0, 0>, sms, 576, 150 * 1024, 1, 0, r);
    case 41: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 0, 0>, sms, 576, 150 * 1024, 1, 0, r);
    case 42: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 0>, sms, 576, 150 * 1024, 1, 0, r);
    case 43: return N != 64 ? 1 : launch_and_read(mma_pipe<0, 0, 1>, sms, 576, 150 * 1024, 1, 0, r);
    case 44: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1>, sms, 576, 150 * 1024, 1, 0, r);
    case 45: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 1>, sms, 576, 150 * 1024, 1, 0, r);
    case 46: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 2>, sms, 576, 150 * 1024, 1, 0, r);
    case 47: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 3>, sms, 576, 150 * 1024, 1, 0, r);
    case 48: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 4>, sms, 576, 150 * 1024, 1, 0, r);
    case 49: return N != 64 ? 1 : launch_and_read(mma_pipe<0, 0, 1, 1>, sms, 576, 150 * 1024, 1, 0, r);
    case 50: return N != 64 ? 1 : launch_and_read(mma_pipe<0, 0, 1, 3>, sms, 576, 150 * 1024, 1, 0, r);
    case 51: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 0, 2>, sms, 576, 150 * 1024, 1, 0, r);
    case 52: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 3, 2>, sms, 576, 150 * 1024, 1, 0, r);
    case 53: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 0, 4>, sms, 576, 150 * 1024, 1, 0, r);
    case 54: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 3, 4>, sms, 576, 150 * 1024, 1, 0, r);
    case 55: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 1, 0, 1>, sms, 576, 150 * 1024, 1, 0, r);
    case 56: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 1, 2, 1>, sms, 576, 150 * 1024, 1, 0, r);
    case 57: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 1, 4, 1>, sms, 576, 150 * 1024, 1, 0, r);
    case 58: return N != 64 ? 1 : launch_and_read(mma_pipe2<8, 3>, sms, 576, 150 * 1024, 1, 0, r);
    case 59: return N != 64 ? 1 : launch_and_read(mma_pipe2<8, 2>, sms, 576, 150 * 1024, 1, 0, r);
    case 60: return N != 64 ? 1 : launch_and_read(mma_pipe2<16, 1>, sms, 576, 150 * 1024, 1, 0, r);
    case 61: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 1, 8, 1>, sms, 576, 150 * 1024, 1, 0, r);
    case 62: return N != 64 ? 1 : launch_and_read(mma_pipe<1, 1, 1, 0, 8>, sms, 576, 150 * 1024, 1, 0, r);
    default: return 1;
  }
}

}  // namespace

// Average cycles per MMA of one issuing stream (kinds 0, 1, 3, 4) or per
// pair MMA (kind 2), and for kinds 3 and 4 the side warps' cycles per
// tcgen05.st / tcgen05.ld.  Returns 0 on success, 1 for an unsupported
// (kind, N, issuers), 2 for a CUDA error, 3 when out of memory; *err gets the
// error bits of the bounded waits (0 when none gave up).
extern "C" int kg_bench_mma_rate(int kind, int n_cols, int issuers, double* cycles_per_mma,
                                 double* side_cycles_per_op, unsigned long long* err) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  Result r;
  int rc = 1;
  switch (n_cols) {
    case 32: rc = run_kind<32>(kind, issuers, sms, r); break;
    case 64: rc = run_kind<64>(kind, issuers, sms, r); break;
    case 80: rc = kind == 2 ? 1 : run_kind<80>(kind, issuers, sms, r); break;
    case 128: rc = run_kind<128>(kind, issuers, sms, r); break;
    case 160: rc = run_kind<160>(kind, issuers, sms, r); break;
    case 256: rc = kind == 1 ? 1 : run_kind<256>(kind, issuers, sms, r); break;
    default: rc = 1;
  }
  if (cycles_per_mma) *cycles_per_mma = r.cycles_per_mma;
  if (side_cycles_per_op) *side_cycles_per_op = r.side_cycles_per_op;
  if (err) *err = r.err;
  return rc;
}

// Timeline of CTA 0 on a ring of nsl (1..3) A slots of 16 MMAs (N = 64) in
// MMA form `form` (see mma_form), or (nsl 4) one slot of 48 MMAs, one CTA per
// SM: 3 clocks per use (wait began, wait returned, use issued), relative to
// the first use; out holds 3 * 256 values.  0 on success.
extern "C" int kg_bench_mma_timeline(int nsl, int form, unsigned long long* out) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t n = 3 * (kIters / 16);
  unsigned long long *d = nullptr, *e = nullptr;
  if (cudaMalloc(&d, n * 8) != cudaSuccess) return 3;
  if (cudaMalloc(&e, (size_t)sms * 4 * 8) != cudaSuccess) {
    cudaFree(d);
    return 3;
  }
  cudaMemset(e, 0, (size_t)sms * 4 * 8);
  // nsl 1..3 with form 0..2; nsl 4: one slot of 48 MMAs per use (form 0)
  auto k = nsl == 4 ? mma_ring_timeline<1, 0, 48>
           : form == 1 ? (nsl == 1 ? mma_ring_timeline<1, 1> : nsl == 2 ? mma_ring_timeline<2, 1> : mma_ring_timeline<3, 1>)
           : form == 2 ? (nsl == 1 ? mma_ring_timeline<1, 2> : nsl == 2 ? mma_ring_timeline<2, 2> : mma_ring_timeline<3, 2>)
                       : (nsl == 1 ? mma_ring_timeline<1> : nsl == 2 ? mma_ring_timeline<2> : mma_ring_timeline<3>);
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
  int rc = 0;
  for (int rep = 0; rep < 2 && rc == 0; ++rep) {
    k<<<sms, 128, 100 * 1024>>>(d, e);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = 2;
  }
  if (rc == 0 && cudaMemcpy(out, d, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess) rc = 2;
  cudaFree(d);
  cudaFree(e);
  return rc;
}
