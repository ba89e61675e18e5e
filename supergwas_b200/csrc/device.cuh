// device.cuh -- parameters, PTX helpers and the shared FP64 epilogue of the
// association kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "params.hpp"

namespace kg {

// A bounded wait gives up after this long and reports KG_ERR_TIMEOUT.
constexpr unsigned long long WAIT_LIMIT_NS = 2000000000ull;

__device__ __forceinline__ unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Exact int64 -> double for |v| < 2^51 without the conversion unit: the
// double 1.5 * 2^52 has unit spacing and a zero low 51-bit mantissa field, so
// adding v to its bit pattern yields the double 1.5 * 2^52 + v exactly
// ("magic number" conversion, Hacker's Delight ch. 17 style).  The caller
// subtracts the bias, usually folded into an FMA.
constexpr double MAGIC_BIAS = 6755399441055744.0;  // 1.5 * 2^52
__device__ __forceinline__ double magic_raw(long long v) {
  return __longlong_as_double(0x4338000000000000LL + v);
}
__device__ __forceinline__ double i2d_exact(long long v) { return magic_raw(v) - MAGIC_BIAS; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Non-blocking test of a phase (mbarrier.test_wait never suspends the thread).
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// As mbar_try, letting the hardware suspend the thread until the phase
// completes (or about 1 ms passes) instead of returning at once, so that a
// waiting warp takes no issue slots from the warps doing the work.
__device__ __forceinline__ bool mbar_try_sleep(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(1000000u)
      : "memory");
  return ok != 0;
}
// Bounded wait: false (and an error bit in counters[2]) after WAIT_LIMIT_NS.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          unsigned long long* counters, unsigned code) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtimer_ns();
  while (!mbar_try(bar, parity)) {
    if (gtimer_ns() - t0 > WAIT_LIMIT_NS) {
      atomicOr(counters + 2, (unsigned long long)code);
      return false;
    }
  }
  return true;
}

// ----------------------------------------------------------- bulk copies
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---------------------------------------------------------------- tcgen05
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
// D[tmem] (+)= A[smem desc] * B[smem desc], kind::i8, int32 accumulate.
__device__ __forceinline__ void tc_mma_i8_ss(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
// D[tmem] (+)= A[tmem] * B[smem desc], kind::i8.
__device__ __forceinline__ void tc_mma_i8_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
// One lane of a converged warp (the lowest active one), chosen by elect.sync.
__device__ __forceinline__ bool elect_one() {
  uint32_t e;
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "elect.sync _|P, 0xffffffff;\n\t"
      "selp.b32 %0, 1, 0, P;\n\t}"
      : "=r"(e));
  return e != 0;
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 32 lanes x 32-bit, 16 consecutive columns per thread.
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// Orders later uses of 16 registers after the preceding tcgen05.wait::ld:
// the registers pass through an (empty) volatile asm that follows the wait.
__device__ __forceinline__ void reg_fence16(uint32_t* r) {
  asm volatile(""
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15]));
}
// 32 lanes x 32-bit, 16 consecutive columns per thread, into r[0..15] (no wait).
__device__ __forceinline__ void tc_ld16p(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// 32 lanes x 32-bit, 8 consecutive columns per thread.
__device__ __forceinline__ void tc_st8(uint32_t taddr, const uint32_t (&r)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(r[0]),
               "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
               : "memory");
}

// Shared-memory matrix descriptor, K-major, no swizzle (core matrix = 8 rows
// x 16 bytes contiguous); lbo = byte distance of K-adjacent core matrices,
// sbo = byte distance of M/N-adjacent 8-row groups.
__device__ __forceinline__ uint64_t sdesc_noswz(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;               // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor: kind::i8, s8 x s8 -> s32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ------------------------------------------- TMEM-A kernels (shared parts)
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

// 128 packed samples (four 32-bit words) -> 32 TMEM columns of int8 A
// operand: column 8q+jj holds, in byte t, sample 32q + 8t + 7 - jj as -128 x
// (jj even) or 64 x (jj odd).  make_b_image_ts lays B out to match.
__device__ __forceinline__ void unpack_stage(const uint32_t (&w)[4], uint32_t (&o)[32]) {
#pragma unroll
  for (int qq = 0; qq < 4; ++qq)
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const uint32_t u = w[qq] * (1u << (2 * h));
      o[qq * 8 + 2 * h] = u & 0x80808080u;
      o[qq * 8 + 2 * h + 1] = u & 0x40404040u;
    }
}

// Bounded wait that also gives up when another role has aborted.  The first
// test is inline (the common case: the phase is already complete); the
// abort flag and the clock are read only every 16 failed tests.  limit_ns:
// how long to wait before giving up (a launch parameter, see wait_limit).
__device__ __forceinline__ bool wait_or_abort(uint32_t bar, uint32_t parity, volatile int* abort,
                                        unsigned long long* counters, unsigned code,
                                        unsigned long long limit_ns = WAIT_LIMIT_NS) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtimer_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_sleep(bar, parity)) return true;
    if ((it & 15u) == 0) {
      if (*abort) return false;
      if (gtimer_ns() - t0 > limit_ns) {
        atomicOr(counters + 2, (unsigned long long)code);
        *abort = 1;
        return false;
      }
    }
  }
}

// The pipeline wait limit of a launch: the caller's value, or WAIT_LIMIT_NS
// when it left it at 0.  Only the waits between the roles of a pipeline use
// it; the final waits for a CTA's own copies and MMAs always allow
// WAIT_LIMIT_NS, so that nothing is still landing when a CTA exits.
__device__ __forceinline__ unsigned long long wait_limit(unsigned long long ns) {
  return ns ? ns : WAIT_LIMIT_NS;
}

// Ring position: slot index and phase parity, advanced without division.
template <int NS>
struct Ring {
  uint32_t slot = 0, phase = 0, used = 0;  // used: laps completed (0 = first)
  __device__ __forceinline__ void next() {
    if (++slot == (uint32_t)NS) {
      slot = 0;
      phase ^= 1u;
      used = 1;
    }
  }
};
// The same with a size chosen at launch.
struct RingN {
  uint32_t slot = 0, phase = 0, used = 0, size;
  __device__ __forceinline__ explicit RingN(uint32_t n) : size(n) {}
  __device__ __forceinline__ void next() {
    if (++slot == size) {
      slot = 0;
      phase ^= 1u;
      used = 1;
    }
  }
};

// ---------------------------------------------------------------- epilogue
// -log10 erfc(z) without underflow (log-domain tail through erfcx).
__device__ __forceinline__ double mlog10_sf(double T) {
  if (!(T > 0.0)) return 0.0;
  const double z = sqrt(0.5 * T);
  if (z < 5.0) return -log10(erfc(z));
  return (z * z - log(erfcx(z))) * 0.43429448190325182765;
}

// Warp-aggregated outputs of one k-mer: tested count, hit record, FP64
// refinement candidate, and (when requested) the per-k-mer arrays.  All 32
// lanes of the warp must call it.
// Warp-aggregated hit records and refinement candidates of one k-mer per
// lane.  All 32 lanes of the warp must call it.
__device__ __forceinline__ void emit_rare(const DevOut& O, unsigned long long local, bool hit, bool cand, double T,
                                          double p, double effect) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned hmask = __ballot_sync(0xffffffffu, hit);
  if (hmask) {
    unsigned long long base = 0;
    const int leader = __ffs(hmask) - 1;
    if ((int)lane == leader) base = atomicAdd(O.counters + 1, (unsigned long long)__popc(hmask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (hit) {
      const unsigned long long slot = base + __popc(hmask & ((1u << lane) - 1u));
      if (slot < O.hit_cap) {
        kg_hit h;
        h.kmer = O.kmer_offset + local;
        h.effect = effect;
        h.pval = p;
        h.chisq = T;
        O.hits[slot] = h;
      } else {
        atomicOr(O.counters + 2, (unsigned long long)ERR_HIT_OVERFLOW);
      }
    }
  }
  const unsigned cmask = __ballot_sync(0xffffffffu, cand);
  if (cmask) {
    unsigned long long base = 0;
    const int leader = __ffs(cmask) - 1;
    if ((int)lane == leader) base = atomicAdd(O.counters + 3, (unsigned long long)__popc(cmask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (cand) {
      const unsigned long long slot = base + __popc(cmask & ((1u << lane) - 1u));
      if (slot < O.cand_cap) O.cand[slot] = O.kmer_offset + local;
      else atomicOr(O.counters + 2, (unsigned long long)ERR_CAND_OVERFLOW);
    }
  }
}

__device__ __forceinline__ void emit_kmer(const DevOut& O, unsigned long long local, bool valid, bool tested,
                                          bool hit, bool cand, double T, double p, double effect, double xxM,
                                          double xyM, double cor) {
  const unsigned lane = threadIdx.x & 31u;
  if (O.weight) {
    const unsigned tot = __reduce_add_sync(0xffffffffu, tested ? O.weight[O.kmer_offset + local] : 0u);
    if (lane == 0 && tot) atomicAdd(O.counters + 0, (unsigned long long)tot);
  } else {
    const unsigned tmask = __ballot_sync(0xffffffffu, tested);
    if (lane == 0 && tmask) atomicAdd(O.counters + 0, (unsigned long long)__popc(tmask));
  }
  emit_rare(O, local, hit, cand, T, p, effect);
  if (valid && O.tested) {
    const unsigned long long g = O.kmer_offset + local;
    O.tested[g] = tested ? 1 : 0;
    O.chisq[g] = T;
    O.pval[g] = p;
    O.effect[g] = effect;
    O.mlog10p[g] = tested ? mlog10_sf(T) : 0.0;
    O.xxM[g] = xxM;
    O.xyM[g] = xyM;
    O.cor[g] = cor;
  }
}

// Statistics and outputs of one k-mer, given c = popcount(x),
// ss = sum_j s_j^2, gs = sum_j g_j e_j, ey = d_y . x.  Must be called by
// all 32 lanes of a warp (warp-aggregated atomics).
__device__ __forceinline__ void finish_kmer(const EpiParams& P, const DevOut& O, unsigned long long local,
                                            bool valid, int c, double ss, double gs, double ey) {
  const int n = P.n;
  bool tested = valid && c > 0 && c < n && !(P.ynorm < 1e-12);
  double cor = 0.0;
  if (tested) {
    const double xcn2 = (double)c * (double)(n - c) / (double)n;  // ||x - mean x||^2
    const double xyc = ey + gs + P.kappa * (double)c;              // x . (y - mean y)
    cor = xyc / (sqrt(xcn2) * P.ynorm);
    tested = !(fabs(cor) < P.corr_thr);                             // src/kgwas.cpp:199,467
  }
  double xxM = 0, xyM = 0, effect = 0, T = 0, p = 1;
  bool cand = false;
  if (tested) {
    xxM = (double)c - ss;
    xyM = P.b * (double)c + ey;
    // compute_hit, src/kgwas.cpp:44-56
    const double eps = 1e-12;
    if (xxM > eps && P.yyM > eps) {
      double r2 = (xyM * xyM) / (xxM * P.yyM);
      if (r2 < 0) r2 = 0;
      if (r2 >= 1) r2 = 1 - 1e-15;
      if (P.refine && r2 >= P.r2_ref) {
        cand = true;  // recomputed in FP64 by refine_kernel, which emits its row
        p = 2.0;
      } else if (O.tested || r2 >= P.r2_cand) {
        T = (double)n * log(1.0 / (1.0 - r2));
        p = erfc(sqrt(0.5 * T));
        effect = xyM / (xxM * P.yyM);
      } else {
        p = 2.0;  // provably above p_thresh; the row is not emitted and no stats are kept
      }
    }
  }
  emit_kmer(O, local, valid, tested, tested && p <= P.p_thresh, cand, T, p, effect, xxM, xyM, cor);
}


// As finish_kmer, for launches without per-k-mer outputs: the Pearson gate
// and the emit / refinement screens compare squares instead of dividing
// (|cor| >= thr  <=>  xyc^2 >= thr^2 ||xc||^2 ||yc||^2;  r2 >= t  <=>
// xyM^2 >= t xxM yyM), and only k-mers that may reach the emit cut evaluate
// the reference formula (src/kgwas.cpp:47-53) exactly.
__device__ __forceinline__ void finish_kmer_fast(const EpiParams& P, const DevOut& O, unsigned long long local,
                                                 bool valid, int c, double ss, double gs, double ey) {
  const int n = P.n;
  bool tested = valid && c > 0 && c < n && !(P.ynorm < 1e-12);
  if (tested && P.corr_thr > 0.0) {
    const double xcn2 = (double)c * (double)(n - c) / (double)n;
    const double xyc = ey + gs + P.kappa * (double)c;
    tested = xyc * xyc >= P.thr2_ynorm2 * xcn2;
  }
  double xxM = 0, xyM = 0, effect = 0, T = 0, p = 1;
  bool cand = false, hit = false;
  if (tested) {
    const double cd = i2d_exact(c);
    xxM = cd - ss;
    xyM = P.b * cd + ey;
    const double eps = 1e-12;
    if (xxM > eps && P.yyM > eps) {
      const double q = xyM * xyM, den = xxM * P.yyM;
      if (P.refine && q >= P.r2_ref * den) {
        cand = true;
      } else if (q >= P.r2_cand * den) {
        double r2 = q / den;
        if (r2 < 0) r2 = 0;
        if (r2 >= 1) r2 = 1 - 1e-15;
        T = (double)n * log(1.0 / (1.0 - r2));
        p = erfc(sqrt(0.5 * T));
        effect = xyM / den;
        hit = p <= P.p_thresh;
      }
    }
  }
  emit_kmer(O, local, valid, tested, hit, cand, T, p, effect, xxM, xyM, 0.0);
}

// Fast screen of one k-mer for kernels that count tested k-mers in a
// register (tested_local, flushed once per warp by the caller): in the common
// case (no hit, no refinement candidate in the warp) it costs one ballot.
// Same decisions and values as finish_kmer_fast.
__device__ __forceinline__ void finish_kmer_lean(const EpiParams& P, const DevOut& O, unsigned long long local,
                                                 bool valid, int c, double cd, double ss, double gs, double ey,
                                                 uint32_t& tested_local) {
  const int n = P.n;
  bool tested = valid && c > 0 && c < n && !(P.ynorm < 1e-12);
  if (P.corr_thr > 0.0) {
    const double xcn2 = cd * (double)(n - c) / (double)n;
    const double xyc = ey + gs + P.kappa * cd;
    tested = tested && xyc * xyc >= P.thr2_ynorm2 * xcn2;
  }
  if (tested) tested_local += O.weight ? O.weight[O.kmer_offset + local] : 1u;
  const double eps = 1e-12;
  const double xxM = cd - ss;
  const double xyM = P.b * cd + ey;
  const double q = xyM * xyM, den = xxM * P.yyM;
  const bool ok = tested && xxM > eps && P.yyM > eps;
  const bool cand = ok && P.refine && q >= P.r2_ref * den;
  const bool maybe = ok && !cand && q >= P.r2_cand * den;
  if (__ballot_sync(0xffffffffu, cand || maybe) == 0u) return;
  double T = 0, p = 1, effect = 0;
  bool hit = false;
  if (maybe) {
    double r2 = q / den;
    if (r2 < 0) r2 = 0;
    if (r2 >= 1) r2 = 1 - 1e-15;
    T = (double)n * log(1.0 / (1.0 - r2));
    p = erfc(sqrt(0.5 * T));
    effect = xyM / den;
    hit = p <= P.p_thresh;
  }
  emit_rare(O, local, hit, cand, T, p, effect);
}

// Adds the per-thread tested counts of a warp to counters[0].
__device__ __forceinline__ void flush_tested(const DevOut& O, uint32_t tested_local) {
  const unsigned tot = __reduce_add_sync(0xffffffffu, tested_local);
  if ((threadIdx.x & 31u) == 0 && tot) atomicAdd(O.counters + 0, (unsigned long long)tot);
}

// ------------------------------------------------- FP64 refinement sums
// Column sums x . v_j of one packed row from byte tables: T[(g*256 + b)*CM + j]
// is the sum of column j over the samples of 8-sample group g whose bit is set
// in b.  Lane l accumulates columns l, l+32, ... over the row's bytes in
// order, one coalesced table row per byte (instead of one V row per set bit).
// nwords: words of the row covered by the tables.  With row2, the column is
// the product of two rows (AND of their words: the 2-D pair test).  Called by
// a whole warp.
template <int CM>
__device__ __forceinline__ void table_row_sums(const uint64_t* __restrict__ row, int nwords,
                                               const double* __restrict__ T, int lane,
                                               double (&acc)[(CM + 31) / 32],
                                               const uint64_t* __restrict__ row2 = nullptr) {
  constexpr int JW = (CM + 31) / 32;
#pragma unroll
  for (int jj = 0; jj < JW; ++jj) acc[jj] = 0.0;
  for (int w = 0; w < nwords; ++w) {
    uint64_t bits = __ldg(row + w);  // one address for the whole warp
    if (row2) bits &= __ldg(row2 + w);
    const double* Tw = T + (size_t)w * (8 * 256 * CM);
    double v[8][JW];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const unsigned b = (unsigned)(bits >> (8 * t)) & 255u;
      const double* e = Tw + (size_t)(t * 256 + b) * CM;
#pragma unroll
      for (int jj = 0; jj < JW; ++jj) {
        const int j = lane + 32 * jj;
        v[t][jj] = (j < CM) ? __ldg(e + j) : 0.0;
      }
    }
#pragma unroll
    for (int t = 0; t < 8; ++t)
#pragma unroll
      for (int jj = 0; jj < JW; ++jj) acc[jj] += v[t][jj];
  }
}

// From the lane-distributed column sums (column 0 = count, 1..k = U columns,
// k+1 = y'): c, ss = sum_j (a_j c + e_j)^2 and ey, identical in every lane.
template <int CM>
__device__ __forceinline__ void refine_reduce(const EpiParams& P, const double (&acc)[(CM + 31) / 32], int lane,
                                              int& c, double& ss, double& ey) {
  constexpr int JW = (CM + 31) / 32;
  c = (int)__shfl_sync(0xffffffffu, acc[0], 0);
  const double cd = (double)c;
  double s2 = 0.0, y = 0.0;
#pragma unroll
  for (int jj = 0; jj < JW; ++jj) {
    const int j = lane + 32 * jj;
    if (j >= 1 && j <= P.k) {
      const double sj = P.a[j - 1] * cd + acc[jj];
      s2 += sj * sj;
    } else if (j == P.k + 1) {
      y = acc[jj];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    y += __shfl_xor_sync(0xffffffffu, y, o);
  }
  ss = s2;
  ey = y;
}

// ------------------------------------------------ many-phenotype helpers
// Shard of a global k-mer index (shard_start ascending, shard_start[0] = 0).
__device__ __forceinline__ int mp_shard(const DevOutMP& O, unsigned long long gk) {
  int lo = 0, hi = O.n_shards - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (O.shard_start[mid] <= gk) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Statistic of one (k-mer, phenotype) from the exact integer sums, as the
// division-free screen of finish_kmer_fast; writes the outcome flags.
__device__ __forceinline__ void mp_eval(const EpiParams& P, bool valid, int c, double ss, double gs, double ey,
                                        bool& tested, bool& hit, bool& cand, double& T, double& p, double& effect) {
  const int n = P.n;
  tested = valid && c > 0 && c < n && !(P.ynorm < 1e-12);
  if (tested && P.corr_thr > 0.0) {
    const double xcn2 = (double)c * (double)(n - c) / (double)n;
    const double xyc = ey + gs + P.kappa * (double)c;
    tested = xyc * xyc >= P.thr2_ynorm2 * xcn2;
  }
  hit = cand = false;
  T = 0;
  p = 1;
  effect = 0;
  if (!tested) return;
  const double xxM = (double)c - ss, xyM = P.b * (double)c + ey;
  const double eps = 1e-12;
  if (!(xxM > eps && P.yyM > eps)) {
    hit = p <= P.p_thresh;
    return;
  }
  const double q = xyM * xyM, den = xxM * P.yyM;
  if (P.refine && q >= P.r2_ref * den) {
    cand = true;
  } else if (q >= P.r2_cand * den) {
    double r2 = q / den;
    if (r2 < 0) r2 = 0;
    if (r2 >= 1) r2 = 1 - 1e-15;
    T = (double)n * log(1.0 / (1.0 - r2));
    p = erfc(sqrt(0.5 * T));
    effect = xyM / den;
    hit = p <= P.p_thresh;
  }
}

// Warp-aggregated hit records and FP64 refinement candidates (k-mer |
// phenotype << 48) of one (k-mer, phenotype) per lane.  mp_emit adds the
// tested count of (shard, phenotype) with one atomic per shard present in the
// warp (match = the lanes of this lane's shard, leader = the lowest of them).
// All 32 lanes of the warp must call them.
__device__ __forceinline__ void mp_emit_rare(const DevOutMP& O, int p, unsigned long long gk, int shard, bool hit,
                                             bool cand, double T, double pv, double effect) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned hm = __ballot_sync(0xffffffffu, hit);
  if (hm) {
    unsigned long long hb = 0;
    const int hl = __ffs(hm) - 1;
    if ((int)lane == hl) hb = atomicAdd(O.counters + 1, (unsigned long long)__popc(hm));
    hb = __shfl_sync(0xffffffffu, hb, hl);
    if (hit) {
      const unsigned long long slot = hb + __popc(hm & ((1u << lane) - 1u));
      if (slot < O.hit_cap) {
        kg_phit hrec;
        hrec.kmer = gk;
        hrec.pheno = p;
        hrec.shard = shard;
        hrec.effect = effect;
        hrec.pval = pv;
        hrec.chisq = T;
        O.hits[slot] = hrec;
      } else {
        atomicOr(O.counters + 2, (unsigned long long)ERR_HIT_OVERFLOW);
      }
    }
  }
  const unsigned cm = __ballot_sync(0xffffffffu, cand);
  if (cm) {
    unsigned long long cb = 0;
    const int cl = __ffs(cm) - 1;
    if ((int)lane == cl) cb = atomicAdd(O.counters + 3, (unsigned long long)__popc(cm));
    cb = __shfl_sync(0xffffffffu, cb, cl);
    if (cand) {
      const unsigned long long slot = cb + __popc(cm & ((1u << lane) - 1u));
      if (slot < O.cand_cap) O.cand[slot] = gk | ((unsigned long long)p << 48);
      else atomicOr(O.counters + 2, (unsigned long long)ERR_CAND_OVERFLOW);
    }
  }
}

__device__ __forceinline__ void mp_emit(const DevOutMP& O, int p, unsigned long long gk, int shard, unsigned match,
                                        bool leader, bool tested, bool hit, bool cand, double T, double pv,
                                        double effect) {
  if (O.weight) {
    // the lanes of one shard (match) add their rows' weights
    const unsigned tot = __reduce_add_sync(match, tested ? O.weight[gk] : 0u);
    if (leader && tot) atomicAdd(O.tested + (size_t)shard * O.n_pheno + p, (unsigned long long)tot);
  } else {
    const unsigned tm = __ballot_sync(0xffffffffu, tested);
    if (leader && (tm & match))
      atomicAdd(O.tested + (size_t)shard * O.n_pheno + p, (unsigned long long)__popc(tm & match));
  }
  mp_emit_rare(O, p, gk, shard, hit, cand, T, pv, effect);
}

}  // namespace kg
