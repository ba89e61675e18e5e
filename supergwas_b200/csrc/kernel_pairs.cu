// kernel_pairs.cu -- the 2-D pair test on the TMEM-A pipeline.
//
// The reference's kgwas_2d (src/kgwas_2d.cpp:237-331) tests every pair
// i < j of its k-mers with the 1-D statistic applied to the product column
// x12 = x_i * x_j: a33 = popcount(x12), xxM = a33 - ||U^T x12||^2,
// xyM = x12.y - (U^T x12).(U^T y), compute_hit.  That is exactly the
// contraction kernel_ts.cu runs, with A = the AND of two packed rows.  A tile
// here is 128 pairs (i, j) sharing i, j in one 128-row j-block:
//   producer  TMA-loads the j-block's packed rows once per unit (a unit is up
//             to `ic` consecutive i of one j-block), no multicast;
//   unpack    ANDs each 128-sample chunk of the resident j rows with the same
//             chunk of row i (a warp-uniform global load) and writes the int8
//             A operand into TMEM (unpack_stage);
//   MMA       tcgen05.mma kind::i8 against the resident limb image;
//   epilogue  limb recombination and the FP64 statistic; pairs that may pass
//             the cut (chi-square >= 12) go to the FP64 refinement list,
//             which pr_refine_kernel recomputes from byte tables.
// Every wait is bounded (KG_ERR_TIMEOUT), as in kernel_ts.cu.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "device.cuh"
#include "kernels.hpp"

namespace kg {

constexpr int PR_TM = 128;
constexpr int PR_KS = 128;
constexpr int PR_SUPER = 4;
constexpr int PR_BOX = 1024;
constexpr uint32_t PR_XBYTES = PR_TM * 128;
constexpr int PR_LU = 3, PR_LY = 5;
constexpr int PR_MAXSLOT = 3;
constexpr int PR_XST_MAX = 12;
constexpr int PR_NBOX_MAX = 8;  // rows of up to 1 KB: 8192 samples
constexpr int PR_WARP_UNPACK0 = 8;

__host__ __device__ constexpr int pr_ug(int N) { return N <= 80 ? 2 : 1; }
__host__ __device__ constexpr int pr_threads(int N) { return 32 * (8 + 4 * pr_ug(N) + 2); }
__host__ __device__ constexpr int pr_nslot(int N) {
  return (512 - 2 * N) / 128 > PR_MAXSLOT ? PR_MAXSLOT : (512 - 2 * N) / 128;
}

struct PrSmem {
  uint32_t x, b, bars, tmem, abort, total;
};
__host__ __device__ inline PrSmem pr_smem(int b_bytes, int xst) {
  PrSmem L;
  L.x = 0;
  L.b = xst * PR_XBYTES;
  L.bars = L.b + ((b_bytes + 127) / 128) * 128;
  L.tmem = L.bars + 8 * (2 * PR_XST_MAX + 2 * PR_MAXSLOT + 4 + 2);
  L.abort = L.tmem + 8;
  L.total = L.abort + 8;
  return L;
}

struct PairUnit {
  unsigned long long jb, i0, i1;
};
// Unit u -> its j-block (the last block whose first unit is <= u) and i range.
__device__ __forceinline__ PairUnit pr_unit(const PairSched& S, unsigned long long u) {
  int lo = 0, hi = S.njb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (S.unit_off[mid] <= u) lo = mid;
    else hi = mid - 1;
  }
  PairUnit U;
  U.jb = (unsigned long long)lo;
  const unsigned long long jend = 128ull * (U.jb + 1) < S.n_kmers ? 128ull * (U.jb + 1) : S.n_kmers;
  const unsigned long long ihi = S.row_end < jend - 1 ? S.row_end : jend - 1;
  U.i0 = S.row_start + (u - S.unit_off[lo]) * S.ic;
  U.i1 = U.i0 + S.ic < ihi ? U.i0 + S.ic : ihi;
  return U;
}

// Warp-aggregated pair records and refinement candidates, one pair per lane.
__device__ __forceinline__ void pr_emit(const DevOutPairs& O, unsigned long long i, unsigned long long j, bool hit,
                                        bool cand, double T, double p, double effect) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned hm = __ballot_sync(0xffffffffu, hit);
  if (hm) {
    unsigned long long base = 0;
    const int ld = __ffs(hm) - 1;
    if ((int)lane == ld) base = atomicAdd(O.counters + 1, (unsigned long long)__popc(hm));
    base = __shfl_sync(0xffffffffu, base, ld);
    if (hit) {
      const unsigned long long slot = base + __popc(hm & ((1u << lane) - 1u));
      if (slot < O.hit_cap) {
        kg_pair h;
        h.a = i;
        h.b = j;
        h.effect = effect;
        h.pval = p;
        h.chisq = T;
        O.hits[slot] = h;
      } else {
        atomicOr(O.counters + 2, (unsigned long long)ERR_HIT_OVERFLOW);
      }
    }
  }
  const unsigned cm = __ballot_sync(0xffffffffu, cand);
  if (cm) {
    unsigned long long base = 0;
    const int ld = __ffs(cm) - 1;
    if ((int)lane == ld) base = atomicAdd(O.counters + 3, (unsigned long long)__popc(cm));
    base = __shfl_sync(0xffffffffu, base, ld);
    if (cand) {
      const unsigned long long slot = base + __popc(cm & ((1u << lane) - 1u));
      if (slot < O.cand_cap) O.cand[slot] = (i << 32) | j;
      else atomicOr(O.counters + 2, (unsigned long long)ERR_CAND_OVERFLOW);
    }
  }
}

template <int N, bool DROP0>
__global__ void __launch_bounds__(pr_threads(N), 1)
    pairs_kernel(const __grid_constant__ CUtensorMap tmap, const uint64_t* __restrict__ x, int wpk, int nbox,
                 int nsub, int xst, const __grid_constant__ PairSched S, const int8_t* __restrict__ Bimg,
                 int b_bytes, const __grid_constant__ EpiParams P, const __grid_constant__ LimbMap LM,
                 const DevOutPairs O) {
  constexpr int UG = pr_ug(N);
  constexpr int WPROD = PR_WARP_UNPACK0 + 4 * UG, WMMA = WPROD + 1;
  constexpr int NSLOT = pr_nslot(N);
  constexpr int A0 = 512 - NSLOT * 128;
  static_assert(NSLOT >= 2 && A0 >= 2 * N, "TMEM budget");
  constexpr uint32_t IDESC = idesc_i8(PR_TM, N);
  constexpr int KU_MAX = (N - 1 - PR_LY) / PR_LU;
  constexpr uint32_t BSTEP = (2 * N * 16) >> 4;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gbase = smem_raw + (base - raw);
  const PrSmem L = pr_smem(b_bytes, xst);
  const uint32_t sx = base + L.x, sb = base + L.b;
  const uint32_t x_full = base + L.bars, x_empty = x_full + 8 * PR_XST_MAX;
  const uint32_t a_full = x_empty + 8 * PR_XST_MAX, a_empty = a_full + 8 * PR_MAXSLOT;
  const uint32_t acc_full = a_empty + 8 * PR_MAXSLOT, acc_empty = acc_full + 16, b_full = acc_empty + 16;
  const uint32_t drain = b_full + 8;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(gbase + L.tmem);
  volatile int* s_abort = reinterpret_cast<volatile int*>(gbase + L.abort);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nsp = (nsub + PR_SUPER - 1) / PR_SUPER;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < xst; ++s) {
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
    mbar_init(drain, 1);
    *s_abort = 0;
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const unsigned long long lim = wait_limit(O.wait_ns);

  if (warp == WPROD) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(&tmap) : "memory");
      mbar_arrive_expect_tx(b_full, (uint32_t)b_bytes);
      for (int off = 0; off < b_bytes; off += 32768) {
        const int len = b_bytes - off < 32768 ? b_bytes - off : 32768;
        bulk_g2s(sb + off, Bimg + off, (uint32_t)len, b_full);
      }
      RingN xr(xst);
      uint32_t last_phase[PR_XST_MAX];
      bool issued[PR_XST_MAX];
      for (int s = 0; s < PR_XST_MAX; ++s) issued[s] = false, last_phase[s] = 0;
      bool ok = true;
      for (unsigned long long u = blockIdx.x; u < S.n_units && ok; u += gridDim.x) {
        const PairUnit U = pr_unit(S, u);
        for (int bx = 0; bx < nbox; ++bx, xr.next()) {
          if (xr.used && !wait_or_abort(x_empty + 8 * xr.slot, xr.phase ^ 1u, s_abort, O.counters, ERR_TIMEOUT_FULL, lim)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(x_full + 8 * xr.slot, PR_XBYTES);
          tma_load_2d(sx + xr.slot * PR_XBYTES, &tmap, bx * 128, (int)(U.jb * PR_TM), x_full + 8 * xr.slot);
          issued[xr.slot] = true;
          last_phase[xr.slot] = xr.phase;
        }
      }
      mbar_wait(b_full, 0, O.counters, ERR_TIMEOUT_FULL);
      for (int s = 0; s < xst; ++s)
        if (issued[s]) mbar_wait(x_full + 8 * s, last_phase[s], O.counters, ERR_TIMEOUT_FULL);
    }
  } else if (warp == WMMA) {
    // ----------------------------------------------------------------- MMA
    const bool leader = elect_one();
    bool ok = __all_sync(0xffffffffu, wait_or_abort(b_full, 0, s_abort, O.counters, ERR_TIMEOUT_FULL, lim));
    const uint64_t bdesc0 = sdesc_noswz(sb, N * 16, 128);
    Ring<NSLOT> ar;
    uint32_t v = 0;  // tiles
    for (unsigned long long u = blockIdx.x; u < S.n_units && ok; u += gridDim.x) {
      const PairUnit U = pr_unit(S, u);
      for (unsigned long long i = U.i0; i < U.i1 && ok; ++i, ++v) {
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
          const int nsub_here = nsub - sp * PR_SUPER < PR_SUPER ? nsub - sp * PR_SUPER : PR_SUPER;
          const uint32_t a_t = tmem + A0 + ar.slot * 128;
          if (leader) {
            uint64_t bk = bd;
            for (int sub = 0; sub < nsub_here; ++sub) {
#pragma unroll
              for (int ks = 0; ks < PR_KS / 32; ++ks) {
                tc_mma_i8_ts(d_t, a_t + sub * 32 + ks * 8, bk, IDESC, (sp | sub | ks) ? 1u : 0u);
                bk += BSTEP;
              }
            }
            tc_commit(a_empty + 8 * ar.slot);
          }
          __syncwarp();
          bd += (uint64_t)(PR_SUPER * (PR_KS / 32) * BSTEP);
        }
        if (!ok) break;
        if (leader) tc_commit(acc_full + 8 * b);
        __syncwarp();
      }
    }
    if (leader) {
      tc_commit(drain);
      mbar_wait(drain, 0, O.counters, ERR_TIMEOUT_MMA);
    }
    __syncwarp();
  } else if (warp >= PR_WARP_UNPACK0) {
    // -------------------------------------------------------------- unpack
    const int grp = (warp - PR_WARP_UNPACK0) >> 2;
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    const int half_row = wpk / 2;  // 16-byte chunks in a packed row
    RingN xr(xst);
    Ring<NSLOT> ar;
    uint32_t turn = 0;
    bool ok = true;
    for (unsigned long long u = blockIdx.x; u < S.n_units && ok; u += gridDim.x) {
      const PairUnit U = pr_unit(S, u);
      // the unit's boxes stay resident for all its tiles
      uint32_t bslot[PR_NBOX_MAX], bphase[PR_NBOX_MAX];
      for (int bx = 0; bx < nbox; ++bx, xr.next()) {
        bslot[bx] = xr.slot;
        bphase[bx] = xr.phase;
      }
      for (unsigned long long i = U.i0; i < U.i1 && ok; ++i) {
        const uint4* xi = reinterpret_cast<const uint4*>(x + i * (unsigned long long)wpk);
        int kc = 0;
        for (int bx = 0; bx < nbox && ok; ++bx) {
          if (i == U.i0 && !__all_sync(0xffffffffu, wait_or_abort(x_full + 8 * bslot[bx], bphase[bx], s_abort,
                                                                  O.counters, ERR_TIMEOUT_FULL, lim))) {
            ok = false;
            break;
          }
          const int kc1 = (bx + 1) * (PR_BOX / PR_KS) < nsub ? (bx + 1) * (PR_BOX / PR_KS) : nsub;
          while (kc < kc1) {
            const int ke = kc + PR_SUPER < kc1 ? kc + PR_SUPER : kc1;
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
            const uint32_t xrow = sx + bslot[bx] * PR_XBYTES + r * 128;
            const uint32_t a_t = tmem + lane_base + A0 + ar.slot * 128;
            // the super-stage's chunks of row i (uniform across the warp) and
            // of the j rows, all loads in flight before the first use
            uint4 wi[PR_SUPER], wj[PR_SUPER];
#pragma unroll
            for (int s4 = 0; s4 < PR_SUPER; ++s4) {
              const int sub = kc + s4;
              wi[s4] = (sub < ke && sub < half_row) ? __ldg(xi + sub) : make_uint4(0u, 0u, 0u, 0u);
              const int c = sub - bx * (PR_BOX / PR_KS);
              if (sub < ke)
                asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];"
                             : "=r"(wj[s4].x), "=r"(wj[s4].y), "=r"(wj[s4].z), "=r"(wj[s4].w)
                             : "r"(xrow + ((c ^ (r & 7)) << 4)));
            }
#pragma unroll
            for (int s4 = 0; s4 < PR_SUPER; ++s4) {
              if (kc + s4 < ke) {
                const uint32_t w4[4] = {wj[s4].x & wi[s4].x, wj[s4].y & wi[s4].y, wj[s4].z & wi[s4].z,
                                        wj[s4].w & wi[s4].w};
                uint32_t o[32];
                unpack_stage(w4, o);
                tc_st32(a_t + s4 * 32, o);
              }
            }
            kc = ke;
            tc_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(a_full + 8 * ar.slot);
            ar.next();
            if (UG == 2) turn ^= 1u;
          }
        }
      }
      if (!ok) break;
      __syncwarp();
      if (lane == 0)
        for (int bx = 0; bx < nbox; ++bx) mbar_arrive(x_empty + 8 * bslot[bx]);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int e = warp >> 2;
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    uint32_t v = 0, jt = 0, evaluated = 0;
    bool ok = true;
    for (unsigned long long u = blockIdx.x; u < S.n_units && ok; u += gridDim.x) {
      const PairUnit U = pr_unit(S, u);
      for (unsigned long long i = U.i0; i < U.i1; ++i, ++v) {
        if ((v & 1u) != (uint32_t)e) continue;
        if (!__all_sync(0xffffffffu, wait_or_abort(acc_full + 8 * e, jt & 1u, s_abort, O.counters, ERR_TIMEOUT_MMA, lim))) {
          ok = false;
          break;
        }
        ++jt;
        tc_fence_after();
        uint32_t d[N];
#pragma unroll
        for (int c16 = 0; c16 < N / 16; ++c16) {
          uint32_t rr[16];
          tc_ld16(tmem + lane_base + e * N + c16 * 16, rr);
          tc_wait_ld();
#pragma unroll
          for (int k = 0; k < 16; ++k) d[c16 * 16 + k] = rr[k];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acc_empty + 8 * e);
        const unsigned long long j = U.jb * PR_TM + r;
        const bool valid = j < S.n_kmers && j > i;
        // limb sums hold -128 * integer sums (see kernel_ts.cu)
        const int c = (-(int)d[0]) >> 7;
        const double cd = i2d_exact(c);
        long long Vy = (long long)(int)d[PR_LY];
#pragma unroll
        for (int l = 1; l < PR_LY; ++l) Vy += (long long)(int)d[PR_LY - l] * (1ll << (8 * l));
        const double sy = LM.scale[P.k];
        const double ey = fma(magic_raw((-Vy) >> 7), sy, -MAGIC_BIAS * sy);
        double ss = 0;
        if (DROP0) {
          const double s0 = P.a[0] * cd;
          ss = s0 * s0;
        }
#pragma unroll
        for (int jj = 0; jj < KU_MAX; ++jj) {
          const int col = jj + (DROP0 ? 1 : 0);
          const int o = 1 + PR_LY + PR_LU * jj;
          long long Vb = (long long)(int)d[o + PR_LU - 1] + (long long)0x4338000000000000LL;
#pragma unroll
          for (int l = 1; l < PR_LU; ++l) Vb += (long long)(int)d[o + PR_LU - 1 - l] * (1ll << (8 * l));
          const double ej = fma(__longlong_as_double(Vb), LM.esc[col], LM.eoff[col]);
          const double sj = fma(P.a[col], cd, ej);
          ss = fma(sj, sj, ss);
        }
        // src/kgwas_2d.cpp:292-318: a33 > 0, xxM > eps, yyM > eps, then compute_hit
        const double eps = 1e-12;
        const double xxM = cd - ss, xyM = P.b * cd + ey;
        const double qv = xyM * xyM, den = xxM * P.yyM;
        const bool okp = valid && c > 0 && xxM > eps && P.yyM > eps;
        evaluated += okp ? 1u : 0u;
        const bool cand = okp && P.refine && qv >= P.r2_ref * den;
        const bool maybe = okp && !cand && qv >= P.r2_cand * den;
        if (__ballot_sync(0xffffffffu, cand || maybe) == 0u) continue;
        double T = 0, p = 1, effect = 0;
        bool hit = false;
        if (maybe) {
          double r2 = qv / den;
          if (r2 < 0) r2 = 0;
          if (r2 >= 1) r2 = 1 - 1e-15;
          T = (double)P.n * log(1.0 / (1.0 - r2));
          p = erfc(sqrt(0.5 * T));
          effect = xyM / den;
          hit = p <= P.p_thresh;
        }
        pr_emit(O, i, j, hit, cand, T, p, effect);
      }
    }
    const unsigned tot = __reduce_add_sync(0xffffffffu, evaluated);
    if (lane == 0 && tot) atomicAdd(O.counters + 0, (unsigned long long)tot);
  }
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// FP64 recomputation of the pair candidates: one warp per pair, column sums
// of x_i * x_j from the byte tables of V (table_row_sums on the AND of the
// two rows), then compute_hit in FP64 (src/kgwas_2d.cpp:300-318).
template <int CM>
__global__ void __launch_bounds__(256) pr_refine_kernel(const uint64_t* __restrict__ x, int wpk, int nwords,
                                                        const double* __restrict__ T,
                                                        const __grid_constant__ EpiParams P, const DevOutPairs O) {
  const int lane = threadIdx.x & 31;
  const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x >> 5);
  unsigned long long ncand = O.counters[3];
  if (ncand > O.cand_cap) ncand = O.cand_cap;
  for (unsigned long long w = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < ncand;
       w += warps) {
    const unsigned long long ent = O.cand[w];
    const unsigned long long i = ent >> 32, j = ent & 0xffffffffull;
    double acc[(CM + 31) / 32];
    table_row_sums<CM>(x + i * (unsigned long long)wpk, nwords, T, lane, acc, x + j * (unsigned long long)wpk);
    int c;
    double ss, ey;
    refine_reduce<CM>(P, acc, lane, c, ss, ey);
    if (lane == 0) {
      const double eps = 1e-12;
      const double xxM = (double)c - ss, xyM = P.b * (double)c + ey;
      if (c > 0 && xxM > eps && P.yyM > eps) {
        double r2 = (xyM * xyM) / (xxM * P.yyM);
        if (r2 < 0) r2 = 0;
        if (r2 >= 1) r2 = 1 - 1e-15;
        const double Tq = (double)P.n * log(1.0 / (1.0 - r2));
        const double p = erfc(sqrt(0.5 * Tq));
        if (p <= P.p_thresh) {
          const unsigned long long slot = atomicAdd(O.counters + 1, 1ull);
          if (slot < O.hit_cap) {
            kg_pair h;
            h.a = i;
            h.b = j;
            h.effect = xyM / (xxM * P.yyM);
            h.pval = p;
            h.chisq = Tq;
            O.hits[slot] = h;
          } else {
            atomicOr(O.counters + 2, (unsigned long long)ERR_HIT_OVERFLOW);
          }
        }
      }
    }
  }
}

// ------------------------------------------------------------------- host

static int pr_ring_depth(int b_bytes, int nbox) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) optin = 0;
  int x = PR_XST_MAX;
  while (x > nbox && pr_smem(b_bytes, x).total + 1024 > (uint32_t)optin) --x;
  return x;
}

bool pairs_supported(int N, int limbs_u, int limbs_y, int kpad, int wpk) {
  if (limbs_u != PR_LU || limbs_y != PR_LY) return false;
  if (N < 16 || N > 128 || N % 16 || pr_nslot(N) < 2) return false;
  if (wpk * 8 < 128) return false;  // one TMA box row is 128 bytes
  const int nbox = (wpk * 8 + 127) / 128;
  if (nbox > PR_NBOX_MAX) return false;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
  // the unit's boxes plus a second unit's, so that loads overlap
  return pr_smem(kpad * N, 2 * nbox).total + 1024 <= (uint32_t)optin;
}

template <int N, bool D0>
static cudaError_t launch_pairs_t(const LaunchPairs& L, const CUtensorMap& tm, cudaStream_t st) {
  const int b_bytes = L.kpad * N;
  const int nbox = (L.wpk * 8 + 127) / 128;
  const int xst = pr_ring_depth(b_bytes, nbox);
  if (xst < 2 * nbox) return cudaErrorInvalidValue;
  const size_t smem = pr_smem(b_bytes, xst).total + 1024;
  cudaError_t e =
      cudaFuncSetAttribute(pairs_kernel<N, D0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  unsigned long long grid = (unsigned long long)L.num_sms;
  if (grid > L.S.n_units) grid = L.S.n_units;
  if (grid == 0) return cudaSuccess;
  pairs_kernel<N, D0><<<(unsigned)grid, pr_threads(N), smem, st>>>(tm, L.x, L.wpk, nbox, L.kpad / PR_KS, xst, L.S,
                                                                   L.Bimg, b_bytes, *L.P, *L.LM, *L.O);
  return cudaGetLastError();
}

cudaError_t launch_pairs(const LaunchPairs& L, cudaStream_t st) {
  if (L.S.n_units == 0) return cudaSuccess;
  CUtensorMap tm;
  if (!mp_tmap(L.x, L.S.n_kmers, L.wpk, &tm)) return cudaErrorInvalidValue;
  const bool d0 = L.drop0;
  switch (L.LM->N) {
#define KG_PR_CASE(NN) \
  case NN: return d0 ? launch_pairs_t<NN, true>(L, tm, st) : launch_pairs_t<NN, false>(L, tm, st);
    KG_PR_CASE(16)
    KG_PR_CASE(32)
    KG_PR_CASE(48)
    KG_PR_CASE(64)
    KG_PR_CASE(80)
    KG_PR_CASE(96)
    KG_PR_CASE(112)
    KG_PR_CASE(128)
#undef KG_PR_CASE
    default: return cudaErrorInvalidValue;
  }
}

template <int CM>
static cudaError_t launch_pr_refine_t(const LaunchPairRefine& L, cudaStream_t st) {
  static int per_sm = 0;
  if (per_sm < 1 &&
      (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pr_refine_kernel<CM>, 256, 0) != cudaSuccess ||
       per_sm < 1))
    per_sm = 1;
  pr_refine_kernel<CM><<<(unsigned)(L.num_sms * per_sm), 256, 0, st>>>(L.x, L.wpk, L.vrows / 64, L.T, *L.P, *L.O);
  return cudaGetLastError();
}

cudaError_t launch_pair_refine(const LaunchPairRefine& L, cudaStream_t st) {
  if (!L.T) return cudaErrorInvalidValue;
  switch (L.cm) {
    case 8: return launch_pr_refine_t<8>(L, st);
    case 12: return launch_pr_refine_t<12>(L, st);
    case 16: return launch_pr_refine_t<16>(L, st);
    case 20: return launch_pr_refine_t<20>(L, st);
    case 24: return launch_pr_refine_t<24>(L, st);
    case 28: return launch_pr_refine_t<28>(L, st);
    case 36: return launch_pr_refine_t<36>(L, st);
    case 44: return launch_pr_refine_t<44>(L, st);
    case 52: return launch_pr_refine_t<52>(L, st);
    case 68: return launch_pr_refine_t<68>(L, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kg
