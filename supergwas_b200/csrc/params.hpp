// params.hpp -- kernel parameter blocks shared by host and device code.
#pragma once
#include <cstdint>

#include "../../include/kgwas_cuda.h"
#include "prep.hpp"

namespace kg {

// Per-phenotype constants of the epilogue (prep.hpp notation).
struct EpiParams {
  int n, k;
  double b, kappa, yyM, ynorm, corr_thr, p_thresh;
  double r2_cand;   // r2 below this cannot give p <= p_thresh (log/erfc skipped)
  int refine;       // 1: k-mers with r2 >= r2_ref go to the FP64 refinement list
  double r2_ref;
  double thr2_ynorm2;  // corr_thr^2 * ynorm^2 (division-free Pearson gate)
  double a[KMAX];
  double g[KMAX];
};

// Column map of the int8 limb contraction (prep.hpp LimbCols).
struct LimbMap {
  int N, count_col;
  int first[KMAX + 1];
  int nl[KMAX + 1];
  double scale[KMAX + 1];
  // Epilogue constants of the kernels whose accumulators hold -128 * digit
  // sums (set_limb_consts): for the recombined integer V, biased to the
  // double 1.5 * 2^52 + V, e = fma(biased, esc, eoff) = V * (-scale / 128)
  // exactly (both factors are powers of two times integers).
  double esc[KMAX + 1];   // -scale / 128
  double eoff[KMAX + 1];  // 1.5 * 2^52 * scale / 128
};

inline void set_limb_consts(LimbMap& L) {
  for (int j = 0; j <= KMAX; ++j) {
    L.esc[j] = -L.scale[j] / 128.0;
    L.eoff[j] = 6755399441055744.0 * L.scale[j] / 128.0;
  }
}

// Device outputs of one launch.
struct DevOut {
  unsigned long long* counters;  // [0] tested, [1] hits, [2] error bits, [3] refinement candidates
  kg_hit* hits;
  unsigned long long hit_cap;
  unsigned long long kmer_offset;  // added to the launch-local k-mer index
  // optional per-k-mer arrays, indexed by kmer_offset + local index
  uint8_t* tested;
  double *chisq, *pval, *effect, *mlog10p, *xxM, *xyM, *cor;
  // FP64 refinement list (global k-mer indices), used when EpiParams::refine
  unsigned long long* cand;
  unsigned long long cand_cap;
  // optional: a tested k-mer counts weight[kmer_offset + local] times in
  // counters[0] (a row that stands for a run of equal rows)
  const uint32_t* weight;
  // pipeline wait limit in ns (0: WAIT_LIMIT_NS)
  unsigned long long wait_ns;
  // test hook of the bounded waits: when non-zero, the row producer of each
  // CTA issues this many row loads and then stops, so that the consumers'
  // waits run out (0: off)
  unsigned long long stall_loads;
};

enum : unsigned { ERR_TIMEOUT_FULL = 1u, ERR_TIMEOUT_MMA = 2u, ERR_HIT_OVERFLOW = 4u, ERR_CAND_OVERFLOW = 8u };

// Chi-square above which the split form hands a k-mer to the FP64
// refinement kernel: there -log10 p ~ T / (2 ln 10) grows with T, so an
// absolute 1e-6 bound needs FP64 accuracy; below it 24-bit U limbs suffice.
constexpr double REFINE_CHISQ = 12.0;

// One phenotype of a multi-phenotype launch (device memory).
struct MPheno {
  EpiParams P;
  LimbMap LM;       // limb columns relative to the phenotype's slot in its group
  int drop0;        // U column 0 carries no limbs (intercept handled in FP64)
  int pad;
};

// Outputs of a multi-phenotype launch.
struct DevOutMP {
  unsigned long long* counters;      // [1] hits, [2] error bits, [3] refinement candidates
  unsigned long long* tested;        // [shard * n_pheno + pheno]
  kg_phit* hits;
  unsigned long long hit_cap;
  unsigned long long* cand;          // kmer | pheno << 48
  unsigned long long cand_cap;
  const unsigned long long* shard_start;  // ascending, global k-mer indices
  int n_shards;
  int n_pheno;
  unsigned long long kmer_offset;
  // optional: a tested (k-mer, phenotype) counts weight[global k-mer] times
  // (a row that stands for a run of equal rows)
  const uint32_t* weight;
  // pipeline wait limit in ns (0: WAIT_LIMIT_NS)
  unsigned long long wait_ns;
  // test hook of the bounded waits, as DevOut::stall_loads (0: off)
  unsigned long long stall_loads;
};

// Outputs of the 2-D pair test (kernel_pairs.cu).
struct DevOutPairs {
  unsigned long long* counters;  // [0] evaluated pairs, [1] hits, [2] error bits, [3] refinement candidates
  kg_pair* hits;
  unsigned long long hit_cap;
  unsigned long long* cand;      // i << 32 | j
  unsigned long long cand_cap;
  unsigned long long wait_ns;    // pipeline wait limit in ns (0: WAIT_LIMIT_NS)
};

// Pair schedule: pairs (i, j), i < j, row_start <= i < row_end, j < n_kmers.
// Unit u covers j-block jb (j in [128 jb, 128 jb + 128)) and up to `ic`
// consecutive i; units of j-block jb are unit_off[jb] .. unit_off[jb+1]-1.
struct PairSched {
  const unsigned long long* unit_off;  // njb + 1 entries (device)
  int njb;
  unsigned long long n_units, n_kmers, row_start, row_end, ic;
};

}  // namespace kg
