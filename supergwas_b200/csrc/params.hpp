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
  double a[KMAX];
  double g[KMAX];
};

// Column map of the int8 limb contraction (prep.hpp LimbCols).
struct LimbMap {
  int N, count_col;
  int first[KMAX + 1];
  int nl[KMAX + 1];
  double scale[KMAX + 1];
};

// Device outputs of one launch.
struct DevOut {
  unsigned long long* counters;  // [0] tested, [1] hits, [2] error bits
  kg_hit* hits;
  unsigned long long hit_cap;
  unsigned long long kmer_offset;  // added to the launch-local k-mer index
  // optional per-k-mer arrays, indexed by kmer_offset + local index
  uint8_t* tested;
  double *chisq, *pval, *effect, *mlog10p, *xxM, *xyM, *cor;
};

enum : unsigned { ERR_TIMEOUT_FULL = 1u, ERR_TIMEOUT_MMA = 2u, ERR_HIT_OVERFLOW = 4u };

}  // namespace kg
