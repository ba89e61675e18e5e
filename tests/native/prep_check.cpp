// prep_check.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the library's real host preparation (supergwas_b200/csrc/prep.cpp)
// and replays, on the CPU, the arithmetic the kernels perform after it:
//   split form: exact integer limb sums (what tcgen05 kind::i8 accumulates in
//               int32 TMEM), recombined to FP64 exactly as the epilogue does;
//   fp64 form : FP64 dot products with the centred columns.
// followed by the same epilogue formulas.  Lets the CPU test suite check the
// rotation / centring / quantisation algebra against the oracle.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../supergwas_b200/csrc/prep.hpp"

extern "C" int prep_emulate(const double* U, int n, int k, const double* y, const uint64_t* x, int64_t m,
                            int wpk, int split, int limbs_u, int limbs_y, double corr_thr, uint8_t* tested,
                            double* chisq, double* effect, double* xxM_o, double* xyM_o, double* cor_o,
                            double* yyM_o) {
  kg::Prepared P;
  if (!kg::prepare(U, n, k, y, P).empty()) return 1;
  kg::LimbCols L;
  if (split && !kg::make_limbs(P, nullptr, n, limbs_u, limbs_y, 256, L).empty()) return 2;
  *yyM_o = P.yyM;
  std::vector<double> e(k + 1);
  for (int64_t j = 0; j < m; ++j) {
    const uint64_t* row = x + (size_t)j * wpk;
    int c = 0;
    if (split) {
      std::vector<long long> acc(L.N, 0);
      for (int i = 0; i < n; ++i)
        if ((row[i >> 6] >> (i & 63)) & 1u)
          for (int col = 0; col < L.N; ++col) acc[col] += L.vals[(size_t)col * L.Kpad + i];
      c = (int)acc[L.count_col];
      for (int t = 0; t <= k; ++t) {
        long long v = 0;
        for (int l = 0; l < L.nl[t]; ++l) v = v * 256 + acc[L.first[t] + l];
        e[t] = (double)v * L.scale[t];
      }
    } else {
      for (int t = 0; t <= k; ++t) e[t] = 0;
      for (int i = 0; i < n; ++i)
        if ((row[i >> 6] >> (i & 63)) & 1u) {
          ++c;
          for (int t = 0; t <= k; ++t) e[t] += P.d[(size_t)t * n + i];
        }
    }
    double ss = 0, gs = 0;
    for (int t = 0; t < k; ++t) {
      const double s = P.a[t] * c + e[t];
      ss += s * s;
      gs += P.g[t] * e[t];
    }
    const double ey = e[k];
    bool tst = c > 0 && c < n && !(P.ynorm < 1e-12);
    double cor = 0;
    if (tst) {
      const double xcn2 = (double)c * (double)(n - c) / n;
      cor = (ey + gs + P.kappa * c) / (std::sqrt(xcn2) * P.ynorm);
      tst = !(std::fabs(cor) < corr_thr);
    }
    double xxM = 0, xyM = 0, T = 0, eff = 0;
    if (tst) {
      xxM = c - ss;
      xyM = P.b * c + ey;
      if (xxM > 1e-12 && P.yyM > 1e-12) {
        double r2 = xyM * xyM / (xxM * P.yyM);
        if (r2 < 0) r2 = 0;
        if (r2 >= 1) r2 = 1 - 1e-15;
        T = n * std::log(1.0 / (1.0 - r2));
        eff = xyM / (xxM * P.yyM);
      }
    }
    tested[j] = tst;
    chisq[j] = T;
    effect[j] = eff;
    xxM_o[j] = xxM;
    xyM_o[j] = xyM;
    cor_o[j] = cor;
  }
  return 0;
}

// The TMEM kernel's B image (make_b_image_ts) against the A operand its
// unpack writes: for every k-mer, the per-limb int32 sums that tcgen05 would
// accumulate (A bytes as the kernel forms them, times the image's B bytes),
// recombined per logical column, must equal -128 * sum_i x_i V_i.  Returns
// the number of (k-mer, column) mismatches, or -1 on a preparation error.
extern "C" int64_t ts_image_check(const double* U, int n, int k, const double* y, const uint64_t* x, int64_t m,
                                  int wpk) {
  kg::Prepared P;
  if (!kg::prepare(U, n, k, y, P).empty()) return -1;
  kg::LimbCols L;
  if (!kg::make_limbs(P, nullptr, n, 3, 5, 256, L).empty()) return -1;
  std::vector<int8_t> img;
  kg::make_b_image_ts(L, img);
  const int N = L.N;
  auto B = [&](int kap, int col) {
    return (int)img[(size_t)(kap / 16) * (N * 16) + (size_t)(col / 8) * 128 + (size_t)(col % 8) * 16 + kap % 16];
  };
  int64_t bad = 0;
  std::vector<long long> acc(N), ref(N);
  for (int64_t r = 0; r < m; ++r) {
    const uint64_t* row = x + (size_t)r * wpk;
    std::fill(acc.begin(), acc.end(), 0);
    std::fill(ref.begin(), ref.end(), 0);
    for (int a = 0; a < L.Kpad / 128; ++a)
      for (int c = 0; c < 32; ++c) {
        const int q = c / 8, jj = c % 8;
        const int bit0 = 128 * a + 32 * q;  // first sample of 32-bit word q of the stage
        uint32_t wq = 0;
        if (bit0 / 64 < wpk) wq = (uint32_t)(row[bit0 / 64] >> (bit0 % 64));
        const uint32_t u = wq << (2 * (jj / 2));
        const uint32_t o = u & ((jj & 1) ? 0x40404040u : 0x80808080u);
        for (int t = 0; t < 4; ++t) {
          const int av = (int)(int8_t)(uint8_t)(o >> (8 * t));
          for (int col = 0; col < N; ++col) acc[col] += (long long)av * B(128 * a + 4 * c + t, col);
        }
      }
    for (int i = 0; i < L.Kpad; ++i)
      if (i / 64 < wpk && ((row[i / 64] >> (i % 64)) & 1u))
        for (int col = 0; col < N; ++col) ref[col] += -128LL * L.vals[(size_t)col * L.Kpad + i];
    auto recomb = [&](const std::vector<long long>& v, int first, int nl) {
      long long s = 0;
      for (int l = 0; l < nl; ++l) s = s * 256 + v[first + l];
      return s;
    };
    if (acc[L.count_col] != ref[L.count_col]) ++bad;
    for (int j = 0; j <= k; ++j)
      if (L.nl[j] > 0 && recomb(acc, L.first[j], L.nl[j]) != recomb(ref, L.first[j], L.nl[j])) ++bad;
    for (int col = 0; col < N; ++col)  // int32 accumulators must not overflow
      if (acc[col] > 2147483647LL || acc[col] < -2147483648LL) ++bad;
  }
  return bad;
}
