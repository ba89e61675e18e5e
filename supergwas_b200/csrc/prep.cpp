// prep.cpp -- see prep.hpp for the algebra.
#include "prep.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace kg {

typedef long double ld;

std::string prepare(const double* U, int n, int k, const double* y, Prepared& P) {
  if (n <= 0) return "n must be positive";
  if (k < 0 || k > KMAX) return "k (U.bin columns) must be in [0, " + std::to_string(KMAX) + "]";
  if (!y) return "y is NULL";
  if (k > 0 && !U) return "U is NULL";
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(y[i])) return "phenotype value is not finite";
  for (size_t i = 0; i < (size_t)n * k; ++i)
    if (!std::isfinite(U[i])) return "U.bin value is not finite";

  P = Prepared();
  P.n = n;
  P.k = k;
  // U^T y and yyM (src/kgwas_utils.hpp:151-153), ynorm of y - mean(y)
  std::vector<ld> Uy(k);
  ld yy = 0, ysum = 0;
  for (int i = 0; i < n; ++i) { yy += (ld)y[i] * y[i]; ysum += y[i]; }
  ld uyy = 0;
  for (int j = 0; j < k; ++j) {
    ld s = 0;
    for (int i = 0; i < n; ++i) s += (ld)U[(size_t)j * n + i] * y[i];
    Uy[j] = s;
    uyy += s * s;
  }
  P.yyM = (double)(yy - uyy);
  const ld ymean = ysum / n;
  P.ymean = (double)ymean;
  ld yc2 = 0;
  for (int i = 0; i < n; ++i) { ld t = (ld)y[i] - ymean; yc2 += t * t; }
  P.ynorm = (double)std::sqrt(yc2);

  // Householder H with H e0 = w/||w||, w = U^T 1; Q = U H.
  std::vector<ld> Q((size_t)n * (k > 0 ? k : 1), 0);
  for (size_t i = 0; i < (size_t)n * k; ++i) Q[i] = U[i];
  std::vector<ld> w(k, 0);
  ld wn2 = 0;
  for (int j = 0; j < k; ++j) {
    ld s = 0;
    for (int i = 0; i < n; ++i) s += U[(size_t)j * n + i];
    w[j] = s;
    wn2 += s * s;
  }
  std::vector<ld> Hm((size_t)k * k, 0);  // H, row-major
  for (int j = 0; j < k; ++j) Hm[(size_t)j * k + j] = 1;
  if (k > 0 && wn2 > 0) {
    const ld wn = std::sqrt(wn2);
    std::vector<ld> v(k);
    ld vv = 0;
    for (int j = 0; j < k; ++j) { v[j] = w[j] / wn - (j == 0 ? 1 : 0); vv += v[j] * v[j]; }
    if (vv > 1e-30L) {
      for (int r = 0; r < k; ++r)
        for (int c = 0; c < k; ++c) Hm[(size_t)r * k + c] -= 2 * v[r] * v[c] / vv;
      // Q = U H: Q[:, c] = sum_r U[:, r] H[r, c]
      for (int c = 0; c < k; ++c)
        for (int i = 0; i < n; ++i) {
          ld s = 0;
          for (int r = 0; r < k; ++r) s += (ld)U[(size_t)r * n + i] * Hm[(size_t)r * k + c];
          Q[(size_t)c * n + i] = s;
        }
    }
  }
  // g = Q^T y = H U^T y (H symmetric)
  P.a.assign(k, 0.0);
  P.g.assign(k, 0.0);
  std::vector<ld> gl(k, 0), al(k, 0);
  for (int c = 0; c < k; ++c) {
    ld s = 0;
    for (int r = 0; r < k; ++r) s += Hm[(size_t)r * k + c] * Uy[r];
    gl[c] = s;
    P.g[c] = (double)s;
  }
  P.d.assign((size_t)(k + 1) * n, 0.0);
  for (int j = 0; j < k; ++j) {
    ld s = 0;
    for (int i = 0; i < n; ++i) s += Q[(size_t)j * n + i];
    al[j] = s / n;
    P.a[j] = (double)al[j];
    for (int i = 0; i < n; ++i) P.d[(size_t)j * n + i] = (double)(Q[(size_t)j * n + i] - al[j]);
  }
  // y' = y - U (U^T y); b = mean(y'); d_y = y' - b
  std::vector<ld> yp(n);
  ld ps = 0;
  for (int i = 0; i < n; ++i) {
    ld s = y[i];
    for (int j = 0; j < k; ++j) s -= (ld)U[(size_t)j * n + i] * Uy[j];
    yp[i] = s;
    ps += s;
  }
  const ld bl = ps / n;
  P.b = (double)bl;
  for (int i = 0; i < n; ++i) P.d[(size_t)k * n + i] = (double)(yp[i] - bl);
  ld kap = bl - ymean;
  for (int j = 0; j < k; ++j) kap += al[j] * gl[j];
  P.kappa = (double)kap;
  // Column 0's centred part is rounding noise when 1 lies in span(U).
  if (k > 0) {
    double mx = 0;
    for (int i = 0; i < n; ++i) mx = std::max(mx, std::fabs(P.d[i]));
    P.drop0 = (mx <= 1e-13 * std::fabs(P.a[0]));
  }
  return "";
}

// Balanced signed-digit decomposition of V into L base-256 digits in [-128,127].
static void digits(int64_t V, int L, int8_t* out) {
  for (int l = L - 1; l >= 0; --l) {
    int64_t r = ((V % 256) + 256) % 256;  // 0..255
    int64_t dgt = r >= 128 ? r - 256 : r;
    out[l] = (int8_t)dgt;
    V = (V - dgt) / 256;
  }
}

std::string make_limbs(const Prepared& p, const int* pos, int n_row, int limbs_u, int limbs_y, int kquant,
                       LimbCols& L) {
  if (limbs_u < 1 || limbs_u > 4 || limbs_y < 1 || limbs_y > 5) return "limbs must be in [1, 4] for U and [1, 5] for y'";
  const int n = p.n, k = p.k;
  if (n_row < n) return "rows hold fewer samples than the overlap";
  L = LimbCols();
  L.Kpad = ((n_row + kquant - 1) / kquant) * kquant;
  // column order: [count, y' limbs, U column 0 (unless dropped), U columns 1..k-1]
  int col = 0;
  L.count_col = col++;
  L.first[k] = col;
  L.nl[k] = limbs_y;
  L.scale[k] = 0.0;
  col += limbs_y;
  for (int j = 0; j < k; ++j) {
    const bool skip = (j == 0 && p.drop0);
    const int nl = skip ? 0 : limbs_u;
    L.first[j] = col;
    L.nl[j] = nl;
    L.scale[j] = 0.0;
    col += nl;
  }
  const int used = col;
  int N = ((used + 15) / 16) * 16;
  if (N < 16) N = 16;
  if (N > 256) return "too many contraction columns for one MMA (" + std::to_string(used) + " > 256)";
  L.N = N;
  L.vals.assign((size_t)N * L.Kpad, 0);
  auto at = [&](int i) { return pos ? pos[i] : i; };
  for (int i = 0; i < n; ++i) L.vals[(size_t)L.count_col * L.Kpad + at(i)] = 1;
  std::vector<int8_t> dg(8);
  for (int j = 0; j <= k; ++j) {
    const int nl = L.nl[j];
    if (nl == 0) continue;
    const double* v = &p.d[(size_t)j * n];
    double mx = 0;
    for (int i = 0; i < n; ++i) mx = std::max(mx, std::fabs(v[i]));
    // half the largest magnitude representable with a top digit in
    // [-127, 127]: the TMEM kernel multiplies half of the samples as 64 x
    // against the digits of -2 V (make_b_image_ts), which must fit too
    const double lim = 127.0 * std::ldexp(1.0, 8 * (nl - 1) - 1);
    int s = 0;
    if (mx > 0) {
      int e;
      std::frexp(lim / mx, &e);   // lim/mx in [2^(e-1), 2^e)
      s = e - 1;                  // mx * 2^s <= lim
    }
    L.scale[j] = std::ldexp(1.0, -s);
    for (int i = 0; i < n; ++i) {
      const int64_t V = (int64_t)std::llround(std::ldexp(v[i], s));
      digits(V, nl, dg.data());
      for (int l = 0; l < nl; ++l) L.vals[(size_t)(L.first[j] + l) * L.Kpad + at(i)] = dg[l];
    }
  }
  return "";
}

void put_b_image_ts(const LimbCols& L, int col0, int N, std::vector<int8_t>& img) {
  // Limb digits of -2 V for every sample, column by column (V = the value a
  // logical column's digits encode; the count column holds V = 1).
  std::vector<int8_t> neg2((size_t)L.N * L.Kpad, 0);
  std::vector<int8_t> dg(8);
  auto regroup = [&](int first, int nl) {
    for (int i = 0; i < L.Kpad; ++i) {
      int64_t V = 0;
      for (int l = 0; l < nl; ++l) V = V * 256 + L.vals[(size_t)(first + l) * L.Kpad + i];
      digits(-2 * V, nl, dg.data());
      for (int l = 0; l < nl; ++l) neg2[(size_t)(first + l) * L.Kpad + i] = dg[l];
    }
  };
  regroup(L.count_col, 1);
  for (int j = 0; j <= KMAX; ++j)
    if (L.nl[j] > 0 && L.first[j] > 0 && L.first[j] + L.nl[j] <= L.N) regroup(L.first[j], L.nl[j]);
  for (int kap = 0; kap < L.Kpad; ++kap) {
    // TMEM column c of a 128-sample stage holds K = 4c..4c+3.  The unpack
    // (unpack_stage in device.cuh) writes, for 32-bit word q of the stage and
    // jj = 0..7, column 8q+jj = (word << 2*(jj/2)) & (jj even ? 0x80808080 :
    // 0x40404040): byte t of it is sample 32q + 8t + 7 - jj, as -128 x (jj
    // even) or 64 x (jj odd).  Odd columns therefore take the digits of -2 V.
    const int a = kap / 128, w = kap % 128, c = w / 4, t = w % 4, q = c / 8, jj = c % 8;
    const int i = 128 * a + 32 * q + 8 * t + 7 - jj;
    const std::vector<int8_t>& src = (jj & 1) ? neg2 : L.vals;
    for (int col = 0; col < L.N; ++col) {
      const int cc = col0 + col;
      const size_t off = (size_t)(kap / 16) * (N * 16) + (size_t)(cc / 8) * 128 + (size_t)(cc % 8) * 16 + kap % 16;
      img[off] = src[(size_t)col * L.Kpad + i];
    }
  }
}

void make_b_image_ts(const LimbCols& L, std::vector<int8_t>& img) {
  img.assign((size_t)L.Kpad * L.N, 0);
  put_b_image_ts(L, 0, L.N, img);
}

void make_b_image(const LimbCols& L, int KC, std::vector<int8_t>& img) {
  const int N = L.N, nchunk = L.Kpad / KC;
  img.assign((size_t)L.Kpad * N, 0);
  for (int q = 0; q < nchunk; ++q)
    for (int k16 = 0; k16 < KC / 16; ++k16)
      for (int col = 0; col < N; ++col)
        for (int kk = 0; kk < 16; ++kk) {
          const int i = q * KC + k16 * 16 + kk;
          const size_t off = (size_t)q * KC * N + (size_t)k16 * (N * 16) + (size_t)(col / 8) * 128 +
                             (size_t)(col % 8) * 16 + kk;
          img[off] = L.vals[(size_t)col * L.Kpad + i];
        }
}

}  // namespace kg
