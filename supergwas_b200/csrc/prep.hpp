// prep.hpp -- host-side FP64 preparation of one phenotype's structure.
//
// The reference evaluates, per k-mer x (0/1 over the n overlap samples),
//   xxM = x.x - ||U^T x||^2 ,  xyM = x.y - (U^T x).(U^T y)      (src/kgwas.cpp:138-166)
//   yyM = ||y||^2 - ||U^T y||^2                                  (src/kgwas_utils.hpp:151-153)
// and the Pearson pre-filter on x - mean(x), y - mean(y)        (src/kgwas.cpp:182-218).
//
// This file rewrites those quantities so that the device only contracts x
// with a few centred FP64 vectors:
//   Q = U H, H the Householder reflection taking e0 to U^T 1 / ||U^T 1||, so
//     Q Q^T = U U^T, column 0 of Q carries the whole intercept and columns
//     1..k-1 sum to zero;
//   q_j = a_j 1 + d_j (a_j = mean, d_j centred), y' = y - U U^T y = b 1 + d_y,
//   g = Q^T y, kappa = b + sum_j a_j g_j - mean(y)  (zero in exact arithmetic).
// With c = popcount(x), e_j = d_j . x and e_y = d_y . x:
//   s_j  = a_j c + e_j                         (= (Q^T x)_j)
//   xxM  = c - sum_j s_j^2
//   xyM  = b c + e_y
//   x.yc = e_y + sum_j g_j e_j + kappa c       (Pearson numerator)
//   ||x - mean x||^2 = c (n - c) / n
// so the only cancellation left (c - s_0^2 for the intercept) happens in FP64
// on exact integers, and every vector the tensor cores see is centred.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace kg {

constexpr int KMAX = 64;      // structure columns supported (r + 1 <= 64)

struct Prepared {
  int n = 0, k = 0;
  double yyM = 0, ynorm = 0, ymean = 0;
  double b = 0, kappa = 0;
  std::vector<double> a, g;     // k each
  std::vector<double> d;        // (k + 1) * n, column j at d[j*n]; column k = d_y
  bool drop0 = false;           // d_0 negligible: skipped by the int8 contraction
};

// Returns an empty string on success, else the error text.
std::string prepare(const double* U_colmajor, int n, int k, const double* y, Prepared& out);

// int8 limb form of the contraction columns for tcgen05 kind::i8.  Column
// order: count (1 for every phenotyped sample), the y' limbs, then the limbs
// of U columns 0 (unless drop0) .. k-1.
struct LimbCols {
  int N = 0;                    // MMA N (columns incl. padding), multiple of 16
  int count_col = 0;            // column holding 1 for every sample (popcount)
  int first[KMAX + 1];          // first limb column of logical column j (j = k: y')
  int nl[KMAX + 1];             // limbs of logical column j (0 = skipped)
  double scale[KMAX + 1];       // 2^-s_j
  // B operand, sample-major values: vals[col * Kpad + i]
  std::vector<int8_t> vals;
  int Kpad = 0;
};

// Quantise the centred columns into signed int8 limbs (balanced digits,
// value = sum_l digit_l 256^(L-1-l) 2^-s).  Overlap sample i sits at bit
// position pos[i] of the packed rows (pos = NULL: position i); rows hold
// n_row samples; Kpad = n_row rounded up to `kquant`.  Positions that hold
// no overlap sample get weight 0 in every column, the count column included.
std::string make_limbs(const Prepared& p, const int* pos, int n_row, int limbs_u, int limbs_y, int kquant,
                       LimbCols& out);

// Lay the B operand out as the shared-memory image of one K chunk after
// another (UMMA K-major, no swizzle: 8-row x 16-byte core matrices, core
// (n8, k16) of chunk q at q*KC*N + k16*(N*16) + n8*128).
void make_b_image(const LimbCols& L, int KC, std::vector<int8_t>& img);

// B operand image for the TMEM-A kernels: the whole Kpad x N matrix in one
// K-major no-swizzle layout (core (n8, k16) at k16*(N*16) + n8*128), with the
// K index permuted inside every 128-sample stage to match the bit unpack
// order: K = 4c + t of column c = 8q + j holds sample 32q + 8t + 7 - j, with
// the digits of V for even j and of -2 V for odd j.
void make_b_image_ts(const LimbCols& L, std::vector<int8_t>& img);
// The columns of L at columns col0 .. col0 + L.N - 1 of an N-column image in
// the same layout (img holds L.Kpad * N bytes): several phenotypes side by
// side in one MMA.
void put_b_image_ts(const LimbCols& L, int col0, int N, std::vector<int8_t>& img);

}  // namespace kg
