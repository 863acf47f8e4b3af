// Device (and host) arithmetic of the scattering-intensity path.
//
// Quartet evaluation is split in two stages:
//
//  stage 1 (q-independent, one thread per group quartet): the Hermite-space
//    density D[T][U][V] of the quartet, summed over its primitive quartets with
//    the reference's cutoffs (src/Integrals.f90:5155-5219), then either
//      * the coefficients h_b of the spherical-Bessel expansion
//        F(q) = sum_b h_b j_b(qH) (q/H)^b  (BesselDeriv, :4708-4746), or
//      * for P = Q (h < cutoffcentre, and always for loop 5) the even
//        polynomial F(q) = sum_s c_s q^{2s} of the P0 table (P_LMN, :3102-3135);
//  stage 2 (per q point, one warp per quartet, lanes over q): the Bessel sum
//    with an accurate generator and the Gaussian factor exp(-q^2 (1/4p+1/4p')).
//
// Everything here is FP64.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define TB_HD __host__ __device__ __forceinline__
#else
#define TB_HD inline
#endif

namespace tb {

// Largest Cartesian exponent per axis handled (g functions, like the
// reference's fill_md_table, src/Variables.f90:938-940).
constexpr int MAXA = 4;
// Largest LLmax (sum of the four shells' angular momenta).
constexpr int LMAXQ = 16;
// Largest Bessel order used (j2 adds two, src/Integrals.f90:5415).
constexpr int LMAXB = LMAXQ + 2;
// Terms of the small-x power series (enough for every order up to LMAXB at
// x below the crossover, see series_terms).
constexpr int SER_K = 24;

// Reference constants.
// acos(-1.0000) evaluated in default (single) precision (src/Variables.f90:994).
#define TB_PI_SP 3.1415927410125732
// The Fortran literal 1.0e-30 of the MD skips is single precision.
#define TB_SKIP30 1.0000000031710769e-30
#define TB_PI 3.141592653589793

// KIND_ELASTIC_J2: the j2 Bessel expansion of total j2 on the elastic density
// product Z_ab Z_cd (integral_k_ijkr_j2, src/Integrals.f90:5903-6083)
// KIND_CMS: the elastic j0 kernel on zi_ab zj_cd, two AO densities from two
// 1-RDMs, over every ordered (bra pair, ket pair) (resolved_cms_integration,
// src/Integrals.f90:2598-2930)
enum Kind { KIND_TOTAL = 0, KIND_ELASTIC = 1, KIND_J2 = 2, KIND_ALIGNED = 3, KIND_ELASTIC_J2 = 4, KIND_CMS = 5 };
// j2 Bessel expansion (order LLmax + 2, P2 weight) / density from 1-RDMs
TB_HD constexpr bool kind_j2(int k) { return k == KIND_J2 || k == KIND_ELASTIC_J2; }
TB_HD constexpr bool kind_elastic(int k) { return k == KIND_ELASTIC || k == KIND_ELASTIC_J2 || k == KIND_CMS; }
enum RecKind { REC_BESSEL = 0, REC_BESSEL_J2 = 1, REC_P0 = 2 };

// Cartesian component i (axis 0, 1, 2 exponent) of an s, p, d or f shell, in
// the order of the molden convention the reference reads
// (src/molden_reader_nikola.py:196-240): p x y z; d xx yy zz xy xz yz;
// f xxx yyy zzz xyy xxy xxz xzz yzz yyz xyz.
TB_HD constexpr int cart_component(int L, int i, int axis) {
  constexpr int t1[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  constexpr int t2[6][3] = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
  constexpr int t3[10][3] = {{3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {1, 2, 0}, {2, 1, 0},
                             {2, 0, 1}, {1, 0, 2}, {0, 1, 2}, {0, 2, 1}, {1, 1, 1}};
  return L == 0 ? 0 : L == 1 ? t1[i][axis] : L == 2 ? t2[i][axis] : t3[i][axis];
}

// number of (T,U,V) with T+U+V <= L
TB_HD constexpr int ntuv(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
// simplex index of (T,U,V)
TB_HD int tuv_index(int T, int U, int V) {
  int s = T + U + V, r = U + V;
  return s * (s + 1) * (s + 2) / 6 + r * (r + 1) / 2 + V;
}

// Packed (T, p) tables with p = T - 2k, k = 0..T/2.
TB_HD constexpr int tp_off(int T) { return (T / 2 + 1) * (T / 2 + 1) - ((T % 2) ? 0 : (T / 2 + 1)); }
TB_HD constexpr int tp_size(int L) { return tp_off(L + 1); }

// Hermite-like expansion coefficients a(T,p) of d^T/dX^T f(|R|) in terms of
// (1/r d/dr)^k f: the recurrence of rrdj0 / Hermite_like_coeffs
// (src/Integrals.f90:7037-7091), a(T,p) = -(T-1) a(T-2,p) - X a(T-1,p-1),
// stored packed as a[tp_off(T) + (T-p)/2].
TB_HD void hermite_table(int L, double X, double *a) {
  a[0] = 1.0;                       // (0,0)
  if (L >= 1) a[tp_off(1)] = -X;    // (1,1)
  for (int T = 2; T <= L; ++T) {
    for (int k = 0; 2 * k <= T; ++k) {
      int p = T - 2 * k;
      double v = 0.0;
      // -(T-1) a(T-2, p), exists if p <= T-2
      if (p <= T - 2) v = -(double)(T - 1) * a[tp_off(T - 2) + (T - 2 - p) / 2];
      // - X a(T-1, p-1), exists if p >= 1
      if (p >= 1) v = v - X * a[tp_off(T - 1) + (T - 1 - (p - 1)) / 2];
      a[tp_off(T) + k] = v;
    }
  }
}

// E^{l1,l2}_t, t = 0..l1+l2, for l1 >= l2 in the order of the reference's
// unrolled tables (src/Variables.f90:31-687): the PA chain from E^{0,0} to
// E^{l1,0}, then the PB chain to E^{l1,l2}; each entry
// a E_{t-1} + P E_t + (t+1) E_{t+1}, left to right.
TB_HD void md_chain(int l1, int l2, double PA, double PB, double a, double *out) {
  double cur[2 * MAXA + 2], nxt[2 * MAXA + 2];
  int len = 1;
  cur[0] = 1.0;
  for (int step = 0; step < l1 + l2; ++step) {
    double P = step < l1 ? PA : PB;
    for (int t = 0; t <= len; ++t) {
      double v = 0.0;
      bool have = false;
      if (t >= 1) { v = a * cur[t - 1]; have = true; }
      if (t <= len - 1) { double w = P * cur[t]; v = have ? v + w : w; }
      if (t + 1 <= len - 1) v = v + (double)(t + 1) * cur[t + 1];
      nxt[t] = v;
    }
    len += 1;
    for (int t = 0; t < len; ++t) cur[t] = nxt[t];
  }
  for (int t = 0; t < len; ++t) out[t] = cur[t];
}

// P_LMN / P_LMN_j2 product factor (src/Integrals.f90:3102-3170) without the
// sign and q power: prod_{odd 3..l-1} prod_{3..m-1} prod_{3..n-1} / prod_{3..r+1 (j2: r+3)}.
TB_HD double p0_factor(int l, int m, int n, bool j2) {
  double prod = 1.0;
  int r = l + m + n;
  for (int i = 3; i <= l - 1; i += 2) prod = prod * i;
  for (int i = 3; i <= m - 1; i += 2) prod = prod * i;
  for (int i = 3; i <= n - 1; i += 2) prod = prod * i;
  int top = j2 ? r + 3 : r + 1;
  for (int i = 3; i <= top; i += 2) prod = prod / i;
  return prod;
}

// Pair-table layout (one entry per unordered group pair gi <= gj):
//  [0..2] P (Gaussian product centre), [3] p = alpha_i + alpha_j,
//  [4] pre = (pi_sp/p)^1.5 exp(-alpha_i alpha_j/p |A-B|^2),
//  [5] 0.25/p, [6..7] pad,
//  [8 + axis*ESZ + (la*(MAXA+1)+lb)*(2*MAXA+1) + t]  E^{la,lb}_t for that axis.
constexpr int E_T = 2 * MAXA + 1;
constexpr int ESZ = (MAXA + 1) * (MAXA + 1) * E_T;
constexpr int PAIR_STRIDE = 8 + 3 * ESZ;

TB_HD int pair_index(int i, int j, int ng) {  // i <= j
  return i * ng - i * (i - 1) / 2 + (j - i);
}
TB_HD int npairs(int ng) { return ng * (ng + 1) / 2; }
// function-pair index for a <= b, ordered by b then a
TB_HD int64_t fpair(int a, int b) { return (int64_t)b * (b + 1) / 2 + a; }

// Sort key of a group quartet from its shells' angular momenta: LLmax first
// (classes), then LK = min(L_bra, L_ket) and whether that is the bra (the
// contracted side of stage 1), then the four shells.  18 bits.
TB_HD uint32_t quartet_key(int Li, int Lj, int Lk, int Lr) {
  const int LL = Li + Lj + Lk + Lr, lb = Li + Lj, lk = Lk + Lr;
  const int LK = lb < lk ? lb : lk, XB = lb < lk ? 1 : 0;
  return (uint32_t)(((LL * 9 + LK) * 2 + XB) * 625 + ((Li * 5 + Lj) * 5 + Lk) * 5 + Lr);
}
constexpr uint32_t KEY_CLASS_DIV = 9 * 2 * 625;  // LLmax = key / KEY_CLASS_DIV
constexpr int KEY_BITS = 18;

// Series coefficients of u_n(x) = j_n(x) (2n+1)!!/x^n = sum_k c_{n,k} y^k,
// y = x^2: c_{n,0} = 1, c_{n,k} = c_{n,k-1} (-1/2) / (k (2n+2k+1)).
TB_HD constexpr double series_coef(int n, int k) {
  double c = 1.0;
  for (int j = 1; j <= k; ++j) c = c * (-0.5) / ((double)j * (double)(2 * n + 2 * j + 1));
  return c;
}

// Crossover x_c(L) between the small-x series branch and the upward
// recurrence, and the number of series terms needed below it.  Chosen from a
// float64 simulation against 40-digit values: both branches stay within
// ~1e-14 of max_b |j_b(x) x^b| for every L here.
TB_HD constexpr double bessel_crossover(int L) { return L <= 12 ? 0.75 * L : (double)L; }
TB_HD constexpr int series_terms(int L) {
  return L <= 2 ? 12 : (L <= 6 ? 16 : (L <= 12 ? 20 : SER_K));
}

}  // namespace tb
