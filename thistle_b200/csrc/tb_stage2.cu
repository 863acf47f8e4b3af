// Stage 2 of the quartet evaluation, one launch per LLmax class: the sum over
// the class's group quartets of F(q) exp(-q^2 (1/4p + 1/4p')) at every q point
// (bessels0rr, src/Integrals.f90:6662-6739, with an accurate generator; the
// P = Q polynomial of set_P0/P_LMN, :3001-3031, :3102-3135).
//
// Layout of the work: lanes over quartets, K quartets per lane, every lane of
// a warp at the same q point.  A warp takes 32 K quartets at a time and walks
// the q tile; per point each lane evaluates its K quartets (the Bessel order
// LB is a compile-time constant of the launch), the warp sums them with a
// butterfly and one lane adds the total into the warp's row of I(q) in shared
// memory.  Quartets are visited in the order of `perm` when given (sorted by
// quarter-octave of H, so that the lanes of a warp take the same branch of
// the Bessel generator at the same q).
//
// Generator, for F = sum_b hhat_b g_b(x), g_b = j_b(x) x^b, x = qH (hhat_b =
// h_b / H^{2b} is prepared by stage 1):
//   x >= x_c(LB): upward recurrence g_{b+1} = (2b+1) g_b - x^2 g_{b-1} from
//                 g_0 = sin x / x, g_1 = g_0 - cos x;
//   x <  x_c(LB): power series of u_n = j_n (2n+1)!! / x^n for the top two
//                 orders, then the stable downward recurrence, accumulated by
//                 Horner in x^2 / (2b+1).
// On uniform q grids z = exp(-q^2 s) e^{i q H} advances by z <- z w,
// w <- w k (w = r e^{i dq H}, r = exp(-(2 q dq + dq^2) s), k = exp(-2 dq^2 s)),
// restarted from direct values every 256 points (and at the start of every q
// chunk): over 256 steps the recurrences drift by ~1e-12 of the term's seed
// magnitude at most (float64 simulation against 30-digit values).
#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_kernels.h"
#include "tb_math.cuh"

namespace tb {

namespace {

#ifndef TB_S2_RESEED
#define TB_S2_RESEED 256
#endif
constexpr int RESEED = TB_S2_RESEED;

// Coefficients that lanes without a quartet point at: a zero record body,
// with room for the [H, s, kind, order] head in front of it.
__device__ const double kZeroRecord[4 + LMAXB + 4] = {0};

// The rare-branch helpers (small-x series, P = Q polynomial) are inlined into
// the checked point loop, which is not unrolled (K copies of each).
#define TB_S2_PATCH_ATTR __forceinline__

// Series coefficients c_{n,k} and the downward-recurrence factors in constant
// memory: FP64 instructions read them as constant-bank operands, where
// literals would first be moved into registers at every use.
struct SeriesTable {
  double c[LMAXB + 2][SER_K + 1];
  double r1[LMAXB + 2];  // 1 / ((2b + 1) (2b + 3))
  double r2[LMAXB + 2];  // 1 / (2b + 1)
};
constexpr SeriesTable make_series_table() {
  SeriesTable t{};
  for (int n = 0; n < LMAXB + 2; ++n) {
    for (int k = 0; k <= SER_K; ++k) t.c[n][k] = series_coef(n, k);
    t.r1[n] = 1.0 / ((2.0 * n + 1.0) * (2.0 * n + 3.0));
    t.r2[n] = 1.0 / (2.0 * n + 1.0);
  }
  return t;
}
__constant__ SeriesTable kSeries = make_series_table();

template <int N, int NK>
__device__ __forceinline__ double series_u(double y) {
  double p = kSeries.c[N][NK];
#pragma unroll
  for (int k = NK - 1; k >= 0; --k) p = fma(p, y, kSeries.c[N][k]);
  return p;
}

// Crossover of the polynomial form (defined below) and the series terms it
// needs: the polynomial-form classes (LB <= 8) switch to the series only
// below poly_crossover(LB), where fewer terms of u_LB, u_LB+1 than
// series_terms (sized for the recurrence crossover 0.75 LB) reach 1e-17:
// the smallest NK with |c_{n,NK+1}| x_c^{2 (NK+1)} <= 1e-17 for both orders
// (6, 8, 10, 11 terms for LB 2-5 against 12-16).
TB_HD constexpr double poly_crossover(int LB);
TB_HD constexpr int poly_series_terms(int LB) {
  const double y = poly_crossover(LB) * poly_crossover(LB);
  for (int nk = 1; nk < SER_K; ++nk) {
    bool ok = true;
    for (int n = LB; n <= LB + 1; ++n) {
      double t = series_coef(n, nk + 1);
      for (int j = 0; j <= nk; ++j) t *= y;
      if ((t < 0 ? -t : t) > 1e-17) ok = false;
    }
    if (ok) return nk;
  }
  return SER_K;
}

// x below the crossover: coefficients read from the record (h[0..LB]).
template <int LB>
__device__ TB_S2_PATCH_ATTR double bessel_small(const double *__restrict__ h, double y) {
  constexpr int NK = LB <= 8 ? poly_series_terms(LB) : series_terms(LB);
  double uhi = series_u<LB + 1, NK>(y);
  double umid = series_u<LB, NK>(y);
  double acc = h[LB] * umid;
#pragma unroll
  for (int b = LB; b >= 1; --b) {
    double ulo = umid - (y * kSeries.r1[b]) * uhi;
    acc = fma(acc, y * kSeries.r2[b], h[b - 1] * ulo);
    uhi = umid;
    umid = ulo;
  }
  return acc;
}

template <int LB>
__device__ __forceinline__ double bessel_up(const double *h, double x, double sn, double cs, double invx) {
  double g0 = sn * invx;
  if (LB == 0) return h[0] * g0;
  double g1 = g0 - cs;
  double F = fma(h[1], g1, h[0] * g0);
  const double y = x * x;
#pragma unroll
  for (int b = 1; b < LB; ++b) {
    double g2 = fma((double)(2 * b + 1), g1, -y * g0);
    F = fma(h[b + 1], g2, F);
    g0 = g1;
    g1 = g2;
  }
  return F;
}

// sum_{j <= n} c_j q2^j (the P = Q polynomial)
__device__ TB_S2_PATCH_ATTR double p0_poly(const double *__restrict__ c, int n, double q2) {
  double F = c[n];
  for (int j = n - 1; j >= 0; --j) F = fma(F, q2, c[j]);
  return F;
}

struct Seed {
  double S, C, wr, wi, g, r;
};

// Direct values at point q: z = g e^{i q H}, the step w = r e^{i dq H}, g
// and r (g = exp(-q^2 s), r = exp(-(2 q dq + dq^2) s)).
__device__ __noinline__ Seed seed_point(double q, double H, double s, double dq) {
  Seed z;
  double sn, cs, sd, cd;
  sincos(q * H, &sn, &cs);
  sincos(dq * H, &sd, &cd);
  z.g = exp(-(q * q) * s);
  z.r = exp(-(2.0 * q * dq + dq * dq) * s);
  z.S = z.g * sn;
  z.C = z.g * cs;
  z.wr = z.r * cd;
  z.wi = z.r * sd;
  return z;
}

template <bool B>
struct BoolTag {
  static constexpr bool value = B;
};

// Quartets per lane K and the register budget.  The polynomial-form orders
// (LB <= 8) take K = 2 (the default pair tile) or 1, the recurrence orders
// always 1.  K = 2 and every recurrence order get 128 registers a thread (4
// blocks of 4 warps or 2 of 8 per SM), K = 1 of a polynomial order 85 (6
// blocks of 4 warps, 3 of 8).  Measured on the AB6 step, two quartets per
// lane at 4 blocks of 4 warps beat 1 (6 blocks), 3 (3 blocks) and 2 at 3 or
// 5 blocks by 1-8 %; smaller molecules may prefer another shape, which the
// plan and batch tuners measure.
TB_HD constexpr int stage2_keff(int LB, int k) { return LB <= 8 ? k : 1; }
template <int LB, int K>
constexpr int stage2_minb() {
  return (K == 1 && LB <= 8) ? 3 : 2;
}

// Crossover of the polynomial form: the smallest x at which its float64 error
// stays within ~2e-13 of the largest term |hhat_b g_b| -- the level the same
// form (and the upward recurrence) has at large x -- from a simulation against
// 40-digit values over random coefficients spanning the H^{-2b} scales.
TB_HD constexpr double poly_crossover(int LB) {
  return LB == 0 ? 0.0 : LB == 1 ? 0.1 : LB == 2 ? 0.5 : LB == 3 ? 1.25 : LB == 4 ? 2.0 : LB == 5 ? 3.0
       : LB == 6 ? 4.0 : LB == 7 ? 5.0 : 6.0;
}

// q points per reduction block: the warp sums QB points at once with a
// reduce-scatter (3 halving rounds over lane bits 4..2, then 2 butterfly
// rounds), so the shuffle latency is paid once per QB points.
#ifndef TB_S2_QB
#define TB_S2_QB 8
#endif
constexpr int QB = TB_S2_QB;
TB_HD constexpr int padded_nq(int nq) { return (nq + QB - 1) / QB * QB; }

template <int LB, int K, bool J2>
__device__ __forceinline__ void stage2_class_body(Stage2ClassArgs &A, int64_t vb, int64_t vgrid) {
  extern __shared__ double sm[];
  const int nq = A.nq, nqb = padded_nq(nq);
  double2 *qs = reinterpret_cast<double2 *>(sm);  // (q, 1/q), padded with the last point
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int NW = blockDim.x >> 5;
  double *acc = sm + 2 * nqb + warp * nqb;
  for (int i = threadIdx.x; i < nqb; i += blockDim.x) {
    const double q = A.q[i < nq ? i : nq - 1];
    qs[i] = make_double2(q, 1.0 / q);
  }
  for (int i = threadIdx.x; i < NW * nqb; i += blockDim.x) sm[2 * nqb + i] = 0.0;
  __syncthreads();

  // polynomial form for the orders whose float64 accuracy it matches (LB <= 8)
  constexpr bool POLY = LB <= 8;
  constexpr double XC = POLY ? poly_crossover(LB) : bessel_crossover(LB);
  constexpr int NA = LB / 2 + 1;                   // A: powers q^0, q^2, .., q^{2 (NA-1)}
  constexpr int NB = LB >= 1 ? (LB - 1) / 2 + 1 : 1;  // B: q times powers of q^2
  const int64_t per = 32 * K;
  const int64_t nb = (A.nquart + per - 1) / per;
  // work item = (batch of 32 K quartets, chunk of the q tile); chunks start
  // on reseed points, so splitting a small class over q costs no accuracy
  const int chunk = A.chunk > 0 ? A.chunk : nqb;
  const int nch = (nqb + chunk - 1) / chunk;
  const int64_t nitems = nb * nch;
  const double dq = A.dq;
  const int jsel = (lane / (32 / QB)) & (QB - 1);
  for (int64_t it = vb * NW + warp; it < nitems; it += vgrid * NW) {
    const int64_t bt = it / nch;
    const int m0 = (int)(it - bt * nch) * chunk, m1 = min(nqb, m0 + chunk);
    // per quartet: z = exp(-q^2 s) e^{i q H} = C + i S advances by z <- z w,
    // w = r e^{i dq H}, w <- w kk (r, kk the Gaussian's ratios); the Gaussian
    // g itself (g <- g rg, rg <- rg kk) only through the patched prefix
    double H[K], invH[K], kk[K], S[K], C[K], wr[K], wi[K], g[K], rg[K];
    double hh[POLY ? 1 : K][POLY ? 1 : LB + 1];  // recurrence form: hhat_b
    double pa[POLY ? K : 1][NA], pb[POLY ? K : 1][NB];  // polynomial form
    long long qcb[K];  // bits of x_c / H: below it the series branch
    const double *hm[K];
    int p0n[K];  // P = Q polynomial order, or -1 for a Bessel quartet
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int64_t slot = bt * per + k * 32 + lane;
      const double *rec = kZeroRecord;
      double h = 1.0;
      p0n[k] = -1;
      bool bessel = false;
      if (slot < A.nquart) {
        const int64_t idx = A.perm ? (int64_t)A.perm[A.pbase + slot] - A.pbase : slot;
        rec = A.rec + idx * A.rs;
        if ((int)rec[2] == REC_P0) p0n[k] = (int)rec[3];
        else {
          h = rec[0];
          bessel = true;
        }
      }
      hm[k] = rec + 4;
      H[k] = h;
      invH[k] = 1.0 / h;
      qcb[k] = bessel ? __double_as_longlong(XC / h) : 0;
      if constexpr (POLY) {
        // sum_b hhat_b g_b(x) = (A(x) sin x + B(x) cos x) / x with
        // x g_b = P_b(x^2) sin x + x Q_b(x^2) cos x, P_0 = 1, Q_0 = 0,
        // P_1 = 1, Q_1 = -1 and (P, Q)_{b+1} = (2b+1) (P, Q)_b - x^2 (P, Q)_{b-1};
        // in q (x = qH, the 1/q left to the warp):
        //   F q = sum_j A_j H^{2j-1} q^{2j} sin + q sum_j B_j H^{2j} q^{2j} cos
        double Ac[NA], Bc[NB], Pm[NA], Pc[NA], Qm[NB], Qc[NB];
#pragma unroll
        for (int j = 0; j < NA; ++j) Ac[j] = Pm[j] = Pc[j] = 0.0;
#pragma unroll
        for (int j = 0; j < NB; ++j) Bc[j] = Qm[j] = Qc[j] = 0.0;
        if (bessel) {
          Pm[0] = 1.0;  // b = 0
          Ac[0] = hm[k][0];
          if (LB >= 1) {
            Pc[0] = 1.0;  // b = 1
            Qc[0] = -1.0;
            Ac[0] += hm[k][1];
            Bc[0] = -hm[k][1];
          }
#pragma unroll
          for (int bb = 1; bb < LB; ++bb) {
            const double c = (double)(2 * bb + 1), hb = hm[k][bb + 1];
            double Pn[NA], Qn[NB];
#pragma unroll
            for (int j = 0; j < NA; ++j) Pn[j] = c * Pc[j] - (j > 0 ? Pm[j - 1] : 0.0);
#pragma unroll
            for (int j = 0; j < NB; ++j) Qn[j] = c * Qc[j] - (j > 0 ? Qm[j - 1] : 0.0);
#pragma unroll
            for (int j = 0; j < NA; ++j) {
              Ac[j] = fma(hb, Pn[j], Ac[j]);
              Pm[j] = Pc[j];
              Pc[j] = Pn[j];
            }
#pragma unroll
            for (int j = 0; j < NB; ++j) {
              Bc[j] = fma(hb, Qn[j], Bc[j]);
              Qm[j] = Qc[j];
              Qc[j] = Qn[j];
            }
          }
        }
        double hp = invH[k];  // H^{2j-1}
#pragma unroll
        for (int j = 0; j < NA; ++j) {
          pa[k][j] = Ac[j] * hp;
          hp *= h * h;
        }
        hp = 1.0;  // H^{2j}
#pragma unroll
        for (int j = 0; j < NB; ++j) {
          pb[k][j] = Bc[j] * hp;
          hp *= h * h;
        }
      } else {
#pragma unroll
        for (int b = 0; b <= LB; ++b) hh[k][b] = p0n[k] < 0 ? hm[k][b] : 0.0;
      }
      kk[k] = exp(-2.0 * dq * dq * rec[1]);
      S[k] = C[k] = wr[k] = wi[k] = g[k] = rg[k] = 0.0;
    }
    // last point (exclusive) at which any lane of the warp may need a patch:
    // on an ascending uniform tile the series region of a quartet is a
    // prefix of its points (q < x_c / H), P = Q lanes need every point.
    // Point 0 (below every crossover, often the drivers' 1e-10 off the grid)
    // is taken apart by the block that starts the tile, so it alone makes no
    // prefix.
    int mse = 0;
    {
      int lane_end = 0;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (p0n[k] >= 0) lane_end = nqb;
        else if (qcb[k] > 0) {
          int e = nqb;
          if (A.uniform && nq > 1) {
            const double q1 = qs[1].x, qc = __longlong_as_double(qcb[k]);
            e = qc <= q1 ? 0 : (int)min((double)nqb, ceil((qc - q1) / dq) + 3.0);
          }
          lane_end = max(lane_end, e);
        }
      }
      mse = (int)__reduce_max_sync(0xffffffffu, (unsigned)lane_end);
    }
    // One lean point of the tile for the warp's 32 K quartets, all K as
    // straight-line code.  Polynomial form: sum_k (A_k S_k + q B_k C_k) is
    // F q summed over the lanes' quartets (J2: F q^3), the common 1/q (1/q^3)
    // applied once.
    auto point = [&](const int m) -> double {
      const double2 qq = qs[m];
      const double q = qq.x, iq = qq.y;
      double FA = 0.0, FB = 0.0;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if constexpr (POLY) {
          const double y = q * q;
          double ae = pa[k][NA - 1], bo = pb[k][NB - 1];
#pragma unroll
          for (int t = NA - 2; t >= 0; --t) ae = fma(ae, y, pa[k][t]);
#pragma unroll
          for (int t = NB - 2; t >= 0; --t) bo = fma(bo, y, pb[k][t]);
          FA = fma(ae, S[k], FA);
          FB = fma(bo, C[k], FB);
        } else {
          // the recurrence is linear in (sin, cos): fed z it gives F g
          double f = bessel_up<LB>(hh[k], q * H[k], S[k], C[k], iq * invH[k]);
          if (J2) f *= iq * iq;
          FA += f;
        }
      }
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double s2 = fma(S[k], wr[k], C[k] * wi[k]);
        C[k] = fma(C[k], wr[k], -S[k] * wi[k]);
        S[k] = s2;
        wr[k] *= kk[k];
        wi[k] *= kk[k];
      }
      if constexpr (POLY) return fma(q, FB, FA) * (J2 ? iq * iq * iq : iq);
      else return FA;
    };
    // One checked point: each lane evaluates, per quartet, only the branch its
    // point falls in -- the P = Q polynomial, the small-x series (both times
    // the Gaussian g), or the lean form -- and advances the rotation and g.
    auto cpoint = [&](const int m) -> double {
      const double2 qq = qs[m];
      const double q = qq.x, iq = qq.y;
      const long long qb = __double_as_longlong(q);
      double tot = 0.0;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        double v;
        if (p0n[k] >= 0) {
          v = p0_poly(hm[k], p0n[k], q * q) * g[k];
        } else if (qb < qcb[k]) {
          const double x = q * H[k];
          v = bessel_small<LB>(hm[k], x * x) * g[k];
          if (J2) v *= iq * iq;
        } else {
          if constexpr (POLY) {
            const double y = q * q;
            double ae = pa[k][NA - 1], bo = pb[k][NB - 1];
#pragma unroll
            for (int t = NA - 2; t >= 0; --t) ae = fma(ae, y, pa[k][t]);
#pragma unroll
            for (int t = NB - 2; t >= 0; --t) bo = fma(bo, y, pb[k][t]);
            v = fma(q, bo * C[k], ae * S[k]) * (J2 ? iq * iq * iq : iq);
          } else {
            v = bessel_up<LB>(hh[k], q * H[k], S[k], C[k], iq * invH[k]);
            if (J2) v *= iq * iq;
          }
        }
        tot += v;
      }
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double s2 = fma(S[k], wr[k], C[k] * wi[k]);
        C[k] = fma(C[k], wr[k], -S[k] * wi[k]);
        S[k] = s2;
        wr[k] *= kk[k];
        wi[k] *= kk[k];
        g[k] *= rg[k];
        rg[k] *= kk[k];
      }
      return tot;
    };
    auto seed = [&](const int m, auto checked) {
      const double q = qs[m].x;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const Seed z = seed_point(q, H[k], hm[k][-3], dq);
        S[k] = z.S;
        C[k] = z.C;
        wr[k] = z.wr;
        wi[k] = z.wi;
        if constexpr (decltype(checked)::value) {
          g[k] = z.g;
          rg[k] = z.r;
        }
      }
    };
    auto reduce = [&](double *Fv, const int mb) {
      // reduce-scatter: after the halving rounds over lane bits 4, 3, 2 the
      // lane holds point jsel summed over 8 lanes; two butterfly rounds finish
#pragma unroll
      for (int half = QB / 2, bit = 16; half >= 1; half >>= 1, bit >>= 1) {
        const bool up = lane & bit;
#pragma unroll
        for (int i = 0; i < half; ++i) {
          const double send = up ? Fv[i] : Fv[i + half];
          const double keep = up ? Fv[i + half] : Fv[i];
          Fv[i] = keep + __shfl_xor_sync(0xffffffffu, send, bit);
        }
      }
      double t = Fv[0];
#pragma unroll
      for (int bit = 32 / QB / 2; bit >= 1; bit >>= 1) t += __shfl_xor_sync(0xffffffffu, t, bit);
      if ((lane & (32 / QB - 1)) == 0) acc[mb + jsel] += t;
    };
    // Seeds (direct sincos / exp) at the chunk start and every RESEED points
    // after it, all on block boundaries; on a non-uniform tile at every
    // point, and when q[0] lies off the grid (the drivers' 1e-10) again at
    // point 1.  The checked points come first, one at a time with a butterfly
    // sum each (mse bounds a prefix; the whole chunk on a non-uniform tile),
    // rounded up to a block boundary; the rest take the lean path in blocks
    // of QB points, without the Gaussian g, point 0 with the checked branches.
    const bool every = !A.uniform;
    const bool off0 = m0 == 0 && !A.first_on_grid;
    int mce = every ? m1 : max(mse, m0);
    mce = min(m1, m0 + (max(mce - m0, 0) + QB - 1) / QB * QB);
#pragma unroll 1
    for (int m = m0; m < mce; ++m) {
      if (every || ((m - m0) & (RESEED - 1)) == 0 || (off0 && m == 1)) seed(m, BoolTag<true>());
      double t = cpoint(m);
#pragma unroll
      for (int bit = 16; bit >= 1; bit >>= 1) t += __shfl_xor_sync(0xffffffffu, t, bit);
      if (lane == 0) acc[m] += t;
    }
    for (int mb = mce; mb < m1; mb += QB) {
      double Fv[QB];
      if (mb == 0) {
        // point 0 with the checked points' branches, then the lean
        // recurrence (reseeded at point 1 when point 0 lies off the grid)
        seed(0, BoolTag<true>());
        Fv[0] = cpoint(0);
        if (off0) seed(1, BoolTag<false>());
#pragma unroll
        for (int j = 1; j < QB; ++j) Fv[j] = point(j);
      } else {
        if (((mb - m0) & (RESEED - 1)) == 0) seed(mb, BoolTag<false>());
#pragma unroll
        for (int j = 0; j < QB; ++j) Fv[j] = point(mb + j);
      }
      reduce(Fv, mb);
    }
  }
  __syncthreads();
  // fixed-order sum of the warp rows, added to this block's partial row
  for (int i = threadIdx.x; i < nq; i += blockDim.x) {
    double t = 0.0;
    for (int w = 0; w < NW; ++w) t += sm[2 * nqb + w * nqb + i];
    A.partial[(size_t)vb * A.pstride + i] += t;
  }
}

template <int LB, int K, bool J2>
__global__ void __launch_bounds__(STAGE2_MAXWARPS * 32, (stage2_minb<LB, K>())) stage2_class_kernel(Stage2ClassArgs A) {
  // geometry blockIdx.y of a batch
  A.rec += blockIdx.y * A.gs_rec;
  A.partial += blockIdx.y * A.gs_partial;
  stage2_class_body<LB, K, J2>(A, blockIdx.x, gridDim.x);
}

// Molecule batches: item i's virtual blocks are pre[i] .. pre[i+1]-1.
__device__ __forceinline__ int s2_batch_item(const int64_t *__restrict__ pre, int n, int64_t b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One virtual block of a batch item, as a separately allocated function: the
// persistent kernel calls the body of every order through one switch.
template <int LB, int K, bool J2>
__device__ __noinline__ void stage2_item(const Stage2ClassArgs *__restrict__ d, int it, int64_t vb, int64_t vgrid) {
  Stage2ClassArgs A = d[it];
  stage2_class_body<LB, K, J2>(A, vb, vgrid);
}

// The persistent molecule-batch kernel: a block takes the next virtual block
// from the counter, runs it, and repeats until none is left.  Items are
// ordered heaviest order first by the host, so the tail is short work.
template <int KS, bool J2>
__global__ void __launch_bounds__(STAGE2_MAXWARPS * 32, 2)
    stage2_persistent(const Stage2ClassArgs *__restrict__ d, const int64_t *__restrict__ pre, int n, int64_t blocks,
                      unsigned long long *__restrict__ next) {
  __shared__ long long take;
  for (;;) {
    __syncthreads();  // the previous virtual block's shared-memory reads are done
    if (threadIdx.x == 0) take = (long long)atomicAdd(next, 1ull);
    __syncthreads();
    const int64_t b = take;
    if (b >= blocks) return;
    const int it = s2_batch_item(pre, n, b);
    const int64_t vb = b - pre[it], vgrid = pre[it + 1] - pre[it];
    const int lb = d[it].lb;
    if constexpr (J2) {
      switch (lb) {
#define TB_C(n_) case n_: stage2_item<n_, stage2_keff(n_, KS), true>(d, it, vb, vgrid); break;
        TB_C(2) TB_C(3) TB_C(4) TB_C(5) TB_C(6) TB_C(7) TB_C(8) TB_C(9) TB_C(10)
        TB_C(11) TB_C(12) TB_C(13) TB_C(14) TB_C(15) TB_C(16) TB_C(17) TB_C(18)
#undef TB_C
        default: break;
      }
    } else {
      switch (lb) {
#define TB_C(n_) case n_: stage2_item<n_, stage2_keff(n_, KS), false>(d, it, vb, vgrid); break;
        TB_C(0) TB_C(1) TB_C(2) TB_C(3) TB_C(4) TB_C(5) TB_C(6) TB_C(7) TB_C(8)
        TB_C(9) TB_C(10) TB_C(11) TB_C(12) TB_C(13) TB_C(14) TB_C(15) TB_C(16)
#undef TB_C
        default: break;
      }
    }
  }
}

size_t class_smem(int nq, int nw) { return sizeof(double) * (size_t)padded_nq(nq) * (2 + nw); }

template <int LB, int K, bool J2>
cudaError_t launch_class_lk(const Stage2ClassArgs &a, int grid, int ngeom, int nw, cudaStream_t st) {
  size_t smem = class_smem(a.nq, nw);
  cudaError_t e =
      cudaFuncSetAttribute(stage2_class_kernel<LB, K, J2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  stage2_class_kernel<LB, K, J2><<<dim3(grid, ngeom), nw * 32, smem, st>>>(a);
  return cudaGetLastError();
}

template <int LB, bool J2>
cudaError_t launch_class_l(const Stage2ClassArgs &a, int grid, int ngeom, Stage2Tile t, cudaStream_t st) {
  if constexpr (LB <= 8)
    if (t.k == 2) return launch_class_lk<LB, 2, J2>(a, grid, ngeom, t.nw, st);
  return launch_class_lk<LB, 1, J2>(a, grid, ngeom, t.nw, st);
}

template <class F>
int occupancy(F *kernel, int nw, size_t smem) {
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 1;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, nw * 32, smem) != cudaSuccess) return 1;
  return nb > 0 ? nb : 1;
}

template <int LB, bool J2>
int blocks_per_sm_l(int nq, Stage2Tile t) {
  const size_t smem = class_smem(nq, t.nw);
  if constexpr (LB <= 8)
    if (t.k == 2) return occupancy(stage2_class_kernel<LB, 2, J2>, t.nw, smem);
  return occupancy(stage2_class_kernel<LB, 1, J2>, t.nw, smem);
}

template <int KS, bool J2>
cudaError_t launch_persistent_k(const Stage2ClassArgs *d, const int64_t *pre, int n, int64_t blocks, int nqmax,
                                int grid, int nw, unsigned long long *next, cudaStream_t st) {
  const size_t smem = class_smem(nqmax, nw);
  cudaError_t e =
      cudaFuncSetAttribute(stage2_persistent<KS, J2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  stage2_persistent<KS, J2><<<grid, nw * 32, smem, st>>>(d, pre, n, blocks, next);
  return cudaGetLastError();
}

}  // namespace

bool stage2_tile_valid(Stage2Tile t) { return (t.k == 1 || t.k == 2) && (t.nw == 4 || t.nw == 8); }

int stage2_persistent_blocks_per_sm(bool j2, int nqmax, Stage2Tile t) {
  const size_t smem = class_smem(nqmax, t.nw);
  if (j2) return t.k == 2 ? occupancy(stage2_persistent<2, true>, t.nw, smem)
                          : occupancy(stage2_persistent<1, true>, t.nw, smem);
  return t.k == 2 ? occupancy(stage2_persistent<2, false>, t.nw, smem)
                  : occupancy(stage2_persistent<1, false>, t.nw, smem);
}

cudaError_t launch_stage2_persistent(bool j2, const Stage2ClassArgs *d, const int64_t *pre, int n, int64_t blocks,
                                     int nqmax, int grid, Stage2Tile t, unsigned long long *next, cudaStream_t st) {
  if (n <= 0 || blocks <= 0 || grid <= 0) return cudaSuccess;
  if (!stage2_tile_valid(t)) return cudaErrorInvalidValue;
  if (j2) return t.k == 2 ? launch_persistent_k<2, true>(d, pre, n, blocks, nqmax, grid, t.nw, next, st)
                          : launch_persistent_k<1, true>(d, pre, n, blocks, nqmax, grid, t.nw, next, st);
  return t.k == 2 ? launch_persistent_k<2, false>(d, pre, n, blocks, nqmax, grid, t.nw, next, st)
                  : launch_persistent_k<1, false>(d, pre, n, blocks, nqmax, grid, t.nw, next, st);
}

int stage2_quartets_per_warp(int LB, Stage2Tile t) { return 32 * stage2_keff(LB, t.k); }

// total / elastic classes have LB = LLmax (0..16), j2 classes LLmax + 2 (2..18)
int stage2_class_blocks_per_sm(int LB, bool j2, int nq, Stage2Tile t) {
  if (j2) {
    switch (LB) {
#define TB_B(n) case n: return blocks_per_sm_l<n, true>(nq, t);
      TB_B(2) TB_B(3) TB_B(4) TB_B(5) TB_B(6) TB_B(7) TB_B(8) TB_B(9) TB_B(10)
      TB_B(11) TB_B(12) TB_B(13) TB_B(14) TB_B(15) TB_B(16) TB_B(17) TB_B(18)
#undef TB_B
      default: return 1;
    }
  }
  switch (LB) {
#define TB_B(n) case n: return blocks_per_sm_l<n, false>(nq, t);
    TB_B(0) TB_B(1) TB_B(2) TB_B(3) TB_B(4) TB_B(5) TB_B(6) TB_B(7) TB_B(8)
    TB_B(9) TB_B(10) TB_B(11) TB_B(12) TB_B(13) TB_B(14) TB_B(15) TB_B(16)
#undef TB_B
    default: return 1;
  }
}

cudaError_t launch_stage2_class(int LB, const Stage2ClassArgs &a, int grid, int ngeom, Stage2Tile t,
                                cudaStream_t st) {
  if (a.nquart <= 0 || grid <= 0) return cudaSuccess;
  if (!stage2_tile_valid(t)) return cudaErrorInvalidValue;
  if (a.j2) {
    switch (LB) {
#define TB_L(n) case n: return launch_class_l<n, true>(a, grid, ngeom, t, st);
      TB_L(2) TB_L(3) TB_L(4) TB_L(5) TB_L(6) TB_L(7) TB_L(8) TB_L(9) TB_L(10)
      TB_L(11) TB_L(12) TB_L(13) TB_L(14) TB_L(15) TB_L(16) TB_L(17) TB_L(18)
#undef TB_L
      default: return cudaErrorInvalidValue;
    }
  }
  switch (LB) {
#define TB_L(n) case n: return launch_class_l<n, false>(a, grid, ngeom, t, st);
    TB_L(0) TB_L(1) TB_L(2) TB_L(3) TB_L(4) TB_L(5) TB_L(6) TB_L(7) TB_L(8)
    TB_L(9) TB_L(10) TB_L(11) TB_L(12) TB_L(13) TB_L(14) TB_L(15) TB_L(16)
#undef TB_L
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace tb
