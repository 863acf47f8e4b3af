// Adjoint of the total-j0 intensity with respect to the Gaussian centres: for
// a cotangent v(q) the vector-Jacobian product
//   g_c = sum_q v(q) dI(q)/dA_c        (A_c the centre of group c, 3 numbers)
// No reference counterpart (THISTLE computes I(q) only); the derivatives are
// those of the forward path of tot_integration (src/Integrals.f90:8-472,
// 5068-5226).  Per group quartet the forward value is
//   I_Q(q) = w K K' exp(-q^2 s) sum_TUV D_TUV G_TUV(q; H),
//   G_TUV = d^T/dHx d^U/dHy d^V/dHz j0(q|H|) = sum_k a_x a_y a_z J_b(q),
//   J_b(q) = j_b(qH) (q/H)^b,  b = (T-k1) + (U-k2) + (V-k3)
// (a the rrdj0 Hermite-like tables), or the P = Q polynomial when H is below
// cutoffcentre.  The geometry enters through K K' (the Gaussian-product
// prefactors), H = P_kr - P_ij and the McMurchie-Davidson coefficients inside
// D; the pair density rho is fixed.
//
// Stage A (q side, per quartet): Jbar_b = H^{-2b} sum_q v(q) exp(-q^2 s)
//   g_b(qH) for b <= LLmax + 1 (g_b = j_b x^b: upward recurrence above the
//   crossover, series below it), or the moments M_s = sum_q v exp(-q^2 s)
//   q^{2s} for P = Q quartets.  A thread per quartet, no cross-lane sums.
// Stage B (function-quartet side, thread per quartet):
//   Abar_TUV = w K K' sum_k a a a Jbar_b   (T+U+V <= LLmax + 1), then over the
//   function quartets, with the convolutions C of the forward stage 1 and
//   their centre derivatives dC (from dE/dA_i = 2 a_i E^{la+1,lb} - la
//   E^{la-1,lb} - (a_i/p) E^{la,lb}_{t-1} + 2 mu X E^{la,lb}, K excluded):
//     S0   = sum rho Abar.C C C             (-> d(K K')/dA: -2 mu X S0)
//     gH   = sum rho Abar_{TUV+e}.C C C      (-> dH/dA = -a_i/p, +a_k/p'), 0 for P = Q
//     gE_i = sum rho Abar.dC_i C C, gE_k likewise (dE/dA_j = -dE/dA_i)
//   and the four centres' gradients go into per-warp rows of shared memory
//   in a fixed order (deterministic), then into per-block partial rows.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "tb_kernels.h"
#include "tb_math.cuh"
#include "tb_stage1.cuh"

namespace tb {

namespace {

constexpr int DE_T = 2 * MAXA + 2;  // t = 0 .. 2 MAXA + 1

__device__ void emd(int l1, int l2, double PA, double PB, double a, double *out) {
  if (l1 >= l2) md_chain(l1, l2, PA, PB, a, out);
  else md_chain(l2, l1, PB, PA, a, out);
}

// dE^{la,lb}_t / dA_i (first centre of the pair), transposed like the E table:
// element t of (axis, la, lb) at dsoa[((axis (maxa+1) + la) (maxa+1) + lb) DE_T + t][pair].
__global__ void pair_dtables_kernel(int ng, int maxa, const int *__restrict__ gstart, const double *__restrict__ ga,
                                    const double *__restrict__ xyz, double *__restrict__ dsoa, int64_t gs_xyz,
                                    int64_t gs_dsoa) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t npair = npairs(ng);
  if (p >= npair) return;
  xyz += blockIdx.y * gs_xyz;
  dsoa += blockIdx.y * gs_dsoa;
  int i = 0, rem = p;
  while (rem >= ng - i) { rem -= ng - i; ++i; }
  const int j = i + rem;
  const int fi = gstart[i], fj = gstart[j];
  const double ai = ga[fi], aj = ga[fj], gp = ai + aj, mu = ai * aj / gp;
  for (int ax = 0; ax < 3; ++ax) {
    const double xi = xyz[3 * fi + ax], xj = xyz[3 * fj + ax];
    const double P = (ai * xi + aj * xj) / gp, X = xi - xj;
    const double PA = P - xi, PB = P - xj, a = 0.5 / gp;
    double E0[DE_T], Ep[DE_T], Em[DE_T];
    for (int la = 0; la <= maxa; ++la)
      for (int lb = 0; lb <= maxa; ++lb) {
        emd(la, lb, PA, PB, a, E0);
        emd(la + 1, lb, PA, PB, a, Ep);
        if (la > 0) emd(la - 1, lb, PA, PB, a, Em);
        const int64_t slot = ((int64_t)(ax * (maxa + 1) + la) * (maxa + 1) + lb) * DE_T;
        for (int t = 0; t < DE_T; ++t) {
          double d = 0.0;
          if (t <= la + lb + 1) d = 2.0 * ai * Ep[t];
          if (la > 0 && t <= la + lb - 1) d -= la * Em[t];
          if (t >= 1 && t - 1 <= la + lb) d -= ai / gp * E0[t - 1];
          if (t <= la + lb) d += 2.0 * mu * X * E0[t];
          dsoa[(slot + t) * npair + p] = d;
        }
      }
  }
}

// ---------------------------------------------------------------------------
// stage A
// ---------------------------------------------------------------------------
template <int N, int NK>
__device__ __forceinline__ double series_un(double y) {
  double p = series_coef(N, NK);
#pragma unroll
  for (int k = NK - 1; k >= 0; --k) p = fma(p, y, series_coef(N, k));
  return p;
}

// g_b = j_b(x) x^b for b = 0..LB1 below the crossover: series for the top two
// orders, downward recurrence, g_b = y^b / (2b+1)!! u_b.
template <int LB1>
__device__ __noinline__ void gb_small(double y, double *g) {
  constexpr int NK = series_terms(LB1);
  double uhi = series_un<LB1 + 1, NK>(y);
  double umid = series_un<LB1, NK>(y);
  double u[LB1 + 1];
  u[LB1] = umid;
#pragma unroll
  for (int b = LB1; b >= 1; --b) {
    double ulo = umid - (y * (1.0 / ((2.0 * b + 1.0) * (2.0 * b + 3.0)))) * uhi;
    u[b - 1] = ulo;
    uhi = umid;
    umid = ulo;
  }
  double w = 1.0;
#pragma unroll
  for (int b = 0; b <= LB1; ++b) {
    g[b] = w * u[b];
    w *= y / (2.0 * b + 3.0);
  }
}

// The q grid is staged through shared memory in chunks of AQ_CHUNK points as
// (q, 1/q, v(q)), so a point costs no division and no global load.  On an
// ascending grid the points below the crossover x = qH < XC form a prefix
// of each quartet's points; the warp walks the longest such prefix of its
// lanes with the per-point branch (series or recurrence) and the rest
// without it.
constexpr int AQ_CHUNK = 2048;

template <int LB1>
__global__ void __launch_bounds__(128) adjoint_q_kernel(AdjointQArgs A) {
  extern __shared__ double aq[];  // [AQ_CHUNK][3]: q, 1/q, v
  A.rec += blockIdx.y * A.gs_rec;
  A.adj += blockIdx.y * A.gs_rec;
  A.v += (int64_t)blockIdx.y * A.nq;
  const int64_t slot = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = slot < A.nquart;
  const int64_t idx = !act ? 0 : (A.perm ? (int64_t)A.perm[A.pbase + slot] - A.pbase : slot);
  const double *rec = A.rec + idx * A.rs;
  const bool p0 = act && (int)rec[2] == REC_P0;
  const double H = (act && !p0) ? rec[0] : 1.0, s = act ? rec[1] : 0.0, invH = 1.0 / H;
  constexpr double XC = bessel_crossover(LB1);
  double acc[LB1 + 1];
#pragma unroll
  for (int b = 0; b <= LB1; ++b) acc[b] = 0.0;
  const double dq = A.dq;
  double sd = 0.0, cd = 1.0;
  sincos(dq * H, &sd, &cd);
  const double kk = exp(-2.0 * dq * dq * s);
  double sn = 0.0, cs = 0.0, g = 0.0, r = 0.0;
  // series points of this lane: q H < XC (an ascending prefix on uniform grids)
  const double qc = XC * invH;
  for (int c0 = 0; c0 < A.nq; c0 += AQ_CHUNK) {
    const int cn = min(AQ_CHUNK, A.nq - c0);
    __syncthreads();
    for (int i = threadIdx.x; i < cn; i += blockDim.x) {
      const double q = A.q[c0 + i];
      aq[3 * i] = q;
      aq[3 * i + 1] = 1.0 / q;
      aq[3 * i + 2] = A.v[c0 + i];
    }
    __syncthreads();
    int pe = 0;  // this lane's points (in the chunk) that may need the series
    if (act && !p0) {
      if (!A.uniform) pe = cn;
      else {
        while (pe < cn && aq[3 * pe] < qc) ++pe;
      }
    }
    const int mse = (int)__reduce_max_sync(0xffffffffu, (unsigned)pe);
    if (!act) continue;
    auto seed = [&](int m) {
      const double q = aq[3 * m];
      sincos(q * H, &sn, &cs);
      g = exp(-(q * q) * s);
      r = exp(-(2.0 * q * dq + dq * dq) * s);
    };
    auto advance = [&]() {
      const double s2 = fma(sn, cd, cs * sd);
      cs = fma(cs, cd, -sn * sd);
      sn = s2;
      g *= r;
      r *= kk;
    };
    // seeds at the chunk start, every 64 points, at every point of a
    // non-uniform grid, and at point 1 when q[0] lies off the grid
    auto reseed_at = [&](int m) {
      const int gm = c0 + m;
      return m == 0 || !A.uniform || (gm & 63) == 0 || (gm == 1 && !A.first_on_grid);
    };
    if (p0) {
      // moments sum_q v exp(-q^2 s) q^{2s}
      for (int m = 0; m < cn; ++m) {
        if (reseed_at(m)) seed(m);
        const double q = aq[3 * m], w = aq[3 * m + 2] * g, q2 = q * q;
        double t = w;
#pragma unroll
        for (int b = 0; b <= LB1; ++b) {
          acc[b] += t;
          t *= q2;
        }
        advance();
      }
      continue;
    }
    auto up = [&](int m) {
      const double q = aq[3 * m], w = aq[3 * m + 2] * g, x = q * H;
      double gb[LB1 + 1];
      gb[0] = sn * (aq[3 * m + 1] * invH);
      gb[1] = gb[0] - cs;
      const double y = x * x;
#pragma unroll
      for (int b = 1; b < LB1; ++b) gb[b + 1] = fma((double)(2 * b + 1), gb[b], -y * gb[b - 1]);
#pragma unroll
      for (int b = 0; b <= LB1; ++b) acc[b] = fma(w, gb[b], acc[b]);
    };
    int m = 0;
    for (; m < mse; ++m) {
      if (reseed_at(m)) seed(m);
      if (aq[3 * m] * H >= XC) up(m);
      else {
        const double q = aq[3 * m], w = aq[3 * m + 2] * g, x = q * H;
        double gb[LB1 + 1];
        gb_small<LB1>(x * x, gb);
#pragma unroll
        for (int b = 0; b <= LB1; ++b) acc[b] = fma(w, gb[b], acc[b]);
      }
      advance();
    }
    for (; m < cn; ++m) {
      if (reseed_at(m)) seed(m);
      up(m);
      advance();
    }
  }
  if (!act) return;
  double *out = A.adj + idx * A.rs;
  if (p0) {
#pragma unroll
    for (int b = 0; b <= LB1; ++b) out[b] = acc[b];
  } else {
    const double ih2 = invH * invH;
    double f = 1.0;
#pragma unroll
    for (int b = 0; b <= LB1; ++b) {
      out[b] = acc[b] * f;
      f *= ih2;
    }
  }
}

// ---------------------------------------------------------------------------
// stage B
// ---------------------------------------------------------------------------
constexpr int ADJ_THREADS = 64;
// Threads per quartet of stage B: PA x PC split the bra x ket function pairs
// of the heavy classes (their partial sums are combined in a fixed order).
TB_HD constexpr int adj_pa(int L) { return L >= 6 ? 4 : (L >= 4 ? 2 : 1); }
TB_HD constexpr int adj_pc(int L) { return L >= 6 ? 4 : (L >= 4 ? 2 : 1); }

template <int L>
__device__ __forceinline__ int adx(int T, int U, int V) {  // simplex index of order L+1
  return ntuv(L + 1) - ntuv(L + 1 - T) + U * (L + 2 - T) - (U * (U - 1)) / 2 + V;
}

__device__ __forceinline__ const double *dsoa_slot(const AdjointFArgs &A, int axis, int la, int lb, int pair) {
  const int m1 = A.s1.emaxa + 1;
  return A.dsoa + (int64_t)((axis * m1 + la) * m1 + lb) * DE_T * A.s1.npair + pair;
}

// A read-only load the compiler may not merge with an earlier load of the
// same address: the ket E tables are read twice per function quartet rather
// than held in registers across the Abar contraction.
__device__ __forceinline__ double ld_nc(const double *p) {
  double v;
  asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

#ifndef TB_ADJ_MINB_LO
#define TB_ADJ_MINB_LO 1
#endif
#ifndef TB_ADJ_MINB_HI
#define TB_ADJ_MINB_HI 1
#endif
// resident blocks per SM the register allocation is sized for (L <= 3, L >= 4)
TB_HD constexpr int adj_minb(int L) { return L <= 3 ? TB_ADJ_MINB_LO : TB_ADJ_MINB_HI; }

template <int L, bool SPLIT>
__global__ void __launch_bounds__(ADJ_THREADS, adj_minb(L)) adjoint_f_kernel(AdjointFArgs A) {
  {
    const int64_t g = blockIdx.y;  // geometry of a batch
    A.s1.pairtab += g * A.s1.gs_pair;
    A.s1.esoa += g * A.s1.gs_esoa;
    A.adj += g * A.s1.gs_rec;
    A.dsoa += g * A.gs_dsoa;
    A.xyz += g * A.gs_xyz;
    A.gpart += g * A.gs_gpart;
  }
  constexpr int L1 = L + 1;
  constexpr int NA = ntuv(L1);
  constexpr int TM = L < 2 * MAXA ? L : 2 * MAXA;          // last E index
  constexpr int TD = L1 < 2 * MAXA + 1 ? L1 : 2 * MAXA + 1;  // last dE index
  extern __shared__ double sm[];
  const int ng = A.s1.ng;
  constexpr int QPB0 = SPLIT ? ADJ_THREADS / (adj_pa(L) * adj_pc(L)) : ADJ_THREADS;
  double *gw = sm + (size_t)QPB0 * NA + (threadIdx.x >> 5) * 3 * ng;  // this warp's gradient row
  for (int i = threadIdx.x; i < (ADJ_THREADS / 32) * 3 * ng; i += ADJ_THREADS) sm[(size_t)QPB0 * NA + i] = 0.0;
  __syncthreads();
  const Stage1Args &S = A.s1;
  const int64_t n = S.qend - S.qbegin;
  const int lane = threadIdx.x & 31;
  constexpr int PA = SPLIT ? adj_pa(L) : 1, PC = SPLIT ? adj_pc(L) : 1, P = PA * PC;
  constexpr int QPB = ADJ_THREADS / P;  // quartets per block and round
  const int gsub = threadIdx.x % P, grp = threadIdx.x / P, pa = gsub % PA, pc = gsub / PA;
  const unsigned gmask = P == 32 ? 0xffffffffu : (((1u << P) - 1u) << (lane - gsub));
  double *Ab = sm + grp;  // the group's Abar_TUV at Ab[adx * QPB]
  // this thread's bra tables: be[ax][t] at sbe[(ax (L+1) + t) ADJ_THREADS], bd likewise
  double *sbe = sm + (size_t)QPB0 * NA + (ADJ_THREADS / 32) * 3 * ng + threadIdx.x;
  double *sbd = sbe + 3 * (L + 1) * ADJ_THREADS;
#define BE(ax, t) sbe[((ax) * (L + 1) + (t)) * ADJ_THREADS]
#define BD(ax, t) sbd[((ax) * (L1 + 1) + (t)) * ADJ_THREADS]
  for (int64_t base = (int64_t)blockIdx.x * QPB; base < n; base += (int64_t)gridDim.x * QPB) {
    const int64_t qi = S.qbegin + base + grp;
    const bool act = base + grp < n;  // whole groups
    double gi[3] = {0, 0, 0}, gj[3] = {0, 0, 0}, gk[3] = {0, 0, 0}, gr[3] = {0, 0, 0};
    int ci = 0, cj = 0, ck = 0, cr = 0;
    if (act) {
      const QuartetHead Q = quartet_head<KIND_TOTAL>(S, qi);
      ci = Q.gi; cj = Q.gj; ck = Q.gk; cr = Q.gr;
      const double *jb = A.adj + S.recbase + (qi - S.qbegin) * (int64_t)S.rs;
      const double wpp = loop_weight(Q.loop) * Q.tb[4] * Q.tk[4];
      // Abar up to order L+1, entries shared out over the group
      int cnt = 0;
      if (Q.p0) {
        for (int T = 0; T <= L1; ++T)
          for (int U = 0; U <= L1 - T; ++U)
            for (int V = 0; V <= L1 - T - U; ++V) {
              if ((cnt++ % P) != gsub) continue;
              double a = 0.0;
              if (!((T | U | V) & 1)) {
                const int k = (T + U + V) / 2;
                a = p0_factor(T, U, V, false) * jb[k];
                if (k & 1) a = -a;
              }
              Ab[adx<L>(T, U, V) * QPB] = wpp * a;
            }
      } else {
        double ax[tp_size(L1)], ay[tp_size(L1)], az[tp_size(L1)];
        hermite_table(L1, Q.Hx, ax);
        hermite_table(L1, Q.Hy, ay);
        hermite_table(L1, Q.Hz, az);
        for (int T = 0; T <= L1; ++T)
          for (int U = 0; U <= L1 - T; ++U)
            for (int V = 0; V <= L1 - T - U; ++V) {
              if ((cnt++ % P) != gsub) continue;
              double a = 0.0;
              for (int k1 = 0; 2 * k1 <= T; ++k1)
                for (int k2 = 0; 2 * k2 <= U; ++k2)
                  for (int k3 = 0; 2 * k3 <= V; ++k3)
                    a += ax[tp_off(T) + k1] * ay[tp_off(U) + k2] * az[tp_off(V) + k3] *
                         jb[(T - k1) + (U - k2) + (V - k3)];
              Ab[adx<L>(T, U, V) * QPB] = wpp * a;
            }
      }
      if (P > 1) __syncwarp(gmask);
      const int pb = pair_index(Q.gi, Q.gj, ng), pk = pair_index(Q.gk, Q.gr, ng);
      const int64_t np = S.npair;
      double S0 = 0.0, gH[3] = {0, 0, 0}, gEi[3] = {0, 0, 0}, gEk[3] = {0, 0, 0};
      const int si = S.gstart[Q.gi], ni = S.gcount[Q.gi];
      const int sj = S.gstart[Q.gj], nj = S.gcount[Q.gj];
      const int sk = S.gstart[Q.gk], nk = S.gcount[Q.gk];
      const int sr = S.gstart[Q.gr], nr = S.gcount[Q.gr];
      for (int ab = pa; ab < ni * nj; ab += PA) {
        const int fa = si + ab / nj, fb = sj + ab % nj;
        const int la = S.flmn[fa], lb = S.flmn[fb];
        const int64_t rowp = fpair(min(fa, fb), max(fa, fb)) * S.np;
        const int lab[3][2] = {{la & 0xff, lb & 0xff}, {(la >> 8) & 0xff, (lb >> 8) & 0xff},
                               {(la >> 16) & 0xff, (lb >> 16) & 0xff}};
        // bra E (signed, skips as forward) and bra dE/dA_i (signed), in this
        // thread's shared-memory slots: they stay fixed over the ket loop
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          const double *e = esoa_slot(S, Q.skip & (1 << ax), ax, lab[ax][0], lab[ax][1], pb);
          const double *d = dsoa_slot(A, ax, lab[ax][0], lab[ax][1], pb);
#pragma unroll
          for (int t = 0; t <= L; ++t) {
            const double v = t <= TM ? e[t * np] : 0.0;
            BE(ax, t) = (t & 1) ? -v : v;
          }
#pragma unroll
          for (int t = 0; t <= L1; ++t) {
            const double v = t <= TD ? d[t * np] : 0.0;
            BD(ax, t) = (t & 1) ? -v : v;
          }
        }
        for (int cd = pc; cd < nk * nr; cd += PC) {
          const int fc = sk + cd / nr, fd = sr + cd % nr;
          double z = S.rho[rowp + fpair(min(fc, fd), max(fc, fd))];
          if (!(fabs(z) >= S.cutoffz)) continue;  // below cutoffz: the quartet adds exactly zero
          const int lc = S.flmn[fc], ld = S.flmn[fd];
          const int lcd[3][2] = {{lc & 0xff, ld & 0xff}, {(lc >> 8) & 0xff, (ld >> 8) & 0xff},
                                 {(lc >> 16) & 0xff, (ld >> 16) & 0xff}};
          const double *ke_p[3], *kd_p[3];
#pragma unroll
          for (int ax = 0; ax < 3; ++ax) {
            const bool sk2 = ax == 0 ? (Q.skip & 8) : (ax == 1 ? (Q.skip & 16) : false);
            ke_p[ax] = esoa_slot(S, sk2, ax, lcd[ax][0], lcd[ax][1], pk);
            kd_p[ax] = dsoa_slot(A, ax, lcd[ax][0], lcd[ax][1], pk);
          }
          // per axis the forward convolution C[T] = sum_t be[t] ke[T - t], T <= L+1
          double C[3][L1 + 1];
#pragma unroll
          for (int ax = 0; ax < 3; ++ax) {
            double ke[L + 1];
#pragma unroll
            for (int t = 0; t <= L; ++t) ke[t] = t <= TM ? ke_p[ax][t * np] : 0.0;
#pragma unroll
            for (int T = 0; T <= L1; ++T) {
              double c = 0.0;
#pragma unroll
              for (int t = 0; t <= T; ++t)
                if (t <= L && T - t <= L) c = fma(BE(ax, t), ke[T - t], c);
              C[ax][T] = c;
            }
          }
          // contractions of Abar with two of the three convolutions
          double Y[3][L1 + 1];
#pragma unroll
          for (int i = 0; i <= L1; ++i) Y[0][i] = Y[1][i] = Y[2][i] = 0.0;
#pragma unroll
          for (int T = 0; T <= L1; ++T)
#pragma unroll
            for (int U = 0; U <= L1 - T; ++U) {
              double w = 0.0;
              const double cxy = C[0][T] * C[1][U];
#pragma unroll
              for (int V = 0; V <= L1 - T - U; ++V) {
                const double a = Ab[adx<L>(T, U, V) * QPB];
                w = fma(a, C[2][V], w);
                Y[2][V] = fma(a, cxy, Y[2][V]);
              }
              Y[0][T] = fma(w, C[1][U], Y[0][T]);
              Y[1][U] = fma(w, C[0][T], Y[1][U]);
            }
          double s0 = 0.0, h0 = 0.0, h1 = 0.0, h2 = 0.0;
#pragma unroll
          for (int T = 0; T <= L; ++T) {
            s0 = fma(C[0][T], Y[0][T], s0);
            h0 = fma(C[0][T], Y[0][T + 1], h0);
            h1 = fma(C[1][T], Y[1][T + 1], h1);
            h2 = fma(C[2][T], Y[2][T + 1], h2);
          }
          S0 = fma(z, s0, S0);
          gH[0] = fma(z, h0, gH[0]);
          gH[1] = fma(z, h1, gH[1]);
          gH[2] = fma(z, h2, gH[2]);
          // centre derivatives of the convolutions, as correlations with Y:
          //   sum_T (bd * ke)[T] Y[T] = sum_t bd[t] sum_s ke[s] Y[t + s]
          //   sum_T (be * kd)[T] Y[T] = sum_t be[t] sum_s kd[s] Y[t + s]
#pragma unroll
          for (int ax = 0; ax < 3; ++ax) {
            double ke[L + 1], kd[L1 + 1];
#pragma unroll
            for (int t = 0; t <= L; ++t) ke[t] = t <= TM ? ld_nc(ke_p[ax] + t * np) : 0.0;
#pragma unroll
            for (int t = 0; t <= L1; ++t) kd[t] = t <= TD ? ld_nc(kd_p[ax] + t * np) : 0.0;
            double e = 0.0, k = 0.0;
#pragma unroll
            for (int t = 0; t <= L1; ++t) {
              double zi = 0.0, zk = 0.0;
#pragma unroll
              for (int s2 = 0; s2 <= L1 - t; ++s2) {
                if (s2 <= L) zi = fma(ke[s2], Y[ax][t + s2], zi);
                if (t <= L) zk = fma(kd[s2], Y[ax][t + s2], zk);
              }
              e = fma(BD(ax, t), zi, e);
              if (t <= L) k = fma(BE(ax, t), zk, k);
            }
            gEi[ax] = fma(z, e, gEi[ax]);
            gEk[ax] = fma(z, k, gEk[ax]);
          }
        }
      }
      if (P > 1) {
        // fixed-order sum of the group's partial sums (in its first thread)
        S0 = group_sum<P>(S0, gmask);
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          gH[ax] = group_sum<P>(gH[ax], gmask);
          gEi[ax] = group_sum<P>(gEi[ax], gmask);
          gEk[ax] = group_sum<P>(gEk[ax], gmask);
        }
        if (gsub != 0) S0 = gH[0] = gH[1] = gH[2] = gEi[0] = gEi[1] = gEi[2] = gEk[0] = gEk[1] = gEk[2] = 0.0;
        __syncwarp(gmask);  // Abar is rewritten by the next round
      }
      if (Q.p0) gH[0] = gH[1] = gH[2] = 0.0;  // the P = Q polynomial does not depend on H
      const double pij = Q.tb[3], pkr = Q.tk[3];
      const int hi = S.gstart[Q.gi], hj = S.gstart[Q.gj], hk = S.gstart[Q.gk], hr = S.gstart[Q.gr];
      const double ai = A.ga[hi], aj = A.ga[hj], ak = A.ga[hk], ar = A.ga[hr];
      const double muij = ai * aj / pij, mukr = ak * ar / pkr;
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const double Xij = A.xyz[3 * hi + ax] - A.xyz[3 * hj + ax];
        const double Xkr = A.xyz[3 * hk + ax] - A.xyz[3 * hr + ax];
        gi[ax] = -2.0 * muij * Xij * S0 - ai / pij * gH[ax] + gEi[ax];
        gj[ax] = 2.0 * muij * Xij * S0 - aj / pij * gH[ax] - gEi[ax];
        gk[ax] = -2.0 * mukr * Xkr * S0 + ak / pkr * gH[ax] + gEk[ax];
        gr[ax] = 2.0 * mukr * Xkr * S0 + ar / pkr * gH[ax] - gEk[ax];
      }
    }
    // fixed-order accumulation into the warp's row: lane 0 adds lane 0's
    // twelve values, then lane 1's, ...
    for (int l = 0; l < 32; ++l) {
      const int c4[4] = {__shfl_sync(0xffffffffu, ci, l), __shfl_sync(0xffffffffu, cj, l),
                         __shfl_sync(0xffffffffu, ck, l), __shfl_sync(0xffffffffu, cr, l)};
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const double v0 = __shfl_sync(0xffffffffu, gi[ax], l), v1 = __shfl_sync(0xffffffffu, gj[ax], l);
        const double v2 = __shfl_sync(0xffffffffu, gk[ax], l), v3 = __shfl_sync(0xffffffffu, gr[ax], l);
        if (lane == 0) {
          gw[3 * c4[0] + ax] += v0;
          gw[3 * c4[1] + ax] += v1;
          gw[3 * c4[2] + ax] += v2;
          gw[3 * c4[3] + ax] += v3;
        }
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * ng; i += ADJ_THREADS) {
    double t = 0.0;
    for (int w = 0; w < ADJ_THREADS / 32; ++w) t += sm[(size_t)QPB0 * NA + w * 3 * ng + i];
    A.gpart[(size_t)blockIdx.x * A.gstride + i] += t;
  }
#undef BE
#undef BD
}

}  // namespace

cudaError_t launch_pair_dtables(int ng, int maxa, const int *gstart, const double *ga, const double *xyz,
                                double *dsoa, int ngeom, int64_t gs_xyz, int64_t gs_dsoa, cudaStream_t st) {
  const int n = npairs(ng);
  pair_dtables_kernel<<<dim3((n + 127) / 128, ngeom), 128, 0, st>>>(ng, maxa, gstart, ga, xyz, dsoa, gs_xyz,
                                                                     gs_dsoa);
  return cudaGetLastError();
}

int64_t dsoa_doubles(int ng, int maxa) { return (int64_t)3 * (maxa + 1) * (maxa + 1) * DE_T * npairs(ng); }

cudaError_t launch_adjoint_q(int LB1, const AdjointQArgs &a, int ngeom, cudaStream_t st) {
  if (a.nquart <= 0) return cudaSuccess;
  const dim3 grid((unsigned)((a.nquart + 127) / 128), ngeom);
  const size_t smem = sizeof(double) * 3 * (size_t)std::min(a.nq, AQ_CHUNK);
  switch (LB1) {
#define TB_Q(n)                                                                                              \
  case n:                                                                                                    \
    if (smem > 48 * 1024) {                                                                                  \
      cudaError_t e = cudaFuncSetAttribute(adjoint_q_kernel<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                           (int)smem);                                                       \
      if (e != cudaSuccess) return e;                                                                        \
    }                                                                                                        \
    adjoint_q_kernel<n><<<grid, 128, smem, st>>>(a);                                                         \
    break;
    TB_Q(1) TB_Q(2) TB_Q(3) TB_Q(4) TB_Q(5) TB_Q(6) TB_Q(7) TB_Q(8) TB_Q(9)
#undef TB_Q
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int L, bool SPLIT>
static cudaError_t launch_adjoint_f_l(const AdjointFArgs &a, int grid, int ngeom, cudaStream_t st) {
  const int qpb = SPLIT ? ADJ_THREADS / (adj_pa(L) * adj_pc(L)) : ADJ_THREADS;
  const size_t smem = sizeof(double) * ((size_t)qpb * ntuv(L + 1) + (ADJ_THREADS / 32) * 3 * (size_t)a.s1.ng +
                                        (size_t)ADJ_THREADS * 3 * (2 * L + 3));
  cudaError_t e =
      cudaFuncSetAttribute(adjoint_f_kernel<L, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  adjoint_f_kernel<L, SPLIT><<<dim3(grid, ngeom), ADJ_THREADS, smem, st>>>(a);
  return cudaGetLastError();
}

int adjoint_f_quartets_per_block(int L, bool split) {
  return split ? ADJ_THREADS / (adj_pa(L) * adj_pc(L)) : ADJ_THREADS;
}

cudaError_t launch_adjoint_f(int L, const AdjointFArgs &a, int grid, int ngeom, bool split, cudaStream_t st) {
  if (a.s1.qend <= a.s1.qbegin) return cudaSuccess;
  switch (L) {
#define TB_F(n)                                                                     \
  case n:                                                                           \
    return split ? launch_adjoint_f_l<n, true>(a, grid, ngeom, st)                  \
                 : launch_adjoint_f_l<n, false>(a, grid, ngeom, st);
    TB_F(0) TB_F(1) TB_F(2) TB_F(3) TB_F(4) TB_F(5) TB_F(6) TB_F(7) TB_F(8)
#undef TB_F
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace tb
