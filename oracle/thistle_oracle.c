/*
 * THISTLE scattering-intensity oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C CPU restatement of the reference Fortran routines that the
 * thistle_b200 CUDA path replaces.  It exists to check the product, never to
 * be the product: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs load it.  The product library never
 * links or calls this file.
 *
 * Every routine follows the reference loop order and arithmetic order
 * (built with -ffp-contract=off so that no FMA contraction changes rounding):
 *
 *   fill_md_table          src/Variables.f90:8-946
 *   variables_total        src/Variables.f90:948-1153 (z11/z22 :1045-1065,
 *                          pair centres and E12 :1113-1128, ddx remap :1132-1148)
 *   variables_elastic      src/Variables.f90:1159-1279
 *   tot_integration        src/Integrals.f90:8-472 (loops L1..L5, weights 8,4,4,2,1)
 *   tot_integration_j2     src/Integrals.f90:954-1424
 *   elastic_integration    src/Integrals.f90:1575-1939
 *   tot_integration_aligned src/Integrals.f90:1425-1573 (all ng^4 quartets)
 *   tot_integral_ijkr_pzero src/Integrals.f90:4955-5067
 *   tot_integral_k_ijkr    src/Integrals.f90:5068-5226
 *   tot_integral_k_ijkr_j2 src/Integrals.f90:5230-5420
 *   tot_integral_k_ijkr_alig src/Integrals.f90:5588-5727
 *   integral_ijkr_pzero    src/Integrals.f90:4751-4863
 *   integral_k_ijkr        src/Integrals.f90:5730-5900
 *   BesselDeriv            src/Integrals.f90:4708-4746
 *   BesselDeriv2j          src/Integrals.f90:6370-6434
 *   rrdj2a / rrdj2b        src/Integrals.f90:6902-6952
 *   Hermite_like_coeffs    src/Integrals.f90:7037-7059
 *   rrdj0                  src/Integrals.f90:7062-7091
 *   bessels0rr             src/Integrals.f90:6662-6739
 *   dphrec                 src/Integrals.f90:7147-7184
 *   set_P0 / P_LMN         src/Integrals.f90:3001-3031, 3102-3135
 *   set_P0_j2 / P_LMN_j2   src/Integrals.f90:3034-3064, 3137-3170
 *   group_start/count      src/main_calculation.f90:85-93
 *   QCOORD3                src/main_calculation.f90:864-929
 *
 * Reference quirks kept on purpose: single-precision pi in E12
 * (acos(-1.0000), src/Variables.f90:994), the fixed 100-term backward start of
 * dphrec (bessel_mode 0), the 1.0e-30 single-precision MD skips where the
 * reference has them active, the sum(h_saved)==0 early return of the elastic
 * kernel, and loop 1's h=(..)**0.5 against sqrt() elsewhere.
 *
 * bessel_mode 1 replaces only dphrec's starting order (100) by one that grows
 * with x, giving accurate j_n where the reference's recurrence has not
 * converged (x = qH above about 75); everything else is unchanged.
 *
 * Pins: the Julia port's known-answer tests (test/runtests.jl:57-157) and the
 * documented form-factor values (docs/src/kernels.md:76-79) are reproduced by
 * tests/test_oracle_kat.py; analytic sum rules pin the full driver.  No stored
 * I(q) output of the reference exists, so full-I(q) parity is against this file.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define DIM 20
/* Fortran literal 1.0e-30 is default (single) real. */
#define SKIP30 ((double)1.0e-30f)
/* acos(-1.0000) evaluated in single precision (src/Variables.f90:994). */
#define PI_SP ((double)3.14159265358979323846f)

enum { ORC_OK = 0, ORC_ERR_ARG = -1, ORC_ERR_L = -2, ORC_ERR_MEM = -3 };

/* ------------------------------------------------------------------------ */
/* Special functions                                                         */
/* ------------------------------------------------------------------------ */

/* Fortran x**n for integer n >= 0, by repeated multiplication. */
static double ipow(double x, int n) {
    double r = 1.0;
    for (int i = 0; i < n; ++i) r *= x;
    return r;
}

/* dphrec (src/Integrals.f90:7147-7184) for one argument.  rbes[k] = j_k(x)
 * for k < lmax1.  leps1 is the backward-recurrence start (100 in the
 * reference). */
static void dphrec1(double x, double *rbes, int leps1, int lmax1) {
    double xx = x * x;
    for (int k = 0; k < leps1; ++k) rbes[k] = 0.0;
    rbes[leps1 - 1] = 1.0;
    rbes[leps1 - 2] = 1.0;
    double cx = cos(x), sx = sin(x);
    double rneu2 = cx + x * sx;
    for (long K = 3; K <= leps1; ++K) {
        long LU = leps1 - K + 2;                 /* 1-based */
        rbes[LU - 2] = rbes[LU - 1] - xx / (4.0 * LU * LU - 1.0) * rbes[LU];
    }
    double A = rbes[0] * rneu2 - xx / 3.0 * rbes[1] * cx;
    for (int k = 0; k < leps1; ++k) rbes[k] = rbes[k] / A;
    double cu = 1.0 / x;
    for (long K = 1; K <= lmax1; ++K) {
        double W = 2.0 * (K - 1);
        cu = x / (W + 1.0) * cu;
        rbes[K - 1] = cu * rbes[K - 1];
    }
}

static int dphrec_start(double x, int bessel_mode) {
    if (bessel_mode == 0) return 100;
    /* Miller start well beyond the turning point n ~ x. */
    double s = x + 12.0 * cbrt(x > 1.0 ? x : 1.0) + 40.0;
    int n = (int)ceil(s);
    return n < 100 ? 100 : n;
}

/* bessels0rr (src/Integrals.f90:6662-6739): F(q) = j0(qH) h0 +
 * sum_{b=1..order} j_b(qH) (q/H)^b h_b. */
static void bessels0rr(double *hsum, int order, const double *mu, int nq, double H,
                       const double *h_saved, int bessel_mode, double *scratch) {
    for (int iq = 0; iq < nq; ++iq) {
        double pmu = H * mu[iq];
        double invpmu = mu[iq] / H;
        double s = sin(pmu);
        double acc = s / pmu * h_saved[0];
        int leps = dphrec_start(pmu, bessel_mode);
        dphrec1(pmu, scratch, leps, order + 1);
        for (int beta = 1; beta <= order; ++beta)
            acc = acc + scratch[beta] * ipow(invpmu, beta) * h_saved[beta];
        hsum[iq] = acc;
    }
}

/* rrdj0 (src/Integrals.f90:7062-7091); a[L][p] (0-based). */
static void rrdj0(int lmax, double x, double a[DIM][DIM]) {
    memset(a, 0, sizeof(double) * DIM * DIM);
    a[0][0] = 1.0;
    a[1][1] = -x;
    for (int l = 2; l <= lmax; ++l) a[l][0] = -(double)(l - 1) * a[l - 2][0];
    for (int l = 2; l <= lmax; ++l)
        for (int p = 1; p <= l; ++p)
            a[l][p] = -(double)(l - 1) * a[l - 2][p] - x * a[l - 1][p - 1];
}

/* Hermite_like_coeffs (src/Integrals.f90:7037-7059). */
static void hermite_like(double a[DIM][DIM], int LLmax, double Hx) {
    memset(a, 0, sizeof(double) * DIM * DIM);
    a[0][0] = 1.0;
    if (LLmax > 0) a[1][1] = -Hx;
    for (int L = 2; L <= LLmax; ++L) {
        a[L][0] = -(double)(L - 1) * a[L - 2][0];
        for (int ka = 1; ka <= LLmax; ++ka)
            a[L][ka] = -Hx * a[L - 1][ka - 1] - (double)(L - 1) * a[L - 2][ka];
    }
}

/* BesselDeriv (src/Integrals.f90:4708-4746): BD[0..LLmax]. */
static void bessel_deriv(double *BD, int LL, int MM, int NN, double a[DIM][DIM],
                         double b[DIM][DIM], double c[DIM][DIM], int LLmax) {
    for (int i = 0; i <= LLmax; ++i) BD[i] = 0.0;
    for (int ii = 0; ii <= LL; ++ii) {
        double C1 = a[LL][ii];
        if (fabs(C1) < SKIP30) continue;
        for (int jj = 0; jj <= MM; ++jj) {
            double Ct2 = b[MM][jj];
            if (fabs(Ct2) < SKIP30) continue;
            double C2 = C1 * Ct2;
            for (int kk = 0; kk <= NN; ++kk) {
                double Ct3 = c[NN][kk];
                if (fabs(Ct3) < SKIP30) continue;
                double C3 = C2 * Ct3;
                int temp = LL + MM + NN - ii - jj - kk;
                int ceil_ = temp / 2 + temp % 2;
                int hOrder = ceil_ + ii + jj + kk;
                BD[hOrder] = BD[hOrder] + C3;
            }
        }
    }
}

/* rrdj2a / rrdj2b (src/Integrals.f90:6902-6952), kept in the reference's
 * column-shifted layout: a[L][p+2] holds the rrdj0 coefficient a(L,p). */
static void rrdj2a(int lmax, double x, double a[DIM][DIM]) {
    memset(a, 0, sizeof(double) * DIM * DIM);
    a[0][2] = 1.0;
    a[1][3] = -x;
    for (int l = 2; l <= lmax; ++l) a[l][2] = -(double)(l - 1) * a[l - 2][2];
    for (int l = 2; l <= lmax; ++l)
        for (int p = 1; p <= l; ++p)
            if (p + 2 < DIM) a[l][p + 2] = -(double)(l - 1) * a[l - 2][p + 2] - x * a[l - 1][p + 1];
}

static void rrdj2b(int lmax, double a[DIM][DIM], double b[DIM][DIM]) {
    memset(b, 0, sizeof(double) * DIM * DIM);
    for (int l = 1; l <= lmax; ++l)
        for (int p = 0; p <= l; ++p) {
            double carg = (l + p) / 2.0;
            if (p + 2 < DIM) b[l][p] = 2.0 * ceil(carg) * a[l][p + 2];
        }
}

/* BesselDeriv2j (src/Integrals.f90:6370-6434): BD[0..DIM-1]. */
static void bessel_deriv2j(double *BD, double hz, double h, int LL, int MM, int NN,
                           double a[DIM][DIM], double b[DIM][DIM], double c[DIM][DIM],
                           double ap[DIM][DIM], double bp[DIM][DIM], double cp[DIM][DIM]) {
    double pi = acos(-1.0);
    double eta = 3.0 * (hz * hz) - h * h;
    for (int i = 0; i < DIM; ++i) BD[i] = 0.0;
    for (int ii = 0; ii <= LL + 2; ++ii) {
        double C1 = a[LL][ii], C1p = ap[LL][ii];
        for (int jj = 0; jj <= MM + 2; ++jj) {
            double Ct2 = b[MM][jj], Ct2p = bp[MM][jj];
            for (int kk = 0; kk <= NN + 2; ++kk) {
                double Ct3 = c[NN][kk], Ct3p = cp[NN][kk];
                double C3 = C1 * Ct2 * Ct3 * eta + C1p * Ct2 * Ct3 + C1 * Ct2p * Ct3 + C1 * Ct2 * Ct3p;
                int hOrder = (int)ceil((LL + MM + NN + ii + jj + kk) / 2.0 - 1.0);
                if (hOrder >= 0 && hOrder < DIM) BD[hOrder] = BD[hOrder] + C3;
            }
        }
    }
    double f = 0.25 * pow(5.0 / pi, 0.5);
    for (int i = 0; i < DIM; ++i) BD[i] = f * BD[i];
}

/* P_LMN / P_LMN_j2 (src/Integrals.f90:3102-3170) for one (l,m,n). */
static double p_lmn(int l, int m, int n, double q, int j2) {
    double prod = 1.0;
    int r = l + m + n;
    for (int i = 3; i <= l - 1; i += 2) prod = prod * i;
    for (int i = 3; i <= m - 1; i += 2) prod = prod * i;
    for (int i = 3; i <= n - 1; i += 2) prod = prod * i;
    int top = j2 ? r + 3 : r + 1;
    for (int i = 3; i <= top; i += 2) prod = prod / i;
    double sgn = ipow(-1.0, r / 2);
    if (!j2) return prod * sgn * ipow(q, r);
    return (l + m - 2 * n) / 4.0 * prod * sgn * ipow(q, r);
}

/* ------------------------------------------------------------------------ */
/* McMurchie-Davidson coefficients (fill_md_table, src/Variables.f90:8-946)  */
/* ------------------------------------------------------------------------ */

/* E^{l1,l2}_t for l1 >= l2 in the reference's unrolled order: the PA chain
 * from E^{0,0} up to E^{l1,0}, then the PB chain up to E^{l1,l2}.  Each step
 * is a*E_{t-1} + P*E_t + (t+1)*E_{t+1}, left to right. */
static void md_chain(int l1, int l2, double PA, double PB, double a, double *out) {
    double cur[2 * 8 + 2], nxt[2 * 8 + 2];
    int len = 1;
    cur[0] = 1.0;
    for (int step = 0; step < l1 + l2; ++step) {
        double P = step < l1 ? PA : PB;
        for (int t = 0; t <= len; ++t) {
            double v = 0.0;
            int have = 0;
            if (t >= 1) { v = a * cur[t - 1]; have = 1; }
            if (t <= len - 1) { double w = P * cur[t]; v = have ? v + w : w; have = 1; }
            if (t + 1 <= len - 1) { double w = (double)(t + 1) * cur[t + 1]; v = v + w; }
            nxt[t] = v;
        }
        len += 1;
        for (int t = 0; t < len; ++t) cur[t] = nxt[t];
    }
    for (int t = 0; t < len; ++t) out[t] = cur[t];
}

/* ------------------------------------------------------------------------ */
/* Setup shared by all calculation types                                     */
/* ------------------------------------------------------------------------ */

typedef struct {
    int ngto, ng, maxl, nq, dt, dl;
    const double *ga, *xx, *yy, *zz, *q;
    const int *l, *m, *n;
    int *gs, *gc;                  /* 1-based function index of group head, count */
    double *px, *py, *pz;          /* (ng,ng) column-major */
    double *e12;                   /* (nq,ng,ng) */
    double *ddx, *ddy, *ddz;       /* (dt,dl,dl,ng,ng) */
    double *p0;                    /* (nq,4maxl+1,4maxl+1,4maxl+1) */
    int p0d;
} setup_t;

#define PX(S, i, j) ((S)->px[(i) + (size_t)(S)->ng * (j)])
#define PY(S, i, j) ((S)->py[(i) + (size_t)(S)->ng * (j)])
#define PZ(S, i, j) ((S)->pz[(i) + (size_t)(S)->ng * (j)])
#define E12(S, iq, i, j) ((S)->e12[(iq) + (size_t)(S)->nq * ((i) + (size_t)(S)->ng * (j))])
/* pointer to ddx(:,:,:,gj,gi) (0-based gi,gj) */
#define DDP(S, arr, gj, gi) ((arr) + (size_t)(S)->dt * (S)->dl * (S)->dl * ((gj) + (size_t)(S)->ng * (gi)))

static void free_setup(setup_t *S) {
    free(S->gs); free(S->gc); free(S->px); free(S->py); free(S->pz); free(S->e12);
    free(S->ddx); free(S->ddy); free(S->ddz); free(S->p0);
    memset(S, 0, sizeof(*S));
}

/* fill_md_table (src/Variables.f90:8-946) for one Cartesian axis, written
 * straight through the remap of src/Variables.f90:1132-1148 into the
 * group-indexed table dd = ddx(t, l(u)+1, l(v)+1, group(v), group(u)). */
static void md_axis(setup_t *S, const int *lax, const double *x, const int *g0, double *dd) {
    int N = S->ngto;
    double E[2 * 8 + 2];
    for (int i = 0; i < N; ++i) {
        for (int j = i; j < N; ++j) {
            double gaP = S->ga[i] + S->ga[j];
            double Px = (S->ga[i] * x[i] + S->ga[j] * x[j]) / gaP;
            int ii = i, jj = j;
            if (i != j && lax[i] < lax[j]) { ii = j; jj = i; }   /* l1 >= l2 */
            double PA = Px - x[ii], PB = Px - x[jj];
            double a = 0.5 / gaP;
            int l1 = lax[ii], l2 = lax[jj];
            md_chain(l1, l2, PA, PB, a, E);
            for (int pass = 0; pass < 2; ++pass) {
                if (pass == 1 && ii == jj) break;
                int u = pass == 0 ? ii : jj, v = pass == 0 ? jj : ii;
                double *blk = DDP(S, dd, g0[v], g0[u]);
                for (int t = 0; t <= l1 + l2; ++t)
                    blk[t + S->dt * (lax[u] + S->dl * lax[v])] = E[t];
            }
        }
    }
}

/* p0kind: 0 none, 1 set_P0, 2 set_P0_j2 */
static int build_setup(setup_t *S, int ngto, const double *ga, const int *l, const int *m,
                       const int *n, const double *xx, const double *yy, const double *zz,
                       const int *group, const double *q, int nq, int p0kind) {
    memset(S, 0, sizeof(*S));
    S->ngto = ngto; S->ga = ga; S->l = l; S->m = m; S->n = n;
    S->xx = xx; S->yy = yy; S->zz = zz; S->q = q; S->nq = nq;
    int ng = 0, maxl = 0;
    for (int i = 0; i < ngto; ++i) {
        if (group[i] > ng) ng = group[i];
        if (group[i] < 1) return ORC_ERR_ARG;
        if (l[i] > maxl) maxl = l[i];
    }
    if (ng <= 0) return ORC_ERR_ARG;
    for (int i = 0; i < ngto; ++i) if (m[i] > 4 || n[i] > 4) return ORC_ERR_L;
    if (maxl > 4) return ORC_ERR_L;
    /* the reference sizes every table by maxval(l) (src/main_calculation.f90:63-64) */
    int maxa = maxl;
    for (int i = 0; i < ngto; ++i) { if (m[i] > maxa) maxa = m[i]; if (n[i] > maxa) maxa = n[i]; }
    S->ng = ng; S->maxl = maxa; S->dt = 2 * maxa + 1; S->dl = maxa + 1;
    S->gs = calloc(ng, sizeof(int)); S->gc = calloc(ng, sizeof(int));
    for (int g = 1; g <= ng; ++g)
        for (int j = 0; j < ngto; ++j)
            if (group[j] == g) {
                int c = 0;
                for (int k = 0; k < ngto; ++k) c += group[k] == g;
                S->gs[g - 1] = j + 1;
                S->gc[g - 1] = c;
                break;
            }
    size_t ng2 = (size_t)ng * ng;
    S->px = calloc(ng2, sizeof(double)); S->py = calloc(ng2, sizeof(double));
    S->pz = calloc(ng2, sizeof(double)); S->e12 = calloc(ng2 * nq, sizeof(double));
    size_t dsz = (size_t)S->dt * S->dl * S->dl * ng2;
    S->ddx = calloc(dsz, sizeof(double)); S->ddy = calloc(dsz, sizeof(double));
    S->ddz = calloc(dsz, sizeof(double));
    if (!S->px || !S->py || !S->pz || !S->e12 || !S->ddx || !S->ddy || !S->ddz) return ORC_ERR_MEM;
    int *g0 = malloc(sizeof(int) * ngto);
    for (int i = 0; i < ngto; ++i) g0[i] = group[i] - 1;
    md_axis(S, l, xx, g0, S->ddx);
    md_axis(S, m, yy, g0, S->ddy);
    md_axis(S, n, zz, g0, S->ddz);
    free(g0);
    double pi = PI_SP;
    for (int jj = 0; jj < ng; ++jj) {
        int j = S->gs[jj] - 1;
        for (int ii = 0; ii < ng; ++ii) {
            int i = S->gs[ii] - 1;
            double gaP = ga[i] + ga[j];
            PX(S, ii, jj) = (ga[i] * xx[i] + ga[j] * xx[j]) / gaP;
            PY(S, ii, jj) = (ga[i] * yy[i] + ga[j] * yy[j]) / gaP;
            PZ(S, ii, jj) = (ga[i] * zz[i] + ga[j] * zz[j]) / gaP;
            double dx = xx[i] - xx[j], dy = yy[i] - yy[j], dz = zz[i] - zz[j];
            double pre = pow(pi / gaP, 1.5);
            double kab = exp(-ga[i] * ga[j] / gaP * (pow(dx, 2.0) + pow(dy, 2.0) + pow(dz, 2.0)));
            for (int iq = 0; iq < nq; ++iq)
                E12(S, iq, ii, jj) = pre * exp(-q[iq] * q[iq] * 0.25 / gaP) * kab;
        }
    }
    if (p0kind) {
        int lmax4 = 4 * maxl;
        S->p0d = lmax4 + 1;
        size_t psz = (size_t)nq * S->p0d * S->p0d * S->p0d;
        S->p0 = calloc(psz, sizeof(double));
        if (!S->p0) return ORC_ERR_MEM;
        double fj2 = sqrt(5.0 / acos(-1.0));
        for (int k = 0; k <= lmax4; k += 2)
            for (int j = 0; j <= lmax4; j += 2)
                for (int i = 0; i <= lmax4; i += 2)
                    for (int iq = 0; iq < nq; ++iq) {
                        if (p0kind == 1) {
                            S->p0[iq + (size_t)nq * (i + S->p0d * (j + (size_t)S->p0d * k))] = p_lmn(i, j, k, q[iq], 0);
                        } else {
                            double v = p_lmn(k, j, i, q[iq], 1);
                            S->p0[iq + (size_t)nq * (k + S->p0d * (j + (size_t)S->p0d * i))] = v * fj2;
                        }
                    }
    }
    return ORC_OK;
}

#define P0AT(S, iq, L, M, N) ((S)->p0[(iq) + (size_t)(S)->nq * ((L) + (S)->p0d * ((M) + (size_t)(S)->p0d * (N)))])

/* ------------------------------------------------------------------------ */
/* Per-quartet kernels                                                       */
/* ------------------------------------------------------------------------ */

/* ztot of every primitive quartet of a group quartet, dense over the
 * positions (a,b,c,d) of (i',j',k',r') inside groups (gi,gj,gk,gr). */
typedef struct { int si, sj, sk, sr; const double *z; } zblock_t;
#define ZAT(Z, a, b, c, d) ((Z)->z[(((size_t)(a) * (Z)->sj + (b)) * (Z)->sk + (c)) * (Z)->sr + (d)])

typedef struct { int kind; int bessel_mode; double cutoff1, cutoff2, cutoffcentre; } kopts_t;
enum { K_TOTAL = 0, K_ELASTIC = 1, K_J2 = 2, K_ELASTIC_J2 = 3 };

/* |E|<1e-30 skips active per kernel (bit k = k-th of MDL MDM MDN MDLp MDMp MDNp) */
#define SKIP_PZERO   0x1f   /* tot_integral_ijkr_pzero :5010-5031 */
#define SKIP_KIJKR   0x00   /* tot_integral_k_ijkr: all commented out :5172-5193 */
#define SKIP_ELASTIC 0x1f   /* integral_k_ijkr :5834-5855, integral_ijkr_pzero :4811-4832 */
#define SKIP_J2      0x0f   /* tot_integral_k_ijkr_j2 (MDMp, MDNp not skipped) */
#define SKIP_ALIG    0x1f   /* tot_integral_k_ijkr_alig */

typedef void (*visit_fn)(void *, int, int, int, int, int, int, double);

/* The six-deep MD loop shared by every per-quartet kernel, in the reference
 * order: (i,j,k,r) primitives, then ll,mm,nn (bra), llp,mmp,nnp (ket). */
static void hermite_loop(const setup_t *S, int gi, int gj, int gk, int gr,
                         const double *dx1, const double *dy1, const double *dz1,
                         const double *dx2, const double *dy2, const double *dz2,
                         const zblock_t *Z, double cutoff1, double cutoff2, int skip, int sign_bra,
                         visit_fn visit, void *ctx) {
    const int *l = S->l, *m = S->m, *n = S->n;
    int dt = S->dt, dl = S->dl;
#define DXA(arr, t, a, b) (arr)[(t) + dt * ((a) + dl * (b))]
    int i0 = S->gs[gi] - 1, j0 = S->gs[gj] - 1, k0 = S->gs[gk] - 1, r0 = S->gs[gr] - 1;
    for (int pi_ = 0; pi_ < S->gc[gi]; ++pi_) {
        int i = i0 + pi_;
        for (int pj = 0; pj < S->gc[gj]; ++pj) {
            int j = j0 + pj;
            for (int pk = 0; pk < S->gc[gk]; ++pk) {
                int k = k0 + pk;
                for (int pr = 0; pr < S->gc[gr]; ++pr) {
                    int r = r0 + pr;
                    double ztot = ZAT(Z, pi_, pj, pk, pr);
                    if (fabs(ztot) < cutoff1) continue;
                    for (int ll = 0; ll <= l[i] + l[j]; ++ll) {
                        double MDL = DXA(dx1, ll, l[i], l[j]);
                        if ((skip & 1) && fabs(MDL) < SKIP30) continue;
                        double prod1 = MDL * ztot;
                        for (int mm = 0; mm <= m[i] + m[j]; ++mm) {
                            double MDM = DXA(dy1, mm, m[i], m[j]);
                            if ((skip & 2) && fabs(MDM) < SKIP30) continue;
                            double prod2 = MDM * prod1;
                            for (int nn = 0; nn <= n[i] + n[j]; ++nn) {
                                double H1 = (sign_bra && ((ll + mm + nn) & 1)) ? -1.0 : 1.0;
                                double MDN = DXA(dz1, nn, n[i], n[j]);
                                if ((skip & 4) && fabs(MDN) < SKIP30) continue;
                                double prod3 = MDN * H1 * prod2;
                                for (int llp = 0; llp <= l[k] + l[r]; ++llp) {
                                    double MDLp = DXA(dx2, llp, l[k], l[r]);
                                    if ((skip & 8) && fabs(MDLp) < SKIP30) continue;
                                    double prod4 = MDLp * prod3;
                                    for (int mmp = 0; mmp <= m[k] + m[r]; ++mmp) {
                                        double MDMp = DXA(dy2, mmp, m[k], m[r]);
                                        if ((skip & 16) && fabs(MDMp) < SKIP30) continue;
                                        double prod5 = MDMp * prod4;
                                        for (int nnp = 0; nnp <= n[k] + n[r]; ++nnp) {
                                            double MDNp = DXA(dz2, nnp, n[k], n[r]);
                                            if ((skip & 32) && fabs(MDNp) < SKIP30) continue;
                                            double prod6 = MDNp * prod5;
                                            if (fabs(prod6) > cutoff2)
                                                visit(ctx, ll, mm, nn, llp, mmp, nnp, prod6);
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
    }
#undef DXA
}

typedef struct { double *h_saved; const double *h_pre2; int Ld; } hctx_t;
static void visit_h(void *c, int ll, int mm, int nn, int llp, int mmp, int nnp, double prod6) {
    hctx_t *h = (hctx_t *)c;
    int L = ll + llp, M = mm + mmp, N = nn + nnp;
    const double *row = h->h_pre2 + (size_t)DIM * (L + h->Ld * (M + (size_t)h->Ld * N));
    for (int b = 0; b < DIM; ++b) h->h_saved[b] = h->h_saved[b] + row[b] * prod6;
}

typedef struct { double *f; const setup_t *S; } p0ctx_t;
static void visit_p0(void *c, int ll, int mm, int nn, int llp, int mmp, int nnp, double prod6) {
    p0ctx_t *p = (p0ctx_t *)c;
    const setup_t *S = p->S;
    int L = ll + llp, M = mm + mmp, N = nn + nnp;
    for (int iq = 0; iq < S->nq; ++iq) p->f[iq] = p->f[iq] + prod6 * P0AT(S, iq, L, M, N);
}

/* LLmax from the group heads (src/Integrals.f90:5111-5114). */
static int llmax_of(const setup_t *S, int gi, int gj, int gk, int gr) {
    int hd[4] = {S->gs[gi] - 1, S->gs[gj] - 1, S->gs[gk] - 1, S->gs[gr] - 1};
    int L = 0;
    for (int t = 0; t < 4; ++t) L += S->l[hd[t]] + S->m[hd[t]] + S->n[hd[t]];
    return L;
}

static size_t kernel_work_doubles(void) { return (size_t)DIM * 21 * 21 * 21 + 4096; }

/* tot_integral_k_ijkr (K_TOTAL), integral_k_ijkr (K_ELASTIC),
 * tot_integral_k_ijkr_j2 (K_J2), integral_k_ijkr_j2 (K_ELASTIC_J2,
 * src/Integrals.f90:5903-6083: the j2 tables and Bessel order of
 * tot_integral_k_ijkr_j2 with the elastic density and |E| < 1e-30 skips on
 * MDL..MDMp, no zero-sum return). */
static int kernel_k_ijkr(const setup_t *S, const kopts_t *o, int gi, int gj, int gk, int gr,
                         double hx, double hy, double hz, double h,
                         const double *dx1, const double *dy1, const double *dz1,
                         const double *dx2, const double *dy2, const double *dz2,
                         const zblock_t *Z, double *f, double *work) {
    int LLmax = llmax_of(S, gi, gj, gk, gr);
    if (LLmax + 1 > DIM) return ORC_ERR_L;
    if ((o->kind == K_J2 || o->kind == K_ELASTIC_J2) && LLmax + 3 > DIM) return ORC_ERR_L;
    static const double zero20[DIM][DIM];
    double a[DIM][DIM], b[DIM][DIM], c[DIM][DIM], ap[DIM][DIM], bp[DIM][DIM], cp[DIM][DIM];
    memcpy(ap, zero20, sizeof ap); memcpy(bp, zero20, sizeof bp); memcpy(cp, zero20, sizeof cp);
    int Ld = LLmax + 1;
    double *h_pre2 = work;
    memset(h_pre2, 0, sizeof(double) * DIM * Ld * Ld * Ld);
    if (o->kind == K_TOTAL) {
        rrdj0(LLmax, hx, a); rrdj0(LLmax, hy, b); rrdj0(LLmax, hz, c);
    } else if (o->kind == K_ELASTIC) {
        hermite_like(a, LLmax, hx); hermite_like(b, LLmax, hy); hermite_like(c, LLmax, hz);
    } else {
        rrdj2a(LLmax, hx, a); rrdj2a(LLmax, hy, b); rrdj2a(LLmax, hz, c);
        rrdj2b(LLmax, a, ap); rrdj2b(LLmax, b, bp); rrdj2b(LLmax, c, cp);
        for (int x = 0; x < DIM; ++x) for (int y = 0; y < DIM; ++y) cp[x][y] = -2.0 * cp[x][y];
    }
    double BD[DIM];
    for (int k = 0; k <= LLmax; ++k)
        for (int j = 0; j <= LLmax - k; ++j)
            for (int i = 0; i <= LLmax - k - j; ++i) {
                int L, M, N;
                for (int t = 0; t < DIM; ++t) BD[t] = 0.0;
                if (o->kind == K_TOTAL) {        /* BesselDeriv(BD,k,j,i) -> h_pre2(:,k+1,j+1,i+1) */
                    L = k; M = j; N = i;
                    bessel_deriv(BD, L, M, N, a, b, c, LLmax);
                } else if (o->kind == K_ELASTIC) { /* BesselDeriv(BD,i,j,k) -> h_pre2(:,i+1,j+1,k+1) */
                    L = i; M = j; N = k;
                    bessel_deriv(BD, L, M, N, a, b, c, LLmax);
                } else {
                    L = i; M = j; N = k;
                    bessel_deriv2j(BD, hz, h, L, M, N, a, b, c, ap, bp, cp);
                }
                double *row = h_pre2 + (size_t)DIM * (L + Ld * (M + (size_t)Ld * N));
                for (int t = 0; t < DIM; ++t) row[t] = BD[t];
            }
    double h_saved[DIM];
    for (int t = 0; t < DIM; ++t) h_saved[t] = 0.0;
    hctx_t hc = {h_saved, h_pre2, Ld};
    int skip = o->kind == K_TOTAL ? SKIP_KIJKR
             : (o->kind == K_ELASTIC || o->kind == K_ELASTIC_J2) ? SKIP_ELASTIC : SKIP_J2;
    hermite_loop(S, gi, gj, gk, gr, dx1, dy1, dz1, dx2, dy2, dz2, Z, o->cutoff1, o->cutoff2,
                 skip, 1, visit_h, &hc);
    double *scratch = h_pre2 + (size_t)DIM * Ld * Ld * Ld;
    if (o->kind == K_ELASTIC) {
        double s = 0.0;
        for (int t = 0; t < DIM; ++t) s += h_saved[t];
        if (s == 0.0) { for (int iq = 0; iq < S->nq; ++iq) f[iq] = 0.0; return ORC_OK; }
    }
    if (o->kind == K_J2 || o->kind == K_ELASTIC_J2) {
        bessels0rr(f, LLmax + 2, S->q, S->nq, h, h_saved, o->bessel_mode, scratch);
        for (int iq = 0; iq < S->nq; ++iq) f[iq] = f[iq] / pow(S->q[iq], 2.0);
    } else {
        bessels0rr(f, LLmax, S->q, S->nq, h, h_saved, o->bessel_mode, scratch);
    }
    return ORC_OK;
}

/* tot_integral_ijkr_pzero / integral_ijkr_pzero (P0 table chosen at setup). */
static void kernel_pzero(const setup_t *S, const kopts_t *o, int gi, int gj, int gk, int gr,
                         const double *dx1, const double *dy1, const double *dz1,
                         const double *dx2, const double *dy2, const double *dz2,
                         const zblock_t *Z, double *f) {
    for (int iq = 0; iq < S->nq; ++iq) f[iq] = 0.0;
    p0ctx_t pc = {f, S};
    hermite_loop(S, gi, gj, gk, gr, dx1, dy1, dz1, dx2, dy2, dz2, Z, o->cutoff1, o->cutoff2,
                 (o->kind == K_ELASTIC || o->kind == K_ELASTIC_J2) ? SKIP_ELASTIC : SKIP_PZERO, 1, visit_p0, &pc);
}

/* ------------------------------------------------------------------------ */
/* Densities                                                                 */
/* ------------------------------------------------------------------------ */

typedef struct {
    int nmat, nmo;
    int *m1, *m2, *m3, *m4;        /* 0-based, bubble-sorted within pairs */
    const double *total;
    const double *mmod;            /* (nmo, ngto) column-major */
    double *zao;                   /* elastic Z (ngto, ngto) column-major */
    double *zao2;                  /* resolved CMS: the ket's Z (zj); NULL otherwise */
    /* optional: the contracted density already summed over the rows,
     * rho[P(x,y) * np + P(u,v)] = ztot for functions x,y (electron 1) and
     * u,v (electron 2), P(x,y) = max(x,y)(max(x,y)+1)/2 + min(x,y) */
    const double *rho;
    long np;
} dens_t;

#define MMOD(D, a, b) ((D)->mmod[(a) + (size_t)(D)->nmo * (b)])

/* z11(:,x,y), z22(:,x,y) of variables_total (src/Variables.f90:1049-1054) */
static void zvec(const dens_t *D, int x, int y, double *z1, double *z2) {
    for (int t = 0; t < D->nmat; ++t) {
        z1[t] = D->total[t] * (MMOD(D, D->m1[t], x) * MMOD(D, D->m2[t], y) +
                               MMOD(D, D->m1[t], y) * MMOD(D, D->m2[t], x));
        z2[t] = MMOD(D, D->m3[t], x) * MMOD(D, D->m4[t], y) +
                MMOD(D, D->m3[t], y) * MMOD(D, D->m4[t], x);
    }
}

/* ztot(i',j',k',r') = zcontrred(J,K,R,I) + zcontrred2(R,I,J,K) with
 * zcontrred(a,b,jj,ii)  = 1/8 sum_t z1(t,j'_a,i'_ii) z2(t,k'_b,r'_jj)
 * zcontrred2(jj,ii,a,b) = 1/8 sum_t z2(t,j'_a,i'_ii) z1(t,k'_b,r'_jj)
 * (the dgemm pairs of src/Integrals.f90:109-127 and the four other loops). */
static long pair_index(int x, int y) {
    return x >= y ? (long)x * (x + 1) / 2 + y : (long)y * (y + 1) / 2 + x;
}

static void build_total_block(const setup_t *S, const dens_t *D, int gi, int gj, int gk, int gr,
                              double *zblk, double *buf) {
    int si = S->gc[gi], sj = S->gc[gj], sk = S->gc[gk], sr = S->gc[gr];
    if (D->rho) {
        /* same ztot, read from the summed density */
        for (int a = 0; a < si; ++a)
            for (int b = 0; b < sj; ++b) {
                const double *row = D->rho + (size_t)pair_index(S->gs[gi] - 1 + a, S->gs[gj] - 1 + b) * D->np;
                for (int c = 0; c < sk; ++c)
                    for (int d = 0; d < sr; ++d)
                        zblk[(((size_t)a * sj + b) * sk + c) * sr + d] =
                            row[pair_index(S->gs[gk] - 1 + c, S->gs[gr] - 1 + d)];
            }
        return;
    }
    size_t nm = D->nmat;
    double *b1 = buf, *b2 = buf + nm * si * sj;
    double *k1 = b2 + nm * si * sj, *k2 = k1 + nm * sk * sr;
    for (int a = 0; a < si; ++a)
        for (int b = 0; b < sj; ++b)
            zvec(D, S->gs[gj] - 1 + b, S->gs[gi] - 1 + a, b1 + nm * (a * sj + b), b2 + nm * (a * sj + b));
    for (int c = 0; c < sk; ++c)
        for (int d = 0; d < sr; ++d)
            zvec(D, S->gs[gk] - 1 + c, S->gs[gr] - 1 + d, k1 + nm * (c * sr + d), k2 + nm * (c * sr + d));
    for (int a = 0; a < si; ++a)
        for (int b = 0; b < sj; ++b)
            for (int c = 0; c < sk; ++c)
                for (int d = 0; d < sr; ++d) {
                    const double *u1 = b1 + nm * (a * sj + b), *u2 = b2 + nm * (a * sj + b);
                    const double *v1 = k1 + nm * (c * sr + d), *v2 = k2 + nm * (c * sr + d);
                    double s1 = 0.0, s2 = 0.0;
                    for (size_t t = 0; t < nm; ++t) s1 += u1[t] * v2[t];
                    for (size_t t = 0; t < nm; ++t) s2 += u2[t] * v1[t];
                    zblk[(((size_t)a * sj + b) * sk + c) * sr + d] = (1.0 / 8.0) * s1 + (1.0 / 8.0) * s2;
                }
}

/* elastic: ztot = Zb(K,R) * Za(I,J) (src/Integrals.f90:5821-5825); the
 * resolved CMS passes za = zi(I,J), zb = zj(K,R) (src/Integrals.f90:2687-2688),
 * zi and zj from two 1-RDMs */
static void build_elastic_block(const setup_t *S, const dens_t *D, int gi, int gj, int gk, int gr,
                                double *zblk) {
    int si = S->gc[gi], sj = S->gc[gj], sk = S->gc[gk], sr = S->gc[gr];
    size_t N = S->ngto;
    const double *zk = D->zao2 ? D->zao2 : D->zao;
    for (int a = 0; a < si; ++a)
        for (int b = 0; b < sj; ++b) {
            double z1 = D->zao[(S->gs[gi] - 1 + a) + N * (S->gs[gj] - 1 + b)];
            for (int c = 0; c < sk; ++c)
                for (int d = 0; d < sr; ++d) {
                    double zb = zk[(S->gs[gk] - 1 + c) + N * (S->gs[gr] - 1 + d)];
                    zblk[(((size_t)a * sj + b) * sk + c) * sr + d] = zb * z1;
                }
        }
}

/* variables_elastic Z (src/Variables.f90:1199-1217); variables_resolved_cms
 * forms zi and zj the same way from its two 1-RDMs (src/Variables.f90:1322-1345) */
static void build_zao_into(const setup_t *S, dens_t *D, const double *onerdm, int nmo1, double *zout) {
    int N = S->ngto;
    for (int ii = 0; ii < N; ++ii)
        for (int jj = 0; jj < N; ++jj) {
            double temp = 0.0;
            for (int cc = 0; cc < nmo1; ++cc)
                for (int cc2 = 0; cc2 < nmo1; ++cc2) {
                    double o1 = onerdm[cc + (size_t)nmo1 * cc2];
                    temp = temp + o1 * MMOD(D, cc, ii) * MMOD(D, cc2, jj);
                    temp = temp + o1 * MMOD(D, cc, jj) * MMOD(D, cc2, ii);
                }
            zout[ii + (size_t)N * jj] = temp / 2.0;
        }
}

static void build_zao(const setup_t *S, dens_t *D, const double *onerdm, int nmo1) {
    build_zao_into(S, D, onerdm, nmo1, D->zao);
}

/* ------------------------------------------------------------------------ */
/* Quartet enumeration: the five loops of tot_integration                    */
/* ------------------------------------------------------------------------ */

typedef struct { int i, j, k, r, loop; } quartet_t;

long orc_count_quartets(int ng) {
    long c = 0;
    for (int i = 0; i < ng; ++i) {
        long mm = ng - 1 - i;
        c += mm * (mm * (mm - 1) / 2) + mm * mm;
    }
    c += (long)ng * ((long)ng * (ng - 1) / 2) + (long)ng * (ng - 1) / 2 + ng;
    return c;
}

static long enum_quartets(int ng, quartet_t *out) {
    long c = 0;
    for (int i = 0; i < ng; ++i) for (int j = i + 1; j < ng; ++j)          /* :79-168 */
        for (int k = i + 1; k < ng; ++k) for (int r = k + 1; r < ng; ++r)
            out[c++] = (quartet_t){i, j, k, r, 1};
    for (int i = 0; i < ng; ++i) for (int j = i + 1; j < ng; ++j)          /* :178-252 */
        for (int r = i + 1; r < ng; ++r) out[c++] = (quartet_t){i, j, i, r, 2};
    for (int i = 0; i < ng; ++i) for (int k = 0; k < ng; ++k)              /* :258-333 */
        for (int r = k + 1; r < ng; ++r) out[c++] = (quartet_t){i, i, k, r, 3};
    for (int i = 0; i < ng; ++i) for (int k = i + 1; k < ng; ++k)          /* :340-408 */
        out[c++] = (quartet_t){i, i, k, k, 4};
    for (int i = 0; i < ng; ++i) out[c++] = (quartet_t){i, i, i, i, 5};   /* :416-468 */
    return c;
}

/* elastic_integration_j2 (src/Integrals.f90:1941-2365) splits loop 2: (i,j,i,r)
 * for i < j < r with weight 8 (loop id 6), and (i,j,i,j) with weight 4;
 * loops 1, 3, 4, 5 as above (fewer quartets than enum_quartets: loop 2 takes
 * each unordered {j, r} once). */
static long enum_quartets_elastic_j2(int ng, quartet_t *out) {
    long c = 0;
    for (int i = 0; i < ng; ++i) for (int j = i + 1; j < ng; ++j)          /* :2005-2074 */
        for (int k = i + 1; k < ng; ++k) for (int r = k + 1; r < ng; ++r)
            out[c++] = (quartet_t){i, j, k, r, 1};
    for (int i = 0; i < ng; ++i) for (int j = i + 1; j < ng; ++j) {        /* :2080-2150 */
        for (int r = j + 1; r < ng; ++r) out[c++] = (quartet_t){i, j, i, r, 6};
        out[c++] = (quartet_t){i, j, i, j, 2};
    }
    for (int i = 0; i < ng; ++i) for (int k = 0; k < ng; ++k)
        for (int r = k + 1; r < ng; ++r) out[c++] = (quartet_t){i, i, k, r, 3};
    for (int i = 0; i < ng; ++i) for (int k = i + 1; k < ng; ++k)
        out[c++] = (quartet_t){i, i, k, k, 4};
    for (int i = 0; i < ng; ++i) out[c++] = (quartet_t){i, i, i, i, 5};
    return c;
}

/* resolved_cms_integration (src/Integrals.f90:2598-2930): no bra-ket symmetry
 * (zi on the bra, zj on the ket), so every bra pair meets every ket pair:
 *   loop 7:  i < j, k < r  weight 4   (:2657-2727)
 *   loop 8:  i = j, k < r  weight 2   (:2734-2794)
 *   loop 9:  i < j, k = r  weight 2   (:2799-2859)
 *   loop 10: i = j, k = r  weight 1   (:2864-2926)
 * each with P = Q only for h < cutoffcentre. */
static long count_quartets_cms(int ng) {
    long np = (long)ng * (ng + 1) / 2;
    return np * np;
}

static long enum_quartets_cms(int ng, quartet_t *out) {
    long c = 0;
    for (int i = 0; i < ng; ++i) for (int j = i + 1; j < ng; ++j)
        for (int k = 0; k < ng; ++k) for (int r = k + 1; r < ng; ++r)
            out[c++] = (quartet_t){i, j, k, r, 7};
    for (int i = 0; i < ng; ++i) for (int k = 0; k < ng; ++k)
        for (int r = k + 1; r < ng; ++r) out[c++] = (quartet_t){i, i, k, r, 8};
    for (int i = 0; i < ng; ++i) for (int j = i + 1; j < ng; ++j)
        for (int k = 0; k < ng; ++k) out[c++] = (quartet_t){i, j, k, k, 9};
    for (int i = 0; i < ng; ++i) for (int k = 0; k < ng; ++k) out[c++] = (quartet_t){i, i, k, k, 10};
    return c;
}

/* Fill 5 ints per quartet (i,j,k,r,loop), 0-based groups, in reference order. */
long orc_enum_quartets(int ng, int *out) {
    long nq = orc_count_quartets(ng);
    quartet_t *tmp = malloc(sizeof(quartet_t) * (size_t)nq);
    if (!tmp) return -1;
    enum_quartets(ng, tmp);
    for (long c = 0; c < nq; ++c) {
        out[5 * c] = tmp[c].i; out[5 * c + 1] = tmp[c].j; out[5 * c + 2] = tmp[c].k;
        out[5 * c + 3] = tmp[c].r; out[5 * c + 4] = tmp[c].loop;
    }
    free(tmp);
    return nq;
}

static const double loop_weight[11] = {0.0, 8.0, 4.0, 4.0, 2.0, 1.0, 8.0, 4.0, 2.0, 2.0, 1.0};

/* One group quartet: f (nq) before the weight and the e12 factors. */
static int eval_quartet(const setup_t *S, const dens_t *D, const kopts_t *o, const quartet_t *Q,
                        double *f, double *zblk, double *zbuf, double *work) {
    int i = Q->i, j = Q->j, k = Q->k, r = Q->r;
    double hx = PX(S, k, r) - PX(S, i, j);
    double hy = PY(S, k, r) - PY(S, i, j);
    double hz = PZ(S, k, r) - PZ(S, i, j);
    double h = (Q->loop == 1 || Q->loop == 7) ? pow(hx * hx + hy * hy + hz * hz, 0.5)
                                              : sqrt(hx * hx + hy * hy + hz * hz);
    zblock_t Z = {S->gc[i], S->gc[j], S->gc[k], S->gc[r], zblk};
    if (o->kind == K_ELASTIC || o->kind == K_ELASTIC_J2) build_elastic_block(S, D, i, j, k, r, zblk);
    else build_total_block(S, D, i, j, k, r, zblk, zbuf);
    const double *dx1 = DDP(S, S->ddx, j, i), *dy1 = DDP(S, S->ddy, j, i), *dz1 = DDP(S, S->ddz, j, i);
    const double *dx2 = DDP(S, S->ddx, r, k), *dy2 = DDP(S, S->ddy, r, k), *dz2 = DDP(S, S->ddz, r, k);
    if (Q->loop == 5 || h < o->cutoffcentre) {
        kernel_pzero(S, o, i, j, k, r, dx1, dy1, dz1, dx2, dy2, dz2, &Z, f);
        return ORC_OK;
    }
    return kernel_k_ijkr(S, o, i, j, k, r, hx, hy, hz, h, dx1, dy1, dz1, dx2, dy2, dz2, &Z, f, work);
}

static int max_group(const setup_t *S) {
    int g = 1;
    for (int i = 0; i < S->ng; ++i) if (S->gc[i] > g) g = S->gc[i];
    return g;
}

/* Sum over a quartet list; deterministic for any thread count: each chunk of
 * CH quartets is summed in order, then the chunk sums are added in order. */
static int run_quartets(const setup_t *S, const dens_t *D, const kopts_t *o, const quartet_t *Qs,
                        long nquart, const double *wts, double *result, int nthreads) {
    const long CH = 16;
    long nch = (nquart + CH - 1) / CH;
    int nq = S->nq;
    double *part = calloc((size_t)(nch > 0 ? nch : 1) * nq, sizeof(double));
    if (!part) return ORC_ERR_MEM;
    int mg = max_group(S);
    size_t zbsz = (size_t)mg * mg * mg * mg;
    size_t zbuf_sz = (size_t)(D->nmat > 0 ? D->nmat : 1) * 4 * mg * mg;
    int err = ORC_OK;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel
    {
        double *zblk = malloc(sizeof(double) * zbsz);
        double *zbuf = (o->kind == K_ELASTIC || o->kind == K_ELASTIC_J2 || D->rho) ? NULL
                                                                              : malloc(sizeof(double) * zbuf_sz);
        double *work = malloc(sizeof(double) * kernel_work_doubles());
        double *f = malloc(sizeof(double) * nq);
#pragma omp for schedule(dynamic, 1)
        for (long ch = 0; ch < nch; ++ch) {
            double *acc = part + (size_t)ch * nq;
            for (long c = ch * CH; c < nquart && c < (ch + 1) * CH; ++c) {
                const quartet_t *Q = &Qs[c];
                int e = eval_quartet(S, D, o, Q, f, zblk, zbuf, work);
                if (e != ORC_OK) { err = e; continue; }
                double w = wts ? wts[c] : loop_weight[Q->loop];
                for (int iq = 0; iq < nq; ++iq)
                    acc[iq] = acc[iq] + w * f[iq] * E12(S, iq, Q->i, Q->j) * E12(S, iq, Q->k, Q->r);
            }
        }
        free(zblk); free(zbuf); free(work); free(f);
    }
    for (int iq = 0; iq < nq; ++iq) result[iq] = 0.0;
    for (long ch = 0; ch < nch; ++ch)
        for (int iq = 0; iq < nq; ++iq) result[iq] += part[(size_t)ch * nq + iq];
    free(part);
    return err;
}

static int build_dens(dens_t *D, const double *mmod, int nmo, const int *mat, const double *total, int nmat) {
    memset(D, 0, sizeof(*D));
    D->nmat = nmat; D->nmo = nmo; D->mmod = mmod; D->total = total;
    D->m1 = malloc(sizeof(int) * (nmat > 0 ? nmat : 1)); D->m2 = malloc(sizeof(int) * (nmat > 0 ? nmat : 1));
    D->m3 = malloc(sizeof(int) * (nmat > 0 ? nmat : 1)); D->m4 = malloc(sizeof(int) * (nmat > 0 ? nmat : 1));
    for (int t = 0; t < nmat; ++t) {
        int a = mat[t], b = mat[t + nmat], c = mat[t + 2 * nmat], d = mat[t + 3 * nmat];
        if (a < 1 || b < 1 || c < 1 || d < 1 || a > nmo || b > nmo || c > nmo || d > nmo) return ORC_ERR_ARG;
        /* bubble_sort of each index pair (src/Variables.f90:1000-1009) */
        if (a > b) { int x = a; a = b; b = x; }
        if (c > d) { int x = c; c = d; d = x; }
        D->m1[t] = a - 1; D->m2[t] = b - 1; D->m3[t] = c - 1; D->m4[t] = d - 1;
    }
    return ORC_OK;
}

static void free_dens(dens_t *D) {
    free(D->m1); free(D->m2); free(D->m3); free(D->m4); free(D->zao); free(D->zao2);
}

/*
 * Full driver in the shape of total_scattering_calculation_2 with readrdm
 * (src/main_calculation.f90:501-849):
 *   type 1: total j0 (set_P0, variables_total, tot_integration)
 *   type 2: elastic j0 (set_P0, variables_elastic, elastic_integration)
 *   type 7: total j2 (set_P0_j2, variables_total, tot_integration_j2)
 *   type 8: elastic j2 (set_P0_j2, variables_elastic, elastic_integration_j2)
 *   type 9: resolved CMS (set_P0, variables_resolved_cms, resolved_cms_integration):
 *           onerdm holds two (nmo1,nmo1) matrices back to back, the bra's
 *           (zi) then the ket's (zj)
 * mmod is (nmo, ngto) column-major; mat is (nmat,4) column-major, 1-based;
 * onerdm is (nmo1,nmo1) column-major.  quartets: optional 5 ints per quartet
 * (i,j,k,r,loop) with 0-based groups, evaluated with the loop's weight, or with
 * weights[c] when weights is non-NULL.  NULL runs the reference's five loops.
 */
int orc_scattering_ex(int type, int ngto, const double *ga, const int *l, const int *m, const int *n,
                      const double *xx, const double *yy, const double *zz, const int *group,
                      const double *mmod, int nmo, const int *mat, const double *total, int nmat,
                      const double *onerdm, int nmo1, const double *q, int nq,
                      double cutoffz, double cutoffmd, double cutoffcentre, int bessel_mode, int nthreads,
                      const int *quartets, long nquart, const double *weights, const double *rho,
                      double *result);

int orc_scattering(int type, int ngto, const double *ga, const int *l, const int *m, const int *n,
                   const double *xx, const double *yy, const double *zz, const int *group,
                   const double *mmod, int nmo, const int *mat, const double *total, int nmat,
                   const double *onerdm, int nmo1, const double *q, int nq,
                   double cutoffz, double cutoffmd, double cutoffcentre, int bessel_mode, int nthreads,
                   const int *quartets, long nquart, const double *weights, double *result) {
    return orc_scattering_ex(type, ngto, ga, l, m, n, xx, yy, zz, group, mmod, nmo, mat, total, nmat, onerdm,
                             nmo1, q, nq, cutoffz, cutoffmd, cutoffcentre, bessel_mode, nthreads, quartets,
                             nquart, weights, NULL, result);
}

/* The same driver; with rho non-NULL (types 1 and 7) the per-quartet
 * contraction of the 2-RDM rows (zcontrred, zcontrred2) is read from the
 * summed pair density instead of being formed from the rows quartet by
 * quartet: rho[P(x,y) np + P(u,v)] = 1/8 sum_t [z11(t,x,y) z22(t,u,v) +
 * z22(t,x,y) z11(t,u,v)], np = ngto(ngto+1)/2 (see build_total_block).
 * Everything after the contraction is unchanged. */
int orc_scattering_ex(int type, int ngto, const double *ga, const int *l, const int *m, const int *n,
                      const double *xx, const double *yy, const double *zz, const int *group,
                      const double *mmod, int nmo, const int *mat, const double *total, int nmat,
                      const double *onerdm, int nmo1, const double *q, int nq,
                      double cutoffz, double cutoffmd, double cutoffcentre, int bessel_mode, int nthreads,
                      const int *quartets, long nquart, const double *weights, const double *rho,
                      double *result) {
    if (type != 1 && type != 2 && type != 7 && type != 8 && type != 9) return ORC_ERR_ARG;
    setup_t S;
    int e = build_setup(&S, ngto, ga, l, m, n, xx, yy, zz, group, q, nq, (type == 7 || type == 8) ? 2 : 1);
    if (e != ORC_OK) { free_setup(&S); return e; }
    dens_t D;
    kopts_t o = {type == 1 ? K_TOTAL : (type == 2 || type == 9) ? K_ELASTIC : type == 7 ? K_J2 : K_ELASTIC_J2,
                 bessel_mode, cutoffz, cutoffmd, cutoffcentre};
    if (type == 2 || type == 8 || type == 9) {
        memset(&D, 0, sizeof D);
        D.mmod = mmod; D.nmo = nmo;
        if (nmo1 > nmo) { free_setup(&S); return ORC_ERR_ARG; }
        D.zao = malloc(sizeof(double) * (size_t)ngto * ngto);
        build_zao(&S, &D, onerdm, nmo1);
        if (type == 9) {
            D.zao2 = malloc(sizeof(double) * (size_t)ngto * ngto);
            build_zao_into(&S, &D, onerdm + (size_t)nmo1 * nmo1, nmo1, D.zao2);
        }
    } else {
        e = build_dens(&D, mmod, nmo, mat, total, nmat);
        if (e != ORC_OK) { free_dens(&D); free_setup(&S); return e; }
        D.rho = rho;
        D.np = (long)ngto * (ngto + 1) / 2;
    }
    quartet_t *Qs;
    long nqt;
    if (quartets) {
        nqt = nquart;
        Qs = malloc(sizeof(quartet_t) * (size_t)(nqt > 0 ? nqt : 1));
        for (long c = 0; c < nqt; ++c) {
            Qs[c] = (quartet_t){quartets[5 * c], quartets[5 * c + 1], quartets[5 * c + 2],
                                quartets[5 * c + 3], quartets[5 * c + 4]};
            if (Qs[c].loop < 1 || Qs[c].loop > 10) { e = ORC_ERR_ARG; }
        }
    } else {
        nqt = type == 9 ? count_quartets_cms(S.ng) : orc_count_quartets(S.ng);
        Qs = malloc(sizeof(quartet_t) * (size_t)nqt);
        if (type == 8) nqt = enum_quartets_elastic_j2(S.ng, Qs);
        else if (type == 9) nqt = enum_quartets_cms(S.ng, Qs);
        else enum_quartets(S.ng, Qs);
    }
    if (e == ORC_OK) e = run_quartets(&S, &D, &o, Qs, nqt, weights, result, nthreads);
    free(Qs);
    free_dens(&D);
    free_setup(&S);
    return e;
}

/* ------------------------------------------------------------------------ */
/* Aligned (non-averaged) total intensity                                    */
/* ------------------------------------------------------------------------ */

typedef struct { double *hr, *hi; const double *e1r, *e1i, *e2r, *e2i; int nq, d; } alctx_t;
static void visit_al(void *c, int ll, int mm, int nn, int llp, int mmp, int nnp, double prod6) {
    alctx_t *a = (alctx_t *)c;
    size_t d = a->d, nq = a->nq;
    size_t o1 = nq * (llp + d * (mmp + d * nnp)), o2 = nq * (ll + d * (mm + d * nn));
    for (size_t iq = 0; iq < nq; ++iq) {
        double ar = a->e1r[o1 + iq], ai = a->e1i[o1 + iq], br = a->e2r[o2 + iq], bi = a->e2i[o2 + iq];
        double pr = ar * br - ai * bi, pi_ = ar * bi + ai * br;
        a->hr[iq] = a->hr[iq] + pr * prod6;
        a->hi[iq] = a->hi[iq] + pi_ * prod6;
    }
}

/*
 * tot_integration_aligned (src/Integrals.f90:1425-1573) with
 * tot_integral_k_ijkr_alig (:5588-5727): all ng^4 ordered quartets, no
 * symmetry and no P=Q branch, complex result (re, im) per q vector.
 * qal is (3, nq) column-major.  E12 is evaluated at |q| on the (nq,ng,ng)
 * group layout (the reference's own CASE(3) cannot run as written: it
 * allocates q_abs twice, src/main_calculation.f90:97,172, and reads the
 * (3131,ng,ng) table as (3131,ngto,ngto)).
 */
int orc_aligned(int ngto, const double *ga, const int *l, const int *m, const int *n,
                const double *xx, const double *yy, const double *zz, const int *group,
                const double *mmod, int nmo, const int *mat, const double *total, int nmat,
                const double *qal, int nq, double cutoffz, double cutoffmd, int nthreads,
                double *result_re, double *result_im) {
    double *qabs = malloc(sizeof(double) * nq);
    for (int iq = 0; iq < nq; ++iq)
        qabs[iq] = sqrt(pow(qal[3 * iq], 2.0) + pow(qal[3 * iq + 1], 2.0) + pow(qal[3 * iq + 2], 2.0));
    setup_t S;
    int e = build_setup(&S, ngto, ga, l, m, n, xx, yy, zz, group, qabs, nq, 0);
    if (e != ORC_OK) { free_setup(&S); free(qabs); return e; }
    dens_t D;
    e = build_dens(&D, mmod, nmo, mat, total, nmat);
    if (e != ORC_OK) { free_dens(&D); free_setup(&S); free(qabs); return e; }
    int d = 4 * S.maxl + 1;
    size_t esz = (size_t)nq * d * d * d;
    double *e1r = malloc(sizeof(double) * esz), *e1i = malloc(sizeof(double) * esz);
    double *e2r = malloc(sizeof(double) * esz), *e2i = malloc(sizeof(double) * esz);
    /* exponent1 = (i q)^LMN, exponent2 = (-i q)^LMN (src/main_calculation.f90:194-205) */
    for (int N = 0; N < d; ++N) for (int M = 0; M < d; ++M) for (int L = 0; L < d; ++L)
        for (int iq = 0; iq < nq; ++iq) {
            double comp[3] = {qal[3 * iq], qal[3 * iq + 1], qal[3 * iq + 2]};
            int pw[3] = {L, M, N};
            for (int sgn = 0; sgn < 2; ++sgn) {
                double rr = 1.0, ri = 0.0;
                for (int ax = 0; ax < 3; ++ax) {
                    double zr = 0.0, zi = (sgn == 0 ? 1.0 : -1.0) * comp[ax];
                    double pr = 1.0, pim = 0.0;
                    for (int t = 0; t < pw[ax]; ++t) { double a = pr * zr - pim * zi, b = pr * zi + pim * zr; pr = a; pim = b; }
                    double a = rr * pr - ri * pim, b = rr * pim + ri * pr; rr = a; ri = b;
                }
                size_t idx = iq + (size_t)nq * (L + (size_t)d * (M + (size_t)d * N));
                if (sgn == 0) { e1r[idx] = rr; e1i[idx] = ri; } else { e2r[idx] = rr; e2i[idx] = ri; }
            }
        }
    int ng = S.ng;
    long nall = (long)ng * ng * ng * ng;
    const long CH = 16;
    long nch = (nall + CH - 1) / CH;
    double *part = calloc((size_t)nch * nq * 2, sizeof(double));
    int mg = max_group(&S);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel
    {
        double *zblk = malloc(sizeof(double) * (size_t)mg * mg * mg * mg);
        double *zbuf = malloc(sizeof(double) * (size_t)(nmat > 0 ? nmat : 1) * 4 * mg * mg);
        double *hr = malloc(sizeof(double) * nq), *hi = malloc(sizeof(double) * nq);
#pragma omp for schedule(dynamic, 1)
        for (long ch = 0; ch < nch; ++ch) {
            double *acc = part + (size_t)ch * nq * 2;
            for (long c = ch * CH; c < nall && c < (ch + 1) * CH; ++c) {
                int i = (int)(c / ((long)ng * ng * ng)), j = (int)((c / ((long)ng * ng)) % ng);
                int k = (int)((c / ng) % ng), r = (int)(c % ng);
                double Hx = PX(&S, k, r) - PX(&S, i, j), Hy = PY(&S, k, r) - PY(&S, i, j);
                double Hz = PZ(&S, k, r) - PZ(&S, i, j);
                build_total_block(&S, &D, i, j, k, r, zblk, zbuf);
                zblock_t Z = {S.gc[i], S.gc[j], S.gc[k], S.gc[r], zblk};
                for (int iq = 0; iq < nq; ++iq) { hr[iq] = 0.0; hi[iq] = 0.0; }
                alctx_t ac = {hr, hi, e1r, e1i, e2r, e2i, nq, d};
                hermite_loop(&S, i, j, k, r, DDP(&S, S.ddx, j, i), DDP(&S, S.ddy, j, i), DDP(&S, S.ddz, j, i),
                             DDP(&S, S.ddx, r, k), DDP(&S, S.ddy, r, k), DDP(&S, S.ddz, r, k), &Z,
                             cutoffz, cutoffmd, SKIP_ALIG, 0, visit_al, &ac);
                for (int iq = 0; iq < nq; ++iq) {
                    /* f = h * exp(i qx Hx) * exp(i qy Hy) * exp(i qz Hz) */
                    double fr = hr[iq], fi = hi[iq];
                    double ang[3] = {qal[3 * iq] * Hx, qal[3 * iq + 1] * Hy, qal[3 * iq + 2] * Hz};
                    for (int ax = 0; ax < 3; ++ax) {
                        double cr = cos(ang[ax]), ci = sin(ang[ax]);
                        double a = fr * cr - fi * ci, b = fr * ci + fi * cr; fr = a; fi = b;
                    }
                    double w = E12(&S, iq, i, j) * E12(&S, iq, k, r);
                    acc[2 * iq] += fr * w;
                    acc[2 * iq + 1] += fi * w;
                }
            }
        }
        free(zblk); free(zbuf); free(hr); free(hi);
    }
    for (int iq = 0; iq < nq; ++iq) { result_re[iq] = 0.0; result_im[iq] = 0.0; }
    for (long ch = 0; ch < nch; ++ch)
        for (int iq = 0; iq < nq; ++iq) {
            result_re[iq] += part[((size_t)ch * nq + iq) * 2];
            result_im[iq] += part[((size_t)ch * nq + iq) * 2 + 1];
        }
    free(part); free(e1r); free(e1i); free(e2r); free(e2i);
    free_dens(&D); free_setup(&S); free(qabs);
    return ORC_OK;
}

/*
 * The aligned intensity of orc_aligned evaluated on a quartet list with
 * weights instead of all ng^4 ordered quartets, real part only.  Exchanging
 * the two functions of a pair leaves a term of tot_integration_aligned
 * unchanged, and exchanging bra and ket conjugates it (H -> -H, (iq)^L <->
 * (-iq)^L), so the ordered sum equals the sum of w Re f over the five loops'
 * list with their weights 8,4,4,2,1 (orc_enum_quartets).  Per quartet the
 * hermite_loop terms of tot_integral_k_ijkr_alig (src/Integrals.f90:5588-5727)
 * are first summed into D_TUV = sum prod6 (-1)^(ll+mm+nn) at T = ll+llp,
 * U = mm+mmp, V = nn+nnp, since (iq)^(llp,mmp,nnp) (-iq)^(ll,mm,nn) =
 * (-1)^(ll+mm+nn) i^(T+U+V) qx^T qy^U qz^V; then f(q) = sum D_TUV
 * i^(T+U+V) qx^T qy^U qz^V times the three phase factors and E12 E12'.
 * rho as in orc_scattering_ex (NULL: formed from the rows).
 */
typedef struct { double *D; int d; } dtctx_t;
static void visit_dtuv(void *c, int ll, int mm, int nn, int llp, int mmp, int nnp, double prod6) {
    dtctx_t *a = (dtctx_t *)c;
    double sg = ((ll + mm + nn) & 1) ? -1.0 : 1.0;
    size_t idx = (size_t)(ll + llp) + a->d * ((size_t)(mm + mmp) + a->d * (size_t)(nn + nnp));
    a->D[idx] = a->D[idx] + sg * prod6;
}

int orc_aligned_list(int ngto, const double *ga, const int *l, const int *m, const int *n,
                     const double *xx, const double *yy, const double *zz, const int *group,
                     const double *mmod, int nmo, const int *mat, const double *total, int nmat,
                     const double *rho, const double *qal, int nq, const int *quartets, long nquart,
                     double cutoffz, double cutoffmd, int nthreads, double *result_re) {
    double *qabs = malloc(sizeof(double) * nq);
    for (int iq = 0; iq < nq; ++iq)
        qabs[iq] = sqrt(pow(qal[3 * iq], 2.0) + pow(qal[3 * iq + 1], 2.0) + pow(qal[3 * iq + 2], 2.0));
    setup_t S;
    int e = build_setup(&S, ngto, ga, l, m, n, xx, yy, zz, group, qabs, nq, 0);
    if (e != ORC_OK) { free_setup(&S); free(qabs); return e; }
    dens_t D;
    e = build_dens(&D, mmod, nmo, mat, total, nmat);
    if (e != ORC_OK) { free_dens(&D); free_setup(&S); free(qabs); return e; }
    D.rho = rho;
    D.np = (long)ngto * (ngto + 1) / 2;
    int d = 4 * S.maxl + 1;
    /* powers qx^t, qy^t, qz^t, t < d, per q vector */
    double *pw = malloc(sizeof(double) * (size_t)nq * 3 * d);
    for (int iq = 0; iq < nq; ++iq)
        for (int ax = 0; ax < 3; ++ax) {
            double v = 1.0;
            for (int t = 0; t < d; ++t) { pw[((size_t)iq * 3 + ax) * d + t] = v; v *= qal[3 * iq + ax]; }
        }
    const long CH = 16;
    long nch = (nquart + CH - 1) / CH;
    double *part = calloc((size_t)(nch > 0 ? nch : 1) * nq, sizeof(double));
    int mg = max_group(&S);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel
    {
        double *zblk = malloc(sizeof(double) * (size_t)mg * mg * mg * mg);
        double *zbuf = rho ? NULL : malloc(sizeof(double) * (size_t)(nmat > 0 ? nmat : 1) * 4 * mg * mg);
        double *Dt = malloc(sizeof(double) * (size_t)d * d * d);
        int *nzi = malloc(sizeof(int) * (size_t)d * d * d * 3);
        double *nzv = malloc(sizeof(double) * (size_t)d * d * d);
#pragma omp for schedule(dynamic, 1)
        for (long ch = 0; ch < nch; ++ch) {
            double *acc = part + (size_t)ch * nq;
            for (long c = ch * CH; c < nquart && c < (ch + 1) * CH; ++c) {
                int i = quartets[5 * c], j = quartets[5 * c + 1], k = quartets[5 * c + 2], r = quartets[5 * c + 3];
                double w = loop_weight[quartets[5 * c + 4]];
                double Hx = PX(&S, k, r) - PX(&S, i, j), Hy = PY(&S, k, r) - PY(&S, i, j);
                double Hz = PZ(&S, k, r) - PZ(&S, i, j);
                build_total_block(&S, &D, i, j, k, r, zblk, zbuf);
                zblock_t Z = {S.gc[i], S.gc[j], S.gc[k], S.gc[r], zblk};
                memset(Dt, 0, sizeof(double) * (size_t)d * d * d);
                dtctx_t dc = {Dt, d};
                hermite_loop(&S, i, j, k, r, DDP(&S, S.ddx, j, i), DDP(&S, S.ddy, j, i), DDP(&S, S.ddz, j, i),
                             DDP(&S, S.ddx, r, k), DDP(&S, S.ddy, r, k), DDP(&S, S.ddz, r, k), &Z,
                             cutoffz, cutoffmd, SKIP_ALIG, 0, visit_dtuv, &dc);
                int nnz = 0;
                for (int V = 0; V < d; ++V) for (int U = 0; U < d; ++U) for (int T = 0; T < d; ++T) {
                    double v = Dt[(size_t)T + d * ((size_t)U + d * (size_t)V)];
                    if (v != 0.0) { nzi[3 * nnz] = T; nzi[3 * nnz + 1] = U; nzi[3 * nnz + 2] = V; nzv[nnz++] = v; }
                }
                if (nnz == 0) continue;
                for (int iq = 0; iq < nq; ++iq) {
                    const double *px = pw + (size_t)iq * 3 * d, *py = px + d, *pz = py + d;
                    double hr = 0.0, hi = 0.0;
                    for (int t = 0; t < nnz; ++t) {
                        int T = nzi[3 * t], U = nzi[3 * t + 1], V = nzi[3 * t + 2];
                        double term = nzv[t] * px[T] * py[U] * pz[V];
                        switch ((T + U + V) & 3) {
                            case 0: hr += term; break;
                            case 1: hi += term; break;
                            case 2: hr -= term; break;
                            default: hi -= term; break;
                        }
                    }
                    double fr = hr, fi = hi;
                    double ang[3] = {qal[3 * iq] * Hx, qal[3 * iq + 1] * Hy, qal[3 * iq + 2] * Hz};
                    for (int ax = 0; ax < 3; ++ax) {
                        double cr = cos(ang[ax]), ci = sin(ang[ax]);
                        double a = fr * cr - fi * ci, b = fr * ci + fi * cr; fr = a; fi = b;
                    }
                    acc[iq] += w * fr * E12(&S, iq, i, j) * E12(&S, iq, k, r);
                }
            }
        }
        free(zblk); free(zbuf); free(Dt); free(nzi); free(nzv);
    }
    for (int iq = 0; iq < nq; ++iq) result_re[iq] = 0.0;
    for (long ch = 0; ch < nch; ++ch)
        for (int iq = 0; iq < nq; ++iq) result_re[iq] += part[(size_t)ch * nq + iq];
    free(part); free(pw);
    free_dens(&D); free_setup(&S); free(qabs);
    return ORC_OK;
}

/*
 * Algorithmic work of the q-independent part of tot_integral_k_ijkr
 * (src/Integrals.f90:5155-5219): T_E = the number of innermost h_saved
 * updates that pass both cutoffs (|ztot| >= cutoffz, |prod6| > cutoffmd;
 * the MD |E| < 1e-30 skips are commented out there), for each listed
 * quartet.  Quartets on the P = Q branch (loop 5, or |H| < cutoffcentre)
 * count the terms of tot_integral_ijkr_pzero (:4955-5067, with its active
 * MD skips) instead and are flagged in is_p0.  rho as in orc_scattering_ex.
 */
typedef struct { long n; } cntctx_t;
static void visit_count(void *c, int ll, int mm, int nn, int llp, int mmp, int nnp, double prod6) {
    (void)ll; (void)mm; (void)nn; (void)llp; (void)mmp; (void)nnp; (void)prod6;
    ((cntctx_t *)c)->n += 1;
}

int orc_count_te(int ngto, const double *ga, const int *l, const int *m, const int *n,
                 const double *xx, const double *yy, const double *zz, const int *group,
                 const double *mmod, int nmo, const int *mat, const double *total, int nmat,
                 const double *rho, double cutoffz, double cutoffmd, double cutoffcentre,
                 const int *quartets, long nquart, int nthreads, long *te, int *is_p0) {
    double q1 = 1.0;
    setup_t S;
    int e = build_setup(&S, ngto, ga, l, m, n, xx, yy, zz, group, &q1, 1, 1);
    if (e != ORC_OK) { free_setup(&S); return e; }
    dens_t D;
    e = build_dens(&D, mmod, nmo, mat, total, nmat);
    if (e != ORC_OK) { free_dens(&D); free_setup(&S); return e; }
    D.rho = rho;
    D.np = (long)ngto * (ngto + 1) / 2;
    int mg = max_group(&S);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel
    {
        double *zblk = malloc(sizeof(double) * (size_t)mg * mg * mg * mg);
        double *zbuf = rho ? NULL : malloc(sizeof(double) * (size_t)(nmat > 0 ? nmat : 1) * 4 * mg * mg);
#pragma omp for schedule(dynamic, 64)
        for (long c = 0; c < nquart; ++c) {
            int i = quartets[5 * c], j = quartets[5 * c + 1], k = quartets[5 * c + 2], r = quartets[5 * c + 3];
            int loop = quartets[5 * c + 4];
            double hx = PX(&S, k, r) - PX(&S, i, j), hy = PY(&S, k, r) - PY(&S, i, j);
            double hz = PZ(&S, k, r) - PZ(&S, i, j);
            double h = loop == 1 ? pow(hx * hx + hy * hy + hz * hz, 0.5) : sqrt(hx * hx + hy * hy + hz * hz);
            int p0 = loop == 5 || h < cutoffcentre;
            build_total_block(&S, &D, i, j, k, r, zblk, zbuf);
            zblock_t Z = {S.gc[i], S.gc[j], S.gc[k], S.gc[r], zblk};
            cntctx_t cc = {0};
            hermite_loop(&S, i, j, k, r, DDP(&S, S.ddx, j, i), DDP(&S, S.ddy, j, i), DDP(&S, S.ddz, j, i),
                         DDP(&S, S.ddx, r, k), DDP(&S, S.ddy, r, k), DDP(&S, S.ddz, r, k), &Z,
                         cutoffz, cutoffmd, p0 ? SKIP_PZERO : SKIP_KIJKR, 1, visit_count, &cc);
            te[c] = cc.n;
            is_p0[c] = p0;
        }
        free(zblk); free(zbuf);
    }
    free_dens(&D); free_setup(&S);
    return ORC_OK;
}

/*
 * Elastic aligned intensity, CASE(4) of total_scattering_calculation
 * (src/main_calculation.f90:218-265): F(q) of elastic_integration_alig
 * (src/Integrals.f90:2366-2490) with integral_k_ijkr_alig (:6085-6190) --
 * every ordered group pair (i, j), H = P_ij, the pair's functions with
 * ztot = Z(a, b), the three MD factors with their |E| < 1e-30 skips and the
 * product kept when |prod3| > 1e-30, times (i qx)^ll (i qy)^mm (i qz)^nn,
 * e^{i qx Hx} e^{i qy Hy} e^{i qz Hz} and e12(|q|, i, j) -- and the result
 * |F|^2.  qal is (3, nq) column-major; Z comes from the 1-RDM as for type 2.
 */
int orc_elastic_aligned(int ngto, const double *ga, const int *l, const int *m, const int *n,
                        const double *xx, const double *yy, const double *zz, const int *group,
                        const double *mmod, int nmo, const double *onerdm, int nmo1, const double *qal, int nq,
                        double *f_re, double *f_im, double *result) {
    double *qabs = malloc(sizeof(double) * nq);
    for (int iq = 0; iq < nq; ++iq)
        qabs[iq] = sqrt(pow(qal[3 * iq], 2.0) + pow(qal[3 * iq + 1], 2.0) + pow(qal[3 * iq + 2], 2.0));
    setup_t S;
    int e = build_setup(&S, ngto, ga, l, m, n, xx, yy, zz, group, qabs, nq, 0);
    if (e != ORC_OK) { free_setup(&S); free(qabs); return e; }
    if (nmo1 > nmo) { free_setup(&S); free(qabs); return ORC_ERR_ARG; }
    dens_t D;
    memset(&D, 0, sizeof D);
    D.mmod = mmod; D.nmo = nmo;
    D.zao = malloc(sizeof(double) * (size_t)ngto * ngto);
    build_zao(&S, &D, onerdm, nmo1);
    int dt = S.dt, dl = S.dl;
    for (int iq = 0; iq < nq; ++iq) { f_re[iq] = 0.0; f_im[iq] = 0.0; }
    for (int gi = 0; gi < S.ng; ++gi)
        for (int gj = 0; gj < S.ng; ++gj) {
            const double Hx = PX(&S, gi, gj), Hy = PY(&S, gi, gj), Hz = PZ(&S, gi, gj);
            const double *dx1 = DDP(&S, S.ddx, gj, gi), *dy1 = DDP(&S, S.ddy, gj, gi), *dz1 = DDP(&S, S.ddz, gj, gi);
#define DXA(arr, t, a, b) (arr)[(t) + dt * ((a) + dl * (b))]
            for (int iq = 0; iq < nq; ++iq) {
                const double qx = qal[3 * iq], qy = qal[3 * iq + 1], qz = qal[3 * iq + 2];
                double hr = 0.0, hi = 0.0;
                for (int i = S.gs[gi] - 1; i < S.gs[gi] - 1 + S.gc[gi]; ++i)
                    for (int j = S.gs[gj] - 1; j < S.gs[gj] - 1 + S.gc[gj]; ++j) {
                        double ztot = D.zao[i + (size_t)ngto * j];
                        for (int ll = 0; ll <= l[i] + l[j]; ++ll) {
                            double MDL = DXA(dx1, ll, l[i], l[j]);
                            if (fabs(MDL) < SKIP30) continue;
                            double prod1 = MDL * ztot;
                            for (int mm = 0; mm <= m[i] + m[j]; ++mm) {
                                double MDM = DXA(dy1, mm, m[i], m[j]);
                                if (fabs(MDM) < SKIP30) continue;
                                double prod2 = MDM * prod1;
                                for (int nn = 0; nn <= n[i] + n[j]; ++nn) {
                                    double MDN = DXA(dz1, nn, n[i], n[j]);
                                    if (fabs(MDN) < SKIP30) continue;
                                    double prod3 = MDN * prod2;
                                    if (!(fabs(prod3) > SKIP30)) continue;
                                    /* exponent1 = (i qx)^ll (i qy)^mm (i qz)^nn */
                                    double er = 1.0, ei = 0.0;
                                    const double comp[3] = {qx, qy, qz};
                                    const int pw[3] = {ll, mm, nn};
                                    for (int ax = 0; ax < 3; ++ax)
                                        for (int t = 0; t < pw[ax]; ++t) {
                                            double a = -ei * comp[ax], b = er * comp[ax];
                                            er = a; ei = b;
                                        }
                                    hr = hr + er * prod3;
                                    hi = hi + ei * prod3;
                                }
                            }
                        }
                    }
                double fr = hr, fi = hi;
                const double ang[3] = {qx * Hx, qy * Hy, qz * Hz};
                for (int ax = 0; ax < 3; ++ax) {
                    double cr = cos(ang[ax]), ci = sin(ang[ax]);
                    double a = fr * cr - fi * ci, b = fr * ci + fi * cr; fr = a; fi = b;
                }
                const double w = E12(&S, iq, gi, gj);
                f_re[iq] += fr * w;
                f_im[iq] += fi * w;
            }
#undef DXA
        }
    for (int iq = 0; iq < nq; ++iq) result[iq] = f_re[iq] * f_re[iq] + f_im[iq] * f_im[iq];
    free_dens(&D); free_setup(&S); free(qabs);
    return ORC_OK;
}

/* The q vectors of CASE(4) (src/main_calculation.f90:227-241) for nq points:
 * ss = (linspace(0, pi/2, nq) - pi) / 2, k0 = 3.00 * 1.889726125 * 0.529,
 * q = 2 k0 cos(ss) (sin ss, 0, cos ss); written (3, nq) column-major. */
void orc_elastic_aligned_grid(int nq, double *qal) {
    const double pi = acos(-1.0);
    const double k0 = 3.00 * 1.889726125 * 0.529;
    for (int mm = 0; mm < nq; ++mm) {
        double ss = nq > 1 ? (pi / 2.0) * (double)mm / (double)(nq - 1) : 0.0;
        ss = (ss - pi) / 2.0;
        const double rr = 2.0 * k0 * cos(ss);
        qal[3 * mm] = rr * sin(ss) * cos(0.0);
        qal[3 * mm + 1] = rr * sin(ss) * sin(0.0);
        qal[3 * mm + 2] = rr * cos(ss);
    }
}

/* QCOORD3 (src/main_calculation.f90:864-929): the 3131-vector aligned grid. */
void orc_qcoord3(double k0, double *qx, double *qy, double *qz) {
    const int nn = 30;
    double pi = acos(-1.0);
    int npt[30] = {0};
    double ldk0 = sqrt(3.0) / 2.0 * k0 / (nn + 1.0);
    for (int i = 2; i <= nn + 1; ++i) npt[i - 2] = (int)ceil(pi / asin(1.0 / (2.0 * i)));
    for (int t = 0; t < 3131; ++t) { qx[t] = 1.0e-10; qy[t] = 1.0e-10; qz[t] = 1.0e-10; }
    qy[1] = ldk0;
    qz[1] = k0 * (1 - sqrt(1.0 - 1.0 / pow(nn + 1.0, 2)));
    int pos = 2;
    for (int i = 1; i <= 5; ++i) {
        pos = pos + 1;
        double qqx = sin(i * pi / 3.0) * ldk0, qqy = cos(i * pi / 3.0) * ldk0;
        qx[pos - 1] = qqx; qy[pos - 1] = qqy;
        qz[pos - 1] = k0 * (1.0 - sqrt(1.0 - (qqx * qqx + qqy * qqy) / (k0 * k0)));
    }
    for (int i = 2; i <= nn + 1; ++i) {
        pos = pos + 1;
        double rc = i * ldk0, ang = 2.0 * pi / npt[i - 2];
        qy[pos - 1] = rc;
        qz[pos - 1] = k0 * (1.0 - sqrt(fabs(1.0 - pow((double)i, 2.0) / pow(nn + 1.0, 2))));
        for (int j = 1; j <= npt[i - 2] - 1; ++j) {
            pos = pos + 1;
            double qqx = sin(j * ang) * rc, qqy = cos(j * ang) * rc;
            qx[pos - 1] = qqx; qy[pos - 1] = qqy;
            qz[pos - 1] = k0 * (1.0 - sqrt(fabs(1.0 - (qqx * qqx + qqy * qqy) / (k0 * k0))));
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Routine-level exports for known-answer tests                              */
/* ------------------------------------------------------------------------ */

/*
 * tot_integral_k_ijkr with the Fortran argument meaning (src/Integrals.f90:5068):
 * l,m,n per function; group_start/group_count per group (1-based starts);
 * dx1..dz2 each (dt, dl, dl) column-major; gi..gr 1-based; zcontr is
 * (spj,spk,spr,spi) and zcontr2 (spr,spi,spj,spk), column-major.
 * kind: 0 total j0, 1 elastic (za (spi,spj) in zcontr, zb (spk,spr) in zcontr2),
 * 2 total j2.  pzero != 0 runs the P=Q kernel with a P0 table built for q.
 */
int orc_kernel_quartet(int kind, int pzero, const double *mu, int nq, int ngto, const int *l,
                       const int *m, const int *n, int ng, const int *group_start,
                       const int *group_count, double hx, double hy, double hz, double h,
                       const double *dx1, const double *dy1, const double *dz1,
                       const double *dx2, const double *dy2, const double *dz2, int dt, int dl,
                       int gi, int gj, int gk, int gr, const double *zcontr, const double *zcontr2,
                       double cutoff1, double cutoff2, int bessel_mode, double *f) {
    setup_t S;
    memset(&S, 0, sizeof S);
    S.ngto = ngto; S.ng = ng; S.l = l; S.m = m; S.n = n; S.q = mu; S.nq = nq; S.dt = dt; S.dl = dl;
    S.gs = (int *)group_start; S.gc = (int *)group_count;
    gi -= 1; gj -= 1; gk -= 1; gr -= 1;
    int si = S.gc[gi], sj = S.gc[gj], sk = S.gc[gk], sr = S.gc[gr];
    double *zblk = malloc(sizeof(double) * (size_t)si * sj * sk * sr);
    for (int a = 0; a < si; ++a) for (int b = 0; b < sj; ++b)
        for (int c = 0; c < sk; ++c) for (int d = 0; d < sr; ++d) {
            double v;
            if (kind == K_ELASTIC) v = zcontr2[c + (size_t)sk * d] * zcontr[a + (size_t)si * b];
            else v = zcontr[b + (size_t)sj * (c + (size_t)sk * (d + (size_t)sr * a))] +
                     zcontr2[d + (size_t)sr * (a + (size_t)si * (b + (size_t)sj * c))];
            zblk[(((size_t)a * sj + b) * sk + c) * sr + d] = v;
        }
    zblock_t Z = {si, sj, sk, sr, zblk};
    kopts_t o = {kind, bessel_mode, cutoff1, cutoff2, 0.0};
    int e = ORC_OK;
    if (pzero) {
        int maxl = (dl - 1);
        S.p0d = 4 * maxl + 1;
        S.p0 = calloc((size_t)nq * S.p0d * S.p0d * S.p0d, sizeof(double));
        double fj2 = sqrt(5.0 / acos(-1.0));
        for (int k = 0; k < S.p0d; k += 2) for (int j = 0; j < S.p0d; j += 2) for (int i = 0; i < S.p0d; i += 2)
            for (int iq = 0; iq < nq; ++iq) {
                if (kind != K_J2) S.p0[iq + (size_t)nq * (i + S.p0d * (j + (size_t)S.p0d * k))] = p_lmn(i, j, k, mu[iq], 0);
                else S.p0[iq + (size_t)nq * (k + S.p0d * (j + (size_t)S.p0d * i))] = p_lmn(k, j, i, mu[iq], 1) * fj2;
            }
        kernel_pzero(&S, &o, gi, gj, gk, gr, dx1, dy1, dz1, dx2, dy2, dz2, &Z, f);
        free(S.p0);
    } else {
        double *work = malloc(sizeof(double) * kernel_work_doubles());
        e = kernel_k_ijkr(&S, &o, gi, gj, gk, gr, hx, hy, hz, h, dx1, dy1, dz1, dx2, dy2, dz2, &Z, f, work);
        free(work);
    }
    free(zblk);
    return e;
}

/* dphrec for a vector of x: rbes (lmax1, nx) column-major, j_k(x) in row k. */
void orc_dphrec(const double *x, int nx, int leps1, int lmax1, double *rbes) {
    double *tmp = malloc(sizeof(double) * (size_t)(leps1 > 0 ? leps1 : 1));
    for (int i = 0; i < nx; ++i) {
        dphrec1(x[i], tmp, leps1, lmax1);
        for (int k = 0; k < lmax1; ++k) rbes[k + (size_t)lmax1 * i] = tmp[k];
    }
    free(tmp);
}

/* bessels0rr on one H for a vector of q (bessel_mode as in orc_scattering). */
void orc_bessels0rr(int order, const double *mu, int nq, double H, const double *h_saved,
                    int bessel_mode, double *f) {
    double *scratch = malloc(sizeof(double) * 4096);
    bessels0rr(f, order, mu, nq, H, h_saved, bessel_mode, scratch);
    free(scratch);
}

/* The McMurchie-Davidson coefficients E^{l1,l2}_t in the reference order. */
void orc_md_chain(int l1, int l2, double PA, double PB, double a, double *out) {
    md_chain(l1, l2, PA, PB, a, out);
}

/* ------------------------------------------------------------------------ */
/* Nuclear-electron term of electron scattering (types 5 and 6)              */
/* ------------------------------------------------------------------------ */

/* BesselSum (src/Integrals.f90:6328-6366): F = sum_b h_b j_b(qH) (q/H)^b.
 * bessel_mode 0 keeps the reference's upward recurrence
 *   h_r = ((2r-1)/(qH) h_{r-1} - h_{r-2} q/H) q/H,
 * bessel_mode 1 takes the j_b of the stable backward recurrence instead (the
 * quantity the upward form approximates; it loses digits for qH below ~b). */
static void bessel_sum(double *f, const double *mu, int nq, double H, int LLmax, const double *h_saved,
                       int bessel_mode, double *scratch) {
    if (bessel_mode != 0) {
        bessels0rr(f, LLmax, mu, nq, H, h_saved, 1, scratch);
        return;
    }
    for (int iq = 0; iq < nq; ++iq) {
        double Pmu = H * mu[iq];
        double h0 = sin(Pmu) / Pmu;
        double sum = h0 * h_saved[0];
        if (LLmax >= 1) {
            double muOH = mu[iq] / H;
            double h1 = (sin(Pmu) / (Pmu * Pmu) - cos(Pmu) / Pmu) * muOH;
            sum = sum + h_saved[1] * h1;
            for (int ra = 2; ra <= LLmax; ++ra) {
                double hr = ((double)(2 * ra - 1) / Pmu * h1 - h0 * muOH) * muOH;
                sum = sum + hr * h_saved[ra];
                h0 = h1;
                h1 = hr;
            }
        }
        f[iq] = sum;
    }
}

/*
 * nuclei_electron_integration (src/Integrals.f90:2493-2596) with
 * integral_k_ij (:6192-6326) and integral_ij_pzero (:4865-4953):
 *   Ine(q) = sum_a sum_{group pairs (i,k), ordered} Zn_a F_ik(q) e12(q,i,k),
 * H = R_a - P_ik, F from the pair's Hermite expansion against the AO density
 * Z of the 1-RDM (variables_elastic).  geom is (natoms,3) column-major.
 */
int orc_nuclear(int ngto, const double *ga, const int *l, const int *m, const int *n,
                const double *xx, const double *yy, const double *zz, const int *group,
                const double *mmod, int nmo, const double *onerdm, int nmo1, const double *q, int nq,
                double cutoffz, double cutoffmd, double cutoffcentre, const double *Zn, const double *geom,
                int natoms, int bessel_mode, double *ine) {
    (void)cutoffz;  /* integral_k_ij has its |ztot| < cutoff1 test commented out (:6268-6273) */
    if (nmo1 > nmo || natoms < 0) return ORC_ERR_ARG;
    setup_t S;
    int e = build_setup(&S, ngto, ga, l, m, n, xx, yy, zz, group, q, nq, 1);
    if (e != ORC_OK) { free_setup(&S); return e; }
    dens_t D;
    memset(&D, 0, sizeof D);
    D.mmod = mmod; D.nmo = nmo;
    D.zao = malloc(sizeof(double) * (size_t)ngto * ngto);
    build_zao(&S, &D, onerdm, nmo1);
    for (int iq = 0; iq < nq; ++iq) ine[iq] = 0.0;
    double *f = malloc(sizeof(double) * (size_t)nq);
    double *scratch = malloc(sizeof(double) * 4096);
    double *h_pre2 = malloc(sizeof(double) * (size_t)DIM * 21 * 21 * 21);
    const size_t N = (size_t)ngto;
    for (int na = 0; na < natoms; ++na)
        for (int gi = 0; gi < S.ng; ++gi)
            for (int gk = 0; gk < S.ng; ++gk) {
                double hx = geom[na] - PX(&S, gi, gk);
                double hy = geom[na + natoms] - PY(&S, gi, gk);
                double hz = geom[na + 2 * natoms] - PZ(&S, gi, gk);
                double h = sqrt(hx * hx + hy * hy + hz * hz);
                const double *dx1 = DDP(&S, S.ddx, gk, gi), *dy1 = DDP(&S, S.ddy, gk, gi),
                             *dz1 = DDP(&S, S.ddz, gk, gi);
                int i0 = S.gs[gi] - 1, k0 = S.gs[gk] - 1;
                int LLmax = S.l[i0] + S.m[i0] + S.n[i0] + S.l[k0] + S.m[k0] + S.n[k0];
                int Ld = LLmax + 1;
                double a[DIM][DIM], b[DIM][DIM], c[DIM][DIM], h_saved[DIM];
                int pzero = h < cutoffcentre;
                if (!pzero) {
                    hermite_like(a, LLmax, hx); hermite_like(b, LLmax, hy); hermite_like(c, LLmax, hz);
                    double BD[DIM];
                    for (int kk = 0; kk <= LLmax; ++kk)
                        for (int jj = 0; jj <= LLmax - kk; ++jj)
                            for (int ii = 0; ii <= LLmax - kk - jj; ++ii) {
                                bessel_deriv(BD, ii, jj, kk, a, b, c, LLmax);
                                double *row = h_pre2 + (size_t)DIM * (ii + Ld * (jj + (size_t)Ld * kk));
                                for (int t = 0; t < DIM; ++t) row[t] = BD[t];
                            }
                    for (int t = 0; t < DIM; ++t) h_saved[t] = 0.0;
                } else {
                    for (int iq = 0; iq < nq; ++iq) f[iq] = 0.0;
                }
                for (int pi = 0; pi < S.gc[gi]; ++pi)
                    for (int pk = 0; pk < S.gc[gk]; ++pk) {
                        int fi = i0 + pi, fk = k0 + pk;
                        double ztot = D.zao[fi + N * fk];
                        for (int ll = 0; ll <= l[fi] + l[fk]; ++ll) {
                            double MDL = dx1[ll + S.dt * (l[fi] + S.dl * l[fk])];
                            if (fabs(MDL) < SKIP30) continue;
                            double prod1 = MDL * ztot;
                            for (int mm = 0; mm <= m[fi] + m[fk]; ++mm) {
                                double MDM = dy1[mm + S.dt * (m[fi] + S.dl * m[fk])];
                                if (fabs(MDM) < SKIP30) continue;
                                double prod2 = MDM * prod1;
                                for (int nn = 0; nn <= n[fi] + n[fk]; ++nn) {
                                    double H1 = ((ll + mm + nn) & 1) ? -1.0 : 1.0;
                                    double MDN = dz1[nn + S.dt * (n[fi] + S.dl * n[fk])];
                                    if (fabs(MDN) < SKIP30) continue;
                                    double prod3 = MDN * H1 * prod2;
                                    if (!(fabs(prod3) > cutoffmd)) continue;
                                    if (pzero) {
                                        for (int iq = 0; iq < nq; ++iq) f[iq] += prod3 * P0AT(&S, iq, ll, mm, nn);
                                    } else {
                                        const double *row = h_pre2 + (size_t)DIM * (ll + Ld * (mm + (size_t)Ld * nn));
                                        for (int t = 0; t < DIM; ++t) h_saved[t] += row[t] * prod3;
                                    }
                                }
                            }
                        }
                    }
                if (!pzero) bessel_sum(f, q, nq, h, LLmax, h_saved, bessel_mode, scratch);
                for (int iq = 0; iq < nq; ++iq) ine[iq] = ine[iq] + Zn[na] * f[iq] * E12(&S, iq, gi, gk);
            }
    free(f); free(scratch); free(h_pre2);
    free_dens(&D);
    free_setup(&S);
    return ORC_OK;
}
