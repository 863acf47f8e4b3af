// CUDA kernels of the scattering-intensity path (sm_100a, FP64 throughout).
//
//  tb_pair_tables   Gaussian-product tables per unordered group pair
//                   (src/Variables.f90:1113-1148 and fill_md_table :8-946)
//  (stage 1, per group quartet: tb_stage1.cuh, one translation unit per kind)
//  tb_stage2        the quartet x q Bessel sum (bessels0rr :6662-6739 with an
//                   accurate generator), warp per quartet, lanes over q,
//                   accumulated per warp in shared memory
//  tb_reduce        fixed-order sum of the per-block partial I(q)
//  ghat_emit / ghat_runs / sym_small: the density transform's gathers
//                   (variables_total z11/z22 :1045-1065 re-expressed as a
//                   4-index transform, whose GEMM passes are in tb_transform.cu)
#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_kernels.h"
#include "tb_math.cuh"

namespace tb {

// ---------------------------------------------------------------------------
// pair tables
// ---------------------------------------------------------------------------
int64_t esoa_doubles(int ng, int maxa) {
  return 2 * (int64_t)3 * (maxa + 1) * (maxa + 1) * E_T * npairs(ng);
}

// One thread per unordered group pair.  Besides the pair record it writes the
// transposed E table: element t of (axis, la, lb) at
// esoa[((axis (maxa+1) + la) (maxa+1) + lb) E_T + t][pair], zero for
// t > la + lb, and a second copy with |E| < 1e-30 set to zero (the MD skips).
__device__ __forceinline__ void pair_table_one(int p, int ng, int maxa, const int *__restrict__ gstart,
                                               const int *__restrict__ flmn, const double *__restrict__ ga,
                                               const double *__restrict__ xyz, double *__restrict__ tab,
                                               double *__restrict__ esoa) {
  const int64_t npair = npairs(ng);
  if (p >= npair) return;
  const int64_t skipoff = (int64_t)3 * (maxa + 1) * (maxa + 1) * E_T * npair;
  int i = 0, rem = p;
  while (rem >= ng - i) { rem -= ng - i; ++i; }
  int j = i + rem;
  int fi = gstart[i], fj = gstart[j];
  double ai = ga[fi], aj = ga[fj];
  double gaP = ai + aj;
  double *t = tab + (size_t)p * PAIR_STRIDE;
  double d2 = 0.0;
  for (int ax = 0; ax < 3; ++ax) {
    double xi = xyz[3 * fi + ax], xj = xyz[3 * fj + ax];
    double P = (ai * xi + aj * xj) / gaP;
    t[ax] = P;
    double d = xi - xj;
    d2 = d2 + d * d;
    double PA = P - xi, PB = P - xj, a = 0.5 / gaP;
    double E[2 * MAXA + 2];
    double *dst = t + 8 + ax * ESZ;
    for (int la = 0; la <= maxa; ++la)
      for (int lb = 0; lb <= maxa; ++lb) {
        // larger exponent first, with its own centre (src/Variables.f90:36-48)
        if (la >= lb) md_chain(la, lb, PA, PB, a, E);
        else md_chain(lb, la, PB, PA, a, E);
        for (int tt = 0; tt <= la + lb; ++tt) dst[(la * (MAXA + 1) + lb) * E_T + tt] = E[tt];
        const int64_t slot = ((int64_t)(ax * (maxa + 1) + la) * (maxa + 1) + lb) * E_T;
        for (int tt = 0; tt < E_T; ++tt) {
          double v = tt <= la + lb ? E[tt] : 0.0;
          esoa[(slot + tt) * npair + p] = v;
          esoa[skipoff + (slot + tt) * npair + p] = fabs(v) < TB_SKIP30 ? 0.0 : v;
        }
      }
  }
  t[3] = gaP;
  t[4] = pow(TB_PI_SP / gaP, 1.5) * exp(-ai * aj / gaP * d2);
  t[5] = 0.25 / gaP;
  t[6] = 0.0;
  t[7] = 0.0;
}

__global__ void pair_tables_kernel(int ng, int maxa, const int *__restrict__ gstart,
                                   const int *__restrict__ flmn, const double *__restrict__ ga,
                                   const double *__restrict__ xyz, double *__restrict__ tab,
                                   double *__restrict__ esoa, int64_t gs_xyz, int64_t gs_tab, int64_t gs_esoa) {
  // geometry blockIdx.y of a batch
  pair_table_one(blockIdx.x * blockDim.x + threadIdx.x, ng, maxa, gstart, flmn, ga, xyz + blockIdx.y * gs_xyz,
                 tab + blockIdx.y * gs_tab, esoa + blockIdx.y * gs_esoa);
}

__device__ __forceinline__ int desc_item(const int64_t *__restrict__ pre, int n, int64_t b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void pair_tables_batch_kernel(const PairDesc *__restrict__ d, const int64_t *__restrict__ pre, int n) {
  const int it = desc_item(pre, n, blockIdx.x);
  const PairDesc D = d[it];
  pair_table_one((int)(blockIdx.x - pre[it]) * blockDim.x + threadIdx.x, D.ng, D.maxa, D.gstart, D.flmn, D.ga, D.xyz,
                 D.tab, D.esoa);
}

__global__ void reduce_desc_kernel(const ReduceDesc *__restrict__ d) {
  const ReduceDesc D = d[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.nq) return;
  double t = 0.0;
  for (int b = 0; b < D.rows; ++b) t += D.partial[(size_t)b * D.nq + i];
  D.out[i] = t;
}

// ---------------------------------------------------------------------------
// stage 2: the Bessel sum, warp per quartet, lanes over q
// ---------------------------------------------------------------------------

// u_n(y) = sum_k c_{n,k} y^k, Horner in y
template <int N, int K>
__device__ __forceinline__ double series_u(double y) {
  double p = series_coef(N, K);
#pragma unroll
  for (int k = K - 1; k >= 0; --k) p = fma(p, y, series_coef(N, k));
  return p;
}

// F = sum_{b<=LB} hh[b] j_b(x) x^b for x = q H (hh already divided by H^{2b}).
// F = sum_{b<=LB} hh[b] j_b(x) x^b for x = q H (hh already divided by H^{2b}),
// given sin x, cos x and 1/x.
template <int LB>
__device__ __forceinline__ double bessel_sum(const double *hh, double x, double sn, double cs, double invx) {
  if (LB == 0) return hh[0] * (sn * invx);
  const double y = x * x;
  if (x >= bessel_crossover(LB)) {
    // upward: g0 = sin x / x, g1 = g0 - cos x, g_{b+1} = (2b+1) g_b - x^2 g_{b-1}
    double g0 = sn * invx;
    double g1 = g0 - cs;
    double F = fma(hh[1], g1, hh[0] * g0);
#pragma unroll
    for (int b = 1; b < LB; ++b) {
      double g2 = fma((double)(2 * b + 1), g1, -y * g0);
      F = fma(hh[b + 1], g2, F);
      g0 = g1;
      g1 = g2;
    }
    return F;
  }
  // small x: series for u_LB, u_{LB+1}; downward u_{b-1} = u_b - y u_{b+1}/((2b+1)(2b+3));
  // Horner in y/(2b+1) for the x^{2b}/(2b+1)!! weights.
  constexpr int K = series_terms(LB);
  double uhi = series_u<LB + 1, K>(y);
  double umid = series_u<LB, K>(y);
  double acc = hh[LB] * umid;
#pragma unroll
  for (int b = LB; b >= 1; --b) {
    double ulo = umid - (y * (1.0 / ((2.0 * b + 1.0) * (2.0 * b + 3.0)))) * uhi;
    acc = fma(acc, y * (1.0 / (2.0 * b + 1.0)), hh[b - 1] * ulo);
    uhi = umid;
    umid = ulo;
  }
  return acc;
}

// Generic q grids: sincos and exp at every point.
template <int LB>
__device__ __forceinline__ void bessel_points_direct(const double *hh, double H, double invH, double s, bool j2,
                                                     const double *q_s, const double *q2_s, const double *iq_s,
                                                     double *acc, int i0, int nq) {
  for (int iq = i0; iq < nq; iq += 32) {
    double q = q_s[iq], q2 = q2_s[iq];
    double x = q * H, sn, cs;
    sincos(x, &sn, &cs);
    double F = bessel_sum<LB>(hh, x, sn, cs, iq_s[iq] * invH);
    F *= exp(-q2 * s);
    if (j2) F *= iq_s[iq] * iq_s[iq];
    acc[iq] += F;
  }
}

// Uniform q grids (q_i = q_first + (i - first) dq): the lane's points are
// 32 dq apart, so sin/cos advance by a rotation through 32 dq H and the
// Gaussian exp(-q^2 s) by g *= r, r *= k with r = exp(-(2 q D + D^2) s),
// k = exp(-2 D^2 s), D = 32 dq; both restart from direct values every 16 steps.
template <int LB>
__device__ __forceinline__ void bessel_points_uniform(const double *hh, double H, double invH, double s, bool j2,
                                                      const double *q_s, const double *iq_s, double dq,
                                                      double *acc, int i0, int nq) {
  const double Dq = 32.0 * dq;
  double sd, cd;
  sincos(Dq * H, &sd, &cd);
  const double kk = exp(-2.0 * Dq * Dq * s);
  int m = 0;
  double sn = 0, cs = 0, g = 0, r = 0;
  for (int iq = i0; iq < nq; iq += 32, ++m) {
    double q = q_s[iq];
    double x = q * H;
    if ((m & 15) == 0) {
      sincos(x, &sn, &cs);
      g = exp(-(q * q) * s);
      r = exp(-(2.0 * q * Dq + Dq * Dq) * s);
    }
    double F = bessel_sum<LB>(hh, x, sn, cs, iq_s[iq] * invH);
    F *= g;
    if (j2) F *= iq_s[iq] * iq_s[iq];
    acc[iq] += F;
    double sn2 = fma(sn, cd, cs * sd);
    cs = fma(cs, cd, -sn * sd);
    sn = sn2;
    g *= r;
    r *= kk;
  }
}

template <int LB>
__device__ __noinline__ void stage2_bessel(const double *__restrict__ c, double H, double s, bool j2,
                                           const double *q_s, const double *q2_s, const double *iq_s,
                                           double *acc, int nq, int lane, int uniform, int first_on_grid,
                                           double dq) {
  double hh[LB + 1];
#pragma unroll
  for (int b = 0; b <= LB; ++b) hh[b] = c[b];
  const double invH = 1.0 / H;
  if (!uniform) {
    bessel_points_direct<LB>(hh, H, invH, s, j2, q_s, q2_s, iq_s, acc, lane, nq);
    return;
  }
  int i0 = lane;
  if (!first_on_grid && lane == 0) {
    bessel_points_direct<LB>(hh, H, invH, s, j2, q_s, q2_s, iq_s, acc, 0, 1);
    i0 = 32;
  }
  bessel_points_uniform<LB>(hh, H, invH, s, j2, q_s, iq_s, dq, acc, i0, nq);
}

__device__ __noinline__ void stage2_p0(const double *__restrict__ c, int ns, double s, const double *q2_s,
                                       double *acc, int nq, int lane) {
  for (int iq = lane; iq < nq; iq += 32) {
    double q2 = q2_s[iq];
    double F = c[ns - 1];
    for (int k = ns - 2; k >= 0; --k) F = fma(F, q2, c[k]);
    acc[iq] += F * exp(-q2 * s);
  }
}

__device__ __forceinline__ void stage2_dispatch(int LB, const double *c, double H, double s, bool j2,
                                                const double *q_s, const double *q2_s, const double *iq_s,
                                                double *acc, int nq, int lane, int uniform, int first_on_grid,
                                                double dq) {
  switch (LB) {
#define TB_CASE(n) \
  case n: stage2_bessel<n>(c, H, s, j2, q_s, q2_s, iq_s, acc, nq, lane, uniform, first_on_grid, dq); break;
    TB_CASE(0) TB_CASE(1) TB_CASE(2) TB_CASE(3) TB_CASE(4) TB_CASE(5) TB_CASE(6) TB_CASE(7)
    TB_CASE(8) TB_CASE(9) TB_CASE(10) TB_CASE(11) TB_CASE(12) TB_CASE(13) TB_CASE(14)
    TB_CASE(15) TB_CASE(16) TB_CASE(17) TB_CASE(18)
#undef TB_CASE
    default: break;
  }
}

__global__ void __launch_bounds__(256) stage2_kernel(Stage2Args A) {
  extern __shared__ double sm[];
  const int nqp = A.nqp;
  double *q_s = sm, *q2_s = sm + nqp, *iq_s = sm + 2 * nqp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double *acc = sm + (3 + warp) * nqp;
  for (int i = threadIdx.x; i < A.nq; i += blockDim.x) {
    double q = A.q[i];
    q_s[i] = q;
    q2_s[i] = q * q;
    iq_s[i] = 1.0 / q;
  }
  for (int i = threadIdx.x; i < nw * nqp; i += blockDim.x) sm[3 * nqp + i] = 0.0;
  __syncthreads();
  const int64_t gw = (int64_t)blockIdx.x * nw + warp, W = (int64_t)gridDim.x * nw;
  const int64_t nchunks = (A.nquart + A.chunk - 1) / A.chunk;
  for (int64_t ch = gw; ch < nchunks; ch += W) {
    int64_t q0 = ch * A.chunk, q1 = min(A.nquart, q0 + A.chunk);
    for (int64_t qi = q0; qi < q1; ++qi) {
      int c = 0;
      while (c < A.ncls - 1 && qi >= A.cls_end[c]) ++c;
      const double *r = A.rec + A.cls_recoff[c] + (qi - A.cls_begin[c]) * (int64_t)A.cls_rs[c];
      double H = r[0], s = r[1];
      int kind = (int)r[2], LB = (int)r[3];
      if (kind == REC_P0) stage2_p0(r + 4, LB + 1, s, q2_s, acc, A.nq, lane);
      else
        stage2_dispatch(LB, r + 4, H, s, kind == REC_BESSEL_J2, q_s, q2_s, iq_s, acc, A.nq, lane, A.uniform,
                        A.first_on_grid, A.dq);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < A.nq; i += blockDim.x) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += sm[(3 + w) * nqp + i];
    A.partial[(size_t)blockIdx.x * A.pstride + i] = t;
  }
}

// Sum of nblocks partial rows (row stride nq) at every q point of geometry
// blockIdx.y: a block takes 32 points, lane = point; warp w adds rows w,
// w + 8, w + 16, .. in order, then the 8 warp sums are added in warp order
// (a fixed order whatever the launch).
constexpr int REDUCE_WARPS = 8;
__global__ void __launch_bounds__(REDUCE_WARPS * 32)
    reduce_kernel(const double *__restrict__ partial, int nblocks, int nq, double *__restrict__ out, int64_t gs_in) {
  __shared__ double sm[REDUCE_WARPS][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + lane;
  partial += blockIdx.y * gs_in;
  double t = 0.0;
  if (i < nq)
    for (int b = w; b < nblocks; b += REDUCE_WARPS) t += partial[(size_t)b * nq + i];
  sm[w][lane] = t;
  __syncthreads();
  if (w == 0 && i < nq) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < REDUCE_WARPS; ++k) s += sm[k][lane];
    out[(int64_t)blockIdx.y * nq + i] = s;
  }
}

// ---------------------------------------------------------------------------
// density transform helpers
// ---------------------------------------------------------------------------

// Ghat[x][y][z][w] = sum of Gamma_t/8 over the eight index placements of
// every row (both orders inside each pair, both pair orders); see tb_density.cu.
// Deterministic in two steps: every (row, placement) emits (flat index,
// value); after a stable sort by index each run of equal indices is summed
// in its sorted (row, placement) order by the run's first element.
__global__ void ghat_emit_kernel(const int *__restrict__ mat, const double *__restrict__ total, int nmat, int n,
                                 int *__restrict__ keys, double *__restrict__ vals) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nmat) return;
  int a = mat[t] - 1, b = mat[t + nmat] - 1, c = mat[t + 2 * nmat] - 1, d = mat[t + 3 * nmat] - 1;
  double v = total[t] * 0.125;
  int P[8][4] = {{a, b, c, d}, {b, a, c, d}, {a, b, d, c}, {b, a, d, c},
                 {c, d, a, b}, {d, c, a, b}, {c, d, b, a}, {d, c, b, a}};
  for (int k = 0; k < 8; ++k) {
    keys[8 * t + k] = ((P[k][0] * n + P[k][1]) * n + P[k][2]) * n + P[k][3];
    vals[8 * t + k] = v;
  }
}

__global__ void ghat_runs_kernel(const int *__restrict__ keys, const double *__restrict__ vals, int64_t m,
                                 double *__restrict__ G) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m || (i > 0 && keys[i - 1] == keys[i])) return;
  double s = vals[i];
  for (int64_t j = i + 1; j < m && keys[j] == keys[i]; ++j) s += vals[j];
  G[keys[i]] = s;
}

// out = 0.5 (in + in^T) for a small n x n matrix
__global__ void sym_small_kernel(const double *__restrict__ in, int n, double *__restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * n) return;
  int r = i / n, c = i % n;
  out[i] = 0.5 * (in[r * n + c] + in[c * n + r]);
}

// ---------------------------------------------------------------------------
// quartet enumeration
// ---------------------------------------------------------------------------
// The five loops of tot_integration visit, for bra pair (i,j):
//   i <  j : kets (k,r) with k < r and k >= i          (loops 1 and 2)
//   i == j : every ket (k,r) with k < r                 (loop 3)
//            and (k,k) with k >= i                      (loops 4 and 5)
// bra_off[b] is the first quartet of bra pair b (pair_index order).
// all_pairs (the resolved CMS): every ket (k <= r) for every bra, in pair order.
__global__ void quartet_fill_kernel(int ng, const int64_t *__restrict__ bra_off, int nbra, int64_t nquart,
                                    const int *__restrict__ gL, uint64_t *__restrict__ quart,
                                    uint32_t *__restrict__ keys, int all_pairs) {
  int64_t qi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= nquart) return;
  int lo = 0, hi = nbra - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (bra_off[mid] <= qi) lo = mid; else hi = mid - 1;
  }
  int b = lo;
  int i = 0, rem = b;
  while (rem >= ng - i) { rem -= ng - i; ++i; }
  int j = i + rem;
  int64_t m = qi - bra_off[b];
  int k, r;
  int64_t noff_all = (int64_t)ng * (ng - 1) / 2;
  if (all_pairs) {
    k = 0;
    while (m >= ng - k) { m -= ng - k; ++k; }
    r = k + (int)m;
  } else if (i < j || m < noff_all) {
    // m-th off-diagonal pair (k < r) starting at k = (i < j ? i : 0)
    k = i < j ? i : 0;
    while (m >= ng - 1 - k) { m -= ng - 1 - k; ++k; }
    r = k + 1 + (int)m;
  } else {
    k = i + (int)(m - noff_all);
    r = k;
  }
  quart[qi] = (uint64_t)i | ((uint64_t)j << 16) | ((uint64_t)k << 32) | ((uint64_t)r << 48);
  int Li = gL[i], Lj = gL[j], Lk = gL[k], Lr = gL[r];
  keys[qi] = quartet_key(Li, Lj, Lk, Lr);
}

// ---------------------------------------------------------------------------
// host-side launchers
// ---------------------------------------------------------------------------
cudaError_t launch_pair_tables(int ng, int maxa, const int *gstart, const int *flmn, const double *ga,
                               const double *xyz, double *tab, double *esoa, int ngeom, int64_t gs_xyz,
                               int64_t gs_tab, int64_t gs_esoa, cudaStream_t st) {
  int n = npairs(ng);
  pair_tables_kernel<<<dim3((n + 127) / 128, ngeom), 128, 0, st>>>(ng, maxa, gstart, flmn, ga, xyz, tab, esoa,
                                                                    gs_xyz, gs_tab, gs_esoa);
  return cudaGetLastError();
}

#ifndef TB_S1_XK_MIN
#define TB_S1_XK_MIN 4
#endif
// LLmax 4-6 always; 7-8 with at least this many quartets per SM.  On the
// 7-atom AB6 step the split contracted-side kernels take class 7 (7315
// quartets, 49 per SM) in 0.52 ms where the register kernel's 32 threads per
// quartet took 1.10; class 8 (441 quartets, 3 per SM: a thread per quartet
// leaves the convolution kernel on a few SMs) stays on the register kernel
// (0.33 ms against 0.76).
#ifndef TB_S1_XK_HIGH_PER_SM
#define TB_S1_XK_HIGH_PER_SM 16
#endif
#ifndef TB_S1_TPL_MAXL
#define TB_S1_TPL_MAXL 3
#endif
bool stage1_tpl(int kind, int L, int shells_canonical) {
  return kind == KIND_TOTAL && shells_canonical && L <= TB_S1_TPL_MAXL;
}

cudaError_t launch_stage1_tpl(int kind, int tuple, const Stage1Args &a, int ngeom, cudaStream_t st) {
  if (kind == KIND_TOTAL) return launch_stage1_tpl_k<KIND_TOTAL>(tuple, a, ngeom, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage1_tpl_batch(int kind, int tuple, const Stage1Args *d, const int64_t *pre, int n,
                                    int64_t blocks, cudaStream_t st) {
  if (kind == KIND_TOTAL) return launch_stage1_tpl_batch_k<KIND_TOTAL>(tuple, d, pre, n, blocks, st);
  return cudaErrorInvalidValue;
}

bool stage1_xk(int L, int64_t nquart, int nsm) {
  if (L < TB_S1_XK_MIN) return false;
  if (L <= 6) return true;
  return L <= 8 && nquart >= (int64_t)TB_S1_XK_HIGH_PER_SM * nsm;
}

cudaError_t launch_stage1_xk(int kind, int L, int LK, bool XB, const Stage1Args &a, int ngeom, cudaStream_t st) {
  if (kind == KIND_TOTAL) return launch_stage1_xk_k<KIND_TOTAL>(L, LK, XB, a, ngeom, st);
  if (kind == KIND_ELASTIC) return launch_stage1_xk_k<KIND_ELASTIC>(L, LK, XB, a, ngeom, st);
  if (kind == KIND_ALIGNED) return launch_stage1_xk_k<KIND_ALIGNED>(L, LK, XB, a, ngeom, st);
  if (kind == KIND_ELASTIC_J2) return launch_stage1_xk_k<KIND_ELASTIC_J2>(L, LK, XB, a, ngeom, st);
  if (kind == KIND_CMS) return launch_stage1_xk_k<KIND_CMS>(L, LK, XB, a, ngeom, st);
  return launch_stage1_xk_k<KIND_J2>(L, LK, XB, a, ngeom, st);
}

cudaError_t launch_stage1_xsplit(int kind, int L, int LK, bool XB, const Stage1Args &a, double *xbuf, int nout,
                                 cudaStream_t st, bool with_xc) {
  if (kind == KIND_TOTAL) return launch_stage1_xsplit_k<KIND_TOTAL>(L, LK, XB, a, xbuf, nout, with_xc, st);
  if (kind == KIND_ELASTIC) return launch_stage1_xsplit_k<KIND_ELASTIC>(L, LK, XB, a, xbuf, nout, with_xc, st);
  if (kind == KIND_ALIGNED) return launch_stage1_xsplit_k<KIND_ALIGNED>(L, LK, XB, a, xbuf, nout, with_xc, st);
  if (kind == KIND_ELASTIC_J2) return launch_stage1_xsplit_k<KIND_ELASTIC_J2>(L, LK, XB, a, xbuf, nout, with_xc, st);
  if (kind == KIND_CMS) return launch_stage1_xsplit_k<KIND_CMS>(L, LK, XB, a, xbuf, nout, with_xc, st);
  return launch_stage1_xsplit_k<KIND_J2>(L, LK, XB, a, xbuf, nout, with_xc, st);
}

bool stage1_xct(int kind, int LK, int shells_canonical) {
  return kind == KIND_TOTAL && shells_canonical && LK <= 3;
}

cudaError_t launch_stage1_xct(int kind, int tuple, bool XB, const Stage1Args &a, double *xbuf, int xstride,
                              int64_t xbase, cudaStream_t st) {
  if (kind == KIND_TOTAL) return launch_stage1_xct_k<KIND_TOTAL>(tuple, XB, a, xbuf, xstride, xbase, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage1_xct_batch(int kind, int tuple, bool XB, const Stage1Args *d, const int64_t *pre, int n,
                                    int64_t blocks, double *xbuf, cudaStream_t st) {
  if (kind == KIND_TOTAL) return launch_stage1_xct_batch_k<KIND_TOTAL>(tuple, XB, d, pre, n, blocks, xbuf, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage1_xsplit_batch(int kind, int L, int LK, int XB, const Stage1Args *d, const int64_t *prexc,
                                       int64_t blocksxc, const int64_t *pre, int64_t blocks, int n, double *xbuf,
                                       cudaStream_t st) {
#define TB_K(k) return launch_stage1_xsplit_batch_k<k>(L, LK, XB, d, prexc, blocksxc, pre, blocks, n, xbuf, st)
  if (kind == KIND_TOTAL) TB_K(KIND_TOTAL);
  if (kind == KIND_ELASTIC) TB_K(KIND_ELASTIC);
  if (kind == KIND_ALIGNED) TB_K(KIND_ALIGNED);
  if (kind == KIND_ELASTIC_J2) TB_K(KIND_ELASTIC_J2);
  if (kind == KIND_CMS) TB_K(KIND_CMS);
  TB_K(KIND_J2);
#undef TB_K
}

cudaError_t launch_pair_tables_batch(const PairDesc *d, const int64_t *pre, int n, int64_t blocks, cudaStream_t st) {
  if (n <= 0 || blocks <= 0) return cudaSuccess;
  pair_tables_batch_kernel<<<(unsigned)blocks, 128, 0, st>>>(d, pre, n);
  return cudaGetLastError();
}

cudaError_t launch_reduce_desc(const ReduceDesc *d, int n, int nqmax, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  reduce_desc_kernel<<<dim3((nqmax + 127) / 128, n), 128, 0, st>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_stage1_batch(int kind, int L, int LK, int XB, const Stage1Args *d, const int64_t *pre, int n,
                                int64_t blocks, cudaStream_t st) {
  if (kind == KIND_TOTAL) return launch_stage1_batch_k<KIND_TOTAL>(L, LK, XB, d, pre, n, blocks, st);
  if (kind == KIND_ELASTIC) return launch_stage1_batch_k<KIND_ELASTIC>(L, LK, XB, d, pre, n, blocks, st);
  if (kind == KIND_ALIGNED) return launch_stage1_batch_k<KIND_ALIGNED>(L, LK, XB, d, pre, n, blocks, st);
  if (kind == KIND_ELASTIC_J2) return launch_stage1_batch_k<KIND_ELASTIC_J2>(L, LK, XB, d, pre, n, blocks, st);
  if (kind == KIND_CMS) return launch_stage1_batch_k<KIND_CMS>(L, LK, XB, d, pre, n, blocks, st);
  return launch_stage1_batch_k<KIND_J2>(L, LK, XB, d, pre, n, blocks, st);
}

cudaError_t launch_stage1(int kind, int L, const Stage1Args &a, int ngeom, cudaStream_t st) {
  // instantiated in tb_stage1_{total,elastic,j2,aligned,elastic_j2,cms}.cu
  if (kind == KIND_TOTAL) return launch_stage1_k<KIND_TOTAL>(L, a, ngeom, st);
  if (kind == KIND_ELASTIC) return launch_stage1_k<KIND_ELASTIC>(L, a, ngeom, st);
  if (kind == KIND_ALIGNED) return launch_stage1_k<KIND_ALIGNED>(L, a, ngeom, st);
  if (kind == KIND_ELASTIC_J2) return launch_stage1_k<KIND_ELASTIC_J2>(L, a, ngeom, st);
  if (kind == KIND_CMS) return launch_stage1_k<KIND_CMS>(L, a, ngeom, st);
  return launch_stage1_k<KIND_J2>(L, a, ngeom, st);
}

size_t stage2_smem_bytes(int nqp, int nwarps) { return sizeof(double) * (size_t)nqp * (3 + nwarps); }

cudaError_t launch_stage2(const Stage2Args &a, int grid, int nwarps, cudaStream_t st) {
  size_t smem = stage2_smem_bytes(a.nqp, nwarps);
  cudaError_t e = cudaFuncSetAttribute(stage2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  stage2_kernel<<<grid, nwarps * 32, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_reduce(const double *partial, int nblocks, int nq, double *out, cudaStream_t st) {
  reduce_kernel<<<(nq + 31) / 32, REDUCE_WARPS * 32, 0, st>>>(partial, nblocks, nq, out, 0);
  return cudaGetLastError();
}

cudaError_t launch_reduce_batch(const double *partial, int nblocks, int nq, int64_t gs_in, double *out, int ngeom,
                                cudaStream_t st) {
  reduce_kernel<<<dim3((nq + 31) / 32, ngeom), REDUCE_WARPS * 32, 0, st>>>(partial, nblocks, nq, out, gs_in);
  return cudaGetLastError();
}

cudaError_t launch_ghat_emit(const int *mat, const double *total, int nmat, int n, int *keys, double *vals,
                             cudaStream_t st) {
  if (nmat <= 0) return cudaSuccess;
  ghat_emit_kernel<<<(nmat + 255) / 256, 256, 0, st>>>(mat, total, nmat, n, keys, vals);
  return cudaGetLastError();
}

cudaError_t launch_ghat_runs(const int *keys, const double *vals, int64_t m, double *G, cudaStream_t st) {
  if (m <= 0) return cudaSuccess;
  ghat_runs_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(keys, vals, m, G);
  return cudaGetLastError();
}


cudaError_t launch_quartet_fill(int ng, const int64_t *bra_off, int64_t nquart, const int *gL,
                                uint64_t *quart, uint32_t *keys, bool all_pairs, cudaStream_t st) {
  if (nquart <= 0) return cudaSuccess;
  quartet_fill_kernel<<<(unsigned)((nquart + 255) / 256), 256, 0, st>>>(ng, bra_off, npairs(ng), nquart, gL,
                                                                        quart, keys, all_pairs ? 1 : 0);
  return cudaGetLastError();
}

int stage2_blocks_per_sm(int nqp, int nwarps) {
  int nb = 0;
  size_t smem = stage2_smem_bytes(nqp, nwarps);
  cudaFuncSetAttribute(stage2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, stage2_kernel, nwarps * 32, smem) != cudaSuccess) return 1;
  return nb > 0 ? nb : 1;
}

__global__ void iota_kernel(uint32_t *v, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (uint32_t)i;
}

cudaError_t launch_iota(uint32_t *v, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  iota_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(v, n);
  return cudaGetLastError();
}

cudaError_t launch_sym_small(const double *in, int n, double *out, cudaStream_t st) {
  sym_small_kernel<<<(n * n + 127) / 128, 128, 0, st>>>(in, n, out);
  return cudaGetLastError();
}

}  // namespace tb
