// Stage 1 of the quartet evaluation: per group quartet, the Hermite-space
// density D[T][U][V] summed over its primitive (function) quartets with the
// reference's cutoffs (tot_integral_k_ijkr, src/Integrals.f90:5155-5219, and
// the pzero / elastic / j2 variants), then either the Bessel expansion
// coefficients h_b (BesselDeriv :4708-4746, BesselDeriv2j :6370-6434) or the
// P = Q polynomial (P_LMN :3102-3135, P_LMN_j2 :3137-3170).
//
// Two kernels produce D:
//   stage1_reg_kernel<L, K>   LLmax <= 8: D lives in registers with a
//       compile-time shape.  S = stage1_reg_split(L) threads share a quartet;
//       thread s of the group owns the entries with V = s (mod S), all S walk
//       the same function quartets (no divergence inside a warp whose
//       quartets have equal shell types, the order the class sort produces).
//       Per function quartet the six-deep loop of the reference becomes three
//       full-length 1-D convolutions and one outer product, all unrolled.
//   stage1_smem_kernel<L, K>  LLmax 9..16 (f and g shells): each thread keeps
//       a partial density in its own shared-memory column; S threads split the
//       function-quartet loop and are summed in a fixed order.
// Both hand D to the same epilogue through a shared-memory column.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_kernels.h"
#include "tb_math.cuh"

namespace tb {

__device__ __forceinline__ void unpack_quartet(uint64_t pk, int &gi, int &gj, int &gk, int &gr) {
  gi = (int)(pk & 0xffff);
  gj = (int)((pk >> 16) & 0xffff);
  gk = (int)((pk >> 32) & 0xffff);
  gr = (int)((pk >> 48) & 0xffff);
}

// The five loops of tot_integration give these weights (src/Integrals.f90:158,243,325,402,462).
__device__ __forceinline__ int quartet_loop(int gi, int gj, int gk, int gr) {
  if (gi == gj) return gk == gr ? (gi == gk ? 5 : 4) : 3;
  return gk == gi ? 2 : 1;
}
__device__ __forceinline__ double loop_weight(int loop) {
  return loop == 1 ? 8.0 : (loop <= 3 ? 4.0 : (loop == 4 ? 2.0 : 1.0));
}

// Simplex layout of D[T][U][V], T+U+V <= L, with V contiguous:
// idx = ntuv(L) - ntuv(L-T) + U (L-T+1) - U (U-1)/2 + V.
template <int L>
__device__ __forceinline__ int dindex(int T, int U, int V) {
  return ntuv(L) - ntuv(L - T) + U * (L - T + 1) - (U * (U - 1)) / 2 + V;
}

// Sum over the S lanes of one quartet's thread group (result in its first lane).
template <int S>
__device__ __forceinline__ double group_sum(double v, unsigned mask) {
#pragma unroll
  for (int off = S / 2; off > 0; off >>= 1) v += __shfl_down_sync(mask, v, off, S);
  return v;
}

#ifndef TB_S1_PF_MAXL
#define TB_S1_PF_MAXL -1
#endif
// contracted-side kernel instances for LLmax 7 and 8 as well
#ifndef TB_S1_XK_HIGH
#define TB_S1_XK_HIGH 1
#endif
#ifndef TB_S1_MB_LO
#define TB_S1_MB_LO 2
#endif
#ifndef TB_S1_MB_3
#define TB_S1_MB_3 3
#endif
// Largest LLmax handled by the register kernel, and its threads per quartet.
constexpr int STAGE1_REG_MAXL = 8;
TB_HD constexpr int stage1_reg_split(int L) { return L <= 4 ? 1 : (L == 5 ? 2 : (L == 6 ? 4 : 8)); }
// The heaviest classes have few quartets with many function quartets each:
// P groups of S threads split the bra function pairs of a quartet, and the P
// partial densities are summed in a fixed order.
TB_HD constexpr int stage1_reg_parts(int L) { return L >= 7 ? 4 : 1; }
// Threads per quartet of the shared-memory kernel.
TB_HD constexpr int stage1_smem_split(int L) { return L <= 15 ? 32 : 16; }
TB_HD constexpr int stage1_split(int L) {
  return L <= STAGE1_REG_MAXL ? stage1_reg_split(L) * stage1_reg_parts(L) : stage1_smem_split(L);
}
// Resident blocks asked of the register allocator: the largest count whose
// register cap (65536 / (128 x blocks)) still holds the kernel without spills.
TB_HD constexpr int stage1_reg_minblocks(int L) { return L <= TB_S1_MB_LO ? 4 : (L == 3 ? TB_S1_MB_3 : 2); }
// Classes whose density and ket coefficients of the next function quartet are
// loaded before the current one is used (a one-deep software pipeline hiding
// the gather latency where registers allow it).
TB_HD constexpr int stage1_prefetch(int L) { return L <= TB_S1_PF_MAXL; }
// Register entries of one thread: (T, U, j) with V = S j + s <= L - T - U for some s.
TB_HD constexpr int reg_entries(int L, int S) {
  int n = 0;
  for (int T = 0; T <= L; ++T)
    for (int U = 0; U <= L - T; ++U) n += (L - T - U) / S + 1;
  return n;
}

struct QuartetHead {
  int gi, gj, gk, gr, loop;
  double w;  // loop weight
  bool p0;
  int skip;
  double Hx, Hy, Hz, h;
  const double *tb, *tk;
};

template <int KIND>
__device__ __forceinline__ QuartetHead quartet_head(const Stage1Args &A, int64_t qi) {
  QuartetHead Q;
  unpack_quartet(A.quartets[qi], Q.gi, Q.gj, Q.gk, Q.gr);
  Q.tb = A.pairtab + (size_t)pair_index(Q.gi, Q.gj, A.ng) * PAIR_STRIDE;
  Q.tk = A.pairtab + (size_t)pair_index(Q.gk, Q.gr, A.ng) * PAIR_STRIDE;
  // hx = px(k,r) - px(i,j)  (src/Integrals.f90:83-86)
  Q.Hx = Q.tk[0] - Q.tb[0];
  Q.Hy = Q.tk[1] - Q.tb[1];
  Q.Hz = Q.tk[2] - Q.tb[2];
  Q.h = sqrt(Q.Hx * Q.Hx + Q.Hy * Q.Hy + Q.Hz * Q.Hz);
  Q.loop = quartet_loop(Q.gi, Q.gj, Q.gk, Q.gr);
  Q.w = loop_weight(Q.loop);
  // the aligned kernel has no P = Q branch (tot_integral_k_ijkr_alig, src/Integrals.f90:5588-5727)
  Q.p0 = KIND == KIND_ALIGNED ? false : (Q.loop == 5 || Q.h < A.cutoffcentre);
  if (KIND == KIND_CMS) {
    // resolved_cms_integration: weight 2 for each off-diagonal side (4, 2, 2,
    // 1), and the P = Q branch only where h < cutoffcentre, loop 4 included
    // (src/Integrals.f90:2698-2716, 2908-2919)
    Q.w = (Q.gi < Q.gj ? 2.0 : 1.0) * (Q.gk < Q.gr ? 2.0 : 1.0);
    Q.p0 = Q.h < A.cutoffcentre;
  }
  // |E| < 1e-30 skips that the reference keeps (bit: MDL MDM MDN MDLp MDMp):
  // a skipped factor removes every term it multiplies, i.e. it is a zero.
  Q.skip = (Q.p0 || KIND == KIND_ALIGNED || kind_elastic(KIND)) ? 0x1f : (KIND == KIND_TOTAL ? 0x00 : 0x0f);
  return Q;
}

// From the quartet's Hermite density (entry k at D[k * dstride], the whole
// density visible to every thread of the group) to its record
// [H, 1/4p+1/4p', kind, order, coefficients...].  Thread `sub` of the S-group
// handles every S-th term; the group leader writes the record.
// Stage-2 order key: P = Q quartets first (bucket 0), then quarter octaves of H.
__device__ __forceinline__ uint32_t h_bucket(double h) {
  int b = (int)floor(4.0 * log2(h)) + 32;
  return (uint32_t)min(max(b, 1), 63);
}

template <int L, int KIND, int S>
__device__ __forceinline__ void stage1_finish(const Stage1Args &A, const QuartetHead &Q, const double *D, int dstride,
                                              int64_t qi, int sub, unsigned gmask) {
  if (A.s2key && sub == 0) A.s2key[qi] = ((uint32_t)A.cls << 6) | (Q.p0 ? 0u : h_bucket(Q.h));
  const double pre = Q.w * Q.tb[4] * Q.tk[4];
  double *r = A.rec + A.recbase + (qi - A.qbegin) * (int64_t)A.rs;
  const bool leader = sub == 0;
  if (KIND == KIND_ALIGNED) {
    // [Hx, Hy, Hz, 1/4p+1/4p', w K K' D_TUV...]: the q-vector kernel forms
    // sum_TUV D_TUV (i qx)^T (i qy)^U (i qz)^V exp(i q.H) itself
    if (!leader) return;
    r[0] = Q.Hx;
    r[1] = Q.Hy;
    r[2] = Q.Hz;
    r[3] = Q.tb[5] + Q.tk[5];
    for (int k = 0; k < ntuv(L); ++k) r[4 + k] = pre * D[k * dstride];
    return;
  }
  if (Q.p0) {
    // F(q) = sum_s c_s q^{2s}, c_s = (-1)^s sum_{T+U+V=2s, even} D P0-factor
    constexpr int NS = L / 2 + 1;
    double cs[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) cs[k] = 0.0;
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < NS; ++k)
      for (int T = 0; T <= 2 * k; T += 2)
        for (int U = 0; U <= 2 * k - T; U += 2) {
          if ((cnt++ % S) != sub) continue;
          int V = 2 * k - T - U;
          double f = p0_factor(T, U, V, kind_j2(KIND));
          if (kind_j2(KIND)) f = (T + U - 2 * V) / 4.0 * f;
          cs[k] += D[dindex<L>(T, U, V) * dstride] * f;
        }
#pragma unroll
    for (int k = 0; k < NS; ++k) cs[k] = group_sum<S>(cs[k], gmask);
    if (!leader) return;
    if (A.p0count) atomicAdd(A.p0count, 1ull);
    const double fj2 = sqrt(5.0 / TB_PI);
    r[0] = 0.0;
    r[1] = Q.tb[5] + Q.tk[5];
    r[2] = (double)REC_P0;
    r[3] = (double)(NS - 1);
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      double acc = kind_j2(KIND) ? cs[k] * fj2 : cs[k];
      r[4 + k] = pre * ((k & 1) ? -acc : acc);
    }
    return;
  }

  // Bessel expansion: h[b] = sum_TUV D[TUV] sum_{p} a(T,px) b(U,py) c(V,pz),
  // b = (T+px)/2 + (U+py)/2 + (V+pz)/2 (BesselDeriv); for j2 the four-term
  // BesselDeriv2j form with two extra orders (src/Integrals.f90:6370-6434).
  constexpr int LB = kind_j2(KIND) ? L + 2 : L;
  constexpr int TP = tp_size(L);
  double ax[TP], ay[TP], az[TP];
  hermite_table(L, Q.Hx, ax);
  hermite_table(L, Q.Hy, ay);
  hermite_table(L, Q.Hz, az);
  double hh[LB + 1];
#pragma unroll
  for (int b = 0; b <= LB; ++b) hh[b] = 0.0;
  const double eta = 3.0 * (Q.Hz * Q.Hz) - Q.h * Q.h;
  int cnt = 0;
  for (int T = 0; T <= L; ++T)
    for (int U = 0; U <= L - T; ++U)
      for (int V = 0; V <= L - T - U; ++V) {
        if ((cnt++ % S) != sub) continue;
        double d = D[dindex<L>(T, U, V) * dstride];
        if (d == 0.0) continue;
        for (int k1 = 0; 2 * k1 <= T; ++k1) {
          double cx = ax[tp_off(T) + k1];
          double cx1 = (double)(2 * (T - k1)) * cx;
          for (int k2 = 0; 2 * k2 <= U; ++k2) {
            double cy = ay[tp_off(U) + k2];
            double cy1 = (double)(2 * (U - k2)) * cy;
            for (int k3 = 0; 2 * k3 <= V; ++k3) {
              double cz = az[tp_off(V) + k3];
              int s3 = (T - k1) + (U - k2) + (V - k3);
              if (!kind_j2(KIND)) {
                hh[s3] += d * (cx * cy * cz);
              } else {
                double cz1 = (double)(2 * (V - k3)) * cz;
                hh[s3 + 2] += d * (cx * cy * cz * eta);
                hh[s3 + 1] += d * (cx1 * cy * cz + cx * cy1 * cz - 2.0 * (cx * cy * cz1));
              }
            }
          }
        }
      }
#pragma unroll
  for (int b = 0; b <= LB; ++b) hh[b] = group_sum<S>(hh[b], gmask);
  if (!leader) return;
  if (kind_j2(KIND)) {
    const double f = 0.25 * sqrt(5.0 / TB_PI);
#pragma unroll
    for (int b = 0; b <= LB; ++b) hh[b] *= f;
  }
  if (KIND == KIND_ELASTIC || KIND == KIND_CMS) {
    // integral_k_ijkr returns F = 0 when sum(h_saved) == 0 (src/Integrals.f90:5883-5886)
    double sum = 0.0;
#pragma unroll
    for (int b = 0; b <= LB; ++b) sum += hh[b];
    if (sum == 0.0) {
#pragma unroll
      for (int b = 0; b <= LB; ++b) hh[b] = 0.0;
    }
  }
  r[0] = Q.h;
  r[1] = Q.tb[5] + Q.tk[5];
  r[2] = (double)(kind_j2(KIND) ? REC_BESSEL_J2 : REC_BESSEL);
  r[3] = (double)LB;
  // hhat_b = h_b / H^{2b}: F = sum_b hhat_b j_b(x) x^b, x = qH
  const double invH2 = 1.0 / (Q.h * Q.h);
  double f = pre;
#pragma unroll
  for (int b = 0; b <= LB; ++b) {
    r[4 + b] = hh[b] * f;
    f *= invH2;
  }
}

// ---------------------------------------------------------------------------
// register kernel (LLmax <= 8)
// ---------------------------------------------------------------------------
// E^{la,lb}_t of one axis of one group pair in the transposed table: element t
// of slot (axis, la, lb) at e[(slot * E_T + t) * npairs], zero for t > la + lb.
__device__ __forceinline__ const double *esoa_slot(const Stage1Args &A, bool skipped, int axis, int la, int lb,
                                                   int pair) {
  const int m1 = A.emaxa + 1;
  const int slot = (axis * m1 + la) * m1 + lb;
  return A.esoa + (skipped ? A.eskip : 0) + (int64_t)slot * E_T * A.npair + pair;
}

// Molecule batches: launch blocks are spread over items (one plan's quartet
// range each); pre[i] is item i's first block, pre[n] the total.
__device__ __forceinline__ int batch_item(const int64_t *__restrict__ pre, int n, int64_t b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Geometry blockIdx.y of a batch: its pair tables, E tables, records and
// P = Q counter; the stage-2 order keys are written for geometry 0 only.
__device__ __forceinline__ void stage1_geometry(Stage1Args &A) {
  const int64_t g = blockIdx.y;
  if (g == 0) return;
  A.pairtab += g * A.gs_pair;
  A.esoa += g * A.gs_esoa;
  A.rec += g * A.gs_rec;
  if (A.p0count) A.p0count += g * MAXCLS;
  A.s2key = nullptr;
}

template <int L, int KIND>
__device__ __forceinline__ void stage1_reg_body(Stage1Args &A, int64_t vb) {
  constexpr int S = stage1_reg_split(L);
  constexpr int PP = stage1_reg_parts(L);
  constexpr int G = S * PP;              // threads per quartet
  constexpr int NE = reg_entries(L, S);
  constexpr int NG = 128 / S;            // density columns per block: one per S threads
  constexpr int TMAX = L < 2 * MAXA ? L : 2 * MAXA;  // last E index an axis can reach
  extern __shared__ double sD[];         // ntuv(L) x NG
  const int gsub = threadIdx.x % G;      // thread within the quartet's group
  const int sub = gsub % S, part = gsub / S, grp = threadIdx.x / S;
  const int lane = threadIdx.x & 31;
  const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lane - gsub));
  const int64_t qi = A.qbegin + (vb * blockDim.x + threadIdx.x) / G;
  // whole groups leave together (S divides 32)
  if (qi >= A.qend) return;
  const QuartetHead Q = quartet_head<KIND>(A, qi);
  const int pb = pair_index(Q.gi, Q.gj, A.ng), pk = pair_index(Q.gk, Q.gr, A.ng);
  const int64_t np = A.npair;

  double D[NE];
#pragma unroll
  for (int e = 0; e < NE; ++e) D[e] = 0.0;

  const int si = A.gstart[Q.gi], ni = A.gcount[Q.gi];
  const int sj = A.gstart[Q.gj], nj = A.gcount[Q.gj];
  const int sk = A.gstart[Q.gk], nk = A.gcount[Q.gk];
  const int sr = A.gstart[Q.gr], nr = A.gcount[Q.gr];
  for (int ab = part; ab < ni * nj; ab += PP) {
    {
      const int ia = ab / nj, ib = ab - ia * nj;
      const int fa = si + ia, fb = sj + ib;
      const int la = A.flmn[fa], lb = A.flmn[fb];
      const int64_t rowp = kind_elastic(KIND) ? 0 : fpair(min(fa, fb), max(fa, fb)) * A.np;
      const double zab = kind_elastic(KIND) ? A.zao[(size_t)fa * A.ngto + fb] : 0.0;
      // bra coefficients with the (-1)^t sign of src/Integrals.f90:5181
      double bx[L + 1], by[L + 1], bz[L + 1];
      {
        const double *ex = esoa_slot(A, Q.skip & 1, 0, la & 0xff, lb & 0xff, pb);
        const double *ey = esoa_slot(A, Q.skip & 2, 1, (la >> 8) & 0xff, (lb >> 8) & 0xff, pb);
        const double *ez = esoa_slot(A, Q.skip & 4, 2, (la >> 16) & 0xff, (lb >> 16) & 0xff, pb);
#pragma unroll
        for (int t = 0; t <= L; ++t) {
          double vx = t <= TMAX ? ex[t * np] : 0.0;
          double vy = t <= TMAX ? ey[t * np] : 0.0;
          double vz = t <= TMAX ? ez[t * np] : 0.0;
          bx[t] = (t & 1) ? -vx : vx;
          by[t] = (t & 1) ? -vy : vy;
          bz[t] = (t & 1) ? -vz : vz;
        }
      }
      // ket function pairs; the density and ket coefficients of the next pair
      // are loaded before the current one is used (one-deep software pipeline)
      const int ncd = nk * nr;
      auto fetch = [&](int ic, int id, double &zo, double *kxo, double *kyo, double *kzo) {
        const int fc = sk + ic, fd = sr + id;
        if (kind_elastic(KIND)) zo = A.zket[(size_t)fc * A.ngto + fd] * zab;
        else zo = A.rho[rowp + fpair(min(fc, fd), max(fc, fd))];
        const int lc = A.flmn[fc], ld = A.flmn[fd];
        const double *ex = esoa_slot(A, Q.skip & 8, 0, lc & 0xff, ld & 0xff, pk);
        const double *ey = esoa_slot(A, Q.skip & 16, 1, (lc >> 8) & 0xff, (ld >> 8) & 0xff, pk);
        const double *ez = esoa_slot(A, false, 2, (lc >> 16) & 0xff, (ld >> 16) & 0xff, pk);
#pragma unroll
        for (int t = 0; t <= TMAX; ++t) {
          kxo[t] = ex[t * np];
          kyo[t] = ey[t * np];
          kzo[t] = ez[t * np];
        }
      };
      constexpr bool PF = stage1_prefetch(L);
      double zn = 0.0, kxn[TMAX + 1], kyn[TMAX + 1], kzn[TMAX + 1];
      if (PF) fetch(0, 0, zn, kxn, kyn, kzn);
      int icn = 0, idn = 0;
      for (int cd = 0; cd < ncd; ++cd) {
        {
          double z, kx[TMAX + 1], ky[TMAX + 1], kz[TMAX + 1];
          if constexpr (PF) {
            z = zn;
#pragma unroll
            for (int t = 0; t <= TMAX; ++t) {
              kx[t] = kxn[t];
              ky[t] = kyn[t];
              kz[t] = kzn[t];
            }
          } else {
            fetch(icn, idn, z, kx, ky, kz);
          }
          if (++idn == nr) {
            idn = 0;
            ++icn;
          }
          if (PF && cd + 1 < ncd) fetch(icn, idn, zn, kxn, kyn, kzn);
          // the reference skips primitive quartets with |ztot| < cutoffz
          z = fabs(z) < A.cutoffz ? 0.0 : z;
          // C_axis[T] = sum_t b[t] k[T - t] over the full (zero-padded) range
          double Cx[L + 1], Cy[L + 1], Cz[L + 1];
#pragma unroll
          for (int T = 0; T <= L; ++T) {
            double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
            for (int t = 0; t <= T; ++t) {
              if (T - t > TMAX) continue;
              sx = fma(bx[t], kx[T - t], sx);
              sy = fma(by[t], ky[T - t], sy);
              sz = fma(bz[t], kz[T - t], sz);
            }
            Cx[T] = sx * z;
            Cy[T] = sy;
            Cz[T] = sz;
          }
          // this thread's z values: V = S j + sub
          double Czs[L / S + 1];
#pragma unroll
          for (int j = 0; j <= L / S; ++j) {
            double v = Cz[S * j];
#pragma unroll
            for (int u = 1; u < S; ++u)
              if (S * j + u <= L) v = sub == u ? Cz[S * j + u] : v;
            Czs[j] = v;
          }
          int e = 0;
#pragma unroll
          for (int T = 0; T <= L; ++T)
#pragma unroll
            for (int U = 0; U <= L - T; ++U) {
              const double w = Cx[T] * Cy[U];
#pragma unroll
              for (int j = 0; j <= (L - T - U) / S; ++j, ++e) D[e] = fma(w, Czs[j], D[e]);
            }
        }
      }
    }
  }
  // hand the density to the epilogue through the group's shared column
  double *col = sD + grp;
  {
    int e = 0;
#pragma unroll
    for (int T = 0; T <= L; ++T)
#pragma unroll
      for (int U = 0; U <= L - T; ++U)
#pragma unroll
        for (int j = 0; j <= (L - T - U) / S; ++j, ++e) {
          const int V = S * j + sub;
          if (S == 1 || V <= L - T - U) col[dindex<L>(T, U, V) * NG] = D[e];
        }
  }
  if (G > 1) __syncwarp(gmask);
  if (PP > 1) {
    // fixed-order sum of the P partial densities into the first part's column
    double *col0 = sD + (threadIdx.x - gsub) / S;
    for (int k = gsub; k < ntuv(L); k += G) {
      double t = col0[k * NG];
#pragma unroll
      for (int p = 1; p < PP; ++p) t += col0[k * NG + p];
      col0[k * NG] = t;
    }
    __syncwarp(gmask);
    col = col0;
  }
  stage1_finish<L, KIND, G>(A, Q, col, NG, qi, gsub, gmask);
}

template <int L, int KIND>
__global__ void __launch_bounds__(128, stage1_reg_minblocks(L)) stage1_reg_kernel(Stage1Args A) {
  stage1_geometry(A);
  stage1_reg_body<L, KIND>(A, blockIdx.x);
}

template <int L, int KIND>
__global__ void __launch_bounds__(128, stage1_reg_minblocks(L))
    stage1_reg_batch(const Stage1Args *__restrict__ d, const int64_t *__restrict__ pre, int n) {
  const int it = batch_item(pre, n, blockIdx.x);
  Stage1Args A = d[it];
  stage1_reg_body<L, KIND>(A, blockIdx.x - pre[it]);
}

// ---------------------------------------------------------------------------
// shell-templated kernel (total j0, LLmax <= 3), thread per quartet
// ---------------------------------------------------------------------------
// The register kernel's arithmetic for one shell tuple (Li, Lj, Lk, Lr) of a
// class, on plans whose s-f groups hold their Cartesian components in the
// cart_component order: every function's exponents, and with them every E
// index, are compile-time constants, so all of a quartet's density and E
// loads are independent (issued ahead of the arithmetic) and repeated E
// values and convolutions are shared between function quartets.  The values
// and the order of the operations are those of stage1_reg_kernel, so the
// density D_TUV is bit-identical to it.
#ifndef TB_S1_TPL_MAXL
#define TB_S1_TPL_MAXL 3
#endif

template <int Li, int Lj, int Lk, int Lr, int KIND>
__device__ __forceinline__ void stage1_tpl_body(const Stage1Args &A, int64_t vb) {
  constexpr int L = Li + Lj + Lk + Lr;
  constexpr int ni = (Li + 1) * (Li + 2) / 2, nj = (Lj + 1) * (Lj + 2) / 2;
  constexpr int nk = (Lk + 1) * (Lk + 2) / 2, nr = (Lr + 1) * (Lr + 2) / 2;
  constexpr int TMAX = L < 2 * MAXA ? L : 2 * MAXA;
  extern __shared__ double sD[];  // ntuv(L) x 128
  const int64_t qi = A.qbegin + vb * blockDim.x + threadIdx.x;
  if (qi >= A.qend) return;
  const QuartetHead Q = quartet_head<KIND>(A, qi);
  const int si = A.gstart[Q.gi], sj = A.gstart[Q.gj], sk = A.gstart[Q.gk], sr = A.gstart[Q.gr];
  const double *tb = A.pairtab + (size_t)pair_index(Q.gi, Q.gj, A.ng) * PAIR_STRIDE + 8;
  const double *tk = A.pairtab + (size_t)pair_index(Q.gk, Q.gr, A.ng) * PAIR_STRIDE + 8;
  // E^{l1 l2}_t of one axis of a pair, with this quartet's |E| < 1e-30 skip
  auto ecoef = [&](const double *tab, int ax, int l1, int l2, int t, bool skip) -> double {
    const double v = tab[ax * ESZ + (l1 * (MAXA + 1) + l2) * E_T + t];
    return (skip && fabs(v) < TB_SKIP30) ? 0.0 : v;
  };
  double D[ntuv(L)];
#pragma unroll
  for (int e = 0; e < ntuv(L); ++e) D[e] = 0.0;
#pragma unroll
  for (int a = 0; a < ni; ++a)
#pragma unroll
    for (int b = 0; b < nj; ++b) {
      const int fa = si + a, fb = sj + b;
      const int64_t rowp = fpair(min(fa, fb), max(fa, fb)) * A.np;
      // bra coefficients with the (-1)^t sign of src/Integrals.f90:5181
      double bx[L + 1], by[L + 1], bz[L + 1];
#pragma unroll
      for (int t = 0; t <= L; ++t) {
        const int x1 = cart_component(Li, a, 0), x2 = cart_component(Lj, b, 0);
        const int y1 = cart_component(Li, a, 1), y2 = cart_component(Lj, b, 1);
        const int z1 = cart_component(Li, a, 2), z2 = cart_component(Lj, b, 2);
        const double vx = (t <= TMAX && t <= x1 + x2) ? ecoef(tb, 0, x1, x2, t, Q.skip & 1) : 0.0;
        const double vy = (t <= TMAX && t <= y1 + y2) ? ecoef(tb, 1, y1, y2, t, Q.skip & 2) : 0.0;
        const double vz = (t <= TMAX && t <= z1 + z2) ? ecoef(tb, 2, z1, z2, t, Q.skip & 4) : 0.0;
        bx[t] = (t & 1) ? -vx : vx;
        by[t] = (t & 1) ? -vy : vy;
        bz[t] = (t & 1) ? -vz : vz;
      }
#pragma unroll
      for (int c = 0; c < nk; ++c)
#pragma unroll
        for (int d = 0; d < nr; ++d) {
          const int fc = sk + c, fd = sr + d;
          double z = A.rho[rowp + fpair(min(fc, fd), max(fc, fd))];
          const int x1 = cart_component(Lk, c, 0), x2 = cart_component(Lr, d, 0);
          const int y1 = cart_component(Lk, c, 1), y2 = cart_component(Lr, d, 1);
          const int z1 = cart_component(Lk, c, 2), z2 = cart_component(Lr, d, 2);
          double kx[TMAX + 1], ky[TMAX + 1], kz[TMAX + 1];
#pragma unroll
          for (int t = 0; t <= TMAX; ++t) {
            kx[t] = t <= x1 + x2 ? ecoef(tk, 0, x1, x2, t, Q.skip & 8) : 0.0;
            ky[t] = t <= y1 + y2 ? ecoef(tk, 1, y1, y2, t, Q.skip & 16) : 0.0;
            kz[t] = t <= z1 + z2 ? ecoef(tk, 2, z1, z2, t, false) : 0.0;
          }
          // the reference skips primitive quartets with |ztot| < cutoffz
          z = fabs(z) < A.cutoffz ? 0.0 : z;
          double Cx[L + 1], Cy[L + 1], Cz[L + 1];
#pragma unroll
          for (int T = 0; T <= L; ++T) {
            double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
            for (int t = 0; t <= T; ++t) {
              if (T - t > TMAX) continue;
              sx = fma(bx[t], kx[T - t], sx);
              sy = fma(by[t], ky[T - t], sy);
              sz = fma(bz[t], kz[T - t], sz);
            }
            Cx[T] = sx * z;
            Cy[T] = sy;
            Cz[T] = sz;
          }
          int e = 0;
#pragma unroll
          for (int T = 0; T <= L; ++T)
#pragma unroll
            for (int U = 0; U <= L - T; ++U) {
              const double w = Cx[T] * Cy[U];
#pragma unroll
              for (int V = 0; V <= L - T - U; ++V, ++e) D[e] = fma(w, Cz[V], D[e]);
            }
        }
    }
  double *col = sD + threadIdx.x;
#pragma unroll
  for (int e = 0; e < ntuv(L); ++e) col[e * 128] = D[e];
  stage1_finish<L, KIND, 1>(A, Q, col, 128, qi, 0, 1u << (threadIdx.x & 31));
}

template <int Li, int Lj, int Lk, int Lr, int KIND>
__global__ void __launch_bounds__(128) stage1_tpl_kernel(Stage1Args A) {
  stage1_geometry(A);
  stage1_tpl_body<Li, Lj, Lk, Lr, KIND>(A, blockIdx.x);
}

// Molecule batches: item i (one plan's quartets of this shell tuple) owns
// blocks pre[i] .. pre[i+1]-1.
template <int Li, int Lj, int Lk, int Lr, int KIND>
__global__ void __launch_bounds__(128)
    stage1_tpl_batch(const Stage1Args *__restrict__ d, const int64_t *__restrict__ pre, int n) {
  const int it = batch_item(pre, n, blockIdx.x);
  const Stage1Args A = d[it];
  stage1_tpl_body<Li, Lj, Lk, Lr, KIND>(A, blockIdx.x - pre[it]);
}

// One launch per shell tuple of a class's sub-range (s = Li..Lr, packed as
// ((Li 5 + Lj) 5 + Lk) 5 + Lr).
template <int K>
cudaError_t launch_stage1_tpl_k(int tuple, const Stage1Args &a, int ngeom, cudaStream_t st) {
  const int64_t n = a.qend - a.qbegin;
  if (n <= 0) return cudaSuccess;
#define TB_TPL(i, j, k, r)                                                                             \
  case ((i * 5 + j) * 5 + k) * 5 + r: {                                                              \
    const size_t smem = (size_t)ntuv(i + j + k + r) * sizeof(double) * 128;                          \
    cudaError_t e = cudaFuncSetAttribute(stage1_tpl_kernel<i, j, k, r, K>,                           \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);    \
    if (e != cudaSuccess) return e;                                                                  \
    stage1_tpl_kernel<i, j, k, r, K><<<dim3((unsigned)((n + 127) / 128), ngeom), 128, smem, st>>>(a); \
    return cudaGetLastError();                                                                       \
  }
  switch (tuple) {
    TB_TPL(0, 0, 0, 0)
    TB_TPL(1, 0, 0, 0) TB_TPL(0, 1, 0, 0) TB_TPL(0, 0, 1, 0) TB_TPL(0, 0, 0, 1)
#if TB_S1_TPL_MAXL >= 2
    TB_TPL(2, 0, 0, 0) TB_TPL(0, 2, 0, 0) TB_TPL(0, 0, 2, 0) TB_TPL(0, 0, 0, 2)
    TB_TPL(1, 1, 0, 0) TB_TPL(1, 0, 1, 0) TB_TPL(1, 0, 0, 1) TB_TPL(0, 1, 1, 0) TB_TPL(0, 1, 0, 1) TB_TPL(0, 0, 1, 1)
#endif
#if TB_S1_TPL_MAXL >= 3
    TB_TPL(3, 0, 0, 0) TB_TPL(0, 3, 0, 0) TB_TPL(0, 0, 3, 0) TB_TPL(0, 0, 0, 3)
    TB_TPL(2, 1, 0, 0) TB_TPL(2, 0, 1, 0) TB_TPL(2, 0, 0, 1) TB_TPL(1, 2, 0, 0) TB_TPL(0, 2, 1, 0) TB_TPL(0, 2, 0, 1)
    TB_TPL(1, 0, 2, 0) TB_TPL(0, 1, 2, 0) TB_TPL(0, 0, 2, 1) TB_TPL(1, 0, 0, 2) TB_TPL(0, 1, 0, 2) TB_TPL(0, 0, 1, 2)
    TB_TPL(1, 1, 1, 0) TB_TPL(1, 1, 0, 1) TB_TPL(1, 0, 1, 1) TB_TPL(0, 1, 1, 1)
#endif
    default: break;
  }
#undef TB_TPL
  return cudaErrorInvalidValue;
}

template <int K>
cudaError_t launch_stage1_tpl_batch_k(int tuple, const Stage1Args *d, const int64_t *pre, int n, int64_t blocks,
                                      cudaStream_t st) {
  if (n <= 0 || blocks <= 0) return cudaSuccess;
#define TB_TPL(i, j, k, r)                                                                           \
  case ((i * 5 + j) * 5 + k) * 5 + r: {                                                            \
    const size_t smem = (size_t)ntuv(i + j + k + r) * sizeof(double) * 128;                        \
    cudaError_t e = cudaFuncSetAttribute(stage1_tpl_batch<i, j, k, r, K>,                          \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
    if (e != cudaSuccess) return e;                                                                \
    stage1_tpl_batch<i, j, k, r, K><<<(unsigned)blocks, 128, smem, st>>>(d, pre, n);               \
    return cudaGetLastError();                                                                     \
  }
  switch (tuple) {
    TB_TPL(0, 0, 0, 0)
    TB_TPL(1, 0, 0, 0) TB_TPL(0, 1, 0, 0) TB_TPL(0, 0, 1, 0) TB_TPL(0, 0, 0, 1)
#if TB_S1_TPL_MAXL >= 2
    TB_TPL(2, 0, 0, 0) TB_TPL(0, 2, 0, 0) TB_TPL(0, 0, 2, 0) TB_TPL(0, 0, 0, 2)
    TB_TPL(1, 1, 0, 0) TB_TPL(1, 0, 1, 0) TB_TPL(1, 0, 0, 1) TB_TPL(0, 1, 1, 0) TB_TPL(0, 1, 0, 1) TB_TPL(0, 0, 1, 1)
#endif
#if TB_S1_TPL_MAXL >= 3
    TB_TPL(3, 0, 0, 0) TB_TPL(0, 3, 0, 0) TB_TPL(0, 0, 3, 0) TB_TPL(0, 0, 0, 3)
    TB_TPL(2, 1, 0, 0) TB_TPL(2, 0, 1, 0) TB_TPL(2, 0, 0, 1) TB_TPL(1, 2, 0, 0) TB_TPL(0, 2, 1, 0) TB_TPL(0, 2, 0, 1)
    TB_TPL(1, 0, 2, 0) TB_TPL(0, 1, 2, 0) TB_TPL(0, 0, 2, 1) TB_TPL(1, 0, 0, 2) TB_TPL(0, 1, 0, 2) TB_TPL(0, 0, 1, 2)
    TB_TPL(1, 1, 1, 0) TB_TPL(1, 1, 0, 1) TB_TPL(1, 0, 1, 1) TB_TPL(0, 1, 1, 1)
#endif
    default: break;
  }
#undef TB_TPL
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// shared-memory kernel (LLmax 9..16)
// ---------------------------------------------------------------------------
template <int L, int KIND>
__device__ __forceinline__ void stage1_smem_body(Stage1Args &A, int64_t vb) {
  // Each thread owns a column of the block's shared array; element k of its
  // (partial) Hermite density sits at sD[k * blockDim.x + threadIdx.x].
  constexpr int S = stage1_smem_split(L);
  extern __shared__ double sD[];
  const int nthr = blockDim.x;
  const int sub = threadIdx.x % S;
  const int lane = threadIdx.x & 31;
  const unsigned gmask = S == 32 ? 0xffffffffu : (((1u << S) - 1u) << (lane - sub));
  const int64_t qi = A.qbegin + (vb * blockDim.x + threadIdx.x) / S;
  if (qi >= A.qend) return;
  double *D = sD + threadIdx.x;
  const QuartetHead Q = quartet_head<KIND>(A, qi);
  const int skip = Q.skip;

  constexpr int NT = ntuv(L);
  for (int k = 0; k < NT; ++k) D[k * nthr] = 0.0;

  const int si = A.gstart[Q.gi], ni = A.gcount[Q.gi];
  const int sj = A.gstart[Q.gj], nj = A.gcount[Q.gj];
  const int sk = A.gstart[Q.gk], nk = A.gcount[Q.gk];
  const int sr = A.gstart[Q.gr], nr = A.gcount[Q.gr];
  const double *Eb = Q.tb + 8, *Ek = Q.tk + 8;
  const int nket = nk * nr, nprim = ni * nj * nket;
  int cur_ab = -1;
  double bx[L + 1], by[L + 1], bz[L + 1];
  int nx1 = 0, ny1 = 0, nz1 = 0;
  int64_t rowp = 0;
  double zab = 0.0;
  for (int pidx = sub; pidx < nprim; pidx += S) {
    const int ab = pidx / nket, cd = pidx - ab * nket;
    if (ab != cur_ab) {
      cur_ab = ab;
      const int fa = si + ab / nj, fb = sj + ab % nj;
      const int la = A.flmn[fa], lb = A.flmn[fb];
      rowp = kind_elastic(KIND) ? 0 : fpair(min(fa, fb), max(fa, fb)) * A.np;
      zab = kind_elastic(KIND) ? A.zao[(size_t)fa * A.ngto + fb] : 0.0;
      const int lx1 = la & 0xff, ly1 = (la >> 8) & 0xff, lz1 = (la >> 16) & 0xff;
      const int lx2 = lb & 0xff, ly2 = (lb >> 8) & 0xff, lz2 = (lb >> 16) & 0xff;
      nx1 = lx1 + lx2;
      ny1 = ly1 + ly2;
      nz1 = lz1 + lz2;
      const double *ex = Eb + 0 * ESZ + (lx1 * (MAXA + 1) + lx2) * E_T;
      const double *ey = Eb + 1 * ESZ + (ly1 * (MAXA + 1) + ly2) * E_T;
      const double *ez = Eb + 2 * ESZ + (lz1 * (MAXA + 1) + lz2) * E_T;
#pragma unroll
      for (int t = 0; t <= L; ++t) {
        double vx = t <= nx1 ? ex[t] : 0.0, vy = t <= ny1 ? ey[t] : 0.0, vz = t <= nz1 ? ez[t] : 0.0;
        if ((skip & 1) && fabs(vx) < TB_SKIP30) vx = 0.0;
        if ((skip & 2) && fabs(vy) < TB_SKIP30) vy = 0.0;
        if ((skip & 4) && fabs(vz) < TB_SKIP30) vz = 0.0;
        bx[t] = (t & 1) ? -vx : vx;
        by[t] = (t & 1) ? -vy : vy;
        bz[t] = (t & 1) ? -vz : vz;
      }
    }
    const int fc = sk + cd / nr, fd = sr + cd % nr;
    double ztot;
    if (kind_elastic(KIND)) ztot = A.zket[(size_t)fc * A.ngto + fd] * zab;
    else ztot = A.rho[rowp + fpair(min(fc, fd), max(fc, fd))];
    if (fabs(ztot) < A.cutoffz) continue;
    const int lc = A.flmn[fc], ld = A.flmn[fd];
    const int lx3 = lc & 0xff, ly3 = (lc >> 8) & 0xff, lz3 = (lc >> 16) & 0xff;
    const int lx4 = ld & 0xff, ly4 = (ld >> 8) & 0xff, lz4 = (ld >> 16) & 0xff;
    const int nx2 = lx3 + lx4, ny2 = ly3 + ly4, nz2 = lz3 + lz4;
    const double *ex = Ek + 0 * ESZ + (lx3 * (MAXA + 1) + lx4) * E_T;
    const double *ey = Ek + 1 * ESZ + (ly3 * (MAXA + 1) + ly4) * E_T;
    const double *ez = Ek + 2 * ESZ + (lz3 * (MAXA + 1) + lz4) * E_T;
    double cx[L + 1], cy[L + 1], cz[L + 1];
    const int nx = nx1 + nx2, ny = ny1 + ny2, nz = nz1 + nz2;
    for (int T = 0; T <= nx; ++T) {
      double acc = 0.0;
      for (int t = max(0, T - nx2); t <= min(T, nx1); ++t) {
        double e = ex[T - t];
        if ((skip & 8) && fabs(e) < TB_SKIP30) e = 0.0;
        acc = fma(bx[t], e, acc);
      }
      cx[T] = acc * ztot;
    }
    for (int U = 0; U <= ny; ++U) {
      double acc = 0.0;
      for (int u = max(0, U - ny2); u <= min(U, ny1); ++u) {
        double e = ey[U - u];
        if ((skip & 16) && fabs(e) < TB_SKIP30) e = 0.0;
        acc = fma(by[u], e, acc);
      }
      cy[U] = acc;
    }
    for (int V = 0; V <= nz; ++V) {
      double acc = 0.0;
      for (int v = max(0, V - nz2); v <= min(V, nz1); ++v) acc = fma(bz[v], ez[V - v], acc);
      cz[V] = acc;
    }
    for (int T = 0; T <= nx; ++T) {
      const int baseT = ntuv(L) - ntuv(L - T);
      for (int U = 0; U <= ny; ++U) {
        const double w = cx[T] * cy[U];
        double *row = D + (baseT + U * (L - T + 1) - (U * (U - 1)) / 2) * nthr;
        for (int V = 0; V <= nz; ++V) row[V * nthr] = fma(w, cz[V], row[V * nthr]);
      }
    }
  }
  // fixed-order sum of the S partial densities into the group's first column
  __syncwarp(gmask);
  const int base = threadIdx.x - sub;
  for (int k = sub; k < NT; k += S) {
    double t = 0.0;
    for (int j = 0; j < S; ++j) t += sD[k * nthr + base + j];
    sD[k * nthr + base] = t;
  }
  __syncwarp(gmask);
  stage1_finish<L, KIND, S>(A, Q, sD + base, nthr, qi, sub, gmask);
}

template <int L, int KIND>
__global__ void stage1_smem_kernel(Stage1Args A) {
  stage1_geometry(A);
  stage1_smem_body<L, KIND>(A, blockIdx.x);
}

template <int L, int KIND>
__global__ void stage1_smem_batch(const Stage1Args *__restrict__ d, const int64_t *__restrict__ pre, int n) {
  const int it = batch_item(pre, n, blockIdx.x);
  Stage1Args A = d[it];
  stage1_smem_body<L, KIND>(A, blockIdx.x - pre[it]);
}

// ---------------------------------------------------------------------------
// contracted-side kernel (LLmax 4..6), thread per quartet
// ---------------------------------------------------------------------------
// The quartets of one launch share LK = min(L_bra, L_ket) and which side it
// is (XB: the bra).  That side is contracted with the pair density first,
//   X_o(t'u'v') = sum_c rho(o, c) E_c^x(t') E_c^y(u') E_c^z(v')   (o on the other side),
// and its Hermite box then convolved once per function pair of the other side,
//   D(T U V) += sum B_o(t u v) X_o(T-t, U-u, V-v),
// every shape compile-time (the other side has order L - LK), so a function
// quartet costs ntuv(LK) FMAs instead of the three zero-padded convolutions
// and the outer product of stage1_reg_kernel.

// The function pairs of a quartet's two sides, and the outer pair o's
// functions: (fa, fb) on the bra (XB false) or (fc, fd) on the ket (XB true).
struct XkSides {
  int si, ni, sj, nj, sk, nk, sr, nr, pb, pk, nout, nin;
};

template <bool XB>
__device__ __forceinline__ XkSides xk_sides(const Stage1Args &A, const QuartetHead &Q) {
  XkSides S;
  S.pb = pair_index(Q.gi, Q.gj, A.ng);
  S.pk = pair_index(Q.gk, Q.gr, A.ng);
  S.si = A.gstart[Q.gi]; S.ni = A.gcount[Q.gi];
  S.sj = A.gstart[Q.gj]; S.nj = A.gcount[Q.gj];
  S.sk = A.gstart[Q.gk]; S.nk = A.gcount[Q.gk];
  S.sr = A.gstart[Q.gr]; S.nr = A.gcount[Q.gr];
  const int nab = S.ni * S.nj, ncd = S.nk * S.nr;
  S.nout = XB ? ncd : nab;
  S.nin = XB ? nab : ncd;
  return S;
}

// Outer pair o's E coefficients (order LO), with the bra's (-1)^t sign of
// src/Integrals.f90:5181 when the outer side is the bra.
template <int LO, bool XB>
__device__ __forceinline__ void xk_outer(const Stage1Args &A, const QuartetHead &Q, const XkSides &S, int o, int &fa,
                                         int &fb, int &fc, int &fd, double *ox, double *oy, double *oz) {
  if (XB) { fc = S.sk + o / S.nr; fd = S.sr + o % S.nr; fa = fb = 0; }
  else { fa = S.si + o / S.nj; fb = S.sj + o % S.nj; fc = fd = 0; }
  if (ox == nullptr) return;
  const int64_t np = A.npair;
  const int l1 = XB ? A.flmn[fc] : A.flmn[fa], l2 = XB ? A.flmn[fd] : A.flmn[fb];
  const int pr = XB ? S.pk : S.pb;
  const double *ex = esoa_slot(A, XB ? (Q.skip & 8) : (Q.skip & 1), 0, l1 & 0xff, l2 & 0xff, pr);
  const double *ey = esoa_slot(A, XB ? (Q.skip & 16) : (Q.skip & 2), 1, (l1 >> 8) & 0xff, (l2 >> 8) & 0xff, pr);
  const double *ez = esoa_slot(A, XB ? false : (Q.skip & 4), 2, (l1 >> 16) & 0xff, (l2 >> 16) & 0xff, pr);
#pragma unroll
  for (int t = 0; t <= LO; ++t) {
    const double sg = (!XB && (t & 1)) ? -1.0 : 1.0;
    ox[t] = sg * ex[t * np];
    oy[t] = sg * ey[t * np];
    oz[t] = sg * ez[t * np];
  }
}

// X_o over the contracted side's function pairs c:
//   X_o(t'u'v') = sum_c rho(o, c) E_c^x(t') E_c^y(u') E_c^z(v')
template <int LK, int KIND, bool XB>
__device__ __forceinline__ void xk_contract(const Stage1Args &A, const QuartetHead &Q, const XkSides &S, int fa,
                                            int fb, int fc, int fd, double *X) {
  constexpr int NX = ntuv(LK);
  const int64_t np = A.npair;
#pragma unroll
  for (int e = 0; e < NX; ++e) X[e] = 0.0;
  int64_t rowp = 0;
  double zo = 0.0;
  if (!XB) {
    rowp = kind_elastic(KIND) ? 0 : fpair(min(fa, fb), max(fa, fb)) * A.np;
    zo = kind_elastic(KIND) ? A.zao[(size_t)fa * A.ngto + fb] : 0.0;
  } else {
    zo = kind_elastic(KIND) ? A.zket[(size_t)fc * A.ngto + fd] : 0.0;
  }
  for (int c = 0; c < S.nin; ++c) {
    int ga, gb2, gc, gd;
    if (XB) { ga = S.si + c / S.nj; gb2 = S.sj + c % S.nj; gc = fc; gd = fd; }
    else { gc = S.sk + c / S.nr; gd = S.sr + c % S.nr; ga = fa; gb2 = fb; }
    double z;
    if (kind_elastic(KIND)) z = (XB ? A.zao : A.zket)[(size_t)(XB ? ga : gc) * A.ngto + (XB ? gb2 : gd)] * zo;
    else {
      const int64_t rp = XB ? fpair(min(ga, gb2), max(ga, gb2)) * A.np : rowp;
      z = A.rho[rp + fpair(min(gc, gd), max(gc, gd))];
    }
    // the reference skips primitive quartets with |ztot| < cutoffz
    z = fabs(z) < A.cutoffz ? 0.0 : z;
    const int l1 = XB ? A.flmn[ga] : A.flmn[gc], l2 = XB ? A.flmn[gb2] : A.flmn[gd];
    const int pr = XB ? S.pb : S.pk;
    const double *ex = esoa_slot(A, XB ? (Q.skip & 1) : (Q.skip & 8), 0, l1 & 0xff, l2 & 0xff, pr);
    const double *ey = esoa_slot(A, XB ? (Q.skip & 2) : (Q.skip & 16), 1, (l1 >> 8) & 0xff, (l2 >> 8) & 0xff, pr);
    const double *ez = esoa_slot(A, XB ? (Q.skip & 4) : false, 2, (l1 >> 16) & 0xff, (l2 >> 16) & 0xff, pr);
    double cx[LK + 1], cy[LK + 1], cz[LK + 1];
#pragma unroll
    for (int t = 0; t <= LK; ++t) {
      const double sg = (XB && (t & 1)) ? -1.0 : 1.0;
      cx[t] = sg * ex[t * np];
      cy[t] = sg * ey[t * np];
      cz[t] = sg * ez[t * np];
    }
    int e = 0;
#pragma unroll
    for (int t = 0; t <= LK; ++t) {
      const double w1 = z * cx[t];
#pragma unroll
      for (int u = 0; u <= LK - t; ++u) {
        const double w2 = w1 * cy[u];
#pragma unroll
        for (int v = 0; v <= LK - t - u; ++v, ++e) X[e] = fma(w2, cz[v], X[e]);
      }
    }
  }
}

// D += O (x) X over the two simplices
template <int L, int LK>
__device__ __forceinline__ void xk_convolve(double *D, const double *ox, const double *oy, const double *oz,
                                            const double *X) {
  constexpr int LO = L - LK;
#pragma unroll
  for (int t = 0; t <= LO; ++t)
#pragma unroll
    for (int u = 0; u <= LO - t; ++u) {
      const double oxy = ox[t] * oy[u];
#pragma unroll
      for (int v = 0; v <= LO - t - u; ++v) {
        const double b = oxy * oz[v];
        int e = 0;
#pragma unroll
        for (int t2 = 0; t2 <= LK; ++t2)
#pragma unroll
          for (int u2 = 0; u2 <= LK - t2; ++u2)
#pragma unroll
            for (int v2 = 0; v2 <= LK - t2 - u2; ++v2, ++e) {
              const int k = dindex<L>(t + t2, u + u2, v + v2);
              D[k] = fma(b, X[e], D[k]);
            }
      }
    }
}

// Fused form: a thread per quartet, contraction and convolution per outer
// pair (geometry and molecule batches).  With xbuf given, X_o is read from
// the contraction kernel's buffer instead (stage1_xc_kernel, row stride
// xstride doubles per quartet).
template <int L, int KIND, int LK, bool XB>
__device__ __forceinline__ void stage1_xk_body(Stage1Args &A, int64_t vb, const double *__restrict__ xbuf = nullptr,
                                               int xstride = 0) {
  constexpr int LO = L - LK;  // order of the convolved (outer) side
  constexpr int NT = ntuv(L), NX = ntuv(LK);
  constexpr int NG = 128;
  extern __shared__ double sD[];
  const int64_t qi = A.qbegin + vb * blockDim.x + threadIdx.x;
  if (qi >= A.qend) return;
  const QuartetHead Q = quartet_head<KIND>(A, qi);
  const XkSides S = xk_sides<XB>(A, Q);
  double D[NT];
#pragma unroll
  for (int e = 0; e < NT; ++e) D[e] = 0.0;
  const double *xq = xbuf ? xbuf + (qi - A.qbegin) * (int64_t)xstride : nullptr;
  for (int o = 0; o < S.nout; ++o) {
    int fa, fb, fc, fd;
    double ox[LO + 1], oy[LO + 1], oz[LO + 1];
    xk_outer<LO, XB>(A, Q, S, o, fa, fb, fc, fd, ox, oy, oz);
    double X[NX];
    if (xq) {
#pragma unroll
      for (int e = 0; e < NX; ++e) X[e] = xq[o * NX + e];
    } else {
      xk_contract<LK, KIND, XB>(A, Q, S, fa, fb, fc, fd, X);
    }
    xk_convolve<L, LK>(D, ox, oy, oz, X);
  }
  double *col = sD + threadIdx.x;
#pragma unroll
  for (int k = 0; k < NT; ++k) col[k * NG] = D[k];
  stage1_finish<L, KIND, 1>(A, Q, col, NG, qi, 0, 0xffffffffu);
}

// Contraction alone, at high occupancy: G threads per quartet (G a power of
// two >= its outer pairs), thread o computing X_o; the G threads of a quartet
// read the same inner-pair coefficients (one transaction per warp).  X_o goes
// to xbuf[(qi - qbegin) * xstride + o * NX + e].
template <int L, int KIND, int LK, bool XB>
__device__ __forceinline__ void stage1_xc_body(const Stage1Args &A, int64_t t, double *__restrict__ xbuf, int G,
                                               int xstride) {
  constexpr int NX = ntuv(LK);
  const int64_t qi = A.qbegin + t / G;
  const int o = (int)(t % G);
  if (qi >= A.qend) return;
  const QuartetHead Q = quartet_head<KIND>(A, qi);
  const XkSides S = xk_sides<XB>(A, Q);
  if (o >= S.nout) return;
  int fa, fb, fc, fd;
  xk_outer<L - LK, XB>(A, Q, S, o, fa, fb, fc, fd, nullptr, nullptr, nullptr);
  double X[NX];
  xk_contract<LK, KIND, XB>(A, Q, S, fa, fb, fc, fd, X);
  double *xo = xbuf + (qi - A.qbegin) * (int64_t)xstride + o * NX;
#pragma unroll
  for (int e = 0; e < NX; ++e) xo[e] = X[e];
}

template <int L, int KIND, int LK, bool XB>
__global__ void __launch_bounds__(128) stage1_xc_kernel(Stage1Args A, double *__restrict__ xbuf, int G, int xstride) {
  stage1_xc_body<L, KIND, LK, XB>(A, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, xbuf, G, xstride);
}

// Shell-templated contraction (total j0, contracted side LK <= 3, plans with
// canonical shells): stage1_xc_body's arithmetic for one pair of inner shells
// (L1, L2) -- the inner function pairs and their Cartesian exponents are
// compile-time, so the density and E loads of a thread are independent of
// each other and issued ahead of the products.  X_o goes to
// xbuf[(qi - xbase) xstride + o NX + e] like stage1_xc_body's.
template <int L1, int L2, bool XB, int KIND>
__device__ __forceinline__ void stage1_xct_body(const Stage1Args &A, int64_t t, double *__restrict__ xbuf, int G,
                                                int xstride, int64_t xbase) {
  constexpr int LK = L1 + L2, NX = ntuv(LK);
  constexpr int n1 = (L1 + 1) * (L1 + 2) / 2, n2 = (L2 + 1) * (L2 + 2) / 2;
  const int64_t qi = A.qbegin + t / G;
  const int o = (int)(t % G);
  if (qi >= A.qend) return;
  const QuartetHead Q = quartet_head<KIND>(A, qi);
  const XkSides S = xk_sides<XB>(A, Q);
  if (o >= S.nout) return;
  int fa, fb, fc, fd;
  xk_outer<0, XB>(A, Q, S, o, fa, fb, fc, fd, nullptr, nullptr, nullptr);
  const int s1 = XB ? S.si : S.sk, s2 = XB ? S.sj : S.sr;
  const double *tab = A.pairtab + (size_t)(XB ? S.pb : S.pk) * PAIR_STRIDE + 8;
  const bool skx = XB ? (Q.skip & 1) : (Q.skip & 8), sky = XB ? (Q.skip & 2) : (Q.skip & 16);
  const bool skz = XB ? (Q.skip & 4) : false;
  auto ecoef = [&](int ax, int l1, int l2, int tt, bool skip) -> double {
    const double v = tab[ax * ESZ + (l1 * (MAXA + 1) + l2) * E_T + tt];
    return (skip && fabs(v) < TB_SKIP30) ? 0.0 : v;
  };
  int64_t rowp = 0;
  double zo = 0.0;
  if (!XB) {
    rowp = kind_elastic(KIND) ? 0 : fpair(min(fa, fb), max(fa, fb)) * A.np;
    zo = kind_elastic(KIND) ? A.zao[(size_t)fa * A.ngto + fb] : 0.0;
  } else {
    zo = kind_elastic(KIND) ? A.zket[(size_t)fc * A.ngto + fd] : 0.0;
  }
  double X[NX];
#pragma unroll
  for (int e = 0; e < NX; ++e) X[e] = 0.0;
#pragma unroll
  for (int c1 = 0; c1 < n1; ++c1)
#pragma unroll
    for (int c2 = 0; c2 < n2; ++c2) {
      const int g1 = s1 + c1, g2 = s2 + c2;  // (ga, gb2) on the bra side, (gc, gd) on the ket side
      double z;
      if (kind_elastic(KIND)) {
        z = (XB ? A.zao : A.zket)[(size_t)g1 * A.ngto + g2] * zo;
      } else {
        const int64_t rp = XB ? fpair(min(g1, g2), max(g1, g2)) * A.np : rowp;
        z = XB ? A.rho[rp + fpair(min(fc, fd), max(fc, fd))] : A.rho[rp + fpair(min(g1, g2), max(g1, g2))];
      }
      // the reference skips primitive quartets with |ztot| < cutoffz
      z = fabs(z) < A.cutoffz ? 0.0 : z;
      const int x1 = cart_component(L1, c1, 0), x2 = cart_component(L2, c2, 0);
      const int y1 = cart_component(L1, c1, 1), y2 = cart_component(L2, c2, 1);
      const int z1 = cart_component(L1, c1, 2), z2 = cart_component(L2, c2, 2);
      double cx[LK + 1], cy[LK + 1], cz[LK + 1];
#pragma unroll
      for (int tt = 0; tt <= LK; ++tt) {
        const double sg = (XB && (tt & 1)) ? -1.0 : 1.0;
        cx[tt] = sg * (tt <= x1 + x2 ? ecoef(0, x1, x2, tt, skx) : 0.0);
        cy[tt] = sg * (tt <= y1 + y2 ? ecoef(1, y1, y2, tt, sky) : 0.0);
        cz[tt] = sg * (tt <= z1 + z2 ? ecoef(2, z1, z2, tt, skz) : 0.0);
      }
      int e = 0;
#pragma unroll
      for (int tt = 0; tt <= LK; ++tt) {
        const double w1 = z * cx[tt];
#pragma unroll
        for (int u = 0; u <= LK - tt; ++u) {
          const double w2 = w1 * cy[u];
#pragma unroll
          for (int v = 0; v <= LK - tt - u; ++v, ++e) X[e] = fma(w2, cz[v], X[e]);
        }
      }
    }
  double *xo = xbuf + (qi - xbase) * (int64_t)xstride + o * NX;
#pragma unroll
  for (int e = 0; e < NX; ++e) xo[e] = X[e];
}

template <int L1, int L2, bool XB, int KIND>
__global__ void __launch_bounds__(128) stage1_xct_kernel(Stage1Args A, double *__restrict__ xbuf, int G, int xstride,
                                                         int64_t xbase) {
  stage1_xct_body<L1, L2, XB, KIND>(A, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, xbuf, G, xstride, xbase);
}

// Molecule batches: item i (one plan's quartets of one shell tuple inside a
// split sub-range) owns blocks pre[i] .. pre[i+1]-1; its X rows start A.xoff
// doubles into the batch's buffer at its first quartet.
template <int L1, int L2, bool XB, int KIND>
__global__ void __launch_bounds__(128)
    stage1_xct_batch(const Stage1Args *__restrict__ d, const int64_t *__restrict__ pre, int n,
                     double *__restrict__ xbuf) {
  const int it = batch_item(pre, n, blockIdx.x);
  const Stage1Args A = d[it];
  stage1_xct_body<L1, L2, XB, KIND>(A, (blockIdx.x - pre[it]) * blockDim.x + threadIdx.x, xbuf + A.xoff, A.xg,
                                    A.xstride, A.qbegin);
}

// One launch per shell tuple ((Li 5 + Lj) 5 + Lk) 5 + Lr: its inner shells
// are (Li, Lj) when the bra is the contracted side (XB), else (Lk, Lr).
template <int K>
cudaError_t launch_stage1_xct_k(int tuple, bool XB, const Stage1Args &a, double *xbuf, int xstride, int64_t xbase,
                                cudaStream_t st) {
  const int64_t n = a.qend - a.qbegin;
  if (n <= 0) return cudaSuccess;
  const int Li = tuple / 125, Lj = (tuple / 25) % 5, Lk = (tuple / 5) % 5, Lr = tuple % 5;
  const int L1 = XB ? Li : Lk, L2 = XB ? Lj : Lr;
  const int Lo1 = XB ? Lk : Li, Lo2 = XB ? Lr : Lj;
  const int nout = (Lo1 + 1) * (Lo1 + 2) / 2 * ((Lo2 + 1) * (Lo2 + 2) / 2);
  int G = 1;
  while (G < nout) G *= 2;
  const int64_t nthr = n * G;
  const unsigned grid = (unsigned)((nthr + 127) / 128);
#define TB_XCT(l1, l2)                                                                          \
  if (L1 == l1 && L2 == l2) {                                                                  \
    if (XB) stage1_xct_kernel<l1, l2, true, K><<<grid, 128, 0, st>>>(a, xbuf, G, xstride, xbase);  \
    else stage1_xct_kernel<l1, l2, false, K><<<grid, 128, 0, st>>>(a, xbuf, G, xstride, xbase);    \
    return cudaGetLastError();                                                                 \
  }
  TB_XCT(0, 0)
  TB_XCT(1, 0) TB_XCT(0, 1)
  TB_XCT(2, 0) TB_XCT(1, 1) TB_XCT(0, 2)
  TB_XCT(3, 0) TB_XCT(2, 1) TB_XCT(1, 2) TB_XCT(0, 3)
#undef TB_XCT
  return cudaErrorInvalidValue;
}

template <int K>
cudaError_t launch_stage1_xct_batch_k(int tuple, bool XB, const Stage1Args *d, const int64_t *pre, int n,
                                      int64_t blocks, double *xbuf, cudaStream_t st) {
  if (n <= 0 || blocks <= 0) return cudaSuccess;
  const int Li = tuple / 125, Lj = (tuple / 25) % 5, Lk = (tuple / 5) % 5, Lr = tuple % 5;
  const int L1 = XB ? Li : Lk, L2 = XB ? Lj : Lr;
#define TB_XCT(l1, l2)                                                                             \
  if (L1 == l1 && L2 == l2) {                                                                     \
    if (XB) stage1_xct_batch<l1, l2, true, K><<<(unsigned)blocks, 128, 0, st>>>(d, pre, n, xbuf);  \
    else stage1_xct_batch<l1, l2, false, K><<<(unsigned)blocks, 128, 0, st>>>(d, pre, n, xbuf);    \
    return cudaGetLastError();                                                                    \
  }
  TB_XCT(0, 0)
  TB_XCT(1, 0) TB_XCT(0, 1)
  TB_XCT(2, 0) TB_XCT(1, 1) TB_XCT(0, 2)
  TB_XCT(3, 0) TB_XCT(2, 1) TB_XCT(1, 2) TB_XCT(0, 3)
#undef TB_XCT
  return cudaErrorInvalidValue;
}


// Molecule batches: item i's contraction threads in blocks prexc[i] ..
template <int L, int KIND, int LK, bool XB>
__global__ void __launch_bounds__(128)
    stage1_xc_batch(const Stage1Args *__restrict__ d, const int64_t *__restrict__ prexc, int n,
                    double *__restrict__ xbuf) {
  const int it = batch_item(prexc, n, blockIdx.x);
  const Stage1Args A = d[it];
  stage1_xc_body<L, KIND, LK, XB>(A, (blockIdx.x - prexc[it]) * blockDim.x + threadIdx.x, xbuf + A.xoff, A.xg,
                                  A.xstride);
}

// Convolution and epilogue from the contraction kernel's X.
template <int L, int KIND, int LK, bool XB>
__global__ void __launch_bounds__(128, 2) stage1_xb_kernel(Stage1Args A, const double *__restrict__ xbuf,
                                                           int xstride) {
  stage1_xk_body<L, KIND, LK, XB>(A, blockIdx.x, xbuf, xstride);
}

template <int L, int KIND, int LK, bool XB>
__global__ void __launch_bounds__(128, 2)
    stage1_xb_batch(const Stage1Args *__restrict__ d, const int64_t *__restrict__ pre, int n,
                    const double *__restrict__ xbuf) {
  const int it = batch_item(pre, n, blockIdx.x);
  Stage1Args A = d[it];
  stage1_xk_body<L, KIND, LK, XB>(A, blockIdx.x - pre[it], xbuf + A.xoff, A.xstride);
}

template <int L, int KIND, int LK, bool XB>
__global__ void __launch_bounds__(128, 2) stage1_xk_kernel(Stage1Args A) {
  stage1_geometry(A);
  stage1_xk_body<L, KIND, LK, XB>(A, blockIdx.x);
}

template <int L, int KIND, int LK, bool XB>
__global__ void __launch_bounds__(128, 2)
    stage1_xk_batch(const Stage1Args *__restrict__ d, const int64_t *__restrict__ pre, int n) {
  const int it = batch_item(pre, n, blockIdx.x);
  Stage1Args A = d[it];
  stage1_xk_body<L, KIND, LK, XB>(A, blockIdx.x - pre[it]);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// threads per block of the shared-memory kernel so that the Hermite densities
// of the block fit in 96 KB (2 blocks per SM)
static inline int stage1_smem_threads(int L) {
  int t = 128;
  while (t > stage1_smem_split(L) && (size_t)ntuv(L) * sizeof(double) * t > 96 * 1024) t /= 2;
  return t;
}

template <int L, int K>
static cudaError_t launch_stage1_l(const Stage1Args &a, int64_t n, int ngeom, cudaStream_t st) {
  if constexpr (L <= STAGE1_REG_MAXL) {
    constexpr int S = stage1_reg_split(L);
    const int thr = 128;
    size_t smem = (size_t)ntuv(L) * sizeof(double) * (thr / S);
    cudaError_t e =
        cudaFuncSetAttribute(stage1_reg_kernel<L, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int64_t threads = n * S * stage1_reg_parts(L);
    stage1_reg_kernel<L, K><<<dim3((unsigned)((threads + thr - 1) / thr), ngeom), thr, smem, st>>>(a);
  } else {
    constexpr int S = stage1_smem_split(L);
    int thr = stage1_smem_threads(L);
    size_t smem = (size_t)ntuv(L) * sizeof(double) * thr;
    cudaError_t e =
        cudaFuncSetAttribute(stage1_smem_kernel<L, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int64_t threads = n * S;
    stage1_smem_kernel<L, K><<<dim3((unsigned)((threads + thr - 1) / thr), ngeom), thr, smem, st>>>(a);
  }
  return cudaGetLastError();
}

template <int L, int K, int LK, bool XB>
static cudaError_t launch_stage1_xk_l(const Stage1Args &a, int64_t n, int ngeom, cudaStream_t st) {
  const int thr = 128;
  const size_t smem = (size_t)ntuv(L) * sizeof(double) * thr;
  cudaError_t e =
      cudaFuncSetAttribute(stage1_xk_kernel<L, K, LK, XB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  stage1_xk_kernel<L, K, LK, XB><<<dim3((unsigned)((n + thr - 1) / thr), ngeom), thr, smem, st>>>(a);
  return cudaGetLastError();
}

template <int K>
cudaError_t launch_stage1_xk_k(int L, int LK, bool XB, const Stage1Args &a, int ngeom, cudaStream_t st) {
  const int64_t n = a.qend - a.qbegin;
  if (n <= 0) return cudaSuccess;
#define TB_XK(l, lk)                                                                         \
  if (L == l && LK == lk)                                                                   \
    return XB ? launch_stage1_xk_l<l, K, lk, true>(a, n, ngeom, st)                         \
              : launch_stage1_xk_l<l, K, lk, false>(a, n, ngeom, st);
  TB_XK(3, 0) TB_XK(3, 1)
  TB_XK(4, 0) TB_XK(4, 1) TB_XK(4, 2)
  TB_XK(5, 0) TB_XK(5, 1) TB_XK(5, 2)
  TB_XK(6, 0) TB_XK(6, 1) TB_XK(6, 2) TB_XK(6, 3)
#if TB_S1_XK_HIGH
  TB_XK(7, 0) TB_XK(7, 1) TB_XK(7, 2) TB_XK(7, 3)
  TB_XK(8, 0) TB_XK(8, 1) TB_XK(8, 2) TB_XK(8, 3) TB_XK(8, 4)
#endif
#undef TB_XK
  return cudaErrorInvalidValue;
}

// Contracted-side classes of a single geometry in two kernels: the
// contraction into xbuf (G threads per quartet), then convolution + epilogue.
template <int L, int K, int LK, bool XB>
static cudaError_t launch_stage1_xsplit_l(const Stage1Args &a, int64_t n, double *xbuf, int nout, bool with_xc,
                                          cudaStream_t st) {
  int G = 1;
  while (G < nout) G *= 2;
  const int xstride = nout * ntuv(LK);
  const int64_t nthr = n * G;
  cudaError_t e = cudaSuccess;
  if (with_xc) {  // otherwise X was written by the shell-templated contraction
    stage1_xc_kernel<L, K, LK, XB><<<(unsigned)((nthr + 127) / 128), 128, 0, st>>>(a, xbuf, G, xstride);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const int thr = 128;
  const size_t smem = (size_t)ntuv(L) * sizeof(double) * thr;
  e = cudaFuncSetAttribute(stage1_xb_kernel<L, K, LK, XB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  stage1_xb_kernel<L, K, LK, XB><<<(unsigned)((n + thr - 1) / thr), thr, smem, st>>>(a, xbuf, xstride);
  return cudaGetLastError();
}

template <int K>
cudaError_t launch_stage1_xsplit_k(int L, int LK, bool XB, const Stage1Args &a, double *xbuf, int nout, bool with_xc,
                                   cudaStream_t st) {
  const int64_t n = a.qend - a.qbegin;
  if (n <= 0) return cudaSuccess;
#define TB_XS(l, lk)                                                                         \
  if (L == l && LK == lk)                                                                   \
    return XB ? launch_stage1_xsplit_l<l, K, lk, true>(a, n, xbuf, nout, with_xc, st)        \
              : launch_stage1_xsplit_l<l, K, lk, false>(a, n, xbuf, nout, with_xc, st);
  TB_XS(4, 0) TB_XS(4, 1) TB_XS(4, 2)
  TB_XS(5, 0) TB_XS(5, 1) TB_XS(5, 2)
  TB_XS(6, 0) TB_XS(6, 1) TB_XS(6, 2) TB_XS(6, 3)
#if TB_S1_XK_HIGH
  TB_XS(7, 0) TB_XS(7, 1) TB_XS(7, 2) TB_XS(7, 3)
  TB_XS(8, 0) TB_XS(8, 1) TB_XS(8, 2) TB_XS(8, 3) TB_XS(8, 4)
#endif
#undef TB_XS
  return cudaErrorInvalidValue;
}

template <int L, int K, int LK, bool XB>
static cudaError_t launch_stage1_xsplit_batch_l(const Stage1Args *d, const int64_t *prexc, int64_t blocksxc,
                                                const int64_t *pre, int64_t blocks, int n, double *xbuf,
                                                cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  if (blocksxc > 0) {  // otherwise X was written by the shell-templated contraction
    stage1_xc_batch<L, K, LK, XB><<<(unsigned)blocksxc, 128, 0, st>>>(d, prexc, n, xbuf);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const size_t smem = (size_t)ntuv(L) * sizeof(double) * 128;
  e = cudaFuncSetAttribute(stage1_xb_batch<L, K, LK, XB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  stage1_xb_batch<L, K, LK, XB><<<(unsigned)blocks, 128, smem, st>>>(d, pre, n, xbuf);
  return cudaGetLastError();
}

template <int K>
cudaError_t launch_stage1_xsplit_batch_k(int L, int LK, int XB, const Stage1Args *d, const int64_t *prexc,
                                         int64_t blocksxc, const int64_t *pre, int64_t blocks, int n, double *xbuf,
                                         cudaStream_t st) {
  if (n <= 0 || blocks <= 0) return cudaSuccess;
#define TB_XSB(l, lk)                                                                                   \
  if (L == l && LK == lk)                                                                             \
    return XB ? launch_stage1_xsplit_batch_l<l, K, lk, true>(d, prexc, blocksxc, pre, blocks, n, xbuf, st) \
              : launch_stage1_xsplit_batch_l<l, K, lk, false>(d, prexc, blocksxc, pre, blocks, n, xbuf, st);
  TB_XSB(4, 0) TB_XSB(4, 1) TB_XSB(4, 2)
  TB_XSB(5, 0) TB_XSB(5, 1) TB_XSB(5, 2)
  TB_XSB(6, 0) TB_XSB(6, 1) TB_XSB(6, 2) TB_XSB(6, 3)
#if TB_S1_XK_HIGH
  TB_XSB(7, 0) TB_XSB(7, 1) TB_XSB(7, 2) TB_XSB(7, 3)
  TB_XSB(8, 0) TB_XSB(8, 1) TB_XSB(8, 2) TB_XSB(8, 3) TB_XSB(8, 4)
#endif
#undef TB_XSB
  return cudaErrorInvalidValue;
}

// Molecule batches: one launch over every item (one plan's quartet range of
// class L, and for the contracted-side kernel of one (LK, XB)); item i owns
// blocks pre[i] .. pre[i+1]-1 (stage1_item_blocks of its quartets).
template <int L, int K>
static cudaError_t launch_stage1_batch_l(int LK, int XB, const Stage1Args *d, const int64_t *pre, int n,
                                         int64_t blocks, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  if constexpr (L >= 3 && L <= (TB_S1_XK_HIGH ? 8 : 6)) {
    if (LK >= 0) {
#define TB_XB(lk)                                                                                         \
  if constexpr (lk <= L / 2)                                                                            \
    if (LK == lk) {                                                                                     \
    const size_t smem = (size_t)ntuv(L) * sizeof(double) * 128;                                         \
    if (XB) {                                                                                           \
      e = cudaFuncSetAttribute(stage1_xk_batch<L, K, lk, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                               (int)smem);                                                              \
      if (e == cudaSuccess) stage1_xk_batch<L, K, lk, true><<<(unsigned)blocks, 128, smem, st>>>(d, pre, n); \
    } else {                                                                                            \
      e = cudaFuncSetAttribute(stage1_xk_batch<L, K, lk, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                               (int)smem);                                                              \
      if (e == cudaSuccess) stage1_xk_batch<L, K, lk, false><<<(unsigned)blocks, 128, smem, st>>>(d, pre, n); \
    }                                                                                                   \
    return e != cudaSuccess ? e : cudaGetLastError();                                                   \
  }
      TB_XB(0) TB_XB(1) TB_XB(2) TB_XB(3) TB_XB(4)
#undef TB_XB
      return cudaErrorInvalidValue;
    }
  }
  if constexpr (L <= STAGE1_REG_MAXL) {
    constexpr int S = stage1_reg_split(L);
    const size_t smem = (size_t)ntuv(L) * sizeof(double) * (128 / S);
    e = cudaFuncSetAttribute(stage1_reg_batch<L, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    stage1_reg_batch<L, K><<<(unsigned)blocks, 128, smem, st>>>(d, pre, n);
  } else {
    const int thr = stage1_smem_threads(L);
    const size_t smem = (size_t)ntuv(L) * sizeof(double) * thr;
    e = cudaFuncSetAttribute(stage1_smem_batch<L, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    stage1_smem_batch<L, K><<<(unsigned)blocks, thr, smem, st>>>(d, pre, n);
  }
  return cudaGetLastError();
}

template <int K>
cudaError_t launch_stage1_batch_k(int L, int LK, int XB, const Stage1Args *d, const int64_t *pre, int n,
                                  int64_t blocks, cudaStream_t st) {
  if (n <= 0 || blocks <= 0) return cudaSuccess;
  switch (L) {
#define TB_S1(l) case l: return launch_stage1_batch_l<l, K>(LK, XB, d, pre, n, blocks, st);
    TB_S1(0) TB_S1(1) TB_S1(2) TB_S1(3) TB_S1(4) TB_S1(5) TB_S1(6) TB_S1(7) TB_S1(8)
    TB_S1(9) TB_S1(10) TB_S1(11) TB_S1(12) TB_S1(13) TB_S1(14) TB_S1(15) TB_S1(16)
#undef TB_S1
    default: return cudaErrorInvalidValue;
  }
}

template <int K>
cudaError_t launch_stage1_k(int L, const Stage1Args &a, int ngeom, cudaStream_t st) {
  int64_t n = a.qend - a.qbegin;
  if (n <= 0) return cudaSuccess;
  switch (L) {
#define TB_S1(l) case l: return launch_stage1_l<l, K>(a, n, ngeom, st);
    TB_S1(0) TB_S1(1) TB_S1(2) TB_S1(3) TB_S1(4) TB_S1(5) TB_S1(6) TB_S1(7) TB_S1(8)
    TB_S1(9) TB_S1(10) TB_S1(11) TB_S1(12) TB_S1(13) TB_S1(14) TB_S1(15) TB_S1(16)
#undef TB_S1
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace tb
