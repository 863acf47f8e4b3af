// Elastic aligned intensity (calculation type 4): the Fourier transform of
// the one-electron density on q vectors,
//   F(q) = sum over ordered group pairs (i, j) of e12(|q|, i, j) e^{i q.P_ij}
//          sum_{a in i, b in j} Z(a, b) sum_{tuv} E^x_t E^y_u E^z_v (i qx)^t (i qy)^u (i qz)^v
// (elastic_integration_alig, src/Integrals.f90:2366-2490, with
// integral_k_ijkr_alig, :6085-6190), and the intensity |F(q)|^2 of CASE(4)
// (src/main_calculation.f90:218-265).  The two orders of a pair (i, j),
// (j, i) give the same term (Z symmetric, E^{ab}_t of the product, P and e12
// symmetric), so the pairs i <= j are summed with weight 2 (1 on the
// diagonal).
//
// Two kernels: records (a thread per unordered group pair: P, 1/4p,
// weight x (pi_sp/p)^1.5 K, L, and the pair's Hermite density D_tuv with
// the reference's |E| < 1e-30 skips and its |term| > 1e-30 test on each
// product Z E E E, summed in the reference's order), then the q kernel (a
// thread per q vector, the records staged through shared memory in chunks;
// per record a nested complex Horner in i qz, i qy, i qx, the phase
// sincos(q.P) and the Gaussian exp(-q^2/4p)).  Records and sums run in a
// fixed order, so the result is deterministic.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_stage1.cuh"

namespace tb {

namespace {

constexpr int FF_LMAX = 2 * MAXA;  // la + lb <= 8
constexpr int FF_RS = 6 + (FF_LMAX + 1) * (FF_LMAX + 2) * (FF_LMAX + 3) / 6;  // [P, s, w, L, D...]
constexpr int FF_CHUNK = 32;  // records staged per round

// position of (t, u, v), t + u + v <= L, in a Hermite density of order L
// (the layout of dindex<L> with L a runtime value)
__device__ __forceinline__ int dindex_rt(int L, int t, int u, int v) {
  return ntuv(L) - ntuv(L - t) + u * (L - t + 1) - (u * (u - 1)) / 2 + v;
}

__global__ void __launch_bounds__(128) ff_records_kernel(Stage1Args A, double *__restrict__ rec) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.npair) return;
  int gi = 0, rem = (int)p;
  while (rem >= A.ng - gi) {
    rem -= A.ng - gi;
    ++gi;
  }
  const int gj = gi + rem;
  const double *tb = A.pairtab + (size_t)p * PAIR_STRIDE;
  const int si = A.gstart[gi], ni = A.gcount[gi], sj = A.gstart[gj], nj = A.gcount[gj];
  const int fl0 = A.flmn[si], fl1 = A.flmn[sj];
  const int L = (fl0 & 0xff) + ((fl0 >> 8) & 0xff) + ((fl0 >> 16) & 0xff) + (fl1 & 0xff) + ((fl1 >> 8) & 0xff) +
                ((fl1 >> 16) & 0xff);
  double *r = rec + p * FF_RS;
  r[0] = tb[0];
  r[1] = tb[1];
  r[2] = tb[2];
  r[3] = tb[5];                              // 1/4p
  r[4] = (gi == gj ? 1.0 : 2.0) * tb[4];     // weight x (pi_sp/p)^1.5 K
  r[5] = (double)L;
  double *D = r + 6;
  const int nt = ntuv(L);
  for (int e = 0; e < nt; ++e) D[e] = 0.0;
  const int64_t np = A.npair;
  for (int x = 0; x < ni; ++x)
    for (int y = 0; y < nj; ++y) {
      const int fa = si + x, fb = sj + y;
      const double z = A.zao[(size_t)fa * A.ngto + fb];
      const int la = A.flmn[fa], lb = A.flmn[fb];
      const int lx = (la & 0xff) + (lb & 0xff), ly = ((la >> 8) & 0xff) + ((lb >> 8) & 0xff);
      const int lz = ((la >> 16) & 0xff) + ((lb >> 16) & 0xff);
      const double *ex = esoa_slot(A, true, 0, la & 0xff, lb & 0xff, (int)p);
      const double *ey = esoa_slot(A, true, 1, (la >> 8) & 0xff, (lb >> 8) & 0xff, (int)p);
      const double *ez = esoa_slot(A, true, 2, (la >> 16) & 0xff, (lb >> 16) & 0xff, (int)p);
      for (int t = 0; t <= lx; ++t) {
        const double mdl = ex[t * np];
        if (mdl == 0.0) continue;  // |E| < 1e-30 is stored as zero
        const double p1 = mdl * z;
        for (int u = 0; u <= ly; ++u) {
          const double mdm = ey[u * np];
          if (mdm == 0.0) continue;
          const double p2 = mdm * p1;
          for (int v = 0; v <= lz; ++v) {
            const double mdn = ez[v * np];
            if (mdn == 0.0) continue;
            const double p3 = mdn * p2;
            if (!(fabs(p3) > TB_SKIP30)) continue;
            D[dindex_rt(L, t, u, v)] += p3;
          }
        }
      }
    }
}

// F(q) per q vector over all records: out_re / out_im, |F|^2 into out_abs2
__global__ void __launch_bounds__(128) ff_q_kernel(const double *__restrict__ rec, int64_t nrec,
                                                   const double *__restrict__ qv, int nq, double *__restrict__ out_re,
                                                   double *__restrict__ out_im, double *__restrict__ out_abs2) {
  __shared__ double sr[FF_CHUNK * FF_RS];
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = iq < nq;
  const double qx = act ? qv[3 * iq] : 0.0, qy = act ? qv[3 * iq + 1] : 0.0, qz = act ? qv[3 * iq + 2] : 0.0;
  const double q2 = qx * qx + qy * qy + qz * qz;
  double fr = 0.0, fi = 0.0;
  for (int64_t c0 = 0; c0 < nrec; c0 += FF_CHUNK) {
    const int nc = (int)(nrec - c0 < FF_CHUNK ? nrec - c0 : FF_CHUNK);
    __syncthreads();
    for (int e = threadIdx.x; e < nc * FF_RS; e += blockDim.x) sr[e] = rec[c0 * FF_RS + e];
    __syncthreads();
    if (!act) continue;
    for (int c = 0; c < nc; ++c) {
      const double *r = sr + c * FF_RS;
      const int L = (int)r[5];
      const double *D = r + 6;
      // h = sum_t (i qx)^t sum_u (i qy)^u sum_v D_tuv (i qz)^v, nested complex Horner
      double hr = 0.0, hi = 0.0;
      for (int t = L; t >= 0; --t) {
        double ur = 0.0, ui = 0.0;
        for (int u = L - t; u >= 0; --u) {
          double vr = 0.0, vi = 0.0;
          for (int v = L - t - u; v >= 0; --v) {
            const double a = -vi * qz, b = vr * qz;  // (vr + i vi) (i qz)
            vr = a + D[dindex_rt(L, t, u, v)];
            vi = b;
          }
          const double a = -ui * qy, b = ur * qy;
          ur = a + vr;
          ui = b + vi;
        }
        const double a = -hi * qx, b = hr * qx;
        hr = a + ur;
        hi = b + ui;
      }
      double sn, cs;
      sincos(qx * r[0] + qy * r[1] + qz * r[2], &sn, &cs);
      const double g = r[4] * exp(-q2 * r[3]);
      fr = fma(g, hr * cs - hi * sn, fr);
      fi = fma(g, hr * sn + hi * cs, fi);
    }
  }
  if (!act) return;
  out_re[iq] = fr;
  out_im[iq] = fi;
  out_abs2[iq] = fr * fr + fi * fi;
}

}  // namespace

int64_t form_factor_record_doubles(int64_t npair) { return npair * FF_RS; }

cudaError_t launch_form_factor(const Stage1Args &a, double *rec, const double *qv, int nq, double *out_re,
                               double *out_im, double *out_abs2, cudaStream_t st) {
  if (a.npair <= 0 || nq <= 0) return cudaSuccess;
  ff_records_kernel<<<(unsigned)((a.npair + 127) / 128), 128, 0, st>>>(a, rec);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  ff_q_kernel<<<(nq + 127) / 128, 128, 0, st>>>(rec, a.npair, qv, nq, out_re, out_im, out_abs2);
  return cudaGetLastError();
}

}  // namespace tb
