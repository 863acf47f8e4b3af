// Nuclear-electron term of electron scattering (types 5 and 6): records of
// the (nucleus a, ordered group pair (i, k)) items of
// nuclei_electron_integration (src/Integrals.f90:2493-2596), integral_k_ij
// (:6192-6326) and integral_ij_pzero (:4865-4953):
//   Ine(q) = sum_a sum_(i,k) Zn_a F_ik(q; H = R_a - P_ik) e12(q, i, k),
// F_ik the Hermite expansion of the pair against the AO density Z of the
// 1-RDM.  Per item a thread forms the pair's Hermite density
//   D_TUV = sum_{f in i, f' in k} Z(f, f') (-1)^{T+U+V} E^x_T E^y_U E^z_V
// (E from the pair tables, |E| < 1e-30 zeroed as the reference skips them)
// and hands it to the quartet epilogue with the nucleus in the ket's place:
// weight Zn_a K_ik, Gaussian exponent 1/4p_ik, P = Q branch below
// cutoffcentre.  The records then go through the stage-2 class kernels.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_stage1.cuh"

namespace tb {

namespace {

// item: a | gi << 16 | gk << 40 (nucleus, ordered group pair)
template <int L>
__global__ void __launch_bounds__(128) nuclear_kernel(Stage1Args A, const uint64_t *__restrict__ items,
                                                      const double *__restrict__ nucrec) {
  constexpr int NT = ntuv(L);
  constexpr int NG = 128;
  extern __shared__ double sD[];
  const int64_t qi = A.qbegin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= A.qend) return;
  const uint64_t it = items[qi];
  const int a = (int)(it & 0xffff), gi = (int)((it >> 16) & 0xffffff), gk = (int)((it >> 40) & 0xffffff);
  const bool swap = gi > gk;  // the table holds the pair (min, max)
  const int pr = swap ? pair_index(gk, gi, A.ng) : pair_index(gi, gk, A.ng);
  QuartetHead Q;
  Q.gi = gi; Q.gj = gk; Q.gk = 0; Q.gr = 0;
  Q.loop = 5;  // weight 1
  Q.w = 1.0;
  Q.tb = A.pairtab + (size_t)pr * PAIR_STRIDE;
  Q.tk = nucrec + (size_t)a * 8;  // [R_a, 0, Zn_a, 0, ...]: ket prefactor Zn_a, no Gaussian
  Q.Hx = Q.tk[0] - Q.tb[0];
  Q.Hy = Q.tk[1] - Q.tb[1];
  Q.Hz = Q.tk[2] - Q.tb[2];
  Q.h = sqrt(Q.Hx * Q.Hx + Q.Hy * Q.Hy + Q.Hz * Q.Hz);
  Q.p0 = Q.h < A.cutoffcentre;
  Q.skip = 0x1f;
  double D[NT];
#pragma unroll
  for (int e = 0; e < NT; ++e) D[e] = 0.0;
  const int64_t np = A.npair;
  const int si = A.gstart[gi], ni = A.gcount[gi], sk = A.gstart[gk], nk = A.gcount[gk];
  for (int x = 0; x < ni; ++x)
    for (int y = 0; y < nk; ++y) {
      const int fi = si + x, fk = sk + y;
      const double z = A.zao[(size_t)fi * A.ngto + fk];
      const int l1 = A.flmn[swap ? fk : fi], l2 = A.flmn[swap ? fi : fk];
      const double *ex = esoa_slot(A, true, 0, l1 & 0xff, l2 & 0xff, pr);
      const double *ey = esoa_slot(A, true, 1, (l1 >> 8) & 0xff, (l2 >> 8) & 0xff, pr);
      const double *ez = esoa_slot(A, true, 2, (l1 >> 16) & 0xff, (l2 >> 16) & 0xff, pr);
      double cx[L + 1], cy[L + 1], cz[L + 1];
#pragma unroll
      for (int t = 0; t <= L; ++t) {
        const double sg = (t & 1) ? -1.0 : 1.0;  // (-1)^{ll+mm+nn}, one factor per axis
        cx[t] = sg * ex[t * np];
        cy[t] = sg * ey[t * np];
        cz[t] = sg * ez[t * np];
      }
      int e = 0;
#pragma unroll
      for (int t = 0; t <= L; ++t) {
        const double w1 = z * cx[t];
#pragma unroll
        for (int u = 0; u <= L - t; ++u) {
          const double w2 = w1 * cy[u];
#pragma unroll
          for (int v = 0; v <= L - t - u; ++v, ++e) D[e] = fma(w2, cz[v], D[e]);
        }
      }
    }
  double *col = sD + threadIdx.x;
#pragma unroll
  for (int k = 0; k < NT; ++k) col[k * NG] = D[k];
  stage1_finish<L, KIND_TOTAL, 1>(A, Q, col, NG, qi, 0, 0xffffffffu);
}

template <int L>
cudaError_t launch_nuclear_l(const Stage1Args &a, const uint64_t *items, const double *nucrec, cudaStream_t st) {
  const int64_t n = a.qend - a.qbegin;
  const size_t smem = (size_t)ntuv(L) * sizeof(double) * 128;
  cudaError_t e = cudaFuncSetAttribute(nuclear_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  nuclear_kernel<L><<<(unsigned)((n + 127) / 128), 128, smem, st>>>(a, items, nucrec);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_nuclear(int L, const Stage1Args &a, const uint64_t *items, const double *nucrec,
                           cudaStream_t st) {
  if (a.qend <= a.qbegin) return cudaSuccess;
  switch (L) {
#define TB_N(l) case l: return launch_nuclear_l<l>(a, items, nucrec, st);
    TB_N(0) TB_N(1) TB_N(2) TB_N(3) TB_N(4) TB_N(5) TB_N(6) TB_N(7) TB_N(8)
#undef TB_N
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace tb
