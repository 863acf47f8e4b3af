// The MO -> primitive transform of the densities (total / j2 pair density,
// elastic and resolved-CMS AO densities) on the device; part of the plan
// (tb_plan.cu).
#include "tb_plan_internal.h"

using namespace tb;

// ---------------------------------------------------------------------------
// density transform on the device
// ---------------------------------------------------------------------------
// rho(ab,cd) = 1/8 sum_t G_t [S12_t(ab) S34_t(cd) + S34_t(ab) S12_t(cd)],
// S12_t(ab) = C_{m1 a} C_{m2 b} + C_{m1 b} C_{m2 a}: the ztot of
// src/Integrals.f90:5163 for every pair of primitive pairs.  With
// Ghat[x][y][z][w] = G_t/8 summed over the eight placements of each row this
// is the 4-index transform rho = sum Ghat C_x,a C_y,b C_z,c C_w,d, run as
// four DGEMM passes: m4 -> d, m3 -> c (pack c<=d), m2 -> b, m1 -> a (a<=b).


int density_alloc(thistle_plan *P) {
  int rc = THISTLE_OK;
  const int n = P->nmo, ngto = P->ngto;
  const int64_t np = P->np, n2 = (int64_t)n * n, n3 = n2 * n, n4 = n3 * n;
  TB_TRY(dalloc(&P->d_C, (size_t)n * ngto, "MO coefficients"));
  if (kind_elastic(P->kind)) {
    const size_t nz = (size_t)P->nzao;
    TB_TRY(dalloc(&P->d_zao, nz * ngto * ngto, "AO density"));
    TB_TRY(dalloc(&P->d_D, nz * P->nmo1 * P->nmo1, "1-RDM"));
    TB_TRY(dalloc(&P->d_Ds, nz * P->nmo1 * P->nmo1, "1-RDM"));
    TB_TRY(dalloc(&P->d_Y, nz * P->nmo1 * ngto, "1-RDM x C"));
    TB_TRY(dalloc(&P->d_Ct, (size_t)n * transform_ct_width(ngto), "transform C^T"));
  } else {
    TB_TRY(dalloc(&P->d_rho, (size_t)(np * np), "pair density"));
    TB_TRY(dalloc(&P->d_mat, (size_t)P->nmat * 4, "2-RDM indices"));
    TB_TRY(dalloc(&P->d_tot, (size_t)P->nmat, "2-RDM values"));
    TB_TRY(dalloc(&P->d_G, (size_t)n4, "Ghat"));
    TB_TRY(dalloc(&P->d_T1, (size_t)(n3 * ngto), "transform T1"));
    TB_TRY(dalloc(&P->d_V, (size_t)(n2 * np), "transform V"));
    TB_TRY(dalloc(&P->d_T3, (size_t)((int64_t)n * ngto * np), "transform T3"));
    TB_TRY(dalloc(&P->d_Ct, (size_t)n * transform_ct_width(ngto), "transform C^T"));
    const int64_t m = std::max<int64_t>(8 * (int64_t)P->nmat, 1);
    TB_TRY(dalloc(&P->d_gk0, (size_t)m, "Ghat keys"));
    TB_TRY(dalloc(&P->d_gk1, (size_t)m, "Ghat keys"));
    TB_TRY(dalloc(&P->d_gv0, (size_t)m, "Ghat values"));
    TB_TRY(dalloc(&P->d_gv1, (size_t)m, "Ghat values"));
    P->gbits = 1;
    while (P->gbits < 31 && ((int64_t)1 << P->gbits) < n4) ++P->gbits;
    TB_TRYC(cub::DeviceRadixSort::SortPairs(nullptr, P->gsort_bytes, P->d_gk0, P->d_gk1, P->d_gv0, P->d_gv1,
                                            (int)m, 0, P->gbits, P->st));
    TB_TRY(dalloc((char **)&P->d_gsort_tmp, P->gsort_bytes, "Ghat sort scratch"));
  }
done:
  return rc;
}

int density_upload(thistle_plan *P, const double *mmod, const int32_t *mat, const double *total,
                          const double *onerdm) {
  TB_CK(cudaMemcpyAsync(P->d_C, mmod, sizeof(double) * (size_t)P->nmo * P->ngto, cudaMemcpyHostToDevice, P->st));
  if (kind_elastic(P->kind)) {
    TB_CK(cudaMemcpyAsync(P->d_D, onerdm, sizeof(double) * (size_t)P->nzao * P->nmo1 * P->nmo1,
                          cudaMemcpyHostToDevice, P->st));
  } else if (P->nmat > 0) {
    TB_CK(cudaMemcpyAsync(P->d_mat, mat, sizeof(int) * (size_t)P->nmat * 4, cudaMemcpyHostToDevice, P->st));
    TB_CK(cudaMemcpyAsync(P->d_tot, total, sizeof(double) * (size_t)P->nmat, cudaMemcpyHostToDevice, P->st));
  }
  return THISTLE_OK;
}

// Pair density (total, j2) or AO density (elastic) from the device-resident
// inputs, every GEMM pass on the FP64 tensor cores (tb_transform.cu).
int density_run(thistle_plan *P) {
  int rc = THISTLE_OK;
  const int n = P->nmo, ngto = P->ngto, cw = transform_ct_width(ngto);
  const int64_t np = P->np, n2 = (int64_t)n * n, n3 = n2 * n, n4 = n3 * n;
  TB_TRYC(launch_transform_ct(P->d_C, n, ngto, P->d_Ct, P->st));
  P->launches += 1;
  if (kind_elastic(P->kind)) {
    // Z = C1^T sym(D) C1 (variables_elastic, src/Variables.f90:1199-1217),
    // C1 the first nmo1 MOs: Y(i, a) = sum_j Ds(i, j) C(j, a), then
    // Z(a, b) = sum_i C(i, a) Y(i, b)
    // (the resolved CMS: the same for each of its two 1-RDMs)
    const int k = P->nmo1;
    for (int z = 0; z < P->nzao; ++z) {
      const int64_t dk = (int64_t)z * k * k;
      TB_TRYC(launch_sym_small(P->d_D + dk, k, P->d_Ds + dk, P->st));
      DmmaGemmArgs g{};
      g.A = P->d_Ds + dk; g.sak = k; g.a_batch = 0;
      g.B = P->d_Ct; g.sbk = cw; g.sbj = 1;
      g.M = k; g.N = ngto; g.K = k;
      g.D = P->d_Y + (int64_t)z * k * ngto; g.sdm = 1; g.sdj = k; g.d_batch = 0;
      TB_TRYC(launch_dmma_gemm(g, 0, true, 1, P->st));
      g.A = P->d_Ct; g.sak = cw;
      g.B = P->d_Y + (int64_t)z * k * ngto; g.sbk = 1; g.sbj = k;
      g.M = ngto; g.N = ngto; g.K = k;
      g.D = P->d_zao + (int64_t)z * ngto * ngto; g.sdm = 1; g.sdj = ngto;
      TB_TRYC(launch_dmma_gemm(g, 0, false, 1, P->st));
      P->launches += 3;
    }
    goto done;
  }
  if (P->nmat == 0) {
    // otherwise the last pass writes every element
    TB_TRYC(cudaMemsetAsync(P->d_rho, 0, sizeof(double) * (size_t)(np * np), P->st));
    goto done;
  }
  TB_TRYC(cudaMemsetAsync(P->d_G, 0, sizeof(double) * (size_t)n4, P->st));
  {
    const int64_t m = 8 * (int64_t)P->nmat;
    size_t bytes = P->gsort_bytes;
    TB_TRYC(launch_ghat_emit(P->d_mat, P->d_tot, P->nmat, n, P->d_gk0, P->d_gv0, P->st));
    TB_TRYC(cub::DeviceRadixSort::SortPairs(P->d_gsort_tmp, bytes, P->d_gk0, P->d_gk1, P->d_gv0, P->d_gv1, (int)m,
                                            0, P->gbits, P->st));
    TB_TRYC(launch_ghat_runs(P->d_gk1, P->d_gv1, m, P->d_G, P->st));
    P->launches += 3;
  }
  {
    DmmaGemmArgs g{};
    // T1[xyz](a) = sum_w C(w, a) Ghat[x][y][z][w]: (ngto x n^3), leading dimension ngto
    g.A = P->d_Ct; g.sak = cw; g.a_batch = 0;
    g.B = P->d_G; g.sbk = 1; g.sbj = n;
    g.M = ngto; g.N = (int)n3; g.K = n;
    g.D = P->d_T1; g.sdm = 1; g.sdj = ngto; g.d_batch = 0;
    TB_TRYC(launch_dmma_gemm(g, 0, false, 1, P->st));
    // V[xy](fpair(c, d)) = sum_z T1[xyz](d) C(z, c) for c <= d, one batch per xy
    g.A = P->d_T1; g.sak = ngto; g.a_batch = (int64_t)n * ngto;
    g.B = P->d_Ct; g.sbk = cw; g.sbj = 1;
    g.M = ngto; g.N = ngto; g.K = n;
    g.D = P->d_V; g.sdm = 0; g.sdj = 0; g.d_batch = np;
    TB_TRYC(launch_dmma_gemm(g, 1, true, (int)n2, P->st));
    // T3[x](p, b) = sum_y V[xy](p) C(y, b), one batch per x
    g.A = P->d_V; g.sak = np; g.a_batch = (int64_t)n * np;
    g.M = (int)np; g.N = ngto; g.K = n;
    g.D = P->d_T3; g.sdm = 1; g.sdj = np; g.d_batch = (int64_t)ngto * np;
    TB_TRYC(launch_dmma_gemm(g, 0, true, n, P->st));
    // rho(p, fpair(a, b)) = sum_x T3[x](p, b) C(x, a) for a <= b, one batch per b
    g.A = P->d_T3; g.sak = (int64_t)ngto * np; g.a_batch = np;
    g.M = (int)np; g.N = ngto; g.K = n;
    g.D = P->d_rho; g.sdm = 1; g.sdj = np; g.d_batch = 0;
    TB_TRYC(launch_dmma_gemm(g, 2, true, ngto, P->st));
    P->launches += 4;
  }
done:
  return rc;
}

