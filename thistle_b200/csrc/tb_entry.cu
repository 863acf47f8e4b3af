// Entry 1 (thistle_total_scattering) and the terms its other calculation
// types add around the plan: the nuclear-electron and nuclear-nuclear terms
// of electron scattering, the elastic aligned form factor and the
// reference's q grids.
#include "tb_plan_internal.h"

using namespace tb;

// ---------------------------------------------------------------------------
// nuclear-electron term of electron scattering (types 5, 6): elastic plans
// ---------------------------------------------------------------------------
// Ine(q) = sum_a sum_(i,k) Zn_a F_ik(q) e12(q, i, k) over the nuclei and the
// ordered group pairs (nuclei_electron_integration, src/Integrals.f90:2493-2596),
// for the plan's current centres; geom is (natoms, 3) column-major.
int nuclear_term(thistle_plan *P, const double *Zn, const double *geom, int natoms, double *host_out) {
  if (P->kind != KIND_ELASTIC) return fail(THISTLE_ERR_TYPE, "the nuclear term needs an elastic plan (the 1-RDM)");
  if (!Zn || !geom || natoms < 1) return fail(THISTLE_ERR_ARG, "nuclear charges and positions are required");
  if (natoms >= (1 << 16)) return fail(THISTLE_ERR_SHAPE, "at most 65535 nuclei");
  if (!finite_all(Zn, natoms) || !finite_all(geom, 3 * (int64_t)natoms))
    return fail(THISTLE_ERR_NONFINITE, "non-finite nuclear charge or position");
  if (P->ngeom != 1) return fail(THISTLE_ERR_SHAPE, "the nuclear term is computed for single-geometry plans");
  int rc = THISTLE_OK;
  uint64_t *d_items = nullptr;
  double *d_nuc = nullptr, *d_rec = nullptr, *d_out = nullptr;
  // pair tables of the current centres
  TB_TRYC(launch_pair_tables(P->ng, P->maxa, P->d_gstart, P->d_flmn, P->d_ga, P->d_xyz, P->d_pairtab, P->d_esoa, 1,
                             3 * (int64_t)P->ngto, gs_pair(P), gs_esoa(P), P->st));
  {
    const int ng = P->ng;
    std::vector<std::vector<uint64_t>> byL(2 * 4 + 1);
    for (int a = 0; a < natoms; ++a)
      for (int gi = 0; gi < ng; ++gi)
        for (int gk = 0; gk < ng; ++gk) {
          const int L = P->gL[gi] + P->gL[gk];
          if (L < 0 || L > 8) {
            rc = fail(THISTLE_ERR_ANGMOM, "pair order above 8");
            goto done;
          }
          byL[L].push_back((uint64_t)a | ((uint64_t)gi << 16) | ((uint64_t)gk << 40));
        }
    std::vector<uint64_t> items;
    std::vector<int64_t> beg(10, 0), rec0(10, 0);
    std::vector<int> rsL(10, 0);
    int64_t recn = 0;
    for (int L = 0; L <= 8; ++L) {
      beg[L] = (int64_t)items.size();
      items.insert(items.end(), byL[L].begin(), byL[L].end());
      rsL[L] = L + 7 + ((L + 7) & 1);
      rec0[L] = recn;
      recn += (int64_t)byL[L].size() * rsL[L];
    }
    beg[9] = (int64_t)items.size();
    std::vector<double> nuc((size_t)natoms * 8, 0.0);
    for (int a = 0; a < natoms; ++a) {
      for (int d = 0; d < 3; ++d) nuc[(size_t)a * 8 + d] = geom[a + (size_t)natoms * d];
      nuc[(size_t)a * 8 + 4] = Zn[a];
    }
    TB_TRY(dalloc(&d_items, items.size(), "nuclear items"));
    TB_TRY(dalloc(&d_nuc, nuc.size(), "nuclei"));
    TB_TRY(dalloc(&d_rec, (size_t)std::max<int64_t>(recn, 1), "nuclear records"));
    TB_TRY(dalloc(&d_out, (size_t)P->nq, "nuclear term"));
    TB_TRYC(cudaMemcpyAsync(d_items, items.data(), sizeof(uint64_t) * items.size(), cudaMemcpyHostToDevice, P->st));
    TB_TRYC(cudaMemcpyAsync(d_nuc, nuc.data(), sizeof(double) * nuc.size(), cudaMemcpyHostToDevice, P->st));
    for (int L = 0; L <= 8; ++L) {
      if (beg[L + 1] == beg[L]) continue;
      Stage1Args a = stage1_args(P, nullptr, beg[L], beg[L + 1], d_rec, rec0[L], rsL[L]);
      TB_TRYC(launch_nuclear(L, a, d_items, d_nuc, P->st));
    }
    TB_TRYC(cudaMemsetAsync(P->d_partial, 0, sizeof(double) * (size_t)P->s2_rows * P->nq, P->st));
    for (int q0 = 0; q0 < P->nq; q0 += P->s2_qtile) {
      const int tn = std::min(P->s2_qtile, P->nq - q0);
      int uniform = 0, first_on_grid = 0;
      double dq = 0.0;
      grid_info(P->hq.data() + q0, tn, uniform, first_on_grid, dq);
      for (int L = 0; L <= 8; ++L) {
        const int64_t nL = beg[L + 1] - beg[L];
        if (nL == 0) continue;
        Stage2ClassArgs s;
        s.rec = d_rec + rec0[L];
        s.rs = rsL[L];
        s.nquart = nL;
        s.perm = nullptr;
        s.pbase = 0;
        s.gs_rec = 0;
        s.gs_partial = 0;
        s.q = P->d_q + q0;
        s.nq = tn;
        s.uniform = uniform;
        s.first_on_grid = first_on_grid;
        s.dq = dq;
        s.chunk = 0;
        s.j2 = false;
        s.lb = L;
        s.partial = P->d_partial + q0;
        s.pstride = P->nq;
        const int64_t per_block = (int64_t)stage2_quartets_per_warp(L, P->s2_tile) * P->s2_tile.nw;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nL + per_block - 1) / per_block, P->s2_rows));
        TB_TRYC(launch_stage2_class(L, s, grid, 1, P->s2_tile, P->st));
      }
    }
    TB_TRYC(launch_reduce_batch(P->d_partial, P->s2_rows, P->nq, (int64_t)P->s2_rows * P->nq, d_out, 1, P->st));
    TB_TRYC(cudaMemcpyAsync(host_out, d_out, sizeof(double) * P->nq, cudaMemcpyDeviceToHost, P->st));
  }
done:
  cudaStreamSynchronize(P->st);
  dfree(d_items);
  dfree(d_nuc);
  dfree(d_rec);
  dfree(d_out);
  return rc;
}

// Inn(q) = sum_ij Zn_i Zn_j sinc(q R_ij), sinc(x) = 1 for |x| < 1e-10
// (src/main_calculation.f90:302-311, 853-861)
// ---------------------------------------------------------------------------
// elastic aligned intensity (type 4): F(q) on q vectors from the AO density
// ---------------------------------------------------------------------------
// F(q) of elastic_integration_alig (src/Integrals.f90:2366-2490) for the
// plan's current centres on nq q vectors (3 interleaved doubles each, host);
// re / im / abs2 (host, any may be NULL) get F and |F|^2 (tb_formfactor.cu).
int form_factor(thistle_plan *P, const double *qvec, int nq, double *re, double *im, double *abs2) {
  if (!kind_elastic(P->kind)) return fail(THISTLE_ERR_TYPE, "the form factor needs an elastic plan (the 1-RDM)");
  if (!qvec || nq <= 0) return fail(THISTLE_ERR_ARG, "empty q-vector list");
  if (!finite_all(qvec, 3 * (int64_t)nq)) return fail(THISTLE_ERR_NONFINITE, "non-finite q vector");
  if (P->ngeom != 1) return fail(THISTLE_ERR_SHAPE, "the form factor is computed for single-geometry plans");
  int rc = THISTLE_OK;
  double *d_rec = nullptr, *d_qv = nullptr, *d_out = nullptr;
  std::vector<double> h((size_t)3 * nq);
  TB_TRY(dalloc(&d_rec, (size_t)form_factor_record_doubles(npairs(P->ng)), "form-factor records"));
  TB_TRY(dalloc(&d_qv, (size_t)3 * nq, "q vectors"));
  TB_TRY(dalloc(&d_out, (size_t)3 * nq, "form factor"));
  TB_TRYC(cudaMemcpyAsync(d_qv, qvec, sizeof(double) * 3 * (size_t)nq, cudaMemcpyHostToDevice, P->st));
  TB_TRYC(launch_pair_tables(P->ng, P->maxa, P->d_gstart, P->d_flmn, P->d_ga, P->d_xyz, P->d_pairtab, P->d_esoa, 1,
                             3 * (int64_t)P->ngto, gs_pair(P), gs_esoa(P), P->st));
  {
    const Stage1Args a = stage1_args(P, P->d_quart, 0, 0, nullptr, 0, 0);
    TB_TRYC(launch_form_factor(a, d_rec, d_qv, nq, d_out, d_out + nq, d_out + 2 * (size_t)nq, P->st));
  }
  P->launches = 3;
  TB_TRYC(cudaMemcpyAsync(h.data(), d_out, sizeof(double) * 3 * (size_t)nq, cudaMemcpyDeviceToHost, P->st));
  TB_TRYC(cudaStreamSynchronize(P->st));
  P->fwd_valid = false;  // the pair tables were rebuilt
  if (re) std::copy(h.begin(), h.begin() + nq, re);
  if (im) std::copy(h.begin() + nq, h.begin() + 2 * (size_t)nq, im);
  if (abs2) std::copy(h.begin() + 2 * (size_t)nq, h.end(), abs2);
done:
  dfree(d_rec);
  dfree(d_qv);
  dfree(d_out);
  return rc;
}

// The q vectors of CASE(4) (src/main_calculation.f90:227-241) for nq points:
// ss = (linspace(0, pi/2, nq) - pi) / 2, k0 = 3.00 * 1.889726125 * 0.529,
// q = 2 k0 cos(ss) (sin ss, 0, cos ss), written (3, nq) column-major.
void elastic_aligned_grid(int nq, double *qal) {
  const double pi = std::acos(-1.0), k0 = 3.00 * 1.889726125 * 0.529;
  for (int mm = 0; mm < nq; ++mm) {
    double ss = nq > 1 ? (pi / 2.0) * (double)mm / (double)(nq - 1) : 0.0;
    ss = (ss - pi) / 2.0;
    const double rr = 2.0 * k0 * std::cos(ss);
    qal[3 * mm] = rr * std::sin(ss) * std::cos(0.0);
    qal[3 * mm + 1] = rr * std::sin(ss) * std::sin(0.0);
    qal[3 * mm + 2] = rr * std::cos(ss);
  }
}

void nuclear_nuclear(const double *Zn, const double *geom, int natoms, const double *q, int nq, double *out) {
  for (int k = 0; k < nq; ++k) out[k] = 0.0;
  for (int i = 0; i < natoms; ++i)
    for (int j = 0; j < natoms; ++j) {
      double r2 = 0.0;
      for (int d = 0; d < 3; ++d) {
        const double x = geom[i + (size_t)natoms * d] - geom[j + (size_t)natoms * d];
        r2 += x * x;
      }
      const double R = std::sqrt(r2);
      for (int k = 0; k < nq; ++k) {
        const double a = q[k] * R;
        out[k] += Zn[i] * Zn[j] * (std::fabs(a) < 1e-10 ? 1.0 : std::sin(a) / a);
      }
    }
}

// The reference's aligned q grid (QCOORD3, src/main_calculation.f90:864-929):
// the origin, one point on the +y axis, a hexagon of radius dk, then rings of
// radius i dk (i = 2..31) with ceil(pi / asin(1/(2i))) points each starting on
// +y, every point lifted onto the Ewald sphere of radius k0; dk =
// sqrt(3)/2 k0/31.  Unused slots and zero components are 1e-10, as there.
void qcoord3_grid(double k0, double *qal /* (3, 3131) column-major */) {
  const int nring = 30, npts = 3131;
  const double pi = std::acos(-1.0);
  const double dk = std::sqrt(3.0) / 2.0 * k0 / (nring + 1.0);
  double *qx = qal, *qy = qal + 1, *qz = qal + 2;  // stride 3
  for (int t = 0; t < npts; ++t) qx[3 * t] = qy[3 * t] = qz[3 * t] = 1.0e-10;
  auto lift = [&](double x, double y) { return k0 * (1.0 - std::sqrt(std::fabs(1.0 - (x * x + y * y) / (k0 * k0)))); };
  int pos = 1;  // 0-based slot of the +y point
  qy[3 * pos] = dk;
  qz[3 * pos] = k0 * (1.0 - std::sqrt(1.0 - 1.0 / ((nring + 1.0) * (nring + 1.0))));
  for (int i = 1; i <= 5; ++i) {
    ++pos;
    const double x = std::sin(i * pi / 3.0) * dk, y = std::cos(i * pi / 3.0) * dk;
    qx[3 * pos] = x;
    qy[3 * pos] = y;
    qz[3 * pos] = k0 * (1.0 - std::sqrt(1.0 - (x * x + y * y) / (k0 * k0)));
  }
  for (int i = 2; i <= nring + 1; ++i) {
    const int np = (int)std::ceil(pi / std::asin(1.0 / (2.0 * i)));
    const double rc = i * dk, ang = 2.0 * pi / np;
    ++pos;
    qy[3 * pos] = rc;
    qz[3 * pos] = k0 * (1.0 - std::sqrt(std::fabs(1.0 - std::pow((double)i, 2.0) / ((nring + 1.0) * (nring + 1.0)))));
    for (int j = 1; j <= np - 1; ++j) {
      ++pos;
      const double x = std::sin(j * ang) * rc, y = std::cos(j * ang) * rc;
      qx[3 * pos] = x;
      qy[3 * pos] = y;
      qz[3 * pos] = lift(x, y);
    }
  }
}

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

int thistle_qcoord3(double k0, double *q_al) {
  if (!q_al) return fail(THISTLE_ERR_ARG, "null argument");
  if (!std::isfinite(k0) || !(k0 > 0.0)) return fail(THISTLE_ERR_ARG, "k0 must be finite and positive");
  qcoord3_grid(k0, q_al);
  return THISTLE_OK;
}

int thistle_plan_form_factor(thistle_plan *P, const double *qvec, int32_t nq, double *re_host, double *im_host,
                             double *abs2_host) {
  if (!P) return fail(THISTLE_ERR_ARG, "null plan");
  return form_factor(P, qvec, nq, re_host, im_host, abs2_host);
}

int thistle_elastic_aligned_grid(int32_t nq, double *q_al) {
  if (nq <= 0 || !q_al) return fail(THISTLE_ERR_ARG, "nq must be positive and q_al non-null");
  elastic_aligned_grid(nq, q_al);
  return THISTLE_OK;
}

int thistle_plan_nuclear(thistle_plan *P, const double *Zn, const double *geom, int32_t natoms, double *ine_host) {
  if (!P || !ine_host) return fail(THISTLE_ERR_ARG, "null argument");
  return nuclear_term(P, Zn, geom, natoms, ine_host);
}

int thistle_total_scattering(int32_t type, const double *Zn, const double *geom, int32_t natoms, int32_t maxl,
                             int32_t ngto, int32_t ng, const double *ga, const int32_t *l, const int32_t *m,
                             const int32_t *n, const double *xx, const double *yy, const double *zz,
                             const double *mmod, int32_t norbs, const double *q, int32_t nq, const int32_t *group,
                             double cutoffz, double cutoffmd, double cutoffcentre, const int32_t *mat,
                             const double *total, int32_t nmat, const double *onerdm, int32_t nmo1,
                             double *q_abs_out, double *result_out) {
  if (!result_out) return fail(THISTLE_ERR_ARG, "null result");
  if (maxl < 0) return fail(THISTLE_ERR_ARG, "maxl must be >= 0");
  if (type == THISTLE_TOTAL_ELECTRON || type == THISTLE_ELASTIC_ELECTRON) {
    // I_e - 2 Ine + Inn (src/main_calculation.f90:277-329, 330-...), I_e the
    // total (type 5) or elastic (type 6) j0 intensity
    if (!Zn || !geom || natoms < 1) return fail(THISTLE_ERR_ARG, "electron scattering needs Zn and geom");
    if (!onerdm || nmo1 <= 0) return fail(THISTLE_ERR_ARG, "electron scattering needs the 1-RDM");
    if (!q || nq <= 0) return fail(THISTLE_ERR_ARG, "empty q grid");
    thistle_plan *E = nullptr, *T = nullptr;
    int rc = plan_create(&E, THISTLE_ELASTIC_J0, ngto, ga, l, m, n, xx, yy, zz, group, mmod, norbs, nullptr, nullptr,
                         0, onerdm, nmo1, q, nq, cutoffz, cutoffmd, cutoffcentre);
    if (rc != THISTLE_OK) return rc;
    std::vector<double> ie((size_t)nq), ine((size_t)nq), inn((size_t)nq);
    if (ng != E->ng) rc = fail(THISTLE_ERR_SHAPE, "ng differs from maxval(group)");
    if (rc == THISTLE_OK && type == THISTLE_TOTAL_ELECTRON) {
      rc = plan_create(&T, THISTLE_TOTAL_J0, ngto, ga, l, m, n, xx, yy, zz, group, mmod, norbs, mat, total, nmat,
                       nullptr, 0, q, nq, cutoffz, cutoffmd, cutoffcentre);
      if (rc == THISTLE_OK) rc = thistle_plan_execute(T, ie.data());
    }
    if (rc == THISTLE_OK && type == THISTLE_ELASTIC_ELECTRON) rc = thistle_plan_execute(E, ie.data());
    if (rc == THISTLE_OK) rc = nuclear_term(E, Zn, geom, natoms, ine.data());
    if (rc == THISTLE_OK) {
      nuclear_nuclear(Zn, geom, natoms, q, nq, inn.data());
      for (int k = 0; k < nq; ++k) result_out[k] = ie[k] - 2.0 * ine[k] + inn[k];
      if (q_abs_out)
        for (int k = 0; k < nq; ++k) q_abs_out[k] = q[k];
    }
    if (T) thistle_plan_destroy(T);
    thistle_plan_destroy(E);
    return rc;
  }
  if (type == THISTLE_ELASTIC_ALIGNED) {
    // CASE(4): |F(q)|^2 on the reference's own grid of nq vectors, whatever q
    // holds; q_abs_out gets |q| (src/main_calculation.f90:218-265)
    if (!onerdm || nmo1 <= 0) return fail(THISTLE_ERR_ARG, "the elastic aligned intensity needs the 1-RDM");
    if (nq <= 0) return fail(THISTLE_ERR_ARG, "nq must be positive");
    std::vector<double> qal((size_t)3 * nq), qabs((size_t)nq);
    elastic_aligned_grid(nq, qal.data());
    for (int i = 0; i < nq; ++i)
      qabs[i] = std::sqrt(qal[3 * i] * qal[3 * i] + qal[3 * i + 1] * qal[3 * i + 1] + qal[3 * i + 2] * qal[3 * i + 2]);
    thistle_plan *E = nullptr;
    int rc = plan_create(&E, THISTLE_ELASTIC_J0, ngto, ga, l, m, n, xx, yy, zz, group, mmod, norbs, nullptr, nullptr,
                         0, onerdm, nmo1, qabs.data(), nq, cutoffz, cutoffmd, cutoffcentre);
    if (rc != THISTLE_OK) return rc;
    if (ng != E->ng) rc = fail(THISTLE_ERR_SHAPE, "ng differs from maxval(group)");
    if (rc == THISTLE_OK) rc = form_factor(E, qal.data(), nq, nullptr, nullptr, result_out);
    if (rc == THISTLE_OK && q_abs_out) std::copy(qabs.begin(), qabs.end(), q_abs_out);
    thistle_plan_destroy(E);
    return rc;
  }
  // type 3 evaluates on the reference's own aligned grid (QCOORD3 with
  // k0 = 10.583544175, 3131 vectors), whatever q holds; q_abs_out gets |q|
  std::vector<double> qal;
  if (type == THISTLE_TOTAL_ALIGNED) {
    if (nq != 3131) return fail(THISTLE_ERR_SHAPE, "type 3 runs on the 3131-vector QCOORD3 grid: nq must be 3131");
    qal.resize(3 * 3131);
    qcoord3_grid(10.583544175, qal.data());
    q = qal.data();
  }
  thistle_plan *P = nullptr;
  int rc = plan_create(&P, type, ngto, ga, l, m, n, xx, yy, zz, group, mmod, norbs, mat, total, nmat, onerdm, nmo1,
                       q, nq, cutoffz, cutoffmd, cutoffcentre);
  if (rc != THISTLE_OK) return rc;
  if (ng != P->ng) {
    plan_free(P);
    return fail(THISTLE_ERR_SHAPE, "ng differs from maxval(group)");
  }
  PhaseTrace tr;
  rc = thistle_plan_execute(P, result_out);
  tr.mark("execute");
  if (rc == THISTLE_OK && q_abs_out) {
    for (int i = 0; i < nq; ++i)
      q_abs_out[i] = type == THISTLE_TOTAL_ALIGNED
                         ? std::sqrt(q[3 * i] * q[3 * i] + q[3 * i + 1] * q[3 * i + 1] + q[3 * i + 2] * q[3 * i + 2])
                         : q[i];
  }
  thistle_plan_destroy(P);
  return rc;
}

}  // extern "C"
