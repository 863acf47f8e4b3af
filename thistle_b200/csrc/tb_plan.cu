// Host side of the C-ABI: validation, device set-up and the execution order
// of the scattering-intensity path.
//
// Reference map:
//   group_start/group_count       src/main_calculation.f90:85-93
//   z11/z22 and the per-quartet dgemm pair (zcontrred, zcontrred2)
//                                 src/Variables.f90:1045-1065, src/Integrals.f90:109-127
//       -> one 4-index transform rho(ab,cd) = sum Ghat C C C C on the device
//   pair centres, E12, MD tables  src/Variables.f90:1113-1148
//   the five quartet loops        src/Integrals.f90:79-468 (bra pair i<=j, ket pair k<=r)
//   per-quartet kernels           src/Integrals.f90:4955-5226 and variants
#include "tb_plan_internal.h"

using namespace tb;

thread_local std::string g_err;

namespace tb {
int set_error(int code, const std::string &msg) { return fail(code, msg); }
}  // namespace tb

// ---------------------------------------------------------------------------
// validation
// ---------------------------------------------------------------------------
bool finite_all(const double *a, int64_t n) {
  // x - x is 0 for finite x and NaN for NaN or Inf: one branch-free pass
  double acc = 0.0;
  for (int64_t i = 0; i < n; ++i) acc += a[i] - a[i];
  return acc == 0.0;
}

int check_basis(thistle_plan *P, int32_t ngto, const double *ga, const int32_t *l, const int32_t *m,
                       const int32_t *n, const double *xx, const double *yy, const double *zz,
                       const int32_t *group) {
  if (ngto <= 0) return fail(THISTLE_ERR_ARG, "ngto must be positive");
  if (!ga || !l || !m || !n || !xx || !yy || !zz || !group) return fail(THISTLE_ERR_ARG, "null basis array");
  if (!finite_all(ga, ngto) || !finite_all(xx, ngto) || !finite_all(yy, ngto) || !finite_all(zz, ngto))
    return fail(THISTLE_ERR_NONFINITE, "non-finite exponent or centre");
  int ng = 0, maxa = 0;
  for (int i = 0; i < ngto; ++i) {
    if (!(ga[i] > 0.0)) return fail(THISTLE_ERR_ARG, "exponent must be positive (function " + std::to_string(i + 1) + ")");
    if (l[i] < 0 || m[i] < 0 || n[i] < 0) return fail(THISTLE_ERR_ARG, "negative angular exponent");
    if (l[i] > MAXA || m[i] > MAXA || n[i] > MAXA || l[i] + m[i] + n[i] > MAXA)
      return fail(THISTLE_ERR_ANGMOM,
                  "McMurchie-Davidson coefficients are only implemented up to g functions (function " +
                      std::to_string(i + 1) + ")");
    maxa = std::max(maxa, std::max(l[i], std::max(m[i], n[i])));
    if (group[i] < 1) return fail(THISTLE_ERR_SHAPE, "group ids are 1-based");
    ng = std::max(ng, (int)group[i]);
  }
  if (ng > 65535) return fail(THISTLE_ERR_SHAPE, "more than 65535 groups");
  P->ngto = ngto;
  P->ng = ng;
  P->maxa = maxa;
  P->gstart.assign(ng, -1);
  P->gcount.assign(ng, 0);
  P->gL.assign(ng, 0);
  P->flmn.resize(ngto);
  for (int i = 0; i < ngto; ++i) {
    int g = group[i] - 1;
    if (P->gstart[g] < 0) P->gstart[g] = i;
    else if (group[i - 1] != group[i])
      return fail(THISTLE_ERR_SHAPE, "functions of group " + std::to_string(g + 1) + " are not contiguous");
    P->gcount[g] += 1;
    P->flmn[i] = l[i] | (m[i] << 8) | (n[i] << 16);
  }
  for (int g = 0; g < ng; ++g) {
    if (P->gstart[g] < 0) return fail(THISTLE_ERR_SHAPE, "group " + std::to_string(g + 1) + " has no function");
    int h = P->gstart[g];
    P->gL[g] = l[h] + m[h] + n[h];
    if (P->gL[g] <= 3) {
      bool ok = P->gcount[g] == (P->gL[g] + 1) * (P->gL[g] + 2) / 2;
      for (int i = 0; ok && i < P->gcount[g]; ++i)
        ok = l[h + i] == cart_component(P->gL[g], i, 0) && m[h + i] == cart_component(P->gL[g], i, 1) &&
             n[h + i] == cart_component(P->gL[g], i, 2);
      if (!ok) P->shells_canonical = 0;
    }
    for (int i = h; i < h + P->gcount[g]; ++i) {
      if (ga[i] != ga[h] || xx[i] != xx[h] || yy[i] != yy[h] || zz[i] != zz[h] ||
          l[i] + m[i] + n[i] != P->gL[g])
        return fail(THISTLE_ERR_SHAPE, "group " + std::to_string(g + 1) +
                                           " mixes exponents, centres or shells (one shell per group)");
    }
  }
  return THISTLE_OK;
}

int check_q(const double *q, int32_t nq) {
  if (!q || nq <= 0) return fail(THISTLE_ERR_ARG, "empty q grid");
  for (int i = 0; i < nq; ++i) {
    if (!std::isfinite(q[i])) return fail(THISTLE_ERR_NONFINITE, "non-finite q");
    if (!(q[i] > 0.0))
      return fail(THISTLE_ERR_Q, "q must be > 0 (the reference divides by q; its drivers put 1e-10 for 0)");
  }
  return THISTLE_OK;
}

// ---------------------------------------------------------------------------
// quartet classes
// ---------------------------------------------------------------------------
int64_t bra_count(int i, int j, int ng, bool all_pairs) {
  if (all_pairs) return npairs(ng);  // resolved CMS: every ket pair
  if (i < j) return (int64_t)(ng - i) * (ng - i - 1) / 2;
  return (int64_t)ng * (ng - 1) / 2 + (ng - i);
}

static inline int class_key(int Li, int Lj, int Lk, int Lr) {
  return ((((Li + Lj + Lk + Lr) * 5 + Li) * 5 + Lj) * 5 + Lk) * 5 + Lr;
}

// Quartet counts per class key, without enumerating quartets.
void class_counts(const std::vector<int> &gL, std::vector<int64_t> &cnt, bool all_pairs) {
  int ng = (int)gL.size();
  cnt.assign(17 * 625, 0);
  if (all_pairs) {
    // every (bra pair, ket pair): products of the pair counts per (La, Lb)
    int64_t pc[5][5] = {};
    for (int i = 0; i < ng; ++i)
      for (int j = i; j < ng; ++j) ++pc[gL[i]][gL[j]];
    for (int a = 0; a < 25; ++a)
      for (int b = 0; b < 25; ++b)
        if (pc[a / 5][a % 5] && pc[b / 5][b % 5])
          cnt[class_key(a / 5, a % 5, b / 5, b % 5)] += pc[a / 5][a % 5] * pc[b / 5][b % 5];
    return;
  }
  // off[k][a][b]: #{(k',r): k <= k' < r, gL[k']=a, gL[r]=b}; diag[k][a]: #{k' >= k: gL[k'] = a}
  std::vector<int64_t> off((size_t)(ng + 1) * 25, 0), after(5, 0), diag((size_t)(ng + 1) * 5, 0);
  for (int k = ng - 1; k >= 0; --k) {
    for (int t = 0; t < 25; ++t) off[(size_t)k * 25 + t] = off[(size_t)(k + 1) * 25 + t];
    for (int b = 0; b < 5; ++b) off[(size_t)k * 25 + gL[k] * 5 + b] += after[b];
    after[gL[k]] += 1;
    for (int a = 0; a < 5; ++a) diag[(size_t)k * 5 + a] = diag[(size_t)(k + 1) * 5 + a];
    diag[(size_t)k * 5 + gL[k]] += 1;
  }
  for (int i = 0; i < ng; ++i)
    for (int j = i; j < ng; ++j) {
      int Li = gL[i], Lj = gL[j];
      const int64_t *o = &off[(size_t)(i < j ? i : 0) * 25];
      for (int a = 0; a < 5; ++a)
        for (int b = 0; b < 5; ++b)
          if (o[a * 5 + b]) cnt[class_key(Li, Lj, a, b)] += o[a * 5 + b];
      if (i == j)
        for (int a = 0; a < 5; ++a)
          if (diag[(size_t)i * 5 + a]) cnt[class_key(Li, Lj, a, a)] += diag[(size_t)i * 5 + a];
    }
}

// Sorted-by-key layout -> contiguous LLmax classes and record offsets.
// The 625 shell tuples ((Li 5 + Lj) 5 + Lk) 5 + Lr in class-sort order:
// LLmax, then the sub-range (LK, XB), then the tuple (the order of quartet_key).
static const std::vector<int> &tuple_sort_order() {
  static const std::vector<int> order = [] {
    std::vector<int> o(625);
    for (int t = 0; t < 625; ++t) o[t] = t;
    std::stable_sort(o.begin(), o.end(), [](int a, int b) {
      const uint32_t ka = quartet_key(a / 125, (a / 25) % 5, (a / 5) % 5, a % 5);
      const uint32_t kb = quartet_key(b / 125, (b / 25) % 5, (b / 5) % 5, b % 5);
      return ka / 625 < kb / 625;
    });
    return o;
  }();
  return order;
}

int setup_classes(thistle_plan *P, const std::vector<int64_t> &cnt, int kind) {
  int64_t pos = 0, recoff = 0;
  P->ncls = 0;
  int maxg[5] = {0, 0, 0, 0, 0};  // most functions of a group, per shell L
  for (int g = 0; g < P->ng; ++g)
    if (P->gL[g] >= 0 && P->gL[g] <= 4) maxg[P->gL[g]] = std::max(maxg[P->gL[g]], P->gcount[g]);
  const std::vector<int> &order = tuple_sort_order();
  size_t oi = 0;  // order is sorted by LLmax: each class's tuples are a contiguous run
  for (int LL = 0; LL <= LMAXQ; ++LL) {
    const size_t o0 = oi;
    while (oi < order.size() && quartet_key(order[oi] / 125, (order[oi] / 25) % 5, (order[oi] / 5) % 5,
                                            order[oi] % 5) / KEY_CLASS_DIV == (uint32_t)LL)
      ++oi;
    int64_t c = 0;
    for (size_t j = o0; j < oi; ++j) c += cnt[LL * 625 + order[j]];
    if (c == 0) continue;
    if (P->ncls >= MAXCLS) return fail(THISTLE_ERR_ARG, "too many quartet classes");
    int k = P->ncls++;
    P->cls_L[k] = LL;
    P->cls_begin[k] = pos;
    P->cls_end[k] = pos + c;
    // [H, s, kind, order] + up to LL+3 coefficients; aligned: [H vector, s] + D_TUV
    int rs = kind == KIND_ALIGNED ? 4 + ntuv(LL) : LL + 7;
    rs += rs & 1;
    P->cls_rs[k] = rs;
    P->cls_recoff[k] = recoff;
    // sub-ranges in key order: (LK, XB) ascending, tuples ascending within
    P->cls_sub[k].clear();
    P->cls_tup[k].clear();
    int64_t sp = pos;
    size_t j = o0;
    while (j < oi) {
      const int sub = (int)((quartet_key(order[j] / 125, (order[j] / 25) % 5, (order[j] / 5) % 5, order[j] % 5) /
                             625) % 18);
      int64_t sc = 0;
      int nout = 0;
      const int LK = sub / 2, XB = sub % 2;
      for (; j < oi; ++j) {
        const int t = order[j];
        const int Li = t / 125, Lj = (t / 25) % 5, Lk = (t / 5) % 5, Lr = t % 5;
        if ((int)((quartet_key(Li, Lj, Lk, Lr) / 625) % 18) != sub) break;
        if (cnt[LL * 625 + t] == 0) continue;
        P->cls_tup[k].push_back(TupleRange{t, sp + sc, sp + sc + cnt[LL * 625 + t]});
        sc += cnt[LL * 625 + t];
        // the outer side is the ket when LK is the bra's
        nout = std::max(nout, XB ? maxg[Lk] * maxg[Lr] : maxg[Li] * maxg[Lj]);
      }
      if (sc > 0) P->cls_sub[k].push_back(SubRange{LK, XB, sp, sp + sc, nout});
      sp += sc;
    }
    recoff += c * rs;
    pos += c;
  }
  P->nquart = pos;
  P->rec_total = recoff;
  return THISTLE_OK;
}

// ---------------------------------------------------------------------------
// quartets on the device: enumerate in bra-pair order, then a stable radix
// sort on the class key so that each LLmax class is contiguous and each warp
// of stage 1 sees quartets with identical loop bounds.
// ---------------------------------------------------------------------------
int quartets_alloc(thistle_plan *P) {
  const int ng = P->ng, nb = npairs(ng);
  std::vector<int64_t> off(nb + 1);
  int64_t acc = 0;
  for (int i = 0, b = 0; i < ng; ++i)
    for (int j = i; j < ng; ++j, ++b) {
      off[b] = acc;
      acc += bra_count(i, j, ng, P->kind == KIND_CMS);
    }
  off[nb] = acc;
  if (acc != P->nquart) return fail(THISTLE_ERR_ARG, "internal: quartet count mismatch");
  if (acc >= ((int64_t)1 << 31)) return fail(THISTLE_ERR_ARG, "more than 2^31 group quartets");
  int rc = THISTLE_OK;
  TB_TRY(dalloc(&P->d_braoff, (size_t)nb + 1, "bra offsets"));
  TB_TRY(dalloc(&P->d_gL, (size_t)ng, "group L"));
  TB_TRY(dalloc(&P->d_k0, (size_t)acc, "quartet keys"));
  TB_TRY(dalloc(&P->d_k1, (size_t)acc, "quartet keys"));
  TB_TRY(dalloc(&P->d_v0, (size_t)acc, "quartets"));
  TB_TRY(dalloc(&P->d_quart, (size_t)acc, "quartets"));
  TB_TRYC(cudaMemcpyAsync(P->d_braoff, off.data(), sizeof(int64_t) * (nb + 1), cudaMemcpyHostToDevice, P->st));
  TB_TRYC(cudaMemcpyAsync(P->d_gL, P->gL.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, P->st));
  TB_TRYC(cub::DeviceRadixSort::SortPairs(nullptr, P->sort_tmp_bytes, P->d_k0, P->d_k1, P->d_v0, P->d_quart,
                                          (int)acc, 0, KEY_BITS, P->st));
  TB_TRY(dalloc((char **)&P->d_sort_tmp, P->sort_tmp_bytes, "sort scratch"));
done:
  return rc;
}

int quartets_run(thistle_plan *P) {
  int rc = THISTLE_OK;
  TB_TRYC(launch_quartet_fill(P->ng, P->d_braoff, P->nquart, P->d_gL, P->d_v0, P->d_k0, P->kind == KIND_CMS,
                              P->st));
  P->launches += 1;
  TB_TRYC(cub::DeviceRadixSort::SortPairs(P->d_sort_tmp, P->sort_tmp_bytes, P->d_k0, P->d_k1, P->d_v0, P->d_quart,
                                          (int)P->nquart, 0, KEY_BITS, P->st));
done:
  return rc;
}

// ---------------------------------------------------------------------------
// plan lifecycle
// ---------------------------------------------------------------------------
void plan_free(thistle_plan *P) {
  if (!P) return;
  dfree(P->d_gstart); dfree(P->d_gcount); dfree(P->d_flmn); dfree(P->d_ga); dfree(P->d_xyz);
  dfree(P->d_q); dfree(P->d_pairtab); dfree(P->d_esoa); dfree(P->d_rho); dfree(P->d_zao); dfree(P->d_rec);
  dfree(P->d_partial); dfree(P->d_result); dfree(P->d_quart);
  dfree(P->d_mat); dfree(P->d_C); dfree(P->d_tot); dfree(P->d_D); dfree(P->d_Ds); dfree(P->d_Y);
  dfree(P->d_G); dfree(P->d_T1); dfree(P->d_V); dfree(P->d_T3); dfree(P->d_Ct);
  dfree(P->d_gk0); dfree(P->d_gk1); dfree(P->d_gv0); dfree(P->d_gv1); dfree(P->d_gsort_tmp);
  dfree(P->d_xbuf);
  dfree(P->d_braoff); dfree(P->d_gL); dfree(P->d_k0); dfree(P->d_k1); dfree(P->d_v0); dfree(P->d_p0count);
  dfree(P->d_s2key); dfree(P->d_s2key_sorted); dfree(P->d_iota); dfree(P->d_perm);
  dfree(P->d_dsoa); dfree(P->d_adj); dfree(P->d_gpart); dfree(P->d_v); dfree(P->d_grad);
  if (P->gx_fwd) cudaGraphExecDestroy(P->gx_fwd);
  if (P->gx_vjp) cudaGraphExecDestroy(P->gx_vjp);
  dfree(P->d_s2sort_tmp);
  dfree(P->d_sort_tmp);
  if (P->have_ev) {
    for (int i = 0; i < 10; ++i) cudaEventDestroy(P->ev[i]);
    for (int r = 0; r < P->rev_made; ++r)
      for (int i = 0; i < 6; ++i) cudaEventDestroy(P->rev[r][i]);
  }
  if (P->ev_join) cudaEventDestroy(P->ev_join);
  if (P->ev_join3) cudaEventDestroy(P->ev_join3);
  for (int c = 0; c < MAXCLS; ++c)
    if (P->ev_cls[c]) cudaEventDestroy(P->ev_cls[c]);
  if (P->st2) cudaStreamDestroy(P->st2);
  if (P->st3) cudaStreamDestroy(P->st3);
  if (P->st && P->own_stream) cudaStreamDestroy(P->st);
  delete P;
}

int64_t gs_pair(const thistle_plan *P) { return (int64_t)npairs(P->ng) * PAIR_STRIDE; }
int64_t gs_esoa(const thistle_plan *P) { return esoa_doubles(P->ng, P->maxa); }
int64_t gs_rec(const thistle_plan *P) { return std::max<int64_t>(P->rec_total, 1); }

void drop_graphs(thistle_plan *P) {
  if (P->gx_fwd) cudaGraphExecDestroy(P->gx_fwd);
  if (P->gx_vjp) cudaGraphExecDestroy(P->gx_vjp);
  P->gx_fwd = P->gx_vjp = nullptr;
}

// (Re)allocates the per-geometry buffers for G geometries (the adjoint's on
// its next use); the partial-row count s2_rows must be set.
int geo_alloc(thistle_plan *P, int G) {
  int rc = THISTLE_OK;
  drop_graphs(P);
  dfree(P->d_xyz); dfree(P->d_pairtab); dfree(P->d_esoa); dfree(P->d_rec); dfree(P->d_partial);
  dfree(P->d_p0count); dfree(P->d_result);
  dfree(P->d_dsoa); dfree(P->d_adj); dfree(P->d_gpart); dfree(P->d_v); dfree(P->d_grad);
  P->ngeom = G;
  TB_TRY(dalloc(&P->d_xyz, (size_t)G * 3 * P->ngto, "centres"));
  TB_TRY(dalloc(&P->d_pairtab, (size_t)G * gs_pair(P), "pair tables"));
  TB_TRY(dalloc(&P->d_esoa, (size_t)G * gs_esoa(P), "transposed E tables"));
  TB_TRY(dalloc(&P->d_rec, (size_t)G * gs_rec(P), "quartet records"));
  TB_TRY(dalloc(&P->d_partial, (size_t)G * 2 * P->s2_rows * P->nq, "partial sums"));
  TB_TRY(dalloc(&P->d_p0count, (size_t)G * MAXCLS, "P0 counters"));
  TB_TRY(dalloc(&P->d_result, (size_t)G * P->nq, "result"));
  P->fwd_valid = false;
done:
  return rc;
}

int upload_centres(thistle_plan *P, const double *xx, const double *yy, const double *zz) {
  std::vector<double> xyz((size_t)P->ngto * 3);
  for (int i = 0; i < P->ngto; ++i) {
    xyz[3 * i] = xx[i];
    xyz[3 * i + 1] = yy[i];
    xyz[3 * i + 2] = zz[i];
  }
  // geometry 0 (the only one outside batches)
  if (P->hxyz.size() >= xyz.size() && std::equal(xyz.begin(), xyz.end(), P->hxyz.begin()))
    return THISTLE_OK;  // unchanged: records stay valid
  TB_CK(cudaMemcpyAsync(P->d_xyz, xyz.data(), sizeof(double) * xyz.size(), cudaMemcpyHostToDevice, P->st));
  TB_CK(cudaStreamSynchronize(P->st));
  if (P->hxyz.size() < xyz.size()) P->hxyz.resize(xyz.size());
  std::copy(xyz.begin(), xyz.end(), P->hxyz.begin());
  P->fwd_valid = false;
  return THISTLE_OK;
}

// All geometries of a batch from one host array (ngeom x ngto x 3, interleaved).
int upload_centres_batch(thistle_plan *P, const double *xyz) {
  const size_t n = (size_t)P->ngeom * 3 * P->ngto;
  if (P->hxyz.size() == n && std::equal(xyz, xyz + n, P->hxyz.begin())) return THISTLE_OK;
  TB_CK(cudaMemcpyAsync(P->d_xyz, xyz, sizeof(double) * n, cudaMemcpyHostToDevice, P->st));
  TB_CK(cudaStreamSynchronize(P->st));
  P->hxyz.assign(xyz, xyz + n);
  P->fwd_valid = false;
  return THISTLE_OK;
}

// Resident stage-2 blocks per SM of every class for the plan's q tile and
// pair tile, and the partial-row count (one row per resident block).  The
// aligned kernel instead takes quartet slices, one partial row each.
void stage2_layout(thistle_plan *P) {
  int maxbps = 1;
  for (int b = 0; b <= LMAXB; ++b) P->s2_bps[b] = 0;
  for (int c = 0; c < P->ncls && P->kind != KIND_ALIGNED; ++c) {
    const int LB = P->cls_L[c] + (kind_j2(P->kind) ? 2 : 0);
    P->s2_bps[LB] = stage2_class_blocks_per_sm(LB, kind_j2(P->kind), P->s2_qtile, P->s2_tile);
    maxbps = std::max(maxbps, P->s2_bps[LB]);
  }
  if (P->kind == KIND_ALIGNED)
    P->s2_rows = std::min(std::max(1, 4 * P->nsm / std::max(1, (P->nq + 127) / 128)), 4 * P->nsm);
  else
    P->s2_rows = P->nsm * maxbps;
}

int plan_create(thistle_plan **out, int32_t type, int32_t ngto, const double *ga, const int32_t *l,
                       const int32_t *m, const int32_t *n, const double *xx, const double *yy, const double *zz,
                       const int32_t *group, const double *mmod, int32_t norbs, const int32_t *mat,
                       const double *total, int32_t nmat, const double *onerdm, int32_t nmo1, const double *q,
                       int32_t nq, double cutoffz, double cutoffmd, double cutoffcentre) {
  if (!out) return fail(THISTLE_ERR_ARG, "null plan pointer");
  *out = nullptr;
  if (type == THISTLE_TOTAL_J1)
    return fail(THISTLE_ERR_TYPE,
                "type 10 (total j1): the reference's tot_integration_j1 stops before integrating "
                "(src/Integrals.f90:526-527), so there is no result to reproduce");
  if (type != THISTLE_TOTAL_J0 && type != THISTLE_ELASTIC_J0 && type != THISTLE_TOTAL_J2 &&
      type != THISTLE_TOTAL_ALIGNED && type != THISTLE_ELASTIC_J2 && type != THISTLE_RESOLVED_CMS)
    return fail(THISTLE_ERR_TYPE, "calculation type " + std::to_string(type) + " is not provided by this entry");
  thistle_plan *P = new thistle_plan();
  int rc = THISTLE_OK;
  std::vector<int64_t> cnt;
  PhaseTrace tr;
  TB_TRY(check_basis(P, ngto, ga, l, m, n, xx, yy, zz, group));
  tr.mark("basis checks");
  if (type == THISTLE_TOTAL_ALIGNED) {
    // q holds nq vectors, (3, nq) column-major like the reference's q_al
    if (!q || nq <= 0) { rc = fail(THISTLE_ERR_ARG, "empty q-vector list"); goto done; }
    if (!finite_all(q, 3 * (int64_t)nq)) { rc = fail(THISTLE_ERR_NONFINITE, "non-finite q vector"); goto done; }
  } else {
    TB_TRY(check_q(q, nq));
  }
  if (!std::isfinite(cutoffz) || !std::isfinite(cutoffmd) || !std::isfinite(cutoffcentre) || cutoffz < 0 ||
      cutoffmd < 0 || cutoffcentre < 0) {
    rc = fail(THISTLE_ERR_ARG, "cutoffs must be finite and non-negative");
    goto done;
  }
  if (!mmod || norbs <= 0) { rc = fail(THISTLE_ERR_ARG, "missing MO coefficients"); goto done; }
  if (!finite_all(mmod, (int64_t)norbs * ngto)) { rc = fail(THISTLE_ERR_NONFINITE, "non-finite MO coefficient"); goto done; }
  P->type = type;
  P->kind = type == THISTLE_TOTAL_J0 ? KIND_TOTAL
            : type == THISTLE_ELASTIC_J0 ? KIND_ELASTIC
            : type == THISTLE_ELASTIC_J2 ? KIND_ELASTIC_J2
            : type == THISTLE_RESOLVED_CMS ? KIND_CMS
            : type == THISTLE_TOTAL_ALIGNED ? KIND_ALIGNED : KIND_J2;
  P->nq = nq;
  P->qdim = type == THISTLE_TOTAL_ALIGNED ? 3 : 1;
  P->hq.assign(q, q + (int64_t)P->qdim * nq);
  P->nmo = norbs;
  P->cutoffz = cutoffz;
  P->cutoffmd = cutoffmd;
  P->cutoffcentre = cutoffcentre;
  P->np = (int64_t)ngto * (ngto + 1) / 2;
  if (kind_elastic(P->kind)) {
    if (!onerdm || nmo1 <= 0 || nmo1 > norbs) { rc = fail(THISTLE_ERR_ARG, "1-RDM must be (nmo1,nmo1) with nmo1 <= norbs"); goto done; }
    P->nzao = P->kind == KIND_CMS ? 2 : 1;  // the resolved CMS takes two 1-RDMs, back to back
    if (!finite_all(onerdm, (int64_t)P->nzao * nmo1 * nmo1)) {
      rc = fail(THISTLE_ERR_NONFINITE, "non-finite 1-RDM");
      goto done;
    }
    P->nmo1 = nmo1;
  } else {
    if (nmat < 0 || (nmat > 0 && (!mat || !total))) { rc = fail(THISTLE_ERR_ARG, "missing 2-RDM rows"); goto done; }
    if (norbs > 215) {
      rc = fail(THISTLE_ERR_ARG, "at most 215 MOs for the 2-RDM transform (norbs^4 must index in 32 bits)");
      goto done;
    }
    {
      // branch-free range pass; the offending row is looked up only on failure
      int32_t lo = 1, hi = 1;
      for (int64_t i = 0; i < (int64_t)nmat * 4; ++i) {
        lo = std::min(lo, mat[i]);
        hi = std::max(hi, mat[i]);
      }
      if (lo < 1 || hi > norbs)
        for (int64_t i = 0; i < (int64_t)nmat * 4; ++i)
          if (mat[i] < 1 || mat[i] > norbs) {
            rc = fail(THISTLE_ERR_SHAPE, "2-RDM index out of range 1..norbs at row " + std::to_string(i % nmat + 1));
            goto done;
          }
    }
    if (nmat > 0 && !finite_all(total, nmat)) { rc = fail(THISTLE_ERR_NONFINITE, "non-finite 2-RDM value"); goto done; }
    P->nmat = nmat;
  }
  tr.mark("density input checks");
  class_counts(P->gL, cnt, P->kind == KIND_CMS);
  tr.mark("class counts");
  TB_TRY(setup_classes(P, cnt, P->kind));
  tr.mark("classes");
  TB_TRYC(cudaStreamCreateWithFlags(&P->st, cudaStreamNonBlocking));
  for (int i = 0; i < 10; ++i) TB_TRYC(cudaEventCreate(&P->ev[i]));
  P->have_ev = true;  // the ring's stage events are made as executions reach their slots
  // the stage-2 streams and their events (made here: executions may be
  // captured into a graph)
  TB_TRYC(cudaStreamCreateWithFlags(&P->st2, cudaStreamNonBlocking));
  TB_TRYC(cudaEventCreateWithFlags(&P->ev_join, cudaEventDisableTiming));
  TB_TRYC(cudaStreamCreateWithFlags(&P->st3, cudaStreamNonBlocking));
  TB_TRYC(cudaEventCreateWithFlags(&P->ev_join3, cudaEventDisableTiming));
  for (int c = 0; c < MAXCLS; ++c) TB_TRYC(cudaEventCreateWithFlags(&P->ev_cls[c], cudaEventDisableTiming));
  tr.mark("stream, events");
  TB_TRY(dalloc(&P->d_gstart, (size_t)P->ng, "groups"));
  TB_TRY(dalloc(&P->d_gcount, (size_t)P->ng, "groups"));
  TB_TRY(dalloc(&P->d_flmn, (size_t)ngto, "functions"));
  TB_TRY(dalloc(&P->d_ga, (size_t)ngto, "exponents"));
  TB_TRY(dalloc(&P->d_q, (size_t)P->qdim * nq, "q"));
  TB_TRYC(cudaMemcpyAsync(P->d_gstart, P->gstart.data(), sizeof(int) * P->ng, cudaMemcpyHostToDevice, P->st));
  TB_TRYC(cudaMemcpyAsync(P->d_gcount, P->gcount.data(), sizeof(int) * P->ng, cudaMemcpyHostToDevice, P->st));
  TB_TRYC(cudaMemcpyAsync(P->d_flmn, P->flmn.data(), sizeof(int) * ngto, cudaMemcpyHostToDevice, P->st));
  TB_TRYC(cudaMemcpyAsync(P->d_ga, ga, sizeof(double) * ngto, cudaMemcpyHostToDevice, P->st));
  if (P->qdim == 3) {
    // (3, nq) column-major = the vectors' components interleaved
    TB_TRYC(cudaMemcpyAsync(P->d_q, q, sizeof(double) * 3 * nq, cudaMemcpyHostToDevice, P->st));
  } else {
    TB_TRYC(cudaMemcpyAsync(P->d_q, q, sizeof(double) * nq, cudaMemcpyHostToDevice, P->st));
  }
  tr.mark("small buffers, uploads");
  TB_TRY(density_alloc(P));
  TB_TRY(density_upload(P, mmod, mat, total, onerdm));
  tr.mark("density buffers");
  TB_TRY(quartets_alloc(P));
  tr.mark("quartet buffers");
  {
    int dev = 0;
    TB_TRYC(cudaGetDevice(&dev));
    TB_TRYC(cudaDeviceGetAttribute(&P->nsm, cudaDevAttrMultiProcessorCount, dev));
    P->s2_qtile = std::min(nq, STAGE2_QTILE);
    stage2_layout(P);
    // contraction buffer of the split contracted-side stage 1: the largest
    // sub-range's quartets x outer pairs x ntuv(LK), up to 2 GB (larger
    // sub-ranges keep the fused kernel)
    {
      int64_t need = 0;
      for (int c = 0; c < P->ncls; ++c) {
        if (!stage1_xk(P->cls_L[c], P->cls_end[c] - P->cls_begin[c], P->nsm)) continue;
        for (const SubRange &u : P->cls_sub[c]) {
          const int64_t x = (u.end - u.begin) * (int64_t)u.nout * ntuv(u.LK);
          if (x <= (int64_t(1) << 28)) need = std::max(need, x);
        }
      }
      if (need > 0) {
        TB_TRY(dalloc(&P->d_xbuf, (size_t)need, "stage-1 contraction buffer"));
        P->xbuf_len = need;
      }
    }
    TB_TRY(geo_alloc(P, 1));
    TB_TRY(upload_centres(P, xx, yy, zz));
    const int64_t n = std::max<int64_t>(P->nquart, 1);
    TB_TRY(dalloc(&P->d_s2key, (size_t)n, "stage-2 keys"));
    TB_TRY(dalloc(&P->d_s2key_sorted, (size_t)n, "stage-2 keys"));
    TB_TRY(dalloc(&P->d_iota, (size_t)n, "quartet indices"));
    TB_TRY(dalloc(&P->d_perm, (size_t)n, "stage-2 order"));
    TB_TRYC(cub::DeviceRadixSort::SortPairs(nullptr, P->s2sort_bytes, P->d_s2key, P->d_s2key_sorted, P->d_iota,
                                            P->d_perm, (int)n, 0, 11, P->st));
    TB_TRY(dalloc((char **)&P->d_s2sort_tmp, P->s2sort_bytes, "stage-2 sort scratch"));
    TB_TRYC(launch_iota(P->d_iota, P->nquart, P->st));
  }
  TB_TRYC(cudaStreamSynchronize(P->st));
  tr.mark("stage-2 buffers");
  P->launches = 0;
  TB_TRYC(cudaEventRecord(P->ev[6], P->st));
  TB_TRY(density_run(P));
  TB_TRYC(cudaEventRecord(P->ev[7], P->st));
  TB_TRY(quartets_run(P));
  TB_TRYC(cudaEventRecord(P->ev[8], P->st));
  TB_TRYC(cudaStreamSynchronize(P->st));
  tr.mark("density transform, quartets");
  {
    float t = 0;
    if (cudaEventElapsedTime(&t, P->ev[6], P->ev[7]) == cudaSuccess) P->ms[4] = t;
    if (cudaEventElapsedTime(&t, P->ev[7], P->ev[8]) == cudaSuccess) P->ms[5] = t;
  }
done:
  if (rc != THISTLE_OK) {
    plan_free(P);
    return rc;
  }
  *out = P;
  return THISTLE_OK;
}

// A tile q[0..n) is "uniform" when q[1..n) is an arithmetic progression to
// within 2e-14 of its largest value; q[0] may sit off it (the drivers put
// 1e-10 where the grid starts at 0).
void grid_info(const double *q, int n, int &uniform, int &first_on_grid, double &dq) {
  uniform = 0;
  first_on_grid = 0;
  dq = 0.0;
  if (n < 4) return;
  dq = (q[n - 1] - q[1]) / (double)(n - 2);
  if (!(dq > 0.0)) return;
  double tol = 2e-14 * std::max(std::fabs(q[n - 1]), std::fabs(q[1]));
  for (int i = 1; i < n; ++i)
    if (std::fabs(q[i] - (q[1] + (double)(i - 1) * dq)) > tol) return;
  uniform = 1;
  first_on_grid = std::fabs(q[0] - (q[1] - dq)) <= tol ? 1 : 0;
}

// Pair tables, stage 1 per class, the stage-2 visiting order (when `order`),
// stage 2 per class and q tile, and the fixed-order reduction into d_out.
// Stage-1 arguments of one class of a quartet list.
Stage1Args stage1_args(const thistle_plan *P, const uint64_t *d_quart, int64_t qbegin, int64_t qend,
                              double *d_rec, int64_t recbase, int rs) {
  Stage1Args a;
  a.quartets = d_quart;
  a.qbegin = qbegin;
  a.qend = qend;
  a.pairtab = P->d_pairtab;
  a.ng = P->ng;
  a.gstart = P->d_gstart;
  a.gcount = P->d_gcount;
  a.flmn = P->d_flmn;
  a.rho = P->d_rho;
  a.np = P->np;
  a.zao = P->d_zao;
  a.zket = P->kind == KIND_CMS ? P->d_zao + (int64_t)P->ngto * P->ngto : P->d_zao;
  a.ngto = P->ngto;
  a.cutoffz = P->cutoffz;
  a.cutoffmd = P->cutoffmd;
  a.cutoffcentre = P->cutoffcentre;
  a.esoa = P->d_esoa;
  a.eskip = esoa_doubles(P->ng, P->maxa) / 2;
  a.emaxa = P->maxa;
  a.npair = npairs(P->ng);
  a.rec = d_rec;
  a.recbase = recbase;
  a.rs = rs;
  a.p0count = nullptr;
  a.s2key = nullptr;
  a.cls = 0;
  a.gs_pair = gs_pair(P);
  a.gs_esoa = gs_esoa(P);
  a.shells_canonical = P->shells_canonical;
  a.gs_rec = gs_rec(P);
  a.xoff = 0;
  a.xstride = 0;
  a.xg = 0;
  return a;
}

#ifndef TB_S2_SIDE_WAVES
#define TB_S2_SIDE_WAVES 16
#endif

int run_stages(thistle_plan *P, const uint64_t *d_quart, const int64_t *cb, const int64_t *ce,
                      const int *cL, int ncls, double *d_rec, const int64_t *recoff, const int *rs,
                      const std::vector<SubRange> *subs, double *d_out, bool order, int ngeom,
                      const std::vector<TupleRange> *tups) {
  // stage events (not while a graph is being captured); a ring slot's events
  // are made the first time an execution reaches it
  const int slot = (int)(P->ring_next % thistle_plan::NRING);
  if (!P->capturing && slot >= P->rev_made) {
    for (int i = 0; i < 6; ++i) TB_CK(cudaEventCreate(&P->rev[slot][i]));
    P->rev_made = slot + 1;
  }
  cudaEvent_t *E = P->rev[slot];
  auto mark = [&](int i) -> cudaError_t { return P->capturing ? cudaSuccess : cudaEventRecord(E[i], P->st); };
  if (!P->capturing) P->ring_next += 1;
  TB_CK(mark(0));
  TB_CK(launch_pair_tables(P->ng, P->maxa, P->d_gstart, P->d_flmn, P->d_ga, P->d_xyz, P->d_pairtab, P->d_esoa,
                           ngeom, 3 * (int64_t)P->ngto, gs_pair(P), gs_esoa(P), P->st));
  P->launches += 1;
  TB_CK(cudaMemsetAsync(P->d_p0count, 0, sizeof(int64_t) * MAXCLS * ngeom, P->st));
  const bool aligned = P->kind == KIND_ALIGNED;
  if (!aligned)
    TB_CK(cudaMemsetAsync(P->d_partial, 0, sizeof(double) * (size_t)2 * P->s2_rows * P->nq * ngeom, P->st));
  // Pipelined stages: each class's visiting order is sorted right after its
  // stage 1 (its keys, bits 0-5: the H bucket; the stable radix sort gives the
  // order the sort over all quartets by (class, bucket) gives), so its stage 2
  // may start while the later classes' stage 1 runs.  Needs each class's sort
  // to fit the scratch sized for the whole sort.
  bool pipe = P->pipeline && order && !aligned;
  for (int c = 0; c < ncls && pipe; ++c) {
    size_t need = 0;
    if (ce[c] > cb[c])
      TB_CK(cub::DeviceRadixSort::SortPairs(nullptr, need, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                            (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)(ce[c] - cb[c]), 0,
                                            6, P->st));
    pipe = need <= P->s2sort_bytes;
  }
  bool m5 = false;  // E5: the first class's stage 2 may start
  TB_CK(mark(1));
  for (int c = 0; c < ncls; ++c) {
    Stage1Args a = stage1_args(P, d_quart, cb[c], ce[c], d_rec, recoff[c], rs[c]);
    a.p0count = (unsigned long long *)(P->d_p0count + c);
    a.s2key = (order && P->kind != KIND_ALIGNED) ? P->d_s2key : nullptr;
    a.cls = c;
    if (tups && stage1_tpl(P->kind, cL[c], P->shells_canonical)) {
      // shell-templated kernels, one launch per shell tuple of the class
      for (const TupleRange &u : tups[c]) {
        Stage1Args b = a;
        b.qbegin = u.begin;
        b.qend = u.end;
        b.recbase = recoff[c] + (u.begin - cb[c]) * (int64_t)rs[c];
        TB_CK(launch_stage1_tpl(P->kind, u.tuple, b, ngeom, P->st));
        P->launches += 1;
      }
    } else if (stage1_xk(cL[c], (ce[c] - cb[c]) * ngeom, P->nsm)) {
      for (const SubRange &u : subs[c]) {
        Stage1Args b = a;
        b.qbegin = u.begin;
        b.qend = u.end;
        b.recbase = recoff[c] + (u.begin - cb[c]) * (int64_t)rs[c];
        const int64_t need = (u.end - u.begin) * (int64_t)u.nout * ntuv(u.LK);
        if (ngeom == 1 && u.nout > 0 && P->d_xbuf && need <= P->xbuf_len) {
          if (tups && stage1_xct(P->kind, u.LK, P->shells_canonical)) {
            // the contraction per shell tuple (templated), then the
            // convolution of the whole sub-range from the same buffer
            for (const TupleRange &w : tups[c]) {
              if (w.begin < u.begin || w.end > u.end) continue;
              Stage1Args bt = b;
              bt.qbegin = w.begin;
              bt.qend = w.end;
              TB_CK(launch_stage1_xct(P->kind, w.tuple, u.XB != 0, bt, P->d_xbuf, u.nout * ntuv(u.LK), u.begin,
                                      P->st));
              P->launches += 1;
            }
            TB_CK(launch_stage1_xsplit(P->kind, cL[c], u.LK, u.XB != 0, b, P->d_xbuf, u.nout, P->st, false));
            P->launches += 1;
          } else {
            TB_CK(launch_stage1_xsplit(P->kind, cL[c], u.LK, u.XB != 0, b, P->d_xbuf, u.nout, P->st));
            P->launches += 2;
          }
        } else {
          TB_CK(launch_stage1_xk(P->kind, cL[c], u.LK, u.XB != 0, b, ngeom, P->st));
          P->launches += 1;
        }
      }
    } else {
      TB_CK(launch_stage1(P->kind, cL[c], a, ngeom, P->st));
      P->launches += 1;
    }
    if (pipe && ce[c] > cb[c]) {
      size_t bytes = P->s2sort_bytes;
      TB_CK(cub::DeviceRadixSort::SortPairs(P->d_s2sort_tmp, bytes, P->d_s2key + cb[c], P->d_s2key_sorted + cb[c],
                                            P->d_iota + cb[c], P->d_perm + cb[c], (int)(ce[c] - cb[c]), 0, 6,
                                            P->st));
      P->launches += 1;
      TB_CK(cudaEventRecord(P->ev_cls[c], P->st));
      if (!m5) TB_CK(mark(5));
      m5 = true;
    }
  }
  TB_CK(mark(2));
  if (aligned) TB_CK(mark(5));
  int64_t nall = ncls > 0 ? ce[ncls - 1] : 0;
  if (P->kind == KIND_ALIGNED) {
    TB_CK(cudaMemsetAsync(P->d_partial, 0, sizeof(double) * (size_t)P->s2_rows * P->nq, P->st));
    for (int c = 0; c < ncls; ++c) {
      AlignedArgs s;
      s.rec = d_rec + recoff[c];
      s.rs = rs[c];
      s.nquart = ce[c] - cb[c];
      s.qv = P->d_q;
      s.nq = P->nq;
      s.partial = P->d_partial;
      s.pstride = P->nq;
      const int slices = (int)std::max<int64_t>(1, std::min<int64_t>(P->s2_rows, (s.nquart + 31) / 32));
      TB_CK(launch_aligned(cL[c], s, slices, P->st));
      P->launches += 1;
    }
    TB_CK(mark(3));
    TB_CK(launch_reduce(P->d_partial, P->s2_rows, P->nq, d_out, P->st));
    P->launches += 1;
    TB_CK(mark(4));
    return THISTLE_OK;
  }
  if (!pipe) {
    if (order && nall > 0) {
      size_t bytes = P->s2sort_bytes;
      TB_CK(cub::DeviceRadixSort::SortPairs(P->d_s2sort_tmp, bytes, P->d_s2key, P->d_s2key_sorted, P->d_iota,
                                            P->d_perm, (int)nall, 0, 11, P->st));
      P->launches += 1;
    }
    // every class's stage 2 waits for the whole of stage 1 (and the sort)
    for (int c = 0; c < ncls; ++c) TB_CK(cudaEventRecord(P->ev_cls[c], P->st));
  }
  if (!m5) TB_CK(mark(5));
  // classes with fewer warp batches than TB_S2_SIDE_WAVES waves of resident
  // warps run on the side stream st2, the others on st3, so the small classes
  // overlap the large ones instead of leaving most of the GPU idle; the
  // side-stream classes add into the second block of partial rows
  const int64_t prow = (int64_t)P->s2_rows * P->nq;
  auto small_class = [&](int c) {
    const int LB = cL[c] + (kind_j2(P->kind) ? 2 : 0);
    const int64_t per_warp = stage2_quartets_per_warp(LB, P->s2_tile);
    const int bps = P->s2_bps[LB] > 0 ? P->s2_bps[LB] : 1;
    return (ce[c] - cb[c] + per_warp - 1) / per_warp * ngeom < (int64_t)TB_S2_SIDE_WAVES * P->nsm * bps * P->s2_tile.nw;
  };
  bool used2 = false, used3 = false;
  for (int q0 = 0; q0 < P->nq; q0 += P->s2_qtile) {
    const int tn = std::min(P->s2_qtile, P->nq - q0);
    int uniform = 0, first_on_grid = 0;
    double dq = 0.0;
    grid_info(P->hq.data() + q0, tn, uniform, first_on_grid, dq);
    for (int c = 0; c < ncls; ++c) {
      if (ce[c] <= cb[c]) continue;
      const int LB = cL[c] + (kind_j2(P->kind) ? 2 : 0);
      Stage2ClassArgs s;
      s.rec = d_rec + recoff[c];
      s.rs = rs[c];
      s.nquart = ce[c] - cb[c];
      s.perm = order ? P->d_perm : nullptr;
      s.gs_rec = gs_rec(P);
      s.gs_partial = 2 * prow;
      s.pbase = cb[c];
      s.q = P->d_q + q0;
      s.nq = tn;
      s.uniform = uniform;
      s.first_on_grid = first_on_grid;
      s.dq = dq;
      s.j2 = kind_j2(P->kind);
      s.lb = LB;
      const bool side = small_class(c);
      s.partial = P->d_partial + (side ? prow : 0) + q0;
      s.pstride = P->nq;
      // a class too small to fill the GPU several times over is also split
      // over q, in chunks of 64 points (the reseed interval)
      const int64_t per_warp = stage2_quartets_per_warp(LB, P->s2_tile);
      const int NW = P->s2_tile.nw;
      const int bps = P->s2_bps[LB] > 0 ? P->s2_bps[LB] : 1;
      const int64_t resident = (int64_t)P->nsm * bps * NW;
      const int64_t nbatch = (s.nquart + per_warp - 1) / per_warp * ngeom;
      const int nseg = (tn + 63) / 64;
      int nch = (int)std::min<int64_t>(nseg, std::max<int64_t>(1, (8 * resident + nbatch - 1) / nbatch));
      s.chunk = nch <= 1 ? 0 : 64 * ((nseg + nch - 1) / nch);
      if (s.chunk > 0) nch = (tn + s.chunk - 1) / s.chunk;
      const int64_t items = nbatch / ngeom * nch;
      const int64_t nblk = (items + NW - 1) / NW;
      const int grid = (int)std::min<int64_t>(nblk, std::min(P->s2_rows, P->nsm * bps));
      if (grid <= 0) continue;
      cudaStream_t sc = side ? P->st2 : P->st3;
      TB_CK(cudaStreamWaitEvent(sc, P->ev_cls[c], 0));
      (side ? used2 : used3) = true;
      TB_CK(launch_stage2_class(LB, s, grid, ngeom, P->s2_tile, sc));
      P->launches += 1;
    }
  }
  if (used2) {
    TB_CK(cudaEventRecord(P->ev_join, P->st2));
    TB_CK(cudaStreamWaitEvent(P->st, P->ev_join, 0));
  }
  if (used3) {
    TB_CK(cudaEventRecord(P->ev_join3, P->st3));
    TB_CK(cudaStreamWaitEvent(P->st, P->ev_join3, 0));
  }
  TB_CK(mark(3));
  TB_CK(launch_reduce_batch(P->d_partial, 2 * P->s2_rows, P->nq, 2 * prow, d_out, ngeom, P->st));
  P->launches += 1;
  TB_CK(mark(4));
  return THISTLE_OK;
}

int plan_exec(thistle_plan *P, double *d_out) {
  int rc = run_stages(P, P->d_quart, P->cls_begin, P->cls_end, P->cls_L, P->ncls, P->d_rec, P->cls_recoff,
                      P->cls_rs, P->cls_sub, d_out, true, P->ngeom, P->cls_tup);
  P->fwd_valid = rc == THISTLE_OK;
  return rc;
}

// Stage intervals of one execution's ring events: pair tables E0-E1, stage 1
// E1-E2, stage 2 E5-E3 (from the moment the first class's stage 2 may start:
// it overlaps the later classes' stage 1), reduction E3-E4.
static const int kStageFrom[4] = {0, 1, 5, 3}, kStageTo[4] = {1, 2, 3, 4};

void read_timings(thistle_plan *P) {
  if (P->ring_next == 0) return;
  cudaEvent_t *E = P->rev[(P->ring_next - 1) % thistle_plan::NRING];
  for (int i = 0; i < 4; ++i) {
    float t = 0;
    if (cudaEventElapsedTime(&t, E[kStageFrom[i]], E[kStageTo[i]]) == cudaSuccess) P->ms[i] = t;
  }
}

// Vector-Jacobian product of total j0 with respect to the group centres:
// grad[g][3 c + axis] = sum_q v[g](q) dI_g(q)/dA_c for every geometry g of the
// batch (tb_adjoint.cu).  The forward records must be those of the current
// centres (adjoint_ready runs the forward stages otherwise).
int adjoint_check(thistle_plan *P) {
  if (P->kind != KIND_TOTAL) return fail(THISTLE_ERR_TYPE, "the adjoint is provided for total j0 (type 1)");
  for (int c = 0; c < P->ncls; ++c)
    if (P->cls_L[c] > 8) return fail(THISTLE_ERR_ANGMOM, "the adjoint covers LLmax <= 8 (s, p, d shells)");
  return THISTLE_OK;
}

int adjoint_alloc(thistle_plan *P) {
  int rc = THISTLE_OK;
  const int G = P->ngeom;
  if (!P->d_dsoa) {
    TB_TRY(dalloc(&P->d_dsoa, (size_t)G * dsoa_doubles(P->ng, P->maxa), "dE tables"));
    TB_TRY(dalloc(&P->d_adj, (size_t)G * gs_rec(P), "adjoint records"));
    // partial gradient rows = the most stage-B blocks of a launch (8 per SM;
    // at their register count about 4 are resident)
    P->adj_rows = 8 * P->nsm;
    TB_TRY(dalloc(&P->d_gpart, (size_t)G * P->adj_rows * 3 * P->ng, "gradient rows"));
  }
  if (!P->d_v) {
    TB_TRY(dalloc(&P->d_v, (size_t)G * P->nq, "cotangent"));
    TB_TRY(dalloc(&P->d_grad, (size_t)G * 3 * P->ng, "gradient"));
  }
done:
  return rc;
}

// The adjoint stages proper (no allocation, no synchronisation: capturable).
int adjoint_stages(thistle_plan *P, const double *d_v, double *d_grad) {
  int rc = THISTLE_OK;
  const int G = P->ngeom;
  const int64_t gs_dsoa = dsoa_doubles(P->ng, P->maxa), gs_gpart = (int64_t)P->adj_rows * 3 * P->ng;
  TB_TRYC(launch_pair_dtables(P->ng, P->maxa, P->d_gstart, P->d_ga, P->d_xyz, P->d_dsoa, G, 3 * (int64_t)P->ngto,
                              gs_dsoa, P->st));
  P->launches += 1;
  {
    int uniform = 0, first_on_grid = 0;
    double dq = 0.0;
    grid_info(P->hq.data(), P->nq, uniform, first_on_grid, dq);
    for (int c = 0; c < P->ncls; ++c) {
      AdjointQArgs a;
      a.rec = P->d_rec + P->cls_recoff[c];
      a.adj = P->d_adj + P->cls_recoff[c];
      a.rs = P->cls_rs[c];
      a.nquart = P->cls_end[c] - P->cls_begin[c];
      a.perm = P->d_perm;
      a.pbase = P->cls_begin[c];
      a.q = P->d_q;
      a.v = d_v;
      a.nq = P->nq;
      a.uniform = uniform;
      a.first_on_grid = first_on_grid;
      a.dq = dq;
      a.gs_rec = gs_rec(P);
      TB_TRYC(launch_adjoint_q(P->cls_L[c] + 1, a, G, P->st));
      P->launches += 1;
    }
  }
  TB_TRYC(cudaMemsetAsync(P->d_gpart, 0, sizeof(double) * (size_t)G * gs_gpart, P->st));
  for (int c = 0; c < P->ncls; ++c) {
    AdjointFArgs a;
    a.s1 = stage1_args(P, P->d_quart, P->cls_begin[c], P->cls_end[c], P->d_rec, P->cls_recoff[c], P->cls_rs[c]);
    a.adj = P->d_adj;
    a.dsoa = P->d_dsoa;
    a.ga = P->d_ga;
    a.xyz = P->d_xyz;
    a.gpart = P->d_gpart;
    a.gstride = 3 * P->ng;
    a.gs_dsoa = gs_dsoa;
    a.gs_xyz = 3 * (int64_t)P->ngto;
    a.gs_gpart = gs_gpart;
    const int64_t n = P->cls_end[c] - P->cls_begin[c];
    // a class with too few quartets (over all geometries) to keep every SM
    // busy several times over splits each quartet across a thread group
    const bool split = n * G < (int64_t)4 * P->nsm * 64;
    const int qpb = adjoint_f_quartets_per_block(P->cls_L[c], split);
    const int grid = (int)std::min<int64_t>(P->adj_rows, (n + qpb - 1) / qpb);
    TB_TRYC(launch_adjoint_f(P->cls_L[c], a, grid, G, split, P->st));
    P->launches += 1;
  }
  TB_TRYC(launch_reduce_batch(P->d_gpart, P->adj_rows, 3 * P->ng, gs_gpart, d_grad, G, P->st));
  P->launches += 1;
done:
  return rc;
}

// Forward stages of the batch into d_result, through the captured graph when enabled.
int forward_batch(thistle_plan *P) {
  if (!P->use_graph) return plan_exec(P, P->d_result);
  if (!P->gx_fwd) {
    // capture once (all buffers exist); replays use the same pointers
    cudaGraph_t g = nullptr;
    TB_CK(cudaStreamBeginCapture(P->st, cudaStreamCaptureModeThreadLocal));
    P->capturing = true;
    int rc = run_stages(P, P->d_quart, P->cls_begin, P->cls_end, P->cls_L, P->ncls, P->d_rec, P->cls_recoff,
                        P->cls_rs, P->cls_sub, P->d_result, true, P->ngeom, P->cls_tup);
    P->capturing = false;
    cudaError_t e = cudaStreamEndCapture(P->st, &g);
    if (rc != THISTLE_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    TB_CK(e);
    e = cudaGraphInstantiate(&P->gx_fwd, g, 0);
    cudaGraphDestroy(g);
    TB_CK(e);
  }
  TB_CK(cudaGraphLaunch(P->gx_fwd, P->st));
  P->fwd_valid = true;
  return THISTLE_OK;
}

int plan_vjp(thistle_plan *P, const double *d_v, double *d_grad) {
  int rc = adjoint_check(P);
  if (rc != THISTLE_OK) return rc;
  TB_TRY(adjoint_alloc(P));
  if (!P->fwd_valid) TB_TRY(forward_batch(P));
  if (!P->use_graph || d_v != P->d_v || d_grad != P->d_grad) {
    TB_TRY(adjoint_stages(P, d_v, d_grad));
  } else {
    if (!P->gx_vjp) {
      cudaGraph_t g = nullptr;
      TB_TRYC(cudaStreamBeginCapture(P->st, cudaStreamCaptureModeThreadLocal));
      P->capturing = true;
      rc = adjoint_stages(P, d_v, d_grad);
      P->capturing = false;
      cudaError_t e = cudaStreamEndCapture(P->st, &g);
      if (rc != THISTLE_OK) {
        if (g) cudaGraphDestroy(g);
        goto done;
      }
      TB_TRYC(e);
      e = cudaGraphInstantiate(&P->gx_vjp, g, 0);
      cudaGraphDestroy(g);
      TB_TRYC(e);
    }
    TB_TRYC(cudaGraphLaunch(P->gx_vjp, P->st));
  }
done:
  return rc;
}

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

int thistle_plan_vjp(thistle_plan *P, const double *v_host, double *grad_host) {
  if (!P || !v_host || !grad_host) return fail(THISTLE_ERR_ARG, "null argument");
  if (!finite_all(v_host, P->nq)) return fail(THISTLE_ERR_NONFINITE, "non-finite cotangent");
  P->launches = 0;
  int rc = adjoint_check(P);
  if (rc != THISTLE_OK) return rc;
  if (P->ngeom != 1) return fail(THISTLE_ERR_SHAPE, "plan holds a geometry batch: use thistle_plan_vjp_batch");
  TB_TRY(adjoint_alloc(P));
  TB_TRYC(cudaMemcpyAsync(P->d_v, v_host, sizeof(double) * P->nq, cudaMemcpyHostToDevice, P->st));
  TB_TRY(plan_vjp(P, P->d_v, P->d_grad));
  TB_TRYC(cudaMemcpyAsync(grad_host, P->d_grad, sizeof(double) * 3 * P->ng, cudaMemcpyDeviceToHost, P->st));
  TB_TRYC(cudaStreamSynchronize(P->st));
done:
  return rc;
}

int thistle_plan_set_batch(thistle_plan *P, int32_t ngeom) {
  if (!P) return fail(THISTLE_ERR_ARG, "null plan");
  if (ngeom < 1 || ngeom > 65535) return fail(THISTLE_ERR_ARG, "ngeom must be 1..65535");
  if (P->kind == KIND_ALIGNED && ngeom != 1) return fail(THISTLE_ERR_TYPE, "aligned plans hold one geometry");
  if (P->kind == KIND_CMS && ngeom != 1) return fail(THISTLE_ERR_TYPE, "resolved CMS plans hold one geometry");
  if (ngeom == P->ngeom) return THISTLE_OK;
  TB_CK(cudaStreamSynchronize(P->st));
  // every geometry starts at geometry 0's centres
  std::vector<double> g0(P->hxyz.begin(), P->hxyz.begin() + 3 * (size_t)P->ngto);
  int rc = geo_alloc(P, ngeom);
  if (rc != THISTLE_OK) return rc;
  std::vector<double> all((size_t)ngeom * g0.size());
  for (int g = 0; g < ngeom; ++g) std::copy(g0.begin(), g0.end(), all.begin() + (size_t)g * g0.size());
  P->hxyz.clear();
  return upload_centres_batch(P, all.data());
}

int thistle_plan_set_centres_batch(thistle_plan *P, const double *xyz) {
  if (!P || !xyz) return fail(THISTLE_ERR_ARG, "null argument");
  const int64_t n = (int64_t)P->ngeom * 3 * P->ngto;
  if (!finite_all(xyz, n)) return fail(THISTLE_ERR_NONFINITE, "non-finite centre");
  for (int g = 0; g < P->ngeom; ++g)
    for (int k = 0; k < P->ng; ++k) {
      const double *h = xyz + ((size_t)g * P->ngto + P->gstart[k]) * 3;
      for (int i = P->gstart[k]; i < P->gstart[k] + P->gcount[k]; ++i)
        for (int ax = 0; ax < 3; ++ax)
          if (xyz[((size_t)g * P->ngto + i) * 3 + ax] != h[ax])
            return fail(THISTLE_ERR_SHAPE, "functions of one group must share a centre");
    }
  return upload_centres_batch(P, xyz);
}

int thistle_plan_set_centres_batch_device(thistle_plan *P, const double *xyz_dev) {
  if (!P || !xyz_dev) return fail(THISTLE_ERR_ARG, "null argument");
  TB_CK(cudaMemcpyAsync(P->d_xyz, xyz_dev, sizeof(double) * (size_t)P->ngeom * 3 * P->ngto,
                        cudaMemcpyDeviceToDevice, P->st));
  P->hxyz.clear();  // the host copy no longer describes the device centres
  P->fwd_valid = false;
  return THISTLE_OK;
}
int thistle_plan_execute_batch_device(thistle_plan *P, double *result_dev) {
  if (!P || !result_dev) return fail(THISTLE_ERR_ARG, "null argument");
  P->launches = 0;
  int rc = forward_batch(P);
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaMemcpyAsync(result_dev, P->d_result, sizeof(double) * P->ngeom * P->nq, cudaMemcpyDeviceToDevice,
                        P->st));
  return THISTLE_OK;
}

int thistle_plan_execute_batch(thistle_plan *P, double *result_host) {
  if (!P || !result_host) return fail(THISTLE_ERR_ARG, "null argument");
  P->launches = 0;
  int rc = forward_batch(P);
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaMemcpyAsync(result_host, P->d_result, sizeof(double) * P->ngeom * P->nq, cudaMemcpyDeviceToHost,
                        P->st));
  TB_CK(cudaStreamSynchronize(P->st));
  return THISTLE_OK;
}

int thistle_plan_vjp_batch(thistle_plan *P, const double *v_host, double *grad_host) {
  if (!P || !v_host || !grad_host) return fail(THISTLE_ERR_ARG, "null argument");
  if (!finite_all(v_host, (int64_t)P->ngeom * P->nq)) return fail(THISTLE_ERR_NONFINITE, "non-finite cotangent");
  P->launches = 0;
  int rc = adjoint_check(P);
  if (rc != THISTLE_OK) return rc;
  TB_TRY(adjoint_alloc(P));
  TB_TRYC(cudaMemcpyAsync(P->d_v, v_host, sizeof(double) * P->ngeom * P->nq, cudaMemcpyHostToDevice, P->st));
  TB_TRY(plan_vjp(P, P->d_v, P->d_grad));
  TB_TRYC(cudaMemcpyAsync(grad_host, P->d_grad, sizeof(double) * P->ngeom * 3 * P->ng, cudaMemcpyDeviceToHost,
                          P->st));
  TB_TRYC(cudaStreamSynchronize(P->st));
done:
  return rc;
}

int thistle_plan_vjp_batch_device(thistle_plan *P, const double *v_dev, double *grad_dev) {
  if (!P || !v_dev || !grad_dev) return fail(THISTLE_ERR_ARG, "null argument");
  P->launches = 0;
  int rc = adjoint_check(P);
  if (rc != THISTLE_OK) return rc;
  TB_TRY(adjoint_alloc(P));
  TB_TRYC(cudaMemcpyAsync(P->d_v, v_dev, sizeof(double) * P->ngeom * P->nq, cudaMemcpyDeviceToDevice, P->st));
  TB_TRY(plan_vjp(P, P->d_v, P->d_grad));
  TB_TRYC(cudaMemcpyAsync(grad_dev, P->d_grad, sizeof(double) * P->ngeom * 3 * P->ng, cudaMemcpyDeviceToDevice,
                          P->st));
done:
  return rc;
}

// Stage-2 q tile (points per shared-memory tile) or pair tile changed:
// recompute the resident blocks per class and the partial-row count, and
// reallocate the partial sums (the only buffer sized by it).  Centres,
// records and captured graphs of other shapes are dropped or kept as they
// stay valid: the records do, the graphs do not.
static int stage2_relayout(thistle_plan *P) {
  TB_CK(cudaStreamSynchronize(P->st));
  drop_graphs(P);
  stage2_layout(P);
  dfree(P->d_partial);
  P->d_partial = nullptr;
  return dalloc(&P->d_partial, (size_t)P->ngeom * 2 * P->s2_rows * P->nq, "partial sums");
}

static int set_qtile(thistle_plan *P, int qt) {
  P->s2_qtile = std::max(1, std::min(qt, std::min(P->nq, STAGE2_QTILE)));
  return stage2_relayout(P);
}

static int set_tile(thistle_plan *P, Stage2Tile t) {
  P->s2_tile = t;
  return stage2_relayout(P);
}

// Geometries per second of forward + adjoint at the plan's current shape
// (3 timed runs after 2 untimed ones), or a negative status.
static int time_batch(thistle_plan *P, cudaEvent_t e0, cudaEvent_t e1, double *gps) {
  const int reps = 3;
  int rc = adjoint_alloc(P);
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaMemsetAsync(P->d_v, 0, sizeof(double) * P->ngeom * P->nq, P->st));
  for (int w = 0; w < 2 + reps && rc == THISTLE_OK; ++w) {
    if (w == 2) TB_CK(cudaEventRecord(e0, P->st));
    P->fwd_valid = false;
    rc = forward_batch(P);
    if (rc == THISTLE_OK) rc = plan_vjp(P, P->d_v, P->d_grad);
  }
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaEventRecord(e1, P->st));
  TB_CK(cudaEventSynchronize(e1));
  float ms = 0;
  TB_CK(cudaEventElapsedTime(&ms, e0, e1));
  *gps = ms > 0 ? P->ngeom * reps / (ms * 1e-3) : 0.0;
  return THISTLE_OK;
}

int thistle_plan_autotune_batch(thistle_plan *P, int32_t gmax, int32_t *g_best, int32_t *qtile_best,
                                double *geoms_per_s) {
  if (!P || !g_best || !qtile_best || !geoms_per_s) return fail(THISTLE_ERR_ARG, "null argument");
  if (gmax < 1) return fail(THISTLE_ERR_ARG, "gmax must be >= 1");
  int rc = adjoint_check(P);
  if (rc != THISTLE_OK) return rc;
  const int qfull = std::min(P->nq, STAGE2_QTILE);
  int qts[2] = {qfull, std::max(64, (qfull / 2 + 63) / 64 * 64)};
  const int nqt = qts[1] < qfull ? 2 : 1;
  const Stage2Tile tiles[4] = {{2, 4}, {2, 8}, {1, 4}, {1, 8}};
  double best = -1.0;
  int bestG = 1, bestQ = qfull;
  Stage2Tile bestT = tiles[0];
  cudaEvent_t e0, e1;
  TB_CK(cudaEventCreate(&e0));
  TB_CK(cudaEventCreate(&e1));
  // batch size and q tile at the default pair tile, then the pair tiles at
  // the best of those
  rc = set_tile(P, tiles[0]);
  for (int G = 1; G <= gmax && rc == THISTLE_OK; G *= 2) {
    bool fits = true;
    for (int t = 0; t < nqt && fits; ++t) {
      rc = thistle_plan_set_batch(P, G);
      if (rc == THISTLE_OK) rc = set_qtile(P, qts[t]);
      double gps = 0.0;
      if (rc == THISTLE_OK) rc = time_batch(P, e0, e1, &gps);
      if (rc == THISTLE_ERR_NOMEM) {
        fits = false;  // no room for this batch: keep the best so far
        rc = THISTLE_OK;
        break;
      }
      if (rc != THISTLE_OK) break;
      if (gps > best) {
        best = gps;
        bestG = G;
        bestQ = qts[t];
      }
    }
    if (!fits) break;
  }
  if (rc == THISTLE_OK) rc = thistle_plan_set_batch(P, bestG);
  if (rc == THISTLE_OK) rc = set_qtile(P, bestQ);
  for (int t = 1; t < 4 && rc == THISTLE_OK; ++t) {
    rc = set_tile(P, tiles[t]);
    double gps = 0.0;
    if (rc == THISTLE_OK) rc = time_batch(P, e0, e1, &gps);
    if (rc == THISTLE_OK && gps > best) {
      best = gps;
      bestT = tiles[t];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != THISTLE_OK) return rc;
  TB_TRY(set_tile(P, bestT));
  *g_best = bestG;
  *qtile_best = bestQ;
  *geoms_per_s = best;
done:
  return rc;
}

int thistle_plan_set_stage2_tile(thistle_plan *P, int32_t quartets_per_lane, int32_t warps_per_block) {
  if (!P) return fail(THISTLE_ERR_ARG, "null plan");
  const Stage2Tile t{quartets_per_lane, warps_per_block};
  if (!stage2_tile_valid(t)) return fail(THISTLE_ERR_ARG, "stage-2 tile: quartets per lane 1 or 2, warps 4 or 8");
  if (P->kind == KIND_ALIGNED) return fail(THISTLE_ERR_TYPE, "aligned plans have no stage-2 pair tile");
  if (t.k == P->s2_tile.k && t.nw == P->s2_tile.nw) return THISTLE_OK;
  return set_tile(P, t);
}

int thistle_plan_stage2_tile(const thistle_plan *P, int32_t *quartets_per_lane, int32_t *warps_per_block) {
  if (!P || !quartets_per_lane || !warps_per_block) return fail(THISTLE_ERR_ARG, "null argument");
  *quartets_per_lane = P->s2_tile.k;
  *warps_per_block = P->s2_tile.nw;
  return THISTLE_OK;
}

int thistle_plan_set_pipeline(thistle_plan *P, int32_t enable) {
  if (!P) return fail(THISTLE_ERR_ARG, "null plan");
  TB_CK(cudaStreamSynchronize(P->st));
  drop_graphs(P);
  P->pipeline = enable != 0;
  return THISTLE_OK;
}

int thistle_plan_use_graph(thistle_plan *P, int32_t enable) {
  if (!P) return fail(THISTLE_ERR_ARG, "null plan");
  TB_CK(cudaStreamSynchronize(P->st));
  drop_graphs(P);
  P->use_graph = enable != 0;
  return THISTLE_OK;
}

int thistle_plan_vjp_device(thistle_plan *P, const double *v_dev, double *grad_dev) {
  if (!P || !v_dev || !grad_dev) return fail(THISTLE_ERR_ARG, "null argument");
  if (P->ngeom != 1) return fail(THISTLE_ERR_SHAPE, "plan holds a geometry batch: use thistle_plan_vjp_batch_device");
  P->launches = 0;
  return plan_vjp(P, v_dev, grad_dev);
}

int thistle_plan_execute_aligned(thistle_plan *P, double *re_host, double *im_host) {
  if (!P || !re_host) return fail(THISTLE_ERR_ARG, "null argument");
  if (P->kind != KIND_ALIGNED) return fail(THISTLE_ERR_TYPE, "not an aligned plan (type 3)");
  P->launches = 0;
  int rc = plan_exec(P, P->d_result);
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaMemcpyAsync(re_host, P->d_result, sizeof(double) * P->nq, cudaMemcpyDeviceToHost, P->st));
  TB_CK(cudaStreamSynchronize(P->st));
  // the ordered quartet sum is real: bra-ket exchange conjugates each term
  if (im_host)
    for (int i = 0; i < P->nq; ++i) im_host[i] = 0.0;
  read_timings(P);
  return THISTLE_OK;
}

const char *thistle_last_error_string(void) { return g_err.c_str(); }

int thistle_version(void) { return 100; }

int thistle_plan_create(thistle_plan **plan, int32_t type, int32_t ngto, const double *ga, const int32_t *l,
                        const int32_t *m, const int32_t *n, const double *xx, const double *yy, const double *zz,
                        const int32_t *group, const double *mmod, int32_t norbs, const int32_t *mat,
                        const double *total, int32_t nmat, const double *onerdm, int32_t nmo1, const double *q,
                        int32_t nq, double cutoffz, double cutoffmd, double cutoffcentre) {
  return plan_create(plan, type, ngto, ga, l, m, n, xx, yy, zz, group, mmod, norbs, mat, total, nmat, onerdm, nmo1,
                     q, nq, cutoffz, cutoffmd, cutoffcentre);
}

int thistle_plan_set_stream(thistle_plan *P, void *stream) {
  if (!P) return fail(THISTLE_ERR_ARG, "null plan");
  TB_CK(cudaStreamSynchronize(P->st));
  if (P->own_stream) cudaStreamDestroy(P->st);
  P->st = (cudaStream_t)stream;
  P->own_stream = false;
  return THISTLE_OK;
}

int thistle_plan_set_centres(thistle_plan *P, const double *xx, const double *yy, const double *zz) {
  if (!P || !xx || !yy || !zz) return fail(THISTLE_ERR_ARG, "null argument");
  if (!finite_all(xx, P->ngto) || !finite_all(yy, P->ngto) || !finite_all(zz, P->ngto))
    return fail(THISTLE_ERR_NONFINITE, "non-finite centre");
  for (int g = 0; g < P->ng; ++g) {
    int h = P->gstart[g];
    for (int i = h; i < h + P->gcount[g]; ++i)
      if (xx[i] != xx[h] || yy[i] != yy[h] || zz[i] != zz[h])
        return fail(THISTLE_ERR_SHAPE, "functions of one group must share a centre");
  }
  return upload_centres(P, xx, yy, zz);
}

int thistle_plan_execute_device(thistle_plan *P, double *result_dev) {
  if (!P || !result_dev) return fail(THISTLE_ERR_ARG, "null argument");
  P->launches = 0;
  return plan_exec(P, result_dev);
}

int thistle_plan_recompute_device(thistle_plan *P, double *result_dev) {
  if (!P || !result_dev) return fail(THISTLE_ERR_ARG, "null argument");
  P->launches = 0;
  TB_CK(cudaEventRecord(P->ev[6], P->st));
  int rc = density_run(P);
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaEventRecord(P->ev[7], P->st));
  rc = quartets_run(P);
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaEventRecord(P->ev[8], P->st));
  return plan_exec(P, result_dev);
}

int thistle_plan_execute(thistle_plan *P, double *result_host) {
  if (!P || !result_host) return fail(THISTLE_ERR_ARG, "null argument");
  P->launches = 0;
  int rc = plan_exec(P, P->d_result);
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaMemcpyAsync(result_host, P->d_result, sizeof(double) * P->nq, cudaMemcpyDeviceToHost, P->st));
  TB_CK(cudaStreamSynchronize(P->st));
  read_timings(P);
  return THISTLE_OK;
}

int thistle_plan_execute_quartets(thistle_plan *P, const int32_t *quartets, int64_t nquart, double *result_host) {
  if (!P || !result_host || (nquart > 0 && !quartets) || nquart < 0) return fail(THISTLE_ERR_ARG, "null argument");
  // host-side class sort of the (small) list
  std::vector<std::pair<int, uint64_t>> items((size_t)nquart);
  for (int64_t t = 0; t < nquart; ++t) {
    int gi = quartets[4 * t], gj = quartets[4 * t + 1], gk = quartets[4 * t + 2], gr = quartets[4 * t + 3];
    if (gi < 0 || gj < 0 || gk < 0 || gr < 0 || gi >= P->ng || gj >= P->ng || gk >= P->ng || gr >= P->ng ||
        gi > gj || gk > gr)
      return fail(THISTLE_ERR_SHAPE, "quartet " + std::to_string(t) + " needs 0 <= gi <= gj < ng, 0 <= gk <= gr < ng");
    int key = (int)quartet_key(P->gL[gi], P->gL[gj], P->gL[gk], P->gL[gr]);
    items[t] = {key, (uint64_t)gi | ((uint64_t)gj << 16) | ((uint64_t)gk << 32) | ((uint64_t)gr << 48)};
  }
  std::stable_sort(items.begin(), items.end(),
                   [](const std::pair<int, uint64_t> &a, const std::pair<int, uint64_t> &b) { return a.first < b.first; });
  int64_t cb[MAXCLS], ce[MAXCLS], ro[MAXCLS];
  int cL[MAXCLS], rs[MAXCLS], ncls = 0;
  std::vector<SubRange> sub[MAXCLS];
  int64_t roff = 0;
  for (int64_t t = 0; t < nquart;) {
    int LL = items[t].first / (int)KEY_CLASS_DIV;
    int64_t u = t;
    while (u < nquart && items[u].first / (int)KEY_CLASS_DIV == LL) ++u;
    for (int64_t w = t; w < u;) {
      const int sk = (items[w].first / 625) % 18;
      int64_t x = w;
      while (x < u && (items[x].first / 625) % 18 == sk) ++x;
      sub[ncls].push_back(SubRange{sk / 2, sk % 2, w, x});
      w = x;
    }
    cb[ncls] = t; ce[ncls] = u; cL[ncls] = LL;
    rs[ncls] = P->kind == KIND_ALIGNED ? 4 + ntuv(LL) : LL + 7;
    rs[ncls] += rs[ncls] & 1;
    ro[ncls] = roff;
    roff += (u - t) * rs[ncls];
    ++ncls;
    t = u;
  }
  std::vector<uint64_t> packed((size_t)nquart);
  for (int64_t t = 0; t < nquart; ++t) packed[t] = items[t].second;
  uint64_t *dq = nullptr;
  double *drec = nullptr;
  int rc = THISTLE_OK;
  P->launches = 0;
  TB_TRY(dalloc(&dq, (size_t)nquart, "quartet list"));
  TB_TRY(dalloc(&drec, (size_t)roff, "quartet records"));
  TB_TRYC(cudaMemcpyAsync(dq, packed.data(), sizeof(uint64_t) * nquart, cudaMemcpyHostToDevice, P->st));
  if (nquart == 0) {
    TB_TRYC(cudaMemsetAsync(P->d_result, 0, sizeof(double) * P->nq, P->st));
  } else {
    TB_TRY(run_stages(P, dq, cb, ce, cL, ncls, drec, ro, rs, sub, P->d_result, false, 1, nullptr));
  }
  TB_TRYC(cudaMemcpyAsync(result_host, P->d_result, sizeof(double) * P->nq, cudaMemcpyDeviceToHost, P->st));
  TB_TRYC(cudaStreamSynchronize(P->st));
done:
  dfree(dq);
  dfree(drec);
  return rc;
}

int thistle_plan_records(const thistle_plan *P, const double **rec_dev, int32_t *ncls, int64_t *cls_begin,
                         int64_t *cls_end, int64_t *cls_recoff, int32_t *cls_rs, const double **q_dev) {
  if (!P || !rec_dev || !ncls || !cls_begin || !cls_end || !cls_recoff || !cls_rs || !q_dev)
    return fail(THISTLE_ERR_ARG, "null argument");
  if (P->kind == KIND_ALIGNED)
    return fail(THISTLE_ERR_TYPE, "aligned plans hold Hermite-density records, not Bessel-sum records");
  *rec_dev = P->d_rec;
  *q_dev = P->d_q;
  *ncls = P->ncls;
  for (int c = 0; c < P->ncls; ++c) {
    cls_begin[c] = P->cls_begin[c];
    cls_end[c] = P->cls_end[c];
    cls_recoff[c] = P->cls_recoff[c];
    cls_rs[c] = P->cls_rs[c];
  }
  return THISTLE_OK;
}

int thistle_plan_density(const thistle_plan *P, double *out, int64_t count, int64_t *needed) {
  if (!P || !needed) return fail(THISTLE_ERR_ARG, "null argument");
  if (P->kind == KIND_ALIGNED || P->kind == KIND_TOTAL || P->kind == KIND_J2) {
    *needed = P->np * P->np;
  } else {
    *needed = (int64_t)P->nzao * P->ngto * P->ngto;  // type 9: zi then zj
  }
  if (!out) return THISTLE_OK;
  if (count < *needed) return fail(THISTLE_ERR_ARG, "output holds " + std::to_string(count) + " doubles, the density " +
                                                       std::to_string(*needed));
  const double *src = kind_elastic(P->kind) ? P->d_zao : P->d_rho;
  TB_CK(cudaStreamSynchronize(P->st));
  TB_CK(cudaMemcpy(out, src, sizeof(double) * (size_t)*needed, cudaMemcpyDeviceToHost));
  return THISTLE_OK;
}

int thistle_plan_info(const thistle_plan *P, int64_t *info) {
  if (!P || !info) return fail(THISTLE_ERR_ARG, "null argument");
  info[0] = P->nquart;
  info[1] = P->ncls;
  info[2] = P->ng;
  info[3] = P->ngto;
  info[4] = P->nq;
  info[5] = P->launches;
  return THISTLE_OK;
}

int thistle_plan_class_counts(const thistle_plan *P, int64_t *out) {
  if (!P || !out) return fail(THISTLE_ERR_ARG, "null argument");
  int64_t p0[MAXCLS] = {0};
  TB_CK(cudaMemcpy(p0, P->d_p0count, sizeof(int64_t) * MAXCLS, cudaMemcpyDeviceToHost));
  for (int i = 0; i <= LMAXQ; ++i) { out[3 * i] = i; out[3 * i + 1] = 0; out[3 * i + 2] = 0; }
  for (int c = 0; c < P->ncls; ++c) {
    out[3 * P->cls_L[c] + 1] = P->cls_end[c] - P->cls_begin[c];
    out[3 * P->cls_L[c] + 2] = p0[c];
  }
  return THISTLE_OK;
}

int thistle_plan_stage_totals(thistle_plan *P, double *ms4, int64_t *nexec) {
  if (!P || !ms4 || !nexec) return fail(THISTLE_ERR_ARG, "null argument");
  TB_CK(cudaStreamSynchronize(P->st));
  for (int i = 0; i < 4; ++i) ms4[i] = 0.0;
  int64_t first = std::max(P->ring_base, P->ring_next - thistle_plan::NRING);
  for (int64_t k = first; k < P->ring_next; ++k) {
    cudaEvent_t *E = P->rev[k % thistle_plan::NRING];
    for (int i = 0; i < 4; ++i) {
      float t = 0;
      TB_CK(cudaEventElapsedTime(&t, E[kStageFrom[i]], E[kStageTo[i]]));
      ms4[i] += t;
    }
  }
  *nexec = P->ring_next - first;
  P->ring_base = P->ring_next;
  read_timings(P);
  return THISTLE_OK;
}

int thistle_plan_timings(const thistle_plan *P, double *ms) {
  if (!P || !ms) return fail(THISTLE_ERR_ARG, "null argument");
  for (int i = 0; i < 6; ++i) ms[i] = P->ms[i];
  return THISTLE_OK;
}

int thistle_plan_destroy(thistle_plan *P) {
  if (P) {
    PhaseTrace tr;
    if (P->st) cudaStreamSynchronize(P->st);
    plan_free(P);
    tr.mark("plan destroy");
  }
  return THISTLE_OK;
}

}  // extern "C"
