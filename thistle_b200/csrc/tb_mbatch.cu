// Molecule batches: several plans (any bases) run as one launch per stage and
// class over descriptor tables, optionally replayed from a CUDA graph.
#include "tb_plan_internal.h"

using namespace tb;

// ---------------------------------------------------------------------------
// molecule batches: several plans (any bases), one launch per stage and class
// ---------------------------------------------------------------------------
struct thistle_batch {
  std::vector<thistle_plan *> plans;
  cudaStream_t st = nullptr;
  int kind = 0, nqmax = 0, rows = 64;  // partial rows per plan: a class's blocks in one launch
  int64_t nq_total = 0;
  std::vector<int64_t> out_off;
  PairDesc *d_pair = nullptr;
  int64_t *d_pair_pre = nullptr, pair_blocks = 0;
  struct S1 {
    int L, LK, XB, n;
    Stage1Args *d;
    int64_t *pre, blocks;
    bool split;            // contraction kernel + convolution kernel through d_xbuf
    int64_t *prexc, blocksxc;
  };
  struct S2 {
    int LB, n;
    Stage2ClassArgs *d;
    int64_t *pre, blocks;
  };
  std::vector<S1> s1;
  std::vector<S2> s2;
  ReduceDesc *d_red = nullptr;
  double *d_partial = nullptr, *d_out = nullptr, *d_xbuf = nullptr;
  int64_t partial_len = 0;
  bool use_graph = false;
  cudaGraphExec_t gx = nullptr;
  int64_t launches = 0;
};

void batch_free(thistle_batch *B) {
  if (!B) return;
  dfree(B->d_pair); dfree(B->d_pair_pre); dfree(B->d_red); dfree(B->d_partial); dfree(B->d_out);
  for (auto &x : B->s1) { dfree(x.d); dfree(x.pre); dfree(x.prexc); }
  dfree(B->d_xbuf);
  for (auto &x : B->s2) { dfree(x.d); dfree(x.pre); }
  if (B->gx) cudaGraphExecDestroy(B->gx);
  delete B;
}

template <class T>
static int upload_vec(T **dst, const std::vector<T> &v, cudaStream_t st, const char *what) {
  int rc = dalloc(dst, v.size(), what);
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
  return THISTLE_OK;
}

int batch_run(thistle_batch *B) {
  cudaStream_t st = B->st;
  B->launches = 0;
  TB_CK(launch_pair_tables_batch(B->d_pair, B->d_pair_pre, (int)B->plans.size(), B->pair_blocks, st));
  B->launches += 1;
  for (auto &x : B->s1) {
    if (x.split) {
      TB_CK(launch_stage1_xsplit_batch(B->kind, x.L, x.LK, x.XB, x.d, x.prexc, x.blocksxc, x.pre, x.blocks, x.n,
                                       B->d_xbuf, st));
      B->launches += 2;
    } else {
      TB_CK(launch_stage1_batch(B->kind, x.L, x.LK, x.XB, x.d, x.pre, x.n, x.blocks, st));
      B->launches += 1;
    }
  }
  TB_CK(cudaMemsetAsync(B->d_partial, 0, sizeof(double) * B->partial_len, st));
  for (auto &x : B->s2) {
    TB_CK(launch_stage2_class_batch(x.LB, kind_j2(B->kind), x.d, x.pre, x.n, x.blocks, B->nqmax, st));
    B->launches += 1;
  }
  TB_CK(launch_reduce_desc(B->d_red, (int)B->plans.size(), B->nqmax, st));
  B->launches += 1;
  return THISTLE_OK;
}

int batch_exec(thistle_batch *B) {
  int rc = THISTLE_OK;
  // work a plan queued on its own stream (centres, an execution) comes first
  for (thistle_plan *P : B->plans)
    if (P->st != B->st) TB_CK(cudaStreamSynchronize(P->st));
  if (!B->use_graph) {
    rc = batch_run(B);
  } else {
    if (!B->gx) {
      cudaGraph_t g = nullptr;
      TB_CK(cudaStreamBeginCapture(B->st, cudaStreamCaptureModeThreadLocal));
      rc = batch_run(B);
      cudaError_t e = cudaStreamEndCapture(B->st, &g);
      if (rc != THISTLE_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      TB_CK(e);
      e = cudaGraphInstantiate(&B->gx, g, 0);
      cudaGraphDestroy(g);
      TB_CK(e);
    }
    TB_CK(cudaGraphLaunch(B->gx, B->st));
  }
  // the batch rewrote every plan's pair tables and records for its current centres
  for (thistle_plan *P : B->plans) P->fwd_valid = rc == THISTLE_OK;
  return rc;
}

int batch_create(thistle_batch **out, thistle_plan *const *plans, int32_t n) {
  if (!out || !plans || n < 1) return fail(THISTLE_ERR_ARG, "need at least one plan");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    const thistle_plan *P = plans[i];
    if (!P) return fail(THISTLE_ERR_ARG, "null plan in the batch");
    if (P->kind != plans[0]->kind) return fail(THISTLE_ERR_TYPE, "plans of one batch must share the calculation type");
    if (P->kind == KIND_ALIGNED) return fail(THISTLE_ERR_TYPE, "aligned plans cannot be batched");
    if (P->kind == KIND_CMS) return fail(THISTLE_ERR_TYPE, "resolved CMS plans cannot be batched");
    if (P->ngeom != 1) return fail(THISTLE_ERR_SHAPE, "batched plans hold one geometry each");
    if (P->nq > STAGE2_QTILE) return fail(THISTLE_ERR_SHAPE, "batched plans need nq <= 1024");
  }
  thistle_batch *B = new thistle_batch();
  int rc = THISTLE_OK;
  B->plans.assign(plans, plans + n);
  B->st = plans[0]->st;
  B->kind = plans[0]->kind;
  {
    // every plan once on its own: records, and the stage-2 visiting order
    for (thistle_plan *P : B->plans) {
      TB_TRY(plan_exec(P, P->d_result));
      TB_TRYC(cudaStreamSynchronize(P->st));
    }
    std::vector<PairDesc> pd;
    std::vector<int64_t> ppre(1, 0);
    std::vector<ReduceDesc> rd;
    int64_t poff = 0, ooff = 0;
    for (thistle_plan *P : B->plans) {
      pd.push_back(PairDesc{P->ng, P->maxa, P->d_gstart, P->d_flmn, P->d_ga, P->d_xyz, P->d_pairtab, P->d_esoa});
      ppre.push_back(ppre.back() + (npairs(P->ng) + 127) / 128);
      B->nqmax = std::max(B->nqmax, P->nq);
      B->out_off.push_back(ooff);
      rd.push_back(ReduceDesc{nullptr, B->rows, P->nq, nullptr});  // pointers below
      poff += (int64_t)B->rows * P->nq;
      ooff += P->nq;
    }
    B->partial_len = poff;
    B->nq_total = ooff;
    TB_TRY(dalloc(&B->d_partial, (size_t)std::max<int64_t>(poff, 1), "batch partial sums"));
    TB_TRY(dalloc(&B->d_out, (size_t)std::max<int64_t>(ooff, 1), "batch results"));
    std::vector<double *> part(n);
    poff = 0;
    for (int i = 0; i < n; ++i) {
      part[i] = B->d_partial + poff;
      rd[i].partial = part[i];
      rd[i].out = B->d_out + B->out_off[i];
      poff += (int64_t)B->rows * plans[i]->nq;
    }
    B->pair_blocks = ppre.back();
    TB_TRY(upload_vec(&B->d_pair, pd, B->st, "batch pair descriptors"));
    TB_TRY(upload_vec(&B->d_pair_pre, ppre, B->st, "batch pair prefix"));
    TB_TRY(upload_vec(&B->d_red, rd, B->st, "batch reduce descriptors"));
    // stage 1: items grouped by (L, LK, XB); the kernel choice per L counts
    // the quartets of every plan
    int64_t ltot[LMAXQ + 1] = {0};
    for (thistle_plan *P : B->plans)
      for (int c = 0; c < P->ncls; ++c) ltot[P->cls_L[c]] += P->cls_end[c] - P->cls_begin[c];
    std::vector<std::pair<std::array<int, 4>, Stage1Args>> items;  // (L, LK, XB, nout)
    for (thistle_plan *P : B->plans)
      for (int c = 0; c < P->ncls; ++c) {
        Stage1Args a = stage1_args(P, P->d_quart, P->cls_begin[c], P->cls_end[c], P->d_rec, P->cls_recoff[c],
                                   P->cls_rs[c]);
        const int L = P->cls_L[c];
        if (stage1_xk(L, ltot[L], P->nsm)) {
          for (const SubRange &u : P->cls_sub[c]) {
            Stage1Args b = a;
            b.qbegin = u.begin;
            b.qend = u.end;
            b.recbase = P->cls_recoff[c] + (u.begin - P->cls_begin[c]) * (int64_t)P->cls_rs[c];
            items.push_back({{L, u.LK, u.XB, u.nout}, b});
          }
        } else {
          items.push_back({{L, -1, 0, 0}, a});
        }
      }
    auto same = [](const std::array<int, 4> &x, const std::array<int, 4> &y) {
      return x[0] == y[0] && x[1] == y[1] && x[2] == y[2];
    };
    std::stable_sort(items.begin(), items.end(), [](const auto &x, const auto &y) {
      return std::array<int, 3>{x.first[0], x.first[1], x.first[2]} <
             std::array<int, 3>{y.first[0], y.first[1], y.first[2]};
    });
    int64_t xneed = 0;
    for (size_t i = 0; i < items.size();) {
      size_t j = i;
      std::vector<Stage1Args> d;
      std::vector<int64_t> pre(1, 0), prexc(1, 0);
      const int L = items[i].first[0], LK = items[i].first[1];
      // contracted side: split through the batch's contraction buffer when
      // every item knows its outer-pair count and the group fits in 2 GB
      bool split = LK >= 0;
      int64_t xoff = 0;
      while (j < items.size() && same(items[j].first, items[i].first)) {
        Stage1Args a = items[j].second;
        const int64_t nq = a.qend - a.qbegin;
        const int nout = items[j].first[3];
        if (LK >= 0 && nout > 0) {
          int G = 1;
          while (G < nout) G *= 2;
          a.xg = G;
          a.xstride = nout * ntuv(LK);
          a.xoff = xoff;
          xoff += nq * a.xstride;
          prexc.push_back(prexc.back() + (nq * G + 127) / 128);
        } else {
          split = false;
        }
        d.push_back(a);
        pre.push_back(pre.back() + stage1_item_blocks(L, LK >= 0, nq));
        ++j;
      }
      if (xoff > (int64_t(1) << 28)) split = false;
      if (split) xneed = std::max(xneed, xoff);
      thistle_batch::S1 x{L, LK, items[i].first[2], (int)d.size(), nullptr, nullptr, pre.back(), split, nullptr,
                          split ? prexc.back() : 0};
      TB_TRY(upload_vec(&x.d, d, B->st, "batch stage-1 descriptors"));
      TB_TRY(upload_vec(&x.pre, pre, B->st, "batch stage-1 prefix"));
      if (split) TB_TRY(upload_vec(&x.prexc, prexc, B->st, "batch contraction prefix"));
      B->s1.push_back(x);
      i = j;
    }
    if (xneed > 0) TB_TRY(dalloc(&B->d_xbuf, (size_t)xneed, "batch contraction buffer"));
    // stage 2: items grouped by Bessel order
    std::vector<std::pair<int, std::pair<Stage2ClassArgs, int64_t>>> s2items;
    for (int i = 0; i < n; ++i) {
      thistle_plan *P = plans[i];
      int uniform = 0, first_on_grid = 0;
      double dq = 0.0;
      grid_info(P->hq.data(), P->nq, uniform, first_on_grid, dq);
      for (int c = 0; c < P->ncls; ++c) {
        const int LB = P->cls_L[c] + (kind_j2(P->kind) ? 2 : 0);
        Stage2ClassArgs s;
        s.rec = P->d_rec + P->cls_recoff[c];
        s.rs = P->cls_rs[c];
        s.nquart = P->cls_end[c] - P->cls_begin[c];
        s.perm = P->d_perm;
        s.pbase = P->cls_begin[c];
        s.q = P->d_q;
        s.nq = P->nq;
        s.uniform = uniform;
        s.first_on_grid = first_on_grid;
        s.dq = dq;
        s.chunk = 0;
        s.j2 = kind_j2(P->kind);
        s.partial = part[i];
        s.pstride = P->nq;
        s.gs_rec = 0;
        s.gs_partial = 0;
        // one block per STAGE2_WARPS batches of quartets, at most `rows`
        // (the other plans of the launch fill the GPU)
        const int64_t per = (int64_t)stage2_quartets_per_warp(LB) * STAGE2_WARPS;
        const int64_t vg = std::min<int64_t>(B->rows, (s.nquart + per - 1) / per);
        if (vg <= 0) continue;
        s2items.push_back({LB, {s, vg}});
      }
    }
    std::stable_sort(s2items.begin(), s2items.end(),
                     [](const auto &x, const auto &y) { return x.first < y.first; });
    for (size_t i = 0; i < s2items.size();) {
      size_t j = i;
      std::vector<Stage2ClassArgs> d;
      std::vector<int64_t> pre(1, 0);
      while (j < s2items.size() && s2items[j].first == s2items[i].first) {
        d.push_back(s2items[j].second.first);
        pre.push_back(pre.back() + s2items[j].second.second);
        ++j;
      }
      thistle_batch::S2 x{s2items[i].first, (int)d.size(), nullptr, nullptr, pre.back()};
      TB_TRY(upload_vec(&x.d, d, B->st, "batch stage-2 descriptors"));
      TB_TRY(upload_vec(&x.pre, pre, B->st, "batch stage-2 prefix"));
      B->s2.push_back(x);
      i = j;
    }
    TB_TRYC(cudaStreamSynchronize(B->st));
  }
done:
  if (rc != THISTLE_OK) {
    batch_free(B);
    return rc;
  }
  *out = B;
  return THISTLE_OK;
}

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

int thistle_batch_create(thistle_batch **batch, thistle_plan *const *plans, int32_t nplans) {
  return batch_create(batch, plans, nplans);
}

int thistle_batch_use_graph(thistle_batch *B, int32_t enable) {
  if (!B) return fail(THISTLE_ERR_ARG, "null batch");
  TB_CK(cudaStreamSynchronize(B->st));
  if (B->gx) cudaGraphExecDestroy(B->gx);
  B->gx = nullptr;
  B->use_graph = enable != 0;
  return THISTLE_OK;
}

int thistle_batch_execute_device(thistle_batch *B, double *result_dev) {
  if (!B || !result_dev) return fail(THISTLE_ERR_ARG, "null argument");
  int rc = batch_exec(B);
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaMemcpyAsync(result_dev, B->d_out, sizeof(double) * B->nq_total, cudaMemcpyDeviceToDevice, B->st));
  return THISTLE_OK;
}

int thistle_batch_execute(thistle_batch *B, double *result_host) {
  if (!B || !result_host) return fail(THISTLE_ERR_ARG, "null argument");
  int rc = batch_exec(B);
  if (rc != THISTLE_OK) return rc;
  TB_CK(cudaMemcpyAsync(result_host, B->d_out, sizeof(double) * B->nq_total, cudaMemcpyDeviceToHost, B->st));
  TB_CK(cudaStreamSynchronize(B->st));
  return THISTLE_OK;
}

int thistle_batch_info(const thistle_batch *B, int64_t *info) {
  if (!B || !info) return fail(THISTLE_ERR_ARG, "null argument");
  info[0] = (int64_t)B->plans.size();
  info[1] = B->nq_total;
  info[2] = B->launches;
  return THISTLE_OK;
}

int thistle_batch_destroy(thistle_batch *B) {
  if (B) {
    if (B->st) cudaStreamSynchronize(B->st);
    batch_free(B);
  }
  return THISTLE_OK;
}

}  // extern "C"
