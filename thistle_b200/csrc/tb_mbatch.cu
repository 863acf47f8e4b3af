// Molecule batches: several plans (any bases) run over descriptor tables,
// optionally replayed from a CUDA graph.  Stage 1 is one launch per kernel
// shape (L, LK, XB); stage 2, the dominant stage, is ONE persistent launch
// over every (plan, class, block) item of the batch.
#include <map>

#include "tb_plan_internal.h"

using namespace tb;

struct thistle_batch {
  std::vector<thistle_plan *> plans;
  cudaStream_t st = nullptr;
  int kind = 0, nqmax = 0;
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
    bool tpl = false;      // shell-templated kernel of shell tuple XB (LK = -2)
    // split groups of canonical total-j0 plans: the shell-templated
    // contraction, one launch per shell tuple, replaces the generic one
    struct Xct {
      int tuple, n;
      Stage1Args *d;
      int64_t *pre, blocks;
    };
    std::vector<Xct> xct;
  };
  std::vector<S1> s1;
  // stage 2: items (plan, class) heaviest Bessel order first, item i owning
  // virtual blocks s2_pre[i] .. s2_pre[i+1]-1, each with its own partial row
  Stage2Tile tile;
  Stage2ClassArgs *d_s2 = nullptr;
  int64_t *d_s2pre = nullptr, s2_blocks = 0;
  int n_s2 = 0, s2_grid = 0;
  unsigned long long *d_next = nullptr;  // the persistent launch's work counter
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
  for (auto &x : B->s1) {
    dfree(x.d); dfree(x.pre); dfree(x.prexc);
    for (auto &y : x.xct) { dfree(y.d); dfree(y.pre); }
  }
  dfree(B->d_xbuf);
  dfree(B->d_s2); dfree(B->d_s2pre); dfree(B->d_next);
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
    if (x.tpl) {
      TB_CK(launch_stage1_tpl_batch(B->kind, x.XB, x.d, x.pre, x.n, x.blocks, st));
      B->launches += 1;
    } else if (x.split) {
      for (auto &y : x.xct) {
        TB_CK(launch_stage1_xct_batch(B->kind, y.tuple, x.XB != 0, y.d, y.pre, y.n, y.blocks, B->d_xbuf, st));
        B->launches += 1;
      }
      TB_CK(launch_stage1_xsplit_batch(B->kind, x.L, x.LK, x.XB, x.d, x.prexc, x.xct.empty() ? x.blocksxc : 0,
                                       x.pre, x.blocks, x.n, B->d_xbuf, st));
      B->launches += x.xct.empty() ? 2 : 1;
    } else {
      TB_CK(launch_stage1_batch(B->kind, x.L, x.LK, x.XB, x.d, x.pre, x.n, x.blocks, st));
      B->launches += 1;
    }
  }
  TB_CK(cudaMemsetAsync(B->d_partial, 0, sizeof(double) * B->partial_len, st));
  TB_CK(cudaMemsetAsync(B->d_next, 0, sizeof(unsigned long long), st));
  TB_CK(launch_stage2_persistent(kind_j2(B->kind), B->d_s2, B->d_s2pre, B->n_s2, B->s2_blocks, B->nqmax, B->s2_grid,
                                 B->tile, B->d_next, st));
  B->launches += 1;
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

// Stage-2 items of the batch for its pair tile: every (plan, class) with
// quartets, heaviest Bessel order first (the persistent launch's tail is then
// light work), each with up to one GPU's worth of virtual blocks.  A virtual
// block adds into its own partial row of its plan, so the partial rows of a
// plan are the sum of its items' virtual blocks, and the reduction over them
// does not depend on which resident block ran which virtual block.
static int batch_stage2_setup(thistle_batch *B) {
  int rc = THISTLE_OK;
  const int n = (int)B->plans.size();
  const bool j2 = kind_j2(B->kind);
  dfree(B->d_s2); dfree(B->d_s2pre); dfree(B->d_red); dfree(B->d_partial);
  B->d_s2 = nullptr;
  B->d_s2pre = nullptr;
  B->d_red = nullptr;
  B->d_partial = nullptr;
  const int nsm = B->plans[0]->nsm;
  const int bps = stage2_persistent_blocks_per_sm(j2, B->nqmax, B->tile);
  const int64_t cap = (int64_t)nsm * bps;
  struct Item {
    int LB, plan;
    int64_t row, vg;
    Stage2ClassArgs s;
  };
  std::vector<Item> items;
  std::vector<int64_t> prow(n, 0);
  for (int i = 0; i < n; ++i) {
    thistle_plan *P = B->plans[i];
    int uniform = 0, first_on_grid = 0;
    double dq = 0.0;
    grid_info(P->hq.data(), P->nq, uniform, first_on_grid, dq);
    for (int c = 0; c < P->ncls; ++c) {
      const int LB = P->cls_L[c] + (j2 ? 2 : 0);
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
      s.j2 = j2;
      s.lb = LB;
      s.pstride = P->nq;
      s.gs_rec = 0;
      s.gs_partial = 0;
      const int64_t per = (int64_t)stage2_quartets_per_warp(LB, B->tile) * B->tile.nw;
      const int64_t vg = std::min<int64_t>(cap, (s.nquart + per - 1) / per);
      if (vg <= 0) continue;
      items.push_back(Item{LB, i, prow[i], vg, s});
      prow[i] += vg;
    }
  }
  std::stable_sort(items.begin(), items.end(), [](const Item &x, const Item &y) { return x.LB > y.LB; });
  std::vector<int64_t> poff(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    prow[i] = std::max<int64_t>(prow[i], 1);  // a plan without quartets still reduces one zero row
    poff[i + 1] = poff[i] + prow[i] * B->plans[i]->nq;
  }
  B->partial_len = poff[n];
  TB_TRY(dalloc(&B->d_partial, (size_t)std::max<int64_t>(B->partial_len, 1), "batch partial sums"));
  {
    std::vector<ReduceDesc> rd;
    for (int i = 0; i < n; ++i)
      rd.push_back(ReduceDesc{B->d_partial + poff[i], (int)prow[i], B->plans[i]->nq, B->d_out + B->out_off[i]});
    std::vector<Stage2ClassArgs> d;
    std::vector<int64_t> pre(1, 0);
    for (Item &it : items) {
      it.s.partial = B->d_partial + poff[it.plan] + it.row * B->plans[it.plan]->nq;
      d.push_back(it.s);
      pre.push_back(pre.back() + it.vg);
    }
    B->n_s2 = (int)d.size();
    B->s2_blocks = pre.back();
    B->s2_grid = (int)std::max<int64_t>(1, std::min<int64_t>(cap, B->s2_blocks));
    TB_TRY(upload_vec(&B->d_red, rd, B->st, "batch reduce descriptors"));
    if (!d.empty()) {
      TB_TRY(upload_vec(&B->d_s2, d, B->st, "batch stage-2 descriptors"));
      TB_TRY(upload_vec(&B->d_s2pre, pre, B->st, "batch stage-2 prefix"));
    }
    TB_TRYC(cudaStreamSynchronize(B->st));
  }
done:
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
    int64_t ooff = 0;
    for (thistle_plan *P : B->plans) {
      pd.push_back(PairDesc{P->ng, P->maxa, P->d_gstart, P->d_flmn, P->d_ga, P->d_xyz, P->d_pairtab, P->d_esoa});
      ppre.push_back(ppre.back() + (npairs(P->ng) + 127) / 128);
      B->nqmax = std::max(B->nqmax, P->nq);
      B->out_off.push_back(ooff);
      ooff += P->nq;
    }
    B->nq_total = ooff;
    TB_TRY(dalloc(&B->d_out, (size_t)std::max<int64_t>(ooff, 1), "batch results"));
    TB_TRY(dalloc(&B->d_next, 1, "batch work counter"));
    B->pair_blocks = ppre.back();
    TB_TRY(upload_vec(&B->d_pair, pd, B->st, "batch pair descriptors"));
    TB_TRY(upload_vec(&B->d_pair_pre, ppre, B->st, "batch pair prefix"));
    // stage 1: items grouped by (L, LK, XB); the kernel choice per L counts
    // the quartets of every plan
    int64_t ltot[LMAXQ + 1] = {0};
    for (thistle_plan *P : B->plans)
      for (int c = 0; c < P->ncls; ++c) ltot[P->cls_L[c]] += P->cls_end[c] - P->cls_begin[c];
    std::vector<std::pair<std::array<int, 6>, Stage1Args>> items;  // (L, LK, XB, nout, plan, class)
    for (int pi = 0; pi < n; ++pi)
      for (int c = 0; c < plans[pi]->ncls; ++c) {
        thistle_plan *P = plans[pi];
        Stage1Args a = stage1_args(P, P->d_quart, P->cls_begin[c], P->cls_end[c], P->d_rec, P->cls_recoff[c],
                                   P->cls_rs[c]);
        const int L = P->cls_L[c];
        if (stage1_tpl(P->kind, L, P->shells_canonical) && !P->cls_tup[c].empty()) {
          // shell-templated kernels: items keyed (L, -2, shell tuple)
          for (const TupleRange &u : P->cls_tup[c]) {
            Stage1Args b = a;
            b.qbegin = u.begin;
            b.qend = u.end;
            b.recbase = P->cls_recoff[c] + (u.begin - P->cls_begin[c]) * (int64_t)P->cls_rs[c];
            items.push_back({{L, -2, u.tuple, 0, pi, c}, b});
          }
        } else if (stage1_xk(L, ltot[L], P->nsm)) {
          for (const SubRange &u : P->cls_sub[c]) {
            Stage1Args b = a;
            b.qbegin = u.begin;
            b.qend = u.end;
            b.recbase = P->cls_recoff[c] + (u.begin - P->cls_begin[c]) * (int64_t)P->cls_rs[c];
            items.push_back({{L, u.LK, u.XB, u.nout, pi, c}, b});
          }
        } else {
          items.push_back({{L, -1, 0, 0, pi, c}, a});
        }
      }
    auto same = [](const std::array<int, 6> &x, const std::array<int, 6> &y) {
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
      // every item knows its outer-pair count and the group fits in 2 GB; a
      // larger set of items of one key becomes several groups, which run one
      // after another through the same buffer
      constexpr int64_t XLIMIT = int64_t(1) << 28;
      bool split = LK >= 0;
      int64_t xoff = 0;
      while (j < items.size() && same(items[j].first, items[i].first)) {
        Stage1Args a = items[j].second;
        const int64_t nq = a.qend - a.qbegin;
        const int nout = items[j].first[3];
        if (LK >= 0 && nout > 0 && !d.empty() && xoff + nq * nout * ntuv(LK) > XLIMIT) break;
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
        pre.push_back(pre.back() + (LK == -2 ? (nq + 127) / 128 : stage1_item_blocks(L, LK >= 0, nq)));
        ++j;
      }
      if (xoff > XLIMIT) split = false;
      if (split) xneed = std::max(xneed, xoff);
      thistle_batch::S1 x{L, LK, items[i].first[2], (int)d.size(), nullptr, nullptr, pre.back(), split, nullptr,
                          split ? prexc.back() : 0};
      x.tpl = LK == -2;
      // the shell-templated contraction when every plan of the group takes
      // it and its shell tuples tile each sub-range
      bool xct = split && stage1_xct(B->kind, LK, 1);
      std::map<int, std::vector<Stage1Args>> bytup;
      for (size_t t = i; t < j && xct; ++t) {
        const thistle_plan *P = plans[items[t].first[4]];
        const int c = items[t].first[5];
        const Stage1Args &a = d[t - i];
        xct = stage1_xct(P->kind, LK, P->shells_canonical);
        int64_t covered = 0;
        for (const TupleRange &w : P->cls_tup[c]) {
          if (!xct || w.begin < a.qbegin || w.end > a.qend) continue;
          Stage1Args bt = a;
          bt.qbegin = w.begin;
          bt.qend = w.end;
          bt.xoff = a.xoff + (w.begin - a.qbegin) * (int64_t)a.xstride;
          bytup[w.tuple].push_back(bt);
          covered += w.end - w.begin;
        }
        if (covered != a.qend - a.qbegin) xct = false;
      }
      if (xct) {
        for (auto &kv : bytup) {
          std::vector<int64_t> tp(1, 0);
          for (const Stage1Args &bt : kv.second) tp.push_back(tp.back() + ((bt.qend - bt.qbegin) * bt.xg + 127) / 128);
          thistle_batch::S1::Xct y{kv.first, (int)kv.second.size(), nullptr, nullptr, tp.back()};
          TB_TRY(upload_vec(&y.d, kv.second, B->st, "batch contraction descriptors"));
          TB_TRY(upload_vec(&y.pre, tp, B->st, "batch contraction prefix"));
          x.xct.push_back(y);
        }
      }
      TB_TRY(upload_vec(&x.d, d, B->st, "batch stage-1 descriptors"));
      TB_TRY(upload_vec(&x.pre, pre, B->st, "batch stage-1 prefix"));
      if (split) TB_TRY(upload_vec(&x.prexc, prexc, B->st, "batch contraction prefix"));
      B->s1.push_back(x);
      i = j;
    }
    if (xneed > 0) TB_TRY(dalloc(&B->d_xbuf, (size_t)xneed, "batch contraction buffer"));
    TB_TRY(batch_stage2_setup(B));
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

int thistle_batch_set_stage2_tile(thistle_batch *B, int32_t quartets_per_lane, int32_t warps_per_block) {
  if (!B) return fail(THISTLE_ERR_ARG, "null batch");
  const Stage2Tile t{quartets_per_lane, warps_per_block};
  if (!stage2_tile_valid(t)) return fail(THISTLE_ERR_ARG, "stage-2 tile: quartets per lane 1 or 2, warps 4 or 8");
  if (t.k == B->tile.k && t.nw == B->tile.nw) return THISTLE_OK;
  TB_CK(cudaStreamSynchronize(B->st));
  if (B->gx) cudaGraphExecDestroy(B->gx);
  B->gx = nullptr;
  B->tile = t;
  return batch_stage2_setup(B);
}

int thistle_batch_stage2_tile(const thistle_batch *B, int32_t *quartets_per_lane, int32_t *warps_per_block) {
  if (!B || !quartets_per_lane || !warps_per_block) return fail(THISTLE_ERR_ARG, "null argument");
  *quartets_per_lane = B->tile.k;
  *warps_per_block = B->tile.nw;
  return THISTLE_OK;
}

int thistle_batch_autotune(thistle_batch *B, int32_t *quartets_per_lane, int32_t *warps_per_block,
                           double *molecules_per_s) {
  if (!B || !quartets_per_lane || !warps_per_block || !molecules_per_s) return fail(THISTLE_ERR_ARG, "null argument");
  const Stage2Tile tiles[4] = {{2, 4}, {2, 8}, {1, 4}, {1, 8}};
  const int reps = 3;
  double best = -1.0;
  Stage2Tile bestT = B->tile;
  cudaEvent_t e0, e1;
  TB_CK(cudaEventCreate(&e0));
  TB_CK(cudaEventCreate(&e1));
  int rc = THISTLE_OK;
  for (int t = 0; t < 4 && rc == THISTLE_OK; ++t) {
    rc = thistle_batch_set_stage2_tile(B, tiles[t].k, tiles[t].nw);
    for (int w = 0; w < 2 + reps && rc == THISTLE_OK; ++w) {
      if (w == 2 && cudaEventRecord(e0, B->st) != cudaSuccess) rc = fail(THISTLE_ERR_CUDA, "event record");
      if (rc == THISTLE_OK) rc = batch_exec(B);
    }
    float ms = 0;
    if (rc == THISTLE_OK && (cudaEventRecord(e1, B->st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                             cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
      rc = fail(THISTLE_ERR_CUDA, "batch autotune timing");
    const double mps = ms > 0 ? B->plans.size() * reps / (ms * 1e-3) : 0.0;
    if (rc == THISTLE_OK && mps > best) {
      best = mps;
      bestT = tiles[t];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != THISTLE_OK) return rc;
  rc = thistle_batch_set_stage2_tile(B, bestT.k, bestT.nw);
  if (rc != THISTLE_OK) return rc;
  *quartets_per_lane = bestT.k;
  *warps_per_block = bestT.nw;
  *molecules_per_s = best;
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
