// Internal declarations shared by the host-side units of the C-ABI
// (tb_plan.cu: validation, classes, quartets, plan lifecycle, execution, the
// adjoint and geometry batches; tb_density.cu: the density transform;
// tb_entry.cu: Entry 1, the electron and elastic-aligned terms and the q
// grids; tb_mbatch.cu: molecule batches).  Not part of the C-ABI: the
// functions below have hidden visibility.
#pragma once
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tb_kernels.h"
#include "tb_math.cuh"
#include "thistle_b200.h"

using namespace tb;

extern thread_local std::string g_err;

// THISTLE_B200_TRACE=1 prints the host-side duration of the set-up phases to stderr.
struct PhaseTrace {
  bool on = std::getenv("THISTLE_B200_TRACE") != nullptr;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  void mark(const char *what) {
    if (!on) return;
    auto t1 = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[thistle_b200] %-28s %9.3f ms\n", what,
                 std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  }
};

inline int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define TB_CK(x)                                                                            \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) return fail(THISTLE_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Device buffers come from the process-wide cache (tb_pool.cu).
template <class T>
inline int dalloc(T **p, size_t n, const char *what) {
  *p = nullptr;
  if (n == 0) n = 1;
  void *v = nullptr;
  cudaError_t e = pool_malloc(&v, n * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? THISTLE_ERR_NOMEM : THISTLE_ERR_CUDA,
                std::string("cudaMalloc of ") + what + " (" + std::to_string(n * sizeof(T)) + " bytes): " +
                    cudaGetErrorString(e));
  }
  *p = (T *)v;
  return THISTLE_OK;
}
template <class T>
inline void dfree(T *&p) {
  if (p) pool_free((void *)p);
  p = nullptr;
}

// Quartets of one LLmax class with equal (LK, XB) (see quartet_key).
struct SubRange {
  int LK, XB;
  int64_t begin, end;
  int nout = 0;  // most function pairs of an outer (convolved) side; 0: unknown
};

// quartets of one shell tuple ((Li 5 + Lj) 5 + Lk) 5 + Lr within a class
struct TupleRange {
  int tuple;
  int64_t begin, end;
};

struct thistle_plan {
  int type = 0, kind = 0;
  int ngto = 0, ng = 0, nmo = 0, nmo1 = 0, nzao = 1, nq = 0, maxa = 0, nmat = 0;
  int shells_canonical = 1;  // s, p, d, f groups: complete shells in cart_component order
  double cutoffz = 0, cutoffmd = 0, cutoffcentre = 0;
  std::vector<int> gstart, gcount, gL, flmn;
  std::vector<double> hq;            // host copy of the q grid (aligned: interleaved q vectors)
  int qdim = 1;                      // 3 for aligned plans (q vectors)
  int64_t nquart = 0, np = 0;
  int ncls = 0;
  int cls_L[MAXCLS];
  int64_t cls_begin[MAXCLS], cls_end[MAXCLS], cls_recoff[MAXCLS];
  int cls_rs[MAXCLS];
  std::vector<SubRange> cls_sub[MAXCLS];
  std::vector<TupleRange> cls_tup[MAXCLS];
  double *d_xbuf = nullptr;  // contraction output of the split contracted-side stage 1
  int64_t xbuf_len = 0;
  int64_t rec_total = 0;
  int *d_gstart = nullptr, *d_gcount = nullptr, *d_flmn = nullptr;
  double *d_ga = nullptr, *d_xyz = nullptr, *d_q = nullptr, *d_pairtab = nullptr, *d_esoa = nullptr;
  double *d_rho = nullptr, *d_zao = nullptr, *d_rec = nullptr, *d_partial = nullptr, *d_result = nullptr;
  uint64_t *d_quart = nullptr;
  // device-resident density inputs and transform workspaces
  int *d_mat = nullptr;
  double *d_C = nullptr, *d_tot = nullptr, *d_D = nullptr, *d_Ds = nullptr, *d_Y = nullptr;
  double *d_G = nullptr, *d_T1 = nullptr, *d_V = nullptr, *d_T3 = nullptr, *d_Ct = nullptr;
  // Ghat build: (index, value) per row placement, sorted by index
  int *d_gk0 = nullptr, *d_gk1 = nullptr;
  double *d_gv0 = nullptr, *d_gv1 = nullptr;
  void *d_gsort_tmp = nullptr;
  size_t gsort_bytes = 0;
  int gbits = 0;
  // grouped GEMM of the transform's last pass (one group per b)
  // quartet enumeration workspaces
  int64_t *d_braoff = nullptr;
  int *d_gL = nullptr;
  uint32_t *d_k0 = nullptr, *d_k1 = nullptr;
  uint64_t *d_v0 = nullptr;
  void *d_sort_tmp = nullptr;
  size_t sort_tmp_bytes = 0;
  int64_t *d_p0count = nullptr;      // P=Q quartets per class in the last execution
  // stage-2 visiting order: keys written by stage 1, sorted with the quartet index
  uint32_t *d_s2key = nullptr, *d_s2key_sorted = nullptr, *d_iota = nullptr, *d_perm = nullptr;
  void *d_s2sort_tmp = nullptr;
  size_t s2sort_bytes = 0;
  int nsm = 0, s2_rows = 0, s2_qtile = 0;
  int s2_bps[LMAXB + 1];             // resident stage-2 blocks per SM, per Bessel order
  Stage2Tile s2_tile;                // stage-2 pair tile (quartets per lane, warps per block)
  cudaStream_t st = nullptr;
  bool own_stream = true;
  // stage-2 classes too small to fill the GPU run on st2, joined into st
  // before the reduction, into partial rows s2_rows .. 2 s2_rows - 1 of each
  // geometry (the others use rows 0 .. s2_rows - 1)
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_join = nullptr;
  // the other stage-2 classes run on st3; class c's stage 2 waits for
  // ev_cls[c], recorded on st once its stage 1 and its visiting-order sort
  // are done, so stage 2 of the first classes overlaps stage 1 of the later
  cudaStream_t st3 = nullptr;
  cudaEvent_t ev_join3 = nullptr;
  cudaEvent_t ev_cls[MAXCLS] = {};
  cudaEvent_t ev[10];
  // per-execution stage events: slot = execution index mod NRING
  static const int NRING = 64;
  cudaEvent_t rev[64][6];
  int rev_made = 0;  // slots 0 .. rev_made-1 hold events (made as executions first reach them)
  int64_t ring_next = 0, ring_base = 0;
  bool have_ev = false;
  float ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int64_t launches = 0;              // own kernels launched by the last call
  // geometry batches: ngeom copies of the centres, tables, records and results
  int ngeom = 1;
  bool capturing = false;            // inside a CUDA-graph capture (no event records)
  bool use_graph = false;
  bool pipeline = true;  // stage 2 of a class may start before the later classes' stage 1
  cudaGraphExec_t gx_fwd = nullptr, gx_vjp = nullptr;
  std::vector<double> hxyz;          // host copy of the centres (interleaved, ngeom x ngto x 3)
  bool fwd_valid = false;            // records and visiting order match the current centres
  // adjoint workspaces (allocated by the first vector-Jacobian product)
  double *d_dsoa = nullptr, *d_adj = nullptr, *d_gpart = nullptr, *d_v = nullptr, *d_grad = nullptr;
  int adj_rows = 0;
};

#define TB_TRY(x)                    \
  do {                               \
    rc = (x);                        \
    if (rc != THISTLE_OK) goto done; \
  } while (0)
#define TB_TRYC(x)                                                                                        \
  do {                                                                                                    \
    cudaError_t e_ = (x);                                                                                 \
    if (e_ != cudaSuccess) {                                                                              \
      rc = fail(THISTLE_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));                       \
      goto done;                                                                                          \
    }                                                                                                     \
  } while (0)

#define TB_INTERNAL __attribute__((visibility("hidden")))

TB_INTERNAL bool finite_all(const double *a, int64_t n);
TB_INTERNAL int check_basis(thistle_plan *P, int32_t ngto, const double *ga, const int32_t *l, const int32_t *m,
                       const int32_t *n, const double *xx, const double *yy, const double *zz,
                       const int32_t *group);
TB_INTERNAL int check_q(const double *q, int32_t nq);
TB_INTERNAL int64_t bra_count(int i, int j, int ng, bool all_pairs);
TB_INTERNAL void class_counts(const std::vector<int> &gL, std::vector<int64_t> &cnt, bool all_pairs);
TB_INTERNAL int setup_classes(thistle_plan *P, const std::vector<int64_t> &cnt, int kind);
TB_INTERNAL int quartets_alloc(thistle_plan *P);
TB_INTERNAL int quartets_run(thistle_plan *P);
TB_INTERNAL void plan_free(thistle_plan *P);
TB_INTERNAL int64_t gs_pair(const thistle_plan *P);
TB_INTERNAL int64_t gs_esoa(const thistle_plan *P);
TB_INTERNAL int64_t gs_rec(const thistle_plan *P);
TB_INTERNAL void drop_graphs(thistle_plan *P);
TB_INTERNAL int geo_alloc(thistle_plan *P, int G);
TB_INTERNAL int upload_centres(thistle_plan *P, const double *xx, const double *yy, const double *zz);
TB_INTERNAL int upload_centres_batch(thistle_plan *P, const double *xyz);
TB_INTERNAL int plan_create(thistle_plan **out, int32_t type, int32_t ngto, const double *ga, const int32_t *l,
                       const int32_t *m, const int32_t *n, const double *xx, const double *yy, const double *zz,
                       const int32_t *group, const double *mmod, int32_t norbs, const int32_t *mat,
                       const double *total, int32_t nmat, const double *onerdm, int32_t nmo1, const double *q,
                       int32_t nq, double cutoffz, double cutoffmd, double cutoffcentre);
TB_INTERNAL void stage2_layout(thistle_plan *P);
TB_INTERNAL void grid_info(const double *q, int n, int &uniform, int &first_on_grid, double &dq);
TB_INTERNAL Stage1Args stage1_args(const thistle_plan *P, const uint64_t *d_quart, int64_t qbegin, int64_t qend,
                              double *d_rec, int64_t recbase, int rs);
TB_INTERNAL int run_stages(thistle_plan *P, const uint64_t *d_quart, const int64_t *cb, const int64_t *ce,
                      const int *cL, int ncls, double *d_rec, const int64_t *recoff, const int *rs,
                      const std::vector<SubRange> *subs, double *d_out, bool order, int ngeom,
                      const std::vector<TupleRange> *tups);
TB_INTERNAL int plan_exec(thistle_plan *P, double *d_out);
TB_INTERNAL void read_timings(thistle_plan *P);
TB_INTERNAL int adjoint_check(thistle_plan *P);
TB_INTERNAL int adjoint_alloc(thistle_plan *P);
TB_INTERNAL int adjoint_stages(thistle_plan *P, const double *d_v, double *d_grad);
TB_INTERNAL int forward_batch(thistle_plan *P);
TB_INTERNAL int plan_vjp(thistle_plan *P, const double *d_v, double *d_grad);
TB_INTERNAL int density_alloc(thistle_plan *P);
TB_INTERNAL int density_upload(thistle_plan *P, const double *mmod, const int32_t *mat, const double *total,
                          const double *onerdm);
TB_INTERNAL int density_run(thistle_plan *P);
TB_INTERNAL int nuclear_term(thistle_plan *P, const double *Zn, const double *geom, int natoms, double *host_out);
TB_INTERNAL int form_factor(thistle_plan *P, const double *qvec, int nq, double *re, double *im, double *abs2);
TB_INTERNAL void elastic_aligned_grid(int nq, double *qal);
TB_INTERNAL void nuclear_nuclear(const double *Zn, const double *geom, int natoms, const double *q, int nq, double *out);
TB_INTERNAL void batch_free(thistle_batch *B);
TB_INTERNAL int batch_run(thistle_batch *B);
TB_INTERNAL int batch_exec(thistle_batch *B);
TB_INTERNAL int batch_create(thistle_batch **out, thistle_plan *const *plans, int32_t n);
TB_INTERNAL void qcoord3_grid(double k0, double *qal /* (3, 3131) column-major */);
