// Internal launch interface between the plan code and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace tb {

struct Stage1Args {
  const uint64_t *quartets;   // packed gi | gj<<16 | gk<<32 | gr<<48, sorted by class
  int64_t qbegin, qend;       // this launch's quartet range (one LLmax class)
  const double *pairtab;      // PAIR_STRIDE doubles per unordered group pair
  int ng;
  const int *gstart, *gcount; // 0-based first function and size of each group
  const int *flmn;            // l | m<<8 | n<<16 per function
  const double *rho;          // pair density (np x np), total / j2
  int64_t np;
  const double *zao;          // AO density (ngto x ngto), elastic; the bra's for KIND_CMS
  const double *zket;         // the ket's AO density: zao, or the second one for KIND_CMS
  int ngto;
  double cutoffz, cutoffmd, cutoffcentre;
  const double *esoa;         // E^{la,lb}_t transposed: [variant][axis][la][lb][t][pair]
  int64_t eskip;              // offset of the variant with |E| < 1e-30 set to zero
  int emaxa;                  // la, lb range of the transposed table (0..emaxa)
  int64_t npair;              // group pairs (the table's innermost extent)
  double *rec;                // records: [H, 1/4p+1/4p', kind, order, coefs...]
  int64_t recbase;
  int rs;
  unsigned long long *p0count; // P=Q quartets counted for this launch's class
  uint32_t *s2key;            // optional: stage-2 order key per quartet, (cls << 6) | h bucket
  int cls;                    // this launch's class index (for s2key)
  // geometry batches: blockIdx.y is the geometry; its tables, records and
  // counters sit these many elements after geometry 0's
  int64_t gs_pair, gs_esoa, gs_rec;
  // molecule batches, split contracted side: this item's X rows start xoff
  // doubles into the batch's contraction buffer, xstride per quartet, xg
  // contraction threads per quartet
  int64_t xoff;
  int xstride, xg;
  // every group of an s, p, d or f shell holds its (L+1)(L+2)/2 Cartesian
  // components in the order cart_component gives (the shell-templated
  // stage-1 kernels rely on it)
  int shells_canonical;
};

constexpr int MAXCLS = 20;

struct Stage2Args {
  const double *rec;
  int ncls;
  int64_t cls_begin[MAXCLS], cls_end[MAXCLS], cls_recoff[MAXCLS];
  int cls_rs[MAXCLS];
  int64_t nquart;
  int chunk;
  const double *q;
  int nq, nqp;
  int uniform;                // q (this tile) is uniform from index 1 with step dq
  int first_on_grid;          // q[0] lies on that grid too
  double dq;
  double *partial;            // this q tile's column of a (gridDim.x x pstride) array
  int64_t pstride;
};

// Stage 2 of one LLmax class: lanes over quartets, K quartets per lane.
struct Stage2ClassArgs {
  const double *rec;          // the class's first record
  int rs;                     // record stride (doubles)
  int64_t nquart;             // quartets in the class
  const uint32_t *perm;       // optional: slot -> quartet index (class-relative after subtracting pbase)
  int64_t pbase;
  const double *q;            // this q tile
  int nq;
  int uniform, first_on_grid; // q[1..nq) uniform with step dq; q[0] on that grid too
  double dq;
  int chunk;                  // q points per work item (multiple of 64), 0 = the whole tile
  int j2;                     // Bessel records are j2 (F / q^2)
  int lb;                     // Bessel order (read by the persistent molecule-batch kernel)
  double *partial;            // gridDim.x rows of pstride doubles, accumulated (+=)
  int64_t pstride;
  int64_t gs_rec, gs_partial; // per-geometry strides (blockIdx.y is the geometry)
};
// Stage-2 pair tile: quartets per lane k (1 or 2; orders above 8 always use
// 1) and warps per block nw (4 or 8).  Every shape sums the same quartets at
// the same points; only the order of the floating-point additions differs.
struct Stage2Tile {
  int k = 2;
  int nw = 4;
};
constexpr int STAGE2_MAXWARPS = 8;
// q points a stage-2 block holds in shared memory at once
constexpr int STAGE2_QTILE = 1024;
bool stage2_tile_valid(Stage2Tile t);
int stage2_quartets_per_warp(int LB, Stage2Tile t);
int stage2_class_blocks_per_sm(int LB, bool j2, int nq, Stage2Tile t);
cudaError_t launch_stage2_class(int LB, const Stage2ClassArgs &a, int grid, int ngeom, Stage2Tile t,
                                cudaStream_t st);
// Molecule batches: ONE persistent launch over every (plan, class, block)
// item.  Item i (descriptor d[i], Bessel order d[i].lb) owns the virtual
// blocks pre[i] .. pre[i+1]-1; resident blocks take virtual blocks from the
// atomic counter *next (zero before the launch) until all `blocks` are done,
// so no block waits on another.  Each virtual block writes its own partial
// row, which keeps the result independent of the schedule.
int stage2_persistent_blocks_per_sm(bool j2, int nqmax, Stage2Tile t);
cudaError_t launch_stage2_persistent(bool j2, const Stage2ClassArgs *d, const int64_t *pre, int n, int64_t blocks,
                                     int nqmax, int grid, Stage2Tile t, unsigned long long *next, cudaStream_t st);

// Aligned intensity of one LLmax class on q vectors (tb_aligned.cu).
struct AlignedArgs {
  const double *rec;          // class records [Hx, Hy, Hz, s, w K K' D_TUV...]
  int rs;
  int64_t nquart;
  const double *qv;           // nq vectors, (qx, qy, qz) interleaved
  int nq;
  double *partial;            // gridDim.y rows of pstride doubles, accumulated (+=)
  int64_t pstride;
};
cudaError_t launch_aligned(int L, const AlignedArgs &a, int slices, cudaStream_t st);

// Adjoint (tb_adjoint.cu): vector-Jacobian product of total j0 w.r.t. the centres.
struct AdjointQArgs {
  const double *rec;          // the class's forward records
  double *adj;                // per quartet: Jbar_b (b <= LLmax+1) or P = Q moments, same slots as rec
  int rs;
  int64_t nquart;
  const uint32_t *perm;       // optional visiting order (as stage 2)
  int64_t pbase;
  const double *q, *v;        // q grid and cotangent, nq each
  int nq;
  int uniform, first_on_grid;
  double dq;
  int64_t gs_rec;             // per-geometry record stride (blockIdx.y; v advances by nq)
};
struct AdjointFArgs {
  Stage1Args s1;              // the class's quartets, tables and density (as stage 1)
  const double *adj;          // stage-A output
  const double *dsoa;         // dE/dA_i table
  const double *ga, *xyz;     // per function
  double *gpart;              // gridDim.x rows of gstride doubles (3 per group), accumulated (+=)
  int64_t gstride;
  int64_t gs_dsoa, gs_xyz, gs_gpart;  // per-geometry strides (blockIdx.y); adj uses s1.gs_rec
};
int64_t dsoa_doubles(int ng, int maxa);
int adjoint_f_quartets_per_block(int L, bool split);
cudaError_t launch_pair_dtables(int ng, int maxa, const int *gstart, const double *ga, const double *xyz,
                                double *dsoa, int ngeom, int64_t gs_xyz, int64_t gs_dsoa, cudaStream_t st);
cudaError_t launch_adjoint_q(int LB1, const AdjointQArgs &a, int ngeom, cudaStream_t st);
cudaError_t launch_adjoint_f(int L, const AdjointFArgs &a, int grid, int ngeom, bool split, cudaStream_t st);

// Process-wide cache of device buffers (tb_pool.cu).
cudaError_t pool_malloc(void **p, size_t bytes);
void pool_free(void *p);

// Sets the calling thread's error string (thistle_last_error_string) and returns code.
int set_error(int code, const std::string &msg);

// Doubles of the transposed E table (both variants) for ng groups.
int64_t esoa_doubles(int ng, int maxa);
cudaError_t launch_pair_tables(int ng, int maxa, const int *gstart, const int *flmn, const double *ga,
                               const double *xyz, double *tab, double *esoa, int ngeom, int64_t gs_xyz,
                               int64_t gs_tab, int64_t gs_esoa, cudaStream_t st);
template <int K>
cudaError_t launch_stage1_k(int L, const Stage1Args &a, int ngeom, cudaStream_t st);
// Shell-templated stage 1 (one shell tuple ((Li 5 + Lj) 5 + Lk) 5 + Lr per
// launch): whether a class of this kind and LLmax takes it, and its launcher.
bool stage1_tpl(int kind, int L, int shells_canonical);
template <int K>
cudaError_t launch_stage1_tpl_k(int tuple, const Stage1Args &a, int ngeom, cudaStream_t st);
cudaError_t launch_stage1_tpl(int kind, int tuple, const Stage1Args &a, int ngeom, cudaStream_t st);
// molecule batches: n items of one shell tuple (descriptors d), item i's
// blocks pre[i] .. pre[i+1]-1 (128 quartets each)
template <int K>
cudaError_t launch_stage1_tpl_batch_k(int tuple, const Stage1Args *d, const int64_t *pre, int n, int64_t blocks,
                                      cudaStream_t st);
cudaError_t launch_stage1_tpl_batch(int kind, int tuple, const Stage1Args *d, const int64_t *pre, int n,
                                    int64_t blocks, cudaStream_t st);
cudaError_t launch_stage1(int kind, int L, const Stage1Args &a, int ngeom, cudaStream_t st);
template <int K>
cudaError_t launch_stage1_xk_k(int L, int LK, bool XB, const Stage1Args &a, int ngeom, cudaStream_t st);
// Whether a class of LLmax L with nquart quartets (summed over the plans of a
// molecule batch) goes through the contracted-side kernel, by sub-range of
// equal (LK = min(L_bra, L_ket), XB = L_bra < L_ket)
bool stage1_xk(int L, int64_t nquart, int nsm);
template <int K>
cudaError_t launch_stage1_batch_k(int L, int LK, int XB, const Stage1Args *d, const int64_t *pre, int n,
                                  int64_t blocks, cudaStream_t st);
cudaError_t launch_stage1_batch(int kind, int L, int LK, int XB, const Stage1Args *d, const int64_t *pre, int n,
                                int64_t blocks, cudaStream_t st);
int64_t stage1_item_blocks(int L, bool xk, int64_t n);
cudaError_t launch_stage1_xk(int kind, int L, int LK, bool XB, const Stage1Args &a, int ngeom, cudaStream_t st);
// nuclear-electron records of items a | gi << 16 | gk << 40 in [a.qbegin, a.qend)
// of pair order L (tb_nuclear.cu); nucrec holds [R_a, 0, Zn_a, 0, 0, 0] per nucleus
cudaError_t launch_nuclear(int L, const Stage1Args &a, const uint64_t *items, const double *nucrec,
                           cudaStream_t st);
// the same sub-range of one geometry as two kernels through xbuf (at least
// (qend - qbegin) * nout * ntuv(LK) doubles; nout = most outer function pairs)
// (with_xc false: the convolution alone, X already written by the
// shell-templated contraction launch_stage1_xct, one launch per shell tuple)
template <int K>
cudaError_t launch_stage1_xsplit_k(int L, int LK, bool XB, const Stage1Args &a, double *xbuf, int nout, bool with_xc,
                                   cudaStream_t st);
cudaError_t launch_stage1_xsplit(int kind, int L, int LK, bool XB, const Stage1Args &a, double *xbuf, int nout,
                                 cudaStream_t st, bool with_xc = true);
template <int K>
cudaError_t launch_stage1_xct_k(int tuple, bool XB, const Stage1Args &a, double *xbuf, int xstride, int64_t xbase,
                                cudaStream_t st);
// whether a contracted-side sub-range (kind, LK) takes the shell-templated
// contraction, and its launcher (a: the tuple's quartets; xbase: the first
// quartet of the sub-range, the buffer's row 0)
bool stage1_xct(int kind, int LK, int shells_canonical);
cudaError_t launch_stage1_xct(int kind, int tuple, bool XB, const Stage1Args &a, double *xbuf, int xstride,
                              int64_t xbase, cudaStream_t st);
// molecule batches: the shell-templated contraction over n items of one
// shell tuple (item i: blocks pre[i] .. pre[i+1]-1, X at xbuf + d[i].xoff
// from its first quartet, d[i].xg threads per quartet)
template <int K>
cudaError_t launch_stage1_xct_batch_k(int tuple, bool XB, const Stage1Args *d, const int64_t *pre, int n,
                                      int64_t blocks, double *xbuf, cudaStream_t st);
cudaError_t launch_stage1_xct_batch(int kind, int tuple, bool XB, const Stage1Args *d, const int64_t *pre, int n,
                                    int64_t blocks, double *xbuf, cudaStream_t st);
// molecule batches: the contraction (blocks from prexc; none when blocksxc is
// 0, X then written by launch_stage1_xct_batch) then the convolution (blocks
// from pre, as the fused kernel) over every item of one (L, LK, XB)
template <int K>
cudaError_t launch_stage1_xsplit_batch_k(int L, int LK, int XB, const Stage1Args *d, const int64_t *prexc,
                                         int64_t blocksxc, const int64_t *pre, int64_t blocks, int n, double *xbuf,
                                         cudaStream_t st);
cudaError_t launch_stage1_xsplit_batch(int kind, int L, int LK, int XB, const Stage1Args *d, const int64_t *prexc,
                                       int64_t blocksxc, const int64_t *pre, int64_t blocks, int n, double *xbuf,
                                       cudaStream_t st);
size_t stage2_smem_bytes(int nqp, int nwarps);
cudaError_t launch_stage2(const Stage2Args &a, int grid, int nwarps, cudaStream_t st);
cudaError_t launch_reduce(const double *partial, int nblocks, int nq, double *out, cudaStream_t st);
// geometry batches: ngeom independent (nblocks x nq) partial arrays, gs_in apart, into ngeom rows of out
cudaError_t launch_reduce_batch(const double *partial, int nblocks, int nq, int64_t gs_in, double *out, int ngeom,
                                cudaStream_t st);
cudaError_t launch_ghat_emit(const int *mat, const double *total, int nmat, int n, int *keys, double *vals,
                             cudaStream_t st);
cudaError_t launch_ghat_runs(const int *keys, const double *vals, int64_t m, double *G, cudaStream_t st);
// Density transform on the FP64 tensor cores (tb_transform.cu): D(m, j) =
// sum_{k < K} A(m, k) B(k, j) with A(m, k) = A[m + k sak + batch a_batch]
// (m contiguous) and B(k, j) = B[k sbk + j sbj], one of sbk, sbj equal to 1
// (b_jcontig: sbj == 1).  mode 0 stores D[m sdm + j sdj + batch d_batch];
// mode 1 the packed lower triangle j <= m at D[batch d_batch + m(m+1)/2 + j];
// mode 2 the columns j <= batch at D[(batch(batch+1)/2 + j) sdj + m].
struct DmmaGemmArgs {
  const double *A;
  int64_t sak, a_batch;
  const double *B;
  int64_t sbk, sbj;
  int M, N, K;
  double *D;
  int64_t sdm, sdj, d_batch;
};
cudaError_t launch_dmma_gemm(const DmmaGemmArgs &g, int mode, bool b_jcontig, int nbatch, cudaStream_t st);
// Ct[k][a] = C(k, a) (C column-major n x ngto), rows of transform_ct_width(ngto) doubles
int transform_ct_width(int ngto);
cudaError_t launch_transform_ct(const double *C, int n, int ngto, double *Ct, cudaStream_t st);
cudaError_t launch_iota(uint32_t *v, int64_t n, cudaStream_t st);
// elastic aligned intensity (tb_formfactor.cu): one record per unordered group
// pair (form_factor_record_doubles(npair) doubles at rec), then F(q) on nq q
// vectors (3 interleaved doubles each): real and imaginary part and |F|^2
int64_t form_factor_record_doubles(int64_t npair);
cudaError_t launch_form_factor(const Stage1Args &a, double *rec, const double *qv, int nq, double *out_re,
                               double *out_im, double *out_abs2, cudaStream_t st);
// molecule batches: pair tables of every item (blocks pre[i] .. pre[i+1]-1 of 128 pairs)
struct PairDesc {
  int ng, maxa;
  const int *gstart, *flmn;
  const double *ga, *xyz;
  double *tab, *esoa;
};
cudaError_t launch_pair_tables_batch(const PairDesc *d, const int64_t *pre, int n, int64_t blocks, cudaStream_t st);
// molecule batches: item i sums rows[i] partial rows of nq[i] points into out[i]
struct ReduceDesc {
  const double *partial;
  int rows, nq;
  double *out;
};
cudaError_t launch_reduce_desc(const ReduceDesc *d, int n, int nqmax, cudaStream_t st);
cudaError_t launch_sym_small(const double *in, int n, double *out, cudaStream_t st);
int stage2_blocks_per_sm(int nqp, int nwarps);
// all_pairs: every ket pair for every bra pair (the resolved CMS) instead of the five loops
cudaError_t launch_quartet_fill(int ng, const int64_t *bra_off, int64_t nquart, const int *gL,
                                uint64_t *quart, uint32_t *keys, bool all_pairs, cudaStream_t st);

}  // namespace tb
