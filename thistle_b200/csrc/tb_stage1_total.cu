// Stage-1 kernels of one calculation kind (see tb_stage1.cuh); one
// translation unit per kind so that the builds run in parallel.
#include "tb_stage1.cuh"

namespace tb {
template cudaError_t launch_stage1_k<KIND_TOTAL>(int L, const Stage1Args &a, int ngeom, cudaStream_t st);
template cudaError_t launch_stage1_tpl_k<KIND_TOTAL>(int tuple, const Stage1Args &a, int ngeom, cudaStream_t st);
template cudaError_t launch_stage1_xct_batch_k<KIND_TOTAL>(int tuple, bool XB, const Stage1Args *d, const int64_t *pre,
                                                           int n, int64_t blocks, double *xbuf, cudaStream_t st);
template cudaError_t launch_stage1_tpl_batch_k<KIND_TOTAL>(int tuple, const Stage1Args *d, const int64_t *pre, int n,
                                                           int64_t blocks, cudaStream_t st);
template cudaError_t launch_stage1_xct_k<KIND_TOTAL>(int tuple, bool XB, const Stage1Args &a, double *xbuf, int xstride,
                                                     int64_t xbase, cudaStream_t st);
template cudaError_t launch_stage1_xk_k<KIND_TOTAL>(int L, int LK, bool XB, const Stage1Args &a, int ngeom,
                                                      cudaStream_t st);
template cudaError_t launch_stage1_xsplit_k<KIND_TOTAL>(int L, int LK, bool XB, const Stage1Args &a, double *xbuf,
                                                     int nout, bool with_xc, cudaStream_t st);
template cudaError_t launch_stage1_xsplit_batch_k<KIND_TOTAL>(int L, int LK, int XB, const Stage1Args *d,
                                                           const int64_t *prexc, int64_t blocksxc, const int64_t *pre,
                                                           int64_t blocks, int n, double *xbuf, cudaStream_t st);
template cudaError_t launch_stage1_batch_k<KIND_TOTAL>(int L, int LK, int XB, const Stage1Args *d, const int64_t *pre,
                                                         int n, int64_t blocks, cudaStream_t st);

// Blocks one molecule-batch item of n quartets of class L needs (xk: the
// contracted-side kernel), matching the launchers above.
int64_t stage1_item_blocks(int L, bool xk, int64_t n) {
  if (n <= 0) return 0;
  if (xk) return (n + 127) / 128;
  if (L <= STAGE1_REG_MAXL) return (n * stage1_reg_split(L) * stage1_reg_parts(L) + 127) / 128;
  const int thr = stage1_smem_threads(L);
  return (n * stage1_smem_split(L) + thr - 1) / thr;
}
}  // namespace tb
