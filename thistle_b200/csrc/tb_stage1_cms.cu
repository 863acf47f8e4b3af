// Stage-1 kernels of one calculation kind (see tb_stage1.cuh); one
// translation unit per kind so that the builds run in parallel.
#include "tb_stage1.cuh"

namespace tb {
template cudaError_t launch_stage1_k<KIND_CMS>(int L, const Stage1Args &a, int ngeom, cudaStream_t st);
template cudaError_t launch_stage1_xk_k<KIND_CMS>(int L, int LK, bool XB, const Stage1Args &a, int ngeom,
                                                      cudaStream_t st);
template cudaError_t launch_stage1_xsplit_k<KIND_CMS>(int L, int LK, bool XB, const Stage1Args &a, double *xbuf,
                                                     int nout, bool with_xc, cudaStream_t st);
template cudaError_t launch_stage1_xsplit_batch_k<KIND_CMS>(int L, int LK, int XB, const Stage1Args *d,
                                                           const int64_t *prexc, int64_t blocksxc, const int64_t *pre,
                                                           int64_t blocks, int n, double *xbuf, cudaStream_t st);
template cudaError_t launch_stage1_batch_k<KIND_CMS>(int L, int LK, int XB, const Stage1Args *d, const int64_t *pre,
                                                         int n, int64_t blocks, cudaStream_t st);
}  // namespace tb
