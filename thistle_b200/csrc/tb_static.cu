// Stage 2 (the quartet x q Bessel sum) for callers that cannot allocate device
// memory.  Its only scratch -- one row of partial I(q) sums per thread block --
// lives in a fixed array compiled into this library instead of a cudaMalloc'd
// buffer; the caller hands in the stage-1 records, the q grid and the output.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "tb_kernels.h"
#include "thistle_b200.h"

namespace {

constexpr int kStaticBlocks = 296;  // two blocks on each of the B200's 148 SMs
constexpr int kStaticMaxQ = 1024;   // q points per call
constexpr int kMaxDevices = 64;

// Partial sums of every call on a device: 296 x 1024 doubles (2.4 MB), held by
// each GPU that loads the library until the process exits.  Every launch
// writes each row element it later reads, so nothing needs clearing.
static __device__ __align__(256) double g_partial_static[kStaticBlocks * kStaticMaxQ];

std::mutex g_mu;
double *g_scratch[kMaxDevices] = {nullptr};

}  // namespace

extern "C" int thistle_bessel_sum_static(const double *rec_dev, int32_t ncls, const int64_t *cls_begin,
                                         const int64_t *cls_end, const int64_t *cls_recoff, const int32_t *cls_rs,
                                         const double *q_dev, int32_t nq, double *result_dev, void *stream) {
  if (!rec_dev || !cls_begin || !cls_end || !cls_recoff || !cls_rs || !q_dev || !result_dev)
    return tb::set_error(THISTLE_ERR_ARG, "null argument");
  if (ncls < 1 || ncls > tb::MAXCLS) return tb::set_error(THISTLE_ERR_ARG, "ncls must be 1..20");
  if (nq < 1 || nq > kStaticMaxQ)
    return tb::set_error(THISTLE_ERR_ARG, "nq = " + std::to_string(nq) + " exceeds the static scratch (at most " +
                                              std::to_string(kStaticMaxQ) + " q points per call)");
  // the stage-2 kernel walks quartets 0 .. cls_end[ncls-1]: the table must start at 0
  if (cls_begin[0] != 0)
    return tb::set_error(THISTLE_ERR_SHAPE, "the first class must begin at quartet 0 (cls_begin[0] = " +
                                                std::to_string(cls_begin[0]) + ")");
  int64_t nquart = 0;
  for (int c = 0; c < ncls; ++c) {
    if (cls_begin[c] < 0 || cls_end[c] < cls_begin[c] || (c > 0 && cls_begin[c] != cls_end[c - 1]) ||
        cls_recoff[c] < 0 || cls_rs[c] < 4)
      return tb::set_error(THISTLE_ERR_SHAPE, "class table must be contiguous ranges with strides >= 4");
    nquart = cls_end[c];
  }
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return tb::set_error(THISTLE_ERR_CUDA, std::string("device query: ") + cudaGetErrorString(e));
  if (dev >= kMaxDevices) return tb::set_error(THISTLE_ERR_ARG, "device ordinal above 63");
  double *scratch = nullptr;
  {
    // first call on this device: host address of the device array, with the
    // device current
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_partial_static);
      if (e != cudaSuccess)
        return tb::set_error(THISTLE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_scratch[dev] = (double *)p;
    }
    scratch = g_scratch[dev];
  }
  const int nwarps = 8;
  int grid = std::min(kStaticBlocks, nsm * tb::stage2_blocks_per_sm(nq, nwarps));
  tb::Stage2Args s;
  s.rec = rec_dev;
  s.ncls = ncls;
  for (int c = 0; c < ncls; ++c) {
    s.cls_begin[c] = cls_begin[c];
    s.cls_end[c] = cls_end[c];
    s.cls_recoff[c] = cls_recoff[c];
    s.cls_rs[c] = cls_rs[c];
  }
  s.nquart = nquart;
  s.chunk = 4;
  s.q = q_dev;
  s.nq = nq;
  s.nqp = nq;
  s.partial = scratch;
  s.pstride = nq;
  s.uniform = 0;  // q is only on the device here: sincos/exp at every point
  s.first_on_grid = 0;
  s.dq = 0.0;
  cudaStream_t st = (cudaStream_t)stream;
  e = tb::launch_stage2(s, grid, nwarps, st);
  if (e == cudaSuccess) e = tb::launch_reduce(scratch, grid, nq, result_dev, st);
  if (e != cudaSuccess) return tb::set_error(THISTLE_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return THISTLE_OK;
}
