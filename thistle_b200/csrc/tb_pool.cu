// Device-memory cache shared by the plans of a process.
//
// A plan holds several GB (the pair density alone is Np^2 doubles) and the
// drop-in entry point builds and drops a plan per call, so cudaMalloc,
// and cudaFree (which also synchronises the device) would cost
// tens of milliseconds per call.  Buffers a plan releases stay cached, per
// device, and are handed to the next request of a similar size (at least the
// requested bytes, at most twice them); a failed cudaMalloc first returns
// every cached buffer of the device to the driver and tries again.  A plan
// synchronises its stream before it releases anything, so a reused buffer
// has no work pending on it.  thistle_release_device_cache() empties the
// cache of the current device.
#include <cuda_runtime.h>

#include <mutex>
#include <unordered_map>
#include <vector>

#include "tb_kernels.h"
#include "thistle_b200.h"

namespace tb {

namespace {

struct Block {
  void *p;
  size_t bytes;
  int dev;
};

std::mutex g_mu;
std::vector<Block> g_free;                  // cached, unused
std::unordered_map<void *, Block> g_live;   // handed out

size_t round_bytes(size_t n) {
  const size_t big = size_t(2) << 20, small = 512;
  if (n == 0) n = 1;
  return n >= (size_t(1) << 20) ? (n + big - 1) / big * big : (n + small - 1) / small * small;
}

// Frees the cached blocks of `dev` (g_mu held).
void drop_cached(int dev) {
  std::vector<Block> keep;
  for (const Block &b : g_free) {
    if (b.dev == dev) cudaFree(b.p);
    else keep.push_back(b);
  }
  g_free.swap(keep);
}

}  // namespace

cudaError_t pool_malloc(void **p, size_t bytes) {
  *p = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const size_t need = round_bytes(bytes);
  std::lock_guard<std::mutex> lock(g_mu);
  int best = -1;
  for (int i = 0; i < (int)g_free.size(); ++i) {
    const Block &b = g_free[i];
    if (b.dev != dev || b.bytes < need || b.bytes > 2 * need) continue;
    if (best < 0 || b.bytes < g_free[best].bytes) best = i;
  }
  if (best >= 0) {
    Block b = g_free[best];
    g_free.erase(g_free.begin() + best);
    g_live[b.p] = b;
    *p = b.p;
    return cudaSuccess;
  }
  e = cudaMalloc(p, need);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    drop_cached(dev);
    e = cudaMalloc(p, need);
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    return e;
  }
  g_live[*p] = Block{*p, need, dev};
  return cudaSuccess;
}

void pool_free(void *p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_live.find(p);
  if (it == g_live.end()) return;
  g_free.push_back(it->second);
  g_live.erase(it);
}

}  // namespace tb

extern "C" {

int thistle_release_device_cache(void) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return tb::set_error(THISTLE_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(tb::g_mu);
  tb::drop_cached(dev);
  return THISTLE_OK;
}

int thistle_device_cache_bytes(int64_t *cached, int64_t *in_use) {
  if (!cached || !in_use) return tb::set_error(THISTLE_ERR_ARG, "null argument");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return tb::set_error(THISTLE_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(tb::g_mu);
  int64_t c = 0, u = 0;
  for (const auto &b : tb::g_free)
    if (b.dev == dev) c += (int64_t)b.bytes;
  for (const auto &kv : tb::g_live)
    if (kv.second.dev == dev) u += (int64_t)kv.second.bytes;
  *cached = c;
  *in_use = u;
  return THISTLE_OK;
}

}  // extern "C"
