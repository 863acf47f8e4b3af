// The MO -> primitive transform of the 2-RDM (and the AO density of the
// 1-RDM) on the FP64 tensor cores: every pass is a GEMM whose inner
// dimension is the MO count,
//   D(m, j) = sum_k A(m, k) B(k, j),   k < K = n (a few tens),
// run by one hand-written kernel on mma.sync.aligned.m8n8k4 (f64 in, f64
// accumulate).  The chain replaces the reference's z11/z22 build and its
// per-quartet dgemm pair (src/Variables.f90:1045-1065, src/Integrals.f90:
// 109-127): rho(ab,cd) = sum Ghat[x][y][z][w] C(x,a) C(y,b) C(z,c) C(w,d),
// with Ghat the rows' eight index placements (tb_density.cu), as
//   T1[x y z](a) = sum_w C(w,a) Ghat[x][y][z][w]
//   V[x y](c<=d) = sum_z T1[x y z](d) C(z,c)        (packed pair c <= d)
//   T3[x](p, b)  = sum_y V[x y](p) C(y,b)
//   rho(p, (a<=b)) = sum_x T3[x](p, b) C(x,a)       (columns a <= b of each b)
// and the elastic Z = C1^T sym(D) C1 (src/Variables.f90:1199-1217) as two
// more of them.
//
// Tiling: a block of 4 warps owns a 64 x 64 tile of D; each warp a 32 x 32
// quarter as 4 x 4 fragments of 8 x 8.  A and B are staged k-major in shared
// memory ([k][m], [k][j]) with a row pitch of 68 doubles: the fragment loads
// (lane t reads row t & 3, column t >> 2) then touch 16 distinct bank pairs
// per half-warp.  K is staged in chunks of at most 64 (one chunk for the
// MO counts of the benchmark molecules), zero-padded to a multiple of 4.
// Sums over k run in order inside each fragment, so results do not depend
// on the launch configuration.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "tb_kernels.h"

namespace tb {

namespace {

constexpr int TG_M = 64, TG_N = 64, TG_KC = 64, TG_LD = 68;
constexpr int TG_THREADS = 128;

__device__ __forceinline__ void dmma884(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// Epilogues: 0 plain (D[m sdm + j sdj + batch d_batch]); 1 packed lower
// triangle of each batch (j <= m at D[batch d_batch + m(m+1)/2 + j]); 2 the
// columns j <= b of batch b at D[(b(b+1)/2 + j) sdj + m] (the pair density).
template <int MODE, bool BJ>
__global__ void __launch_bounds__(TG_THREADS) dmma_gemm_kernel(DmmaGemmArgs g) {
  extern __shared__ __align__(16) double tg_sm[];
  const int kcap = g.K < TG_KC ? (g.K + 3) / 4 * 4 : TG_KC;
  double *As = tg_sm;                 // [k][m]
  double *Bs = tg_sm + kcap * TG_LD;  // [k][j]
  const int64_t batch = blockIdx.z;
  const int m0 = blockIdx.x * TG_M, j0 = blockIdx.y * TG_N;
  int nlim = g.N;
  if (MODE == 2) nlim = min(nlim, (int)batch + 1);
  if (j0 >= nlim) return;
  if (MODE == 1 && j0 > m0 + TG_M - 1) return;  // only j > m: nothing stored
  const double *A = g.A + batch * g.a_batch;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  const int fr = lane & 3, fc = lane >> 2;  // fragment row (k) and column (m or j)
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  for (int k0 = 0; k0 < g.K; k0 += TG_KC) {
    const int kc = min(TG_KC, g.K - k0), kr = (kc + 3) / 4 * 4;
    if (k0 > 0) __syncthreads();
    // A: m contiguous in global memory
    for (int e = threadIdx.x; e < kr * TG_M; e += TG_THREADS) {
      const int k = e / TG_M, m = e % TG_M;
      double v = 0.0;
      if (k < kc && m0 + m < g.M) v = A[(int64_t)(m0 + m) + (int64_t)(k0 + k) * g.sak];
      As[k * TG_LD + m] = v;
    }
    if (BJ) {  // B: j contiguous
      for (int e = threadIdx.x; e < kr * TG_N; e += TG_THREADS) {
        const int k = e / TG_N, j = e % TG_N;
        double v = 0.0;
        if (k < kc && j0 + j < g.N) v = g.B[(int64_t)(k0 + k) * g.sbk + (j0 + j)];
        Bs[k * TG_LD + j] = v;
      }
    } else {  // B: k contiguous
      for (int e = threadIdx.x; e < kr * TG_N; e += TG_THREADS) {
        const int j = e / kr, k = e % kr;
        double v = 0.0;
        if (k < kc && j0 + j < g.N) v = g.B[(int64_t)(k0 + k) + (int64_t)(j0 + j) * g.sbj];
        Bs[k * TG_LD + j] = v;
      }
    }
    __syncthreads();
    for (int kk = 0; kk < kr; kk += 4) {
      const double *ar = As + (kk + fr) * TG_LD + wm + fc;
      const double *br = Bs + (kk + fr) * TG_LD + wn + fc;
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = ar[8 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = br[8 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma884(acc[i][j], af[i], bf[j]);
    }
  }
  // fragment element (i, j, h): m = m0 + wm + 8 i + fc, column j0 + wn + 8 j + 2 fr + h
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + wm + 8 * i + fc;
    if (m >= g.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = j0 + wn + 8 * j + 2 * fr + h;
        if (c >= nlim) continue;
        if (MODE == 0) {
          g.D[(int64_t)m * g.sdm + (int64_t)c * g.sdj + batch * g.d_batch] = acc[i][j][h];
        } else if (MODE == 1) {
          if (c <= m) g.D[batch * g.d_batch + (int64_t)m * (m + 1) / 2 + c] = acc[i][j][h];
        } else {
          g.D[(batch * (batch + 1) / 2 + c) * g.sdj + m] = acc[i][j][h];
        }
      }
  }
}

// Ct[k][a] = C(k, a) for a < ngto (C column-major n x ngto), zero up to cw
__global__ void tg_transpose_kernel(const double *__restrict__ C, int n, int ngto, int cw, double *__restrict__ Ct) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * cw) return;
  const int k = e / cw, a = e % cw;
  Ct[e] = a < ngto ? C[(int64_t)a * n + k] : 0.0;
}

template <int MODE, bool BJ>
cudaError_t launch_mode(const DmmaGemmArgs &g, int nbatch, cudaStream_t st) {
  const int kcap = g.K < TG_KC ? (g.K + 3) / 4 * 4 : TG_KC;
  const size_t smem = sizeof(double) * 2 * (size_t)kcap * TG_LD;
  cudaError_t e = cudaFuncSetAttribute(dmma_gemm_kernel<MODE, BJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)((g.M + TG_M - 1) / TG_M), (unsigned)((g.N + TG_N - 1) / TG_N), (unsigned)nbatch);
  dmma_gemm_kernel<MODE, BJ><<<grid, TG_THREADS, smem, st>>>(g);
  return cudaGetLastError();
}

}  // namespace

int transform_ct_width(int ngto) { return (ngto + 7) / 8 * 8; }

cudaError_t launch_transform_ct(const double *C, int n, int ngto, double *Ct, cudaStream_t st) {
  const int cw = transform_ct_width(ngto);
  tg_transpose_kernel<<<(n * cw + 255) / 256, 256, 0, st>>>(C, n, ngto, cw, Ct);
  return cudaGetLastError();
}

cudaError_t launch_dmma_gemm(const DmmaGemmArgs &g, int mode, bool b_jcontig, int nbatch, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || nbatch <= 0) return cudaSuccess;
  if (g.K <= 0 || nbatch > 65535) return cudaErrorInvalidValue;
  if ((g.N + TG_N - 1) / TG_N > 65535) {
    // plain stores: split the columns into launches of at most 65535 tiles
    if (mode != 0) return cudaErrorInvalidValue;
    const int step = 65535 * TG_N;
    for (int j = 0; j < g.N; j += step) {
      DmmaGemmArgs h = g;
      h.B = g.B + (int64_t)j * g.sbj;
      h.D = g.D + (int64_t)j * g.sdj;
      h.N = std::min(step, g.N - j);
      cudaError_t e = launch_dmma_gemm(h, 0, b_jcontig, nbatch, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  if (mode == 0) return b_jcontig ? launch_mode<0, true>(g, nbatch, st) : launch_mode<0, false>(g, nbatch, st);
  if (mode == 1) return b_jcontig ? launch_mode<1, true>(g, nbatch, st) : launch_mode<1, false>(g, nbatch, st);
  if (mode == 2) return b_jcontig ? launch_mode<2, true>(g, nbatch, st) : launch_mode<2, false>(g, nbatch, st);
  return cudaErrorInvalidValue;
}

}  // namespace tb
