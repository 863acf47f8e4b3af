// Aligned (not orientationally averaged) total intensity on Cartesian q
// vectors: tot_integration_aligned with tot_integral_k_ijkr_alig
// (src/Integrals.f90:1425-1573, 5588-5727), tables of
// src/main_calculation.f90:194-205.
//
// Per group quartet the reference forms
//   h(q) = sum prod6 (i q)^{l'm'n'} (-i q)^{lmn},  f = h exp(i q.H) E12 E12'
// over all ng^4 ordered quartets.  With the Hermite density D_TUV of stage 1
// (bra sign included) h(q) = sum_TUV D_TUV (i qx)^T (i qy)^U (i qz)^V.
// Exchanging bra and ket turns D_TUV into (-1)^{T+U+V} D_TUV and H into -H,
// i.e. f into its complex conjugate, and exchanging the two functions of a
// pair leaves f unchanged; so the ordered sum equals
//   sum over the five-loop quartet list of  w Re f,
// w the loop weight (8, 4, 4, 2, 1), and its imaginary part vanishes.
//
// Layout: one thread per q vector (128 per block), blockIdx.y slices the
// class's quartets; a block stages QC records in shared memory and every
// thread evaluates them for its vector.  Per quartet and vector:
//   Z_TU = sum_V D_TUV (i qz)^V,  Y_T = sum_U (i qy)^U Z_TU,
//   X = sum_T (i qx)^T Y_T,  Re f = exp(-q^2 s) (Re X cos q.H - Im X sin q.H).
// Each block adds its slice's sum into row blockIdx.y of the partial array
// (launches of one stream run in order, so the sum is deterministic).
#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_kernels.h"
#include "tb_math.cuh"

namespace tb {

namespace {

constexpr int AL_THREADS = 128;
constexpr int AL_QC = 32;  // records staged per round (fewer for long records)
__host__ __device__ inline int al_qc(int rs) { return rs * AL_QC * 8 <= 160 * 1024 ? AL_QC : (160 * 1024 / 8) / rs; }

template <int L>
__device__ __forceinline__ constexpr int al_dindex(int T, int U, int V) {
  return ntuv(L) - ntuv(L - T) + U * (L - T + 1) - (U * (U - 1)) / 2 + V;
}

template <int L>
__global__ void __launch_bounds__(AL_THREADS) aligned_kernel(AlignedArgs A) {
  extern __shared__ double sr[];
  const int iq = blockIdx.x * AL_THREADS + threadIdx.x;
  const bool act = iq < A.nq;
  const double qx = act ? A.qv[3 * iq] : 0.0, qy = act ? A.qv[3 * iq + 1] : 0.0, qz = act ? A.qv[3 * iq + 2] : 0.0;
  const double q2 = qx * qx + qy * qy + qz * qz;
  // (-1)^floor(n/2) q^n: (i q)^n is this for even n and i times it for odd n
  double xs[L + 1], ys[L + 1], zs[L + 1];
  xs[0] = ys[0] = zs[0] = 1.0;
#pragma unroll
  for (int n = 1; n <= L; ++n) {
    xs[n] = xs[n - 1] * qx;
    ys[n] = ys[n - 1] * qy;
    zs[n] = zs[n - 1] * qz;
  }
#pragma unroll
  for (int n = 2; n <= L; n += 4) {
    xs[n] = -xs[n];
    ys[n] = -ys[n];
    zs[n] = -zs[n];
    if (n + 1 <= L) {
      xs[n + 1] = -xs[n + 1];
      ys[n + 1] = -ys[n + 1];
      zs[n + 1] = -zs[n + 1];
    }
  }
  const int64_t per = (A.nquart + gridDim.y - 1) / gridDim.y;
  const int64_t q0 = (int64_t)blockIdx.y * per, q1 = min(A.nquart, q0 + per);
  const int rs = A.rs;
  double acc = 0.0;
  const int qc = al_qc(rs);
  for (int64_t c0 = q0; c0 < q1; c0 += qc) {
    const int n = (int)min((int64_t)qc, q1 - c0);
    __syncthreads();
    for (int i = threadIdx.x; i < n * rs; i += AL_THREADS) sr[i] = A.rec[c0 * rs + i];
    __syncthreads();
    for (int t = 0; t < n; ++t) {
      const double *r = sr + t * rs;
      const double *D = r + 4;
      double Xr = 0.0, Xi = 0.0;
#pragma unroll
      for (int T = 0; T <= L; ++T) {
        double Yr = 0.0, Yi = 0.0;
#pragma unroll
        for (int U = 0; U <= L - T; ++U) {
          double Zr = 0.0, Zi = 0.0;
#pragma unroll
          for (int V = 0; V <= L - T - U; ++V) {
            const double d = D[al_dindex<L>(T, U, V)];
            if (V & 1) Zi = fma(d, zs[V], Zi);
            else Zr = fma(d, zs[V], Zr);
          }
          if (U & 1) {
            Yr = fma(-ys[U], Zi, Yr);
            Yi = fma(ys[U], Zr, Yi);
          } else {
            Yr = fma(ys[U], Zr, Yr);
            Yi = fma(ys[U], Zi, Yi);
          }
        }
        if (T & 1) {
          Xr = fma(-xs[T], Yi, Xr);
          Xi = fma(xs[T], Yr, Xi);
        } else {
          Xr = fma(xs[T], Yr, Xr);
          Xi = fma(xs[T], Yi, Xi);
        }
      }
      double sn, cs;
      sincos(qx * r[0] + qy * r[1] + qz * r[2], &sn, &cs);
      acc = fma(exp(-q2 * r[3]), Xr * cs - Xi * sn, acc);
    }
  }
  if (act) A.partial[(size_t)blockIdx.y * A.pstride + iq] += acc;
}

template <int L>
cudaError_t launch_aligned_l(const AlignedArgs &a, int slices, cudaStream_t st) {
  const size_t smem = sizeof(double) * (size_t)al_qc(a.rs) * a.rs;
  cudaError_t e = cudaFuncSetAttribute(aligned_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((a.nq + AL_THREADS - 1) / AL_THREADS, slices);
  aligned_kernel<L><<<grid, AL_THREADS, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_aligned(int L, const AlignedArgs &a, int slices, cudaStream_t st) {
  if (a.nquart <= 0 || a.nq <= 0) return cudaSuccess;
  switch (L) {
#define TB_A(n) case n: return launch_aligned_l<n>(a, slices, st);
    TB_A(0) TB_A(1) TB_A(2) TB_A(3) TB_A(4) TB_A(5) TB_A(6) TB_A(7) TB_A(8)
    TB_A(9) TB_A(10) TB_A(11) TB_A(12) TB_A(13) TB_A(14) TB_A(15) TB_A(16)
#undef TB_A
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace tb
