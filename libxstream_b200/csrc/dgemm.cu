/*
 * Plain FP64 GEMM on the FP64 tensor cores (DMMA, mma.sync m8n8k4): C = alpha*A*B + beta*C,
 * column-major, no transposes. The baseline the Ozaki int8 form is measured against.
 *
 * CTA tile 128 x 128, 8 warps of 64 x 32 (8 x 4 DMMA tiles, 128 accumulator registers), K step 16,
 * one CTA per SM; a 4-stage cp.async ring stages A as [k][m] and B as [n][k] (both as stored in global memory),
 * rows padded (A by 8, B by 2 doubles) so that the fragment loads of a warp touch every bank
 * exactly twice. Out-of-range rows, columns and k read as zero (cp.async zero fill); the epilogue
 * writes only in-range elements.
 */
#include "internal.h"
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

constexpr int kBM = 128, kBN = 128, kBK = 16, kStages = 4, kThreads = 256;
constexpr int kAStride = kBM + 8; /* doubles per k row of the A tile */
constexpr int kBStride = kBK + 2; /* doubles per n row of the B tile */
constexpr int kATile = kBK * kAStride, kBTile = kBN * kBStride;

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

/* 16-byte (or 8-byte) asynchronous copy global -> shared; src_bytes < size zero-fills the rest. */
template <int SIZE>
__device__ __forceinline__ void cp_async(void* dst, const void* src, int src_bytes) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  if constexpr (16 == SIZE) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
  }
  else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
  }
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

/* VEC = 2: 16-byte copies (lda, ldb even and 16-byte aligned bases); VEC = 1: 8-byte copies. */
template <int VEC>
__device__ __forceinline__ void load_tiles(double* sa, double* sb, const double* __restrict__ A, const double* __restrict__ B,
  int M, int N, int K, long long lda, long long ldb, int m0, int n0, int k0) {
  constexpr int A_CHUNKS = kBK * kBM / VEC, B_CHUNKS = kBN * kBK / VEC;
  for (int c = threadIdx.x; c < A_CHUNKS; c += kThreads) { /* A: column k has m contiguous */
    const int kk = c / (kBM / VEC), mm = (c - kk * (kBM / VEC)) * VEC;
    const int gm = m0 + mm, gk = k0 + kk;
    const int valid = (gk < K) ? max(0, min(VEC, M - gm)) : 0;
    const double* src = A + (valid > 0 ? (long long)gk * lda + gm : 0);
    cp_async<8 * VEC>(sa + kk * kAStride + mm, src, 8 * valid);
  }
  for (int c = threadIdx.x; c < B_CHUNKS; c += kThreads) { /* B: column n has k contiguous */
    const int nn = c / (kBK / VEC), kk = (c - nn * (kBK / VEC)) * VEC;
    const int gn = n0 + nn, gk = k0 + kk;
    const int valid = (gn < N) ? max(0, min(VEC, K - gk)) : 0;
    const double* src = B + (valid > 0 ? (long long)gn * ldb + gk : 0);
    cp_async<8 * VEC>(sb + nn * kBStride + kk, src, 8 * valid);
  }
}

template <int VEC>
__global__ void __launch_bounds__(kThreads, 1)
  xs_dgemm_kernel(int M, int N, int K, double alpha, const double* __restrict__ A, long long lda, const double* __restrict__ B,
    long long ldb, double beta, double* __restrict__ C, long long ldc) {
  extern __shared__ double smem[];
  double* const sA = smem;
  double* const sB = smem + kStages * kATile;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int wm = (warp & 1) * 64, wn = (warp >> 1) * 32;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int nk = (K + kBK - 1) / kBK;
  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) load_tiles<VEC>(sA + s * kATile, sB + s * kBTile, A, B, M, N, K, lda, ldb, m0, n0, s * kBK);
    cp_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_wait<kStages - 2>();
    __syncthreads();
    { /* refill the stage consumed in the previous iteration */
      const int nt = kt + kStages - 1;
      if (nt < nk) load_tiles<VEC>(sA + (nt % kStages) * kATile, sB + (nt % kStages) * kBTile, A, B, M, N, K, lda, ldb, m0, n0, nt * kBK);
      cp_commit();
    }
    const double* const a = sA + (kt % kStages) * kATile;
    const double* const b = sB + (kt % kStages) * kBTile;
#pragma unroll
    for (int ks = 0; ks < kBK / 4; ++ks) {
      double fa[8], fb[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) fa[i] = a[(ks * 4 + t) * kAStride + wm + i * 8 + g];
#pragma unroll
      for (int j = 0; j < 4; ++j) fb[j] = b[(wn + j * 8 + g) * kBStride + ks * 4 + t];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], fa[i], fb[j]);
    }
  }
  cp_wait<0>();
  /* epilogue: lane holds C(g, 2t) and C(g, 2t+1) of every 8 x 8 tile */
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int row = m0 + wm + i * 8 + g;
    if (row >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int col = n0 + wn + j * 8 + 2 * t + h;
        if (col < N) {
          double* const p = C + row + (long long)col * ldc;
          *p = (0.0 == beta) ? alpha * acc[i][j][h] : fma(alpha, acc[i][j][h], beta * *p);
        }
      }
    }
  }
}

constexpr size_t smem_bytes() { return sizeof(double) * kStages * (kATile + kBTile); }

template <int VEC>
cudaError_t launch(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb, double beta, double* C,
  int ldc, cudaStream_t s) {
  const cudaError_t r = (cudaError_t)xs_func_smem((const void*)xs_dgemm_kernel<VEC>, smem_bytes());
  if (cudaSuccess != r) return r;
  const dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
  xs_dgemm_kernel<VEC><<<grid, kThreads, smem_bytes(), s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  return cudaGetLastError();
}

}  // namespace

extern "C" int xs_dgemm(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb, double beta,
  double* C, int ldc, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (M < 0 || N < 0 || K < 0 || lda < (M > 1 ? M : 1) || ldb < (K > 1 ? K : 1) || ldc < (M > 1 ? M : 1)) {
    return (int)cudaErrorInvalidValue;
  }
  if (0 == M || 0 == N) return 0;
  const bool vec = (0 == (lda & 1)) && (0 == (ldb & 1)) && (0 == ((uintptr_t)A & 15)) && (0 == ((uintptr_t)B & 15));
  void* prof = xs_profile_begin(stream);
  const cudaError_t r = vec ? launch<2>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, s)
                            : launch<1>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, s);
  xs_profile_end(prof, "dgemm", 2.0 * M * N * (double)K, 0.0, stream);
  return (int)r;
}
