/*
 * Ozaki scheme-1 FP64 GEMM on the int8 tensor cores (tcgen05 with tensor-memory accumulators).
 *
 * C = alpha * op(A) * op(B) + beta * C, FP64, column-major (BLAS conventions). Each row of op(A)
 * and each column of op(B) is scaled by its largest power of two (the biased exponent of its
 * largest entry) and split into `nslices` signed 7-bit digits of the aligned 53-bit significand,
 * as the reference does (samples/ozaki/kernels/ozaki_common.cl:789-834 digit rule,
 * samples/ozaki/kernels/ozaki1_int8.cl:428-589 preprocessing): digit s holds bits
 * [46-7s, 52-7s] of the aligned significand; the eighth digit (bits [0,3]) is stored multiplied by
 * 8, so that every digit s carries weight 2^(46-7s) and a slice pair (sa, sb) weighs
 * 2^(92-7(sa+sb)). All pairs with sa + sb <= cutoff are multiplied on the tensor cores (int8 x int8
 * -> exact int32 sums); pairs of one anti-diagonal d = sa + sb share one tensor-memory
 * accumulator (their scales are equal), so one FP64 recombination per diagonal suffices:
 *   C(i,j) += alpha * 2^(ea_i + eb_j - 2058 - 7d) * D_d(i,j)        (ozaki1_int8.cl:740-790).
 * Exactness of the int32 sums: |digit| <= 127 and a diagonal holds at most 8 pairs, so a K range
 * of at most 16384 keeps |D_d| < 8 * 16384 * 127^2 < 2^31; longer K runs in chunks of 16384.
 *
 * Device layout: digit planes dA[s][M][Kp] and dB[s][N][Kp] (int8, K contiguous, Kp = K rounded
 * up to 16, zero padded), exponents ea[M], eb[N] (int32).
 *
 * GEMM kernel, two forms (GemmForm): one CTA per 128 x BN tile of C, 6 warps. Warp 0 (one lane)
 * streams (pair, k-block) tiles of both operands into a shared-memory ring with TMA (3-D tensor maps
 * over the digit planes, 128-byte swizzle, out-of-range rows and k read as zero); warp 1 owns all 512
 * tensor-memory columns and one lane issues tcgen05.mma (M=128, N=BN, K=32) per 32-byte K step,
 * committing each stage back to the producer and each finished diagonal to the epilogue; warps 2-5
 * (one tensor-memory lane quarter each) read a finished int32 accumulator with tcgen05.ld, scale it
 * and add it in FP64, then hand it back, so the tensor cores work on diagonal d+1 while diagonal d is
 * being recombined.
 *  - partial form (BN = 128, 6 stages; M*N up to 4096^2): two 128-column accumulators and the tile's
 *    FP64 partial sum (two 32-bit columns per C column) share tensor memory; the partial sum stays
 *    there from diagonal to diagonal (tcgen05.st), so C is read once (beta) at the first diagonal and
 *    written once at the last;
 *  - read-modify-write form (BN = 256, 4 stages; larger products): two 256-column accumulators, each
 *    diagonal added into C. A 256-wide tile needs 25 % fewer operand bytes per MAC; above 4096^2 that
 *    outweighs the per-diagonal C traffic (measured; neither a CTA pair sharing B tiles nor shorter
 *    K ranges per launch were faster).
 * Every mbarrier wait is bounded: a stalled pipeline ends the kernel with an error status (per-call
 * abort word and the library's device error word) instead of a hang.
 */
#include "internal.h"
#include "tc_ptx.cuh"
#include "ozaki_digits.cuh"
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <string.h>

extern "C" unsigned* xs_device_error_ptr(void);

namespace {
using namespace xs_tc;
using namespace xs_oz;

/* Two forms of the GEMM kernel (GemmForm): 128 x 128 C tiles whose FP64 partial sum stays in tensor
   memory across anti-diagonals (C read and written once; 6 stages), and 128 x 256 tiles that add each
   diagonal into C (read-modify-write per diagonal; 4 stages, 25 % fewer operand bytes per MAC). The
   first is faster up to M*N = 4096^2, the second above (measured on B200). */
constexpr int kBM = 128, kBK = 128;
template <bool PARTIAL>
struct GemmForm {
  static constexpr int BN = PARTIAL ? 128 : 256, STAGES = PARTIAL ? 6 : 4;
  static constexpr int ATILE = kBM * kBK, BTILE = BN * kBK;
  static constexpr uint32_t PART_COL = 2 * BN; /* tensor-memory column of the FP64 partial sum (2 per C column) */
  static constexpr size_t smem_bytes() {
    return 1024 /* alignment slack */ + (size_t)STAGES * (ATILE + BTILE) + (2 * STAGES + 4) * sizeof(uint64_t) +
           16 /* tensor-memory address */ + BN * sizeof(int);
  }
};
constexpr long long kPartialMaxMN = 4096ll * 4096ll; /* largest M*N run by the tensor-memory partial form */
constexpr int kMaxSlices = 8;
constexpr int kMaxPairs = kMaxSlices * kMaxSlices;
constexpr int kMaxGroups = 2 * kMaxSlices - 1;
constexpr int kKChunkBlocks = 16384 / kBK; /* k-blocks per launch: keeps every diagonal's int32 sum exact */
constexpr int kGemmThreads = 192;
constexpr int kGroupM = 8; /* row panels per rasterization group */
constexpr unsigned kErrOzakiTimeout = 4u; /* device error word bit: an Ozaki pipeline wait timed out */

/* ------------------------------------------------------------------------------ slicing */

/* Row maxima of the biased exponent, rows contiguous in memory: element (r, k) at x[r + k*ld].
   Grid (ceil(R/256), k-chunks); partial maxima meet in emax[] (zeroed by the caller) by atomicMax. */
__global__ void xs_oz_rowexp_rc(const double* __restrict__ x, long long ld, int R, int K, int kchunk, int* __restrict__ emax) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const int k0 = blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
  int e = 0;
  for (int k = k0; k < k1; ++k) e = max(e, biased_exp(x[r + (long long)k * ld]));
  if (0 != e) atomicMax(emax + r, e);
}

/* Row maxima with k contiguous: element (r, k) at x[k + r*ld]; one warp per row. */
__global__ void xs_oz_rowexp_kc(const double* __restrict__ x, long long ld, int R, int K, int* __restrict__ emax) {
  const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (r >= R) return;
  const double* const row = x + (long long)r * ld;
  int e = 0;
  for (int k = lane; k < K; k += 32) e = max(e, biased_exp(row[k]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, o));
  if (0 == lane) emax[r] = e;
}

/* Digits of 16 consecutive k of one row into the planes d[s][r][k0 .. k0+15]. */
__device__ __forceinline__ void slice16(const double (&v)[16], int erow, int ns, signed char* __restrict__ d, long long plane,
  long long off) {
  unsigned long long al[16];
  unsigned sg[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    int be;
    unsigned long long mt;
    ieee_split(v[j], sg[j], be, mt);
    const int sh = erow - be;
    al[j] = (0 != mt && sh <= 52) ? (mt >> sh) : 0ull;
  }
  for (int s = 0; s < ns; ++s) {
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t x = 0;
#pragma unroll
      for (int b = 0; b < 4; ++b) x |= ((uint32_t)(slice_digit(al[q * 4 + b], sg[q * 4 + b], s) & 0xFF)) << (8 * b);
      w[q] = x;
    }
    *reinterpret_cast<uint4*>(d + s * plane + off) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

/* Slicing with k contiguous (element (r, k) at x[k + r*ld]): one thread per (row, 16 k). */
__global__ void xs_oz_slice_kc(const double* __restrict__ x, long long ld, int R, int K, int Kp, const int* __restrict__ emax,
  int ns, signed char* __restrict__ d) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int kg = Kp / 16;
  if (t >= (long long)R * kg) return;
  const int r = (int)(t / kg), k0 = (int)(t - (long long)r * kg) * 16;
  const double* const row = x + (long long)r * ld;
  double v[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = (k0 + j < K) ? row[k0 + j] : 0.0;
  slice16(v, emax[r], ns, d, (long long)R * Kp, (long long)r * Kp + k0);
}

/* Slicing with rows contiguous (element (r, k) at x[r + k*ld]): threads of a block run over rows
   (coalesced reads), blockIdx.y over groups of 16 k. */
__global__ void xs_oz_slice_rc(const double* __restrict__ x, long long ld, int R, int K, int Kp, const int* __restrict__ emax,
  int ns, signed char* __restrict__ d) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const int k0 = blockIdx.y * 16;
  double v[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = (k0 + j < K) ? x[r + (long long)(k0 + j) * ld] : 0.0;
  slice16(v, emax[r], ns, d, (long long)R * Kp, (long long)r * Kp + k0);
}

/* C = beta * C (K == 0 or alpha == 0). */
__global__ void xs_oz_scale_c(double* __restrict__ c, long long ldc, int M, int N, double beta) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)M * N) return;
  const int j = (int)(t / M), i = (int)(t - (long long)j * M);
  double* const p = c + i + (long long)j * ldc;
  *p = (0.0 == beta) ? 0.0 : beta * *p;
}

/* ------------------------------------------------------------------------------ GEMM */

struct OzGroup {
  int p0, p1;  /* pairs [p0, p1) of the pair list */
  int eshift;  /* -2058 - 7d for diagonal d */
  int pad;
};

struct OzGemmArgs {
  int M, N, kb0, kb1; /* k-blocks [kb0, kb1) of 128 */
  int ngroups;
  int first; /* 1: this launch applies beta to C */
  double alpha, beta;
  const int* ea;
  const int* eb;
  double* C;
  long long ldc;
  unsigned* abort; /* per-call abort word (zeroed by the host before the first launch) */
  unsigned* dev_err;
  long long wait_limit; /* bound of every pipeline wait, clock cycles */
  unsigned char sa[kMaxPairs], sb[kMaxPairs];
  OzGroup g[kMaxGroups];
};

/* alpha * v * 2^E added to c, exactly scaled by 2^E whenever that is a normal number. */
__device__ __forceinline__ double add_scaled(double c, int v, int E, double alpha) {
  double t;
  if (E >= -1022 && E <= 1023) t = (double)v * __longlong_as_double((long long)(E + 1023) << 52);
  else t = ldexp((double)v, E);
  return fma(alpha, t, c);
}

template <bool PARTIAL>
__global__ void __launch_bounds__(kGemmThreads, 1)
  xs_ozaki_gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
    const __grid_constant__ OzGemmArgs args) {
  using F = GemmForm<PARTIAL>;
  constexpr int kBN = F::BN, kStages = F::STAGES, kATileBytes = F::ATILE, kBTileBytes = F::BTILE;
  constexpr uint32_t kPartCol = F::PART_COL;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* const smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* const sA = smem;
  unsigned char* const sB = smem + kStages * kATileBytes;
  uint64_t* const bars = (uint64_t*)(sB + kStages * kBTileBytes);
  uint64_t* const full = bars;
  uint64_t* const empty = bars + kStages;
  uint64_t* const accf = bars + 2 * kStages;
  uint64_t* const acce = accf + 2;
  uint32_t* const tmem_slot = (uint32_t*)(acce + 2);
  int* const s_eb = (int*)(tmem_slot + 4);
  unsigned* const abort = args.abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  /* tile order: groups of kGroupM row panels sweep the column panels together, so that the CTAs of
     one wave share their A row panels and B column panels in L2 */
  int n0, m0;
  {
    const int ntm = (args.M + kBM - 1) / kBM, ntn = (args.N + kBN - 1) / kBN;
    const int id = blockIdx.x, per_group = kGroupM * ntn, g = id / per_group, first = g * kGroupM;
    const int gsize = min(kGroupM, ntm - first), r = id - g * per_group;
    m0 = (first + r % gsize) * kBM;
    n0 = (r / gsize) * kBN;
  }
  if (0 == threadIdx.x) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&accf[i], 1);
      mbar_init(&acce[i], 128);
    }
    fence_barrier_init();
    prefetch_tensormap(&mapA);
    prefetch_tensormap(&mapB);
  }
  if (1 == warp) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  for (int j = threadIdx.x; j < kBN; j += blockDim.x) s_eb[j] = (n0 + j < args.N) ? args.eb[n0 + j] : 0;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (0 == warp) { /* TMA producer */
    if (0 == lane) {
      int it = 0;
      bool ok = true;
      for (int g = 0; g < args.ngroups && ok; ++g) {
        for (int p = args.g[g].p0; p < args.g[g].p1 && ok; ++p) {
          const int za = args.sa[p], zb = args.sb[p];
          for (int kb = args.kb0; kb < args.kb1; ++kb, ++it) {
            const int stage = it % kStages;
            const uint32_t ph = (uint32_t)(it / kStages) & 1u;
            if (!(ok = mbar_wait(&empty[stage], ph ^ 1u, abort, 1u, args.wait_limit))) break;
            mbar_arrive_expect_tx(&full[stage], kATileBytes + kBTileBytes);
            tma_load_3d(sA + stage * kATileBytes, &mapA, kb * kBK, m0, za, &full[stage]);
            tma_load_3d(sB + stage * kBTileBytes, &mapB, kb * kBK, n0, zb, &full[stage]);
          }
        }
      }
    }
  }
  else if (1 == warp) { /* MMA issuer */
    if (0 == lane) {
      const uint32_t idesc = idesc_i8(kBM, kBN);
      int it = 0;
      bool ok = true;
      for (int g = 0; g < args.ngroups && ok; ++g) {
        const int buf = g & 1, use = g >> 1;
        if (!(ok = mbar_wait(&acce[buf], ((uint32_t)use & 1u) ^ 1u, abort, 2u, args.wait_limit))) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(buf * kBN);
        uint32_t acc = 0;
        for (int p = args.g[g].p0; p < args.g[g].p1 && ok; ++p) {
          for (int kb = args.kb0; kb < args.kb1; ++kb, ++it) {
            const int stage = it % kStages;
            const uint32_t ph = (uint32_t)(it / kStages) & 1u;
            if (!(ok = mbar_wait(&full[stage], ph, abort, 2u, args.wait_limit))) break;
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA + stage * kATileBytes), b0 = smem_u32(sB + stage * kBTileBytes);
#pragma unroll
            for (int kk = 0; kk < kBK / 32; ++kk) {
              mma_i8(d, desc_k_sw128(a0 + kk * 32), desc_k_sw128(b0 + kk * 32), idesc, acc);
              acc = 1;
            }
            mma_commit(&empty[stage]);
          }
        }
        if (ok) mma_commit(&accf[buf]);
      }
    }
  }
  else if constexpr (PARTIAL) { /* epilogue: warps 2..5, tensor-memory lane quarter warp % 4; this lane's row
                                   of the tile keeps its FP64 partial sum in tensor memory across diagonals */
    const int q = warp & 3;
    const int row = m0 + q * 32 + lane;
    const bool rok = row < args.M;
    const int ear = rok ? args.ea[row] : 0;
    const uint32_t tlane = tmem + ((uint32_t)(q * 32) << 16);
    const bool read_c = (0 == args.first) || 0.0 != args.beta;
    for (int g = 0; g < args.ngroups; ++g) {
      const int buf = g & 1, use = g >> 1;
      if (!mbar_wait(&accf[buf], (uint32_t)use & 1u, abort, 8u, args.wait_limit)) break;
      tc_fence_after();
      const int eshift = args.g[g].eshift;
      const bool first_g = (0 == g), last_g = (g + 1 == args.ngroups);
      for (int c0 = 0; c0 < kBN; c0 += 16) {
        uint32_t v[16], pw[32];
        tmem_ld16(tlane + (uint32_t)(buf * kBN + c0), v);
        if (!first_g) tmem_ld32(tlane + kPartCol + (uint32_t)(2 * c0), pw);
        tmem_ld_wait();
        const int ncol = min(16, args.N - (n0 + c0));
        double* const crow = args.C + row + (long long)(n0 + c0) * args.ldc;
        double part[16];
        if (first_g) { /* the partial sum starts as beta * C (the call's first launch) or C (a later K range) */
#pragma unroll
          for (int j = 0; j < 16; ++j) part[j] = (rok && j < ncol && read_c) ? crow[(long long)j * args.ldc] : 0.0;
          if (0 != args.first) {
#pragma unroll
            for (int j = 0; j < 16; ++j) part[j] *= args.beta;
          }
        }
        else {
#pragma unroll
          for (int j = 0; j < 16; ++j) part[j] = __hiloint2double((int)pw[2 * j + 1], (int)pw[2 * j]);
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int iv = (int)v[j];
          if (0 != iv) part[j] = add_scaled(part[j], iv, ear + s_eb[c0 + j] + eshift, args.alpha);
        }
        if (last_g) {
          if (rok) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              if (j < ncol) crow[(long long)j * args.ldc] = part[j];
            }
          }
        }
        else {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            pw[2 * j] = (uint32_t)__double2loint(part[j]);
            pw[2 * j + 1] = (uint32_t)__double2hiint(part[j]);
          }
          tmem_st32(tlane + kPartCol + (uint32_t)(2 * c0), pw);
        }
      }
      if (!last_g) tmem_st_wait(); /* the partial sums are in tensor memory before the next diagonal reads them */
      tc_fence_before();
      mbar_arrive(&acce[buf]);
    }
  }
  else { /* epilogue: warps 2..5, tensor-memory lane quarter warp % 4; each diagonal is added into C */
    const int q = warp & 3;
    const int row = m0 + q * 32 + lane;
    const bool rok = row < args.M;
    const int ear = rok ? args.ea[row] : 0;
    const uint32_t tlane = tmem + ((uint32_t)(q * 32) << 16);
    for (int g = 0; g < args.ngroups; ++g) {
      const int buf = g & 1, use = g >> 1;
      if (!mbar_wait(&accf[buf], (uint32_t)use & 1u, abort, 8u, args.wait_limit)) break;
      tc_fence_after();
      const int eshift = args.g[g].eshift;
      const bool beta_now = (0 != args.first) && (0 == g);
      for (int c0 = 0; c0 < kBN; c0 += 32) {
        uint32_t v[32];
        tmem_ld32(tlane + (uint32_t)(buf * kBN + c0), v);
        tmem_ld_wait();
        if (rok) { /* all 32 loads of the chunk first, then the updates and the stores (no load waits for a
                      store it cannot be proven independent of) */
          double* const crow = args.C + row + (long long)(n0 + c0) * args.ldc;
          const int ncol = min(32, args.N - (n0 + c0));
          const bool read_c = !beta_now || 0.0 != args.beta;
          double cv[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) cv[j] = (j < ncol && read_c) ? crow[(long long)j * args.ldc] : 0.0;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            double c = beta_now ? args.beta * cv[j] : cv[j];
            const int iv = (int)v[j];
            if (0 != iv) c = add_scaled(c, iv, ear + s_eb[c0 + j] + eshift, args.alpha);
            cv[j] = c;
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (j < ncol) crow[(long long)j * args.ldc] = cv[j];
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&acce[buf]);
    }
  }
  if (0 != *(volatile unsigned*)abort) { /* let copies and MMAs still in flight land before TMEM goes */
    for (int i = 0; i < 200; ++i) __nanosleep(1000);
  }
  tc_fence_before();
  __syncthreads();
  if (1 == warp) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
  if (0 == threadIdx.x && 0 != *(volatile unsigned*)abort) atomicOr(args.dev_err, kErrOzakiTimeout);
}

/* ------------------------------------------------------------------------------ host */

PFN_cuTensorMapEncodeTiled_v12000 encode_fn(void) {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (nullptr == fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaSuccess == cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) &&
        cudaDriverEntryPointSuccess == q) {
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
  }
  return fn;
}

/* 3-D map over digit planes d[s][R][Kp] (int8), box 128 (k) x rows x 1, 128-byte swizzle. */
int make_plane_map(CUtensorMap* map, const void* base, int Kp, int R, int ns, int box_rows) {
  const PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
  if (nullptr == fn) return (int)cudaErrorNotSupported;
  const cuuint64_t dims[3] = {(cuuint64_t)Kp, (cuuint64_t)R, (cuuint64_t)ns};
  const cuuint64_t strides[2] = {(cuuint64_t)Kp, (cuuint64_t)Kp * (cuuint64_t)R};
  const cuuint32_t box[3] = {(cuuint32_t)kBK, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (CUDA_SUCCESS == r) ? 0 : (int)cudaErrorInvalidValue;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

/* Exponents and digit planes of op(X) viewed as R rows of K entries: element (r, k) at
   x[r + k*ld] when rows_contiguous, else at x[k + r*ld]. */
int slice_operand(const double* x, long long ld, bool rows_contiguous, int R, int K, int Kp, int ns, int* emax,
  signed char* planes, cudaStream_t s) {
  if (rows_contiguous) {
    const int kchunk = 256;
    xs_oz_rowexp_rc<<<dim3((R + 255) / 256, (K + kchunk - 1) / kchunk), 256, 0, s>>>(x, ld, R, K, kchunk, emax);
    xs_oz_slice_rc<<<dim3((R + 127) / 128, Kp / 16), 128, 0, s>>>(x, ld, R, K, Kp, emax, ns, planes);
  }
  else {
    xs_oz_rowexp_kc<<<(R + 7) / 8, 256, 0, s>>>(x, ld, R, K, emax);
    const long long n = (long long)R * (Kp / 16);
    xs_oz_slice_kc<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, ld, R, K, Kp, emax, ns, planes);
  }
  return (int)cudaGetLastError();
}

}  // namespace

extern "C" {

size_t xs_ozaki_gemm_scratch_bytes(int M, int N, int K, int nslices) {
  const size_t Kp = align_up((size_t)(K > 0 ? K : 1), 16);
  return align_up((size_t)nslices * M * Kp, 1024) + align_up((size_t)nslices * N * Kp, 1024) + align_up(sizeof(int) * M, 256) +
         align_up(sizeof(int) * N, 256) + 256;
}

int xs_ozaki_gemm(char transa, char transb, int M, int N, int K, double alpha, const double* a, int lda, const double* b,
  int ldb, double beta, double* c, int ldc, int nslices, int cutoff, void* scratch, size_t scratch_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const bool ta = ('T' == transa || 't' == transa || 'C' == transa || 'c' == transa);
  const bool tb = ('T' == transb || 't' == transb || 'C' == transb || 'c' == transb);
  if (M < 0 || N < 0 || K < 0 || nslices < 1 || nslices > kMaxSlices || ldc < (M > 1 ? M : 1)) return (int)cudaErrorInvalidValue;
  if (0 == M || 0 == N) return 0;
  if (0 == K || 0.0 == alpha) {
    if (1.0 == beta) return 0;
    const long long n = (long long)M * N;
    xs_oz_scale_c<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(c, ldc, M, N, beta);
    return (int)cudaGetLastError();
  }
  if (lda < (ta ? K : M) || ldb < (tb ? N : K)) return (int)cudaErrorInvalidValue;
  if (nullptr == scratch || scratch_bytes < xs_ozaki_gemm_scratch_bytes(M, N, K, nslices)) return (int)cudaErrorInvalidValue;
  const int maxcut = 2 * (nslices - 1);
  if (cutoff < 0 || cutoff > maxcut) cutoff = maxcut;
  const int Kp = (int)align_up((size_t)K, 16);
  char* p = (char*)scratch;
  signed char* const dA = (signed char*)p;
  p += align_up((size_t)nslices * M * Kp, 1024);
  signed char* const dB = (signed char*)p;
  p += align_up((size_t)nslices * N * Kp, 1024);
  int* const ea = (int*)p;
  p += align_up(sizeof(int) * M, 256);
  int* const eb = (int*)p;
  p += align_up(sizeof(int) * N, 256);
  unsigned* const abort = (unsigned*)p;
  int r = (int)cudaMemsetAsync(ea, 0, (size_t)(p - (char*)ea) + 256, s);
  if (0 != r) return r;
  /* rows of op(A): A(i, k) at a[i + k*lda] ('N') or a[k + i*lda] ('T'); columns of op(B): B(k, j)
     at b[k + j*ldb] ('N', k contiguous) or b[j + k*ldb] ('T') */
  void* prof = xs_profile_begin(stream);
  if (0 != (r = slice_operand(a, lda, !ta, M, K, Kp, nslices, ea, dA, s))) return r;
  if (0 != (r = slice_operand(b, ldb, tb, N, K, Kp, nslices, eb, dB, s))) return r;
  xs_profile_end(prof, "ozaki_slice", 0.0, 8.0 * ((double)M * K + (double)K * N), stream);
  CUtensorMap mapA, mapB;
  if (0 != (r = make_plane_map(&mapA, dA, Kp, M, nslices, kBM))) return r;
  const bool partial = (long long)M * N <= kPartialMaxMN;
  if (0 != (r = make_plane_map(&mapB, dB, Kp, N, nslices, partial ? GemmForm<true>::BN : GemmForm<false>::BN))) return r;
  OzGemmArgs args;
  memset(&args, 0, sizeof(args));
  args.M = M;
  args.N = N;
  args.alpha = alpha;
  args.beta = beta;
  args.ea = ea;
  args.eb = eb;
  args.C = c;
  args.ldc = ldc;
  args.abort = abort;
  args.dev_err = xs_device_error_ptr();
  args.wait_limit = xs_wait_limit();
  if (nullptr == args.dev_err) return (int)cudaErrorInvalidValue;
  int np = 0, ng = 0;
  for (int d = 0; d <= cutoff; ++d) { /* pairs ordered by anti-diagonal, one accumulation group each */
    const int p0 = np;
    for (int sa = 0; sa < nslices; ++sa) {
      const int sb = d - sa;
      if (sb < 0 || sb >= nslices) continue;
      args.sa[np] = (unsigned char)sa;
      args.sb[np] = (unsigned char)sb;
      ++np;
    }
    if (np > p0) {
      args.g[ng].p0 = p0;
      args.g[ng].p1 = np;
      args.g[ng].eshift = -2058 - 7 * d;
      ++ng;
    }
  }
  args.ngroups = ng;
  const size_t smem = partial ? GemmForm<true>::smem_bytes() : GemmForm<false>::smem_bytes();
  void (*const kernel)(const CUtensorMap, const CUtensorMap, const OzGemmArgs) =
    partial ? xs_ozaki_gemm_kernel<true> : xs_ozaki_gemm_kernel<false>;
  if (0 != (r = xs_func_smem((const void*)kernel, smem))) return r;
  const int nkb = (K + kBK - 1) / kBK, bn = partial ? GemmForm<true>::BN : GemmForm<false>::BN;
  const dim3 grid(((N + bn - 1) / bn) * ((M + kBM - 1) / kBM));
  for (int kb0 = 0; kb0 < nkb; kb0 += kKChunkBlocks) {
    args.kb0 = kb0;
    args.kb1 = (kb0 + kKChunkBlocks < nkb) ? kb0 + kKChunkBlocks : nkb;
    args.first = (0 == kb0) ? 1 : 0;
    prof = xs_profile_begin(stream);
    kernel<<<grid, kGemmThreads, smem, s>>>(mapA, mapB, args);
    if (0 != (r = (int)cudaGetLastError())) return r;
    const double kc = (double)(args.kb1 - args.kb0) * kBK;
    xs_profile_end(prof, "ozaki_gemm", 2.0 * M * N * (kc < K ? kc : K), 0.0, stream);
  }
  return 0;
}

}  // extern "C"
