/*
 * Ozaki scheme-2 FP64 GEMM on the int8 tensor cores: Chinese-remainder (CRT) form.
 *
 * C = alpha * op(A) * op(B) + beta * C, FP64, column-major (BLAS conventions), the second scheme of
 * the reference's Ozaki sample (samples/ozaki/kernels/ozaki2_int8.cl:13-45, host set-up
 * samples/ozaki/ozaki_opencl.c:406-426). Each row of op(A) and each column of op(B) is scaled by its
 * largest power of two and turned into integers of MB bits (the aligned significands of
 * xs_oz::ieee_split, truncated to MB bits; MB = 53 keeps every bit of the largest entry). The exact
 * integer product A_int * B_int is then computed modulo q moduli m_1..m_q (pairwise coprime, at most
 * 256, so residues are unsigned bytes): one unsigned 8-bit GEMM per modulus on the tensor cores
 * (tcgen05.mma kind::i8, u8 x u8 -> exact int32 sums over up to 32768 k, reduced modulo m_i in the
 * epilogue and kept as one byte per modulus and output), and the integer is reconstructed from its
 * residues by the CRT with the "fractional" formula
 *     x / P = frac( sum_i r_i * y_i / m_i ),   P = prod m_i,  y_i = (P / m_i)^-1 mod m_i,
 * evaluated as a 128-bit binary fraction in integer arithmetic (y_i / m_i rounded to 2^-128; the sum
 * wraps modulo 2^128, which takes the fractional part, and read as a signed number it is centred:
 * x in [-P/2, P/2)), multiplied by P in double precision and scaled back:
 * C(i,j) = x * 2^(ea_i + eb_j - 2150 + 2 (53 - MB)).
 * The modulus count decides the precision: P must exceed 2 K 2^(2 MB), so q moduli carry
 * MB = floor((log2 P - ceil(log2 K) - 2) / 2) bits per input (capped at 53); the default takes the fewest
 * moduli that give MB = 53 for this K (16 up to K = 2^17).
 *
 * Device layout: residue planes rA[q][M][Kp] and rB[q][N][Kp] (u8, K contiguous, zero padded),
 * exponents ea[M], eb[N], residues of C R[q][N][M] (u8, column-major per modulus).
 *
 * GEMM kernel: persistent, one CTA per SM, 10 warps, the pipeline of the scheme-1 kernel over work
 * units (modulus, 128 x 256 tile of C) taken modulus-major and strided by the grid: warp 0 streams
 * the k-blocks of both operands' residue planes into a 4-stage shared-memory ring with TMA (128-byte
 * swizzle); warp 1 owns two 128 x 256 int32 accumulators in tensor memory and one lane issues the
 * MMAs; warps 2-9 (two per tensor-memory lane quarter, one column half each) reduce a finished
 * accumulator modulo m_i and store the bytes while the tensor cores work on the next unit. Every
 * mbarrier wait is bounded (per-call abort word, library device error word).
 */
#include "internal.h"
#include "tc_ptx.cuh"
#include "ozaki_digits.cuh"
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

extern "C" unsigned* xs_device_error_ptr(void);

namespace {
using namespace xs_tc;
using namespace xs_oz;

constexpr int kMaxMod = 20;
constexpr int kBM = 128, kBN = 256, kBK = 128, kStages = 4;
constexpr int kThreads = 320; /* producer, MMA issuer, 8 epilogue warps */
constexpr int kGroupM = 8;
/* k-blocks per launch: 32768 * 255^2 < 2^31 keeps every int32 sum exact */
constexpr int kKChunkBlocks = 32768 / kBK;
constexpr int kATileBytes = kBM * kBK, kBTileBytes = kBN * kBK;
constexpr unsigned kErrOzakiTimeout = 4u;

/* Pairwise coprime moduli <= 256, largest first (products of primes where composite). */
constexpr unsigned kModuli[kMaxMod] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                                       223, 217, 211, 199, 197, 193, 191, 181, 179, 173};

struct Oz2Consts {
  unsigned mod[kMaxMod];
  /* 32-bit residues (mod31): magic = floor(2^39 / m_i) + 1; c18 = 2^18 mod m_i, c36 = 2^36 mod m_i;
     cneg = -2^54 mod m_i */
  unsigned magic[kMaxMod], c18[kMaxMod], c36[kMaxMod], cneg[kMaxMod];
  double phi, plo; /* P as a double-double */
  int nmod, mb;
  /* w_i = y_i / m_i as a 128-bit binary fraction (floor(2^128 y_i / m_i)), least significant word
     first; y_i = (P / m_i)^-1 mod m_i */
  unsigned w[kMaxMod][4];
};

/* --------------------------------------------------------------------------- preprocessing */

/* Row maxima of the biased exponent, rows contiguous (element (r, k) at x[r + k*ld]); partial
   maxima meet in emax[] (zeroed by the caller) by atomicMax. */
__global__ void xs_oz2_rowexp_rc(const double* __restrict__ x, long long ld, int R, int K, int kchunk, int* __restrict__ emax) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const int k0 = blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
  int e = 0;
  for (int k = k0; k < k1; ++k) e = max(e, biased_exp(x[r + (long long)k * ld]));
  if (0 != e) atomicMax(emax + r, e);
}

/* Row maxima with k contiguous (element (r, k) at x[k + r*ld]); one warp per row. */
__global__ void xs_oz2_rowexp_kc(const double* __restrict__ x, long long ld, int R, int K, int* __restrict__ emax) {
  const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (r >= R) return;
  const double* const row = x + (long long)r * ld;
  int e = 0;
  for (int k = lane; k < K; k += 32) e = max(e, biased_exp(row[k]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, o));
  if (0 == lane) emax[r] = e;
}

/* |v| scaled to the row's largest exponent and truncated to mb bits, and its sign. */
__device__ __forceinline__ unsigned long long aligned_int(double v, int erow, int mb, unsigned& sign) {
  int be;
  unsigned long long mt;
  ieee_split(v, sign, be, mt);
  const int sh = erow - be + 53 - mb;
  return (0 != mt && sh < 64) ? (mt >> sh) : 0ull;
}


/* x mod m for x < 2^31 and m <= 256 from magic = floor(2^39 / m) + 1 (< 2^32 for m >= 129): the
   product x * magic / 2^39 is x/m + x*e/2^39 with 0 < e <= 1, x*e/2^39 < 2^-8 <= 1/m, and x/m is at
   most 1 - 1/m above an integer, so the shifted high product is floor(x / m) exactly. */
__device__ __forceinline__ unsigned mod31(unsigned x, unsigned m, unsigned magic) {
  return x - (__umulhi(x, magic) >> 7) * m;
}

/* 16 consecutive k of one row as signed integers (-1)^s u, u < 2^53. A negative value is held as
   u' = 2^54 - u (so that -u = u' + e (mod m) with e = -2^54 mod m), and u' <= 2^54 as 18-bit limbs
   a0 + a1 2^18 + a2 2^36: its residue is that of x = a0 + a1 c18 + a2 c36 + s e < 2^27
   (c = 2^18, 2^36 mod m), all 32-bit arithmetic. */
struct Limbs16 {
  unsigned a0[16], a1[16], a2[16], sg[16];
};

__device__ __forceinline__ void limbs16(const double (&v)[16], int erow, int mb, Limbs16& L) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    unsigned long long u = aligned_int(v[j], erow, mb, L.sg[j]);
    if (L.sg[j]) u = (1ull << 54) - u;
    L.a0[j] = (unsigned)u & 0x3ffffu;
    L.a1[j] = (unsigned)(u >> 18) & 0x3ffffu;
    L.a2[j] = (unsigned)(u >> 36);
  }
}

/* The 16 residues modulo m_i as bytes (k ascending). */
__device__ __forceinline__ uint4 residue_bytes16(const Limbs16& L, const Oz2Consts& cs, int i) {
  const unsigned m = cs.mod[i], mg = cs.magic[i], c1 = cs.c18[i], c2 = cs.c36[i], e = cs.cneg[i];
  unsigned r[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) r[j] = mod31(L.a0[j] + L.a1[j] * c1 + L.a2[j] * c2 + L.sg[j] * e, m, mg);
  uint32_t w[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    w[q] = __byte_perm(__byte_perm(r[4 * q], r[4 * q + 1], 0x0040u), __byte_perm(r[4 * q + 2], r[4 * q + 3], 0x0040u), 0x5410u);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

/* k contiguous (element (r, k) at x[k + r*ld]): one thread per (row, 16 k); VEC: 16-byte loads
   (x 16-byte aligned and ld even). */
template <bool VEC>
__global__ void xs_oz2_res_kc(const double* __restrict__ x, long long ld, int R, int K, int Kp, const int* __restrict__ emax,
  const __grid_constant__ Oz2Consts cs, unsigned char* __restrict__ d) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int kg = Kp / 16;
  if (t >= (long long)R * kg) return;
  const int r = (int)(t / kg), k0 = (int)(t - (long long)r * kg) * 16;
  const double* const row = x + (long long)r * ld;
  double v[16];
  if (VEC && k0 + 16 <= K) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double2 t2 = *reinterpret_cast<const double2*>(row + k0 + 2 * j);
      v[2 * j] = t2.x;
      v[2 * j + 1] = t2.y;
    }
  }
  else {
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = (k0 + j < K) ? row[k0 + j] : 0.0;
  }
  Limbs16 L;
  limbs16(v, emax[r], cs.mb, L);
  unsigned char* const dst = d + (long long)r * Kp + k0;
  const long long plane = (long long)R * Kp;
  for (int i = 0; i < cs.nmod; ++i) *reinterpret_cast<uint4*>(dst + i * plane) = residue_bytes16(L, cs, i);
}

/* rows contiguous (element (r, k) at x[r + k*ld]): a block of 256 threads takes 32 rows x 128 k,
   lane = row (coalesced loads), warp = 16 k. The residue bytes of four moduli at a time go through
   shared memory (rows padded to 144 bytes: the 16-byte chunks of 8 lanes fall in distinct banks) and
   leave as whole 128-byte row segments of each plane, so no 32-byte sector is written in part. */
constexpr int kRcRows = 32, kRcK = 128, kRcPitch = kRcK + 16, kRcMods = 4;
__global__ void __launch_bounds__(256) xs_oz2_res_rc(const double* __restrict__ x, long long ld, int R, int K, int Kp,
  const int* __restrict__ emax, const __grid_constant__ Oz2Consts cs, unsigned char* __restrict__ d) {
  __shared__ __align__(16) unsigned char tile[kRcMods][kRcRows * kRcPitch];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r0 = blockIdx.x * kRcRows, kt0 = blockIdx.y * kRcK;
  const int r = r0 + lane, k0 = kt0 + warp * 16;
  double v[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = (r < R && k0 + j < K) ? x[r + (long long)(k0 + j) * ld] : 0.0;
  Limbs16 L;
  limbs16(v, (r < R) ? emax[r] : 0, cs.mb, L);
  const long long plane = (long long)R * Kp;
  /* write-out role: row wr of the tile, 16-byte chunk wc */
  const int wr = threadIdx.x >> 3, wc = threadIdx.x & 7;
  const bool wok = (r0 + wr < R) && (kt0 + wc * 16 < Kp);
  unsigned char* const dst = d + (long long)(r0 + wr) * Kp + kt0 + wc * 16;
  for (int i0 = 0; i0 < cs.nmod; i0 += kRcMods) {
    const int nm = min(kRcMods, cs.nmod - i0);
    for (int ii = 0; ii < nm; ++ii) {
      *reinterpret_cast<uint4*>(&tile[ii][lane * kRcPitch + warp * 16]) = residue_bytes16(L, cs, i0 + ii);
    }
    __syncthreads();
    if (wok) {
      for (int ii = 0; ii < nm; ++ii) {
        *reinterpret_cast<uint4*>(dst + (i0 + ii) * plane) = *reinterpret_cast<const uint4*>(&tile[ii][wr * kRcPitch + wc * 16]);
      }
    }
    __syncthreads();
  }
}

/* C = beta * C (K == 0 or alpha == 0). */
__global__ void xs_oz2_scale_c(double* __restrict__ c, long long ldc, int M, int N, double beta) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)M * N) return;
  const long long j = t / M, i = t - j * M;
  double* const p = c + i + j * ldc;
  *p = (0.0 == beta) ? 0.0 : beta * *p;
}

/* ------------------------------------------------------------------------------------ GEMM */

struct Oz2GemmArgs {
  int M, N, kb0, kb1; /* k-blocks [kb0, kb1) of 128 */
  int nmod;
  int first; /* 1: the first k-chunk (residues are written, not accumulated) */
  unsigned mod[kMaxMod];
  unsigned magic[kMaxMod]; /* floor(2^39 / m_i) + 1 */
  unsigned char* R; /* [nmod][N][M] */
  unsigned* abort;
  unsigned* dev_err;
  long long wait_limit; /* bound of every pipeline wait, clock cycles */
};

constexpr size_t gemm_smem_bytes() {
  return 1024 /* alignment slack */ + (size_t)kStages * (kATileBytes + kBTileBytes) + 16 * sizeof(uint64_t) + 16;
}

/* instruction descriptor of tcgen05.mma kind::i8 with unsigned 8-bit A and B, s32 accumulator */
__host__ __device__ constexpr uint32_t idesc_u8(int M, int N) {
  return (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

/* Work unit u of the persistent GEMM: modulus q = u / ntiles (modulus-major, so the CTAs resident at
   one time read the residue planes of one or two moduli and those stay in L2), C tile by grouped
   rasterization (kGroupM row panels sweep the column panels together). */
__device__ __forceinline__ void unit_coords(int u, int ntiles, int ntm, int ntn, int& q, int& m0, int& n0) {
  q = u / ntiles;
  const int id = u - q * ntiles, per_group = kGroupM * ntn, g = id / per_group, first = g * kGroupM;
  const int gsize = min(kGroupM, ntm - first), r = id - g * per_group;
  m0 = (first + r % gsize) * kBM;
  n0 = (r / gsize) * kBN;
}

__global__ void __launch_bounds__(kThreads, 1)
  xs_ozaki2_gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
    const __grid_constant__ Oz2GemmArgs args) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* const smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* const sA = smem;
  unsigned char* const sB = smem + kStages * kATileBytes;
  uint64_t* const bars = (uint64_t*)(sB + kStages * kBTileBytes);
  uint64_t* const full = bars;
  uint64_t* const empty = bars + kStages;
  uint64_t* const accf = bars + 2 * kStages;
  uint64_t* const acce = accf + 2;
  uint32_t* const tmem_slot = (uint32_t*)(bars + 16);
  unsigned* const abort = args.abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntm = (args.M + kBM - 1) / kBM, ntn = (args.N + kBN - 1) / kBN, ntiles = ntm * ntn;
  const int nunits = ntiles * args.nmod;
  if (0 == threadIdx.x) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&accf[i], 1);
      mbar_init(&acce[i], kThreads - 64);
    }
    fence_barrier_init();
    prefetch_tensormap(&mapA);
    prefetch_tensormap(&mapB);
  }
  if (1 == warp) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (0 == warp) { /* TMA producer */
    if (0 == lane) {
      int it = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
        int q, m0, n0;
        unit_coords(u, ntiles, ntm, ntn, q, m0, n0);
        for (int kb = args.kb0; kb < args.kb1; ++kb, ++it) {
          const int stage = it % kStages;
          const uint32_t ph = (uint32_t)(it / kStages) & 1u;
          if (!(ok = mbar_wait(&empty[stage], ph ^ 1u, abort, 1u, args.wait_limit))) break;
          mbar_arrive_expect_tx(&full[stage], kATileBytes + kBTileBytes);
          tma_load_3d(sA + stage * kATileBytes, &mapA, kb * kBK, m0, q, &full[stage]);
          tma_load_3d(sB + stage * kBTileBytes, &mapB, kb * kBK, n0, q, &full[stage]);
        }
      }
    }
  }
  else if (1 == warp) { /* MMA issuer */
    if (0 == lane) {
      const uint32_t idesc = idesc_u8(kBM, kBN);
      int it = 0;
      bool ok = true;
      for (int u = blockIdx.x, i = 0; u < nunits && ok; u += gridDim.x, ++i) {
        const int buf = i & 1, use = i >> 1;
        if (!(ok = mbar_wait(&acce[buf], ((uint32_t)use & 1u) ^ 1u, abort, 2u, args.wait_limit))) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(buf * kBN);
        uint32_t acc = 0;
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
        if (ok) mma_commit(&accf[buf]);
      }
    }
  }
  else { /* epilogue: warps 2..9, tensor-memory lane quarter warp % 4 and column half (warp - 2) / 4;
            thread = one row of the tile, 128 columns */
    const int qd = warp & 3, cb = ((warp - 2) >> 2) * (kBN / 2);
    for (int u = blockIdx.x, i = 0; u < nunits; u += gridDim.x, ++i) {
      const int buf = i & 1, use = i >> 1;
      int q, m0, n0;
      unit_coords(u, ntiles, ntm, ntn, q, m0, n0);
      const int row = m0 + qd * 32 + lane;
      const bool rok = row < args.M;
      if (!mbar_wait(&accf[buf], (uint32_t)use & 1u, abort, 8u, args.wait_limit)) break;
      tc_fence_after();
      const unsigned m = args.mod[q];
      const unsigned mg = args.magic[q];
      unsigned char* const plane = args.R + (size_t)q * args.M * args.N;
      for (int c0 = cb; c0 < cb + kBN / 2; c0 += 32) {
        uint32_t v[32];
        tmem_ld32(tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(buf * kBN + c0), v);
        tmem_ld_wait();
        if (rok) {
          const int ncol = min(32, args.N - (n0 + c0));
          unsigned char* const dst = plane + row + (size_t)(n0 + c0) * args.M;
          if (!args.first) { /* a later k-chunk: add the residues so far */
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] += (j < ncol) ? dst[(size_t)j * args.M] : 0u;
          }
          if (32 == ncol) {
#pragma unroll
            for (int j = 0; j < 32; ++j) dst[(size_t)j * args.M] = (unsigned char)mod31(v[j], m, mg); /* < 2^31 */
          }
          else {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              if (j < ncol) dst[(size_t)j * args.M] = (unsigned char)mod31(v[j], m, mg);
            }
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

/* ---------------------------------------------------------------------------- reconstruction */

/* x * 2^E from the 128-bit fraction S of x / P (see xs_oz2_reconstruct). */
__device__ __forceinline__ double crt_value(const uint32_t (&S)[4], const Oz2Consts& cs, int E) {
  /* fraction = (T + U 2^-64) 2^-64, T the signed upper and U the unsigned lower 64 bits; T as a
     double plus the (exact, |.| <= 2^10) rest of its rounding */
  const long long T = (long long)(((unsigned long long)S[3] << 32) | S[2]);
  const unsigned long long U = ((unsigned long long)S[1] << 32) | S[0];
  const double th = __ll2double_rn(T);
  const double tl = __ll2double_rn(T - __double2ll_rn(th)) + __ull2double_rn(U) * 0x1p-64;
  const double x = fma(th, cs.phi, fma(th, cs.plo, tl * cs.phi)); /* x * 2^64 */
  E -= 64;
  return (E >= -1022 && E <= 1023) ? x * __longlong_as_double((long long)(E + 1023) << 52) /* exact */ : ldexp(x, E);
}

/* C(i,j) = alpha * x * 2^E + beta * C(i,j), x the centred integer with residues R[.][j][i]. A thread
   takes V consecutive rows i (one V-byte load per plane; V = 4 needs M % 4 == 0), grid rows take
   columns j (strided when N exceeds the grid).
   x / P = frac(sum_i r_i w_i) is summed as a 128-bit binary fraction: the wrap-around modulo 2^128
   takes the fractional part and the two's-complement reading of the sum centres it to [-1/2, 1/2)
   (x in [-P/2, P/2)). With w_i rounded down to 2^-128 the fraction is off by less than
   nmod * 255 * 2^-128 < 2^-115, i.e. x by less than 2^-115 P. */
template <int V>
__global__ void __launch_bounds__(256) xs_oz2_reconstruct(const unsigned char* __restrict__ R, int M, int N,
  const int* __restrict__ ea, const int* __restrict__ eb, const __grid_constant__ Oz2Consts cs, double alpha, double beta,
  double* __restrict__ C, long long ldc) {
  const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * V;
  if (i0 >= M) return;
  const size_t plane = (size_t)M * N;
  int ia[V];
#pragma unroll
  for (int v = 0; v < V; ++v) ia[v] = (i0 + v < M) ? ea[i0 + v] : 0;
  /* V residues per word; the next column's loads are in flight while this column is computed */
  unsigned res[kMaxMod], nxt[kMaxMod];
  auto load = [&](unsigned (&dst)[kMaxMod], int j) {
    const size_t off = (size_t)j * M + i0;
#pragma unroll
    for (int q = 0; q < kMaxMod; ++q) {
      if (4 == V) dst[q] = (q < cs.nmod) ? *reinterpret_cast<const unsigned*>(R + (size_t)q * plane + off) : 0u;
      else dst[q] = (q < cs.nmod) ? R[(size_t)q * plane + off] : 0u;
    }
  };
  if (blockIdx.y < N) load(res, blockIdx.y);
  for (int j = blockIdx.y; j < N; j += gridDim.y) {
    if (j + gridDim.y < N) load(nxt, j + gridDim.y);
    const int ib = eb[j];
    double* const cp = C + i0 + (long long)j * ldc;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      /* sum_i r_i w_i column by column: word k of the product sums to < 20 * 2^8 * 2^32 < 2^45 in
         64 bits, so no carry moves until the columns are combined (modulo 2^128) at the end */
      unsigned long long acc[4] = {0ull, 0ull, 0ull, 0ull};
#pragma unroll
      for (int q = 0; q < kMaxMod; ++q) {
        if (q < cs.nmod) {
          const unsigned r = __byte_perm(res[q], 0u, 0x4440u + v);
#pragma unroll
          for (int w = 0; w < 4; ++w) acc[w] += (unsigned long long)r * cs.w[q][w];
        }
      }
      uint32_t S[4];
      unsigned long long t = acc[0];
      S[0] = (uint32_t)t;
      t = acc[1] + (t >> 32);
      S[1] = (uint32_t)t;
      t = acc[2] + (t >> 32);
      S[2] = (uint32_t)t;
      t = acc[3] + (t >> 32);
      S[3] = (uint32_t)t;
      if (i0 + v < M) {
        const double val = (0 != ia[v] && 0 != ib) ? crt_value(S, cs, ia[v] + ib - 2150 + 2 * (53 - cs.mb)) : 0.0;
        cp[v] = (0.0 == beta) ? alpha * val : fma(alpha, val, beta * cp[v]);
      }
    }
#pragma unroll
    for (int q = 0; q < kMaxMod; ++q) res[q] = nxt[q];
  }
}

/* ------------------------------------------------------------------------------------ host */

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

/* 3-D map over residue planes d[q][R][Kp] (u8), box 128 (k) x rows x 1, 128-byte swizzle. */
int make_plane_map(CUtensorMap* map, const void* base, int Kp, int R, int nq, int box_rows) {
  const PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
  if (nullptr == fn) return (int)cudaErrorNotSupported;
  const cuuint64_t dims[3] = {(cuuint64_t)Kp, (cuuint64_t)R, (cuuint64_t)nq};
  const cuuint64_t strides[2] = {(cuuint64_t)Kp, (cuuint64_t)Kp * (cuuint64_t)R};
  const cuuint32_t box[3] = {(cuuint32_t)kBK, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (CUDA_SUCCESS == r) ? 0 : (int)cudaErrorInvalidValue;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

unsigned gcd_host(unsigned a, unsigned b) {
  while (0 != b) {
    const unsigned t = a % b;
    a = b;
    b = t;
  }
  return a;
}

/* inverse of a modulo m (gcd(a, m) == 1), extended Euclid */
unsigned inv_mod(unsigned a, unsigned m) {
  long long t = 0, nt = 1, r = m, nr = a % m;
  while (0 != nr) {
    const long long q = r / nr, tt = t - q * nt, rr = r - q * nr;
    t = nt;
    nt = tt;
    r = nr;
    nr = rr;
  }
  return (unsigned)((t % (long long)m + (long long)m) % (long long)m);
}

/* log2 of the product of the first n moduli */
double log2_product(int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += log2((double)kModuli[i]);
  return s;
}

/* Constants of the CRT with the first nmod moduli for inner dimension K. Returns the mantissa bits
   the inputs keep (0 if nmod cannot hold even one bit). */
int make_consts(int nmod, int K, Oz2Consts* cs) {
  memset(cs, 0, sizeof(*cs));
  cs->nmod = nmod;
  for (int i = 0; i < nmod; ++i) {
    for (int j = 0; j < i; ++j) {
      if (1u != gcd_host(kModuli[i], kModuli[j])) return 0;
    }
  }
  /* P as a double-double: exact from a 128-bit integer up to 16 factors <= 2^8, from a long double
     beyond */
  unsigned __int128 P = 1;
  long double Pld = 1.0L;
  for (int i = 0; i < nmod; ++i) {
    Pld *= (long double)kModuli[i];
    if (i < 16) P *= kModuli[i];
  }
  if (nmod <= 16) {
    cs->phi = (double)P;
    const unsigned __int128 hi = (unsigned __int128)cs->phi;
    cs->plo = (P >= hi) ? (double)(P - hi) : -(double)(hi - P);
  }
  else {
    cs->phi = (double)Pld;
    cs->plo = (double)(Pld - (long double)cs->phi);
  }
  for (int i = 0; i < nmod; ++i) {
    const unsigned m = kModuli[i];
    cs->mod[i] = m;
    cs->magic[i] = (unsigned)((1ull << 39) / m + 1ull);
    cs->c18[i] = (unsigned)((1ull << 18) % m);
    cs->c36[i] = (unsigned)((1ull << 36) % m);
    cs->cneg[i] = (unsigned)((m - (1ull << 54) % m) % m);
  }
  for (int i = 0; i < nmod; ++i) {
    const unsigned m = kModuli[i];
    unsigned pm = 1; /* (P / m_i) mod m_i */
    for (int j = 0; j < nmod; ++j) {
      if (j != i) pm = (pm * (kModuli[j] % m)) % m;
    }
    unsigned long long rem = inv_mod(pm, m); /* y_i < m_i: floor(2^128 y_i / m_i) by long division */
    for (int k = 3; k >= 0; --k) {
      const unsigned long long num = rem << 32;
      cs->w[i][k] = (unsigned)(num / m);
      rem = num % m;
    }
  }
  int lgk = 0;
  while ((1ll << lgk) < (long long)K) ++lgk;
  const int mb = (int)floor((log2_product(nmod) - 1.0 - lgk - 1.0) / 2.0);
  cs->mb = (mb > 53) ? 53 : mb;
  return (cs->mb > 0) ? cs->mb : 0;
}

/* Fewest moduli that keep all 53 bits for inner dimension K. */
int default_nmod(int K) {
  int lgk = 0;
  while ((1ll << lgk) < (long long)K) ++lgk;
  for (int n = 1; n <= kMaxMod; ++n) {
    if (log2_product(n) - 1.0 >= 2.0 * 53 + lgk + 1.0) return n;
  }
  return kMaxMod;
}

int residue_operand(const double* x, long long ld, bool rows_contiguous, int R, int K, int Kp, const Oz2Consts& cs, int* emax,
  unsigned char* planes, cudaStream_t s) {
  if (rows_contiguous) {
    const int kchunk = 256;
    xs_oz2_rowexp_rc<<<dim3((R + 255) / 256, (K + kchunk - 1) / kchunk), 256, 0, s>>>(x, ld, R, K, kchunk, emax);
    xs_oz2_res_rc<<<dim3((R + kRcRows - 1) / kRcRows, (Kp + kRcK - 1) / kRcK), 256, 0, s>>>(x, ld, R, K, Kp, emax, cs, planes);
  }
  else {
    xs_oz2_rowexp_kc<<<(R + 7) / 8, 256, 0, s>>>(x, ld, R, K, emax);
    const long long n = (long long)R * (Kp / 16);
    if (0 == ((uintptr_t)x & 15) && 0 == (ld & 1)) {
      xs_oz2_res_kc<true><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, ld, R, K, Kp, emax, cs, planes);
    }
    else {
      xs_oz2_res_kc<false><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, ld, R, K, Kp, emax, cs, planes);
    }
  }
  return (int)cudaGetLastError();
}

}  // namespace

extern "C" {

int xs_ozaki2_default_moduli(int K) { return default_nmod(K > 0 ? K : 1); }

size_t xs_ozaki2_gemm_scratch_bytes(int M, int N, int K, int nmod) {
  if (nmod <= 0) nmod = default_nmod(K > 0 ? K : 1);
  const size_t Kp = align_up((size_t)(K > 0 ? K : 1), 16);
  return align_up((size_t)nmod * M * Kp, 1024) + align_up((size_t)nmod * N * Kp, 1024) + align_up((size_t)nmod * M * N, 1024) +
         align_up(sizeof(int) * M, 256) + align_up(sizeof(int) * N, 256) + 256;
}

int xs_ozaki2_gemm(char transa, char transb, int M, int N, int K, double alpha, const double* a, int lda, const double* b,
  int ldb, double beta, double* c, int ldc, int nmod, void* scratch, size_t scratch_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const bool ta = ('T' == transa || 't' == transa || 'C' == transa || 'c' == transa);
  const bool tb = ('T' == transb || 't' == transb || 'C' == transb || 'c' == transb);
  if (M < 0 || N < 0 || K < 0 || nmod < 0 || nmod > kMaxMod || ldc < (M > 1 ? M : 1)) return (int)cudaErrorInvalidValue;
  if (0 == M || 0 == N) return 0;
  if (0 == K || 0.0 == alpha) {
    if (1.0 == beta) return 0;
    const long long n = (long long)M * N;
    xs_oz2_scale_c<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(c, ldc, M, N, beta);
    return (int)cudaGetLastError();
  }
  if (lda < (ta ? K : M) || ldb < (tb ? N : K)) return (int)cudaErrorInvalidValue;
  if (0 == nmod) nmod = default_nmod(K);
  Oz2Consts cs;
  if (0 == make_consts(nmod, K, &cs)) return (int)cudaErrorInvalidValue; /* too few moduli for this K */
  if (nullptr == scratch || scratch_bytes < xs_ozaki2_gemm_scratch_bytes(M, N, K, nmod)) return (int)cudaErrorInvalidValue;
  const int Kp = (int)align_up((size_t)K, 16);
  char* p = (char*)scratch;
  unsigned char* const rA = (unsigned char*)p;
  p += align_up((size_t)nmod * M * Kp, 1024);
  unsigned char* const rB = (unsigned char*)p;
  p += align_up((size_t)nmod * N * Kp, 1024);
  unsigned char* const rC = (unsigned char*)p;
  p += align_up((size_t)nmod * M * N, 1024);
  int* const ea = (int*)p;
  p += align_up(sizeof(int) * M, 256);
  int* const eb = (int*)p;
  p += align_up(sizeof(int) * N, 256);
  unsigned* const abort = (unsigned*)p;
  int r = (int)cudaMemsetAsync(ea, 0, (size_t)(p - (char*)ea) + 256, s);
  if (0 != r) return r;
  void* prof = xs_profile_begin(stream);
  if (0 != (r = residue_operand(a, lda, !ta, M, K, Kp, cs, ea, rA, s))) return r;
  if (0 != (r = residue_operand(b, ldb, tb, N, K, Kp, cs, eb, rB, s))) return r;
  xs_profile_end(prof, "ozaki2_residues", 0.0, 8.0 * ((double)M * K + (double)K * N), stream);
  CUtensorMap mapA, mapB;
  if (0 != (r = make_plane_map(&mapA, rA, Kp, M, nmod, kBM))) return r;
  if (0 != (r = make_plane_map(&mapB, rB, Kp, N, nmod, kBN))) return r;
  Oz2GemmArgs args;
  memset(&args, 0, sizeof(args));
  args.M = M;
  args.N = N;
  args.nmod = nmod;
  for (int i = 0; i < nmod; ++i) {
    args.mod[i] = cs.mod[i];
    args.magic[i] = cs.magic[i];
  }
  args.R = rC;
  args.abort = abort;
  args.dev_err = xs_device_error_ptr();
  args.wait_limit = xs_wait_limit();
  if (nullptr == args.dev_err) return (int)cudaErrorInvalidValue;
  const size_t smem = gemm_smem_bytes();
  if (0 != (r = xs_func_smem((const void*)xs_ozaki2_gemm_kernel, smem))) return r;
  const int nkb = (K + kBK - 1) / kBK;
  const long long nunits = (long long)((N + kBN - 1) / kBN) * ((M + kBM - 1) / kBM) * nmod;
  const dim3 grid((unsigned)(nunits < xs_sm_count() ? nunits : xs_sm_count()));
  for (int kb0 = 0; kb0 < nkb; kb0 += kKChunkBlocks) {
    args.kb0 = kb0;
    args.kb1 = (kb0 + kKChunkBlocks < nkb) ? kb0 + kKChunkBlocks : nkb;
    args.first = (0 == kb0) ? 1 : 0;
    prof = xs_profile_begin(stream);
    xs_ozaki2_gemm_kernel<<<grid, kThreads, smem, s>>>(mapA, mapB, args);
    if (0 != (r = (int)cudaGetLastError())) return r;
    const double kc = (double)(args.kb1 - args.kb0) * kBK;
    xs_profile_end(prof, "ozaki2_gemm", 2.0 * M * N * (kc < K ? kc : K), 0.0, stream);
  }
  prof = xs_profile_begin(stream);
  const long long n = (long long)M * N;
  const int V = (0 == M % 4) ? 4 : 1;
  /* about four waves of resident blocks; each thread walks its columns */
  const int rgx = (M + 256 * V - 1) / (256 * V), rgy = max(1, min(N, min(65535, 12 * xs_sm_count() / rgx)));
  const dim3 rgrid((unsigned)rgx, (unsigned)rgy);
  if (4 == V) xs_oz2_reconstruct<4><<<rgrid, 256, 0, s>>>(rC, M, N, ea, eb, cs, alpha, beta, c, ldc);
  else xs_oz2_reconstruct<1><<<rgrid, 256, 0, s>>>(rC, M, N, ea, eb, cs, alpha, beta, c, ldc);
  r = (int)cudaGetLastError();
  xs_profile_end(prof, "ozaki2_reconstruct", 0.0, (double)nmod * n + 16.0 * n, stream);
  return r;
}

}  // extern "C"
