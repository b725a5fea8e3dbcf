/*
 * Ozaki scheme-1 form of the stack path: C[c] += A[a] * B[b] over a stack of FP64 blocks of one
 * shape (m, n, k <= 64), with the block products on the int8 tensor cores (tcgen05).
 *
 * 1. Pool slicing (once per call): every block of the A pool (m x k, column-major) is split per row,
 *    every block of the B pool (k x n, row-major as libsmm_acc_transpose leaves it) per column, into
 *    s signed 7-bit digits under the row's / column's own power-of-two scale (the digit rule of
 *    ozaki_common.cl:789-834 and the per-row/per-column exponents of ozaki1_int8.cl:428-589, applied
 *    to each block). Digits are stored MMA-ready: per block and slice a K-major tile of
 *    rows8 x KP bytes (rows rounded up to 8 for A, 16 for B; KP = k rounded up to 32) made of core
 *    matrices of 8 rows x 16 bytes; exponents per block row / column.
 * 2. The stack is grouped by c (the plain path's grouping sort) and cut into chunks of L entries,
 *    one CTA per chunk (10 warps, 1 CTA per SM).
 * 3. Per entry, warp 0 copies the entry's A and B digit tiles into a shared-memory stage with bulk
 *    copies. The B slices sit between zero slices, so the K-major operand starting at slice
 *    index d0 - sa spans B slices d0-sa .. d0-sa+W-1: one tcgen05.mma (M=64, N=W*n16, K=32) of A
 *    slice sa against it puts pair (sa, d-sa) of every diagonal d in [d0, d0+W) into column block
 *    d-d0 of the accumulator. Summed over sa, column block j holds the exact int32 sum of all pairs
 *    of diagonal d0+j (|sum| <= 8 * 127^2 * 64 < 2^23). Windows of W diagonals cover 0..cutoff;
 *    each (entry, window) owns one buffer of a tensor-memory ring, so the tensor cores run ahead of
 *    the epilogue.
 * 4. Warps 2-9 (epilogue): per (entry, window) they read the accumulator (M=64 layout: rows 16q..16q+15
 *    in lanes 32q..32q+15 of quarter q), combine the window's diagonals in FP64 with weights
 *    2^(-7j), scale by 2^(ea_i - 1029) * 2^(eb_j - 1029) * 2^(-7 d0) (exact powers of two) and add to
 *    the FP64 sum of the current segment (run of equal c) held in registers. A segment is written
 *    once: straight into C when it lies inside the chunk, else as a piece that the combine kernel
 *    adds up in chunk order (deterministic), as the plain path does.
 * Every mbarrier wait is bounded (per-call abort word, library device error word bit 2).
 */
#include "internal.h"
#include "ozaki_digits.cuh"
#include "tc_ptx.cuh"
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

namespace {
using namespace xs_tc;
using namespace xs_oz;

constexpr int kMaxSlices = 8;
constexpr int kMaxWin = 16;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr int kTmemCols = 512;
constexpr unsigned kErrOzakiTimeout = 4u;
constexpr unsigned kErrBadOffset = 8u;
constexpr int kMaxChunk = 1024; /* entries per chunk (their keys are staged in shared memory) */
constexpr int kXSlots = 8;      /* exponent ring: row exponents of A and column exponents of B per entry */

/* ------------------------------------------------------------------------- pool slicing */

/* Block blk, row r (< R) of K entries: element (r, kk) at x[blk*bs + r*rs + kk*cs]. Writes the digit
   tiles d[blk][s][rows8][KP] (core matrices of 8 rows x 16 bytes: row group g at g*KP*8, k-chunk c
   at c*128, row r%8 at 16*(r%8)) and the row exponents e[blk][64]. 64 threads per block. */
__global__ void __launch_bounds__(128) xs_ozs_slice_pool(const double* __restrict__ x, int nblk, long long bs, int rs, int cs,
  int R, int K, int KP, int rows8, int ns, unsigned char* __restrict__ d, int* __restrict__ e) {
  const int blk = blockIdx.x * 2 + (threadIdx.x >> 6), r = threadIdx.x & 63;
  if (blk >= nblk) return;
  const double* const xb = x + (long long)blk * bs;
  int emax = 0;
  if (r < R) {
    for (int kk = 0; kk < K; ++kk) emax = max(emax, biased_exp(xb[(long long)r * rs + (long long)kk * cs]));
  }
  e[(long long)blk * 64 + r] = emax;
  if (r >= rows8) return;
  unsigned char* const out = d + (long long)blk * ns * rows8 * KP + (r >> 3) * (KP * 8) + (r & 7) * 16;
  for (int k0 = 0; k0 < KP; k0 += 16) {
    unsigned long long al[16];
    unsigned sg[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int kk = k0 + j;
      const double v = (r < R && kk < K) ? xb[(long long)r * rs + (long long)kk * cs] : 0.0;
      int be;
      unsigned long long mt;
      ieee_split(v, sg[j], be, mt);
      const int sh = emax - be;
      al[j] = (0 != mt && sh <= 52) ? (mt >> sh) : 0ull;
    }
    for (int s = 0; s < ns; ++s) {
      uint32_t w[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t v = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) v |= ((uint32_t)(slice_digit(al[q * 4 + b], sg[q * 4 + b], s) & 0xFF)) << (8 * b);
        w[q] = v;
      }
      *reinterpret_cast<uint4*>(out + (long long)s * rows8 * KP + (k0 >> 4) * 128) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

/* ------------------------------------------------------------------------- stack kernel */

struct OzWin {
  int d0, W;        /* diagonals d0 .. d0+W-1 */
  int sa_lo, sa_hi; /* A slices with at least one pair in the window */
};

struct OzSmmArgs {
  const unsigned* keys;           /* grouped c offsets (1-based) */
  const unsigned long long* vals; /* grouped (a | b << 32) offsets (1-based) */
  int S, L, nchunks;
  int m, n, k, KP, rowsA, rowsB, ns, Wmax;
  int na, nb;
  long long mk, kn;
  const unsigned char* dA;
  const unsigned char* dB;
  const int* eA;
  const int* eB;
  unsigned sliceA, sliceB;     /* bytes of one slice tile: rowsA*KP, rowsB*KP */
  unsigned stage_bytes, offB;  /* stage: A tiles at 0, B area (zero pads around the slices) at offB */
  int nstages;
  int nwin;
  OzWin win[kMaxWin];
  int nbuf, bufcols; /* tensor-memory ring */
  double* C;
  double* pieces; /* [chunk][2][m*n] */
  unsigned* abort;
  unsigned* dev_err;
  long long wait_limit; /* bound of every pipeline wait, clock cycles */
};

__device__ __forceinline__ double pow2_or_zero(int e) { /* 2^(e - 1029) for a biased exponent e, 0 for e < 7 */
  return (e >= 7) ? __longlong_as_double((long long)(e - 6) << 52) : 0.0;
}

__device__ __forceinline__ void entry_blocks(const OzSmmArgs& g, unsigned long long v, int& ab, int& bb, bool& ok) {
  const long long ao = (long long)(unsigned)v - 1, bo = (long long)(unsigned)(v >> 32) - 1;
  ab = (int)(ao / g.mk);
  bb = (int)(bo / g.kn);
  ok = (ao >= 0 && bo >= 0 && ao == (long long)ab * g.mk && bo == (long long)bb * g.kn && ab < g.na && bb < g.nb);
  if (!ok) {
    ab = 0;
    bb = 0;
  }
}

__global__ void __launch_bounds__(kThreads, 1) xs_ozs_smm_kernel(const __grid_constant__ OzSmmArgs g) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* const smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  int* const xring = (int*)(smem + (size_t)g.nstages * g.stage_bytes); /* [kXSlots][128]: eA row, eB col */
  unsigned* const s_keys = (unsigned*)(xring + kXSlots * 128);           /* [kMaxChunk] */
  int2* const s_blk = (int2*)(s_keys + kMaxChunk);                       /* [kMaxChunk]: A, B block index */
  uint64_t* const bars = (uint64_t*)(s_blk + kMaxChunk);
  uint64_t* const full = bars;                 /* [nstages] */
  uint64_t* const empty = bars + 8;            /* [nstages] */
  uint64_t* const accf = bars + 16;            /* [nbuf] */
  uint64_t* const acce = bars + 32;            /* [nbuf] */
  uint64_t* const xfull = bars + 48;           /* [kXSlots] */
  uint64_t* const xempty = bars + 56;          /* [kXSlots] */
  uint32_t* const tmem_slot = (uint32_t*)(bars + 64);
  unsigned* const abort = g.abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ch = blockIdx.x;
  const int p0 = ch * g.L, p1 = min(g.S, p0 + g.L);
  if (0 == threadIdx.x) {
    for (int i = 0; i < g.nstages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < g.nbuf; ++i) {
      mbar_init(&accf[i], 1);
      mbar_init(&acce[i], 32 * kEpiWarps);
    }
    for (int i = 0; i < kXSlots; ++i) {
      mbar_init(&xfull[i], 1);
      mbar_init(&xempty[i], 32 * kEpiWarps);
    }
    fence_barrier_init();
  }
  if (1 == warp) {
    tmem_alloc(tmem_slot, kTmemCols);
    tmem_relinquish();
  }
  { /* zero every stage once: the pads around the B slices and the A tail stay zero (bulk copies
       only write the slice tiles) */
    uint4* const z = (uint4*)smem;
    const int nz = (int)((size_t)g.nstages * g.stage_bytes / 16);
    for (int i = threadIdx.x; i < nz; i += blockDim.x) z[i] = make_uint4(0, 0, 0, 0);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    for (int i = threadIdx.x; i < p1 - p0; i += blockDim.x) {
      s_keys[i] = g.keys[p0 + i];
      int ab, bb;
      bool ok;
      entry_blocks(g, g.vals[p0 + i], ab, bb, ok);
      if (!ok) atomicOr(g.dev_err, kErrBadOffset);
      s_blk[i] = make_int2(ab, bb);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int nent = p1 - p0;

  if (0 == warp) { /* producer */
    if (0 == lane) {
      const unsigned padB = (unsigned)(g.Wmax - 1) * g.sliceB;
      for (int e = 0; e < nent; ++e) {
        const int stage = e % g.nstages;
        const uint32_t ph = (uint32_t)(e / g.nstages) & 1u;
        const int ab = s_blk[e].x, bb = s_blk[e].y;
        { /* exponents of the entry's A rows and B columns into the exponent ring */
          const int xs = e % kXSlots;
          if (!mbar_wait(&xempty[xs], ((uint32_t)(e / kXSlots) & 1u) ^ 1u, abort, 1u, g.wait_limit)) break;
          mbar_arrive_expect_tx(&xfull[xs], 512);
          bulk_load(xring + xs * 128, g.eA + (size_t)ab * 64, 256, &xfull[xs]);
          bulk_load(xring + xs * 128 + 64, g.eB + (size_t)bb * 64, 256, &xfull[xs]);
        }
        if (!mbar_wait(&empty[stage], ph ^ 1u, abort, 1u, g.wait_limit)) break;
        unsigned char* const st = smem + (size_t)stage * g.stage_bytes;
        const unsigned bytesA = (unsigned)g.ns * g.sliceA, bytesB = (unsigned)g.ns * g.sliceB;
        mbar_arrive_expect_tx(&full[stage], bytesA + bytesB);
        bulk_load(st, g.dA + (size_t)ab * bytesA, bytesA, &full[stage]);
        bulk_load(st + g.offB + padB, g.dB + (size_t)bb * bytesB, bytesB, &full[stage]);
      }
    }
  }
  else if (1 == warp) { /* MMA issuer */
    if (0 == lane) {
      const uint32_t sbo = (uint32_t)g.KP * 8u;
      int grp = 0;
      bool ok = true;
      for (int e = 0; e < nent && ok; ++e) {
        const int stage = e % g.nstages;
        const uint32_t ph = (uint32_t)(e / g.nstages) & 1u;
        if (!(ok = mbar_wait(&full[stage], ph, abort, 2u, g.wait_limit))) break;
        tc_fence_after();
        const uint32_t sA = smem_u32(smem + (size_t)stage * g.stage_bytes);
        const uint32_t sB = sA + g.offB;
        for (int w = 0; w < g.nwin && ok; ++w, ++grp) {
          const int buf = grp % g.nbuf, use = grp / g.nbuf;
          if (!(ok = mbar_wait(&acce[buf], ((uint32_t)use & 1u) ^ 1u, abort, 2u, g.wait_limit))) break;
          tc_fence_after();
          const OzWin& wn = g.win[w];
          const uint32_t idesc = idesc_i8(64, wn.W * g.rowsB);
          const uint32_t d = tmem + (uint32_t)(buf * g.bufcols);
          uint32_t acc = 0;
          for (int sa = wn.sa_lo; sa <= wn.sa_hi; ++sa) {
            const uint32_t a0 = sA + (uint32_t)sa * g.sliceA;
            const uint32_t b0 = sB + (uint32_t)(g.Wmax - 1 + wn.d0 - sa) * g.sliceB;
            for (int ks = 0; ks < g.KP / 32; ++ks) {
              mma_i8(d, desc_k_noswz(a0 + ks * 256, 128, sbo), desc_k_noswz(b0 + ks * 256, 128, sbo), idesc, acc);
              acc = 1;
            }
          }
          mma_commit(&accf[buf]);
        }
        if (ok) mma_commit(&empty[stage]);
      }
    }
  }
  else { /* epilogue: warps 2..9 */
    const int ew = warp - 2, q = warp & 3, half = ew >> 2;
    const int row = 16 * q + lane;
    const bool rok = (lane < 16) && (row < g.m);
    const int nch = g.rowsB / 8, chalf = (nch + 1) / 2;
    const int c_lo = half * chalf, c_hi = min(nch, c_lo + chalf);
    const int mn = g.m * g.n;
    const bool headcross = (p0 > 0) && (g.keys[p0 - 1] == s_keys[0]);
    const bool tailcross = (p1 < g.S) && (s_keys[nent - 1] == g.keys[p1]);
    double acc[4][8];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[c][j] = 0.0;
    int seg_start = p0;
    unsigned seg_key = (nent > 0) ? s_keys[0] : 0u;
    int grp = 0;
    bool ok = true;
    /* writes the finished segment [seg_start, seg_end) of key seg_key */
    auto flush = [&](int seg_end) {
      if (rok) {
        double* dst;
        long long stride;
        int slot = -1;
        if (seg_start == p0 && headcross) slot = 0;
        else if (seg_end == p1 && tailcross) slot = 1;
        if (slot >= 0) dst = g.pieces + ((size_t)ch * 2 + slot) * mn;
        else dst = g.C + ((size_t)seg_key - 1);
        stride = g.m;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int cc = c_lo + c;
          if (cc < c_hi) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int col = cc * 8 + j;
              if (col < g.n) {
                double* const p = dst + row + (long long)col * stride;
                *p = (slot >= 0) ? acc[c][j] : (*p + acc[c][j]);
              }
            }
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[c][j] = 0.0;
    };
    for (int e = 0; e < nent && ok; ++e) {
      const unsigned key = s_keys[e];
      if (key != seg_key) {
        flush(p0 + e);
        seg_start = p0 + e;
        seg_key = key;
      }
      const int xs = e % kXSlots;
      if (!(ok = mbar_wait(&xfull[xs], (uint32_t)(e / kXSlots) & 1u, abort, 8u, g.wait_limit))) break;
      const int* const xe = xring + xs * 128;
      const double rs = rok ? pow2_or_zero(xe[row]) : 0.0;
      for (int w = 0; w < g.nwin; ++w, ++grp) {
        const int buf = grp % g.nbuf, use = grp / g.nbuf;
        if (!(ok = mbar_wait(&accf[buf], (uint32_t)use & 1u, abort, 8u, g.wait_limit))) break;
        tc_fence_after();
        const OzWin& wn = g.win[w];
        const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(buf * g.bufcols);
        const double rw = rs * __longlong_as_double((long long)(1023 - 7 * wn.d0) << 52);
        /* two passes of up to two 8-column chunks: the window's diagonals are combined in FP64 with
           weights 2^(-7 jb), then scaled and added to the segment sum */
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
          double t[2][8];
#pragma unroll
          for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int j = 0; j < 8; ++j) t[c][j] = 0.0;
          double wd = 1.0;
          for (int jb = 0; jb < wn.W; ++jb, wd *= 0.0078125) {
            uint32_t v[2][8];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              const int cc = c_lo + 2 * pass + c;
              if (cc < c_hi) tmem_ld8(tbase + (uint32_t)(jb * g.rowsB + cc * 8), v[c]);
            }
            tmem_ld_wait();
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              if (c_lo + 2 * pass + c < c_hi) {
#pragma unroll
                for (int j = 0; j < 8; ++j) { /* exact int32 -> double: 2^52 + 2^31 + v, minus the offset */
                  const double dv = __hiloint2double(0x43300000, (int)(v[c][j] ^ 0x80000000u)) - 4503601774854144.0;
                  t[c][j] = fma(dv, wd, t[c][j]);
                }
              }
            }
          }
          if (rok) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              const int cc = c_lo + 2 * pass + c;
              if (cc < c_hi) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                  const int col = cc * 8 + j;
                  const double cs = (col < g.n) ? pow2_or_zero(xe[64 + col]) : 0.0;
                  acc[2 * pass + c][j] = fma(t[c][j], rw * cs, acc[2 * pass + c][j]);
                }
              }
            }
          }
        }
        tc_fence_before();
        mbar_arrive(&acce[buf]);
      }
      if (ok) mbar_arrive(&xempty[xs]);
    }
    if (ok && nent > 0) flush(p1);
  }
  if (0 != *(volatile unsigned*)abort) {
    for (int i = 0; i < 200; ++i) __nanosleep(1000);
  }
  tc_fence_before();
  __syncthreads();
  if (1 == warp) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
  if (0 == threadIdx.x && 0 != *(volatile unsigned*)abort) atomicOr(g.dev_err, kErrOzakiTimeout);
}

/* Sums the pieces of every chunk-crossing segment in chunk order and adds them to C once. Chunk ch
   owns the segment that leaves it through its tail when that segment starts in ch. */
__global__ void xs_ozs_combine(const unsigned* __restrict__ keys, int S, int L, int m, int n, const double* __restrict__ pieces,
  double* __restrict__ C, const unsigned* __restrict__ abort) {
  const int ch = blockIdx.x;
  if (0 != *(volatile const unsigned*)abort) return;
  const int p0 = ch * L, p1 = min(S, p0 + L);
  if (p1 >= S) return;
  const unsigned key = keys[p1 - 1];
  if (keys[p1] != key) return;                                            /* no tail crossing */
  if (keys[p0] == key && p0 > 0 && keys[p0 - 1] == key) return;          /* started in an earlier chunk */
  const int mn = m * n;
  for (int idx = threadIdx.x; idx < mn; idx += blockDim.x) {
    double s = pieces[((size_t)ch * 2 + 1) * mn + idx];
    for (int c2 = ch + 1; (size_t)c2 * L < (size_t)S && keys[(size_t)c2 * L] == key; ++c2) s += pieces[((size_t)c2 * 2 + 0) * mn + idx];
    C[(size_t)key - 1 + idx] += s;
  }
}

/* ---------------------------------------------------------------------------- planning */

struct OzPlan {
  int KP, rowsA, rowsB, ns, cutoff, Wmax, nwin, nbuf, bufcols, nstages;
  OzWin win[kMaxWin];
  unsigned sliceA, sliceB, stage_bytes, offB;
  size_t smem;
  size_t poolA, poolB; /* digit bytes per block */
};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int plan_oz(int m, int n, int k, int ns, int cutoff, OzPlan* p) {
  if (m < 1 || n < 1 || k < 1 || m > 64 || n > 64 || k > 64 || ns < 1 || ns > kMaxSlices) return -1;
  p->ns = ns;
  p->cutoff = (cutoff < 0 || cutoff > 2 * (ns - 1)) ? 2 * (ns - 1) : cutoff;
  p->KP = (k <= 32) ? 32 : 64;
  p->rowsA = (m + 7) / 8 * 8;
  p->rowsB = (n + 15) / 16 * 16; /* MMA N must be a multiple of 16 */
  p->Wmax = 256 / p->rowsB;
  if (p->Wmax > p->cutoff + 1) p->Wmax = p->cutoff + 1;
  p->nwin = 0;
  for (int d0 = 0; d0 <= p->cutoff; d0 += p->Wmax) {
    if (p->nwin == kMaxWin) return -1;
    OzWin& w = p->win[p->nwin++];
    w.d0 = d0;
    w.W = (d0 + p->Wmax - 1 <= p->cutoff) ? p->Wmax : p->cutoff + 1 - d0;
    w.sa_lo = (d0 - (ns - 1) > 0) ? d0 - (ns - 1) : 0;
    w.sa_hi = (d0 + w.W - 1 < ns - 1) ? d0 + w.W - 1 : ns - 1;
  }
  p->bufcols = p->Wmax * p->rowsB;
  p->nbuf = kTmemCols / p->bufcols;
  if (p->nbuf > 16) p->nbuf = 16;
  p->sliceA = (unsigned)(p->rowsA * p->KP);
  p->sliceB = (unsigned)(p->rowsB * p->KP);
  /* A: s tiles, the last one read as 64 rows; B: (Wmax-1) zero tiles, s tiles, (Wmax-1) zero tiles */
  const size_t bytesA = (size_t)(ns - 1) * p->sliceA + (size_t)64 * p->KP;
  p->offB = (unsigned)align_up(bytesA, 128);
  const size_t bytesB = (size_t)(ns + 2 * (p->Wmax - 1)) * p->sliceB;
  p->stage_bytes = (unsigned)align_up(p->offB + bytesB, 128);
  const size_t budget = 188 * 1024;
  p->nstages = (int)(budget / p->stage_bytes);
  if (p->nstages > 8) p->nstages = 8;
  if (p->nstages < 1) return -1;
  p->smem = 128 + (size_t)p->nstages * p->stage_bytes + sizeof(int) * kXSlots * 128 + sizeof(unsigned) * kMaxChunk +
            sizeof(int2) * kMaxChunk + 80 * sizeof(uint64_t);
  if (p->smem < 120 * 1024) p->smem = 120 * 1024; /* one CTA per SM: it owns all 512 TMEM columns */
  p->poolA = (size_t)ns * p->sliceA;
  p->poolB = (size_t)ns * p->sliceB;
  return 0;
}

struct OzLayout {
  size_t dA, dB, eA, eB, keys0, keys1, keys2, vals0, vals1, vals2, pieces, sort, abort, total;
  int L, nchunks;
};

void layout_oz(const OzPlan& p, int S, int m, int n, int na, int nb, OzLayout* l) {
  const int part = S < xs_stack_group_max() ? S : xs_stack_group_max();
  const int target = 4 * xs_sm_count();
  l->L = (part + target - 1) / target;
  if (l->L < 8) l->L = 8;
  if (l->L > kMaxChunk) l->L = kMaxChunk;
  l->nchunks = (part + l->L - 1) / l->L;
  size_t o = 0;
  l->dA = o;
  o = align_up(o + p.poolA * (size_t)na, 256);
  l->dB = o;
  o = align_up(o + p.poolB * (size_t)nb, 256);
  l->eA = o;
  o = align_up(o + sizeof(int) * 64 * (size_t)na, 256);
  l->eB = o;
  o = align_up(o + sizeof(int) * 64 * (size_t)nb, 256);
  const size_t ks = align_up(sizeof(unsigned) * (size_t)part, 256), vs = align_up(sizeof(unsigned long long) * (size_t)part, 256);
  l->keys0 = o;
  o += ks;
  l->keys1 = o;
  o += ks;
  l->keys2 = o;
  o += ks;
  l->vals0 = o;
  o += vs;
  l->vals1 = o;
  o += vs;
  l->vals2 = o;
  o += vs;
  l->pieces = o;
  o = align_up(o + sizeof(double) * 2 * (size_t)l->nchunks * m * n, 256);
  l->sort = o;
  o = align_up(o + xs_stack_sort_scratch_bytes(part), 256);
  l->abort = o;
  o += 256;
  l->total = o;
}

}  // namespace

extern "C" {

size_t xs_smm_ozaki_scratch_bytes(int S, int m, int n, int k, int na, int nb, int nslices) {
  OzPlan p;
  OzLayout l;
  if (0 >= S || 0 != plan_oz(m, n, k, nslices, -1, &p)) return 0;
  layout_oz(p, S, m, n, na, nb, &l);
  return l.total;
}

int xs_launch_smm_ozaki(const int* dev_stack, int S, int m, int n, int k, const double* a, int na, const double* b, int nb,
  double* c, int nslices, int cutoff, void* scratch, size_t scratch_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  OzPlan p;
  OzLayout l;
  if (0 >= S) return 0;
  if (na < 1 || nb < 1 || 0 != plan_oz(m, n, k, nslices, cutoff, &p)) return (int)cudaErrorInvalidValue;
  layout_oz(p, S, m, n, na, nb, &l);
  if (nullptr == scratch || scratch_bytes < l.total) return (int)cudaErrorInvalidValue;
  char* const base = (char*)scratch;
  unsigned char* const dA = (unsigned char*)(base + l.dA);
  unsigned char* const dB = (unsigned char*)(base + l.dB);
  int* const eA = (int*)(base + l.eA);
  int* const eB = (int*)(base + l.eB);
  unsigned* const abort = (unsigned*)(base + l.abort);
  int r = (int)cudaMemsetAsync(abort, 0, 256, s);
  if (0 != r) return r;
  void* prof = xs_profile_begin(stream);
  /* A block: element (i, kk) at i + kk*m; B block (k x n row-major): column j element kk at kk*n + j */
  xs_ozs_slice_pool<<<(na + 1) / 2, 128, 0, s>>>(a, na, (long long)m * k, 1, m, m, k, p.KP, p.rowsA, p.ns, dA, eA);
  xs_ozs_slice_pool<<<(nb + 1) / 2, 128, 0, s>>>(b, nb, (long long)k * n, 1, n, n, k, p.KP, p.rowsB, p.ns, dB, eB);
  if (0 != (r = (int)cudaGetLastError())) return r;
  xs_profile_end(prof, "ozaki_slice_pools", 0.0, 8.0 * ((double)na * m * k + (double)nb * k * n), stream);
  if (0 != (r = xs_func_smem((const void*)xs_ozs_smm_kernel, p.smem))) return r;
  const int part_max = xs_stack_group_max();
  for (int off = 0; off < S; off += part_max) {
    const int P = (S - off < part_max) ? S - off : part_max;
    unsigned* const k0 = (unsigned*)(base + l.keys0);
    unsigned* const k1 = (unsigned*)(base + l.keys1);
    unsigned* const kout = (unsigned*)(base + l.keys2);
    unsigned long long* const v0 = (unsigned long long*)(base + l.vals0);
    unsigned long long* const v1 = (unsigned long long*)(base + l.vals1);
    unsigned long long* const vout = (unsigned long long*)(base + l.vals2);
    prof = xs_profile_begin(stream);
    if (0 != (r = xs_stack_group(dev_stack + 3 * (size_t)off, P, k0, v0, k1, v1, kout, vout, nullptr, base + l.sort, stream))) return r;
    xs_profile_end(prof, "sort", 0.0, 48.0 * P, stream);
    OzSmmArgs g;
    memset(&g, 0, sizeof(g));
    g.keys = kout;
    g.vals = vout;
    g.S = P;
    g.L = l.L;
    g.nchunks = (P + l.L - 1) / l.L;
    g.m = m;
    g.n = n;
    g.k = k;
    g.KP = p.KP;
    g.rowsA = p.rowsA;
    g.rowsB = p.rowsB;
    g.ns = p.ns;
    g.Wmax = p.Wmax;
    g.na = na;
    g.nb = nb;
    g.mk = (long long)m * k;
    g.kn = (long long)k * n;
    g.dA = dA;
    g.dB = dB;
    g.eA = eA;
    g.eB = eB;
    g.sliceA = p.sliceA;
    g.sliceB = p.sliceB;
    g.stage_bytes = p.stage_bytes;
    g.offB = p.offB;
    g.nstages = p.nstages;
    g.nwin = p.nwin;
    for (int w = 0; w < p.nwin; ++w) g.win[w] = p.win[w];
    g.nbuf = p.nbuf;
    g.bufcols = p.bufcols;
    g.C = c;
    g.pieces = (double*)(base + l.pieces);
    g.abort = abort;
    g.dev_err = xs_device_error_ptr();
    g.wait_limit = xs_wait_limit();
    if (nullptr == g.dev_err) return (int)cudaErrorInvalidValue;
    prof = xs_profile_begin(stream);
    xs_ozs_smm_kernel<<<g.nchunks, kThreads, p.smem, s>>>(g);
    if (0 != (r = (int)cudaGetLastError())) return r;
    xs_profile_end(prof, "ozaki_smm", 2.0 * m * n * (double)k * P, 0.0, stream);
    prof = xs_profile_begin(stream);
    xs_ozs_combine<<<g.nchunks, 256, 0, s>>>(kout, P, l.L, m, n, g.pieces, c, abort);
    if (0 != (r = (int)cudaGetLastError())) return r;
    xs_profile_end(prof, "ozaki_combine", 0.0, 0.0, stream);
  }
  return 0;
}

}  // extern "C"
