/*
 * Stable device grouping of stacks by their c offset (the first step of the plain FP64 stack path),
 * for one stack or a batch of stacks in one cooperative kernel.
 *
 * The c offsets of one stack are few distinct values spread over a large range (C blocks of one
 * shape in a pool), so they are mapped to dense bucket ids id = (c - cmin) / g, where g is the gcd
 * of all differences c - c0 (for a pool of equal blocks g is the block size). Phase 0 of the kernel
 * splits each stack into keys (c) and payload (a | b << 32) and gathers cmin, cmax and g per stack;
 * then an LSD counting sort over the ids runs with digits of at most 2048 buckets: a single pass when
 * a stack touches at most 2048 distinct C blocks (the common case), two or three otherwise. Per pass:
 * per-tile digit histograms -> digit bases -> stable scatter (rank within a tile from warp match
 * masks and per-warp counts). Every tile belongs to one stack and every stack is sorted inside its
 * own range of the output; equal keys keep stack order, so the permutation is bit-exact and
 * reproducible. Grid-wide barriers spin on a global counter with an iteration limit; on timeout the
 * kernel sets the call's error flag (the stack kernel then writes nothing) and the library's device
 * error word, and returns instead of hanging.
 */
#include "internal.h"
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

/* Library-wide device error word: bit 0 = a grid barrier of the grouping sort timed out, bit 2 = a
   pipeline wait of the Ozaki GEMM timed out. */
__device__ unsigned xs_device_error_word;

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kRadixBits = 11;
constexpr int kRadix = 1 << kRadixBits;
constexpr unsigned kSpinLimit = 1u << 24;
constexpr int kMaxGroupTiles = 256; /* the owner-warp digit scan covers at most 256 tiles per stack */

/* Control block of one call, zero-initialised by one memset at the start of the call:
   ctl[0] holds the grid barrier, the error flag and the stack kernels' work-queue counters (its four
   statistics words serve as the queues of the tile-class groups 1..4, `queue` is spare);
   ctl[1 + g] the statistics of stack g of the call (the minimum kept as its complement, atomicMax). */
struct SortCtl {
  unsigned ncmin, cmax, gcd, pad0;
  unsigned bar_count, bar_gen, err, queue;
};

/* gcd by Stein's binary method (shifts and subtractions, no integer division). */
__device__ __forceinline__ unsigned gcd_u(unsigned a, unsigned b) {
  if (0 == a) return b;
  if (0 == b) return a;
  const int sh = __ffs(a | b) - 1;
  a >>= __ffs(a) - 1;
  do {
    b >>= __ffs(b) - 1;
    if (a > b) {
      const unsigned t = a;
      a = b;
      b = t;
    }
    b -= a;
  } while (0 != b);
  return a << sh;
}

/* Extend a running gcd by x; skips the gcd when g already divides x (the common case). */
__device__ __forceinline__ unsigned gcd_acc(unsigned g, unsigned x) {
  return (0 != g && 0 == x % g) ? g : gcd_u(g, x);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

/* Bounded grid barrier (all CTAs are co-resident: cooperative launch). The arrival counter only
   grows (it is zeroed with the control block at the start of the call): barrier number `epoch`
   (0, 1, ...) of the launch is passed once it reaches (epoch + 1) * gridDim.x, so the last CTA to
   arrive resets nothing and the others leave on their next poll. Returns false on timeout or if
   another CTA reported an error. */
__device__ __forceinline__ bool grid_sync(SortCtl* ctl, int& epoch) {
  __shared__ int s_ok;
  __syncthreads();
  if (0 == threadIdx.x) {
    const unsigned target = (unsigned)(epoch + 1) * gridDim.x;
    __threadfence();
    unsigned seen = atomicAdd(&ctl->bar_count, 1u) + 1u;
    int ok = 1;
    unsigned spins = 0;
    while (seen < target) {
      if (++spins > kSpinLimit) {
        atomicExch(&ctl->err, 1u);
        atomicOr(&xs_device_error_word, 1u);
        ok = 0;
        break;
      }
      seen = *(volatile unsigned*)&ctl->bar_count;
    }
    __threadfence();
    if (0 != *(volatile unsigned*)&ctl->err) ok = 0;
    s_ok = ok;
  }
  ++epoch;
  __syncthreads();
  return 0 != s_ok;
}

/* Bucket id (c - cmin) / g. g divides every c - cmin, so the quotient is an exact integer below
   2^32 and the double product x * (1/g) is within far less than 0.5 of it: rounding recovers it. */
__device__ __forceinline__ unsigned bucket_of(unsigned c, unsigned cmin, double inv_g) {
  return __double2uint_rn((double)(c - cmin) * inv_g);
}

/* floor(x / d) for d >= 1 from m = floor(2^32 / d) (m = 0 for d = 1): the high product is q or
   q - 1, one correction step fixes it. */
__device__ __forceinline__ unsigned div_floor(unsigned x, unsigned d, unsigned m) {
  if (1u >= d) return x;
  unsigned q = __umulhi(x, m);
  if ((unsigned long long)(q + 1u) * d <= x) ++q;
  return q;
}

/* For each of this lane's E digits, the lanes of the warp holding the same digit (what
   __match_any_sync returns), from one ballot per digit bit: bits 0..nbits-1 and bit kRadixBits, which
   only the no-entry digit kRadix sets. Ballots cost far less than match instructions. */
template <int E>
__device__ __forceinline__ void match_digits(const int (&dig)[E], int nbits, unsigned (&peers)[E]) {
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const bool x = 0 != ((dig[r] >> kRadixBits) & 1);
    const unsigned v = __ballot_sync(0xffffffffu, x);
    peers[r] = x ? v : ~v;
  }
  for (int b = 0; b < nbits; ++b) {
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const bool x = 0 != ((dig[r] >> b) & 1);
      const unsigned v = __ballot_sync(0xffffffffu, x);
      peers[r] &= x ? v : ~v;
    }
  }
}

/* Block-wide exclusive scan of R values held PER per thread (thread i owns [i*PER, (i+1)*PER));
   returns the block total. */
template <int PER>
__device__ __forceinline__ int block_exscan(int (&v)[PER], int* s_wsum) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int sum = 0;
#pragma unroll
  for (int j = 0; j < PER; ++j) sum += v[j];
  int x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (31 == lane) s_wsum[warp] = x;
  __syncthreads();
  int run = x - sum, total = 0;
  for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) {
    if (w2 < warp) run += s_wsum[w2];
    total += s_wsum[w2];
  }
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int t = v[j];
    v[j] = run;
    run += t;
  }
  __syncthreads();
  return total;
}

/* Grouping sort of a batch of stacks. Tile t belongs to stack s with tile_begin[s] <= t <
   tile_begin[s] + ntiles[s]; it covers entries [lt*T, min(S_s, (lt+1)*T)) of that stack (lt =
   t - tile_begin[s], T = kSortThreads*E). Warp w owns the contiguous sub-range [w0, w0 + 32E) of
   the tile and lane l holds entries w0 + l + 32r (r < E) in registers for the whole kernel, so every
   phase costs about one round trip to memory. Output positions of stack s are off[s] + local.
   Histogram table: rows hist[t][0..kRadix) per tile, then one totals row per stack. */
template <int E>
__global__ void __launch_bounds__(kSortThreads) xs_stack_group_kernel(xs_sort_batch_t desc, unsigned* __restrict__ k0,
  unsigned long long* __restrict__ v0, unsigned* __restrict__ k1, unsigned long long* __restrict__ v1,
  unsigned* __restrict__ kout, unsigned long long* __restrict__ vout, int* __restrict__ seglist,
  int* __restrict__ hist, SortCtl* ctl, unsigned long long* __restrict__ stamps) {
  __shared__ __align__(16) unsigned short s_wc[kSortWarps][kRadix]; /* (b) reuses it as int[kRadix] */
  __shared__ int s_base[kRadix]; /* digit histogram in (a), digit write positions in (b)/(c) */
  __shared__ int s_wsum[kSortWarps];
  __shared__ unsigned s_red[3][kSortWarps];
  __shared__ int s_radix[XS_MAX_BATCH]; /* digit range R of every stack of the batch */
  /* per-stack tables of the descriptor, read with compile-time indices only (an index computed at
     run time would make every thread copy the whole descriptor to local memory) */
  __shared__ int s_tb[XS_MAX_BATCH], s_nt[XS_MAX_BATCH], s_gidx[XS_MAX_BATCH];
  __shared__ unsigned s_blk[XS_MAX_BATCH];
#pragma unroll
  for (int s2 = 0; s2 < XS_MAX_BATCH; ++s2) {
    if (s2 == (int)threadIdx.x) {
      s_tb[s2] = desc.tile_begin[s2];
      s_nt[s2] = desc.ntiles[s2];
      s_gidx[s2] = desc.gidx[s2];
      s_blk[s2] = desc.blk[s2];
    }
  }
  __syncthreads();
  const int tile = blockIdx.x, ntiles_all = gridDim.x, nstacks = desc.nstacks;
  int si = 0;
  while (si + 1 < nstacks && s_tb[si + 1] <= tile) ++si;
  const int* stack = nullptr;
  int fmt = 0, S = 0, off = 0;
#pragma unroll
  for (int s2 = 0; s2 < XS_MAX_BATCH; ++s2) {
    if (s2 == si) {
      stack = desc.stack[s2];
      fmt = desc.format[s2];
      S = desc.S[s2];
      off = desc.off[s2];
    }
  }
  /* parameter format: 1-based (a, b, c) triples, or 6-int records with 0-based (a, b, c) at +3 */
  const int pstride = (0 != fmt) ? 6 : 3, pbase = (0 != fmt) ? 3 : 0;
  const int pone = (0 != fmt) ? 1 : 0;
  const int tb = s_tb[si], G = s_nt[si];
  const int lt = tile - tb, T = kSortThreads * E;
  const int t0 = min(S, lt * T), t1 = min(S, t0 + T);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int w0 = min(t1, t0 + warp * 32 * E), w1 = min(t1, w0 + 32 * E);
  unsigned key[E];
  unsigned long long val[E];
  SortCtl* const sctl = ctl + 1 + s_gidx[si];
  const unsigned blk = s_blk[si];
  int epoch = 0; /* grid barriers passed */
  /* optional phase timestamps (stamps != nullptr): [tile][8] */
#define XS_STAMP(slot) \
  do { \
    if (nullptr != stamps && 0 == threadIdx.x) stamps[tile * 8 + (slot)] = global_ns(); \
  } while (0)
  XS_STAMP(0);
  /* the stack kernel launched after this one may be scheduled now (programmatic dependent launch);
     it waits for this kernel's completion before it reads the grouped stack */
  asm volatile("griddepcontrol.launch_dependents;" :::);

  /* phase 0: load + bucket statistics of this stack */
  {
    const unsigned c0 = (unsigned)(stack[pbase + 2] + pone);
    unsigned lo = 0xFFFFFFFFu, hi = 0u, gg = 0u;
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int i = w0 + lane + 32 * r;
      key[r] = 0u;
      val[r] = 0ull;
      if (i < w1) {
        const int* const e = stack + (size_t)pstride * i + pbase;
        const int a = e[0] + pone, b = e[1] + pone;
        key[r] = (unsigned)(e[2] + pone);
        val[r] = (unsigned long long)(unsigned)a | ((unsigned long long)(unsigned)b << 32);
      }
    }
#pragma unroll
    for (int r = 0; r < E; ++r) {
      if (w0 + lane + 32 * r < w1) {
        const unsigned c = key[r];
        lo = min(lo, c);
        hi = max(hi, c);
        if (0 == blk) gg = gcd_acc(gg, (c > c0) ? c - c0 : c0 - c);
      }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if (0 == blk) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) gg = gcd_acc(gg, __shfl_xor_sync(0xffffffffu, gg, o));
    }
    if (0 == lane) {
      s_red[0][warp] = lo;
      s_red[1][warp] = hi;
      s_red[2][warp] = gg;
    }
    __syncthreads();
    if (0 == threadIdx.x) {
      for (int w = 1; w < kSortWarps; ++w) {
        lo = min(lo, s_red[0][w]);
        hi = max(hi, s_red[1][w]);
        if (0 == blk) gg = gcd_acc(gg, s_red[2][w]);
      }
      if (lo != 0xFFFFFFFFu) {
        atomicMax(&sctl->ncmin, ~lo);
        atomicMax(&sctl->cmax, hi);
      }
      if (0 != gg) {
        unsigned old = *(volatile unsigned*)&sctl->gcd;
        while (0 == old || gcd_u(old, gg) != old) { /* no CAS once the global gcd divides this one */
          const unsigned assumed = old;
          old = atomicCAS(&sctl->gcd, assumed, gcd_u(assumed, gg));
          if (old == assumed) break;
        }
      }
      if (0 == tile && nullptr != seglist) seglist[0] = 0;
    }
    for (int i = tile * kSortThreads + (int)threadIdx.x; i < desc.nzero; i += ntiles_all * kSortThreads) desc.zero[i] = 0;
    XS_STAMP(1);
    if (!grid_sync(ctl, epoch)) return;
    XS_STAMP(2);
  }
  /* per-stack digit plan; every CTA derives the same pass count and table mode for the whole batch
     (the number of grid barriers must be uniform) */
  int passes_all = 0, rows_max = 0;
  for (int s2 = 0; s2 < nstacks; ++s2) {
    const SortCtl* const c2 = ctl + 1 + s_gidx[s2];
    const unsigned g2 = (0 != s_blk[s2]) ? s_blk[s2] : *(volatile const unsigned*)&c2->gcd;
    const unsigned nb2 = (0 == g2) ? 1u : (*(volatile const unsigned*)&c2->cmax - ~*(volatile const unsigned*)&c2->ncmin) / g2 + 1u;
    int b2 = 0;
    while (b2 < 32 && (nb2 - 1u) >> b2) ++b2;
    const int p2 = (b2 + kRadixBits - 1) / kRadixBits;
    if (0 == threadIdx.x) s_radix[s2] = (0 == p2) ? 1 : 1 << ((b2 + p2 - 1) / p2);
    if (p2 > passes_all) passes_all = p2;
    if (s_nt[s2] > rows_max) rows_max = s_nt[s2];
  }
  const unsigned cmin = ~*(volatile unsigned*)&sctl->ncmin, g = (0 != blk) ? blk : *(volatile unsigned*)&sctl->gcd;
  const unsigned cmax = *(volatile unsigned*)&sctl->cmax;
  const unsigned nb = (0 == g) ? 1u : (cmax - cmin) / g + 1u;
  const double inv_g = (0 == g) ? 0.0 : 1.0 / (double)g;
  const unsigned gm = (1u < g) ? (unsigned)((1ull << 32) / g) : 0u;

  int bits = 0;
  while (bits < 32 && (nb - 1u) >> bits) ++bits;
  const int passes = (bits + kRadixBits - 1) / kRadixBits;
  if (0 == passes) { /* a single C block: already grouped, keep stack order */
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int i = w0 + lane + 32 * r;
      if (i < w1) {
        kout[off + i] = key[r];
        vout[off + i] = val[r];
      }
    }
  }
  const int rb = (0 == passes) ? 0 : (bits + passes - 1) / passes, R = 1 << rb;
  const bool direct = rows_max <= 64; /* up to 64 tiles per stack: each CTA scans its stack's rows itself */
  for (int pass = 0; pass < passes_all; ++pass) {
    const bool active = pass < passes;
    const int shift = pass * rb;
    const bool last = (pass + 1 == passes);
    unsigned* const kdst = last ? kout : ((0 == (pass & 1)) ? k1 : k0);
    unsigned long long* const vdst = last ? vout : ((0 == (pass & 1)) ? v1 : v0);
    int dig[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
      /* bucket id: an exact quotient (g = gcd divides c - cmin) or floor((c - cmin) / blk) */
      const unsigned id = (0 != blk) ? div_floor(key[r] - cmin, g, gm) : bucket_of(key[r], cmin, inv_g);
      dig[r] = (active && w0 + lane + 32 * r < w1) ? (int)((id >> shift) & (R - 1)) : kRadix;
    }
    /* (a) tile histogram, row hist[tile][0..R); per-warp counters zeroed for (c) */
    for (int d = threadIdx.x; d < R; d += blockDim.x) s_base[d] = 0;
    for (int j = threadIdx.x; j < kSortWarps * (kRadix / 8); j += blockDim.x) { /* 8 counters per 16-byte store */
      if (8 * (j & (kRadix / 8 - 1)) < R) reinterpret_cast<uint4*>(&s_wc[0][0])[j] = make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) { /* shared-memory atomics: lanes of a hot C block serialise on one counter,
                                     which costs less than matching the digits first */
      if (kRadix != dig[r]) atomicAdd(&s_base[dig[r]], 1);
    }
    __syncthreads();
    if (direct) { /* 16-bit counts (a tile holds at most kTileLarge entries): half the bytes to read in (b) */
      unsigned short* const row16 = reinterpret_cast<unsigned short*>(hist) + (size_t)tile * kRadix;
      for (int d = threadIdx.x; d < R; d += blockDim.x) row16[d] = (unsigned short)s_base[d];
    }
    else {
      for (int d = threadIdx.x; d < R; d += blockDim.x) hist[(size_t)tile * kRadix + d] = s_base[d];
    }
    if (0 == pass) XS_STAMP(3);
    if (!grid_sync(ctl, epoch)) return;
    if (0 == pass) XS_STAMP(4);
    /* (b) digit bases of this tile inside its stack. Data written by other CTAs in this kernel is
       read with __ldcg (from L2), never through a possibly stale L1 line. Thread i owns digits
       [i*per, (i+1)*per). */
    constexpr int PER = kRadix / kSortThreads;
    const int per = (R + kSortThreads - 1) / kSortThreads;
    int tot[PER], pre[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) tot[j] = pre[j] = 0;
    if (direct) { /* coalesced: thread t sums the digit pairs (2q, 2q + 1), q = t, t + 256, ..., of the stack's
                     16-bit rows, eight rows per round of loads; the sums move through shared memory to
                     the contiguous ownership the scan below uses */
      static_assert(0 == PER % 2, "digit pairs");
      int ctot[PER], cpre[PER];
#pragma unroll
      for (int j = 0; j < PER; ++j) ctot[j] = cpre[j] = 0;
      if (active) {
        const unsigned short* const rows16 = reinterpret_cast<const unsigned short*>(hist) + (size_t)tb * kRadix;
        for (int tt = 0; tt < G; tt += 8) {
          unsigned h[8][PER / 2];
#pragma unroll
          for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int j2 = 0; j2 < PER / 2; ++j2) {
              const int q = j2 * kSortThreads + (int)threadIdx.x;
              h[u][j2] = (tt + u < G && 2 * q < R)
                           ? __ldcg(reinterpret_cast<const unsigned*>(rows16 + (size_t)(tt + u) * kRadix) + q) : 0u;
            }
#pragma unroll
          for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int j2 = 0; j2 < PER / 2; ++j2) {
              const int lo = (int)(h[u][j2] & 0xFFFFu), hi = (2 * (j2 * kSortThreads + (int)threadIdx.x) + 1 < R) ? (int)(h[u][j2] >> 16) : 0;
              ctot[2 * j2] += lo;
              ctot[2 * j2 + 1] += hi;
              if (tt + u < lt) {
                cpre[2 * j2] += lo;
                cpre[2 * j2 + 1] += hi;
              }
            }
        }
      }
      int* const s_pre = reinterpret_cast<int*>(&s_wc[0][0]); /* the per-warp counters are zero and unused until (c) */
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        const int d = 2 * ((j / 2) * kSortThreads + (int)threadIdx.x) + (j & 1);
        if (d < R) {
          s_base[d] = ctot[j];
          s_pre[d] = cpre[j];
        }
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        const int d = threadIdx.x * per + j;
        const bool ok = j < per && d < R;
        tot[j] = ok ? s_base[d] : 0;
        pre[j] = ok ? s_pre[d] : 0;
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < PER; ++j) { /* the counters are zero again for (c) */
        const int d = j * kSortThreads + (int)threadIdx.x;
        if (d < R) s_pre[d] = 0;
      }
    }
    else { /* owner warps: one per (stack, digit), scanning that stack's tile column in place (32
              tiles per step, all loads issued first); totals to the stack's totals row */
      for (int q = tile * kSortWarps + warp; q < nstacks * kRadix; q += ntiles_all * kSortWarps) {
        const int s2 = q / kRadix, d = q - s2 * kRadix;
        if (d >= s_radix[s2]) continue; /* digits the stack does not use */
        const int tb2 = s_tb[s2], G2 = s_nt[s2];
        constexpr int kSteps = kMaxGroupTiles / 32;
        int h[kSteps];
#pragma unroll
        for (int st = 0; st < kSteps; ++st) {
          const int tt = 32 * st + lane;
          h[st] = (tt < G2) ? __ldcg(hist + (size_t)(tb2 + tt) * kRadix + d) : 0;
        }
        int run = 0;
#pragma unroll
        for (int st = 0; st < kSteps; ++st) {
          int x = h[st];
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
          }
          const int tt = 32 * st + lane;
          if (tt < G2) hist[(size_t)(tb2 + tt) * kRadix + d] = run + x - h[st];
          run += __shfl_sync(0xffffffffu, x, 31);
        }
        if (0 == lane) hist[(size_t)(ntiles_all + s2) * kRadix + d] = run;
      }
      if (!grid_sync(ctl, epoch)) return;
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        const int d = threadIdx.x * per + j;
        const bool ok = active && j < per && d < R;
        tot[j] = ok ? __ldcg(hist + (size_t)(ntiles_all + si) * kRadix + d) : 0;
        pre[j] = ok ? __ldcg(hist + (size_t)tile * kRadix + d) : 0;
      }
    }
    block_exscan<PER>(tot, s_wsum);
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int d = threadIdx.x * per + j;
      if (j < per && d < R) s_base[d] = off + tot[j] + pre[j];
    }
    if (0 == pass) XS_STAMP(5);
    /* (c) stable scatter: per-warp counts -> per-warp offsets -> ordered placement */
    unsigned peers[E];
    match_digits<E>(dig, rb, peers);
#pragma unroll
    for (int r = 0; r < E; ++r) {
      if (kRadix != dig[r] && 0 == __popc(peers[r] & ((1u << lane) - 1u))) {
        s_wc[warp][dig[r]] += (unsigned short)__popc(peers[r]);
      }
      __syncwarp();
    }
    __syncthreads();
    for (int dd = threadIdx.x; dd < R; dd += blockDim.x) {
      int run = 0;
#pragma unroll
      for (int w2 = 0; w2 < kSortWarps; ++w2) {
        const int c = s_wc[w2][dd];
        s_wc[w2][dd] = (unsigned short)run;
        run += c;
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int rank = __popc(peers[r] & ((1u << lane) - 1u));
      if (kRadix != dig[r]) {
        const int pos = s_base[dig[r]] + s_wc[warp][dig[r]] + rank;
        kdst[pos] = key[r];
        vdst[pos] = val[r];
      }
      __syncwarp();
      if (kRadix != dig[r] && 0 == rank) s_wc[warp][dig[r]] += (unsigned short)__popc(peers[r]);
      __syncwarp();
    }
    if (0 == pass) XS_STAMP(6);
    if (pass + 1 < passes_all) {
      if (!grid_sync(ctl, epoch)) return;
      if (pass + 1 < passes) {
#pragma unroll
        for (int r = 0; r < E; ++r) {
          const int i = w0 + lane + 32 * r;
          if (i < w1) {
            key[r] = __ldcg(kdst + off + i);
            val[r] = __ldcg(vdst + off + i);
          }
        }
      }
    }
  }
  XS_STAMP(7);
#undef XS_STAMP
}

/* ------------------------------------------------------------------ one-cluster grouping (small stacks) */

/* One-cluster grouping: 16 CTAs of 512 threads, 4 entries per thread (32768 entries at most). */
constexpr int kClusterMax = 16;
constexpr int kClThreads = 512;
constexpr int kClWarps = kClThreads / 32;
constexpr int kClE = 4;
constexpr int kClusterEntries = kClusterMax * kClThreads * kClE;
/* dynamic shared memory: per-warp digit counters [kClWarps][kRadix] (u16), then the digit totals of
   every CTA of the cluster [kClusterMax][kRadix] (int) */
constexpr size_t kClSmem = sizeof(unsigned short) * kClWarps * kRadix + sizeof(int) * kClusterMax * kRadix;


/* Grouping of one stack of at most kClusterEntries entries by ONE thread-block cluster: a stable LSD
   counting sort over the bucket ids of the c offsets, with the same per-digit order as
   xs_stack_group_kernel (stack order within a digit, hence the same output). Bucket ids: with blk > 0
   (the C block size: the blocks of one stack do not overlap, so distinct blocks lie at least blk
   apart) id = (c - cmin) / blk, which needs only the minimum and maximum of the offsets; with
   blk == 0 the gcd of the offset differences divides them exactly. The CTAs exchange data only by
   pushing it into each other's shared memory, each push followed by a cluster barrier: their
   statistics, then per pass their digit totals, from which every CTA derives its write positions
   locally (totals over the cluster, exclusive scan over the digits, counts of the CTAs before it).
   Within a CTA, each warp counts its entries per digit from match masks (one count per distinct
   digit and entry round) and places them in stack order. No grid barrier, global table, atomic or
   memset (CTA 0 clears the error word and the segment list); cluster barriers are hardware
   barriers of co-scheduled CTAs and cannot hang. */
template <int E>
__global__ void __launch_bounds__(kClThreads) xs_stack_group_cluster_kernel(const int* __restrict__ stack, int S, int format,
  unsigned blk, unsigned* __restrict__ k0, unsigned long long* __restrict__ v0, unsigned* __restrict__ k1,
  unsigned long long* __restrict__ v1, unsigned* __restrict__ kout, unsigned long long* __restrict__ vout,
  int* __restrict__ seglist, int* __restrict__ zero, int nzero, SortCtl* ctl, int heavy, unsigned blk_magic,
  unsigned long long* __restrict__ stamps) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  unsigned short (*const s_wc)[kRadix] = reinterpret_cast<unsigned short (*)[kRadix]>(s_dyn);
  int (*const s_all)[kRadix] = reinterpret_cast<int (*)[kRadix]>(s_dyn + sizeof(unsigned short) * kClWarps * kRadix);
  __shared__ __align__(16) int s_base[kRadix]; /* digit write positions of this CTA */
  __shared__ int s_wsum[kClWarps];
  __shared__ unsigned s_red[3][kClWarps];
  __shared__ unsigned s_stat[kClusterMax][3]; /* cmin, cmax, gcd of every CTA, pushed by each */
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank(), ncta = (int)cluster.num_blocks();
  /* optional phase timestamps (stamps != nullptr): [rank][8] */
#define XS_CSTAMP(slot) \
  do { \
    if (nullptr != stamps && 0 == threadIdx.x) stamps[rank * 8 + (slot)] = global_ns(); \
  } while (0)
  XS_CSTAMP(0);
  asm volatile("griddepcontrol.launch_dependents;" :::);
  /* every CTA of the cluster must be running before another one writes into its shared memory: arrive
     now, wait before the first push (the stack loads overlap the barrier) */
  asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
  const int pstride = (0 != format) ? 6 : 3, pbase = (0 != format) ? 3 : 0, pone = (0 != format) ? 1 : 0;
  const int T = kClThreads * E;
  const int t0 = min(S, rank * T), t1 = min(S, t0 + T);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int w0 = min(t1, t0 + warp * 32 * E), w1 = min(t1, w0 + 32 * E);
  unsigned key[E];
  unsigned long long val[E];
  if (0 == rank && 0 == threadIdx.x) {
    ctl->err = 0u;
    if (nullptr != seglist) seglist[0] = 0;
  }
  for (int i = rank * kClThreads + (int)threadIdx.x; i < nzero; i += ncta * kClThreads) zero[i] = 0;
  { /* load + statistics */
    unsigned lo = 0xFFFFFFFFu, hi = 0u, gg = 0u;
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int i = w0 + lane + 32 * r;
      key[r] = 0u;
      val[r] = 0ull;
      if (i < w1) {
        const int* const e = stack + (size_t)pstride * i + pbase;
        const int a = e[0] + pone, b = e[1] + pone;
        key[r] = (unsigned)(e[2] + pone);
        val[r] = (unsigned long long)(unsigned)a | ((unsigned long long)(unsigned)b << 32);
        lo = min(lo, key[r]);
        hi = max(hi, key[r]);
      }
    }
    if (0 == blk) { /* gcd of the differences to the stack's first offset */
      const unsigned c0 = (unsigned)(stack[pbase + 2] + pone);
#pragma unroll
      for (int r = 0; r < E; ++r) {
        if (w0 + lane + 32 * r < w1) gg = gcd_acc(gg, (key[r] > c0) ? key[r] - c0 : c0 - key[r]);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) gg = gcd_acc(gg, __shfl_xor_sync(0xffffffffu, gg, o));
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if (0 == lane) {
      s_red[0][warp] = lo;
      s_red[1][warp] = hi;
      s_red[2][warp] = gg;
    }
    __syncthreads();
    if (0 == warp) {
      lo = (lane < kClWarps) ? s_red[0][lane] : 0xFFFFFFFFu;
      hi = (lane < kClWarps) ? s_red[1][lane] : 0u;
      lo = __reduce_min_sync(0xffffffffu, lo);
      hi = __reduce_max_sync(0xffffffffu, hi);
      if (0 == lane && 0 == blk) {
        for (int w = 1; w < kClWarps; ++w) gg = gcd_acc(gg, s_red[2][w]);
      }
      gg = __shfl_sync(0xffffffffu, gg, 0);
    }
    XS_CSTAMP(1);
    asm volatile("barrier.cluster.wait.aligned;" ::: "memory");
    if (0 == warp && lane < ncta) { /* push this CTA's statistics to every CTA of the cluster */
      unsigned* const st = cluster.map_shared_rank(&s_stat[rank][0], lane);
      st[0] = lo;
      st[1] = hi;
      st[2] = gg;
    }
  }
  cluster.sync();
  XS_CSTAMP(2);
  /* every warp combines the cluster's statistics, lane q taking CTA q's (ncta <= 16 < 32) */
  const unsigned cmin = __reduce_min_sync(0xffffffffu, (lane < ncta) ? s_stat[lane][0] : 0xFFFFFFFFu);
  const unsigned cmax = __reduce_max_sync(0xffffffffu, (lane < ncta) ? s_stat[lane][1] : 0u);
  unsigned g = blk, gm = blk_magic; /* blk > 0: floor(2^32 / blk) from the host */
  if (0 == blk) {
    g = (lane < ncta) ? s_stat[lane][2] : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) g = gcd_acc(g, __shfl_xor_sync(0xffffffffu, g, o));
    gm = (1u < g) ? (unsigned)((1ull << 32) / g) : 0u;
  }
  const unsigned nb = (0 == g) ? 1u : div_floor(cmax - cmin, g, gm) + 1u;
  int bits = 0;
  while (bits < 32 && (nb - 1u) >> bits) ++bits;
  const int passes = (bits + kRadixBits - 1) / kRadixBits;
  if (0 == passes) { /* a single C block: already grouped, keep stack order */
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int i = w0 + lane + 32 * r;
      if (i < w1) {
        kout[i] = key[r];
        vout[i] = val[r];
      }
    }
  }
  const int rb = (0 == passes) ? 0 : (bits + passes - 1) / passes, R = 1 << rb;
  unsigned id[E];
#pragma unroll
  for (int r = 0; r < E; ++r) id[r] = (0 == g) ? 0u : div_floor(key[r] - cmin, g, gm);
  for (int pass = 0; pass < passes; ++pass) {
    const int shift = pass * rb;
    const bool last = (pass + 1 == passes);
    unsigned* const kdst = last ? kout : ((0 == (pass & 1)) ? k1 : k0);
    unsigned long long* const vdst = last ? vout : ((0 == (pass & 1)) ? v1 : v0);
    int dig[E];
#pragma unroll
    for (int r = 0; r < E; ++r) dig[r] = (w0 + lane + 32 * r < w1) ? (int)((id[r] >> shift) & (R - 1)) : kRadix;
    /* (a) per-warp digit counts: the leader of each group of equal digits adds the group's size */
    if (R >= 8) {
      for (int j = threadIdx.x; j < kClWarps * (R / 8); j += kClThreads) { /* 8 counters per 16-byte store */
        reinterpret_cast<uint4*>(&s_wc[j / (R / 8)][0])[j % (R / 8)] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    else if ((int)threadIdx.x < kClWarps * R) s_wc[threadIdx.x / R][threadIdx.x % R] = 0;
    __syncthreads();
    unsigned peers[E];
    match_digits<E>(dig, rb, peers);
#pragma unroll
    for (int r = 0; r < E; ++r) {
      if (kRadix != dig[r] && 0 == __popc(peers[r] & ((1u << lane) - 1u))) {
        s_wc[warp][dig[r]] += (unsigned short)__popc(peers[r]);
      }
      __syncwarp();
    }
    __syncthreads();
    if (0 == pass) XS_CSTAMP(3);
    /* (b) per digit: exclusive prefix over the warps in place; the CTA's totals go to every CTA.
       Thread i owns the four digits [4i, 4i + 4) here and in (c), read and written as vectors
       (counts < 2^16: a CTA holds kClThreads * E entries); digits >= R are never used. */
    static_assert(kRadix == 4 * kClThreads, "four digits per thread");
    const int d4 = 4 * (int)threadIdx.x;
    if (d4 < R) {
      unsigned run0 = 0u, run1 = 0u, run2 = 0u, run3 = 0u;
#pragma unroll
      for (int w2 = 0; w2 < kClWarps; ++w2) {
        uint2* const p = reinterpret_cast<uint2*>(&s_wc[w2][d4]);
        const uint2 c = *p;
        *p = make_uint2(run0 | (run1 << 16), run2 | (run3 << 16));
        run0 += c.x & 0xFFFFu;
        run1 += c.x >> 16;
        run2 += c.y & 0xFFFFu;
        run3 += c.y >> 16;
      }
      const int4 t4 = make_int4((int)run0, (int)run1, (int)run2, (int)run3);
      for (int q = 0; q < ncta; ++q) *cluster.map_shared_rank(reinterpret_cast<int4*>(&s_all[rank][d4]), q) = t4;
    }
    cluster.sync();
    if (0 == pass) XS_CSTAMP(4);
    /* (c) write positions: exclusive scan of the cluster totals over the digits plus the counts of
       the CTAs before this one. */
    int tot[4] = {0, 0, 0, 0}, pre[4] = {0, 0, 0, 0};
    if (d4 < R) {
      for (int q = 0; q < ncta; ++q) {
        const int4 c = *reinterpret_cast<const int4*>(&s_all[q][d4]);
        tot[0] += c.x;
        tot[1] += c.y;
        tot[2] += c.z;
        tot[3] += c.w;
        if (q < rank) {
          pre[0] += c.x;
          pre[1] += c.y;
          pre[2] += c.z;
          pre[3] += c.w;
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (d4 + j >= R) tot[j] = pre[j] = 0;
      }
    }
    if (1 == passes && 0 < heavy) { /* C blocks with >= heavy entries first, then the rest; id order within each */
      int hv[4];
      bool isheavy[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        isheavy[j] = tot[j] >= heavy;
        hv[j] = isheavy[j] ? tot[j] : 0;
        tot[j] -= hv[j];
      }
      const int nheavy = block_exscan<4>(hv, s_wsum);
      block_exscan<4>(tot, s_wsum);
#pragma unroll
      for (int j = 0; j < 4; ++j) tot[j] = isheavy[j] ? hv[j] : nheavy + tot[j];
    }
    else block_exscan<4>(tot, s_wsum);
    if (d4 < R) *reinterpret_cast<int4*>(&s_base[d4]) = make_int4(tot[0] + pre[0], tot[1] + pre[1], tot[2] + pre[2], tot[3] + pre[3]);
    __syncthreads();
    if (0 == pass) XS_CSTAMP(5);
    /* (d) stable placement in stack order: CTA base + warp offset + rank within the warp */
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int rank_w = __popc(peers[r] & ((1u << lane) - 1u));
      if (kRadix != dig[r]) {
        const int pos = s_base[dig[r]] + s_wc[warp][dig[r]] + rank_w;
        kdst[pos] = key[r];
        vdst[pos] = val[r];
      }
      __syncwarp();
      if (kRadix != dig[r] && 0 == rank_w) s_wc[warp][dig[r]] += (unsigned short)__popc(peers[r]);
      __syncwarp();
    }
    if (0 == pass) XS_CSTAMP(6);
    if (!last) { /* this pass's output is visible to the whole cluster, and s_all may be overwritten */
      cluster.sync();
#pragma unroll
      for (int r = 0; r < E; ++r) {
        const int i = w0 + lane + 32 * r;
        if (i < w1) {
          key[r] = __ldcg(kdst + i);
          val[r] = __ldcg(vdst + i);
          id[r] = (0 == g) ? 0u : div_floor(key[r] - cmin, g, gm);
        }
      }
    }
  }
  XS_CSTAMP(7);
#undef XS_CSTAMP
}

/* Entries per thread kept in registers: 8 (tiles of 2048) or 16 (tiles of 4096). */
constexpr int kTileSmall = kSortThreads * 8, kTileLarge = kSortThreads * 16;

int sort_grid_max(void) {
  static int grid[XS_MAXDEV]; /* per device, 0 until computed */
  const int dev = xs_device_slot();
  if (0 == grid[dev]) {
    int a = 0, b = 0;
    if (cudaSuccess != cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, xs_stack_group_kernel<8>, kSortThreads, 0)) a = 1;
    if (cudaSuccess != cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, xs_stack_group_kernel<16>, kSortThreads, 0)) b = 1;
    const int per_sm = a < b ? a : b;
    grid[dev] = xs_sm_count() * (per_sm < 1 ? 1 : per_sm);
  }
  return grid[dev];
}

/* Tiles of a batch: kTileSmall entries each, or kTileLarge when the small tiles do not fit on the
   device at once or one stack would need more than kMaxGroupTiles of them. Fills ntiles/tile_begin
   and returns the grid (0 if the batch is larger than one launch takes). */
int plan_tiles(xs_sort_batch_t* d, int* large) {
  const int gmax = sort_grid_max();
  for (int pass = 0; pass < 2; ++pass) {
    const int T = pass ? kTileLarge : kTileSmall;
    int total = 0, fits = 1;
    for (int s = 0; s < d->nstacks; ++s) {
      const int nt = (d->S[s] + T - 1) / T;
      d->ntiles[s] = nt < 1 ? 1 : nt;
      d->tile_begin[s] = total;
      total += d->ntiles[s];
      if (d->ntiles[s] > kMaxGroupTiles) fits = 0;
    }
    if (fits && total <= gmax) {
      *large = pass;
      return total;
    }
  }
  return 0;
}

int group_launch(const xs_sort_batch_t& desc0, unsigned* k0, unsigned long long* v0, unsigned* k1, unsigned long long* v1,
  unsigned* kout, unsigned long long* vout, int* seglist, void* sort_scratch, cudaStream_t s, unsigned long long* stamps,
  int clear_ctl) {
  xs_sort_batch_t desc = desc0;
  int large = 0;
  const int grid = plan_tiles(&desc, &large);
  if (0 == grid) return (int)cudaErrorInvalidValue; /* callers split batches above the launch limit */
  SortCtl* ctl = (SortCtl*)sort_scratch;
  int* hist = (int*)((char*)sort_scratch + xs_sort_ctl_bytes());
  if (clear_ctl) {
    int ng = 0;
    for (int i = 0; i < desc.nstacks; ++i) ng = desc.gidx[i] + 1 > ng ? desc.gidx[i] + 1 : ng;
    const cudaError_t r = cudaMemsetAsync(ctl, 0, sizeof(SortCtl) * (size_t)(1 + ng), s);
    if (cudaSuccess != r) return (int)r;
  }
  else { /* a later grouping launch of the call: its grid barriers count from zero again */
    const cudaError_t r = cudaMemsetAsync(&ctl->bar_count, 0, sizeof(unsigned), s);
    if (cudaSuccess != r) return (int)r;
  }
  void* args[] = {&desc, &k0, &v0, &k1, &v1, &kout, &vout, &seglist, &hist, &ctl, &stamps};
  return (int)cudaLaunchCooperativeKernel(
    large ? (const void*)xs_stack_group_kernel<16> : (const void*)xs_stack_group_kernel<8>, dim3(grid), dim3(kSortThreads),
    args, 0, s);
}

/* Launches the one-cluster grouping with ncta CTAs (a power of two <= kClusterMax). Returns
   cudaErrorNotSupported, launching nothing, when the device cannot run a cluster of that size. */
int cluster_group_launch(const int* stack, int S, int format, unsigned blk, unsigned* k0, unsigned long long* v0, unsigned* k1,
  unsigned long long* v1, unsigned* kout, unsigned long long* vout, int* seglist, int* zero, int nzero, SortCtl* ctl, int ncta,
  int heavy, cudaStream_t s, unsigned long long* stamps = nullptr) {
  static int ok[XS_MAXDEV][kClusterMax + 1]; /* per device and cluster size: 0 unknown, 1 supported, -1 not */
  auto kernel = xs_stack_group_cluster_kernel<kClE>;
  int* const okp = &ok[xs_device_slot()][ncta];
  const size_t smem = kClSmem;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)ncta);
  cfg.blockDim = dim3(kClThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)ncta;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (0 == *okp) {
    int nclusters = 0;
    cudaError_t r = cudaSuccess;
    /* static + dynamic shared memory exceed the default 48 KB per CTA */
    r = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (cudaSuccess == r && ncta > 8) r = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (cudaSuccess == r) r = cudaOccupancyMaxActiveClusters(&nclusters, kernel, &cfg);
    *okp = (cudaSuccess == r && 0 < nclusters) ? 1 : -1;
    if (cudaSuccess != r) (void)cudaGetLastError(); /* not sticky: clear it */
  }
  if (0 > *okp) return (int)cudaErrorNotSupported;
  const unsigned blk_magic = (1u < blk) ? (unsigned)((1ull << 32) / blk) : 0u;
  return (int)cudaLaunchKernelEx(&cfg, kernel, stack, S, format, blk, k0, v0, k1, v1, kout, vout, seglist, zero, nzero, ctl, heavy,
    blk_magic, stamps);
}

}  // namespace

extern "C" {

size_t xs_sort_ctl_bytes(void) { return (sizeof(SortCtl) * (1 + XS_MAX_CALL_STACKS) + 255) / 256 * 256; }

int xs_sort_clear_ctl(void* sort_scratch, int nstacks, void* stream) {
  return (int)cudaMemsetAsync(sort_scratch, 0, sizeof(SortCtl) * (size_t)(1 + nstacks), (cudaStream_t)stream);
}

size_t xs_stack_sort_scratch_bytes_batch(const xs_sort_batch_t* desc) {
  xs_sort_batch_t d = *desc;
  int large = 0;
  const int grid = plan_tiles(&d, &large);
  const size_t rows = (size_t)(grid > 0 ? grid : sort_grid_max()) + (size_t)XS_MAX_BATCH;
  return xs_sort_ctl_bytes() + sizeof(int) * rows * kRadix;
}

int xs_stack_group_fits(const xs_sort_batch_t* desc) {
  xs_sort_batch_t d = *desc;
  int large = 0;
  return plan_tiles(&d, &large) > 0 ? 1 : 0;
}

size_t xs_stack_sort_scratch_bytes(int S) {
  xs_sort_batch_t d;
  d.nstacks = 1;
  d.S[0] = S;
  return xs_stack_sort_scratch_bytes_batch(&d);
}

int xs_stack_group_cluster_max(void) { return kClusterEntries; }

int xs_stack_group_max(void) { return (sort_grid_max() < kMaxGroupTiles ? sort_grid_max() : kMaxGroupTiles) * kTileLarge; }

int xs_stack_group_batch(const xs_sort_batch_t* desc, unsigned* k0, unsigned long long* v0, unsigned* k1,
  unsigned long long* v1, unsigned* kout, unsigned long long* vout, int* seglist, void* sort_scratch, void* stream) {
  return group_launch(*desc, k0, v0, k1, v1, kout, vout, seglist, sort_scratch, (cudaStream_t)stream, nullptr, 0);
}

int xs_stack_group(const int* dev_stack, int S, unsigned* k0, unsigned long long* v0, unsigned* k1,
  unsigned long long* v1, unsigned* kout, unsigned long long* vout, int* seglist, void* sort_scratch, void* stream) {
  return xs_stack_group_ex(dev_stack, S, 0, 0u, k0, v0, k1, v1, kout, vout, seglist, nullptr, 0, 0, sort_scratch, stream);
}

int xs_stack_group_ex(const int* dev_stack, int S, int format, unsigned blk, unsigned* k0, unsigned long long* v0, unsigned* k1,
  unsigned long long* v1, unsigned* kout, unsigned long long* vout, int* seglist, int* zero, int nzero, int heavy,
  void* sort_scratch, void* stream) {
  if (0 < S && S <= kClusterEntries) { /* one cluster of up to 16 CTAs */
    int ncta = 1;
    while (ncta * kClThreads * kClE < S) ncta <<= 1;
    const int r = cluster_group_launch(dev_stack, S, format, blk, k0, v0, k1, v1, kout, vout, seglist, zero, nzero,
      (SortCtl*)sort_scratch, ncta, heavy, (cudaStream_t)stream);
    if (cudaErrorNotSupported != r) return r; /* else: the cooperative kernel below */
  }
  xs_sort_batch_t d;
  memset(&d, 0, sizeof(d));
  d.zero = zero;
  d.nzero = (nullptr != zero) ? nzero : 0;
  d.nstacks = 1;
  d.stack[0] = dev_stack;
  d.format[0] = format;
  d.S[0] = S;
  d.off[0] = 0;
  d.gidx[0] = 0;
  d.blk[0] = blk;
  return group_launch(d, k0, v0, k1, v1, kout, vout, seglist, sort_scratch, (cudaStream_t)stream, nullptr, 1);
}

unsigned* xs_sort_queue_counter(void* sort_scratch, int which) {
  SortCtl* const c = (SortCtl*)sort_scratch;
  unsigned* const q[4] = {&c->ncmin, &c->cmax, &c->gcd, &c->pad0};
  return q[which & 3];
}
const unsigned* xs_sort_error_flag(void* sort_scratch) { return &((SortCtl*)sort_scratch)->err; }
int xs_sort_launch_tiles(void) { return sort_grid_max() < kMaxGroupTiles ? sort_grid_max() : kMaxGroupTiles; }
int xs_sort_tile_entries(int large) { return large ? kTileLarge : kTileSmall; }

/* Device address of the error word for kernels of other translation units (one per device). */
unsigned* xs_device_error_ptr(void) {
  static unsigned* addr[64];
  int dev = 0;
  if (cudaSuccess != cudaGetDevice(&dev) || dev < 0 || dev >= 64) return NULL;
  if (NULL == addr[dev]) {
    void* p = NULL;
    if (cudaSuccess != cudaGetSymbolAddress(&p, xs_device_error_word)) return NULL;
    addr[dev] = (unsigned*)p;
  }
  return addr[dev];
}

int xs_device_error_fetch(unsigned* host_dst, void* stream) {
  unsigned* const p = xs_device_error_ptr();
  if (nullptr == p) return (int)cudaErrorInvalidSymbol;
  return (int)cudaMemcpyAsync(host_dst, p, sizeof(unsigned), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
}

int xs_device_error_read(unsigned* value) {
  return (int)cudaMemcpyFromSymbol(value, xs_device_error_word, sizeof(unsigned));
}

int xs_device_error_clear(void) {
  const unsigned zero = 0;
  return (int)cudaMemcpyToSymbol(xs_device_error_word, &zero, sizeof(zero));
}

int libxstream_b200_device_error(int reset) {
  unsigned e = 0;
  if (EXIT_SUCCESS != xs_ensure_device()) return -1;
  if (cudaSuccess != xs_device_error_read(&e)) return -1;
  if (0 != reset && 0 != e && cudaSuccess != xs_device_error_clear()) return -1;
  return (int)e;
}

/* Diagnostic variant: the grouping of one stack (C block size blk, 0: gcd statistics) by the kernel
   the library would use for it (one cluster up to 32768 entries, else the cooperative kernel), with
   per-CTA phase timestamps (ns, %globaltimer) written to stamps[tile * 8 + phase]; allocates and
   frees its own buffers, synchronous. Returns the number of tiles (CTAs), or a negative CUDA error
   code. */
int xs_stack_group_profile(const int* dev_stack, int S, unsigned blk, unsigned long long* host_stamps, int capacity,
  void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  xs_sort_batch_t d;
  memset(&d, 0, sizeof(d));
  d.nstacks = 1;
  d.stack[0] = dev_stack;
  d.S[0] = S;
  d.off[0] = 0;
  d.gidx[0] = 0;
  d.blk[0] = blk;
  xs_sort_batch_t dp = d;
  int large = 0, ncta = 0;
  if (0 < S && S <= kClusterEntries) {
    ncta = 1;
    while (ncta * kClThreads * kClE < S) ncta <<= 1;
  }
  const int grid = (0 < ncta) ? ncta : plan_tiles(&dp, &large);
  if (0 == grid || capacity < grid * 8) return -(int)cudaErrorInvalidValue;
  const size_t ks = sizeof(unsigned) * (size_t)S, vs = sizeof(unsigned long long) * (size_t)S;
  char* buf = nullptr;
  const size_t scr = xs_stack_sort_scratch_bytes(S);
  const size_t total = 3 * ks + 3 * vs + scr + 8 * sizeof(unsigned long long) * grid + 8192;
  cudaError_t r = cudaMallocAsync((void**)&buf, total, s);
  if (cudaSuccess != r) return -(int)r;
  char* p = buf;
  unsigned* k0 = (unsigned*)p; p += ks;
  unsigned* k1 = (unsigned*)p; p += ks;
  unsigned* ko = (unsigned*)p; p += ks;
  p = (char*)(((uintptr_t)p + 255) & ~(uintptr_t)255);
  unsigned long long* v0 = (unsigned long long*)p; p += vs;
  unsigned long long* v1 = (unsigned long long*)p; p += vs;
  unsigned long long* vo = (unsigned long long*)p; p += vs;
  unsigned long long* st = (unsigned long long*)p; p += 8 * sizeof(unsigned long long) * grid;
  int* seg = (int*)p; p += 256;
  p = (char*)(((uintptr_t)p + 255) & ~(uintptr_t)255);
  int rc = (0 < ncta) ? cluster_group_launch(dev_stack, S, 0, blk, k0, v0, k1, v1, ko, vo, seg, nullptr, 0, (SortCtl*)p, ncta, 0, s, st)
                      : cudaErrorNotSupported;
  if (cudaErrorNotSupported == rc) rc = group_launch(d, k0, v0, k1, v1, ko, vo, seg, p, s, st, 1);
  if (0 == rc) rc = (int)cudaMemcpyAsync(host_stamps, st, 8 * sizeof(unsigned long long) * grid, cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(buf, s);
  if (cudaSuccess == (cudaError_t)rc) rc = (int)cudaStreamSynchronize(s);
  return (0 == rc) ? grid : -rc;
}

}  // extern "C"
