/*
 * Stable device sort of a stack by its c offset (the grouping step of the plain FP64 stack path).
 *
 * The c offsets of one stack are few distinct values spread over a large range (C blocks of one
 * shape in a pool), so they are first mapped to dense bucket ids id = (c - cmin) / g, where g is the
 * gcd of all differences c - c0 (for a pool of equal blocks g is the block size). The extract kernel
 * one cooperative kernel computes cmin, cmax and g (phase 0, while it splits the stack into keys
 * and payload) and then runs an LSD counting sort over the ids with digits of at most 2048
 * buckets: a single pass when the stack touches at most 2048 distinct C blocks (the common case),
 * two or three otherwise. Per pass: per-tile digit histograms -> one exclusive scan per digit over the tiles ->
 * stable scatter (rank within a tile from warp match masks and per-warp counts). The ordering of
 * equal keys is the stack order, so the permutation is bit-exact and reproducible.
 * Grid-wide barriers spin on a global counter with an iteration limit; on timeout the kernel sets
 * an error flag and returns, and the host reports the error instead of hanging.
 */
#include "internal.h"
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kRadixBits = 11;
constexpr int kRadix = 1 << kRadixBits;
constexpr unsigned kSpinLimit = 1u << 24;

/* Zero-initialised by one memset per call: the minimum is kept as its complement (atomicMax). */
struct SortCtl {
  unsigned ncmin, cmax, gcd, pad0;
  unsigned bar_count, bar_gen, err, pad1;
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

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

/* Bounded grid barrier (all CTAs are co-resident: cooperative launch). Returns false on timeout
   or if another CTA reported an error. */
__device__ bool grid_sync(SortCtl* ctl) {
  __shared__ int s_ok;
  __syncthreads();
  if (0 == threadIdx.x) {
    volatile unsigned* const vgen = &ctl->bar_gen;
    const unsigned gen = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(&ctl->bar_count, 1u);
    int ok = 1;
    if (arrived == gridDim.x - 1) {
      atomicExch(&ctl->bar_count, 0u);
      __threadfence();
      atomicAdd(&ctl->bar_gen, 1u);
    }
    else {
      unsigned spins = 0;
      while (*vgen == gen) {
        if (++spins > kSpinLimit) {
          atomicExch(&ctl->err, 1u);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    if (0 != *(volatile unsigned*)&ctl->err) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return 0 != s_ok;
}

/* Extend a running gcd by x; skips the gcd when g already divides x (the common case). */
__device__ __forceinline__ unsigned gcd_acc(unsigned g, unsigned x) {
  return (0 != g && 0 == x % g) ? g : gcd_u(g, x);
}

/* Bucket id (c - cmin) / g. g divides every c - cmin, so the quotient is an exact integer below
   2^32 and the double product x * (1/g) is within far less than 0.5 of it: rounding recovers it. */
__device__ __forceinline__ unsigned bucket_of(unsigned c, unsigned cmin, double inv_g) {
  return __double2uint_rn((double)(c - cmin) * inv_g);
}

/* Block-wide exclusive scan of R values held PER per thread (thread i owns [i*PER, (i+1)*PER)). */
template <int PER>
__device__ __forceinline__ void block_exscan(int (&v)[PER], int* s_wsum) {
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
  int run = x - sum;
  for (int w2 = 0; w2 < warp; ++w2) run += s_wsum[w2];
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int t = v[j];
    v[j] = run;
    run += t;
  }
  __syncthreads();
}

/* Extract + stable LSD counting sort of a stack by bucket id, one cooperative kernel.
   Layout: CTA = tile of up to kSortThreads*E consecutive entries; warp w owns the contiguous
   sub-range [w0, w0 + 32E) and lane l holds entries w0 + l + 32r (r < E) in registers for the
   whole kernel, so every phase costs about one round trip to memory.
   Phase 0: load the AoS stack, contribute min(c), max(c) and the gcd of c - c0 (one set of atomics
   per CTA). Per pass (radix R = 2^rb <= 2048 buckets, as few passes as the bucket range needs):
   tile histograms hist[tile][digit] -> barrier -> digit bases of this tile (exclusive scan over
   digits of the digit totals plus the prefix over lower tiles; computed directly when the table is
   small, else by one owner thread per digit and a second barrier) -> stable scatter: each warp
   counts its digits, the counts become per-warp offsets, each warp places its entries in order
   (ranks inside 32 entries from match masks). Later passes reload their tile from the previous
   pass's output after a barrier. */
template <int E>
__global__ void __launch_bounds__(kSortThreads) xs_stack_group_kernel(const int* __restrict__ stack, int S,
  unsigned* __restrict__ k0, unsigned long long* __restrict__ v0, unsigned* __restrict__ k1,
  unsigned long long* __restrict__ v1, unsigned* __restrict__ kout, unsigned long long* __restrict__ vout,
  int* __restrict__ seglist, int* __restrict__ hist, SortCtl* ctl, unsigned long long* __restrict__ stamps) {
  __shared__ unsigned short s_wc[kSortWarps][kRadix];
  __shared__ int s_base[kRadix]; /* digit histogram in (a), digit write positions in (b)/(c) */
  __shared__ int s_wsum[kSortWarps];
  __shared__ unsigned s_red[3][kSortWarps];
  const int G = gridDim.x, tile = blockIdx.x;
  const int T = (S + G - 1) / G, t0 = min(S, tile * T), t1 = min(S, t0 + T);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int w0 = min(t1, t0 + warp * 32 * E), w1 = min(t1, w0 + 32 * E);
  unsigned key[E];
  unsigned long long val[E];
  /* optional phase timestamps (stamps != nullptr): [tile][8] */
#define XS_STAMP(slot) \
  do { \
    if (nullptr != stamps && 0 == threadIdx.x) stamps[tile * 8 + (slot)] = global_ns(); \
  } while (0)
  XS_STAMP(0);

  /* phase 0: load + bucket statistics */
  {
    const unsigned c0 = (unsigned)stack[2];
    unsigned lo = 0xFFFFFFFFu, hi = 0u, gg = 0u;
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int i = w0 + lane + 32 * r;
      key[r] = 0u;
      val[r] = 0ull;
      if (i < w1) {
        const int a = stack[3 * i + 0], b = stack[3 * i + 1];
        key[r] = (unsigned)stack[3 * i + 2];
        val[r] = (unsigned long long)(unsigned)a | ((unsigned long long)(unsigned)b << 32);
      }
    }
#pragma unroll
    for (int r = 0; r < E; ++r) {
      if (w0 + lane + 32 * r < w1) {
        const unsigned c = key[r];
        lo = min(lo, c);
        hi = max(hi, c);
        gg = gcd_acc(gg, (c > c0) ? c - c0 : c0 - c);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      gg = gcd_acc(gg, __shfl_xor_sync(0xffffffffu, gg, o));
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
        gg = gcd_acc(gg, s_red[2][w]);
      }
      if (lo != 0xFFFFFFFFu) {
        atomicMax(&ctl->ncmin, ~lo);
        atomicMax(&ctl->cmax, hi);
      }
      if (0 != gg) {
        unsigned old = *(volatile unsigned*)&ctl->gcd;
        while (0 == old || gcd_u(old, gg) != old) { /* no CAS once the global gcd divides this one */
          const unsigned assumed = old;
          old = atomicCAS(&ctl->gcd, assumed, gcd_u(assumed, gg));
          if (old == assumed) break;
        }
      }
      if (0 == tile) seglist[0] = 0;
    }
    XS_STAMP(1);
    if (!grid_sync(ctl)) return;
    XS_STAMP(2);
  }
  const unsigned cmin = ~*(volatile unsigned*)&ctl->ncmin, g = *(volatile unsigned*)&ctl->gcd;
  const unsigned cmax = *(volatile unsigned*)&ctl->cmax;
  const unsigned nb = (0 == g) ? 1u : (cmax - cmin) / g + 1u;
  const double inv_g = (0 == g) ? 0.0 : 1.0 / (double)g;
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
    return;
  }
  const int rb = (bits + passes - 1) / passes, R = 1 << rb;
  const bool direct = (size_t)G * R <= 32768; /* small table: each CTA scans it itself */
  for (int pass = 0; pass < passes; ++pass) {
    const int shift = pass * rb;
    const bool last = (pass + 1 == passes);
    unsigned* const kdst = last ? kout : ((0 == (pass & 1)) ? k1 : k0);
    unsigned long long* const vdst = last ? vout : ((0 == (pass & 1)) ? v1 : v0);
    int dig[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
      dig[r] = (w0 + lane + 32 * r < w1) ? (int)((bucket_of(key[r], cmin, inv_g) >> shift) & (R - 1)) : kRadix;
    }
    /* (a) tile histogram, row hist[tile][0..R); per-warp counters zeroed for (c) */
    for (int d = threadIdx.x; d < R; d += blockDim.x) s_base[d] = 0;
    for (int j = threadIdx.x; j < kSortWarps * kRadix; j += blockDim.x) {
      if ((j & (kRadix - 1)) < R) (&s_wc[0][0])[j] = 0;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) {
      if (kRadix != dig[r]) atomicAdd(&s_base[dig[r]], 1);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < R; d += blockDim.x) hist[(size_t)tile * R + d] = s_base[d];
    if (0 == pass) XS_STAMP(3);
    if (!grid_sync(ctl)) return;
    if (0 == pass) XS_STAMP(4);
    /* (b) digit bases of this tile. Data written by other CTAs in this kernel is read with __ldcg
       (from L2), never through a possibly stale L1 line; table reads are unrolled by 8. */
    /* thread i owns digits [i*per, (i+1)*per): all threads share the R digits */
    constexpr int PER = kRadix / kSortThreads;
    const int per = (R + kSortThreads - 1) / kSortThreads;
    int tot[PER], pre[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) tot[j] = pre[j] = 0;
    if (direct) {
      for (int tt = 0; tt < G; tt += 8) {
        int h[8][PER];
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
          for (int j = 0; j < PER; ++j) {
            const int d = threadIdx.x * per + j;
            h[u][j] = (j < per && tt + u < G && d < R) ? __ldcg(hist + (size_t)(tt + u) * R + d) : 0;
          }
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
          for (int j = 0; j < PER; ++j) {
            tot[j] += h[u][j];
            pre[j] += (tt + u < tile) ? h[u][j] : 0;
          }
      }
    }
    else { /* one owner warp per digit scans its column in place (32 tiles per step, all loads issued
              first), totals to the extra row G */
      for (int d = tile * kSortWarps + warp; d < R; d += G * kSortWarps) {
        constexpr int kMaxSteps = 8; /* G <= 256 tiles */
        int h[kMaxSteps];
#pragma unroll
        for (int q = 0; q < kMaxSteps; ++q) {
          const int tt = 32 * q + lane;
          h[q] = (tt < G) ? __ldcg(hist + (size_t)tt * R + d) : 0;
        }
        int run = 0;
#pragma unroll
        for (int q = 0; q < kMaxSteps; ++q) {
          int x = h[q];
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
          }
          const int tt = 32 * q + lane;
          if (tt < G) hist[(size_t)tt * R + d] = run + x - h[q];
          run += __shfl_sync(0xffffffffu, x, 31);
        }
        if (0 == lane) hist[(size_t)G * R + d] = run;
      }
      if (!grid_sync(ctl)) return;
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        const int d = threadIdx.x * per + j;
        tot[j] = (j < per && d < R) ? __ldcg(hist + (size_t)G * R + d) : 0;
        pre[j] = (j < per && d < R) ? __ldcg(hist + (size_t)tile * R + d) : 0;
      }
    }
    block_exscan<PER>(tot, s_wsum);
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int d = threadIdx.x * per + j;
      if (j < per && d < R) s_base[d] = tot[j] + pre[j];
    }
    if (0 == pass) XS_STAMP(5);
    /* (c) stable scatter: per-warp counts -> per-warp offsets -> ordered placement */
    unsigned peers[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
      peers[r] = __match_any_sync(0xffffffffu, dig[r]);
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
    if (!last) {
      if (!grid_sync(ctl)) return;
#pragma unroll
      for (int r = 0; r < E; ++r) {
        const int i = w0 + lane + 32 * r;
        if (i < w1) {
          key[r] = __ldcg(kdst + i);
          val[r] = __ldcg(vdst + i);
        }
      }
    }
  }
  XS_STAMP(7);
#undef XS_STAMP
}

/* Entries per thread kept in registers: 8 (tiles of 2048) or 16 (tiles of 4096). */
constexpr int kTileSmall = kSortThreads * 8, kTileLarge = kSortThreads * 16;

int sort_grid_max(void) {
  static int grid = 0;
  if (0 == grid) {
    int a = 0, b = 0;
    if (cudaSuccess != cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, xs_stack_group_kernel<8>, kSortThreads, 0)) a = 1;
    if (cudaSuccess != cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, xs_stack_group_kernel<16>, kSortThreads, 0)) b = 1;
    const int per_sm = a < b ? a : b;
    grid = xs_sm_count() * (per_sm < 1 ? 1 : per_sm);
    if (grid > 256) grid = 256; /* the owner-warp digit scan covers at most 256 tiles */
  }
  return grid;
}

/* Tiles: as few as possible of at most kTileSmall entries, or of kTileLarge when the stack needs more
   tiles than fit on the device. Returns the grid (0 if the stack is larger than one launch takes). */
int sort_grid(int S, int* large) {
  const int gmax = sort_grid_max();
  int grid = (S + kTileSmall - 1) / kTileSmall;
  *large = 0;
  if (grid > gmax) {
    grid = (S + kTileLarge - 1) / kTileLarge;
    *large = 1;
    if (grid > gmax) return 0;
  }
  return grid < 1 ? 1 : grid;
}

}  // namespace

extern "C" {

size_t xs_stack_sort_scratch_bytes(int S) {
  int large = 0;
  const size_t G = (size_t)sort_grid(S, &large);
  return sizeof(SortCtl) + 256 + sizeof(int) * ((G + 1) * kRadix);
}

int xs_stack_group_max(void) { return sort_grid_max() * kTileLarge; }

static int xs_stack_group_impl(const int* dev_stack, int S, unsigned* k0, unsigned long long* v0, unsigned* k1,
  unsigned long long* v1, unsigned* kout, unsigned long long* vout, int* seglist, void* sort_scratch, void* stream,
  unsigned long long* stamps) {
  cudaStream_t s = (cudaStream_t)stream;
  SortCtl* ctl = (SortCtl*)sort_scratch;
  int* hist = (int*)((char*)sort_scratch + sizeof(SortCtl) + 256);
  int large = 0;
  int grid = sort_grid(S, &large);
  if (0 == grid) return (int)cudaErrorInvalidValue; /* callers split stacks above xs_stack_group_max() */
  cudaError_t r = cudaMemsetAsync(ctl, 0, sizeof(SortCtl), s);
  if (cudaSuccess != r) return (int)r;
  void* args[] = {&dev_stack, &S, &k0, &v0, &k1, &v1, &kout, &vout, &seglist, &hist, &ctl, &stamps};
  return (int)cudaLaunchCooperativeKernel(
    large ? (const void*)xs_stack_group_kernel<16> : (const void*)xs_stack_group_kernel<8>, dim3(grid), dim3(kSortThreads),
    args, 0, s);
}

int xs_stack_group(const int* dev_stack, int S, unsigned* k0, unsigned long long* v0, unsigned* k1,
  unsigned long long* v1, unsigned* kout, unsigned long long* vout, int* seglist, void* sort_scratch, void* stream) {
  return xs_stack_group_impl(dev_stack, S, k0, v0, k1, v1, kout, vout, seglist, sort_scratch, stream, nullptr);
}

/* Diagnostic variant: the grouping of one stack with per-CTA phase timestamps (ns, %globaltimer)
   written to stamps[tile * 8 + phase]; allocates and frees its own buffers, synchronous. Returns the
   number of tiles (CTAs), or a negative CUDA error code. */
int xs_stack_group_profile(const int* dev_stack, int S, unsigned long long* host_stamps, int capacity, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  int large = 0;
  const int grid = sort_grid(S, &large);
  if (0 == grid || capacity < grid * 8) return -(int)cudaErrorInvalidValue;
  const size_t ks = sizeof(unsigned) * (size_t)S, vs = sizeof(unsigned long long) * (size_t)S;
  char* buf = nullptr;
  const size_t scr = xs_stack_sort_scratch_bytes(S);
  const size_t total = 3 * ks + 3 * vs + sizeof(int) * 2 + scr + 8 * sizeof(unsigned long long) * grid + 4096;
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
  int rc = xs_stack_group_impl(dev_stack, S, k0, v0, k1, v1, ko, vo, seg, p, s, st);
  if (0 == rc) rc = (int)cudaMemcpyAsync(host_stamps, st, 8 * sizeof(unsigned long long) * grid, cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(buf, s);
  if (cudaSuccess == (cudaError_t)rc) rc = (int)cudaStreamSynchronize(s);
  return (0 == rc) ? grid : -rc;
}

int xs_stack_sort_error(void* sort_scratch, int* err, void* stream) {
  SortCtl* ctl = (SortCtl*)sort_scratch;
  unsigned e = 0;
  cudaError_t r = cudaMemcpyAsync(&e, &ctl->err, sizeof(e), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
  if (cudaSuccess == r) r = cudaStreamSynchronize((cudaStream_t)stream);
  *err = (int)e;
  return (int)r;
}

}  // extern "C"
