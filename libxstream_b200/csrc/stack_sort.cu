/*
 * Stable device sort of a stack by its c offset (the grouping step of the plain FP64 stack path).
 *
 * The c offsets of one stack are few distinct values spread over a large range (C blocks of one
 * shape in a pool), so they are first mapped to dense bucket ids id = (c - cmin) / g, where g is the
 * gcd of all differences c - c0 (for a pool of equal blocks g is the block size). The extract kernel
 * computes cmin, cmax and g with atomics while it splits the stack into keys and payload. One
 * cooperative kernel then runs an LSD counting sort over the ids with 2048-bucket digits: a single
 * pass when the stack touches at most 2048 distinct C blocks (the common case), two or three
 * otherwise. Per pass: per-tile digit histograms -> one exclusive scan per digit over the tiles ->
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

__device__ __forceinline__ unsigned gcd_u(unsigned a, unsigned b) {
  while (0 != b) {
    const unsigned t = a % b;
    a = b;
    b = t;
  }
  return a;
}

/* Extract kernel (replaces the plain split): keys, payload, and the bucket-mapping statistics. */
__global__ void xs_extract_stats_kernel(const int* __restrict__ stack, int S, unsigned* __restrict__ keys,
  unsigned long long* __restrict__ vals, int* __restrict__ seglist, SortCtl* __restrict__ ctl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned c0 = (unsigned)stack[2];
  unsigned lo = 0xFFFFFFFFu, hi = 0u, gg = 0u;
  if (0 == i) seglist[0] = 0;
  if (i < S) {
    const int a = stack[3 * i + 0], b = stack[3 * i + 1], c = stack[3 * i + 2];
    keys[i] = (unsigned)c;
    vals[i] = (unsigned long long)(unsigned)a | ((unsigned long long)(unsigned)b << 32);
    lo = hi = (unsigned)c;
    gg = ((unsigned)c > c0) ? (unsigned)c - c0 : c0 - (unsigned)c;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    gg = gcd_u(gg, __shfl_xor_sync(0xffffffffu, gg, o));
  }
  /* one set of global atomics per CTA */
  __shared__ unsigned s_lo[32], s_hi[32], s_g[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (0 == lane) {
    s_lo[warp] = lo;
    s_hi[warp] = hi;
    s_g[warp] = gg;
  }
  __syncthreads();
  if (0 == threadIdx.x) {
    for (int w = 1; w < nw; ++w) {
      lo = min(lo, s_lo[w]);
      hi = max(hi, s_hi[w]);
      gg = gcd_u(gg, s_g[w]);
    }
    if (lo != 0xFFFFFFFFu) {
      atomicMax(&ctl->ncmin, ~lo);
      atomicMax(&ctl->cmax, hi);
    }
    if (0 != gg) {
      unsigned old = *(volatile unsigned*)&ctl->gcd, assumed;
      while (gcd_u(old, gg) != old || 0 == old) { /* skip the CAS when the global gcd already divides */
        assumed = old;
        old = atomicCAS(&ctl->gcd, assumed, gcd_u(assumed, gg));
        if (old == assumed) break;
      }
    }
  }
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
        __nanosleep(64);
      }
    }
    __threadfence();
    if (0 != *(volatile unsigned*)&ctl->err) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return 0 != s_ok;
}

__device__ __forceinline__ unsigned bucket_of(unsigned c, unsigned cmin, unsigned g) {
  return (0 == g) ? 0u : (c - cmin) / g;
}

/* Cooperative LSD counting sort of (keys, vals) by bucket id. hist holds kRadix * gridDim.x ints. */
__global__ void __launch_bounds__(kSortThreads) xs_stack_sort_kernel(int S, unsigned* __restrict__ k0,
  unsigned long long* __restrict__ v0, unsigned* __restrict__ k1, unsigned long long* __restrict__ v1,
  unsigned* __restrict__ kout, unsigned long long* __restrict__ vout, int* __restrict__ hist, SortCtl* ctl) {
  __shared__ unsigned short s_wc[kSortWarps][kRadix];
  __shared__ int s_base[kRadix]; /* digit histogram in (a), digit write positions in (c)/(d) */
  int* const s_hist = s_base;
  const int G = gridDim.x, tile = blockIdx.x;
  const int T = (S + G - 1) / G, t0 = min(S, tile * T), t1 = min(S, t0 + T);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned cmin = ~ctl->ncmin, g = ctl->gcd;
  const unsigned nb = (0 == g) ? 1u : (ctl->cmax - cmin) / g + 1u;
  int bits = 0;
  while (bits < 32 && (nb - 1u) >> bits) ++bits;
  const int passes = (bits + kRadixBits - 1) / kRadixBits;
  if (0 == passes) { /* a single C block: already grouped, keep stack order */
    for (int i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
      kout[i] = __ldcg(k0 + i);
      vout[i] = __ldcg(v0 + i);
    }
    return;
  }
  const unsigned* kin = k0;
  const unsigned long long* vin = v0;
  for (int pass = 0; pass < passes; ++pass) {
    const int shift = pass * kRadixBits;
    const bool last = (pass + 1 == passes);
    unsigned* const kdst = last ? kout : ((0 == (pass & 1)) ? k1 : k0);
    unsigned long long* const vdst = last ? vout : ((0 == (pass & 1)) ? v1 : v0);
    /* (a) tile histogram */
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) s_hist[d] = 0;
    __syncthreads();
    for (int i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
      atomicAdd(&s_hist[(bucket_of(__ldcg(kin + i), cmin, g) >> shift) & (kRadix - 1)], 1);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) hist[(size_t)d * G + tile] = s_hist[d];
    if (!grid_sync(ctl)) return;
    /* (b) exclusive scan over the tiles of each digit this CTA owns (one digit per warp); the
       digit totals go to the extra row hist[kRadix * G + d]. Data written by other CTAs in this
       kernel is read with __ldcg (L2), never through a possibly stale L1 line. */
    for (int d = tile * kSortWarps + warp; d < kRadix; d += G * kSortWarps) {
      int run = 0;
      for (int base = 0; base < G; base += 32) {
        const int t = base + lane;
        const int v = (t < G) ? __ldcg(hist + (size_t)d * G + t) : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += y;
        }
        if (t < G) hist[(size_t)d * G + t] = run + x - v;
        run += __shfl_sync(0xffffffffu, x, 31);
      }
      if (0 == lane) hist[(size_t)kRadix * G + d] = run;
    }
    if (!grid_sync(ctl)) return;
    /* (c) digit bases for this tile: exclusive scan of the digit totals plus the tile prefix */
    {
      /* block-wide exclusive scan of kRadix totals: each thread scans kRadix / kSortThreads values */
      constexpr int PER = kRadix / kSortThreads;
      int v[PER], sum = 0;
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        v[j] = __ldcg(hist + (size_t)kRadix * G + threadIdx.x * PER + j);
        sum += v[j];
      }
      int x = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      __shared__ int s_wsum[kSortWarps];
      if (31 == lane) s_wsum[warp] = x;
      __syncthreads();
      int wpre = 0;
      for (int w2 = 0; w2 < warp; ++w2) wpre += s_wsum[w2];
      int run = wpre + x - sum;
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        const int d = threadIdx.x * PER + j;
        s_base[d] = run + __ldcg(hist + (size_t)d * G + tile);
        run += v[j];
      }
    }
    __syncthreads();
    /* (d) stable scatter, one round of blockDim entries at a time */
    for (int r0 = t0; r0 < t1; r0 += blockDim.x) {
      for (int j = threadIdx.x; j < kSortWarps * kRadix; j += blockDim.x) (&s_wc[0][0])[j] = 0;
      __syncthreads();
      const int i = r0 + threadIdx.x;
      const bool valid = i < t1;
      unsigned key = 0;
      unsigned long long val = 0;
      int d = kRadix; /* invalid lanes get a digit of their own */
      if (valid) {
        key = __ldcg(kin + i);
        val = __ldcg(vin + i);
        d = (int)((bucket_of(key, cmin, g) >> shift) & (kRadix - 1));
      }
      const unsigned peers = __match_any_sync(0xffffffffu, d);
      const int rank = __popc(peers & ((1u << lane) - 1u));
      if (valid && 0 == rank) s_wc[warp][d] = (unsigned short)__popc(peers);
      __syncthreads();
      if (valid) {
        int before = 0;
        for (int w2 = 0; w2 < warp; ++w2) before += s_wc[w2][d];
        const int pos = s_base[d] + before + rank;
        kdst[pos] = key;
        vdst[pos] = val;
      }
      __syncthreads();
      for (int dd = threadIdx.x; dd < kRadix; dd += blockDim.x) {
        int tot = 0;
#pragma unroll
        for (int w2 = 0; w2 < kSortWarps; ++w2) tot += s_wc[w2][dd];
        s_base[dd] += tot;
      }
      __syncthreads();
    }
    if (!last) {
      if (!grid_sync(ctl)) return;
      kin = kdst;
      vin = vdst;
    }
  }
}

int sort_grid_size(void) {
  static int grid = 0;
  if (0 == grid) {
    int per_sm = 0;
    if (cudaSuccess != cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, xs_stack_sort_kernel, kSortThreads, 0)) {
      per_sm = 1;
    }
    if (per_sm < 1) per_sm = 1;
    grid = xs_sm_count() * (per_sm < 2 ? per_sm : 2);
  }
  return grid;
}

}  // namespace

extern "C" {

size_t xs_stack_sort_scratch_bytes(int S) {
  const size_t G = (size_t)sort_grid_size();
  (void)S;
  return sizeof(SortCtl) + 256 + sizeof(int) * ((size_t)kRadix * G + kRadix);
}

int xs_stack_extract(const int* dev_stack, int S, unsigned* keys, unsigned long long* vals, int* seglist, void* sort_scratch,
  void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  SortCtl* const ctl = (SortCtl*)sort_scratch;
  cudaError_t r = cudaMemsetAsync(ctl, 0, sizeof(SortCtl), s);
  if (cudaSuccess != r) return (int)r;
  xs_extract_stats_kernel<<<(S + 255) / 256, 256, 0, s>>>(dev_stack, S, keys, vals, seglist, ctl);
  return (int)cudaGetLastError();
}

int xs_stack_sort(int S, unsigned* k0, unsigned long long* v0, unsigned* k1, unsigned long long* v1, unsigned* kout,
  unsigned long long* vout, void* sort_scratch, void* stream) {
  SortCtl* ctl = (SortCtl*)sort_scratch;
  int* hist = (int*)((char*)sort_scratch + sizeof(SortCtl) + 256);
  /* tiles of at least kMinTile entries: fewer tiles mean smaller digit histograms to scan */
  constexpr int kMinTile = 1024;
  int grid = sort_grid_size();
  const int tiles_needed = (S + kMinTile - 1) / kMinTile;
  if (grid > tiles_needed) grid = tiles_needed > 0 ? tiles_needed : 1;
  void* args[] = {&S, &k0, &v0, &k1, &v1, &kout, &vout, &hist, &ctl};
  return (int)cudaLaunchCooperativeKernel((const void*)xs_stack_sort_kernel, dim3(grid), dim3(kSortThreads), args, 0,
    (cudaStream_t)stream);
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
