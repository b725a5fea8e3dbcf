/*
 * sm_100a kernels for the DBCSR stack path: plain FP64 stack multiply, batched in-place transpose,
 * block norms, and the FP64 tensor-pipe peak probe.
 *
 * Plain FP64 stack multiply (replaces samples/smm/kernels/multiply.cl:80-701 and the launch in
 * samples/smm/smm_kernel.c:462-507). Semantics per stack entry (a, b, c), 1-based offsets:
 *     C(i,j) += sum_kk A(i,kk) * B(kk,j),   A(i,kk) = a[a-1 + kk*m + i]   (m x k, column-major)
 *                                           B(kk,j) = b[b-1 + kk*n + j]   (pre-transposed k x n)
 *                                           C(i,j)  = c[c-1 + j*m + i]    (m x n, column-major)
 * (multiply.cl:12-15 ADX/BDX/CDX with IDX/IDT from libxstream_common.h:86-87).
 *
 * B200 design, instead of the reference's one-work-group-per-mini-batch with FP atomics at every
 * change of c (multiply.cl:621-695):
 *   1. The stack's c offsets are sorted stably (device radix sort): entries of one C block become
 *      a contiguous segment, in stack order.
 *   2. The sorted stack is cut into chunks of L entries (perfect load balance whatever the c
 *      distribution). One warp owns one chunk and one warp sub-tile of C (8*MT x 8*NT). It streams
 *      DMMA fragments (mma.sync m8n8k4 f64) straight from L2/HBM into registers, one k-panel ahead
 *      of the tensor pipe, and keeps the C sub-tile in registers across the whole segment.
 *   3. A segment that lies inside one chunk is written back once (red.global.add.f64: a single
 *      writer per element, so the result is deterministic). A segment that crosses chunk
 *      boundaries leaves one partial tile ("piece") per chunk in scratch; a second kernel sums the
 *      pieces of each such segment in a fixed order and writes the block once.
 *   The result is bitwise reproducible from run to run, unlike FP atomics.
 */
#include "internal.h"
#include "tc_ptx.cuh"
#include "../../include/libxstream_b200.h"
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

namespace {

/* Warps of the combine kernel (its warp partials go through dynamic shared memory). */
constexpr int kCombineWarps = 16;

/* Programmatic dependent launch: a kernel launched with pdl_launch may be scheduled while the
   kernel before it in the stream is still running (once that kernel's CTAs have all passed
   pdl_trigger or exited); it must call pdl_wait before it reads anything its predecessor writes.
   Both are no-ops for a kernel launched the ordinary way. */
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

template <typename... KArgs, typename... Args>
cudaError_t pdl_launch(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

/* Release/acquire fence at GPU scope: orders this thread's piece stores before its (relaxed) arrival
   increment, and a CTA's reads of the other CTAs' pieces after the increment that found them all
   published. Lighter than the sequentially consistent __threadfence(). */
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

/* Bring a block of `count` contiguous doubles into L2 (one prefetch per 128-byte line, by 32 lanes). */
__device__ __forceinline__ void prefetch_block_l2(const double* p, int count, int lane) {
  for (int x = 16 * lane; x < count + 15; x += 16 * 32) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p + (x < count ? x : count - 1)));
  }
}

__device__ __forceinline__ void dmma_m8n8k4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

/* Per-lane geometry of a warp sub-tile (8*MT x 8*NT of C): which fragment rows/columns it loads. */
template <int MT, int NT>
struct Tile {
  bool rok[MT], cok[NT];
  int r0, c0;
  __device__ __forceinline__ void init(int sub, int nsub_n, int m, int n, int g) {
    const int sm = sub / nsub_n, sn = sub - sm * nsub_n;
    r0 = sm * 8 * MT;
    c0 = sn * 8 * NT;
#pragma unroll
    for (int i = 0; i < MT; ++i) rok[i] = r0 + 8 * i + g < m;
#pragma unroll
    for (int j = 0; j < NT; ++j) cok[j] = c0 + 8 * j + g < n;
  }
};

/* Write-back of a finished C sub-tile: each element has exactly one writer (red.global.add.f64). */
template <int MT, int NT>
__device__ __forceinline__ void commit_tile(double* __restrict__ C, size_t coff, const double (&acc)[MT][NT][2], int m,
  int n, int g, int t, const Tile<MT, NT>& tl, double alpha) {
#pragma unroll
  for (int i = 0; i < MT; ++i) {
    const int r = tl.r0 + 8 * i + g;
    if (r < m) {
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const int cc = tl.c0 + 8 * j + 2 * t;
        if (cc < n) atomicAdd(C + coff + (size_t)cc * m + r, alpha * acc[i][j][0]);
        if (cc + 1 < n) atomicAdd(C + coff + (size_t)(cc + 1) * m + r, alpha * acc[i][j][1]);
      }
    }
  }
}

/* How a warp holds its C sub-tile, for the merge and combine code that sums pieces ([REGS][32]
   doubles, element r of lane l at r * 32 + l) and writes a finished sum back: the DMMA fragments of an
   8*MT x 8*NT sub-tile (element (i, j, h) at (i * NT + j) * 2 + h). */
struct StackTask;
template <int MT, int NT>
struct DmmaLayout {
  static constexpr int REGS = MT * NT * 2;
  __device__ static __forceinline__ void commit(const StackTask& tk, int sub, size_t coff, const double (&sum)[REGS]);
};

/* Shared memory of the stack kernel: per warp two partial tiles (head / tail piece) + metadata. */
template <int MT, int NT>
__host__ __device__ constexpr size_t smm_smem_bytes(int warps) {
  return (size_t)warps * (2 * MT * NT * 2 * 32 * sizeof(double) + 4 * sizeof(int));
}

/* Registers per thread the kernel may use: tiles up to 3x3 run 3 CTAs of 4 warps per SM. */
__host__ __device__ constexpr int smm_min_blocks(int mt, int nt) { return (mt * nt <= 9) ? 3 : 2; }

/* The stack kernel. M_, N_, K_ > 0 make the block shape a compile-time constant (every fragment
   load is then one load at an immediate offset from a per-lane base pointer); 0 means runtime.
   CTA = W warps = W consecutive chunks of L sorted entries, one warp sub-tile of C each. Per warp:
   DMMA fragments of the next k-panel (KP k-steps of 4) are loaded while the current panel runs;
   a segment that ends inside the chunk is written back at once; pieces of segments crossing chunk
   boundaries are merged inside the CTA through shared memory in warp order, and only segments that
   cross the CTA's own boundaries leave a CTA-level piece in global scratch for the combine kernel. */
/* What the stack kernel needs to know about one stack: one task for a single call, one per stack
   for a batch. keys/vals are the stack's grouped entries, pieces its CTA-level piece slots. */
struct StackTask {
  const double* a;
  const double* b;
  double* c;
  const unsigned* keys;
  const unsigned long long* vals;
  double* pieces;
  int S, m, n, k;
  int L, nchunks, ngroups, nsub_n, nsub;
  int item_begin; /* first work item of this stack (batch) */
  int cls;        /* tile class (MT - 1) * 4 + (NT - 1) (batch) */
  int sid;        /* stack index within the call: tag of its segment-list entries */
  int kind;       /* unified batch kernel: 0 = register kernel of tile class cls, else 1 + staged shape index */
  double alpha;   /* C += alpha * A * B (1 for the LIBSMM ABI) */
  int* arrive;    /* per (CTA group, sub-tile) arrival counters of CTA-crossing segments, zero at launch:
                     the stack kernel combines them itself; nullptr: they go to the combine kernel */
  const int* raw; /* the caller's parameter stack (input of the grouping), for the L2 prefetch */
  int rstride;    /* ints per parameter record (3 or 6) */
  int rbase;      /* a-offset position within a record (b follows) */
  int rshift;     /* added to a record's offsets to make them 0-based (-1: 1-based, 0: 0-based) */
  int npf;        /* records whose A and B blocks are prefetched into L2 (0: none) */
  int Ls[3];      /* entries per chunk in the CTA groups [0, slotn), [slotn, 2 slotn), [2 slotn, ...) */
  int slotn;      /* CTA groups per length class (the SM count when the lengths differ) */
};

/* First entry of chunk c (0 <= c <= nchunks; S at the end) when CTA group b = c / W holds W chunks
   of Ls[class of b] entries. The host makes the three lengths equal (chunk c starts at c L), or, for
   a one-wave launch of several CTAs per SM, longer for the CTAs launched first on their SM and
   shorter for the last ones: the SM's warp schedulers favour its older CTAs, so equal chunks leave
   the last-launched CTA's warps running alone at the end. */
__device__ __forceinline__ int chunk_first(const StackTask& tk, int W, int c) {
  const int b = c / W, w = c - b * W, sn = tk.slotn;
  const long long n0 = min(b, sn), n1 = min(max(b - sn, 0), sn), n2 = max(b - 2 * sn, 0);
  const int Lb = (b < sn) ? tk.Ls[0] : ((b < 2 * sn) ? tk.Ls[1] : tk.Ls[2]);
  const long long f = (long long)W * (n0 * tk.Ls[0] + n1 * tk.Ls[1] + n2 * tk.Ls[2]) + (long long)w * Lb;
  return (int)min(f, (long long)tk.S);
}

/* Bulk prefetch into L2 of the A and B blocks of the first tk.npf parameter records, dealt round-robin
   over the CTAs (record i to CTA i mod grid), so that every SM's copy unit issues a share. It reads only the caller's inputs (the raw stack and the pools), so a stack kernel
   runs it before pdl_wait, while the grouping that precedes it in the stream still runs and the
   pools would otherwise be fetched only at the first copy. A block's window is widened to 16-byte
   boundaries (the bulk-copy granule); a widened window never leaves the block's page. */
__device__ __forceinline__ void prefetch_block(const double* p, uint32_t bytes) {
  const uint64_t s = (uint64_t)p, s0 = s & ~15ull, s1 = (s + bytes + 15ull) & ~15ull;
  xs_tc::bulk_prefetch_l2((const void*)s0, (uint32_t)(s1 - s0));
}
__device__ __forceinline__ void prefetch_operands(const StackTask& tk) {
  if (0 >= tk.npf) return;
  const uint32_t abytes = (uint32_t)(tk.m * tk.k * sizeof(double)), bbytes = (uint32_t)(tk.k * tk.n * sizeof(double));
  const int nthreads = (int)(gridDim.x * blockDim.x);
  for (int i = (int)(blockIdx.x + gridDim.x * threadIdx.x); i < tk.npf; i += nthreads) {
    const int* const e = tk.raw + (size_t)tk.rstride * i + tk.rbase;
    prefetch_block(tk.a + (e[0] + tk.rshift), abytes);
    prefetch_block(tk.b + (e[1] + tk.rshift), bbytes);
  }
}

template <int MT, int NT>
__device__ __forceinline__ void DmmaLayout<MT, NT>::commit(const StackTask& tk, int sub, size_t coff, const double (&sum)[REGS]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  double tile[MT][NT][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      tile[i][j][0] = sum[(i * NT + j) * 2 + 0];
      tile[i][j][1] = sum[(i * NT + j) * 2 + 1];
    }
  Tile<MT, NT> tl;
  tl.init(sub, tk.nsub_n, tk.m, tk.n, g);
  commit_tile<MT, NT>(tk.c, coff, tile, tk.m, tk.n, g, t, tl, tk.alpha);
}

/* Segment-list entry: stack index (high 8 bits) and CTA group (low 24 bits). */
__device__ __forceinline__ int seg_tag(int sid, int group) { return (sid << 24) | group; }

/* Pieces per first-level combine of a long CTA-crossing segment. */
constexpr int kFan = 8;

/* Scratch slot of piece q of the segment whose first group is j0: the tail piece of group j0 (q = 0),
   else the head piece of group j0 + q. */
__device__ __forceinline__ int piece_slot(int j0, int q) { return (0 == q) ? 2 * j0 + 1 : 2 * (j0 + q); }

/* Groups j0 <= j <= j1 (j0, j1 returned) that hold entries of the segment with key x, for a segment
   that the CTA group j (W chunks, chunk_first) holds and that crosses j's first boundary (head: the
   entry before the group's first one has key x) and/or its last one (tail: the first entry of group
   j + 1 has key x). Keys are sorted, so the boundaries a segment
   crosses are consecutive: one warp tests 32 boundaries per round (one load per lane). */
__device__ __forceinline__ void segment_groups(const StackTask& tk, int W, int j, unsigned x, bool head, bool tail, int& j0,
  int& j1) {
  const int lane = threadIdx.x & 31;
  const unsigned* __restrict__ const keys = tk.keys;
  j0 = j;
  if (head) { /* boundary j - q is crossed iff the entry before group j - q's first one has key x */
    for (int q0 = 1;; q0 += 32) {
      const int gq = j - q0 - lane;
      const bool crossed = (gq >= 1) && __ldcg(keys + (size_t)chunk_first(tk, W, gq * W) - 1) == x;
      const unsigned m = __ballot_sync(0xFFFFFFFFu, crossed);
      if (0xFFFFFFFFu != m) {
        j0 = j - q0 - (__ffs(~m) - 1);
        break;
      }
    }
  }
  j1 = j;
  if (tail) { /* group j + 1 holds x; group j + q (q >= 2) does iff its first entry has key x */
    for (int q0 = 2;; q0 += 32) {
      const int gq = j + q0 + lane;
      const bool crossed = (gq < tk.ngroups) && __ldcg(keys + (size_t)chunk_first(tk, W, gq * W)) == x;
      const unsigned m = __ballot_sync(0xFFFFFFFFu, crossed);
      if (0xFFFFFFFFu != m) {
        j1 = j + q0 - 1 + (__ffs(~m) - 1);
        break;
      }
    }
  }
}

/* The CTA-level segment ranges of CTA group `group` (W chunks of L entries): probe[0] = the first
   group holding the segment that enters the CTA (group if none enters), probe[1] = the last group
   holding the segment that leaves it (group if none leaves). They depend on the grouped keys only, so
   one warp computes them while the CTA's first copies are in flight, and the merge at the end does
   not wait for these loads. Called by a whole warp; lane 0 writes probe. */
__device__ __forceinline__ void probe_boundaries(const StackTask& tk, int W, int group, int* probe) {
  const int S = tk.S, first = chunk_first(tk, W, group * W), lastp = chunk_first(tk, W, (group + 1) * W) - 1;
  const unsigned* __restrict__ const keys = tk.keys;
  const unsigned k0 = keys[first], k1 = keys[lastp];
  const bool hx = (0 < first) && keys[first - 1] == k0;
  const bool tx = (lastp + 1 < S) && keys[lastp + 1] == k1;
  int j0, j1, unused;
  segment_groups(tk, W, group, k0, hx, false, j0, unused);
  segment_groups(tk, W, group, k1, false, tx, unused, j1);
  if (0 == (threadIdx.x & 31)) {
    probe[0] = j0;
    probe[1] = j1;
  }
}

/* CTA-level merge of the warps' partial tiles. Chains start at warp 0's head piece (a segment
   entering the CTA) and at every tail piece (a segment starting in that warp's chunk); a chain
   continues through the head pieces of the following warps while the previous piece reaches the end
   of its chunk. A chain that stays inside the CTA is written back at once; one that crosses the CTA's
   boundaries becomes a CTA-level piece in global scratch (slot 2j for a piece that continues a
   segment of the previous group, 2j + 1 for one that starts in group j). Without arrival counters
   (tk.arrive == nullptr) the tail pieces are listed for the combine kernel. With them, the CTA finds
   the groups j0..j1 of the segment (its np = j1 - j0 + 1 pieces, piece q from group j0 + q) and
   publishes its piece (fence, then one atomic increment): a segment of at most kFan pieces has one
   counter, and the CTA whose increment completes it combines all pieces; a longer one is combined
   in two levels, kFan consecutive pieces per first-level counter (the CTA completing one sums them
   and then arrives at the segment's counter) and the first-level sums at the end. The CTA records
   what it completed in duty[slot] = {1, j0, np, key, level, first-level group} for finish_segments.
   piece_at(w, slot) is warp w's head (slot 0) or tail (slot 1) piece in shared memory, [REGS][32]
   doubles; meta[w][4] holds its head / head-spans / tail flags; probe (nullptr: found here) holds the
   CTA's segment ranges from probe_boundaries. Called by all threads after a CTA barrier. */
template <typename Lay, typename PieceAt>
__device__ __forceinline__ void cta_merge(const StackTask& tk, int group, int sub, int* __restrict__ seglist,
  const int* meta, int W, PieceAt piece_at, int (*duty)[6], const int* probe = nullptr) {
  constexpr int REGS = Lay::REGS;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int S = tk.S, L = tk.L, nchunks = tk.nchunks, nsub = tk.nsub;
  if (threadIdx.x < 12) duty[threadIdx.x / 6][threadIdx.x % 6] = 0;
  __syncthreads();
  for (int start = 0; start < 2; ++start) {
    const bool from_head = (0 == start);
    if (warp >= W) break; /* warps beyond the W chunk owners (a producer warp) hold no pieces */
    if (from_head && 0 != warp) continue;
    if (0 == meta[warp * 4 + (from_head ? 0 : 2)]) continue;
    double sum[REGS];
    const double* src = piece_at(warp, from_head ? 0 : 1) + lane;
#pragma unroll
    for (int r = 0; r < REGS; ++r) sum[r] = src[r * 32];
    bool spans = from_head ? (0 != meta[warp * 4 + 1]) : true;
    int cur = warp;
    while (spans && cur + 1 < W && group * W + cur + 1 < nchunks) {
      ++cur;
      src = piece_at(cur, 0) + lane;
#pragma unroll
      for (int r = 0; r < REGS; ++r) sum[r] += src[r * 32];
      spans = (0 != meta[cur * 4 + 1]);
    }
    const int c_first = group * W + warp; /* chunk where this chain starts */
    /* the chain's segment: the CTA's first key (head chain) or the last key of its first chunk */
    const unsigned key = from_head ? tk.keys[chunk_first(tk, W, group * W)] : tk.keys[chunk_first(tk, W, c_first + 1) - 1];
    if (from_head || spans) { /* the segment crosses a CTA boundary: CTA-level piece */
      const int slot = from_head ? 2 * group : 2 * group + 1;
      double* const dst = tk.pieces + ((size_t)slot * nsub + sub) * REGS * 32 + lane;
#pragma unroll
      for (int r = 0; r < REGS; ++r) dst[r * 32] = sum[r];
      if (nullptr == tk.arrive) {
        if (!from_head && 0 == sub && 0 == lane) {
          const int slotidx = atomicAdd(seglist, 1);
          seglist[1 + slotidx] = seg_tag(tk.sid, group);
        }
      }
      else {
        int j0, j1;
        if (nullptr != probe) { /* a head chain continues the segment entering the CTA; a spanning chain leaves it */
          j0 = from_head ? probe[0] : group;
          j1 = spans ? probe[1] : group;
        }
        else segment_groups(tk, W, group, key, from_head, spans, j0, j1);
        const int np = j1 - j0 + 1, q = group - j0;
        const int level = (np <= kFan) ? 2 : 1, i1 = q / kFan;
        const int target = (2 == level) ? np : min(kFan, np - i1 * kFan);
        int* const counter = (2 == level) ? tk.arrive + (size_t)j0 * nsub + sub
                                          : tk.arrive + (size_t)tk.ngroups * nsub + (size_t)piece_slot(j0, i1 * kFan) * nsub + sub;
        fence_acq_rel_gpu(); /* the piece is visible device-wide before the arrival */
        __syncwarp();
        int last = 0;
        if (0 == lane) {
          last = (atomicAdd(counter, 1) == target - 1) ? 1 : 0;
          if (last) fence_acq_rel_gpu(); /* acquire: the pieces this increment completed are visible */
        }
        if (0 != __shfl_sync(0xFFFFFFFFu, last, 0) && 0 == lane) {
          int* const d = duty[from_head ? 0 : 1];
          d[1] = j0;
          d[2] = np;
          d[3] = (int)key;
          d[4] = level;
          d[5] = i1;
          d[0] = 1;
        }
      }
    }
    else Lay::commit(tk, sub, (size_t)key - 1, sum);
  }
}

/* Sums count pieces, piece i at slot slot_of(i), in a fixed order: warp w takes pieces w, w + W, ...
   (two in flight), the warps' partials are added in warp order through red ([W - 1][REGS][32]
   doubles of shared memory no longer in use). The tree depends only on count and W, so the result is
   reproducible; it is valid in warp 0. Called by all threads; contains a CTA barrier. */
template <int REGS, typename SlotOf>
__device__ __forceinline__ void sum_pieces(const StackTask& tk, int sub, int count, SlotOf slot_of, double* red,
  double (&acc)[REGS]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
  const int nsub = tk.nsub;
#pragma unroll
  for (int r = 0; r < REGS; ++r) acc[r] = 0.0;
  int q = warp;
  for (; q + W < count; q += 2 * W) {
    const double* const p0 = tk.pieces + ((size_t)slot_of(q) * nsub + sub) * REGS * 32 + lane;
    const double* const p1 = tk.pieces + ((size_t)slot_of(q + W) * nsub + sub) * REGS * 32 + lane;
    double v0[REGS], v1[REGS];
#pragma unroll
    for (int r = 0; r < REGS; ++r) {
      v0[r] = __ldcg(p0 + r * 32);
      v1[r] = __ldcg(p1 + r * 32);
    }
#pragma unroll
    for (int r = 0; r < REGS; ++r) acc[r] += v0[r];
#pragma unroll
    for (int r = 0; r < REGS; ++r) acc[r] += v1[r];
  }
  if (q < count) {
    const double* const p0 = tk.pieces + ((size_t)slot_of(q) * nsub + sub) * REGS * 32 + lane;
#pragma unroll
    for (int r = 0; r < REGS; ++r) acc[r] += __ldcg(p0 + r * 32);
  }
  if (0 != warp) {
#pragma unroll
    for (int r = 0; r < REGS; ++r) red[((warp - 1) * REGS + r) * 32 + lane] = acc[r];
  }
  __syncthreads();
  if (0 == warp) {
    for (int w2 = 0; w2 < W - 1; ++w2) {
#pragma unroll
      for (int r = 0; r < REGS; ++r) acc[r] += red[(w2 * REGS + r) * 32 + lane];
    }
  }
}

/* Completes the combines this CTA's arrivals finished (duty, filled by cta_merge). A first-level
   duty sums its kFan (or fewer) pieces, stores the sum over the group's first piece and arrives at
   the segment's counter; the CTA completing that counter (or a duty of a short segment) sums the
   segment's pieces or first-level sums in order and writes the block once. Called by all threads
   after a CTA barrier that follows cta_merge; ends with a barrier. */
template <typename Lay>
__device__ __forceinline__ void finish_segments(const StackTask& tk, int sub, int (*duty)[6], double* red) {
  constexpr int REGS = Lay::REGS;
  __shared__ int s_go;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nsub = tk.nsub;
  for (int d = 0; d < 2; ++d) {
    if (0 == duty[d][0]) continue; /* uniform: shared memory read after a barrier */
    const int j0 = duty[d][1], np = duty[d][2], level = duty[d][4], i1 = duty[d][5];
    const unsigned key = (unsigned)duty[d][3];
    fence_acq_rel_gpu(); /* the other CTAs published their pieces before their arrivals */
    double acc[REGS];
    int count = np, stride = 1; /* what the final sum covers: pieces 0, stride, 2 * stride, ... */
    if (1 == level) {
      const int q1 = i1 * kFan, n1 = min(kFan, np - q1);
      sum_pieces<REGS>(tk, sub, n1, [&](int i) { return piece_slot(j0, q1 + i); }, red, acc);
      if (0 == warp) { /* the first-level sum replaces the group's first piece */
        double* const dst = tk.pieces + ((size_t)piece_slot(j0, q1) * nsub + sub) * REGS * 32 + lane;
#pragma unroll
        for (int r = 0; r < REGS; ++r) __stcg(dst + r * 32, acc[r]);
        fence_acq_rel_gpu();
        __syncwarp();
        int last = 0;
        if (0 == lane) {
          last = (atomicAdd(tk.arrive + (size_t)j0 * nsub + sub, 1) == (np + kFan - 1) / kFan - 1) ? 1 : 0;
          if (last) fence_acq_rel_gpu();
          s_go = last;
        }
      }
      __syncthreads();
      const int go = s_go;
      __syncthreads(); /* red and s_go may be reused */
      if (!go) continue;
      fence_acq_rel_gpu();
      count = (np + kFan - 1) / kFan;
      stride = kFan;
    }
    sum_pieces<REGS>(tk, sub, count, [&](int i) { return piece_slot(j0, i * stride); }, red, acc);
    if (0 == warp) Lay::commit(tk, sub, (size_t)key - 1, acc);
    __syncthreads();
  }
}

/* One work item of the stack kernel: CTA group `group` (W = blockDim.x / 32 consecutive chunks of
   L grouped entries) and warp sub-tile `sub` of C (8*MT x 8*NT) of one stack. M_, N_, K_ > 0 make
   the block shape a compile-time constant (every fragment load is then one load at an immediate
   offset from a per-lane base pointer); 0 means runtime. Per warp: DMMA fragments of the next
   k-panel (KP k-steps of 4) are loaded while the current panel runs, the A/B blocks two entries ahead
   are prefetched into L2, and the C sub-tile stays in registers for a whole segment (run of equal
   c); a segment that ends inside the chunk is written back at once. Pieces of segments crossing
   chunk boundaries are merged inside the CTA through shared memory in warp order; only segments that
   cross the CTA's own boundaries leave a CTA-level piece in global scratch for the combine kernel.
   Ends with a CTA barrier, so shared memory can be reused for the next item. */
template <int M_, int N_, int K_, int MT, int NT, int KP>
__device__ __forceinline__ void smm_item(const StackTask& tk, int group, int sub, int* __restrict__ seglist,
  double* __restrict__ smem) {
  constexpr int REGS = MT * NT * 2;
  const int m = M_ ? M_ : tk.m, n = N_ ? N_ : tk.n, k = K_ ? K_ : tk.k;
  const double* __restrict__ const A = tk.a;
  const double* __restrict__ const B = tk.b;
  double* __restrict__ const C = tk.c;
  const unsigned* __restrict__ const keys = tk.keys;
  const unsigned long long* __restrict__ const vals = tk.vals;
  const int S = tk.S, L = tk.L, nchunks = tk.nchunks, nsub_n = tk.nsub_n;
  const int W = blockDim.x >> 5;
  double* const sp = smem;                                       /* [W][2][REGS][32] */
  int* const meta = (int*)(smem + (size_t)W * 2 * REGS * 32);    /* [W][4]: head, head_spans, tail, spare */
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int chunk = group * W + warp;
  const int KS = (k + 3) >> 2;
  const int npan = (KS + KP - 1) / KP;
  Tile<MT, NT> tl;
  tl.init(sub, nsub_n, m, n, g);
  const int klim = (k - t + 3) >> 2; /* k-steps in which this lane's k index is inside the block */
  const unsigned a_lane = (unsigned)(t * m + tl.r0 + g), b_lane = (unsigned)(t * n + tl.c0 + g);
  if (0 == lane) {
    meta[warp * 4 + 0] = 0;
    meta[warp * 4 + 1] = 0;
    meta[warp * 4 + 2] = 0;
  }
  __syncwarp();
  if (chunk < nchunks) {
    const int p0 = chunk_first(tk, W, chunk), p1 = chunk_first(tk, W, chunk + 1);
    const bool headcross = (0 < p0) && (keys[p0 - 1] == keys[p0]);
    const bool tailcross = (p1 < S) && (keys[p1 - 1] == keys[p1]);

    double acc[MT][NT][2];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    /* fragments of panel `pan` of the entry with payload v: A(row, 4ks+t) and B(4ks+t, col) */
    auto load = [&](double (&fa)[KP][MT], double (&fb)[KP][NT], unsigned long long v, int pan) {
      const double* const ap = A + ((unsigned)v - 1u + a_lane);
      const double* const bp = B + ((unsigned)(v >> 32) - 1u + b_lane);
#pragma unroll
      for (int p = 0; p < KP; ++p) {
        const int ks = pan * KP + p;
        const bool ok = ks < klim;
#pragma unroll
        for (int i = 0; i < MT; ++i) fa[p][i] = (ok && tl.rok[i]) ? __ldg(ap + 4 * ks * m + 8 * i) : 0.0;
#pragma unroll
        for (int j = 0; j < NT; ++j) fb[p][j] = (ok && tl.cok[j]) ? __ldg(bp + 4 * ks * n + 8 * j) : 0.0;
      }
    };
    auto mma = [&](const double (&fa)[KP][MT], const double (&fb)[KP][NT], int pan) {
#pragma unroll
      for (int p = 0; p < KP; ++p) {
        if (pan * KP + p < KS) {
#pragma unroll
          for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j) dmma_m8n8k4(acc[i][j][0], acc[i][j][1], fa[p][i], fb[p][j]);
        }
      }
    };

    double fa0[KP][MT], fb0[KP][NT], fa1[KP][MT], fb1[KP][NT];
    /* payload pipeline: entry e (cur), e+1 (nxt), e+2 (nn); blocks of e+2 are prefetched into L2 */
    unsigned key_cur = keys[p0];
    unsigned long long v_cur = vals[p0];
    unsigned long long v_nxt = (p0 + 1 < p1) ? vals[p0 + 1] : 0ull;
    unsigned long long v_nn = (p0 + 2 < p1) ? vals[p0 + 2] : 0ull;
    unsigned key_nxt = (p0 + 1 < p1) ? keys[p0 + 1] : 0u;
    int e = p0, pan = 0, segstart = p0;
    load(fa0, fb0, v_cur, 0);
    if (p0 + 1 < p1) {
      prefetch_block_l2(A + ((unsigned)v_nxt - 1u), m * k, lane);
      prefetch_block_l2(B + ((unsigned)(v_nxt >> 32) - 1u), k * n, lane);
    }

    /* One step: prefetch the next panel into (fan, fbn), run the current one from (fac, fbc),
       finish a segment when its last entry is done, advance. Returns false when the chunk is done. */
    auto step = [&](double (&fac)[KP][MT], double (&fbc)[KP][NT], double (&fan)[KP][MT], double (&fbn)[KP][NT]) -> bool {
      const bool last_pan = (pan + 1 == npan);
      const int e2 = last_pan ? e + 1 : e;
      const int pan2 = last_pan ? 0 : pan + 1;
      if (e2 < p1) load(fan, fbn, last_pan ? v_nxt : v_cur, pan2);
      mma(fac, fbc, pan);
      if (last_pan) {
        const bool seg_end = (e + 1 == p1) || (key_nxt != key_cur);
        if (seg_end) {
          const bool crossl = headcross && (segstart == p0);
          const bool crossr = tailcross && (e + 1 == p1);
          if (!crossl && !crossr) {
            commit_tile<MT, NT>(C, (size_t)key_cur - 1, acc, m, n, g, t, tl, tk.alpha);
          }
          else { /* piece: head slot if it continues a segment from the previous chunk, else tail */
            const int slot = crossl ? 0 : 1;
            double* const dst = sp + ((size_t)(warp * 2 + slot) * REGS) * 32 + lane;
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
              for (int j = 0; j < NT; ++j) {
                dst[((i * NT + j) * 2 + 0) * 32] = acc[i][j][0];
                dst[((i * NT + j) * 2 + 1) * 32] = acc[i][j][1];
              }
            if (0 == lane) {
              if (crossl) {
                meta[warp * 4 + 0] = 1;
                meta[warp * 4 + 1] = crossr ? 1 : 0;
              }
              else meta[warp * 4 + 2] = 1;
            }
          }
#pragma unroll
          for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
          segstart = e + 1;
        }
        if (e + 1 < p1) {
          v_cur = v_nxt;
          key_cur = key_nxt;
          if (e + 2 < p1) {
            v_nxt = v_nn;
            key_nxt = keys[e + 2];
            prefetch_block_l2(A + ((unsigned)v_nxt - 1u), m * k, lane);
            prefetch_block_l2(B + ((unsigned)(v_nxt >> 32) - 1u), k * n, lane);
            if (e + 3 < p1) v_nn = vals[e + 3];
          }
        }
      }
      e = e2;
      pan = pan2;
      return e < p1;
    };
    for (;;) {
      if (!step(fa0, fb0, fa1, fb1)) break;
      if (!step(fa1, fb1, fa0, fb0)) break;
    }
  }
  __syncthreads();
  __shared__ int duty[2][6];
  cta_merge<DmmaLayout<MT, NT>>(tk, group, sub, seglist, meta, W,
    [&](int w, int slot) -> const double* { return sp + ((size_t)(w * 2 + slot) * REGS) * 32; }, duty);
  __syncthreads();
  if (nullptr != tk.arrive) finish_segments<DmmaLayout<MT, NT>>(tk, sub, duty, sp);
}

template <int M_, int N_, int K_, int MT, int NT, int KP>
__global__ void __launch_bounds__(128, smm_min_blocks(MT, NT))
  xs_smm_dmma_kernel(const __grid_constant__ StackTask tk, int* __restrict__ seglist, const unsigned* __restrict__ err) {
  extern __shared__ double smem[];
  prefetch_operands(tk);
  pdl_wait();
  pdl_trigger();
  if (0 != *(volatile const unsigned*)err) return; /* the grouping failed: write nothing */
  const int group = blockIdx.x / tk.nsub, sub = blockIdx.x - group * tk.nsub;
  smm_item<M_, N_, K_, MT, NT, KP>(tk, group, sub, seglist, smem);
}

/* ------------------------------------------------- staged stack kernel (bulk copies into shared memory) */

/* Device error word bit: a wait of the staged stack kernel for its bulk copies timed out. */
constexpr unsigned kErrStagedTimeout = 16u;

/* Geometry of the staged kernel for an M_ x N_ x K_ block shape whose whole C block is one warp tile
   (MT = ceil(M_/8), NT = ceil(N_/8), both <= 4). A stage holds the 16-byte-aligned windows around one
   A block and one B block as the bulk copies bring them (a block that starts 8 bytes past a 16-byte
   boundary is copied from that boundary, so a window is at most 8 bytes longer than its block). Per
   warp: a ring of R stages, reused for the warp's two partial tiles once the ring is drained; then R
   mbarriers per warp and the merge metadata [W][4]. */
template <int M_, int N_, int K_>
struct Staged {
  static constexpr int MT = (M_ + 7) / 8, NT = (N_ + 7) / 8, REGS = MT * NT * 2, KS = (K_ + 3) / 4;
  static constexpr int SA = (M_ * K_ * 8 + 8 + 15) / 16 * 16;
  static constexpr int SB = (K_ * N_ * 8 + 8 + 15) / 16 * 16;
  static constexpr int STAGE = SA + SB;
  static constexpr int PIECES = 2 * REGS * 32 * (int)sizeof(double);
  /* k-index of lane t (t = lane % 4) in DMMA step s. The four k-indices of a step may be any four
     indices of the block as long as A and B use the same ones, so they are chosen to spread the
     warp's shared-memory fragment reads over all banks: lanes t = 0..3 read columns kk(s, t) of A
     (rows of B), ld = M_ (N_) doubles apart. With stride Q between them (kk = base + Q*t) the columns
     start Q*M_*8 bytes apart; when Q*M_ mod 16 is 4 or 12 (in doubles) the four 4-lane groups of a
     half-warp land on four disjoint sets of banks. Full groups of 4*Q indices use stride Q; the
     remainder uses Q too when that costs no extra step, else stride 1. */
  static constexpr bool spread_one(int q, int ld) { return (q * ld) % 16 == 4 || (q * ld) % 16 == 12; }
  static constexpr bool spread(int q) { return spread_one(q, M_) && spread_one(q, N_); }
  /* a stride that spreads both operands, else one that spreads A (the larger share of the loads
     when m >= n), else B */
  static constexpr int Q = spread(1) ? 1 : spread(2) ? 2 : spread(4) ? 4
                         : spread_one(1, M_) ? 1 : spread_one(2, M_) ? 2 : spread_one(4, M_) ? 4
                         : spread_one(1, N_) ? 1 : spread_one(2, N_) ? 2 : spread_one(4, N_) ? 4 : 1;
  static constexpr int GQ = (K_ / (4 * Q)) * Q; /* steps in full groups */
  static constexpr int RS = KS - GQ;             /* remainder steps */
  static constexpr int QR = (RS == Q) ? Q : 1;
  __device__ static __forceinline__ int kidx(int s, int t) {
    return (s < GQ) ? 4 * Q * (s / Q) + (s % Q) + Q * t
                    : 4 * GQ + ((1 == QR) ? 4 * (s - GQ) + t : (s - GQ) + QR * t);
  }
  __host__ __device__ static constexpr int warp_bytes(int R) { return (R * STAGE > PIECES) ? R * STAGE : PIECES; }
  /* + 256 bytes of slack: fragment reads of padding rows / columns may pass the last stage by up to
     8 * MT - M_ (8 * NT - N_) doubles */
  __host__ __device__ static constexpr size_t smem_bytes(int W, int R) {
    return (size_t)W * warp_bytes(R) + (size_t)W * R * sizeof(uint64_t) + (size_t)W * 4 * sizeof(int) + 256;
  }
};

/* Waits (bounded, ignoring the abort word) for a stage whose copies were issued, so that no copy
   still lands in shared memory after the warp gave up. */
__device__ __forceinline__ void drain_stage(uint64_t* bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!xs_tc::mbar_try_wait(bar, parity) && clock64() - t0 < 400000000ll) {
  }
}

/* The staged stack kernel: the same chunks, segments, pieces and CTA merge as the register kernel,
   but lane 0 of each warp streams the A and B blocks of the next R-1 entries of its chunk into the
   warp's shared-memory ring with bulk copies (cp.async.bulk, completion counted in bytes on one
   mbarrier per stage), and the tensor pipe takes every DMMA fragment from shared memory. The L2
   latency is then hidden behind whole entries instead of one k-panel, and no registers hold data in
   flight. The entries' keys and payloads sit in registers (lane j holds entries j and 32 + j of the
   current window) and are broadcast with shuffles. For block shapes whose C block is one warp tile.
   Every wait is bounded: a copy that does not land in time sets the grouping error word (the
   combine then writes nothing) and a device error bit, and the warp stops once the copies it has in
   flight have landed (again bounded).

   One CTA group `group` (W = blockDim.x / 32 chunks) of that kernel, so that a persistent kernel can
   run several: rings = W rings of warp_bytes(R) bytes; bars = W x R mbarriers (count 1) initialised
   before the first item; phase = bit q: parity of the next phase of this warp's barrier q, carried
   from item to item; meta [W][4], s_probe[2], duty[2][6] in shared memory. Returns false (uniformly
   over the CTA) when a copy did not land in time, with no copy left in flight. Contains CTA barriers;
   the caller separates consecutive items by one. */
template <int M_, int N_, int K_, int R>
__device__ __forceinline__ bool staged_item(const StackTask& tk, int group, int* __restrict__ seglist, unsigned* __restrict__ err,
  long long wait_limit, unsigned char* rings, uint64_t* bars, int* meta, unsigned& phase, int* s_probe, int (*duty)[6]) {
  using G = Staged<M_, N_, K_>;
  constexpr int MT = G::MT, NT = G::NT, REGS = G::REGS, KS = G::KS;
  constexpr unsigned FULL = 0xFFFFFFFFu;
  const int W = blockDim.x >> 5;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  unsigned char* const ring = rings + (size_t)warp * G::warp_bytes(R);
  uint64_t* const bar = bars + warp * R;
  if (0 == lane) {
    meta[warp * 4 + 0] = 0;
    meta[warp * 4 + 1] = 0;
    meta[warp * 4 + 2] = 0;
  }
  __syncwarp();
  const double* __restrict__ const A = tk.a;
  const double* __restrict__ const B = tk.b;
  const unsigned* __restrict__ const keys = tk.keys;
  const unsigned long long* __restrict__ const vals = tk.vals;
  const int S = tk.S, L = tk.L;
  const int chunk = group * W + warp;
  Tile<MT, NT> tl;
  tl.init(0, 1, M_, N_, g);
  /* per-lane fragment offsets (doubles): full k groups (stride Q), remainder steps (stride QR) */
  const int lane_af = g + G::Q * M_ * t, lane_bf = g + G::Q * N_ * t;
  const int lane_ar = g + G::QR * M_ * t, lane_br = g + G::QR * N_ * t;
  double acc[MT][NT][2], hacc[MT][NT][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = hacc[i][j][0] = hacc[i][j][1] = 0.0;
  int head = 0, hspans = 0, tail = 0;
  bool bad = false;
  if (chunk < tk.nchunks) {
    const int p0 = chunk_first(tk, W, chunk), p1 = chunk_first(tk, W, chunk + 1);
    const bool headcross = (0 < p0) && (keys[p0 - 1] == keys[p0]);
    const bool tailcross = (p1 < S) && (keys[p1 - 1] == keys[p1]);
    int wb = p0; /* first entry of the current window */
    unsigned kc = 0u, kn = 0u;
    unsigned long long vc = 0ull, vn = 0ull;
    if (p0 + lane < p1) {
      kc = keys[p0 + lane];
      vc = vals[p0 + lane];
    }
    if (p0 + 32 + lane < p1) {
      kn = keys[p0 + 32 + lane];
      vn = vals[p0 + 32 + lane];
    }
    { /* the C blocks of the segments that start in the first 64 entries go to L2 now, so that their
         read-modify-write at the segment's end hits L2 */
      const unsigned pc = __shfl_up_sync(FULL, kc, 1), pn = __shfl_up_sync(FULL, kn, 1), c31 = __shfl_sync(FULL, kc, 31);
      if (p0 + lane < p1 && (0 == lane || pc != kc)) prefetch_block(tk.c + (kc - 1u), (uint32_t)(M_ * N_ * 8));
      if (p0 + 32 + lane < p1 && ((0 == lane) ? c31 : pn) != kn) prefetch_block(tk.c + (kn - 1u), (uint32_t)(M_ * N_ * 8));
    }
    auto key_of = [&](int e) -> unsigned { /* e - wb in [0, 64) */
      const int i = e - wb;
      const unsigned x0 = __shfl_sync(FULL, kc, i & 31), x1 = __shfl_sync(FULL, kn, i & 31);
      return (i < 32) ? x0 : x1;
    };
    auto val_of = [&](int e) -> unsigned long long {
      const int i = e - wb;
      const unsigned long long x0 = __shfl_sync(FULL, vc, i & 31), x1 = __shfl_sync(FULL, vn, i & 31);
      return (i < 32) ? x0 : x1;
    };
    /* lane 0: bulk copies of entry e's A and B windows into stage (e - p0) % R */
    auto issue = [&](int e, unsigned long long v) {
      if (0 == lane) {
        unsigned char* const dst = ring + ((e - p0) % R) * G::STAGE;
        const uintptr_t as = (uintptr_t)(A + ((unsigned)v - 1u)), bs = (uintptr_t)(B + ((unsigned)(v >> 32) - 1u));
        const uintptr_t a0 = as & ~(uintptr_t)15, a1 = (as + (uintptr_t)M_ * K_ * 8 + 15) & ~(uintptr_t)15;
        const uintptr_t b0 = bs & ~(uintptr_t)15, b1 = (bs + (uintptr_t)K_ * N_ * 8 + 15) & ~(uintptr_t)15;
        uint64_t* const sb = &bar[(e - p0) % R];
        xs_tc::mbar_arrive_expect_tx(sb, (uint32_t)((a1 - a0) + (b1 - b0)));
        xs_tc::bulk_load(dst, (const void*)a0, (uint32_t)(a1 - a0), sb);
        xs_tc::bulk_load(dst + G::SA, (const void*)b0, (uint32_t)(b1 - b0), sb);
      }
    };
    for (int q = 0; q < R - 1 && p0 + q < p1; ++q) issue(p0 + q, val_of(p0 + q));
    if (0 == warp && nullptr != tk.arrive) probe_boundaries(tk, W, group, s_probe);
    int issued = min(R - 1, p1 - p0), segstart = p0, e = p0;
    unsigned key_cur = key_of(p0);
    for (; e < p1; ++e) {
      if (e - wb == 32) { /* next window of entry info (its loads have 32 - R entries to land) */
        wb += 32;
        kc = kn;
        vc = vn;
        kn = 0u;
        vn = 0ull;
        if (wb + 32 + lane < p1) {
          kn = keys[wb + 32 + lane];
          vn = vals[wb + 32 + lane];
        }
      }
      if (e + R - 1 < p1) { /* refill the stage that entry e - 1 used */
        issue(e + R - 1, val_of(e + R - 1));
        ++issued;
      }
      const unsigned long long v = val_of(e);
      const int st = (e - p0) % R;
      const bool ok =
        __all_sync(FULL, xs_tc::mbar_wait(&bar[st], (((phase >> st) & 1u) + (uint32_t)((e - p0) / R)) & 1u, err, 2u, wait_limit) ? 1 : 0);
      if (!ok) {
        bad = true;
        break;
      }
      const double* const sA = (const double*)(ring + st * G::STAGE) + (((uintptr_t)(A + ((unsigned)v - 1u)) >> 3) & 1u);
      const double* const sB =
        (const double*)(ring + st * G::STAGE + G::SA) + (((uintptr_t)(B + ((unsigned)(v >> 32) - 1u)) >> 3) & 1u);
      /* fragments: lane (g, t) reads A(8i + g, kidx(ks, t)) and B(kidx(ks, t), 8j + g). Rows beyond
         m and columns beyond n read whatever follows in shared memory (the stage, the next one, or
         the slack after the last): they only reach C entries that are never written back. k indices
         beyond k occur only in the remainder steps, where both fragments are zeroed. */
#pragma unroll
      for (int ks = 0; ks < KS; ++ks) {
        double fa[MT], fb[NT];
        if (ks < G::GQ) { /* full groups: kidx = kc + Q*t, always inside the block */
          constexpr int Q = G::Q;
          const int kc = 4 * Q * (ks / Q) + ks % Q;
#pragma unroll
          for (int i = 0; i < MT; ++i) fa[i] = sA[lane_af + kc * M_ + 8 * i];
#pragma unroll
          for (int j = 0; j < NT; ++j) fb[j] = sB[lane_bf + kc * N_ + 8 * j];
        }
        else {
          constexpr int QR = G::QR;
          const int kc = 4 * G::GQ + ((1 == QR) ? 4 * (ks - G::GQ) : (ks - G::GQ));
          const bool kin = kc + QR * t < K_;
#pragma unroll
          for (int i = 0; i < MT; ++i) fa[i] = kin ? sA[lane_ar + kc * M_ + 8 * i] : 0.0;
#pragma unroll
          for (int j = 0; j < NT; ++j) fb[j] = kin ? sB[lane_br + kc * N_ + 8 * j] : 0.0;
        }
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) dmma_m8n8k4(acc[i][j][0], acc[i][j][1], fa[i], fb[j]);
      }
      const bool last = (e + 1 == p1);
      const unsigned key_nxt = key_of(last ? e : e + 1);
      if (last || key_nxt != key_cur) { /* the segment ends with entry e */
        const bool crossl = headcross && (segstart == p0);
        const bool crossr = tailcross && last;
        if (!crossl && !crossr) commit_tile<MT, NT>(tk.c, (size_t)key_cur - 1, acc, M_, N_, g, t, tl, tk.alpha);
        else if (!crossr) { /* continues a segment of the previous chunk: head piece */
#pragma unroll
          for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j) {
              hacc[i][j][0] = acc[i][j][0];
              hacc[i][j][1] = acc[i][j][1];
            }
          head = 1;
        }
        else if (crossl) { /* the whole chunk is one segment crossing both ends */
          head = 1;
          hspans = 1;
        }
        else tail = 1;
        if (!crossr) {
#pragma unroll
          for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
        }
        segstart = e + 1;
      }
      key_cur = key_nxt;
      __syncwarp();
    }
    if (bad) { /* entries e .. issued - 1 have copies in flight */
      for (int q = e - p0; q < issued; ++q) drain_stage(&bar[q % R], (((phase >> (q % R)) & 1u) + (uint32_t)(q / R)) & 1u);
    }
    else { /* stage q completed ceil((n - q) / R) phases in this item */
      const int n = p1 - p0;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        if (q < n && 0 != (((n - q + R - 1) / R) & 1)) phase ^= 1u << q;
      }
    }
  }
  __syncwarp();
  if (!bad) { /* the ring is drained: the warp's pieces go to its own region */
    double* const sp = (double*)ring; /* [2][REGS][32] */
    if (head) {
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          sp[((i * NT + j) * 2 + 0) * 32 + lane] = hspans ? acc[i][j][0] : hacc[i][j][0];
          sp[((i * NT + j) * 2 + 1) * 32 + lane] = hspans ? acc[i][j][1] : hacc[i][j][1];
        }
    }
    if (tail) {
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          sp[(REGS + (i * NT + j) * 2 + 0) * 32 + lane] = acc[i][j][0];
          sp[(REGS + (i * NT + j) * 2 + 1) * 32 + lane] = acc[i][j][1];
        }
    }
    if (0 == lane) {
      meta[warp * 4 + 0] = head;
      meta[warp * 4 + 1] = hspans;
      meta[warp * 4 + 2] = tail;
    }
  }
  if (__syncthreads_or(bad ? 1 : 0)) return false;
  cta_merge<DmmaLayout<MT, NT>>(tk, group, 0, seglist, meta, W, [&](int w, int slot) -> const double* {
    return (const double*)(rings + (size_t)w * G::warp_bytes(R)) + (size_t)slot * REGS * 32;
  }, duty, (nullptr != tk.arrive && group * W < tk.nchunks) ? s_probe : nullptr);
  if (nullptr != tk.arrive) {
    __syncthreads();
    finish_segments<DmmaLayout<MT, NT>>(tk, 0, duty, (double*)rings);
  }
  return true;
}

/* The staged stack kernel: one CTA group per CTA (see staged_item). */
template <int M_, int N_, int K_, int R>
__global__ void __launch_bounds__(128, smm_min_blocks((M_ + 7) / 8, (N_ + 7) / 8))
  xs_smm_staged_kernel(const __grid_constant__ StackTask tk, int* __restrict__ seglist, unsigned* __restrict__ err,
    unsigned* __restrict__ dev_err, long long wait_limit) {
  using G = Staged<M_, N_, K_>;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ int s_probe[2];
  __shared__ int duty[2][6];
  prefetch_operands(tk);
  pdl_wait();
  pdl_trigger();
  if (0 != *(volatile const unsigned*)err) return;
  const int W = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t* const bars = (uint64_t*)(smraw + (size_t)W * G::warp_bytes(R));
  int* const meta = (int*)(smraw + (size_t)W * G::warp_bytes(R) + (size_t)W * R * sizeof(uint64_t));
  if (0 == lane) {
#pragma unroll
    for (int q = 0; q < R; ++q) xs_tc::mbar_init(&bars[warp * R + q], 1);
    xs_tc::fence_barrier_init();
  }
  __syncwarp();
  unsigned phase = 0u;
  if (!staged_item<M_, N_, K_, R>(tk, blockIdx.x, seglist, err, wait_limit, smraw, bars, meta, phase, s_probe, duty)) {
    if (0 == threadIdx.x && nullptr != dev_err) atomicOr(dev_err, kErrStagedTimeout);
  }
}

/* ------------------------------------ warp-specialised staged stack kernel (one producer warp) */

/* Shared memory of the warp-specialised kernel: NC rings of R stages (Staged geometry), then a full
   and an empty mbarrier per stage, the merge metadata [NC][4] and 256 bytes of slack. */
template <int M_, int N_, int K_>
__host__ __device__ constexpr size_t ws_smem_bytes(int NC, int R) {
  return (size_t)NC * Staged<M_, N_, K_>::warp_bytes(R) + (size_t)2 * NC * R * sizeof(uint64_t) + (size_t)NC * 4 * sizeof(int) + 256;
}

/* The staged stack kernel with its copies taken off the compute warps: a CTA of NC consumer warps
   (one chunk of L grouped entries each, the same segments, pieces and merge as the staged kernel)
   and one producer warp, whose lane w streams the A and B blocks of consumer w's entries into w's
   ring of R stages (cp.async.bulk of the 16-byte-aligned windows, completion counted in bytes on the
   stage's full barrier) as soon as w releases a stage (one arrival on its empty barrier). A consumer
   only waits for its stage, runs the DMMAs from shared memory and releases it; the producer keeps
   the next entry's payload in a register, so an issue never waits for a global load. Every wait is
   bounded: a timed-out wait sets the grouping error word (which the other roles and CTAs poll), the
   producer stops issuing and waits (bounded) for the copies still in flight, and the kernel sets a
   device error bit and returns without writing. */
template <int M_, int N_, int K_, int NC, int R, int MINB>
__global__ void __launch_bounds__(32 * (NC + 1), MINB)
  xs_smm_ws_kernel(const __grid_constant__ StackTask tk, int* __restrict__ seglist, unsigned* __restrict__ err,
    unsigned* __restrict__ dev_err, long long wait_limit) {
  using G = Staged<M_, N_, K_>;
  constexpr int MT = G::MT, NT = G::NT, REGS = G::REGS, KS = G::KS;
  constexpr unsigned FULL = 0xFFFFFFFFu;
  extern __shared__ __align__(128) unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int group = blockIdx.x;
  uint64_t* const fullb = (uint64_t*)(smraw + (size_t)NC * G::warp_bytes(R));
  uint64_t* const emptyb = fullb + NC * R;
  int* const meta = (int*)(emptyb + NC * R); /* [NC][4]: head, head spans the chunk, tail, entries consumed */
  if (warp < NC && 0 == lane) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      xs_tc::mbar_init(&fullb[warp * R + q], 1);
      xs_tc::mbar_init(&emptyb[warp * R + q], 1);
    }
    xs_tc::fence_barrier_init();
    meta[warp * 4 + 0] = 0;
    meta[warp * 4 + 1] = 0;
    meta[warp * 4 + 2] = 0;
    meta[warp * 4 + 3] = 0;
  }
  prefetch_operands(tk);
  pdl_wait();
  pdl_trigger();
  if (__syncthreads_or((0 != *(volatile const unsigned*)err) ? 1 : 0)) return; /* the grouping failed: write nothing */
  const double* __restrict__ const A = tk.a;
  const double* __restrict__ const B = tk.b;
  const unsigned* __restrict__ const keys = tk.keys;
  const unsigned long long* __restrict__ const vals = tk.vals;
  const int S = tk.S, L = tk.L;
  bool bad = false;
  int issued = 0; /* producer lane w: entries of chunk w whose copies were issued */
  if (NC == warp) { /* ------------------------------------------------------------- producer */
    const int chunk = group * NC + lane;
    const int p0 = (lane < NC && chunk < tk.nchunks) ? chunk_first(tk, NC, chunk) : 0;
    const int n = (lane < NC && chunk < tk.nchunks) ? chunk_first(tk, NC, chunk + 1) - p0 : 0;
    unsigned char* const ring = smraw + (size_t)lane * G::warp_bytes(R);
    unsigned long long vnext = (0 < n) ? vals[p0] : 0ull;
    long long t_prog = clock64();
    while (__any_sync(FULL, issued < n)) {
      bool ready = false;
      if (issued < n) {
        ready = (issued < R) || xs_tc::mbar_test_wait(&emptyb[lane * R + issued % R], (uint32_t)((issued / R - 1) & 1));
      }
      if (ready) {
        const unsigned long long v = vnext;
        if (issued + 1 < n) vnext = vals[p0 + issued + 1];
        const int st = issued % R;
        unsigned char* const dst = ring + st * G::STAGE;
        const uintptr_t as = (uintptr_t)(A + ((unsigned)v - 1u)), bs = (uintptr_t)(B + ((unsigned)(v >> 32) - 1u));
        const uintptr_t a0 = as & ~(uintptr_t)15, a1 = (as + (uintptr_t)M_ * K_ * 8 + 15) & ~(uintptr_t)15;
        const uintptr_t b0 = bs & ~(uintptr_t)15, b1 = (bs + (uintptr_t)K_ * N_ * 8 + 15) & ~(uintptr_t)15;
        uint64_t* const sb = &fullb[lane * R + st];
        xs_tc::mbar_arrive_expect_tx(sb, (uint32_t)((a1 - a0) + (b1 - b0)));
        xs_tc::bulk_load(dst, (const void*)a0, (uint32_t)(a1 - a0), sb);
        xs_tc::bulk_load(dst + G::SA, (const void*)b0, (uint32_t)(b1 - b0), sb);
        ++issued;
      }
      if (__any_sync(FULL, ready)) t_prog = clock64();
      else { /* nobody released a stage: back off; give up on an abort or when the bound is passed */
        if (0 != *(volatile const unsigned*)err) break;
        if (clock64() - t_prog > wait_limit) {
          if (0 == lane) atomicOr(err, 2u);
          break;
        }
        __nanosleep(64);
      }
    }
  }
  else { /* ------------------------------------------------------------------------ consumer */
    unsigned char* const ring = smraw + (size_t)warp * G::warp_bytes(R);
    const int chunk = group * NC + warp;
    Tile<MT, NT> tl;
    tl.init(0, 1, M_, N_, g);
    const int lane_af = g + G::Q * M_ * t, lane_bf = g + G::Q * N_ * t;
    const int lane_ar = g + G::QR * M_ * t, lane_br = g + G::QR * N_ * t;
    double acc[MT][NT][2], hacc[MT][NT][2];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = hacc[i][j][0] = hacc[i][j][1] = 0.0;
    int head = 0, hspans = 0, tail = 0, consumed = 0;
    if (chunk < tk.nchunks) {
      const int p0 = chunk_first(tk, NC, chunk), p1 = chunk_first(tk, NC, chunk + 1);
      const bool headcross = (0 < p0) && (keys[p0 - 1] == keys[p0]);
      const bool tailcross = (p1 < S) && (keys[p1 - 1] == keys[p1]);
      int wb = p0;
      unsigned kc = 0u, kn = 0u;
      unsigned long long vc = 0ull, vn = 0ull;
      if (p0 + lane < p1) {
        kc = keys[p0 + lane];
        vc = vals[p0 + lane];
      }
      if (p0 + 32 + lane < p1) {
        kn = keys[p0 + 32 + lane];
        vn = vals[p0 + 32 + lane];
      }
      auto key_of = [&](int e) -> unsigned {
        const int i = e - wb;
        const unsigned x0 = __shfl_sync(FULL, kc, i & 31), x1 = __shfl_sync(FULL, kn, i & 31);
        return (i < 32) ? x0 : x1;
      };
      auto val_of = [&](int e) -> unsigned long long {
        const int i = e - wb;
        const unsigned long long x0 = __shfl_sync(FULL, vc, i & 31), x1 = __shfl_sync(FULL, vn, i & 31);
        return (i < 32) ? x0 : x1;
      };
      int segstart = p0, e = p0;
      unsigned key_cur = key_of(p0);
      for (; e < p1; ++e) {
        if (e - wb == 32) {
          wb += 32;
          kc = kn;
          vc = vn;
          kn = 0u;
          vn = 0ull;
          if (wb + 32 + lane < p1) {
            kn = keys[wb + 32 + lane];
            vn = vals[wb + 32 + lane];
          }
        }
        const unsigned long long v = val_of(e);
        const int st = (e - p0) % R;
        const bool ok =
          __all_sync(FULL, xs_tc::mbar_wait(&fullb[warp * R + st], (uint32_t)(((e - p0) / R) & 1), err, 2u, wait_limit) ? 1 : 0);
        if (!ok) {
          bad = true;
          break;
        }
        const double* const sA = (const double*)(ring + st * G::STAGE) + (((uintptr_t)(A + ((unsigned)v - 1u)) >> 3) & 1u);
        const double* const sB =
          (const double*)(ring + st * G::STAGE + G::SA) + (((uintptr_t)(B + ((unsigned)(v >> 32) - 1u)) >> 3) & 1u);
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
          double fa[MT], fb[NT];
          if (ks < G::GQ) {
            constexpr int Q = G::Q;
            const int kk = 4 * Q * (ks / Q) + ks % Q;
#pragma unroll
            for (int i = 0; i < MT; ++i) fa[i] = sA[lane_af + kk * M_ + 8 * i];
#pragma unroll
            for (int j = 0; j < NT; ++j) fb[j] = sB[lane_bf + kk * N_ + 8 * j];
          }
          else {
            constexpr int QR = G::QR;
            const int kk = 4 * G::GQ + ((1 == QR) ? 4 * (ks - G::GQ) : (ks - G::GQ));
            const bool kin = kk + QR * t < K_;
#pragma unroll
            for (int i = 0; i < MT; ++i) fa[i] = kin ? sA[lane_ar + kk * M_ + 8 * i] : 0.0;
#pragma unroll
            for (int j = 0; j < NT; ++j) fb[j] = kin ? sB[lane_br + kk * N_ + 8 * j] : 0.0;
          }
#pragma unroll
          for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j) dmma_m8n8k4(acc[i][j][0], acc[i][j][1], fa[i], fb[j]);
        }
        __syncwarp(); /* every lane's fragment reads of the stage are done: hand it back */
        if (0 == lane) xs_tc::mbar_arrive(&emptyb[warp * R + st]);
        ++consumed;
        const bool last = (e + 1 == p1);
        const unsigned key_nxt = key_of(last ? e : e + 1);
        if (last || key_nxt != key_cur) {
          const bool crossl = headcross && (segstart == p0);
          const bool crossr = tailcross && last;
          if (!crossl && !crossr) commit_tile<MT, NT>(tk.c, (size_t)key_cur - 1, acc, M_, N_, g, t, tl, tk.alpha);
          else if (!crossr) {
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
              for (int j = 0; j < NT; ++j) {
                hacc[i][j][0] = acc[i][j][0];
                hacc[i][j][1] = acc[i][j][1];
              }
            head = 1;
          }
          else if (crossl) {
            head = 1;
            hspans = 1;
          }
          else tail = 1;
          if (!crossr) {
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
              for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
          }
          segstart = e + 1;
        }
        key_cur = key_nxt;
      }
    }
    __syncwarp();
    if (0 == lane) meta[warp * 4 + 3] = consumed;
    if (!bad) { /* every stage of this warp was consumed, so no copy is in flight: pieces go to its ring */
      double* const sp = (double*)ring;
      if (head) {
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) {
            sp[((i * NT + j) * 2 + 0) * 32 + lane] = hspans ? acc[i][j][0] : hacc[i][j][0];
            sp[((i * NT + j) * 2 + 1) * 32 + lane] = hspans ? acc[i][j][1] : hacc[i][j][1];
          }
      }
      if (tail) {
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) {
            sp[(REGS + (i * NT + j) * 2 + 0) * 32 + lane] = acc[i][j][0];
            sp[(REGS + (i * NT + j) * 2 + 1) * 32 + lane] = acc[i][j][1];
          }
      }
      if (0 == lane) {
        meta[warp * 4 + 0] = head;
        meta[warp * 4 + 1] = hspans;
        meta[warp * 4 + 2] = tail;
      }
    }
  }
  if (__syncthreads_or((bad || (NC == warp && 0 != *(volatile const unsigned*)err)) ? 1 : 0)) {
    /* the producer waits (bounded) for every copy it issued that its consumer did not take */
    if (NC == warp && lane < NC) {
      for (int q = meta[lane * 4 + 3]; q < issued; ++q) drain_stage(&fullb[lane * R + q % R], (uint32_t)((q / R) & 1));
    }
    if (0 == threadIdx.x && nullptr != dev_err) atomicOr(dev_err, kErrStagedTimeout);
    return;
  }
  __shared__ int duty[2][6];
  cta_merge<DmmaLayout<MT, NT>>(tk, group, 0, seglist, meta, NC, [&](int w, int slot) -> const double* {
    return (const double*)(smraw + (size_t)w * G::warp_bytes(R)) + (size_t)slot * REGS * 32;
  }, duty);
  if (nullptr != tk.arrive) {
    __syncthreads();
    finish_segments<DmmaLayout<MT, NT>>(tk, 0, duty, (double*)smraw);
  }
}

/* ------------------------------------------------------ register-blocked FMA stack kernel (small blocks) */

/* C layout of the FMA kernel: the 32 lanes form an LR x LC lane grid (LC = 32 / LR); lane (lr, lc),
   lr = lane % LR, lc = lane / LR, holds the RB x CB elements in rows lr + LR*a (a < RB) and columns
   lc*CB + b (b < CB) of C, element (a, b) at a*CB + b. Consecutive lanes hold consecutive rows, so
   their A loads and C write-backs are contiguous; a lane's columns are contiguous, so its B loads
   are pairs. */
template <int LR, int RB, int CB>
struct FmaLayout {
  static constexpr int LC = 32 / LR;
  static constexpr int REGS = RB * CB;
  __device__ static __forceinline__ void commit(const StackTask& tk, int, size_t coff, const double (&sum)[REGS]) {
    const int lane = threadIdx.x & 31, lr = lane % LR, lc = lane / LR, m = tk.m, n = tk.n;
#pragma unroll
    for (int a = 0; a < RB; ++a) {
      const int row = lr + LR * a;
      if (row < m) {
#pragma unroll
        for (int b = 0; b < CB; ++b) {
          const int col = lc * CB + b;
          if (col < n) atomicAdd(tk.c + coff + (size_t)col * m + row, tk.alpha * sum[a * CB + b]);
        }
      }
    }
  }
};

/* Shared memory of the FMA kernel, in doubles per warp: a ring of D stages, each the entry's A block
   (m*k, column-major) rounded up to an even count followed by its B block (k*n, row-major); 32 doubles
   of slack (reads of padding rows and columns pass the last stage by less than the slack); the head
   piece [REGS][32]. The tail piece reuses the ring once it is drained. Then the merge metadata. The
   slack is the lane grid's column count rounded up to even: a lane's B reads pass the end of a row
   of n by at most LC*CB - n doubles. */
__host__ __device__ constexpr int fma_stage(int m, int n, int k) { return ((m * k + 1) / 2 * 2 + k * n + 1) / 2 * 2; }
__host__ __device__ constexpr int fma_ring(int m, int n, int k, int D, int regs, int slack) {
  return (D * fma_stage(m, n, k) + slack > regs * 32) ? D * fma_stage(m, n, k) + slack : regs * 32;
}
__host__ __device__ constexpr size_t fma_smem_bytes(int m, int n, int k, int D, int regs, int slack, int W) {
  return (size_t)W * (fma_ring(m, n, k, D, regs, slack) + regs * 32) * sizeof(double) + (size_t)W * 4 * sizeof(int);
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(xs_tc::smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

/* The FMA stack kernel: the chunks, segments, pieces and merge of the other stack kernels, with C held
   as FmaLayout<LR, RB, CB> register blocks and plain FP64 FMAs instead of padded DMMA tiles, so a
   small or odd block (4^3, 5^3, 6x6x18, 13x4x16, 32x9x9, 16x64x9) issues no padding work. Each warp
   streams the A and B blocks of the next D - 1 entries of its chunk into its ring with 8-byte
   cp.async copies (lane l copies elements l, l + 32, ... of the entry's A | B window, one commit
   group per entry), so D - 1 entries are in flight per warp without holding registers. Per k index a
   lane reads RB values of A (a column of A: the lanes of one lane-grid column read consecutive rows)
   and CB of B (one row of B, in pairs when the row length is even) and issues RB*CB FMAs. M_, N_, K_
   > 0 fix the block shape at compile time; 0 means runtime (m <= LR*RB, n <= LC*CB). */
template <int M_, int N_, int K_, int LR, int RB, int CB, int D>
__global__ void __launch_bounds__(128, 2)
  xs_smm_fma_kernel(const __grid_constant__ StackTask tk, int* __restrict__ seglist, const unsigned* __restrict__ err) {
  using Lay = FmaLayout<LR, RB, CB>;
  constexpr int REGS = Lay::REGS, SLACK = (Lay::LC * CB + 1) / 2 * 2;
  constexpr unsigned FULL = 0xFFFFFFFFu;
  extern __shared__ __align__(16) double fsm[];
  __shared__ int s_probe[2];
  prefetch_operands(tk);
  pdl_wait();
  pdl_trigger();
  if (__syncthreads_or((0 != *(volatile const unsigned*)err) ? 1 : 0)) return;
  const int m = M_ ? M_ : tk.m, n = N_ ? N_ : tk.n, k = K_ ? K_ : tk.k;
  const int W = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lr = lane % LR, lc = lane / LR;
  const int stage = fma_stage(m, n, k), sa = (m * k + 1) / 2 * 2, mk = m * k, tot = m * k + k * n;
  const int region = fma_ring(m, n, k, D, REGS, SLACK) + REGS * 32;
  double* const ring = fsm + (size_t)warp * region;
  double* const hpiece = ring + fma_ring(m, n, k, D, REGS, SLACK);
  int* const meta = (int*)(fsm + (size_t)W * region);
  if (0 == lane) {
    meta[warp * 4 + 0] = 0;
    meta[warp * 4 + 1] = 0;
    meta[warp * 4 + 2] = 0;
  }
  const double* __restrict__ const A = tk.a;
  const double* __restrict__ const B = tk.b;
  const unsigned* __restrict__ const keys = tk.keys;
  const unsigned long long* __restrict__ const vals = tk.vals;
  const int S = tk.S, L = tk.L;
  const int chunk = blockIdx.x * W + warp;
  double acc[REGS];
#pragma unroll
  for (int r = 0; r < REGS; ++r) acc[r] = 0.0;
  int head = 0, hspans = 0, tail = 0;
  if (chunk < tk.nchunks) {
    const int p0 = chunk_first(tk, W, chunk), p1 = chunk_first(tk, W, chunk + 1);
    const bool headcross = (0 < p0) && (keys[p0 - 1] == keys[p0]);
    const bool tailcross = (p1 < S) && (keys[p1 - 1] == keys[p1]);
    int wb = p0;
    unsigned kc = 0u, kn = 0u;
    unsigned long long vc = 0ull, vn = 0ull;
    if (p0 + lane < p1) {
      kc = keys[p0 + lane];
      vc = vals[p0 + lane];
    }
    if (p0 + 32 + lane < p1) {
      kn = keys[p0 + 32 + lane];
      vn = vals[p0 + 32 + lane];
    }
    auto key_of = [&](int e) -> unsigned {
      const int i = e - wb;
      const unsigned x0 = __shfl_sync(FULL, kc, i & 31), x1 = __shfl_sync(FULL, kn, i & 31);
      return (i < 32) ? x0 : x1;
    };
    auto val_of = [&](int e) -> unsigned long long {
      const int i = e - wb;
      const unsigned long long x0 = __shfl_sync(FULL, vc, i & 31), x1 = __shfl_sync(FULL, vn, i & 31);
      return (i < 32) ? x0 : x1;
    };
    /* copies of entry e's A | B window into its stage: lane l takes elements l, l + 32, ... */
    auto issue = [&](int e, unsigned long long v) {
      double* const dst = ring + ((e - p0) % D) * stage;
      const double* const as = A + ((unsigned)v - 1u);
      const double* const bs = B + ((unsigned)(v >> 32) - 1u);
      for (int x = lane; x < tot; x += 32) {
        if (x < mk) cp_async8(dst + x, as + x);
        else cp_async8(dst + sa + (x - mk), bs + (x - mk));
      }
    };
    for (int q = 0; q < D - 1; ++q) {
      if (p0 + q < p1) issue(p0 + q, val_of(p0 + q));
      cp_async_commit();
    }
    if (0 == warp) probe_boundaries(tk, W, blockIdx.x, s_probe);
    int segstart = p0;
    unsigned key_cur = key_of(p0);
    for (int e = p0; e < p1; ++e) {
      if (e - wb == 32) {
        wb += 32;
        kc = kn;
        vc = vn;
        kn = 0u;
        vn = 0ull;
        if (wb + 32 + lane < p1) {
          kn = keys[wb + 32 + lane];
          vn = vals[wb + 32 + lane];
        }
      }
      cp_async_wait<D - 2>(); /* entry e's group has landed (this lane's copies) */
      __syncwarp();           /* ... and every lane's; all lanes are done with entry e - 1's stage */
      if (e + D - 1 < p1) issue(e + D - 1, val_of(e + D - 1));
      cp_async_commit();
      const double* const sA = ring + ((e - p0) % D) * stage;
      const double* const sB = sA + sa;
      auto fma_k = [&](int kk) {
        double fa[RB], fb[CB];
#pragma unroll
        for (int a = 0; a < RB; ++a) fa[a] = sA[kk * m + lr + LR * a];
        const double* const brow = sB + kk * n + lc * CB;
        if (0 == (CB & 1) && 0 == (n & 1)) { /* 16-byte aligned pairs: the stage and B part start even */
#pragma unroll
          for (int b = 0; b < CB; b += 2) {
            const double2 x = *(const double2*)(brow + b);
            fb[b] = x.x;
            fb[b + 1] = x.y;
          }
        }
        else {
#pragma unroll
          for (int b = 0; b < CB; ++b) fb[b] = brow[b];
        }
#pragma unroll
        for (int a = 0; a < RB; ++a)
#pragma unroll
          for (int b = 0; b < CB; ++b) acc[a * CB + b] = fma(fa[a], fb[b], acc[a * CB + b]);
      };
      if (0 < K_) {
#pragma unroll
        for (int kk = 0; kk < K_; ++kk) fma_k(kk);
      }
      else {
        for (int kk = 0; kk < k; ++kk) fma_k(kk);
      }
      const bool last = (e + 1 == p1);
      const unsigned key_nxt = key_of(last ? e : e + 1);
      if (last || key_nxt != key_cur) { /* the segment ends with entry e */
        const bool crossl = headcross && (segstart == p0);
        const bool crossr = tailcross && last;
        if (!crossl && !crossr) Lay::commit(tk, 0, (size_t)key_cur - 1, acc);
        else if (!crossr) { /* continues the previous chunk's segment: head piece */
#pragma unroll
          for (int r = 0; r < REGS; ++r) hpiece[r * 32 + lane] = acc[r];
          head = 1;
        }
        else if (crossl) { /* the whole chunk is one segment crossing both ends */
          head = 1;
          hspans = 1;
        }
        else tail = 1;
        if (!crossr) {
#pragma unroll
          for (int r = 0; r < REGS; ++r) acc[r] = 0.0;
        }
        segstart = e + 1;
      }
      key_cur = key_nxt;
    }
  }
  cp_async_wait<0>();
  __syncwarp();
  if (hspans) {
#pragma unroll
    for (int r = 0; r < REGS; ++r) hpiece[r * 32 + lane] = acc[r];
  }
  if (tail) { /* the ring is drained: the tail piece goes to its start */
#pragma unroll
    for (int r = 0; r < REGS; ++r) ring[r * 32 + lane] = acc[r];
  }
  if (0 == lane) {
    meta[warp * 4 + 0] = head;
    meta[warp * 4 + 1] = hspans;
    meta[warp * 4 + 2] = tail;
  }
  __syncthreads();
  __shared__ int duty[2][6];
  cta_merge<Lay>(tk, blockIdx.x, 0, seglist, meta, W, [&](int w, int slot) -> const double* {
    const double* const base = fsm + (size_t)w * region;
    return (0 == slot) ? base + fma_ring(m, n, k, D, REGS, SLACK) : base;
  }, duty, s_probe);
  __syncthreads();
  finish_segments<Lay>(tk, 0, duty, fsm);
}

/* Task table of a batch (kernel parameter: read through the constant bank). */
constexpr int kMaxBatchTasks = 32;
struct BatchTasks {
  int ntasks, nitems;
  StackTask t[kMaxBatchTasks];
};

/* Register groups of the tile classes: group 0 holds the classes with MT*NT <= 9 fragments (168
   registers: the unified batch kernel runs them), group 1 the larger ones. */
__host__ __device__ constexpr int batch_group(int mt, int nt) { return (mt * nt <= 9) ? 0 : 1; }
/* k-steps per register panel: 4 for small tiles, 2 for mid-size, 1 for the largest (whose
   accumulators alone take 48-64 registers) */
__host__ __device__ constexpr int batch_kp(int mt, int nt) { return (mt * nt <= 4) ? 4 : ((mt * nt < 12) ? 2 : 1); }

/* One tile class of the register kernel as a separate (not inlined) function of the unified batch
   kernel, so that each class gets its own register allocation instead of sharing one with the other
   classes' code. */
template <int MT, int NT>
__device__ __noinline__ void batch_item(const StackTask& tk, int group, int sub, int* seglist, double* smem) {
  smm_item<0, 0, 0, MT, NT, batch_kp(MT, NT)>(tk, group, sub, seglist, smem);
}

template <int GRP, int MT, int NT>
__device__ __forceinline__ void batch_dispatch(int cls, const StackTask& tk, int group, int sub, int* seglist, double* smem) {
  if constexpr (batch_group(MT, NT) == GRP) {
    if ((MT - 1) * 4 + (NT - 1) == cls) batch_item<MT, NT>(tk, group, sub, seglist, smem);
  }
}

/* Sum the pieces of one CTA-crossing segment for one sub-tile in a fixed order and write the block
   once. The segment starts in CTA group j0 (its tail piece) and continues through the head pieces of
   the following groups while their first entry still belongs to it; all threads of the CTA find that
   count in one parallel probe of group-start keys, then its warps sum the pieces round-robin (warp w
   takes pieces w, w+CW, ...) and warp 0 adds the warp partials in warp order: the summation tree
   depends only on the number of pieces, so the result is deterministic. */
template <int MT, int NT>
__device__ __forceinline__ void combine_one(const StackTask& tk, int W, int j0, int sub, double* __restrict__ red) {
  constexpr int REGS = MT * NT * 2;
  constexpr int CW = kCombineWarps;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const unsigned* __restrict__ const keys = tk.keys;
  const double* __restrict__ const pieces = tk.pieces;
  const int ngroups = tk.ngroups, nsub = tk.nsub;
  const unsigned xkey = keys[chunk_first(tk, W, (j0 + 1) * W) - 1];
  /* pieces = 1 + number of following groups that start inside the segment (a prefix, keys sorted) */
  int np = 1;
  for (int base = j0 + 1;; base += blockDim.x) {
    const int j = base + (int)threadIdx.x;
    const int inside = (j < ngroups) && (keys[(size_t)chunk_first(tk, W, j * W)] == xkey);
    const int cnt = __syncthreads_count(inside);
    np += cnt;
    if (cnt < (int)blockDim.x) break;
  }
  double acc[REGS];
#pragma unroll
  for (int r = 0; r < REGS; ++r) acc[r] = 0.0;
  int q = warp;
  for (; q + CW < np; q += 2 * CW) { /* two pieces in flight per step */
    const int s0 = (0 == q) ? 2 * j0 + 1 : 2 * (j0 + q), s1 = 2 * (j0 + q + CW);
    const double* const p0 = pieces + ((size_t)s0 * nsub + sub) * REGS * 32 + lane;
    const double* const p1 = pieces + ((size_t)s1 * nsub + sub) * REGS * 32 + lane;
    double v0[REGS], v1[REGS];
#pragma unroll
    for (int r = 0; r < REGS; ++r) {
      v0[r] = p0[r * 32];
      v1[r] = p1[r * 32];
    }
#pragma unroll
    for (int r = 0; r < REGS; ++r) acc[r] += v0[r];
#pragma unroll
    for (int r = 0; r < REGS; ++r) acc[r] += v1[r];
  }
  if (q < np) {
    const int s0 = (0 == q) ? 2 * j0 + 1 : 2 * (j0 + q);
    const double* const p0 = pieces + ((size_t)s0 * nsub + sub) * REGS * 32 + lane;
#pragma unroll
    for (int r = 0; r < REGS; ++r) acc[r] += p0[r * 32];
  }
  if (0 != warp) {
#pragma unroll
    for (int r = 0; r < REGS; ++r) red[((warp - 1) * REGS + r) * 32 + lane] = acc[r];
  }
  __syncthreads();
  if (0 == warp) {
    for (int w2 = 0; w2 < CW - 1; ++w2) {
#pragma unroll
      for (int r = 0; r < REGS; ++r) acc[r] += red[(w2 * REGS + r) * 32 + lane];
    }
    Tile<MT, NT> tl;
    tl.init(sub, tk.nsub_n, tk.m, tk.n, g);
    double tile[MT][NT][2];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        tile[i][j][0] = acc[(i * NT + j) * 2 + 0];
        tile[i][j][1] = acc[(i * NT + j) * 2 + 1];
      }
    commit_tile<MT, NT>(tk.c, (size_t)xkey - 1, tile, tk.m, tk.n, g, t, tl, tk.alpha);
  }
  __syncthreads();
}

/* Combine of a single stack: grid-stride over (segment-list entry, sub-tile). */
template <int MT, int NT>
__global__ void __launch_bounds__(32 * kCombineWarps)
  xs_smm_combine_kernel(const __grid_constant__ StackTask tk, int W, const int* __restrict__ seglist,
    const unsigned* __restrict__ err) {
  extern __shared__ double red[]; /* [CW - 1][REGS][32] */
  pdl_wait();
  if (0 != *(volatile const unsigned*)err) return;
  const int count = seglist[0];
  for (int w = blockIdx.x; w < count * tk.nsub; w += gridDim.x) {
    const int li = w / tk.nsub, sub = w - li * tk.nsub;
    combine_one<MT, NT>(tk, W, seglist[1 + li] & 0xFFFFFF, sub, red);
  }
}

/* ------------------------------------------------- unified persistent batch kernel (one launch) */

/* Shapes the unified batch kernel runs with their staged item function (every shape with a staged
   kernel; 2 CTAs per SM leave 255 registers for the largest, 16 fragments); X(index, m, n, k). */
#define XS_UNI_STAGED(X) \
  X(0, 4, 4, 4) X(1, 8, 8, 8) X(2, 9, 9, 9) X(3, 13, 13, 13) X(4, 16, 16, 16) X(5, 22, 22, 22) X(6, 23, 23, 23) \
  X(7, 23, 22, 13) X(8, 22, 22, 23) X(9, 32, 9, 9) X(10, 13, 4, 16) X(11, 16, 26, 5) X(12, 26, 26, 26) \
  X(13, 26, 23, 26) X(14, 22, 32, 32) X(15, 16, 64, 9)
constexpr int kUniMinBlocks = 2; /* CTAs per SM */
constexpr int kUniW = 4;       /* warps per CTA */
constexpr int kUniR = 2;       /* bulk-copy stages per warp of the staged items */
constexpr int kUniHeader = 128; /* shared memory before an item's area: mbarriers [W][R], merge metadata [W][4] */
constexpr size_t cmax_sz(size_t a, size_t b) { return a > b ? a : b; }
/* shared memory of an item: the staged shapes' rings (+ slack), the register kernel's pieces (3 x 3
   fragments at most) */
#define XS_UNI_AREA(i, M, N, K) (size_t)kUniW * Staged<M, N, K>::warp_bytes(kUniR) + 256,
constexpr size_t kUniAreas[] = {XS_UNI_STAGED(XS_UNI_AREA) smm_smem_bytes<4, 4>(kUniW)};
#undef XS_UNI_AREA
constexpr size_t uni_area_max(int i) {
  return (i + 1 == (int)(sizeof(kUniAreas) / sizeof(*kUniAreas))) ? kUniAreas[i] : cmax_sz(kUniAreas[i], uni_area_max(i + 1));
}
constexpr size_t kUniArea = uni_area_max(0);
constexpr size_t kUniSmem = kUniHeader + kUniArea;

template <int M_, int N_, int K_>
__device__ __forceinline__ bool uni_staged(const StackTask& tk, int group, int* seglist, unsigned* err, long long wait_limit,
  unsigned char* area, uint64_t* bars, int* meta, unsigned* phase, int* s_probe, int (*duty)[6]) {
  unsigned ph = *phase;
  const bool ok = staged_item<M_, N_, K_, kUniR>(tk, group, seglist, err, wait_limit, area, bars, meta, ph, s_probe, duty);
  *phase = ph;
  return ok;
}

/* The unified persistent batch kernel: every stack of the call in one launch. The grid is the number
   of CTAs resident on the device; each CTA takes work items (CTA group x sub-tile of one stack) from
   one queue in the order the host laid them out (heaviest items first) and runs each with its
   stack's kernel: the staged item function of its shape, or the register kernel of its tile class.
   Every stack combines its CTA-crossing segments inside the kernel (arrival counters zeroed by the
   grouping), so nothing follows. A copy that does not land in time stops the CTA with the grouping
   error word and a device error bit set; the other CTAs stop at their next item. */
__global__ void __launch_bounds__(32 * kUniW, kUniMinBlocks)
  xs_smm_uni_kernel(const __grid_constant__ BatchTasks bt, int* __restrict__ seglist, unsigned* __restrict__ queue,
    unsigned* __restrict__ err, unsigned* __restrict__ dev_err, long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ int s_item, s_probe[2], duty[2][6];
  uint64_t* const bars = (uint64_t*)smraw;
  int* const meta = (int*)(smraw + kUniW * kUniR * sizeof(uint64_t));
  unsigned char* const area = smraw + kUniHeader;
  for (int ti = 0; ti < bt.ntasks; ++ti) prefetch_operands(bt.t[ti]);
  pdl_wait();
  pdl_trigger();
  if (__syncthreads_or((0 != *(volatile const unsigned*)err) ? 1 : 0)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (0 == lane) {
#pragma unroll
    for (int q = 0; q < kUniR; ++q) xs_tc::mbar_init(&bars[warp * kUniR + q], 1);
    xs_tc::fence_barrier_init();
  }
  __syncwarp();
  unsigned phase = 0u; /* bit q: parity of the next phase of this warp's barrier q */
  for (;;) {
    if (0 == threadIdx.x) s_item = (0 != *(volatile const unsigned*)err) ? bt.nitems : (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= bt.nitems) break;
    int ti = 0;
    while (ti + 1 < bt.ntasks && bt.t[ti + 1].item_begin <= item) ++ti;
    const StackTask& tk = bt.t[ti];
    const int local = item - tk.item_begin, group = local / tk.nsub, sub = local - group * tk.nsub;
    bool ok = true;
    switch (tk.kind) {
#define XS_UNI_CASE(i, M, N, K) \
  case 1 + i: ok = uni_staged<M, N, K>(tk, group, seglist, err, wait_limit, area, bars, meta, &phase, s_probe, duty); break;
      XS_UNI_STAGED(XS_UNI_CASE)
#undef XS_UNI_CASE
      default: {
        double* const smem = (double*)area;
        const int cls = tk.cls;
        batch_dispatch<0, 1, 1>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 1, 2>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 1, 3>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 1, 4>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 2, 1>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 2, 2>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 2, 3>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 2, 4>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 3, 1>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 3, 2>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 3, 3>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 4, 1>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<0, 4, 2>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<1, 3, 4>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<1, 4, 3>(cls, tk, group, sub, seglist, smem);
        batch_dispatch<1, 4, 4>(cls, tk, group, sub, seglist, smem);
      }
    }
    if (!ok) { /* uniform over the CTA */
      if (0 == threadIdx.x && nullptr != dev_err) atomicOr(dev_err, kErrStagedTimeout);
      break;
    }
    __syncthreads(); /* the next item reuses shared memory */
  }
}

/* Index of (m, n, k) in the unified kernel's staged shapes, -1 if it has none. */
int uni_staged_index(int m, int n, int k) {
#define XS_UNI_FIND(i, M, N, K) \
  if (M == m && N == n && K == k) return i;
  XS_UNI_STAGED(XS_UNI_FIND)
#undef XS_UNI_FIND
  return -1;
}

struct SmmPlan {
  int nsub_m, nsub_n, nsub, nchunks, L, W, ngroups;
  int Ls[3], slotn; /* chunk lengths per CTA length class (chunk_first) */
  int no_combine; /* the stack kernel only: CTA-crossing pieces are combined by the caller */
  size_t off_keys_in, off_keys_tmp, off_keys_out, off_vals_in, off_vals_tmp, off_vals_out, off_seglist, off_pieces;
  size_t off_arrive, off_sort, total;
};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

/* Launches the stack and combine kernels of one stack; with occ != nullptr it only reports how many
   CTAs of W = pl.W warps fit on one SM (the plan sizes chunks from that). */
typedef cudaError_t (*launch_fn_t)(const SmmPlan& pl, const StackTask& tk, int* seglist, const unsigned* err,
  cudaStream_t s, int* occ);

launch_fn_t find_launcher(int m, int n, int k, const xs_smm_params_t* prm);
struct WsEntry;
const WsEntry* find_ws(int m, int n, int k, int wpb);
int fma_piece_regs(int m, int n, int k);

/* Work decomposition and scratch layout of one call. An open chunk length (prm->chunk <= 0) is
   sized so that the grid is one full wave of resident CTAs: L = ceil(S * nsub / (resident * W)). */
/* Fraction of the chunk length moved from the CTA groups launched last on their SM to the ones
   launched first (chunk_first), for one-wave launches of three CTAs per SM of stacks the one-cluster
   grouping takes: 12 % (measured on B200: 23^3 and 22^3 stacks of 30000 entries 6-12 % shorten the
   step by about 1.5 %, 18 % and more lengthen it; 32x9x9 at 10^5 entries and the shapes that run two
   CTAs per SM were slower with it, so they keep equal chunks); LIBXSTREAM_B200_CHUNK_SKEW (percent,
   0 = equal chunks) overrides the 12 %. */
static double chunk_skew() {
  static const double v = []() -> double {
    const char* const env = getenv("LIBXSTREAM_B200_CHUNK_SKEW");
    const double pc = (nullptr != env) ? atof(env) : 12.0;
    return (0.0 < pc && pc < 50.0) ? pc / 100.0 : 0.0;
  }();
  return v;
}

/* Chunks that start before S under the plan's lengths (the host side of chunk_first). */
static int plan_nchunks(const SmmPlan& pl, int S) {
  if (pl.Ls[0] == pl.Ls[1] && pl.Ls[1] == pl.Ls[2]) return (S + pl.L - 1) / pl.L;
  const long long cap0 = (long long)pl.W * pl.slotn * pl.Ls[0], cap1 = (long long)pl.W * pl.slotn * pl.Ls[1];
  if (S <= cap0) return (int)((S + pl.Ls[0] - 1) / pl.Ls[0]);
  if (S <= cap0 + cap1) return pl.W * pl.slotn + (int)((S - cap0 + pl.Ls[1] - 1) / pl.Ls[1]);
  return 2 * pl.W * pl.slotn + (int)((S - cap0 - cap1 + pl.Ls[2] - 1) / pl.Ls[2]);
}

int plan_smm(int S, int m, int n, int k, const xs_smm_params_t* prm, SmmPlan* pl) {
  const int mt = prm->mt, nt = prm->nt;
  double auto_skew = 0.0;
  if (mt < 1 || mt > 8 || nt < 1 || nt > 8) return -1; /* tiles beyond 4 fragments: staged kernels only */
  pl->no_combine = 0;
  pl->nsub_m = ((m + 7) / 8 + mt - 1) / mt;
  pl->nsub_n = ((n + 7) / 8 + nt - 1) / nt;
  if (XS_KP_FMA == prm->kp) pl->nsub_m = pl->nsub_n = 1; /* the FMA lane grid covers the whole block */
  pl->nsub = pl->nsub_m * pl->nsub_n;
  pl->W = (prm->wpb >= 1 && prm->wpb <= 4) ? prm->wpb : 4;
  if (0 == prm->generic && 4 < prm->wpb && nullptr != find_ws(m, n, k, prm->wpb) && (m + 7) / 8 == mt && (n + 7) / 8 == nt) {
    pl->W = prm->wpb; /* warp-specialised kernel: wpb consumer warps, one chunk each */
  }
  if (0 < prm->chunk) pl->L = prm->chunk;
  else {
    int occ = 0;
    StackTask none = {};
    none.m = m; /* the shape sizes the shared memory of runtime-shape kernels */
    none.n = n;
    none.k = k;
    const launch_fn_t fn = find_launcher(m, n, k, prm);
    if (cudaSuccess != fn(*pl, none, nullptr, nullptr, 0, &occ) || occ < 1) occ = 1;
    const long resident = (long)occ * xs_sm_count();
    const long L = ((long)S * pl->nsub + resident * pl->W - 1) / (resident * pl->W);
    pl->L = (int)(L < 1 ? 1 : L);
    auto_skew = (3 == occ && 1 == pl->nsub && S <= xs_stack_group_cluster_max()) ? chunk_skew() : 0.0;
  }
  pl->Ls[0] = pl->Ls[1] = pl->Ls[2] = pl->L;
  pl->slotn = 1 << 29;
  {
    const int d = (int)(auto_skew * pl->L + 0.5);
    if (0 < d && d < pl->L) { /* a one-wave launch of three CTAs per SM: the first-launched third of the
                                 CTA groups takes L + d entries per chunk, the last third L - d */
      pl->Ls[0] = pl->L + d;
      pl->Ls[2] = pl->L - d;
      pl->slotn = xs_sm_count();
    }
  }
  pl->nchunks = plan_nchunks(*pl, S);
  pl->ngroups = (pl->nchunks + pl->W - 1) / pl->W;
  size_t off = 0;
  const size_t ks = align_up(sizeof(unsigned) * (size_t)S, 256), vs = align_up(sizeof(unsigned long long) * (size_t)S, 256);
  pl->off_keys_in = off;
  off += ks;
  pl->off_keys_tmp = off;
  off += ks;
  pl->off_keys_out = off;
  off += ks;
  pl->off_vals_in = off;
  off += vs;
  pl->off_vals_tmp = off;
  off += vs;
  pl->off_vals_out = off;
  off += vs;
  pl->off_seglist = off;
  off = align_up(off + sizeof(int) * ((size_t)pl->ngroups + 1), 256);
  pl->off_pieces = off; /* two pieces per CTA group and sub-tile, one warp's accumulators each */
  const int regs = (XS_KP_FMA == prm->kp) ? fma_piece_regs(m, n, k) : mt * nt * 2;
  if (0 >= regs) return -1;
  off = align_up(off + sizeof(double) * (size_t)2 * pl->ngroups * pl->nsub * regs * 32, 256);
  pl->off_arrive = off; /* segment counters [ngroups][nsub], then first-level counters [2 ngroups][nsub] */
  off = align_up(off + sizeof(int) * (size_t)3 * pl->ngroups * pl->nsub, 256);
  pl->off_sort = off;
  off = align_up(off + xs_stack_sort_scratch_bytes(S), 256);
  pl->total = off;
  return 0;
}

/* The combine kernel of one stack (CTA-crossing segments), MT x NT warp tiles. */
template <int MT, int NT>
cudaError_t launch_combine(const SmmPlan& pl, const StackTask& tk, const int* seglist, const unsigned* err, cudaStream_t s) {
  const int cgrid = max(1, min(pl.ngroups * pl.nsub, 2 * xs_sm_count()));
  const size_t csmem = sizeof(double) * (kCombineWarps - 1) * (MT * NT * 2) * 32;
  {
    const cudaError_t r = (cudaError_t)xs_func_smem((const void*)xs_smm_combine_kernel<MT, NT>, csmem);
    if (cudaSuccess != r) return r;
  }
  void* prof = xs_profile_begin(s);
  const cudaError_t r = pdl_launch(xs_smm_combine_kernel<MT, NT>, cgrid, 32 * kCombineWarps, csmem, s, tk, pl.W, seglist, err);
  xs_profile_end(prof, "combine", 0.0, 0.0, s);
  return r;
}

template <int M_, int N_, int K_, int MT, int NT, int KP>
cudaError_t launch_dmma(const SmmPlan& pl, const StackTask& tk, int* seglist, const unsigned* err, cudaStream_t s,
  int* occ) {
  cudaError_t r;
  const size_t smem = smm_smem_bytes<MT, NT>(pl.W);
  r = (cudaError_t)xs_func_smem((const void*)xs_smm_dmma_kernel<M_, N_, K_, MT, NT, KP>, smem);
  if (cudaSuccess != r) return r;
  if (nullptr != occ) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, xs_smm_dmma_kernel<M_, N_, K_, MT, NT, KP>, 32 * pl.W, smem);
  }
  void* prof = xs_profile_begin(s);
  r = pdl_launch(xs_smm_dmma_kernel<M_, N_, K_, MT, NT, KP>, pl.ngroups * pl.nsub, 32 * pl.W, smem, s, tk, seglist, err);
  if (cudaSuccess != r) return r;
  const double m = tk.m, n = tk.n, k = tk.k;
  xs_profile_end(prof, "smm", 2.0 * m * n * k * (double)tk.S, 8.0 * tk.S * (m * k + k * n + 2.0 * m * n), s);
  return (pl.no_combine || nullptr != tk.arrive) ? cudaSuccess : launch_combine<MT, NT>(pl, tk, seglist, err, s);
}

/* The staged kernel of one block shape with an R-deep ring per warp, then the combine. */
template <int M_, int N_, int K_, int R>
cudaError_t launch_staged(const SmmPlan& pl, const StackTask& tk, int* seglist, const unsigned* err, cudaStream_t s,
  int* occ) {
  using G = Staged<M_, N_, K_>;
  cudaError_t r;
  const size_t smem = G::smem_bytes(pl.W, R);
  r = (cudaError_t)xs_func_smem((const void*)xs_smm_staged_kernel<M_, N_, K_, R>, smem);
  if (cudaSuccess != r) return r;
  if (nullptr != occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, xs_smm_staged_kernel<M_, N_, K_, R>, 32 * pl.W, smem);
  if (1 != pl.nsub) return cudaErrorInvalidValue; /* one warp tile per C block */
  void* prof = xs_profile_begin(s);
  r = pdl_launch(xs_smm_staged_kernel<M_, N_, K_, R>, pl.ngroups, 32 * pl.W, smem, s, tk, seglist, (unsigned*)err,
    xs_device_error_ptr(), xs_wait_limit());
  if (cudaSuccess != r) return r;
  const double m = M_, n = N_, k = K_;
  xs_profile_end(prof, "smm", 2.0 * m * n * k * (double)tk.S, 8.0 * tk.S * (m * k + k * n + 2.0 * m * n), s);
  return (pl.no_combine || nullptr != tk.arrive) ? cudaSuccess : launch_combine<G::MT, G::NT>(pl, tk, seglist, err, s);
}

/* The warp-specialised staged kernel of one block shape: NC consumer warps + one producer warp per
   CTA, rings of R stages, MINB CTAs per SM; then the combine (when the stack kernel does not combine
   its CTA-crossing segments itself). */
template <int M_, int N_, int K_, int NC, int R, int MINB>
cudaError_t launch_ws(const SmmPlan& pl, const StackTask& tk, int* seglist, const unsigned* err, cudaStream_t s, int* occ) {
  using G = Staged<M_, N_, K_>;
  cudaError_t r;
  const size_t smem = ws_smem_bytes<M_, N_, K_>(NC, R);
  r = (cudaError_t)xs_func_smem((const void*)xs_smm_ws_kernel<M_, N_, K_, NC, R, MINB>, smem);
  if (cudaSuccess != r) return r;
  if (nullptr != occ) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, xs_smm_ws_kernel<M_, N_, K_, NC, R, MINB>, 32 * (NC + 1), smem);
  }
  if (1 != pl.nsub || NC != pl.W) return cudaErrorInvalidValue; /* one warp tile per C block, NC chunks per CTA */
  void* prof = xs_profile_begin(s);
  r = pdl_launch(xs_smm_ws_kernel<M_, N_, K_, NC, R, MINB>, pl.ngroups, 32 * (NC + 1), smem, s, tk, seglist, (unsigned*)err,
    xs_device_error_ptr(), xs_wait_limit());
  if (cudaSuccess != r) return r;
  const double m = M_, n = N_, k = K_;
  xs_profile_end(prof, "smm", 2.0 * m * n * k * (double)tk.S, 8.0 * tk.S * (m * k + k * n + 2.0 * m * n), s);
  return (pl.no_combine || nullptr != tk.arrive) ? cudaSuccess : launch_combine<G::MT, G::NT>(pl, tk, seglist, err, s);
}

/* The FMA kernel: FmaLayout<LR, RB, CB> tiles, D-deep cp.async ring per warp. Its CTA-crossing segments
   are combined inside the kernel (the combine kernel takes DMMA-layout pieces only). */
template <int M_, int N_, int K_, int LR, int RB, int CB, int D>
cudaError_t launch_fma(const SmmPlan& pl, const StackTask& tk, int* seglist, const unsigned* err, cudaStream_t s, int* occ) {
  constexpr int REGS = RB * CB, SLACK = (32 / LR * CB + 1) / 2 * 2;
  const int m = M_ ? M_ : tk.m, n = N_ ? N_ : tk.n, k = K_ ? K_ : tk.k;
  if (m < 1 || n < 1 || k < 1 || m > LR * RB || n > 32 / LR * CB) return cudaErrorInvalidValue;
  const size_t smem = fma_smem_bytes(m, n, k, D, REGS, SLACK, pl.W);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t r = (cudaError_t)xs_func_smem((const void*)xs_smm_fma_kernel<M_, N_, K_, LR, RB, CB, D>, smem);
  if (cudaSuccess != r) return r;
  if (nullptr != occ) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, xs_smm_fma_kernel<M_, N_, K_, LR, RB, CB, D>, 32 * pl.W, smem);
  }
  if (1 != pl.nsub || nullptr == tk.arrive) return cudaErrorInvalidValue;
  void* prof = xs_profile_begin(s);
  r = pdl_launch(xs_smm_fma_kernel<M_, N_, K_, LR, RB, CB, D>, pl.ngroups, 32 * pl.W, smem, s, tk, seglist, err);
  if (cudaSuccess != r) return r;
  xs_profile_end(prof, "smm", 2.0 * m * n * k * (double)tk.S, 8.0 * tk.S * ((double)m * k + (double)k * n + 2.0 * m * n), s);
  return cudaSuccess;
}

/* FMA kernels: shapes compiled with their own lane grids, then runtime-shape classes (k <= 80) for any
   block whose C fits the class's lane grid; a shape takes the class with the fewest padded elements. */
struct FmaEntry {
  int m, n, k; /* 0: runtime */
  int mmax, nmax;
  int regs;  /* accumulators per lane (RB * CB): the size of a piece is regs * 32 doubles */
  int D;     /* ring depth */
  int slack; /* doubles after the last stage */
  launch_fn_t fn;
};
#define XS_FMA(M, N, K, LR, RB, CB, D) \
  {M, N, K, M, N, RB * CB, D, (32 / LR * CB + 1) / 2 * 2, &launch_fma<M, N, K, LR, RB, CB, D>}
#define XS_FMA_RT(LR, RB, CB, D) \
  {0, 0, 0, LR * RB, 32 / LR * CB, RB * CB, D, (32 / LR * CB + 1) / 2 * 2, &launch_fma<0, 0, 0, LR, RB, CB, D>}
static const FmaEntry fma_table[] = {
  XS_FMA(4, 4, 4, 4, 1, 1, 8), XS_FMA(5, 5, 5, 8, 1, 2, 8), XS_FMA(6, 6, 18, 8, 1, 2, 6), XS_FMA(13, 4, 16, 16, 1, 2, 6),
  XS_FMA(32, 9, 9, 16, 2, 5, 4), XS_FMA(16, 64, 9, 8, 2, 16, 3), XS_FMA(7, 10, 5, 8, 1, 3, 8),
  XS_FMA_RT(8, 1, 1, 8), XS_FMA_RT(8, 1, 2, 8), XS_FMA_RT(8, 2, 2, 6), XS_FMA_RT(8, 2, 4, 6), XS_FMA_RT(16, 2, 4, 4),
  XS_FMA_RT(16, 2, 8, 4), XS_FMA_RT(8, 2, 8, 4), XS_FMA_RT(8, 2, 16, 3), XS_FMA_RT(16, 2, 16, 3),
};
constexpr int kFmaMaxK = 80;

const FmaEntry* find_fma(int m, int n, int k) {
  const FmaEntry* best = nullptr;
  for (const FmaEntry& e : fma_table) {
    if (0 != e.m) {
      if (e.m == m && e.n == n && e.k == k) return &e;
      continue;
    }
    if (m > e.mmax || n > e.nmax || k > kFmaMaxK) continue;
    if (nullptr == best || e.mmax * e.nmax < best->mmax * best->nmax) best = &e;
  }
  return best;
}

/* Accumulators per lane of the FMA kernel that runs (m, n, k), 0 if none does. */
int fma_piece_regs(int m, int n, int k) {
  const FmaEntry* const f = find_fma(m, n, k);
  return (nullptr != f) ? f->regs : 0;
}

/* Runtime-shape kernels: any (m, n, k), warp sub-tile MT x NT, KP in {2, 4}. */
#define XS_KP_ENTRY(MT, NT) {&launch_dmma<0, 0, 0, MT, NT, 2>, &launch_dmma<0, 0, 0, MT, NT, 4>}
static const launch_fn_t launch_table[4][4][2] = {
  {XS_KP_ENTRY(1, 1), XS_KP_ENTRY(1, 2), XS_KP_ENTRY(1, 3), XS_KP_ENTRY(1, 4)},
  {XS_KP_ENTRY(2, 1), XS_KP_ENTRY(2, 2), XS_KP_ENTRY(2, 3), XS_KP_ENTRY(2, 4)},
  {XS_KP_ENTRY(3, 1), XS_KP_ENTRY(3, 2), XS_KP_ENTRY(3, 3), XS_KP_ENTRY(3, 4)},
  {XS_KP_ENTRY(4, 1), XS_KP_ENTRY(4, 2), XS_KP_ENTRY(4, 3), XS_KP_ENTRY(4, 4)},
};

/* Shape-specialised kernels for the square block sizes DBCSR workloads use most. */
struct SpecEntry {
  int m, n, k, mt, nt, kp;
  launch_fn_t fn;
};
#define XS_SPEC(S, MT, KP) {S, S, S, MT, MT, KP, &launch_dmma<S, S, S, MT, MT, KP>}
#define XS_STAGED(S, R) {S, S, S, (S + 7) / 8, (S + 7) / 8, 0, &launch_staged<S, S, S, R>}
#define XS_STAGED3(M, N, K, R) {M, N, K, (M + 7) / 8, (N + 7) / 8, 0, &launch_staged<M, N, K, R>}
static const SpecEntry spec_table[] = {
  XS_SPEC(4, 1, 1), XS_SPEC(5, 1, 2), XS_SPEC(8, 1, 2), XS_SPEC(9, 2, 3), XS_SPEC(16, 2, 2), XS_SPEC(16, 2, 4),
  XS_SPEC(32, 4, 2), XS_SPEC(32, 4, 4), XS_SPEC(45, 3, 2), XS_SPEC(45, 3, 4), XS_SPEC(64, 4, 2), XS_SPEC(64, 4, 4),
};

/* Shapes with a staged kernel: it runs whenever the warp tile covers the whole C block (any kp),
   unless the runtime-shape kernel is forced (generic). Each was measured against the register
   kernel on stacks of 30000 entries; 5^3 (no gain) and 32^3 (slower: a 256-byte column stride puts
   every fragment column on the same banks) keep the register kernel, like every shape not listed. */
static const SpecEntry staged_table[] = {
  XS_STAGED(13, 2), XS_STAGED(22, 2), XS_STAGED(23, 2), XS_STAGED(26, 2),
  XS_STAGED3(23, 22, 13, 2), XS_STAGED3(22, 22, 23, 2), XS_STAGED3(32, 9, 9, 2), XS_STAGED3(13, 4, 16, 2),
  XS_STAGED(4, 2), XS_STAGED(8, 2), XS_STAGED(9, 2), XS_STAGED(16, 2), XS_STAGED3(16, 26, 5, 2), XS_STAGED3(26, 23, 26, 2),
  XS_STAGED3(22, 32, 32, 2), XS_STAGED3(16, 64, 9, 2),
};

/* Shapes with a warp-specialised staged kernel, selected by the warps-per-CTA parameter (wpb = NC,
   the consumer warps; values above 4, which the other kernels do not take). */
struct WsEntry {
  int m, n, k, nc;
  launch_fn_t fn;
};
#define XS_WS(M, N, K, NC, R, MINB) {M, N, K, NC, &launch_ws<M, N, K, NC, R, MINB>}
static const WsEntry ws_table[] = {
  XS_WS(23, 23, 23, 12, 2, 1), XS_WS(23, 23, 23, 6, 2, 2), XS_WS(23, 23, 23, 8, 3, 1),
};

const WsEntry* find_ws(int m, int n, int k, int wpb) {
  for (const WsEntry& e : ws_table) {
    if (e.m == m && e.n == n && e.k == k && e.nc == wpb) return &e;
  }
  return nullptr;
}

cudaError_t launch_unsupported(const SmmPlan&, const StackTask&, int*, const unsigned*, cudaStream_t, int*) {
  return cudaErrorInvalidValue;
}

launch_fn_t find_launcher(int m, int n, int k, const xs_smm_params_t* prm) {
  if (XS_KP_FMA == prm->kp) {
    const FmaEntry* const f = find_fma(m, n, k);
    return (nullptr != f) ? f->fn : &launch_unsupported;
  }
  if (0 == prm->generic) {
    if (4 < prm->wpb) {
      const WsEntry* const w = find_ws(m, n, k, prm->wpb);
      if (nullptr != w && (m + 7) / 8 == prm->mt && (n + 7) / 8 == prm->nt) return w->fn;
    }
    for (const SpecEntry& e : staged_table) {
      if (e.m == m && e.n == n && e.k == k && e.mt == prm->mt && e.nt == prm->nt) return e.fn;
    }
    for (const SpecEntry& e : spec_table) {
      if (e.m == m && e.n == n && e.k == k && e.mt == prm->mt && e.nt == prm->nt && e.kp == prm->kp) return e.fn;
    }
  }
  if (prm->mt > 4 || prm->nt > 4) return &launch_unsupported; /* no register kernel for such tiles */
  return launch_table[prm->mt - 1][prm->nt - 1][(4 == prm->kp) ? 1 : 0];
}

/* ------------------------------------------------------------- unified batch: plan and launch */

/* One part of a batch: a stack, or a slice of a stack larger than one grouping launch takes. */
struct UniPart {
  int stack, first, S;
  int kind;   /* 0: register kernel of tile class (mt, nt); else 1 + staged shape index */
  int mt, nt; /* warp tile in 8 x 8 fragments */
  int nsub, nsub_n, L, ngroups;
  double item_cost;
};

/* Work items per resident CTA the plan aims for: enough for the queue to even out items of unequal
   speed, few enough that an item's start (first copies in flight) and merge stay a small share. A
   batch of one part has items of equal speed: one per CTA. Otherwise one per kUniItemCost cost units
   of work per CTA, between 6 and 16 (measured on B200: a 186k-triple mixed batch, 25k units per CTA,
   is fastest with 6 items per CTA, a 2M-triple one, 275k units, with 12-24). */
constexpr double kUniItemsMin = 6.0, kUniItemsMax = 16.0, kUniItemCost = 4000.0;

struct UniPlan {
  int nparts, ntotal, nitems, ngroups_total, occ;
  UniPart part[kMaxBatchTasks];
  int order[kMaxBatchTasks]; /* parts by descending item cost */
  size_t off_part[kMaxBatchTasks], pieces_off[kMaxBatchTasks], arrive_off[kMaxBatchTasks];
  size_t off_keys_in, off_keys_tmp, off_keys_out, off_vals_in, off_vals_tmp, off_vals_out, off_seglist, off_pieces;
  size_t off_arrive, narrive, off_sort, total;
};

/* Tile of at most 4 x 4 fragments for a block of fm x fn fragments: the fewest padded fragments,
   then the fewest sub-tiles. */
void uni_tiles(int fm, int fn, int* mt, int* nt) {
  long best = -1;
  for (int a = 1; a <= 4; ++a) {
    for (int b = 1; b <= 4; ++b) {
      const long subs = (long)((fm + a - 1) / a) * ((fn + b - 1) / b);
      const long cost = subs * a * b * 64 + subs;
      if (best < 0 || cost < best) {
        best = cost;
        *mt = a;
        *nt = b;
      }
    }
  }
}

/* CTAs of the unified kernel resident per SM on the active device (cached per device). */
int uni_occupancy(void) {
  static int occ_cached[XS_MAXDEV]; /* 0 until set up */
  const int dev = xs_device_slot();
  if (0 == occ_cached[dev]) {
    int o = 0;
    if (cudaSuccess != (cudaError_t)xs_func_smem((const void*)xs_smm_uni_kernel, kUniSmem) ||
        cudaSuccess != cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, xs_smm_uni_kernel, 32 * kUniW, kUniSmem) || o < 1) {
      return 0;
    }
    occ_cached[dev] = o;
  }
  return occ_cached[dev];
}

/* Work decomposition of a batch for the unified kernel: stacks split into parts of at most
   xs_stack_group_max() entries; per part its kernel (the staged item function of its shape, or the
   register kernel of a tile class of at most 4 x 4 fragments) and a chunk length L chosen so that every
   work item (kUniW chunks x one sub-tile) costs about the same (kUniItemsMin..kUniItemsMax items per
   resident CTA). Returns the
   number of parts, -1 if the batch has too many parts or the kernel cannot be set up. */
int plan_uni(const libxstream_b200_stack_t* st, int ns, UniPlan* up) {
  const int smax = xs_stack_group_max();
  up->nparts = 0;
  up->ntotal = 0;
  for (int i = 0; i < ns; ++i) {
    if (0 >= st[i].stack_size) continue;
    const int m = st[i].m, n = st[i].n, k = st[i].k, fm = (m + 7) / 8, fn = (n + 7) / 8;
    xs_smm_params_t prm;
    xs_params_lookup(3, m, n, k, st[i].stack_size, &prm);
    const int sidx = uni_staged_index(m, n, k);
    int mt = prm.mt, nt = prm.nt;
    if (0 > sidx && (mt > fm || nt > fn)) uni_tiles(fm, fn, &mt, &nt);
    for (int first = 0; first < st[i].stack_size; first += smax) {
      if (up->nparts == kMaxBatchTasks) return -1;
      UniPart& p = up->part[up->nparts++];
      p.stack = i;
      p.first = first;
      p.S = min(smax, st[i].stack_size - first);
      p.kind = (0 <= sidx) ? 1 + sidx : 0;
      p.mt = (0 <= sidx) ? fm : mt;
      p.nt = (0 <= sidx) ? fn : nt;
      p.nsub_n = (0 <= sidx) ? 1 : (fn + p.nt - 1) / p.nt;
      p.nsub = (0 <= sidx) ? 1 : ((fm + p.mt - 1) / p.mt) * p.nsub_n;
      up->ntotal += p.S;
    }
  }
  if (0 == up->nparts) return 0;
  up->occ = uni_occupancy();
  if (0 >= up->occ) return -1;
  /* cost units: DMMA instructions per entry per warp plus a fixed per-entry overhead */
  double total = 0;
  for (int q = 0; q < up->nparts; ++q) {
    const UniPart& p = up->part[q];
    total += (double)p.S * p.nsub * (p.mt * p.nt * ((st[p.stack].k + 3) / 4) + 8);
  }
  const double per_cta = total / ((double)up->occ * xs_sm_count());
  const double items = (1 == up->nparts) ? 1.0 : fmin(kUniItemsMax, fmax(kUniItemsMin, per_cta / kUniItemCost));
  const double target = per_cta / items;
  size_t off = 0, poff = 0, narrive = 0;
  up->ngroups_total = 0;
  up->nitems = 0;
  for (int q = 0; q < up->nparts; ++q) {
    UniPart& p = up->part[q];
    const double per_entry = p.mt * p.nt * ((st[p.stack].k + 3) / 4) + 8;
    long L = (long)(target / (kUniW * per_entry) + 0.5);
    if (L < 1) L = 1;
    if (L > p.S) L = p.S;
    p.L = (int)L;
    const int nchunks = (int)((p.S + L - 1) / L);
    p.ngroups = (nchunks + kUniW - 1) / kUniW;
    p.item_cost = (double)kUniW * L * per_entry;
    up->off_part[q] = off;
    off += (size_t)p.S;
    up->pieces_off[q] = poff;
    poff += (size_t)2 * p.ngroups * p.nsub * (p.mt * p.nt * 2) * 32;
    up->arrive_off[q] = narrive;
    narrive += (size_t)3 * p.ngroups * p.nsub;
    up->ngroups_total += p.ngroups;
    up->nitems += p.ngroups * p.nsub;
    up->order[q] = q;
  }
  for (int a = 1; a < up->nparts; ++a) { /* heaviest items first (insertion sort, stable) */
    const int v = up->order[a];
    int b = a - 1;
    while (b >= 0 && up->part[up->order[b]].item_cost < up->part[v].item_cost) {
      up->order[b + 1] = up->order[b];
      --b;
    }
    up->order[b + 1] = v;
  }
  const size_t N = (size_t)up->ntotal;
  size_t o = 0;
  const size_t ks = align_up(sizeof(unsigned) * N, 256), vs = align_up(sizeof(unsigned long long) * N, 256);
  up->off_keys_in = o;
  o += ks;
  up->off_keys_tmp = o;
  o += ks;
  up->off_keys_out = o;
  o += ks;
  up->off_vals_in = o;
  o += vs;
  up->off_vals_tmp = o;
  o += vs;
  up->off_vals_out = o;
  o += vs;
  up->off_seglist = o;
  o = align_up(o + sizeof(int) * ((size_t)up->ngroups_total + 1), 256);
  up->off_pieces = o;
  o = align_up(o + sizeof(double) * poff, 256);
  up->off_arrive = o;
  up->narrive = narrive;
  o = align_up(o + sizeof(int) * narrive, 256);
  up->off_sort = o;
  o = align_up(o + xs_sort_ctl_bytes() + sizeof(int) * ((size_t)xs_sort_launch_tiles() + XS_MAX_BATCH) * 2048, 256);
  up->total = o;
  return up->nparts;
}

/* ------------------------------------------------------------------------------ transpose */

/* In-place transposes of listed blocks (transpose.cl:28-83 semantics; a bit copy, exact for any
   element type). One CTA handles `nb` blocks at a time: all their elements are gathered into shared
   memory with consecutive threads on consecutive elements of a block (coalesced), each block's
   columns `ld` = m|1 elements apart (an odd stride: the transposed reads of a warp then hit distinct
   banks), then written back as n x m column-major, again with consecutive threads on consecutive
   output elements. */
template <typename T>
__global__ void __launch_bounds__(256) xs_transpose_kernel(const int* __restrict__ trs, int offset, int S, T* __restrict__ data,
  int m, int n, int nb) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ int s_off[256];
  T* const buf = reinterpret_cast<T*>(smem_raw);
  const int mn = m * n, ld = m | 1, bsz = ld * n, step = blockDim.x;
  /* the thread stride as (blocks, columns, rows) for the input walk and (blocks, rows, columns) for
     the output walk, so that indices advance by additions and carries only */
  const int sb = step / mn, sr = step - sb * mn;
  const int sj_in = sr / m, si_in = sr - sj_in * m;  /* input: e = b*mn + j*m + i */
  const int si_out = sr / n, sj_out = sr - si_out * n; /* output: e = b*mn + i*n + j */
  const int t = threadIdx.x;
  const int tb = t / mn, tr = t - tb * mn;
  const int tj_in = tr / m, ti_in = tr - tj_in * m, ti_out = tr / n, tj_out = tr - ti_out * n;
  for (int b0 = blockIdx.x * nb; b0 < S; b0 += gridDim.x * nb) {
    const int nbl = min(nb, S - b0);
    for (int q = t; q < nbl; q += step) s_off[q] = trs[offset + b0 + q];
    __syncthreads();
    { /* gather: eight independent loads in flight per thread, then the shared-memory stores */
      int b = tb, j = tj_in, i = ti_in;
      while (b < nbl) {
        T v[8];
        int pos[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          pos[u] = -1;
          if (b < nbl) {
            v[u] = data[s_off[b] + j * m + i];
            pos[u] = b * bsz + j * ld + i;
          }
          i += si_in;
          if (i >= m) {
            i -= m;
            ++j;
          }
          j += sj_in;
          if (j >= n) {
            j -= n;
            ++b;
          }
          b += sb;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          if (pos[u] >= 0) buf[pos[u]] = v[u];
        }
      }
    }
    __syncthreads();
    {
      int b = tb, i = ti_out, j = tj_out;
      while (b < nbl) { /* output (j, i) of the n x m result at i*n + j = input (i, j) */
        data[s_off[b] + i * n + j] = buf[b * bsz + j * ld + i];
        j += sj_out;
        if (j >= n) {
          j -= n;
          ++i;
        }
        i += si_out;
        if (i >= m) {
          i -= m;
          ++b;
        }
        b += sb;
      }
    }
    __syncthreads();
  }
}

/* ---------------------------------------------------------------------------------- norms */

__global__ void xs_norms_kernel(const double* __restrict__ mat, int nblks, const int* __restrict__ offsets,
  const int* __restrict__ nelems, float* __restrict__ norms) {
  const int lane = threadIdx.x & 31;
  const int blk = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (blk >= nblks) return;
  const double* const p = mat + offsets[blk];
  const int ne = nelems[blk];
  double s = 0.0;
  for (int e = lane; e < ne; e += 32) s = fma(p[e], p[e], s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (0 == lane) norms[blk] = (float)sqrt(s);
}

/* ------------------------------------------------------------------------ FP64 peak probe */

__global__ void xs_dmma_peak_kernel(double* out, int iters) {
  const double a = 1.0 + threadIdx.x * 1e-6, b = 1.0 - threadIdx.x * 1e-6;
  double c[8][2];
#pragma unroll
  for (int u = 0; u < 8; ++u) c[u][0] = c[u][1] = 0.0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 8; ++u) dmma_m8n8k4(c[u][0], c[u][1], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int u = 0; u < 8; ++u) s += c[u][0] + c[u][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" {

int xs_smm_f64_specialized(int m, int n, int k, int* mt_kp_pairs, int capacity) {
  int count = 0;
  auto scan = [&](const SpecEntry* table, size_t len) {
    for (size_t i = 0; i < len; ++i) {
      const SpecEntry& e = table[i];
      if (e.m == m && e.n == n && e.k == k) {
        if (count < capacity && nullptr != mt_kp_pairs) {
          mt_kp_pairs[3 * count + 0] = e.mt;
          mt_kp_pairs[3 * count + 1] = e.nt;
          mt_kp_pairs[3 * count + 2] = e.kp;
        }
        ++count;
      }
    }
  };
  scan(staged_table, sizeof(staged_table) / sizeof(*staged_table)); /* staged kernels first (kp = 0) */
  scan(spec_table, sizeof(spec_table) / sizeof(*spec_table));
  return count;
}

int xs_smm_fma_supported(int m, int n, int k) {
  const FmaEntry* const f = find_fma(m, n, k);
  if (nullptr == f) return 0;
  /* the lane grid covers the block; its ring (4 warps per CTA) must also fit shared memory: the check
     launch_fma makes, without a device call */
  return (fma_smem_bytes(m, n, k, f->D, f->regs, f->slack, 4) <= 227 * 1024) ? 1 : 0;
}

size_t xs_smm_f64_scratch_bytes(int stack_size, int m, int n, int k, const xs_smm_params_t* params) {
  SmmPlan pl;
  if (stack_size > xs_stack_group_max()) stack_size = xs_stack_group_max(); /* processed in parts */
  if (0 >= stack_size || 0 != plan_smm(stack_size, m, n, k, params, &pl)) return 0;
  return pl.total;
}

int xs_launch_smm_f64(const int* dev_stack, int S, const double* a, const double* b, double* c, int m, int n, int k,
  const xs_smm_params_t* prm, void* scratch, size_t scratch_bytes, void* stream) {
  return xs_launch_smm_f64_ex(dev_stack, S, 0, 1.0, a, b, c, m, n, k, prm, scratch, scratch_bytes, stream);
}

/* Operand bytes (A and B blocks, counted per parameter record) that a stack kernel prefetches into L2
   while the grouping runs: 64 MB, about half the L2, so that the prefetched blocks are not evicted
   before they are used; LIBXSTREAM_B200_PREFETCH_MB overrides it (0: no prefetch). */
static long long prefetch_budget() {
  static const long long v = []() -> long long {
    const char* const env = getenv("LIBXSTREAM_B200_PREFETCH_MB");
    const long long mb = (nullptr != env) ? atoll(env) : 64;
    return (0 < mb) ? (mb << 20) : 0;
  }();
  return v;
}

/* Sets the prefetch fields of tk: the first records of the stack whose A and B blocks fit the budget.
   Records of less than 1 KB of A and B get none: their prefetches cost more than they save (5x5x5 at
   10^5 entries measured 3 % slower with them, 8x8x8 unchanged, 22^3..32^3 1.4-2.3 % faster). */
static void set_prefetch(StackTask& tk, const int* dev_stack, int S, int format, long long budget) {
  const long long per = (long long)tk.k * (tk.m + tk.n) * (long long)sizeof(double);
  if (per < 1024) budget = 0;
  tk.raw = dev_stack;
  tk.rstride = (0 != format) ? 6 : 3;
  tk.rbase = (0 != format) ? 3 : 0;
  tk.rshift = (0 != format) ? 0 : -1;
  tk.npf = (0 < per) ? (int)((budget / per < S) ? budget / per : S) : 0;
}

int xs_launch_smm_f64_ex(const int* dev_stack, int S, int format, double alpha, const double* a, const double* b, double* c,
  int m, int n, int k, const xs_smm_params_t* prm, void* scratch, size_t scratch_bytes, void* stream) {
  SmmPlan pl;
  cudaStream_t s = (cudaStream_t)stream;
  if (0 >= S) return 0;
  const int smax = xs_stack_group_max();
  if (S > smax) { /* C += A*B is additive over the stack: run it in consecutive parts */
    for (int off = 0; off < S; off += smax) {
      const int r = xs_launch_smm_f64_ex(dev_stack + (0 != format ? 6 : 3) * (size_t)off, min(smax, S - off), format, alpha, a, b,
        c, m, n, k, prm, scratch, scratch_bytes, stream);
      if (0 != r) return r;
    }
    return 0;
  }
  if (0 != plan_smm(S, m, n, k, prm, &pl) || scratch_bytes < pl.total || nullptr == scratch) return (int)cudaErrorInvalidValue;
  char* const base = (char*)scratch;
  unsigned* const keys_in = (unsigned*)(base + pl.off_keys_in);
  unsigned* const keys_tmp = (unsigned*)(base + pl.off_keys_tmp);
  unsigned* const keys_out = (unsigned*)(base + pl.off_keys_out);
  unsigned long long* const vals_in = (unsigned long long*)(base + pl.off_vals_in);
  unsigned long long* const vals_tmp = (unsigned long long*)(base + pl.off_vals_tmp);
  unsigned long long* const vals_out = (unsigned long long*)(base + pl.off_vals_out);
  int* const seglist = (int*)(base + pl.off_seglist);
  void* const sort_scratch = base + pl.off_sort;
  int* const arrive = (int*)(base + pl.off_arrive);
  void* prof = xs_profile_begin(s);
  const int r = xs_stack_group_ex(dev_stack, S, format, (unsigned)(m * n), keys_in, vals_in, keys_tmp, vals_tmp, keys_out,
    vals_out, seglist, arrive, 3 * pl.ngroups * pl.nsub, pl.L * pl.W, sort_scratch, s);
  if (0 != r) return r;
  xs_profile_end(prof, "sort", 0.0, 48.0 * S, s);
  StackTask tk = {};
  tk.alpha = alpha;
  tk.a = a;
  tk.b = b;
  tk.c = c;
  tk.keys = keys_out;
  tk.vals = vals_out;
  tk.pieces = (double*)(base + pl.off_pieces);
  tk.S = S;
  tk.m = m;
  tk.n = n;
  tk.k = k;
  tk.L = pl.L;
  tk.nchunks = pl.nchunks;
  tk.ngroups = pl.ngroups;
  tk.nsub_n = pl.nsub_n;
  tk.nsub = pl.nsub;
  tk.arrive = arrive; /* CTA-crossing segments are combined inside the stack kernel */
  tk.Ls[0] = pl.Ls[0];
  tk.Ls[1] = pl.Ls[1];
  tk.Ls[2] = pl.Ls[2];
  tk.slotn = pl.slotn;
  set_prefetch(tk, dev_stack, S, format, prefetch_budget());
  const launch_fn_t fn = find_launcher(m, n, k, prm);
  return (int)fn(pl, tk, seglist, xs_sort_error_flag(sort_scratch), s, nullptr);
}

size_t xs_smm_batch_scratch_bytes(const libxstream_b200_stack_t* stacks, int nstacks) {
  UniPlan up;
  if (0 >= plan_uni(stacks, nstacks, &up)) return 0;
  return up.total;
}

/* A batch of stacks: one grouping launch for up to XS_MAX_BATCH parts (more only when the parts
   exceed the tiles one grouping launch takes), then one launch of the unified persistent kernel for
   every part; no combine launch. */
int xs_launch_smm_batch(const libxstream_b200_stack_t* st, int ns, void* scratch, size_t scratch_bytes, void* stream) {
  UniPlan up;
  cudaStream_t s = (cudaStream_t)stream;
  const int np = plan_uni(st, ns, &up);
  if (0 > np) return (int)cudaErrorInvalidValue;
  if (0 == np) return 0;
  if (scratch_bytes < up.total || nullptr == scratch) return (int)cudaErrorInvalidValue;
  char* const base = (char*)scratch;
  unsigned* const k0 = (unsigned*)(base + up.off_keys_in);
  unsigned* const k1 = (unsigned*)(base + up.off_keys_tmp);
  unsigned* const kout = (unsigned*)(base + up.off_keys_out);
  unsigned long long* const v0 = (unsigned long long*)(base + up.off_vals_in);
  unsigned long long* const v1 = (unsigned long long*)(base + up.off_vals_tmp);
  unsigned long long* const vout = (unsigned long long*)(base + up.off_vals_out);
  int* const seglist = (int*)(base + up.off_seglist);
  double* const pieces = (double*)(base + up.off_pieces);
  void* const sort_scratch = base + up.off_sort;
  int* const arrive = (int*)(base + up.off_arrive);
  /* grouping: one control block for the call, then as few grouping launches as the tiles need; the
     first one also zeroes every part's arrival counters */
  int r = xs_sort_clear_ctl(sort_scratch, up.nparts, s);
  if (0 != r) return r;
  void* prof = xs_profile_begin(s);
  xs_sort_batch_t sb;
  memset(&sb, 0, sizeof(sb));
  sb.zero = (0 < up.narrive) ? arrive : nullptr;
  sb.nzero = (int)up.narrive;
  int tiles = 0;
  const int launch_tiles = xs_sort_launch_tiles(), tile_entries = xs_sort_tile_entries(1);
  for (int q = 0; q <= up.nparts; ++q) {
    const int nt = (q < up.nparts) ? (up.part[q].S + tile_entries - 1) / tile_entries : 0;
    if (q == up.nparts || sb.nstacks == XS_MAX_BATCH || tiles + nt > launch_tiles) {
      if (0 < sb.nstacks) {
        r = xs_stack_group_batch(&sb, k0, v0, k1, v1, kout, vout, seglist, sort_scratch, s);
        if (0 != r) return r;
        sb.zero = nullptr;
        sb.nzero = 0;
      }
      sb.nstacks = 0;
      tiles = 0;
    }
    if (q == up.nparts) break;
    const UniPart& p = up.part[q];
    sb.gidx[sb.nstacks] = q;
    sb.stack[sb.nstacks] = st[p.stack].dev_param_stack + 3 * (size_t)p.first;
    sb.format[sb.nstacks] = 0;
    sb.S[sb.nstacks] = p.S;
    sb.off[sb.nstacks] = (int)up.off_part[q];
    sb.blk[sb.nstacks] = (unsigned)(st[p.stack].m * st[p.stack].n);
    ++sb.nstacks;
    tiles += nt;
  }
  xs_profile_end(prof, "sort", 0.0, 48.0 * up.ntotal, s);
  /* task table in item order (heaviest items first) */
  BatchTasks bt;
  memset(&bt, 0, sizeof(bt));
  double flops = 0, bytes = 0, pf_total = 0;
  for (int i = 0; i < up.nparts; ++i) {
    const libxstream_b200_stack_t& d = st[up.part[i].stack];
    pf_total += 8.0 * d.k * (double)(d.m + d.n) * up.part[i].S;
  }
  /* the prefetch budget is shared by the parts in proportion to their operand bytes */
  const double pf_scale = (pf_total > (double)prefetch_budget()) ? (double)prefetch_budget() / pf_total : 1.0;
  for (int i = 0; i < up.nparts; ++i) {
    const int q = up.order[i];
    const UniPart& p = up.part[q];
    const libxstream_b200_stack_t& d = st[p.stack];
    StackTask tk = {};
    tk.alpha = 1.0;
    tk.a = (const double*)d.a;
    tk.b = (const double*)d.b;
    tk.c = (double*)d.c;
    tk.keys = kout + up.off_part[q];
    tk.vals = vout + up.off_part[q];
    tk.pieces = pieces + up.pieces_off[q];
    tk.arrive = arrive + up.arrive_off[q];
    tk.S = p.S;
    tk.m = d.m;
    tk.n = d.n;
    tk.k = d.k;
    tk.L = p.L;
    tk.Ls[0] = tk.Ls[1] = tk.Ls[2] = p.L;
    tk.slotn = 1 << 29;
    tk.nchunks = (p.S + p.L - 1) / p.L;
    tk.ngroups = p.ngroups;
    tk.nsub_n = p.nsub_n;
    tk.nsub = p.nsub;
    tk.cls = (p.mt - 1) * 4 + (p.nt - 1);
    tk.kind = p.kind;
    tk.sid = q;
    tk.item_begin = bt.nitems;
    set_prefetch(tk, d.dev_param_stack + 3 * (size_t)p.first, p.S, 0,
      (long long)(pf_scale * 8.0 * d.k * (double)(d.m + d.n) * p.S));
    bt.t[bt.ntasks++] = tk;
    bt.nitems += p.ngroups * p.nsub;
    flops += 2.0 * d.m * d.n * d.k * (double)p.S;
    bytes += 8.0 * p.S * ((double)d.m * d.k + (double)d.k * d.n + 2.0 * d.m * d.n);
  }
  const int grid = max(1, min(bt.nitems, up.occ * xs_sm_count()));
  prof = xs_profile_begin(s);
  r = (int)pdl_launch(xs_smm_uni_kernel, grid, 32 * kUniW, kUniSmem, s, bt, seglist, xs_sort_queue_counter(sort_scratch, 0),
    (unsigned*)xs_sort_error_flag(sort_scratch), xs_device_error_ptr(), xs_wait_limit());
  xs_profile_end(prof, "smm_batch", flops, bytes, s);
  return r;
}

int xs_launch_transpose(const int* trs, int offset, int S, void* data, int esize, int m, int n, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (0 >= S) return 0;
  const int mn = m * n;
  const size_t bbytes = (size_t)(m | 1) * n * esize;
  /* blocks per CTA: up to 24 KB of shared memory, but at least one CTA per SM when there are blocks
     enough (small blocks would otherwise give too few CTAs) */
  int nb = (int)((24 * 1024) / bbytes);
  if (nb < 1) nb = 1;
  const int per_sm = (S + xs_sm_count() - 1) / xs_sm_count();
  if (nb > per_sm) nb = per_sm;
  if (nb > 256) nb = 256; /* block offsets staged per CTA */
  const size_t smem = bbytes * nb;
  if (smem > 227 * 1024) return (int)cudaErrorInvalidValue; /* a block larger than shared memory */
  const int threads = (nb * mn >= 256) ? 256 : ((nb * mn + 31) / 32) * 32;
  int grid = (S + nb - 1) / nb;
  if (grid > 16 * xs_sm_count()) grid = 16 * xs_sm_count();
  cudaError_t r;
  void* const prof = xs_profile_begin(s);
  if (8 == esize) {
    if (cudaSuccess != (r = (cudaError_t)xs_func_smem((const void*)xs_transpose_kernel<unsigned long long>, smem))) return (int)r;
    xs_transpose_kernel<unsigned long long><<<grid, threads, smem, s>>>(trs, offset, S, (unsigned long long*)data, m, n, nb);
  }
  else if (4 == esize) {
    if (cudaSuccess != (r = (cudaError_t)xs_func_smem((const void*)xs_transpose_kernel<unsigned>, smem))) return (int)r;
    xs_transpose_kernel<unsigned><<<grid, threads, smem, s>>>(trs, offset, S, (unsigned*)data, m, n, nb);
  }
  else return (int)cudaErrorInvalidValue;
  r = cudaGetLastError();
  xs_profile_end(prof, "trans", 0.0, 2.0 * esize * (double)mn * S, s);
  return (int)r;
}

int xs_launch_norms(const double* mat, int nblks, const int* offsets, const int* nelems, float* norms, void* stream) {
  if (0 >= nblks) return 0;
  void* const prof = xs_profile_begin(stream);
  xs_norms_kernel<<<(nblks + 7) / 8, 256, 0, (cudaStream_t)stream>>>(mat, nblks, offsets, nelems, norms);
  const cudaError_t r = cudaGetLastError();
  xs_profile_end(prof, "norms", 0.0, 0.0, stream);
  return (int)r;
}

double xs_fp64_peak_tflops(void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const int sms = xs_sm_count(), threads = 256, blocks = sms * 8, iters = 4096;
  double* out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float ms = 0.f;
  double result = -1.0;
  if (cudaSuccess != cudaMallocAsync((void**)&out, sizeof(double) * blocks * threads, s)) return -1.0;
  if (cudaSuccess == cudaEventCreate(&e0) && cudaSuccess == cudaEventCreate(&e1)) {
    xs_dmma_peak_kernel<<<blocks, threads, 0, s>>>(out, 64); /* warm-up */
    cudaEventRecord(e0, s);
    xs_dmma_peak_kernel<<<blocks, threads, 0, s>>>(out, iters);
    cudaEventRecord(e1, s);
    if (cudaSuccess == cudaEventSynchronize(e1) && cudaSuccess == cudaEventElapsedTime(&ms, e0, e1) && 0 < ms) {
      const double flops = 2.0 * 8 * 8 * 4 * 8 * (double)iters * blocks * (threads / 32);
      result = flops / (ms * 1e-3) * 1e-12;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFreeAsync(out, s);
  cudaStreamSynchronize(s);
  return result;
}

}  // extern "C"
