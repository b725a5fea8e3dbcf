/*
 * Exhaustive autotuner of the plain FP64 stack kernel (and the timing of the Ozaki form), the
 * counterpart of the reference's tuning driver (samples/smm/tune_multiply.py: OpenTuner search over
 * the JIT parameters, records written as samples/smm/params/tune_multiply_*.csv). Here the space is
 * small and precompiled, so it is searched exhaustively on the device: for one shape and stack size
 * the tuner builds synthetic pools and a stack (counter-based hash, reproducible from the seed),
 * times every candidate (tile class MT x NT with MT <= ceil(m/8), NT <= ceil(n/8), both <= 4, and
 * k-panel KP in {2, 4}; chunk length sized per launch) with CUDA events and returns all times, so
 * that callers can pick the best and train the predictor on the whole sweep.
 */
#include "internal.h"
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

namespace {

__device__ __forceinline__ uint32_t hash32(uint32_t x) { /* lowbias32 integer hash (public domain) */
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

/* x[i] = uniform in [-1, 1) from hash(seed, i) */
__global__ void xs_tune_fill(double* __restrict__ x, size_t n, uint32_t seed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t h = hash32((uint32_t)i * 2654435761u ^ hash32(seed ^ (uint32_t)(i >> 32)));
    x[i] = (double)h * (2.0 / 4294967296.0) - 1.0;
  }
}

/* S triples (1-based block offsets): a, b uniform over the pools, c skewed towards low block ids
   (floor(nc * u^2)) so that C blocks receive uneven numbers of updates */
__global__ void xs_tune_stack(int* __restrict__ stack, int S, int na, int nb, int nc, int mk, int kn, int mn, uint32_t seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S) return;
  const uint32_t h0 = hash32(seed ^ hash32(3u * (uint32_t)i + 0u)), h1 = hash32(seed ^ hash32(3u * (uint32_t)i + 1u));
  const uint32_t h2 = hash32(seed ^ hash32(3u * (uint32_t)i + 2u));
  const double u = (double)h2 / 4294967296.0;
  const int c = min(nc - 1, (int)(nc * u * u));
  stack[3 * i + 0] = (int)(h0 % (uint32_t)na) * mk + 1;
  stack[3 * i + 1] = (int)(h1 % (uint32_t)nb) * kn + 1;
  stack[3 * i + 2] = c * mn + 1;
}

int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

}  // namespace

extern "C" {

/* Candidate configurations of the plain kernels for (m, n): writes up to cap (mt, nt, kp) triples,
   the DMMA tile classes first, then (1, 1, XS_KP_FMA) when an FMA lane grid covers the block (a k
   whose ring does not fit shared memory is timed as not applicable). */
int xs_tune_candidates(int m, int n, int* mt_nt_kp, int cap) {
  const int mt_max = clampi((m + 7) / 8, 1, 4), nt_max = clampi((n + 7) / 8, 1, 4);
  int count = 0;
  auto add = [&](int mt, int nt, int kp) {
    if (count < cap && nullptr != mt_nt_kp) {
      mt_nt_kp[3 * count + 0] = mt;
      mt_nt_kp[3 * count + 1] = nt;
      mt_nt_kp[3 * count + 2] = kp;
    }
    ++count;
  };
  for (int mt = 1; mt <= mt_max; ++mt) {
    for (int nt = 1; nt <= nt_max; ++nt) {
      for (int kp = 2; kp <= 4; kp += 2) add(mt, nt, kp);
    }
  }
  if (xs_smm_fma_supported(m, n, 1)) add(1, 1, XS_KP_FMA);
  return count;
}

/* Times every candidate (and, with ozaki_slices > 0 and m, n, k <= 64, the Ozaki form with that
   many slices, triangle of pairs) on synthetic data; ms_out[i] = milliseconds per call of candidate
   i (candidates in xs_tune_candidates order, the Ozaki time last; -1 for a candidate that does not
   take this shape). Returns the number of times written, or a negative CUDA error. Synchronous;
   allocates and frees its own buffers. */
int xs_tune(int m, int n, int k, int S, int reps, int ozaki_slices, uint32_t seed, float* ms_out, int cap, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (m < 1 || n < 1 || k < 1 || S < 1 || reps < 1 || nullptr == ms_out) return -(int)cudaErrorInvalidValue;
  int cand[3 * 33];
  const int nc_cand = xs_tune_candidates(m, n, cand, 33);
  const int with_oz = (ozaki_slices > 0 && m <= 64 && n <= 64 && k <= 64) ? 1 : 0;
  if (cap < nc_cand + with_oz) return -(int)cudaErrorInvalidValue;
  const int na = clampi(S / 8, 16, 8192), nb = na, nc = clampi(S / 32, 8, 2048);
  const size_t mk = (size_t)m * k, kn = (size_t)k * n, mn = (size_t)m * n;
  size_t scratch_bytes = 0;
  for (int i = 0; i < nc_cand; ++i) {
    xs_smm_params_t p = {0, cand[3 * i], cand[3 * i + 1], cand[3 * i + 2], 0, 4, 0};
    const size_t b = xs_smm_f64_scratch_bytes(S, m, n, k, &p); /* 0: not runnable (an FMA candidate for this k) */
    if (b > scratch_bytes) scratch_bytes = b;
  }
  if (with_oz) {
    const size_t b = xs_smm_ozaki_scratch_bytes(S, m, n, k, na, nb, ozaki_slices);
    if (b > scratch_bytes) scratch_bytes = b;
  }
  double *a = nullptr, *b = nullptr, *c = nullptr;
  int* stack = nullptr;
  void* scratch = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int r = (int)cudaMallocAsync((void**)&a, sizeof(double) * mk * na, s);
  if (0 == r) r = (int)cudaMallocAsync((void**)&b, sizeof(double) * kn * nb, s);
  if (0 == r) r = (int)cudaMallocAsync((void**)&c, sizeof(double) * mn * nc, s);
  if (0 == r) r = (int)cudaMallocAsync((void**)&stack, sizeof(int) * 3 * (size_t)S, s);
  if (0 == r) r = (int)cudaMallocAsync(&scratch, scratch_bytes, s);
  if (0 == r) r = (int)cudaEventCreate(&e0);
  if (0 == r) r = (int)cudaEventCreate(&e1);
  if (0 == r) {
    xs_tune_fill<<<1024, 256, 0, s>>>(a, mk * na, seed);
    xs_tune_fill<<<1024, 256, 0, s>>>(b, kn * nb, seed + 1u);
    xs_tune_stack<<<(S + 255) / 256, 256, 0, s>>>(stack, S, na, nb, nc, (int)mk, (int)kn, (int)mn, seed + 2u);
    r = (int)cudaMemsetAsync(c, 0, sizeof(double) * mn * nc, s);
  }
  for (int i = 0; i < nc_cand + with_oz && 0 == r; ++i) {
    const bool oz = (i == nc_cand);
    xs_smm_params_t p = {0, oz ? 1 : cand[3 * i], oz ? 1 : cand[3 * i + 1], oz ? 2 : cand[3 * i + 2], 0, 4, 0};
    if (!oz && XS_KP_FMA == p.kp && !xs_smm_fma_supported(m, n, k)) {
      ms_out[i] = -1.f; /* the FMA kernel does not take this shape */
      continue;
    }
    auto call = [&]() -> int {
      if (oz) {
        return xs_launch_smm_ozaki(stack, S, m, n, k, a, na, b, nb, c, ozaki_slices, ozaki_slices - 1, scratch, scratch_bytes, s);
      }
      return xs_launch_smm_f64(stack, S, a, b, c, m, n, k, &p, scratch, scratch_bytes, s);
    };
    r = call(); /* warm-up */
    if (0 == r) r = (int)cudaEventRecord(e0, s);
    for (int rep = 0; rep < reps && 0 == r; ++rep) r = call();
    if (0 == r) r = (int)cudaEventRecord(e1, s);
    if (0 == r) r = (int)cudaEventSynchronize(e1);
    float ms = 0.f;
    if (0 == r) r = (int)cudaEventElapsedTime(&ms, e0, e1);
    ms_out[i] = ms / (float)reps;
  }
  const int r2 = (int)cudaStreamSynchronize(s);
  if (nullptr != e0) cudaEventDestroy(e0);
  if (nullptr != e1) cudaEventDestroy(e1);
  cudaFreeAsync(scratch, s);
  cudaFreeAsync(stack, s);
  cudaFreeAsync(c, s);
  cudaFreeAsync(b, s);
  cudaFreeAsync(a, s);
  if (0 == r) r = r2;
  return (0 == r) ? nc_cand + with_oz : -r;
}

}  // extern "C"
