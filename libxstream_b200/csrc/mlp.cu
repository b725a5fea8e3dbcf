/*
 * Learned parameter predictor: a 3-layer MLP (FP32, width 64) that maps a stack's shape
 * (m, n, k, stack size, exponent spread of the inputs) to the autotuner's best kernel configuration
 * (one of 32 DMMA tile classes MT x NT x KP, or the register-blocked FMA kernel) and to the
 * plain-vs-Ozaki choice. The counterpart of the
 * reference's learned parameter prediction (samples/smm/tune_multiply.py driving LIBXS predict
 * models, params/*.bin), rebuilt as this library's own network and kernels.
 *
 * Network: x (27 features) -> h1 = relu(x W1 + b1) (64) -> h2 = relu(h1 W2 + b2) (64) -> y = h2 W3 + b3
 * (34 outputs: 32 DMMA configuration logits, the FMA kernel's logit, 1 Ozaki logit). Features: one-hot ceil(m/8) and ceil(n/8)
 * (the 8x8 DMMA fragment counts, 1..10, which decide the tile classes), log2 k / 6.5, (k mod 8)/8,
 * log10 S / 5, spread / 40, log2(m n k S) / 40, (m mod 8)/8, (n mod 8)/8.
 * Loss per sample: cross-entropy of the masked softmax p against the soft target
 * q_c ~ exp(-(r_c - 1) / 0.02) over the applicable configurations, r_c = t_c / t_best (0 when the
 * configuration does not apply: configurations within a few percent of the best share the target
 * mass), plus the binary cross-entropy of the Ozaki logit against "the Ozaki form was faster" when
 * that was measured.
 * Training runs on the device with the kernels below (forward, loss gradient, backward, weight
 * gradients with a fixed-order reduction so that training is deterministic, Adam); inference is
 * the same forward pass followed by a masked argmax.
 */
#include "internal.h"
#include <cuda_runtime.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define XS_MLP_F 27
#define XS_MLP_H 64
#define XS_MLP_K 33 /* configurations: 32 DMMA tile classes, then the FMA kernel (index 32) */
#define XS_MLP_O (XS_MLP_K + 1)
#define XS_MLP_NW (XS_MLP_F * XS_MLP_H + XS_MLP_H + XS_MLP_H * XS_MLP_H + XS_MLP_H + XS_MLP_H * XS_MLP_O + XS_MLP_O)

namespace {

constexpr int F = XS_MLP_F, H = XS_MLP_H, K = XS_MLP_K, O = XS_MLP_O, NW = XS_MLP_NW;
constexpr int oW1 = 0, ob1 = oW1 + F * H, oW2 = ob1 + H, ob2 = oW2 + H * H, oW3 = ob2 + H, ob3 = oW3 + H * O;
constexpr int kWChunks = 16; /* sample chunks of the weight-gradient reduction */

__host__ __device__ inline int mt_max_of(int m) { return min(4, max(1, (m + 7) / 8)); }

/* configuration c = (mt-1)*8 + (nt-1)*2 + (kp == 4) applies to (m, n); c = 32, the FMA kernel, where the
   caller says it does (fma_ok: its lane grids cover the block and its ring fits shared memory) */
constexpr int kFmaConfig = 32;
__host__ __device__ inline bool config_valid(int c, int m, int n, bool fma_ok) {
  return (kFmaConfig == c) ? fma_ok : ((c >> 3) + 1 <= mt_max_of(m) && ((c >> 1) & 3) + 1 <= mt_max_of(n));
}

__device__ void features(const int* raw, float* x) {
  const float k = (float)raw[2], S = fmaxf((float)raw[3], 1.f);
  const int fm = min(10, max(1, (raw[0] + 7) / 8)), fn = min(10, max(1, (raw[1] + 7) / 8));
  for (int i = 0; i < 20; ++i) x[i] = 0.f;
  x[fm - 1] = 1.f;
  x[10 + fn - 1] = 1.f;
  x[20] = log2f(k) / 6.5f;
  x[21] = (float)(raw[2] & 7) / 8.f;
  x[22] = log10f(S) / 5.f;
  x[23] = (float)raw[4] / 40.f;
  x[24] = (log2f((float)raw[0]) + log2f((float)raw[1]) + log2f(k) + log2f(S)) / 40.f;
  x[25] = (float)(raw[0] & 7) / 8.f;
  x[26] = (float)(raw[1] & 7) / 8.f;
}

__device__ void load_weights(const float* __restrict__ W, float* sW) {
  for (int i = threadIdx.x; i < NW; i += blockDim.x) sW[i] = W[i];
  __syncthreads();
}

/* forward pass of one sample from smem weights; h1, h2 may be null (inference) */
__device__ void forward_one(const float* sW, const float* x, float* h1o, float* h2o, float* y) {
  float h1[H], h2[H];
#pragma unroll 4
  for (int h = 0; h < H; ++h) {
    float s = sW[ob1 + h];
#pragma unroll
    for (int f = 0; f < F; ++f) s = fmaf(x[f], sW[oW1 + f * H + h], s);
    h1[h] = fmaxf(s, 0.f);
  }
  for (int j = 0; j < H; ++j) {
    float s = sW[ob2 + j];
#pragma unroll 8
    for (int h = 0; h < H; ++h) s = fmaf(h1[h], sW[oW2 + h * H + j], s);
    h2[j] = fmaxf(s, 0.f);
  }
  for (int o = 0; o < O; ++o) {
    float s = sW[ob3 + o];
#pragma unroll 8
    for (int j = 0; j < H; ++j) s = fmaf(h2[j], sW[oW3 + j * O + o], s);
    y[o] = s;
  }
  if (nullptr != h1o) {
    for (int h = 0; h < H; ++h) h1o[h] = h1[h];
    for (int j = 0; j < H; ++j) h2o[j] = h2[j];
  }
}

__global__ void xs_mlp_fwd(const float* __restrict__ W, const int* __restrict__ raw, int N, float* __restrict__ X,
  float* __restrict__ H1, float* __restrict__ H2, float* __restrict__ Y) {
  extern __shared__ float sW[];
  load_weights(W, sW);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  float x[F];
  features(raw + 5 * (size_t)i, x);
  for (int f = 0; f < F; ++f) X[(size_t)i * F + f] = x[f];
  forward_one(sW, x, H1 + (size_t)i * H, H2 + (size_t)i * H, Y + (size_t)i * O);
}

/* loss and dL/dy per sample (already divided by N) */
constexpr float kTargetTemp = 0.02f;
__global__ void xs_mlp_loss(const float* __restrict__ Y, const float* __restrict__ R, const float* __restrict__ Z, int N,
  float* __restrict__ dY, float* __restrict__ loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float* y = Y + (size_t)i * O;
  const float* r = R + (size_t)i * K;
  float ymax = -INFINITY;
  for (int c = 0; c < K; ++c) {
    if (r[c] > 0.f) ymax = fmaxf(ymax, y[c]);
  }
  float zp = 0.f, zq = 0.f;
  for (int c = 0; c < K; ++c) {
    if (r[c] > 0.f) {
      zp += expf(y[c] - ymax);
      zq += expf(-(r[c] - 1.f) / kTargetTemp);
    }
  }
  const float lzp = logf(zp);
  float* dy = dY + (size_t)i * O;
  const float inv = 1.f / (float)N;
  float l = 0.f;
  for (int c = 0; c < K; ++c) {
    if (r[c] > 0.f) {
      const float q = expf(-(r[c] - 1.f) / kTargetTemp) / zq, lp = y[c] - ymax - lzp;
      l -= q * lp;
      dy[c] = (expf(lp) - q) * inv;
    }
    else dy[c] = 0.f;
  }
  const float zi = Z[i];
  if (zi >= 0.f) {
    const float yk = y[K];
    const float sg = 1.f / (1.f + expf(-yk));
    l += fmaxf(yk, 0.f) - yk * zi + log1pf(expf(-fabsf(yk))); /* BCE with logits */
    dy[K] = (sg - zi) * inv;
  }
  else dy[K] = 0.f;
  loss[i] = l;
}

__global__ void xs_mlp_bwd(const float* __restrict__ W, const float* __restrict__ H1, const float* __restrict__ H2,
  const float* __restrict__ dY, int N, float* __restrict__ dH1, float* __restrict__ dH2) {
  extern __shared__ float sW[];
  load_weights(W, sW);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float* dy = dY + (size_t)i * O;
  const float* h1 = H1 + (size_t)i * H;
  const float* h2 = H2 + (size_t)i * H;
  float g2[H];
  for (int j = 0; j < H; ++j) {
    float s = 0.f;
    for (int o = 0; o < O; ++o) s = fmaf(dy[o], sW[oW3 + j * O + o], s);
    g2[j] = (h2[j] > 0.f) ? s : 0.f;
    dH2[(size_t)i * H + j] = g2[j];
  }
  for (int h = 0; h < H; ++h) {
    float s = 0.f;
#pragma unroll 8
    for (int j = 0; j < H; ++j) s = fmaf(g2[j], sW[oW2 + h * H + j], s);
    dH1[(size_t)i * H + h] = (h1[h] > 0.f) ? s : 0.f;
  }
}

/* Partial weight gradients over sample chunk blockIdx.y, in sample order (deterministic). */
__global__ void xs_mlp_wgrad(const float* __restrict__ X, const float* __restrict__ H1, const float* __restrict__ H2,
  const float* __restrict__ dH1, const float* __restrict__ dH2, const float* __restrict__ dY, int N, float* __restrict__ part) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= NW) return;
  const int per = (N + kWChunks - 1) / kWChunks, i0 = blockIdx.y * per, i1 = min(N, i0 + per);
  const float *in, *g;
  int ld_in, ld_g, a, b;
  if (w < ob1) { a = w / H; b = w % H; in = X; ld_in = F; g = dH1; ld_g = H; }
  else if (w < oW2) { a = -1; b = w - ob1; in = nullptr; ld_in = 0; g = dH1; ld_g = H; }
  else if (w < ob2) { a = (w - oW2) / H; b = (w - oW2) % H; in = H1; ld_in = H; g = dH2; ld_g = H; }
  else if (w < oW3) { a = -1; b = w - ob2; in = nullptr; ld_in = 0; g = dH2; ld_g = H; }
  else if (w < ob3) { a = (w - oW3) / O; b = (w - oW3) % O; in = H2; ld_in = H; g = dY; ld_g = O; }
  else { a = -1; b = w - ob3; in = nullptr; ld_in = 0; g = dY; ld_g = O; }
  float s = 0.f;
  if (a >= 0) {
    for (int i = i0; i < i1; ++i) s = fmaf(in[(size_t)i * ld_in + a], g[(size_t)i * ld_g + b], s);
  }
  else {
    for (int i = i0; i < i1; ++i) s += g[(size_t)i * ld_g + b];
  }
  part[(size_t)blockIdx.y * NW + w] = s;
}

__global__ void xs_mlp_reduce(const float* __restrict__ part, float* __restrict__ G) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= NW) return;
  float s = 0.f;
  for (int c = 0; c < kWChunks; ++c) s += part[(size_t)c * NW + w];
  G[w] = s;
}

__global__ void xs_mlp_adam(float* __restrict__ W, const float* __restrict__ G, float* __restrict__ M1, float* __restrict__ M2,
  int t, float lr) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= NW) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float g = G[w];
  const float m = b1 * M1[w] + (1.f - b1) * g, v = b2 * M2[w] + (1.f - b2) * g * g;
  M1[w] = m;
  M2[w] = v;
  const float mh = m / (1.f - powf(b1, (float)t)), vh = v / (1.f - powf(b2, (float)t));
  W[w] -= lr * mh / (sqrtf(vh) + eps);
}

/* Inference only: features, forward pass and selection per sample with the activations in registers
   (layer by layer over the inputs, four or two weights per shared-memory load), writing nothing but
   the selected configuration, its probability and the Ozaki probability. The same fmaf sequence per
   output as forward_one, so the logits are bitwise those of xs_mlp_fwd. */
__global__ void __launch_bounds__(128) xs_mlp_infer(const float* __restrict__ W, const int* __restrict__ raw,
  const unsigned char* __restrict__ fma_ok, int N, unsigned char* __restrict__ cfg, float* __restrict__ conf,
  float* __restrict__ pz) {
  extern __shared__ __align__(16) float sW[];
  load_weights(W, sW);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  static_assert(0 == (oW1 % 4) && 0 == (oW2 % 4) && 0 == (H % 4) && 0 == (oW3 % 2) && 0 == (O % 2), "vector weight loads");
  float x[F];
  features(raw + 5 * (size_t)i, x);
  float h1[H], h2[H], y[O];
#pragma unroll
  for (int h = 0; h < H; ++h) h1[h] = sW[ob1 + h];
#pragma unroll
  for (int f = 0; f < F; ++f) {
#pragma unroll
    for (int h = 0; h < H; h += 4) {
      const float4 w = *reinterpret_cast<const float4*>(sW + oW1 + f * H + h);
      h1[h] = fmaf(x[f], w.x, h1[h]);
      h1[h + 1] = fmaf(x[f], w.y, h1[h + 1]);
      h1[h + 2] = fmaf(x[f], w.z, h1[h + 2]);
      h1[h + 3] = fmaf(x[f], w.w, h1[h + 3]);
    }
  }
#pragma unroll
  for (int h = 0; h < H; ++h) h1[h] = fmaxf(h1[h], 0.f);
#pragma unroll
  for (int j = 0; j < H; ++j) h2[j] = sW[ob2 + j];
#pragma unroll
  for (int h = 0; h < H; ++h) {
#pragma unroll
    for (int j = 0; j < H; j += 4) {
      const float4 w = *reinterpret_cast<const float4*>(sW + oW2 + h * H + j);
      h2[j] = fmaf(h1[h], w.x, h2[j]);
      h2[j + 1] = fmaf(h1[h], w.y, h2[j + 1]);
      h2[j + 2] = fmaf(h1[h], w.z, h2[j + 2]);
      h2[j + 3] = fmaf(h1[h], w.w, h2[j + 3]);
    }
  }
#pragma unroll
  for (int j = 0; j < H; ++j) h2[j] = fmaxf(h2[j], 0.f);
#pragma unroll
  for (int o = 0; o < O; ++o) y[o] = sW[ob3 + o];
#pragma unroll
  for (int j = 0; j < H; ++j) {
#pragma unroll
    for (int o = 0; o < O; o += 2) {
      const float2 w = *reinterpret_cast<const float2*>(sW + oW3 + j * O + o);
      y[o] = fmaf(h2[j], w.x, y[o]);
      y[o + 1] = fmaf(h2[j], w.y, y[o + 1]);
    }
  }
  const int m = raw[5 * (size_t)i], n = raw[5 * (size_t)i + 1];
  const bool fok = (nullptr != fma_ok) && 0 != fma_ok[i];
  int best = 0;
  float ymax = -INFINITY;
#pragma unroll
  for (int c = 0; c < K; ++c) {
    if (config_valid(c, m, n, fok) && y[c] > ymax) {
      ymax = y[c];
      best = c;
    }
  }
  float z = 0.f;
#pragma unroll
  for (int c = 0; c < K; ++c) {
    if (config_valid(c, m, n, fok)) z += expf(y[c] - ymax);
  }
  cfg[i] = (unsigned char)best;
  if (nullptr != conf) conf[i] = 1.f / z;
  if (nullptr != pz) pz[i] = 1.f / (1.f + expf(-y[K]));
}

struct Dev {
  float *W, *X, *H1, *H2, *Y, *dY, *dH1, *dH2, *R, *Z, *loss, *part, *G, *M1, *M2;
  int* raw;
};

void dev_free(Dev& d) {
  void* ptrs[] = {d.W, d.X, d.H1, d.H2, d.Y, d.dY, d.dH1, d.dH2, d.R, d.Z, d.loss, d.part, d.G, d.M1, d.M2, d.raw};
  for (void* p : ptrs) cudaFree(p);
  memset(&d, 0, sizeof(d));
}

int dev_alloc(Dev& d, int N) {
  memset(&d, 0, sizeof(d));
  const size_t n = (size_t)(N > 0 ? N : 1);
  int r = 0;
  r |= (int)cudaMalloc(&d.W, sizeof(float) * NW);
  r |= (int)cudaMalloc(&d.X, sizeof(float) * n * F);
  r |= (int)cudaMalloc(&d.H1, sizeof(float) * n * H);
  r |= (int)cudaMalloc(&d.H2, sizeof(float) * n * H);
  r |= (int)cudaMalloc(&d.Y, sizeof(float) * n * O);
  r |= (int)cudaMalloc(&d.dY, sizeof(float) * n * O);
  r |= (int)cudaMalloc(&d.dH1, sizeof(float) * n * H);
  r |= (int)cudaMalloc(&d.dH2, sizeof(float) * n * H);
  r |= (int)cudaMalloc(&d.R, sizeof(float) * n * K);
  r |= (int)cudaMalloc(&d.Z, sizeof(float) * n);
  r |= (int)cudaMalloc(&d.loss, sizeof(float) * n);
  r |= (int)cudaMalloc(&d.part, sizeof(float) * kWChunks * NW);
  r |= (int)cudaMalloc(&d.G, sizeof(float) * NW);
  r |= (int)cudaMalloc(&d.M1, sizeof(float) * NW);
  r |= (int)cudaMalloc(&d.M2, sizeof(float) * NW);
  r |= (int)cudaMalloc(&d.raw, sizeof(int) * 5 * n);
  if (0 != r) {
    dev_free(d);
    return (int)cudaErrorMemoryAllocation;
  }
  return 0;
}

/* one forward + loss + backward + weight-gradient pass into d.G */
int grad_pass(Dev& d, int N, cudaStream_t s) {
  const int tb = 128, nb = (N + tb - 1) / tb;
  const size_t smem = sizeof(float) * NW;
  xs_mlp_fwd<<<nb, tb, smem, s>>>(d.W, d.raw, N, d.X, d.H1, d.H2, d.Y);
  xs_mlp_loss<<<nb, tb, 0, s>>>(d.Y, d.R, d.Z, N, d.dY, d.loss);
  xs_mlp_bwd<<<nb, tb, smem, s>>>(d.W, d.H1, d.H2, d.dY, N, d.dH1, d.dH2);
  xs_mlp_wgrad<<<dim3((NW + 127) / 128, kWChunks), 128, 0, s>>>(d.X, d.H1, d.H2, d.dH1, d.dH2, d.dY, N, d.part);
  xs_mlp_reduce<<<(NW + 127) / 128, 128, 0, s>>>(d.part, d.G);
  return (int)cudaGetLastError();
}

int set_smem_attrs(void) {
  const size_t smem = sizeof(float) * NW;
  int r = xs_func_smem((const void*)xs_mlp_fwd, smem);
  if (0 == r) r = xs_func_smem((const void*)xs_mlp_infer, smem);
  return (0 != r) ? r : xs_func_smem((const void*)xs_mlp_bwd, smem);
}

/* ------------------------------------------------------------------ installed predictor table */

constexpr int kGridDim = 80;  /* m, n, k in 1..80 */
constexpr int kGridS = 3;     /* stack-size buckets: 1e3, 1e4, 1e5 */
unsigned char* g_cfg = nullptr;
unsigned char* g_conf = nullptr; /* confidence * 255 */
pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;

int s_bucket(int S) { return (S < 3000) ? 0 : ((S < 30000) ? 1 : 2); }

}  // namespace

extern "C" {

int xs_mlp_nweights(void) { return NW; }

int xs_mlp_train(const int* raw, const float* R, const float* Z, int N, int steps, float lr, float* weights, float* loss_hist) {
  Dev d;
  if (N < 1 || steps < 0 || nullptr == weights) return (int)cudaErrorInvalidValue;
  int r = set_smem_attrs();
  if (0 != r) return r;
  if (0 != (r = dev_alloc(d, N))) return r;
  cudaStream_t s = nullptr;
  r = (int)cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (0 == r) r = (int)cudaMemcpyAsync(d.raw, raw, sizeof(int) * 5 * (size_t)N, cudaMemcpyHostToDevice, s);
  if (0 == r) r = (int)cudaMemcpyAsync(d.R, R, sizeof(float) * K * (size_t)N, cudaMemcpyHostToDevice, s);
  if (0 == r) r = (int)cudaMemcpyAsync(d.Z, Z, sizeof(float) * (size_t)N, cudaMemcpyHostToDevice, s);
  if (0 == r) r = (int)cudaMemcpyAsync(d.W, weights, sizeof(float) * NW, cudaMemcpyHostToDevice, s);
  if (0 == r) r = (int)cudaMemsetAsync(d.M1, 0, sizeof(float) * NW, s);
  if (0 == r) r = (int)cudaMemsetAsync(d.M2, 0, sizeof(float) * NW, s);
  float* lh = (float*)malloc(sizeof(float) * (size_t)N);
  for (int t = 1; t <= steps && 0 == r; ++t) {
    r = grad_pass(d, N, s);
    if (0 == r) {
      xs_mlp_adam<<<(NW + 127) / 128, 128, 0, s>>>(d.W, d.G, d.M1, d.M2, t, lr);
      r = (int)cudaGetLastError();
    }
    if (0 == r && nullptr != loss_hist && nullptr != lh) {
      r = (int)cudaMemcpyAsync(lh, d.loss, sizeof(float) * (size_t)N, cudaMemcpyDeviceToHost, s);
      if (0 == r) r = (int)cudaStreamSynchronize(s);
      double sum = 0;
      for (int i = 0; i < N; ++i) sum += lh[i];
      loss_hist[t - 1] = (float)(sum / N);
    }
  }
  if (0 == r) r = (int)cudaMemcpyAsync(weights, d.W, sizeof(float) * NW, cudaMemcpyDeviceToHost, s);
  if (0 == r) r = (int)cudaStreamSynchronize(s);
  free(lh);
  if (nullptr != s) cudaStreamDestroy(s);
  dev_free(d);
  return r;
}

int xs_mlp_grad(const float* weights, const int* raw, const float* R, const float* Z, int N, float* grad, float* loss) {
  Dev d;
  if (N < 1) return (int)cudaErrorInvalidValue;
  int r = set_smem_attrs();
  if (0 != r) return r;
  if (0 != (r = dev_alloc(d, N))) return r;
  r = (int)cudaMemcpy(d.raw, raw, sizeof(int) * 5 * (size_t)N, cudaMemcpyHostToDevice);
  if (0 == r) r = (int)cudaMemcpy(d.R, R, sizeof(float) * K * (size_t)N, cudaMemcpyHostToDevice);
  if (0 == r) r = (int)cudaMemcpy(d.Z, Z, sizeof(float) * (size_t)N, cudaMemcpyHostToDevice);
  if (0 == r) r = (int)cudaMemcpy(d.W, weights, sizeof(float) * NW, cudaMemcpyHostToDevice);
  if (0 == r) r = grad_pass(d, N, nullptr);
  if (0 == r) r = (int)cudaMemcpy(grad, d.G, sizeof(float) * NW, cudaMemcpyDeviceToHost);
  if (0 == r && nullptr != loss) r = (int)cudaMemcpy(loss, d.loss, sizeof(float) * (size_t)N, cudaMemcpyDeviceToHost);
  dev_free(d);
  return r;
}

int xs_mlp_forward(const float* weights, const int* raw, int N, float* y) {
  Dev d;
  if (N < 1) return (int)cudaErrorInvalidValue;
  int r = set_smem_attrs();
  if (0 != r) return r;
  if (0 != (r = dev_alloc(d, N))) return r;
  r = (int)cudaMemcpy(d.raw, raw, sizeof(int) * 5 * (size_t)N, cudaMemcpyHostToDevice);
  if (0 == r) r = (int)cudaMemcpy(d.W, weights, sizeof(float) * NW, cudaMemcpyHostToDevice);
  if (0 == r) {
    xs_mlp_fwd<<<(N + 127) / 128, 128, sizeof(float) * NW>>>(d.W, d.raw, N, d.X, d.H1, d.H2, d.Y);
    r = (int)cudaGetLastError();
  }
  if (0 == r) r = (int)cudaMemcpy(y, d.Y, sizeof(float) * O * (size_t)N, cudaMemcpyDeviceToHost);
  dev_free(d);
  return r;
}

/* Inference for N queries (m, n, k, S, spread): configuration index, its probability, Ozaki
   probability (conf, pz may be null). Synchronous. Device memory: the weights and about 30 bytes per
   query (queries, FMA flags and the three results); the training buffers are not touched. */
int xs_mlp_predict(const float* weights, const int* raw, int N, unsigned char* cfg, float* conf, float* pz) {
  if (N < 1) return 0;
  int r = set_smem_attrs();
  if (0 != r) return r;
  float *dW = nullptr, *dconf = nullptr, *dpz = nullptr;
  int* draw = nullptr;
  unsigned char *dcfg = nullptr, *dfma = nullptr;
  /* where the FMA kernel takes the shape (host-side rule, the same one its launcher applies) */
  unsigned char* const fma_ok = (unsigned char*)malloc((size_t)N);
  if (nullptr == fma_ok) r = (int)cudaErrorMemoryAllocation;
  else {
    for (int i = 0; i < N; ++i) fma_ok[i] = (unsigned char)xs_smm_fma_supported(raw[5 * (size_t)i], raw[5 * (size_t)i + 1], raw[5 * (size_t)i + 2]);
  }
  if (0 == r) r = (int)cudaMalloc(&dW, sizeof(float) * NW);
  if (0 == r) r = (int)cudaMalloc(&draw, sizeof(int) * 5 * (size_t)N);
  if (0 == r) r = (int)cudaMalloc(&dcfg, (size_t)N);
  if (0 == r) r = (int)cudaMalloc(&dfma, (size_t)N);
  if (0 == r) r = (int)cudaMalloc(&dconf, sizeof(float) * (size_t)N);
  if (0 == r) r = (int)cudaMalloc(&dpz, sizeof(float) * (size_t)N);
  if (0 == r) r = (int)cudaMemcpy(dfma, fma_ok, (size_t)N, cudaMemcpyHostToDevice);
  if (0 == r) r = (int)cudaMemcpy(draw, raw, sizeof(int) * 5 * (size_t)N, cudaMemcpyHostToDevice);
  if (0 == r) r = (int)cudaMemcpy(dW, weights, sizeof(float) * NW, cudaMemcpyHostToDevice);
  if (0 == r) {
    xs_mlp_infer<<<(N + 127) / 128, 128, sizeof(float) * NW>>>(dW, draw, dfma, N, dcfg, dconf, dpz);
    r = (int)cudaGetLastError();
  }
  if (0 == r) r = (int)cudaMemcpy(cfg, dcfg, (size_t)N, cudaMemcpyDeviceToHost);
  if (0 == r && nullptr != conf) r = (int)cudaMemcpy(conf, dconf, sizeof(float) * (size_t)N, cudaMemcpyDeviceToHost);
  if (0 == r && nullptr != pz) r = (int)cudaMemcpy(pz, dpz, sizeof(float) * (size_t)N, cudaMemcpyDeviceToHost);
  cudaFree(dpz);
  cudaFree(dconf);
  cudaFree(dfma);
  cudaFree(dcfg);
  cudaFree(draw);
  cudaFree(dW);
  free(fma_ok);
  return r;
}

/* Installs the predictor: one inference launch over every shape m, n, k in 1..80 and the three
   stack-size buckets; lookups then read the resulting table on the host (graph-capture safe). */
int xs_mlp_install(const float* weights) {
  const int N = kGridDim * kGridDim * kGridDim * kGridS;
  int* raw = (int*)malloc(sizeof(int) * 5 * (size_t)N);
  unsigned char* cfg = (unsigned char*)malloc((size_t)N);
  float* conf = (float*)malloc(sizeof(float) * (size_t)N);
  unsigned char* conf8 = (unsigned char*)malloc((size_t)N);
  if (nullptr == raw || nullptr == cfg || nullptr == conf || nullptr == conf8) {
    free(raw);
    free(cfg);
    free(conf);
    free(conf8);
    return (int)cudaErrorMemoryAllocation;
  }
  static const int S_of[kGridS] = {1000, 10000, 100000};
  for (int i = 0; i < N; ++i) {
    int t = i;
    const int sb = t % kGridS;
    t /= kGridS;
    const int k = t % kGridDim + 1;
    t /= kGridDim;
    const int n = t % kGridDim + 1, m = t / kGridDim + 1;
    int* q = raw + 5 * (size_t)i;
    q[0] = m;
    q[1] = n;
    q[2] = k;
    q[3] = S_of[sb];
    q[4] = 0;
  }
  int r = xs_mlp_predict(weights, raw, N, cfg, conf, nullptr);
  if (0 == r) {
    for (int i = 0; i < N; ++i) conf8[i] = (unsigned char)(fminf(fmaxf(conf[i], 0.f), 1.f) * 255.f + 0.5f);
    pthread_mutex_lock(&g_lock);
    free(g_cfg);
    free(g_conf);
    g_cfg = cfg;
    g_conf = conf8;
    pthread_mutex_unlock(&g_lock);
    cfg = nullptr;
    conf8 = nullptr;
  }
  free(raw);
  free(cfg);
  free(conf);
  free(conf8);
  return r;
}

void xs_mlp_uninstall(void) {
  pthread_mutex_lock(&g_lock);
  free(g_cfg);
  free(g_conf);
  g_cfg = nullptr;
  g_conf = nullptr;
  pthread_mutex_unlock(&g_lock);
}

/* Predicted configuration for a shape from the installed table: returns 1 and fills mt, nt, kp (kp =
   XS_KP_FMA: the FMA kernel) and the confidence (0..1) when a predictor is installed and the shape is
   inside the table, else 0. */
int xs_mlp_lookup(int m, int n, int k, int S, int* mt, int* nt, int* kp, float* confidence) {
  int found = 0;
  if (m < 1 || n < 1 || k < 1 || m > kGridDim || n > kGridDim || k > kGridDim) return 0;
  pthread_mutex_lock(&g_lock);
  if (nullptr != g_cfg) {
    const size_t i = (((size_t)(m - 1) * kGridDim + (n - 1)) * kGridDim + (k - 1)) * kGridS + s_bucket(S);
    const int c = g_cfg[i];
    *mt = (kFmaConfig == c) ? 1 : (c >> 3) + 1;
    *nt = (kFmaConfig == c) ? 1 : ((c >> 1) & 3) + 1;
    *kp = (kFmaConfig == c) ? XS_KP_FMA : ((c & 1) ? 4 : 2);
    if (nullptr != confidence) *confidence = (float)g_conf[i] / 255.f;
    found = 1;
  }
  pthread_mutex_unlock(&g_lock);
  return found;
}

}  // extern "C"
