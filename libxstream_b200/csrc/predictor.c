/*
 * Host API of the autotuner and of the learned parameter predictor (C). The exhaustive tuner times
 * every precompiled configuration of the plain stack kernel on synthetic data of a given shape; the
 * predictor (a small MLP, trained on the tuner's sweeps by the device kernels in mlp.cu) proposes a
 * configuration for shapes without a tuned record. Lookup order in the stack path: tuned record ->
 * exhaustive tuning on the spot when LIBXSTREAM_B200_AUTOTUNE=1, the stream is not being captured
 * and the predictor is absent or its confidence is below LIBXSTREAM_B200_MLP_MINCONF (default 0.5)
 * -> predicted configuration -> default heuristic (no predictor installed).
 */
#include "internal.h"
#include "../../include/libxstream_b200.h"
#include <cuda_runtime_api.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int libxstream_b200_tune_candidates(int m, int n, int* mt_nt_kp, int capacity) {
  return xs_tune_candidates(m, n, mt_nt_kp, capacity);
}

int libxstream_b200_tune(int m, int n, int k, int stack_size, int reps, int ozaki_slices, unsigned seed, float* ms_out,
  int capacity, void* stream) {
  int r;
  if (EXIT_SUCCESS != xs_smm_ensure_init()) return -1;
  if (NULL == stream) stream = xs_default_stream();
  r = xs_tune(m, n, k, stack_size, reps, ozaki_slices, seed, ms_out, capacity, stream);
  if (0 > r) xs_record_error(-r, "tune");
  return r;
}

int libxstream_b200_mlp_nweights(void) { return xs_mlp_nweights(); }

int libxstream_b200_mlp_train(const int* raw, const float* r, const float* z, int n, int steps, float lr, float* weights,
  float* loss_hist) {
  if (EXIT_SUCCESS != xs_smm_ensure_init()) return EXIT_FAILURE;
  return xs_record_error(xs_mlp_train(raw, r, z, n, steps, lr, weights, loss_hist), "mlp_train");
}

int libxstream_b200_mlp_grad(const float* weights, const int* raw, const float* r, const float* z, int n, float* grad,
  float* loss) {
  if (EXIT_SUCCESS != xs_smm_ensure_init()) return EXIT_FAILURE;
  return xs_record_error(xs_mlp_grad(weights, raw, r, z, n, grad, loss), "mlp_grad");
}

int libxstream_b200_mlp_forward(const float* weights, const int* raw, int n, float* y) {
  if (EXIT_SUCCESS != xs_smm_ensure_init()) return EXIT_FAILURE;
  return xs_record_error(xs_mlp_forward(weights, raw, n, y), "mlp_forward");
}

int libxstream_b200_mlp_predict(const float* weights, const int* raw, int n, unsigned char* config, float* confidence,
  float* p_ozaki) {
  if (EXIT_SUCCESS != xs_smm_ensure_init()) return EXIT_FAILURE;
  return xs_record_error(xs_mlp_predict(weights, raw, n, config, confidence, p_ozaki), "mlp_predict");
}

int libxstream_b200_mlp_install(const float* weights, int nweights) {
  if (NULL == weights) {
    xs_mlp_uninstall();
    return EXIT_SUCCESS;
  }
  if (nweights != xs_mlp_nweights()) return xs_record_error(1, "mlp_install: wrong number of weights");
  if (EXIT_SUCCESS != xs_smm_ensure_init()) return EXIT_FAILURE;
  return xs_record_error(xs_mlp_install(weights), "mlp_install");
}

/* Text file: a header line "XS_MLP <nweights>" then one weight per line. */
int xs_mlp_load_file(const char* path) {
  FILE* const f = (NULL != path) ? fopen(path, "r") : NULL;
  const int nw = xs_mlp_nweights();
  float* w;
  int count = 0, hdr = 0, result;
  if (NULL == f) return EXIT_FAILURE;
  w = (float*)malloc(sizeof(float) * (size_t)nw);
  if (NULL == w || 1 != fscanf(f, "XS_MLP %d", &hdr) || hdr != nw) {
    free(w);
    fclose(f);
    return EXIT_FAILURE;
  }
  while (count < nw && 1 == fscanf(f, "%f", &w[count])) ++count;
  fclose(f);
  result = (count == nw) ? libxstream_b200_mlp_install(w, nw) : EXIT_FAILURE;
  free(w);
  return result;
}

int libxstream_b200_mlp_lookup(int m, int n, int k, int stack_size, int* mt_nt_kp, float* confidence) {
  if (NULL == mt_nt_kp) return 0;
  return xs_mlp_lookup(m, n, k, stack_size, mt_nt_kp, mt_nt_kp + 1, mt_nt_kp + 2, confidence);
}

static int xs_autotune_enabled(void) {
  static int v = -1;
  if (0 > v) {
    const char* const env = getenv("LIBXSTREAM_B200_AUTOTUNE");
    v = (NULL != env && '1' == *env) ? 1 : 0;
  }
  return v;
}

void xs_autotune_if_needed(int m, int n, int k, int stack_size, void* stream) {
  xs_smm_params_t p;
  int source = XS_PARAMS_DEFAULT, cand[3 * 33], nc, best = -1, i; /* 32 DMMA tile classes + the FMA kernel */
  float ms[34];
  enum cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStream_t s = NULL;
  if (!xs_autotune_enabled()) return;
  xs_params_lookup_ex(3, m, n, k, stack_size, &p, &source);
  if (XS_PARAMS_TUNED == source || XS_PARAMS_PREDICTED == source) return;
  if (cudaSuccess != cudaStreamIsCapturing((cudaStream_t)stream, &cs) || cudaStreamCaptureStatusNone != cs) return;
  nc = xs_tune_candidates(m, n, cand, 33);
  if (nc > 33) return;
  if (cudaSuccess != cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) return;
  if (nc == xs_tune(m, n, k, stack_size, 2, 0, 12345u, ms, 34, s)) {
    for (i = 0; i < nc; ++i) { /* a negative time: the candidate does not take this shape */
      if (0.f <= ms[i] && (0 > best || ms[i] < ms[best])) best = i;
    }
  }
  cudaStreamDestroy(s);
  if (0 <= best) {
    p.chunk = 0;
    p.mt = cand[3 * best];
    p.nt = cand[3 * best + 1];
    p.kp = cand[3 * best + 2];
    p.wpb = 4;
    p.generic = 0;
    p.sorted = 0;
    xs_params_set(3, m, n, k, &p, 2e-6 * m * n * k * (double)stack_size / ms[best]);
    if (2 <= xs_verbosity()) {
      fprintf(stderr, "INFO LIBSMM/B200: tuned %ix%ix%i S=%i: mt=%i nt=%i kp=%i (%.3f ms)\n", m, n, k, stack_size, p.mt, p.nt,
        p.kp, ms[best]);
    }
  }
}
