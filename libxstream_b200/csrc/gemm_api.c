/*
 * Dense FP64 GEMM entry points: the Ozaki scheme-1 form on the int8 tensor cores and the plain
 * FP64 DMMA form it is compared with. Both take device pointers and a stream, enqueue their work
 * and return without synchronising (samples/ozaki/ozaki_opencl.h:413-421 ozaki_gemm semantics);
 * scratch comes from the device's stream-ordered memory pool and is released in stream order.
 */
#include "internal.h"
#include "../../include/libxstream_b200.h"
#include <stdio.h>
#include <stdlib.h>

int libxstream_b200_ozaki_gemm(char transa, char transb, int M, int N, int K, double alpha, const double* a, int lda,
  const double* b, int ldb, double beta, double* c, int ldc, int nslices, int trim, void* stream) {
  void* scratch = NULL;
  size_t nbytes;
  int r, cutoff;
  if (EXIT_SUCCESS != xs_smm_ensure_init()) return EXIT_FAILURE;
  if (NULL == stream) stream = xs_default_stream();
  if (0 >= nslices) nslices = 8; /* the reference's FP64 default (ozaki_opencl.c:422) */
  if (8 < nslices) return xs_record_error(1, "ozaki_gemm: nslices > 8");
  cutoff = 2 * (nslices - 1) - (0 < trim ? trim : 0); /* ozaki_opencl.c:460-463 */
  if (0 > cutoff) cutoff = 0;
  nbytes = (0 < M && 0 < N && 0 < K && 0.0 != alpha) ? xs_ozaki_gemm_scratch_bytes(M, N, K, nslices) : 0;
  if (0 < nbytes && EXIT_SUCCESS != xs_scratch_alloc(&scratch, nbytes, stream)) return EXIT_FAILURE;
  r = xs_ozaki_gemm(transa, transb, M, N, K, alpha, a, lda, b, ldb, beta, c, ldc, nslices, cutoff, scratch, nbytes, stream);
  if (NULL != scratch) xs_scratch_free(scratch, stream);
  return xs_record_error(r, "ozaki_gemm");
}

int libxstream_b200_ozaki2_gemm(char transa, char transb, int M, int N, int K, double alpha, const double* a, int lda,
  const double* b, int ldb, double beta, double* c, int ldc, int nmoduli, void* stream) {
  void* scratch = NULL;
  size_t nbytes;
  int r;
  if (EXIT_SUCCESS != xs_smm_ensure_init()) return EXIT_FAILURE;
  if (NULL == stream) stream = xs_default_stream();
  if (0 > nmoduli || 20 < nmoduli) return xs_record_error(1, "ozaki2_gemm: nmoduli outside 0..20");
  if (0 == nmoduli) nmoduli = xs_ozaki2_default_moduli(K); /* full FP64 input precision for this K */
  nbytes = (0 < M && 0 < N && 0 < K && 0.0 != alpha) ? xs_ozaki2_gemm_scratch_bytes(M, N, K, nmoduli) : 0;
  if (0 < nbytes && EXIT_SUCCESS != xs_scratch_alloc(&scratch, nbytes, stream)) return EXIT_FAILURE;
  r = xs_ozaki2_gemm(transa, transb, M, N, K, alpha, a, lda, b, ldb, beta, c, ldc, nmoduli, scratch, nbytes, stream);
  if (NULL != scratch) xs_scratch_free(scratch, stream);
  return xs_record_error(r, "ozaki2_gemm");
}

int libxstream_b200_dgemm(char transa, char transb, int M, int N, int K, double alpha, const double* a, int lda,
  const double* b, int ldb, double beta, double* c, int ldc, void* stream) {
  if (EXIT_SUCCESS != xs_smm_ensure_init()) return EXIT_FAILURE;
  if (('N' != transa && 'n' != transa) || ('N' != transb && 'n' != transb)) {
    return xs_record_error(1, "dgemm: only transa = transb = 'N'");
  }
  if (NULL == stream) stream = xs_default_stream();
  return xs_record_error(xs_dgemm(M, N, K, alpha, a, lda, b, ldb, beta, c, ldc, stream), "dgemm");
}

int libxstream_b200_process_ozaki(const int* dev_param_stack, int stack_size, int m, int n, int k, const double* dev_a,
  int na, const double* dev_b, int nb, double* dev_c, int nslices, int trim, void* stream) {
  void* scratch = NULL;
  size_t nbytes;
  int r, cutoff;
  if (0 >= stack_size) return EXIT_SUCCESS;
  if (m < 1 || n < 1 || k < 1 || m > 64 || n > 64 || k > 64) return -1; /* not handled: use the plain path */
  if (EXIT_SUCCESS != xs_smm_ensure_init()) return EXIT_FAILURE;
  if (NULL == stream) stream = xs_default_stream();
  if (0 >= nslices) nslices = 7;
  if (8 < nslices || 1 > na || 1 > nb) return xs_record_error(1, "process_ozaki: invalid arguments");
  cutoff = 2 * (nslices - 1) - (0 < trim ? trim : 0);
  if (0 > cutoff) cutoff = 0;
  nbytes = xs_smm_ozaki_scratch_bytes(stack_size, m, n, k, na, nb, nslices);
  if (0 == nbytes || EXIT_SUCCESS != xs_scratch_alloc(&scratch, nbytes, stream)) return EXIT_FAILURE;
  r = xs_launch_smm_ozaki(dev_param_stack, stack_size, m, n, k, dev_a, na, dev_b, nb, dev_c, nslices, cutoff, scratch, nbytes,
    stream);
  xs_scratch_free(scratch, stream);
  return xs_record_error(r, "process_ozaki");
}
