/*
 * CPU oracle for the DBCSR SMM stack path. TEST INFRASTRUCTURE ONLY: this file is the checker the
 * parity tests, the smoke test and the CPU-baseline leg of bench.py compare against. The product
 * (libxstream_b200) never links, loads or calls it.
 *
 * It restates, in plain C, what the reference computes:
 *   - stack multiply: for each triple (a, b, c) of 1-based element offsets, in stack order,
 *     C(m x n, ldc=m) += A(m x k, lda=m) * B(k x n). This is the host reference of
 *     samples/smm/acc_bench.c:357-394 (libxs_gemm_index with 'N','N', lda=m, ldb=k, ldc=m,
 *     alpha=beta=1, index base 1), where B is column-major k x n (ldb=k); the device kernel
 *     samples/smm/kernels/multiply.cl:12-15 reads the same B after libsmm_acc_transpose, i.e.
 *     row-major k x n (BDX(K,N) = bdata[K*SN + N + b0]). Both layouts are provided.
 *   - batched transpose: samples/smm/kernels/transpose.cl:36-45 (m x n column-major block at
 *     matrix + trs_stack[offset + i] becomes n x m column-major, in place).
 *   - Ozaki scheme-1 digit slicing: samples/ozaki/kernels/ozaki_common.cl:789-834 and
 *     samples/ozaki/kernels/ozaki1_int8.cl:440-498 (per-row / per-column maximum exponent, aligned
 *     53-bit mantissa, 7-bit signed digits) and the pair loop with its scale
 *     2^(low_a + low_b - 104) * expa * expb (ozaki1_int8.cl:740-790).
 * The arithmetic of the reference's host path lives in LIBXS (libxs_gemm_index, not vendored, no
 * pinned version); the semantics above are those of its call site in acc_bench.c.
 * Built with -ffp-contract=off so that products and sums round exactly as written.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#if defined(_OPENMP)
#include <omp.h>
#endif

/* One triple: C(i,j) += sum_kk A(i,kk) * B(kk,j); b_rowmajor selects B(kk,j) = b[kk*n + j]
   (device contract, after transpose) instead of b[j*k + kk] (host contract, ldb = k). */
static void smm_entry(const double* a, const double* b, double* c, int m, int n, int k, int b_rowmajor) {
  int i, j, kk;
  for (j = 0; j < n; ++j) {
    for (kk = 0; kk < k; ++kk) {
      const double bv = b_rowmajor ? b[(size_t)kk * n + j] : b[(size_t)j * k + kk];
      const double* const acol = a + (size_t)kk * m;
      double* const ccol = c + (size_t)j * m;
      for (i = 0; i < m; ++i) ccol[i] += acol[i] * bv;
    }
  }
}

/* Sequential stack multiply in stack order (the semantics every other variant must match). */
void oracle_smm_f64(const int* stack, int S, const double* a, const double* b, double* c, int m, int n, int k,
  int b_rowmajor) {
  int s;
  for (s = 0; s < S; ++s) {
    smm_entry(a + stack[3 * s] - 1, b + stack[3 * s + 1] - 1, c + stack[3 * s + 2] - 1, m, n, k, b_rowmajor);
  }
}

/* Multi-threaded stack multiply: thread t owns the C blocks whose offset hashes to t, so every
   block is updated by one thread in stack order and the result equals oracle_smm_f64 bitwise. */
void oracle_smm_f64_omp(const int* stack, int S, const double* a, const double* b, double* c, int m, int n, int k,
  int b_rowmajor, int nthreads) {
#if defined(_OPENMP)
  if (0 >= nthreads) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    const int nt = omp_get_num_threads(), tid = omp_get_thread_num();
    int s;
    for (s = 0; s < S; ++s) {
      const unsigned cblk = (unsigned)(stack[3 * s + 2] - 1) / (unsigned)(m * n);
      if ((int)((cblk * 2654435761u) % (unsigned)nt) == tid) {
        smm_entry(a + stack[3 * s] - 1, b + stack[3 * s + 1] - 1, c + stack[3 * s + 2] - 1, m, n, k, b_rowmajor);
      }
    }
  }
#else
  (void)nthreads;
  oracle_smm_f64(stack, S, a, b, c, m, n, k, b_rowmajor);
#endif
}

/* One triple with B column-major (ldb = k, the host contract of acc_bench.c:369-374) for the timed
   baseline: an 8 x 4 register tile of C (generic GCC vectors of 4 doubles, fused multiply-adds) over
   the rows in steps of 8, a scalar loop for the remaining rows -- the structure of a tuned host
   small-GEMM kernel such as the LIBXS JIT kernels the reference's host path runs. */
typedef double xs_v4d __attribute__((vector_size(32)));

__attribute__((optimize("fp-contract=fast"))) static void smm_entry_fast(const double* a, const double* b, double* c,
  int m, int n, int k) {
  int i0 = 0, j0, jj, kk, i;
  for (; i0 + 8 <= m; i0 += 8) {
    for (j0 = 0; j0 < n; j0 += 4) {
      const int nj = (n - j0 < 4) ? n - j0 : 4;
      xs_v4d acc[4][2];
      for (jj = 0; jj < 4; ++jj) {
        if (jj < nj) {
          memcpy(&acc[jj][0], c + (size_t)(j0 + jj) * m + i0, sizeof(xs_v4d));
          memcpy(&acc[jj][1], c + (size_t)(j0 + jj) * m + i0 + 4, sizeof(xs_v4d));
        }
        else acc[jj][0] = acc[jj][1] = (xs_v4d){0, 0, 0, 0};
      }
      if (4 == nj) {
        for (kk = 0; kk < k; ++kk) {
          xs_v4d a0, a1;
          memcpy(&a0, a + (size_t)kk * m + i0, sizeof(a0));
          memcpy(&a1, a + (size_t)kk * m + i0 + 4, sizeof(a1));
          for (jj = 0; jj < 4; ++jj) {
            const double bv = b[(size_t)(j0 + jj) * k + kk];
            acc[jj][0] += a0 * bv;
            acc[jj][1] += a1 * bv;
          }
        }
      }
      else {
        for (kk = 0; kk < k; ++kk) {
          xs_v4d a0, a1;
          memcpy(&a0, a + (size_t)kk * m + i0, sizeof(a0));
          memcpy(&a1, a + (size_t)kk * m + i0 + 4, sizeof(a1));
          for (jj = 0; jj < nj; ++jj) {
            const double bv = b[(size_t)(j0 + jj) * k + kk];
            acc[jj][0] += a0 * bv;
            acc[jj][1] += a1 * bv;
          }
        }
      }
      for (jj = 0; jj < nj; ++jj) {
        memcpy(c + (size_t)(j0 + jj) * m + i0, &acc[jj][0], sizeof(xs_v4d));
        memcpy(c + (size_t)(j0 + jj) * m + i0 + 4, &acc[jj][1], sizeof(xs_v4d));
      }
    }
  }
  if (i0 < m) { /* remaining rows */
    int j;
    for (j = 0; j < n; ++j) {
      double* const cj = c + (size_t)j * m;
      const double* const bj = b + (size_t)j * k;
      for (kk = 0; kk < k; ++kk) {
        const double bv = bj[kk];
        const double* const ak = a + (size_t)kk * m;
        for (i = i0; i < m; ++i) cj[i] += ak[i] * bv;
      }
    }
  }
}

/* Timed CPU baseline: the host SMM path with all threads (B column-major). Thread t owns
   the C blocks whose offset hashes to t, so each block is still updated in stack order by one
   thread; results differ from oracle_smm_f64 only by FMA rounding. */
void oracle_smm_f64_fast(const int* stack, int S, const double* a, const double* b, double* c, int m, int n, int k,
  int nthreads) {
#if defined(_OPENMP)
  if (0 >= nthreads) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    const int nt = omp_get_num_threads(), tid = omp_get_thread_num();
    int s;
    for (s = 0; s < S; ++s) {
      const unsigned cblk = (unsigned)(stack[3 * s + 2] - 1) / (unsigned)(m * n);
      if ((int)((cblk * 2654435761u) % (unsigned)nt) == tid) {
        smm_entry_fast(a + stack[3 * s] - 1, b + stack[3 * s + 1] - 1, c + stack[3 * s + 2] - 1, m, n, k);
      }
    }
  }
#else
  int s;
  (void)nthreads;
  for (s = 0; s < S; ++s) smm_entry_fast(a + stack[3 * s] - 1, b + stack[3 * s + 1] - 1, c + stack[3 * s + 2] - 1, m, n, k);
#endif
}

int oracle_max_threads(void) {
#if defined(_OPENMP)
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* In-place transpose of each listed m x n column-major block (0-based offsets) to n x m. */
void oracle_transpose_f64(const int* trs, int offset, int S, double* data, int m, int n) {
  double* const tmp = (double*)malloc(sizeof(double) * (size_t)m * n);
  int s, i, j;
  if (NULL == tmp) return;
  for (s = 0; s < S; ++s) {
    double* const mat = data + trs[offset + s];
    memcpy(tmp, mat, sizeof(double) * (size_t)m * n);
    for (i = 0; i < m; ++i)
      for (j = 0; j < n; ++j) mat[(size_t)i * n + j] = tmp[(size_t)j * m + i];
  }
  free(tmp);
}

/* Frobenius norm per block (c_calculate_norms semantics of this library). */
void oracle_norms(const double* mat, int nblks, const int* offsets, const int* nelems, float* norms) {
  int b, e;
  for (b = 0; b < nblks; ++b) {
    double s = 0.0;
    for (e = 0; e < nelems[b]; ++e) s += mat[offsets[b] + e] * mat[offsets[b] + e];
    norms[b] = (float)sqrt(s);
  }
}

/* Relative max-norm error per C block: max over blocks of max|x - r| / max|r| within the block
   (the per-block metric of the north star; a block of all-zero reference uses absolute error). */
double oracle_block_relerr(const double* x, const double* r, int nblocks, int blocksize) {
  double worst = 0.0;
  int blk, e;
  for (blk = 0; blk < nblocks; ++blk) {
    double dmax = 0.0, rmax = 0.0;
    for (e = 0; e < blocksize; ++e) {
      const double d = fabs(x[(size_t)blk * blocksize + e] - r[(size_t)blk * blocksize + e]);
      const double a = fabs(r[(size_t)blk * blocksize + e]);
      if (d > dmax || d != d) dmax = (d != d) ? INFINITY : d;
      if (a > rmax) rmax = a;
    }
    {
      const double rel = (0 < rmax) ? dmax / rmax : dmax;
      if (rel > worst) worst = rel;
    }
  }
  return worst;
}

/* ------------------------------------------------------------------ Ozaki scheme 1 (int8) */

/* IEEE-754 binary64 split: sign, biased exponent, 53-bit significand with the implicit bit.
   Zero, subnormal, Inf and NaN give exponent 0 and significand 0 (ozaki_common.cl:789-806). */
static void ieee_split(double v, int* sign, int* bexp, uint64_t* mant) {
  uint64_t bits;
  memcpy(&bits, &v, sizeof(bits));
  *sign = (int)(bits >> 63);
  *bexp = (int)((bits >> 52) & 2047u);
  *mant = (bits & 0x000FFFFFFFFFFFFFull) | 0x0010000000000000ull;
  if (0 == *bexp || 2047 == *bexp) {
    *mant = 0;
    *bexp = 0;
  }
}

/* Digit s of an aligned significand: bits [52-7s .. max(0, 52-7s-6)], signed (ozaki_common.cl:814-834). */
static int slice_digit(uint64_t aligned, int sign, int s) {
  const int high = 52 - 7 * s;
  const int low = high - 6 > 0 ? high - 6 : 0;
  const int width = high - low + 1;
  int d = 0;
  if (width > 0 && high >= 0) d = (int)((aligned >> low) & ((1u << width) - 1u));
  return sign ? -d : d;
}

int oracle_slice_low_bit(int s) {
  const int high = 52 - 7 * s;
  return high - 6 > 0 ? high - 6 : 0;
}

/* Slice the rows of an M x K matrix x (element (r, kk) at x[r*rs + kk*cs]) into nslices int8
   planes digits[s][r][kk] (row-major, K contiguous) with per-row biased max exponent emax[r]
   (ozaki1_int8.cl:440-498 for A; B is the same with rows = columns of B). */
void oracle_ozaki_slice(const double* x, int M, int K, long rs, long cs, int nslices, signed char* digits, int* emax) {
  int r, kk, s;
  for (r = 0; r < M; ++r) {
    int e = 0;
    for (kk = 0; kk < K; ++kk) {
      int sg, be;
      uint64_t mt;
      ieee_split(x[(size_t)r * rs + (size_t)kk * cs], &sg, &be, &mt);
      if (be > e) e = be;
    }
    emax[r] = e;
    for (kk = 0; kk < K; ++kk) {
      int sg, be;
      uint64_t mt, aligned = 0;
      ieee_split(x[(size_t)r * rs + (size_t)kk * cs], &sg, &be, &mt);
      if (0 != mt) {
        const int shift = e - be;
        aligned = (shift <= 52) ? (mt >> shift) : 0;
      }
      for (s = 0; s < nslices; ++s) digits[((size_t)s * M + r) * K + kk] = (signed char)slice_digit(aligned, sg, s);
    }
  }
}

/* Ozaki GEMM C(M x N, col-major ldc=M) += A(M x K, col-major) * B(K x N, col-major), scheme 1
   with nslices slices, all pairs with sa + sb <= cutoff (cutoff < 0: all pairs). Integer pair
   products are exact in int64; each pair is scaled by 2^(low_sa + low_sb - 104) * 2^(ea-1023) *
   2^(eb-1023) and accumulated in FP64 in (sa, sb) order (ozaki1_int8.cl:740-790). */
void oracle_ozaki_gemm(const double* A, const double* B, double* C, int M, int N, int K, int nslices, int cutoff) {
  signed char* const da = (signed char*)malloc((size_t)nslices * M * K);
  signed char* const db = (signed char*)malloc((size_t)nslices * N * K);
  int* const ea = (int*)malloc(sizeof(int) * (size_t)M);
  int* const eb = (int*)malloc(sizeof(int) * (size_t)N);
  int i, j, kk, sa, sb;
  if (NULL == da || NULL == db || NULL == ea || NULL == eb) goto done;
  oracle_ozaki_slice(A, M, K, 1, M, nslices, da, ea);      /* rows of A: element (i, kk) at i + kk*M */
  oracle_ozaki_slice(B, N, K, K, 1, nslices, db, eb);      /* columns of B: element (kk, j) at kk + j*K */
  for (j = 0; j < N; ++j) {
    for (i = 0; i < M; ++i) {
      double acc = 0.0;
      if (0 == ea[i] || 0 == eb[j]) continue;
      for (sa = 0; sa < nslices; ++sa) {
        for (sb = 0; sb < nslices; ++sb) {
          int64_t dot = 0;
          if (0 <= cutoff && sa + sb > cutoff) continue;
          for (kk = 0; kk < K; ++kk) {
            dot += (int64_t)da[((size_t)sa * M + i) * K + kk] * (int64_t)db[((size_t)sb * N + j) * K + kk];
          }
          acc += ldexp((double)dot, oracle_slice_low_bit(sa) + oracle_slice_low_bit(sb) - 104 + (ea[i] - 1023) + (eb[j] - 1023));
        }
      }
      C[(size_t)j * M + i] += acc;
    }
  }
done:
  free(da);
  free(db);
  free(ea);
  free(eb);
}

/* Ozaki scheme-1 stack multiply: for every entry, C[c] += A[a] * B[b] where each row of the A block
   and each column of the B block is sliced with its own row / column exponent (the rule of
   oracle_ozaki_slice applied per block), all slice pairs with sa + sb <= cutoff are multiplied in
   int64 and scaled and accumulated in FP64 in (sa, sb) order, per entry in stack order. B blocks
   are k x n row-major when b_rowmajor (the device layout after libsmm_acc_transpose), else
   column-major. */
void oracle_ozaki_smm(const int* stack, int S, const double* a, const double* b, double* c, int m, int n, int k,
  int b_rowmajor, int nslices, int cutoff) {
  signed char* const da = (signed char*)malloc((size_t)nslices * m * k);
  signed char* const db = (signed char*)malloc((size_t)nslices * n * k);
  double* const blk = (double*)malloc(sizeof(double) * (size_t)m * n);
  int* const ea = (int*)malloc(sizeof(int) * (size_t)m);
  int* const eb = (int*)malloc(sizeof(int) * (size_t)n);
  int e, i, j, kk, sa, sb;
  if (NULL == da || NULL == db || NULL == blk || NULL == ea || NULL == eb) goto done;
  for (e = 0; e < S; ++e) {
    const double* const A = a + stack[3 * e + 0] - 1;
    const double* const B = b + stack[3 * e + 1] - 1;
    double* const C = c + stack[3 * e + 2] - 1;
    oracle_ozaki_slice(A, m, k, 1, m, nslices, da, ea);
    if (b_rowmajor) oracle_ozaki_slice(B, n, k, 1, n, nslices, db, eb); /* column j: element kk at kk*n + j */
    else oracle_ozaki_slice(B, n, k, k, 1, nslices, db, eb);            /* column j: element kk at kk + j*k */
    for (j = 0; j < n; ++j) {
      for (i = 0; i < m; ++i) {
        double acc = 0.0;
        if (0 != ea[i] && 0 != eb[j]) {
          for (sa = 0; sa < nslices; ++sa) {
            for (sb = 0; sb < nslices; ++sb) {
              int64_t dot = 0;
              if (0 <= cutoff && sa + sb > cutoff) continue;
              for (kk = 0; kk < k; ++kk) {
                dot += (int64_t)da[((size_t)sa * m + i) * k + kk] * (int64_t)db[((size_t)sb * n + j) * k + kk];
              }
              acc += ldexp((double)dot, oracle_slice_low_bit(sa) + oracle_slice_low_bit(sb) - 104 + (ea[i] - 1023) + (eb[j] - 1023));
            }
          }
        }
        blk[(size_t)j * m + i] = acc;
      }
    }
    for (i = 0; i < m * n; ++i) C[i] += blk[i];
  }
done:
  free(da);
  free(db);
  free(blk);
  free(ea);
  free(eb);
}
