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

/* Stable order of the stack by C offset (LSD radix sort of c - 1 in two 16-bit digits): perm[i] is
   the stack index of the i-th entry in grouped order. Returns 0, or -1 if memory ran out. */
static int group_by_c(const int* stack, int S, int* perm) {
  int* const tmp = (int*)malloc(sizeof(int) * (size_t)(S > 0 ? S : 1));
  size_t* const cnt = (size_t*)malloc(sizeof(size_t) * 65537);
  int pass, i;
  if (NULL == tmp || NULL == cnt) {
    free(tmp);
    free(cnt);
    return -1;
  }
  for (i = 0; i < S; ++i) tmp[i] = i;
  for (pass = 0; pass < 2; ++pass) {
    const int sh = 16 * pass;
    const int* const src = (0 == pass) ? tmp : perm;
    int* const dst = (0 == pass) ? perm : tmp;
    memset(cnt, 0, sizeof(size_t) * 65537);
    for (i = 0; i < S; ++i) ++cnt[1 + ((((unsigned)stack[3 * src[i] + 2] - 1u) >> sh) & 0xFFFFu)];
    for (i = 0; i < 65536; ++i) cnt[i + 1] += cnt[i];
    for (i = 0; i < S; ++i) dst[cnt[(((unsigned)stack[3 * src[i] + 2] - 1u) >> sh) & 0xFFFFu]++] = src[i];
  }
  memcpy(perm, tmp, sizeof(int) * (size_t)S);
  free(tmp);
  free(cnt);
  return 0;
}

/* Timed CPU baseline: the host SMM path with all threads (B column-major), balanced the way the
   reference splits its host loop into tasks of equal length (libxs_gemm_index_task(..., tid, ntasks),
   samples/smm/acc_bench.c:380-384). The stack is first ordered by C offset (stable), then cut into
   nthreads contiguous ranges of equal entry count, so every thread does the same number of block
   products whatever the C distribution (a Zipf-hot C block no longer lands on one thread). A
   segment (run of equal C) inside a range is accumulated straight into C by its only owner; the
   segments that cross a range boundary are accumulated into private partial tiles (head / tail of
   each range), which are added to C afterwards in thread order, so the result is deterministic.
   Results differ from oracle_smm_f64 only by rounding (FMA, and the partial sums). */
void oracle_smm_f64_fast(const int* stack, int S, const double* a, const double* b, double* c, int m, int n, int k,
  int nthreads) {
  const size_t mn = (size_t)m * n;
  int* perm;
  double* part;
  int nt, t;
  if (0 >= S) return;
#if defined(_OPENMP)
  if (0 >= nthreads) nthreads = omp_get_max_threads();
#else
  nthreads = 1;
#endif
  nt = (nthreads < S) ? nthreads : S;
  if (0 >= nt) nt = 1;
  perm = (int*)malloc(sizeof(int) * (size_t)S);
  part = (double*)malloc(sizeof(double) * 2 * mn * (size_t)nt);
  if (NULL == perm || NULL == part || 0 != group_by_c(stack, S, perm)) {
    free(perm);
    free(part);
    return;
  }
#define XS_C_OF(I) (stack[3 * perm[I] + 2])
#if defined(_OPENMP)
#pragma omp parallel for num_threads(nt) schedule(static, 1)
#endif
  for (t = 0; t < nt; ++t) {
    const int p0 = (int)((long long)S * t / nt), p1 = (int)((long long)S * (t + 1) / nt);
    const int crossl = (0 < p0) && XS_C_OF(p0 - 1) == XS_C_OF(p0);
    const int crossr = (p1 < S) && XS_C_OF(p1) == XS_C_OF(p1 - 1);
    double* const head = part + 2 * mn * (size_t)t;
    double* const tail = head + mn;
    int q = p0;
    memset(head, 0, sizeof(double) * 2 * mn);
    while (q < p1) {
      const int cq = XS_C_OF(q);
      int r = q + 1, i;
      double* dst;
      while (r < p1 && XS_C_OF(r) == cq) ++r;
      if (q == p0 && crossl) dst = head;       /* continues a segment of the previous range */
      else if (r == p1 && crossr) dst = tail;  /* continues into the next range */
      else dst = c + cq - 1;                   /* this thread's own C block */
      for (i = q; i < r; ++i) smm_entry_fast(a + stack[3 * perm[i]] - 1, b + stack[3 * perm[i] + 1] - 1, dst, m, n, k);
      q = r;
    }
  }
  for (t = 0; t < nt; ++t) { /* partial tiles of boundary-crossing segments, in thread order */
    const int p0 = (int)((long long)S * t / nt), p1 = (int)((long long)S * (t + 1) / nt);
    const int crossl = (0 < p0) && XS_C_OF(p0 - 1) == XS_C_OF(p0);
    const int crossr = (p1 < S) && XS_C_OF(p1) == XS_C_OF(p1 - 1);
    const int whole = crossl && XS_C_OF(p0) == XS_C_OF(p1 - 1); /* one segment spans the range: all in head */
    const double* const head = part + 2 * mn * (size_t)t;
    size_t e;
    if (crossl) {
      double* const dst = c + XS_C_OF(p0) - 1;
      for (e = 0; e < mn; ++e) dst[e] += head[e];
    }
    if (crossr && !whole) {
      double* const dst = c + XS_C_OF(p1 - 1) - 1;
      for (e = 0; e < mn; ++e) dst[e] += head[mn + e];
    }
  }
#undef XS_C_OF
  free(perm);
  free(part);
}

/* Largest share of the stack's entries that one thread of oracle_smm_f64_fast processes, relative to
   the mean (1.0 = perfectly balanced). */
double oracle_fast_balance(int S, int nthreads) {
  int t, nt = (nthreads < S) ? nthreads : S;
  long long most = 0;
  if (0 >= nt) return 1.0;
  for (t = 0; t < nt; ++t) {
    const long long len = (long long)S * (t + 1) / nt - (long long)S * t / nt;
    if (len > most) most = len;
  }
  return (double)most * nt / (double)S;
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
