/*
 * DBCSR LIBSMM accelerator ABI: batched small-matrix multiply ("stack" process) and batched
 * in-place transpose, implemented with hand-written sm_100a kernels.
 *
 * Reference interface replaced: samples/smm/acc_libsmm.h:31-49 (types and prototypes),
 * implemented there by samples/smm/smm_acc.c:43-604, samples/smm/smm_kernel.c:82-528 and
 * samples/smm/smm_trans.c:48-228.
 *
 * Data contract (identical to the reference):
 *   - A, B and C are flat pools of blocks; all blocks of one call have the same shape.
 *   - libsmm_acc_process: dev_param_stack holds stack_size triples (a, b, c) of 1-based element
 *     offsets. For each triple C[c..] += A[a..] * B[b..] where the A block is m x k column-major,
 *     the B block has already been transposed by libsmm_acc_transpose (k x n stored row-major,
 *     i.e. element (kk, j) at kk*n + j) and the C block is m x n column-major.
 *   - libsmm_acc_transpose: dev_trs_stack[offset + i] (0-based element offsets) lists blocks that
 *     are transposed in place from m x n column-major to n x m column-major. Bit-exact.
 * Return codes: 0 = success; libsmm_acc_process returns -1 for a stack it does not handle
 * (inhomogeneous, m*n > max_kernel_dim^2, unsupported type) so that DBCSR falls back to its host
 * path; c_calculate_norms returns -1 in the reference (unimplemented) and is implemented here.
 */
#ifndef LIBXSTREAM_B200_LIBSMM_ACC_H
#define LIBXSTREAM_B200_LIBSMM_ACC_H

#include "dbcsr_acc.h"

#if defined(__cplusplus)
extern "C" {
#endif

/** Element type ids as DBCSR numbers them (replaces acc_libsmm.h:31-36). */
typedef enum libsmm_acc_data_t {
  dbcsr_type_real_4 = 1,
  dbcsr_type_real_8 = 3,
  dbcsr_type_complex_4 = 5,
  dbcsr_type_complex_8 = 7
} libsmm_acc_data_t;

/** Reference-counted init/finalize (replaces acc_libsmm.h:38-39, smm_acc.c:43-481). */
int libsmm_acc_init(void);
int libsmm_acc_finalize(void);
/** 1: concurrent calls from several host threads on different streams are allowed (acc_libsmm.h:40). */
c_dbcsr_acc_bool_t libsmm_acc_is_thread_safe(void);

/** Batched in-place transpose (replaces acc_libsmm.h:42-43, smm_trans.c:48). */
int libsmm_acc_transpose(const int* dev_trs_stack, int offset, int stack_size, void* dev_data, libsmm_acc_data_t datatype,
  int m, int n, int max_kernel_dim, void* stream);

/** Stack multiply C += A*B (replaces acc_libsmm.h:45-47, smm_acc.c:575-593). */
int libsmm_acc_process(const int* host_param_stack, const int* dev_param_stack, int stack_size, libsmm_acc_data_t datatype,
  const void* dev_a_data, const void* dev_b_data, void* dev_c_data, int m_max, int n_max, int k_max, int max_kernel_dim,
  c_dbcsr_acc_bool_t def_mnk, void* stack_stream, void* c_stream);

/**
 * Frobenius norm of each of nblks blocks: norms[i] = sqrt(sum_j mat[offsets[i] + j]^2) for
 * j < nelems[i], computed in FP64 and stored as float. All pointers are device pointers.
 * The reference stubs this out (acc_libsmm.h:49, smm_acc.c:596-604 returns -1).
 */
int c_calculate_norms(const double* mat, int nblks, const int* offsets, const int* nelems, float* norms, void* stream_ptr);

#if defined(__cplusplus)
}
#endif

#endif /* LIBXSTREAM_B200_LIBSMM_ACC_H */
