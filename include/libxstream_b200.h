/*
 * Extension entry points of the B200 SMM library: additions beside the DBCSR ABI, for tuning,
 * measurement and batched execution. None of them changes what libsmm_acc_process computes.
 * Each declaration names the part of the reference it corresponds to, or says that it has none.
 */
#ifndef LIBXSTREAM_B200_H
#define LIBXSTREAM_B200_H

#include "libsmm_acc.h"

#if defined(__cplusplus)
extern "C" {
#endif

/** One homogeneous FP64 stack of a batch: stack_size (a, b, c) triples of 1-based element offsets
    (device memory) into the pools a, b (B already transposed, k x n row-major) and c, as for
    libsmm_acc_process. */
typedef struct libxstream_b200_stack_t {
  const int* dev_param_stack;
  int stack_size;
  int m, n, k;
  const void* a;
  const void* b;
  void* c;
} libxstream_b200_stack_t;

/** All stacks of one multiplication in one call: equivalent to one libsmm_acc_process per stack
    (FP64, homogeneous, def_mnk = 1), but grouped together (one grouping launch for up to 16 stacks)
    and run by one persistent stack kernel whose CTAs take work items from all stacks, heaviest
    first, and combine C blocks that cross CTAs themselves; the call is capturable in a CUDA graph (libxstream_b200_graph_begin/end). Stacks may share pools; if two
    stacks update the same C block their contributions are added atomically (correct, but not
    bitwise reproducible). Returns -1 (nothing done) if any stack is one libsmm_acc_process would not
    handle (m*n > max_kernel_dim^2, nonpositive sizes), else 0 or a CUDA error. No counterpart in the
    reference, which launches one homogeneous stack per call (samples/smm/smm_acc.c:575-593). */
int libxstream_b200_process_batch(const libxstream_b200_stack_t* stacks, int nstacks, int max_kernel_dim, void* stream);

/** The suitability rule of libsmm_acc_process: 1 if the stack is handled on the GPU, else 0.
    Replaces libsmm_acc_process_suitable (samples/smm/smm_acc.c:527-573). */
int libxstream_b200_process_suitable(
  c_dbcsr_acc_bool_t def_mnk, libsmm_acc_data_t datatype, int stack_size, int m, int n, int k, int max_kernel_dim);

/** Device-side error word of the library: bit 0 = a grid barrier of the grouping sort timed out (the
    affected call then wrote nothing), bit 2 = a pipeline wait of an Ozaki kernel timed out, bit 3 = an
    Ozaki stack entry with an offset that is not a multiple of the block size, bit 4 = a wait of the
    staged stack kernel for its block copies timed out. reset != 0 clears it. Synchronises the device.
    The ACC calls report the same word: c_dbcsr_acc_stream_sync and c_dbcsr_acc_device_synchronize
    read it after the synchronisation and return nonzero (error slot: cudaErrorTimeout) when it is
    set; from then on libsmm_acc_process, libsmm_acc_transpose and the batch, DBM and allocation-free
    stack calls return nonzero without doing work, until c_dbcsr_acc_clear_errors consumes the word
    (as the reference's error slot is consumed, src/libxstream_dbcsr.c:57-62). No counterpart in the
    reference for the word itself. */
int libxstream_b200_device_error(int reset);

/** Bound, in GPU clock cycles, of every pipeline wait of the kernels launched after this call (the
    staged stack kernel's waits for its block copies and the Ozaki kernels' mbarrier waits); cycles
    <= 0 restores the default of 4e9 cycles (about two seconds). A wait that runs out sets its bit
    in the device error word and the kernel stops early (the C blocks of that call are then
    incomplete; nothing faults or hangs). A launch
    captured into a CUDA graph keeps the bound that was set when it was captured. Meant for tests of
    the error path and for callers that want a shorter bound. No counterpart in the reference. */
void libxstream_b200_set_wait_limit(long long cycles);
long long libxstream_b200_get_wait_limit(void);

/** Last CUDA error code recorded by the library (0 if none); cleared by c_dbcsr_acc_clear_errors.
    Corresponds to the reference's error slot (libxstream/libxstream_opencl.h:156-194). */
int libxstream_b200_last_error(void);

/** FP64 tensor-pipe (DMMA) peak of the active device in TFLOP/s, measured by a short kernel on
    the given stream (NULL: per-thread default stream). No counterpart in the reference. */
double libxstream_b200_fp64_peak(void* stream);

/** Set the kernel parameters used for FP64 stacks of shape (m, n, k): chunk = entries per warp
    (0: size to each stack), mt/nt = warp sub-tile in 8x8 DMMA tiles (1..4), kp = k-steps per
    register panel (2 or 4), wpb = warps per CTA (1..4). Replaces the OPENCL_LIBSMM_SMM_* tunables
    (samples/smm/smm_kernel.c:194-278). Returns 0 on success. */
int libxstream_b200_set_params(int m, int n, int k, int chunk, int mt, int nt, int kp, int wpb);

/** Read back the parameters used for (m, n, k, stack_size): out6 = {chunk, mt, nt, kp, wpb, sorted}. */
int libxstream_b200_get_params(int m, int n, int k, int stack_size, int* out6);

/** Forget all tuned parameters (defaults apply afterwards). */
void libxstream_b200_clear_params(void);

/** Load tuned parameters from a CSV file (DEVICE;TYPEID;M;N;K;S;GFLOPS;L;MT;NT;KP;WPB), as the
    reference loads OPENCL_LIBSMM_SMM_PARAMS (samples/smm/smm_acc.c:92-152). Returns the number of
    records, or -1 if the file cannot be read. */
int libxstream_b200_load_params(const char* csv_path);

/** Test hook: the nth following device scratch allocation fails (0 disables). No counterpart in
    the reference; used to check that allocation failures surface as nonzero return codes. */
void libxstream_b200_inject_alloc_failure(int nth);

/** Launch profile: when enabled (also by LIBXSTREAM_B200_PROFILE=1), each kernel launch is timed
    with events on its stream and filed under its kernel name with the work it states (flops,
    bytes). Counterpart of the reference's LIBXSTREAM_PROFILE per-kernel histogram
    (src/libxstream.c:2629-2723). */
void libxstream_b200_profile_enable(int on);
void libxstream_b200_profile_reset(void);
/** Totals for one kernel name; waits for its pending launches. Returns 0, or -1 if never launched. */
int libxstream_b200_profile_query(const char* kernel, long* launches, double* ms, double* gflop, double* gbyte);
/** Names of the profiled kernels, ';'-separated, into names[capacity]; returns the length used. */
int libxstream_b200_profile_kernels(char* names, int capacity);

/** A timing-enabled event (c_dbcsr_acc_event_create makes events without timing) and the time in
    ms between two recorded ones (waits for `stop`; -1 on error). No counterpart in the reference. */
int libxstream_b200_event_create_timed(void** event_p);
double libxstream_b200_event_elapsed_ms(void* start, void* stop);

/** CUDA-graph capture of library calls: begin capturing the calls made on `stream` by this thread,
    end the capture into an executable graph (nkernels, if given, receives its number of kernel
    nodes), replay it on a stream, destroy it. A captured libsmm_acc_process replays with the
    arguments and buffers it was captured with. No counterpart in the reference (it enqueues every
    kernel individually, samples/smm/smm_kernel.c:462-507). */
int libxstream_b200_graph_begin(void* stream);
int libxstream_b200_graph_end(void* stream, void** graph_exec, int* nkernels);
int libxstream_b200_graph_launch(void* graph_exec, void* stream);
int libxstream_b200_graph_destroy(void* graph_exec);

/** Allocation-free stack multiply, for callers that cannot let the library allocate device memory
    per call: applications that reserve nearly all device memory for their own allocator at
    start-up, or code that must not take the driver's allocation locks or risk the device
    synchronisation a growing memory pool or cudaFree can cause. Same arguments, results and
    return codes as libsmm_acc_process, with two differences: it never hands the stack to a DBM
    launch hook (libxstream_b200_set_dbm_launch_fn), and it never runs the exhaustive autotuner
    (tuning allocates), so with LIBXSTREAM_B200_AUTOTUNE=1 a shape not yet tuned runs with the
    predicted or default parameters. Its scratch is a fixed 8 MiB device array inside the
    library (held by every GPU that uses the library until the process exits), so a stack that
    needs more (libxstream_b200_process_scratch_bytes) is rejected with a nonzero return and a
    message. The first call on a device looks up the array's device address: make it before any
    stream capture. All calls on a device share the array; calls that overlap on the GPU race and
    must be ordered by the caller. This entry point has no counterpart in the reference. */
int libxstream_b200_process_noalloc(const int* host_param_stack, const int* dev_param_stack, int stack_size,
  libsmm_acc_data_t datatype, const void* dev_a_data, const void* dev_b_data, void* dev_c_data, int m_max, int n_max,
  int k_max, int max_kernel_dim, c_dbcsr_acc_bool_t def_mnk, void* stack_stream, void* c_stream);
/** Size of the allocation-free entry point's scratch array (8 MiB), and the scratch a stack of
    stack_size (m, n, k) FP64 entries needs with the current parameters (0 for an invalid shape). */
size_t libxstream_b200_noalloc_scratch_bytes(void);
size_t libxstream_b200_process_scratch_bytes(int stack_size, int m, int n, int k);

/**
 * Ozaki scheme-1 FP64 GEMM on the int8 tensor cores: C = alpha*op(A)*op(B) + beta*C with
 * column-major device operands (op = 'N' or 'T'), each row of op(A) / column of op(B) split into
 * nslices (1..8; <= 0 means 8) int8 digit slices under power-of-two scaling, slice pairs with
 * sa + sb <= 2*(nslices-1) - trim multiplied with exact int32 sums and recombined in FP64.
 * Replaces ozaki_gemm (samples/ozaki/ozaki_opencl.h:420-421; nslices and trim play the roles of
 * ozaki_init's ndecomp and oztrim, ozaki_opencl.h:328-329) for Scheme 1. Enqueued on stream
 * (NULL: the per-thread default stream); returns 0 on success.
 */
int libxstream_b200_ozaki_gemm(char transa, char transb, int M, int N, int K, double alpha, const double* a, int lda,
  const double* b, int ldb, double beta, double* c, int ldc, int nslices, int trim, void* stream);

/**
 * Ozaki scheme-2 (Chinese remainder) FP64 GEMM on the int8 tensor cores: C = alpha*op(A)*op(B) +
 * beta*C with column-major device operands (op = 'N' or 'T'). Rows of op(A) / columns of op(B) are
 * scaled by their largest power of two and truncated to integers, whose product is computed modulo
 * nmoduli pairwise coprime moduli <= 256 (one unsigned 8-bit tensor-core GEMM each, exact int32 sums)
 * and reconstructed by the CRT in double-double arithmetic. nmoduli 1..20 sets the precision (inputs
 * keep floor((log2 P - log2 K - 2) / 2) bits, at most 53); 0 takes the fewest moduli that keep all 53
 * (16 for K <= 4096). Replaces ozaki_gemm for Scheme 2 (samples/ozaki/ozaki_opencl.h:420-421 with
 * ozaki_init kind 2, ozaki_opencl.h:321-329; nmoduli plays the role of ndecomp). Enqueued on stream
 * (NULL: the per-thread default stream); returns 0 on success.
 */
int libxstream_b200_ozaki2_gemm(char transa, char transb, int M, int N, int K, double alpha, const double* a, int lda,
  const double* b, int ldb, double beta, double* c, int ldc, int nmoduli, void* stream);

/**
 * Plain FP64 GEMM on the FP64 tensor cores (DMMA): C = alpha*A*B + beta*C, column-major device
 * operands, transa = transb = 'N' only (other values return nonzero). The baseline for
 * libxstream_b200_ozaki_gemm; no counterpart in the reference (which compares with host DGEMM).
 */
int libxstream_b200_dgemm(char transa, char transb, int M, int N, int K, double alpha, const double* a, int lda,
  const double* b, int ldb, double beta, double* c, int ldc, void* stream);

/**
 * Ozaki scheme-1 form of libsmm_acc_process for FP64 stacks of one shape with m, n, k <= 64:
 * C[c] += A[a]*B[b] with every block row of A / column of B split into nslices (1..8; <= 0 means 7)
 * int8 digit slices under its own power-of-two scale and the slice pairs with
 * sa + sb <= 2*(nslices-1) - trim multiplied on the int8 tensor cores (exact int32 sums), then
 * recombined and accumulated in FP64. Same data contract as libsmm_acc_process (1-based offsets,
 * B pool already transposed to k x n row-major), plus the pool sizes na, nb in blocks; every offset
 * must be a multiple of the block size (otherwise bit 3 of libxstream_b200_device_error is set).
 * Returns -1 for shapes it does not handle (use libsmm_acc_process), 0 on success. No counterpart in
 * the reference, whose Ozaki code is dense GEMM only (samples/ozaki).
 */
int libxstream_b200_process_ozaki(const int* dev_param_stack, int stack_size, int m, int n, int k, const double* dev_a,
  int na, const double* dev_b, int nb, double* dev_c, int nslices, int trim, void* stream);

/**
 * Exhaustive autotuner of the plain stack kernel (replaces samples/smm/tune_multiply.py's OpenTuner
 * search; the space here is the precompiled tile classes). libxstream_b200_tune_candidates writes
 * the (mt, nt, kp) triples tried for (m, n) and returns their count (the DMMA tile classes, then
 * (1, 1, -1), the register-blocked FMA kernel, where its lane grids cover m x n); libxstream_b200_tune times each
 * on synthetic data of the given shape and stack size (reps calls after one warm-up; seed fixes the
 * data) and, with ozaki_slices > 0 and m, n, k <= 64, the Ozaki form last; ms_out receives the
 * milliseconds per call (-1 for a candidate that does not take the shape). Returns the number of times
 * written, < 0 on error. Synchronous.
 */
int libxstream_b200_tune_candidates(int m, int n, int* mt_nt_kp, int capacity);
int libxstream_b200_tune(int m, int n, int k, int stack_size, int reps, int ozaki_slices, unsigned seed, float* ms_out,
  int capacity, void* stream);

/**
 * Learned parameter predictor: 3-layer FP32 MLP (width 64) from (m, n, k, stack size, exponent
 * spread) to the best of the 32 tile classes (c = (mt-1)*8 + (nt-1)*2 + (kp==4)) and to the
 * plain-vs-Ozaki choice. Samples are raw int quintuples (m, n, k, S, spread); r[N][32] holds each
 * configuration's time divided by the best (0 = not applicable), z[N] is 1 when the Ozaki form was
 * faster, 0 when not, -1 when unmeasured. Training (Adam, device kernels) updates weights in place
 * and records the mean loss per step; grad/forward expose one pass for checking; predict runs the
 * inference kernel; install builds the lookup table used by libsmm_acc_process for shapes without
 * a tuned record (LIBXSTREAM_B200_MLP=<file> installs one at init). No counterpart in the reference
 * beyond its use of LIBXS predict models (samples/smm/tune_multiply.py).
 */
int libxstream_b200_mlp_nweights(void);
int libxstream_b200_mlp_train(const int* raw, const float* r, const float* z, int n, int steps, float lr, float* weights,
  float* loss_hist);
int libxstream_b200_mlp_grad(const float* weights, const int* raw, const float* r, const float* z, int n, float* grad,
  float* loss);
int libxstream_b200_mlp_forward(const float* weights, const int* raw, int n, float* y);
int libxstream_b200_mlp_predict(const float* weights, const int* raw, int n, unsigned char* config, float* confidence,
  float* p_ozaki);
int libxstream_b200_mlp_install(const float* weights, int nweights);
int libxstream_b200_mlp_lookup(int m, int n, int k, int stack_size, int* mt_nt_kp, float* confidence);

/**
 * DBM interplay (samples/smm/smm_acc_opencl.h:114-118). libxstream_b200_dbm_launch_fn_t is the
 * reference's opencl_libsmm_acc_dbm_launch_fn_t: ntasks records, param_format = m | n << 8 | k << 16
 * for one shape (0: mixed shapes). libxstream_b200_set_dbm_launch_fn replaces
 * opencl_libsmm_acc_set_dbm_launch_fn: once set (non-NULL), libsmm_acc_process hands FP64 stacks of
 * one shape to that function with alpha = 1. libxstream_b200_dbm_launch runs such a batch with this
 * library's stack kernels -- 6-int records (m, n, k, a, b, c), 0-based offsets, C += alpha*A*B,
 * layouts as for libsmm_acc_process -- the reuse of LIBSMM kernels by DBM that
 * opencl_libsmm_acc_process(..., param_format) offers (smm_kernel.c:82-88); mixed shapes return -1.
 */
typedef int (*libxstream_b200_dbm_launch_fn_t)(void* stream, double alpha, int ntasks, int param_format, const int* params_host,
  const int* params, const double* pack_a_data, const double* pack_b_data, double* shard_c_data);
void libxstream_b200_set_dbm_launch_fn(libxstream_b200_dbm_launch_fn_t launch_fn);
int libxstream_b200_dbm_launch(void* stream, double alpha, int ntasks, int param_format, const int* params_host,
  const int* params, const double* pack_a_data, const double* pack_b_data, double* shard_c_data);

#if defined(__cplusplus)
}
#endif

#endif /* LIBXSTREAM_B200_H */
