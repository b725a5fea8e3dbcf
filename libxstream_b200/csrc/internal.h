/*
 * Internal declarations shared by the C host layer (acc_runtime.c, smm_acc.c, smm_params.c) and
 * the CUDA translation units (smm_kernels.cu and friends). Nothing here is part of the public ABI.
 */
#ifndef LIBXSTREAM_B200_INTERNAL_H
#define LIBXSTREAM_B200_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#if defined(__cplusplus)
extern "C" {
#endif

/* ---------------------------------------------------------------- runtime state (acc_runtime.c) */

/** Make sure the calling thread has the active device current; returns 0 on success. */
int xs_ensure_device(void);
/** Active device id (set by c_dbcsr_acc_set_active_device, default 0). */
int xs_active_device(void);
/** Device ids the runtime tracks per device (SM counts, pools, kernel set-up). */
#define XS_MAXDEV 64
/** The active device as an index of per-device caches, in [0, XS_MAXDEV). */
int xs_device_slot(void);
/** Make the dynamic shared memory limit of kernel `func` on the active device at least `bytes`
    (function attributes are per device): set on first use per device and when a larger size is
    asked for; returns a CUDA error code. */
int xs_func_smem(const void* func, size_t bytes);
/** Number of SMs of the active device (cached). */
int xs_sm_count(void);
/** Record a CUDA error code (nonzero) in the error slot; returns EXIT_FAILURE if code != 0. */
int xs_record_error(int cuda_error, const char* where);
/** Last recorded error code (0 if none). */
int xs_last_error(void);
/** Last recorded error code, and reset the slot. */
int xs_consume_error(void);
/** LIBSMM initialised (lazily, reference counted once) and the active device current. */
int xs_smm_ensure_init(void);
/** Verbosity from LIBXSTREAM_B200_VERBOSE (0 = quiet). */
int xs_verbosity(void);
/** The stream used when the caller passes NULL: the per-thread default stream. */
void* xs_default_stream(void);
/** Stream-ordered scratch allocation from the device's memory pool (no host sync). */
int xs_scratch_alloc(void** ptr, size_t nbytes, void* stream);
int xs_scratch_free(void* ptr, void* stream);
/** Test hook: make the n-th following scratch allocation fail (0 disables). */
void xs_inject_alloc_failure(int nth);
/** Default bound of a kernel's pipeline wait, in clock cycles (about two seconds at 1.965 GHz). */
#define XS_DEFAULT_WAIT_LIMIT 4000000000LL
/** Bound of the kernels' pipeline waits in clock cycles, passed to every launch that has such waits
    (libxstream_b200_set_wait_limit; XS_DEFAULT_WAIT_LIMIT unless set). */
long long xs_wait_limit(void);
/** 1 once a synchronisation found the device error word set, until c_dbcsr_acc_clear_errors. */
int xs_device_fault_pending(void);

/* ------------------------------------------------------------------ launch profile (profile.c) */

/** 1 if per-kernel launch profiling is on. */
int xs_profile_enabled(void);
/** Record a start event on the stream (NULL when profiling is off). */
void* xs_profile_begin(void* stream);
/** Record the stop event and file the launch under `name` with its stated work. */
void xs_profile_end(void* token, const char* name, double flops, double bytes, void* stream);

/* ------------------------------------------------ kernel launchers (smm_kernels.cu, C linkage) */

/** Parameters of the plain FP64 stack kernel; chosen by the parameter table / autotuner. */
typedef struct xs_smm_params_t {
  int chunk;   /* entries per work item (L) */
  int mt, nt;  /* warp sub-tile, in units of 8x8 DMMA tiles (1..4 each) */
  int kp;      /* k-steps (of 4) per register panel: 2 or 4 (1..4 for shape-specialised kernels); 0: staged
                  kernel; XS_KP_FMA: register-blocked FMA kernel (no DMMA tiles) */
  int generic; /* 1: always use the runtime-shape kernel even if a specialised one exists */
  int wpb;     /* warps per CTA */
  int sorted;  /* 1: the stack is known to be grouped by c (skip the device sort) */
} xs_smm_params_t;

/** kp value that selects the register-blocked FMA stack kernel (small blocks). */
#define XS_KP_FMA (-1)
/** Where a lookup's parameters came from. */
#define XS_PARAMS_DEFAULT 0   /* default heuristic */
#define XS_PARAMS_TUNED 1     /* tuned record (table / CSV / autotuner) */
#define XS_PARAMS_PREDICTED 2 /* learned predictor */
#define XS_PARAMS_LOWCONF 3   /* predictor below its confidence threshold (its prediction is used) */
void xs_params_lookup_ex(int type, int m, int n, int k, int stack_size, xs_smm_params_t* out, int* source);
/** Runs the exhaustive tuner for (m, n, k, stack_size) and records the best configuration when
    LIBXSTREAM_B200_AUTOTUNE=1, no tuned record exists, the predictor is absent or not confident,
    and the stream is not being captured. */
void xs_autotune_if_needed(int m, int n, int k, int stack_size, void* stream);
int xs_mlp_load_file(const char* path);

/** Shape-specialised kernels compiled for (m, n, k): writes up to capacity (mt, nt, kp) triples,
    returns how many exist. */
int xs_smm_f64_specialized(int m, int n, int k, int* mt_nt_kp, int capacity);

/** 1 if the register-blocked FMA kernel takes blocks of m x n x k. */
int xs_smm_fma_supported(int m, int n, int k);

/** Size in bytes of the device scratch needed by xs_launch_smm_f64 for this call. */
size_t xs_smm_f64_scratch_bytes(int stack_size, int m, int n, int k, const xs_smm_params_t* params);

/**
 * Plain FP64 stack multiply: sort by c (stable), chunked DMMA accumulation, single write-back per
 * C block piece, deterministic combine of pieces. scratch must hold xs_smm_f64_scratch_bytes().
 * Returns a cudaError_t value (0 = success).
 */
int xs_launch_smm_f64(const int* dev_stack, int stack_size, const double* a, const double* b, double* c, int m, int n,
  int k, const xs_smm_params_t* params, void* scratch, size_t scratch_bytes, void* stream);
/** Same with C += alpha*A*B and the stack in parameter format `format` (0: 1-based (a, b, c) triples;
    otherwise 6-int records whose 0-based (a, b, c) offsets sit at +3, the DBM task layout). */
int xs_launch_smm_f64_ex(const int* dev_stack, int stack_size, int format, double alpha, const double* a, const double* b,
  double* c, int m, int n, int k, const xs_smm_params_t* params, void* scratch, size_t scratch_bytes, void* stream);

/** Device address of the library's device error word (current device). */
unsigned* xs_device_error_ptr(void);
/** Enqueue a copy of the current device's error word into host memory (pinned) on the stream. */
int xs_device_error_fetch(unsigned* host_dst, void* stream);
/** Read (synchronously) / reset the current device's error word; return a cudaError_t value. */
int xs_device_error_read(unsigned* value);
int xs_device_error_clear(void);

/** Ozaki scheme-1 FP64 GEMM on the int8 tensor cores (ozaki_gemm.cu): C = alpha*op(A)*op(B) + beta*C,
    column-major, nslices in 1..8, slice pairs with sa + sb <= cutoff (cutoff < 0: all pairs).
    scratch must hold xs_ozaki_gemm_scratch_bytes(). Returns a cudaError_t value. */
size_t xs_ozaki_gemm_scratch_bytes(int M, int N, int K, int nslices);
int xs_ozaki_gemm(char transa, char transb, int M, int N, int K, double alpha, const double* a, int lda, const double* b,
  int ldb, double beta, double* c, int ldc, int nslices, int cutoff, void* scratch, size_t scratch_bytes, void* stream);

/** Ozaki scheme-2 (CRT) FP64 GEMM on the int8 tensor cores (ozaki2_gemm.cu): C = alpha*op(A)*op(B) +
    beta*C, column-major, nmod moduli (1..20; 0: the fewest that keep all 53 bits for this K).
    scratch must hold xs_ozaki2_gemm_scratch_bytes(). Returns a cudaError_t value. */
int xs_ozaki2_default_moduli(int K);
size_t xs_ozaki2_gemm_scratch_bytes(int M, int N, int K, int nmod);
int xs_ozaki2_gemm(char transa, char transb, int M, int N, int K, double alpha, const double* a, int lda, const double* b,
  int ldb, double beta, double* c, int ldc, int nmod, void* scratch, size_t scratch_bytes, void* stream);

/** Ozaki scheme-1 stack multiply (ozaki_smm.cu): C[c] += A[a]*B[b] for one shape m, n, k <= 64 with
    int8 tensor-core slice products; A pool of na m x k column-major blocks, B pool of nb k x n
    row-major blocks, 1-based block-aligned offsets. Returns a cudaError_t value. */
size_t xs_smm_ozaki_scratch_bytes(int S, int m, int n, int k, int na, int nb, int nslices);
int xs_launch_smm_ozaki(const int* dev_stack, int S, int m, int n, int k, const double* a, int na, const double* b, int nb,
  double* c, int nslices, int cutoff, void* scratch, size_t scratch_bytes, void* stream);

/** Exhaustive autotuner (tune.cu): candidate (mt, nt, kp) triples of the plain kernel for (m, n),
    and the time per call of each (plus the Ozaki form with ozaki_slices > 0) on synthetic data. */
int xs_tune_candidates(int m, int n, int* mt_nt_kp, int cap);
int xs_tune(int m, int n, int k, int S, int reps, int ozaki_slices, unsigned seed, float* ms_out, int cap, void* stream);

/** Learned parameter predictor (mlp.cu): 3-layer FP32 MLP, raw inputs (m, n, k, S, spread) per sample,
    r[N][32] time ratios (0 = configuration not applicable), z[N] Ozaki label (1, 0, or -1 unknown). */
int xs_mlp_nweights(void);
int xs_mlp_train(const int* raw, const float* r, const float* z, int N, int steps, float lr, float* weights, float* loss_hist);
int xs_mlp_grad(const float* weights, const int* raw, const float* r, const float* z, int N, float* grad, float* loss);
int xs_mlp_forward(const float* weights, const int* raw, int N, float* y);
int xs_mlp_predict(const float* weights, const int* raw, int N, unsigned char* cfg, float* conf, float* pz);
int xs_mlp_install(const float* weights);
void xs_mlp_uninstall(void);
int xs_mlp_lookup(int m, int n, int k, int S, int* mt, int* nt, int* kp, float* confidence);

/** Plain FP64 DMMA GEMM (dgemm.cu): C = alpha*A*B + beta*C, column-major, no transposes. */
int xs_dgemm(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb, double beta, double* C,
  int ldc, void* stream);

/** Stable grouping of stacks by c (stack_sort.cu), one cooperative kernel for one stack or a batch:
    splits each AoS stack into keys (c) and payload (a | b << 32), resets the segment list, and
    writes each stack's grouped order to (kout, vout) at its offset off[s], using (k0, v0) and
    (k1, v1) as ping-pong buffers for multi-pass sorts. */
#define XS_MAX_BATCH 16       /* stacks per grouping launch */
#define XS_MAX_CALL_STACKS 64 /* stacks per library call (statistics slots in the control block) */
typedef struct xs_sort_batch_t {
  int nstacks;
  int gidx[XS_MAX_BATCH];       /* index of the stack within the call (statistics slot) */
  const int* stack[XS_MAX_BATCH];
  int format[XS_MAX_BATCH];     /* 0: (a, b, c) triples of 1-based offsets; else 6-int records, 0-based (a, b, c) at +3 */
  int S[XS_MAX_BATCH];          /* entries per stack (>= 1) */
  int off[XS_MAX_BATCH];        /* first output position of each stack */
  int tile_begin[XS_MAX_BATCH]; /* filled by the launcher */
  int ntiles[XS_MAX_BATCH];     /* filled by the launcher */
  unsigned blk[XS_MAX_BATCH];   /* > 0: the stack's C block size (its blocks do not overlap): bucket ids
                                   floor((c - cmin) / blk), no gcd statistics; 0: gcd of the offsets */
  int* zero;                    /* nzero ints the grouping kernel sets to 0 before it ends (or nullptr) */
  int nzero;
} xs_sort_batch_t;
size_t xs_sort_ctl_bytes(void);
/** Zero the call's control block (barrier, error flag, queue, statistics of nstacks stacks). */
int xs_sort_clear_ctl(void* sort_scratch, int nstacks, void* stream);
/** Tiles one grouping launch takes at most, and entries per tile (small / large tiles). */
int xs_sort_launch_tiles(void);
int xs_sort_tile_entries(int large);
size_t xs_stack_sort_scratch_bytes(int S);
size_t xs_stack_sort_scratch_bytes_batch(const xs_sort_batch_t* desc);
/** Largest stack the one-cluster grouping kernel takes (entries). */
int xs_stack_group_cluster_max(void);
/** Largest single stack xs_stack_group takes in one launch (larger stacks are processed in parts). */
int xs_stack_group_max(void);
/** 1 if the batch fits one grouping launch. */
int xs_stack_group_fits(const xs_sort_batch_t* desc);
/** Grouping of a batch that fits one launch; the control block must have been cleared for the call
    (xs_sort_clear_ctl) before the first launch of the call. */
int xs_stack_group(const int* dev_stack, int S, unsigned* k0, unsigned long long* v0, unsigned* k1,
  unsigned long long* v1, unsigned* kout, unsigned long long* vout, int* seglist, void* sort_scratch, void* stream);
/** As xs_stack_group, for either parameter format; also zeroes nzero ints at zero (nullptr: none).
    blk > 0: the C block size (blocks of the stack do not overlap), which spares the gcd statistics.
    heavy > 0: in a single-pass grouping (stacks of at most 32768 entries over at most 2048 block
    positions), the C blocks with at least `heavy` entries come first, then the others, each class in
    offset order (entries of one block stay in stack order). */
int xs_stack_group_ex(const int* dev_stack, int S, int format, unsigned blk, unsigned* k0, unsigned long long* v0, unsigned* k1,
  unsigned long long* v1, unsigned* kout, unsigned long long* vout, int* seglist, int* zero, int nzero, int heavy,
  void* sort_scratch, void* stream);
int xs_stack_group_batch(const xs_sort_batch_t* desc, unsigned* k0, unsigned long long* v0, unsigned* k1,
  unsigned long long* v1, unsigned* kout, unsigned long long* vout, int* seglist, void* sort_scratch, void* stream);
/** Device addresses inside the sort scratch: the work-queue counters of the stack kernels (one per
    tile-class group 0..3, zeroed with the statistics at every call) and the error flag a timed-out
    grid barrier sets. */
unsigned* xs_sort_queue_counter(void* sort_scratch, int which);
const unsigned* xs_sort_error_flag(void* sort_scratch);

/** Batch of stacks (include/libxstream_b200.h: libxstream_b200_stack_t): scratch size and launch. */
struct libxstream_b200_stack_t;
size_t xs_smm_batch_scratch_bytes(const struct libxstream_b200_stack_t* stacks, int nstacks);
int xs_launch_smm_batch(const struct libxstream_b200_stack_t* stacks, int nstacks, void* scratch, size_t scratch_bytes,
  void* stream);

/** In-place batched transpose of m x n blocks (element size esize: 4 or 8). Returns cudaError_t. */
int xs_launch_transpose(const int* dev_trs_stack, int offset, int stack_size, void* data, int esize, int m, int n,
  void* stream);

/** Block Frobenius norms (c_calculate_norms). Returns cudaError_t. */
int xs_launch_norms(const double* mat, int nblks, const int* offsets, const int* nelems, float* norms, void* stream);

/** Measured FP64 DMMA peak (TFLOP/s) via a short microbenchmark on the active device. */
double xs_fp64_peak_tflops(void* stream);

/* ------------------------------------------------------------- parameter table (smm_params.c) */

/** Look up tuned parameters for (type, m, n, k); fills defaults if none are known. */
void xs_params_lookup(int type, int m, int n, int k, int stack_size, xs_smm_params_t* out);
/** Default heuristic parameters (used when the table has no entry). */
void xs_params_default(int m, int n, int k, int stack_size, xs_smm_params_t* out);
/** Load a CSV parameter table (returns number of records or -1). */
int xs_params_load_csv(const char* path);
/** Drop all table entries. */
void xs_params_clear(void);
/** Insert/replace one record. */
int xs_params_set(int type, int m, int n, int k, const xs_smm_params_t* p, double gflops);

#if defined(__cplusplus)
}
#endif

#endif /* LIBXSTREAM_B200_INTERNAL_H */
