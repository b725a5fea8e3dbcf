/*
 * LIBSMM host layer (C): libsmm_acc_init/finalize/is_thread_safe/process/transpose and
 * c_calculate_norms, dispatching to the precompiled sm_100a kernels in smm_kernels.cu.
 *
 * Replaces samples/smm/smm_acc.c:43-604 (init, finalize, thread safety, suitability, process),
 * samples/smm/smm_kernel.c:82-528 (parameter resolution + launch) and samples/smm/smm_trans.c:48-228
 * (transpose). Behaviour kept from the reference:
 *   - init/finalize are reference counted; c_dbcsr_acc_init alone is enough for DBCSR
 *     (smm_acc.c:51-62), so process/transpose initialise lazily;
 *   - a stack is handled iff def_mnk != 0, 0 < m*n <= max_kernel_dim^2, 0 < k, type is handled
 *     (smm_acc.c:527-573); otherwise a non-empty stack returns -1 (host fallback,
 *     smm_kernel.c:524-526) and an empty stack returns 0;
 *   - transpose of a 1x1 block, of an unsupported type or of m*n > max_kernel_dim^2 is a
 *     successful no-op (smm_trans.c:54-68);
 *   - host_param_stack and c_stream are accepted and not needed (smm_kernel.c:86-87).
 * FP64 (dbcsr_type_real_8) is the type this library computes; FP32 stacks return -1 so that DBCSR
 * takes its host path, which the reference also does when built without OPENCL_LIBSMM_F32.
 * Parameters come from the table (B200SMM_PARAMS=<csv> loads one, =0 disables it) or from the
 * default heuristic; LIBXSTREAM_B200_VERBOSE=2 prints the choice per shape, 3 prints every launch.
 * Device-side errors (a bounded wait that gave up) are read at the synchronisation points
 * (c_dbcsr_acc_stream_sync, c_dbcsr_acc_device_synchronize); once one was seen, the stack calls
 * here return EXIT_FAILURE without work until c_dbcsr_acc_clear_errors.
 */
#include "internal.h"
#include "../../include/libsmm_acc.h"
#include "../../include/libxstream_b200.h"
#include <dlfcn.h>
#include <pthread.h>
#include <string.h>
#include <unistd.h>
#include <stdio.h>
#include <stdlib.h>

static pthread_mutex_t xs_smm_lock = PTHREAD_MUTEX_INITIALIZER;
static int xs_smm_initialized = 0;

int libsmm_acc_init(void) {
  int result = EXIT_SUCCESS;
  pthread_mutex_lock(&xs_smm_lock);
  if (0 == xs_smm_initialized) {
    const char* const env = getenv("B200SMM_PARAMS");
    result = c_dbcsr_acc_init();
    if (EXIT_SUCCESS == result && NULL != env && '\0' != *env && '0' != *env) {
      const int n = xs_params_load_csv(env);
      if (0 > n) fprintf(stderr, "WARNING LIBSMM/B200: cannot read parameter file \"%s\"\n", env);
      else if (2 <= xs_verbosity()) fprintf(stderr, "INFO LIBSMM/B200: %i tuned record(s) from %s\n", n, env);
    }
  }
  if (EXIT_SUCCESS == result) ++xs_smm_initialized;
  pthread_mutex_unlock(&xs_smm_lock);
  if (EXIT_SUCCESS == result && 1 == xs_smm_initialized) { /* learned predictor */
    const char* const mlp = getenv("LIBXSTREAM_B200_MLP");
    if (NULL != mlp && '\0' != *mlp) {
      if ('0' != *mlp && EXIT_SUCCESS == xs_ensure_device() && EXIT_SUCCESS != xs_mlp_load_file(mlp)) {
        fprintf(stderr, "WARNING LIBSMM/B200: cannot load predictor \"%s\"\n", mlp);
      }
    }
    else { /* the predictor shipped next to the library: <dir of the .so>/../params/mlp_b200.txt */
      Dl_info info;
      if (0 != dladdr((void*)&libsmm_acc_init, &info) && NULL != info.dli_fname) {
        char path[4096];
        const char* const slash = strrchr(info.dli_fname, '/');
        const int dirlen = (NULL != slash) ? (int)(slash - info.dli_fname) : 1;
        snprintf(path, sizeof(path), "%.*s/../params/mlp_b200.txt", dirlen, NULL != slash ? info.dli_fname : ".");
        if (0 == access(path, R_OK) && EXIT_SUCCESS == xs_ensure_device() && EXIT_SUCCESS == xs_mlp_load_file(path) &&
            2 <= xs_verbosity()) {
          fprintf(stderr, "INFO LIBSMM/B200: predictor %s\n", path);
        }
      }
    }
  }
  return result;
}

int libsmm_acc_finalize(void) {
  int result = EXIT_SUCCESS;
  pthread_mutex_lock(&xs_smm_lock);
  if (0 < xs_smm_initialized) {
    --xs_smm_initialized;
    if (0 == xs_smm_initialized) result = c_dbcsr_acc_finalize();
  }
  pthread_mutex_unlock(&xs_smm_lock);
  return result;
}

c_dbcsr_acc_bool_t libsmm_acc_is_thread_safe(void) { return 1; }

static int xs_lazy_init(void) {
  int result = EXIT_SUCCESS;
  if (0 == xs_smm_initialized) result = libsmm_acc_init();
  if (EXIT_SUCCESS == result) result = xs_ensure_device();
  return result;
}

int xs_smm_ensure_init(void) { return xs_lazy_init(); }

int libxstream_b200_process_suitable(
  c_dbcsr_acc_bool_t def_mnk, libsmm_acc_data_t datatype, int stack_size, int m, int n, int k, int max_kernel_dim) {
  const long mn = (long)m * n;
  if (0 >= m || 0 >= n || 0 >= k || 0 >= stack_size || 0 == def_mnk) return 0;
  if (mn > (long)max_kernel_dim * max_kernel_dim) return 0;
  return (dbcsr_type_real_8 == datatype) ? 1 : 0;
}

static int xs_process_format(const int* dev_param_stack, int stack_size, int format, double alpha, libsmm_acc_data_t datatype,
  const void* dev_a_data, const void* dev_b_data, void* dev_c_data, int m_max, int n_max, int k_max, int max_kernel_dim,
  c_dbcsr_acc_bool_t def_mnk, void* stack_stream);

/* DBM launch hook (samples/smm/smm_kernel.c:71-76, smm_acc.c:579-585): when set, FP64 stacks of one
   shape go to the caller's kernel with the shape packed as m | n << 8 | k << 16. */
static libxstream_b200_dbm_launch_fn_t xs_dbm_launch_fn = NULL;

void libxstream_b200_set_dbm_launch_fn(libxstream_b200_dbm_launch_fn_t launch_fn) { xs_dbm_launch_fn = launch_fn; }

int libsmm_acc_process(const int* host_param_stack, const int* dev_param_stack, int stack_size, libsmm_acc_data_t datatype,
  const void* dev_a_data, const void* dev_b_data, void* dev_c_data, int m_max, int n_max, int k_max, int max_kernel_dim,
  c_dbcsr_acc_bool_t def_mnk, void* stack_stream, void* c_stream) {
  if (NULL != xs_dbm_launch_fn && dbcsr_type_real_8 == datatype && 0 != def_mnk && 0 < stack_size && m_max < 128 && n_max < 128 &&
      k_max < 128) {
    return xs_dbm_launch_fn(stack_stream, 1.0, stack_size, m_max | (n_max << 8) | (k_max << 16), host_param_stack, dev_param_stack,
      (const double*)dev_a_data, (const double*)dev_b_data, (double*)dev_c_data);
  }
  return xs_process_format(dev_param_stack, stack_size, 0, 1.0, datatype, dev_a_data, dev_b_data, dev_c_data, m_max, n_max,
    k_max, max_kernel_dim, def_mnk, stack_stream);
}

/* The DBM side (opencl_libsmm_acc_process with param_format != 0, smm_kernel.c:82-88 and
   multiply.cl:96-99): ntasks 6-int records (m, n, k, a, b, c) with 0-based offsets, all of the
   shape packed into param_format (m | n << 8 | k << 16), C += alpha * A * B. Mixed shapes
   (param_format 0) are not handled here (-1). The signature is libxstream_b200_dbm_launch_fn_t, so
   this function can itself be installed as the hook. */
int libxstream_b200_dbm_launch(void* stream, double alpha, int ntasks, int param_format, const int* params_host,
  const int* params, const double* pack_a_data, const double* pack_b_data, double* shard_c_data) {
  const int m = param_format & 255, n = (param_format >> 8) & 255, k = (param_format >> 16) & 255;
  (void)params_host;
  if (0 >= ntasks) return EXIT_SUCCESS;
  if (0 == m || 0 == n || 0 == k) return -1;
  return xs_process_format(params, ntasks, 1, alpha, dbcsr_type_real_8, pack_a_data, pack_b_data, shard_c_data, m, n, k, 80, 1,
    stream);
}

static int xs_process_format(const int* dev_param_stack, int stack_size, int format, double alpha, libsmm_acc_data_t datatype,
  const void* dev_a_data, const void* dev_b_data, void* dev_c_data, int m_max, int n_max, int k_max, int max_kernel_dim,
  c_dbcsr_acc_bool_t def_mnk, void* stack_stream) {
  xs_smm_params_t prm;
  void* stream = (NULL != stack_stream) ? stack_stream : xs_default_stream();
  void* scratch = NULL;
  size_t nbytes;
  int result;
  if (0 == stack_size) return EXIT_SUCCESS;
  if (!libxstream_b200_process_suitable(def_mnk, datatype, stack_size, m_max, n_max, k_max, max_kernel_dim)) {
    if (2 <= xs_verbosity()) {
      fprintf(stderr, "INFO LIBSMM/B200: SMM-kernel %ix%ix%i (type %i) ss=%i is %s\n", m_max, n_max, k_max, (int)datatype,
        stack_size, 0 == def_mnk ? "inhomogeneous" : "not handled");
    }
    return (0 < stack_size) ? -1 : EXIT_SUCCESS;
  }
  if (NULL == dev_param_stack || NULL == dev_a_data || NULL == dev_b_data || NULL == dev_c_data) return EXIT_FAILURE;
  if (xs_device_fault_pending()) return EXIT_FAILURE; /* a device error not yet cleared */
  result = xs_lazy_init();
  if (EXIT_SUCCESS != result) return result;
  xs_autotune_if_needed(m_max, n_max, k_max, stack_size, stream);
  xs_params_lookup((int)datatype, m_max, n_max, k_max, stack_size, &prm);
  if (3 <= xs_verbosity()) {
    fprintf(stderr, "INFO LIBSMM/B200: SMM-kernel %ix%ix%i L=%i MT=%i NT=%i KP=%i WPB=%i ss=%i\n", m_max, n_max, k_max,
      prm.chunk, prm.mt, prm.nt, prm.kp, prm.wpb, stack_size);
  }
  nbytes = xs_smm_f64_scratch_bytes(stack_size, m_max, n_max, k_max, &prm);
  result = xs_scratch_alloc(&scratch, nbytes, stream);
  if (EXIT_SUCCESS == result) {
    result = xs_record_error(xs_launch_smm_f64_ex(dev_param_stack, stack_size, format, alpha, (const double*)dev_a_data,
                               (const double*)dev_b_data, (double*)dev_c_data, m_max, n_max, k_max, &prm, scratch, nbytes,
                               stream),
      "libsmm_acc_process");
    if (EXIT_SUCCESS != xs_scratch_free(scratch, stream)) result = EXIT_FAILURE;
  }
  return result;
}

int libsmm_acc_transpose(const int* dev_trs_stack, int offset, int stack_size, void* dev_data, libsmm_acc_data_t datatype,
  int m, int n, int max_kernel_dim, void* stream) {
  const long mn = (long)m * n;
  int esize, result;
  if (0 == stack_size || 1 == mn) return EXIT_SUCCESS;
  if (0 > stack_size || 0 > offset || 0 >= m || 0 >= n) return EXIT_FAILURE;
  if (mn > (long)max_kernel_dim * max_kernel_dim) return EXIT_SUCCESS;
  if (dbcsr_type_real_8 == datatype) esize = 8;
  else if (dbcsr_type_real_4 == datatype) esize = 4;
  else return EXIT_SUCCESS;
  if (NULL == dev_trs_stack || NULL == dev_data) return EXIT_FAILURE;
  if (xs_device_fault_pending()) return EXIT_FAILURE;
  result = xs_lazy_init();
  if (EXIT_SUCCESS != result) return result;
  return xs_record_error(xs_launch_transpose(dev_trs_stack, offset, stack_size, dev_data, esize, m, n,
                           NULL != stream ? stream : xs_default_stream()),
    "libsmm_acc_transpose");
}

int c_calculate_norms(const double* mat, int nblks, const int* offsets, const int* nelems, float* norms, void* stream_ptr) {
  int result;
  if (0 == nblks) return EXIT_SUCCESS;
  if (0 > nblks || NULL == mat || NULL == offsets || NULL == nelems || NULL == norms) return EXIT_FAILURE;
  result = xs_lazy_init();
  if (EXIT_SUCCESS != result) return result;
  return xs_record_error(
    xs_launch_norms(mat, nblks, offsets, nelems, norms, NULL != stream_ptr ? stream_ptr : xs_default_stream()),
    "c_calculate_norms");
}

/* ------------------------------------------------------------------- extension entry points */

static int xs_process_batch_part(const libxstream_b200_stack_t* stacks, int nstacks, void* stream) {
  void* scratch = NULL;
  size_t nbytes = xs_smm_batch_scratch_bytes(stacks, nstacks);
  int result;
  if (0 == nbytes) { /* too many parts for one launch set: split the list */
    const int half = nstacks / 2;
    if (1 >= nstacks) return EXIT_FAILURE;
    result = xs_process_batch_part(stacks, half, stream);
    if (EXIT_SUCCESS == result) result = xs_process_batch_part(stacks + half, nstacks - half, stream);
    return result;
  }
  result = xs_scratch_alloc(&scratch, nbytes, stream);
  if (EXIT_SUCCESS == result) {
    result = xs_record_error(xs_launch_smm_batch(stacks, nstacks, scratch, nbytes, stream), "libxstream_b200_process_batch");
    if (EXIT_SUCCESS != xs_scratch_free(scratch, stream)) result = EXIT_FAILURE;
  }
  return result;
}

int libxstream_b200_process_batch(const libxstream_b200_stack_t* stacks, int nstacks, int max_kernel_dim, void* stream) {
  int i, nonempty = 0, result;
  if (0 >= nstacks) return EXIT_SUCCESS;
  if (NULL == stacks) return EXIT_FAILURE;
  for (i = 0; i < nstacks; ++i) {
    const libxstream_b200_stack_t* const d = stacks + i;
    if (0 > d->stack_size) return -1;
    if (0 == d->stack_size) continue;
    if (!libxstream_b200_process_suitable(1, dbcsr_type_real_8, d->stack_size, d->m, d->n, d->k, max_kernel_dim)) return -1;
    if (NULL == d->dev_param_stack || NULL == d->a || NULL == d->b || NULL == d->c) return EXIT_FAILURE;
    ++nonempty;
  }
  if (0 == nonempty) return EXIT_SUCCESS;
  if (xs_device_fault_pending()) return EXIT_FAILURE;
  result = xs_lazy_init();
  if (EXIT_SUCCESS != result) return result;
  return xs_process_batch_part(stacks, nstacks, NULL != stream ? stream : xs_default_stream());
}

int libxstream_b200_last_error(void) { return xs_last_error(); }

double libxstream_b200_fp64_peak(void* stream) {
  if (EXIT_SUCCESS != xs_lazy_init()) return -1.0;
  return xs_fp64_peak_tflops(NULL != stream ? stream : xs_default_stream());
}

int libxstream_b200_set_params(int m, int n, int k, int chunk, int mt, int nt, int kp, int wpb) {
  xs_smm_params_t p;
  p.chunk = chunk;
  p.mt = mt;
  p.nt = nt;
  p.kp = kp;
  p.wpb = wpb;
  p.sorted = 0;
  p.generic = 0;
  return xs_params_set((int)dbcsr_type_real_8, m, n, k, &p, 0.0);
}

int libxstream_b200_get_params(int m, int n, int k, int stack_size, int* out6) {
  xs_smm_params_t p;
  if (NULL == out6) return EXIT_FAILURE;
  xs_params_lookup((int)dbcsr_type_real_8, m, n, k, stack_size, &p);
  out6[0] = p.chunk;
  out6[1] = p.mt;
  out6[2] = p.nt;
  out6[3] = p.kp;
  out6[4] = p.wpb;
  out6[5] = p.sorted;
  return EXIT_SUCCESS;
}

void libxstream_b200_clear_params(void) { xs_params_clear(); }

int libxstream_b200_load_params(const char* csv_path) { return xs_params_load_csv(csv_path); }

void libxstream_b200_inject_alloc_failure(int nth) { xs_inject_alloc_failure(nth); }
