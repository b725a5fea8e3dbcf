/*
 * Allocation-free entry point of the FP64 stack multiply.
 *
 * libsmm_acc_process takes its per-call scratch (the grouped copy of the stack, the sort's bucket
 * tables, the partial tiles of C blocks that span several CTAs) from the device's stream-ordered
 * memory pool. Some callers cannot allow that: an application that reserves nearly all device
 * memory for its own allocator at start-up (so any later allocation can fail at an arbitrary point),
 * or a code path that must not take the driver's allocation locks or risk the implicit device
 * synchronisation a growing pool or cudaFree can cause. For them, libxstream_b200_process_noalloc
 * runs the same kernels with the same results on a fixed scratch area that is part of the library
 * image: a file-scope device array of XS_NOALLOC_SCRATCH_BYTES (8 MiB) that every GPU on which the
 * library is used holds until the process exits. Nothing is allocated or freed per call. Unlike
 * libsmm_acc_process it does not pass stacks to an installed DBM launch hook and does not run the
 * exhaustive autotuner (which allocates its own buffers): it uses the predicted or default
 * parameters of a shape that was not tuned.
 *
 * Limits and rules:
 *   - a call whose stack needs more scratch than the array holds is rejected (nonzero return, a
 *     message on stderr) before any work is queued; libxstream_b200_process_scratch_bytes tells in
 *     advance what a stack needs (with the default parameters on a B200, 8 MiB covers stacks of up
 *     to about 100000 entries of 23x23x23 blocks and about 88000 of 64x64x64 blocks);
 *   - the first call on a device looks up the device address of the array (once per device, with
 *     that device current); make that first call before any stream capture;
 *   - every call on a device uses the same array, and the array keeps what the last call left in
 *     it (each call clears the parts that must start at zero); calls whose work overlaps on the
 *     GPU -- on different streams, or from several host threads -- race on it and must be ordered
 *     by the caller (one stream, or events).
 * This entry point has no counterpart in the reference.
 */
#include "internal.h"
#include "../../include/libxstream_b200.h"
#include <cuda_runtime.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>

#define XS_NOALLOC_SCRATCH_BYTES ((size_t)8 << 20)
#define XS_NOALLOC_MAXDEV 64

/* The scratch area. Host code must not use this name as an address: only the device address
   obtained by cudaGetSymbolAddress is passed to kernels. */
static __device__ __align__(256) unsigned char xs_noalloc_scratch[XS_NOALLOC_SCRATCH_BYTES];

static pthread_mutex_t xs_noalloc_lock = PTHREAD_MUTEX_INITIALIZER;
static void* xs_noalloc_addr[XS_NOALLOC_MAXDEV];

/* Device address of the scratch array on the calling thread's current CUDA device (looked up once
   per device). cudaGetSymbolAddress resolves on that device, so the cache is indexed by it too. */
static int xs_noalloc_scratch_address(void** addr) {
  int result = EXIT_SUCCESS, device = -1;
  if (cudaSuccess != cudaGetDevice(&device)) return xs_record_error((int)cudaGetLastError(), "cudaGetDevice");
  if (0 > device || XS_NOALLOC_MAXDEV <= device) return EXIT_FAILURE;
  pthread_mutex_lock(&xs_noalloc_lock);
  if (nullptr == xs_noalloc_addr[device]) {
    void* p = nullptr;
    const cudaError_t r = cudaGetSymbolAddress(&p, xs_noalloc_scratch);
    if (cudaSuccess == r && nullptr != p) xs_noalloc_addr[device] = p;
    else result = xs_record_error((int)(cudaSuccess != r ? r : cudaErrorInvalidSymbol), "cudaGetSymbolAddress");
  }
  *addr = xs_noalloc_addr[device];
  pthread_mutex_unlock(&xs_noalloc_lock);
  return result;
}

extern "C" {

size_t libxstream_b200_noalloc_scratch_bytes(void) { return XS_NOALLOC_SCRATCH_BYTES; }

size_t libxstream_b200_process_scratch_bytes(int stack_size, int m, int n, int k) {
  xs_smm_params_t prm;
  if (0 >= stack_size || 0 >= m || 0 >= n || 0 >= k || EXIT_SUCCESS != xs_smm_ensure_init()) return 0;
  xs_params_lookup((int)dbcsr_type_real_8, m, n, k, stack_size, &prm);
  return xs_smm_f64_scratch_bytes(stack_size, m, n, k, &prm);
}

int libxstream_b200_process_noalloc(const int* host_param_stack, const int* dev_param_stack, int stack_size,
  libsmm_acc_data_t datatype, const void* dev_a_data, const void* dev_b_data, void* dev_c_data, int m_max, int n_max,
  int k_max, int max_kernel_dim, c_dbcsr_acc_bool_t def_mnk, void* stack_stream, void* c_stream) {
  xs_smm_params_t prm;
  void* scratch = nullptr;
  size_t nbytes;
  int result;
  (void)host_param_stack;
  (void)c_stream;
  if (0 == stack_size) return EXIT_SUCCESS;
  if (!libxstream_b200_process_suitable(def_mnk, datatype, stack_size, m_max, n_max, k_max, max_kernel_dim)) {
    return (0 < stack_size) ? -1 : EXIT_SUCCESS;
  }
  if (nullptr == dev_param_stack || nullptr == dev_a_data || nullptr == dev_b_data || nullptr == dev_c_data) {
    return EXIT_FAILURE;
  }
  if (xs_device_fault_pending()) return EXIT_FAILURE; /* a device error not yet cleared */
  result = xs_smm_ensure_init();
  if (EXIT_SUCCESS != result) return result;
  xs_params_lookup((int)datatype, m_max, n_max, k_max, stack_size, &prm);
  nbytes = xs_smm_f64_scratch_bytes(stack_size, m_max, n_max, k_max, &prm);
  if (nbytes > XS_NOALLOC_SCRATCH_BYTES) {
    fprintf(stderr,
      "ERROR LIBSMM/B200: libxstream_b200_process_noalloc: a stack of %i %ix%ix%i entries needs %zu bytes of scratch, "
      "more than the %zu bytes of the allocation-free entry point (use libsmm_acc_process, or split the stack)\n",
      stack_size, m_max, n_max, k_max, nbytes, XS_NOALLOC_SCRATCH_BYTES);
    return EXIT_FAILURE;
  }
  result = xs_noalloc_scratch_address(&scratch);
  if (EXIT_SUCCESS != result) return result;
  return xs_record_error(xs_launch_smm_f64(dev_param_stack, stack_size, (const double*)dev_a_data,
                           (const double*)dev_b_data, (double*)dev_c_data, m_max, n_max, k_max, &prm, scratch,
                           XS_NOALLOC_SCRATCH_BYTES, nullptr != stack_stream ? stack_stream : xs_default_stream()),
    "libxstream_b200_process_noalloc");
}

}  // extern "C"
