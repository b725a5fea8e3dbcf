/*
 * DBCSR ACC runtime (c_dbcsr_acc_*) on the CUDA runtime: devices, streams, events and memory.
 *
 * Replaces the reference's OpenCL runtime layer:
 *   src/libxstream_dbcsr.c:37-304   (the 26 ACC wrappers),
 *   src/libxstream_stream.c:54-320  (queues: create with priority, sync, wait),
 *   src/libxstream_event.c:14-169   (marker events: record, device-side wait, query, host sync),
 *   src/libxstream_mem.c:702-1481   (device/host allocation, copies, memset, info),
 *   src/libxstream.c:451-1870       (init/finalize, device count, active device, error slot).
 * Design: streams are cudaStream_t created non-blocking; events are cudaEvent_t without timing;
 * device memory comes from the device's default memory pool through cudaMallocFromPoolAsync
 * (the pool keeps freed memory, so repeated allocations are cheap); host memory is pinned
 * (cudaHostAlloc). A NULL stream on the copy/memset calls means "synchronous", as in the reference.
 */
#include "internal.h"
#include "../../include/dbcsr_acc.h"
#include <cuda_runtime_api.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

static pthread_mutex_t xs_lock = PTHREAD_MUTEX_INITIALIZER;
static int xs_init_count = 0;
static int xs_ndevices = -1;
static int xs_device = 0;
static int xs_error = 0;
static int xs_verbose = -1;
static int xs_smcount[XS_MAXDEV];
static int xs_pool_ready[XS_MAXDEV];
static int xs_alloc_fail_countdown = 0;
static __thread int xs_thread_device = -1;
/* Bound of the kernels' pipeline waits in clock cycles (0: XS_DEFAULT_WAIT_LIMIT). */
static long long xs_wait_cycles = 0;
/* Set once a synchronisation found the device error word non-zero; cleared by
   c_dbcsr_acc_clear_errors. While it is set, the stack calls refuse work. */
static int xs_device_fault = 0;
/* Pinned host words that receive copies of each device's error word at stream synchronisation. */
static unsigned* xs_err_mirror[XS_MAXDEV];

int xs_verbosity(void) {
  if (0 > xs_verbose) {
    const char* const env = getenv("LIBXSTREAM_B200_VERBOSE");
    xs_verbose = (NULL != env && '\0' != *env) ? atoi(env) : 0;
  }
  return xs_verbose;
}

int xs_record_error(int cuda_error, const char* where) {
  if (0 != cuda_error) {
    xs_error = cuda_error;
    if (0 != xs_verbosity()) {
      fprintf(stderr, "ERROR ACC/B200: %s failed: %s (%i)\n", NULL != where ? where : "call",
        cudaGetErrorString((cudaError_t)cuda_error), cuda_error);
    }
    return EXIT_FAILURE;
  }
  return EXIT_SUCCESS;
}

int xs_last_error(void) { return xs_error; }

int xs_consume_error(void) {
  const int e = xs_error;
  xs_error = 0;
  return e;
}

void xs_inject_alloc_failure(int nth) { xs_alloc_fail_countdown = nth; }

long long xs_wait_limit(void) {
  const long long w = __atomic_load_n(&xs_wait_cycles, __ATOMIC_RELAXED);
  return (0 < w) ? w : XS_DEFAULT_WAIT_LIMIT;
}

void libxstream_b200_set_wait_limit(long long cycles) { __atomic_store_n(&xs_wait_cycles, 0 < cycles ? cycles : 0, __ATOMIC_RELAXED); }

long long libxstream_b200_get_wait_limit(void) { return xs_wait_limit(); }

int xs_device_fault_pending(void) { return __atomic_load_n(&xs_device_fault, __ATOMIC_RELAXED); }

/* A device error word read back from the GPU: non-zero means a kernel's bounded wait gave up (or a
   kernel found an input it could not use) and its results are incomplete. That becomes the error
   slot's code (cudaErrorTimeout), a nonzero return, and the sticky flag the stack calls check. */
static int xs_device_status(unsigned word) {
  if (0 == word) return EXIT_SUCCESS;
  __atomic_store_n(&xs_device_fault, 1, __ATOMIC_RELAXED);
  xs_error = (int)cudaErrorTimeout;
  if (0 != xs_verbosity()) {
    fprintf(stderr, "ERROR ACC/B200: a kernel reported a device-side error (error word 0x%x): results are incomplete\n", word);
  }
  return EXIT_FAILURE;
}

/* Pinned host word of the active device for copies of its error word (allocated on first use). */
static unsigned* xs_error_mirror(void) {
  const int d = xs_device_slot();
  unsigned* m = __atomic_load_n(&xs_err_mirror[d], __ATOMIC_ACQUIRE);
  if (NULL == m) {
    void* p = NULL;
    pthread_mutex_lock(&xs_lock);
    m = xs_err_mirror[d];
    if (NULL == m && cudaSuccess == cudaHostAlloc(&p, 64, cudaHostAllocPortable)) {
      *(volatile unsigned*)p = 0;
      m = (unsigned*)p;
      __atomic_store_n(&xs_err_mirror[d], m, __ATOMIC_RELEASE);
    }
    pthread_mutex_unlock(&xs_lock);
    if (NULL == m) (void)cudaGetLastError();
  }
  return m;
}

static int xs_count_devices(void) {
  if (0 > xs_ndevices) {
    int n = 0;
    if (cudaSuccess != cudaGetDeviceCount(&n)) {
      (void)cudaGetLastError();
      n = 0;
    }
    xs_ndevices = (XS_MAXDEV < n ? XS_MAXDEV : n);
  }
  return xs_ndevices;
}

/* Keep freed pool memory cached: repeated per-call scratch allocations then cost no driver call. */
static int xs_setup_pool(int device) {
  if (0 == xs_pool_ready[device]) {
    cudaMemPool_t pool;
    uint64_t threshold = UINT64_MAX;
    int r = (int)cudaDeviceGetDefaultMemPool(&pool, device);
    if (cudaSuccess == r) r = (int)cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    if (cudaSuccess != r) return xs_record_error(r, "memory pool setup");
    if (cudaSuccess != cudaDeviceGetAttribute(&xs_smcount[device], cudaDevAttrMultiProcessorCount, device)) {
      xs_smcount[device] = 148;
    }
    xs_pool_ready[device] = 1;
  }
  return EXIT_SUCCESS;
}

int xs_ensure_device(void) {
  if (xs_thread_device != xs_device) {
    if (xs_device >= xs_count_devices()) return EXIT_FAILURE;
    if (cudaSuccess != cudaSetDevice(xs_device)) return xs_record_error((int)cudaGetLastError(), "cudaSetDevice");
    pthread_mutex_lock(&xs_lock);
    {
      const int r = xs_setup_pool(xs_device);
      pthread_mutex_unlock(&xs_lock);
      if (EXIT_SUCCESS != r) return r;
    }
    xs_thread_device = xs_device;
  }
  return EXIT_SUCCESS;
}

int xs_active_device(void) { return xs_device; }

int xs_device_slot(void) {
  const int d = xs_device;
  return (0 <= d && d < XS_MAXDEV) ? d : 0;
}

/* (device, kernel) -> dynamic shared memory limit already set */
#define XS_FUNC_SLOTS 512
static struct {
  int dev, bytes;
  const void* func;
} xs_func_smem_set[XS_FUNC_SLOTS];
static int xs_func_smem_n = 0;
static pthread_mutex_t xs_func_lock = PTHREAD_MUTEX_INITIALIZER;

int xs_func_smem(const void* func, size_t bytes) {
  const int dev = xs_device_slot();
  int i, r = 0, slot = -1;
  if (bytes <= 48 * 1024) return 0; /* the default limit */
  pthread_mutex_lock(&xs_func_lock);
  for (i = 0; i < xs_func_smem_n; ++i) {
    if (xs_func_smem_set[i].dev == dev && xs_func_smem_set[i].func == func) {
      slot = i;
      break;
    }
  }
  if (0 > slot || xs_func_smem_set[slot].bytes < (int)bytes) {
    r = (int)cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (cudaSuccess == r) {
      if (0 > slot && xs_func_smem_n < XS_FUNC_SLOTS) slot = xs_func_smem_n++; /* a full table: set every time */
      if (0 <= slot) {
        xs_func_smem_set[slot].dev = dev;
        xs_func_smem_set[slot].func = func;
        xs_func_smem_set[slot].bytes = (int)bytes;
      }
    }
  }
  pthread_mutex_unlock(&xs_func_lock);
  return r;
}

int xs_sm_count(void) {
  const int d = xs_device;
  return (0 <= d && d < XS_MAXDEV && 0 < xs_smcount[d]) ? xs_smcount[d] : 148;
}

void* xs_default_stream(void) { return (void*)cudaStreamPerThread; }

int xs_scratch_alloc(void** ptr, size_t nbytes, void* stream) {
  cudaMemPool_t pool;
  int r;
  *ptr = NULL;
  if (0 == nbytes) return EXIT_SUCCESS;
  if (0 < xs_alloc_fail_countdown && 0 == --xs_alloc_fail_countdown) return EXIT_FAILURE; /* injected */
  r = (int)cudaDeviceGetDefaultMemPool(&pool, xs_device);
  if (cudaSuccess == r) r = (int)cudaMallocFromPoolAsync(ptr, nbytes, pool, (cudaStream_t)stream);
  return xs_record_error(r, "cudaMallocFromPoolAsync");
}

int xs_scratch_free(void* ptr, void* stream) {
  if (NULL == ptr) return EXIT_SUCCESS;
  return xs_record_error((int)cudaFreeAsync(ptr, (cudaStream_t)stream), "cudaFreeAsync");
}

/* ------------------------------------------------------------------------- init / finalize */

int c_dbcsr_acc_init(void) {
  int result = EXIT_SUCCESS;
  pthread_mutex_lock(&xs_lock);
  if (0 == xs_init_count) {
    const char* const env = getenv("LIBXSTREAM_B200_DEVICE");
    const int n = xs_count_devices();
    if (0 >= n) result = EXIT_FAILURE;
    else {
      const int d = (NULL != env && '\0' != *env) ? atoi(env) : 0;
      xs_device = (0 <= d && d < n) ? d : 0;
    }
  }
  if (EXIT_SUCCESS == result) ++xs_init_count;
  pthread_mutex_unlock(&xs_lock);
  if (EXIT_SUCCESS == result) result = xs_ensure_device();
  return result;
}

int c_dbcsr_acc_finalize(void) {
  int result = EXIT_SUCCESS;
  pthread_mutex_lock(&xs_lock);
  if (0 < xs_init_count) --xs_init_count;
  pthread_mutex_unlock(&xs_lock);
  return result;
}

void c_dbcsr_acc_clear_errors(void) {
  xs_error = 0;
  (void)cudaGetLastError();
  if (0 < xs_init_count && EXIT_SUCCESS == xs_ensure_device()) { /* consume the device error word */
    unsigned w = 0;
    if (cudaSuccess != xs_device_error_read(&w) || 0 != w) (void)xs_device_error_clear();
    (void)cudaGetLastError();
  }
  __atomic_store_n(&xs_device_fault, 0, __ATOMIC_RELAXED);
}

/* ---------------------------------------------------------------------------------- devices */

int c_dbcsr_acc_get_ndevices(int* ndevices) {
  if (NULL == ndevices) return EXIT_FAILURE;
  *ndevices = xs_count_devices();
  return EXIT_SUCCESS;
}

int c_dbcsr_acc_set_active_device(int device_id) {
  if (0 > device_id || device_id >= xs_count_devices()) return EXIT_FAILURE;
  xs_device = device_id;
  xs_thread_device = -1;
  return xs_ensure_device();
}

int c_dbcsr_acc_device_synchronize(void) {
  unsigned w = 0;
  int r;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  r = xs_record_error((int)cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  if (EXIT_SUCCESS == r) r = xs_record_error(xs_device_error_read(&w), "device error word");
  return (EXIT_SUCCESS == r) ? xs_device_status(w) : r;
}

/* ---------------------------------------------------------------------------------- streams */

int c_dbcsr_acc_stream_priority_range(int* least, int* greatest) {
  int lo = 0, hi = 0;
  if (NULL == least && NULL == greatest) return EXIT_FAILURE;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  if (cudaSuccess != cudaDeviceGetStreamPriorityRange(&lo, &hi)) return xs_record_error((int)cudaGetLastError(), "priority");
  if (NULL != least) *least = lo;
  if (NULL != greatest) *greatest = hi;
  return EXIT_SUCCESS;
}

int c_dbcsr_acc_stream_create(void** stream_p, const char* name, int priority) {
  cudaStream_t s = NULL;
  int lo = 0, hi = 0, r;
  (void)name;
  if (NULL == stream_p) return EXIT_FAILURE;
  *stream_p = NULL;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  if (cudaSuccess != cudaDeviceGetStreamPriorityRange(&lo, &hi)) lo = hi = 0;
  /* priorities outside [greatest, least] (e.g. -1 as "default" on a device whose range is 0..0) clamp */
  if (priority > lo) priority = lo;
  if (priority < hi) priority = hi;
  r = (int)cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, priority);
  if (cudaSuccess == r) *stream_p = (void*)s;
  return xs_record_error(r, "cudaStreamCreateWithPriority");
}

int c_dbcsr_acc_stream_destroy(void* stream) {
  if (NULL == stream) return EXIT_SUCCESS;
  return xs_record_error((int)cudaStreamDestroy((cudaStream_t)stream), "cudaStreamDestroy");
}

/* The device error word is copied into a pinned host word on the same stream just before the
   synchronisation, so reading it costs no extra round trip. */
int c_dbcsr_acc_stream_sync(void* stream) {
  const cudaStream_t s = NULL != stream ? (cudaStream_t)stream : cudaStreamPerThread;
  unsigned* mirror;
  int r;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  mirror = xs_error_mirror();
  if (NULL != mirror && EXIT_SUCCESS != xs_record_error(xs_device_error_fetch(mirror, s), "device error word")) {
    return EXIT_FAILURE;
  }
  r = xs_record_error((int)cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return (EXIT_SUCCESS == r && NULL != mirror) ? xs_device_status(*(volatile unsigned*)mirror) : r;
}

int c_dbcsr_acc_stream_wait_event(void* stream, void* event) {
  if (NULL == event) return EXIT_FAILURE;
  return xs_record_error(
    (int)cudaStreamWaitEvent(NULL != stream ? (cudaStream_t)stream : cudaStreamPerThread, (cudaEvent_t)event, 0),
    "cudaStreamWaitEvent");
}

/* ----------------------------------------------------------------------------------- events */

int c_dbcsr_acc_event_create(void** event_p) {
  cudaEvent_t e = NULL;
  int r;
  if (NULL == event_p) return EXIT_FAILURE;
  *event_p = NULL;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  r = (int)cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  if (cudaSuccess == r) *event_p = (void*)e;
  return xs_record_error(r, "cudaEventCreate");
}

int c_dbcsr_acc_event_destroy(void* event) {
  if (NULL == event) return EXIT_SUCCESS;
  return xs_record_error((int)cudaEventDestroy((cudaEvent_t)event), "cudaEventDestroy");
}

int c_dbcsr_acc_event_record(void* event, void* stream) {
  if (NULL == event) return EXIT_FAILURE;
  return xs_record_error(
    (int)cudaEventRecord((cudaEvent_t)event, NULL != stream ? (cudaStream_t)stream : cudaStreamPerThread), "cudaEventRecord");
}

int c_dbcsr_acc_event_query(void* event, c_dbcsr_acc_bool_t* has_occurred) {
  cudaError_t r;
  if (NULL == has_occurred) return EXIT_FAILURE;
  if (NULL == event) { /* an empty event counts as occurred (soft error, as the reference) */
    *has_occurred = 1;
    return EXIT_SUCCESS;
  }
  r = cudaEventQuery((cudaEvent_t)event);
  if (cudaSuccess == r) *has_occurred = 1;
  else if (cudaErrorNotReady == r) *has_occurred = 0;
  else { /* error state: report occurred and succeed, like src/libxstream_event.c:131-134 */
    (void)cudaGetLastError();
    *has_occurred = 1;
  }
  return EXIT_SUCCESS;
}

int c_dbcsr_acc_event_synchronize(void* event) {
  if (NULL == event) return EXIT_SUCCESS;
  return xs_record_error((int)cudaEventSynchronize((cudaEvent_t)event), "cudaEventSynchronize");
}

/* ----------------------------------------------------------------------------------- memory */

int c_dbcsr_acc_dev_mem_allocate(void** dev_mem, size_t nbytes) {
  int r;
  if (NULL == dev_mem) return EXIT_FAILURE;
  *dev_mem = NULL;
  if (0 == nbytes) return EXIT_SUCCESS;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  r = xs_scratch_alloc(dev_mem, nbytes, (void*)cudaStreamPerThread);
  /* the allocation must be usable from any stream once this call returns */
  if (EXIT_SUCCESS == r) r = xs_record_error((int)cudaStreamSynchronize(cudaStreamPerThread), "allocate sync");
  if (EXIT_SUCCESS != r) *dev_mem = NULL;
  return r;
}

int c_dbcsr_acc_dev_mem_deallocate(void* dev_mem) {
  int r;
  if (NULL == dev_mem) return EXIT_SUCCESS;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  /* work queued on any stream may still use the buffer: finish it before returning it to the pool */
  r = xs_record_error((int)cudaDeviceSynchronize(), "deallocate sync");
  if (EXIT_SUCCESS == r) r = xs_scratch_free(dev_mem, (void*)cudaStreamPerThread);
  if (EXIT_SUCCESS == r) r = xs_record_error((int)cudaStreamSynchronize(cudaStreamPerThread), "deallocate");
  return r;
}

int c_dbcsr_acc_dev_mem_set_ptr(void** dev_mem, void* other, size_t lb) {
  if (NULL == dev_mem) return EXIT_FAILURE;
  *dev_mem = (NULL != other) ? (void*)((char*)other + lb) : NULL;
  return EXIT_SUCCESS;
}

int c_dbcsr_acc_host_mem_allocate(void** host_mem, size_t nbytes, void* stream) {
  int r;
  (void)stream;
  if (NULL == host_mem) return EXIT_FAILURE;
  *host_mem = NULL;
  if (0 == nbytes) return EXIT_SUCCESS;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  r = (int)cudaHostAlloc(host_mem, nbytes, cudaHostAllocPortable);
  if (cudaSuccess != r) *host_mem = NULL;
  return xs_record_error(r, "cudaHostAlloc");
}

int c_dbcsr_acc_host_mem_deallocate(void* host_mem, void* stream) {
  if (NULL == host_mem) return EXIT_SUCCESS;
  if (NULL != stream && cudaSuccess != cudaStreamSynchronize((cudaStream_t)stream)) {
    return xs_record_error((int)cudaGetLastError(), "host free sync");
  }
  return xs_record_error((int)cudaFreeHost(host_mem), "cudaFreeHost");
}

static int xs_copy(void* dst, const void* src, size_t nbytes, enum cudaMemcpyKind kind, void* stream, const char* what) {
  cudaStream_t s;
  int r;
  if (NULL == dst || NULL == src || 0 == nbytes || dst == src) return EXIT_SUCCESS;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  s = (NULL != stream) ? (cudaStream_t)stream : cudaStreamPerThread;
  r = (int)cudaMemcpyAsync(dst, src, nbytes, kind, s);
  if (cudaSuccess == r && NULL == stream) r = (int)cudaStreamSynchronize(s);
  return xs_record_error(r, what);
}

int c_dbcsr_acc_memcpy_h2d(const void* host_mem, void* dev_mem, size_t nbytes, void* stream) {
  return xs_copy(dev_mem, host_mem, nbytes, cudaMemcpyHostToDevice, stream, "memcpy_h2d");
}

int c_dbcsr_acc_memcpy_d2h(const void* dev_mem, void* host_mem, size_t nbytes, void* stream) {
  return xs_copy(host_mem, dev_mem, nbytes, cudaMemcpyDeviceToHost, stream, "memcpy_d2h");
}

int c_dbcsr_acc_memcpy_d2d(const void* devmem_src, void* devmem_dst, size_t nbytes, void* stream) {
  return xs_copy(devmem_dst, devmem_src, nbytes, cudaMemcpyDeviceToDevice, stream, "memcpy_d2d");
}

int c_dbcsr_acc_memset_zero(void* dev_mem, size_t offset, size_t nbytes, void* stream) {
  cudaStream_t s;
  int r;
  if (0 == nbytes) return EXIT_SUCCESS;
  if (NULL == dev_mem) return EXIT_FAILURE;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  s = (NULL != stream) ? (cudaStream_t)stream : cudaStreamPerThread;
  r = (int)cudaMemsetAsync((char*)dev_mem + offset, 0, nbytes, s);
  if (cudaSuccess == r && NULL == stream) r = (int)cudaStreamSynchronize(s);
  return xs_record_error(r, "memset_zero");
}

int c_dbcsr_acc_dev_mem_info(size_t* mem_free, size_t* mem_total) {
  size_t f = 0, t = 0;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  if (cudaSuccess != cudaMemGetInfo(&f, &t)) return xs_record_error((int)cudaGetLastError(), "cudaMemGetInfo");
  if (NULL != mem_free) *mem_free = f;
  if (NULL != mem_total) *mem_total = t;
  return EXIT_SUCCESS;
}

/* DBCSR normally provides these; weak definitions keep the library usable on its own. */
__attribute__((weak)) void c_dbcsr_timeset(const char** routineN, const int* routineN_len, int* handle) {
  (void)routineN;
  (void)routineN_len;
  if (NULL != handle) *handle = 0;
}

__attribute__((weak)) void c_dbcsr_timestop(const int* handle) { (void)handle; }
