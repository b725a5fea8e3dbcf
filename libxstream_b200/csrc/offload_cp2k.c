/*
 * CP2K offload API (include/offload_cp2k.h) over the c_dbcsr_acc_* runtime of this library: thin
 * wrappers that abort on failure, as src/libxstream_cp2k.c:13-196 does. Memset with a non-zero value
 * is a CUDA memset (the DBCSR layer only clears). offloadMemcpyToSymbol has no symbol table to copy
 * into (the reference accepts only the empty case, libxstream_cp2k.c:73-79); offloadEnsureMallocHeapSize
 * raises the device-side malloc heap limit when it is below the request.
 */
#include "internal.h"
#include "../../include/dbcsr_acc.h"
#include "../../include/offload_cp2k.h"
#include <cuda_runtime_api.h>
#include <stdio.h>

static void xs_offload_expect(int result, const char* name) {
  if (EXIT_SUCCESS != result) {
    const int e = xs_last_error();
    fprintf(stderr, "ERROR OFFLOAD/B200: %s failed (%s)\n", name, 0 != e ? cudaGetErrorName((cudaError_t)e) : "unknown");
    abort();
  }
}

const char* offloadGetErrorName(offloadError_t error) { return cudaGetErrorName((cudaError_t)error); }

offloadError_t offloadGetLastError(void) { return (offloadError_t)xs_consume_error(); }

void offloadMemsetAsync(void* ptr, int val, size_t size, offloadStream_t stream) {
  int r;
  if (0 == val) r = c_dbcsr_acc_memset_zero(ptr, 0, size, stream);
  else {
    cudaStream_t s = (NULL != stream) ? (cudaStream_t)stream : cudaStreamPerThread;
    r = (EXIT_SUCCESS == xs_ensure_device()) ? xs_record_error((int)cudaMemsetAsync(ptr, val, size, s), "memset") : EXIT_FAILURE;
    if (EXIT_SUCCESS == r && NULL == stream) r = xs_record_error((int)cudaStreamSynchronize(s), "memset");
  }
  xs_offload_expect(r, "offloadMemsetAsync");
}

void offloadMemset(void* ptr, int val, size_t size) { offloadMemsetAsync(ptr, val, size, NULL); }

void offloadMemcpyAsyncHtoD(void* ptr_dev, const void* ptr_hst, size_t size, offloadStream_t stream) {
  xs_offload_expect(c_dbcsr_acc_memcpy_h2d(ptr_hst, ptr_dev, size, stream), "offloadMemcpyAsyncHtoD");
}

void offloadMemcpyAsyncDtoH(void* ptr_hst, const void* ptr_dev, size_t size, offloadStream_t stream) {
  xs_offload_expect(c_dbcsr_acc_memcpy_d2h(ptr_dev, ptr_hst, size, stream), "offloadMemcpyAsyncDtoH");
}

void offloadMemcpyAsyncDtoD(void* dst, const void* src, size_t size, offloadStream_t stream) {
  xs_offload_expect(c_dbcsr_acc_memcpy_d2d(src, dst, size, stream), "offloadMemcpyAsyncDtoD");
}

void offloadMemcpyHtoD(void* ptr_dev, const void* ptr_hst, size_t size) { offloadMemcpyAsyncHtoD(ptr_dev, ptr_hst, size, NULL); }

void offloadMemcpyDtoH(void* ptr_hst, const void* ptr_dev, size_t size) { offloadMemcpyAsyncDtoH(ptr_hst, ptr_dev, size, NULL); }

void offloadMemcpyToSymbol(const void* symbol, const void* src, size_t count) {
  if (NULL != symbol && NULL != src && 0 != count) {
    fprintf(stderr, "ERROR OFFLOAD/B200: offloadMemcpyToSymbol has no device symbols to copy into\n");
    abort();
  }
}

void offloadEventCreate(offloadEvent_t* event) { xs_offload_expect(c_dbcsr_acc_event_create(event), "offloadEventCreate"); }

void offloadEventDestroy(offloadEvent_t event) { xs_offload_expect(c_dbcsr_acc_event_destroy(event), "offloadEventDestroy"); }

void offloadEventSynchronize(offloadEvent_t event) {
  xs_offload_expect(c_dbcsr_acc_event_synchronize(event), "offloadEventSynchronize");
}

void offloadEventRecord(offloadEvent_t event, offloadStream_t stream) {
  xs_offload_expect(c_dbcsr_acc_event_record(event, stream), "offloadEventRecord");
}

bool offloadEventQuery(offloadEvent_t event) {
  c_dbcsr_acc_bool_t has_occurred = 0;
  xs_offload_expect(c_dbcsr_acc_event_query(event, &has_occurred), "offloadEventQuery");
  return 0 != has_occurred;
}

void offloadStreamCreate(offloadStream_t* stream) {
  xs_offload_expect(c_dbcsr_acc_stream_create(stream, "Offload Stream", 0), "offloadStreamCreate");
}

void offloadStreamDestroy(offloadStream_t stream) { xs_offload_expect(c_dbcsr_acc_stream_destroy(stream), "offloadStreamDestroy"); }

void offloadStreamSynchronize(offloadStream_t stream) {
  xs_offload_expect(c_dbcsr_acc_stream_sync(stream), "offloadStreamSynchronize");
}

void offloadStreamWaitEvent(offloadStream_t stream, offloadEvent_t event) {
  xs_offload_expect(c_dbcsr_acc_stream_wait_event(stream, event), "offloadStreamWaitEvent");
}

void offloadMallocHost(void** ptr, size_t size) { xs_offload_expect(c_dbcsr_acc_host_mem_allocate(ptr, size, NULL), "offloadMallocHost"); }

void offloadMalloc(void** ptr, size_t size) { xs_offload_expect(c_dbcsr_acc_dev_mem_allocate(ptr, size), "offloadMalloc"); }

void offloadFree(void* ptr) { xs_offload_expect(c_dbcsr_acc_dev_mem_deallocate(ptr), "offloadFree"); }

void offloadFreeHost(void* ptr) { xs_offload_expect(c_dbcsr_acc_host_mem_deallocate(ptr, NULL), "offloadFreeHost"); }

void offloadDeviceSynchronize(void) { xs_offload_expect(c_dbcsr_acc_device_synchronize(), "offloadDeviceSynchronize"); }

void offloadEnsureMallocHeapSize(size_t required_size) {
  size_t current = 0;
  int r = xs_ensure_device();
  if (EXIT_SUCCESS == r) r = xs_record_error((int)cudaDeviceGetLimit(&current, cudaLimitMallocHeapSize), "heap size");
  if (EXIT_SUCCESS == r && current < required_size) {
    r = xs_record_error((int)cudaDeviceSetLimit(cudaLimitMallocHeapSize, required_size), "heap size");
  }
  xs_offload_expect(r, "offloadEnsureMallocHeapSize");
}
