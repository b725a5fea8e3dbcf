/*
 * CP2K "offload" API on the B200 runtime: the names, types and semantics of the reference's
 * libxstream/libxstream_cp2k.h:29-58 (replacing src/libxstream_cp2k.c:23-196), implemented on CUDA
 * streams, events and memory through this library's c_dbcsr_acc_* layer. Like the reference, every
 * function except offloadGetErrorName/offloadGetLastError aborts the process when the underlying call
 * fails; a NULL stream means synchronous.
 */
#ifndef OFFLOAD_CP2K_B200_H
#define OFFLOAD_CP2K_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <stdlib.h>

#if defined(__cplusplus)
extern "C" {
#endif

#define offloadSuccess EXIT_SUCCESS
typedef void* offloadStream_t;
typedef void* offloadEvent_t;
typedef int offloadError_t;

const char* offloadGetErrorName(offloadError_t error);
offloadError_t offloadGetLastError(void);
void offloadMemsetAsync(void* ptr, int val, size_t size, offloadStream_t stream);
void offloadMemset(void* ptr, int val, size_t size);
void offloadMemcpyAsyncHtoD(void* ptr_dev, const void* ptr_hst, size_t size, offloadStream_t stream);
void offloadMemcpyAsyncDtoH(void* ptr_hst, const void* ptr_dev, size_t size, offloadStream_t stream);
void offloadMemcpyAsyncDtoD(void* dst, const void* src, size_t size, offloadStream_t stream);
void offloadMemcpyHtoD(void* ptr_dev, const void* ptr_hst, size_t size);
void offloadMemcpyDtoH(void* ptr_hst, const void* ptr_dev, size_t size);
void offloadMemcpyToSymbol(const void* symbol, const void* src, size_t count);
void offloadEventCreate(offloadEvent_t* event);
void offloadEventDestroy(offloadEvent_t event);
void offloadEventSynchronize(offloadEvent_t event);
void offloadEventRecord(offloadEvent_t event, offloadStream_t stream);
bool offloadEventQuery(offloadEvent_t event);
void offloadStreamCreate(offloadStream_t* stream);
void offloadStreamDestroy(offloadStream_t stream);
void offloadStreamSynchronize(offloadStream_t stream);
void offloadStreamWaitEvent(offloadStream_t stream, offloadEvent_t event);
void offloadMallocHost(void** ptr, size_t size);
void offloadMalloc(void** ptr, size_t size);
void offloadFree(void* ptr);
void offloadFreeHost(void* ptr);
void offloadDeviceSynchronize(void);
void offloadEnsureMallocHeapSize(size_t required_size);

#if defined(__cplusplus)
}
#endif

#endif /* OFFLOAD_CP2K_B200_H */
