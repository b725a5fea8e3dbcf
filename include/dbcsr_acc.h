/*
 * DBCSR accelerator (ACC) runtime ABI, implemented on the CUDA runtime for B200 (sm_100a).
 *
 * These 26 entry points are the ones DBCSR binds when it is built against an accelerator
 * backend. Each declaration below replaces the same-named function of the reference backend:
 *   reference interface: libxstream/libxstream_dbcsr.h:24-64 (declarations),
 *                        src/libxstream_dbcsr.c:37-304 (wrappers),
 *                        samples/smm/acc.h:24-74 (DBCSR's own copy of the prototypes),
 *                        .abi.txt:1-26 (exported names).
 * Conventions kept from the reference:
 *   - every int-returning call returns 0 (EXIT_SUCCESS) on success, nonzero on failure;
 *   - a NULL stream on the memory calls means "synchronous" (the copy has completed on return);
 *   - stream priorities follow CUDA's rule that a lower number is a higher priority;
 *   - c_dbcsr_acc_event_query reports "occurred" when the query itself fails (soft error);
 *   - c_dbcsr_acc_dev_mem_set_ptr(&p, base, lb) sets p = (char*)base + lb.
 */
#ifndef LIBXSTREAM_B200_DBCSR_ACC_H
#define LIBXSTREAM_B200_DBCSR_ACC_H

#include <stddef.h>

#if defined(__cplusplus)
extern "C" {
#endif

/** Boolean used throughout the ACC ABI (replaces libxstream_dbcsr.h:21). */
typedef int c_dbcsr_acc_bool_t;

/** Initialise / finalise the runtime; reference counted (replaces libxstream_dbcsr.h:24-25). */
int c_dbcsr_acc_init(void);
int c_dbcsr_acc_finalize(void);

/** Forget the last recorded error (replaces libxstream_dbcsr.h:28). */
void c_dbcsr_acc_clear_errors(void);

/** Devices (replaces libxstream_dbcsr.h:31-33). */
int c_dbcsr_acc_get_ndevices(int* ndevices);
int c_dbcsr_acc_set_active_device(int device_id);
int c_dbcsr_acc_device_synchronize(void);

/** Streams (replaces libxstream_dbcsr.h:36-42). A lower priority number is a higher priority. */
int c_dbcsr_acc_stream_priority_range(int* least, int* greatest);
int c_dbcsr_acc_stream_create(void** stream_p, const char* name, int priority);
int c_dbcsr_acc_stream_destroy(void* stream);
int c_dbcsr_acc_stream_sync(void* stream);
int c_dbcsr_acc_stream_wait_event(void* stream, void* event);

/** Events (replaces libxstream_dbcsr.h:45-49). */
int c_dbcsr_acc_event_create(void** event_p);
int c_dbcsr_acc_event_destroy(void* event);
int c_dbcsr_acc_event_record(void* event, void* stream);
int c_dbcsr_acc_event_query(void* event, c_dbcsr_acc_bool_t* has_occurred);
int c_dbcsr_acc_event_synchronize(void* event);

/** Memory (replaces libxstream_dbcsr.h:52-61). Device memory comes from the stream-ordered pool. */
int c_dbcsr_acc_dev_mem_allocate(void** dev_mem, size_t nbytes);
int c_dbcsr_acc_dev_mem_deallocate(void* dev_mem);
int c_dbcsr_acc_dev_mem_set_ptr(void** dev_mem, void* other, size_t lb);
int c_dbcsr_acc_host_mem_allocate(void** host_mem, size_t nbytes, void* stream);
int c_dbcsr_acc_host_mem_deallocate(void* host_mem, void* stream);
int c_dbcsr_acc_memcpy_h2d(const void* host_mem, void* dev_mem, size_t nbytes, void* stream);
int c_dbcsr_acc_memcpy_d2h(const void* dev_mem, void* host_mem, size_t nbytes, void* stream);
int c_dbcsr_acc_memcpy_d2d(const void* devmem_src, void* devmem_dst, size_t nbytes, void* stream);
int c_dbcsr_acc_memset_zero(void* dev_mem, size_t offset, size_t nbytes, void* stream);
int c_dbcsr_acc_dev_mem_info(size_t* mem_free, size_t* mem_total);

/**
 * DBCSR's timer hooks (libxstream_dbcsr.h:66-67). DBCSR provides them; this library defines weak
 * no-op versions so it also links and runs standalone.
 */
void c_dbcsr_timeset(const char** routineN, const int* routineN_len, int* handle);
void c_dbcsr_timestop(const int* handle);

#if defined(__cplusplus)
}
#endif

#endif /* LIBXSTREAM_B200_DBCSR_ACC_H */
