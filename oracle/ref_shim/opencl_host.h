/*
 * Host C environment in which the reference's OpenCL C kernels (samples/smm/kernels/multiply.cl,
 * transpose.cl, with the libxstream/opencl/*.h helpers they include) compile as plain C, so that the
 * reference's own kernel code can run on the CPU as a checker of the oracle and of the device
 * results. Test infrastructure only.
 *
 * Execution model: the driver (ref_driver.c) calls the kernel function once per work-item, work-group
 * after work-group, work-item after work-item. That is exact for the configurations the driver builds:
 * no local-memory staging and no barriers in multiply.cl (no SLM_A/B/C/P), and a single work-item per
 * work-group in transpose.cl (WG = 1), where the one work-item does the whole block.
 * Address-space qualifiers vanish, get_group_id/get_local_id read the driver's counters, the global
 * FP atomic add of multiply.cl is a plain add (work-items never run concurrently).
 */
#ifndef XS_REF_OPENCL_HOST_H
#define XS_REF_OPENCL_HOST_H

#include <math.h>
#include <stddef.h>

typedef unsigned long ulong;
typedef unsigned int uint;
typedef unsigned short ushort;

#define kernel
#define __kernel
#define global
#define __global
#define local
#define __local
#define __constant const

extern int xs_ref_group_id, xs_ref_local_id;
#define get_group_id(DIM) xs_ref_group_id
#define get_local_id(DIM) xs_ref_local_id

#define CLK_LOCAL_MEM_FENCE 0
#define barrier(FLAGS) ((void)0)
#define min(A, B) ((A) < (B) ? (A) : (B))
#define max(A, B) ((A) < (B) ? (B) : (A))

/* the FP atomic add the host would select (libxstream_opencl_flags_atomics) */
#define ATOMIC_ADD_GLOBAL(A, B) (*(A) += (B))

#endif
