/*
 * Runs a reference OpenCL C kernel compiled as C (see opencl_host.h): every work-group, and in it
 * every work-item, one after the other. Test infrastructure only. The kernel function is built
 * under the name xs_ref_kernel (-DFN=xs_ref_kernel) with the build parameters of the
 * reference host (samples/smm/smm_kernel.c:339-347, smm_trans.c).
 */
#include "opencl_host.h"

int xs_ref_group_id, xs_ref_local_id;

#if defined(XS_REF_MULTIPLY)
#  if (1 < BS)
void xs_ref_kernel(double* cdata, const double* adata, const double* bdata, const int* param_stack, int param_format,
  int stack_size, int bs);
#  else
void xs_ref_kernel(double* cdata, const double* adata, const double* bdata, const int* param_stack, int param_format);
#  endif

/* C += A*B over the stack (the reference device layout: B blocks k x n row-major) */
void xs_ref_process(const int* stack, int stack_size, int param_format, const double* a, const double* b, double* c) {
  const int bs = BS, ngroups = (stack_size + bs - 1) / bs;
  for (int g = 0; g < ngroups; ++g) {
    xs_ref_group_id = g;
    for (int i = 0; i < WG; ++i) {
      xs_ref_local_id = i;
#  if (1 < BS)
      xs_ref_kernel(c, a, b, stack, param_format, stack_size, bs);
#  else
      xs_ref_kernel(c, a, b, stack, param_format);
#  endif
    }
  }
}
#endif

#if defined(XS_REF_TRANSPOSE)
#  if (1 < BS)
void xs_ref_kernel(int trs_offset, const int* trs_stack, double* matrix, int stack_size, int bs);
#  else
void xs_ref_kernel(int trs_offset, const int* trs_stack, double* matrix);
#  endif

void xs_ref_transpose(const int* trs_stack, int offset, int stack_size, double* matrix) {
  const int bs = BS, ngroups = (stack_size + bs - 1) / bs;
  for (int g = 0; g < ngroups; ++g) {
    xs_ref_group_id = g;
    xs_ref_local_id = 0; /* WG = 1 */
#  if (1 < BS)
    xs_ref_kernel(offset, trs_stack, matrix, stack_size, bs);
#  else
    xs_ref_kernel(offset, trs_stack, matrix);
#  endif
  }
}
#endif
