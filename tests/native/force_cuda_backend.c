/*
 * force_cuda_backend.c — test-only link-time wrapper that runs the
 * reference's own viewport test programs on the CUDA backend.
 *
 * Linked with -Wl,--wrap=mop_viewport_create, so the test program's calls
 * to mop_viewport_create (reference src/core/viewport.c) arrive here; the
 * viewport is created with backend value 4 — MOP_BACKEND_CUDA of the
 * integration patch, resolved by rhi_swap.c — instead of the backend the
 * test names.  The test source and every core object stay unmodified.
 */
#include <mop/mop.h>

#define MOP_BACKEND_CUDA_VALUE 4

MopViewport *__real_mop_viewport_create(const MopViewportDesc *desc);

MopViewport *__wrap_mop_viewport_create(const MopViewportDesc *desc) {
  if (!desc)
    return __real_mop_viewport_create(desc);
  MopViewportDesc d = *desc;
  d.backend = (MopBackendType)MOP_BACKEND_CUDA_VALUE;
  return __real_mop_viewport_create(&d);
}
