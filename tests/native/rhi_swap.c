/*
 * rhi_swap.c — test-only backend resolution for the drop-in harness.
 *
 * Linked in place of the reference's src/rhi/rhi.c (same three functions,
 * rhi.c:15-72) so that the UNMODIFIED reference viewport core resolves
 * backend value 4 — MOP_BACKEND_CUDA in the integration patch (a new
 * enumerator after MOP_BACKEND_VULKAN, backend.h:24-30) — to
 * mop_rhi_backend_cuda().  Everything else in the core is
 * the reference's own object code.
 */
#include "rhi/rhi.h"

#define MOP_BACKEND_CUDA_VALUE 4

const MopRhiBackend *mop_rhi_backend_cuda(void);

const char *mop_backend_name(MopBackendType type) {
  switch ((int)type) {
  case MOP_BACKEND_AUTO:
    return "auto";
  case MOP_BACKEND_CPU:
    return "cpu";
  case MOP_BACKEND_OPENGL:
    return "opengl";
  case MOP_BACKEND_VULKAN:
    return "vulkan";
  case MOP_BACKEND_CUDA_VALUE:
    return "cuda";
  default:
    return "unknown";
  }
}

MopBackendType mop_backend_default(void) { return MOP_BACKEND_CPU; }

const MopRhiBackend *mop_rhi_get_backend(MopBackendType type) {
  if (type == MOP_BACKEND_AUTO)
    type = mop_backend_default();
  switch ((int)type) {
  case MOP_BACKEND_CPU:
    return mop_rhi_backend_cpu();
  case MOP_BACKEND_CUDA_VALUE:
    return mop_rhi_backend_cuda();
  default:
    return NULL;
  }
}
