/*
 * api_internal.h — host-side objects shared by the C-ABI translation units
 * (mopcuda_api.cu: per-viewport frames; batch_api.cu: batched viewports).
 */
#ifndef MOPCUDA_API_INTERNAL_H
#define MOPCUDA_API_INTERNAL_H

#include "../../include/mop_cuda.h"
#include "mopcuda_internal.cuh"

#include <algorithm>
#include <mutex>
#include <vector>

/* Records the message for mopcuda_last_error() and returns code. */
int mc_fail(int code, const char *fmt, ...);
#define fail mc_fail

#define CU_TRY(expr)                                                                      \
  do {                                                                                    \
    cudaError_t e_ = (expr);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(MOPCUDA_ECUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, \
                  __LINE__);                                                              \
  } while (0)

#define FRAME_TIMEOUT_MS 20000

/* ------------------------------------------------------------------------
 * objects
 * ------------------------------------------------------------------------ */
/* Grow-only device buffer. */
struct DevArena {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap)
      return 0;
    size_t n = bytes + bytes / 2 + 4096;
    release();
    if (cudaMalloc(&p, n) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return fail(MOPCUDA_ENOMEM, "cudaMalloc(%zu) failed", n);
    }
    cap = n;
    return 0;
  }
  void release() {
    if (p)
      cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <class T> T *as() const { return (T *)p; }
};

struct HostArena {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap)
      return 0;
    size_t n = bytes + bytes / 2 + 4096;
    if (p)
      cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    if (cudaMallocHost(&p, n) != cudaSuccess) {
      cudaGetLastError();
      return fail(MOPCUDA_ENOMEM, "cudaMallocHost(%zu) failed", n);
    }
    cap = n;
    return 0;
  }
  void release() {
    if (p)
      cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
  template <class T> T *as() const { return (T *)p; }
};

/* One device allocation shared by several buffers (a scene file's meshes);
 * freed with the last of them. */
struct BufferSlab {
  void *d = nullptr;
  uint32_t refs = 0;
};
/* Drops one reference; frees the allocation with the last (device lock
 * held, nothing in flight reads it). */
static inline void mc_slab_release(BufferSlab *s) {
  if (s && --s->refs == 0) {
    cudaFree(s->d);
    delete s;
  }
}

struct MopCudaBuffer {
  void *d = nullptr;
  void *h = nullptr; /* host shadow for buffer_read (null for buffers made on the device) */
  size_t size = 0;
  BufferSlab *slab = nullptr; /* d lies inside slab->d when set */
};

struct MopCudaTexture {
  int w = 0, h = 0;
  bool hdr = false;
  void *d = nullptr;
  void *hcopy = nullptr;
};

struct MopCudaFramebuffer {
  int w = 0, h = 0;
  int ssaa = 1; /* presentation factor when known (fused SSAA output) */
  DevArena pre, out, depth, ids, presented;
  HostArena h_color, h_depth, h_ids;
  bool host_color = false, host_depth = false, host_ids = false;
  bool presented_valid = false;
  uint64_t frame_serial = 0;
  /* asynchronous presented-colour readback: requested for the pending frame
   * (issued once it completes, inside the next launch when frame_end follows)
   * or in flight on the device's copy stream */
  cudaEvent_t rb_done = nullptr;
  bool rb_requested = false, rb_live = false;
  void *rb_dst = nullptr;
  size_t rb_size = 0;
  int rb_ssaa = 1;
  /* framebuffer_create_from_texture: every completed frame's colour is
   * copied into this texture (device and host copies) */
  MopCudaTexture *target = nullptr;
};

/* A frame's environment background: the environment texture and the ray
 * setup of pass_background_hdri_cpu (viewport.c:2128-2177). */
struct SkyState {
  bool on = false;
  const MopCudaTexture *env = nullptr;
  float fwd[3] = {0, 0, 0}, right[3] = {0, 0, 0}, up[3] = {0, 0, 0};
  float half_w = 0, half_h = 0, rotation = 0, intensity = 1;
};

struct MopCudaDevice {
  int ordinal = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr; /* asynchronous readbacks */
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t pick_ev = nullptr; /* the allocation-free pick's bounded wait */
  cudaEvent_t stage_ev[MOPCUDA_STAGES + 1] = {};
  bool stage_timing = false;
  float stage_ms[MOPCUDA_STAGES] = {};
  std::mutex mu;
  /* the launched frame (kept for a re-run after an overflow) */
  MopCudaFramebuffer *fb = nullptr;
  float clear[4] = {0, 0, 0, 1};
  std::vector<DrawRec> draws;
  std::vector<LightRec> lights;
  uint32_t unsupported_draws = 0;
  uint32_t skipped_draws = 0;
  uint32_t ordered_from = UINT32_MAX; /* first draw of the ordered suffix */
  /* the frame being recorded (frame_begin .. frame_end), while the previous
   * one may still run on the device */
  MopCudaFramebuffer *rec_fb = nullptr;
  float rec_clear[4] = {0, 0, 0, 1};
  std::vector<DrawRec> rec_draws;
  std::vector<LightRec> rec_lights;
  uint32_t rec_unsupported = 0, rec_skipped = 0, rec_ordered_from = UINT32_MAX;
  bool frame_open = false;
  bool pending = false;
  /* the completed frame whose readback frame_end issues inside the next
   * launch, once that launch's upload and kernels up to shading are queued
   * (issued earlier, the image copy delays the next frame's start) */
  MopCudaFramebuffer *rb_defer = nullptr;
  int rb_defer_rc = 0;
  int frame_status = 0;
  /* state */
  float exposure = 1.0f;
  uint32_t post = MOPCUDA_POST_GAMMA | MOPCUDA_POST_FXAA;
  float lut[256];
  float fog[6] = {0, 0, 0, 0, 0, 0}; /* MopFogParams: colour RGBA, near, far */
  SkyState rec_sky, sky; /* background of the frame being recorded / launched */
  /* IBL */
  DevArena irr, pf, brdf;
  int irr_w = 0, irr_h = 0, pf_w = 0, pf_h = 0, pf_levels = 0, brdf_size = 0;
  DevArena env, ibl_tab; /* device precompute: the environment map and host tables */
  HostArena h_ibl;
  int env_w = 0, env_h = 0;
  cudaEvent_t ibl_t0 = nullptr, ibl_t1 = nullptr;
  /* scene-file uploads: page-locked and device staging of a mesh section;
   * per-mesh uploads carve their buffers from load_chunk (the device holds
   * one reference on it while it is the current chunk) */
  HostArena h_load;
  DevArena load_stage;
  BufferSlab *load_chunk = nullptr;
  size_t load_chunk_used = 0;
  float ibl_rot = 0.0f, ibl_int = 1.0f;
  bool ibl_on = false;
  /* frame arenas */
  DevArena d_draws, d_lights, clip, world, normal, color, rrec, srec, clipq,
      large_list, large_items, shade_list, counters, pick_xy, pick_out;
  /* visibility keys: two buffers in turn, a frame's shading pass clearing the
   * one the next frame uses; keys_clean[i] = samples of buffer i known clear */
  DevArena keys[2];
  int keys_cur = 0;
  size_t keys_clean[2] = {0, 0};
  HostArena h_draws, h_lights, h_counters, h_pick;
  DevArena deform_params; /* bone matrices / morph weights of a deform call */
  DevArena hdr, frag_head, frags, touched, olist, olist_items; /* blended suffix */
  DevArena wlist, wlist_items; /* wireframe records of the suffix */
  DevArena oscratch;           /* the fold's sort scratch for long fragment lists */
  uint32_t frag_hint = 0, olist_hint = 0;
  HostArena h_deform;
  /* shadow pass: casters recorded between shadow_begin and shadow_end; the
   * map then stays bound for the device's frames until shadow_clear.  Two
   * maps alternate, so a pass does not wait for the frame in flight, which
   * (or its re-run) reads the other one: fr_sh is the map a launched frame
   * was bound to at its frame_end (-1: none) and fr_sh_size its size. */
  std::vector<ShadowDraw> sh_draws;
  bool sh_open = false, sh_bound = false;
  int sh_rec_size = 0, sh_size = 0, sh_cur = 0;
  int fr_sh = -1, fr_sh_size = 0;
  float sh_rec_vp[16] = {};
  DevArena sh_map[2], sh_d_draws, sh_recs, sh_items, sh_ctr;
  HostArena sh_h_draws;
  cudaEvent_t sh_ev = nullptr; /* after the caster table's upload */
  bool sh_ev_live = false;
  cudaEvent_t sh_t0 = nullptr, sh_t1 = nullptr; /* around the pass's clear and kernels */
  uint32_t vertex_cap = 0, rec_cap = 0, clip_cap = 0, large_cap = 0;
  uint32_t extra_hint = 0, rec_hint = 0, clip_hint = 0, large_hint = 0;
  LaunchCfg cfg = {148, SMALL_MAX_SIDE, SMALL_MAX_AREA, 128, 256, 4, 32, 4};
  uint64_t launches = 0;
  float last_ms = 0.0f;
  uint64_t io_h2d = 0, io_d2h = 0; /* bytes moved by the last frame launch */
};


/* Bounded host waits (20 us polls); every device wait of the library. */
int mc_bounded_sync(MopCudaDevice *d, cudaEvent_t ev, int timeout_ms);
int mc_stream_sync(MopCudaDevice *d, int timeout_ms);
/* Completes a launched frame (re-running it on overflow) before state it
 * reads changes. */
int mc_finish_pending(MopCudaDevice *d);
/* Builds the device record of one draw (and appends its lights). */
int mc_build_draw(const MopCudaDraw *c, const float *model, const float *mvp,
                  std::vector<LightRec> &lights, DrawRec &r, bool &skip);
/* Per-draw IBL constants for prefiltered maps of pf_w x pf_h with `levels`
 * levels and a BRDF LUT of brdf_size (no-op when on is false). */
void mc_ibl_consts(bool on, int pf_w, int pf_h, int levels, int brdf_size, DrawRec *draws,
                   uint32_t n);
/* Post-process arguments for the device's current effects. */
void mc_post_args(const MopCudaDevice *d, PostArgs &p);
/* Post-process arguments for effect bits `fx` with the per-byte values `lut`
 * (build_lut of fx) and fog parameters `fog` (colour RGBA, near, far); the
 * buffer pointers and sizes are left to the caller. */
void mc_post_template(uint32_t fx, const float lut[256], const float fog[6], PostArgs &p);
/* Copies a completed frame's colour into its framebuffer's render target,
 * if it has one (device lock held). */
int mc_target_update(MopCudaDevice *d, MopCudaFramebuffer *fb);
/* mop_mat4_multiply order: running sum from 0.0f, no contraction. */
void mc_mat4_mul(const float *a, const float *b, float *c);

#endif
