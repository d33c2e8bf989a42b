/*
 * mopcuda_api.cu — host side of the C ABI declared in include/mop_cuda.h.
 *
 * Owns device memory (grow-only arenas per device, pinned host mirrors per
 * framebuffer), records draws on the host, and launches the frame as one
 * stream-ordered kernel sequence (kernels.cu).  Every host wait is bounded.
 *
 * Reference correspondence: this file plays the role of the CPU backend's
 * RHI implementation (src/backend/cpu/cpu_backend.c), with the per-draw
 * software rasterisation replaced by a deferred whole-frame device launch.
 */
#include "api_internal.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <mutex>
#include <vector>

/* ------------------------------------------------------------------------
 * errors
 * ------------------------------------------------------------------------ */
static thread_local char g_err[512] = "";

int mc_fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

extern "C" const char *mopcuda_last_error(void) { return g_err; }

extern "C" void *mopcuda_host_alloc(size_t bytes) {
  void *p = nullptr;
  if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) {
    cudaGetLastError();
    fail(MOPCUDA_ENOMEM, "cudaMallocHost(%zu) failed", bytes);
    return nullptr;
  }
  return p;
}

extern "C" void mopcuda_host_free(void *p) {
  if (p)
    cudaFreeHost(p);
}

static int finish_frame(MopCudaDevice *d, int timeout_ms, bool defer_readback = false);
static int issue_readback(MopCudaDevice *d, MopCudaFramebuffer *fb);

/* float x86-compatible evaluation of the post-process byte map
 * (postprocess.c:43-86 for one channel value) */
static void build_lut(float lut[256], uint32_t fx) {
  for (int i = 0; i < 256; i++) {
    volatile float c = (float)i / 255.0f;
    if (fx & MOPCUDA_POST_TONEMAP)
      c = c / (c + 1.0f);
    if (fx & MOPCUDA_POST_GAMMA) {
      float x = c > 0.0f ? c : 0.0f;
      c = x <= 0.0031308f ? x * 12.92f : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
    }
    lut[i] = c;
  }
}

/* ------------------------------------------------------------------------
 * device
 * ------------------------------------------------------------------------ */
extern "C" MopCudaDevice *mopcuda_device_create(int ordinal) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    fail(MOPCUDA_ECUDA, "no CUDA device available");
    return nullptr;
  }
  if (ordinal < 0 || ordinal >= n) {
    fail(MOPCUDA_EINVAL, "CUDA ordinal %d out of range (%d devices)", ordinal, n);
    return nullptr;
  }
  if (cudaSetDevice(ordinal) != cudaSuccess) {
    cudaGetLastError();
    fail(MOPCUDA_ECUDA, "cudaSetDevice(%d) failed", ordinal);
    return nullptr;
  }
  MopCudaDevice *d = new MopCudaDevice();
  d->ordinal = ordinal;
  cudaDeviceGetAttribute(&d->num_sms, cudaDevAttrMultiProcessorCount, ordinal);
  d->cfg.num_sms = d->num_sms;
  if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&d->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&d->ev0) != cudaSuccess || cudaEventCreate(&d->ev1) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->pick_ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    fail(MOPCUDA_ECUDA, "stream/event creation failed");
    delete d;
    return nullptr;
  }
  for (int i = 0; i <= MOPCUDA_STAGES; i++)
    cudaEventCreate(&d->stage_ev[i]);
  build_lut(d->lut, d->post);
  return d;
}

/* Polls the event: back to back for the first 2 ms (a frame usually ends
 * within that, and a sleep would add the scheduler's wake-up latency to
 * every frame), then every 20 us until the timeout. */
int mc_bounded_sync(MopCudaDevice *d, cudaEvent_t ev, int timeout_ms) {
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (;;) {
    cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess)
      return MOPCUDA_OK;
    if (e != cudaErrorNotReady)
      return fail(MOPCUDA_ECUDA, "device error: %s", cudaGetErrorString(e));
    clock_gettime(CLOCK_MONOTONIC, &t1);
    double ms = (t1.tv_sec - t0.tv_sec) * 1e3 + (t1.tv_nsec - t0.tv_nsec) * 1e-6;
    if (timeout_ms >= 0 && ms > (double)timeout_ms)
      return fail(MOPCUDA_ETIMEOUT, "frame did not complete within %d ms", timeout_ms);
    if (ms > 2.0) {
      struct timespec nap = {0, 20000};
      nanosleep(&nap, nullptr);
    }
  }
}

int mc_stream_sync(MopCudaDevice *d, int timeout_ms) {
  cudaEvent_t e;
  CU_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEventRecord(e, d->stream);
  int rc = mc_bounded_sync(d, e, timeout_ms);
  cudaEventDestroy(e);
  return rc;
}

int mc_finish_pending(MopCudaDevice *d) {
  return d->pending ? finish_frame(d, FRAME_TIMEOUT_MS) : MOPCUDA_OK;
}

extern "C" void mopcuda_device_destroy(MopCudaDevice *d) {
  if (!d)
    return;
  cudaSetDevice(d->ordinal);
  mc_stream_sync(d, 10000);
  DevArena *arenas[] = {&d->irr,      &d->pf,         &d->brdf,        &d->d_draws,
                        &d->d_lights, &d->clip,       &d->world,       &d->normal,
                        &d->color,    &d->rrec,       &d->srec,
                        &d->clipq,    &d->keys[0],    &d->keys[1],     &d->large_list,
                        &d->large_items,
                        &d->shade_list, &d->counters, &d->pick_xy,     &d->pick_out,
                        &d->deform_params, &d->hdr, &d->frag_head, &d->frags, &d->touched,
                        &d->olist, &d->olist_items, &d->wlist, &d->wlist_items, &d->oscratch, &d->sh_map[0], &d->sh_map[1], &d->sh_d_draws,
                        &d->sh_recs, &d->sh_items, &d->sh_ctr, &d->env, &d->ibl_tab};
  for (DevArena *a : arenas)
    a->release();
  d->h_ibl.release();
  d->h_load.release();
  d->load_stage.release();
  mc_slab_release(d->load_chunk); /* buffers still carved from it keep it */
  d->load_chunk = nullptr;
  if (d->ibl_t0) {
    cudaEventDestroy(d->ibl_t0);
    cudaEventDestroy(d->ibl_t1);
  }
  d->sh_h_draws.release();
  if (d->sh_ev) {
    cudaEventDestroy(d->sh_ev);
    cudaEventDestroy(d->sh_t0);
    cudaEventDestroy(d->sh_t1);
  }
  d->h_draws.release();
  d->h_lights.release();
  d->h_counters.release();
  d->h_pick.release();
  d->h_deform.release();
  cudaEventDestroy(d->ev0);
  cudaEventDestroy(d->ev1);
  if (d->pick_ev)
    cudaEventDestroy(d->pick_ev);
  for (int i = 0; i <= MOPCUDA_STAGES; i++)
    if (d->stage_ev[i])
      cudaEventDestroy(d->stage_ev[i]);
  cudaStreamSynchronize(d->copy_stream);
  cudaStreamDestroy(d->copy_stream);
  cudaStreamDestroy(d->stream);
  delete d;
}

extern "C" uint64_t mopcuda_launch_count(const MopCudaDevice *d) { return d ? d->launches : 0; }

/* ------------------------------------------------------------------------
 * buffers
 * ------------------------------------------------------------------------ */
extern "C" MopCudaBuffer *mopcuda_buffer_create(MopCudaDevice *d, const void *data, size_t size) {
  if (!d || (!data && size)) {
    fail(MOPCUDA_EINVAL, "buffer_create: bad arguments");
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  MopCudaBuffer *b = new MopCudaBuffer();
  b->size = size;
  size_t alloc = size ? size : 16;
  b->h = malloc(alloc);
  if (!b->h || cudaMalloc(&b->d, alloc) != cudaSuccess) {
    cudaGetLastError();
    free(b->h);
    delete b;
    fail(MOPCUDA_ENOMEM, "buffer_create(%zu) failed", size);
    return nullptr;
  }
  if (size) {
    memcpy(b->h, data, size);
    if (cudaMemcpy(b->d, data, size, cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(b->d);
      free(b->h);
      delete b;
      fail(MOPCUDA_ECUDA, "buffer_create: upload failed");
      return nullptr;
    }
  }
  return b;
}

extern "C" void mopcuda_buffer_destroy(MopCudaDevice *d, MopCudaBuffer *b) {
  if (!d || !b)
    return;
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  mc_finish_pending(d);     /* a launched frame may still read it, or re-run */
  mc_stream_sync(d, 10000);
  if (b->slab)
    mc_slab_release(b->slab);
  else
    cudaFree(b->d);
  free(b->h);
  delete b;
}

extern "C" int mopcuda_buffer_update(MopCudaDevice *d, MopCudaBuffer *b, const void *data,
                                     size_t offset, size_t size) {
  if (!d || !b || (!data && size) || offset > b->size || size > b->size - offset)
    return fail(MOPCUDA_EINVAL, "buffer_update: range outside buffer");
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  int rc = mc_finish_pending(d); /* the launched frame reads the old contents */
  if (!rc)
    rc = mc_stream_sync(d, 10000);
  if (rc)
    return rc;
  if (b->h)
    memcpy((uint8_t *)b->h + offset, data, size);
  CU_TRY(cudaMemcpy((uint8_t *)b->d + offset, data, size, cudaMemcpyHostToDevice));
  return MOPCUDA_OK;
}

extern "C" const void *mopcuda_buffer_read(const MopCudaBuffer *b) { return b ? b->h : nullptr; }

extern "C" int mopcuda_buffer_copy_to_host(MopCudaDevice *d, const MopCudaBuffer *b,
                                           size_t offset, void *dst, size_t size) {
  if (!d || !b || (!dst && size) || offset > b->size || size > b->size - offset)
    return fail(MOPCUDA_EINVAL, "buffer_copy_to_host: range outside buffer");
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  int rc = mc_stream_sync(d, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  if (size)
    CU_TRY(cudaMemcpy(dst, (const uint8_t *)b->d + offset, size, cudaMemcpyDeviceToHost));
  return MOPCUDA_OK;
}
extern "C" size_t mopcuda_buffer_size(const MopCudaBuffer *b) { return b ? b->size : 0; }

/* ------------------------------------------------------------------------
 * textures
 * ------------------------------------------------------------------------ */
static MopCudaTexture *tex_create(MopCudaDevice *d, int w, int h, const void *data, size_t bpp,
                                  bool hdr) {
  if (!d || w <= 0 || h <= 0 || !data) {
    fail(MOPCUDA_EINVAL, "texture_create: bad arguments");
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  size_t bytes = (size_t)w * (size_t)h * bpp;
  MopCudaTexture *t = new MopCudaTexture();
  t->w = w;
  t->h = h;
  t->hdr = hdr;
  t->hcopy = malloc(bytes);
  if (!t->hcopy || cudaMalloc(&t->d, bytes) != cudaSuccess) {
    cudaGetLastError();
    free(t->hcopy);
    delete t;
    fail(MOPCUDA_ENOMEM, "texture_create: allocation failed");
    return nullptr;
  }
  memcpy(t->hcopy, data, bytes);
  if (cudaMemcpy(t->d, data, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(t->d);
    free(t->hcopy);
    delete t;
    fail(MOPCUDA_ECUDA, "texture_create: upload failed");
    return nullptr;
  }
  return t;
}

extern "C" MopCudaTexture *mopcuda_texture_create(MopCudaDevice *d, int w, int h,
                                                  const uint8_t *rgba) {
  return tex_create(d, w, h, rgba, 4, false);
}

extern "C" MopCudaTexture *mopcuda_texture_create_hdr(MopCudaDevice *d, int w, int h,
                                                      const float *rgba) {
  return tex_create(d, w, h, rgba, 16, true);
}

extern "C" void mopcuda_texture_destroy(MopCudaDevice *d, MopCudaTexture *t) {
  if (!d || !t)
    return;
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  mc_stream_sync(d, 10000);
  cudaFree(t->d);
  free(t->hcopy);
  delete t;
}

extern "C" int mopcuda_texture_read_rgba8(MopCudaDevice *d, MopCudaTexture *t, uint8_t *out,
                                          size_t out_size) {
  if (!t || t->hdr || !out)
    return fail(MOPCUDA_EINVAL, "texture_read_rgba8: bad arguments");
  size_t need = (size_t)t->w * (size_t)t->h * 4;
  if (out_size < need)
    return fail(MOPCUDA_EINVAL, "texture_read_rgba8: buffer too small");
  memcpy(out, t->hcopy, need);
  return MOPCUDA_OK;
}

/* ------------------------------------------------------------------------
 * framebuffers
 * ------------------------------------------------------------------------ */
static int fb_alloc(MopCudaFramebuffer *fb, int w, int h) {
  size_t s = (size_t)w * (size_t)h;
  int rc = 0;
  rc |= fb->pre.ensure(s * 4);
  rc |= fb->out.ensure(s * 4);
  rc |= fb->depth.ensure(s * 4);
  rc |= fb->ids.ensure(s * 4);
  rc |= fb->presented.ensure(s * 4);
  rc |= fb->h_color.ensure(s * 4);
  rc |= fb->h_depth.ensure(s * 4);
  rc |= fb->h_ids.ensure(s * 4);
  if (rc)
    return MOPCUDA_ENOMEM;
  fb->w = w;
  fb->h = h;
  fb->host_color = fb->host_depth = fb->host_ids = false;
  fb->presented_valid = false;
  return MOPCUDA_OK;
}

extern "C" MopCudaFramebuffer *mopcuda_framebuffer_create(MopCudaDevice *d, int w, int h) {
  /* reference limit: mop_sw_framebuffer_alloc, rasterizer.c:31-35 */
  if (!d || w <= 0 || h <= 0 || w > 16384 || h > 16384) {
    fail(MOPCUDA_EINVAL, "framebuffer dimensions out of range: %dx%d", w, h);
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  MopCudaFramebuffer *fb = new MopCudaFramebuffer();
  if (fb_alloc(fb, w, h)) {
    delete fb;
    return nullptr;
  }
  return fb;
}

static void fb_release(MopCudaFramebuffer *fb) {
  fb->pre.release();
  fb->out.release();
  fb->depth.release();
  fb->ids.release();
  fb->presented.release();
  fb->h_color.release();
  fb->h_depth.release();
  fb->h_ids.release();
}

extern "C" void mopcuda_framebuffer_destroy(MopCudaDevice *d, MopCudaFramebuffer *fb) {
  if (!d || !fb)
    return;
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  mc_stream_sync(d, 10000);
  if (d->fb == fb)
    d->fb = nullptr;
  if (d->rec_fb == fb) {
    d->rec_fb = nullptr;
    d->frame_open = false;
  }
  if (fb->rb_live)
    mc_bounded_sync(d, fb->rb_done, 10000);
  if (fb->rb_done)
    cudaEventDestroy(fb->rb_done);
  fb_release(fb);
  delete fb;
}

extern "C" int mopcuda_framebuffer_resize(MopCudaDevice *d, MopCudaFramebuffer *fb, int w, int h) {
  if (!d || !fb || w <= 0 || h <= 0 || w > 16384 || h > 16384)
    return fail(MOPCUDA_EINVAL, "framebuffer_resize: %dx%d out of range", w, h);
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  int rc = mc_stream_sync(d, 10000);
  if (rc)
    return rc;
  fb_release(fb);
  return fb_alloc(fb, w, h);
}

/* ------------------------------------------------------------------------
 * frame state
 * ------------------------------------------------------------------------ */
extern "C" void mopcuda_set_exposure(MopCudaDevice *d, float e) {
  if (d)
    d->exposure = e;
}

extern "C" void mopcuda_set_post_effects(MopCudaDevice *d, uint32_t fx) {
  if (!d)
    return;
  d->post = fx;
  build_lut(d->lut, fx);
}

extern "C" int mopcuda_set_fog(MopCudaDevice *d, const float color[4], float near_dist,
                               float far_dist) {
  if (!d || !color)
    return fail(MOPCUDA_EINVAL, "set_fog: %s", !d ? "no device" : "no colour");
  memcpy(d->fog, color, 4 * sizeof(float));
  d->fog[4] = near_dist;
  d->fog[5] = far_dist;
  return MOPCUDA_OK;
}

extern "C" int mopcuda_set_ibl(MopCudaDevice *d, const float *irr, int iw, int ih, const float *pf,
                               int pw, int ph, int levels, const float *brdf, int bs, float rot,
                               float intensity) {
  if (!d)
    return fail(MOPCUDA_EINVAL, "set_ibl: no device");
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  int rc = mc_finish_pending(d);
  if (!rc)
    rc = mc_stream_sync(d, 10000);
  if (rc)
    return rc;
  if (!irr) {
    d->ibl_on = false;
    return MOPCUDA_OK;
  }
  if (iw <= 0 || ih <= 0 || !pf || pw <= 0 || ph <= 0 || levels <= 0 || !brdf || bs <= 0)
    return fail(MOPCUDA_EINVAL, "set_ibl: bad map dimensions");
  size_t pf_px = 0;
  for (int l = 0; l < levels; l++) {
    int lw = pw >> l, lh = ph >> l;
    pf_px += (size_t)(lw < 1 ? 1 : lw) * (size_t)(lh < 1 ? 1 : lh);
  }
  size_t ib = (size_t)iw * ih * 16, pb = pf_px * 16, bb = (size_t)bs * bs * 16;
  if (d->irr.ensure(ib) || d->pf.ensure(pb) || d->brdf.ensure(bb))
    return MOPCUDA_ENOMEM;
  CU_TRY(cudaMemcpy(d->irr.p, irr, ib, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(d->pf.p, pf, pb, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(d->brdf.p, brdf, bb, cudaMemcpyHostToDevice));
  d->irr_w = iw;
  d->irr_h = ih;
  d->pf_w = pw;
  d->pf_h = ph;
  d->pf_levels = levels;
  d->brdf_size = bs;
  d->ibl_rot = rot;
  d->ibl_int = intensity;
  d->ibl_on = true;
  return MOPCUDA_OK;
}

/* ------------------------------------------------------------------------
 * frame commands
 * ------------------------------------------------------------------------ */
/* ------------------------------------------------------------------------
 * vertex deformation (mop_skin_apply / mop_morph_apply on the device)
 * ------------------------------------------------------------------------ */
static int deform_check(const MopCudaBuffer *dst, const MopCudaBuffer *bind, uint32_t vc,
                        const MopCudaDeformLayout *l, bool skin) {
  if (!dst || !bind || !l || l->stride == 0 || l->stride % 4 || l->position_offset < 0 ||
      l->position_offset % 4 || (uint32_t)l->position_offset + 12u > l->stride)
    return fail(MOPCUDA_EINVAL, "deform: bad layout");
  if (l->normal_offset >= 0 && (l->normal_offset % 4 || (uint32_t)l->normal_offset + 12u > l->stride))
    return fail(MOPCUDA_EINVAL, "deform: bad normal offset");
  if (skin && (l->joints_offset < 0 || (uint32_t)l->joints_offset + 4u > l->stride ||
               l->weights_offset < 0 || l->weights_offset % 4 ||
               (uint32_t)l->weights_offset + 16u > l->stride))
    return fail(MOPCUDA_EINVAL, "deform: skinning needs joints (ubyte4) and weights (float4)");
  const size_t need = (size_t)vc * l->stride;
  if (need > bind->size || need > dst->size)
    return fail(MOPCUDA_EINVAL, "deform: %u vertices exceed a buffer", vc);
  return MOPCUDA_OK;
}

/* Runs the launch on the device stream, then refreshes dst's host shadow (the
 * core reads deformed vertices back for bounds). */
static int deform_finish(MopCudaDevice *d, MopCudaBuffer *dst, size_t bytes) {
  CU_TRY(cudaGetLastError());
  if (dst->h)
    CU_TRY(cudaMemcpyAsync(dst->h, dst->d, bytes, cudaMemcpyDeviceToHost, d->stream));
  return mc_stream_sync(d, FRAME_TIMEOUT_MS);
}

extern "C" int mopcuda_skin_apply(MopCudaDevice *d, MopCudaBuffer *dst, const MopCudaBuffer *bind,
                                  uint32_t vc, const MopCudaDeformLayout *l, const float *bones,
                                  uint32_t bone_count) {
  if (!d || (bone_count && !bones))
    return fail(MOPCUDA_EINVAL, "skin_apply: bad arguments");
  int rc = deform_check(dst, bind, vc, l, true);
  if (rc)
    return rc;
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  if (d->pending && (rc = finish_frame(d, FRAME_TIMEOUT_MS)))
    return rc; /* the last frame may still read dst */
  const size_t bb = 64ull * bone_count;
  if (d->deform_params.ensure(bb + 16) || d->h_deform.ensure(bb + 16))
    return MOPCUDA_ENOMEM;
  if (bb) {
    memcpy(d->h_deform.p, bones, bb);
    CU_TRY(cudaMemcpyAsync(d->deform_params.p, d->h_deform.p, bb, cudaMemcpyHostToDevice,
                           d->stream));
  }
  DeformLayout dl = {l->stride, l->position_offset, l->normal_offset, l->joints_offset,
                     l->weights_offset};
  d->launches += (uint64_t)mopcuda_launch_skin((const uint8_t *)bind->d, (uint8_t *)dst->d, vc,
                                               dl, d->deform_params.as<float>(), bone_count,
                                               d->num_sms, d->stream);
  return deform_finish(d, dst, (size_t)vc * l->stride);
}

extern "C" int mopcuda_morph_apply(MopCudaDevice *d, MopCudaBuffer *dst,
                                   const MopCudaBuffer *bind, uint32_t vc,
                                   const MopCudaDeformLayout *l, const MopCudaBuffer *targets,
                                   const float *weights, uint32_t target_count) {
  if (!d || (target_count && (!weights || !targets)))
    return fail(MOPCUDA_EINVAL, "morph_apply: bad arguments");
  int rc = deform_check(dst, bind, vc, l, false);
  if (rc)
    return rc;
  if (target_count && (size_t)target_count * vc * 12u > targets->size)
    return fail(MOPCUDA_EINVAL, "morph_apply: targets buffer holds fewer than %u targets",
                target_count);
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  if (d->pending && (rc = finish_frame(d, FRAME_TIMEOUT_MS)))
    return rc;
  const size_t wb = 4ull * target_count;
  if (d->deform_params.ensure(wb + 16) || d->h_deform.ensure(wb + 16))
    return MOPCUDA_ENOMEM;
  if (wb) {
    memcpy(d->h_deform.p, weights, wb);
    CU_TRY(cudaMemcpyAsync(d->deform_params.p, d->h_deform.p, wb, cudaMemcpyHostToDevice,
                           d->stream));
  }
  DeformLayout dl = {l->stride, l->position_offset, l->normal_offset, -1, -1};
  d->launches += (uint64_t)mopcuda_launch_morph(
      (const uint8_t *)bind->d, (uint8_t *)dst->d, vc, dl,
      target_count ? (const float *)targets->d : nullptr, d->deform_params.as<float>(),
      target_count, d->num_sms, d->stream);
  return deform_finish(d, dst, (size_t)vc * l->stride);
}

extern "C" int mopcuda_frame_begin(MopCudaDevice *d, MopCudaFramebuffer *fb, const float clear[4]) {
  if (!d || !fb)
    return fail(MOPCUDA_EINVAL, "frame_begin: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  /* Recording goes to its own lists: the previous frame may still run (its
   * lists stay for a re-run after an overflow) and is completed at
   * frame_end, so the host records while the device renders. */
  d->rec_fb = fb;
  for (int k = 0; k < 4; k++)
    d->rec_clear[k] = clear ? clear[k] : 0.0f;
  d->rec_draws.clear();
  d->rec_lights.clear();
  d->rec_unsupported = 0;
  d->rec_skipped = 0;
  d->rec_ordered_from = UINT32_MAX;
  d->rec_sky = SkyState();
  d->frame_open = true;
  return MOPCUDA_OK;
}

/* Host float helpers for the background's ray setup: the reference's
 * mop_vec3_* operations (math.c:17-50), without contraction. */
static void h_norm3(const float a[3], float o[3]) {
  volatile float l = sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  if (l < 1e-8f) {
    o[0] = o[1] = o[2] = 0.0f;
    return;
  }
  volatile float inv = 1.0f / l;
  o[0] = a[0] * inv;
  o[1] = a[1] * inv;
  o[2] = a[2] * inv;
}
static void h_cross3(const float a[3], const float b[3], float o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

static int record_sky(MopCudaDevice *d, MopCudaFramebuffer *fb, const MopCudaTexture *env,
                      const SkyState &s) {
  if (!env || !env->hdr || !env->d)
    return fail(MOPCUDA_EINVAL, "background: the environment must be an HDR (RGBA32F) texture");
  if (!d->frame_open || d->rec_fb != fb)
    return fail(MOPCUDA_EINVAL, "background outside frame_begin/frame_end");
  d->rec_sky = s;
  d->rec_sky.env = env;
  d->rec_sky.on = true;
  return MOPCUDA_OK;
}

extern "C" int mopcuda_draw_background(MopCudaDevice *d, MopCudaFramebuffer *fb,
                                       const MopCudaTexture *env, const float eye[3],
                                       const float target[3], const float up[3], float fov_deg,
                                       float rotation, float intensity) {
  if (!d || !fb || !eye || !target || !up)
    return fail(MOPCUDA_EINVAL, "draw_background: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  /* pass_background_hdri_cpu's camera basis (viewport.c:2133-2143), the
   * same float operations in the same order */
  SkyState s;
  volatile float fov = fov_deg * (3.14159265358979323846f / 180.0f);
  volatile float aspect = (float)fb->w / (float)fb->h;
  volatile float half_h = tanf(fov * 0.5f);
  s.half_h = half_h;
  s.half_w = half_h * aspect;
  const float f_raw[3] = {target[0] - eye[0], target[1] - eye[1], target[2] - eye[2]};
  h_norm3(f_raw, s.fwd);
  float r_raw[3];
  h_cross3(s.fwd, up, r_raw);
  h_norm3(r_raw, s.right);
  h_cross3(s.right, s.fwd, s.up);
  s.rotation = rotation;
  s.intensity = intensity;
  return record_sky(d, fb, env, s);
}

extern "C" int mopcuda_draw_skybox(MopCudaDevice *d, MopCudaFramebuffer *fb,
                                   const MopCudaTexture *env, const float inv_vp[16],
                                   const float cam_pos[3], float rotation, float intensity) {
  if (!d || !fb || !inv_vp || !cam_pos)
    return fail(MOPCUDA_EINVAL, "draw_skybox: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  /* points of the far plane at ndc (0,0), (1,0), (0,1) through the inverse
   * view-projection give the ray setup: the centre ray D * fwd, and
   * D * right * half_w, D * up * half_h for the unit steps in ndc */
  double p[3][3];
  const double ndc[3][2] = {{0, 0}, {1, 0}, {0, 1}};
  for (int k = 0; k < 3; k++) {
    double v[4];
    for (int r = 0; r < 4; r++)
      v[r] = (double)inv_vp[r] * ndc[k][0] + (double)inv_vp[4 + r] * ndc[k][1] +
             (double)inv_vp[8 + r] + (double)inv_vp[12 + r];
    if (v[3] == 0.0)
      return fail(MOPCUDA_EINVAL, "draw_skybox: inverse view-projection maps ndc to infinity");
    for (int c = 0; c < 3; c++)
      p[k][c] = v[c] / v[3];
  }
  double c0[3], dr[3], du[3];
  for (int c = 0; c < 3; c++) {
    c0[c] = p[0][c] - cam_pos[c];
    dr[c] = p[1][c] - p[0][c];
    du[c] = p[2][c] - p[0][c];
  }
  const double dist = sqrt(c0[0] * c0[0] + c0[1] * c0[1] + c0[2] * c0[2]);
  const double lr = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
  const double lu = sqrt(du[0] * du[0] + du[1] * du[1] + du[2] * du[2]);
  if (!(dist > 0.0) || !(lr > 0.0) || !(lu > 0.0))
    return fail(MOPCUDA_EINVAL, "draw_skybox: degenerate inverse view-projection");
  SkyState s;
  for (int c = 0; c < 3; c++) {
    s.fwd[c] = (float)(c0[c] / dist);
    s.right[c] = (float)(dr[c] / lr);
    s.up[c] = (float)(du[c] / lu);
  }
  s.half_w = (float)(lr / dist);
  s.half_h = (float)(lu / dist);
  s.rotation = rotation;
  s.intensity = intensity;
  return record_sky(d, fb, env, s);
}

static float clamp01f(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }

/* Records one draw.  Opaque lit and opaque flat draws are order-independent;
 * blended draws (smooth or flat), unlit smooth draws (the legacy path with
 * silhouette edge AA), wireframe draws (anti-aliased lines blended over what
 * is there) and draws with the depth test or the depth write off (the core's
 * instanced pass and editor chrome) depend on submission order and start the
 * frame's ordered suffix; zero-opacity filled draws are colour no-ops in the
 * reference and are dropped (lines ignore the opacity). */
int mc_build_draw(const MopCudaDraw *c, const float *model, const float *mvp,
                  std::vector<LightRec> &lights, DrawRec &r, bool &skip) {
  skip = false;
  if (!c->vertex_buffer || !c->index_buffer)
    return fail(MOPCUDA_EINVAL, "draw: missing buffers");
  float op = clamp01f(c->opacity);
  if (op == 0.0f && c->blend_mode != 3 && !c->wireframe) {
    skip = true;
    return MOPCUDA_OK;
  }
  bool lit = c->lights && c->light_count > 0;
  uint32_t stride = 48;
  memset(&r, 0, sizeof r);
  if (c->wireframe)
    r.flags |= DF_WIRE;
  if (c->layout) {
    const MopCudaVertexLayout *L = c->layout;
    stride = L->stride;
    if (stride == 0 || stride % 4 || L->position_offset < 0 || (L->position_offset % 4) ||
        (L->normal_offset >= 0 && L->normal_offset % 4) ||
        (L->color_offset >= 0 && L->color_offset % 4) || (L->uv_offset >= 0 && L->uv_offset % 4))
      return fail(MOPCUDA_EINVAL, "draw: vertex layout must be 4-byte aligned with a position");
    auto fits = [&](int off, int n) { return off < 0 || (uint32_t)off + 4u * (uint32_t)n <= stride; };
    if (!fits(L->position_offset, L->position_components) ||
        !fits(L->normal_offset, L->normal_components) || !fits(L->color_offset, L->color_components) ||
        !fits(L->uv_offset, L->uv_components))
      return fail(MOPCUDA_EINVAL, "draw: attribute outside the vertex stride");
    r.flags |= DF_FLEX;
    r.stride = stride;
    r.off_pos = (int16_t)L->position_offset;
    r.off_nrm = (int16_t)L->normal_offset;
    r.off_col = (int16_t)L->color_offset;
    r.off_uv = (int16_t)L->uv_offset;
    r.n_pos = (int8_t)L->position_components;
    r.n_nrm = (int8_t)L->normal_components;
    r.n_col = (int8_t)L->color_components;
    r.n_uv = (int8_t)L->uv_components;
  }
  if ((size_t)c->vertex_count * stride > c->vertex_buffer->size)
    return fail(MOPCUDA_EINVAL, "draw: vertex_count exceeds the vertex buffer");
  uint32_t tris = c->index_count / 3u;
  if ((size_t)tris * 12u > c->index_buffer->size)
    return fail(MOPCUDA_EINVAL, "draw: index_count exceeds the index buffer");
  memcpy(r.mvp, mvp, sizeof r.mvp);
  memcpy(r.model, model, sizeof r.model);
  r.blend_mode = c->blend_mode;
  memcpy(r.light_dir, c->light_dir, sizeof r.light_dir);
  r.ambient = c->ambient;
  r.opacity = c->opacity;
  r.metallic = c->metallic;
  r.roughness = c->roughness;
  r.depth_bias = c->depth_bias;
  {
    /* per-draw constants the reference recomputes per pixel
     * (rasterizer.c:1712-1727, 2000, 2030-2032), same operations */
    float alpha = r.roughness * r.roughness;
    float alpha2 = alpha * alpha;
    if (alpha2 < 1e-7f)
      alpha2 = 1e-7f;
    r.alpha2 = alpha2;
    r.smith_k = alpha * 0.5f;
    r.one_minus_k = 1.0f - r.smith_k;
    r.f0_dielectric = 0.04f * (1.0f - r.metallic);
    r.diffuse_scale = 1.0f - r.metallic;
  }
  memcpy(r.cam_eye, c->cam_eye, sizeof r.cam_eye);
  r.object_id = c->object_id;
  r.vbuf = (const uint8_t *)c->vertex_buffer->d;
  r.ibuf = (const uint32_t *)c->index_buffer->d;
  if (c->texture && !c->texture->hdr && c->texture->w >= 1 && c->texture->h >= 1) {
    r.tex = (const uint8_t *)c->texture->d;
    r.tex_w = c->texture->w;
    r.tex_h = c->texture->h;
    r.flags |= DF_TEXTURED;
  }
  r.vertex_count = c->vertex_count;
  r.index_count = tris * 3u;
  if (c->smooth)
    r.flags |= DF_SMOOTH;
  if (c->backface_cull)
    r.flags |= DF_CULL;
  if (!c->depth_test)
    r.flags |= DF_NO_DEPTH_TEST;
  else if (!c->depth_write)
    r.flags |= DF_NO_DEPTH_WRITE;
  if (lit) {
    r.flags |= DF_LIT;
    /* the draw's active lights (inactive ones contribute nothing: the
     * reference skips them, rasterizer.c:1504, 1605, 1729); a block equal to the
     * previous draw's is shared, so a frame's draws usually share one list */
    LightRec blk[64];
    std::vector<LightRec> big;
    LightRec *b = c->light_count <= 64 ? blk : (big.resize(c->light_count), big.data());
    uint32_t n = 0;
    for (uint32_t i = 0; i < c->light_count; i++) {
      const MopCudaLight &s = c->lights[i];
      if (!s.active)
        continue;
      LightRec L;
      memset(&L, 0, sizeof L);
      L.type = s.type;
      memcpy(L.position, s.position, sizeof L.position);
      memcpy(L.direction, s.direction, sizeof L.direction);
      memcpy(L.color, s.color, sizeof L.color);
      L.intensity = s.intensity;
      L.range = s.range;
      L.spot_inner_cos = s.spot_inner_cos;
      L.spot_outer_cos = s.spot_outer_cos;
      L.active = s.active;
      /* mop_vec3_normalize(direction) (math.c:43-50), once per frame */
      float dl = sqrtf(L.direction[0] * L.direction[0] + L.direction[1] * L.direction[1] +
                       L.direction[2] * L.direction[2]);
      if (dl < 1e-8f) {
        L.ndir[0] = L.ndir[1] = L.ndir[2] = 0.0f;
      } else {
        float inv = 1.0f / dl;
        for (int k = 0; k < 3; k++)
          L.ndir[k] = L.direction[k] * inv;
      }
      b[n++] = L;
    }
    r.light_count = n;
    if (n && lights.size() >= n &&
        memcmp(lights.data() + (lights.size() - n), b, sizeof(LightRec) * n) == 0) {
      r.light_off = (uint32_t)(lights.size() - n);
    } else {
      r.light_off = (uint32_t)lights.size();
      lights.insert(lights.end(), b, b + n);
    }
  }
  return MOPCUDA_OK;
}

static int record_draw(MopCudaDevice *d, const MopCudaDraw *c, const float *model,
                       const float *mvp) {
  DrawRec r;
  bool skip = false;
  int rc = mc_build_draw(c, model, mvp, d->rec_lights, r, skip);
  if (rc == MOPCUDA_EUNSUPPORTED)
    d->rec_unsupported++;
  if (rc)
    return rc;
  if (skip) {
    d->rec_skipped++;
    return MOPCUDA_OK;
  }
  /* the first blended, unlit smooth, depth-write-off or depth-test-off draw
   * starts the ordered suffix */
  const bool legacy = (r.flags & DF_SMOOTH) && !(r.flags & DF_LIT);
  if ((r.blend_mode != 0 || clamp01f(r.opacity) < 1.0f || legacy ||
       (r.flags & (DF_NO_DEPTH_WRITE | DF_NO_DEPTH_TEST | DF_WIRE))) &&
      d->rec_ordered_from == UINT32_MAX)
    d->rec_ordered_from = (uint32_t)d->rec_draws.size();
  d->rec_draws.push_back(r);
  return MOPCUDA_OK;
}

extern "C" int mopcuda_draw(MopCudaDevice *d, MopCudaFramebuffer *fb, const MopCudaDraw *c) {
  if (!d || !fb || !c)
    return fail(MOPCUDA_EINVAL, "draw: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  if (!d->frame_open || d->rec_fb != fb)
    return fail(MOPCUDA_EINVAL, "draw outside frame_begin/frame_end");
  return record_draw(d, c, c->model, c->mvp);
}

extern "C" int mopcuda_draw_list(MopCudaDevice *d, MopCudaFramebuffer *fb, const MopCudaDraw *c,
                                 uint32_t n) {
  if (!d || !fb || (n && !c))
    return fail(MOPCUDA_EINVAL, "draw_list: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  if (!d->frame_open || d->rec_fb != fb)
    return fail(MOPCUDA_EINVAL, "draw outside frame_begin/frame_end");
  for (uint32_t i = 0; i < n; i++) {
    int rc = record_draw(d, c + i, c[i].model, c[i].mvp);
    if (rc)
      return rc;
  }
  return MOPCUDA_OK;
}

/* mop_mat4_multiply order (math.c:182-194): running sum from 0.0f. */
void mc_mat4_mul(const float *a, const float *b, float *c) {
  float r[16];
  for (int col = 0; col < 4; col++)
    for (int row = 0; row < 4; row++) {
      volatile float s = 0.0f;
      for (int k = 0; k < 4; k++) {
        volatile float p = a[k * 4 + row] * b[col * 4 + k];
        s = s + p;
      }
      r[col * 4 + row] = s;
    }
  memcpy(c, r, sizeof r);
}

extern "C" int mopcuda_draw_instanced(MopCudaDevice *d, MopCudaFramebuffer *fb,
                                      const MopCudaDraw *c, const float *view, const float *proj,
                                      const float *inst, uint32_t n) {
  if (!d || !fb || !c || !view || !proj || (!inst && n))
    return fail(MOPCUDA_EINVAL, "draw_instanced: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  if (!d->frame_open || d->rec_fb != fb)
    return fail(MOPCUDA_EINVAL, "draw outside frame_begin/frame_end");
  for (uint32_t i = 0; i < n; i++) {
    float vm[16], mvp[16];
    mc_mat4_mul(view, inst + 16 * (size_t)i, vm);
    mc_mat4_mul(proj, vm, mvp);
    int rc = record_draw(d, c, inst + 16 * (size_t)i, mvp);
    if (rc)
      return rc;
  }
  return MOPCUDA_OK;
}


void mc_ibl_consts(bool on, int pf_w, int pf_h, int pf_levels, int brdf_size, DrawRec *draws,
                   uint32_t nd) {
  if (on) {
    /* per-draw IBL constants (rasterizer.c:243-265, 280-291), x86 float ops */
    for (uint32_t i = 0; i < nd; i++) {
      DrawRec &r = draws[i];
      int level = (int)(r.roughness * (float)(pf_levels - 1));
      if (level >= pf_levels)
        level = pf_levels - 1;
      if (level < 0)
        level = 0; /* roughness < 0: undefined in the reference */
      size_t off = 0;
      for (int l = 0; l < level; l++) {
        int lw = pf_w >> l, lh = pf_h >> l;
        off += (size_t)(lw < 1 ? 1 : lw) * (size_t)(lh < 1 ? 1 : lh);
      }
      r.pf_off = (uint32_t)off;
      r.pf_lw = pf_w >> level < 1 ? 1 : pf_w >> level;
      r.pf_lh = pf_h >> level < 1 ? 1 : pf_h >> level;
      float rough = r.roughness < 0.0f ? 0.0f : (r.roughness > 1.0f ? 1.0f : r.roughness);
      int row = (int)(rough * (float)(brdf_size - 1) + 0.5f);
      r.brdf_row = row >= brdf_size ? brdf_size - 1 : row;
    }
  }
}

/* The byte the reference writes for a channel value t that reaches the
 * gamma step (postprocess.c:73-78, then the clamp and rounding of :99-112),
 * with this process's powf. */
static int gamma_byte(float t) {
  volatile float x = t > 0.0f ? t : 0.0f;
  volatile float c = x <= 0.0031308f ? x * 12.92f : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
  float v = c;
  if (v > 1.0f)
    v = 1.0f;
  if (v < 0.0f)
    v = 0.0f;
  volatile float q = v * 255.0f + 0.5f;
  return (int)q;
}

/* Thresholds of gamma_byte: thr[k] is the smallest positive float whose byte
 * is at least k + 1.  gamma_byte is non-decreasing in t (checked over every
 * positive float up to 2.0 with glibc 2.39's powf: 255 steps, none down; all
 * larger values and +inf give 255, NaN and t <= 0 give 0), so a value's byte
 * is the number of thresholds at or below it, and a search of this table
 * on the device returns powf's byte without evaluating powf there. */
static void build_gamma_thresholds(float thr[255]) {
  for (int k = 1; k <= 255; k++) {
    uint32_t lo = 1u, hi = 0x7f800000u; /* smallest subnormal .. +inf */
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo) / 2u;
      float t;
      memcpy(&t, &mid, 4);
      if (gamma_byte(t) >= k)
        hi = mid;
      else
        lo = mid + 1u;
    }
    memcpy(&thr[k - 1], &lo, 4);
  }
}

static const float *gamma_thresholds() {
  static float thr[255];
  static std::once_flag once;
  std::call_once(once, [] { build_gamma_thresholds(thr); });
  return thr;
}

void mc_post_template(uint32_t fx, const float lut[256], const float fog[6], PostArgs &p) {
  memset(&p, 0, sizeof p);
  p.effects = fx & (MOPCUDA_POST_GAMMA | MOPCUDA_POST_TONEMAP | MOPCUDA_POST_VIGNETTE |
                    MOPCUDA_POST_FOG | MOPCUDA_POST_FXAA);
  memcpy(p.lut, lut, sizeof p.lut);
  for (int i = 0; i < 256; i++) {
    float v = lut[i];
    if (v > 1.0f)
      v = 1.0f;
    if (v < 0.0f)
      v = 0.0f;
    volatile float q = v * 255.0f + 0.5f; /* postprocess.c:110-112 */
    p.lut8[i] = (uint8_t)(int)q;
  }
  if (fx & MOPCUDA_POST_FOG) {
    p.fog_color[0] = fog[0];
    p.fog_color[1] = fog[1];
    p.fog_color[2] = fog[2];
    p.fog_near = fog[4];
    volatile float range = fog[5] - fog[4]; /* postprocess.c:53 */
    p.fog_range = range;
    memcpy(p.gamma_thr, gamma_thresholds(), sizeof p.gamma_thr);
  }
}

void mc_post_args(const MopCudaDevice *d, PostArgs &p) { mc_post_template(d->post, d->lut, d->fog, p); }

/* Runs between a launch's shading and its post pass: issues the previous
 * frame's deferred readback, then names the readback the post pass must wait
 * for (this framebuffer's image may still be on its way to the host). */
static cudaEvent_t frame_pre_post(void *ctx) {
  MopCudaDevice *d = (MopCudaDevice *)ctx;
  if (d->rb_defer) {
    MopCudaFramebuffer *prev = d->rb_defer;
    d->rb_defer = nullptr;
    d->rb_defer_rc = issue_readback(d, prev);
  }
  return d->fb->rb_live ? d->fb->rb_done : nullptr;
}

static int launch_frame(MopCudaDevice *d) {
  MopCudaFramebuffer *fb = d->fb;
  const uint32_t nd = (uint32_t)d->draws.size();
  uint64_t V = 0, T = 0;
  for (uint32_t i = 0; i < nd; i++) {
    d->draws[i].vbase = (uint32_t)V;
    d->draws[i].tbase = (uint32_t)T;
    V += d->draws[i].vertex_count;
    T += d->draws[i].index_count / 3u;
  }
  if (T >= (1ull << (32 - ORDER_FAN_BITS)) || V >= (1ull << 31))
    return fail(MOPCUDA_EINVAL, "frame too large: %llu triangles", (unsigned long long)T);
  const size_t S = (size_t)fb->w * (size_t)fb->h;
  /* capacities: grow from the last frame's observed counts */
  uint32_t extra = (uint32_t)(T / 8 + 1024);
  if (extra < d->extra_hint)
    extra = d->extra_hint;
  uint32_t vcap = (uint32_t)V + extra;
  /* one record slot per triangle, then the clipped triangles' fans */
  uint32_t fan_cap = (uint32_t)(T / 8 + 1024);
  if (fan_cap < d->rec_hint)
    fan_cap = d->rec_hint;
  uint32_t rcap = (uint32_t)T + fan_cap;
  uint32_t ccap = (uint32_t)(T / 8 + 1024);
  if (ccap < d->clip_hint)
    ccap = d->clip_hint;
  uint32_t lcap = (uint32_t)(T / 16 + 1024);
  if (lcap < d->large_hint)
    lcap = d->large_hint;
  int rc = 0;
  rc |= d->d_draws.ensure(sizeof(DrawRec) * (nd ? nd : 1));
  rc |= d->d_lights.ensure(sizeof(LightRec) * (d->lights.size() + 1));
  rc |= d->clip.ensure(16ull * vcap);
  rc |= d->world.ensure(16ull * vcap);
  rc |= d->normal.ensure(16ull * vcap);
  rc |= d->color.ensure(16ull * vcap);
  rc |= d->rrec.ensure(sizeof(RasterRec) * (size_t)rcap);
  rc |= d->srec.ensure(sizeof(ShadeRec) * (size_t)rcap);
  rc |= d->clipq.ensure(4ull * ccap);
  for (int i = 0; i < 2; i++) {
    const void *was = d->keys[i].p;
    rc |= d->keys[i].ensure(8ull * S);
    if (d->keys[i].p != was)
      d->keys_clean[i] = 0;
  }
  rc |= d->large_list.ensure(4ull * lcap);
  rc |= d->large_items.ensure(4ull * lcap);
  rc |= d->shade_list.ensure(4ull * S);
  rc |= d->counters.ensure(sizeof(Counters));
  rc |= d->h_draws.ensure(sizeof(DrawRec) * (nd ? nd : 1));
  rc |= d->h_lights.ensure(sizeof(LightRec) * (d->lights.size() + 1));
  rc |= d->h_counters.ensure(sizeof(Counters));
  /* blended suffix: per-sample composition buffers and fragment lists */
  const bool ordered = d->ordered_from < nd;
  const uint32_t t_split = ordered ? d->draws[d->ordered_from].tbase : (uint32_t)T;
  uint32_t fcap = 0, ocap = 0;
  if (ordered) {
    fcap = (uint32_t)std::min<size_t>(std::max<size_t>(d->frag_hint, S + 65536), 0xfffffff0u);
    ocap = std::max<uint32_t>(d->olist_hint, (uint32_t)(T - t_split) + fan_cap);
    rc |= d->hdr.ensure(16ull * S);
    rc |= d->frag_head.ensure(4ull * S);
    rc |= d->touched.ensure(4ull * S);
    rc |= d->frags.ensure(8ull * fcap);
    rc |= d->olist.ensure(4ull * ocap);
    rc |= d->olist_items.ensure(4ull * ocap);
    rc |= d->oscratch.ensure(16ull * fcap);
    bool wire = false;
    for (uint32_t i = d->ordered_from; i < nd && !wire; i++)
      wire = (d->draws[i].flags & DF_WIRE) != 0;
    if (wire) {
      /* line plots mark fragment payloads with bit 31 (FRAG_WIRE_BIT) */
      if (T >= (1ull << (31 - ORDER_FAN_BITS)))
        return fail(MOPCUDA_EUNSUPPORTED, "frame: wireframe draws in a frame of %llu triangles",
                    (unsigned long long)T);
      rc |= d->wlist.ensure(4ull * ocap);
      rc |= d->wlist_items.ensure(4ull * ocap);
    }
  }
  if (rc)
    return MOPCUDA_ENOMEM;
  d->vertex_cap = vcap;
  d->rec_cap = rcap;
  d->clip_cap = ccap;
  d->large_cap = lcap;
  mc_ibl_consts(d->ibl_on, d->pf_w, d->pf_h, d->pf_levels, d->brdf_size, d->draws.data(), nd);
  if (nd)
    memcpy(d->h_draws.p, d->draws.data(), sizeof(DrawRec) * nd);
  if (!d->lights.empty())
    memcpy(d->h_lights.p, d->lights.data(), sizeof(LightRec) * d->lights.size());

  FrameArgs a;
  memset(&a, 0, sizeof a);
  a.draws = d->d_draws.as<DrawRec>();
  a.draw_count = nd;
  a.lights = d->d_lights.as<LightRec>();
  a.light_total = (uint32_t)d->lights.size();
  a.total_vertices = (uint32_t)V;
  a.total_tris = (uint32_t)T;
  a.clip = d->clip.as<float4>();
  a.world = d->world.as<float4>();
  a.normal = d->normal.as<float4>();
  a.color = d->color.as<float4>();
  a.vertex_cap = vcap;
  a.rrec = d->rrec.as<RasterRec>();
  a.srec = d->srec.as<ShadeRec>();
  a.rec_cap = rcap;
  a.clipq = d->clipq.as<uint32_t>();
  a.clip_cap = ccap;
  a.width = fb->w;
  a.height = fb->h;
  const int kb = d->keys_cur;
  a.keys = d->keys[kb].as<unsigned long long>();
  a.keys_next = d->keys[kb ^ 1].as<unsigned long long>();
  a.large_list = d->large_list.as<uint32_t>();
  a.large_items = d->large_items.as<uint32_t>();
  a.large_cap = lcap;
  a.shade_list = d->shade_list.as<uint32_t>();
  a.ctr = d->counters.as<Counters>();
  memcpy(a.clear, d->clear, sizeof a.clear);
  a.exposure = d->exposure;
  if (d->ibl_on) {
    a.irr = d->irr.as<float>();
    a.irr_w = d->irr_w;
    a.irr_h = d->irr_h;
    a.pf = d->pf.as<float>();
    a.pf_w = d->pf_w;
    a.pf_h = d->pf_h;
    a.pf_levels = d->pf_levels;
    a.brdf = d->brdf.as<float>();
    a.brdf_size = d->brdf_size;
    a.ibl_rotation = d->ibl_rot;
    a.ibl_intensity = d->ibl_int;
  }
  a.pre = fb->pre.as<uchar4>();
  a.depth = fb->depth.as<float>();
  a.ids = fb->ids.as<uint32_t>();
  if (d->sky.on) {
    const SkyState &k = d->sky;
    a.sky = (const float4 *)k.env->d;
    a.sky_w = k.env->w;
    a.sky_h = k.env->h;
    memcpy(a.sky_fwd, k.fwd, sizeof a.sky_fwd);
    memcpy(a.sky_right, k.right, sizeof a.sky_right);
    memcpy(a.sky_up, k.up, sizeof a.sky_up);
    a.sky_half_w = k.half_w;
    a.sky_half_h = k.half_h;
    a.sky_rotation = k.rotation;
    a.sky_intensity = k.intensity;
  }
  a.small_side = d->cfg.small_side;
  a.small_area = d->cfg.small_area;
  if (ordered) {
    a.t_split = t_split;
    a.hdr = d->hdr.as<float4>();
    a.frag_head = d->frag_head.as<uint32_t>();
    a.frags = d->frags.as<uint2>();
    a.frag_cap = fcap;
    a.touched = d->touched.as<uint32_t>();
    a.olist = d->olist.as<uint32_t>();
    a.olist_items = d->olist_items.as<uint32_t>();
    a.olist_cap = ocap;
    a.oscratch = d->oscratch.as<ulonglong2>();
    a.oscratch_count = &d->counters.as<Counters>()->scratch_count;
    a.oscratch_cap = fcap;
    for (uint32_t i = d->ordered_from; i < nd; i++) {
      if (d->draws[i].flags & DF_NO_DEPTH_TEST)
        a.ordered_keep_all = 1;
      if (d->draws[i].flags & DF_WIRE)
        a.wire = 1;
    }
    if (a.wire) {
      a.wlist = d->wlist.as<uint32_t>();
      a.wlist_items = d->wlist_items.as<uint32_t>();
      a.wlist_cap = ocap;
    }
  }

  if (d->fr_sh >= 0) { /* the map bound at this frame's frame_end */
    const DevArena &m = d->sh_map[d->fr_sh];
    a.shadow_keys = m.as<uint32_t>();
    a.shadow_vp = (const float *)(m.as<uint8_t>() + 4 * (size_t)d->fr_sh_size * d->fr_sh_size);
    a.shadow_w = a.shadow_h = d->fr_sh_size;
  }

  PostArgs p;
  mc_post_args(d, p);
  p.pre = fb->pre.as<uchar4>();
  p.out = fb->out.as<uchar4>();
  int sf = fb->ssaa >= 1 && fb->ssaa <= 4 && fb->w % fb->ssaa == 0 && fb->h % fb->ssaa == 0
               ? fb->ssaa
               : 1;
  p.presented = sf > 1 ? fb->presented.as<uchar4>() : nullptr;
  p.depth = fb->depth.as<float>();
  p.width = fb->w;
  p.height = fb->h;
  p.ssaa = sf;

  cudaStream_t s = d->stream;
  CU_TRY(cudaEventRecord(d->ev0, s));
  if (nd)
    CU_TRY(cudaMemcpyAsync(d->d_draws.p, d->h_draws.p, sizeof(DrawRec) * nd,
                           cudaMemcpyHostToDevice, s));
  if (!d->lights.empty())
    CU_TRY(cudaMemcpyAsync(d->d_lights.p, d->h_lights.p, sizeof(LightRec) * d->lights.size(),
                           cudaMemcpyHostToDevice, s));
  CU_TRY(cudaMemsetAsync(d->counters.p, 0, sizeof(Counters), s));
  /* this frame dirties its key buffer and its shading pass clears the other */
  const bool keys_clear = d->keys_clean[kb] >= S;
  d->keys_clean[0] = d->keys_clean[1] = 0;
  if (!keys_clear)
    CU_TRY(cudaMemsetAsync(a.keys, 0xff, 8ull * S, s));
  d->rb_defer_rc = MOPCUDA_OK;
  d->launches += (uint64_t)mopcuda_launch_frame(a, p, d->cfg, s,
                                                d->stage_timing ? d->stage_ev : nullptr,
                                                frame_pre_post, d);
  CU_TRY(cudaGetLastError());
  d->keys_clean[kb ^ 1] = S;
  d->keys_cur = kb ^ 1;
  CU_TRY(cudaMemcpyAsync(d->h_counters.p, d->counters.p, sizeof(Counters), cudaMemcpyDeviceToHost,
                         s));
  CU_TRY(cudaEventRecord(d->ev1, s));
  fb->host_color = fb->host_depth = fb->host_ids = false;
  fb->presented_valid = sf > 1;
  fb->frame_serial++;
  d->pending = true;
  d->io_h2d = sizeof(DrawRec) * (uint64_t)nd + sizeof(LightRec) * (uint64_t)d->lights.size();
  d->io_d2h = sizeof(Counters);
  return d->rb_defer_rc; /* the previous frame's readback, issued by the hook */
}

extern "C" int mopcuda_frame_io_bytes(MopCudaDevice *d, uint64_t *h2d, uint64_t *d2h) {
  if (!d || !h2d || !d2h)
    return fail(MOPCUDA_EINVAL, "frame_io_bytes: bad arguments");
  *h2d = d->io_h2d;
  *d2h = d->io_d2h;
  return MOPCUDA_OK;
}


/* Waits for the launched frame; re-runs it with larger arenas if any
 * capacity overflowed (the counters say by how much). */
static int finish_frame(MopCudaDevice *d, int timeout_ms, bool defer_readback) {
  for (int attempt = 0; d->pending; attempt++) {
    int rc = mc_bounded_sync(d, d->ev1, timeout_ms);
    if (rc) {
      /* a wait that ran out leaves the frame pending (a later wait resumes
       * it); a device error loses it */
      if (rc != MOPCUDA_ETIMEOUT)
        d->pending = false;
      return rc;
    }
    d->pending = false;
    cudaEventElapsedTime(&d->last_ms, d->ev0, d->ev1);
    if (d->stage_timing)
      for (int i = 0; i < MOPCUDA_STAGES; i++)
        cudaEventElapsedTime(&d->stage_ms[i], d->stage_ev[i], d->stage_ev[i + 1]);
    const Counters *c = d->h_counters.as<Counters>();
    if (!c->overflow) {
      if (d->fb && d->fb->target && (rc = mc_target_update(d, d->fb)))
        return rc;
      if (d->fb && d->fb->rb_requested) {
        if (defer_readback) {
          d->rb_defer = d->fb; /* issued inside the caller's next launch */
          return MOPCUDA_OK;
        }
        return issue_readback(d, d->fb);
      }
      break;
    }
    if (c->overflow & 512u)
      return fail(MOPCUDA_EUNSUPPORTED,
                  "frame: the large triangles' raster items exceed 2^32 in one frame");
    if (attempt >= 4)
      return fail(MOPCUDA_ENOMEM, "frame arenas overflowed repeatedly (flags %u)", c->overflow);
    d->rec_hint = c->rec_count + c->rec_count / 4 + 1024;
    d->clip_hint = c->clip_count + c->clip_count / 4 + 1024;
    d->extra_hint = c->extra_vertices + c->extra_vertices / 4 + 1024;
    d->large_hint = c->large_count + c->large_count / 4 + 1024;
    if (c->overflow & 16u)
      d->frag_hint = c->frag_count + c->frag_count / 4 + 65536;
    if (c->overflow & 32u)
      d->olist_hint = c->olist_count + c->olist_count / 4 + 1024;
    if (c->overflow & 128u)
      d->olist_hint = std::max(d->olist_hint, c->wire_count + c->wire_count / 4 + 1024);
    if (c->overflow & 1u)
      d->rec_hint *= 2;
    if (c->overflow & 2u)
      d->extra_hint *= 2;
    if (c->overflow & 4u)
      d->clip_hint *= 2;
    if (c->overflow & 8u)
      d->large_hint *= 2;
    rc = launch_frame(d);
    if (rc)
      return rc;
  }
  return MOPCUDA_OK;
}

extern "C" int mopcuda_frame_end(MopCudaDevice *d, MopCudaFramebuffer *fb) {
  if (!d || !fb)
    return fail(MOPCUDA_EINVAL, "frame_end: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  if (!d->frame_open || d->rec_fb != fb)
    return fail(MOPCUDA_EINVAL, "frame_end without frame_begin");
  d->frame_open = false;
  cudaSetDevice(d->ordinal);
  /* the previous frame completes (or re-runs) with its own lists before its
   * pinned staging is reused */
  int rc;
  if (d->pending && (rc = finish_frame(d, FRAME_TIMEOUT_MS, true)))
    return rc;
  d->fb = d->rec_fb;
  memcpy(d->clear, d->rec_clear, sizeof d->clear);
  d->draws.swap(d->rec_draws);
  d->lights.swap(d->rec_lights);
  d->unsupported_draws = d->rec_unsupported;
  d->skipped_draws = d->rec_skipped;
  d->ordered_from = d->rec_ordered_from;
  d->sky = d->rec_sky;
  d->fr_sh = d->sh_bound ? d->sh_cur : -1;
  d->fr_sh_size = d->sh_size;
  rc = launch_frame(d);
  if (d->rb_defer) { /* the launch stopped before its post pass */
    MopCudaFramebuffer *prev = d->rb_defer;
    d->rb_defer = nullptr;
    int rrc = issue_readback(d, prev);
    if (!rc)
      rc = rrc;
  }
  if (rc)
    return rc;
  if (d->unsupported_draws)
    return fail(MOPCUDA_EUNSUPPORTED, "%u draw(s) outside the order-independent path were skipped",
                d->unsupported_draws);
  return MOPCUDA_OK;
}

extern "C" int mopcuda_frame_wait(MopCudaDevice *d, int timeout_ms) {
  if (!d)
    return fail(MOPCUDA_EINVAL, "frame_wait: no device");
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  return finish_frame(d, timeout_ms);
}

extern "C" float mopcuda_frame_gpu_time_ms(MopCudaDevice *d) { return d ? d->last_ms : 0.0f; }

/* ------------------------------------------------------------------------
 * shadow pass (pass_shadow, viewport.c:2288-2442: casters rasterised into a
 * depth map from the light, then bound for the frame's shading)
 * ------------------------------------------------------------------------ */
extern "C" int mopcuda_shadow_begin(MopCudaDevice *d, int size, const float light_vp[16]) {
  if (!d || !light_vp || size <= 0 || size > 16384)
    return fail(MOPCUDA_EINVAL, "shadow_begin: bad arguments (size %d)", size);
  std::lock_guard<std::mutex> lk(d->mu);
  d->sh_draws.clear();
  d->sh_open = true;
  d->sh_rec_size = size;
  memcpy(d->sh_rec_vp, light_vp, sizeof d->sh_rec_vp);
  return MOPCUDA_OK;
}

/* One caster of the open pass (the device lock held). */
static int add_caster(MopCudaDevice *d, const MopCudaBuffer *vertices, uint32_t vertex_count,
                      uint32_t stride, const MopCudaBuffer *indices, uint32_t index_count,
                      const float model[16]) {
  if (!vertices || !indices)
    return fail(MOPCUDA_EINVAL, "shadow_draw: bad arguments");
  if (stride < 12 || stride % 4 != 0)
    return fail(MOPCUDA_EINVAL, "shadow_draw: stride %u (needs >= 12, a multiple of 4)", stride);
  if ((uint64_t)vertex_count * stride > vertices->size ||
      (uint64_t)index_count * 4u > indices->size)
    return fail(MOPCUDA_EINVAL, "shadow_draw: %u vertices / %u indices exceed the buffers",
                vertex_count, index_count);
  ShadowDraw s;
  s.verts = (const uint8_t *)vertices->d;
  s.idx = (const uint32_t *)indices->d;
  s.vertex_count = vertex_count;
  s.stride = stride;
  s.tri_count = index_count / 3u;
  s.tri_off = 0;
  mc_mat4_mul(d->sh_rec_vp, model, s.mvp); /* mop_mat4_multiply(light_vp, model) */
  if (s.tri_count)
    d->sh_draws.push_back(s);
  return MOPCUDA_OK;
}

extern "C" int mopcuda_shadow_draw(MopCudaDevice *d, const MopCudaBuffer *vertices,
                                   uint32_t vertex_count, uint32_t stride,
                                   const MopCudaBuffer *indices, uint32_t index_count,
                                   const float model[16]) {
  if (!d || !model)
    return fail(MOPCUDA_EINVAL, "shadow_draw: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  if (!d->sh_open)
    return fail(MOPCUDA_EINVAL, "shadow_draw outside shadow_begin/shadow_end");
  return add_caster(d, vertices, vertex_count, stride, indices, index_count, model);
}

extern "C" int mopcuda_shadow_draw_list(MopCudaDevice *d, const MopCudaShadowCaster *c,
                                        uint32_t n) {
  if (!d || (n && !c))
    return fail(MOPCUDA_EINVAL, "shadow_draw_list: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  if (!d->sh_open)
    return fail(MOPCUDA_EINVAL, "shadow_draw outside shadow_begin/shadow_end");
  for (uint32_t i = 0; i < n; i++) {
    int rc = add_caster(d, c[i].vertices, c[i].vertex_count, c[i].stride, c[i].indices,
                        c[i].index_count, c[i].model);
    if (rc)
      return rc;
  }
  return MOPCUDA_OK;
}

extern "C" int mopcuda_shadow_end(MopCudaDevice *d) {
  if (!d)
    return fail(MOPCUDA_EINVAL, "shadow_end: no device");
  std::lock_guard<std::mutex> lk(d->mu);
  if (!d->sh_open)
    return fail(MOPCUDA_EINVAL, "shadow_end without shadow_begin");
  d->sh_open = false;
  cudaSetDevice(d->ordinal);
  int rc;
  /* the pass writes the map the last one did not; only a frame in flight
   * bound to that map (an older pass's) has to complete first */
  const int t = 1 - d->sh_cur;
  if (d->pending && d->fr_sh == t && (rc = finish_frame(d, FRAME_TIMEOUT_MS)))
    return rc;
  if (!d->sh_ev) {
    CU_TRY(cudaEventCreateWithFlags(&d->sh_ev, cudaEventDisableTiming));
    CU_TRY(cudaEventCreate(&d->sh_t0));
    CU_TRY(cudaEventCreate(&d->sh_t1));
  }
  if (d->sh_ev_live && (rc = mc_bounded_sync(d, d->sh_ev, FRAME_TIMEOUT_MS)))
    return rc;
  const uint32_t n = (uint32_t)d->sh_draws.size();
  uint64_t T = 0;
  for (ShadowDraw &s : d->sh_draws) {
    s.tri_off = (uint32_t)T;
    T += s.tri_count;
  }
  if (T >= (1ull << 31))
    return fail(MOPCUDA_EINVAL, "shadow pass too large: %llu triangles", (unsigned long long)T);
  const size_t S = (size_t)d->sh_rec_size;
  rc = 0;
  rc |= d->sh_map[t].ensure(4 * S * S + 64); /* texels, then the light's view-projection */
  rc |= d->sh_d_draws.ensure(sizeof(ShadowDraw) * (n ? n : 1));
  rc |= d->sh_h_draws.ensure(sizeof(ShadowDraw) * n + 64);
  rc |= d->sh_recs.ensure(sizeof(ShadowRec) * (size_t)(T ? T : 1));
  rc |= d->sh_items.ensure(8 * (size_t)(T ? T : 1));
  rc |= d->sh_ctr.ensure(sizeof(ShadowCounters));
  if (rc)
    return MOPCUDA_ENOMEM;
  cudaStream_t st = d->stream;
  /* page-locked staging: the caster table, then the view-projection */
  uint8_t *hp = d->sh_h_draws.as<uint8_t>();
  const size_t db = sizeof(ShadowDraw) * n;
  if (n)
    memcpy(hp, d->sh_draws.data(), db);
  memcpy(hp + db, d->sh_rec_vp, 64);
  if (n)
    CU_TRY(cudaMemcpyAsync(d->sh_d_draws.p, hp, db, cudaMemcpyHostToDevice, st));
  CU_TRY(cudaMemcpyAsync(d->sh_map[t].as<uint8_t>() + 4 * S * S, hp + db, 64,
                         cudaMemcpyHostToDevice, st));
  CU_TRY(cudaEventRecord(d->sh_ev, st));
  d->sh_ev_live = true;
  CU_TRY(cudaEventRecord(d->sh_t0, st));
  /* cleared to 1.0 (viewport.c:2370-2373): the key 0xffffffff */
  CU_TRY(cudaMemsetAsync(d->sh_map[t].p, 0xff, 4 * S * S, st));
  CU_TRY(cudaMemsetAsync(d->sh_ctr.p, 0, sizeof(ShadowCounters), st));
  ShadowArgs a;
  a.draws = d->sh_d_draws.as<ShadowDraw>();
  a.draw_count = n;
  a.tri_total = (uint32_t)T;
  a.map = d->sh_map[t].as<uint32_t>();
  a.size = (int)S;
  a.small_area = SHADOW_SMALL_AREA;
  a.recs = d->sh_recs.as<ShadowRec>();
  a.items = d->sh_items.as<unsigned long long>();
  a.ctr = d->sh_ctr.as<ShadowCounters>();
  a.num_sms = d->num_sms;
  d->launches += (uint64_t)mopcuda_launch_shadow(a, st);
  CU_TRY(cudaGetLastError());
  CU_TRY(cudaEventRecord(d->sh_t1, st));
  d->sh_size = (int)S;
  d->sh_cur = t;
  d->sh_bound = true;
  return MOPCUDA_OK;
}

extern "C" float mopcuda_shadow_gpu_time_ms(MopCudaDevice *d) {
  if (!d || !d->sh_t1)
    return 0.0f;
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  if (mc_bounded_sync(d, d->sh_t1, FRAME_TIMEOUT_MS))
    return 0.0f;
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, d->sh_t0, d->sh_t1);
  return ms;
}

extern "C" int mopcuda_shadow_clear(MopCudaDevice *d) {
  if (!d)
    return fail(MOPCUDA_EINVAL, "shadow_clear: no device");
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  int rc;
  if (d->pending && (rc = finish_frame(d, FRAME_TIMEOUT_MS)))
    return rc;
  d->sh_bound = false;
  d->sh_open = false;
  return MOPCUDA_OK;
}

extern "C" int mopcuda_shadow_read(MopCudaDevice *d, float *out, size_t out_bytes) {
  if (!d || !out)
    return fail(MOPCUDA_EINVAL, "shadow_read: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  if (!d->sh_bound)
    return fail(MOPCUDA_EINVAL, "shadow_read: no shadow map bound");
  const size_t n = (size_t)d->sh_size * (size_t)d->sh_size;
  if (out_bytes < 4 * n)
    return fail(MOPCUDA_EINVAL, "shadow_read: %zu bytes, %zu needed", out_bytes, 4 * n);
  cudaSetDevice(d->ordinal);
  int rc = mc_stream_sync(d, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  CU_TRY(cudaMemcpy(out, d->sh_map[d->sh_cur].p, 4 * n, cudaMemcpyDeviceToHost));
  uint32_t *k = (uint32_t *)out;
  for (size_t i = 0; i < n; i++) { /* keys -> depth values, in place */
    uint32_t b = k[i];
    b = b == 0xffffffffu ? 0x3f800000u : ((b & 0x80000000u) ? (b & 0x7fffffffu) : ~b);
    k[i] = b;
  }
  return MOPCUDA_OK;
}

/* ------------------------------------------------------------------------
 * readbacks
 * ------------------------------------------------------------------------ */
static int ready(MopCudaDevice *d, MopCudaFramebuffer *fb) {
  if (!d || !fb)
    return fail(MOPCUDA_EINVAL, "readback: bad arguments");
  cudaSetDevice(d->ordinal);
  if (d->fb == fb && d->pending)
    return finish_frame(d, FRAME_TIMEOUT_MS);
  return MOPCUDA_OK;
}

static int fetch(MopCudaDevice *d, DevArena &src, HostArena &dst, size_t bytes, bool &valid) {
  if (valid)
    return MOPCUDA_OK;
  CU_TRY(cudaMemcpyAsync(dst.p, src.p, bytes, cudaMemcpyDeviceToHost, d->stream));
  int rc = mc_stream_sync(d, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  valid = true;
  return MOPCUDA_OK;
}

extern "C" const uint8_t *mopcuda_read_color(MopCudaDevice *d, MopCudaFramebuffer *fb, int *w,
                                             int *h) {
  if (!d || !fb)
    return nullptr;
  std::lock_guard<std::mutex> lk(d->mu);
  if (ready(d, fb) || fetch(d, fb->out, fb->h_color, (size_t)fb->w * fb->h * 4, fb->host_color))
    return nullptr;
  if (w)
    *w = fb->w;
  if (h)
    *h = fb->h;
  return fb->h_color.as<uint8_t>();
}

extern "C" const uint32_t *mopcuda_read_object_id(MopCudaDevice *d, MopCudaFramebuffer *fb, int *w,
                                                  int *h) {
  if (!d || !fb)
    return nullptr;
  std::lock_guard<std::mutex> lk(d->mu);
  if (ready(d, fb) || fetch(d, fb->ids, fb->h_ids, (size_t)fb->w * fb->h * 4, fb->host_ids))
    return nullptr;
  if (w)
    *w = fb->w;
  if (h)
    *h = fb->h;
  return fb->h_ids.as<uint32_t>();
}

extern "C" const float *mopcuda_read_depth(MopCudaDevice *d, MopCudaFramebuffer *fb, int *w,
                                           int *h) {
  if (!d || !fb)
    return nullptr;
  std::lock_guard<std::mutex> lk(d->mu);
  if (ready(d, fb) || fetch(d, fb->depth, fb->h_depth, (size_t)fb->w * fb->h * 4, fb->host_depth))
    return nullptr;
  if (w)
    *w = fb->w;
  if (h)
    *h = fb->h;
  return fb->h_depth.as<float>();
}

extern "C" int mopcuda_read_color_resolved(MopCudaDevice *d, MopCudaFramebuffer *fb, int sf,
                                           uint8_t *out, size_t out_size) {
  if (!d || !fb || !out || sf <= 0 || fb->w % sf || fb->h % sf)
    return fail(MOPCUDA_EINVAL, "read_color_resolved: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  int rc = ready(d, fb);
  if (rc)
    return rc;
  size_t need = (size_t)(fb->w / sf) * (size_t)(fb->h / sf) * 4;
  if (out_size < need)
    return fail(MOPCUDA_EINVAL, "read_color_resolved: buffer too small");
  const void *src = fb->out.p;
  if (sf > 1) {
    if (!(fb->presented_valid && fb->ssaa == sf)) {
      d->launches += (uint64_t)mopcuda_launch_box(fb->out.as<uchar4>(), fb->w, fb->h, sf,
                                                  fb->presented.as<uchar4>(), d->stream);
      CU_TRY(cudaGetLastError());
    }
    src = fb->presented.p;
  }
  CU_TRY(cudaMemcpyAsync(out, src, need, cudaMemcpyDeviceToHost, d->stream));
  return mc_stream_sync(d, FRAME_TIMEOUT_MS);
}

/* Asynchronous readback of the presented image (no reference counterpart:
 * the synchronous read is mop_viewport_read_color).  The copy runs on the
 * device's copy stream once the frame has completed; when frame_end launches
 * the next frame, it is queued inside that launch (frame_pre_post), after
 * the frame's upload and kernels up to shading, so it overlaps their work;
 * the next frame's post pass, which overwrites the image, waits for it. */
static int issue_readback(MopCudaDevice *d, MopCudaFramebuffer *fb) {
  fb->rb_requested = false;
  if (!fb->rb_done)
    CU_TRY(cudaEventCreateWithFlags(&fb->rb_done, cudaEventDisableTiming));
  const void *src = fb->rb_ssaa > 1 ? fb->presented.p : fb->out.p;
  CU_TRY(cudaStreamWaitEvent(d->copy_stream, d->ev1, 0));
  CU_TRY(cudaMemcpyAsync(fb->rb_dst, src, fb->rb_size, cudaMemcpyDeviceToHost, d->copy_stream));
  CU_TRY(cudaEventRecord(fb->rb_done, d->copy_stream));
  fb->rb_live = true;
  return MOPCUDA_OK;
}

extern "C" int mopcuda_read_color_resolved_async(MopCudaDevice *d, MopCudaFramebuffer *fb,
                                                 int sf, void *out, size_t out_size) {
  if (!d || !fb || !out || sf <= 0 || fb->w % sf || fb->h % sf)
    return fail(MOPCUDA_EINVAL, "read_color_resolved_async: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  if (sf > 1 && fb->ssaa != sf)
    return fail(MOPCUDA_EINVAL, "read_color_resolved_async: SSAA %d is not the framebuffer's "
                                "presentation factor %d", sf, fb->ssaa);
  const size_t need = (size_t)(fb->w / sf) * (size_t)(fb->h / sf) * 4;
  if (out_size < need)
    return fail(MOPCUDA_EINVAL, "read_color_resolved_async: buffer too small");
  fb->rb_dst = out;
  fb->rb_size = need;
  fb->rb_ssaa = sf;
  fb->rb_requested = true;
  if (d->fb == fb && d->pending)
    return MOPCUDA_OK; /* issued when the frame completes (inside the next launch) */
  return issue_readback(d, fb);
}

extern "C" int mopcuda_readback_wait(MopCudaDevice *d, MopCudaFramebuffer *fb, int timeout_ms) {
  if (!d || !fb)
    return fail(MOPCUDA_EINVAL, "readback_wait: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  int rc;
  if (fb->rb_requested && d->fb == fb && d->pending && (rc = finish_frame(d, timeout_ms)))
    return rc;
  if (!fb->rb_live)
    return MOPCUDA_OK;
  return mc_bounded_sync(d, fb->rb_done, timeout_ms);
}

/* Presentation factor of a framebuffer: lets frame_end fuse the SSAA box
 * into the post pass (the viewport allocates W*ssaa x H*ssaa samples). */
extern "C" int mopcuda_framebuffer_set_ssaa(MopCudaFramebuffer *fb, int sf) {
  if (!fb || sf <= 0)
    return fail(MOPCUDA_EINVAL, "framebuffer_set_ssaa: bad arguments");
  fb->ssaa = sf;
  return MOPCUDA_OK;
}

static int pick_one(MopCudaDevice *d, MopCudaFramebuffer *fb, int x, int y, uint32_t *id,
                    float *dep) {
  *id = 0;
  *dep = 1.0f;
  if (x < 0 || x >= fb->w || y < 0 || y >= fb->h)
    return MOPCUDA_OK;
  int rc = ready(d, fb);
  if (rc)
    return rc;
  size_t i = (size_t)y * (size_t)fb->w + (size_t)x;
  if (fb->host_ids)
    *id = fb->h_ids.as<uint32_t>()[i];
  else
    CU_TRY(cudaMemcpy(id, fb->ids.as<uint32_t>() + i, 4, cudaMemcpyDeviceToHost));
  if (fb->host_depth)
    *dep = fb->h_depth.as<float>()[i];
  else
    CU_TRY(cudaMemcpy(dep, fb->depth.as<float>() + i, 4, cudaMemcpyDeviceToHost));
  return MOPCUDA_OK;
}

extern "C" uint32_t mopcuda_pick_read_id(MopCudaDevice *d, MopCudaFramebuffer *fb, int x, int y) {
  if (!d || !fb)
    return 0;
  std::lock_guard<std::mutex> lk(d->mu);
  uint32_t id;
  float dp;
  return pick_one(d, fb, x, y, &id, &dp) ? 0u : id;
}

extern "C" float mopcuda_pick_read_depth(MopCudaDevice *d, MopCudaFramebuffer *fb, int x, int y) {
  if (!d || !fb)
    return 1.0f;
  std::lock_guard<std::mutex> lk(d->mu);
  uint32_t id;
  float dp;
  return pick_one(d, fb, x, y, &id, &dp) ? 1.0f : dp;
}

extern "C" int mopcuda_pick_batch(MopCudaDevice *d, MopCudaFramebuffer *fb, int sf,
                                  const int32_t *xy, uint32_t n, uint32_t *ids, float *depths,
                                  int32_t *hits) {
  if (!d || !fb || sf <= 0 || (n && (!xy || !ids || !depths || !hits)))
    return fail(MOPCUDA_EINVAL, "pick_batch: bad arguments");
  if (n == 0)
    return MOPCUDA_OK;
  std::lock_guard<std::mutex> lk(d->mu);
  int rc = ready(d, fb);
  if (rc)
    return rc;
  size_t in_b = 8ull * n, out_b = 12ull * n;
  if (d->pick_xy.ensure(in_b) || d->pick_out.ensure(out_b) || d->h_pick.ensure(in_b + out_b))
    return MOPCUDA_ENOMEM;
  memcpy(d->h_pick.p, xy, in_b);
  cudaStream_t s = d->stream;
  CU_TRY(cudaMemcpyAsync(d->pick_xy.p, d->h_pick.p, in_b, cudaMemcpyHostToDevice, s));
  uint32_t *oid = d->pick_out.as<uint32_t>();
  float *odp = (float *)(oid + n);
  int32_t *oht = (int32_t *)(odp + n);
  d->launches += (uint64_t)mopcuda_launch_pick(fb->ids.as<uint32_t>(), fb->depth.as<float>(), fb->w,
                                               fb->h, sf, d->pick_xy.as<int2>(), n, oid, odp, oht, s);
  CU_TRY(cudaGetLastError());
  uint8_t *hb = d->h_pick.as<uint8_t>() + in_b;
  CU_TRY(cudaMemcpyAsync(hb, d->pick_out.p, out_b, cudaMemcpyDeviceToHost, s));
  rc = mc_stream_sync(d, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  memcpy(ids, hb, 4ull * n);
  memcpy(depths, hb + 4ull * n, 4ull * n);
  memcpy(hits, hb + 8ull * n, 4ull * n);
  return MOPCUDA_OK;
}

/* ------------------------------------------------------------------------
 * measurement helpers
 * ------------------------------------------------------------------------ */
extern "C" void mopcuda_set_stage_timing(MopCudaDevice *d, int on) {
  if (d)
    d->stage_timing = on != 0;
}

extern "C" int mopcuda_stage_times(MopCudaDevice *d, float *ms, int n) {
  if (!d || !ms || n < MOPCUDA_STAGES)
    return fail(MOPCUDA_EINVAL, "stage_times: need %d floats", MOPCUDA_STAGES);
  for (int i = 0; i < MOPCUDA_STAGES; i++)
    ms[i] = d->stage_ms[i];
  return MOPCUDA_OK;
}

extern "C" int mopcuda_measure_fp32_peak(MopCudaDevice *d, double *gops) {
  if (!d || !gops)
    return fail(MOPCUDA_EINVAL, "measure_fp32_peak: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  float *tmp = nullptr;
  const int blocks = d->num_sms * 8, iters = 4096;
  CU_TRY(cudaMalloc(&tmp, sizeof(float) * (size_t)blocks));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 0.0;
  for (int rep = 0; rep < 6; rep++) {
    cudaEventRecord(a, d->stream);
    d->launches += (uint64_t)mopcuda_launch_fp32_peak(tmp, blocks, iters, d->stream);
    cudaEventRecord(b, d->stream);
    int rc = mc_bounded_sync(d, b, FRAME_TIMEOUT_MS);
    if (rc) {
      cudaFree(tmp);
      return rc;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    double ops = (double)blocks * 256.0 * (double)iters * 16.0;
    if (rep > 0 && ms > 0.0f && ops / (ms * 1e6) > best)
      best = ops / (ms * 1e6);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(tmp);
  *gops = best;
  return MOPCUDA_OK;
}

/* ------------------------------------------------------------------------
 * Batched pick without any allocation.
 *
 * For callers that cannot allocate device or pinned memory at call time —
 * hosts that run a fixed memory budget with their own allocator, code that
 * must not call cudaMalloc from a latency-critical thread (cudaMalloc and
 * cudaFree synchronise the device), or embedders that forbid allocation
 * after start-up.  The query coordinates and the results are staged in this
 * file-scope device array instead of per-device arenas.  Every GPU that
 * loads the library holds it until the process exits.
 *
 * Set-up: the first call on a device (with that device current) resolves
 * the array's device address with cudaGetSymbolAddress — the host-side name
 * is only a stand-in, not a device address.  Make that first call before
 * any stream capture.  The bounded wait uses an event the device made at
 * mopcuda_device_create (one per MopCudaDevice, so two devices on one GPU
 * never read each other's completion).
 * All calls share the array and it keeps the last call's contents (every
 * slot a call reads is written by that call first); calls whose work
 * overlaps on the GPU race on it, so callers must not overlap them.
 * The results are copied straight into the caller's buffers: the wait is
 * bounded only when they are page-locked (a copy into pageable memory holds
 * the host until the pick kernel ends), and after MOPCUDA_ETIMEOUT the
 * copies stay queued, so xy and the outputs remain in use until the device
 * is synchronised or destroyed.
 * ------------------------------------------------------------------------ */
#define NOALLOC_PICK_BYTES_PER_QUERY 20u /* int2 in, uint32 + float + int32 out */
static __device__ __align__(256) unsigned char
    g_pick_scratch[(size_t)MOPCUDA_NOALLOC_PICK_MAX * NOALLOC_PICK_BYTES_PER_QUERY];

#define NOALLOC_MAX_DEVICES 64
static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[NOALLOC_MAX_DEVICES];

static int noalloc_setup(int ordinal, unsigned char **scratch) {
  if (ordinal < 0 || ordinal >= NOALLOC_MAX_DEVICES)
    return fail(MOPCUDA_EINVAL, "pick_batch_noalloc: device ordinal %d unsupported", ordinal);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[ordinal]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_pick_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError(); /* leave no stale error for a later launch check */
      return fail(MOPCUDA_ECUDA, "pick_batch_noalloc: cudaGetSymbolAddress failed: %s",
                  cudaGetErrorString(e));
    }
    g_noalloc_ptr[ordinal] = p;
  }
  *scratch = (unsigned char *)g_noalloc_ptr[ordinal];
  return MOPCUDA_OK;
}

extern "C" int mopcuda_pick_batch_noalloc(MopCudaDevice *d, MopCudaFramebuffer *fb, int sf,
                                          const int32_t *xy, uint32_t n, uint32_t *ids,
                                          float *depths, int32_t *hits) {
  if (!d || !fb || sf <= 0 || (n && (!xy || !ids || !depths || !hits)))
    return fail(MOPCUDA_EINVAL, "pick_batch_noalloc: bad arguments");
  if (n > MOPCUDA_NOALLOC_PICK_MAX)
    return fail(MOPCUDA_EINVAL, "pick_batch_noalloc: %u queries exceed the limit of %u", n,
                (unsigned)MOPCUDA_NOALLOC_PICK_MAX);
  if (n == 0)
    return MOPCUDA_OK;
  std::lock_guard<std::mutex> lk(d->mu);
  if (d->pending && d->fb == fb)
    return fail(MOPCUDA_EINVAL, "pick_batch_noalloc: frame still pending; call "
                                "mopcuda_frame_wait first (completion may reallocate)");
  CU_TRY(cudaSetDevice(d->ordinal));
  unsigned char *scratch = nullptr;
  int rc = noalloc_setup(d->ordinal, &scratch);
  if (rc)
    return rc;
  cudaEvent_t ev = d->pick_ev;
  int2 *dxy = (int2 *)scratch;
  uint32_t *oid = (uint32_t *)(scratch + 8ull * MOPCUDA_NOALLOC_PICK_MAX);
  float *odp = (float *)(oid + MOPCUDA_NOALLOC_PICK_MAX);
  int32_t *oht = (int32_t *)(odp + MOPCUDA_NOALLOC_PICK_MAX);
  cudaStream_t s = d->stream;
  CU_TRY(cudaMemcpyAsync(dxy, xy, 8ull * n, cudaMemcpyHostToDevice, s));
  d->launches += (uint64_t)mopcuda_launch_pick(fb->ids.as<uint32_t>(), fb->depth.as<float>(),
                                               fb->w, fb->h, sf, dxy, n, oid, odp, oht, s);
  CU_TRY(cudaGetLastError());
  CU_TRY(cudaMemcpyAsync(ids, oid, 4ull * n, cudaMemcpyDeviceToHost, s));
  CU_TRY(cudaMemcpyAsync(depths, odp, 4ull * n, cudaMemcpyDeviceToHost, s));
  CU_TRY(cudaMemcpyAsync(hits, oht, 4ull * n, cudaMemcpyDeviceToHost, s));
  CU_TRY(cudaEventRecord(ev, s));
  return mc_bounded_sync(d, ev, FRAME_TIMEOUT_MS);
}
