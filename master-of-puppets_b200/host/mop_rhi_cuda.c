/*
 * mop_rhi_cuda.c — the CUDA backend's RHI function table (C11).
 *
 * Drop-in counterpart of the CPU backend's table (reference
 * src/backend/cpu/cpu_backend.c:1296-1343): every mandatory entry of
 * MopRhiBackend (src/rhi/rhi.h:132-339) plus the recommended optional ones
 * (frame_submit, frame_gpu_time_ms, set_exposure, set_ibl_textures,
 * texture_read_rgba8, frame_wait_readback, texture_create_ex with BC1/3/5
 * decoded on the device, framebuffer_copy_to_texture and
 * framebuffer_create_from_texture for render-to-texture, draw_skybox for the
 * environment background).  GPU-only effect hooks stay NULL
 * exactly as the CPU table leaves them (every caller NULL-guards them,
 * rhi.h:112-130).
 *
 * This file is compiled against the reference's own headers (it is what a
 * maintainer drops into src/backend/cuda/); each entry forwards to the plain
 * C ABI of include/mop_cuda.h, translating MopRhiDrawCall / MopLight /
 * MopVertexFormat into their POD counterparts.  Readback pointers are the
 * framebuffer's pinned host mirrors: valid until the next frame, resize or
 * destroy, and writable by the core (overlay passes write through them).
 *
 * The device is CUDA ordinal 0 unless MOP_CUDA_DEVICE names another.
 */
#include "rhi/rhi.h"

#include "mop_cuda.h"

#include <stdlib.h>
#include <string.h>

struct MopRhiDevice {
  MopCudaDevice *cu;
  MopCudaLight *lights; /* per-draw conversion scratch */
  uint32_t light_cap;
};

/* The opaque RHI handles are the C-ABI objects themselves. */
#define BUF(b) ((MopCudaBuffer *)(b))
#define TEX(t) ((MopCudaTexture *)(t))
#define FB(f) ((MopCudaFramebuffer *)(f))

static MopRhiDevice *cu_device_create(void) {
  const char *env = getenv("MOP_CUDA_DEVICE");
  int ordinal = env ? atoi(env) : 0;
  MopCudaDevice *cu = mopcuda_device_create(ordinal);
  if (!cu)
    return NULL;
  MopRhiDevice *d = calloc(1, sizeof *d);
  if (!d) {
    mopcuda_device_destroy(cu);
    return NULL;
  }
  d->cu = cu;
  return d;
}

/* The C-ABI device behind an RHI device: the core's CPU-only hooks
 * (shadow pass, IBL maps, post effects) call the C ABI with it. */
MopCudaDevice *mop_rhi_cuda_device(MopRhiDevice *d) { return d ? d->cu : NULL; }

static void cu_device_destroy(MopRhiDevice *d) {
  if (!d)
    return;
  mopcuda_device_destroy(d->cu);
  free(d->lights);
  free(d);
}

static MopRhiBuffer *cu_buffer_create(MopRhiDevice *d, const MopRhiBufferDesc *desc) {
  if (!d || !desc)
    return NULL;
  return (MopRhiBuffer *)mopcuda_buffer_create(d->cu, desc->data, desc->size);
}

static void cu_buffer_destroy(MopRhiDevice *d, MopRhiBuffer *b) {
  mopcuda_buffer_destroy(d->cu, BUF(b));
}

static void cu_buffer_update(MopRhiDevice *d, MopRhiBuffer *b, const void *data, size_t off,
                             size_t size) {
  mopcuda_buffer_update(d->cu, BUF(b), data, off, size);
}

static const void *cu_buffer_read(MopRhiBuffer *b) { return mopcuda_buffer_read(BUF(b)); }

static MopRhiFramebuffer *cu_framebuffer_create(MopRhiDevice *d, const MopRhiFramebufferDesc *desc) {
  if (!d || !desc)
    return NULL;
  return (MopRhiFramebuffer *)mopcuda_framebuffer_create(d->cu, desc->width, desc->height);
}

static void cu_framebuffer_destroy(MopRhiDevice *d, MopRhiFramebuffer *fb) {
  mopcuda_framebuffer_destroy(d->cu, FB(fb));
}

static void cu_framebuffer_resize(MopRhiDevice *d, MopRhiFramebuffer *fb, int w, int h) {
  mopcuda_framebuffer_resize(d->cu, FB(fb), w, h);
}

static void cu_frame_begin(MopRhiDevice *d, MopRhiFramebuffer *fb, MopColor clear) {
  float c[4] = {clear.r, clear.g, clear.b, clear.a};
  mopcuda_frame_begin(d->cu, FB(fb), c);
}

/* The whole recorded frame runs on the device here; readbacks wait for it. */
static void cu_frame_end(MopRhiDevice *d, MopRhiFramebuffer *fb) {
  mopcuda_frame_end(d->cu, FB(fb));
}

static void cu_frame_submit(MopRhiDevice *d, MopRhiFramebuffer *fb) {
  (void)d;
  (void)fb;
}

static void cu_frame_wait_readback(MopRhiDevice *d, MopRhiFramebuffer *fb) {
  (void)fb;
  mopcuda_frame_wait(d->cu, 20000);
}

static int comps(MopAttribFormat f) {
  switch (f) {
  case MOP_FORMAT_FLOAT:
    return 1;
  case MOP_FORMAT_FLOAT2:
    return 2;
  case MOP_FORMAT_FLOAT3:
    return 3;
  case MOP_FORMAT_FLOAT4:
    return 4;
  default:
    return 0; /* read as the reference's default case: zeros */
  }
}

static void layout_attr(const MopVertexFormat *vf, MopAttribSemantic s, int32_t *off, int32_t *n) {
  const MopVertexAttrib *a = mop_vertex_format_find(vf, s);
  *off = a ? (int32_t)a->offset : -1;
  *n = a ? comps(a->format) : 0;
}

/* Translate the draw-call fields the frame path reads (EMIT_DRAW,
 * reference viewport.c:2015-2088). */
static int to_cuda_draw(MopRhiDevice *d, const MopRhiDrawCall *c, MopCudaDraw *o,
                        MopCudaVertexLayout *lay) {
  memset(o, 0, sizeof *o);
  o->vertex_buffer = BUF(c->vertex_buffer);
  o->index_buffer = BUF(c->index_buffer);
  o->vertex_count = c->vertex_count;
  o->index_count = c->index_count;
  o->object_id = c->object_id;
  memcpy(o->model, c->model.d, sizeof o->model);
  memcpy(o->mvp, c->mvp.d, sizeof o->mvp);
  o->light_dir[0] = c->light_dir.x;
  o->light_dir[1] = c->light_dir.y;
  o->light_dir[2] = c->light_dir.z;
  o->ambient = c->ambient;
  o->opacity = c->opacity;
  o->metallic = c->metallic;
  o->roughness = c->roughness;
  o->depth_bias = c->depth_bias;
  o->cam_eye[0] = c->cam_eye.x;
  o->cam_eye[1] = c->cam_eye.y;
  o->cam_eye[2] = c->cam_eye.z;
  o->smooth = c->shading_mode == MOP_SHADING_SMOOTH;
  o->wireframe = c->wireframe;
  o->depth_test = c->depth_test;
  o->depth_write = c->depth_write;
  o->backface_cull = c->backface_cull;
  o->blend_mode = (int32_t)c->blend_mode;
  o->texture = TEX(c->texture);
  if (c->lights && c->light_count) {
    if (c->light_count > d->light_cap) {
      MopCudaLight *n = realloc(d->lights, sizeof(MopCudaLight) * c->light_count);
      if (!n)
        return -1;
      d->lights = n;
      d->light_cap = c->light_count;
    }
    for (uint32_t i = 0; i < c->light_count; i++) {
      const MopLight *s = &c->lights[i];
      MopCudaLight *t = &d->lights[i];
      t->type = (int32_t)s->type;
      t->position[0] = s->position.x;
      t->position[1] = s->position.y;
      t->position[2] = s->position.z;
      t->direction[0] = s->direction.x;
      t->direction[1] = s->direction.y;
      t->direction[2] = s->direction.z;
      t->color[0] = s->color.r;
      t->color[1] = s->color.g;
      t->color[2] = s->color.b;
      t->color[3] = s->color.a;
      t->intensity = s->intensity;
      t->range = s->range;
      t->spot_inner_cos = s->spot_inner_cos;
      t->spot_outer_cos = s->spot_outer_cos;
      t->active = s->active ? 1 : 0;
    }
    o->lights = d->lights;
    o->light_count = c->light_count;
  }
  if (c->vertex_format) {
    const MopVertexFormat *vf = c->vertex_format;
    lay->stride = vf->stride;
    layout_attr(vf, MOP_ATTRIB_POSITION, &lay->position_offset, &lay->position_components);
    layout_attr(vf, MOP_ATTRIB_NORMAL, &lay->normal_offset, &lay->normal_components);
    layout_attr(vf, MOP_ATTRIB_COLOR, &lay->color_offset, &lay->color_components);
    layout_attr(vf, MOP_ATTRIB_TEXCOORD0, &lay->uv_offset, &lay->uv_components);
    o->layout = lay;
  }
  return 0;
}

static void cu_draw(MopRhiDevice *d, MopRhiFramebuffer *fb, const MopRhiDrawCall *c) {
  MopCudaDraw dc;
  MopCudaVertexLayout lay;
  if (to_cuda_draw(d, c, &dc, &lay) == 0)
    mopcuda_draw(d->cu, FB(fb), &dc);
}

static void cu_draw_skybox(MopRhiDevice *d, MopRhiFramebuffer *fb, MopRhiTexture *env,
                           const float *inv_vp, const float *cam_pos, float rotation,
                           float intensity) {
  mopcuda_draw_skybox(d->cu, FB(fb), TEX(env), inv_vp, cam_pos, rotation, intensity);
}

static void cu_draw_instanced(MopRhiDevice *d, MopRhiFramebuffer *fb, const MopRhiDrawCall *c,
                              const MopMat4 *inst, uint32_t n) {
  if (!c || !inst || n == 0)
    return;
  MopCudaDraw dc;
  MopCudaVertexLayout lay;
  if (to_cuda_draw(d, c, &dc, &lay) == 0)
    mopcuda_draw_instanced(d->cu, FB(fb), &dc, c->view.d, c->projection.d, inst[0].d, n);
}

static uint32_t cu_pick_read_id(MopRhiDevice *d, MopRhiFramebuffer *fb, int x, int y) {
  return mopcuda_pick_read_id(d->cu, FB(fb), x, y);
}

static float cu_pick_read_depth(MopRhiDevice *d, MopRhiFramebuffer *fb, int x, int y) {
  return mopcuda_pick_read_depth(d->cu, FB(fb), x, y);
}

static const uint8_t *cu_read_color(MopRhiDevice *d, MopRhiFramebuffer *fb, int *w, int *h) {
  return mopcuda_read_color(d->cu, FB(fb), w, h);
}

static const uint32_t *cu_read_object_id(MopRhiDevice *d, MopRhiFramebuffer *fb, int *w, int *h) {
  return mopcuda_read_object_id(d->cu, FB(fb), w, h);
}

static const float *cu_read_depth(MopRhiDevice *d, MopRhiFramebuffer *fb, int *w, int *h) {
  return mopcuda_read_depth(d->cu, FB(fb), w, h);
}

static MopRhiTexture *cu_texture_create(MopRhiDevice *d, int w, int h, const uint8_t *rgba) {
  return (MopRhiTexture *)mopcuda_texture_create(d->cu, w, h, rgba);
}

static MopRhiTexture *cu_texture_create_hdr(MopRhiDevice *d, int w, int h, const float *rgba) {
  return (MopRhiTexture *)mopcuda_texture_create_hdr(d->cu, w, h, rgba);
}

static MopRhiTexture *cu_texture_create_ex(MopRhiDevice *d, int w, int h, int format, int mips,
                                          const uint8_t *data, size_t size) {
  return (MopRhiTexture *)mopcuda_texture_create_ex(d->cu, w, h, format, mips, data, size);
}

static bool cu_framebuffer_copy_to_texture(MopRhiDevice *d, MopRhiFramebuffer *fb,
                                           MopRhiTexture *t) {
  return mopcuda_framebuffer_copy_to_texture(d->cu, FB(fb), TEX(t)) == MOPCUDA_OK;
}

static MopRhiFramebuffer *cu_framebuffer_create_from_texture(MopRhiDevice *d, MopRhiTexture *t,
                                                             int w, int h) {
  return (MopRhiFramebuffer *)mopcuda_framebuffer_create_from_texture(d->cu, TEX(t), w, h);
}

static void cu_texture_destroy(MopRhiDevice *d, MopRhiTexture *t) {
  mopcuda_texture_destroy(d->cu, TEX(t));
}

static bool cu_texture_read_rgba8(MopRhiDevice *d, MopRhiTexture *t, uint8_t *out, size_t n) {
  return mopcuda_texture_read_rgba8(d->cu, TEX(t), out, n) == MOPCUDA_OK;
}

static float cu_frame_gpu_time_ms(MopRhiDevice *d) { return mopcuda_frame_gpu_time_ms(d->cu); }

static void cu_set_exposure(MopRhiDevice *d, float e) { mopcuda_set_exposure(d->cu, e); }

/* The table-level IBL hook only carries textures (rhi.h:286-293): no
 * rotation, intensity or mip chain.  A core that feeds the CPU path's full
 * state uses mopcuda_set_ibl directly (the sw_ibl_set hook). */
static void cu_set_ibl_textures(MopRhiDevice *d, MopRhiTexture *irr, MopRhiTexture *pf,
                                MopRhiTexture *brdf) {
  (void)irr;
  (void)pf;
  (void)brdf;
  (void)d;
}

static const MopRhiBackend CUDA_BACKEND = {
    .name = "cuda",
    .device_create = cu_device_create,
    .device_destroy = cu_device_destroy,
    .buffer_create = cu_buffer_create,
    .buffer_destroy = cu_buffer_destroy,
    .framebuffer_create = cu_framebuffer_create,
    .framebuffer_destroy = cu_framebuffer_destroy,
    .framebuffer_resize = cu_framebuffer_resize,
    .framebuffer_create_from_texture = cu_framebuffer_create_from_texture,
    .frame_begin = cu_frame_begin,
    .frame_end = cu_frame_end,
    .frame_submit = cu_frame_submit,
    .frame_wait_readback = cu_frame_wait_readback,
    .draw = cu_draw,
    .pick_read_id = cu_pick_read_id,
    .pick_read_depth = cu_pick_read_depth,
    .framebuffer_read_color = cu_read_color,
    .framebuffer_read_object_id = cu_read_object_id,
    .framebuffer_read_depth = cu_read_depth,
    .texture_create = cu_texture_create,
    .texture_create_hdr = cu_texture_create_hdr,
    .texture_create_ex = cu_texture_create_ex,
    .texture_destroy = cu_texture_destroy,
    .draw_instanced = cu_draw_instanced,
    .draw_skybox = cu_draw_skybox,
    .buffer_update = cu_buffer_update,
    .buffer_read = cu_buffer_read,
    .frame_gpu_time_ms = cu_frame_gpu_time_ms,
    .set_exposure = cu_set_exposure,
    .set_ibl_textures = cu_set_ibl_textures,
    .texture_read_rgba8 = cu_texture_read_rgba8,
    .framebuffer_copy_to_texture = cu_framebuffer_copy_to_texture,
};

const MopRhiBackend *mop_rhi_backend_cuda(void) { return &CUDA_BACKEND; }
