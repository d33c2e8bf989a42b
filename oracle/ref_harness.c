/*
 * ref_harness.c — drives the unmodified reference library on its CPU backend.
 *
 * Test infrastructure only (see ref_harness.h).  Scene construction follows
 * the parity rules for the CPU frame path:
 *   - chrome off (mop_viewport_set_chrome, reference viewport.c:3934-3942) so
 *     no gradient quad / grid draws are issued;
 *   - the always-on outline overlay disabled (viewport.c:745);
 *   - lights cleared (the default sun would otherwise drive the shadow pass,
 *     viewport.c:683-692, 2288-2442), then the scene's lights added with their
 *     own cast_shadows flags;
 *   - base colour baked into vertex colours by the caller (CPU shading reads
 *     vertex colour only); metallic/roughness through mop_mesh_set_material.
 * Serial mode nulls the CPU device's tile pool so cpu_draw takes its
 * single-threaded loop (reference cpu_backend.c:29-31, 589-620).
 */
#include "ref_harness.h"

#include "core/viewport_internal.h"
#include "rasterizer/rasterizer_mt.h"

#include <mop/loader/loader.h>
#include <mop/loader/mop_scene.h>
#include <mop/mop.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

typedef struct RefH {
  MopViewport *vp;
  MopTexture **textures;
  uint32_t texture_count;
  int w, h, ssaa;
  int threads;
  MopViewport *tex_vp;  /* owns the render target texture */
  MopTexture *target;
  bool cpu;             /* the viewport runs on the CPU backend */
} RefH;

/* The CPU backend's texture_create mallocs the texture record without
 * clearing hdr_data (cpu_backend.c:811-827) and texture_destroy frees that
 * field (:1064-1072), which faults once the heap hands back reused memory;
 * the harness therefore leaves RGBA8 textures it made on the CPU backend
 * alive (a test-sized leak) and destroys them on the CUDA backend. */
static void harness_texture_release(RefH *h, MopViewport *vp, MopTexture *t) {
  if (t && !h->cpu)
    mop_viewport_destroy_texture(vp, t);
}

static int cmp_double(const void *a, const void *b);

static double now_ms(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec * 1e3 + (double)ts.tv_nsec * 1e-6;
}

#ifdef REFH_CUDA_HOOKS
#include "mop_cuda.h"

MopCudaDevice *mop_rhi_cuda_device(MopRhiDevice *d);

/* The integration patch's shadow pass for the CUDA backend, run as a
 * MOP_STAGE_PRE_SCENE hook (the core gates its own pass_shadow to the CPU
 * backend, viewport.c:3224, and keeps it static): the casters the core would
 * select (active, below the chrome IDs, opaque; viewport.c:2310-2315), the
 * light camera from mopcuda_shadow_light_vp, every caster's RHI buffers
 * rasterised by the C ABI, the map bound for the frame's draws. */
static void cuda_shadow_hook(MopViewport *vp, void *ud) {
  (void)ud;
  MopCudaDevice *cu = mop_rhi_cuda_device(vp->device);
  const MopLight *sun = NULL;
  for (uint32_t i = 0; i < vp->light_count && !sun; i++)
    if (vp->lights[i].active && vp->lights[i].type == MOP_LIGHT_DIRECTIONAL &&
        vp->lights[i].cast_shadows)
      sun = &vp->lights[i];
  uint32_t n = 0;
  float *models = malloc(sizeof(float) * 16 * (vp->mesh_count ? vp->mesh_count : 1));
  struct MopMesh **casters = malloc(sizeof(*casters) * (vp->mesh_count ? vp->mesh_count : 1));
  for (uint32_t i = 0; sun && models && casters && i < vp->mesh_count; i++) {
    struct MopMesh *m = vp->meshes[i];
    if (!m->active || m->object_id >= 0xFFFD0000u || m->blend_mode != MOP_BLEND_OPAQUE)
      continue;
    memcpy(models + 16 * n, m->world_transform.d, sizeof(float) * 16);
    casters[n++] = m;
  }
  float light_vp[16];
  const float dir[3] = {sun ? sun->direction.x : 0.0f, sun ? sun->direction.y : 0.0f,
                        sun ? sun->direction.z : 0.0f};
  if (!n || !mopcuda_shadow_light_vp(models, n, dir, light_vp)) {
    mopcuda_shadow_clear(cu);
  } else {
    mopcuda_shadow_begin(cu, 1024, light_vp);
    for (uint32_t k = 0; k < n; k++)
      mopcuda_shadow_draw(cu, (MopCudaBuffer *)casters[k]->vertex_buffer,
                          casters[k]->vertex_count, (uint32_t)sizeof(MopVertex),
                          (MopCudaBuffer *)casters[k]->index_buffer, casters[k]->index_count,
                          models + 16 * k);
    mopcuda_shadow_end(cu);
  }
  free(models);
  free(casters);
}

/* The integration patch's post-process and IBL rows for the CUDA backend:
 * the core applies vp->post_effects and vp->fog_params itself for its CPU
 * backend only (rg_cleanup, viewport.c:2950-2961) and hands the IBL maps only
 * to the CPU rasteriser; the patch gives all of them to the device.  Run as
 * a MOP_STAGE_PRE_SCENE hook, so the values of the frame being rendered
 * apply. */
static void cuda_post_hook(MopViewport *vp, void *ud) {
  (void)ud;
  MopCudaDevice *cu = mop_rhi_cuda_device(vp->device);
  const float fog[4] = {vp->fog_params.color.r, vp->fog_params.color.g, vp->fog_params.color.b,
                        vp->fog_params.color.a};
  mopcuda_set_post_effects(cu, vp->post_effects);
  mopcuda_set_fog(cu, fog, vp->fog_params.near_dist, vp->fog_params.far_dist);
  /* the IBL row: the maps, rotation and intensity rg_ibl_setup hands the
   * CPU rasteriser (viewport.c:2698-2705); none bound when there are none */
  if (vp->env_irradiance_data)
    mopcuda_set_ibl(cu, vp->env_irradiance_data, vp->env_irradiance_w, vp->env_irradiance_h,
                    vp->env_prefiltered_data, vp->env_prefiltered_w, vp->env_prefiltered_h,
                    vp->env_prefiltered_levels, vp->env_brdf_lut_data, 256, vp->env_rotation,
                    vp->env_intensity);
  else
    mopcuda_set_ibl(cu, NULL, 0, 0, NULL, 0, 0, 0, NULL, 0, 0.0f, 1.0f);
}
#endif

void *refh_create(const RefScene *sc) {
  if (!sc || sc->width <= 0 || sc->height <= 0)
    return NULL;
  RefH *h = calloc(1, sizeof(RefH));
  if (!h)
    return NULL;
  bool cpu = sc->backend == 0;
  h->cpu = cpu;
  MopViewportDesc desc = {.width = sc->width,
                          .height = sc->height,
                          .backend = cpu ? MOP_BACKEND_CPU : (MopBackendType)sc->backend,
                          .reverse_z = false,
                          .ssaa_factor = sc->ssaa};
  if (sc->render_target) {
    /* the host-owned texture comes from another viewport of the backend */
    MopViewportDesc td = desc;
    td.width = td.height = 8;
    td.ssaa_factor = 1;
    h->tex_vp = mop_viewport_create(&td);
    uint8_t *zero = calloc((size_t)sc->width * sc->height, 4);
    if (h->tex_vp && zero)
      h->target = mop_viewport_create_texture(h->tex_vp, sc->width, sc->height, zero);
    /* The CPU backend's cpu_texture_create (cpu_backend.c:811) mallocs its
     * texture record without setting is_hdr / hdr_data, and
     * framebuffer_create_from_texture refuses a target whose is_hdr reads
     * true (:156), so whether a render target works depends on what the
     * allocator hands back.  The harness sets the two fields the reference
     * leaves unset, through the record's layout (cpu_backend.c:43-49). */
    if (cpu && h->target && h->target->rhi_texture) {
      struct CpuTexRecord {
        int width, height;
        uint8_t *data;
        float *hdr_data;
        bool is_hdr;
      } *rec = (struct CpuTexRecord *)(void *)h->target->rhi_texture;
      rec->hdr_data = NULL;
      rec->is_hdr = false;
    }
    free(zero);
    if (!h->target) {
      if (h->tex_vp)
        mop_viewport_destroy(h->tex_vp);
      free(h);
      return NULL;
    }
    desc.render_target = h->target;
  }
  h->vp = mop_viewport_create(&desc);
  if (!h->vp) {
    harness_texture_release(h, h->tex_vp, h->target);
    if (h->tex_vp)
      mop_viewport_destroy(h->tex_vp);
    free(h);
    return NULL;
  }
  MopViewport *vp = h->vp;
  h->w = sc->width;
  h->h = sc->height;
  h->ssaa = vp->ssaa_factor;

  long n = sysconf(_SC_NPROCESSORS_ONLN);
  h->threads = n > 1 ? (int)n : 1;
  /* The CPU device's only member is its tile pool pointer. */
  MopSwThreadPool **pool = (MopSwThreadPool **)vp->device;
  if (!cpu) {
    h->threads = 0;
  } else if (sc->serial) {
    if (*pool) {
      mop_sw_threadpool_destroy(*pool);
      *pool = NULL;
    }
    h->threads = 1;
  } else if (sc->workers > 0) {
    if (*pool)
      mop_sw_threadpool_destroy(*pool);
    *pool = mop_sw_threadpool_create(sc->workers);
    h->threads = sc->workers + 1; /* workers + the calling thread */
  }

#ifdef REFH_CUDA_HOOKS
  if (!cpu) {
    mop_viewport_add_hook(vp, MOP_STAGE_PRE_SCENE, cuda_shadow_hook, NULL);
    mop_viewport_add_hook(vp, MOP_STAGE_PRE_SCENE, cuda_post_hook, NULL);
  }
#endif
  mop_viewport_set_chrome(vp, false);
  mop_viewport_set_overlay_enabled(vp, MOP_OVERLAY_OUTLINE, false);
  mop_viewport_set_clear_color(
      vp, (MopColor){sc->clear_color[0], sc->clear_color[1],
                     sc->clear_color[2], sc->clear_color[3]});
  mop_viewport_set_ambient(vp, sc->ambient);
  mop_viewport_set_exposure(vp, sc->exposure);
  mop_viewport_set_post_effects(vp, sc->post_effects);
  if (sc->fog_on) {
    MopFogParams fog = {{sc->fog_color[0], sc->fog_color[1], sc->fog_color[2], sc->fog_color[3]},
                        sc->fog_near, sc->fog_far};
    mop_viewport_set_fog(vp, &fog);
  }
  if (sc->flat)
    mop_viewport_set_shading(vp, MOP_SHADING_FLAT);
  if (sc->wireframe) {
    mop_viewport_set_render_mode(vp, MOP_RENDER_WIREFRAME);
    if (sc->wireframe == 1 && vp->grid) {
      mop_viewport_remove_mesh(vp, vp->grid);
      vp->grid = NULL;
    }
  }
  mop_viewport_set_camera(
      vp, (MopVec3){sc->eye[0], sc->eye[1], sc->eye[2]},
      (MopVec3){sc->target[0], sc->target[1], sc->target[2]},
      (MopVec3){sc->up[0], sc->up[1], sc->up[2]}, sc->fov_deg, sc->near_plane,
      sc->far_plane);

  mop_viewport_clear_lights(vp);
  for (uint32_t i = 0; i < sc->light_count; i++) {
    const RefLight *L = &sc->lights[i];
    MopLight d = {
        .type = (MopLightType)L->type,
        .position = {L->position[0], L->position[1], L->position[2]},
        .direction = {L->direction[0], L->direction[1], L->direction[2]},
        .color = {L->color[0], L->color[1], L->color[2], L->color[3]},
        .intensity = L->intensity,
        .range = L->range,
        .spot_inner_cos = L->spot_inner_cos,
        .spot_outer_cos = L->spot_outer_cos,
        .active = L->active != 0,
        .cast_shadows = L->cast_shadows != 0,
    };
    MopLight *slot = mop_viewport_add_light(vp, &d);
    /* add_light always activates its slot (reference light.c:26-71). */
    if (slot && !L->active)
      mop_viewport_remove_light(vp, slot);
  }

  if (sc->texture_count) {
    h->textures = calloc(sc->texture_count, sizeof(MopTexture *));
    h->texture_count = sc->texture_count;
    for (uint32_t t = 0; t < sc->texture_count; t++) {
      if (sc->tex_format && sc->tex_format[t] != 0) {
        MopTextureDesc td = {.width = sc->tex_w[t],
                             .height = sc->tex_h[t],
                             .mip_levels = 1,
                             .format = (MopTexFormat)sc->tex_format[t],
                             .data = sc->tex_data[t],
                             .data_size = sc->tex_bytes ? sc->tex_bytes[t] : 0};
        h->textures[t] = mop_tex_create(vp, &td);
      } else {
        h->textures[t] = mop_viewport_create_texture(vp, sc->tex_w[t], sc->tex_h[t],
                                                     sc->tex_data[t]);
      }
    }
  }

  for (uint32_t m = 0; m < sc->mesh_count; m++) {
    const RefMesh *rm = &sc->meshes[m];
    MopMeshDesc md = {.vertices = (const MopVertex *)rm->vertices,
                      .vertex_count = rm->vertex_count,
                      .indices = rm->indices,
                      .index_count = rm->index_count,
                      .object_id = rm->object_id};
    MopMesh *mesh = mop_viewport_add_mesh(vp, &md);
    if (!mesh)
      continue;
    MopMat4 t;
    memcpy(t.d, rm->transform, sizeof(t.d));
    mop_mesh_set_transform(mesh, &t);
    if (rm->has_material) {
      MopMaterial mat = mop_material_default();
      mat.metallic = rm->metallic;
      mat.roughness = rm->roughness;
      mop_mesh_set_material(mesh, &mat);
    }
    if (rm->texture >= 0 && (uint32_t)rm->texture < h->texture_count)
      mop_mesh_set_texture(mesh, h->textures[rm->texture]);
    if (rm->blend_mode > 0)
      mop_mesh_set_blend_mode(mesh, (MopBlendMode)rm->blend_mode);
    if (rm->opacity != 1.0f)
      mop_mesh_set_opacity(mesh, rm->opacity);
  }

  for (uint32_t k = 0; k < sc->instanced_count; k++) {
    const RefInstanced *ri = &sc->instanced[k];
    MopMeshDesc md = {.vertices = (const MopVertex *)ri->vertices,
                      .vertex_count = ri->vertex_count,
                      .indices = ri->indices,
                      .index_count = ri->index_count,
                      .object_id = ri->object_id};
    mop_viewport_add_instanced_mesh(vp, &md, (const MopMat4 *)ri->transforms,
                                    ri->instance_count);
  }

  if (sc->env == 1) {
    MopProceduralSkyDesc sky = {
        .sun_direction = {sc->sun_dir[0], sc->sun_dir[1], sc->sun_dir[2]},
        .turbidity = sc->turbidity,
        .ground_albedo = sc->ground_albedo};
    mop_viewport_set_procedural_sky(vp, &sky);
    MopEnvironmentDesc env = {.type = MOP_ENV_PROCEDURAL_SKY,
                              .rotation = sc->env_rotation,
                              .intensity = sc->env_intensity};
    mop_viewport_set_environment(vp, &env);
    if (sc->env_background)
      mop_viewport_set_environment_background(vp, true);
  }
  return h;
}

int refh_render(void *hp, RefFrame *out) {
  RefH *h = hp;
  if (!h)
    return -1;
  MopViewport *vp = h->vp;
  if (mop_viewport_render(vp) != MOP_RENDER_OK)
    return -2;
  int w = 0, hh = 0;
  const uint8_t *c = mop_viewport_read_color(vp, &w, &hh);
  if (!c)
    return -3;
  if (out->color)
    memcpy(out->color, c, (size_t)w * hh * 4);
  int fw = 0, fh = 0;
  const uint8_t *cf =
      vp->rhi->framebuffer_read_color(vp->device, vp->framebuffer, &fw, &fh);
  if (out->color_full && cf)
    memcpy(out->color_full, cf, (size_t)fw * fh * 4);
  const float *d =
      vp->rhi->framebuffer_read_depth(vp->device, vp->framebuffer, &fw, &fh);
  if (out->depth && d)
    memcpy(out->depth, d, (size_t)fw * fh * sizeof(float));
  const uint32_t *id = vp->rhi->framebuffer_read_object_id(
      vp->device, vp->framebuffer, &fw, &fh);
  if (out->object_id && id)
    memcpy(out->object_id, id, (size_t)fw * fh * sizeof(uint32_t));
  memcpy(out->view, vp->view_matrix.d, sizeof(out->view));
  memcpy(out->proj, vp->projection_matrix.d, sizeof(out->proj));
  out->eye[0] = vp->cam_eye.x;
  out->eye[1] = vp->cam_eye.y;
  out->eye[2] = vp->cam_eye.z;
  MopFrameStats st = mop_viewport_get_stats(vp);
  out->triangle_count = st.triangle_count;
  out->frame_ms = st.frame_time_ms;
  return 0;
}

int refh_pick(void *hp, int n, const int32_t *xy, uint32_t *ids, float *depths,
              int32_t *hits) {
  RefH *h = hp;
  if (!h)
    return -1;
  for (int i = 0; i < n; i++) {
    MopPickResult r = mop_viewport_pick(h->vp, xy[2 * i], xy[2 * i + 1]);
    ids[i] = r.object_id;
    depths[i] = r.depth;
    hits[i] = r.hit ? 1 : 0;
  }
  return 0;
}

int refh_env_maps(void *hp, const float **irr, int32_t *iw, int32_t *ih,
                  const float **pf, int32_t *pw, int32_t *ph, int32_t *levels,
                  const float **brdf, int32_t *brdf_size) {
  RefH *h = hp;
  if (!h || !h->vp->env_irradiance_data)
    return -1;
  MopViewport *vp = h->vp;
  *irr = vp->env_irradiance_data;
  *iw = vp->env_irradiance_w;
  *ih = vp->env_irradiance_h;
  *pf = vp->env_prefiltered_data;
  *pw = vp->env_prefiltered_w;
  *ph = vp->env_prefiltered_h;
  *levels = vp->env_prefiltered_levels;
  *brdf = vp->env_brdf_lut_data;
  *brdf_size = 256; /* BRDF_LUT_SIZE, reference viewport.c:2702 */
  return 0;
}

int refh_scene_save(void *hp, const char *path, uint32_t flags) {
  RefH *h = hp;
  return h ? mop_scene_save(h->vp, path, flags) : -1;
}

int refh_scene_file_mesh(const char *path, uint32_t idx, float *vertices, uint32_t vcap,
                         uint32_t *indices, uint32_t icap, uint32_t *vc, uint32_t *ic,
                         float bbox[6]) {
  MopSceneFile *f = mop_scene_load(path);
  if (!f)
    return -1;
  MopLoadedMesh m;
  int rc = -2;
  if (mop_scene_get_mesh(f, idx, &m)) {
    rc = -3;
    if (m.vertex_count <= vcap && m.index_count <= icap) {
      memcpy(vertices, m.vertices, (size_t)m.vertex_count * sizeof(MopVertex));
      memcpy(indices, m.indices, (size_t)m.index_count * sizeof(uint32_t));
      *vc = m.vertex_count;
      *ic = m.index_count;
      bbox[0] = m.bbox_min.x;
      bbox[1] = m.bbox_min.y;
      bbox[2] = m.bbox_min.z;
      bbox[3] = m.bbox_max.x;
      bbox[4] = m.bbox_max.y;
      bbox[5] = m.bbox_max.z;
      rc = 0;
    }
    free(m.vertices);
    free(m.indices);
  }
  mop_scene_free(f);
  return rc;
}

double refh_time_scene_file(const char *path, int reps) {
  double *t = malloc(sizeof(double) * (size_t)(reps > 0 ? reps : 1));
  for (int r = 0; r < reps; r++) {
    double t0 = now_ms();
    MopSceneFile *f = mop_scene_load(path);
    if (!f) {
      free(t);
      return -1.0;
    }
    uint32_t n = mop_scene_mesh_count(f);
    for (uint32_t k = 0; k < n; k++) {
      MopLoadedMesh m;
      if (mop_scene_get_mesh(f, k, &m)) {
        free(m.vertices);
        free(m.indices);
      }
    }
    mop_scene_free(f);
    t[r] = now_ms() - t0;
  }
  qsort(t, (size_t)reps, sizeof(double), cmp_double);
  double med = t[reps / 2];
  free(t);
  return med;
}

int refh_env_hdr(void *hp, const float **hdr, int32_t *w, int32_t *h) {
  RefH *rh = hp;
  if (!rh || !rh->vp->env_hdr_data)
    return -1;
  *hdr = rh->vp->env_hdr_data;
  *w = rh->vp->env_width;
  *h = rh->vp->env_height;
  return 0;
}

static int cmp_double(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return (x > y) - (x < y);
}

double refh_time_frames(void *hp, int warm, int frames) {
  RefH *h = hp;
  if (!h || frames <= 0)
    return -1.0;
  for (int i = 0; i < warm; i++) {
    mop_viewport_render(h->vp);
    mop_viewport_read_color(h->vp, NULL, NULL);
  }
  double *t = malloc(sizeof(double) * (size_t)frames);
  for (int i = 0; i < frames; i++) {
    double t0 = now_ms();
    mop_viewport_render(h->vp);
    mop_viewport_read_color(h->vp, NULL, NULL);
    t[i] = now_ms() - t0;
  }
  qsort(t, (size_t)frames, sizeof(double), cmp_double);
  double med = t[frames / 2];
  free(t);
  return med;
}

double refh_time_environment(void *hp, int reps) {
  RefH *h = hp;
  if (!h || reps <= 0)
    return -1.0;
  MopViewport *vp = h->vp;
  MopEnvironmentDesc env = {.type = MOP_ENV_PROCEDURAL_SKY,
                            .rotation = vp->env_rotation,
                            .intensity = vp->env_intensity};
  double *t = malloc(sizeof(double) * (size_t)reps);
  for (int i = 0; i < reps; i++) {
    double t0 = now_ms();
    mop_viewport_set_environment(vp, &env); /* sky + the three precomputes */
    t[i] = now_ms() - t0;
  }
  qsort(t, (size_t)reps, sizeof(double), cmp_double);
  double med = t[reps / 2];
  free(t);
  return med;
}

int refh_num_threads(void *hp) {
  RefH *h = hp;
  return h ? h->threads : 0;
}

void refh_destroy(void *hp) {
  RefH *h = hp;
  if (!h)
    return;
  /* Textures belong to the viewport and are released with it. */
  free(h->textures);
  mop_viewport_destroy(h->vp);
  harness_texture_release(h, h->tex_vp, h->target);
  if (h->tex_vp)
    mop_viewport_destroy(h->tex_vp);
  free(h);
}

int refh_bc_decode(int backend, int format, int w, int h, const uint8_t *data, uint32_t size,
                   uint8_t *out) {
  const MopRhiBackend *rhi =
      mop_rhi_get_backend(backend == 0 ? MOP_BACKEND_CPU : (MopBackendType)backend);
  if (!rhi || !rhi->texture_create_ex || !rhi->texture_read_rgba8 || !data || !out)
    return -1;
  MopRhiDevice *dev = rhi->device_create();
  if (!dev)
    return -1;
  int rc = -2;
  MopRhiTexture *t = rhi->texture_create_ex(dev, w, h, format, 1, data, size);
  if (t) {
    rc = rhi->texture_read_rgba8(dev, t, out, (size_t)w * h * 4) ? 0 : -3;
    /* not destroyed on the CPU backend (see harness_texture_release) */
    if (backend != 0)
      rhi->texture_destroy(dev, t);
  }
  rhi->device_destroy(dev);
  return rc;
}

int refh_present_to_texture(void *hp, int tw, int th, uint8_t *out) {
  RefH *h = hp;
  if (!h || tw <= 0 || th <= 0 || !out)
    return -1;
  uint8_t *zero = calloc((size_t)tw * th, 4);
  if (!zero)
    return -1;
  MopTexture *t = mop_viewport_create_texture(h->vp, tw, th, zero);
  free(zero);
  if (!t)
    return -2;
  int ok = mop_viewport_present_to_texture(h->vp, t) ? 1 : 0;
  if (ok && !mop_tex_read_rgba8(h->vp, t, out, (size_t)tw * th * 4))
    ok = -3;
  harness_texture_release(h, h->vp, t);
  return ok;
}

int refh_read_target(void *hp, uint8_t *out) {
  RefH *h = hp;
  if (!h || !h->target || !out)
    return -1;
  return mop_tex_read_rgba8(h->tex_vp, h->target, out, (size_t)h->w * h->h * 4) ? 0 : -2;
}

int refh_deform_probe(const uint8_t *vertices, uint32_t vertex_count, const float *bones,
                      uint32_t bone_count, const float *targets, const float *weights,
                      uint32_t target_count, uint8_t *out) {
  if (!vertices || vertex_count < 3 || !out)
    return -1;
  MopViewportDesc desc = {.width = 16, .height = 16, .backend = MOP_BACKEND_CPU, .ssaa_factor = 1};
  MopViewport *vp = mop_viewport_create(&desc);
  if (!vp)
    return -1;
  mop_viewport_set_chrome(vp, false);
  MopVertexFormat fmt;
  memset(&fmt, 0, sizeof fmt);
  fmt.attribs[0] = (MopVertexAttrib){MOP_ATTRIB_POSITION, MOP_FORMAT_FLOAT3, 0};
  fmt.attribs[1] = (MopVertexAttrib){MOP_ATTRIB_NORMAL, MOP_FORMAT_FLOAT3, 12};
  fmt.attribs[2] = (MopVertexAttrib){MOP_ATTRIB_JOINTS, MOP_FORMAT_UBYTE4, 24};
  fmt.attribs[3] = (MopVertexAttrib){MOP_ATTRIB_WEIGHTS, MOP_FORMAT_FLOAT4, 28};
  fmt.attrib_count = 4;
  fmt.stride = 44;
  const uint32_t idx[3] = {0, 1, 2};
  MopMeshDescEx md = {.vertex_data = vertices, .vertex_count = vertex_count, .indices = idx,
                      .index_count = 3, .object_id = 1, .vertex_format = &fmt};
  MopMesh *m = mop_viewport_add_mesh_ex(vp, &md);
  int rc = -1;
  if (m) {
    if (target_count && targets && weights)
      mop_mesh_set_morph_targets(m, vp, targets, weights, target_count);
    if (bone_count && bones)
      mop_mesh_set_bone_matrices(m, vp, (const MopMat4 *)bones, bone_count);
    mop_viewport_render(vp);
    const void *raw = vp->rhi->buffer_read(m->vertex_buffer);
    if (raw) {
      memcpy(out, raw, (size_t)vertex_count * 44u);
      rc = 0;
    }
  }
  mop_viewport_destroy(vp);
  return rc;
}
