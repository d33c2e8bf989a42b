/*
 * mop_cuda.h — C ABI of the B200 (sm_100a) backend for the Master of Puppets
 * software-rasterizer frame path.
 *
 * Every entry point takes plain pointers, sizes and POD structs; nothing in
 * this header depends on CUDA, C++ or the reference's headers, so it can be
 * bound from C, ctypes or any FFI.  The entry points replace, one for one,
 * the reference's RHI function table entries (src/rhi/rhi.h:132-339) as
 * implemented by its CPU backend (src/backend/cpu/cpu_backend.c); the
 * reference-typed table itself is produced by mop_rhi_backend_cuda() in
 * master-of-puppets_b200/host/mop_rhi_cuda.c on top of these calls.
 *
 * Execution model.  Draws are recorded on the host between frame_begin and
 * frame_end; frame_end runs the whole frame on the device as a fixed
 * sequence of kernels: vertex transform, triangle setup + clipping,
 * rasterisation of every triangle record into a per-sample visibility key
 * (64-bit atomicMin on depth|submission order), resolve of the background and
 * compaction of covered samples, deferred shading with the ACES resolve, then
 * FXAA + gamma + SSAA box.  Results are order-independent and deterministic;
 * object IDs and depth are bit-exact to the reference CPU backend.  Batches
 * and the server (further down) run the same kernels over many viewports.
 *
 * Errors: create calls return NULL; int-returning calls return MOPCUDA_OK
 * (0) or a negative MOPCUDA_E* code; mopcuda_last_error() gives text.
 */
#ifndef MOP_CUDA_H
#define MOP_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MOPCUDA_OK 0
#define MOPCUDA_EINVAL (-1)       /* bad argument                              */
#define MOPCUDA_ENOMEM (-2)       /* device or pinned-host allocation failed   */
#define MOPCUDA_ECUDA (-3)        /* CUDA runtime error                        */
#define MOPCUDA_ETIMEOUT (-4)     /* bounded wait expired (device lost)        */
#define MOPCUDA_EUNSUPPORTED (-5) /* draw state outside the supported path     */

/* post-effect bits (reference include/mop/render/postprocess.h:20-33) */
#define MOPCUDA_POST_GAMMA (1u << 0)
#define MOPCUDA_POST_TONEMAP (1u << 1)
#define MOPCUDA_POST_VIGNETTE (1u << 2)
#define MOPCUDA_POST_FOG (1u << 3)
#define MOPCUDA_POST_FXAA (1u << 4)

typedef struct MopCudaDevice MopCudaDevice;
typedef struct MopCudaBuffer MopCudaBuffer;
typedef struct MopCudaTexture MopCudaTexture;
typedef struct MopCudaFramebuffer MopCudaFramebuffer;

/* Light record; same fields and meaning as MopLight
 * (reference include/mop/core/light.h:37-60). */
typedef struct MopCudaLight {
  int32_t type; /* 0 directional, 1 point, 2 spot */
  float position[3];
  float direction[3];
  float color[4];
  float intensity;
  float range;
  float spot_inner_cos;
  float spot_outer_cos;
  int32_t active;
} MopCudaLight;

/* Flexible vertex layout (reference include/mop/core/vertex_format.h:70):
 * byte offsets of each attribute inside a vertex of `stride` bytes, or -1
 * when absent (normal defaults to (0,1,0), colour to white, uv to 0). */
typedef struct MopCudaVertexLayout {
  uint32_t stride;
  int32_t position_offset;
  int32_t position_components; /* 1..4 */
  int32_t normal_offset;
  int32_t normal_components;
  int32_t color_offset;
  int32_t color_components;
  int32_t uv_offset;
  int32_t uv_components;
} MopCudaVertexLayout;

/* One draw; the fields of MopRhiDrawCall (reference src/rhi/rhi.h:51-110)
 * that the frame path reads.  Matrices are column-major d[col*4+row]. */
typedef struct MopCudaDraw {
  MopCudaBuffer *vertex_buffer;
  MopCudaBuffer *index_buffer;
  uint32_t vertex_count;
  uint32_t index_count;
  uint32_t object_id;
  float model[16];
  float mvp[16];
  float light_dir[3];
  float ambient;
  float opacity;
  float metallic;
  float roughness;
  float depth_bias;
  float cam_eye[3];
  int32_t smooth;        /* MOP_SHADING_SMOOTH                              */
  int32_t wireframe;     /* the triangles' edges as anti-aliased lines       */
  int32_t depth_test;
  int32_t depth_write;
  int32_t backface_cull;
  int32_t blend_mode;    /* MopBlendMode                                    */
  MopCudaTexture *texture;
  const MopCudaLight *lights; /* copied at draw time; NULL = no light list  */
  uint32_t light_count;
  const MopCudaVertexLayout *layout; /* NULL = 48-byte MopVertex           */
} MopCudaDraw;

/* ---- device lifecycle: MopRhiBackend.device_create/destroy (rhi.h:136-137),
 *      cpu_device_create cpu_backend.c:55-75 ---------------------------- */
MopCudaDevice *mopcuda_device_create(int cuda_ordinal);
void mopcuda_device_destroy(MopCudaDevice *dev);
const char *mopcuda_last_error(void);
/* Number of kernel launches issued by this device since creation. */
uint64_t mopcuda_launch_count(const MopCudaDevice *dev);

/* ---- buffers: buffer_create/destroy/update/read (rhi.h:140-143, 230-237),
 *      cpu_backend.c:87-115, 663-667, 1077-1080 ------------------------- */
MopCudaBuffer *mopcuda_buffer_create(MopCudaDevice *dev, const void *data, size_t size);
void mopcuda_buffer_destroy(MopCudaDevice *dev, MopCudaBuffer *buf);
int mopcuda_buffer_update(MopCudaDevice *dev, MopCudaBuffer *buf, const void *data,
                          size_t offset, size_t size);
/* Host shadow of the buffer contents (the core reads vertex data back). */
const void *mopcuda_buffer_read(const MopCudaBuffer *buf);
/* The device bytes [offset, offset + size) of a buffer (no reference
 * counterpart: the device copy, for buffers made on the device without a
 * host copy). */
int mopcuda_buffer_copy_to_host(MopCudaDevice *dev, const MopCudaBuffer *buf, size_t offset,
                                void *dst, size_t size);
size_t mopcuda_buffer_size(const MopCudaBuffer *buf);

/* ---- textures: texture_create/_hdr/destroy (rhi.h:197-211),
 *      cpu_backend.c:811-853, 1064-1072 --------------------------------- */
MopCudaTexture *mopcuda_texture_create(MopCudaDevice *dev, int width, int height,
                                       const uint8_t *rgba);
MopCudaTexture *mopcuda_texture_create_hdr(MopCudaDevice *dev, int width, int height,
                                           const float *rgba);
void mopcuda_texture_destroy(MopCudaDevice *dev, MopCudaTexture *tex);
int mopcuda_texture_read_rgba8(MopCudaDevice *dev, MopCudaTexture *tex, uint8_t *out,
                               size_t out_size);
/* texture_create_ex (rhi.h:211-213), cpu_texture_create_ex
 * (cpu_backend.c:1016-1056): format 0 is RGBA8 (mopcuda_texture_create);
 * 1 BC1, 2 BC3, 3 BC5 (MopTexFormat, texture_pipeline.h:35-41) are copied to
 * the device as stored and decoded there to RGBA8 exactly as
 * bc_decompress_to_rgba8 does (cpu_backend.c:855-1014); BC7 (4) returns NULL
 * with MOPCUDA_EUNSUPPORTED, as the CPU backend refuses it.  mip_levels is
 * ignored (level 0 only, as the CPU backend).  A non-zero data_size smaller
 * than the dimensions imply is refused (the reference would read past it). */
MopCudaTexture *mopcuda_texture_create_ex(MopCudaDevice *dev, int width, int height, int format,
                                          int mip_levels, const uint8_t *data, size_t data_size);

/* ---- framebuffers: framebuffer_create/destroy/resize (rhi.h:146-151),
 *      cpu_backend.c:121-188 ------------------------------------------- */
MopCudaFramebuffer *mopcuda_framebuffer_create(MopCudaDevice *dev, int width, int height);
void mopcuda_framebuffer_destroy(MopCudaDevice *dev, MopCudaFramebuffer *fb);
int mopcuda_framebuffer_resize(MopCudaDevice *dev, MopCudaFramebuffer *fb, int width,
                               int height);
/* Presentation (SSAA) factor of the framebuffer, as the viewport allocates
 * (width*ssaa) x (height*ssaa) samples (reference viewport.c:552-577).  When
 * set, frame_end fuses the box resolve of mop_viewport_read_color
 * (viewport.c:3385-3411) into its post pass. */
int mopcuda_framebuffer_set_ssaa(MopCudaFramebuffer *fb, int ssaa);
/* framebuffer_copy_to_texture (rhi.h:320-321), cpu_framebuffer_copy_to_texture
 * (cpu_backend.c:741-790): the last frame's post-processed colour into an
 * RGBA8 texture of the same size, or of a whole-number factor smaller on both
 * axes (box of sf x sf samples, truncating mean); any other size is refused
 * (MOPCUDA_EINVAL).  Waits for the frame; the texture's device copy (used by
 * later draws) and host copy (mopcuda_texture_read_rgba8) are both updated. */
int mopcuda_framebuffer_copy_to_texture(MopCudaDevice *dev, MopCudaFramebuffer *fb,
                                        MopCudaTexture *target);
/* framebuffer_create_from_texture (rhi.h:155-157),
 * cpu_framebuffer_create_from_texture (cpu_backend.c:143-170): a framebuffer
 * of the texture's size whose every completed frame lands in the texture
 * (the CPU backend rasterises into the texture's pixels; here each frame's
 * colour is copied in when it completes).  NULL for a size mismatch or an
 * HDR texture.  The texture must outlive the framebuffer. */
MopCudaFramebuffer *mopcuda_framebuffer_create_from_texture(MopCudaDevice *dev,
                                                           MopCudaTexture *color, int width,
                                                           int height);

/* ---- vertex deformation: the core's mop_skin_apply / mop_morph_apply
 *      (reference src/core/viewport.c:1572-1680, 1763-1804) on the device.
 *      The core keeps the bind pose and morph targets in backend buffers and
 *      calls these instead of deforming on the host and re-uploading; dst's
 *      host shadow (mopcuda_buffer_read) is refreshed, as the core reads
 *      deformed vertices back for bounds. ------------------------------- */
typedef struct MopCudaDeformLayout {
  uint32_t stride;         /* bytes per vertex, multiple of 4                */
  int32_t position_offset; /* float3                                         */
  int32_t normal_offset;   /* float3, -1 when absent                         */
  int32_t joints_offset;   /* ubyte4 bone indices (skinning only)            */
  int32_t weights_offset;  /* float4 bone weights (skinning only)            */
} MopCudaDeformLayout;
/* dst = bind pose with positions (and normals, renormalised) skinned by up
 * to 4 weighted bones each; bones: bone_count column-major 4x4 (host). */
int mopcuda_skin_apply(MopCudaDevice *dev, MopCudaBuffer *dst, const MopCudaBuffer *bind,
                       uint32_t vertex_count, const MopCudaDeformLayout *layout,
                       const float *bones, uint32_t bone_count);
/* dst = bind pose with positions += weight_t * delta_t over the targets in
 * order (zero weights skipped); targets: target_count x vertex_count x 3
 * floats in a device buffer; weights: host array. */
int mopcuda_morph_apply(MopCudaDevice *dev, MopCudaBuffer *dst, const MopCudaBuffer *bind,
                        uint32_t vertex_count, const MopCudaDeformLayout *layout,
                        const MopCudaBuffer *targets, const float *weights,
                        uint32_t target_count);

/* ---- frame state ------------------------------------------------------ */
/* set_exposure (rhi.h:244): exposure for the ACES resolve
 * (reference mop_sw_hdr_resolve, rasterizer.c:2776). */
void mopcuda_set_exposure(MopCudaDevice *dev, float exposure);
/* Post-effect bits applied after the resolve (mop_postprocess_apply,
 * postprocess.c:24); default GAMMA|FXAA as the viewport sets it.  FOG,
 * TONEMAP, GAMMA and VIGNETTE run per sample in the reference's order; the
 * other bits (bloom, SSAO, ...) belong to GPU effect hooks the CPU path
 * ignores, and are ignored here too. */
void mopcuda_set_post_effects(MopCudaDevice *dev, uint32_t effects);
/* mop_viewport_set_fog (postprocess.c:170-175): the MopFogParams the FOG bit
 * uses (colour RGBA, only RGB read; near and far distances compared with each
 * sample's depth value, postprocess.c:51-65).  A device starts with all zero,
 * as a new viewport does: factor 0, colours unchanged.  Returns EINVAL for a
 * null device or colour. */
int mopcuda_set_fog(MopCudaDevice *dev, const float color[4], float near_dist, float far_dist);
/* IBL maps, as mop_sw_ibl_set (rasterizer.h:212-215): irradiance RGBA32F
 * iw x ih, prefiltered RGBA32F mip chain concatenated (levels), BRDF LUT
 * RGBA32F size x size.  Copied to the device.  NULL irradiance clears. */
int mopcuda_set_ibl(MopCudaDevice *dev, const float *irradiance, int iw, int ih,
                    const float *prefiltered, int pw, int ph, int levels,
                    const float *brdf_lut, int brdf_size, float rotation, float intensity);

/* ---- IBL precompute on the device (environment.c:111-484, 493-620)
 *
 * ibl_from_env computes from an RGBA32F equirectangular environment (w x h,
 * what the core loads for MOP_ENV_HDRI) the maps precompute_irradiance,
 * precompute_prefiltered and precompute_brdf_lut make — irradiance 64x32,
 * prefiltered 128x64 in 5 levels, BRDF LUT 256x256 — and binds them as
 * mopcuda_set_ibl does; ibl_procedural_sky first generates the 512x256
 * Preetham sky of generate_procedural_sky (MOP_ENV_PROCEDURAL_SKY) on the
 * device.  The BRDF LUT is bit-exact; the sky and the two environment
 * convolutions use CUDA's atan2f/asinf/acosf/cosf/expf per sample, so they
 * agree with the core's to float rounding. */
int mopcuda_ibl_from_env(MopCudaDevice *dev, const float *env_rgba, int w, int h, float rotation,
                         float intensity);
int mopcuda_ibl_procedural_sky(MopCudaDevice *dev, const float sun_direction[3], float turbidity,
                               float ground_albedo, float rotation, float intensity);
/* Device time of the last precompute (table upload, sky, three maps). */
float mopcuda_ibl_gpu_time_ms(MopCudaDevice *dev);
/* Copies of the bound maps (any pointer may be NULL); env is the
 * environment the last precompute read (the generated sky included). */
int mopcuda_ibl_read(MopCudaDevice *dev, float *irradiance, size_t irradiance_bytes,
                     float *prefiltered, size_t prefiltered_bytes, float *brdf_lut,
                     size_t brdf_lut_bytes, float *env, size_t env_bytes);

/* ---- .mop v2 scene files straight to device memory (reference
 *      src/loader/mop_scene.c, include/mop/loader/mop_scene.h)
 *
 * scene_file_open maps the file and checks it as mop_scene_load does (magic
 * 0x4D4F5002, version 2, at most 256 sections, the table of contents inside
 * the file); NULL on failure.  The counts and the camera are
 * mop_scene_mesh_count / _light_count / _get_camera; scene_file_light reads
 * light section idx (no reference getter).  scene_file_upload_mesh is
 * mop_scene_get_mesh into device buffers: the section's stored bytes
 * (quantized 18-byte or raw 48-byte vertices, 16- or 32-bit indices) cross
 * PCIe as they are and are decoded on the device into MopVertex and 32-bit
 * index buffers byte-identical to mop_scene_get_mesh's arrays.  With
 * MOPCUDA_LOAD_HOST_SHADOW the buffers also keep the host copy
 * mopcuda_buffer_read returns (the core reads vertices back); otherwise
 * mopcuda_buffer_read returns NULL for them. */
typedef struct MopCudaSceneFile MopCudaSceneFile;
#define MOPCUDA_LOAD_HOST_SHADOW 1u
MopCudaSceneFile *mopcuda_scene_file_open(const char *path);
void mopcuda_scene_file_close(MopCudaSceneFile *file);
uint32_t mopcuda_scene_file_mesh_count(const MopCudaSceneFile *file);
uint32_t mopcuda_scene_file_light_count(const MopCudaSceneFile *file);
int mopcuda_scene_file_camera(const MopCudaSceneFile *file, float eye[3], float target[3],
                              float up[3], float *fov_radians, float *near_plane,
                              float *far_plane);
int mopcuda_scene_file_light(const MopCudaSceneFile *file, uint32_t idx, MopCudaLight *out);
int mopcuda_scene_file_upload_mesh(MopCudaDevice *dev, const MopCudaSceneFile *file, uint32_t idx,
                                   uint32_t flags, MopCudaBuffer **vertices,
                                   MopCudaBuffer **indices, uint32_t *vertex_count,
                                   uint32_t *index_count, float bbox_min[3], float bbox_max[3]);
/* Every mesh of the file in one pass: one host-to-device copy of all stored
 * mesh sections, one decode launch for the vertices and one for the
 * indices, the buffers carved from one device allocation (each still
 * released with mopcuda_buffer_destroy; the allocation goes with the last).
 * vertices / indices receive mesh_count handles; the count arrays may be
 * NULL. */
int mopcuda_scene_file_upload_all(MopCudaDevice *dev, const MopCudaSceneFile *file, uint32_t flags,
                                  MopCudaBuffer **vertices, MopCudaBuffer **indices,
                                  uint32_t *vertex_counts, uint32_t *index_counts);

/* ---- shadow map (pass_shadow, viewport.c:2288-2442, which the core runs
 *      for its CPU backend only; mop_sw_shadow_render_mesh,
 *      rasterizer.c:357-493; mop_sw_shadow_set / _clear, rasterizer.c:146-157)
 *
 * shadow_begin opens a pass of a size x size depth map (the core uses 1024)
 * for the light view-projection light_vp; shadow_draw adds one caster (the
 * core passes every active opaque mesh below the chrome IDs, in mesh order:
 * its vertex buffer with positions as float3 at offset 0 of each `stride`-
 * byte vertex, 48 for MopVertex, its index buffer and world transform);
 * shadow_end rasterises the casters on the device stream and binds the map
 * for this device's later frames, where every directional light's diffuse
 * and specular terms take the 3x3 PCF factor (rasterizer.c:303-348,
 * 1580-1583, 1677-1680, 1802-1805) until shadow_clear.  A frame keeps the
 * map bound at its frame_end; two maps alternate, so a pass recorded while
 * that frame runs does not wait for it. */
int mopcuda_shadow_begin(MopCudaDevice *dev, int size, const float light_vp[16]);
int mopcuda_shadow_draw(MopCudaDevice *dev, const MopCudaBuffer *vertices, uint32_t vertex_count,
                        uint32_t stride, const MopCudaBuffer *indices, uint32_t index_count,
                        const float model[16]);
/* n casters in array order, exactly as n shadow_draw calls (no reference
 * counterpart: for hosts that keep their casters in an array; stops at the
 * first caster that fails). */
typedef struct MopCudaShadowCaster {
  const MopCudaBuffer *vertices;
  uint32_t vertex_count;
  uint32_t stride;
  const MopCudaBuffer *indices;
  uint32_t index_count;
  float model[16];
} MopCudaShadowCaster;
int mopcuda_shadow_draw_list(MopCudaDevice *dev, const MopCudaShadowCaster *casters, uint32_t n);
int mopcuda_shadow_end(MopCudaDevice *dev);
int mopcuda_shadow_clear(MopCudaDevice *dev);
/* Device time of the last shadow pass (map clear + raster), waiting for it
 * (bounded); 0 before the first pass (no reference counterpart). */
float mopcuda_shadow_gpu_time_ms(MopCudaDevice *dev);
/* The bound map as depth values (size * size floats, row-major). */
int mopcuda_shadow_read(MopCudaDevice *dev, float *depth, size_t bytes);

/* ---- frame commands: frame_begin/end/submit, draw, draw_instanced
 *      (rhi.h:160-175, 214-218), cpu_backend.c:197-211, 528-657 -------- */
int mopcuda_frame_begin(MopCudaDevice *dev, MopCudaFramebuffer *fb, const float clear_rgba[4]);
int mopcuda_draw(MopCudaDevice *dev, MopCudaFramebuffer *fb, const MopCudaDraw *draw);
/* n draws in array order, exactly as n mopcuda_draw calls (no reference
 * counterpart: a convenience for hosts that keep their draw calls in an
 * array; stops at the first draw that fails). */
int mopcuda_draw_list(MopCudaDevice *dev, MopCudaFramebuffer *fb, const MopCudaDraw *draws,
                      uint32_t n);
/* The environment background of the frame being recorded
 * (pass_background_hdri_cpu, reference viewport.c:2128-2177, which the core
 * runs on the CPU backend for an HDRI or procedural-sky environment with
 * mop_viewport_set_environment_background on): every sample the draws leave
 * uncovered shows the RGBA32F environment texture `env` (equirectangular)
 * along the ray through the sample, times intensity, resolved as background
 * (no ACES); blended draws composite over it.  eye/target/up/fov_deg are the
 * camera as the viewport holds it for the frame (after its orbit update); the
 * ray setup (forward, right, up, tan of half the fov) is the core's, computed
 * with the same float operations.  Call between frame_begin and frame_end. */
int mopcuda_draw_background(MopCudaDevice *dev, MopCudaFramebuffer *fb,
                            const MopCudaTexture *env, const float eye[3], const float target[3],
                            const float up[3], float fov_deg, float rotation, float intensity);
/* draw_skybox (rhi.h:285-293): the same background from the inverse
 * view-projection and camera position the core hands GPU backends
 * (viewport.c:2209-2218); the ray setup is recovered from the far-plane
 * points at ndc (0,0), (1,0), (0,1), so rays match the core's to float
 * rounding rather than bit for bit. */
int mopcuda_draw_skybox(MopCudaDevice *dev, MopCudaFramebuffer *fb, const MopCudaTexture *env,
                        const float inv_vp[16], const float cam_pos[3], float rotation,
                        float intensity);
/* view/projection multiply per instance as cpu_draw_instanced does
 * (mvp = P * (V * instance), cpu_backend.c:638-657). */
int mopcuda_draw_instanced(MopCudaDevice *dev, MopCudaFramebuffer *fb, const MopCudaDraw *draw,
                           const float *view, const float *projection,
                           const float *instance_models, uint32_t instance_count);
/* Launch the recorded frame (asynchronous; returns after enqueueing). */
int mopcuda_frame_end(MopCudaDevice *dev, MopCudaFramebuffer *fb);
/* Bounded wait for the last launched frame; MOPCUDA_ETIMEOUT after
 * timeout_ms, with the frame still pending: a later wait (or any call that
 * completes the frame first) resumes waiting for it.  A device error
 * (MOPCUDA_ECUDA) ends the frame with its result undefined. */
int mopcuda_frame_wait(MopCudaDevice *dev, int timeout_ms);
/* Device time of the last completed frame (frame_gpu_time_ms, rhi.h:240). */
float mopcuda_frame_gpu_time_ms(MopCudaDevice *dev);

/* ---- readbacks (rhi.h:177-195), cpu_backend.c:673-735.  Returned pointers
 *      are pinned host mirrors owned by the framebuffer, valid until the next
 *      frame, resize or destroy; the caller may write through them. ----- */
const uint8_t *mopcuda_read_color(MopCudaDevice *dev, MopCudaFramebuffer *fb, int *w, int *h);
const uint32_t *mopcuda_read_object_id(MopCudaDevice *dev, MopCudaFramebuffer *fb, int *w,
                                       int *h);
const float *mopcuda_read_depth(MopCudaDevice *dev, MopCudaFramebuffer *fb, int *w, int *h);
/* SSAA box resolve on the device (mop_viewport_read_color,
 * viewport.c:3385-3411) into a caller buffer of (w/ssaa)*(h/ssaa)*4 bytes. */
int mopcuda_read_color_resolved(MopCudaDevice *dev, MopCudaFramebuffer *fb, int ssaa,
                                uint8_t *out, size_t out_size);
/* The same image, read asynchronously (no reference counterpart): the copy
 * into `out` (page-locked memory for a true overlap, mopcuda_host_alloc)
 * starts on a separate copy stream when the frame completes, queued inside
 * the next frame's launch when mopcuda_frame_end follows, and overlaps that
 * frame's work; ssaa must be 1 or the framebuffer's presentation
 * factor.  mopcuda_readback_wait returns once the framebuffer's last
 * requested image is in host memory (it completes the frame first when it
 * is still pending). */
int mopcuda_read_color_resolved_async(MopCudaDevice *dev, MopCudaFramebuffer *fb, int ssaa,
                                      void *out, size_t out_size);
int mopcuda_readback_wait(MopCudaDevice *dev, MopCudaFramebuffer *fb, int timeout_ms);
uint32_t mopcuda_pick_read_id(MopCudaDevice *dev, MopCudaFramebuffer *fb, int x, int y);
float mopcuda_pick_read_depth(MopCudaDevice *dev, MopCudaFramebuffer *fb, int x, int y);
/* Batched pick at presentation pixels (mop_viewport_pick, viewport.c:3687):
 * xy[2n]; outputs ids/depths/hits per query; out-of-range -> (0, 1.0, 0). */
int mopcuda_pick_batch(MopCudaDevice *dev, MopCudaFramebuffer *fb, int ssaa, const int32_t *xy,
                       uint32_t n, uint32_t *ids, float *depths, int32_t *hits);

/* Same results as mopcuda_pick_batch, for callers that cannot allocate at
 * call time (a fixed memory budget with their own allocator, a thread that
 * must not call cudaMalloc/cudaFree because they synchronise the device, an
 * embedder that forbids allocation after start-up).  No counterpart in the
 * reference: its CPU picks read host arrays directly.
 *
 * Nothing is allocated: queries and results are staged in one file-scope
 * device array of MOPCUDA_NOALLOC_PICK_MAX * 20 bytes (1.25 MiB) that every
 * GPU loading the library holds until the process exits.  More than
 * MOPCUDA_NOALLOC_PICK_MAX queries are rejected with MOPCUDA_EINVAL.  xy and
 * the outputs are host memory.  The frame must be complete
 * (mopcuda_frame_wait) — completing it here could reallocate.  The first
 * call on a device resolves the array's device address; make it before any
 * stream capture.  All calls share the array (it keeps the last call's
 * contents): calls that overlap on the GPU race.  The results are copied
 * straight into the caller's arrays, so the 20 s wait bounds the call only
 * when ids, depths and hits are page-locked (mopcuda_host_alloc): a copy
 * into pageable memory holds the host until the pick kernel ends.  After
 * MOPCUDA_ETIMEOUT the copies are still queued: xy and the outputs stay in
 * use until the device is synchronised or destroyed. */
#define MOPCUDA_NOALLOC_PICK_MAX 65536u
int mopcuda_pick_batch_noalloc(MopCudaDevice *dev, MopCudaFramebuffer *fb, int ssaa,
                               const int32_t *xy, uint32_t n, uint32_t *ids, float *depths,
                               int32_t *hits);

/* ---- measurement (no reference counterpart: the reference reports only
 *      wall-clock MopFrameStats, include/mop/util/profile.h:51-81) ------- */
/* Record CUDA events between the frame's stages on the device stream. */
void mopcuda_set_stage_timing(MopCudaDevice *dev, int on);
/* Stage durations of the last completed frame, ms: [0] vertex transform,
 * [1] triangle setup + clipping, [2] visibility raster, [3] resolve of
 * background + compaction, [4] deferred shading + ACES, [5] post (FXAA,
 * gamma, SSAA).  `ms` holds >= 6 floats. */
int mopcuda_stage_times(MopCudaDevice *dev, float *ms, int n);
/* Measured FP32 add/multiply issue rate without FMA, Gop/s: the roofline
 * denominator of the shading stage. */
int mopcuda_measure_fp32_peak(MopCudaDevice *dev, double *gops);
/* Host->device and device->host bytes of the last frame launch itself (draw
 * table + light records up; frame counters down), excluding readbacks. */
int mopcuda_frame_io_bytes(MopCudaDevice *dev, uint64_t *h2d, uint64_t *d2h);

/* ---- batched viewports over a resident scene ---------------------------
 * No counterpart in the reference, which renders one viewport per
 * mop_viewport_render (viewport.c:2990-3320).  A scene holds draws recorded
 * once (buffers, textures, materials, model matrices, lights); a batch binds
 * a scene to N viewports of their own size, camera and SSAA factor and
 * renders all of them with one CUDA graph launch.  Every viewport's colour,
 * depth and object IDs equal what a frame of the same draws through
 * mopcuda_frame_begin/draw/frame_end gives (draws wholly outside a
 * viewport's frustum are skipped; they contribute nothing there).  Exposure,
 * post effects and IBL are the device's at mopcuda_batch_create. */
typedef struct MopCudaScene MopCudaScene;
typedef struct MopCudaBatch MopCudaBatch;

typedef struct MopCudaView {
  float view[16];  /* column-major, as mopcuda_camera_matrices returns */
  float proj[16];
  float eye[3];
  int width, height; /* presented size; the samples are width*ssaa x height*ssaa */
  int ssaa;          /* 1..4 */
  float clear[4];
} MopCudaView;

MopCudaScene *mopcuda_scene_create(MopCudaDevice *dev);
/* The scene's shadow pass, as pass_shadow runs it for the frame
 * (viewport.c:2288-2442): with size > 0, every launch that renders the scene
 * first rasterises its casters (every opaque draw below the editor-chrome
 * IDs, with the model matrices the launch renders) into a size x size depth map
 * from the light camera mopcuda_shadow_light_vp derives for `direction` (the
 * first active directional light with cast_shadows), and its viewports'
 * directional lights take the 3x3 PCF factor as in a plain frame.  size 0
 * turns it off.  Each scene entry of a server launch (a scene as of the
 * requests' submission) gets its own map. */
int mopcuda_scene_set_shadow(MopCudaScene *scene, int size, const float direction[3]);
void mopcuda_scene_destroy(MopCudaScene *scene);
/* Appends a draw (its mvp and cam_eye are ignored: each viewport supplies
 * them).  Same state rules and errors as mopcuda_draw.  Draws go in mesh
 * order; each viewport renders the non-blended ones in that order, then the
 * blended ones (blend_mode != 0) back to front by the squared distance of
 * their model translation to its eye (pass_scene_opaque /
 * pass_scene_transparent, viewport.c:2449-2553).  Refused
 * (MOPCUDA_EUNSUPPORTED): draws with the depth test or the depth write off,
 * a 1,025th blended draw, and wireframe draws in a scene of 2^26 or more
 * triangles.  Returns the draw's index (>= 0) or an error code. */
int mopcuda_scene_add_draw(MopCudaScene *scene, const MopCudaDraw *draw);
/* Replaces draw `index`'s model matrix (TRS update); effective from the next
 * batch submit. */
int mopcuda_scene_set_model(MopCudaScene *scene, uint32_t index, const float model[16]);
uint32_t mopcuda_scene_draw_count(const MopCudaScene *scene);
/* Triangles submitted by the scene's draws (each viewport processes its
 * visible subset). */
uint64_t mopcuda_scene_triangle_count(const MopCudaScene *scene);

/* n in 1..256.  Device memory for every viewport's buffers is allocated
 * here; the work pools grow on demand (a submit that overflows them is
 * re-run after growing). */
MopCudaBatch *mopcuda_batch_create(MopCudaScene *scene, const MopCudaView *views, uint32_t n);
void mopcuda_batch_destroy(MopCudaBatch *batch);
/* New cameras/clear colours for the same viewport sizes and SSAA factors. */
int mopcuda_batch_set_views(MopCudaBatch *batch, const MopCudaView *views, uint32_t n);
/* Launches the batch (asynchronous); waits for the previous one first. */
int mopcuda_batch_submit(MopCudaBatch *batch);
/* Bounded wait for the submitted batch, re-running it if its pools grew. */
int mopcuda_batch_wait(MopCudaBatch *batch, int timeout_ms);
/* Device time of the last completed batch launch, ms. */
float mopcuda_batch_gpu_time_ms(const MopCudaBatch *batch);
/* Copies one viewport's result into host memory: what = 0 colour at sample
 * resolution after post effects (RGBA8), 1 presented colour (SSAA box
 * resolve; = 0 when ssaa is 1), 2 depth (f32, samples), 3 object IDs (u32,
 * samples).  bytes must equal the buffer's size. */
#define MOPCUDA_BATCH_COLOR 0
#define MOPCUDA_BATCH_PRESENTED 1
#define MOPCUDA_BATCH_DEPTH 2
#define MOPCUDA_BATCH_IDS 3
int mopcuda_batch_read(MopCudaBatch *batch, uint32_t view, int what, void *dst, size_t bytes);
/* The same buffer of views first .. first+count-1 in one call: dsts[i] and
 * bytes[i] for view first+i, every size checked before any copy, one wait
 * for all the copies. */
int mopcuda_batch_read_views(MopCudaBatch *batch, uint32_t first, uint32_t count, int what,
                             void *const *dsts, const size_t *bytes);
/* Asynchronous form for the colour buffers (MOPCUDA_BATCH_COLOR or
 * _PRESENTED) of the last submitted launch, which it waits for: the copies
 * are queued once the next submit has queued its stages up to shading, and
 * run while that launch renders (its post passes, which rewrite the images,
 * wait for them); without a next submit, readback_wait queues them.  dsts
 * stay the caller's and should be page-locked; the copies are complete when
 * mopcuda_batch_readback_wait returns 0. */
int mopcuda_batch_read_views_async(MopCudaBatch *batch, uint32_t first, uint32_t count, int what,
                                   void *const *dsts, const size_t *bytes);
int mopcuda_batch_readback_wait(MopCudaBatch *batch, int timeout_ms);
/* Picks on viewport `view` (presented coordinates, top-left sample), as
 * mopcuda_pick_batch. */
int mopcuda_batch_pick(MopCudaBatch *batch, uint32_t view, const int32_t *xy, uint32_t n,
                       uint32_t *ids, float *depths, int32_t *hits);

/* Launch shape of a batch: the small-record limits of the raster (bbox
 * side, area), block sizes of the vertex / setup / small-raster /
 * large-raster / shading stages and the persistent-grid multiplier. */
typedef struct MopCudaBatchConfig {
  int small_side, small_area;
  int vertex_block, setup_block, raster_block, large_block, shade_block;
  int grid_mul;
} MopCudaBatchConfig;
int mopcuda_batch_get_config(const MopCudaBatch *batch, MopCudaBatchConfig *cfg);
/* Validates and applies cfg (the graph is rebuilt at the next submit). */
int mopcuda_batch_set_config(MopCudaBatch *batch, const MopCudaBatchConfig *cfg);
/* Autotuner: coordinate search over MopCudaBatchConfig, timing `reps`
 * launches of the batch per candidate with CUDA events; applies the fastest
 * and writes a one-line JSON report (candidates and their ms) to report
 * (may be NULL).  Results do not depend on the configuration. */
int mopcuda_batch_autotune(MopCudaBatch *batch, int reps, char *report, size_t report_len);
/* Bytes of device memory the batch holds (buffers + pools). */
uint64_t mopcuda_batch_device_bytes(const MopCudaBatch *batch);

/* ---- serving -----------------------------------------------------------
 * No counterpart in the reference (it renders on the caller's thread).  A
 * server keeps scenes resident and serves render and pick requests from any
 * thread with continuous batching: one worker admits queued requests in
 * arrival order while the estimated device bytes of the work in flight stay
 * within hbm_budget and a launch slot is free, fuses up to max_views of
 * them (any mix of scenes) into one launch on the slot's stream, and keeps
 * admitting new arrivals into the next free slot while earlier launches
 * run.  A request larger than the budget runs alone.  Results equal the
 * request's own frame (mopcuda_frame_* of the same draws and camera),
 * whatever it was batched with.  Scenes added to a server take no further
 * draws (mopcuda_scene_add_draw fails) until the server is destroyed; model
 * matrices may change at any time and a request renders them as they were
 * when it was submitted. */
typedef struct MopCudaServer MopCudaServer;

typedef struct MopCudaServerConfig {
  uint64_t hbm_budget;      /* bytes of in-flight work (framebuffers + pools) */
  uint32_t max_views;       /* requests fused into one launch, 1..256 */
  uint32_t max_inflight;    /* launches on the device at once, 1..16 */
  uint32_t batch_window_us; /* after a launch, wait this long for more arrivals */
  uint64_t max_launch_samples; /* samples of one launch at most (a larger request still runs,
                                  alone); 0 = no limit.  Smaller launches finish sooner and
                                  shorten the latency tail at some cost in throughput */
} MopCudaServerConfig;

#define MOPCUDA_REQ_RENDER 0u
#define MOPCUDA_REQ_PICK 1u

typedef struct MopCudaRequest {
  uint32_t kind;  /* MOPCUDA_REQ_RENDER or MOPCUDA_REQ_PICK */
  uint32_t scene; /* id from mopcuda_server_add_scene */
  MopCudaView view;
  /* RENDER: presented RGBA8 (width*height*4 bytes) and optionally the
   * sample-resolution object IDs and depth; NULL skips a buffer.  The
   * memory must stay valid until mopcuda_server_wait returns.  Page-locked
   * buffers (mopcuda_host_alloc) receive the device copy directly; others
   * are staged and copied by the server's worker thread. */
  uint8_t *color;
  uint32_t *ids;
  float *depth;
  /* PICK: pick_n presented-pixel coordinates (copied at submit) and their
   * results, as mopcuda_pick_batch.  The view is rendered for visibility
   * only (no shading). */
  const int32_t *pick_xy;
  uint32_t pick_n;
  uint32_t *pick_ids;
  float *pick_depths;
  int32_t *pick_hits;
} MopCudaRequest;

typedef struct MopCudaServerStats {
  uint64_t submitted, completed, failed;
  uint64_t launches, launched_views, reruns;
  uint64_t peak_inflight_bytes; /* estimated bytes admitted at once */
  uint64_t device_bytes;        /* device memory the launch slots hold now */
  uint32_t max_views_in_launch;
  uint32_t pad;
} MopCudaServerStats;

MopCudaServer *mopcuda_server_create(MopCudaDevice *dev, const MopCudaServerConfig *cfg);
/* Finishes the queued work, then frees the server (not its scenes). */
void mopcuda_server_destroy(MopCudaServer *srv);
/* Returns the scene's id (>= 0) or an error code. */
int mopcuda_server_add_scene(MopCudaServer *srv, MopCudaScene *scene);
int mopcuda_server_submit(MopCudaServer *srv, const MopCudaRequest *req, uint64_t *ticket);
/* Waits up to timeout_ms (0 polls) for a request; on completion returns its
 * status, writes the arrival-to-result latency and forgets the ticket.
 * MOPCUDA_ETIMEOUT: still queued or running. */
int mopcuda_server_wait(MopCudaServer *srv, uint64_t ticket, int timeout_ms, double *latency_ms);
/* Waits until nothing is queued or running. */
int mopcuda_server_drain(MopCudaServer *srv, int timeout_ms);
int mopcuda_server_stats(MopCudaServer *srv, MopCudaServerStats *stats);
/* Page-locked host memory (cudaMallocHost) for request buffers. */
void *mopcuda_host_alloc(size_t bytes);
void mopcuda_host_free(void *p);

/* ---- host-side matrices (the device receives finished matrices) ------- */
/* out = a * b, column-major (mop_mat4_multiply, reference math.c:182-194). */
void mopcuda_mat4_multiply(const float a[16], const float b[16], float out[16]);
/* T * Rz * Ry * Rx * S (mop_mat4_compose_trs, math.c:205-215). */
void mopcuda_mat4_compose_trs(const float position[3], const float rotation[3],
                              const float scale[3], float out[16]);
/* View/projection/eye of a frame after mop_viewport_set_camera: the orbit
 * camera re-derives eye and up each render (viewport.c:1058-1128,
 * camera.c:35-63).  width/height are the presentation size. */
void mopcuda_camera_matrices(const float eye[3], const float target[3], const float up[3],
                             float fov_deg, float near_plane, float far_plane, int width,
                             int height, float view[16], float proj[16], float eye_out[3]);
/* The eye and up vector a frame uses for a camera set with eye/target/up:
 * the orbit parameters mop_viewport_set_camera stores (viewport.c:1079-1091)
 * re-applied as mop_viewport_render does (what mopcuda_draw_background wants
 * when the caller has no viewport core). */
void mopcuda_camera_orbit(const float eye[3], const float target[3], const float up[3],
                          float eye_out[3], float up_out[3]);
/* The shadow pass's light view-projection (viewport.c:2303-2427): a scene
 * box from the casters' world transforms (translation +- 1.5 x the largest
 * column length), an orthographic light camera looking along `direction`
 * from twice the box radius.  Returns 0 (and leaves light_vp alone) when
 * count is 0, 1 otherwise. */
int mopcuda_shadow_light_vp(const float *models, uint32_t count, const float direction[3],
                            float light_vp[16]);

#ifdef __cplusplus
}
#endif
#endif
