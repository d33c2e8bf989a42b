/*
 * ref_harness.h — test-only driver for the reference library's CPU backend.
 *
 * This is oracle infrastructure: it builds a viewport through the reference's
 * public scene API (include/mop/core/viewport.h, scene.h, light.h,
 * environment.h), renders with MOP_BACKEND_CPU, and copies out the buffers a
 * parity test compares.  It is compiled together with the unmodified
 * reference sources into oracle/_ref/libmopref.so by oracle/Makefile.
 *
 * All structs are plain C so that ctypes (tests/, bench.py cpu leg) can bind
 * them without headers.
 */
#ifndef MOP_REF_HARNESS_H
#define MOP_REF_HARNESS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct RefMesh {
  const float *vertices;    /* vertex_count * 12 floats, MopVertex layout   */
  uint32_t vertex_count;
  const uint32_t *indices;
  uint32_t index_count;
  uint32_t object_id;
  float transform[16];      /* column-major world matrix                   */
  float metallic;
  float roughness;
  int32_t has_material;     /* 0: reference defaults (metallic 0, rough .5) */
  int32_t texture;          /* index into RefScene textures, -1 = none      */
  float opacity;
  int32_t blend_mode;       /* > 0: mop_mesh_set_blend_mode before opacity  */
} RefMesh;

/* mop_viewport_add_instanced_mesh (reference viewport.c:3774-3858): one
 * object ID, the default material, no texture; drawn by pass_instanced after
 * the transparent pass with mvp = P * (V * instance) per instance. */
typedef struct RefInstanced {
  const float *vertices;    /* vertex_count * 12 floats, MopVertex layout   */
  uint32_t vertex_count;
  const uint32_t *indices;
  uint32_t index_count;
  uint32_t object_id;
  const float *transforms;  /* instance_count column-major matrices         */
  uint32_t instance_count;
} RefInstanced;

typedef struct RefLight {
  int32_t type;             /* 0 directional, 1 point, 2 spot              */
  float position[3];
  float direction[3];
  float color[4];
  float intensity;
  float range;
  float spot_inner_cos;
  float spot_outer_cos;
  int32_t active;
  int32_t cast_shadows;     /* MopLight.cast_shadows                         */
} RefLight;

typedef struct RefScene {
  int32_t width, height, ssaa;
  float clear_color[4];
  float eye[3], target[3], up[3];
  float fov_deg, near_plane, far_plane;
  float ambient;
  float exposure;
  uint32_t post_effects;
  uint32_t mesh_count;
  const RefMesh *meshes;
  uint32_t texture_count;
  const int32_t *tex_w;
  const int32_t *tex_h;
  const uint8_t *const *tex_data;
  uint32_t light_count;
  const RefLight *lights;
  int32_t env;              /* 0: gradient (no IBL), 1: procedural sky IBL */
  float sun_dir[3];
  float turbidity, ground_albedo;
  float env_rotation, env_intensity;
  int32_t serial;           /* 1: null the tile thread pool (serial path)  */
  int32_t flat;             /* 1: MOP_SHADING_FLAT for the viewport        */
  int32_t workers;          /* >0: replace the tile pool with this many
                               worker threads (default: nproc-1)           */
  int32_t backend;          /* 0: MOP_BACKEND_CPU; 4: the CUDA backend
                               (only in the drop-in harness library)       */
  int32_t fog_on;           /* 1: mop_viewport_set_fog with the values below */
  float fog_color[4];
  float fog_near, fog_far;
  uint32_t instanced_count;
  const RefInstanced *instanced;
  /* per texture: MopTexFormat (0 RGBA8, 1 BC1, 2 BC3, 3 BC5) and the byte
   * size of tex_data[t]; NULL: every texture is RGBA8.  Compressed textures
   * are made with mop_tex_create (texture_create_ex). */
  const int32_t *tex_format;
  const uint32_t *tex_bytes;
  /* 1: the viewport renders into a host texture (MopViewportDesc
   * render_target, made through a helper viewport of the same backend);
   * refh_read_target reads it back */
  int32_t render_target;
  int32_t env_background;   /* 1: mop_viewport_set_environment_background */
  int32_t wireframe;        /* 1: mop_viewport_set_render_mode(WIREFRAME)
                               without the core's hidden grid mesh (with the
                               chrome off it is a zero-opacity blended mesh,
                               which wireframe mode draws as lines); 2: with
                               it */
} RefScene;

typedef struct RefFrame {
  uint8_t *color;           /* presented RGBA8, W*H*4 (after SSAA box)     */
  uint8_t *color_full;      /* optional sample-res RGBA8 (may be NULL)     */
  float *depth;             /* sample-res float                             */
  uint32_t *object_id;      /* sample-res uint32                            */
  float view[16];
  float proj[16];
  float eye[3];
  uint32_t triangle_count;  /* MopFrameStats.triangle_count                 */
  double frame_ms;          /* MopFrameStats.frame_time_ms                  */
} RefFrame;

void *refh_create(const RefScene *scene);
int refh_render(void *h, RefFrame *out);
int refh_pick(void *h, int n, const int32_t *xy, uint32_t *ids, float *depths,
              int32_t *hits);
int refh_env_maps(void *h, const float **irr, int32_t *iw, int32_t *ih,
                  const float **pf, int32_t *pw, int32_t *ph, int32_t *levels,
                  const float **brdf, int32_t *brdf_size);
/* mop_scene_save of the harness's viewport (flags: MOP_SAVE_QUANTIZE = 1). */
int refh_scene_save(void *h, const char *path, uint32_t flags);
/* mop_scene_load + mop_scene_get_mesh(idx): the decoded vertices (12 floats
 * each) and 32-bit indices, and the section's bbox (min, max). */
int refh_scene_file_mesh(const char *path, uint32_t idx, float *vertices, uint32_t vcap,
                         uint32_t *indices, uint32_t icap, uint32_t *vc, uint32_t *ic,
                         float bbox[6]);
/* Median ms of mop_scene_load + mop_scene_get_mesh of every mesh + frees. */
double refh_time_scene_file(const char *path, int reps);
/* The environment map the maps were computed from (the generated sky for
 * env == 1): RGBA32F, w x h. */
int refh_env_hdr(void *h, const float **hdr, int32_t *w, int32_t *hh);
/* Median wall time (ms) of render + read_color over `frames` after `warm`. */
double refh_time_frames(void *h, int warm, int frames);
/* Median ms of mop_viewport_set_environment with the scene's procedural sky
 * (sky generation + the three IBL precomputes, serial on the host). */
double refh_time_environment(void *h, int reps);
int refh_num_threads(void *h);
/* The backend's texture_create_ex + texture_read_rgba8 of one image (backend
 * 0: the CPU backend; 4 in the drop-in library: the CUDA backend): the
 * decoded RGBA8 texels in out (w * h * 4).  0 on success. */
int refh_bc_decode(int backend, int format, int w, int h, const uint8_t *data, uint32_t size,
                   uint8_t *out);
/* mop_viewport_present_to_texture into a new RGBA8 texture of tw x th, read
 * back with mop_tex_read_rgba8.  Returns 1 when the present succeeded, 0 when
 * the core refused it, negative on a harness error. */
int refh_present_to_texture(void *h, int tw, int th, uint8_t *out);
/* The render target's pixels after the last frame (render_target scenes). */
int refh_read_target(void *h, uint8_t *out);
void refh_destroy(void *h);

/* Deformation probe: one mesh of vertex layout position float3 @0, normal
 * float3 @12, joints ubyte4 @24, weights float4 @28 (stride 44) added with
 * mop_viewport_add_mesh_ex; bone matrices (mop_mesh_set_bone_matrices) and/or
 * morph targets (mop_mesh_set_morph_targets) set; one render on the CPU
 * backend; the vertex buffer the core uploaded is copied to out
 * (vertex_count * 44 bytes).  Returns 0 on success. */
int refh_deform_probe(const uint8_t *vertices, uint32_t vertex_count, const float *bones,
                      uint32_t bone_count, const float *targets, const float *weights,
                      uint32_t target_count, uint8_t *out);

#ifdef __cplusplus
}
#endif
#endif
