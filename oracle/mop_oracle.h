/*
 * mop_oracle.h — plain-C restatement of the reference CPU frame path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA backend is compared
 * against; nothing in the product links it.  It restates, serially and in the
 * reference's float evaluation order, the path
 *   cpu_draw (reference src/backend/cpu/cpu_backend.c:528-629)
 *   -> mop_sw_rasterize_triangle_full / mop_sw_rasterize_triangle
 *      (src/rasterizer/rasterizer.c:2458-2612, 1093-1242)
 *   -> smooth multi-light / flat / legacy smooth rasterisers
 *   -> mop_sw_hdr_resolve (rasterizer.c:2776-2803)
 *   -> mop_postprocess_apply (src/render/postprocess.c:24-116)
 *   -> mop_viewport_read_color SSAA box (src/core/viewport.c:3364-3418)
 *   -> mop_viewport_pick (viewport.c:3687-3749)
 * and the camera chain that produces the view/projection matrices
 * (viewport.c:1058-1130, src/interact/camera.c:35-63, src/math/math.c).
 *
 * Parity is pinned against the reference library itself (oracle/_ref, built
 * from the reference sources by oracle/Makefile) on seeded scenes, and against
 * golden fixtures committed under tests/golden/.
 */
#ifndef MOP_ORACLE_H
#define MOP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrLight {
  int32_t type; /* 0 directional, 1 point, 2 spot */
  float position[3];
  float direction[3];
  float color[4];
  float intensity;
  float range;
  float spot_inner_cos;
  float spot_outer_cos;
  int32_t active;
} OrLight;

typedef struct OrDraw {
  const float *vertices; /* vertex_count * 12 floats (MopVertex) */
  uint32_t vertex_count;
  const uint32_t *indices;
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
  int32_t smooth;        /* MOP_SHADING_SMOOTH */
  int32_t depth_test;
  int32_t backface_cull;
  int32_t blend_mode;    /* MopBlendMode */
  const OrLight *lights; /* NULL / 0 = legacy single-light path */
  uint32_t light_count;
  const uint8_t *texture; /* RGBA8 or NULL */
  int32_t tex_w, tex_h;
  /* 0 with depth_test: the depth buffer is saved before the draw and restored
   * after it (cpu_backend.c:536-544, 621-627) */
  int32_t depth_write;
  /* MOP_RENDER_WIREFRAME on a non-zero ID: the triangle's three edges as
   * anti-aliased lines in its flat colour (rasterizer.c:1225-1235) */
  int32_t wireframe;
} OrDraw;

typedef struct OrIBL {
  const float *irr;
  int32_t irr_w, irr_h;
  const float *pf;
  int32_t pf_w, pf_h, pf_levels;
  const float *brdf;
  int32_t brdf_size;
  float rotation;
  float intensity;
} OrIBL;

/* A bound shadow map (mop_sw_shadow_set, reference rasterizer.c:146-151):
 * w x h depth values and the light's view-projection. */
typedef struct OrShadow {
  const float *depth;
  int32_t w, h;
  float vp[16];
} OrShadow;

/* The environment background (pass_background_hdri_cpu, reference
 * viewport.c:2128-2177): every sample's HDR colour before the draws is the
 * equirectangular environment (RGBA32F, w x h) seen along the ray through
 * the sample, times intensity.  The camera is the one mop_viewport_set_camera
 * took (the orbit re-derivation of the eye and up is applied here). */
typedef struct OrSky {
  const float *env;
  int32_t w, h;
  float rotation, intensity;
  float eye[3], target[3], up[3];
  float fov_deg;
} OrSky;

typedef struct OrFrame {
  int32_t width, height; /* sample resolution (presented * ssaa) */
  int32_t ssaa;
  float clear[4];
  float exposure;
  uint32_t post_effects;
  const OrIBL *ibl; /* NULL = no IBL maps bound */
  /* outputs (caller-allocated; NULL to skip) */
  uint8_t *color_full;      /* width*height*4, after resolve + post */
  float *depth;             /* width*height */
  uint32_t *object_id;      /* width*height */
  uint8_t *color_presented; /* (width/ssaa)*(height/ssaa)*4 */
  float *hdr;               /* width*height*4, before resolve */
  const OrShadow *shadow;   /* NULL = no shadow map bound */
  /* MopFogParams, applied when post_effects has MOP_POST_FOG (fog_on) */
  int32_t fog_on;
  float fog_color[4];
  float fog_near, fog_far;
  const OrSky *sky;         /* NULL = no environment background */
} OrFrame;

/* Render one frame of draws in submission order.  Returns 0 on success. */
int oracle_render(OrFrame *frame, const OrDraw *draws, uint32_t draw_count);

/* Camera chain: mop_viewport_set_camera followed by the orbit re-derivation
 * mop_viewport_render performs every frame.  width/height are the
 * presentation size (the projection aspect). */
void oracle_camera(const float eye[3], const float target[3], const float up[3],
                   float fov_deg, float near_plane, float far_plane, int width,
                   int height, float view[16], float proj[16],
                   float eye_out[3]);

/* c = a * b, column-major (mop_mat4_multiply, math.c:182-194). */
void oracle_mat4_multiply(const float a[16], const float b[16], float c[16]);

/* Pick at presentation pixels: ID/depth of the top-left sample of each
 * SSAA block (viewport.c:3687-3749, cpu_backend.c:673-687). */
void oracle_pick(const uint32_t *object_id, const float *depth, int width,
                 int height, int ssaa, int n, const int32_t *xy,
                 uint32_t *ids, float *depths, int32_t *hits);

/* sRGB gamma byte map used by the post-process (postprocess.c:75-82). */
void oracle_gamma_lut(uint8_t lut[256]);

/* One shadow caster: MopVertex array, indices, world transform. */
typedef struct OrShadowMesh {
  const float *vertices; /* vertex_count * 12 floats */
  uint32_t vertex_count;
  const uint32_t *indices;
  uint32_t index_count;
  float model[16];
} OrShadowMesh;

/* The light view-projection of pass_shadow (viewport.c:2303-2427) from the
 * casters' world transforms (count x 16 floats) and the light direction.
 * Returns 0 when count is 0. */
int oracle_shadow_matrix(const float *models, uint32_t count, const float dir[3],
                         float vp[16]);
/* The shadow map of pass_shadow: size x size cleared to 1.0 (viewport.c:
 * 2370-2373), then mop_sw_shadow_render_mesh (rasterizer.c:357-493) for
 * every caster in order. */
void oracle_shadow_render(const OrShadowMesh *meshes, uint32_t count, int size,
                          const float vp[16], float *depth);

/* mop_scene_get_mesh's decode of one .mop v2 mesh section (reference
 * src/loader/mop_scene.c:397-486, dequantize_vertex / oct_decode :142-223):
 * section points at the 48-byte section header; vertices receives
 * vertex_count x 12 floats, indices index_count words.  Returns 0, or -1
 * when the section is shorter than its counts. */
int oracle_mop_decode_mesh(const uint8_t *section, uint64_t size, float *vertices,
                           uint32_t *indices);

/* Vertex deformation the core runs before buffer_update: byte layout of one
 * vertex (stride; offsets of position float3, normal float3 or -1, joints
 * ubyte4, weights float4). */
typedef struct OrDeformLayout {
  uint32_t stride;
  int32_t position_offset, normal_offset, joints_offset, weights_offset;
} OrDeformLayout;

/* mop_skin_apply (reference src/core/viewport.c:1572-1680): dst = bind pose
 * with positions and normals skinned by the bone matrices (column-major). */
void oracle_skin_apply(const OrDeformLayout *l, const uint8_t *bind, uint32_t vertex_count,
                       const float *bones, uint32_t bone_count, uint8_t *dst);
/* mop_morph_apply (viewport.c:1763-1804): dst = bind pose with positions
 * plus the weighted deltas of every target (targets * vertices * 3 floats). */
void oracle_morph_apply(const OrDeformLayout *l, const uint8_t *bind, uint32_t vertex_count,
                        const float *targets, const float *weights, uint32_t target_count,
                        uint8_t *dst);

/* bc_decompress_to_rgba8 (reference src/backend/cpu/cpu_backend.c:855-1014):
 * a BC1 (format 1), BC3 (2) or BC5 (3) image of w x h texels, blocks in
 * row-major order, decoded to RGBA8 (out: w * h * 4 bytes).  Returns 0, or -1
 * for another format. */
int oracle_bc_decode(int format, int w, int h, const uint8_t *blocks, uint8_t *out);

#ifdef __cplusplus
}
#endif
#endif
