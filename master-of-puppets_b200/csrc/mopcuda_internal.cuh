/*
 * mopcuda_internal.cuh — device records and exact-arithmetic helpers.
 *
 * All kernels are compiled with -fmad=false -prec-div=true -prec-sqrt=true
 * -ftz=false: every float expression below is evaluated as the sequence of
 * IEEE single-precision round-to-nearest operations written, in the same
 * order as the reference CPU rasteriser (ISO C11, scalar SSE2, no
 * contraction).  That is what makes depth, coverage and object IDs
 * bit-exact and colour bit-exact except where a transcendental (atan2f,
 * asinf in the IBL lookups) differs between CUDA and glibc.
 */
#ifndef MOPCUDA_INTERNAL_CUH
#define MOPCUDA_INTERNAL_CUH

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "fold.h"

/* ------------------------------------------------------------------------
 * frame records
 * ------------------------------------------------------------------------ */

enum DrawFlags : uint32_t {
  DF_SMOOTH = 1u << 0,
  DF_CULL = 1u << 1,
  DF_LIT = 1u << 2,     /* light list present: _full entry (rasterizer.c:2458) */
  DF_TEXTURED = 1u << 3,
  DF_FLEX = 1u << 4,    /* flexible vertex layout                              */
  /* depth_test && !depth_write: the CPU backend saves the depth buffer before
   * the draw and restores it after (cpu_backend.c:536-544, 575-580), so the
   * draw's fragments test against the depth before it and each other, and
   * its colour and IDs stay while its depth does not */
  DF_NO_DEPTH_WRITE = 1u << 5,
  /* !depth_test: every covered fragment passes (rasterizer.c:1948) and
   * writes depth */
  DF_NO_DEPTH_TEST = 1u << 6,
  /* scene draws of a batch: blended, translucent or unlit smooth — the draw
   * starts its viewport's ordered suffix (set by the host) */
  DF_ORDERED = 1u << 7,
  /* wireframe: the triangle's three edges as anti-aliased lines in its flat
   * colour (rasterizer.c:1225-1235, 743-871); part of the ordered suffix */
  DF_WIRE = 1u << 8,
};

/* One recorded draw, uploaded per frame (the MopRhiDrawCall fields the path
 * reads, plus where its vertices/triangles land in the frame arrays). */
struct DrawRec {
  float mvp[16];
  float model[16];
  float light_dir[3];
  float ambient;
  float opacity;
  float metallic;
  float roughness;
  float depth_bias;
  float cam_eye[3];
  uint32_t object_id;
  const uint8_t *vbuf;     /* device vertex bytes                        */
  const uint32_t *ibuf;    /* device indices                             */
  const uint8_t *tex;      /* device RGBA8 or null                       */
  int32_t tex_w, tex_h;
  uint32_t vertex_count, index_count;
  uint32_t vbase;          /* first slot in the frame vertex arrays      */
  uint32_t tbase;          /* first global triangle index                */
  uint32_t light_off, light_count;
  uint32_t flags;
  uint32_t stride;
  int16_t off_pos, off_nrm, off_col, off_uv; /* -1 = absent             */
  int8_t n_pos, n_nrm, n_col, n_uv;          /* component counts         */
  /* per-draw shading constants, computed on the host with the same
   * operations the reference repeats per pixel (rasterizer.c:1712-1727,
   * 2000, 2030-2032): alpha^2 (clamped), Smith k, 1-k, 0.04(1-m), 1-m */
  float alpha2, smith_k, one_minus_k, f0_dielectric, diffuse_scale;
  /* per-draw IBL lookups (rasterizer.c:243-291): prefiltered mip chosen by
   * roughness (offset in texels, size) and the BRDF LUT row */
  uint32_t pf_off;
  int32_t pf_lw, pf_lh, brdf_row;
  int32_t blend_mode; /* MopBlendMode: 0 opaque, 1 alpha, 2 additive, 3 multiply */
};

struct LightRec {
  int32_t type;
  float position[3];
  float direction[3];
  float color[4];
  float intensity;
  float range;
  float spot_inner_cos;
  float spot_outer_cos;
  int32_t active;
  float ndir[3]; /* mop_vec3_normalize(direction), computed once per frame */
};

/* Per fan-triangle raster record, 64 bytes. */
struct __align__(16) RasterRec {
  float w0[3];      /* edge values at the clamped bbox corner (x0+.5, y0+.5) */
  float dx[3];      /* per-pixel increments                                  */
  float dy[3];      /* per-row increments                                    */
  float zc[3];      /* smooth: sz0..2 ; flat: z_row0, z_dx, z_dy             */
  float inv_area;
  uint32_t order;   /* (triangle << ORDER_FAN_BITS) | fan: submission order  */
  uint16_t x0, y0, x1, y1; /* inclusive clamped bbox; y1 bit 15 = flat       */
};

#define ORDER_FAN_BITS 5
#define REC_FLAT_BIT 0x8000u
/* Record slot t belongs to triangle t.  A clipped triangle's slot holds this
 * marker in y0 and, in `order`, the slot of its first fan record in the
 * overflow region that starts at slot total_tris. */
#define REC_REDIRECT 0xffffu
/* A wireframe triangle's record: x1 holds this marker (no filled raster
 * kernel takes it: its box is empty), w0/dx/dy hold the screen x, y and z of
 * its three vertices. */
#define REC_WIRE_X1 0x8000u
/* Fragment payloads of wireframe frames: bit 31 set marks a line plot, the
 * rest its item index (the frame's triangle count stays below 2^26, so
 * triangle orders keep bit 31 clear). */
#define FRAG_WIRE_BIT 0x80000000u

/* Per fan-triangle shading record, 16 bytes. */
struct __align__(16) ShadeRec {
  union {
    uint32_t v[3];  /* smooth: frame vertex slots of the fan vertices        */
    float col[3];   /* flat: constant colour                                 */
  };
  uint32_t draw;
};

/* Frame counters and error flags, zeroed at frame start. */
struct alignas(8) Counters {
  uint32_t rec_count;         /* fan records of clipped triangles (overflow region) */
  uint32_t extra_vertices;
  /* one 64-bit counter: low word the items of the large records pushed so far
   * (their list offsets, ascending with the list index), high word the number
   * of large records (rasterised as (row, chunk) items); 8-byte aligned */
  uint32_t large_items;
  uint32_t large_count;
  uint32_t clip_count;
  uint32_t overflow;          /* bit0 records, bit1 extra vertices, bit2 clip
                                 queue, bit3 large list, bit9 large-record
                                 items past 2^32                               */
  uint32_t shade_count;       /* covered samples queued for shading              */
  /* ordered (blended) suffix of the frame; overflow bit4 fragment pool,
   * bit5 ordered-record list, bit7 wireframe-record list */
  uint32_t frag_count, touched_count, olist_count, olist_items;
  uint32_t wire_count, wire_items; /* wireframe records queued, their plots */
  uint32_t scratch_count;          /* sort-scratch entries taken by long lists */
  uint32_t pad[2];
};
/* arrays of counters (one per viewport) keep the 64-bit pair aligned */
static_assert(sizeof(Counters) % 8 == 0 && offsetof(Counters, large_items) % 8 == 0,
              "large-record counter pair must be 8-byte aligned");

/* Blended fragments of one sample sorted in registers; a sample with more
 * sorts its list in the fold's global scratch (heapsort). */
#define ORDERED_MAX_FRAGS 48

/* Records whose clamped bbox exceeds these bounds are rasterised as
 * (row, RASTER_CHUNK-sample) items spread over many threads; smaller ones
 * by one thread each. */
#define SMALL_MAX_SIDE 32  /* default small-record limits */
#define SMALL_MAX_AREA 128
#define RASTER_CHUNK 32

struct FrameArgs {
  const DrawRec *draws;
  uint32_t draw_count;
  const LightRec *lights;
  uint32_t light_total;   /* records in `lights` (all draws of the frame) */
  uint32_t total_vertices;
  uint32_t total_tris;
  /* vertex streams (total_vertices + extra capacity) */
  float4 *clip;
  float4 *world;
  float4 *normal;
  float4 *color;
  uint32_t vertex_cap;
  /* records: slot t = triangle t, then the clipped fans' overflow region */
  RasterRec *rrec;
  ShadeRec *srec;
  uint32_t rec_cap;  /* total slots: total_tris + overflow capacity */
  uint32_t *clipq;
  uint32_t clip_cap;
  /* visibility */
  int width, height;                /* sample resolution */
  unsigned long long *keys;         /* per sample: depth_key << 32 | order */
  unsigned long long *keys_next;    /* the next frame's key buffer, cleared by k_shade
                                       (null: none) */
  uint32_t *large_list;             /* record ids of large records */
  uint32_t *large_items;            /* offset of each one's first item (ascending) */
  uint32_t large_cap;
  uint32_t *shade_list;             /* covered sample indices */
  Counters *ctr;
  /* resolve */
  float clear[4];
  float exposure;
  /* IBL */
  const float *irr;
  int irr_w, irr_h;
  const float *pf;
  int pf_w, pf_h, pf_levels;
  const float *brdf;
  int brdf_size;
  float ibl_rotation, ibl_intensity;
  /* outputs */
  uchar4 *pre;     /* resolved RGBA8 before post effects */
  float *depth;
  uint32_t *ids;
  /* small-record limits: bbox side and area (larger records are rasterised
   * item-parallel) */
  int small_side, small_area;
  /* visibility only: shading writes depth and IDs but no colour */
  int no_color;
  /* ordered suffix: triangles t >= t_split (a blended draw and everything
   * after it) are composited per sample in submission order instead of
   * entering the visibility keys; hdr != null when the frame has one */
  uint32_t t_split;
  float4 *hdr;            /* per sample: the opaque pass's colour before ACES */
  uint32_t *frag_head;    /* per sample: first fragment, 0xffffffff = none      */
  uint2 *frags;           /* fragment: (next, order)                            */
  uint32_t frag_cap;
  uint32_t *touched;      /* samples that received a fragment                   */
  uint32_t *olist;        /* live records of the suffix                          */
  uint32_t *olist_items;  /* their (row, chunk) item counts, then offsets        */
  uint32_t olist_cap;
  /* environment background (pass_background_hdri_cpu): every uncovered
   * sample shows the RGBA32F environment (sky_w x sky_h) along the ray
   * sky_fwd + sky_right * ndc_x * sky_half_w + sky_up * ndc_y * sky_half_h,
   * times sky_intensity; null: the clear colour */
  const float4 *sky;
  int sky_w, sky_h;
  float sky_fwd[3], sky_right[3], sky_up[3];
  float sky_half_w, sky_half_h, sky_rotation, sky_intensity;
  /* the suffix holds a depth-test-off draw: its fragments pass whatever the
   * depth, and later ones may pass where the opaque depth is nearer, so
   * every covered fragment of the suffix is kept */
  int ordered_keep_all;
  /* wireframe records in the suffix: their queue and plot counts (then
   * offsets); wire != 0 when the frame has wireframe draws */
  uint32_t *wlist, *wlist_items;
  uint32_t wlist_cap;
  int wire;
  /* sort scratch of the fold for lists longer than ORDERED_MAX_FRAGS:
   * (key, payload) pairs, oscratch_cap entries (at least the fragment pool,
   * so it cannot run out), taken from *oscratch_count */
  ulonglong2 *oscratch;
  uint32_t *oscratch_count;
  uint32_t oscratch_cap;
  /* shadow map bound for directional lights (the rasteriser's shadow state,
   * rasterizer.c:141-157): shadow_w x shadow_h texel keys (shadow_texel),
   * null when none is bound; shadow_vp: the light's view-projection, 16
   * floats in device memory */
  const uint32_t *shadow_keys;
  const float *shadow_vp;
  int shadow_w, shadow_h;
};

/* ------------------------------------------------------------------------
 * shadow pass: depth-only raster of the casters from the light
 * (mop_sw_shadow_render_mesh, rasterizer.c:357-493)
 * ------------------------------------------------------------------------ */
/* One caster mesh; its triangles are [tri_off, tri_off + tri_count) of the
 * pass.  Positions are float3 at offset 0 of each `stride`-byte vertex. */
struct ShadowDraw {
  const uint8_t *verts;
  const uint32_t *idx;
  uint32_t vertex_count, stride, tri_count, tri_off;
  float mvp[16]; /* light view-projection * model (mop_mat4_multiply, on the host) */
};

/* A triangle whose bbox exceeds SHADOW_SMALL_AREA, rasterised by
 * 32-row bands (narrow bboxes) or rows (wide ones); 64 bytes. */
struct __align__(16) ShadowRec {
  float w[3];  /* edge values at (x0 + .5, y0 + .5), winding already flipped */
  float dx[3]; /* per-texel increments */
  float dy[3]; /* per-row increments   */
  float sz[3]; /* window depth of the three vertices */
  float inv_area;
  uint32_t x0y0, x1y1; /* bbox corners, x | y << 16 */
  uint32_t pad;
};

struct ShadowCounters {
  uint32_t recs;           /* large records written */
  uint32_t pad;
  unsigned long long items; /* band / row items of all large records */
};

/* Caster bboxes of at most this many texels are walked by their triangle's
 * thread; larger ones go to the warp-per-chunk raster. */
#define SHADOW_SMALL_AREA 32
/* Large casters up to this bbox width are walked a 32-row band per warp
 * (one row per lane); wider ones a row per warp (one chunk per lane). */
#define SHADOW_SEG 128

struct ShadowArgs {
  const ShadowDraw *draws;
  uint32_t draw_count, tri_total;
  uint32_t *map; /* size x size keys; 0xffffffff (cleared) = depth 1.0 */
  int size;
  int small_area;
  ShadowRec *recs;            /* capacity tri_total */
  unsigned long long *items;  /* per record: item count, then exclusive offsets */
  ShadowCounters *ctr;
  int num_sms;
};

/* Rasterises the pass into s.map (already cleared, counters zeroed); returns
 * the number of kernels launched. */
int mopcuda_launch_shadow(const ShadowArgs &s, cudaStream_t st);

struct PostArgs {
  const uchar4 *pre;
  uchar4 *out;        /* sample-res after post */
  uchar4 *presented;  /* (w/ssaa) x (h/ssaa) or null */
  int width, height, ssaa;
  uint32_t effects;
  float lut[256];     /* per-byte value after tonemap/gamma */
  uint8_t lut8[256];  /* the whole per-channel map when vignette is off */
  /* fog (FOG bit): each sample's depth value moves its colour towards
   * fog_color by clamp((depth - fog_near) / fog_range, 0, 1) */
  const float *depth;
  float fog_color[3];
  float fog_near, fog_range;
  /* gamma_thr[k]: the smallest float whose sRGB value rounds to byte k + 1
   * (host glibc powf); the byte of any value is the count of entries <= it */
  float gamma_thr[255];
};

/* ------------------------------------------------------------------------
 * exact helpers
 * ------------------------------------------------------------------------ */

/* float -> int as the x86-64 reference build converts (cvttss2si):
 * truncation, and INT_MIN for NaN or out-of-range values. */
__device__ __forceinline__ int x86_f2i(float f) {
  if (!(f >= -2147483648.0f && f < 2147483648.0f))
    return (int)0x80000000;
  return (int)f;
}

/* float -> uint8_t through int32 truncation, keeping the low byte. */
__device__ __forceinline__ uint8_t x86_f2u8(float f) { return (uint8_t)(uint32_t)x86_f2i(f); }

/* Order-preserving map of a depth value to 32 bits; -0 and +0 share a key
 * (they compare equal under the reference's strict `<` test). */
__device__ __forceinline__ uint32_t depth_key(float z) {
  uint32_t b = __float_as_uint(z);
  if ((b & 0x7fffffffu) == 0u)
    b = 0u;
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

#define KEY_EMPTY 0xffffffffffffffffull

/* launchers (kernels.cu); each returns the number of kernels it launched */
/* Launch shapes of the frame kernels (chosen by the autotuner). */
struct LaunchCfg {
  int num_sms;
  int small_side, small_area; /* FrameArgs::small_side / small_area */
  int raster_block;   /* threads per block of the small-record raster     */
  int shade_block;    /* threads per block of the shading kernel          */
  int shade_waves;    /* resident blocks per SM targeted by shading       */
  int post_bx, post_by;
};

/* Byte layout of a deformed vertex: stride and offsets (-1: no normal). */
struct DeformLayout {
  uint32_t stride;
  int32_t position_offset, normal_offset, joints_offset, weights_offset;
};

/* Skinning / morph of vc vertices from bind into dst (device pointers). */
int mopcuda_launch_skin(const uint8_t *bind, uint8_t *dst, uint32_t vc, const DeformLayout &l,
                        const float *bones, uint32_t bone_count, int num_sms, cudaStream_t s);
int mopcuda_launch_morph(const uint8_t *bind, uint8_t *dst, uint32_t vc, const DeformLayout &l,
                         const float *targets, const float *weights, uint32_t tc, int num_sms,
                         cudaStream_t s);

/* ------------------------------------------------------------------------
 * batched viewports over one resident scene
 * ------------------------------------------------------------------------ */
#define MOPCUDA_MAX_VIEWS 256

/* One viewport of a batch: its camera, sample resolution and where its
 * sample- and pixel-resolution buffers start in the batch pools. */
struct ViewRec {
  float view[16], proj[16];
  float eye[3];
  float clear[4];
  int width, height; /* sample resolution */
  int ssaa;
  uint32_t scene;    /* index into BatchArgs::scenes */
  uint32_t no_color; /* visibility only (picks): depth and IDs, no shading */
  uint32_t pad;
  unsigned long long sample_off; /* keys, shade list, pre, out, depth, ids */
  unsigned long long pixel_off;  /* presented */
  unsigned long long draw_off;   /* first of the scene's nd slots in view_draws */
};

/* One resident scene of a batch: its draw table for this launch, bounds,
 * lights and IBL maps. */
struct SceneDesc {
  const DrawRec *draws; /* mvp, cam_eye, vbase and tbase unused */
  const struct DrawBound *bounds;
  uint32_t nd;
  uint32_t light_total;
  const LightRec *lights;
  const float *irr, *pf, *brdf;
  int irr_w, irr_h, pf_w, pf_h, pf_levels, brdf_size;
  float ibl_rotation, ibl_intensity;
  /* the scene's shadow map for this launch (null: none): size x size keys,
   * then the light's view-projection */
  const uint32_t *shadow_keys;
  const float *shadow_vp;
  int shadow_size;
};

/* Mesh-local bounding sphere of a draw's vertices; r < 0 (or NaN) means the
 * draw is never culled. */
struct DrawBound {
  float c[3];
  float r;
};

/* Pool sizes that the allocation pass found too small; the host grows the
 * pools to at least these and re-runs the batch. */
struct BatchStatus {
  uint32_t overflow; /* pools: bit0 vertex, bit1 records, bit2 clip queue, bit3 large
                        list, bit4 ordered-record lists, bit5 fragments, bit6 wireframe-
                        record lists; bit8 a viewport with an ordered suffix or wireframe
                        draws in a launch without the buffers for them */
  uint32_t scratch_count; /* the fold's sort scratch, shared by the viewports */
  unsigned long long need_vertex, need_rec, need_clip, need_large, need_olist, need_frag,
      need_wlist;
};

/* Blended draws of one scene a batch viewport sorts back to front. */
#define BATCH_MAX_BLENDED 1024

struct BatchArgs {
  const SceneDesc *scenes;
  const ViewRec *views;
  uint32_t nv;
  FrameArgs *frames;   /* nv, filled by k_batch_prepare / k_batch_alloc */
  DrawRec *view_draws; /* per viewport its scene's nd slots: the visible draws */
  Counters *ctr;       /* nv */
  BatchStatus *status;
  FrameArgs tmpl;      /* exposure and small-record limits */
  /* pools (per-viewport ranges assigned on the device) */
  float4 *clip, *world, *normal, *color;
  unsigned long long vertex_pool;
  RasterRec *rrec;
  ShadeRec *srec;
  unsigned long long rec_pool;
  uint32_t *clipq;
  unsigned long long clip_pool;
  uint32_t *large_list, *large_items;
  unsigned long long large_pool;
  unsigned long long *keys;
  uint32_t *shade_list;
  uchar4 *pre;
  float *depth;
  uint32_t *ids;
  /* ordered suffix (null when no scene of the launch has one): per-sample
   * composition buffers at the viewports' sample offsets, and pools of
   * fragments and suffix-record lists carved per viewport */
  float4 *hdr;
  uint32_t *frag_head, *touched;
  uint2 *frags;
  unsigned long long frag_pool;
  uint32_t *olist, *olist_items;
  unsigned long long olist_pool;
  uint32_t *wlist, *wlist_items; /* wireframe-record lists (null: no wireframe draws) */
  unsigned long long wlist_pool;
  ulonglong2 *oscratch;          /* the fold's sort scratch, frag_pool entries, shared */
  uint32_t *oscratch_count;      /* by the launch's viewports through one counter */
  unsigned long long samples; /* samples of the launch (frag_head's length) */
  /* per-viewport reserves: clipped fans (records, extra vertices, clip
   * queue) T * fan_num / 8 + 1024; large list T * large_num / 16 + 1024;
   * fragments S * frag_num / 4 + 4096 */
  uint32_t fan_num, large_num, frag_num;
};

/* Per-stage launch shape of a batch (the autotuner's search space). */
struct BatchLaunch {
  int num_sms;
  int vertex_block, setup_block, raster_block, large_block, shade_block;
  int grid_mul; /* persistent grids: resident blocks per SM x grid_mul */
  /* filled by mopcuda_batch_grids (occupancy queries, before any capture) */
  int grid_vertex, grid_setup, grid_clip, grid_rsmall, grid_rlarge, grid_shade;
};

/* Computes the persistent grid sizes of cfg from the kernels' occupancy. */
void mopcuda_batch_grids(BatchLaunch &cfg);

/* Launches the device part of one batch on stream s: prepare, allocate,
 * vertex, setup, clip, raster, resolve, shade and post (the caller clears
 * counters and keys first).  post_views[k] lists the viewports with ssaa
 * k+1 (device array, post_count[k] entries); posts holds each viewport's
 * PostArgs.  Returns the number of kernels launched. */
/* parts: which of the launch to enqueue, BATCH_PART_MAIN (uploads done by
 * the caller, then every stage up to shading) and/or BATCH_PART_POST (the
 * post passes, which write the colour images). */
#define BATCH_PART_MAIN 1
#define BATCH_PART_POST 2
/* ordered: the launch has suffix buffers (b.hdr): the suffix kernels run
 * after shading for the viewports that have a suffix. */
int mopcuda_launch_batch(const BatchArgs &b, const PostArgs *posts, const uint32_t *post_views[4],
                         const uint32_t post_count[4], const uint32_t post_tiles[4],
                         const BatchLaunch &cfg, bool shared_lights, bool shadows, bool ordered,
                         cudaStream_t s, int parts = BATCH_PART_MAIN | BATCH_PART_POST);

/* ev (optional, 7 events): stage boundaries
 * vertex | setup+clip | raster | resolve | shade | post */
/* before_post (optional): called on the host once the kernels up to shading
 * are queued, before the post pass is; returns an event the post pass waits
 * for (the readback of the image it overwrites), or null. */
typedef cudaEvent_t (*PrePostHook)(void *ctx);
int mopcuda_launch_frame(const FrameArgs &a, const PostArgs &p, const LaunchCfg &cfg,
                         cudaStream_t s, cudaEvent_t *ev, PrePostHook before_post = nullptr,
                         void *hook_ctx = nullptr);
int mopcuda_launch_fp32_peak(float *out, int blocks, int iters, cudaStream_t s);
#define MOPCUDA_STAGES 6
int mopcuda_launch_box(const uchar4 *src, int width, int height, int sf, uchar4 *dst,
                       cudaStream_t s);
int mopcuda_launch_pick(const uint32_t *ids, const float *depth, int width, int height, int sf,
                        const int2 *xy, uint32_t n, uint32_t *out_id, float *out_depth,
                        int32_t *out_hit, cudaStream_t s);
int mopcuda_shade_occupancy(int block);

#endif
