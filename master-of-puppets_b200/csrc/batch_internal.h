/*
 * batch_internal.h — resident scenes and the launch machinery shared by the
 * batch API (batch_api.cu) and the request server (server.cu).
 */
#ifndef MOPCUDA_BATCH_INTERNAL_H
#define MOPCUDA_BATCH_INTERNAL_H

#include "api_internal.h"

#include <memory>

struct MopCudaScene {
  MopCudaDevice *dev = nullptr;
  std::vector<DrawRec> draws; /* host records; mvp / cam_eye come per viewport */
  std::vector<LightRec> lights;
  std::vector<DrawBound> bounds;
  uint64_t tris = 0, verts = 0;
  uint64_t version = 0;     /* bumps when draws are added */
  uint64_t gen = 0;         /* bumps when a model matrix changes */
  std::shared_ptr<const std::vector<float>> models; /* models as of models_gen */
  uint64_t models_gen = ~0ull;
  bool frozen = false;      /* held by a server: no more draws */
  /* device copies of the immutable parts, uploaded when version changes */
  DevArena d_bounds, d_lights;
  uint64_t dev_version = ~0ull;
  /* IBL maps captured from the device at scene creation */
  DevArena irr, pf, brdf;
  bool ibl_on = false;
  int irr_w = 0, irr_h = 0, pf_w = 0, pf_h = 0, pf_levels = 0, brdf_size = 0;
  float ibl_rot = 0.0f, ibl_int = 1.0f;
  /* shadow pass (mopcuda_scene_set_shadow): map size (0: none) and the
   * directional light's direction */
  int sh_size = 0;
  float sh_dir[3] = {0.0f, 0.0f, 0.0f};
  /* order-dependent draws: blended ones (the core's transparent pass, sorted
   * per viewport) and the triangles of every DF_ORDERED draw */
  uint32_t blended = 0;
  uint64_t ordered_tris = 0;
  bool wire = false; /* has wireframe draws */
  std::mutex mu;
};

/* One scene entry's shadow pass in a launch: the map (texels, then the
 * light's view-projection), the caster table and the raster's work space. */
struct EntryShadow {
  int size = 0;          /* 0: the entry renders without a map */
  uint32_t casters = 0;
  uint64_t tris = 0;
  DevArena map, d_draws, recs, items, ctr;
  HostArena h_draws;     /* caster table, then the view-projection */
};

/* Uploads bounds and lights when the draw list changed (synchronous). */
int mc_scene_sync(MopCudaScene *s);
/* The scene's draw table as of now, with its per-draw IBL constants; with
 * models (nd x 16 floats) the model matrices are taken from there. */
void mc_scene_snapshot(MopCudaScene *s, DrawRec *dst, const std::vector<float> *models);
/* The scene's model matrices now (shared until the next change). */
std::shared_ptr<const std::vector<float>> mc_scene_models(MopCudaScene *s);
/* Estimated device bytes of one viewport of `samples` samples over scene s
 * (sample buffers plus half the worst-case work pools). */
uint64_t mc_view_bytes(const MopCudaScene *s, uint64_t samples, uint64_t pixels);

/* One launch of N viewports over one or more resident scenes: its device
 * buffers and work pools, and the stream it runs on. */
struct LaunchCore {
  MopCudaDevice *dev = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  /* layout */
  uint32_t nv = 0;
  std::vector<ViewRec> vrec;
  std::vector<MopCudaScene *> scenes; /* scene entries, index = ViewRec::scene */
  /* per entry: model matrices to render with (null: the scene's current) */
  std::vector<std::shared_ptr<const std::vector<float>>> scene_models;
  std::vector<uint64_t> scene_draw_off;
  uint64_t total_draws = 0, view_draw_total = 0;
  std::vector<PostArgs> posts;
  std::vector<EntryShadow> shadows; /* per scene entry */
  bool any_shadow = false;
  bool shadow_moved = false; /* stage() reallocated a shadow buffer */
  /* ordered suffix: a scene entry with order-dependent draws gives the
   * launch its per-sample buffers and pools; suffix_moved: stage()
   * reallocated one of them */
  bool any_ordered = false, any_wire = false, suffix_moved = false;
  DevArena hdr, frag_head, touched, frags, olist, olist_items, wlist, wlist_items, oscratch;
  unsigned long long frag_pool = 0, olist_pool = 0, wlist_pool = 0;
  uint32_t frag_num = 4;
  uint32_t post_count[4] = {0, 0, 0, 0}, post_tiles[4] = {0, 0, 0, 0};
  unsigned long long total_samples = 0, total_pixels = 0;
  /* inputs */
  DevArena d_views, d_frames, d_view_draws, d_ctr, d_status, d_posts, d_post_views, d_draws,
      d_scenes;
  HostArena h_views, h_draws, h_scenes, h_status;
  /* work pools */
  DevArena clip, world, normal, color, rrec, srec, clipq, large_list, large_items;
  unsigned long long vertex_pool = 0, rec_pool = 0, clip_pool = 0, large_pool = 0;
  uint32_t fan_num = 1, large_num = 1;
  /* pool sizes below which stage() does not go (a server sizes its slots
   * once for its largest launch, so they do not reallocate while serving) */
  unsigned long long pool_floor[4] = {0, 0, 0, 0};
  /* likewise for the sample- and pixel-resolution buffers */
  unsigned long long sample_floor = 0, pixel_floor = 0;
  /* sample / pixel buffers */
  DevArena keys, shade_list, pre, out, depth, ids, presented;
  /* launch shape */
  MopCudaBatchConfig cfg = {SMALL_MAX_SIDE, SMALL_MAX_AREA, 256, 256, 128, 256, 256, 1};
  float exposure = 1.0f;
  uint32_t post_effects = 0;
  float lut[256];
  float fog[6] = {0, 0, 0, 0, 0, 0};
  uint64_t launches = 0;

  int init(MopCudaDevice *d);
  void release();
  int stage_shadow(size_t k, const DrawRec *dr, SceneDesc &d);
  int stage_suffix();
  /* views[i] renders scene scene_of[i] (index into sc); no_color[i] (may be
   * null) marks visibility-only viewports. */
  int set_layout(const MopCudaView *views, const uint32_t *scene_of, const uint8_t *no_color,
                 uint32_t n, const std::vector<MopCudaScene *> &sc,
                 const std::vector<std::shared_ptr<const std::vector<float>>> *models = nullptr);
  /* Snapshots the scenes' draw tables into pinned memory; sizes the pools. */
  int stage();
  /* Enqueues the launch on `stream` (capturable): parts = BATCH_PART_MAIN
   * (uploads, clears, every stage up to shading) and/or BATCH_PART_POST (the
   * post passes, then the status copies the host reads at completion);
   * `launches` counts the kernels of the parts enqueued. */
  int enqueue(int parts = BATCH_PART_MAIN | BATCH_PART_POST);
  /* After ev1: true when the launch must run again (reserves or pools grew). */
  int after(bool *rerun, int attempt);
  uint64_t device_bytes() const;
  int sync(int timeout_ms);
  /* Frees the pools and sample buffers (they grow back on the next use). */
  void trim();
};

static inline bool mc_block_ok(int n) { return n >= 32 && n <= 256 && n % 32 == 0; }
int mc_check_view(const MopCudaView &v);
/* Work-pool entries one viewport of a scene of T triangles and V vertices
 * may need: vertices, records, clip queue, large list. */
void mc_pool_need(uint64_t T, uint64_t V, uint32_t fan_num, uint32_t large_num,
                  unsigned long long need[4]);

#endif
