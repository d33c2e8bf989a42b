/*
 * batch_api.cu — batched viewports over a resident scene (C ABI in
 * include/mop_cuda.h, "batched viewports").
 *
 * A MopCudaScene keeps the draw records of a scene on the host (the same
 * DrawRec the per-viewport path builds, so every per-draw constant is
 * identical).  A MopCudaBatch binds a scene to up to 256 viewports and
 * renders all of them with one CUDA graph: H2D of cameras and draw records,
 * counter/key clears, then one launch per pipeline stage covering every
 * viewport (kernels.cu, "Batched viewports"), and a D2H of the pool status.
 * The graph is captured once per pool layout / launch configuration and
 * replayed per submit.
 *
 * No counterpart in the reference: mop_viewport_render renders one viewport
 * per call (viewport.c:2990-3320).
 */
#include "api_internal.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

struct MopCudaScene {
  MopCudaDevice *dev = nullptr;
  std::vector<DrawRec> draws;
  std::vector<LightRec> lights;
  std::vector<DrawBound> bounds;
  uint64_t tris = 0, verts = 0;
  uint64_t version = 0; /* bumps when draws are added */
  std::mutex mu;
};

struct MopCudaBatch {
  MopCudaScene *scene = nullptr;
  MopCudaDevice *dev = nullptr;
  uint32_t nv = 0;
  std::vector<ViewRec> vrec;
  std::vector<PostArgs> posts;
  std::vector<uint32_t> post_list[4];
  uint32_t post_count[4] = {0, 0, 0, 0}, post_tiles[4] = {0, 0, 0, 0};
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  /* per-launch inputs and bookkeeping */
  DevArena d_views, d_frames, d_view_draws, d_ctr, d_status, d_posts, d_post_views, d_draws,
      d_lights, d_bounds;
  HostArena h_views, h_draws, h_status;
  uint64_t scene_version = ~0ull;
  uint32_t nd = 0;
  /* work pools (carved per viewport on the device) */
  DevArena clip, world, normal, color, rrec, srec, clipq, large_list, large_items;
  unsigned long long vertex_pool = 0, rec_pool = 0, clip_pool = 0, large_pool = 0;
  uint32_t fan_num = 1, large_num = 1; /* per-viewport reserve numerators */
  /* sample / pixel buffers */
  DevArena keys, shade_list, pre, out, depth, ids, presented, pick_xy, pick_out;
  DevArena irr, pf, brdf; /* the batch's copy of the device's IBL maps */
  HostArena h_pick;
  unsigned long long total_samples = 0, total_pixels = 0;
  /* launch shape */
  MopCudaBatchConfig cfg = {SMALL_MAX_SIDE, SMALL_MAX_AREA, 256, 256, 128, 256, 256, 1};
  FrameArgs tmpl;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool pending = false;
  float last_ms = 0.0f;
  uint64_t launches = 0;
  std::mutex mu;
};


/* ------------------------------------------------------------------------
 * scene
 * ------------------------------------------------------------------------ */
extern "C" MopCudaScene *mopcuda_scene_create(MopCudaDevice *dev) {
  if (!dev) {
    fail(MOPCUDA_EINVAL, "scene_create: no device");
    return nullptr;
  }
  MopCudaScene *s = new MopCudaScene();
  s->dev = dev;
  return s;
}

extern "C" void mopcuda_scene_destroy(MopCudaScene *s) { delete s; }

/* Bounding sphere of the positions the vertex stage reads (read_attrib
 * rules: missing components are 0), in double, then rounded outwards. */
static DrawBound mesh_bound(const MopCudaDraw *c) {
  DrawBound bd;
  bd.c[0] = bd.c[1] = bd.c[2] = 0.0f;
  bd.r = -1.0f;
  const uint8_t *base = (const uint8_t *)mopcuda_buffer_read(c->vertex_buffer);
  if (!base || c->vertex_count == 0)
    return bd;
  uint32_t stride = 48, off = 0, ncomp = 3;
  if (c->layout) {
    stride = c->layout->stride;
    off = (uint32_t)c->layout->position_offset;
    ncomp = (uint32_t)c->layout->position_components;
  }
  auto pos = [&](uint32_t i, double p[3]) {
    const float *f = (const float *)(base + (size_t)i * stride + off);
    for (uint32_t k = 0; k < 3; k++)
      p[k] = k < ncomp ? (double)f[k] : 0.0;
  };
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = 0; i < c->vertex_count; i++) {
    double p[3];
    pos(i, p);
    for (int k = 0; k < 3; k++) {
      if (!isfinite(p[k]))
        return bd; /* never culled */
      lo[k] = std::min(lo[k], p[k]);
      hi[k] = std::max(hi[k], p[k]);
    }
  }
  float cf[3];
  for (int k = 0; k < 3; k++)
    cf[k] = (float)(0.5 * (lo[k] + hi[k]));
  double r2 = 0.0;
  for (uint32_t i = 0; i < c->vertex_count; i++) {
    double p[3];
    pos(i, p);
    double d2 = 0.0;
    for (int k = 0; k < 3; k++)
      d2 += (p[k] - cf[k]) * (p[k] - cf[k]);
    r2 = std::max(r2, d2);
  }
  double r = sqrt(r2) * (1.0 + 1e-6) + 1e-30;
  float rf = (float)r;
  if ((double)rf < r)
    rf = nextafterf(rf, INFINITY);
  memcpy(bd.c, cf, sizeof cf);
  bd.r = rf;
  return bd;
}

extern "C" int mopcuda_scene_add_draw(MopCudaScene *s, const MopCudaDraw *c) {
  if (!s || !c)
    return fail(MOPCUDA_EINVAL, "scene_add_draw: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  DrawRec r;
  bool skip = false;
  const float ident[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  size_t nl = s->lights.size();
  int rc = mc_build_draw(c, c->model, ident, s->lights, r, skip);
  if (rc) {
    s->lights.resize(nl);
    return rc;
  }
  if (skip) { /* zero-opacity: drawn as nothing, keep an empty slot */
    memset(&r, 0, sizeof r);
    memcpy(r.model, c->model, sizeof r.model);
  }
  if ((uint64_t)s->tris + r.index_count / 3u >= (1ull << (32 - ORDER_FAN_BITS)))
    return fail(MOPCUDA_EINVAL, "scene too large");
  s->draws.push_back(r);
  s->bounds.push_back(skip ? DrawBound{{0, 0, 0}, -1.0f} : mesh_bound(c));
  s->tris += r.index_count / 3u;
  s->verts += r.vertex_count;
  s->version++;
  return (int)(s->draws.size() - 1);
}

extern "C" int mopcuda_scene_set_model(MopCudaScene *s, uint32_t index, const float model[16]) {
  if (!s || !model)
    return fail(MOPCUDA_EINVAL, "scene_set_model: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  if (index >= s->draws.size())
    return fail(MOPCUDA_EINVAL, "scene_set_model: index %u out of range", index);
  memcpy(s->draws[index].model, model, sizeof s->draws[index].model);
  return MOPCUDA_OK;
}

extern "C" uint32_t mopcuda_scene_draw_count(const MopCudaScene *s) {
  return s ? (uint32_t)s->draws.size() : 0u;
}

extern "C" uint64_t mopcuda_scene_triangle_count(const MopCudaScene *s) { return s ? s->tris : 0; }

/* ------------------------------------------------------------------------
 * batch
 * ------------------------------------------------------------------------ */
static int check_view(const MopCudaView &v) {
  if (v.width <= 0 || v.height <= 0 || v.ssaa < 1 || v.ssaa > 4)
    return fail(MOPCUDA_EINVAL, "batch view: bad size or ssaa");
  if ((uint64_t)v.width * v.ssaa > 32767u || (uint64_t)v.height * v.ssaa > 32767u)
    return fail(MOPCUDA_EINVAL, "batch view: %dx%d x%d exceeds 32767 samples per side", v.width,
                v.height, v.ssaa);
  return MOPCUDA_OK;
}

static void set_view(ViewRec &r, const MopCudaView &v) {
  memcpy(r.view, v.view, sizeof r.view);
  memcpy(r.proj, v.proj, sizeof r.proj);
  memcpy(r.eye, v.eye, sizeof r.eye);
  memcpy(r.clear, v.clear, sizeof r.clear);
}

static void drop_graph(MopCudaBatch *b) {
  if (b->exec)
    cudaGraphExecDestroy(b->exec);
  if (b->graph)
    cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

static int batch_sync(MopCudaBatch *b, int timeout_ms) {
  cudaEvent_t e;
  CU_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEventRecord(e, b->stream);
  int rc = mc_bounded_sync(b->dev, e, timeout_ms);
  cudaEventDestroy(e);
  return rc;
}

extern "C" void mopcuda_batch_destroy(MopCudaBatch *b) {
  if (!b)
    return;
  cudaSetDevice(b->dev->ordinal);
  if (b->stream)
    batch_sync(b, 10000);
  drop_graph(b);
  DevArena *arenas[] = {&b->d_views, &b->d_frames, &b->d_view_draws, &b->d_ctr, &b->d_status,
                        &b->d_posts, &b->d_post_views, &b->d_draws, &b->d_lights, &b->d_bounds,
                        &b->clip, &b->world, &b->normal, &b->color, &b->rrec, &b->srec,
                        &b->clipq, &b->large_list, &b->large_items, &b->keys, &b->shade_list,
                        &b->pre, &b->out, &b->depth, &b->ids, &b->presented, &b->pick_xy,
                        &b->pick_out, &b->irr, &b->pf, &b->brdf};
  for (DevArena *a : arenas)
    a->release();
  b->h_views.release();
  b->h_draws.release();
  b->h_status.release();
  b->h_pick.release();
  if (b->ev0)
    cudaEventDestroy(b->ev0);
  if (b->ev1)
    cudaEventDestroy(b->ev1);
  if (b->stream)
    cudaStreamDestroy(b->stream);
  delete b;
}

/* Pools for the worst case scaled by `frac` (every draw visible in every
 * viewport is frac = 1). */
static int size_pools(MopCudaBatch *b, unsigned long long vneed, unsigned long long rneed,
                      unsigned long long cneed, unsigned long long lneed) {
  int rc = 0;
  rc |= b->clip.ensure(16ull * vneed);
  rc |= b->world.ensure(16ull * vneed);
  rc |= b->normal.ensure(16ull * vneed);
  rc |= b->color.ensure(16ull * vneed);
  rc |= b->rrec.ensure(sizeof(RasterRec) * rneed);
  rc |= b->srec.ensure(sizeof(ShadeRec) * rneed);
  rc |= b->clipq.ensure(4ull * cneed);
  rc |= b->large_list.ensure(4ull * lneed);
  rc |= b->large_items.ensure(4ull * lneed);
  if (rc)
    return MOPCUDA_ENOMEM;
  auto cap = [](const DevArena &a, size_t el) { return (unsigned long long)(a.cap / el); };
  b->vertex_pool = std::min(std::min(cap(b->clip, 16), cap(b->world, 16)),
                            std::min(cap(b->normal, 16), cap(b->color, 16)));
  b->rec_pool = std::min(cap(b->rrec, sizeof(RasterRec)), cap(b->srec, sizeof(ShadeRec)));
  b->clip_pool = cap(b->clipq, 4);
  b->large_pool = std::min(cap(b->large_list, 4), cap(b->large_items, 4));
  return MOPCUDA_OK;
}

/* Uploads the scene when it changed and refreshes the pinned draw table. */
static int stage_scene(MopCudaBatch *b) {
  MopCudaScene *s = b->scene;
  std::lock_guard<std::mutex> lk(s->mu);
  const uint32_t nd = (uint32_t)s->draws.size();
  if (s->version != b->scene_version) {
    int rc = 0;
    rc |= b->d_draws.ensure(sizeof(DrawRec) * (nd ? nd : 1));
    rc |= b->h_draws.ensure(sizeof(DrawRec) * (nd ? nd : 1));
    rc |= b->d_view_draws.ensure(sizeof(DrawRec) * (size_t)(nd ? nd : 1) * b->nv);
    rc |= b->d_lights.ensure(sizeof(LightRec) * (s->lights.size() + 1));
    rc |= b->d_bounds.ensure(sizeof(DrawBound) * (nd ? nd : 1));
    if (rc)
      return MOPCUDA_ENOMEM;
    if (!s->lights.empty())
      CU_TRY(cudaMemcpy(b->d_lights.p, s->lights.data(), sizeof(LightRec) * s->lights.size(),
                        cudaMemcpyHostToDevice));
    if (nd)
      CU_TRY(cudaMemcpy(b->d_bounds.p, s->bounds.data(), sizeof(DrawBound) * nd,
                        cudaMemcpyHostToDevice));
    b->tmpl.lights = b->d_lights.as<LightRec>();
    b->tmpl.light_total = (uint32_t)s->lights.size();
    b->nd = nd;
    b->scene_version = s->version;
    /* first pools: half the worst case (all draws visible everywhere) */
    const unsigned long long T = s->tris, V = s->verts, fan = T * b->fan_num / 8ull + 1024ull;
    const unsigned long long half = (b->nv + 1ull) / 2ull;
    int prc = size_pools(b, half * (V + fan), half * (T + fan), half * fan,
                         half * (T * b->large_num / 16ull + 1024ull));
    if (prc)
      return prc;
    drop_graph(b);
  }
  DrawRec *h = b->h_draws.as<DrawRec>();
  if (nd)
    memcpy(h, s->draws.data(), sizeof(DrawRec) * nd);
  const FrameArgs &t = b->tmpl;
  mc_ibl_consts(t.pf != nullptr, t.pf_w, t.pf_h, t.pf_levels, t.brdf_size, h, nd);
  return MOPCUDA_OK;
}

static int build_graph(MopCudaBatch *b) {
  drop_graph(b);
  BatchLaunch L;
  memset(&L, 0, sizeof L);
  L.num_sms = b->dev->num_sms;
  L.vertex_block = b->cfg.vertex_block;
  L.setup_block = b->cfg.setup_block;
  L.raster_block = b->cfg.raster_block;
  L.large_block = b->cfg.large_block;
  L.shade_block = b->cfg.shade_block;
  L.grid_mul = b->cfg.grid_mul;
  mopcuda_batch_grids(L);
  b->tmpl.small_side = b->cfg.small_side;
  b->tmpl.small_area = b->cfg.small_area;

  BatchArgs a;
  memset(&a, 0, sizeof a);
  a.scene = b->d_draws.as<DrawRec>();
  a.bounds = b->d_bounds.as<DrawBound>();
  a.nd = b->nd;
  a.views = b->d_views.as<ViewRec>();
  a.nv = b->nv;
  a.frames = b->d_frames.as<FrameArgs>();
  a.view_draws = b->d_view_draws.as<DrawRec>();
  a.ctr = b->d_ctr.as<Counters>();
  a.status = b->d_status.as<BatchStatus>();
  a.tmpl = b->tmpl;
  a.clip = b->clip.as<float4>();
  a.world = b->world.as<float4>();
  a.normal = b->normal.as<float4>();
  a.color = b->color.as<float4>();
  a.vertex_pool = b->vertex_pool;
  a.rrec = b->rrec.as<RasterRec>();
  a.srec = b->srec.as<ShadeRec>();
  a.rec_pool = b->rec_pool;
  a.clipq = b->clipq.as<uint32_t>();
  a.clip_pool = b->clip_pool;
  a.large_list = b->large_list.as<uint32_t>();
  a.large_items = b->large_items.as<uint32_t>();
  a.large_pool = b->large_pool;
  a.keys = b->keys.as<unsigned long long>();
  a.shade_list = b->shade_list.as<uint32_t>();
  a.pre = b->pre.as<uchar4>();
  a.depth = b->depth.as<float>();
  a.ids = b->ids.as<uint32_t>();
  a.fan_num = b->fan_num;
  a.large_num = b->large_num;

  const uint32_t *pv[4];
  for (int k = 0; k < 4; k++)
    pv[k] = b->d_post_views.as<uint32_t>() + (size_t)k * b->nv;

  cudaStream_t s = b->stream;
  CU_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaMemcpyAsync(b->d_views.p, b->h_views.p, sizeof(ViewRec) * b->nv, cudaMemcpyHostToDevice, s);
  if (b->nd)
    cudaMemcpyAsync(b->d_draws.p, b->h_draws.p, sizeof(DrawRec) * b->nd, cudaMemcpyHostToDevice,
                    s);
  cudaMemsetAsync(b->d_ctr.p, 0, sizeof(Counters) * b->nv, s);
  cudaMemsetAsync(b->d_status.p, 0, sizeof(BatchStatus), s);
  cudaMemsetAsync(b->keys.p, 0xff, 8ull * b->total_samples, s);
  int n = mopcuda_launch_batch(a, b->d_posts.as<PostArgs>(), pv, b->post_count, b->post_tiles, L,
                               s);
  cudaMemcpyAsync(b->h_status.p, b->d_status.p, sizeof(BatchStatus), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(b->h_status.as<uint8_t>() + sizeof(BatchStatus), b->d_ctr.p,
                  sizeof(Counters) * b->nv, cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamEndCapture(s, &b->graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b->graph = nullptr;
    return fail(MOPCUDA_ECUDA, "batch graph capture: %s", cudaGetErrorString(e));
  }
  e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    drop_graph(b);
    return fail(MOPCUDA_ECUDA, "batch graph instantiate: %s", cudaGetErrorString(e));
  }
  b->launches = (uint64_t)n;
  return MOPCUDA_OK;
}

extern "C" MopCudaBatch *mopcuda_batch_create(MopCudaScene *scene, const MopCudaView *views,
                                              uint32_t n) {
  if (!scene || !views || n == 0 || n > MOPCUDA_MAX_VIEWS) {
    fail(MOPCUDA_EINVAL, "batch_create: need a scene and 1..%d views", MOPCUDA_MAX_VIEWS);
    return nullptr;
  }
  for (uint32_t i = 0; i < n; i++)
    if (check_view(views[i]))
      return nullptr;
  MopCudaDevice *d = scene->dev;
  cudaSetDevice(d->ordinal);
  MopCudaBatch *b = new MopCudaBatch();
  b->scene = scene;
  b->dev = d;
  b->nv = n;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
    cudaGetLastError();
    fail(MOPCUDA_ECUDA, "batch_create: stream/event creation failed");
    mopcuda_batch_destroy(b);
    return nullptr;
  }
  b->vrec.resize(n);
  b->posts.resize(n);
  unsigned long long so = 0, po = 0;
  PostArgs post;
  mc_post_args(d, post);
  for (uint32_t i = 0; i < n; i++) {
    const MopCudaView &v = views[i];
    ViewRec &r = b->vrec[i];
    memset(&r, 0, sizeof r);
    set_view(r, v);
    r.ssaa = v.ssaa;
    r.width = v.width * v.ssaa;
    r.height = v.height * v.ssaa;
    r.sample_off = so;
    r.pixel_off = po;
    /* 16-sample alignment keeps the resolve's vector stores aligned */
    so += ((unsigned long long)r.width * r.height + 15ull) & ~15ull;
    po += ((unsigned long long)v.width * v.height + 15ull) & ~15ull;
  }
  b->total_samples = so;
  b->total_pixels = po;
  int rc = 0;
  rc |= b->keys.ensure(8ull * so);
  rc |= b->shade_list.ensure(4ull * so);
  rc |= b->pre.ensure(4ull * so);
  rc |= b->out.ensure(4ull * so);
  rc |= b->depth.ensure(4ull * so);
  rc |= b->ids.ensure(4ull * so);
  rc |= b->presented.ensure(4ull * po + 16);
  rc |= b->d_views.ensure(sizeof(ViewRec) * n);
  rc |= b->h_views.ensure(sizeof(ViewRec) * n);
  rc |= b->d_frames.ensure(sizeof(FrameArgs) * n);
  rc |= b->d_ctr.ensure(sizeof(Counters) * n);
  rc |= b->d_status.ensure(sizeof(BatchStatus));
  rc |= b->h_status.ensure(sizeof(BatchStatus) + sizeof(Counters) * n);
  rc |= b->d_posts.ensure(sizeof(PostArgs) * n);
  rc |= b->d_post_views.ensure(4ull * 4ull * n);
  if (rc) {
    mopcuda_batch_destroy(b);
    return nullptr;
  }
  for (uint32_t i = 0; i < n; i++) {
    const ViewRec &r = b->vrec[i];
    PostArgs p = post;
    p.pre = b->pre.as<uchar4>() + r.sample_off;
    p.out = b->out.as<uchar4>() + r.sample_off;
    p.presented = r.ssaa > 1 ? b->presented.as<uchar4>() + r.pixel_off : nullptr;
    p.width = r.width;
    p.height = r.height;
    p.ssaa = r.ssaa;
    b->posts[i] = p;
    const int k = r.ssaa - 1;
    b->post_list[k].push_back(i);
    const uint32_t pw = (uint32_t)(r.width / r.ssaa), ph = (uint32_t)(r.height / r.ssaa);
    b->post_tiles[k] += ((pw + 31u) / 32u) * ((ph + 7u) / 8u);
  }
  std::vector<uint32_t> lists(4ull * n, 0u);
  for (int k = 0; k < 4; k++) {
    b->post_count[k] = (uint32_t)b->post_list[k].size();
    std::copy(b->post_list[k].begin(), b->post_list[k].end(), lists.begin() + (size_t)k * n);
  }
  if (cudaMemcpy(b->d_posts.p, b->posts.data(), sizeof(PostArgs) * n, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(b->d_post_views.p, lists.data(), 4ull * 4ull * n, cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    cudaGetLastError();
    fail(MOPCUDA_ECUDA, "batch_create: upload failed");
    mopcuda_batch_destroy(b);
    return nullptr;
  }
  /* frame state shared by every viewport */
  FrameArgs &t = b->tmpl;
  memset(&t, 0, sizeof t);
  t.exposure = d->exposure;
  if (d->ibl_on) {
    /* own copies: later set_ibl calls on the device must not move them */
    size_t pf_px = 0;
    for (int l = 0; l < d->pf_levels; l++) {
      int lw = d->pf_w >> l, lh = d->pf_h >> l;
      pf_px += (size_t)(lw < 1 ? 1 : lw) * (size_t)(lh < 1 ? 1 : lh);
    }
    const size_t ib = (size_t)d->irr_w * d->irr_h * 16, pb = pf_px * 16,
                 bb = (size_t)d->brdf_size * d->brdf_size * 16;
    if (b->irr.ensure(ib) || b->pf.ensure(pb) || b->brdf.ensure(bb) ||
        cudaMemcpy(b->irr.p, d->irr.p, ib, cudaMemcpyDeviceToDevice) != cudaSuccess ||
        cudaMemcpy(b->pf.p, d->pf.p, pb, cudaMemcpyDeviceToDevice) != cudaSuccess ||
        cudaMemcpy(b->brdf.p, d->brdf.p, bb, cudaMemcpyDeviceToDevice) != cudaSuccess) {
      cudaGetLastError();
      fail(MOPCUDA_ENOMEM, "batch_create: IBL copy failed");
      mopcuda_batch_destroy(b);
      return nullptr;
    }
    t.irr = b->irr.as<float>();
    t.irr_w = d->irr_w;
    t.irr_h = d->irr_h;
    t.pf = b->pf.as<float>();
    t.pf_w = d->pf_w;
    t.pf_h = d->pf_h;
    t.pf_levels = d->pf_levels;
    t.brdf = b->brdf.as<float>();
    t.brdf_size = d->brdf_size;
    t.ibl_rotation = d->ibl_rot;
    t.ibl_intensity = d->ibl_int;
  }
  return b;
}

extern "C" int mopcuda_batch_set_views(MopCudaBatch *b, const MopCudaView *views, uint32_t n) {
  if (!b || !views || n != b->nv)
    return fail(MOPCUDA_EINVAL, "batch_set_views: need %u views", b ? b->nv : 0u);
  std::lock_guard<std::mutex> lk(b->mu);
  for (uint32_t i = 0; i < n; i++) {
    const ViewRec &r = b->vrec[i];
    if (views[i].ssaa != r.ssaa || views[i].width * views[i].ssaa != r.width ||
        views[i].height * views[i].ssaa != r.height)
      return fail(MOPCUDA_EINVAL, "batch_set_views: view %u changed size or ssaa", i);
  }
  for (uint32_t i = 0; i < n; i++)
    set_view(b->vrec[i], views[i]);
  return MOPCUDA_OK;
}

static int launch_graph(MopCudaBatch *b) {
  cudaStream_t s = b->stream;
  CU_TRY(cudaEventRecord(b->ev0, s));
  CU_TRY(cudaGraphLaunch(b->exec, s));
  CU_TRY(cudaEventRecord(b->ev1, s));
  b->pending = true;
  return MOPCUDA_OK;
}

static int finish_batch(MopCudaBatch *b, int timeout_ms);

static int submit_locked(MopCudaBatch *b) {
  cudaSetDevice(b->dev->ordinal);
  int rc = finish_batch(b, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  rc = stage_scene(b);
  if (rc)
    return rc;
  memcpy(b->h_views.p, b->vrec.data(), sizeof(ViewRec) * b->nv);
  if (!b->exec) {
    rc = build_graph(b);
    if (rc)
      return rc;
  }
  return launch_graph(b);
}

extern "C" int mopcuda_batch_submit(MopCudaBatch *b) {
  if (!b)
    return fail(MOPCUDA_EINVAL, "batch_submit: no batch");
  std::lock_guard<std::mutex> lk(b->mu);
  return submit_locked(b);
}

/* Waits; re-runs after growing the per-viewport reserves (a viewport's
 * counters overflowed) or the pools (the allocation pass found them short;
 * the status holds the exact totals). */
static int finish_batch(MopCudaBatch *b, int timeout_ms) {
  for (int attempt = 0; b->pending; attempt++) {
    int rc = mc_bounded_sync(b->dev, b->ev1, timeout_ms);
    b->pending = false;
    if (rc)
      return rc;
    cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
    const BatchStatus *st = b->h_status.as<BatchStatus>();
    const Counters *ctr = (const Counters *)(b->h_status.as<uint8_t>() + sizeof(BatchStatus));
    uint32_t view_over = 0;
    for (uint32_t i = 0; i < b->nv; i++)
      view_over |= ctr[i].overflow;
    if (!st->overflow && !view_over)
      break;
    if (attempt >= 8)
      return fail(MOPCUDA_ENOMEM, "batch pools overflowed repeatedly (flags %u/%u)",
                  st->overflow, view_over);
    if (view_over & 7u) { /* clipped fans: records, extra vertices or clip queue */
      if (b->fan_num >= 256u)
        return fail(MOPCUDA_ENOMEM, "batch: clipped-fan reserve exhausted");
      b->fan_num *= 2u;
    }
    if (view_over & 8u) {
      if (b->large_num >= 512u)
        return fail(MOPCUDA_ENOMEM, "batch: large-record list exhausted");
      b->large_num *= 2u;
    }
    if (st->overflow) {
      const unsigned long long need[4] = {st->need_vertex, st->need_rec, st->need_clip,
                                          st->need_large};
      unsigned long long cap[4] = {b->vertex_pool, b->rec_pool, b->clip_pool, b->large_pool};
      for (int k = 0; k < 4; k++)
        if (need[k] > cap[k])
          cap[k] = need[k] + need[k] / 4 + 4096ull;
      rc = size_pools(b, cap[0], cap[1], cap[2], cap[3]);
      if (rc)
        return rc;
    }
    rc = build_graph(b);
    if (rc)
      return rc;
    rc = launch_graph(b);
    if (rc)
      return rc;
  }
  return MOPCUDA_OK;
}

extern "C" int mopcuda_batch_wait(MopCudaBatch *b, int timeout_ms) {
  if (!b)
    return fail(MOPCUDA_EINVAL, "batch_wait: no batch");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->dev->ordinal);
  return finish_batch(b, timeout_ms);
}

extern "C" float mopcuda_batch_gpu_time_ms(const MopCudaBatch *b) { return b ? b->last_ms : 0.0f; }

extern "C" int mopcuda_batch_read(MopCudaBatch *b, uint32_t view, int what, void *dst,
                                  size_t bytes) {
  if (!b || !dst || view >= b->nv)
    return fail(MOPCUDA_EINVAL, "batch_read: bad arguments");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->dev->ordinal);
  int rc = finish_batch(b, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  const ViewRec &r = b->vrec[view];
  const size_t S = (size_t)r.width * r.height;
  const size_t P = (size_t)(r.width / r.ssaa) * (r.height / r.ssaa);
  const void *src = nullptr;
  size_t n = 0;
  switch (what) {
  case MOPCUDA_BATCH_COLOR:
    src = b->out.as<uchar4>() + r.sample_off;
    n = 4 * S;
    break;
  case MOPCUDA_BATCH_PRESENTED:
    src = r.ssaa > 1 ? (const void *)(b->presented.as<uchar4>() + r.pixel_off)
                     : (const void *)(b->out.as<uchar4>() + r.sample_off);
    n = 4 * P;
    break;
  case MOPCUDA_BATCH_DEPTH:
    src = b->depth.as<float>() + r.sample_off;
    n = 4 * S;
    break;
  case MOPCUDA_BATCH_IDS:
    src = b->ids.as<uint32_t>() + r.sample_off;
    n = 4 * S;
    break;
  default:
    return fail(MOPCUDA_EINVAL, "batch_read: unknown buffer %d", what);
  }
  if (bytes != n)
    return fail(MOPCUDA_EINVAL, "batch_read: buffer is %zu bytes, not %zu", n, bytes);
  CU_TRY(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, b->stream));
  return batch_sync(b, FRAME_TIMEOUT_MS);
}

extern "C" int mopcuda_batch_pick(MopCudaBatch *b, uint32_t view, const int32_t *xy, uint32_t n,
                                  uint32_t *ids, float *depths, int32_t *hits) {
  if (!b || view >= b->nv || (n && (!xy || !ids || !depths || !hits)))
    return fail(MOPCUDA_EINVAL, "batch_pick: bad arguments");
  if (n == 0)
    return MOPCUDA_OK;
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->dev->ordinal);
  int rc = finish_batch(b, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  size_t in_b = 8ull * n, out_b = 12ull * n;
  if (b->pick_xy.ensure(in_b) || b->pick_out.ensure(out_b) || b->h_pick.ensure(in_b + out_b))
    return MOPCUDA_ENOMEM;
  memcpy(b->h_pick.p, xy, in_b);
  cudaStream_t s = b->stream;
  CU_TRY(cudaMemcpyAsync(b->pick_xy.p, b->h_pick.p, in_b, cudaMemcpyHostToDevice, s));
  uint32_t *oid = b->pick_out.as<uint32_t>();
  float *odp = (float *)(oid + n);
  int32_t *oht = (int32_t *)(odp + n);
  const ViewRec &r = b->vrec[view];
  mopcuda_launch_pick(b->ids.as<uint32_t>() + r.sample_off, b->depth.as<float>() + r.sample_off,
                      r.width, r.height, r.ssaa, b->pick_xy.as<int2>(), n, oid, odp, oht, s);
  CU_TRY(cudaGetLastError());
  uint8_t *hb = b->h_pick.as<uint8_t>() + in_b;
  CU_TRY(cudaMemcpyAsync(hb, b->pick_out.p, out_b, cudaMemcpyDeviceToHost, s));
  rc = batch_sync(b, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  memcpy(ids, hb, 4ull * n);
  memcpy(depths, hb + 4ull * n, 4ull * n);
  memcpy(hits, hb + 8ull * n, 4ull * n);
  return MOPCUDA_OK;
}

/* ------------------------------------------------------------------------
 * launch configuration and autotuner
 * ------------------------------------------------------------------------ */
extern "C" int mopcuda_batch_get_config(const MopCudaBatch *b, MopCudaBatchConfig *cfg) {
  if (!b || !cfg)
    return fail(MOPCUDA_EINVAL, "batch_get_config: bad arguments");
  *cfg = b->cfg;
  return MOPCUDA_OK;
}

static bool block_ok(int n) { return n >= 32 && n <= 256 && n % 32 == 0; }

extern "C" int mopcuda_batch_set_config(MopCudaBatch *b, const MopCudaBatchConfig *c) {
  if (!b || !c)
    return fail(MOPCUDA_EINVAL, "batch_set_config: bad arguments");
  if (c->small_side < 1 || c->small_side > 256 || c->small_area < 1 ||
      c->small_area > 65536 || !block_ok(c->vertex_block) || !block_ok(c->setup_block) ||
      !block_ok(c->raster_block) || !block_ok(c->large_block) || !block_ok(c->shade_block) ||
      c->grid_mul < 1 || c->grid_mul > 8)
    return fail(MOPCUDA_EINVAL, "batch_set_config: value out of range");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->dev->ordinal);
  int rc = finish_batch(b, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  b->cfg = *c;
  drop_graph(b);
  return MOPCUDA_OK;
}

/* Median device time of `reps` launches under the current configuration. */
static int time_config(MopCudaBatch *b, int reps, float *ms) {
  int rc = submit_locked(b); /* warm-up; also grows the pools if needed */
  if (!rc)
    rc = finish_batch(b, FRAME_TIMEOUT_MS);
  std::vector<float> t;
  for (int i = 0; i < reps && !rc; i++) {
    rc = submit_locked(b);
    if (!rc)
      rc = finish_batch(b, FRAME_TIMEOUT_MS);
    t.push_back(b->last_ms);
  }
  if (rc)
    return rc;
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return MOPCUDA_OK;
}

extern "C" int mopcuda_batch_autotune(MopCudaBatch *b, int reps, char *report,
                                      size_t report_len) {
  if (!b || reps < 1)
    return fail(MOPCUDA_EINVAL, "batch_autotune: bad arguments");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->dev->ordinal);
  MopCudaBatchConfig best = b->cfg;
  float best_ms = 0.0f;
  int rc = time_config(b, reps, &best_ms);
  if (rc)
    return rc;
  std::string log = "{\"start_ms\": " + std::to_string(best_ms) + ", \"trials\": [";
  bool first = true;
  struct Axis {
    const char *name;
    std::vector<std::pair<int, int>> values;
  };
  const std::vector<Axis> axes = {
      {"small", {{16, 64}, {32, 128}, {32, 256}, {64, 512}}},
      {"raster_block", {{64, 0}, {128, 0}, {256, 0}}},
      {"setup_block", {{128, 0}, {256, 0}}},
      {"large_block", {{128, 0}, {256, 0}}},
      {"shade_block", {{128, 0}, {256, 0}}},
      {"vertex_block", {{128, 0}, {256, 0}}},
      {"grid_mul", {{1, 0}, {2, 0}}},
  };
  for (const Axis &ax : axes)
    for (const auto &val : ax.values) {
      MopCudaBatchConfig c = best;
      std::string nm = ax.name;
      if (nm == "small") {
        c.small_side = val.first;
        c.small_area = val.second;
      } else if (nm == "raster_block") {
        c.raster_block = val.first;
      } else if (nm == "setup_block") {
        c.setup_block = val.first;
      } else if (nm == "large_block") {
        c.large_block = val.first;
      } else if (nm == "shade_block") {
        c.shade_block = val.first;
      } else if (nm == "vertex_block") {
        c.vertex_block = val.first;
      } else {
        c.grid_mul = val.first;
      }
      if (memcmp(&c, &best, sizeof c) == 0)
        continue;
      b->cfg = c;
      drop_graph(b);
      float ms = 0.0f;
      rc = time_config(b, reps, &ms);
      if (rc)
        return rc;
      char buf[160];
      snprintf(buf, sizeof buf, "%s{\"%s\": [%d, %d], \"ms\": %.4f}", first ? "" : ", ", ax.name,
               val.first, val.second, ms);
      log += buf;
      first = false;
      if (ms < best_ms * 0.99f) {
        best = c;
        best_ms = ms;
      }
    }
  b->cfg = best;
  drop_graph(b);
  char tail[256];
  snprintf(tail, sizeof tail,
           "], \"best_ms\": %.4f, \"best\": {\"small_side\": %d, \"small_area\": %d, "
           "\"vertex_block\": %d, \"setup_block\": %d, \"raster_block\": %d, "
           "\"large_block\": %d, \"shade_block\": %d, \"grid_mul\": %d}}",
           best_ms, best.small_side, best.small_area, best.vertex_block, best.setup_block,
           best.raster_block, best.large_block, best.shade_block, best.grid_mul);
  log += tail;
  if (report && report_len) {
    strncpy(report, log.c_str(), report_len - 1);
    report[report_len - 1] = '\0';
  }
  return MOPCUDA_OK;
}

extern "C" uint64_t mopcuda_batch_device_bytes(const MopCudaBatch *b) {
  if (!b)
    return 0;
  const DevArena *arenas[] = {&b->d_views, &b->d_frames, &b->d_view_draws, &b->d_ctr,
                              &b->d_status, &b->d_posts, &b->d_post_views, &b->d_draws,
                              &b->d_lights, &b->d_bounds, &b->clip, &b->world, &b->normal,
                              &b->color, &b->rrec, &b->srec, &b->clipq, &b->large_list,
                              &b->large_items, &b->keys, &b->shade_list, &b->pre, &b->out,
                              &b->depth, &b->ids, &b->presented, &b->pick_xy, &b->pick_out,
                              &b->irr, &b->pf, &b->brdf};
  uint64_t t = 0;
  for (const DevArena *a : arenas)
    t += a->cap;
  return t;
}
