/*
 * batch_api.cu — resident scenes and batched viewports (C ABI in
 * include/mop_cuda.h, "batched viewports").
 *
 * A MopCudaScene keeps the draw records of a scene on the host (the same
 * DrawRec the per-viewport path builds, so every per-draw constant is
 * identical) plus device copies of its draw bounds, lights and IBL maps.  A
 * LaunchCore renders N viewports over one or more scenes in one stream
 * sequence: H2D of cameras and draw tables, counter/key clears, one launch
 * per pipeline stage covering every viewport (kernels.cu, "Batched
 * viewports") and a D2H of the pool status.  A MopCudaBatch captures that
 * sequence once as a CUDA graph and replays it per submit.
 *
 * No counterpart in the reference: mop_viewport_render renders one viewport
 * per call (viewport.c:2990-3320).
 */
#include "batch_internal.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

/* ------------------------------------------------------------------------
 * scene
 * ------------------------------------------------------------------------ */
static int copy_ibl(MopCudaScene *s, const MopCudaDevice *d) {
  s->ibl_on = d->ibl_on;
  if (!d->ibl_on)
    return MOPCUDA_OK;
  size_t pf_px = 0;
  for (int l = 0; l < d->pf_levels; l++) {
    int lw = d->pf_w >> l, lh = d->pf_h >> l;
    pf_px += (size_t)(lw < 1 ? 1 : lw) * (size_t)(lh < 1 ? 1 : lh);
  }
  const size_t ib = (size_t)d->irr_w * d->irr_h * 16, pb = pf_px * 16,
               bb = (size_t)d->brdf_size * d->brdf_size * 16;
  if (s->irr.ensure(ib) || s->pf.ensure(pb) || s->brdf.ensure(bb))
    return MOPCUDA_ENOMEM;
  CU_TRY(cudaMemcpy(s->irr.p, d->irr.p, ib, cudaMemcpyDeviceToDevice));
  CU_TRY(cudaMemcpy(s->pf.p, d->pf.p, pb, cudaMemcpyDeviceToDevice));
  CU_TRY(cudaMemcpy(s->brdf.p, d->brdf.p, bb, cudaMemcpyDeviceToDevice));
  s->irr_w = d->irr_w;
  s->irr_h = d->irr_h;
  s->pf_w = d->pf_w;
  s->pf_h = d->pf_h;
  s->pf_levels = d->pf_levels;
  s->brdf_size = d->brdf_size;
  s->ibl_rot = d->ibl_rot;
  s->ibl_int = d->ibl_int;
  return MOPCUDA_OK;
}

extern "C" MopCudaScene *mopcuda_scene_create(MopCudaDevice *dev) {
  if (!dev) {
    fail(MOPCUDA_EINVAL, "scene_create: no device");
    return nullptr;
  }
  cudaSetDevice(dev->ordinal);
  MopCudaScene *s = new MopCudaScene();
  s->dev = dev;
  {
    std::lock_guard<std::mutex> lk(dev->mu);
    if (mc_stream_sync(dev, 10000) || copy_ibl(s, dev)) {
      delete s;
      return nullptr;
    }
  }
  return s;
}

extern "C" void mopcuda_scene_destroy(MopCudaScene *s) {
  if (!s)
    return;
  cudaSetDevice(s->dev->ordinal);
  s->d_bounds.release();
  s->d_lights.release();
  s->irr.release();
  s->pf.release();
  s->brdf.release();
  delete s;
}

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
  if (s->frozen)
    return fail(MOPCUDA_EINVAL, "scene_add_draw: the scene is held by a server");
  DrawRec r;
  bool skip = false;
  const float ident[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  size_t nl = s->lights.size();
  int rc = mc_build_draw(c, c->model, ident, s->lights, r, skip);
  if (rc) {
    s->lights.resize(nl);
    return rc;
  }
  if (!skip && (r.flags & (DF_NO_DEPTH_WRITE | DF_NO_DEPTH_TEST))) {
    s->lights.resize(nl);
    return fail(MOPCUDA_EUNSUPPORTED,
                "scene_add_draw: batches render depth-tested, depth-writing draws only");
  }
  if (skip) { /* zero opacity: a colour no-op, kept as an empty slot */
    memset(&r, 0, sizeof r);
    memcpy(r.model, c->model, sizeof r.model);
  }
  /* blended, translucent and unlit smooth draws are order-dependent: each
   * viewport composites them in its ordered suffix, the blended ones in
   * the core's back-to-front order for that viewport's eye */
  const float op = r.opacity < 0.0f ? 0.0f : (r.opacity > 1.0f ? 1.0f : r.opacity);
  if (!skip && (r.blend_mode != 0 || op < 1.0f || ((r.flags & DF_SMOOTH) && !(r.flags & DF_LIT)) ||
                (r.flags & DF_WIRE)))
    r.flags |= DF_ORDERED;
  /* line plots mark fragment payloads with bit 31: a viewport's triangles
   * stay below 2^26 when the scene has wireframe draws */
  if ((r.flags & DF_WIRE) || s->wire) {
    if ((uint64_t)s->tris + r.index_count / 3u >= (1ull << (31 - ORDER_FAN_BITS))) {
      s->lights.resize(nl);
      return fail(MOPCUDA_EUNSUPPORTED, "scene_add_draw: wireframe draws in a scene of 2^26 "
                                        "or more triangles");
    }
  }
  if (r.blend_mode != 0 && s->blended >= BATCH_MAX_BLENDED) {
    s->lights.resize(nl);
    return fail(MOPCUDA_EUNSUPPORTED, "scene_add_draw: more than %d blended draws in a scene",
                BATCH_MAX_BLENDED);
  }
  if ((uint64_t)s->tris + r.index_count / 3u >= (1ull << (32 - ORDER_FAN_BITS)))
    return fail(MOPCUDA_EINVAL, "scene too large");
  if (r.blend_mode != 0)
    s->blended++;
  if (r.flags & DF_WIRE)
    s->wire = true;
  if (r.flags & DF_ORDERED)
    s->ordered_tris += r.index_count / 3u;
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
  s->gen++;
  return MOPCUDA_OK;
}

extern "C" int mopcuda_scene_set_shadow(MopCudaScene *s, int size, const float direction[3]) {
  if (!s || size < 0 || size > 16384 || (size > 0 && !direction))
    return fail(MOPCUDA_EINVAL, "scene_set_shadow: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  s->sh_size = size;
  if (size > 0)
    memcpy(s->sh_dir, direction, sizeof s->sh_dir);
  return MOPCUDA_OK;
}

extern "C" uint32_t mopcuda_scene_draw_count(const MopCudaScene *s) {
  return s ? (uint32_t)s->draws.size() : 0u;
}

extern "C" uint64_t mopcuda_scene_triangle_count(const MopCudaScene *s) { return s ? s->tris : 0; }

int mc_scene_sync(MopCudaScene *s) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->dev_version == s->version)
    return MOPCUDA_OK;
  const size_t nd = s->draws.size();
  if (s->d_bounds.ensure(sizeof(DrawBound) * (nd ? nd : 1)) ||
      s->d_lights.ensure(sizeof(LightRec) * (s->lights.size() + 1)))
    return MOPCUDA_ENOMEM;
  if (nd)
    CU_TRY(cudaMemcpy(s->d_bounds.p, s->bounds.data(), sizeof(DrawBound) * nd,
                      cudaMemcpyHostToDevice));
  if (!s->lights.empty())
    CU_TRY(cudaMemcpy(s->d_lights.p, s->lights.data(), sizeof(LightRec) * s->lights.size(),
                      cudaMemcpyHostToDevice));
  s->dev_version = s->version;
  return MOPCUDA_OK;
}

void mc_scene_snapshot(MopCudaScene *s, DrawRec *dst, const std::vector<float> *models) {
  std::lock_guard<std::mutex> lk(s->mu);
  const uint32_t nd = (uint32_t)s->draws.size();
  if (nd)
    memcpy(dst, s->draws.data(), sizeof(DrawRec) * nd);
  if (models && models->size() == 16ull * nd)
    for (uint32_t i = 0; i < nd; i++)
      memcpy(dst[i].model, models->data() + 16ull * i, sizeof dst[i].model);
  mc_ibl_consts(s->ibl_on, s->pf_w, s->pf_h, s->pf_levels, s->brdf_size, dst, nd);
}

std::shared_ptr<const std::vector<float>> mc_scene_models(MopCudaScene *s) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->models || s->models_gen != s->gen || s->models->size() != 16ull * s->draws.size()) {
    auto m = std::make_shared<std::vector<float>>(16ull * s->draws.size());
    for (size_t i = 0; i < s->draws.size(); i++)
      memcpy(m->data() + 16 * i, s->draws[i].model, 16 * sizeof(float));
    s->models = m;
    s->models_gen = s->gen;
  }
  return s->models;
}

void mc_pool_need(uint64_t T, uint64_t V, uint32_t fan_num, uint32_t large_num,
                  unsigned long long need[4]) {
  const unsigned long long fan = T * fan_num / 8ull + 1024ull;
  need[0] = V + fan;
  need[1] = T + fan;
  need[2] = fan;
  need[3] = T * large_num / 16ull + 1024ull;
}

uint64_t mc_view_bytes(const MopCudaScene *s, uint64_t samples, uint64_t pixels) {
  unsigned long long need[4];
  mc_pool_need(s->tris, s->verts, 1, 1, need);
  const uint64_t pools = 64ull * need[0] + (sizeof(RasterRec) + sizeof(ShadeRec)) * need[1] +
                         4ull * need[2] + 8ull * need[3];
  /* an ordered suffix: hdr, list heads and touched samples, a fragment per
   * sample and the suffix-record list */
  const uint64_t suffix =
      s->ordered_tris ? 32ull * samples + (s->wire ? 16ull : 8ull) * (s->ordered_tris + need[2]) +
                            4096ull * 8ull
                      : 0ull;
  return 28ull * samples + 4ull * pixels + pools / 2 + suffix +
         sizeof(DrawRec) * s->draws.size();
}

/* ------------------------------------------------------------------------
 * launch core
 * ------------------------------------------------------------------------ */
int mc_check_view(const MopCudaView &v) {
  if (v.width <= 0 || v.height <= 0 || v.ssaa < 1 || v.ssaa > 4)
    return fail(MOPCUDA_EINVAL, "view: bad size or ssaa");
  if ((uint64_t)v.width * v.ssaa > 32767u || (uint64_t)v.height * v.ssaa > 32767u)
    return fail(MOPCUDA_EINVAL, "view: %dx%d x%d exceeds 32767 samples per side", v.width,
                v.height, v.ssaa);
  return MOPCUDA_OK;
}

static void set_camera(ViewRec &r, const MopCudaView &v) {
  memcpy(r.view, v.view, sizeof r.view);
  memcpy(r.proj, v.proj, sizeof r.proj);
  memcpy(r.eye, v.eye, sizeof r.eye);
  memcpy(r.clear, v.clear, sizeof r.clear);
}

int LaunchCore::init(MopCudaDevice *d) {
  dev = d;
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&ev0) != cudaSuccess || cudaEventCreate(&ev1) != cudaSuccess) {
    cudaGetLastError();
    return fail(MOPCUDA_ECUDA, "launch: stream/event creation failed");
  }
  exposure = d->exposure;
  post_effects = d->post;
  memcpy(lut, d->lut, sizeof lut);
  memcpy(fog, d->fog, sizeof fog);
  return MOPCUDA_OK;
}

int LaunchCore::sync(int timeout_ms) {
  cudaEvent_t e;
  CU_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEventRecord(e, stream);
  int rc = mc_bounded_sync(dev, e, timeout_ms);
  cudaEventDestroy(e);
  return rc;
}

void LaunchCore::release() {
  if (stream)
    sync(10000);
  DevArena *arenas[] = {&d_views, &d_frames, &d_view_draws, &d_ctr, &d_status, &d_posts,
                        &d_post_views, &d_draws, &d_scenes, &clip, &world, &normal, &color,
                        &rrec, &srec, &clipq, &large_list, &large_items, &keys, &shade_list,
                        &pre, &out, &depth, &ids, &presented, &hdr, &frag_head, &touched,
                        &frags, &olist, &olist_items, &wlist, &wlist_items, &oscratch};
  for (DevArena *a : arenas)
    a->release();
  frag_pool = olist_pool = wlist_pool = 0;
  for (EntryShadow &e : shadows) {
    DevArena *sa[] = {&e.map, &e.d_draws, &e.recs, &e.items, &e.ctr};
    for (DevArena *a : sa)
      a->release();
    e.h_draws.release();
  }
  shadows.clear();
  h_views.release();
  h_draws.release();
  h_scenes.release();
  h_status.release();
  if (ev0)
    cudaEventDestroy(ev0);
  if (ev1)
    cudaEventDestroy(ev1);
  if (stream)
    cudaStreamDestroy(stream);
  ev0 = ev1 = nullptr;
  stream = nullptr;
}

void LaunchCore::trim() {
  if (stream)
    sync(10000);
  DevArena *arenas[] = {&clip,       &world, &normal,  &color,      &rrec,      &srec,
                        &clipq,      &large_list, &large_items, &keys, &shade_list, &pre,
                        &out,        &depth, &ids,     &presented,  &hdr,       &frag_head,
                        &touched,    &frags, &olist,   &olist_items, &wlist, &wlist_items,
                        &oscratch};
  for (DevArena *a : arenas)
    a->release();
  vertex_pool = rec_pool = clip_pool = large_pool = 0;
  frag_pool = olist_pool = wlist_pool = 0;
}

uint64_t LaunchCore::device_bytes() const {
  const DevArena *arenas[] = {&d_views, &d_frames, &d_view_draws, &d_ctr, &d_status, &d_posts,
                              &d_post_views, &d_draws, &d_scenes, &clip, &world, &normal, &color,
                              &rrec, &srec, &clipq, &large_list, &large_items, &keys,
                              &shade_list, &pre, &out, &depth, &ids, &presented, &hdr,
                              &frag_head, &touched, &frags, &olist, &olist_items, &wlist,
                              &wlist_items, &oscratch};
  uint64_t t = 0;
  for (const DevArena *a : arenas)
    t += a->cap;
  for (const EntryShadow &e : shadows)
    t += e.map.cap + e.d_draws.cap + e.recs.cap + e.items.cap + e.ctr.cap;
  return t;
}

int LaunchCore::set_layout(const MopCudaView *views, const uint32_t *scene_of,
                           const uint8_t *no_color, uint32_t n,
                           const std::vector<MopCudaScene *> &sc,
                           const std::vector<std::shared_ptr<const std::vector<float>>> *models) {
  if (n == 0 || n > MOPCUDA_MAX_VIEWS)
    return fail(MOPCUDA_EINVAL, "launch: 1..%d views", MOPCUDA_MAX_VIEWS);
  for (uint32_t i = 0; i < n; i++) {
    int rc = mc_check_view(views[i]);
    if (rc)
      return rc;
    if (scene_of[i] >= sc.size())
      return fail(MOPCUDA_EINVAL, "launch: view %u names scene %u of %zu", i, scene_of[i],
                  sc.size());
  }
  nv = n;
  scenes = sc;
  if (models)
    scene_models = *models;
  else
    scene_models.assign(sc.size(), nullptr);
  scene_draw_off.assign(sc.size(), 0);
  if (shadows.size() < sc.size()) /* entries keep their buffers; never shrunk */
    shadows.resize(sc.size());
  total_draws = 0;
  for (size_t k = 0; k < sc.size(); k++) {
    scene_draw_off[k] = total_draws;
    total_draws += sc[k]->draws.size();
  }
  vrec.assign(n, ViewRec());
  posts.assign(n, PostArgs());
  unsigned long long so = 0, po = 0, dro = 0;
  for (uint32_t i = 0; i < n; i++) {
    const MopCudaView &v = views[i];
    ViewRec &r = vrec[i];
    memset(&r, 0, sizeof r);
    set_camera(r, v);
    r.ssaa = v.ssaa;
    r.width = v.width * v.ssaa;
    r.height = v.height * v.ssaa;
    r.scene = scene_of[i];
    r.no_color = no_color && no_color[i] ? 1u : 0u;
    r.sample_off = so;
    r.pixel_off = po;
    r.draw_off = dro;
    /* 16-sample alignment keeps the resolve's vector stores aligned */
    so += ((unsigned long long)r.width * r.height + 15ull) & ~15ull;
    po += ((unsigned long long)v.width * v.height + 15ull) & ~15ull;
    dro += sc[scene_of[i]]->draws.size();
  }
  total_samples = so;
  total_pixels = po;
  view_draw_total = dro;
  int rc = 0;
  const unsigned long long sa = std::max(so, sample_floor), pa = std::max(po, pixel_floor);
  rc |= keys.ensure(8ull * sa);
  rc |= shade_list.ensure(4ull * sa);
  rc |= pre.ensure(4ull * sa);
  rc |= out.ensure(4ull * sa);
  rc |= depth.ensure(4ull * sa);
  rc |= ids.ensure(4ull * sa);
  rc |= presented.ensure(4ull * pa + 16);
  rc |= d_views.ensure(sizeof(ViewRec) * n);
  rc |= h_views.ensure(sizeof(ViewRec) * n);
  rc |= d_frames.ensure(sizeof(FrameArgs) * n);
  rc |= d_ctr.ensure(sizeof(Counters) * n);
  rc |= d_status.ensure(sizeof(BatchStatus));
  rc |= h_status.ensure(sizeof(BatchStatus) + sizeof(Counters) * n);
  rc |= d_posts.ensure(sizeof(PostArgs) * n);
  rc |= d_post_views.ensure(4ull * 4ull * n);
  rc |= d_view_draws.ensure(sizeof(DrawRec) * (dro ? dro : 1));
  rc |= d_draws.ensure(sizeof(DrawRec) * (total_draws ? total_draws : 1));
  rc |= h_draws.ensure(sizeof(DrawRec) * (total_draws ? total_draws : 1));
  rc |= d_scenes.ensure(sizeof(SceneDesc) * sc.size());
  rc |= h_scenes.ensure(sizeof(SceneDesc) * sc.size());
  if (rc)
    return MOPCUDA_ENOMEM;
  PostArgs post;
  mc_post_template(post_effects, lut, fog, post);
  std::vector<uint32_t> lists(4ull * n, 0u);
  for (int k = 0; k < 4; k++)
    post_count[k] = post_tiles[k] = 0;
  for (uint32_t i = 0; i < n; i++) {
    const ViewRec &r = vrec[i];
    PostArgs p = post;
    p.pre = pre.as<uchar4>() + r.sample_off;
    p.out = out.as<uchar4>() + r.sample_off;
    p.presented = r.ssaa > 1 ? presented.as<uchar4>() + r.pixel_off : nullptr;
    p.depth = depth.as<float>() + r.sample_off;
    p.width = r.width;
    p.height = r.height;
    p.ssaa = r.ssaa;
    posts[i] = p;
    if (r.no_color)
      continue; /* visibility only: no post effects */
    const int k = r.ssaa - 1;
    lists[(size_t)k * n + post_count[k]++] = i;
    const uint32_t pw = (uint32_t)(r.width / r.ssaa), ph = (uint32_t)(r.height / r.ssaa);
    post_tiles[k] += ((pw + 31u) / 32u) * ((ph + 7u) / 8u);
  }
  CU_TRY(cudaMemcpyAsync(d_posts.p, posts.data(), sizeof(PostArgs) * n, cudaMemcpyHostToDevice,
                         stream));
  CU_TRY(cudaMemcpyAsync(d_post_views.p, lists.data(), 4ull * 4ull * n, cudaMemcpyHostToDevice,
                         stream));
  return sync(FRAME_TIMEOUT_MS); /* pageable sources: finish before they go */
}

static int size_pools(LaunchCore *b, unsigned long long vneed, unsigned long long rneed,
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

/* Entry k's shadow pass for this launch (pass_shadow, viewport.c:2288-2442):
 * the light camera from its casters' model matrices as of the launch, every
 * caster's light view-projection * model, the caster table staged in
 * page-locked memory; the entry's SceneDesc names the map. */
int LaunchCore::stage_shadow(size_t k, const DrawRec *dr, SceneDesc &d) {
  EntryShadow &e = shadows[k];
  const MopCudaScene *sc = scenes[k];
  const int old_size = e.size;
  const uint32_t old_casters = e.casters;
  e.size = 0;
  e.casters = 0;
  e.tris = 0;
  if (sc->sh_size > 0) {
    std::vector<uint32_t> idx;
    std::vector<float> models;
    for (uint32_t i = 0; i < (uint32_t)sc->draws.size(); i++) {
      const DrawRec &r = dr[i];
      /* casters: every opaque draw below the editor-chrome IDs
       * (viewport.c:2310-2317); empty slots hold dropped draws */
      if (r.vertex_count == 0 || r.index_count < 3u || r.object_id >= 0xFFFD0000u ||
          r.blend_mode != 0)
        continue;
      idx.push_back(i);
      models.insert(models.end(), r.model, r.model + 16);
    }
    float vp[16];
    if (!idx.empty() && mopcuda_shadow_light_vp(models.data(), (uint32_t)idx.size(), sc->sh_dir, vp)) {
      std::vector<ShadowDraw> cas(idx.size());
      uint64_t T = 0;
      for (size_t j = 0; j < idx.size(); j++) {
        const DrawRec &r = dr[idx[j]];
        ShadowDraw &c = cas[j];
        const bool flex = (r.flags & DF_FLEX) != 0;
        c.verts = r.vbuf + (flex ? r.off_pos : 0);
        c.idx = r.ibuf;
        c.vertex_count = r.vertex_count;
        c.stride = flex ? r.stride : 48u;
        c.tri_count = r.index_count / 3u;
        c.tri_off = (uint32_t)T;
        mc_mat4_mul(vp, r.model, c.mvp); /* mop_mat4_multiply(light_vp, model) */
        T += c.tri_count;
      }
      if (T >= (1ull << 31))
        return fail(MOPCUDA_EINVAL, "scene shadow pass too large: %llu triangles",
                    (unsigned long long)T);
      const size_t S = (size_t)sc->sh_size, n = cas.size();
      void *before[6] = {e.map.p, e.d_draws.p, e.recs.p, e.items.p, e.ctr.p, e.h_draws.p};
      int rc = 0;
      rc |= e.map.ensure(4 * S * S + 64);
      rc |= e.d_draws.ensure(sizeof(ShadowDraw) * n);
      rc |= e.recs.ensure(sizeof(ShadowRec) * (size_t)T);
      rc |= e.items.ensure(8 * (size_t)T);
      rc |= e.ctr.ensure(sizeof(ShadowCounters));
      rc |= e.h_draws.ensure(sizeof(ShadowDraw) * n + 64);
      if (rc)
        return MOPCUDA_ENOMEM;
      void *after[6] = {e.map.p, e.d_draws.p, e.recs.p, e.items.p, e.ctr.p, e.h_draws.p};
      if (memcmp(before, after, sizeof before) != 0)
        shadow_moved = true;
      memcpy(e.h_draws.p, cas.data(), sizeof(ShadowDraw) * n);
      memcpy(e.h_draws.as<uint8_t>() + sizeof(ShadowDraw) * n, vp, 64);
      e.size = (int)S;
      e.casters = (uint32_t)n;
      e.tris = T;
      d.shadow_keys = e.map.as<uint32_t>();
      d.shadow_vp = (const float *)(e.map.as<uint8_t>() + 4 * S * S);
      d.shadow_size = (int)S;
    }
  }
  if (e.size != old_size || e.casters != old_casters)
    shadow_moved = true; /* the captured launch no longer matches */
  return MOPCUDA_OK;
}

int LaunchCore::stage() {
  SceneDesc *sd = h_scenes.as<SceneDesc>();
  DrawRec *hd = h_draws.as<DrawRec>();
  for (size_t k = 0; k < scenes.size(); k++) {
    MopCudaScene *s = scenes[k];
    int rc = mc_scene_sync(s);
    if (rc)
      return rc;
    mc_scene_snapshot(s, hd + scene_draw_off[k], scene_models[k].get());
    SceneDesc &d = sd[k];
    memset(&d, 0, sizeof d);
    d.draws = d_draws.as<DrawRec>() + scene_draw_off[k];
    d.bounds = s->d_bounds.as<DrawBound>();
    d.nd = (uint32_t)s->draws.size();
    d.lights = s->d_lights.as<LightRec>();
    d.light_total = (uint32_t)s->lights.size();
    if (s->ibl_on) {
      d.irr = s->irr.as<float>();
      d.irr_w = s->irr_w;
      d.irr_h = s->irr_h;
      d.pf = s->pf.as<float>();
      d.pf_w = s->pf_w;
      d.pf_h = s->pf_h;
      d.pf_levels = s->pf_levels;
      d.brdf = s->brdf.as<float>();
      d.brdf_size = s->brdf_size;
      d.ibl_rotation = s->ibl_rot;
      d.ibl_intensity = s->ibl_int;
    }
    if ((rc = stage_shadow(k, hd + scene_draw_off[k], d)))
      return rc;
  }
  any_shadow = false;
  for (size_t k = 0; k < scenes.size(); k++)
    any_shadow |= shadows[k].size > 0;
  memcpy(h_views.p, vrec.data(), sizeof(ViewRec) * nv);
  /* first pools: half the worst case (every draw visible in every view) */
  unsigned long long want[4] = {0, 0, 0, 0};
  for (uint32_t i = 0; i < nv; i++) {
    const MopCudaScene *s = scenes[vrec[i].scene];
    unsigned long long need[4];
    mc_pool_need(s->tris, s->verts, fan_num, large_num, need);
    for (int k = 0; k < 4; k++)
      want[k] += need[k];
  }
  for (int k = 0; k < 4; k++)
    want[k] = std::max(want[k] / 2 + 4096, pool_floor[k]);
  int rc = stage_suffix();
  if (rc)
    return rc;
  if (vertex_pool < want[0] || rec_pool < want[1] || clip_pool < want[2] ||
      large_pool < want[3])
    return size_pools(this, std::max(want[0], vertex_pool), std::max(want[1], rec_pool),
                      std::max(want[2], clip_pool), std::max(want[3], large_pool));
  return MOPCUDA_OK;
}

/* The ordered suffix's buffers when a scene entry of the launch has
 * order-dependent draws: composition colour, list heads and touched samples
 * per sample; the suffix-record and fragment pools sized for every viewport
 * of such a scene (the device reports larger needs, after() grows them). */
int LaunchCore::stage_suffix() {
  any_ordered = false;
  for (const MopCudaScene *s : scenes)
    any_ordered |= s->ordered_tris > 0;
  if (!any_ordered)
    return MOPCUDA_OK;
  unsigned long long ol = 0, fr = 0, wl = 0;
  any_wire = false;
  for (uint32_t i = 0; i < nv; i++) {
    const MopCudaScene *s = scenes[vrec[i].scene];
    if (!s->ordered_tris)
      continue;
    unsigned long long need[4];
    mc_pool_need(s->tris, s->verts, fan_num, large_num, need);
    ol += s->ordered_tris + need[2];
    fr += (unsigned long long)vrec[i].width * vrec[i].height * frag_num / 4ull + 4096ull;
    if (s->wire) {
      any_wire = true;
      wl += s->ordered_tris + need[2];
    }
  }
  const unsigned long long sa = std::max(total_samples, sample_floor);
  void *before[9] = {hdr.p, frag_head.p, touched.p, frags.p, olist.p, olist_items.p,
                     wlist.p, wlist_items.p, oscratch.p};
  int rc = 0;
  rc |= hdr.ensure(16ull * sa);
  rc |= frag_head.ensure(4ull * sa);
  rc |= touched.ensure(4ull * sa);
  if (olist_pool < ol) {
    rc |= olist.ensure(4ull * ol);
    rc |= olist_items.ensure(4ull * ol);
  }
  if (frag_pool < fr) {
    rc |= frags.ensure(8ull * fr);
    rc |= oscratch.ensure(16ull * fr);
  }
  if (any_wire && wlist_pool < wl) {
    rc |= wlist.ensure(4ull * wl);
    rc |= wlist_items.ensure(4ull * wl);
  }
  if (rc)
    return MOPCUDA_ENOMEM;
  olist_pool = std::min(olist.cap / 4, olist_items.cap / 4);
  frag_pool = std::min(frags.cap / 8, oscratch.cap / 16);
  wlist_pool = std::min(wlist.cap / 4, wlist_items.cap / 4);
  void *after_[9] = {hdr.p, frag_head.p, touched.p, frags.p, olist.p, olist_items.p,
                     wlist.p, wlist_items.p, oscratch.p};
  if (memcmp(before, after_, sizeof before) != 0)
    suffix_moved = true;
  return MOPCUDA_OK;
}

int LaunchCore::enqueue(int parts) {
  BatchLaunch L;
  memset(&L, 0, sizeof L);
  L.num_sms = dev->num_sms;
  L.vertex_block = cfg.vertex_block;
  L.setup_block = cfg.setup_block;
  L.raster_block = cfg.raster_block;
  L.large_block = cfg.large_block;
  L.shade_block = cfg.shade_block;
  L.grid_mul = cfg.grid_mul;
  mopcuda_batch_grids(L);

  BatchArgs a;
  memset(&a, 0, sizeof a);
  a.scenes = d_scenes.as<SceneDesc>();
  a.views = d_views.as<ViewRec>();
  a.nv = nv;
  a.frames = d_frames.as<FrameArgs>();
  a.view_draws = d_view_draws.as<DrawRec>();
  a.ctr = d_ctr.as<Counters>();
  a.status = d_status.as<BatchStatus>();
  a.tmpl.exposure = exposure;
  a.tmpl.small_side = cfg.small_side;
  a.tmpl.small_area = cfg.small_area;
  a.clip = clip.as<float4>();
  a.world = world.as<float4>();
  a.normal = normal.as<float4>();
  a.color = color.as<float4>();
  a.vertex_pool = vertex_pool;
  a.rrec = rrec.as<RasterRec>();
  a.srec = srec.as<ShadeRec>();
  a.rec_pool = rec_pool;
  a.clipq = clipq.as<uint32_t>();
  a.clip_pool = clip_pool;
  a.large_list = large_list.as<uint32_t>();
  a.large_items = large_items.as<uint32_t>();
  a.large_pool = large_pool;
  a.keys = keys.as<unsigned long long>();
  a.shade_list = shade_list.as<uint32_t>();
  a.pre = pre.as<uchar4>();
  a.depth = depth.as<float>();
  a.ids = ids.as<uint32_t>();
  a.fan_num = fan_num;
  a.large_num = large_num;
  a.frag_num = frag_num;
  a.samples = total_samples;
  if (any_ordered) {
    a.hdr = hdr.as<float4>();
    a.frag_head = frag_head.as<uint32_t>();
    a.touched = touched.as<uint32_t>();
    a.frags = frags.as<uint2>();
    a.frag_pool = frag_pool;
    a.olist = olist.as<uint32_t>();
    a.olist_items = olist_items.as<uint32_t>();
    a.olist_pool = olist_pool;
    a.oscratch = oscratch.as<ulonglong2>();
    a.oscratch_count = &d_status.as<BatchStatus>()->scratch_count;
    if (any_wire) {
      a.wlist = wlist.as<uint32_t>();
      a.wlist_items = wlist_items.as<uint32_t>();
      a.wlist_pool = wlist_pool;
    }
  }

  const uint32_t *pv[4];
  for (int k = 0; k < 4; k++)
    pv[k] = d_post_views.as<uint32_t>() + (size_t)k * nv;
  cudaStream_t s = stream;
  if (parts & BATCH_PART_MAIN) {
    CU_TRY(cudaMemcpyAsync(d_views.p, h_views.p, sizeof(ViewRec) * nv, cudaMemcpyHostToDevice,
                           s));
    if (total_draws)
      CU_TRY(cudaMemcpyAsync(d_draws.p, h_draws.p, sizeof(DrawRec) * total_draws,
                             cudaMemcpyHostToDevice, s));
    CU_TRY(cudaMemcpyAsync(d_scenes.p, h_scenes.p, sizeof(SceneDesc) * scenes.size(),
                           cudaMemcpyHostToDevice, s));
    CU_TRY(cudaMemsetAsync(d_ctr.p, 0, sizeof(Counters) * nv, s));
    CU_TRY(cudaMemsetAsync(d_status.p, 0, sizeof(BatchStatus), s));
    CU_TRY(cudaMemsetAsync(keys.p, 0xff, 8ull * total_samples, s));
  }
  uint64_t sh_launches = 0;
  if (parts & BATCH_PART_MAIN)
    for (size_t k = 0; k < scenes.size(); k++) {
      EntryShadow &e = shadows[k];
      if (!e.size)
        continue;
      const size_t S = (size_t)e.size, db = sizeof(ShadowDraw) * e.casters;
      CU_TRY(cudaMemcpyAsync(e.d_draws.p, e.h_draws.p, db, cudaMemcpyHostToDevice, s));
      CU_TRY(cudaMemcpyAsync(e.map.as<uint8_t>() + 4 * S * S, e.h_draws.as<uint8_t>() + db, 64,
                             cudaMemcpyHostToDevice, s));
      /* cleared to 1.0 (viewport.c:2370-2373): the key 0xffffffff */
      CU_TRY(cudaMemsetAsync(e.map.p, 0xff, 4 * S * S, s));
      CU_TRY(cudaMemsetAsync(e.ctr.p, 0, sizeof(ShadowCounters), s));
      ShadowArgs sa;
      sa.draws = e.d_draws.as<ShadowDraw>();
      sa.draw_count = e.casters;
      sa.tri_total = (uint32_t)e.tris;
      sa.map = e.map.as<uint32_t>();
      sa.size = (int)S;
      sa.small_area = SHADOW_SMALL_AREA;
      sa.recs = e.recs.as<ShadowRec>();
      sa.items = e.items.as<unsigned long long>();
      sa.ctr = e.ctr.as<ShadowCounters>();
      sa.num_sms = dev->num_sms;
      sh_launches += (uint64_t)mopcuda_launch_shadow(sa, s);
    }
  launches = sh_launches +
             (uint64_t)mopcuda_launch_batch(a, d_posts.as<PostArgs>(), pv, post_count, post_tiles,
                                            L, scenes.size() == 1, any_shadow, any_ordered, s,
                                            parts);
  CU_TRY(cudaGetLastError());
  if (parts & BATCH_PART_POST) { /* status after the last kernel: read at completion */
    CU_TRY(cudaMemcpyAsync(h_status.p, d_status.p, sizeof(BatchStatus), cudaMemcpyDeviceToHost,
                           s));
    CU_TRY(cudaMemcpyAsync(h_status.as<uint8_t>() + sizeof(BatchStatus), d_ctr.p,
                           sizeof(Counters) * nv, cudaMemcpyDeviceToHost, s));
  }
  return MOPCUDA_OK;
}

int LaunchCore::after(bool *rerun, int attempt) {
  *rerun = false;
  const BatchStatus *st = h_status.as<BatchStatus>();
  const Counters *ctr = (const Counters *)(h_status.as<uint8_t>() + sizeof(BatchStatus));
  uint32_t view_over = 0;
  for (uint32_t i = 0; i < nv; i++)
    view_over |= ctr[i].overflow;
  if (!st->overflow && !view_over)
    return MOPCUDA_OK;
  if (view_over & 512u)
    return fail(MOPCUDA_EUNSUPPORTED,
                "launch: a viewport's large-triangle raster items exceed 2^32");
  if (attempt >= 8)
    return fail(MOPCUDA_ENOMEM, "launch pools overflowed repeatedly (flags %u/%u)", st->overflow,
                view_over);
  if (view_over & 7u) { /* a viewport's clipped fans: records, vertices, clip queue */
    if (fan_num >= 256u)
      return fail(MOPCUDA_ENOMEM, "launch: clipped-fan reserve exhausted");
    fan_num *= 2u;
  }
  if (view_over & 8u) {
    if (large_num >= 512u)
      return fail(MOPCUDA_ENOMEM, "launch: large-record list exhausted");
    large_num *= 2u;
  }
  if (view_over & 32u) { /* a viewport's suffix-record list: the fan reserve */
    if (fan_num >= 256u)
      return fail(MOPCUDA_ENOMEM, "launch: suffix-record list exhausted");
    fan_num *= 2u;
  }
  if (view_over & 128u) { /* a viewport's wireframe-record list: the fan reserve */
    if (fan_num >= 256u)
      return fail(MOPCUDA_ENOMEM, "launch: wireframe-record list exhausted");
    fan_num *= 2u;
  }
  if (view_over & 16u) { /* a viewport's fragments: its counter holds the demand */
    if (frag_num >= (1u << 20))
      return fail(MOPCUDA_ENOMEM, "launch: blended-fragment reserve exhausted");
    unsigned long long want = 2ull * frag_num;
    for (uint32_t i = 0; i < nv; i++) {
      if (!(ctr[i].overflow & 16u))
        continue;
      const unsigned long long S = (unsigned long long)vrec[i].width * vrec[i].height;
      const unsigned long long need = 4ull * ctr[i].frag_count / (S ? S : 1ull) + 1ull;
      want = std::max(want, need + need / 4);
    }
    while (frag_num < want && frag_num < (1u << 20))
      frag_num *= 2u;
  }
  if (st->overflow & 256u)
    return fail(MOPCUDA_ENOMEM, "launch: a viewport has an ordered suffix but the launch has "
                                "no suffix buffers");
  if (view_over & (16u | 32u | 128u)) { /* the reserves grew: pools to match */
    int rc = stage_suffix();
    if (rc)
      return rc;
  }
  if (st->overflow & 112u) { /* the suffix pools */
    const unsigned long long ol = st->need_olist + st->need_olist / 4 + 4096ull;
    const unsigned long long fr = st->need_frag + st->need_frag / 4 + 4096ull;
    const unsigned long long wl = st->need_wlist + st->need_wlist / 4 + 4096ull;
    int rc = 0;
    if ((st->overflow & 64u) && wl > wlist_pool) {
      rc |= wlist.ensure(4ull * wl);
      rc |= wlist_items.ensure(4ull * wl);
      wlist_pool = std::min(wlist.cap / 4, wlist_items.cap / 4);
    }
    if ((st->overflow & 16u) && ol > olist_pool) {
      rc |= olist.ensure(4ull * ol);
      rc |= olist_items.ensure(4ull * ol);
      olist_pool = std::min(olist.cap / 4, olist_items.cap / 4);
    }
    if ((st->overflow & 32u) && fr > frag_pool) {
      rc |= frags.ensure(8ull * fr);
      rc |= oscratch.ensure(16ull * fr);
      frag_pool = std::min(frags.cap / 8, oscratch.cap / 16);
    }
    if (rc)
      return MOPCUDA_ENOMEM;
  }
  if (st->overflow & 15u) {
    const unsigned long long need[4] = {st->need_vertex, st->need_rec, st->need_clip,
                                        st->need_large};
    unsigned long long cap[4] = {vertex_pool, rec_pool, clip_pool, large_pool};
    for (int k = 0; k < 4; k++)
      if (need[k] > cap[k])
        cap[k] = need[k] + need[k] / 4 + 4096ull;
    int rc = size_pools(this, cap[0], cap[1], cap[2], cap[3]);
    if (rc)
      return rc;
  }
  *rerun = true;
  return MOPCUDA_OK;
}

/* ------------------------------------------------------------------------
 * batch: one LaunchCore over one scene, captured as a CUDA graph
 * ------------------------------------------------------------------------ */
/* One device-to-host copy of an asynchronous colour readback. */
struct RbCopy {
  void *dst;
  const void *src;
  size_t n;
};

struct MopCudaBatch {
  MopCudaScene *scene = nullptr;
  LaunchCore core;
  uint64_t scene_version = ~0ull;
  /* a launch is two graphs: every stage up to shading, then the post passes
   * (which write the colour images) and the status copies */
  cudaGraph_t graph = nullptr, graph_post = nullptr;
  cudaGraphExec_t exec = nullptr, exec_post = nullptr;
  bool pending = false;
  /* asynchronous colour readback of the last completed launch: the copies
   * wait in rb_copies until the next launch's first graph is queued (queued
   * before it, they held back its uploads), run on copy_stream, and that
   * launch's post graph waits for rb_done */
  std::vector<RbCopy> rb_copies;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t rb_done = nullptr;
  bool rb_live = false;
  float last_ms = 0.0f;
  DevArena pick_xy, pick_out;
  HostArena h_pick;
  std::mutex mu;
};

static void drop_graph(MopCudaBatch *b) {
  if (b->exec)
    cudaGraphExecDestroy(b->exec);
  if (b->graph)
    cudaGraphDestroy(b->graph);
  if (b->exec_post)
    cudaGraphExecDestroy(b->exec_post);
  if (b->graph_post)
    cudaGraphDestroy(b->graph_post);
  b->exec = b->exec_post = nullptr;
  b->graph = b->graph_post = nullptr;
}

/* Queues the recorded readback copies on the copy stream (the launch they
 * read has completed). */
static int issue_readback(MopCudaBatch *b) {
  if (b->rb_copies.empty())
    return MOPCUDA_OK;
  if (!b->copy_stream) {
    CU_TRY(cudaStreamCreateWithFlags(&b->copy_stream, cudaStreamNonBlocking));
    CU_TRY(cudaEventCreateWithFlags(&b->rb_done, cudaEventDisableTiming));
  }
  std::vector<RbCopy> copies;
  copies.swap(b->rb_copies);
  for (const RbCopy &c : copies)
    CU_TRY(cudaMemcpyAsync(c.dst, c.src, c.n, cudaMemcpyDeviceToHost, b->copy_stream));
  CU_TRY(cudaEventRecord(b->rb_done, b->copy_stream));
  b->rb_live = true;
  return MOPCUDA_OK;
}

/* The readback queued and complete (before the images' memory is freed or
 * moved). */
static int drain_readback(MopCudaBatch *b, int timeout_ms) {
  int rc = issue_readback(b);
  if (rc)
    return rc;
  if (!b->rb_live)
    return MOPCUDA_OK;
  rc = mc_bounded_sync(b->core.dev, b->rb_done, timeout_ms);
  if (!rc)
    b->rb_live = false;
  return rc;
}

extern "C" void mopcuda_batch_destroy(MopCudaBatch *b) {
  if (!b)
    return;
  cudaSetDevice(b->core.dev->ordinal);
  if (b->core.stream)
    b->core.sync(10000);
  b->rb_copies.clear();
  if (b->copy_stream) {
    if (b->rb_live)
      mc_bounded_sync(b->core.dev, b->rb_done, 10000);
    cudaEventDestroy(b->rb_done);
    cudaStreamDestroy(b->copy_stream);
  }
  drop_graph(b);
  b->pick_xy.release();
  b->pick_out.release();
  b->h_pick.release();
  b->core.release();
  delete b;
}

extern "C" MopCudaBatch *mopcuda_batch_create(MopCudaScene *scene, const MopCudaView *views,
                                              uint32_t n) {
  if (!scene || !views || n == 0 || n > MOPCUDA_MAX_VIEWS) {
    fail(MOPCUDA_EINVAL, "batch_create: need a scene and 1..%d views", MOPCUDA_MAX_VIEWS);
    return nullptr;
  }
  MopCudaDevice *d = scene->dev;
  cudaSetDevice(d->ordinal);
  MopCudaBatch *b = new MopCudaBatch();
  b->scene = scene;
  if (b->core.init(d)) {
    mopcuda_batch_destroy(b);
    return nullptr;
  }
  std::vector<uint32_t> scene_of(n, 0u);
  std::vector<MopCudaScene *> sc = {scene};
  if (b->core.set_layout(views, scene_of.data(), nullptr, n, sc)) {
    mopcuda_batch_destroy(b);
    return nullptr;
  }
  b->scene_version = scene->version;
  return b;
}

extern "C" int mopcuda_batch_set_views(MopCudaBatch *b, const MopCudaView *views, uint32_t n) {
  if (!b || !views || n != b->core.nv)
    return fail(MOPCUDA_EINVAL, "batch_set_views: need %u views", b ? b->core.nv : 0u);
  std::lock_guard<std::mutex> lk(b->mu);
  for (uint32_t i = 0; i < n; i++) {
    const ViewRec &r = b->core.vrec[i];
    if (views[i].ssaa != r.ssaa || views[i].width * views[i].ssaa != r.width ||
        views[i].height * views[i].ssaa != r.height)
      return fail(MOPCUDA_EINVAL, "batch_set_views: view %u changed size or ssaa", i);
  }
  for (uint32_t i = 0; i < n; i++)
    set_camera(b->core.vrec[i], views[i]);
  return MOPCUDA_OK;
}

static int capture_part(MopCudaBatch *b, int part, cudaGraph_t *graph, cudaGraphExec_t *exec,
                        uint64_t *launches) {
  LaunchCore &c = b->core;
  CU_TRY(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
  int rc = c.enqueue(part);
  cudaError_t e = cudaStreamEndCapture(c.stream, graph);
  if (rc || e != cudaSuccess) {
    cudaGetLastError();
    if (*graph)
      cudaGraphDestroy(*graph);
    *graph = nullptr;
    return rc ? rc : fail(MOPCUDA_ECUDA, "batch graph capture: %s", cudaGetErrorString(e));
  }
  e = cudaGraphInstantiate(exec, *graph, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(MOPCUDA_ECUDA, "batch graph instantiate: %s", cudaGetErrorString(e));
  }
  *launches += c.launches;
  return MOPCUDA_OK;
}

static int build_graph(MopCudaBatch *b) {
  drop_graph(b);
  uint64_t launches = 0;
  int rc = capture_part(b, BATCH_PART_MAIN, &b->graph, &b->exec, &launches);
  if (!rc)
    rc = capture_part(b, BATCH_PART_POST, &b->graph_post, &b->exec_post, &launches);
  if (rc) {
    drop_graph(b);
    return rc;
  }
  b->core.launches = launches;
  return MOPCUDA_OK;
}

static int launch_graph(MopCudaBatch *b) {
  cudaStream_t s = b->core.stream;
  CU_TRY(cudaEventRecord(b->core.ev0, s));
  CU_TRY(cudaGraphLaunch(b->exec, s));
  /* the previous launch's images go to the host while this one renders;
   * its post passes overwrite them only once they are there */
  const int rrc = issue_readback(b);
  if (b->rb_live)
    CU_TRY(cudaStreamWaitEvent(s, b->rb_done, 0));
  CU_TRY(cudaGraphLaunch(b->exec_post, s));
  CU_TRY(cudaEventRecord(b->core.ev1, s));
  b->pending = true;
  return rrc;
}

/* Waits; re-runs after growing a viewport's reserves or the pools. */
static int finish_batch(MopCudaBatch *b, int timeout_ms) {
  for (int attempt = 0; b->pending; attempt++) {
    int rc = mc_bounded_sync(b->core.dev, b->core.ev1, timeout_ms);
    b->pending = false;
    if (rc)
      return rc;
    cudaEventElapsedTime(&b->last_ms, b->core.ev0, b->core.ev1);
    bool rerun = false;
    rc = b->core.after(&rerun, attempt);
    if (rc)
      return rc;
    if (!rerun)
      break;
    rc = build_graph(b);
    if (rc)
      return rc;
    rc = launch_graph(b);
    if (rc)
      return rc;
  }
  return MOPCUDA_OK;
}

static int submit_locked(MopCudaBatch *b) {
  cudaSetDevice(b->core.dev->ordinal);
  int rc = finish_batch(b, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  if (b->scene->version != b->scene_version) { /* draws were added: new table sizes */
    /* the buffers may move: a pending readback runs to completion first */
    if ((rc = drain_readback(b, FRAME_TIMEOUT_MS)))
      return rc;
    LaunchCore &c = b->core;
    std::vector<uint32_t> scene_of(c.nv, 0u);
    std::vector<MopCudaView> views(c.nv);
    for (uint32_t i = 0; i < c.nv; i++) {
      const ViewRec &r = c.vrec[i];
      MopCudaView &v = views[i];
      memcpy(v.view, r.view, sizeof v.view);
      memcpy(v.proj, r.proj, sizeof v.proj);
      memcpy(v.eye, r.eye, sizeof v.eye);
      memcpy(v.clear, r.clear, sizeof v.clear);
      v.width = r.width / r.ssaa;
      v.height = r.height / r.ssaa;
      v.ssaa = r.ssaa;
    }
    std::vector<MopCudaScene *> sc = {b->scene};
    rc = c.set_layout(views.data(), scene_of.data(), nullptr, c.nv, sc);
    if (rc)
      return rc;
    b->scene_version = b->scene->version;
    drop_graph(b);
  }
  const unsigned long long pools[4] = {b->core.vertex_pool, b->core.rec_pool, b->core.clip_pool,
                                       b->core.large_pool};
  b->core.shadow_moved = b->core.suffix_moved = false;
  rc = b->core.stage();
  if (rc)
    return rc;
  if (pools[0] != b->core.vertex_pool || pools[1] != b->core.rec_pool ||
      pools[2] != b->core.clip_pool || pools[3] != b->core.large_pool ||
      b->core.shadow_moved || b->core.suffix_moved)
    drop_graph(b); /* the pools, the suffix buffers or the shadow passes moved */
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

extern "C" int mopcuda_batch_wait(MopCudaBatch *b, int timeout_ms) {
  if (!b)
    return fail(MOPCUDA_EINVAL, "batch_wait: no batch");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->core.dev->ordinal);
  return finish_batch(b, timeout_ms);
}

extern "C" float mopcuda_batch_gpu_time_ms(const MopCudaBatch *b) { return b ? b->last_ms : 0.0f; }

/* Where viewport `view`'s buffer `what` lives on the device, and its size. */
static int view_buffer(const LaunchCore &c, uint32_t view, int what, const void **src,
                       size_t *n) {
  const ViewRec &r = c.vrec[view];
  const size_t S = (size_t)r.width * r.height;
  const size_t P = (size_t)(r.width / r.ssaa) * (r.height / r.ssaa);
  switch (what) {
  case MOPCUDA_BATCH_COLOR:
    *src = c.out.as<uchar4>() + r.sample_off;
    *n = 4 * S;
    return MOPCUDA_OK;
  case MOPCUDA_BATCH_PRESENTED:
    *src = r.ssaa > 1 ? (const void *)(c.presented.as<uchar4>() + r.pixel_off)
                      : (const void *)(c.out.as<uchar4>() + r.sample_off);
    *n = 4 * P;
    return MOPCUDA_OK;
  case MOPCUDA_BATCH_DEPTH:
    *src = c.depth.as<float>() + r.sample_off;
    *n = 4 * S;
    return MOPCUDA_OK;
  case MOPCUDA_BATCH_IDS:
    *src = c.ids.as<uint32_t>() + r.sample_off;
    *n = 4 * S;
    return MOPCUDA_OK;
  default:
    return fail(MOPCUDA_EINVAL, "batch_read: unknown buffer %d", what);
  }
}

extern "C" int mopcuda_batch_read(MopCudaBatch *b, uint32_t view, int what, void *dst,
                                  size_t bytes) {
  return mopcuda_batch_read_views(b, view, 1, what, &dst, &bytes);
}

extern "C" int mopcuda_batch_read_views(MopCudaBatch *b, uint32_t first, uint32_t count,
                                        int what, void *const *dsts, const size_t *bytes) {
  if (!b || !dsts || !bytes || count == 0 || first >= b->core.nv ||
      count > b->core.nv - first)
    return fail(MOPCUDA_EINVAL, "batch_read: bad arguments");
  for (uint32_t i = 0; i < count; i++)
    if (!dsts[i])
      return fail(MOPCUDA_EINVAL, "batch_read: bad arguments");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->core.dev->ordinal);
  int rc = finish_batch(b, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  const LaunchCore &c = b->core;
  /* every size is checked before the first copy is queued */
  for (uint32_t i = 0; i < count; i++) {
    const void *src;
    size_t n;
    if ((rc = view_buffer(c, first + i, what, &src, &n)))
      return rc;
    if (bytes[i] != n)
      return fail(MOPCUDA_EINVAL, "batch_read: buffer is %zu bytes, not %zu", n, bytes[i]);
  }
  for (uint32_t i = 0; i < count; i++) {
    const void *src;
    size_t n;
    view_buffer(c, first + i, what, &src, &n);
    CU_TRY(cudaMemcpyAsync(dsts[i], src, n, cudaMemcpyDeviceToHost, c.stream));
  }
  return b->core.sync(FRAME_TIMEOUT_MS);
}

extern "C" int mopcuda_batch_read_views_async(MopCudaBatch *b, uint32_t first, uint32_t count,
                                              int what, void *const *dsts,
                                              const size_t *bytes) {
  if (!b || !dsts || !bytes || count == 0 || first >= b->core.nv ||
      count > b->core.nv - first)
    return fail(MOPCUDA_EINVAL, "batch_read_views_async: bad arguments");
  if (what != MOPCUDA_BATCH_COLOR && what != MOPCUDA_BATCH_PRESENTED)
    return fail(MOPCUDA_EINVAL, "batch_read_views_async: colour buffers only (got %d)", what);
  for (uint32_t i = 0; i < count; i++)
    if (!dsts[i])
      return fail(MOPCUDA_EINVAL, "batch_read_views_async: bad arguments");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->core.dev->ordinal);
  int rc = finish_batch(b, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  const LaunchCore &c = b->core;
  std::vector<RbCopy> copies(count);
  for (uint32_t i = 0; i < count; i++) {
    if ((rc = view_buffer(c, first + i, what, &copies[i].src, &copies[i].n)))
      return rc;
    if (bytes[i] != copies[i].n)
      return fail(MOPCUDA_EINVAL, "batch_read_views_async: buffer is %zu bytes, not %zu",
                  copies[i].n, bytes[i]);
    copies[i].dst = dsts[i];
  }
  /* copies recorded earlier for this launch go first */
  if ((rc = issue_readback(b)))
    return rc;
  b->rb_copies.swap(copies);
  return MOPCUDA_OK;
}

extern "C" int mopcuda_batch_readback_wait(MopCudaBatch *b, int timeout_ms) {
  if (!b)
    return fail(MOPCUDA_EINVAL, "batch_readback_wait: no batch");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->core.dev->ordinal);
  return drain_readback(b, timeout_ms);
}

extern "C" int mopcuda_batch_pick(MopCudaBatch *b, uint32_t view, const int32_t *xy, uint32_t n,
                                  uint32_t *ids, float *depths, int32_t *hits) {
  if (!b || view >= b->core.nv || (n && (!xy || !ids || !depths || !hits)))
    return fail(MOPCUDA_EINVAL, "batch_pick: bad arguments");
  if (n == 0)
    return MOPCUDA_OK;
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->core.dev->ordinal);
  int rc = finish_batch(b, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  size_t in_b = 8ull * n, out_b = 12ull * n;
  if (b->pick_xy.ensure(in_b) || b->pick_out.ensure(out_b) || b->h_pick.ensure(in_b + out_b))
    return MOPCUDA_ENOMEM;
  memcpy(b->h_pick.p, xy, in_b);
  LaunchCore &c = b->core;
  cudaStream_t s = c.stream;
  CU_TRY(cudaMemcpyAsync(b->pick_xy.p, b->h_pick.p, in_b, cudaMemcpyHostToDevice, s));
  uint32_t *oid = b->pick_out.as<uint32_t>();
  float *odp = (float *)(oid + n);
  int32_t *oht = (int32_t *)(odp + n);
  const ViewRec &r = c.vrec[view];
  mopcuda_launch_pick(c.ids.as<uint32_t>() + r.sample_off, c.depth.as<float>() + r.sample_off,
                      r.width, r.height, r.ssaa, b->pick_xy.as<int2>(), n, oid, odp, oht, s);
  CU_TRY(cudaGetLastError());
  uint8_t *hb = b->h_pick.as<uint8_t>() + in_b;
  CU_TRY(cudaMemcpyAsync(hb, b->pick_out.p, out_b, cudaMemcpyDeviceToHost, s));
  rc = c.sync(FRAME_TIMEOUT_MS);
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
  *cfg = b->core.cfg;
  return MOPCUDA_OK;
}

static int config_ok(const MopCudaBatchConfig *c) {
  if (c->small_side < 1 || c->small_side > 256 || c->small_area < 1 ||
      c->small_area > 65536 || !mc_block_ok(c->vertex_block) || !mc_block_ok(c->setup_block) ||
      !mc_block_ok(c->raster_block) || !mc_block_ok(c->large_block) ||
      !mc_block_ok(c->shade_block) || c->grid_mul < 1 || c->grid_mul > 8)
    return fail(MOPCUDA_EINVAL, "batch config: value out of range");
  return MOPCUDA_OK;
}

extern "C" int mopcuda_batch_set_config(MopCudaBatch *b, const MopCudaBatchConfig *c) {
  if (!b || !c)
    return fail(MOPCUDA_EINVAL, "batch_set_config: bad arguments");
  int rc = config_ok(c);
  if (rc)
    return rc;
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->core.dev->ordinal);
  rc = finish_batch(b, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  b->core.cfg = *c;
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
  cudaSetDevice(b->core.dev->ordinal);
  MopCudaBatchConfig best = b->core.cfg;
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
  /* coordinate descent: passes over every axis until a pass improves nothing
   * (at most three) */
  int passes = 0;
  for (bool improved = true; improved && passes < 3; passes++) {
    improved = false;
    for (const Axis &ax : axes)
      for (const auto &val : ax.values) {
        MopCudaBatchConfig c = best;
        const std::string nm = ax.name;
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
        b->core.cfg = c;
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
          improved = true;
        }
      }
  }
  b->core.cfg = best;
  drop_graph(b);
  char tail[320];
  snprintf(tail, sizeof tail,
           "], \"passes\": %d, \"best_ms\": %.4f, \"best\": {\"small_side\": %d, \"small_area\": %d, "
           "\"vertex_block\": %d, \"setup_block\": %d, \"raster_block\": %d, "
           "\"large_block\": %d, \"shade_block\": %d, \"grid_mul\": %d}}",
           passes, best_ms, best.small_side, best.small_area, best.vertex_block, best.setup_block,
           best.raster_block, best.large_block, best.shade_block, best.grid_mul);
  log += tail;
  if (report && report_len) {
    strncpy(report, log.c_str(), report_len - 1);
    report[report_len - 1] = '\0';
  }
  return MOPCUDA_OK;
}

extern "C" uint64_t mopcuda_batch_device_bytes(const MopCudaBatch *b) {
  return b ? b->core.device_bytes() + b->pick_xy.cap + b->pick_out.cap : 0;
}
