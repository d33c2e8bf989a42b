/*
 * server.cu — the request server (C ABI in include/mop_cuda.h, "serving").
 *
 * Scenes stay resident on the device.  Clients submit render and pick
 * requests from any thread; one worker thread runs the loop:
 *
 *   completions  every launch slot whose end event has fired hands its
 *                results to the clients (or re-runs after its pools grew);
 *   admission    queued requests are admitted in arrival order while the
 *                estimated device bytes of the work in flight stay within
 *                the HBM budget and a slot is free; up to max_views
 *                admitted requests (any mix of scenes) form one launch;
 *   launch       the launch runs on the slot's own stream, so launches
 *                overlap on the device while new requests keep arriving.
 *
 * A request's result does not depend on what it was batched with: every
 * viewport of a launch is computed exactly as its own frame would be.
 * No counterpart in the reference, which renders on the caller's thread.
 */
#include "batch_internal.h"

#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

using Clock = std::chrono::steady_clock;

struct SrvRequest {
  uint64_t ticket = 0;
  MopCudaRequest req;
  std::shared_ptr<const std::vector<float>> models; /* the scene's models at submit */
  std::vector<int32_t> pick_xy;
  Clock::time_point t_submit, t_done;
  int status = 0; /* 0 queued, 1 running, 2 done, < 0 error */
  uint64_t est_bytes = 0;
  uint64_t samples = 0; /* width * height * ssaa^2 of the view */
  /* result staging offsets in the slot's pinned buffer */
  size_t off_color = 0, off_ids = 0, off_depth = 0, off_pick = 0;
  /* client buffers in page-locked memory receive their DMA directly */
  bool direct_color = false, direct_ids = false, direct_depth = false;
};

struct SrvSlot {
  LaunchCore core;
  std::vector<SrvRequest *> reqs;
  bool busy = false;
  int attempt = 0;
  uint64_t est_bytes = 0;
  HostArena h_io; /* pick inputs, then every result of the launch */
  DevArena d_pick_xy, d_pick_out;
  size_t in_bytes = 0, out_bytes = 0;
};

struct MopCudaServer {
  MopCudaDevice *dev = nullptr;
  MopCudaServerConfig cfg;
  std::vector<MopCudaScene *> scenes;
  std::mutex mu;
  std::condition_variable cv_arrive, cv_done;
  std::deque<SrvRequest *> pending;
  std::unordered_map<uint64_t, SrvRequest *> reqs;
  std::vector<SrvSlot *> slots;
  std::thread worker;
  bool stop = false;
  uint64_t next_ticket = 1;
  uint64_t inflight_bytes = 0;
  uint64_t max_view_samples = 0, max_view_pixels = 0; /* largest request so far */
  MopCudaServerStats st;
};

/* True for page-locked host memory (cudaHostAlloc / cudaHostRegister). */
static bool pinned(const void *p) {
  if (!p)
    return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

static double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

/* Stages a launch of the slot's requests: layout, scene snapshots, the
 * batch kernels, then the result copies and picks. */
static int srv_enqueue(MopCudaServer *s, SrvSlot *sl) {
  LaunchCore &c = sl->core;
  cudaStream_t st = c.stream;
  CU_TRY(cudaEventRecord(c.ev0, st));
  int rc = c.enqueue();
  if (rc)
    return rc;
  if (sl->in_bytes)
    CU_TRY(cudaMemcpyAsync(sl->d_pick_xy.p, sl->h_io.p, sl->in_bytes, cudaMemcpyHostToDevice, st));
  uint8_t *out = sl->h_io.as<uint8_t>() + sl->in_bytes;
  size_t pick_in = 0, pick_out = 0;
  for (size_t i = 0; i < sl->reqs.size(); i++) {
    SrvRequest *r = sl->reqs[i];
    const ViewRec &v = c.vrec[i];
    const size_t S = (size_t)v.width * v.height;
    const size_t P = (size_t)(v.width / v.ssaa) * (v.height / v.ssaa);
    if (r->req.kind == MOPCUDA_REQ_RENDER) {
      if (r->req.color) {
        const void *src = v.ssaa > 1 ? (const void *)(c.presented.as<uchar4>() + v.pixel_off)
                                     : (const void *)(c.out.as<uchar4>() + v.sample_off);
        void *dst = r->direct_color ? (void *)r->req.color : (void *)(out + r->off_color);
        CU_TRY(cudaMemcpyAsync(dst, src, 4 * P, cudaMemcpyDeviceToHost, st));
      }
      if (r->req.ids) {
        void *dst = r->direct_ids ? (void *)r->req.ids : (void *)(out + r->off_ids);
        CU_TRY(cudaMemcpyAsync(dst, c.ids.as<uint32_t>() + v.sample_off, 4 * S,
                               cudaMemcpyDeviceToHost, st));
      }
      if (r->req.depth) {
        void *dst = r->direct_depth ? (void *)r->req.depth : (void *)(out + r->off_depth);
        CU_TRY(cudaMemcpyAsync(dst, c.depth.as<float>() + v.sample_off, 4 * S,
                               cudaMemcpyDeviceToHost, st));
      }
    } else if (r->req.pick_n) {
      const uint32_t n = r->req.pick_n;
      uint32_t *oid = (uint32_t *)(sl->d_pick_out.as<uint8_t>() + pick_out);
      float *odp = (float *)(oid + n);
      int32_t *oht = (int32_t *)(odp + n);
      mopcuda_launch_pick(c.ids.as<uint32_t>() + v.sample_off, c.depth.as<float>() + v.sample_off,
                          v.width, v.height, v.ssaa,
                          (const int2 *)(sl->d_pick_xy.as<uint8_t>() + pick_in), n, oid, odp, oht,
                          st);
      CU_TRY(cudaMemcpyAsync(out + r->off_pick, oid, 12ull * n, cudaMemcpyDeviceToHost, st));
      pick_in += 8ull * n;
      pick_out += 12ull * n;
    }
  }
  CU_TRY(cudaGetLastError());
  CU_TRY(cudaEventRecord(c.ev1, st));
  return MOPCUDA_OK;
}

static int srv_launch(MopCudaServer *s, SrvSlot *sl) {
  LaunchCore &c = sl->core;
  const uint32_t n = (uint32_t)sl->reqs.size();
  std::vector<MopCudaScene *> sc;
  std::vector<std::shared_ptr<const std::vector<float>>> sm;
  std::vector<uint32_t> scene_of(n);
  std::vector<uint8_t> no_color(n);
  std::vector<MopCudaView> views(n);
  size_t in_b = 0, out_b = 0;
  for (uint32_t i = 0; i < n; i++) {
    SrvRequest *r = sl->reqs[i];
    /* one scene entry per (scene, model state): requests see their scene as
     * it was when they were submitted */
    MopCudaScene *scene = s->scenes[r->req.scene];
    uint32_t e = 0;
    while (e < sc.size() && !(sc[e] == scene && sm[e] == r->models))
      e++;
    if (e == sc.size()) {
      sc.push_back(scene);
      sm.push_back(r->models);
    }
    scene_of[i] = e;
    views[i] = r->req.view;
    no_color[i] = r->req.kind == MOPCUDA_REQ_PICK ? 1 : 0;
    const MopCudaView &v = r->req.view;
    const size_t S = (size_t)v.width * v.ssaa * v.height * v.ssaa;
    const size_t P = (size_t)v.width * v.height;
    auto take = [&](size_t bytes) {
      size_t o = out_b;
      out_b += (bytes + 15) & ~(size_t)15;
      return o;
    };
    if (r->req.kind == MOPCUDA_REQ_RENDER) {
      if (r->req.color && !r->direct_color)
        r->off_color = take(4 * P);
      if (r->req.ids && !r->direct_ids)
        r->off_ids = take(4 * S);
      if (r->req.depth && !r->direct_depth)
        r->off_depth = take(4 * S);
    } else {
      r->off_pick = take(12ull * r->req.pick_n);
      in_b += 8ull * r->req.pick_n;
    }
  }
  in_b = (in_b + 15) & ~(size_t)15;
  if (sl->h_io.ensure(in_b + out_b + 16) || sl->d_pick_xy.ensure(in_b + 16) ||
      sl->d_pick_out.ensure(out_b + 16))
    return MOPCUDA_ENOMEM;
  sl->in_bytes = in_b;
  sl->out_bytes = out_b;
  size_t o = 0;
  for (SrvRequest *r : sl->reqs)
    if (r->req.kind == MOPCUDA_REQ_PICK && r->req.pick_n) {
      memcpy(sl->h_io.as<uint8_t>() + o, r->pick_xy.data(), 8ull * r->req.pick_n);
      o += 8ull * r->req.pick_n;
    }
  int rc = c.set_layout(views.data(), scene_of.data(), no_color.data(), n, sc, &sm);
  if (!rc)
    rc = c.stage();
  if (!rc)
    rc = srv_enqueue(s, sl);
  return rc;
}

/* Hands a finished launch's results to the clients. */
static void srv_deliver(SrvSlot *sl) {
  const uint8_t *out = sl->h_io.as<uint8_t>() + sl->in_bytes;
  const LaunchCore &c = sl->core;
  for (size_t i = 0; i < sl->reqs.size(); i++) {
    SrvRequest *r = sl->reqs[i];
    const ViewRec &v = c.vrec[i];
    const size_t S = (size_t)v.width * v.height;
    const size_t P = (size_t)(v.width / v.ssaa) * (v.height / v.ssaa);
    if (r->req.kind == MOPCUDA_REQ_RENDER) {
      if (r->req.color && !r->direct_color)
        memcpy(r->req.color, out + r->off_color, 4 * P);
      if (r->req.ids && !r->direct_ids)
        memcpy(r->req.ids, out + r->off_ids, 4 * S);
      if (r->req.depth && !r->direct_depth)
        memcpy(r->req.depth, out + r->off_depth, 4 * S);
    } else if (r->req.pick_n) {
      const uint32_t n = r->req.pick_n;
      const uint8_t *p = out + r->off_pick;
      memcpy(r->req.pick_ids, p, 4ull * n);
      memcpy(r->req.pick_depths, p + 4ull * n, 4ull * n);
      memcpy(r->req.pick_hits, p + 8ull * n, 4ull * n);
    }
  }
}

static uint64_t held_bytes(const MopCudaServer *s) {
  uint64_t t = 0;
  for (const SrvSlot *sl : s->slots)
    t += sl->core.device_bytes() + sl->d_pick_xy.cap + sl->d_pick_out.cap;
  return t;
}

static void srv_finish(MopCudaServer *s, SrvSlot *sl, int rc, std::unique_lock<std::mutex> &lk) {
  const Clock::time_point now = Clock::now();
  for (SrvRequest *r : sl->reqs) {
    r->status = rc ? rc : 2;
    r->t_done = now;
  }
  if (rc)
    s->st.failed += sl->reqs.size();
  else
    s->st.completed += sl->reqs.size();
  s->inflight_bytes -= sl->est_bytes;
  sl->est_bytes = 0;
  sl->reqs.clear();
  sl->busy = false;
  s->st.device_bytes = held_bytes(s);
  if (s->st.device_bytes > s->cfg.hbm_budget) { /* give back this slot's buffers */
    lk.unlock();
    sl->core.trim();
    lk.lock();
    s->st.device_bytes = held_bytes(s);
  }
  s->cv_done.notify_all();
}

static void srv_loop(MopCudaServer *s) {
  cudaSetDevice(s->dev->ordinal);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    bool progressed = false;
    /* completions */
    for (SrvSlot *sl : s->slots) {
      if (!sl->busy || sl->reqs.empty())
        continue;
      cudaError_t q = cudaEventQuery(sl->core.ev1);
      if (q == cudaErrorNotReady)
        continue;
      progressed = true;
      lk.unlock();
      int rc = MOPCUDA_OK;
      bool rerun = false;
      if (q != cudaSuccess) {
        cudaGetLastError();
        rc = fail(MOPCUDA_ECUDA, "server launch: %s", cudaGetErrorString(q));
      } else {
        rc = sl->core.after(&rerun, sl->attempt);
        if (!rc && rerun) {
          sl->attempt++;
          rc = srv_enqueue(s, sl);
        } else if (!rc) {
          srv_deliver(sl);
        }
      }
      lk.lock();
      if (rerun && !rc) {
        s->st.reruns++;
        continue;
      }
      srv_finish(s, sl, rc, lk);
    }
    /* admission: arrival order, within the budget, up to max_views a launch */
    for (SrvSlot *sl : s->slots) {
      if (sl->busy || s->pending.empty())
        continue;
      std::vector<SrvRequest *> group;
      uint64_t bytes = 0, samples = 0;
      while (!s->pending.empty() && group.size() < s->cfg.max_views) {
        SrvRequest *r = s->pending.front();
        const bool fits = s->inflight_bytes + bytes + r->est_bytes <= s->cfg.hbm_budget;
        const bool alone = s->inflight_bytes == 0 && group.empty(); /* oversize: run it alone */
        if (!fits && !alone)
          break;
        if (s->cfg.max_launch_samples && !group.empty() &&
            samples + r->samples > s->cfg.max_launch_samples)
          break; /* the launch is full: the rest wait for the next slot */
        group.push_back(r);
        bytes += r->est_bytes;
        samples += r->samples;
        s->pending.pop_front();
      }
      if (group.empty())
        break;
      for (SrvRequest *r : group)
        r->status = 1;
      /* size the slot's buffers for a full launch of the largest request
       * seen, so later launches do not stop to reallocate */
      sl->core.sample_floor = s->max_view_samples * s->cfg.max_views;
      sl->core.pixel_floor = s->max_view_pixels * s->cfg.max_views;
      sl->reqs = group;
      sl->busy = true;
      sl->attempt = 0;
      sl->est_bytes = bytes;
      s->inflight_bytes += bytes;
      s->st.peak_inflight_bytes = std::max(s->st.peak_inflight_bytes, s->inflight_bytes);
      s->st.launches++;
      s->st.launched_views += group.size();
      s->st.max_views_in_launch =
          std::max(s->st.max_views_in_launch, (uint32_t)group.size());
      progressed = true;
      lk.unlock();
      int rc = srv_launch(s, sl);
      lk.lock();
      if (rc)
        srv_finish(s, sl, rc, lk);
      s->st.device_bytes = held_bytes(s);
    }
    bool busy = false;
    for (SrvSlot *sl : s->slots)
      busy |= sl->busy;
    if (s->stop && s->pending.empty() && !busy)
      break;
    if (!progressed) {
      if (busy)
        s->cv_arrive.wait_for(lk, std::chrono::microseconds(20));
      else
        s->cv_arrive.wait_for(lk, std::chrono::milliseconds(5));
    } else if (s->cfg.batch_window_us && !s->pending.empty()) {
      s->cv_arrive.wait_for(lk, std::chrono::microseconds(s->cfg.batch_window_us));
    }
  }
}

extern "C" MopCudaServer *mopcuda_server_create(MopCudaDevice *dev,
                                                const MopCudaServerConfig *cfg) {
  if (!dev || !cfg || cfg->max_views == 0 || cfg->max_views > MOPCUDA_MAX_VIEWS ||
      cfg->max_inflight == 0 || cfg->max_inflight > 16) {
    fail(MOPCUDA_EINVAL, "server_create: need a device, 1..%d views and 1..16 launches",
         MOPCUDA_MAX_VIEWS);
    return nullptr;
  }
  cudaSetDevice(dev->ordinal);
  MopCudaServer *s = new MopCudaServer();
  s->dev = dev;
  s->cfg = *cfg;
  memset(&s->st, 0, sizeof s->st);
  for (uint32_t i = 0; i < cfg->max_inflight; i++) {
    SrvSlot *sl = new SrvSlot();
    if (sl->core.init(dev)) {
      delete sl;
      for (SrvSlot *o : s->slots) {
        o->core.release();
        delete o;
      }
      delete s;
      return nullptr;
    }
    s->slots.push_back(sl);
  }
  s->worker = std::thread(srv_loop, s);
  return s;
}

extern "C" void mopcuda_server_destroy(MopCudaServer *s) {
  if (!s)
    return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_arrive.notify_all();
  if (s->worker.joinable())
    s->worker.join();
  cudaSetDevice(s->dev->ordinal);
  for (SrvSlot *sl : s->slots) {
    sl->h_io.release();
    sl->d_pick_xy.release();
    sl->d_pick_out.release();
    sl->core.release();
    delete sl;
  }
  for (auto &kv : s->reqs)
    delete kv.second;
  for (MopCudaScene *sc : s->scenes) {
    std::lock_guard<std::mutex> lk(sc->mu);
    sc->frozen = false;
  }
  delete s;
}

extern "C" int mopcuda_server_add_scene(MopCudaServer *s, MopCudaScene *scene) {
  if (!s || !scene || scene->dev != s->dev)
    return fail(MOPCUDA_EINVAL, "server_add_scene: scene of another device");
  {
    std::lock_guard<std::mutex> lk(scene->mu);
    scene->frozen = true;
  }
  cudaSetDevice(s->dev->ordinal);
  int rc = mc_scene_sync(scene);
  if (rc)
    return rc;
  std::lock_guard<std::mutex> lk(s->mu);
  s->scenes.push_back(scene);
  /* slot pools: half the worst case of a full launch of the largest scene,
   * so serving does not stop to reallocate them */
  unsigned long long need[4];
  mc_pool_need(scene->tris, scene->verts, 1, 1, need);
  for (SrvSlot *sl : s->slots)
    for (int k = 0; k < 4; k++)
      sl->core.pool_floor[k] =
          std::max(sl->core.pool_floor[k], need[k] * s->cfg.max_views / 2 + 4096ull);
  return (int)(s->scenes.size() - 1);
}

extern "C" int mopcuda_server_submit(MopCudaServer *s, const MopCudaRequest *req,
                                     uint64_t *ticket) {
  if (!s || !req || !ticket)
    return fail(MOPCUDA_EINVAL, "server_submit: bad arguments");
  int rc = mc_check_view(req->view);
  if (rc)
    return rc;
  if (req->kind != MOPCUDA_REQ_RENDER && req->kind != MOPCUDA_REQ_PICK)
    return fail(MOPCUDA_EINVAL, "server_submit: unknown request kind %u", req->kind);
  if (req->kind == MOPCUDA_REQ_PICK && req->pick_n &&
      (!req->pick_xy || !req->pick_ids || !req->pick_depths || !req->pick_hits))
    return fail(MOPCUDA_EINVAL, "server_submit: pick buffers missing");
  SrvRequest *r = new SrvRequest();
  r->req = *req;
  r->direct_color = pinned(req->color);
  r->direct_ids = pinned(req->ids);
  r->direct_depth = pinned(req->depth);
  if (req->kind == MOPCUDA_REQ_PICK && req->pick_n)
    r->pick_xy.assign(req->pick_xy, req->pick_xy + 2ull * req->pick_n);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (req->scene >= s->scenes.size()) {
      delete r;
      return fail(MOPCUDA_EINVAL, "server_submit: unknown scene %u", req->scene);
    }
    const MopCudaView &v = req->view;
    const uint64_t S = (uint64_t)v.width * v.ssaa * v.height * v.ssaa;
    const uint64_t P = (uint64_t)v.width * v.height;
    r->est_bytes = mc_view_bytes(s->scenes[req->scene], S, P);
    r->samples = S;
    s->max_view_samples = std::max<uint64_t>(s->max_view_samples, (S + 15) & ~(uint64_t)15);
    s->max_view_pixels = std::max<uint64_t>(s->max_view_pixels, (P + 15) & ~(uint64_t)15);
    r->models = mc_scene_models(s->scenes[req->scene]);
    r->ticket = s->next_ticket++;
    s->reqs[r->ticket] = r;
    s->pending.push_back(r);
    s->st.submitted++;
    *ticket = r->ticket;
  }
  s->cv_arrive.notify_one();
  return MOPCUDA_OK;
}

extern "C" int mopcuda_server_wait(MopCudaServer *s, uint64_t ticket, int timeout_ms,
                                   double *latency_ms) {
  if (!s)
    return fail(MOPCUDA_EINVAL, "server_wait: no server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end())
    return fail(MOPCUDA_EINVAL, "server_wait: unknown ticket %llu", (unsigned long long)ticket);
  SrvRequest *r = it->second;
  const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms),
                                      [&] { return r->status == 2 || r->status < 0; });
  if (!ok)
    return fail(MOPCUDA_ETIMEOUT, "server_wait: request %llu not done",
                (unsigned long long)ticket);
  const int status = r->status;
  if (latency_ms)
    *latency_ms = ms_between(r->t_submit, r->t_done);
  s->reqs.erase(it);
  delete r;
  return status == 2 ? MOPCUDA_OK : status;
}

extern "C" int mopcuda_server_drain(MopCudaServer *s, int timeout_ms) {
  if (!s)
    return fail(MOPCUDA_EINVAL, "server_drain: no server");
  std::unique_lock<std::mutex> lk(s->mu);
  const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] {
    if (!s->pending.empty())
      return false;
    for (SrvSlot *sl : s->slots)
      if (sl->busy)
        return false;
    return true;
  });
  return ok ? MOPCUDA_OK : fail(MOPCUDA_ETIMEOUT, "server_drain: work still in flight");
}

extern "C" int mopcuda_server_stats(MopCudaServer *s, MopCudaServerStats *out) {
  if (!s || !out)
    return fail(MOPCUDA_EINVAL, "server_stats: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  return MOPCUDA_OK;
}
