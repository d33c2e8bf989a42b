/*
 * mop_oracle.c — serial plain-C restatement of the reference CPU frame path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see mop_oracle.h).  Every float
 * expression keeps the reference's evaluation order, because the CPU build
 * (ISO C11, scalar SSE2, no FMA contraction) is bit-reproducible only under
 * the same sequence of IEEE single-precision operations.  Citations are
 * reference file:line.
 *
 * Compiled with -ffp-contract=off (oracle/Makefile).
 */
#include "mop_oracle.h"

#include <math.h>
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI_F ((float)3.14159265358979323846) /* (float)M_PI, rasterizer.c:24 */

/* ------------------------------------------------------------------------
 * vector helpers — math.c:17-50
 * ------------------------------------------------------------------------ */
typedef struct V3 {
  float x, y, z;
} V3;
typedef struct V4 {
  float x, y, z, w;
} V4;

static V3 v3(float x, float y, float z) {
  V3 r = {x, y, z};
  return r;
}
static V3 v3_add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static V3 v3_sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static V3 v3_scale(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static V3 v3_cross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z,
            a.x * b.y - a.y * b.x);
}
static float v3_dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static float v3_len(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
/* math.c:43-50: below 1e-8 the vector collapses to zero; otherwise it is
 * scaled by the reciprocal (not divided). */
static V3 v3_norm(V3 a) {
  float l = v3_len(a);
  if (l < 1e-8f)
    return v3(0.0f, 0.0f, 0.0f);
  float inv = 1.0f / l;
  return v3(a.x * inv, a.y * inv, a.z * inv);
}
static float clamp01(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }

/* column-major element (row r, column c) */
#define MAT(m, r, c) ((m)[(c)*4 + (r)])

/* mop_mat4_mul_vec4, math.c:196-203: each row summed left to right. */
static V4 m4_xform(const float *m, V4 v) {
  V4 r;
  r.x = MAT(m, 0, 0) * v.x + MAT(m, 0, 1) * v.y + MAT(m, 0, 2) * v.z + MAT(m, 0, 3) * v.w;
  r.y = MAT(m, 1, 0) * v.x + MAT(m, 1, 1) * v.y + MAT(m, 1, 2) * v.z + MAT(m, 1, 3) * v.w;
  r.z = MAT(m, 2, 0) * v.x + MAT(m, 2, 1) * v.y + MAT(m, 2, 2) * v.z + MAT(m, 2, 3) * v.w;
  r.w = MAT(m, 3, 0) * v.x + MAT(m, 3, 1) * v.y + MAT(m, 3, 2) * v.z + MAT(m, 3, 3) * v.w;
  return r;
}

/* mop_mat4_multiply, math.c:182-194: the running sum starts at 0.0f. */
void oracle_mat4_multiply(const float a[16], const float b[16], float c[16]) {
  float r[16];
  for (int col = 0; col < 4; col++)
    for (int row = 0; row < 4; row++) {
      float s = 0.0f;
      for (int k = 0; k < 4; k++)
        s += MAT(a, row, k) * MAT(b, k, col);
      MAT(r, row, col) = s;
    }
  memcpy(c, r, sizeof(r));
}

/* mop_mat4_look_at, math.c:111-130 */
static void m4_look_at(V3 eye, V3 center, V3 up, float *m) {
  V3 f = v3_norm(v3_sub(center, eye));
  V3 s = v3_norm(v3_cross(f, up));
  V3 u = v3_cross(s, f);
  memset(m, 0, 16 * sizeof(float));
  MAT(m, 0, 0) = s.x;
  MAT(m, 0, 1) = s.y;
  MAT(m, 0, 2) = s.z;
  MAT(m, 1, 0) = u.x;
  MAT(m, 1, 1) = u.y;
  MAT(m, 1, 2) = u.z;
  MAT(m, 2, 0) = -f.x;
  MAT(m, 2, 1) = -f.y;
  MAT(m, 2, 2) = -f.z;
  MAT(m, 0, 3) = -v3_dot(s, eye);
  MAT(m, 1, 3) = -v3_dot(u, eye);
  MAT(m, 2, 3) = v3_dot(f, eye);
  MAT(m, 3, 3) = 1.0f;
}

/* mop_mat4_perspective, math.c:69-79 */
static void m4_perspective(float fov, float aspect, float n, float f, float *m) {
  float t = tanf(fov * 0.5f);
  memset(m, 0, 16 * sizeof(float));
  MAT(m, 0, 0) = 1.0f / (aspect * t);
  MAT(m, 1, 1) = 1.0f / t;
  MAT(m, 2, 2) = -(f + n) / (f - n);
  MAT(m, 3, 2) = -1.0f;
  MAT(m, 2, 3) = -(2.0f * f * n) / (f - n);
}

/* mop_viewport_set_camera (viewport.c:1058-1093) stores orbit parameters;
 * mop_viewport_render re-applies the orbit camera every frame
 * (viewport.c:3017 -> camera.c:35-63 -> set_camera_orbit viewport.c:1095-1128),
 * so the frame's eye/up come from sinf/cosf of the recovered yaw/pitch. */
/* The orbit re-derivation of the eye and up vector mop_viewport_render
 * applies every frame (from the yaw/pitch mop_viewport_set_camera stored). */
static void orbit_camera(const float eye[3], const float target[3], const float up[3],
                         V3 *cam_eye_out, V3 *cam_up_out) {
  V3 e = v3(eye[0], eye[1], eye[2]);
  V3 t = v3(target[0], target[1], target[2]);
  V3 cam_eye = e, cam_up = v3(up[0], up[1], up[2]);
  V3 off = v3_sub(e, t);
  float dist = v3_len(off);
  if (dist > 1e-6f) {
    float yaw = atan2f(off.x, off.z);
    float pitch = asinf(off.y / dist);
    float sp = sinf(pitch), cp = cosf(pitch);
    float sy = sinf(yaw), cy = cosf(yaw);
    cam_up = v3(-sp * sy, cp, -sp * cy);
    float cp2 = cosf(pitch);
    cam_eye = v3(t.x + dist * cp2 * sinf(yaw), t.y + dist * sinf(pitch),
                 t.z + dist * cp2 * cosf(yaw));
  }
  *cam_eye_out = cam_eye;
  *cam_up_out = cam_up;
}

void oracle_camera(const float eye[3], const float target[3], const float up[3],
                   float fov_deg, float near_plane, float far_plane, int width,
                   int height, float view[16], float proj[16],
                   float eye_out[3]) {
  V3 t = v3(target[0], target[1], target[2]);
  V3 cam_eye, cam_up;
  orbit_camera(eye, target, up, &cam_eye, &cam_up);
  m4_look_at(cam_eye, t, cam_up, view);
  float fov = fov_deg * (3.14159265358979323846f / 180.0f);
  float aspect = (float)width / (float)height;
  m4_perspective(fov, aspect, near_plane, far_plane, proj);
  eye_out[0] = cam_eye.x;
  eye_out[1] = cam_eye.y;
  eye_out[2] = cam_eye.z;
}

/* ------------------------------------------------------------------------
 * framebuffer
 * ------------------------------------------------------------------------ */
typedef struct FB {
  int w, h;
  float *hdr;
  float *depth;
  uint32_t *id;
  uint8_t *color;
} FB;

/* Clip-space vertex (rasterizer.h:60-67).  The tangent is interpolated by the
 * reference but never read on this path, so it is not carried. */
typedef struct CV {
  V4 p;
  V3 n;
  V3 wp;
  float c[4];
  float u, v;
} CV;

/* Screen vertex (rasterizer.h:101-109). */
typedef struct SV {
  float sx, sy, sz, iw;
  V3 n, wp;
  float c[4];
} SV;

/* ------------------------------------------------------------------------
 * per-triangle vertex transform — cpu_prepare_triangle, cpu_backend.c:224-324
 * ------------------------------------------------------------------------ */
static void prepare_vertex(const OrDraw *d, const float *src, CV *o) {
  V4 p = {src[0], src[1], src[2], 1.0f};
  o->p = m4_xform(d->mvp, p);
  if (d->depth_bias != 0.0f)
    o->p.z += d->depth_bias * o->p.w; /* cpu_backend.c:238-242 */
  V4 w = m4_xform(d->model, p);
  o->wp = v3(w.x, w.y, w.z);
  V4 nn = {src[3], src[4], src[5], 0.0f};
  V4 tn = m4_xform(d->model, nn); /* not normalised, not inverse-transposed */
  o->n = v3(tn.x, tn.y, tn.z);
  for (int k = 0; k < 4; k++)
    o->c[k] = src[6 + k];
  o->u = src[10];
  o->v = src[11];
  if (d->texture && d->tex_w >= 1 && d->tex_h >= 1) { /* :276-303 */
    float tu = o->u - floorf(o->u);
    float tv = o->v - floorf(o->v);
    int tx = (int)(tu * (float)(d->tex_w - 1) + 0.5f);
    int ty = (int)(tv * (float)(d->tex_h - 1) + 0.5f);
    if (tx < 0)
      tx = 0;
    if (tx >= d->tex_w)
      tx = d->tex_w - 1;
    if (ty < 0)
      ty = 0;
    if (ty >= d->tex_h)
      ty = d->tex_h - 1;
    const uint8_t *t = d->texture + ((size_t)ty * (size_t)d->tex_w + (size_t)tx) * 4;
    for (int k = 0; k < 4; k++)
      o->c[k] *= (float)t[k] / 255.0f;
  }
}

/* ------------------------------------------------------------------------
 * Sutherland-Hodgman — rasterizer.c:514-626
 * ------------------------------------------------------------------------ */
#define MAX_CLIP 24

static const float PLANES[6][4] = {{1.0f, 0.0f, 0.0f, 1.0f},  {-1.0f, 0.0f, 0.0f, 1.0f},
                                   {0.0f, 1.0f, 0.0f, 1.0f},  {0.0f, -1.0f, 0.0f, 1.0f},
                                   {0.0f, 0.0f, 1.0f, 1.0f},  {0.0f, 0.0f, -1.0f, 1.0f}};

static float plane_dist(const float *pl, V4 p) {
  return pl[0] * p.x + pl[1] * p.y + pl[2] * p.z + pl[3] * p.w;
}

static float lerpf(float a, float b, float t) { return a + t * (b - a); }

/* lerp_vertex, rasterizer.c:528-551 */
static CV cv_lerp(const CV *a, const CV *b, float t) {
  CV r;
  r.p.x = lerpf(a->p.x, b->p.x, t);
  r.p.y = lerpf(a->p.y, b->p.y, t);
  r.p.z = lerpf(a->p.z, b->p.z, t);
  r.p.w = lerpf(a->p.w, b->p.w, t);
  r.n = v3(lerpf(a->n.x, b->n.x, t), lerpf(a->n.y, b->n.y, t), lerpf(a->n.z, b->n.z, t));
  r.wp = v3(lerpf(a->wp.x, b->wp.x, t), lerpf(a->wp.y, b->wp.y, t),
            lerpf(a->wp.z, b->wp.z, t));
  for (int k = 0; k < 4; k++)
    r.c[k] = lerpf(a->c[k], b->c[k], t);
  r.u = lerpf(a->u, b->u, t);
  r.v = lerpf(a->v, b->v, t);
  return r;
}

/* clip_against_plane, rasterizer.c:553-593 */
static int clip_plane(const CV *in, int n, CV *out, const float *pl) {
  if (n < 1)
    return 0;
  int m = 0;
  CV prev = in[n - 1];
  float dp = plane_dist(pl, prev.p);
  for (int i = 0; i < n; i++) {
    CV cur = in[i];
    float dc = plane_dist(pl, cur.p);
    if (dc >= 0.0f) {
      if (dp < 0.0f) {
        float t = dp / (dp - dc);
        if (m < MAX_CLIP)
          out[m++] = cv_lerp(&prev, &cur, t);
      }
      if (m < MAX_CLIP)
        out[m++] = cur;
    } else if (dp >= 0.0f) {
      float t = dp / (dp - dc);
      if (m < MAX_CLIP)
        out[m++] = cv_lerp(&prev, &cur, t);
    }
    prev = cur;
    dp = dc;
  }
  return m;
}

/* mop_sw_clip_polygon, rasterizer.c:598-626 */
static int clip_poly(const CV *in, int n, CV *out) {
  CV a[MAX_CLIP], b[MAX_CLIP];
  int cnt = n > MAX_CLIP ? MAX_CLIP : n;
  memcpy(a, in, sizeof(CV) * (size_t)cnt);
  CV *src = a, *dst = b;
  for (int p = 0; p < 6; p++) {
    cnt = clip_plane(src, cnt, dst, PLANES[p]);
    if (cnt == 0)
      return 0;
    CV *t = src;
    src = dst;
    dst = t;
  }
  memcpy(out, src, sizeof(CV) * (size_t)cnt);
  return cnt;
}

/* ------------------------------------------------------------------------
 * IBL lookups — rasterizer.c:161-301
 * ------------------------------------------------------------------------ */
static void ibl_bilinear(const float *d, int w, int h, float u, float v, float out[3]) {
  u = u - floorf(u);
  v = v - floorf(v);
  float fx = u * (float)(w - 1);
  float fy = v * (float)(h - 1);
  int x0 = (int)fx, y0 = (int)fy;
  int x1 = (x0 + 1) % w;
  int y1 = y0 + 1 < h ? y0 + 1 : h - 1;
  float sx = fx - (float)x0, sy = fy - (float)y0;
  const float *p00 = &d[((size_t)y0 * w + x0) * 4];
  const float *p10 = &d[((size_t)y0 * w + x1) * 4];
  const float *p01 = &d[((size_t)y1 * w + x0) * 4];
  const float *p11 = &d[((size_t)y1 * w + x1) * 4];
  for (int c = 0; c < 3; c++) {
    float top = p00[c] * (1.0f - sx) + p10[c] * sx;
    float bot = p01[c] * (1.0f - sx) + p11[c] * sx;
    out[c] = top * (1.0f - sy) + bot * sy;
  }
}

static void dir_uv(float dx, float dy, float dz, float rot, float *u, float *v) {
  float phi = atan2f(dz, dx) + rot;
  float cdy = dy < -1.0f ? -1.0f : (dy > 1.0f ? 1.0f : dy);
  *u = phi / (2.0f * 3.14159265f) + 0.5f;
  *v = asinf(cdy) / 3.14159265f + 0.5f;
}

static void ibl_irr(const OrIBL *ibl, V3 n, float out[3]) {
  out[0] = out[1] = out[2] = 0.0f;
  if (!ibl || !ibl->irr)
    return;
  float len = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
  if (len < 1e-6f)
    return;
  float u, v;
  dir_uv(n.x / len, n.y / len, n.z / len, ibl->rotation, &u, &v);
  ibl_bilinear(ibl->irr, ibl->irr_w, ibl->irr_h, u, v, out);
  for (int c = 0; c < 3; c++)
    out[c] *= ibl->intensity;
}

static void ibl_pf(const OrIBL *ibl, V3 r, float rough, float out[3]) {
  out[0] = out[1] = out[2] = 0.0f;
  if (!ibl || !ibl->pf)
    return;
  float len = sqrtf(r.x * r.x + r.y * r.y + r.z * r.z);
  if (len < 1e-6f)
    return;
  int level = (int)(rough * (float)(ibl->pf_levels - 1));
  if (level >= ibl->pf_levels)
    level = ibl->pf_levels - 1;
  size_t off = 0;
  for (int l = 0; l < level; l++) {
    int lw = ibl->pf_w >> l, lh = ibl->pf_h >> l;
    off += (size_t)(lw < 1 ? 1 : lw) * (size_t)(lh < 1 ? 1 : lh);
  }
  int lw = ibl->pf_w >> level, lh = ibl->pf_h >> level;
  if (lw < 1)
    lw = 1;
  if (lh < 1)
    lh = 1;
  float u, v;
  dir_uv(r.x / len, r.y / len, r.z / len, ibl->rotation, &u, &v);
  ibl_bilinear(ibl->pf + off * 4, lw, lh, u, v, out);
  for (int c = 0; c < 3; c++)
    out[c] *= ibl->intensity;
}

static void ibl_lut(const OrIBL *ibl, float ndv, float rough, float *sc, float *bi) {
  *sc = 1.0f;
  *bi = 0.0f;
  if (!ibl || !ibl->brdf)
    return;
  ndv = ndv < 0.0f ? 0.0f : (ndv > 1.0f ? 1.0f : ndv);
  rough = rough < 0.0f ? 0.0f : (rough > 1.0f ? 1.0f : rough);
  int n = ibl->brdf_size;
  int x = (int)(ndv * (float)(n - 1) + 0.5f);
  int y = (int)(rough * (float)(n - 1) + 0.5f);
  if (x >= n)
    x = n - 1;
  if (y >= n)
    y = n - 1;
  size_t i = ((size_t)y * n + x) * 4;
  *sc = ibl->brdf[i + 0];
  *bi = ibl->brdf[i + 1];
}

/* ------------------------------------------------------------------------
 * light terms
 * ------------------------------------------------------------------------ */

/* distance falloff shared by the point/spot cases of the per-pixel
 * diffuse and specular helpers (rasterizer.c:1636-1646, 1742-1760). */
static float falloff_inv_sq(const OrLight *L, float dist) {
  if (L->range > 0.0f) {
    float r = dist / L->range;
    float a = 1.0f - r;
    if (a < 0.0f)
      a = 0.0f;
    return a * a;
  }
  float d2 = dist * dist;
  if (d2 < 0.01f)
    d2 = 0.01f;
  return 1.0f / d2;
}

static float spot_cone(const OrLight *L, V3 dir) {
  V3 sd = v3_norm(v3(L->direction[0], L->direction[1], L->direction[2]));
  float ca = -v3_dot(dir, sd);
  if (ca < L->spot_outer_cos)
    return 0.0f;
  if (ca < L->spot_inner_cos) {
    float rs = L->spot_inner_cos - L->spot_outer_cos;
    if (rs > 1e-6f) {
      float t = (ca - L->spot_outer_cos) / rs;
      return t * t * (3.0f - 2.0f * t);
    }
  }
  return 1.0f;
}

/* ------------------------------------------------------------------------
 * shadow map: the rasteriser's bound map (rasterizer.c:141-157), the 3x3 PCF
 * test (rasterizer.c:303-348), the depth-only caster raster (:357-493) and
 * pass_shadow's light camera (viewport.c:2288-2442)
 * ------------------------------------------------------------------------ */
static const OrShadow *g_shadow; /* bound for the frame oracle_render draws */

/* (int) of a float as the x86-64 build converts it (cvttss2si): INT_MIN
 * for NaN and out-of-range values. */
static int x86_f2i(float f) {
  if (!(f >= -2147483648.0f && f < 2147483648.0f))
    return INT32_MIN;
  return (int)f;
}

static float shadow_test_pcf(V3 wp) {
  const OrShadow *s = g_shadow;
  if (!s || !s->depth)
    return 1.0f;
  V4 p = {wp.x, wp.y, wp.z, 1.0f};
  V4 lp = m4_xform(s->vp, p);
  if (lp.w <= 0.0f)
    return 1.0f;
  float inv_w = 1.0f / lp.w;
  float ndcx = lp.x * inv_w;
  float ndcy = lp.y * inv_w;
  float ndcz = (lp.z * inv_w + 1.0f) * 0.5f;
  float u = (ndcx + 1.0f) * 0.5f * (float)s->w;
  float v = (1.0f - ndcy) * 0.5f * (float)s->h;
  int64_t cx = x86_f2i(u), cy = x86_f2i(v);
  float bias = 0.005f;
  int lit = 0, total = 0;
  for (int dy = -1; dy <= 1; dy++) {
    for (int dx = -1; dx <= 1; dx++) {
      int64_t sx = cx + dx, sy = cy + dy;
      if (sx < 0 || sx >= s->w || sy < 0 || sy >= s->h) {
        lit++;
        total++;
        continue;
      }
      float shadow_z = s->depth[sy * (int64_t)s->w + sx];
      if (ndcz <= shadow_z + bias)
        lit++;
      total++;
    }
  }
  return (float)lit / (float)total;
}

static float light_shadow(const OrLight *L, V3 wp) {
  return (L->type == 0 && g_shadow && g_shadow->depth) ? shadow_test_pcf(wp) : 1.0f;
}

/* mop_mat4_ortho, math.c:93-109 */
static void m4_ortho(float l, float r, float b, float t, float n, float f, float *m) {
  float rl = r - l, tb = t - b, fn = f - n;
  memset(m, 0, 16 * sizeof(float));
  if (fabsf(rl) < 1e-9f || fabsf(tb) < 1e-9f || fabsf(fn) < 1e-9f) {
    m[0] = m[5] = m[10] = m[15] = 1.0f;
    return;
  }
  MAT(m, 0, 0) = 2.0f / rl;
  MAT(m, 1, 1) = 2.0f / tb;
  MAT(m, 2, 2) = -2.0f / fn;
  MAT(m, 0, 3) = -(r + l) / rl;
  MAT(m, 1, 3) = -(t + b) / tb;
  MAT(m, 2, 3) = -(f + n) / fn;
  MAT(m, 3, 3) = 1.0f;
}

int oracle_shadow_matrix(const float *models, uint32_t count, const float dir[3],
                         float vp[16]) {
  if (count == 0)
    return 0;
  float smin[3] = {1e9f, 1e9f, 1e9f}, smax[3] = {-1e9f, -1e9f, -1e9f};
  for (uint32_t i = 0; i < count; i++) {
    const float *m = models + 16 * (size_t)i;
    float cx = m[12], cy = m[13], cz = m[14];
    float sx = sqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    float sy = sqrtf(m[4] * m[4] + m[5] * m[5] + m[6] * m[6]);
    float sz = sqrtf(m[8] * m[8] + m[9] * m[9] + m[10] * m[10]);
    float r = sx > sy ? sx : sy;
    if (sz > r)
      r = sz;
    r *= 1.5f;
    if (cx - r < smin[0])
      smin[0] = cx - r;
    if (cy - r < smin[1])
      smin[1] = cy - r;
    if (cz - r < smin[2])
      smin[2] = cz - r;
    if (cx + r > smax[0])
      smax[0] = cx + r;
    if (cy + r > smax[1])
      smax[1] = cy + r;
    if (cz + r > smax[2])
      smax[2] = cz + r;
  }
  V3 ld = v3_norm(v3(dir[0], dir[1], dir[2]));
  float ctx = (smin[0] + smax[0]) * 0.5f;
  float cty = (smin[1] + smax[1]) * 0.5f;
  float ctz = (smin[2] + smax[2]) * 0.5f;
  float dx = smax[0] - smin[0], dy = smax[1] - smin[1], dz = smax[2] - smin[2];
  float radius = sqrtf(dx * dx + dy * dy + dz * dz) * 0.5f;
  if (radius < 1.0f)
    radius = 1.0f;
  V3 eye = v3(ctx - ld.x * radius * 2.0f, cty - ld.y * radius * 2.0f,
              ctz - ld.z * radius * 2.0f);
  V3 up = v3(0.0f, 1.0f, 0.0f);
  if (fabsf(v3_dot(ld, up)) > 0.99f)
    up = v3(1.0f, 0.0f, 0.0f);
  float view[16], proj[16];
  m4_look_at(eye, v3(ctx, cty, ctz), up, view);
  float os = radius * 1.2f;
  m4_ortho(-os, os, -os, os, 0.1f, radius * 4.0f, proj);
  oracle_mat4_multiply(proj, view, vp);
  return 1;
}

static void shadow_mesh(const OrShadowMesh *me, const float *light_vp, int size, float *depth) {
  float mvp[16];
  oracle_mat4_multiply(light_vp, me->model, mvp);
  float half_w = (float)size * 0.5f;
  float half_h = (float)size * 0.5f;
  for (uint32_t i = 0; i + 2 < me->index_count; i += 3) {
    uint32_t ix[3] = {me->indices[i], me->indices[i + 1], me->indices[i + 2]};
    if (ix[0] >= me->vertex_count || ix[1] >= me->vertex_count || ix[2] >= me->vertex_count)
      continue;
    V4 c[3];
    for (int k = 0; k < 3; k++) {
      const float *p = me->vertices + (size_t)ix[k] * 12;
      V4 pos = {p[0], p[1], p[2], 1.0f};
      c[k] = m4_xform(mvp, pos);
    }
    if ((c[0].x < -c[0].w && c[1].x < -c[1].w && c[2].x < -c[2].w) ||
        (c[0].x > c[0].w && c[1].x > c[1].w && c[2].x > c[2].w) ||
        (c[0].y < -c[0].w && c[1].y < -c[1].w && c[2].y < -c[2].w) ||
        (c[0].y > c[0].w && c[1].y > c[1].w && c[2].y > c[2].w) ||
        (c[0].z < -c[0].w && c[1].z < -c[1].w && c[2].z < -c[2].w) ||
        (c[0].z > c[0].w && c[1].z > c[1].w && c[2].z > c[2].w))
      continue;
    if (c[0].w <= 1e-6f || c[1].w <= 1e-6f || c[2].w <= 1e-6f)
      continue;
    float sx[3], sy[3], sz[3];
    for (int k = 0; k < 3; k++) {
      float inv = 1.0f / c[k].w;
      sx[k] = (c[k].x * inv + 1.0f) * half_w;
      sy[k] = (1.0f - c[k].y * inv) * half_h;
      sz[k] = (c[k].z * inv + 1.0f) * 0.5f;
    }
    float fmin_x = sx[0], fmin_y = sy[0], fmax_x = sx[0], fmax_y = sy[0];
    for (int k = 1; k < 3; k++) {
      if (sx[k] < fmin_x)
        fmin_x = sx[k];
      if (sx[k] > fmax_x)
        fmax_x = sx[k];
    }
    for (int k = 1; k < 3; k++) {
      if (sy[k] < fmin_y)
        fmin_y = sy[k];
      if (sy[k] > fmax_y)
        fmax_y = sy[k];
    }
    int min_x = x86_f2i(floorf(fmin_x)), min_y = x86_f2i(floorf(fmin_y));
    int max_x = x86_f2i(ceilf(fmax_x)), max_y = x86_f2i(ceilf(fmax_y));
    if (min_x < 0)
      min_x = 0;
    if (min_y < 0)
      min_y = 0;
    if (max_x >= size)
      max_x = size - 1;
    if (max_y >= size)
      max_y = size - 1;
    if (min_x > max_x || min_y > max_y)
      continue;
    float area = (sx[1] - sx[0]) * (sy[2] - sy[0]) - (sx[2] - sx[0]) * (sy[1] - sy[0]);
    if (fabsf(area) < 1e-6f)
      continue;
    float inv_area = 1.0f / fabsf(area);
    float edx[3] = {sy[1] - sy[2], sy[2] - sy[0], sy[0] - sy[1]};
    float edy[3] = {sx[2] - sx[1], sx[0] - sx[2], sx[1] - sx[0]};
    float px0 = (float)min_x + 0.5f, py0 = (float)min_y + 0.5f;
    float wr[3] = {(sx[2] - sx[1]) * (py0 - sy[1]) - (sy[2] - sy[1]) * (px0 - sx[1]),
                   (sx[0] - sx[2]) * (py0 - sy[2]) - (sy[0] - sy[2]) * (px0 - sx[2]),
                   (sx[1] - sx[0]) * (py0 - sy[0]) - (sy[1] - sy[0]) * (px0 - sx[0])};
    if (area < 0.0f) {
      for (int k = 0; k < 3; k++) {
        edx[k] = -edx[k];
        edy[k] = -edy[k];
        wr[k] = -wr[k];
      }
    }
    for (int y = min_y; y <= max_y; y++) {
      float w0 = wr[0], w1 = wr[1], w2 = wr[2];
      for (int x = min_x; x <= max_x; x++) {
        if (w0 >= 0.0f && w1 >= 0.0f && w2 >= 0.0f) {
          float b0 = w0 * inv_area, b1 = w1 * inv_area, b2 = w2 * inv_area;
          float z = b0 * sz[0] + b1 * sz[1] + b2 * sz[2];
          size_t idx = (size_t)y * (size_t)size + (size_t)x;
          if (z < depth[idx])
            depth[idx] = z;
        }
        w0 += edx[0];
        w1 += edx[1];
        w2 += edx[2];
      }
      wr[0] += edy[0];
      wr[1] += edy[1];
      wr[2] += edy[2];
    }
  }
}

void oracle_shadow_render(const OrShadowMesh *meshes, uint32_t count, int size,
                          const float vp[16], float *depth) {
  for (size_t p = 0; p < (size_t)size * (size_t)size; p++)
    depth[p] = 1.0f;
  for (uint32_t i = 0; i < count; i++)
    shadow_mesh(&meshes[i], vp, size, depth);
}

/* compute_multi_light_rgb, rasterizer.c:1596-1688. */
static void diffuse_rgb(V3 n, V3 wp, const OrLight *Ls, uint32_t cnt, float amb,
                        float out[3]) {
  out[0] = out[1] = out[2] = amb;
  for (uint32_t i = 0; i < cnt; i++) {
    const OrLight *L = &Ls[i];
    if (!L->active)
      continue;
    float ndotl = 0.0f, att = 1.0f, spot = 1.0f;
    if (L->type == 0) {
      V3 dir = v3_norm(v3(L->direction[0], L->direction[1], L->direction[2]));
      ndotl = -v3_dot(n, dir);
    } else if (L->type == 1 || L->type == 2) {
      V3 tl = v3_sub(v3(L->position[0], L->position[1], L->position[2]), wp);
      float dist = v3_len(tl);
      if (dist < 1e-6f)
        dist = 1e-6f;
      V3 dir = v3_scale(tl, 1.0f / dist);
      ndotl = v3_dot(n, dir);
      if (L->type == 2)
        spot = spot_cone(L, dir);
      att = falloff_inv_sq(L, dist);
    }
    if (ndotl < 0.0f)
      ndotl = 0.0f;
    float shadow = light_shadow(L, wp);
    float contrib = ndotl * L->intensity * att * spot * shadow;
    out[0] += contrib * L->color[0];
    out[1] += contrib * L->color[1];
    out[2] += contrib * L->color[2];
  }
}

/* compute_multi_light (flat), rasterizer.c:1497-1588: same as the RGB helper
 * except spot falloff is 1/(1+d^2), colour is ignored, and the total is
 * clamped to [0,1]. */
static float diffuse_flat(V3 n, V3 wp, const OrLight *Ls, uint32_t cnt, float amb) {
  float total = amb;
  for (uint32_t i = 0; i < cnt; i++) {
    const OrLight *L = &Ls[i];
    if (!L->active)
      continue;
    float ndotl = 0.0f, att = 1.0f, spot = 1.0f;
    if (L->type == 0) {
      V3 dir = v3_norm(v3(L->direction[0], L->direction[1], L->direction[2]));
      ndotl = -v3_dot(n, dir);
    } else if (L->type == 1 || L->type == 2) {
      V3 tl = v3_sub(v3(L->position[0], L->position[1], L->position[2]), wp);
      float dist = v3_len(tl);
      if (dist < 1e-6f)
        dist = 1e-6f;
      V3 dir = v3_scale(tl, 1.0f / dist);
      ndotl = v3_dot(n, dir);
      if (L->type == 1) {
        att = falloff_inv_sq(L, dist);
      } else {
        spot = spot_cone(L, dir);
        if (L->range > 0.0f) {
          float r = dist / L->range;
          att = 1.0f - r;
          if (att < 0.0f)
            att = 0.0f;
          att *= att;
        } else {
          att = 1.0f / (1.0f + dist * dist);
        }
      }
    }
    if (ndotl < 0.0f)
      ndotl = 0.0f;
    float shadow = light_shadow(L, wp);
    total += ndotl * L->intensity * att * spot * shadow;
  }
  return clamp01(total);
}

/* compute_multi_specular_ggx, rasterizer.c:1701-1814: spot lights are
 * treated as point lights (no cone), lights with N.L <= 0 are skipped. */
static void specular_ggx(V3 n, V3 wp, V3 vdir, const OrLight *Ls, uint32_t cnt,
                         float rough, float metal, const float base[3], float out[3]) {
  out[0] = out[1] = out[2] = 0.0f;
  float alpha = rough * rough;
  float alpha2 = alpha * alpha;
  if (alpha2 < 1e-7f)
    alpha2 = 1e-7f;
  float ndotv = v3_dot(n, vdir);
  if (ndotv < 1e-4f)
    ndotv = 1e-4f;
  float f0[3];
  for (int c = 0; c < 3; c++)
    f0[c] = 0.04f * (1.0f - metal) + base[c] * metal;
  float k = alpha * 0.5f;
  float g1v = ndotv / (ndotv * (1.0f - k) + k);
  for (uint32_t i = 0; i < cnt; i++) {
    const OrLight *L = &Ls[i];
    if (!L->active)
      continue;
    V3 ldir = v3(0.0f, 0.0f, 0.0f);
    float att = 1.0f;
    if (L->type == 0) {
      V3 d = v3_norm(v3(L->direction[0], L->direction[1], L->direction[2]));
      ldir = v3(-d.x, -d.y, -d.z);
    } else if (L->type == 1 || L->type == 2) {
      V3 tl = v3_sub(v3(L->position[0], L->position[1], L->position[2]), wp);
      float dist = v3_len(tl);
      if (dist < 1e-6f)
        dist = 1e-6f;
      ldir = v3_scale(tl, 1.0f / dist);
      att = falloff_inv_sq(L, dist);
    }
    float ndotl = v3_dot(n, ldir);
    if (ndotl <= 0.0f)
      continue;
    V3 h = v3_norm(v3_add(ldir, vdir));
    float ndoth = v3_dot(n, h);
    if (ndoth < 0.0f)
      ndoth = 0.0f;
    float vdoth = v3_dot(vdir, h);
    if (vdoth < 0.0f)
      vdoth = 0.0f;
    float ndoth2 = ndoth * ndoth;
    float dd = ndoth2 * (alpha2 - 1.0f) + 1.0f;
    float D = alpha2 / (OR_PI_F * dd * dd);
    float g1l = ndotl / (ndotl * (1.0f - k) + k);
    float G = g1v * g1l;
    float omv = 1.0f - vdoth;
    float omv2 = omv * omv;
    float omv5 = omv2 * omv2 * omv;
    float fr[3];
    for (int c = 0; c < 3; c++)
      fr[c] = f0[c] + (1.0f - f0[c]) * omv5;
    float den = 4.0f * ndotl * ndotv;
    if (den < 1e-6f)
      den = 1e-6f;
    float st = D * G / den;
    float shadow = light_shadow(L, wp);
    float wgt = st * L->intensity * att * ndotl * shadow * OR_PI_F;
    for (int c = 0; c < 3; c++)
      out[c] += wgt * fr[c] * L->color[c];
  }
}

/* Per-pixel shading of the smooth multi-light path, rasterizer.c:1963-2099.
 * pc[] are the normalised perspective-correct weights. */
static void shade_ml(const SV *sv, const float pc[3], const OrDraw *d,
                     const OrIBL *ibl, float out[3]) {
  V3 n = v3(pc[0] * sv[0].n.x + pc[1] * sv[1].n.x + pc[2] * sv[2].n.x,
            pc[0] * sv[0].n.y + pc[1] * sv[1].n.y + pc[2] * sv[2].n.y,
            pc[0] * sv[0].n.z + pc[1] * sv[1].n.z + pc[2] * sv[2].n.z);
  n = v3_norm(n);
  float base[3];
  for (int c = 0; c < 3; c++)
    base[c] = pc[0] * sv[0].c[c] + pc[1] * sv[1].c[c] + pc[2] * sv[2].c[c];
  V3 wp = v3(pc[0] * sv[0].wp.x + pc[1] * sv[1].wp.x + pc[2] * sv[2].wp.x,
             pc[0] * sv[0].wp.y + pc[1] * sv[1].wp.y + pc[2] * sv[2].wp.y,
             pc[0] * sv[0].wp.z + pc[1] * sv[1].wp.z + pc[2] * sv[2].wp.z);
  V3 eye = v3(d->cam_eye[0], d->cam_eye[1], d->cam_eye[2]);
  V3 vdir = v3_norm(v3_sub(eye, wp));
  float lit[3], spec[3];
  diffuse_rgb(n, wp, d->lights, d->light_count, d->ambient, lit);
  specular_ggx(n, wp, vdir, d->lights, d->light_count, d->roughness, d->metallic,
               base, spec);
  float ds = 1.0f - d->metallic;
  float env[3] = {0.0f, 0.0f, 0.0f};
  float irr[3] = {0.0f, 0.0f, 0.0f};
  bool has_irr = ibl && ibl->irr;
  if (has_irr)
    ibl_irr(ibl, n, irr);
  {
    float vdn = v3_dot(vdir, n);
    V3 refl = v3(2.0f * vdn * n.x - vdir.x, 2.0f * vdn * n.y - vdir.y,
                 2.0f * vdn * n.z - vdir.z);
    float ndv = v3_dot(n, vdir);
    if (ndv < 0.0f)
      ndv = 0.0f;
    float f0[3];
    for (int c = 0; c < 3; c++)
      f0[c] = 0.04f * (1.0f - d->metallic) + base[c] * d->metallic;
    if (ibl && ibl->pf && ibl->brdf) {
      float pf[3], bs, bb;
      ibl_pf(ibl, refl, d->roughness, pf);
      ibl_lut(ibl, ndv, d->roughness, &bs, &bb);
      for (int c = 0; c < 3; c++)
        env[c] = pf[c] * (f0[c] * bs + bb);
    } else if (d->metallic > 0.01f) {
      /* hemisphere fallback, rasterizer.c:2042-2072 */
      float sky_t = refl.y * 0.5f + 0.5f;
      if (sky_t < 0.0f)
        sky_t = 0.0f;
      if (sky_t > 1.0f)
        sky_t = 1.0f;
      const float sky[3] = {0.35f, 0.38f, 0.45f}, gnd[3] = {0.08f, 0.07f, 0.06f};
      float he[3];
      for (int c = 0; c < 3; c++)
        he[c] = gnd[c] + sky_t * (sky[c] - gnd[c]);
      float mix = d->roughness * d->roughness;
      float avg = (he[0] + he[1] + he[2]) * (1.0f / 3.0f);
      for (int c = 0; c < 3; c++)
        he[c] += mix * (avg - he[c]);
      float om = 1.0f - ndv;
      float om2 = om * om;
      float om5 = om2 * om2 * om;
      for (int c = 0; c < 3; c++) {
        float fe = f0[c] + (1.0f - f0[c]) * om5;
        env[c] = he[c] * fe * d->ambient * 3.0f;
      }
    }
  }
  for (int c = 0; c < 3; c++) {
    float p;
    if (has_irr)
      p = base[c] * (lit[c] + irr[c]) * ds + env[c] + spec[c];
    else
      p = base[c] * lit[c] * ds + env[c] + spec[c];
    out[c] = p < 0.0f ? 0.0f : p;
  }
}

/* ------------------------------------------------------------------------
 * Edge setup shared by the three rasterisers (e.g. rasterizer.c:1842-1924)
 * ------------------------------------------------------------------------ */
typedef struct Edges {
  int x0, y0, x1, y1; /* clamped inclusive bbox */
  float area, inv_area;
  bool flip;
  float dx[3], dy[3]; /* per-pixel / per-row increments */
  float w_row[3];     /* edge values at (x0+.5, y0+.5) */
  float inv_e[3];     /* 1/|edge|, 0 for degenerate edges */
} Edges;

static bool edge_setup(const float sx[3], const float sy[3], int W, int H,
                       bool want_inv_e, Edges *e) {
  float fmin_x = sx[0], fmin_y = sy[0], fmax_x = sx[0], fmax_y = sy[0];
  for (int k = 1; k < 3; k++) {
    if (sx[k] < fmin_x)
      fmin_x = sx[k];
    if (sy[k] < fmin_y)
      fmin_y = sy[k];
    if (sx[k] > fmax_x)
      fmax_x = sx[k];
    if (sy[k] > fmax_y)
      fmax_y = sy[k];
  }
  e->x0 = (int)floorf(fmin_x);
  e->y0 = (int)floorf(fmin_y);
  e->x1 = (int)ceilf(fmax_x);
  e->y1 = (int)ceilf(fmax_y);
  if (e->x0 < 0)
    e->x0 = 0;
  if (e->y0 < 0)
    e->y0 = 0;
  if (e->x1 >= W)
    e->x1 = W - 1;
  if (e->y1 >= H)
    e->y1 = H - 1;
  if (e->x0 > e->x1 || e->y0 > e->y1)
    return false;
  e->area = (sx[1] - sx[0]) * (sy[2] - sy[0]) - (sx[2] - sx[0]) * (sy[1] - sy[0]);
  if (fabsf(e->area) < 1e-6f)
    return false;
  e->flip = e->area < 0.0f;
  e->inv_area = 1.0f / fabsf(e->area);
  /* edge k runs from vertex k+1 to vertex k+2 */
  for (int k = 0; k < 3; k++) {
    int a = (k + 1) % 3, b = (k + 2) % 3;
    e->dx[k] = sy[a] - sy[b];
    e->dy[k] = sx[b] - sx[a];
    if (e->flip) {
      e->dx[k] = -e->dx[k];
      e->dy[k] = -e->dy[k];
    }
  }
  if (want_inv_e)
    for (int k = 0; k < 3; k++) {
      float l = sqrtf(e->dx[k] * e->dx[k] + e->dy[k] * e->dy[k]);
      e->inv_e[k] = (l > 1e-6f) ? 1.0f / l : 0.0f;
    }
  float px = (float)e->x0 + 0.5f, py = (float)e->y0 + 0.5f;
  for (int k = 0; k < 3; k++) {
    int a = (k + 1) % 3, b = (k + 2) % 3;
    float w = (sx[b] - sx[a]) * (py - sy[a]) - (sy[b] - sy[a]) * (px - sx[a]);
    e->w_row[k] = e->flip ? -w : w;
  }
  return true;
}

static void blend_px(int mode, float fa, float *dst, float p[3]) {
  float inv = 1.0f - fa;
  for (int c = 0; c < 3; c++) {
    if (mode == 2)
      p[c] = dst[c] + p[c] * fa;
    else if (mode == 3)
      p[c] = dst[c] * p[c];
    else
      p[c] = p[c] * fa + dst[c] * inv;
  }
}

/* mop_sw_rasterize_triangle_smooth_ml, rasterizer.c:1825-2152 */
static void raster_smooth_ml(const SV sv[3], const OrDraw *d, const OrIBL *ibl, FB *fb) {
  float sx[3] = {sv[0].sx, sv[1].sx, sv[2].sx}, sy[3] = {sv[0].sy, sv[1].sy, sv[2].sy};
  Edges e;
  if (!edge_setup(sx, sy, fb->w, fb->h, true, &e))
    return;
  float op = clamp01(d->opacity);
  float wr[3] = {e.w_row[0], e.w_row[1], e.w_row[2]};
  for (int y = e.y0; y <= e.y1; y++) {
    float w[3] = {wr[0], wr[1], wr[2]};
    for (int x = e.x0; x <= e.x1; x++) {
      if (w[0] >= 0.0f && w[1] >= 0.0f && w[2] >= 0.0f) {
        float d0 = w[0] * e.inv_e[0], d1 = w[1] * e.inv_e[1], d2 = w[2] * e.inv_e[2];
        float min_d = d0;
        if (d1 < min_d)
          min_d = d1;
        if (d2 < min_d)
          min_d = d2;
        if (min_d >= 0.0f) {
          float b0 = w[0] * e.inv_area, b1 = w[1] * e.inv_area, b2 = w[2] * e.inv_area;
          float z = b0 * sv[0].sz + b1 * sv[1].sz + b2 * sv[2].sz;
          size_t idx = (size_t)y * (size_t)fb->w + (size_t)x;
          if (!d->depth_test || z < fb->depth[idx]) {
            float pc[3] = {b0 * sv[0].iw, b1 * sv[1].iw, b2 * sv[2].iw};
            float ip = 1.0f / (pc[0] + pc[1] + pc[2]);
            pc[0] *= ip;
            pc[1] *= ip;
            pc[2] *= ip;
            float p[3];
            shade_ml(sv, pc, d, ibl, p);
            float cov = (min_d < 1.0f && d->blend_mode != 0) ? min_d : 1.0f;
            float fa = op * cov;
            float *hdr = &fb->hdr[idx * 4];
            if (d->blend_mode == 0 && fa >= 1.0f) {
              hdr[0] = p[0];
              hdr[1] = p[1];
              hdr[2] = p[2];
              hdr[3] = 1.0f;
              fb->depth[idx] = z;
              fb->id[idx] = d->object_id;
            } else {
              blend_px(d->blend_mode, fa, hdr, p);
              hdr[0] = p[0];
              hdr[1] = p[1];
              hdr[2] = p[2];
              hdr[3] = 1.0f;
              if (fa > 0.5f) {
                fb->depth[idx] = z;
                fb->id[idx] = d->object_id;
              }
            }
          }
        }
      }
      w[0] += e.dx[0];
      w[1] += e.dx[1];
      w[2] += e.dx[2];
    }
    wr[0] += e.dy[0];
    wr[1] += e.dy[1];
    wr[2] += e.dy[2];
  }
}

/* mop_sw_rasterize_triangle_smooth (no light list), rasterizer.c:1253-1489:
 * single light, Blinn-Phong term, silhouette coverage read from the depth
 * buffer (so the result depends on draw order). */
static void raster_smooth_legacy(const SV sv[3], const OrDraw *d, FB *fb) {
  float sx[3] = {sv[0].sx, sv[1].sx, sv[2].sx}, sy[3] = {sv[0].sy, sv[1].sy, sv[2].sy};
  Edges e;
  if (!edge_setup(sx, sy, fb->w, fb->h, true, &e))
    return;
  V3 nl = v3_norm(v3(d->light_dir[0], d->light_dir[1], d->light_dir[2]));
  float op = clamp01(d->opacity);
  float wr[3] = {e.w_row[0], e.w_row[1], e.w_row[2]};
  for (int y = e.y0; y <= e.y1; y++) {
    float w[3] = {wr[0], wr[1], wr[2]};
    for (int x = e.x0; x <= e.x1; x++) {
      if (w[0] >= 0.0f && w[1] >= 0.0f && w[2] >= 0.0f) {
        float d0 = w[0] * e.inv_e[0], d1 = w[1] * e.inv_e[1], d2 = w[2] * e.inv_e[2];
        float min_d = d0;
        if (d1 < min_d)
          min_d = d1;
        if (d2 < min_d)
          min_d = d2;
        if (min_d >= 0.0f) {
          float b0 = w[0] * e.inv_area, b1 = w[1] * e.inv_area, b2 = w[2] * e.inv_area;
          float z = b0 * sv[0].sz + b1 * sv[1].sz + b2 * sv[2].sz;
          size_t idx = (size_t)y * (size_t)fb->w + (size_t)x;
          if (!d->depth_test || z < fb->depth[idx]) {
            float pc[3] = {b0 * sv[0].iw, b1 * sv[1].iw, b2 * sv[2].iw};
            float ip = 1.0f / (pc[0] + pc[1] + pc[2]);
            pc[0] *= ip;
            pc[1] *= ip;
            pc[2] *= ip;
            V3 n = v3(pc[0] * sv[0].n.x + pc[1] * sv[1].n.x + pc[2] * sv[2].n.x,
                      pc[0] * sv[0].n.y + pc[1] * sv[1].n.y + pc[2] * sv[2].n.y,
                      pc[0] * sv[0].n.z + pc[1] * sv[1].n.z + pc[2] * sv[2].n.z);
            n = v3_norm(n);
            float base[3];
            for (int c = 0; c < 3; c++)
              base[c] = pc[0] * sv[0].c[c] + pc[1] * sv[1].c[c] + pc[2] * sv[2].c[c];
            float ndotl = v3_dot(n, nl);
            if (ndotl < 0.0f)
              ndotl = 0.0f;
            float lit = d->ambient + (1.0f - d->ambient) * ndotl;
            V3 hv = v3_norm(v3(nl.x, nl.y + 1.0f, nl.z));
            float ndoth = v3_dot(n, hv);
            if (ndoth < 0.0f)
              ndoth = 0.0f;
            float spec = ndoth * ndoth;
            spec *= spec;
            spec *= spec;
            spec *= spec;
            spec *= spec;
            spec *= 0.25f;
            float p[3];
            for (int c = 0; c < 3; c++) {
              p[c] = base[c] * lit + spec;
              if (p[c] < 0.0f)
                p[c] = 0.0f;
            }
            float ez = fb->depth[idx];
            bool sil = (ez - z) > 0.005f;
            float cov = (min_d < 1.0f && sil) ? min_d : 1.0f;
            float fa = op * cov;
            float *hdr = &fb->hdr[idx * 4];
            if (d->blend_mode == 0 && fa >= 1.0f) {
              hdr[0] = p[0];
              hdr[1] = p[1];
              hdr[2] = p[2];
              hdr[3] = 1.0f;
              fb->depth[idx] = z;
              fb->id[idx] = d->object_id;
            } else {
              blend_px(d->blend_mode, fa, hdr, p);
              hdr[0] = p[0];
              hdr[1] = p[1];
              hdr[2] = p[2];
              hdr[3] = 1.0f;
              if (fa > 0.5f) {
                fb->depth[idx] = z;
                fb->id[idx] = d->object_id;
              }
            }
          }
        }
      }
      w[0] += e.dx[0];
      w[1] += e.dx[1];
      w[2] += e.dx[2];
    }
    wr[0] += e.dy[0];
    wr[1] += e.dy[1];
    wr[2] += e.dy[2];
  }
}

/* rasterize_filled_triangle, rasterizer.c:890-1087: constant colour, depth
 * stepped incrementally alongside the edge values. */
static void raster_flat(const float sx[3], const float sy[3], const float sz[3], float cr,
                        float cg, float cb, float ca, uint32_t id, bool depth_test,
                        int blend, FB *fb) {
  Edges e;
  if (!edge_setup(sx, sy, fb->w, fb->h, false, &e))
    return;
  float z_dx = (e.dx[0] * sz[0] + e.dx[1] * sz[1] + e.dx[2] * sz[2]) * e.inv_area;
  float z_dy = (e.dy[0] * sz[0] + e.dy[1] * sz[1] + e.dy[2] * sz[2]) * e.inv_area;
  float z_row = (e.w_row[0] * sz[0] + e.w_row[1] * sz[1] + e.w_row[2] * sz[2]) * e.inv_area;
  float wr[3] = {e.w_row[0], e.w_row[1], e.w_row[2]};
  bool opaque = (blend == 0 && ca >= 1.0f);
  for (int y = e.y0; y <= e.y1; y++) {
    float w[3] = {wr[0], wr[1], wr[2]};
    float z = z_row;
    for (int x = e.x0; x <= e.x1; x++) {
      if (w[0] >= 0.0f && w[1] >= 0.0f && w[2] >= 0.0f) {
        size_t idx = (size_t)y * (size_t)fb->w + (size_t)x;
        if (!depth_test || z < fb->depth[idx]) {
          float *hdr = &fb->hdr[idx * 4];
          if (opaque) {
            hdr[0] = cr;
            hdr[1] = cg;
            hdr[2] = cb;
            hdr[3] = 1.0f;
            fb->depth[idx] = z;
            fb->id[idx] = id;
          } else {
            float p[3] = {cr, cg, cb};
            float dst[3] = {hdr[0], hdr[1], hdr[2]};
            for (int c = 0; c < 3; c++) {
              if (blend == 2)
                p[c] = dst[c] + p[c] * ca;
              else if (blend == 3)
                p[c] = dst[c] * p[c];
              else
                p[c] = p[c] * ca + dst[c] * (1.0f - ca);
            }
            hdr[0] = p[0];
            hdr[1] = p[1];
            hdr[2] = p[2];
            hdr[3] = 1.0f;
          }
        }
      }
      w[0] += e.dx[0];
      w[1] += e.dx[1];
      w[2] += e.dx[2];
      z += z_dx;
    }
    wr[0] += e.dy[0];
    wr[1] += e.dy[1];
    wr[2] += e.dy[2];
    z_row += z_dy;
  }
}

/* ------------------------------------------------------------------------
 * triangle front end — mop_sw_rasterize_triangle_full (rasterizer.c:2458-2612)
 * and mop_sw_rasterize_triangle (1093-1242)
 * ------------------------------------------------------------------------ */
static bool outside_same_plane(V4 a, V4 b, V4 c) {
  return (a.x < -a.w && b.x < -b.w && c.x < -c.w) || (a.x > a.w && b.x > b.w && c.x > c.w) ||
         (a.y < -a.w && b.y < -b.w && c.y < -c.w) || (a.y > a.w && b.y > b.w && c.y > c.w) ||
         (a.z < -a.w && b.z < -b.w && c.z < -c.w) || (a.z > a.w && b.z > b.w && c.z > c.w);
}

static bool inside_all(V4 p) {
  return p.x >= -p.w && p.x <= p.w && p.y >= -p.w && p.y <= p.w && p.z >= -p.w && p.z <= p.w;
}

/* Xiaolin Wu anti-aliased lines (mop_sw_draw_line_aa with thickness 1,
 * rasterizer.c:743-871) and their plot (aa_plot, :687-729): the colour
 * blended over the HDR value by the coverage, depth and ID written above
 * coverage 0.5.  The HDR buffer is what the frame's resolve reads, so the
 * plot's byte write is left out. */
static float wu_fpart(float x) { return x - floorf(x); }
static float wu_rfpart(float x) { return 1.0f - wu_fpart(x); }

static void wu_plot(FB *fb, int x, int y, float z, const uint8_t rgb[3], float cov,
                    uint32_t id, bool dt) {
  if (x < 0 || x >= fb->w || y < 0 || y >= fb->h || cov < 0.004f)
    return;
  size_t i = (size_t)y * (size_t)fb->w + (size_t)x;
  if (dt && z >= fb->depth[i])
    return;
  float inv = 1.0f - cov;
  for (int c = 0; c < 3; c++) {
    float src = (float)rgb[c] / 255.0f;
    fb->hdr[i * 4 + c] = src * cov + fb->hdr[i * 4 + c] * inv;
  }
  fb->hdr[i * 4 + 3] = 1.0f;
  if (cov > 0.5f) {
    fb->depth[i] = z;
    fb->id[i] = id;
  }
}

static void wu_line(FB *fb, float x0, float y0, float z0, float x1, float y1, float z1,
                    const uint8_t rgb[3], uint32_t id, bool dt) {
  bool steep = fabsf(y1 - y0) > fabsf(x1 - x0);
  if (steep) { /* walk along y: swap the axes */
    float t = x0;
    x0 = y0;
    y0 = t;
    t = x1;
    x1 = y1;
    y1 = t;
  }
  if (x0 > x1) { /* left to right */
    float t = x0;
    x0 = x1;
    x1 = t;
    t = y0;
    y0 = y1;
    y1 = t;
    t = z0;
    z0 = z1;
    z1 = t;
  }
  float gradient = (x1 - x0 < 0.001f) ? 1.0f : (y1 - y0) / (x1 - x0);
  /* the two end pixels */
  float xe = roundf(x0), ye = y0 + gradient * (xe - x0), gap = wu_rfpart(x0 + 0.5f);
  int xp1 = (int)xe, yp = (int)floorf(ye);
  float c_hi = wu_rfpart(ye) * gap, c_lo = wu_fpart(ye) * gap;
  if (steep) {
    wu_plot(fb, yp, xp1, z0, rgb, c_hi, id, dt);
    wu_plot(fb, yp + 1, xp1, z0, rgb, c_lo, id, dt);
  } else {
    wu_plot(fb, xp1, yp, z0, rgb, c_hi, id, dt);
    wu_plot(fb, xp1, yp + 1, z0, rgb, c_lo, id, dt);
  }
  float intery = ye + gradient;
  xe = roundf(x1);
  ye = y1 + gradient * (xe - x1);
  gap = wu_fpart(x1 + 0.5f);
  int xp2 = (int)xe;
  yp = (int)floorf(ye);
  c_hi = wu_rfpart(ye) * gap;
  c_lo = wu_fpart(ye) * gap;
  if (steep) {
    wu_plot(fb, yp, xp2, z1, rgb, c_hi, id, dt);
    wu_plot(fb, yp + 1, xp2, z1, rgb, c_lo, id, dt);
  } else {
    wu_plot(fb, xp2, yp, z1, rgb, c_hi, id, dt);
    wu_plot(fb, xp2, yp + 1, z1, rgb, c_lo, id, dt);
  }
  /* the pixels between, depth interpolated by the step's fraction */
  float steps = (float)(xp2 - xp1);
  if (steps < 1.0f)
    steps = 1.0f;
  for (int x = xp1 + 1; x < xp2; x++) {
    float t = (float)(x - xp1) / steps;
    float z = z0 + t * (z1 - z0);
    int iy = (int)floorf(intery);
    if (steep) {
      wu_plot(fb, iy, x, z, rgb, wu_rfpart(intery), id, dt);
      wu_plot(fb, iy + 1, x, z, rgb, wu_fpart(intery), id, dt);
    } else {
      wu_plot(fb, x, iy, z, rgb, wu_rfpart(intery), id, dt);
      wu_plot(fb, x, iy + 1, z, rgb, wu_fpart(intery), id, dt);
    }
    intery += gradient;
  }
}

static void triangle(const CV tri[3], const OrDraw *d, const OrIBL *ibl, FB *fb) {
  V4 a = tri[0].p, b = tri[1].p, c = tri[2].p;
  bool lit = d->lights && d->light_count > 0;
  if (outside_same_plane(a, b, c))
    return;
  if (d->backface_cull && a.w > 0.0f && b.w > 0.0f && c.w > 0.0f) {
    float ex = b.x * a.w - a.x * b.w;
    float ey = b.y * a.w - a.y * b.w;
    float fx = c.x * a.w - a.x * c.w;
    float fy = c.y * a.w - a.y * c.w;
    if (ex * fy - ey * fx <= 0.0f)
      return;
  }
  CV clipped[MAX_CLIP];
  const CV *poly;
  int np;
  if (a.w > 0.0f && b.w > 0.0f && c.w > 0.0f && inside_all(a) && inside_all(b) &&
      inside_all(c)) {
    poly = tri;
    np = 3;
  } else {
    np = clip_poly(tri, 3, clipped);
    if (np < 3)
      return;
    poly = clipped;
  }
  V3 nl = v3_norm(v3(d->light_dir[0], d->light_dir[1], d->light_dir[2]));
  float hw = (float)fb->w * 0.5f, hh = (float)fb->h * 0.5f;
  uint8_t ca8 = (uint8_t)(clamp01(d->opacity) * 255.0f); /* :1159 (unlit path) */
  for (int i = 1; i < np - 1; i++) {
    const CV *v[3] = {&poly[0], &poly[i], &poly[i + 1]};
    if (fabsf(v[0]->p.w) < 1e-7f || fabsf(v[1]->p.w) < 1e-7f || fabsf(v[2]->p.w) < 1e-7f)
      continue;
    SV sv[3];
    for (int k = 0; k < 3; k++) {
      float iw = 1.0f / v[k]->p.w;
      sv[k].sx = (v[k]->p.x * iw + 1.0f) * hw;
      sv[k].sy = (1.0f - v[k]->p.y * iw) * hh;
      sv[k].sz = (v[k]->p.z * iw + 1.0f) * 0.5f;
      sv[k].iw = iw;
      sv[k].n = v[k]->n;
      sv[k].wp = v[k]->wp;
      memcpy(sv[k].c, v[k]->c, sizeof(sv[k].c));
    }
    float sarea = (sv[1].sx - sv[0].sx) * (sv[2].sy - sv[0].sy) -
                  (sv[2].sx - sv[0].sx) * (sv[1].sy - sv[0].sy);
    if (d->backface_cull && sarea >= 0.0f)
      continue;
    if (d->smooth && !d->wireframe) {
      if (lit)
        raster_smooth_ml(sv, d, ibl, fb);
      else
        raster_smooth_legacy(sv, d, fb);
      continue;
    }
    /* flat shading */
    V3 fn = v3_norm(v3(v[0]->n.x + v[1]->n.x + v[2]->n.x, v[0]->n.y + v[1]->n.y + v[2]->n.y,
                       v[0]->n.z + v[1]->n.z + v[2]->n.z));
    float avg[3];
    for (int k = 0; k < 3; k++)
      avg[k] = (v[0]->c[k] + v[1]->c[k] + v[2]->c[k]) * (1.0f / 3.0f);
    float col[3], caf;
    if (lit) {
      V3 wp = v3((v[0]->wp.x + v[1]->wp.x + v[2]->wp.x) / 3.0f,
                 (v[0]->wp.y + v[1]->wp.y + v[2]->wp.y) / 3.0f,
                 (v[0]->wp.z + v[1]->wp.z + v[2]->wp.z) / 3.0f);
      float lighting = diffuse_flat(fn, wp, d->lights, d->light_count, d->ambient);
      float ds = 1.0f - d->metallic;
      float env_flat = d->ambient * d->metallic * 0.3f;
      for (int k = 0; k < 3; k++)
        col[k] = avg[k] * (lighting * ds + env_flat);
      caf = clamp01(d->opacity);
    } else {
      float ndotl = v3_dot(fn, nl);
      if (ndotl < 0.0f)
        ndotl = 0.0f;
      float lighting = clamp01(d->ambient + (1.0f - d->ambient) * ndotl);
      for (int k = 0; k < 3; k++)
        col[k] = avg[k] * lighting;
      caf = (float)ca8 / 255.0f;
    }
    for (int k = 0; k < 3; k++)
      if (col[k] < 0.0f)
        col[k] = 0.0f;
    float sx[3] = {sv[0].sx, sv[1].sx, sv[2].sx}, sy[3] = {sv[0].sy, sv[1].sy, sv[2].sy},
          sz[3] = {sv[0].sz, sv[1].sz, sv[2].sz};
    if (d->wireframe) { /* rasterizer.c:1225-1235, 2595-2605 */
      uint8_t rgb[3];
      for (int k = 0; k < 3; k++)
        rgb[k] = (uint8_t)((col[k] > 1.0f ? 1.0f : col[k]) * 255.0f);
      for (int e = 0; e < 3; e++) {
        int f = (e + 1) % 3;
        wu_line(fb, sx[e], sy[e], sz[e], sx[f], sy[f], sz[f], rgb, d->object_id,
                d->depth_test != 0);
      }
      continue;
    }
    raster_flat(sx, sy, sz, col[0], col[1], col[2], caf, d->object_id, d->depth_test != 0,
                d->blend_mode, fb);
  }
}

/* ------------------------------------------------------------------------
 * frame end: ACES resolve, FXAA, post-process, SSAA box
 * ------------------------------------------------------------------------ */
static float aces(float x) { /* rasterizer.c:2770-2774 */
  float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
  float m = (x * (a * x + b)) / (x * (c * x + d) + e);
  return m < 0.0f ? 0.0f : (m > 1.0f ? 1.0f : m);
}

/* float -> uint8_t as the x86-64 reference build converts it: truncate to
 * int32, keep the low byte. */
static uint8_t to_u8(float f) { return (uint8_t)(int32_t)f; }

static void hdr_resolve(FB *fb, float exposure) { /* rasterizer.c:2776-2803 */
  size_t n = (size_t)fb->w * fb->h;
  for (size_t i = 0; i < n; i++) {
    const float *h = &fb->hdr[i * 4];
    uint8_t *o = &fb->color[i * 4];
    if (fb->id[i] == 0) {
      for (int c = 0; c < 3; c++)
        o[c] = to_u8(fminf(h[c], 1.0f) * 255.0f + 0.5f);
      o[3] = 255;
    } else {
      for (int c = 0; c < 3; c++)
        o[c] = to_u8(aces(h[c] * exposure) * 255.0f + 0.5f);
      o[3] = to_u8(h[3] * 255.0f + 0.5f);
    }
  }
}

static float luma8(const uint8_t *p) {
  return 0.299f * (float)p[0] + 0.587f * (float)p[1] + 0.114f * (float)p[2];
}

static void fxaa(FB *fb) { /* mop_sw_fxaa, rasterizer.c:2625-2761 */
  int w = fb->w, h = fb->h;
  if (w < 3 || h < 3)
    return;
  size_t bytes = (size_t)w * h * 4;
  uint8_t *src = malloc(bytes);
  memcpy(src, fb->color, bytes);
#define LU(xx, yy) luma8(&src[((size_t)(yy) * (size_t)w + (size_t)(xx)) * 4])
  for (int y = 1; y < h - 1; y++) {
    for (int x = 1; x < w - 1; x++) {
      float lM = LU(x, y), lN = LU(x, y - 1), lS = LU(x, y + 1), lW = LU(x - 1, y),
            lE = LU(x + 1, y);
      float mn = lM, mx = lM;
      float nb[4] = {lN, lS, lW, lE};
      for (int k = 0; k < 4; k++) {
        if (nb[k] < mn)
          mn = nb[k];
      }
      for (int k = 0; k < 4; k++) {
        if (nb[k] > mx)
          mx = nb[k];
      }
      float range = mx - mn;
      if (range < 0.0625f * mx + 0.004f)
        continue;
      float lNW = LU(x - 1, y - 1), lNE = LU(x + 1, y - 1), lSW = LU(x - 1, y + 1),
            lSE = LU(x + 1, y + 1);
      float avg = (lN + lS + lW + lE) * (2.0f / 12.0f) + (lNW + lNE + lSW + lSE) * (1.0f / 12.0f);
      float sub = fabsf(avg - lM);
      sub = sub / range;
      if (sub > 1.0f)
        sub = 1.0f;
      sub = sub * sub * (3.0f - 2.0f * sub);
      sub *= 0.75f;
      float eh = fabsf(-2.0f * lW + lNW + lSW) + fabsf(-2.0f * lM + lN + lS) * 2.0f +
                 fabsf(-2.0f * lE + lNE + lSE);
      float ev = fabsf(-2.0f * lN + lNW + lNE) + fabsf(-2.0f * lM + lW + lE) * 2.0f +
                 fabsf(-2.0f * lS + lSW + lSE);
      bool horiz = eh >= ev;
      int stx = horiz ? 0 : 1, sty = horiz ? 1 : 0;
      float lp = horiz ? lS : lE, ln = horiz ? lN : lW;
      float gp = fabsf(lp - lM), gn = fabsf(ln - lM);
      int ox = gp >= gn ? stx : -stx, oy = gp >= gn ? sty : -sty;
      int nx = x + ox, ny = y + oy;
      if (nx < 0)
        nx = 0;
      if (nx >= w)
        nx = w - 1;
      if (ny < 0)
        ny = 0;
      if (ny >= h)
        ny = h - 1;
      size_t ci = ((size_t)y * w + x) * 4, ni = ((size_t)ny * w + nx) * 4;
      float ib = 1.0f - sub;
      for (int c = 0; c < 3; c++)
        fb->color[ci + c] = to_u8(src[ci + c] * ib + src[ni + c] * sub);
    }
  }
#undef LU
  free(src);
}

static float srgb(float c) { /* postprocess.c:76-77 */
  return c <= 0.0031308f ? c * 12.92f : 1.055f * powf(c, 1.0f / 2.4f) - 0.055f;
}

void oracle_gamma_lut(uint8_t lut[256]) {
  for (int i = 0; i < 256; i++) {
    float r = (float)(uint8_t)i / 255.0f;
    r = srgb(r > 0.0f ? r : 0.0f);
    if (r > 1.0f)
      r = 1.0f;
    if (r < 0.0f)
      r = 0.0f;
    lut[i] = to_u8(r * 255.0f + 0.5f);
  }
}

/* mop_postprocess_apply, postprocess.c:24-116: FXAA, then per sample fog
 * (from the sample's depth value, :51-65), Reinhard tonemap, sRGB gamma and
 * vignette, clamped and rounded to bytes. */
static void postprocess(FB *fb, uint32_t fx, const OrFrame *f) {
  if (fx == 0)
    return;
  if (fx & 16u)
    fxaa(fb);
  int w = fb->w, h = fb->h;
  float cx = (float)w * 0.5f, cy = (float)h * 0.5f;
  float maxd = sqrtf(cx * cx + cy * cy);
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      uint8_t *p = &fb->color[((size_t)y * w + x) * 4];
      float c[3];
      for (int k = 0; k < 3; k++)
        c[k] = (float)p[k] / 255.0f;
      if ((fx & 8u) && f->fog_on) {
        const float depth = fb->depth[(size_t)y * w + x];
        const float range = f->fog_far - f->fog_near;
        float factor = 0.0f;
        if (range > 0.0f) {
          factor = (depth - f->fog_near) / range;
          if (factor < 0.0f)
            factor = 0.0f;
          if (factor > 1.0f)
            factor = 1.0f;
        }
        for (int k = 0; k < 3; k++)
          c[k] = c[k] + (f->fog_color[k] - c[k]) * factor;
      }
      if (fx & 2u)
        for (int k = 0; k < 3; k++)
          c[k] = c[k] / (c[k] + 1.0f);
      if (fx & 1u)
        for (int k = 0; k < 3; k++)
          c[k] = srgb(c[k] > 0.0f ? c[k] : 0.0f);
      if (fx & 4u) {
        float dx = (float)x - cx, dy = (float)y - cy;
        float dist = sqrtf(dx * dx + dy * dy) / maxd;
        float vg = 1.0f - dist * dist * 0.5f;
        if (vg < 0.0f)
          vg = 0.0f;
        for (int k = 0; k < 3; k++)
          c[k] *= vg;
      }
      for (int k = 0; k < 3; k++) {
        if (c[k] > 1.0f)
          c[k] = 1.0f;
        if (c[k] < 0.0f)
          c[k] = 0.0f;
        p[k] = to_u8(c[k] * 255.0f + 0.5f);
      }
    }
}

/* ------------------------------------------------------------------------
 * frame driver
 * ------------------------------------------------------------------------ */
/* env_sample_bilinear, viewport.c:2099-2124 */
static void sky_bilinear(const float *d, int w, int h, float u, float v, float out[4]) {
  u = u - floorf(u);
  v = v - floorf(v);
  float fx = u * (float)(w - 1), fy = v * (float)(h - 1);
  int x0 = (int)fx, y0 = (int)fy;
  int x1 = (x0 + 1) % w, y1 = y0 + 1;
  if (y1 >= h)
    y1 = h - 1;
  float sx = fx - (float)x0, sy = fy - (float)y0;
  const float *p00 = &d[((size_t)y0 * w + x0) * 4], *p10 = &d[((size_t)y0 * w + x1) * 4];
  const float *p01 = &d[((size_t)y1 * w + x0) * 4], *p11 = &d[((size_t)y1 * w + x1) * 4];
  for (int c = 0; c < 4; c++) {
    float top = p00[c] * (1.0f - sx) + p10[c] * sx;
    float bot = p01[c] * (1.0f - sx) + p11[c] * sx;
    out[c] = top * (1.0f - sy) + bot * sy;
  }
}

/* pass_background_hdri_cpu, viewport.c:2128-2177: the environment along the
 * ray through every sample, into the HDR buffer (alpha 1). */
static void sky_pass(FB *fb, const OrSky *s) {
  V3 cam_eye, cam_up;
  orbit_camera(s->eye, s->target, s->up, &cam_eye, &cam_up);
  V3 t = v3(s->target[0], s->target[1], s->target[2]);
  int sw = fb->w, sh = fb->h;
  float fov = s->fov_deg * (3.14159265358979323846f / 180.0f);
  float aspect = (float)sw / (float)sh;
  float half_h = tanf(fov * 0.5f);
  float half_w = half_h * aspect;
  V3 fwd = v3_norm(v3_sub(t, cam_eye));
  V3 right = v3_norm(v3_cross(fwd, cam_up));
  V3 up = v3_cross(right, fwd);
  const float pi = 3.14159265358979f;
  for (int y = 0; y < sh; y++) {
    float ndc_y = 1.0f - 2.0f * ((float)y + 0.5f) / (float)sh;
    for (int x = 0; x < sw; x++) {
      float ndc_x = 2.0f * ((float)x + 0.5f) / (float)sw - 1.0f;
      float dx = fwd.x + right.x * ndc_x * half_w + up.x * ndc_y * half_h;
      float dy = fwd.y + right.y * ndc_x * half_w + up.y * ndc_y * half_h;
      float dz = fwd.z + right.z * ndc_x * half_w + up.z * ndc_y * half_h;
      float len = sqrtf(dx * dx + dy * dy + dz * dz);
      dx /= len;
      dy /= len;
      dz /= len;
      float phi = atan2f(dz, dx) - s->rotation;
      float cdy = dy < -1.0f ? -1.0f : (dy > 1.0f ? 1.0f : dy);
      float theta = asinf(cdy);
      float eu = phi / (2.0f * pi) + 0.5f;
      float ev = theta / pi + 0.5f;
      float smp[4];
      sky_bilinear(s->env, s->w, s->h, eu, ev, smp);
      float *o = &fb->hdr[((size_t)y * sw + x) * 4];
      o[0] = smp[0] * s->intensity;
      o[1] = smp[1] * s->intensity;
      o[2] = smp[2] * s->intensity;
      o[3] = 1.0f;
    }
  }
}

int oracle_render(OrFrame *f, const OrDraw *draws, uint32_t n) {
  if (!f || f->width <= 0 || f->height <= 0)
    return -1;
  size_t px = (size_t)f->width * f->height;
  FB fb = {f->width, f->height, malloc(px * 16), malloc(px * 4), malloc(px * 4), malloc(px * 4)};
  if (!fb.hdr || !fb.depth || !fb.id || !fb.color) {
    free(fb.hdr);
    free(fb.depth);
    free(fb.id);
    free(fb.color);
    return -2;
  }
  g_shadow = f->shadow;
  /* mop_sw_framebuffer_clear, rasterizer.c:114-134 */
  for (size_t i = 0; i < px; i++) {
    for (int c = 0; c < 4; c++) {
      fb.hdr[i * 4 + c] = f->clear[c];
      fb.color[i * 4 + c] = to_u8(f->clear[c] * 255.0f);
    }
    fb.depth[i] = 1.0f;
    fb.id[i] = 0;
  }
  if (f->sky && f->sky->env && f->sky->w > 0 && f->sky->h > 0)
    sky_pass(&fb, f->sky);
  for (uint32_t di = 0; di < n; di++) {
    const OrDraw *d = &draws[di];
    /* cpu_draw, cpu_backend.c:536-544 and 621-627: a read-only depth test
     * keeps the depth buffer as it was before the draw */
    float *saved = NULL;
    if (d->depth_test && !d->depth_write) {
      saved = malloc(px * 4);
      if (saved)
        memcpy(saved, fb.depth, px * 4);
    }
    for (uint32_t i = 0; i + 2 < d->index_count; i += 3) {
      uint32_t ix[3] = {d->indices[i], d->indices[i + 1], d->indices[i + 2]};
      if (ix[0] >= d->vertex_count || ix[1] >= d->vertex_count || ix[2] >= d->vertex_count)
        continue;
      CV tri[3];
      for (int k = 0; k < 3; k++)
        prepare_vertex(d, d->vertices + (size_t)ix[k] * 12, &tri[k]);
      triangle(tri, d, f->ibl, &fb);
    }
    if (saved) {
      memcpy(fb.depth, saved, px * 4);
      free(saved);
    }
  }
  if (f->hdr)
    memcpy(f->hdr, fb.hdr, px * 16);
  hdr_resolve(&fb, f->exposure);
  postprocess(&fb, f->post_effects, f);
  if (f->color_full)
    memcpy(f->color_full, fb.color, px * 4);
  if (f->depth)
    memcpy(f->depth, fb.depth, px * 4);
  if (f->object_id)
    memcpy(f->object_id, fb.id, px * 4);
  if (f->color_presented) {
    int sf = f->ssaa > 0 ? f->ssaa : 1;
    int pw = f->width / sf, ph = f->height / sf;
    for (int y = 0; y < ph; y++)
      for (int x = 0; x < pw; x++) {
        int acc[4] = {0, 0, 0, 0};
        for (int dy = 0; dy < sf; dy++)
          for (int dx = 0; dx < sf; dx++) {
            const uint8_t *p = &fb.color[(((size_t)(y * sf + dy)) * f->width + x * sf + dx) * 4];
            for (int c = 0; c < 4; c++)
              acc[c] += p[c];
          }
        for (int c = 0; c < 4; c++)
          f->color_presented[((size_t)y * pw + x) * 4 + c] = (uint8_t)(acc[c] / (sf * sf));
      }
  }
  free(fb.hdr);
  free(fb.depth);
  free(fb.id);
  free(fb.color);
  g_shadow = NULL;
  return 0;
}

void oracle_pick(const uint32_t *object_id, const float *depth, int width, int height,
                 int ssaa, int n, const int32_t *xy, uint32_t *ids, float *depths,
                 int32_t *hits) {
  int sw = width * ssaa, sh = height * ssaa;
  for (int i = 0; i < n; i++) {
    int x = xy[2 * i], y = xy[2 * i + 1];
    ids[i] = 0;
    depths[i] = 1.0f;
    hits[i] = 0;
    if (x < 0 || x >= width || y < 0 || y >= height)
      continue;
    int rx = x * ssaa, ry = y * ssaa;
    if (rx < 0 || rx >= sw || ry < 0 || ry >= sh)
      continue;
    uint32_t id = object_id[(size_t)ry * sw + rx];
    if (id != 0) {
      ids[i] = id;
      depths[i] = depth[(size_t)ry * sw + rx];
      hits[i] = 1;
    }
  }
}

/* ------------------------------------------------------------------------
 * vertex deformation (reference src/core/viewport.c:1572-1680, 1763-1804)
 * ------------------------------------------------------------------------ */
void oracle_skin_apply(const OrDeformLayout *l, const uint8_t *bind, uint32_t vc,
                       const float *bones, uint32_t bone_count, uint8_t *dst) {
  memcpy(dst, bind, (size_t)vc * l->stride);
  for (uint32_t v = 0; v < vc; v++) {
    const uint8_t *vert = bind + (size_t)v * l->stride;
    uint8_t *out = dst + (size_t)v * l->stride;
    const uint8_t *jd = vert + l->joints_offset;
    float w[4], p[3];
    memcpy(w, vert + l->weights_offset, sizeof w);
    memcpy(p, vert + l->position_offset, sizeof p);
    float sx = 0, sy = 0, sz = 0;
    for (int b = 0; b < 4; b++) {
      if (w[b] <= 0.0f || jd[b] >= bone_count)
        continue;
      const float *m = bones + 16 * (size_t)jd[b];
      float rx = m[0] * p[0] + m[4] * p[1] + m[8] * p[2] + m[12];
      float ry = m[1] * p[0] + m[5] * p[1] + m[9] * p[2] + m[13];
      float rz = m[2] * p[0] + m[6] * p[1] + m[10] * p[2] + m[14];
      sx += w[b] * rx;
      sy += w[b] * ry;
      sz += w[b] * rz;
    }
    float o[3] = {sx, sy, sz};
    memcpy(out + l->position_offset, o, sizeof o);
    if (l->normal_offset >= 0) {
      float n[3];
      memcpy(n, vert + l->normal_offset, sizeof n);
      float nx = 0, ny = 0, nz = 0;
      for (int b = 0; b < 4; b++) {
        if (w[b] <= 0.0f || jd[b] >= bone_count)
          continue;
        const float *m = bones + 16 * (size_t)jd[b];
        float rx = m[0] * n[0] + m[4] * n[1] + m[8] * n[2];
        float ry = m[1] * n[0] + m[5] * n[1] + m[9] * n[2];
        float rz = m[2] * n[0] + m[6] * n[1] + m[10] * n[2];
        nx += w[b] * rx;
        ny += w[b] * ry;
        nz += w[b] * rz;
      }
      float len = sqrtf(nx * nx + ny * ny + nz * nz);
      if (len > 1e-8f) {
        nx /= len;
        ny /= len;
        nz /= len;
      }
      float on[3] = {nx, ny, nz};
      memcpy(out + l->normal_offset, on, sizeof on);
    }
  }
}

void oracle_morph_apply(const OrDeformLayout *l, const uint8_t *bind, uint32_t vc,
                        const float *targets, const float *weights, uint32_t tc, uint8_t *dst) {
  memcpy(dst, bind, (size_t)vc * l->stride);
  for (uint32_t t = 0; t < tc; t++) {
    float w = weights[t];
    if (w == 0.0f)
      continue;
    const float *d = targets + (size_t)t * vc * 3;
    for (uint32_t v = 0; v < vc; v++) {
      float pos[3];
      uint8_t *q = dst + (size_t)v * l->stride + l->position_offset;
      memcpy(pos, q, sizeof pos);
      pos[0] += w * d[v * 3 + 0];
      pos[1] += w * d[v * 3 + 1];
      pos[2] += w * d[v * 3 + 2];
      memcpy(q, pos, sizeof pos);
    }
  }
}

/* ------------------------------------------------------------------------
 * .mop v2 mesh section decode, mop_scene.c:142-223, 397-486
 * ------------------------------------------------------------------------ */
int oracle_mop_decode_mesh(const uint8_t *sec, uint64_t size, float *out_v, uint32_t *out_i) {
  if (size < 48)
    return -1;
  uint32_t h[4];
  float bmin[3], bmax[3];
  memcpy(h, sec, 16);
  memcpy(bmin, sec + 16, 12);
  memcpy(bmax, sec + 28, 12);
  const uint32_t vc = h[0], ic = h[1];
  const int quant = h[2] == 1, idx16 = h[3] == 2;
  const uint64_t vb = (uint64_t)vc * (quant ? 18u : 48u), ib = (uint64_t)ic * (idx16 ? 2u : 4u);
  const uint64_t vb8 = (vb + 7u) & ~(uint64_t)7u;
  if (48 + vb8 + ib > size)
    return -1;
  const uint8_t *vd = sec + 48, *id = sec + 48 + vb8;
  for (uint32_t k = 0; k < vc; k++) {
    float *o = out_v + (size_t)k * 12;
    if (!quant) {
      memcpy(o, vd + (size_t)k * 48, 48);
      continue;
    }
    uint16_t q[9];
    memcpy(q, vd + (size_t)k * 18, 18);
    for (int i = 0; i < 3; i++) {
      float range = bmax[i] - bmin[i];
      o[i] = bmin[i] + ((float)q[i] / 65535.0f) * range;
    }
    float ox = (float)(int16_t)q[3] / 32767.0f, oy = (float)(int16_t)q[4] / 32767.0f;
    float nz = 1.0f - fabsf(ox) - fabsf(oy);
    if (nz < 0.0f) {
      float tx = (1.0f - fabsf(oy)) * (ox >= 0.0f ? 1.0f : -1.0f);
      float ty = (1.0f - fabsf(ox)) * (oy >= 0.0f ? 1.0f : -1.0f);
      ox = tx;
      oy = ty;
    }
    float nx = ox, ny = oy;
    float len = sqrtf(nx * nx + ny * ny + nz * nz);
    if (len > 1e-8f) {
      nx /= len;
      ny /= len;
      nz /= len;
    }
    o[3] = nx;
    o[4] = ny;
    o[5] = nz;
    o[6] = (float)(q[5] & 0xffu) / 255.0f;
    o[7] = (float)(q[5] >> 8) / 255.0f;
    o[8] = (float)(q[6] & 0xffu) / 255.0f;
    o[9] = (float)(q[6] >> 8) / 255.0f;
    o[10] = (float)q[7] / 65535.0f;
    o[11] = (float)q[8] / 65535.0f;
  }
  for (uint32_t k = 0; k < ic; k++) {
    if (idx16) {
      uint16_t x;
      memcpy(&x, id + (size_t)k * 2, 2);
      out_i[k] = x;
    } else {
      memcpy(&out_i[k], id + (size_t)k * 4, 4);
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------
 * BC texture decode: bc_decode_rgb565, bc1/bc4/bc3/bc5_decode_block and
 * bc_decompress_to_rgba8 (reference cpu_backend.c:859-1014), integer
 * arithmetic with the same truncating divisions.
 * ------------------------------------------------------------------------ */
static void or_rgb565(unsigned c, unsigned o[3]) {
  o[0] = ((c >> 11) & 0x1Fu) * 255u / 31u;
  o[1] = ((c >> 5) & 0x3Fu) * 255u / 63u;
  o[2] = (c & 0x1Fu) * 255u / 31u;
}

/* colour block (8 bytes) -> 16 texels of 4 bytes, texel t = y * 4 + x */
static void or_bc1_block(const uint8_t *b, uint8_t tex[16][4]) {
  unsigned c0 = (unsigned)b[0] | ((unsigned)b[1] << 8), c1 = (unsigned)b[2] | ((unsigned)b[3] << 8);
  unsigned pal[4][4];
  or_rgb565(c0, pal[0]);
  or_rgb565(c1, pal[1]);
  pal[0][3] = pal[1][3] = 255u;
  for (int i = 0; i < 3; i++) {
    if (c0 > c1) {
      pal[2][i] = (2u * pal[0][i] + pal[1][i] + 1u) / 3u;
      pal[3][i] = (pal[0][i] + 2u * pal[1][i] + 1u) / 3u;
    } else {
      pal[2][i] = (pal[0][i] + pal[1][i]) / 2u;
      pal[3][i] = 0u;
    }
  }
  pal[2][3] = 255u;
  pal[3][3] = c0 > c1 ? 255u : 0u;
  unsigned lut = (unsigned)b[4] | ((unsigned)b[5] << 8) | ((unsigned)b[6] << 16) |
                 ((unsigned)b[7] << 24);
  for (int t = 0; t < 16; t++)
    for (int k = 0; k < 4; k++)
      tex[t][k] = (uint8_t)pal[(lut >> (2 * t)) & 3u][k];
}

/* one-channel block (8 bytes) into channel ch of the 16 texels */
static void or_bc4_block(const uint8_t *b, uint8_t tex[16][4], int ch) {
  unsigned a0 = b[0], a1 = b[1], pal[8];
  uint64_t bits = 0;
  for (int i = 0; i < 6; i++)
    bits |= (uint64_t)b[2 + i] << (8 * i);
  pal[0] = a0;
  pal[1] = a1;
  if (a0 > a1) {
    for (unsigned i = 1; i <= 6; i++)
      pal[1 + i] = ((7u - i) * a0 + i * a1 + 3u) / 7u;
  } else {
    for (unsigned i = 1; i <= 4; i++)
      pal[1 + i] = ((5u - i) * a0 + i * a1 + 2u) / 5u;
    pal[6] = 0u;
    pal[7] = 255u;
  }
  for (int t = 0; t < 16; t++)
    tex[t][ch] = (uint8_t)pal[(bits >> (3 * t)) & 7u];
}

int oracle_bc_decode(int format, int w, int h, const uint8_t *blocks, uint8_t *out) {
  if (format < 1 || format > 3 || w <= 0 || h <= 0)
    return -1;
  int bw = (w + 3) / 4, bh = (h + 3) / 4;
  size_t bs = format == 1 ? 8 : 16;
  for (int by = 0; by < bh; by++)
    for (int bx = 0; bx < bw; bx++) {
      const uint8_t *b = blocks + ((size_t)by * bw + bx) * bs;
      uint8_t tex[16][4];
      if (format == 1) {
        or_bc1_block(b, tex);
      } else if (format == 2) {
        or_bc1_block(b + 8, tex);
        or_bc4_block(b, tex, 3);
      } else {
        for (int t = 0; t < 16; t++) {
          tex[t][0] = tex[t][1] = tex[t][2] = 0;
          tex[t][3] = 255;
        }
        or_bc4_block(b, tex, 0);
        or_bc4_block(b + 8, tex, 1);
      }
      for (int ty = 0; ty < 4 && by * 4 + ty < h; ty++)
        for (int tx = 0; tx < 4 && bx * 4 + tx < w; tx++)
          memcpy(out + (((size_t)(by * 4 + ty)) * w + bx * 4 + tx) * 4, tex[ty * 4 + tx], 4);
    }
  return 0;
}
