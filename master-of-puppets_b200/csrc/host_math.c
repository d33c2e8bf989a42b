/*
 * host_math.c — the host-side matrix work of the frame path (C11).
 *
 * The device receives finished matrices; these helpers produce them with
 * the reference's exact float operation order so that mvp, world and
 * camera matrices match the CPU backend bit for bit:
 *   column-major multiply        reference src/math/math.c:182-194
 *   TRS compose T*Rz*Ry*Rx*S     math.c:205-215 (rotations :132-162)
 *   look_at / perspective        math.c:69-79, 111-130
 *   camera chain                 mop_viewport_set_camera viewport.c:1058-1093,
 *                                orbit re-application each frame
 *                                camera.c:35-63 -> viewport.c:1095-1128
 *   ortho, shadow light camera   math.c:93-109, pass_shadow viewport.c:2303-2427
 * sinf/cosf/tanf/atan2f/asinf are the host C library's, as in the reference.
 * Compiled with -ffp-contract=off (no FMA contraction).
 */
#include "../../include/mop_cuda.h"

#include <math.h>
#include <string.h>

#define E(m, r, c) ((m)[(c)*4 + (r)])

void mopcuda_mat4_multiply(const float a[16], const float b[16], float out[16]) {
  if (!a || !b || !out)
    return;
  float r[16];
  for (int c = 0; c < 4; c++)
    for (int row = 0; row < 4; row++) {
      float s = 0.0f;
      for (int k = 0; k < 4; k++)
        s += E(a, row, k) * E(b, k, c);
      E(r, row, c) = s;
    }
  memcpy(out, r, sizeof r);
}

static void ident(float m[16]) {
  memset(m, 0, 16 * sizeof(float));
  m[0] = m[5] = m[10] = m[15] = 1.0f;
}

void mopcuda_mat4_compose_trs(const float pos[3], const float rot[3], const float scl[3],
                              float out[16]) {
  if (!pos || !rot || !scl || !out)
    return;
  float s[16], rx[16], ry[16], rz[16], t[16], m1[16], m2[16], m3[16];
  memset(s, 0, sizeof s);
  E(s, 0, 0) = scl[0];
  E(s, 1, 1) = scl[1];
  E(s, 2, 2) = scl[2];
  E(s, 3, 3) = 1.0f;
  float c = cosf(rot[0]), n = sinf(rot[0]);
  ident(rx);
  E(rx, 1, 1) = c;
  E(rx, 1, 2) = -n;
  E(rx, 2, 1) = n;
  E(rx, 2, 2) = c;
  c = cosf(rot[1]);
  n = sinf(rot[1]);
  ident(ry);
  E(ry, 0, 0) = c;
  E(ry, 0, 2) = n;
  E(ry, 2, 0) = -n;
  E(ry, 2, 2) = c;
  c = cosf(rot[2]);
  n = sinf(rot[2]);
  ident(rz);
  E(rz, 0, 0) = c;
  E(rz, 0, 1) = -n;
  E(rz, 1, 0) = n;
  E(rz, 1, 1) = c;
  ident(t);
  E(t, 0, 3) = pos[0];
  E(t, 1, 3) = pos[1];
  E(t, 2, 3) = pos[2];
  mopcuda_mat4_multiply(rx, s, m1);
  mopcuda_mat4_multiply(ry, m1, m2);
  mopcuda_mat4_multiply(rz, m2, m3);
  mopcuda_mat4_multiply(t, m3, out);
}

typedef struct {
  float x, y, z;
} v3;

static float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

static v3 unit(v3 a) {
  float l = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
  if (l < 1e-8f) {
    v3 z = {0.0f, 0.0f, 0.0f};
    return z;
  }
  float inv = 1.0f / l;
  v3 r = {a.x * inv, a.y * inv, a.z * inv};
  return r;
}

static v3 cross(v3 a, v3 b) {
  v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return r;
}

/* mop_mat4_look_at, math.c:111-130 */
static void look_at(v3 e, v3 t, v3 u, float view[16]) {
  v3 f = unit((v3){t.x - e.x, t.y - e.y, t.z - e.z});
  v3 s = unit(cross(f, u));
  v3 uu = cross(s, f);
  ident(view);
  E(view, 0, 0) = s.x;
  E(view, 0, 1) = s.y;
  E(view, 0, 2) = s.z;
  E(view, 1, 0) = uu.x;
  E(view, 1, 1) = uu.y;
  E(view, 1, 2) = uu.z;
  E(view, 2, 0) = -f.x;
  E(view, 2, 1) = -f.y;
  E(view, 2, 2) = -f.z;
  E(view, 0, 3) = -dot(s, e);
  E(view, 1, 3) = -dot(uu, e);
  E(view, 2, 3) = dot(f, e);
}

/* The orbit parameters mop_viewport_set_camera recovers from eye and
 * target (viewport.c:1079-1091), re-applied by mop_viewport_render: the eye
 * and up vector the frame uses. */
static void orbit(const float eye[3], const float target[3], const float up[3], v3 *e_out,
                  v3 *u_out) {
  v3 e = {eye[0], eye[1], eye[2]}, t = {target[0], target[1], target[2]};
  v3 u = {up[0], up[1], up[2]};
  v3 off = {e.x - t.x, e.y - t.y, e.z - t.z};
  float dist = sqrtf(off.x * off.x + off.y * off.y + off.z * off.z);
  if (dist > 1e-6f) {
    float yaw = atan2f(off.x, off.z);
    float pitch = asinf(off.y / dist);
    float sp = sinf(pitch), cp = cosf(pitch), sy = sinf(yaw), cy = cosf(yaw);
    v3 ou = {-sp * sy, cp, -sp * cy};
    u = ou;
    float cp2 = cosf(pitch);
    v3 oe = {t.x + dist * cp2 * sinf(yaw), t.y + dist * sinf(pitch),
             t.z + dist * cp2 * cosf(yaw)};
    e = oe;
  }
  *e_out = e;
  *u_out = u;
}

void mopcuda_camera_orbit(const float eye[3], const float target[3], const float up[3],
                          float eye_out[3], float up_out[3]) {
  if (!eye || !target || !up || !eye_out || !up_out)
    return;
  v3 e, u;
  orbit(eye, target, up, &e, &u);
  eye_out[0] = e.x;
  eye_out[1] = e.y;
  eye_out[2] = e.z;
  up_out[0] = u.x;
  up_out[1] = u.y;
  up_out[2] = u.z;
}

void mopcuda_camera_matrices(const float eye[3], const float target[3], const float up[3],
                             float fov_deg, float near_plane, float far_plane, int width,
                             int height, float view[16], float proj[16], float eye_out[3]) {
  if (!eye || !target || !up || !view || !proj || !eye_out)
    return;
  v3 t = {target[0], target[1], target[2]};
  v3 e, u;
  orbit(eye, target, up, &e, &u);
  look_at(e, t, u, view);
  float fov = fov_deg * (3.14159265358979323846f / 180.0f);
  float aspect = (float)width / (float)height;
  float th = tanf(fov * 0.5f);
  memset(proj, 0, 16 * sizeof(float));
  E(proj, 0, 0) = 1.0f / (aspect * th);
  E(proj, 1, 1) = 1.0f / th;
  E(proj, 2, 2) = -(far_plane + near_plane) / (far_plane - near_plane);
  E(proj, 3, 2) = -1.0f;
  E(proj, 2, 3) = -(2.0f * far_plane * near_plane) / (far_plane - near_plane);
  eye_out[0] = e.x;
  eye_out[1] = e.y;
  eye_out[2] = e.z;
}

/* mop_mat4_ortho, math.c:93-109 */
static void ortho(float l, float r, float b, float t, float n, float f, float m[16]) {
  float rl = r - l, tb = t - b, fn = f - n;
  if (fabsf(rl) < 1e-9f || fabsf(tb) < 1e-9f || fabsf(fn) < 1e-9f) {
    ident(m);
    return;
  }
  memset(m, 0, 16 * sizeof(float));
  E(m, 0, 0) = 2.0f / rl;
  E(m, 1, 1) = 2.0f / tb;
  E(m, 2, 2) = -2.0f / fn;
  E(m, 0, 3) = -(r + l) / rl;
  E(m, 1, 3) = -(t + b) / tb;
  E(m, 2, 3) = -(f + n) / fn;
  E(m, 3, 3) = 1.0f;
}

/* pass_shadow's light camera, viewport.c:2303-2427 */
int mopcuda_shadow_light_vp(const float *models, uint32_t count, const float direction[3],
                            float light_vp[16]) {
  if (!models || !direction || !light_vp || count == 0)
    return 0;
  float lo[3] = {1e9f, 1e9f, 1e9f}, hi[3] = {-1e9f, -1e9f, -1e9f};
  for (uint32_t i = 0; i < count; i++) {
    const float *m = models + 16 * (size_t)i;
    const float c[3] = {m[12], m[13], m[14]};
    float sx = sqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    float sy = sqrtf(m[4] * m[4] + m[5] * m[5] + m[6] * m[6]);
    float sz = sqrtf(m[8] * m[8] + m[9] * m[9] + m[10] * m[10]);
    float r = sx > sy ? sx : sy;
    if (sz > r)
      r = sz;
    r *= 1.5f;
    for (int k = 0; k < 3; k++)
      if (c[k] - r < lo[k])
        lo[k] = c[k] - r;
    for (int k = 0; k < 3; k++)
      if (c[k] + r > hi[k])
        hi[k] = c[k] + r;
  }
  v3 d = unit((v3){direction[0], direction[1], direction[2]});
  v3 ctr = {(lo[0] + hi[0]) * 0.5f, (lo[1] + hi[1]) * 0.5f, (lo[2] + hi[2]) * 0.5f};
  float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
  float radius = sqrtf(dx * dx + dy * dy + dz * dz) * 0.5f;
  if (radius < 1.0f)
    radius = 1.0f;
  v3 eye = {ctr.x - d.x * radius * 2.0f, ctr.y - d.y * radius * 2.0f,
            ctr.z - d.z * radius * 2.0f};
  v3 up = {0.0f, 1.0f, 0.0f};
  if (fabsf(dot(d, up)) > 0.99f)
    up = (v3){1.0f, 0.0f, 0.0f};
  float view[16], proj[16];
  look_at(eye, ctr, up, view);
  float size = radius * 1.2f;
  ortho(-size, size, -size, size, 0.1f, radius * 4.0f, proj);
  mopcuda_mat4_multiply(proj, view, light_vp);
  return 1;
}
