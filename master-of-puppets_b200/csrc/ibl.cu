/*
 * ibl.cu — image-based-lighting precompute on the device: the procedural
 * sky and the three maps the frame's IBL lookups read (reference
 * src/core/environment.c):
 *
 *   generate_procedural_sky   environment.c:493-620  (512x256 Preetham sky)
 *   precompute_irradiance     environment.c:111-222  (64x32, 128 cosine samples)
 *   precompute_prefiltered    environment.c:224-376  (128x64, 5 levels, 64 GGX samples)
 *   precompute_brdf_lut       environment.c:378-484  (256x256, 64 samples)
 *
 * Every output texel is one thread that sums its samples in the reference's
 * order with the reference's float operations (no contraction).  Values the
 * reference takes from sinf/cosf/tanf/expf of per-texel or per-sample
 * constants — texel directions and tangent frames, Hammersley sample
 * directions, the sky's Preetham coefficients — are computed here on the
 * host with the same C library, so they are bit-identical; the device then
 * only adds, multiplies, divides and takes square roots (all correctly
 * rounded).  The BRDF LUT is therefore bit-exact.  The per-sample atan2f /
 * asinf of the equirectangular lookup and the sky's per-texel acosf / cosf /
 * expf are CUDA's: the x86 C library's differ from them (and from the
 * correctly rounded value) in the last place for a fraction of inputs, so
 * the sky, irradiance and prefiltered maps agree with the core's to float
 * rounding, not bit for bit.
 */
#include "api_internal.h"

#include <math.h>
#include <string.h>

namespace {

constexpr int IRR_W = 64, IRR_H = 32, IRR_SAMPLES = 128;
constexpr int PF_W = 128, PF_H = 64, PF_LEVELS = 5, PF_SAMPLES = 64;
constexpr int BRDF_SIZE = 256, BRDF_SAMPLES = 64;
constexpr int SKY_W = 512, SKY_H = 256;
constexpr float PI_F = 3.14159265358979323846f; /* (float)M_PI */

int pf_texels() {
  int n = 0;
  for (int l = 0; l < PF_LEVELS; l++)
    n += std::max(1, PF_W >> l) * std::max(1, PF_H >> l);
  return n;
}

/* Host tables, one device buffer; float offsets. */
struct IblTables {
  size_t irr_basis, irr_dirs, pf_basis, pf_dirs, brdf_phi, sky_rows, sky_cols, total;
};

IblTables table_layout() {
  IblTables t;
  size_t o = 0;
  t.irr_basis = o;
  o += (size_t)IRR_W * IRR_H * 12;
  t.irr_dirs = o;
  o += (size_t)IRR_SAMPLES * 4;
  t.pf_basis = o;
  o += (size_t)pf_texels() * 12;
  t.pf_dirs = o;
  o += (size_t)PF_LEVELS * PF_SAMPLES * 4;
  t.brdf_phi = o;
  o += (size_t)BRDF_SAMPLES * 4;
  t.sky_rows = o;
  o += (size_t)SKY_H * 4;
  t.sky_cols = o;
  o += (size_t)SKY_W * 4;
  t.total = o;
  return t;
}

/* The texel's direction and tangent frame, environment.c:125-165 (and the
 * same lines of precompute_prefiltered): t, n, b as 3 x float4. */
void texel_frame(int x, int y, int w, int h, float *out) {
  float u = ((float)x + 0.5f) / (float)w;
  float v = ((float)y + 0.5f) / (float)h;
  float phi = (u - 0.5f) * 2.0f * PI_F;
  float theta = (v - 0.5f) * PI_F;
  float ct = cosf(theta);
  float nx = ct * cosf(phi);
  float ny = sinf(theta);
  float nz = ct * sinf(phi);
  float len = sqrtf(nx * nx + ny * ny + nz * nz);
  nx /= len;
  ny /= len;
  nz /= len;
  float upx = 0.0f, upy = 1.0f, upz = 0.0f;
  if (fabsf(ny) > 0.99f) {
    upx = 0.0f;
    upy = 0.0f;
    upz = 1.0f;
  }
  float tx = upy * nz - upz * ny;
  float ty = upz * nx - upx * nz;
  float tz = upx * ny - upy * nx;
  float tlen = sqrtf(tx * tx + ty * ty + tz * tz);
  if (tlen > 1e-6f) {
    tx /= tlen;
    ty /= tlen;
    tz /= tlen;
  }
  float bx = ny * tz - nz * ty;
  float by = nz * tx - nx * tz;
  float bz = nx * ty - ny * tx;
  const float f[12] = {tx, ty, tz, 0.0f, nx, ny, nz, 0.0f, bx, by, bz, 0.0f};
  memcpy(out, f, sizeof f);
}

/* Hammersley point s of n: xi1 = s/n, xi2 = the bit-reversed index. */
void hammersley(int s, int n, float *xi1, float *xi2) {
  *xi1 = (float)s / (float)n;
  uint32_t bits = (uint32_t)s;
  bits = (bits << 16u) | (bits >> 16u);
  bits = ((bits & 0x55555555u) << 1u) | ((bits & 0xAAAAAAAAu) >> 1u);
  bits = ((bits & 0x33333333u) << 2u) | ((bits & 0xCCCCCCCCu) >> 2u);
  bits = ((bits & 0x0F0F0F0Fu) << 4u) | ((bits & 0xF0F0F0F0u) >> 4u);
  bits = ((bits & 0x00FF00FFu) << 8u) | ((bits & 0xFF00FF00u) >> 8u);
  *xi2 = (float)bits * 2.3283064365386963e-10f;
}

float pf_alpha2(int l) {
  float roughness = (float)l / (float)(PF_LEVELS - 1);
  float alpha = roughness * roughness;
  float alpha2 = alpha * alpha;
  return alpha2 < 1e-7f ? 1e-7f : alpha2;
}

void build_tables(const IblTables &L, float *t) {
  memset(t, 0, L.total * sizeof(float));
  for (int y = 0; y < IRR_H; y++)
    for (int x = 0; x < IRR_W; x++)
      texel_frame(x, y, IRR_W, IRR_H, t + L.irr_basis + ((size_t)y * IRR_W + x) * 12);
  for (int s = 0; s < IRR_SAMPLES; s++) { /* environment.c:172-190 */
    float xi1, xi2;
    hammersley(s, IRR_SAMPLES, &xi1, &xi2);
    float cos_theta_s = sqrtf(xi1);
    float sin_theta_s = sqrtf(1.0f - xi1);
    float phi_s = 2.0f * PI_F * xi2;
    float *d = t + L.irr_dirs + (size_t)s * 4;
    d[0] = sin_theta_s * cosf(phi_s);
    d[1] = cos_theta_s;
    d[2] = sin_theta_s * sinf(phi_s);
  }
  size_t off = 0;
  for (int l = 0; l < PF_LEVELS; l++) {
    int w = std::max(1, PF_W >> l), h = std::max(1, PF_H >> l);
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++)
        texel_frame(x, y, w, h, t + L.pf_basis + (off + (size_t)y * w + x) * 12);
    off += (size_t)w * h;
    const float alpha2 = pf_alpha2(l);
    for (int s = 0; s < PF_SAMPLES; s++) { /* environment.c:310-328 */
      float xi1, xi2;
      hammersley(s, PF_SAMPLES, &xi1, &xi2);
      float cos_theta_h = sqrtf((1.0f - xi1) / (1.0f + (alpha2 - 1.0f) * xi1));
      float sin_theta_h = sqrtf(1.0f - cos_theta_h * cos_theta_h);
      float phi_h = 2.0f * PI_F * xi2;
      float *d = t + L.pf_dirs + ((size_t)l * PF_SAMPLES + s) * 4;
      d[0] = sin_theta_h * cosf(phi_h);
      d[1] = cos_theta_h;
      d[2] = sin_theta_h * sinf(phi_h);
    }
  }
  for (int s = 0; s < BRDF_SAMPLES; s++) { /* environment.c:421-439 */
    float xi1, xi2;
    hammersley(s, BRDF_SAMPLES, &xi1, &xi2);
    float phi_h = 2.0f * PI_F * xi2;
    float *d = t + L.brdf_phi + (size_t)s * 4;
    d[0] = cosf(phi_h);
    d[1] = sinf(phi_h);
  }
  for (int y = 0; y < SKY_H; y++) { /* environment.c:561-569 */
    float v = ((float)y + 0.5f) / (float)SKY_H;
    float theta = (v - 0.5f) * PI_F;
    t[L.sky_rows + (size_t)y * 4 + 0] = cosf(theta);
    t[L.sky_rows + (size_t)y * 4 + 1] = sinf(theta);
  }
  for (int x = 0; x < SKY_W; x++) {
    float u = ((float)x + 0.5f) / (float)SKY_W;
    float phi = (u - 0.5f) * 2.0f * PI_F;
    t[L.sky_cols + (size_t)x * 4 + 0] = cosf(phi);
    t[L.sky_cols + (size_t)x * 4 + 1] = sinf(phi);
  }
}

/* Preetham constants of generate_procedural_sky (environment.c:514-551). */
struct SkyArgs {
  float sun[3];
  float A, B, C, D, E;
  float Yz, F0, ground;
};

float perez_host(float theta, float gamma, float A, float B, float C, float D, float E) {
  float ct = cosf(theta);
  if (ct < 0.001f)
    ct = 0.001f;
  float cg = cosf(gamma);
  return (1.0f + A * expf(B / ct)) * (1.0f + C * expf(D * gamma) + E * cg * cg);
}

SkyArgs sky_args(const float sun_dir[3], float turbidity, float ground_albedo) {
  SkyArgs a;
  float T = turbidity;
  if (T < 2.0f)
    T = 2.0f;
  if (T > 10.0f)
    T = 10.0f;
  float sx = sun_dir[0], sy = sun_dir[1], sz = sun_dir[2];
  float slen = sqrtf(sx * sx + sy * sy + sz * sz);
  if (slen < 1e-6f) {
    sx = 0.0f;
    sy = 1.0f;
    sz = 0.0f;
  } else {
    sx /= slen;
    sy /= slen;
    sz /= slen;
  }
  float theta_s = acosf(sy > 1.0f ? 1.0f : (sy < -1.0f ? -1.0f : sy));
  a.A = 0.1787f * T - 1.4630f;
  a.B = -0.3554f * T + 0.4275f;
  a.C = -0.0227f * T + 5.3251f;
  a.D = 0.1206f * T - 2.5771f;
  a.E = -0.0670f * T + 0.3703f;
  float chi = (4.0f / 9.0f - T / 120.0f) * (PI_F - 2.0f * theta_s);
  float Yz = (4.0453f * T - 4.9710f) * tanf(chi) - 0.2155f * T + 2.4192f;
  if (Yz < 0.0f)
    Yz = 0.0f;
  float F0 = perez_host(0.0f, theta_s, a.A, a.B, a.C, a.D, a.E);
  if (F0 < 1e-6f)
    F0 = 1e-6f;
  a.sun[0] = sx;
  a.sun[1] = sy;
  a.sun[2] = sz;
  a.Yz = Yz;
  a.F0 = F0;
  a.ground = ground_albedo;
  return a;
}

/* ------------------------------------------------------------------------
 * device
 * ------------------------------------------------------------------------ */
/* sample_hdr_bilinear, environment.c:32-60 */
__device__ __forceinline__ float4 env_bilinear(const float4 *__restrict__ d, int w, int h, float u,
                                               float v) {
  u = u - floorf(u);
  v = v - floorf(v);
  float fx = u * (float)(w - 1);
  float fy = v * (float)(h - 1);
  int x0 = (int)fx, y0 = (int)fy;
  int x1 = (x0 + 1) % w;
  int y1 = y0 + 1;
  if (y1 >= h)
    y1 = h - 1;
  float sx = fx - (float)x0, sy = fy - (float)y0;
  const float4 p00 = __ldg(d + ((size_t)y0 * w + x0)), p10 = __ldg(d + ((size_t)y0 * w + x1));
  const float4 p01 = __ldg(d + ((size_t)y1 * w + x0)), p11 = __ldg(d + ((size_t)y1 * w + x1));
  float4 o;
  float top, bot;
  top = p00.x * (1.0f - sx) + p10.x * sx;
  bot = p01.x * (1.0f - sx) + p11.x * sx;
  o.x = top * (1.0f - sy) + bot * sy;
  top = p00.y * (1.0f - sx) + p10.y * sx;
  bot = p01.y * (1.0f - sx) + p11.y * sx;
  o.y = top * (1.0f - sy) + bot * sy;
  top = p00.z * (1.0f - sx) + p10.z * sx;
  bot = p01.z * (1.0f - sx) + p11.z * sx;
  o.z = top * (1.0f - sy) + bot * sy;
  o.w = 1.0f;
  return o;
}

/* dir_to_equirect with rotation 0, environment.c:63-70 */
__device__ __forceinline__ float4 env_dir(const float4 *__restrict__ env, int w, int h, float dx,
                                          float dy, float dz) {
  float phi = atan2f(dz, dx) + 0.0f;
  float theta = asinf(dy < -1.0f ? -1.0f : (dy > 1.0f ? 1.0f : dy));
  float u = phi / (2.0f * PI_F) + 0.5f;
  float v = theta / PI_F + 0.5f;
  return env_bilinear(env, w, h, u, v);
}

struct IblDev {
  const float4 *env;
  int env_w, env_h;
  const float4 *tab; /* the host tables (float4 units) */
  IblTables L;       /* float offsets (multiples of 4) */
  float4 *irr, *pf, *brdf, *sky;
  int pf_texels;
  SkyArgs sky_args;
};

/* Both convolutions run a warp per texel: each lane evaluates one of 32
 * consecutive samples (direction, equirect coordinates, bilinear fetch),
 * then the warp adds the 32 values one lane at a time in sample order, so
 * every sum is accumulated in exactly the order of the serial loop. */
static_assert(IRR_SAMPLES % 32 == 0 && PF_SAMPLES % 32 == 0, "samples in whole warps");

__global__ void __launch_bounds__(128) k_ibl_irradiance(IblDev a) {
  const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); /* warp-uniform */
  const int lane = (int)(threadIdx.x & 31u);
  if (i >= IRR_W * IRR_H)
    return;
  const float4 *fr = a.tab + a.L.irr_basis / 4 + (size_t)i * 3;
  const float4 T = fr[0], N = fr[1], B = fr[2];
  const float4 *dirs = a.tab + a.L.irr_dirs / 4;
  float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f, total = 0.0f;
  for (int s0 = 0; s0 < IRR_SAMPLES; s0 += 32) {
    const float4 l = dirs[s0 + lane];
    const float wx = T.x * l.x + N.x * l.y + B.x * l.z;
    const float wy = T.y * l.x + N.y * l.y + B.y * l.z;
    const float wz = T.z * l.x + N.z * l.y + B.z * l.z;
    const float4 c = env_dir(a.env, a.env_w, a.env_h, wx, wy, wz);
#pragma unroll 8
    for (int j = 0; j < 32; j++) {
      acc0 += __shfl_sync(0xffffffffu, c.x, j);
      acc1 += __shfl_sync(0xffffffffu, c.y, j);
      acc2 += __shfl_sync(0xffffffffu, c.z, j);
      total += 1.0f;
    }
  }
  if (lane != 0)
    return;
  float4 o = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
  if (total > 0.0f) {
    o.x = acc0 / total;
    o.y = acc1 / total;
    o.z = acc2 / total;
  }
  a.irr[i] = o;
}

__global__ void __launch_bounds__(128) k_ibl_prefilter(IblDev a) {
  const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); /* warp-uniform */
  const int lane = (int)(threadIdx.x & 31u);
  if (i >= a.pf_texels)
    return;
  int l = 0, base = 0;
  for (; l < PF_LEVELS - 1; l++) { /* the level holding texel i */
    const int n = max(1, PF_W >> l) * max(1, PF_H >> l);
    if (i < base + n)
      break;
    base += n;
  }
  const float4 *fr = a.tab + a.L.pf_basis / 4 + (size_t)i * 3;
  const float4 T = fr[0], N = fr[1], B = fr[2];
  const float vx = N.x, vy = N.y, vz = N.z;
  const float4 *dirs = a.tab + a.L.pf_dirs / 4 + (size_t)l * PF_SAMPLES;
  float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f, total = 0.0f;
  for (int s0 = 0; s0 < PF_SAMPLES; s0 += 32) {
    const float4 h = dirs[s0 + lane];
    const float hx = T.x * h.x + N.x * h.y + B.x * h.z;
    const float hy = T.y * h.x + N.y * h.y + B.y * h.z;
    const float hz = T.z * h.x + N.z * h.y + B.z * h.z;
    const float vdh = vx * hx + vy * hy + vz * hz;
    const float lx = 2.0f * vdh * hx - vx;
    const float ly = 2.0f * vdh * hy - vy;
    const float lz = 2.0f * vdh * hz - vz;
    const float ndl = N.x * lx + N.y * ly + N.z * lz;
    const bool use = !(ndl <= 0.0f); /* the serial loop skips ndl <= 0 */
    float px = 0.0f, py = 0.0f, pz = 0.0f;
    if (use) {
      const float4 c = env_dir(a.env, a.env_w, a.env_h, lx, ly, lz);
      px = c.x * ndl;
      py = c.y * ndl;
      pz = c.z * ndl;
    }
    const unsigned m = __ballot_sync(0xffffffffu, use);
#pragma unroll 8
    for (int j = 0; j < 32; j++) {
      const float qx = __shfl_sync(0xffffffffu, px, j);
      const float qy = __shfl_sync(0xffffffffu, py, j);
      const float qz = __shfl_sync(0xffffffffu, pz, j);
      const float qn = __shfl_sync(0xffffffffu, ndl, j);
      if ((m >> j) & 1u) {
        acc0 += qx;
        acc1 += qy;
        acc2 += qz;
        total += qn;
      }
    }
  }
  if (lane != 0)
    return;
  float4 o = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
  if (total > 0.0f) {
    o.x = acc0 / total;
    o.y = acc1 / total;
    o.z = acc2 / total;
  }
  a.pf[i] = o;
}

__global__ void __launch_bounds__(256) k_ibl_brdf(IblDev a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= BRDF_SIZE * BRDF_SIZE)
    return;
  const int x = i % BRDF_SIZE, y = i / BRDF_SIZE;
  const float roughness = ((float)y + 0.5f) / (float)BRDF_SIZE;
  const float alpha = roughness * roughness;
  float alpha2 = alpha * alpha;
  if (alpha2 < 1e-7f)
    alpha2 = 1e-7f;
  const float k = alpha * 0.5f;
  float ndotv = ((float)x + 0.5f) / (float)BRDF_SIZE;
  if (ndotv < 1e-4f)
    ndotv = 1e-4f;
  const float sin_v = sqrtf(1.0f - ndotv * ndotv);
  const float vx_t = sin_v, vy_t = 0.0f, vz_t = ndotv;
  const float4 *phis = a.tab + a.L.brdf_phi / 4;
  float scale = 0.0f, bias = 0.0f;
  for (int s = 0; s < BRDF_SAMPLES; s++) {
    const float xi1 = (float)s / (float)BRDF_SAMPLES;
    const float cos_theta_h = sqrtf((1.0f - xi1) / (1.0f + (alpha2 - 1.0f) * xi1));
    const float sin_theta_h = sqrtf(1.0f - cos_theta_h * cos_theta_h);
    const float4 ph = phis[s];
    const float hx = sin_theta_h * ph.x;
    const float hy = sin_theta_h * ph.y;
    const float hz = cos_theta_h;
    const float vdh = vx_t * hx + vy_t * hy + vz_t * hz;
    const float lz = 2.0f * vdh * hz - vz_t;
    const float ndl = lz;
    if (ndl <= 0.0f)
      continue;
    const float ndh = hz;
    const float vdh_c = vdh > 0.0f ? vdh : 0.0f;
    const float g1v_t = ndotv / (ndotv * (1.0f - k) + k);
    const float g1l_t = ndl / (ndl * (1.0f - k) + k);
    const float g = g1v_t * g1l_t;
    const float vis = (g * vdh_c) / (ndh * ndotv + 1e-6f);
    const float fc = 1.0f - vdh_c;
    const float fc2 = fc * fc;
    const float fc5 = fc2 * fc2 * fc;
    scale += vis * (1.0f - fc5);
    bias += vis * fc5;
  }
  a.brdf[i] = make_float4(scale / (float)BRDF_SAMPLES, bias / (float)BRDF_SAMPLES, 0.0f, 1.0f);
}

__device__ __forceinline__ float perez_dev(float theta, float gamma, const SkyArgs &s) {
  float ct = cosf(theta);
  if (ct < 0.001f)
    ct = 0.001f;
  float cg = cosf(gamma);
  return (1.0f + s.A * expf(s.B / ct)) * (1.0f + s.C * expf(s.D * gamma) + s.E * cg * cg);
}

/* generate_procedural_sky's per-texel loop, environment.c:559-617 */
__global__ void __launch_bounds__(256) k_ibl_sky(IblDev a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= SKY_W * SKY_H)
    return;
  const int x = i % SKY_W, y = i / SKY_W;
  const SkyArgs &s = a.sky_args;
  const float4 rt = a.tab[a.L.sky_rows / 4 + y], pt = a.tab[a.L.sky_cols / 4 + x];
  const float ct = rt.x;
  const float dx = ct * pt.x;
  const float dy = rt.y;
  const float dz = ct * pt.y;
  if (dy < 0.0f) {
    const float ground = s.ground * s.Yz * 0.1f;
    a.sky[i] = make_float4(ground * 0.8f, ground * 0.85f, ground, 1.0f);
    return;
  }
  float theta_p = acosf(dy);
  if (theta_p < 0.001f)
    theta_p = 0.001f;
  const float gamma = acosf(dx * s.sun[0] + dy * s.sun[1] + dz * s.sun[2]);
  const float Fp = perez_dev(theta_p, gamma, s);
  float lum = s.Yz * (Fp / s.F0);
  if (lum < 0.0f)
    lum = 0.0f;
  const float sky_r = 0.3f + 0.1f * (1.0f - dy);
  const float sky_g = 0.5f + 0.2f * (1.0f - dy);
  const float sky_b = 0.9f + 0.1f * dy;
  float sun_intensity = 0.0f;
  if (gamma < 0.02f)
    sun_intensity = 100.0f * (1.0f - gamma / 0.02f);
  else if (gamma < 0.05f)
    sun_intensity = 5.0f * (1.0f - gamma / 0.05f);
  const float scale = lum * 0.5f;
  a.sky[i] = make_float4(sky_r * scale + sun_intensity, sky_g * scale + sun_intensity * 0.95f,
                         sky_b * scale + sun_intensity * 0.8f, 1.0f);
}

/* Uploads the tables, runs the sky (when sky != null) and the three maps on
 * the device stream, and binds the maps as set_ibl does. */
int run_precompute(MopCudaDevice *d, const float *env_host, int env_w, int env_h,
                   const SkyArgs *sky, float rotation, float intensity) {
  const IblTables L = table_layout();
  const int npf = pf_texels();
  int rc = mc_finish_pending(d); /* frames in flight read the maps */
  if (!rc)
    rc = mc_stream_sync(d, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  const size_t env_bytes = (size_t)env_w * env_h * 16;
  rc = 0;
  rc |= d->ibl_tab.ensure(L.total * 4);
  rc |= d->h_ibl.ensure(L.total * 4 + (env_host ? env_bytes : 0));
  rc |= d->env.ensure(env_bytes);
  rc |= d->irr.ensure((size_t)IRR_W * IRR_H * 16);
  rc |= d->pf.ensure((size_t)npf * 16);
  rc |= d->brdf.ensure((size_t)BRDF_SIZE * BRDF_SIZE * 16);
  if (rc)
    return MOPCUDA_ENOMEM;
  float *h = d->h_ibl.as<float>();
  build_tables(L, h);
  cudaStream_t st = d->stream;
  if (!d->ibl_t0) {
    CU_TRY(cudaEventCreate(&d->ibl_t0));
    CU_TRY(cudaEventCreate(&d->ibl_t1));
  }
  CU_TRY(cudaEventRecord(d->ibl_t0, st));
  CU_TRY(cudaMemcpyAsync(d->ibl_tab.p, h, L.total * 4, cudaMemcpyHostToDevice, st));
  if (env_host) {
    memcpy(h + L.total, env_host, env_bytes);
    CU_TRY(cudaMemcpyAsync(d->env.p, h + L.total, env_bytes, cudaMemcpyHostToDevice, st));
  }
  IblDev a;
  memset(&a, 0, sizeof a);
  a.env = d->env.as<float4>();
  a.env_w = env_w;
  a.env_h = env_h;
  a.tab = d->ibl_tab.as<float4>();
  a.L = L;
  a.irr = d->irr.as<float4>();
  a.pf = d->pf.as<float4>();
  a.brdf = d->brdf.as<float4>();
  a.sky = d->env.as<float4>();
  a.pf_texels = npf;
  int launches = 0;
  if (sky) {
    a.sky_args = *sky;
    k_ibl_sky<<<(SKY_W * SKY_H + 255) / 256, 256, 0, st>>>(a);
    launches++;
  }
  k_ibl_irradiance<<<(IRR_W * IRR_H * 32 + 127) / 128, 128, 0, st>>>(a); /* a warp per texel */
  k_ibl_prefilter<<<(npf * 32 + 127) / 128, 128, 0, st>>>(a);
  k_ibl_brdf<<<(BRDF_SIZE * BRDF_SIZE + 255) / 256, 256, 0, st>>>(a);
  launches += 3;
  CU_TRY(cudaGetLastError());
  CU_TRY(cudaEventRecord(d->ibl_t1, st));
  d->launches += (uint64_t)launches;
  d->env_w = env_w;
  d->env_h = env_h;
  d->irr_w = IRR_W;
  d->irr_h = IRR_H;
  d->pf_w = PF_W;
  d->pf_h = PF_H;
  d->pf_levels = PF_LEVELS;
  d->brdf_size = BRDF_SIZE;
  d->ibl_rot = rotation;
  d->ibl_int = intensity > 0.0f ? intensity : 1.0f;
  d->ibl_on = true;
  /* the staging buffer is reused by the next call: wait for the copies */
  return mc_bounded_sync(d, d->ibl_t1, FRAME_TIMEOUT_MS);
}

} // namespace

extern "C" int mopcuda_ibl_from_env(MopCudaDevice *d, const float *env_rgba, int w, int h,
                                    float rotation, float intensity) {
  if (!d || !env_rgba || w < 2 || h < 2 || w > 16384 || h > 16384)
    return fail(MOPCUDA_EINVAL, "ibl_from_env: bad arguments (%dx%d)", w, h);
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  return run_precompute(d, env_rgba, w, h, nullptr, rotation, intensity);
}

extern "C" int mopcuda_ibl_procedural_sky(MopCudaDevice *d, const float sun_dir[3],
                                          float turbidity, float ground_albedo, float rotation,
                                          float intensity) {
  if (!d || !sun_dir)
    return fail(MOPCUDA_EINVAL, "ibl_procedural_sky: bad arguments");
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  const SkyArgs s = sky_args(sun_dir, turbidity, ground_albedo);
  return run_precompute(d, nullptr, SKY_W, SKY_H, &s, rotation, intensity);
}

extern "C" float mopcuda_ibl_gpu_time_ms(MopCudaDevice *d) {
  if (!d || !d->ibl_t1)
    return 0.0f;
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  if (mc_bounded_sync(d, d->ibl_t1, FRAME_TIMEOUT_MS))
    return 0.0f;
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, d->ibl_t0, d->ibl_t1);
  return ms;
}

extern "C" int mopcuda_ibl_read(MopCudaDevice *d, float *irr, size_t irr_bytes, float *pf,
                                size_t pf_bytes, float *brdf, size_t brdf_bytes, float *env,
                                size_t env_bytes) {
  if (!d)
    return fail(MOPCUDA_EINVAL, "ibl_read: no device");
  std::lock_guard<std::mutex> lk(d->mu);
  if (!d->ibl_on)
    return fail(MOPCUDA_EINVAL, "ibl_read: no IBL maps bound");
  cudaSetDevice(d->ordinal);
  int rc = mc_stream_sync(d, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  size_t pf_px = 0;
  for (int l = 0; l < d->pf_levels; l++)
    pf_px += (size_t)std::max(1, d->pf_w >> l) * (size_t)std::max(1, d->pf_h >> l);
  const struct {
    float *dst;
    size_t have, need;
    const DevArena *src;
  } parts[4] = {{irr, irr_bytes, (size_t)d->irr_w * d->irr_h * 16, &d->irr},
                {pf, pf_bytes, pf_px * 16, &d->pf},
                {brdf, brdf_bytes, (size_t)d->brdf_size * d->brdf_size * 16, &d->brdf},
                {env, env_bytes, (size_t)d->env_w * d->env_h * 16, &d->env}};
  for (const auto &p : parts) {
    if (!p.dst)
      continue;
    if (p.have < p.need || !p.src->p || p.need == 0)
      return fail(MOPCUDA_EINVAL, "ibl_read: %zu bytes given, %zu needed", p.have, p.need);
    CU_TRY(cudaMemcpy(p.dst, p.src->p, p.need, cudaMemcpyDeviceToHost));
  }
  return MOPCUDA_OK;
}
