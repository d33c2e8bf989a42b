/*
 * kernels.cu — sm_100a kernels of the CUDA frame path.
 *
 * Stage map (reference file:line of the CPU code each stage reproduces):
 *   k_vertex     per-vertex transform     cpu_prepare_triangle[_ex]
 *                                         cpu_backend.c:224-324, 412-526
 *   k_setup      cull / trivial accept /  mop_sw_rasterize_triangle_full
 *                screen map / edge setup  rasterizer.c:2458-2612, 1825-1924
 *   k_clip       Sutherland-Hodgman fan   rasterizer.c:514-626
 *   k_raster_*   coverage + depth into a  rasterizer.c:1926-1960 (the
 *                64-bit atomicMin key     incremental edge walk and the
 *                buffer (small records:   strict depth test; replaces the
 *                thread each; large:      single-threaded centroid binning
 *                (row, chunk) items)      of rasterizer_mt.c)
 *   k_resolve    background + compaction  rasterizer.c:2785-2792
 *   k_shade      deferred shading + ACES  rasterizer.c:1961-2108, 2776-2803
 *   k_post       FXAA + post + SSAA box   rasterizer.c:2625-2761,
 *                                         postprocess.c:24-116,
 *                                         viewport.c:3385-3411
 *   k_pick       batched pick             viewport.c:3687-3749
 *
 * Every float expression keeps the reference's operand order; the file is
 * compiled with -fmad=false so nothing is contracted into FMA.
 */
#include "mopcuda_internal.cuh"

/* Programmatic dependent launch.  The frame's kernels from the vertex pass
 * to the post pass are launched with programmatic stream serialisation: a
 * kernel may be scheduled while its predecessor drains, and its first
 * statement, pdl_wait(), holds every thread until the predecessor has
 * completed and its writes are visible (griddepcontrol.wait).  A kernel
 * launched without the attribute passes pdl_wait() at once, so the kernels
 * stay correct wherever they are launched from.  No kernel triggers early:
 * a successor starts once all of its predecessor's blocks have exited. */
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename Arg>
static void pdl(void (*k)(Arg), dim3 grid, dim3 block, cudaStream_t s, Arg arg) {
  cudaLaunchConfig_t c = {};
  c.gridDim = grid;
  c.blockDim = block;
  c.dynamicSmemBytes = 0;
  c.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  c.attrs = at;
  c.numAttrs = 1;
  cudaLaunchKernelEx(&c, k, arg);
}

#define PI_F 3.14159274f /* (float)M_PI */

/* (uint8_t) of a value already clamped to [0, 255.5] (or NaN): plain
 * truncation agrees with the x86 conversion there (NaN -> 0 on both after
 * taking the low byte of INT_MIN / 0). */
__device__ __forceinline__ uint8_t u8_of(float v) { return (uint8_t)__float2int_rz(v); }

/* ------------------------------------------------------------------------
 * small vector math (reference math.c:17-50, 196-203)
 * ------------------------------------------------------------------------ */
struct V3 {
  float x, y, z;
};

__device__ __forceinline__ V3 mk3(float x, float y, float z) {
  V3 r;
  r.x = x;
  r.y = y;
  r.z = z;
  return r;
}
__device__ __forceinline__ V3 add3(V3 a, V3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 scale3(V3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ V3 norm3(V3 a) {
  float l = len3(a);
  if (l < 1e-8f)
    return mk3(0.0f, 0.0f, 0.0f);
  float inv = 1.0f / l;
  return mk3(a.x * inv, a.y * inv, a.z * inv);
}
__device__ __forceinline__ float clamp01(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }

/* rows of a column-major matrix times (x, y, z, w), summed left to right */
__device__ __forceinline__ float4 xform(const float *m, float x, float y, float z, float w) {
  float4 r;
  r.x = m[0] * x + m[4] * y + m[8] * z + m[12] * w;
  r.y = m[1] * x + m[5] * y + m[9] * z + m[13] * w;
  r.z = m[2] * x + m[6] * y + m[10] * z + m[14] * w;
  r.w = m[3] * x + m[7] * y + m[11] * z + m[15] * w;
  return r;
}

__device__ __forceinline__ int find_draw_by(const DrawRec *draws, uint32_t n, uint32_t g,
                                            bool by_vertex) {
  uint32_t lo = 0, hi = n; /* last draw with base <= g */
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    uint32_t b = by_vertex ? draws[mid].vbase : draws[mid].tbase;
    if (b <= g)
      lo = mid;
    else
      hi = mid;
  }
  return (int)lo;
}

/* ------------------------------------------------------------------------
 * k_vertex — one thread per (draw, vertex)
 * ------------------------------------------------------------------------ */
__device__ __forceinline__ void read_attr(const uint8_t *v, int off, int n, float dflt_last,
                                          int want, float *out) {
  /* read_attrib_float{2,3,4}, cpu_backend.c:332-410: missing components are
   * zero, except a 4-component read's last one which defaults to 1. */
  for (int k = 0; k < want; k++)
    out[k] = 0.0f;
  if (want == 4)
    out[3] = dflt_last;
  if (off < 0 || n <= 0)
    return;
  const float *f = (const float *)(v + off);
  int m = n < want ? n : want;
  for (int k = 0; k < m; k++)
    out[k] = __ldg(f + k);
}

__device__ __forceinline__ void vertex_item(const FrameArgs &a, uint32_t g) {
  const DrawRec &d = a.draws[find_draw_by(a.draws, a.draw_count, g, true)];
  uint32_t i = g - d.vbase;
  float pos[3], nrm[3], col[4], uv[2];
  if (!(d.flags & DF_FLEX)) {
    const float *v = (const float *)(d.vbuf + (size_t)i * 48u);
    float4 q0 = __ldg((const float4 *)v);
    float4 q1 = __ldg((const float4 *)v + 1);
    float4 q2 = __ldg((const float4 *)v + 2);
    pos[0] = q0.x; pos[1] = q0.y; pos[2] = q0.z;
    nrm[0] = q0.w; nrm[1] = q1.x; nrm[2] = q1.y;
    col[0] = q1.z; col[1] = q1.w; col[2] = q2.x; col[3] = q2.y;
    uv[0] = q2.z; uv[1] = q2.w;
  } else {
    const uint8_t *v = d.vbuf + (size_t)i * d.stride;
    read_attr(v, d.off_pos, d.n_pos, 1.0f, 3, pos);
    if (d.off_nrm >= 0) {
      read_attr(v, d.off_nrm, d.n_nrm, 1.0f, 3, nrm);
    } else {
      nrm[0] = 0.0f; nrm[1] = 1.0f; nrm[2] = 0.0f;
    }
    if (d.off_col >= 0) {
      read_attr(v, d.off_col, d.n_col, 1.0f, 4, col);
    } else {
      col[0] = col[1] = col[2] = col[3] = 1.0f;
    }
    read_attr(v, d.off_uv, d.n_uv, 1.0f, 2, uv);
  }
  float4 c = xform(d.mvp, pos[0], pos[1], pos[2], 1.0f);
  if (d.depth_bias != 0.0f)
    c.z += d.depth_bias * c.w; /* cpu_backend.c:238-242 */
  float4 w = xform(d.model, pos[0], pos[1], pos[2], 1.0f);
  float4 n = xform(d.model, nrm[0], nrm[1], nrm[2], 0.0f);
  if (d.flags & DF_TEXTURED) { /* nearest texel at the vertex, :276-303 */
    float tu = uv[0] - floorf(uv[0]);
    float tv = uv[1] - floorf(uv[1]);
    int tx = x86_f2i(tu * (float)(d.tex_w - 1) + 0.5f);
    int ty = x86_f2i(tv * (float)(d.tex_h - 1) + 0.5f);
    tx = tx < 0 ? 0 : (tx >= d.tex_w ? d.tex_w - 1 : tx);
    ty = ty < 0 ? 0 : (ty >= d.tex_h ? d.tex_h - 1 : ty);
    uchar4 t = __ldg((const uchar4 *)d.tex + ((size_t)ty * (size_t)d.tex_w + (size_t)tx));
    col[0] *= (float)t.x / 255.0f;
    col[1] *= (float)t.y / 255.0f;
    col[2] *= (float)t.z / 255.0f;
    col[3] *= (float)t.w / 255.0f;
  }
  a.clip[g] = c;
  a.world[g] = make_float4(w.x, w.y, w.z, 0.0f);
  a.normal[g] = make_float4(n.x, n.y, n.z, 1.0f / c.w); /* .w: 1/w for perspective weights */
  a.color[g] = make_float4(col[0], col[1], col[2], col[3]);
}

__global__ void k_vertex(FrameArgs a) {
  pdl_wait();
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < a.total_vertices)
    vertex_item(a, g);
}

/* ------------------------------------------------------------------------
 * lighting (rasterizer.c:1497-1814) and IBL (161-301)
 * ------------------------------------------------------------------------ */
__device__ __forceinline__ float falloff_inv_sq(const LightRec &L, float dist) {
  if (L.range > 0.0f) {
    float r = dist / L.range;
    float at = 1.0f - r;
    if (at < 0.0f)
      at = 0.0f;
    return at * at;
  }
  float d2 = dist * dist;
  if (d2 < 0.01f)
    d2 = 0.01f;
  return 1.0f / d2;
}

__device__ __forceinline__ float spot_cone(const LightRec &L, V3 dir) {
  V3 sd = mk3(L.ndir[0], L.ndir[1], L.ndir[2]);
  float ca = -dot3(dir, sd);
  if (ca < L.spot_outer_cos)
    return 0.0f;
  if (ca < L.spot_inner_cos) {
    float rs = L.spot_inner_cos - L.spot_outer_cos;
    if (rs > 1e-6f) {
      float t = (ca - L.spot_outer_cos) / rs;
      return t * t * (3.0f - 2.0f * t);
    }
  }
  return 1.0f;
}

/* Shadow-map texel from its key: 0xffffffff is the cleared value 1.0,
 * otherwise the inverse of depth_key. */
__device__ __forceinline__ float shadow_texel(uint32_t k) {
  if (k == 0xffffffffu)
    return 1.0f;
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

/* shadow_test_pcf, rasterizer.c:303-348: the world position through the
 * light's view-projection, 3x3 texels around the truncated texel coordinate
 * (out-of-map texels count as lit), lit when ndc z <= texel + 0.005; the
 * result is lit / 9.  The texel coordinate converts as the x86 build does
 * (cvttss2si); the neighbour offsets are taken in 64 bits so INT_MIN +- 1
 * stays out of the map. */
__device__ __noinline__ float shadow_pcf_at(const uint32_t *__restrict__ keys,
                                           const float *__restrict__ vp, int sw, int sh,
                                           float px, float py, float pz) {
  const float4 lp = xform(vp, px, py, pz, 1.0f);
  if (lp.w <= 0.0f)
    return 1.0f;
  const float inv_w = 1.0f / lp.w;
  const float ndcx = lp.x * inv_w;
  const float ndcy = lp.y * inv_w;
  const float ndcz = (lp.z * inv_w + 1.0f) * 0.5f;
  const float u = (ndcx + 1.0f) * 0.5f * (float)sw;
  const float v = (1.0f - ndcy) * 0.5f * (float)sh;
  const long long cx = x86_f2i(u), cy = x86_f2i(v);
  int lit = 0;
  for (int dy = -1; dy <= 1; dy++) {
    for (int dx = -1; dx <= 1; dx++) {
      const long long sx = cx + dx, sy = cy + dy;
      if (sx < 0 || sx >= sw || sy < 0 || sy >= sh) {
        lit++;
        continue;
      }
      const float sz = shadow_texel(__ldg(keys + (size_t)sy * (size_t)sw + sx));
      if (ndcz <= sz + 0.005f)
        lit++;
    }
  }
  return (float)lit / 9.0f;
}

/* Kept out of line: frames without a shadow map never call it, and the
 * shading loops keep their registers. */
__device__ __forceinline__ float shadow_pcf(const FrameArgs &a, V3 wp) {
  if (!a.shadow_keys) /* a batch viewport whose scene has no map */
    return 1.0f;
  return shadow_pcf_at(a.shadow_keys, a.shadow_vp, a.shadow_w, a.shadow_h, wp.x, wp.y, wp.z);
}

/* compute_multi_light (flat path), rasterizer.c:1497-1588; directional
 * lights are shadowed when a shadow map is bound (:1580-1583). */
template <bool SH>
__device__ float diffuse_flat(const FrameArgs &a, V3 n, V3 wp, const LightRec *Ls, uint32_t cnt,
                              float amb) {
  float total = amb;
  for (uint32_t i = 0; i < cnt; i++) {
    const LightRec &L = Ls[i];
    if (!L.active)
      continue;
    float ndotl = 0.0f, att = 1.0f, spot = 1.0f;
    if (L.type == 0) {
      V3 dir = mk3(L.ndir[0], L.ndir[1], L.ndir[2]);
      ndotl = -dot3(n, dir);
    } else if (L.type == 1 || L.type == 2) {
      V3 tl = sub3(mk3(L.position[0], L.position[1], L.position[2]), wp);
      float dist = len3(tl);
      if (dist < 1e-6f)
        dist = 1e-6f;
      V3 dir = scale3(tl, 1.0f / dist);
      ndotl = dot3(n, dir);
      if (L.type == 1) {
        att = falloff_inv_sq(L, dist);
      } else {
        spot = spot_cone(L, dir);
        if (L.range > 0.0f) {
          float r = dist / L.range;
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
    const float shadow = (SH && L.type == 0) ? shadow_pcf(a, wp) : 1.0f;
    total += ndotl * L.intensity * att * spot * shadow;
  }
  return clamp01(total);
}

/* compute_multi_light_rgb (rasterizer.c:1596-1688) and
 * compute_multi_specular_ggx (1701-1814) evaluated in one pass over the
 * lights.  For point and spot lights both reference helpers compute the same
 * to-light vector, distance, direction, N.L and inverse-square / range
 * falloff from the same operands in the same order, so those values are
 * computed once here; each helper's own accumulation order is unchanged. */
template <bool SH>
__device__ void lights_smooth(const FrameArgs &a, V3 n, V3 wp, V3 vdir, const LightRec *Ls,
                              const DrawRec &d, const float base[3], float lit[3],
                              float spec[3]) {
  lit[0] = lit[1] = lit[2] = d.ambient;
  spec[0] = spec[1] = spec[2] = 0.0f;
  const float alpha2 = d.alpha2, k = d.smith_k, omk = d.one_minus_k;
  float ndotv = dot3(n, vdir);
  if (ndotv < 1e-4f)
    ndotv = 1e-4f;
  float f0[3];
  for (int c = 0; c < 3; c++)
    f0[c] = d.f0_dielectric + base[c] * d.metallic;
  const float g1v = ndotv / (ndotv * omk + k);
  const uint32_t cnt = d.light_count;
  for (uint32_t i = 0; i < cnt; i++) {
    const LightRec &L = Ls[i];
    if (!L.active)
      continue;
    float ndl_d = 0.0f, ndl_s, att = 1.0f, spot = 1.0f;
    V3 ldir;
    if (L.type == 0) {
      const V3 nd = mk3(L.ndir[0], L.ndir[1], L.ndir[2]);
      ndl_d = -dot3(n, nd);
      ldir = mk3(-nd.x, -nd.y, -nd.z);
      ndl_s = dot3(n, ldir);
    } else if (L.type == 1 || L.type == 2) {
      const V3 tl = sub3(mk3(L.position[0], L.position[1], L.position[2]), wp);
      float dist = len3(tl);
      if (dist < 1e-6f)
        dist = 1e-6f;
      ldir = scale3(tl, 1.0f / dist);
      ndl_d = dot3(n, ldir);
      ndl_s = ndl_d;
      if (L.type == 2)
        spot = spot_cone(L, ldir);
      att = falloff_inv_sq(L, dist);
    } else {
      ldir = mk3(0.0f, 0.0f, 0.0f);
      ndl_s = dot3(n, ldir);
    }
    /* both helpers shadow directional lights from the same world position
     * when a shadow map is bound (rasterizer.c:1677-1680, 1802-1805) */
    const float shadow = (SH && L.type == 0) ? shadow_pcf(a, wp) : 1.0f;
    /* diffuse (rasterizer.c:1673-1687) */
    float ndotl = ndl_d < 0.0f ? 0.0f : ndl_d;
    const float contrib = ndotl * L.intensity * att * spot * shadow;
    lit[0] += contrib * L.color[0];
    lit[1] += contrib * L.color[1];
    lit[2] += contrib * L.color[2];
    /* specular (rasterizer.c:1763-1813): spot lights carry no cone factor */
    if (ndl_s <= 0.0f)
      continue;
    const V3 h = norm3(add3(ldir, vdir));
    float ndoth = dot3(n, h);
    if (ndoth < 0.0f)
      ndoth = 0.0f;
    float vdoth = dot3(vdir, h);
    if (vdoth < 0.0f)
      vdoth = 0.0f;
    const float ndoth2 = ndoth * ndoth;
    const float dd = ndoth2 * (alpha2 - 1.0f) + 1.0f;
    const float D = alpha2 / (PI_F * dd * dd);
    const float g1l = ndl_s / (ndl_s * omk + k);
    const float G = g1v * g1l;
    const float omv = 1.0f - vdoth;
    const float omv2 = omv * omv;
    const float omv5 = omv2 * omv2 * omv;
    float den = 4.0f * ndl_s * ndotv;
    if (den < 1e-6f)
      den = 1e-6f;
    const float st = D * G / den;
    const float wgt = st * L.intensity * att * ndl_s * shadow * PI_F;
    for (int c = 0; c < 3; c++) {
      const float fr = f0[c] + (1.0f - f0[c]) * omv5;
      spec[c] += wgt * fr * L.color[c];
    }
  }
}

__device__ __forceinline__ void ibl_bilinear(const float *d, int w, int h, float u, float v,
                                             float out[3]) {
  u = u - floorf(u);
  v = v - floorf(v);
  float fx = u * (float)(w - 1);
  float fy = v * (float)(h - 1);
  int x0 = (int)fx, y0 = (int)fy;
  x0 = x0 < 0 ? 0 : (x0 > w - 1 ? w - 1 : x0);
  y0 = y0 < 0 ? 0 : (y0 > h - 1 ? h - 1 : y0);
  int x1 = (x0 + 1) % w;
  int y1 = y0 + 1 < h ? y0 + 1 : h - 1;
  float sx = fx - (float)x0, sy = fy - (float)y0;
  const float4 p00 = __ldg((const float4 *)d + ((size_t)y0 * w + x0));
  const float4 p10 = __ldg((const float4 *)d + ((size_t)y0 * w + x1));
  const float4 p01 = __ldg((const float4 *)d + ((size_t)y1 * w + x0));
  const float4 p11 = __ldg((const float4 *)d + ((size_t)y1 * w + x1));
  float a00[3] = {p00.x, p00.y, p00.z}, a10[3] = {p10.x, p10.y, p10.z};
  float a01[3] = {p01.x, p01.y, p01.z}, a11[3] = {p11.x, p11.y, p11.z};
  for (int c = 0; c < 3; c++) {
    float top = a00[c] * (1.0f - sx) + a10[c] * sx;
    float bot = a01[c] * (1.0f - sx) + a11[c] * sx;
    out[c] = top * (1.0f - sy) + bot * sy;
  }
}

/* dir_to_uv, rasterizer.c:216-222.  atan2f/asinf are CUDA's; glibc's differ
 * in the last ulp for some inputs, which perturbs IBL colour by at most a
 * rounding step. */
__device__ __forceinline__ void dir_uv(float dx, float dy, float dz, float rot, float *u,
                                       float *v) {
  float phi = atan2f(dz, dx) + rot;
  float cdy = dy < -1.0f ? -1.0f : (dy > 1.0f ? 1.0f : dy);
  *u = phi / (2.0f * 3.14159265f) + 0.5f;
  *v = asinf(cdy) / 3.14159265f + 0.5f;
}

__device__ void ibl_irr(const FrameArgs &a, V3 n, float out[3]) {
  out[0] = out[1] = out[2] = 0.0f;
  float len = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
  if (len < 1e-6f)
    return;
  float u, v;
  dir_uv(n.x / len, n.y / len, n.z / len, a.ibl_rotation, &u, &v);
  ibl_bilinear(a.irr, a.irr_w, a.irr_h, u, v, out);
  for (int c = 0; c < 3; c++)
    out[c] *= a.ibl_intensity;
}

/* The mip level and its offset/size depend only on the draw's roughness;
 * the host computes them once per draw (rasterizer.c:243-265). */
__device__ void ibl_pf(const FrameArgs &a, const DrawRec &d, V3 r, float out[3]) {
  out[0] = out[1] = out[2] = 0.0f;
  float len = sqrtf(r.x * r.x + r.y * r.y + r.z * r.z);
  if (len < 1e-6f)
    return;
  float u, v;
  dir_uv(r.x / len, r.y / len, r.z / len, a.ibl_rotation, &u, &v);
  ibl_bilinear(a.pf + (size_t)d.pf_off * 4, d.pf_lw, d.pf_lh, u, v, out);
  for (int c = 0; c < 3; c++)
    out[c] *= a.ibl_intensity;
}

/* BRDF LUT at (N.V, roughness); the roughness row is per draw, computed on
 * the host (rasterizer.c:280-291). */
__device__ __forceinline__ void ibl_lut(const FrameArgs &a, const DrawRec &d, float ndv, float *sc,
                                        float *bi) {
  ndv = ndv < 0.0f ? 0.0f : (ndv > 1.0f ? 1.0f : ndv);
  int n = a.brdf_size;
  int x = (int)(ndv * (float)(n - 1) + 0.5f);
  int y = d.brdf_row;
  if (x >= n)
    x = n - 1;
  float4 t = __ldg((const float4 *)a.brdf + ((size_t)y * n + x));
  *sc = t.x;
  *bi = t.y;
}

/* Per-sample shading of the smooth multi-light path (rasterizer.c:1963-2099)
 * from the normalised perspective-correct weights pc[]. */
template <bool SH>
__device__ void shade_smooth(const FrameArgs &a, const DrawRec &d, const LightRec *Ls,
                             const uint32_t v[3], const float4 N[3], const float pc[3],
                             float out[3]) {
  float4 C[3], W[3];
  for (int k = 0; k < 3; k++) {
    C[k] = a.color[v[k]];
    W[k] = a.world[v[k]];
  }
  V3 n = mk3(pc[0] * N[0].x + pc[1] * N[1].x + pc[2] * N[2].x,
             pc[0] * N[0].y + pc[1] * N[1].y + pc[2] * N[2].y,
             pc[0] * N[0].z + pc[1] * N[1].z + pc[2] * N[2].z);
  n = norm3(n);
  float base[3];
  base[0] = pc[0] * C[0].x + pc[1] * C[1].x + pc[2] * C[2].x;
  base[1] = pc[0] * C[0].y + pc[1] * C[1].y + pc[2] * C[2].y;
  base[2] = pc[0] * C[0].z + pc[1] * C[1].z + pc[2] * C[2].z;
  V3 wp = mk3(pc[0] * W[0].x + pc[1] * W[1].x + pc[2] * W[2].x,
              pc[0] * W[0].y + pc[1] * W[1].y + pc[2] * W[2].y,
              pc[0] * W[0].z + pc[1] * W[1].z + pc[2] * W[2].z);
  V3 vdir = norm3(sub3(mk3(d.cam_eye[0], d.cam_eye[1], d.cam_eye[2]), wp));
  float lit[3], spec[3];
  lights_smooth<SH>(a, n, wp, vdir, Ls, d, base, lit, spec);
  const float ds = d.diffuse_scale;
  float env[3] = {0.0f, 0.0f, 0.0f}, irr[3] = {0.0f, 0.0f, 0.0f};
  bool has_irr = a.irr != nullptr;
  if (has_irr)
    ibl_irr(a, n, irr);
  {
    float vdn = dot3(vdir, n);
    V3 refl = mk3(2.0f * vdn * n.x - vdir.x, 2.0f * vdn * n.y - vdir.y, 2.0f * vdn * n.z - vdir.z);
    float ndv = dot3(n, vdir);
    if (ndv < 0.0f)
      ndv = 0.0f;
    float f0[3];
    for (int c = 0; c < 3; c++)
      f0[c] = d.f0_dielectric + base[c] * d.metallic;
    if (a.pf != nullptr && a.brdf != nullptr) {
      float pf[3], bs, bb;
      ibl_pf(a, d, refl, pf);
      ibl_lut(a, d, ndv, &bs, &bb);
      for (int c = 0; c < 3; c++)
        env[c] = pf[c] * (f0[c] * bs + bb);
    } else if (d.metallic > 0.01f) { /* hemisphere fallback, :2042-2072 */
      float sky_t = refl.y * 0.5f + 0.5f;
      if (sky_t < 0.0f)
        sky_t = 0.0f;
      if (sky_t > 1.0f)
        sky_t = 1.0f;
      const float sky[3] = {0.35f, 0.38f, 0.45f}, gnd[3] = {0.08f, 0.07f, 0.06f};
      float he[3];
      for (int c = 0; c < 3; c++)
        he[c] = gnd[c] + sky_t * (sky[c] - gnd[c]);
      float mix = d.roughness * d.roughness;
      float avg = (he[0] + he[1] + he[2]) * (1.0f / 3.0f);
      for (int c = 0; c < 3; c++)
        he[c] += mix * (avg - he[c]);
      float om = 1.0f - ndv;
      float om2 = om * om;
      float om5 = om2 * om2 * om;
      for (int c = 0; c < 3; c++) {
        float fe = f0[c] + (1.0f - f0[c]) * om5;
        env[c] = he[c] * fe * d.ambient * 3.0f;
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
 * triangle setup
 * ------------------------------------------------------------------------ */

/* Clip-space vertex with the attributes the flat colour needs. */
struct CV {
  float4 p;
  V3 n, wp;
  float c[4];
};

__device__ __forceinline__ CV load_cv(const FrameArgs &a, uint32_t g) {
  CV r;
  r.p = a.clip[g];
  float4 n = a.normal[g], w = a.world[g], c = a.color[g];
  r.n = mk3(n.x, n.y, n.z);
  r.wp = mk3(w.x, w.y, w.z);
  r.c[0] = c.x;
  r.c[1] = c.y;
  r.c[2] = c.z;
  r.c[3] = c.w;
  return r;
}

/* Edge setup shared by the rasterisers (e.g. rasterizer.c:1842-1924).
 * Returns false when the reference returns before its pixel loop. */
__device__ bool edge_setup(const float sx[3], const float sy[3], int W, int H, RasterRec &r) {
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
  int x0 = x86_f2i(floorf(fmin_x)), y0 = x86_f2i(floorf(fmin_y));
  int x1 = x86_f2i(ceilf(fmax_x)), y1 = x86_f2i(ceilf(fmax_y));
  if (x0 < 0)
    x0 = 0;
  if (y0 < 0)
    y0 = 0;
  if (x1 >= W)
    x1 = W - 1;
  if (y1 >= H)
    y1 = H - 1;
  if (x0 > x1 || y0 > y1)
    return false;
  float area = (sx[1] - sx[0]) * (sy[2] - sy[0]) - (sx[2] - sx[0]) * (sy[1] - sy[0]);
  if (fabsf(area) < 1e-6f)
    return false;
  bool flip = area < 0.0f;
  r.inv_area = 1.0f / fabsf(area);
  for (int k = 0; k < 3; k++) {
    int p = (k + 1) % 3, q = (k + 2) % 3;
    float ex = sy[p] - sy[q], ey = sx[q] - sx[p];
    r.dx[k] = flip ? -ex : ex;
    r.dy[k] = flip ? -ey : ey;
  }
  float px = (float)x0 + 0.5f, py = (float)y0 + 0.5f;
  for (int k = 0; k < 3; k++) {
    int p = (k + 1) % 3, q = (k + 2) % 3;
    float w = (sx[q] - sx[p]) * (py - sy[p]) - (sy[q] - sy[p]) * (px - sx[p]);
    r.w0[k] = flip ? -w : w;
  }
  r.x0 = (uint16_t)x0;
  r.y0 = (uint16_t)y0;
  r.x1 = (uint16_t)x1;
  r.y1 = (uint16_t)y1;
  return true;
}

__device__ __forceinline__ void mark_dead(RasterRec &r) {
  r.x0 = 1;
  r.x1 = 0;
  r.y0 = 1;
  r.y1 = 0;
}

/* Screen mapping, cull and edge setup of one fan triangle (the body of the
 * fan loop, rasterizer.c:2532-2609).  Fills `rr`/`sr`; returns false if the
 * reference would draw nothing for it. */
template <bool SH>
__device__ bool fan_setup(const FrameArgs &a, const DrawRec &d, const CV v[3], const uint32_t slot[3],
                          uint32_t order, RasterRec &rr, ShadeRec &sr) {
  if (fabsf(v[0].p.w) < 1e-7f || fabsf(v[1].p.w) < 1e-7f || fabsf(v[2].p.w) < 1e-7f)
    return false;
  float hw = (float)a.width * 0.5f, hh = (float)a.height * 0.5f;
  float sx[3], sy[3], sz[3];
  for (int k = 0; k < 3; k++) {
    float iw = 1.0f / v[k].p.w;
    sx[k] = (v[k].p.x * iw + 1.0f) * hw;
    sy[k] = (1.0f - v[k].p.y * iw) * hh;
    sz[k] = (v[k].p.z * iw + 1.0f) * 0.5f;
  }
  float sarea = (sx[1] - sx[0]) * (sy[2] - sy[0]) - (sx[2] - sx[0]) * (sy[1] - sy[0]);
  if ((d.flags & DF_CULL) && sarea >= 0.0f)
    return false;
  const bool wire = (d.flags & DF_WIRE) != 0;
  if (wire) { /* the edges are drawn whatever the area (rasterizer.c:1225-1235) */
    for (int k = 0; k < 3; k++) {
      rr.w0[k] = sx[k];
      rr.dx[k] = sy[k];
      rr.dy[k] = sz[k];
    }
    rr.x0 = rr.y0 = rr.y1 = 0;
    rr.x1 = (uint16_t)REC_WIRE_X1;
  } else if (!edge_setup(sx, sy, a.width, a.height, rr)) {
    return false;
  }
  rr.order = order;
  sr.draw = (uint32_t)(&d - a.draws);
  if ((d.flags & DF_SMOOTH) && !wire) {
    rr.zc[0] = sz[0];
    rr.zc[1] = sz[1];
    rr.zc[2] = sz[2];
    sr.v[0] = slot[0];
    sr.v[1] = slot[1];
    sr.v[2] = slot[2];
    return true;
  }
  /* flat: constant colour and incremental depth (rasterizer.c:2549-2609,
   * 1164-1232, 971-974); a wireframe triangle takes the same colour */
  if (!wire) {
    rr.y1 |= REC_FLAT_BIT;
    rr.zc[0] = (rr.w0[0] * sz[0] + rr.w0[1] * sz[1] + rr.w0[2] * sz[2]) * rr.inv_area;
    rr.zc[1] = (rr.dx[0] * sz[0] + rr.dx[1] * sz[1] + rr.dx[2] * sz[2]) * rr.inv_area;
    rr.zc[2] = (rr.dy[0] * sz[0] + rr.dy[1] * sz[1] + rr.dy[2] * sz[2]) * rr.inv_area;
  }
  V3 fn = norm3(mk3(v[0].n.x + v[1].n.x + v[2].n.x, v[0].n.y + v[1].n.y + v[2].n.y,
                    v[0].n.z + v[1].n.z + v[2].n.z));
  float avg[3];
  for (int k = 0; k < 3; k++)
    avg[k] = (v[0].c[k] + v[1].c[k] + v[2].c[k]) * (1.0f / 3.0f);
  float col[3];
  if (d.flags & DF_LIT) {
    V3 wp = mk3((v[0].wp.x + v[1].wp.x + v[2].wp.x) / 3.0f, (v[0].wp.y + v[1].wp.y + v[2].wp.y) / 3.0f,
                (v[0].wp.z + v[1].wp.z + v[2].wp.z) / 3.0f);
    float lighting = diffuse_flat<SH>(a, fn, wp, a.lights + d.light_off, d.light_count, d.ambient);
    float ds = 1.0f - d.metallic;
    float env_flat = d.ambient * d.metallic * 0.3f;
    for (int k = 0; k < 3; k++)
      col[k] = avg[k] * (lighting * ds + env_flat);
  } else {
    V3 nl = norm3(mk3(d.light_dir[0], d.light_dir[1], d.light_dir[2]));
    float ndotl = dot3(fn, nl);
    if (ndotl < 0.0f)
      ndotl = 0.0f;
    float lighting = clamp01(d.ambient + (1.0f - d.ambient) * ndotl);
    for (int k = 0; k < 3; k++)
      col[k] = avg[k] * lighting;
  }
  for (int k = 0; k < 3; k++)
    sr.col[k] = col[k] < 0.0f ? 0.0f : col[k];
  return true;
}

__device__ __forceinline__ bool outside_same_plane(float4 a, float4 b, float4 c) {
  return (a.x < -a.w && b.x < -b.w && c.x < -c.w) || (a.x > a.w && b.x > b.w && c.x > c.w) ||
         (a.y < -a.w && b.y < -b.w && c.y < -c.w) || (a.y > a.w && b.y > b.w && c.y > c.w) ||
         (a.z < -a.w && b.z < -b.w && c.z < -c.w) || (a.z > a.w && b.z > b.w && c.z > c.w);
}

__device__ __forceinline__ bool inside_all(float4 p) {
  return p.x >= -p.w && p.x <= p.w && p.y >= -p.w && p.y <= p.w && p.z >= -p.w && p.z <= p.w;
}

/* Warp-aggregated allocation of one slot from *counter: the converged lanes
 * with the same counter (a batch warp can hold items of several viewports,
 * each with its own counters) share a single atomicAdd and take
 * consecutive slots in lane order. */
__device__ __forceinline__ uint32_t warp_alloc1(uint32_t *counter) {
  const uint32_t mask = __activemask();
  const uint32_t peers = __match_any_sync(mask, (unsigned long long)(uintptr_t)counter);
  const uint32_t lane = threadIdx.x & 31u;
  const int leader = __ffs(peers) - 1;
  uint32_t base = 0;
  if ((int)lane == leader)
    base = atomicAdd(counter, (uint32_t)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}

__device__ __forceinline__ bool rec_live(const RasterRec &r, int W, int H) {
  int y1 = (int)(r.y1 & 0x7fffu);
  /* live records always lie inside the framebuffer; anything else is dead
   * or an unwritten slot of an overflowed frame (which the host re-runs) */
  return (int)r.x0 <= (int)r.x1 && (int)r.y0 <= y1 && (int)r.x1 < W && y1 < H;
}

/* Records of the ordered suffix (a blended draw and all after it) are
 * composited per sample in submission order instead. */
__device__ __forceinline__ bool rec_ordered(const FrameArgs &a, const RasterRec &r) {
  return a.hdr != nullptr && (r.order >> ORDER_FAN_BITS) >= a.t_split;
}

/* Records above the small-record limits (bbox side / area, tunable) are
 * rasterised item-parallel by k_raster_large. */
__device__ __forceinline__ bool rec_large(const FrameArgs &a, const RasterRec &r) {
  int w = (int)r.x1 - (int)r.x0 + 1, h = (int)(r.y1 & 0x7fffu) - (int)r.y0 + 1;
  return w > a.small_side || h > a.small_side || w * h > a.small_area;
}

__device__ __forceinline__ uint32_t rec_items(const RasterRec &r) {
  uint32_t w = (uint32_t)r.x1 - (uint32_t)r.x0 + 1u;
  uint32_t h = (uint32_t)(r.y1 & 0x7fffu) - (uint32_t)r.y0 + 1u;
  return h * ((w + RASTER_CHUNK - 1u) / RASTER_CHUNK);
}

/* Queue a large record for item-parallel rasterisation. */
/* Queues a large record: one 64-bit atomic takes its list slot (high word)
 * and the offset of its first item (low word) together, so the offsets come
 * out ascending with the slot and no scan pass is needed.  An item total
 * past 2^32 carries into the slot count: flagged (bit 9), the frame fails. */
__device__ __forceinline__ void push_large(const FrameArgs &a, uint32_t rid, const RasterRec &r) {
  const uint32_t n = rec_items(r);
  const unsigned long long old = atomicAdd(
      reinterpret_cast<unsigned long long *>(&a.ctr->large_items), (1ull << 32) | n);
  const uint32_t q = (uint32_t)(old >> 32), off = (uint32_t)old;
  if (off + n < off)
    atomicOr(&a.ctr->overflow, 512u);
  if (q < a.large_cap) {
    a.large_list[q] = rid;
    a.large_items[q] = off;
  } else {
    atomicOr(&a.ctr->overflow, 8u);
  }
}

/* Marks slot t dead (or as a redirect to clipped fan records) with one
 * 16-byte store of the record's tail (inv_area, order, bbox). */
__device__ __forceinline__ void write_rec_tail(RasterRec *slot, uint32_t order, uint16_t y0) {
  uint4 tail;
  tail.x = 0u;                        /* inv_area */
  tail.y = order;
  tail.z = 1u | ((uint32_t)y0 << 16); /* x0 = 1, y0 */
  tail.w = 0u;                        /* x1 = 0 < x0: never rasterised */
  reinterpret_cast<uint4 *>(slot)[3] = tail;
}

/* k_setup — one thread per triangle (mop_sw_rasterize_triangle_full
 * rasterizer.c:2458-2530 up to the fan loop).  Slot t of the record arrays
 * belongs to triangle t. */
template <bool SH>
__device__ __forceinline__ void setup_item(const FrameArgs &a, uint32_t t) {
  const DrawRec &d = a.draws[find_draw_by(a.draws, a.draw_count, t, false)];
  const uint32_t lt = t - d.tbase;
  const uint32_t i0 = __ldg(d.ibuf + 3u * lt), i1 = __ldg(d.ibuf + 3u * lt + 1u),
                 i2 = __ldg(d.ibuf + 3u * lt + 2u);
  int status = 0; /* 0 dead, 1 single fan triangle, 2 needs clipping */
  RasterRec rr;
  ShadeRec sr;
  if (!(i0 >= d.vertex_count || i1 >= d.vertex_count || i2 >= d.vertex_count)) {
    const uint32_t g[3] = {d.vbase + i0, d.vbase + i1, d.vbase + i2};
    const float4 A = a.clip[g[0]], B = a.clip[g[1]], C = a.clip[g[2]];
    if (!outside_same_plane(A, B, C)) {
      bool culled = false;
      if ((d.flags & DF_CULL) && A.w > 0.0f && B.w > 0.0f && C.w > 0.0f) {
        float ex = B.x * A.w - A.x * B.w;
        float ey = B.y * A.w - A.y * B.w;
        float fx = C.x * A.w - A.x * C.w;
        float fy = C.y * A.w - A.y * C.w;
        culled = (ex * fy - ey * fx <= 0.0f);
      }
      if (!culled) {
        if (A.w > 0.0f && B.w > 0.0f && C.w > 0.0f && inside_all(A) && inside_all(B) &&
            inside_all(C)) {
          CV v[3];
          if ((d.flags & (DF_SMOOTH | DF_WIRE)) == DF_SMOOTH) {
            /* smooth records reference the vertex streams */
            v[0].p = A;
            v[1].p = B;
            v[2].p = C;
          } else { /* flat needs normals, colours and positions for its colour */
            for (int k = 0; k < 3; k++)
              v[k] = load_cv(a, g[k]);
          }
          status = fan_setup<SH>(a, d, v, g, t << ORDER_FAN_BITS, rr, sr) ? 1 : 0;
        } else {
          status = 2;
        }
      }
    }
  }
  if (status == 1) {
    a.rrec[t] = rr;
    a.srec[t] = sr;
    if (rec_live(rr, a.width, a.height) && rec_large(a, rr))
      push_large(a, t, rr);
  } else if (status == 2) {
    write_rec_tail(&a.rrec[t], 0u, REC_REDIRECT); /* k_clip fills in the target */
    uint32_t q = warp_alloc1(&a.ctr->clip_count);
    if (q < a.clip_cap)
      a.clipq[q] = t;
    else
      atomicOr(&a.ctr->overflow, 4u);
  } else {
    write_rec_tail(&a.rrec[t], 0u, 0u);
  }
}

/* 5 blocks of 256 per SM (48 registers): the setup waits on vertex gathers
 * and more resident warps hide them. */
template <bool SH>
__global__ void __launch_bounds__(256, 5) k_setup(FrameArgs a) {
  pdl_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < a.total_tris)
    setup_item<SH>(a, t);
}

/* Sutherland-Hodgman (rasterizer.c:514-626) on the triangles queued by
 * k_setup; one thread per queued triangle. */
#define MAX_CLIP 24

__device__ __forceinline__ float lerpf(float x, float y, float t) { return x + t * (y - x); }

__device__ __forceinline__ CV cv_lerp(const CV &p, const CV &q, float t) {
  CV r;
  r.p.x = lerpf(p.p.x, q.p.x, t);
  r.p.y = lerpf(p.p.y, q.p.y, t);
  r.p.z = lerpf(p.p.z, q.p.z, t);
  r.p.w = lerpf(p.p.w, q.p.w, t);
  r.n = mk3(lerpf(p.n.x, q.n.x, t), lerpf(p.n.y, q.n.y, t), lerpf(p.n.z, q.n.z, t));
  r.wp = mk3(lerpf(p.wp.x, q.wp.x, t), lerpf(p.wp.y, q.wp.y, t), lerpf(p.wp.z, q.wp.z, t));
  for (int k = 0; k < 4; k++)
    r.c[k] = lerpf(p.c[k], q.c[k], t);
  return r;
}

__device__ __forceinline__ float plane_dist(int pl, float4 p) {
  /* the reference multiplies by every plane coefficient, zeros included */
  const float nx[6] = {1.0f, -1.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  const float ny[6] = {0.0f, 0.0f, 1.0f, -1.0f, 0.0f, 0.0f};
  const float nz[6] = {0.0f, 0.0f, 0.0f, 0.0f, 1.0f, -1.0f};
  return nx[pl] * p.x + ny[pl] * p.y + nz[pl] * p.z + 1.0f * p.w;
}

__device__ __forceinline__ uint32_t clip_items(const FrameArgs &a) {
  const uint32_t n_q = a.ctr->clip_count;
  return n_q > a.clip_cap ? a.clip_cap : n_q;
}

template <bool SH>
__device__ __forceinline__ void clip_item(const FrameArgs &a, uint32_t qi) {
  {
    uint32_t t = a.clipq[qi];
    const DrawRec &d = a.draws[find_draw_by(a.draws, a.draw_count, t, false)];
    uint32_t lt = t - d.tbase;
    CV buf0[MAX_CLIP], buf1[MAX_CLIP];
    for (int k = 0; k < 3; k++)
      buf0[k] = load_cv(a, d.vbase + __ldg(d.ibuf + 3u * lt + k));
    CV *src = buf0, *dst = buf1;
    int cnt = 3;
    for (int pl = 0; pl < 6 && cnt > 0; pl++) {
      /* a plane every vertex is inside of returns the polygon unchanged (same
       * vertices, same order): skip its copy */
      bool all_in = true;
      for (int i = 0; i < cnt; i++)
        all_in &= plane_dist(pl, src[i].p) >= 0.0f;
      if (all_in)
        continue;
      int m = 0;
      CV prev = src[cnt - 1];
      float dp = plane_dist(pl, prev.p);
      for (int i = 0; i < cnt; i++) {
        CV cur = src[i];
        float dc = plane_dist(pl, cur.p);
        if (dc >= 0.0f) {
          if (dp < 0.0f) {
            float tt = dp / (dp - dc);
            if (m < MAX_CLIP)
              dst[m++] = cv_lerp(prev, cur, tt);
          }
          if (m < MAX_CLIP)
            dst[m++] = cur;
        } else if (dp >= 0.0f) {
          float tt = dp / (dp - dc);
          if (m < MAX_CLIP)
            dst[m++] = cv_lerp(prev, cur, tt);
        }
        prev = cur;
        dp = dc;
      }
      cnt = m;
      CV *tmp = src;
      src = dst;
      dst = tmp;
    }
    if (cnt < 3)
      return; /* slot t stays a redirect that no fragment references */
    /* store the polygon's vertices, then one record per fan triangle */
    uint32_t e = atomicAdd(&a.ctr->extra_vertices, (uint32_t)cnt);
    uint32_t nf = (uint32_t)cnt - 2u;
    uint32_t r = a.total_tris + atomicAdd(&a.ctr->rec_count, nf);
    if (a.total_vertices + e + (uint32_t)cnt > a.vertex_cap || r + nf > a.rec_cap) {
      atomicOr(&a.ctr->overflow, (a.total_vertices + e + (uint32_t)cnt > a.vertex_cap) ? 2u : 1u);
      return;
    }
    uint32_t vs = a.total_vertices + e;
    for (int k = 0; k < cnt; k++) {
      const CV &c = src[k];
      a.clip[vs + k] = c.p;
      a.normal[vs + k] = make_float4(c.n.x, c.n.y, c.n.z, 1.0f / c.p.w);
      a.world[vs + k] = make_float4(c.wp.x, c.wp.y, c.wp.z, 0.0f);
      a.color[vs + k] = make_float4(c.c[0], c.c[1], c.c[2], c.c[3]);
    }
    for (int i = 1; i < cnt - 1; i++) {
      CV fv[3] = {src[0], src[i], src[i + 1]};
      uint32_t slot[3] = {vs, vs + (uint32_t)i, vs + (uint32_t)i + 1u};
      RasterRec rr;
      ShadeRec sr;
      if (!fan_setup<SH>(a, d, fv, slot, (t << ORDER_FAN_BITS) | (uint32_t)(i - 1), rr, sr)) {
        mark_dead(rr);
        rr.order = (t << ORDER_FAN_BITS) | (uint32_t)(i - 1);
        sr.draw = (uint32_t)(&d - a.draws);
      }
      a.rrec[r + i - 1] = rr;
      a.srec[r + i - 1] = sr;
      if (rec_live(rr, a.width, a.height) && rec_large(a, rr))
        push_large(a, r + (uint32_t)i - 1u, rr);
    }
    write_rec_tail(&a.rrec[t], r, REC_REDIRECT);
  }
}

template <bool SH>
__global__ void k_clip(FrameArgs a) {
  pdl_wait();
  const uint32_t n_q = clip_items(a);
  for (uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x; qi < n_q;
       qi += gridDim.x * blockDim.x)
    clip_item<SH>(a, qi);
}

/* ------------------------------------------------------------------------
 * visibility: every fragment of every live record does a 64-bit atomicMin
 * of (depth_key << 32 | submission order) into the per-sample key buffer.
 * The minimum is the fragment the reference keeps: nearest depth, and on an
 * exact tie the earliest submitted (strict `z < depth`, rasterizer.c:1960).
 * ------------------------------------------------------------------------ */
/* Walk samples [xs, xe] of row y of record r, starting from edge values
 * w0..w2 (and flat depth z) already folded to (y, xs). */
__device__ __forceinline__ void raster_span(const FrameArgs &a, const RasterRec &r, bool flat, int y,
                                            int xs, int xe, float w0, float w1, float w2, float z) {
  unsigned long long *row = a.keys + (size_t)y * (size_t)a.width;
  bool seen = false;
  for (int x = xs; x <= xe; x++) {
    if (w0 >= 0.0f && w1 >= 0.0f && w2 >= 0.0f) {
      seen = true;
      float zz = z;
      if (!flat) {
        float b0 = w0 * r.inv_area, b1 = w1 * r.inv_area, b2 = w2 * r.inv_area;
        zz = b0 * r.zc[0] + b1 * r.zc[1] + b2 * r.zc[2];
      }
      if (zz < 1.0f)
        atomicMin(row + x, ((unsigned long long)depth_key(zz) << 32) | (unsigned long long)r.order);
    } else if (seen) {
      break; /* edge values are monotone along a row: coverage has ended */
    }
    w0 = __fadd_rn(w0, r.dx[0]);
    w1 = __fadd_rn(w1, r.dx[1]);
    w2 = __fadd_rn(w2, r.dx[2]);
    if (flat)
      z = __fadd_rn(z, r.zc[1]);
  }
}

/* Small records: one thread walks the whole (<= 128-sample) bbox, row by
 * row, exactly as the reference's loops step (rasterizer.c:1926-2151). */
__device__ __forceinline__ uint32_t raster_small_items(const FrameArgs &a) {
  const uint32_t n = a.total_tris + a.ctr->rec_count;
  return n > a.rec_cap ? a.rec_cap : n;
}

__device__ __forceinline__ void raster_small_item(const FrameArgs &a, uint32_t rid) {
  {
    const RasterRec r = a.rrec[rid];
    if (!rec_live(r, a.width, a.height) || rec_large(a, r) || rec_ordered(a, r))
      return;
    const bool flat = (r.y1 & REC_FLAT_BIT) != 0;
    const int y1 = (int)(r.y1 & 0x7fffu);
    float wr0 = r.w0[0], wr1 = r.w0[1], wr2 = r.w0[2], zr = r.zc[0];
    for (int y = (int)r.y0; y <= y1; y++) {
      raster_span(a, r, flat, y, (int)r.x0, (int)r.x1, wr0, wr1, wr2, zr);
      wr0 = __fadd_rn(wr0, r.dy[0]);
      wr1 = __fadd_rn(wr1, r.dy[1]);
      wr2 = __fadd_rn(wr2, r.dy[2]);
      if (flat)
        zr = __fadd_rn(zr, r.zc[2]);
    }
  }
}

__global__ void k_raster_small(FrameArgs a) {
  pdl_wait();
  const uint32_t n = raster_small_items(a);
  for (uint32_t rid = blockIdx.x * blockDim.x + threadIdx.x; rid < n;
       rid += gridDim.x * blockDim.x)
    raster_small_item(a, rid);
}

/* Exclusive scan of a record list's item counts (the ordered, wireframe and
 * shadow lists) by one block of 1024:
 * tiles of 4096 counts (4 consecutive per thread), warp-shuffle scans, the
 * next tile's counts loaded before the current one is scanned; part holds
 * >= 32 words. */
#define LARGE_SCAN_PER 4
template <typename T>
__device__ __forceinline__ void items_scan_block(T *items, uint32_t n, T *total_out, T *part) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t tile = 1024u * LARGE_SCAN_PER;
  T nxt[LARGE_SCAN_PER];
#pragma unroll
  for (int k = 0; k < LARGE_SCAN_PER; k++) {
    const uint32_t i = tid * LARGE_SCAN_PER + (uint32_t)k;
    nxt[k] = i < n ? items[i] : (T)0;
  }
  T carry = 0;
  for (uint32_t base = 0; base < n; base += tile) {
    T v[LARGE_SCAN_PER];
    T sum = 0;
#pragma unroll
    for (int k = 0; k < LARGE_SCAN_PER; k++) {
      v[k] = nxt[k];
      sum += v[k];
      const uint32_t j = base + tile + tid * LARGE_SCAN_PER + (uint32_t)k;
      nxt[k] = j < n ? items[j] : (T)0;
    }
    T x = sum; /* inclusive scan of the per-thread sums within the warp */
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o)
        x += y;
    }
    if (lane == 31u)
      part[warp] = x;
    __syncthreads();
    if (warp == 0) {
      T w = part[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= (uint32_t)o)
          w += y;
      }
      part[lane] = w;
    }
    __syncthreads();
    T run = carry + (warp ? part[warp - 1] : (T)0) + x - sum;
    const T total = part[31];
#pragma unroll
    for (int k = 0; k < LARGE_SCAN_PER; k++) {
      const uint32_t i = base + tid * LARGE_SCAN_PER + (uint32_t)k;
      if (i < n)
        items[i] = run;
      run += v[k];
    }
    carry += total;
    __syncthreads(); /* part is reused by the next tile */
  }
  if (tid == 0)
    *total_out = carry;
}

/* Large records: one thread per (row, RASTER_CHUNK-sample chunk); the edge
 * values at the chunk start come from the exact fold. */
__device__ __forceinline__ void raster_large_item(const FrameArgs &a, uint32_t it) {
  uint32_t nl = a.ctr->large_count;
  if (nl > a.large_cap)
    nl = a.large_cap;
  {
    uint32_t lo = 0, hi = nl; /* last record with offset <= it */
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) >> 1;
      if (a.large_items[mid] <= it)
        lo = mid;
      else
        hi = mid;
    }
    const uint32_t rid = a.large_list[lo];
    if (rid >= a.rec_cap)
      return;
    const RasterRec r = a.rrec[rid];
    if (!rec_live(r, a.width, a.height) || rec_ordered(a, r))
      return;
    const bool flat = (r.y1 & REC_FLAT_BIT) != 0;
    const uint32_t w = (uint32_t)r.x1 - (uint32_t)r.x0 + 1u;
    const uint32_t chunks = (w + RASTER_CHUNK - 1u) / RASTER_CHUNK;
    const uint32_t local = it - a.large_items[lo];
    const int jr = (int)(local / chunks), kc = (int)((local % chunks) * RASTER_CHUNK);
    const int y = (int)r.y0 + jr;
    if (y > (int)(r.y1 & 0x7fffu))
      return;
    const int xs = (int)r.x0 + kc, xe = min((int)r.x1, xs + RASTER_CHUNK - 1);
    float w0 = fold_add(fold_add(r.w0[0], r.dy[0], jr), r.dx[0], kc);
    float w1 = fold_add(fold_add(r.w0[1], r.dy[1], jr), r.dx[1], kc);
    float w2 = fold_add(fold_add(r.w0[2], r.dy[2], jr), r.dx[2], kc);
    float z = flat ? fold_add(fold_add(r.zc[0], r.zc[2], jr), r.zc[1], kc) : 0.0f;
    raster_span(a, r, flat, y, xs, xe, w0, w1, w2, z);
  }
}

__global__ void k_raster_large(FrameArgs a) {
  pdl_wait();
  const uint32_t total = a.ctr->large_items;
  for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < total;
       it += gridDim.x * blockDim.x)
    raster_large_item(a, it);
}

/* ------------------------------------------------------------------------
 * resolve and shading
 * ------------------------------------------------------------------------ */
__device__ __forceinline__ float aces(float x) { /* rasterizer.c:2770-2774 */
  float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
  float m = (x * (a * x + b)) / (x * (c * x + d) + e);
  return m < 0.0f ? 0.0f : (m > 1.0f ? 1.0f : m);
}

/* The environment background's HDR colour at sample (x, y)
 * (pass_background_hdri_cpu, viewport.c:2145-2175): the ray through the
 * sample centre, normalised with divisions, to equirectangular (u, v) with
 * atan2f / asinf (CUDA's; glibc's differ in the last ulp for some inputs, as
 * in the IBL lookups), a bilinear sample (env_sample_bilinear, :2099-2124)
 * times the intensity. */
__device__ __forceinline__ void sky_hdr(const FrameArgs &a, int x, int y, float out[3]) {
  const float ndc_y = 1.0f - 2.0f * ((float)y + 0.5f) / (float)a.height;
  const float ndc_x = 2.0f * ((float)x + 0.5f) / (float)a.width - 1.0f;
  float d[3];
  for (int c = 0; c < 3; c++)
    d[c] = a.sky_fwd[c] + a.sky_right[c] * ndc_x * a.sky_half_w + a.sky_up[c] * ndc_y * a.sky_half_h;
  const float len = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  d[0] /= len;
  d[1] /= len;
  d[2] /= len;
  const float pi = 3.14159265358979f;
  const float phi = atan2f(d[2], d[0]) - a.sky_rotation;
  const float cdy = d[1] < -1.0f ? -1.0f : (d[1] > 1.0f ? 1.0f : d[1]);
  const float theta = asinf(cdy);
  float u = phi / (2.0f * pi) + 0.5f, v = theta / pi + 0.5f;
  u = u - floorf(u);
  v = v - floorf(v);
  const int w = a.sky_w, h = a.sky_h;
  const float fx = u * (float)(w - 1), fy = v * (float)(h - 1);
  int x0 = (int)fx, y0 = (int)fy;
  x0 = x0 < 0 ? 0 : (x0 > w - 1 ? w - 1 : x0); /* u, v in [0, 1): already inside */
  y0 = y0 < 0 ? 0 : (y0 > h - 1 ? h - 1 : y0);
  const int x1 = (x0 + 1) % w, y1 = y0 + 1 < h ? y0 + 1 : h - 1;
  const float sx = fx - (float)x0, sy = fy - (float)y0;
  const float4 p00 = __ldg(a.sky + (size_t)y0 * w + x0), p10 = __ldg(a.sky + (size_t)y0 * w + x1);
  const float4 p01 = __ldg(a.sky + (size_t)y1 * w + x0), p11 = __ldg(a.sky + (size_t)y1 * w + x1);
  const float q00[3] = {p00.x, p00.y, p00.z}, q10[3] = {p10.x, p10.y, p10.z};
  const float q01[3] = {p01.x, p01.y, p01.z}, q11[3] = {p11.x, p11.y, p11.z};
  for (int c = 0; c < 3; c++) {
    const float top = q00[c] * (1.0f - sx) + q10[c] * sx;
    const float bot = q01[c] * (1.0f - sx) + q11[c] * sx;
    out[c] = (top * (1.0f - sy) + bot * sy) * a.sky_intensity;
  }
}

/* The background sample's resolved colour (id 0: no ACES, rasterizer.c:2785-2792). */
__device__ __forceinline__ uchar4 sky_resolved(const FrameArgs &a, uint32_t i) {
  float h[3];
  sky_hdr(a, (int)(i % (uint32_t)a.width), (int)(i / (uint32_t)a.width), h);
  return make_uchar4(x86_f2u8(fminf(h[0], 1.0f) * 255.0f + 0.5f),
                     x86_f2u8(fminf(h[1], 1.0f) * 255.0f + 0.5f),
                     x86_f2u8(fminf(h[2], 1.0f) * 255.0f + 0.5f), 255);
}

/* Writes the background (clear colour resolved with id 0 and depth 1,
 * rasterizer.c:2785-2792) to every sample with 16-byte stores — k_shade
 * overwrites the covered ones — and queues covered samples for shading in
 * sample order (each thread owns 8 consecutive samples; one atomicAdd per
 * block iteration).  Blocks of 256 threads. */
#define RESOLVE_PER_THREAD 8

/* This thread's 8 keys of the chunk at blk (full chunks only; the ragged
 * tail is read sample by sample). */
__device__ __forceinline__ void resolve_load_keys(const FrameArgs &a, uint32_t blk,
                                                  ulonglong2 kk[RESOLVE_PER_THREAD / 2]) {
  const uint32_t S = (uint32_t)a.width * (uint32_t)a.height;
  const uint32_t i0 = blk + threadIdx.x * RESOLVE_PER_THREAD;
  if (i0 + RESOLVE_PER_THREAD <= S) {
    const ulonglong2 *kp = reinterpret_cast<const ulonglong2 *>(a.keys + i0);
#pragma unroll
    for (int k = 0; k < RESOLVE_PER_THREAD / 2; k++)
      kk[k] = kp[k];
  }
}

/* One block iteration of the resolve: samples [blk, blk + 256 * 8), with
 * this thread's keys already loaded (resolve_load_keys). */
__device__ __forceinline__ void resolve_chunk_keys(const FrameArgs &a, uint32_t blk,
                                                   const ulonglong2 kk[RESOLVE_PER_THREAD / 2],
                                                   uint32_t *s_warp, uint32_t *s_base_p) {
  uint32_t &s_base = *s_base_p;
  const uint32_t S = (uint32_t)a.width * (uint32_t)a.height;
  const uchar4 bg = make_uchar4(x86_f2u8(fminf(a.clear[0], 1.0f) * 255.0f + 0.5f),
                                x86_f2u8(fminf(a.clear[1], 1.0f) * 255.0f + 0.5f),
                                x86_f2u8(fminf(a.clear[2], 1.0f) * 255.0f + 0.5f), 255);
  const uint32_t bgw = (uint32_t)bg.x | ((uint32_t)bg.y << 8) | ((uint32_t)bg.z << 16) |
                       ((uint32_t)bg.w << 24);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  {
    const uint32_t i0 = blk + threadIdx.x * RESOLVE_PER_THREAD;
    uint32_t mask = 0;
    if (i0 + RESOLVE_PER_THREAD <= S) {
#pragma unroll
      for (int k = 0; k < RESOLVE_PER_THREAD / 2; k++) {
        const ulonglong2 v = kk[k];
        if (v.x != KEY_EMPTY)
          mask |= 1u << (2 * k);
        if (v.y != KEY_EMPTY)
          mask |= 1u << (2 * k + 1);
      }
      const uint4 c4 = make_uint4(bgw, bgw, bgw, bgw);
      const float4 d4 = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
      const uint4 z4 = make_uint4(0u, 0u, 0u, 0u);
      uint4 *pc = reinterpret_cast<uint4 *>(a.pre + i0);
      float4 *pd = reinterpret_cast<float4 *>(a.depth + i0);
      uint4 *pi = reinterpret_cast<uint4 *>(a.ids + i0);
      pc[0] = c4;
      pc[1] = c4;
      pd[0] = d4;
      pd[1] = d4;
      pi[0] = z4;
      pi[1] = z4;
    } else {
      for (int k = 0; k < RESOLVE_PER_THREAD; k++) {
        const uint32_t i = i0 + (uint32_t)k;
        if (i < S) {
          if (a.keys[i] != KEY_EMPTY)
            mask |= 1u << k;
          a.pre[i] = bg;
          a.depth[i] = 1.0f;
          a.ids[i] = 0u;
        }
      }
    }
    if (a.sky) /* the environment background replaces the clear colour */
      for (int k = 0; k < RESOLVE_PER_THREAD; k++) {
        const uint32_t i = i0 + (uint32_t)k;
        if (i < S && !((mask >> k) & 1u))
          a.pre[i] = sky_resolved(a, i);
      }
    const uint32_t c = (uint32_t)__popc(mask);
    uint32_t incl = c;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o)
        incl += v;
    }
    if (lane == 31)
      s_warp[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t run = 0;
      for (int w = 0; w < 8; w++) {
        uint32_t x = s_warp[w];
        s_warp[w] = run;
        run += x;
      }
      s_base = run ? atomicAdd(&a.ctr->shade_count, run) : 0u;
    }
    __syncthreads();
    uint32_t pos = s_base + s_warp[warp] + incl - c;
    for (int k = 0; k < RESOLVE_PER_THREAD; k++)
      if ((mask >> k) & 1u)
        a.shade_list[pos++] = i0 + (uint32_t)k;
    __syncthreads();
  }
}

__device__ __forceinline__ void resolve_chunk(const FrameArgs &a, uint32_t blk, uint32_t *s_warp,
                                              uint32_t *s_base_p) {
  ulonglong2 kk[RESOLVE_PER_THREAD / 2];
  resolve_load_keys(a, blk, kk);
  resolve_chunk_keys(a, blk, kk, s_warp, s_base_p);
}

/* The next chunk's keys are loaded before this chunk's barriers and
 * compaction atomic, so they are in flight while the block waits. */
__global__ void __launch_bounds__(256) k_resolve(FrameArgs a) {
  pdl_wait();
  __shared__ uint32_t s_warp[8];
  __shared__ uint32_t s_base;
  const uint32_t S = (uint32_t)a.width * (uint32_t)a.height;
  const uint32_t per_iter = 256u * RESOLVE_PER_THREAD, stride = gridDim.x * per_iter;
  ulonglong2 nk[RESOLVE_PER_THREAD / 2];
  uint32_t blk = blockIdx.x * per_iter;
  if (blk < S)
    resolve_load_keys(a, blk, nk);
  for (; blk < S; blk += stride) {
    ulonglong2 ck[RESOLVE_PER_THREAD / 2];
#pragma unroll
    for (int k = 0; k < RESOLVE_PER_THREAD / 2; k++)
      ck[k] = nk[k];
    if (blk + stride < S)
      resolve_load_keys(a, blk + stride, nk);
    resolve_chunk_keys(a, blk, ck, s_warp, &s_base);
  }
}

/* The three edge values after k sequential additions of their increments
 * (fold_add for each edge).  Short folds (k <= FOLD_SERIAL_MAX) step the
 * first two edges as one paired add (__fadd2_rn: two IEEE round-to-nearest
 * single additions in one instruction) and the third alone, for as many
 * steps as the longest short fold among the warp's converged lanes, each
 * lane's steps past its own k predicated off; longer folds take the
 * binade-skipping path per edge. */
__device__ __forceinline__ void fold3(float w[3], const float d[3], int k) {
  if (k <= FOLD_SERIAL_MAX) {
    const int km = (int)__reduce_max_sync(__activemask(), (unsigned)k);
    float2 p = make_float2(w[0], w[1]);
    const float2 dp = make_float2(d[0], d[1]);
    float q = w[2];
#pragma unroll
    for (int i = 0; i < FOLD_SERIAL_MAX; i++) {
      if (i >= km)
        break;
      if (i < k) {
        p = __fadd2_rn(p, dp);
        q = __fadd_rn(q, d[2]);
      }
    }
    w[0] = p.x;
    w[1] = p.y;
    w[2] = q;
  } else {
    for (int e = 0; e < 3; e++)
      w[e] = fold_add_long(w[e], d[e], k);
  }
}

/* Edge values of record r at row jr, column kc of its bbox: the row fold
 * from the corner, then the column fold along the row, as the reference
 * steps them. */
__device__ __forceinline__ void fold_rec(const RasterRec &r, int jr, int kc, float w[3]) {
  w[0] = r.w0[0];
  w[1] = r.w0[1];
  w[2] = r.w0[2];
  fold3(w, r.dy, jr);
  fold3(w, r.dx, kc);
}

/* Deferred shading of one covered sample: the winning record's exact edge
 * values at the sample (fold from the bbox corner), barycentrics, depth,
 * perspective-correct weights, multi-light + IBL shading (smooth) or the
 * record's constant colour (flat), then the ACES resolve. */
#define SHADE_SMEM_LIGHTS 64

/* Stages the frame's light records in shared memory when they fit; returns
 * the array the shading reads. */
__device__ __forceinline__ const LightRec *stage_lights(const FrameArgs &a, LightRec *s_lights) {
  if (a.light_total > SHADE_SMEM_LIGHTS)
    return a.lights;
  const uint32_t words = a.light_total * (uint32_t)(sizeof(LightRec) / 4);
  const uint32_t *src = reinterpret_cast<const uint32_t *>(a.lights);
  uint32_t *dst = reinterpret_cast<uint32_t *>(s_lights);
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x)
    dst[i] = src[i];
  __syncthreads();
  return s_lights;
}

/* Shades covered sample shade_list[j] (lights: the frame's light array). */
template <bool SH>
__device__ __forceinline__ void shade_item(const FrameArgs &a, uint32_t j, const LightRec *lights) {
  {
    const uint32_t px = a.shade_list[j];
    const unsigned long long k = a.keys[px];
    const uint32_t t = (uint32_t)k >> ORDER_FAN_BITS;
    const uint32_t fan = (uint32_t)k & ((1u << ORDER_FAN_BITS) - 1u);
    uint32_t rid = 0xffffffffu;
    RasterRec r;
    if (t < a.total_tris) {
      r = a.rrec[t];
      if (r.y0 == REC_REDIRECT) {
        rid = r.order + fan;
        if (rid < a.rec_cap)
          r = a.rrec[rid];
        else
          rid = 0xffffffffu;
      } else if (fan == 0u) {
        rid = t;
      }
    }
    if (rid >= a.rec_cap) { /* overflowed frame: the host re-runs it */
      a.pre[px] = make_uchar4(0, 0, 0, 255);
      a.depth[px] = 1.0f;
      a.ids[px] = 0u;
      return;
    }
    const int x = (int)(px % (uint32_t)a.width), y = (int)(px / (uint32_t)a.width);
    const ShadeRec s = a.srec[rid];
    const DrawRec &d = a.draws[s.draw < a.draw_count ? s.draw : 0];
    const LightRec *Ls = lights + d.light_off;
    const int jr = y - (int)r.y0, kc = x - (int)r.x0;
    float hdr[3], depth;
    if (r.y1 & REC_FLAT_BIT) {
      depth = fold_add(fold_add(r.zc[0], r.zc[2], jr), r.zc[1], kc);
      hdr[0] = s.col[0];
      hdr[1] = s.col[1];
      hdr[2] = s.col[2];
    } else {
      float w[3];
      fold_rec(r, jr, kc, w);
      float b0 = w[0] * r.inv_area, b1 = w[1] * r.inv_area, b2 = w[2] * r.inv_area;
      depth = b0 * r.zc[0] + b1 * r.zc[1] + b2 * r.zc[2];
      if (a.no_color || s.v[0] >= a.vertex_cap || s.v[1] >= a.vertex_cap ||
          s.v[2] >= a.vertex_cap) {
        hdr[0] = hdr[1] = hdr[2] = 0.0f; /* visibility-only view (bad vertex slots are
                                           unreachable for live records) */
      } else {
        const float4 N[3] = {a.normal[s.v[0]], a.normal[s.v[1]], a.normal[s.v[2]]};
        float pc[3] = {b0 * N[0].w, b1 * N[1].w, b2 * N[2].w}; /* .w = 1/clip.w */
        float ip = 1.0f / (pc[0] + pc[1] + pc[2]);
        pc[0] *= ip;
        pc[1] *= ip;
        pc[2] *= ip;
        shade_smooth<SH>(a, d, Ls, s.v, N, pc, hdr);
      }
    }
    a.pre[px] = make_uchar4(u8_of(aces(hdr[0] * a.exposure) * 255.0f + 0.5f),
                            u8_of(aces(hdr[1] * a.exposure) * 255.0f + 0.5f),
                            u8_of(aces(hdr[2] * a.exposure) * 255.0f + 0.5f), 255);
    a.depth[px] = depth;
    a.ids[px] = d.object_id;
    if (a.hdr) /* the blended suffix composites over this colour */
      a.hdr[px] = make_float4(hdr[0], hdr[1], hdr[2], 1.0f);
  }
}

/* 4 blocks of 256 per SM (64 registers): the kernel is issue-bound and the
 * extra warps hide the dependent-latency stalls of the lighting chains. */
/* With keys_next set, the kernel also clears the next frame's key buffer
 * (keys alternate between two buffers): 16-byte stores g + m * step (g the
 * thread's index, step the grid's threads), two per shaded sample and the
 * rest after the last one, so the writes spread over a kernel whose time is
 * arithmetic, and no frame waits for a clear of its own. */
template <bool SH>
__global__ void __launch_bounds__(256, 4) k_shade(FrameArgs a) {
  pdl_wait();
  __shared__ LightRec s_lights[SHADE_SMEM_LIGHTS];
  const LightRec *lights = stage_lights(a, s_lights);
  const uint32_t n = a.ctr->shade_count;
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x, step = gridDim.x * blockDim.x;
  const size_t S = (size_t)a.width * (size_t)a.height;
  const uint32_t nk = a.keys_next ? (uint32_t)(S >> 1) : 0u;
  uint4 *kn = reinterpret_cast<uint4 *>(a.keys_next);
  const uint4 ones = make_uint4(~0u, ~0u, ~0u, ~0u);
  uint32_t j = g;
  for (; j < n; j += step) {
    const uint32_t c = 2u * j - g; /* = g + 2 * iteration * step */
    if (c < nk) {
      kn[c] = ones;
      if (c + step < nk)
        kn[c + step] = ones;
    }
    shade_item<SH>(a, j, lights);
  }
  for (uint32_t c = 2u * j - g; c < nk; c += step)
    kn[c] = ones;
  if (nk && (S & 1u) && g == 0u)
    a.keys_next[S - 1u] = ~0ull;
}

/* ------------------------------------------------------------------------
 * k_post — FXAA (rasterizer.c:2625-2761), tonemap/gamma/vignette
 * (postprocess.c:24-116) and the SSAA box (viewport.c:3385-3411).  A block
 * of 32x8 threads owns 32x8 presented pixels: it stages their samples plus
 * a one-sample halo (and each sample's luma) in shared memory with
 * coalesced loads, then each thread filters its ssaa x ssaa samples.
 * ------------------------------------------------------------------------ */
#define POST_BX 32
#define POST_BY 8

__device__ __forceinline__ float luma(uchar4 p) {
  return 0.299f * (float)p.x + 0.587f * (float)p.y + 0.114f * (float)p.z;
}

/* FXAA of tile sample (i, j) from its 3x3 neighbourhood in the tile. */
template <int TW>
__device__ __forceinline__ uchar4 fxaa_tile(const uchar4 (*tc)[TW], const float (*tl)[TW], int i,
                                            int j) {
  const uchar4 c = tc[i][j];
  const float lM = tl[i][j], lN = tl[i - 1][j], lS = tl[i + 1][j], lW = tl[i][j - 1],
              lE = tl[i][j + 1];
  float mn = lM, mx = lM;
  if (lN < mn) mn = lN;
  if (lS < mn) mn = lS;
  if (lW < mn) mn = lW;
  if (lE < mn) mn = lE;
  if (lN > mx) mx = lN;
  if (lS > mx) mx = lS;
  if (lW > mx) mx = lW;
  if (lE > mx) mx = lE;
  const float range = mx - mn;
  if (range < 0.0625f * mx + 0.004f)
    return c;
  const float lNW = tl[i - 1][j - 1], lNE = tl[i - 1][j + 1], lSW = tl[i + 1][j - 1],
              lSE = tl[i + 1][j + 1];
  const float avg =
      (lN + lS + lW + lE) * (2.0f / 12.0f) + (lNW + lNE + lSW + lSE) * (1.0f / 12.0f);
  float sub = fabsf(avg - lM);
  sub = sub / range;
  if (sub > 1.0f)
    sub = 1.0f;
  sub = sub * sub * (3.0f - 2.0f * sub);
  sub *= 0.75f;
  const float eh = fabsf(-2.0f * lW + lNW + lSW) + fabsf(-2.0f * lM + lN + lS) * 2.0f +
                   fabsf(-2.0f * lE + lNE + lSE);
  const float ev = fabsf(-2.0f * lN + lNW + lNE) + fabsf(-2.0f * lM + lW + lE) * 2.0f +
                   fabsf(-2.0f * lS + lSW + lSE);
  const bool horiz = eh >= ev;
  const float lp = horiz ? lS : lE, ln = horiz ? lN : lW;
  const float gp = fabsf(lp - lM), gn = fabsf(ln - lM);
  const bool pos = gp >= gn;
  const int ni = horiz ? (pos ? i + 1 : i - 1) : i;
  const int nj = horiz ? j : (pos ? j + 1 : j - 1);
  const uchar4 nb = tc[ni][nj];
  const float ib = 1.0f - sub;
  uchar4 o = c;
  o.x = u8_of((float)c.x * ib + (float)nb.x * sub);
  o.y = u8_of((float)c.y * ib + (float)nb.y * sub);
  o.z = u8_of((float)c.z * ib + (float)nb.z * sub);
  return o;
}

/* The sample tile of one block: rows -1 .. POST_BY*SF of the block's pixels'
 * samples and columns -OX .. POST_BX*SF+OX-1, so that each row is whole
 * 16-byte chunks of the image; NBUF colour tiles, the next one filling by
 * asynchronous copies while the current one is filtered. */
template <int SF> struct PostSmem {
  static constexpr int OX = 4; /* tile column of the block's first own sample */
  static constexpr int TW = POST_BX * SF + 2 * OX, TH = POST_BY * SF + 2;
  static constexpr int NBUF = SF <= 3 ? 2 : 1; /* within 48 KB of static shared memory */
  alignas(16) uchar4 c[NBUF][TH][TW];
  float l[TH][TW];
  float lut[256];
  uint8_t lut8[256];
  float thr[256]; /* gamma byte thresholds (FOG bit only); thr[255] = +inf */
};

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

/* Samples of the tile that lie off the image are neither copied nor read:
 * FXAA reads the neighbours of samples at least one away from every edge,
 * and every presented pixel's samples are on the image. */
__device__ __forceinline__ bool post_vec(const PostArgs &a) {
  return (a.width & 3) == 0 && ((uintptr_t)a.pre & 15u) == 0u;
}

/* Issues this thread's copies of tile (bx, by) into colour buffer c (one
 * commit group).  With 16-byte rows (post_vec) a copy moves 4 samples. */
template <int SF>
__device__ __forceinline__ void post_fetch(const PostArgs &a, bool vec,
                                           uchar4 (*c)[PostSmem<SF>::TW], int bx, int by) {
  constexpr int TW = PostSmem<SF>::TW, TH = PostSmem<SF>::TH, OX = PostSmem<SF>::OX;
  const int tid = threadIdx.y * POST_BX + threadIdx.x;
  const int w = a.width, h = a.height;
  const int sx0 = bx * POST_BX * SF - OX, sy0 = by * POST_BY * SF - 1;
  if (vec) {
    for (int i = tid; i < (TW / 4) * TH; i += POST_BX * POST_BY) {
      const int ty = i / (TW / 4), tx = 4 * (i % (TW / 4));
      const int sy = sy0 + ty, sx = sx0 + tx;
      if (sy >= 0 && sy < h && sx >= 0 && sx < w)
        cp_async16(&c[ty][tx], a.pre + (size_t)sy * w + sx);
    }
  } else {
    for (int i = tid; i < TW * TH; i += POST_BX * POST_BY) {
      const int ty = i / TW, tx = i % TW;
      const int sy = sy0 + ty, sx = sx0 + tx;
      if (sy >= 0 && sy < h && sx >= 0 && sx < w)
        cp_async4(&c[ty][tx], a.pre + (size_t)sy * w + sx);
    }
  }
  cp_async_commit();
}

/* The luma of the samples this thread copied (its own copies are visible
 * to it once waited for). */
template <int SF>
__device__ __forceinline__ void post_luma(const PostArgs &a, bool vec,
                                          const uchar4 (*c)[PostSmem<SF>::TW],
                                          float (*l)[PostSmem<SF>::TW], int bx, int by) {
  constexpr int TW = PostSmem<SF>::TW, TH = PostSmem<SF>::TH, OX = PostSmem<SF>::OX;
  const int tid = threadIdx.y * POST_BX + threadIdx.x;
  const int w = a.width, h = a.height;
  const int sx0 = bx * POST_BX * SF - OX, sy0 = by * POST_BY * SF - 1;
  if (vec) {
    for (int i = tid; i < (TW / 4) * TH; i += POST_BX * POST_BY) {
      const int ty = i / (TW / 4), tx = 4 * (i % (TW / 4));
      const int sy = sy0 + ty, sx = sx0 + tx;
      if (sy >= 0 && sy < h && sx >= 0 && sx < w) {
        const uint4 q = *reinterpret_cast<const uint4 *>(&c[ty][tx]);
        float4 o;
        o.x = luma(*reinterpret_cast<const uchar4 *>(&q.x));
        o.y = luma(*reinterpret_cast<const uchar4 *>(&q.y));
        o.z = luma(*reinterpret_cast<const uchar4 *>(&q.z));
        o.w = luma(*reinterpret_cast<const uchar4 *>(&q.w));
        *reinterpret_cast<float4 *>(&l[ty][tx]) = o;
      }
    }
  } else {
    for (int i = tid; i < TW * TH; i += POST_BX * POST_BY) {
      const int ty = i / TW, tx = i % TW;
      const int sy = sy0 + ty, sx = sx0 + tx;
      if (sy >= 0 && sy < h && sx >= 0 && sx < w)
        l[ty][tx] = luma(c[ty][tx]);
    }
  }
}

template <int SF>
__device__ __forceinline__ void post_load_luts(const PostArgs &a, PostSmem<SF> &sm) {
  const int tid = threadIdx.y * POST_BX + threadIdx.x;
  for (int i = tid; i < 256; i += POST_BX * POST_BY) {
    sm.lut[i] = a.lut[i];
    sm.lut8[i] = a.lut8[i];
    if (a.effects & 8u)
      sm.thr[i] = i < 255 ? a.gamma_thr[i] : __int_as_float(0x7f800000);
  }
}

/* The byte of channel value t after the sRGB step, clamp and rounding
 * (postprocess.c:73-78, 99-112): the number of thresholds at or below t,
 * found by a binary search of the 255 sorted thresholds (thr[255] = +inf
 * keeps every probe in range).  NaN compares below every threshold: 0, as
 * the reference's `c > 0 ? c : 0` gives. */
__device__ __forceinline__ uint8_t gamma_byte_of(const float *thr, float t) {
  int n = 0;
#pragma unroll
  for (int step = 128; step >= 1; step >>= 1)
    if (t >= thr[n + step - 1])
      n += step;
  return (uint8_t)n;
}

/* One sample of the post-process with the FOG bit (postprocess.c:43-112):
 * the byte colour to [0, 1], fog from the sample's depth value, Reinhard,
 * sRGB, vignette, clamp, rounding — the reference's float operations in its
 * order.  Without vignette the sRGB step and rounding are the exact threshold
 * search; with vignette the sRGB value itself is needed and powf is taken as
 * the double-precision pow rounded to float (glibc's powf, 0.82 ulp, differs
 * from it by one ulp for 0.06 % of inputs, which moves the byte only when the
 * product lands within that ulp of a rounding boundary). */
__device__ __forceinline__ uchar4 post_fog_sample(const PostArgs &a, const float *thr, uchar4 c,
                                                  float depth, float vg) {
  const uint32_t fx = a.effects;
  float factor = 0.0f;
  if (a.fog_range > 0.0f) {
    factor = (depth - a.fog_near) / a.fog_range;
    if (factor < 0.0f)
      factor = 0.0f;
    if (factor > 1.0f)
      factor = 1.0f;
  }
  const uint8_t in[3] = {c.x, c.y, c.z};
  uint8_t o[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    float v = (float)in[k] / 255.0f;
    v = v + (a.fog_color[k] - v) * factor;
    if (fx & 2u)
      v = v / (v + 1.0f);
    if ((fx & 1u) && !(fx & 4u)) {
      o[k] = gamma_byte_of(thr, v);
      continue;
    }
    if (fx & 1u) {
      const float x = v > 0.0f ? v : 0.0f;
      v = x <= 0.0031308f ? x * 12.92f
                          : 1.055f * (float)pow((double)x, (double)(1.0f / 2.4f)) - 0.055f;
    }
    if (fx & 4u)
      v *= vg;
    if (v > 1.0f)
      v = 1.0f;
    if (v < 0.0f)
      v = 0.0f;
    o[k] = u8_of(v * 255.0f + 0.5f);
  }
  return make_uchar4(o[0], o[1], o[2], c.w);
}

template <int SF, int TW>
__device__ __forceinline__ void post_pixel(const PostArgs &a, const uchar4 (*s_c)[TW],
                                           const float (*s_l)[TW], const float *s_lut,
                                           const uint8_t *s_lut8, const float *s_thr, int px,
                                           int py);

/* Filters tile (bx, by) from colour buffer `buf` once its copies have
 * landed: this thread's lumas, a barrier, then each thread's pixel (FXAA,
 * the tonemap/gamma map and the SSAA box).  Block-uniform; ends with a
 * barrier so the caller may refill the buffers. */
template <int SF>
__device__ __forceinline__ void post_filter(const PostArgs &a, bool vec, PostSmem<SF> &sm, int buf,
                                            int bx, int by) {
  constexpr int TW = PostSmem<SF>::TW;
  post_luma<SF>(a, vec, sm.c[buf], sm.l, bx, by);
  __syncthreads();
  const int pw = a.width / SF, ph = a.height / SF;
  const int px = bx * POST_BX + (int)threadIdx.x;
  const int py = by * POST_BY + (int)threadIdx.y;
  if (px < pw && py < ph)
    post_pixel<SF, TW>(a, sm.c[buf], sm.l, sm.lut, sm.lut8, sm.thr, px, py);
  __syncthreads();
}

/* One tile of POST_BX x POST_BY presented pixels (bx, by), copied and
 * filtered with nothing in flight around it. */
template <int SF>
__device__ __forceinline__ void post_tile(const PostArgs &a, PostSmem<SF> &sm, int bx, int by) {
  const bool vec = post_vec(a);
  post_fetch<SF>(a, vec, sm.c[0], bx, by);
  cp_async_wait<0>();
  post_filter<SF>(a, vec, sm, 0, bx, by);
}

template <int SF, int TW>
__device__ __forceinline__ void post_pixel(const PostArgs &a, const uchar4 (*s_c)[TW],
                                           const float (*s_l)[TW], const float *s_lut,
                                           const uint8_t *s_lut8, const float *s_thr, int px,
                                           int py) {
  const int w = a.width, h = a.height, pw = w / SF;
  const bool fx = (a.effects & 16u) && w >= 3 && h >= 3;
  uint32_t acc[4] = {0, 0, 0, 0};
#pragma unroll
  for (int dy = 0; dy < SF; dy++)
#pragma unroll
    for (int dx = 0; dx < SF; dx++) {
      const int x = px * SF + dx, y = py * SF + dy;
      const int ti = (int)threadIdx.y * SF + dy + 1,
                tj = (int)threadIdx.x * SF + dx + PostSmem<SF>::OX;
      uchar4 c = s_c[ti][tj];
      if (fx && x >= 1 && y >= 1 && x < w - 1 && y < h - 1)
        c = fxaa_tile<TW>(s_c, s_l, ti, tj);
      if (a.effects & 8u) {
        float vg = 1.0f;
        if (a.effects & 4u) {
          const float cx = (float)w * 0.5f, cy = (float)h * 0.5f;
          const float maxd = sqrtf(cx * cx + cy * cy);
          const float ddx = (float)x - cx, ddy = (float)y - cy;
          const float dist = sqrtf(ddx * ddx + ddy * ddy) / maxd;
          vg = 1.0f - dist * dist * 0.5f;
          if (vg < 0.0f)
            vg = 0.0f;
        }
        c = post_fog_sample(a, s_thr, c, a.depth[(size_t)y * w + x], vg);
      } else if (a.effects != 0u && !(a.effects & 4u)) {
        /* without vignette the post-process is a fixed byte map */
        c.x = s_lut8[c.x];
        c.y = s_lut8[c.y];
        c.z = s_lut8[c.z];
      } else if (a.effects != 0u) {
        float v[3] = {s_lut[c.x], s_lut[c.y], s_lut[c.z]};
        if (a.effects & 4u) {
          const float cx = (float)w * 0.5f, cy = (float)h * 0.5f;
          const float maxd = sqrtf(cx * cx + cy * cy);
          const float ddx = (float)x - cx, ddy = (float)y - cy;
          const float dist = sqrtf(ddx * ddx + ddy * ddy) / maxd;
          float vg = 1.0f - dist * dist * 0.5f;
          if (vg < 0.0f)
            vg = 0.0f;
          for (int k = 0; k < 3; k++)
            v[k] *= vg;
        }
        for (int k = 0; k < 3; k++) {
          if (v[k] > 1.0f)
            v[k] = 1.0f;
          if (v[k] < 0.0f)
            v[k] = 0.0f;
        }
        c.x = u8_of(v[0] * 255.0f + 0.5f);
        c.y = u8_of(v[1] * 255.0f + 0.5f);
        c.z = u8_of(v[2] * 255.0f + 0.5f);
      }
      a.out[(size_t)y * w + x] = c;
      acc[0] += c.x;
      acc[1] += c.y;
      acc[2] += c.z;
      acc[3] += c.w;
    }
  if (a.presented) {
    const uint32_t n = (uint32_t)(SF * SF);
    a.presented[(size_t)py * pw + px] =
        make_uchar4((uint8_t)(acc[0] / n), (uint8_t)(acc[1] / n), (uint8_t)(acc[2] / n),
                    (uint8_t)(acc[3] / n));
  }
}

/* Persistent: each block loads the tables once and takes tiles blockIdx.x,
 * blockIdx.x + gridDim.x, ... in row-major tile order; with two colour
 * buffers the copies of the next tile are in flight while the current one
 * is filtered. */
template <int SF>
__global__ void __launch_bounds__(POST_BX *POST_BY) k_post(PostArgs a) {
  pdl_wait();
  __shared__ PostSmem<SF> sm;
  post_load_luts<SF>(a, sm);
  const bool vec = post_vec(a);
  const uint32_t tx = ((uint32_t)(a.width / SF) + POST_BX - 1u) / POST_BX;
  const uint32_t ty = ((uint32_t)(a.height / SF) + POST_BY - 1u) / POST_BY;
  const uint32_t nt = tx * ty;
  if (PostSmem<SF>::NBUF == 1) {
    for (uint32_t t = blockIdx.x; t < nt; t += gridDim.x)
      post_tile<SF>(a, sm, (int)(t % tx), (int)(t / tx));
    return;
  }
  uint32_t t = blockIdx.x;
  if (t < nt)
    post_fetch<SF>(a, vec, sm.c[0], (int)(t % tx), (int)(t / tx));
  for (int buf = 0; t < nt; t += gridDim.x, buf ^= 1) {
    const uint32_t tn = t + gridDim.x;
    if (tn < nt) { /* the other buffer was released by the last filter's barrier */
      post_fetch<SF>(a, vec, sm.c[buf ^ (PostSmem<SF>::NBUF - 1)], (int)(tn % tx),
                     (int)(tn / tx));
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    post_filter<SF>(a, vec, sm, buf & (PostSmem<SF>::NBUF - 1), (int)(t % tx), (int)(t / tx));
  }
}

/* Blocks of k_post<SF> resident on one SM (queried once per factor). */
template <int SF> static int post_resident() {
  static int nb = 0;
  if (nb == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_post<SF>, POST_BX * POST_BY, 0) !=
            cudaSuccess ||
        nb < 1) {
      cudaGetLastError();
      nb = 1;
    }
  }
  return nb;
}

template __global__ void k_post<1>(PostArgs);
template __global__ void k_post<2>(PostArgs);
template __global__ void k_post<3>(PostArgs);
template __global__ void k_post<4>(PostArgs);

/* SSAA box of an already post-processed buffer (read_color path). */
__global__ void k_box(const uchar4 *src, int width, int height, int sf, uchar4 *dst) {
  const int pw = width / sf, ph = height / sf;
  int px = blockIdx.x * blockDim.x + threadIdx.x;
  int py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= pw || py >= ph)
    return;
  uint32_t acc[4] = {0, 0, 0, 0};
  for (int dy = 0; dy < sf; dy++)
    for (int dx = 0; dx < sf; dx++) {
      uchar4 c = src[(size_t)(py * sf + dy) * width + px * sf + dx];
      acc[0] += c.x;
      acc[1] += c.y;
      acc[2] += c.z;
      acc[3] += c.w;
    }
  uint32_t n = (uint32_t)(sf * sf);
  dst[(size_t)py * pw + px] = make_uchar4((uint8_t)(acc[0] / n), (uint8_t)(acc[1] / n),
                                          (uint8_t)(acc[2] / n), (uint8_t)(acc[3] / n));
}

/* ------------------------------------------------------------------------
 * k_pick — mop_viewport_pick at presentation pixels (viewport.c:3687-3749):
 * ID and depth of the top-left sample of the SSAA block.
 * ------------------------------------------------------------------------ */
__global__ void k_pick(const uint32_t *ids, const float *depth, int width, int height, int sf,
                       const int2 *xy, uint32_t n, uint32_t *out_id, float *out_depth,
                       int32_t *out_hit) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  int2 q = xy[i];
  uint32_t id = 0;
  float dp = 1.0f;
  int pw = width / sf, ph = height / sf;
  if (q.x >= 0 && q.x < pw && q.y >= 0 && q.y < ph) {
    size_t s = (size_t)(q.y * sf) * (size_t)width + (size_t)(q.x * sf);
    id = ids[s];
    if (id != 0)
      dp = depth[s];
  }
  out_id[i] = id;
  out_depth[i] = dp;
  out_hit[i] = id != 0 ? 1 : 0;
}

/* ------------------------------------------------------------------------
 * launchers (called from mopcuda_api.cu)
 * ------------------------------------------------------------------------ */
static inline unsigned blocks_for(uint32_t n, unsigned bs) { return (n + bs - 1u) / bs; }

__global__ void k_ocount(FrameArgs a);
__global__ void k_oscan(FrameArgs a);
__global__ void k_oraster(FrameArgs a);
template <bool SH, bool WIRE> __global__ void k_ofold(FrameArgs a);
__global__ void k_wcount(FrameArgs a);
__global__ void k_wscan(FrameArgs a);
__global__ void k_wplot(FrameArgs a);

/* The legacy smooth path's shading (mop_sw_rasterize_triangle_smooth,
 * rasterizer.c:1371-1420): interpolated normal and vertex colour, one
 * directional light (light_dir) with ambient, a view-independent Blinn-Phong
 * term of power 32 and weight 0.25, clamped at zero. */
__device__ void shade_legacy(const FrameArgs &a, const DrawRec &d, const uint32_t v[3],
                             const float4 N[3], const float pc[3], float out[3]) {
  const float4 C0 = a.color[v[0]], C1 = a.color[v[1]], C2 = a.color[v[2]];
  const V3 n = norm3(mk3(pc[0] * N[0].x + pc[1] * N[1].x + pc[2] * N[2].x,
                         pc[0] * N[0].y + pc[1] * N[1].y + pc[2] * N[2].y,
                         pc[0] * N[0].z + pc[1] * N[1].z + pc[2] * N[2].z));
  const float fr = pc[0] * C0.x + pc[1] * C1.x + pc[2] * C2.x;
  const float fg = pc[0] * C0.y + pc[1] * C1.y + pc[2] * C2.y;
  const float fb = pc[0] * C0.z + pc[1] * C1.z + pc[2] * C2.z;
  const V3 nl = norm3(mk3(d.light_dir[0], d.light_dir[1], d.light_dir[2]));
  float ndotl = dot3(n, nl);
  if (ndotl < 0.0f)
    ndotl = 0.0f;
  const float lit = d.ambient + (1.0f - d.ambient) * ndotl;
  const V3 hv = norm3(mk3(nl.x, nl.y + 1.0f, nl.z));
  float ndoth = dot3(n, hv);
  if (ndoth < 0.0f)
    ndoth = 0.0f;
  float spec = ndoth * ndoth;
  spec *= spec;
  spec *= spec;
  spec *= spec;
  spec *= spec;
  spec *= 0.25f;
  const float p[3] = {fr * lit + spec, fg * lit + spec, fb * lit + spec};
  for (int c = 0; c < 3; c++)
    out[c] = p[c] < 0.0f ? 0.0f : p[c];
}

int mopcuda_launch_frame(const FrameArgs &a, const PostArgs &p, const LaunchCfg &cfg,
                         cudaStream_t s, cudaEvent_t *ev, PrePostHook before_post,
                         void *hook_ctx) {
  int launches = 0;
  const uint32_t S = (uint32_t)a.width * (uint32_t)a.height;
  if (ev)
    cudaEventRecord(ev[0], s);
  /* the kernels from here to the post pass follow one another with
   * programmatic dependent launches (pdl) */
  if (a.total_vertices) {
    pdl(k_vertex, blocks_for(a.total_vertices, 256), 256, s, a);
    launches++;
  }
  if (ev)
    cudaEventRecord(ev[1], s);
  if (a.total_tris) {
    const unsigned cg = blocks_for(a.clip_cap < 65536u ? a.clip_cap : 65536u, 128);
    if (a.shadow_keys) {
      pdl(k_setup<true>, blocks_for(a.total_tris, 256), 256, s, a);
      pdl(k_clip<true>, cg, 128, s, a);
    } else {
      pdl(k_setup<false>, blocks_for(a.total_tris, 256), 256, s, a);
      pdl(k_clip<false>, cg, 128, s, a);
    }
    launches += 2;
  }
  if (ev)
    cudaEventRecord(ev[2], s);
  if (a.total_tris) {
    const int rb = cfg.raster_block > 0 ? cfg.raster_block : 128;
    const uint32_t rec_grid = blocks_for(a.rec_cap < (1u << 22) ? a.rec_cap : (1u << 22),
                                         (unsigned)rb);
    pdl(k_raster_small, rec_grid, rb, s, a);
    pdl(k_raster_large, cfg.num_sms * 8, 256, s, a);
    launches += 2;
  }
  if (ev)
    cudaEventRecord(ev[3], s);
  pdl(k_resolve, cfg.num_sms * 8, 256, s, a);
  if (ev)
    cudaEventRecord(ev[4], s);
  const int sb = cfg.shade_block > 0 ? cfg.shade_block : 256;
  const int waves = cfg.shade_waves > 0 ? cfg.shade_waves : 4;
  if (a.shadow_keys)
    pdl(k_shade<true>, cfg.num_sms * waves, sb, s, a);
  else
    pdl(k_shade<false>, cfg.num_sms * waves, sb, s, a);
  launches += 2;
  if (a.hdr) { /* blended suffix, composited in submission order */
    cudaMemsetAsync(a.frag_head, 0xff, sizeof(uint32_t) * (size_t)S, s);
    const uint32_t nrec = a.rec_cap < (1u << 22) ? a.rec_cap : (1u << 22);
    pdl(k_ocount, blocks_for(nrec, 256), 256, s, a);
    pdl(k_oscan, 1, 1024, s, a);
    pdl(k_oraster, cfg.num_sms * 8, 256, s, a);
    launches += 3;
    if (a.wire) { /* wireframe draws: their line plots join the fragment lists */
      pdl(k_wcount, blocks_for(nrec, 256), 256, s, a);
      pdl(k_wscan, 1, 1024, s, a);
      pdl(k_wplot, cfg.num_sms * 8, 256, s, a);
      launches += 3;
      if (a.shadow_keys)
        pdl(k_ofold<true, true>, cfg.num_sms * 8, 128, s, a);
      else
        pdl(k_ofold<false, true>, cfg.num_sms * 8, 128, s, a);
    } else if (a.shadow_keys) {
      pdl(k_ofold<true, false>, cfg.num_sms * 8, 128, s, a);
    } else {
      pdl(k_ofold<false, false>, cfg.num_sms * 8, 128, s, a);
    }
    launches += 1;
  }
  if (ev)
    cudaEventRecord(ev[5], s);
  /* the previous frame's image may still be on its way to the host */
  cudaEvent_t post_wait = before_post ? before_post(hook_ctx) : nullptr;
  if (post_wait)
    cudaStreamWaitEvent(s, post_wait, 0);
  const int sf = p.ssaa;
  dim3 pb(POST_BX, POST_BY);
  const uint32_t tiles = blocks_for((uint32_t)(p.width / sf), POST_BX) *
                         blocks_for((uint32_t)(p.height / sf), POST_BY);
  auto pgrid = [&](int resident) {
    const uint32_t g = (uint32_t)cfg.num_sms * (uint32_t)resident;
    return tiles < g ? (tiles ? tiles : 1u) : g;
  };
  switch (sf) {
  case 2:
    pdl(k_post<2>, pgrid(post_resident<2>()), pb, s, p);
    break;
  case 3:
    pdl(k_post<3>, pgrid(post_resident<3>()), pb, s, p);
    break;
  case 4:
    pdl(k_post<4>, pgrid(post_resident<4>()), pb, s, p);
    break;
  default:
    pdl(k_post<1>, pgrid(post_resident<1>()), pb, s, p);
    break;
  }
  launches++;
  if (ev)
    cudaEventRecord(ev[6], s);
  return launches;
}

int mopcuda_shade_occupancy(int block) {
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_shade<false>, block, 0);
  return nb > 0 ? nb : 1;
}

/* FP32 add/multiply issue peak without FMA: the denominator of the shading
 * roofline (the frame path is compiled with -fmad=false).  Each thread runs
 * 8 independent chains of alternating FMUL and FADD. */
__global__ void k_fp32_peak(float *out, int iters, float a, float b) {
  float x[8];
  for (int k = 0; k < 8; k++)
    x[k] = (float)(threadIdx.x + k) * 1e-3f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) {
      x[k] = __fmul_rn(x[k], a);
      x[k] = __fadd_rn(x[k], b);
    }
  }
  float s = 0.0f;
  for (int k = 0; k < 8; k++)
    s += x[k];
  if (s == 123.456f)
    out[blockIdx.x] = s;
}

int mopcuda_launch_fp32_peak(float *out, int blocks, int iters, cudaStream_t s) {
  k_fp32_peak<<<blocks, 256, 0, s>>>(out, iters, 0.999999f, 1e-7f);
  return 1;
}

int mopcuda_launch_box(const uchar4 *src, int width, int height, int sf, uchar4 *dst,
                       cudaStream_t s) {
  dim3 b(16, 16);
  dim3 g(blocks_for((uint32_t)(width / sf), 16), blocks_for((uint32_t)(height / sf), 16));
  k_box<<<g, b, 0, s>>>(src, width, height, sf, dst);
  return 1;
}

int mopcuda_launch_pick(const uint32_t *ids, const float *depth, int width, int height, int sf,
                        const int2 *xy, uint32_t n, uint32_t *out_id, float *out_depth,
                        int32_t *out_hit, cudaStream_t s) {
  if (n == 0)
    return 0;
  k_pick<<<blocks_for(n, 128), 128, 0, s>>>(ids, depth, width, height, sf, xy, n, out_id,
                                             out_depth, out_hit);
  return 1;
}


/* ========================================================================
 * Ordered suffix: blended draws (and every draw after the first one) in
 * submission order per sample — mop_sw_rasterize_triangle_smooth_ml's
 * blended branch (rasterizer.c:2094-2140) and the flat opaque path
 * (:890-1024), which read and write the colour, depth and ID the earlier
 * fragments left.  The records are rasterised into per-sample fragment
 * lists (fragments at or behind the opaque pass's depth can never pass: the
 * depth only decreases), each sample sorts its list by submission order and
 * folds it sequentially.
 * ======================================================================== */
__device__ __forceinline__ uint32_t ordered_record_items(const FrameArgs &a) {
  return raster_small_items(a);
}

/* Queues record rid if it is a live record of the suffix, with its
 * (row, chunk) count. */
__device__ __forceinline__ void ocount_item(const FrameArgs &a, uint32_t rid) {
  const RasterRec r = a.rrec[rid];
  if (!rec_live(r, a.width, a.height) || !rec_ordered(a, r))
    return;
  const uint32_t q = atomicAdd(&a.ctr->olist_count, 1u);
  if (q < a.olist_cap) {
    a.olist[q] = rid;
    a.olist_items[q] = rec_items(r);
  } else {
    atomicOr(&a.ctr->overflow, 32u);
  }
}

__global__ void __launch_bounds__(256) k_ocount(FrameArgs a) {
  pdl_wait();
  const uint32_t n = ordered_record_items(a);
  for (uint32_t rid = blockIdx.x * blockDim.x + threadIdx.x; rid < n;
       rid += gridDim.x * blockDim.x)
    ocount_item(a, rid);
}

__global__ void __launch_bounds__(1024) k_oscan(FrameArgs a) {
  pdl_wait();
  __shared__ uint32_t part[32];
  uint32_t n = a.ctr->olist_count;
  if (n > a.olist_cap)
    n = a.olist_cap;
  items_scan_block(a.olist_items, n, &a.ctr->olist_items, part);
}

/* Links a fragment into sample px's list.  Node and touched-list slots come
 * from warp-aggregated allocations (one atomic per group of converged lanes,
 * not one per fragment on two shared counters); the fold sorts each list,
 * so the order of the slots does not matter. */
__device__ __forceinline__ void push_fragment(const FrameArgs &a, uint32_t px, uint32_t order) {
  const uint32_t node = warp_alloc1(&a.ctr->frag_count);
  if (node >= a.frag_cap) {
    atomicOr(&a.ctr->overflow, 16u);
    return;
  }
  const uint32_t prev = atomicExch(&a.frag_head[px], node);
  a.frags[node] = make_uint2(prev, order);
  if (prev == 0xffffffffu) /* first fragment of this sample */
    a.touched[warp_alloc1(&a.ctr->touched_count)] = px;
}

/* One (row, 32-sample chunk) item of a suffix record (nl: records queued):
 * the reference's edge walk from the folded chunk start; covered samples in
 * front of the opaque depth get a fragment. */
__device__ __forceinline__ void oraster_item(const FrameArgs &a, uint32_t it, uint32_t nl) {
  uint32_t lo = 0, hi = nl;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a.olist_items[mid] <= it)
      lo = mid;
    else
      hi = mid;
  }
  const uint32_t rid = a.olist[lo];
  if (rid >= a.rec_cap)
    return;
  const RasterRec r = a.rrec[rid];
  const bool flat = (r.y1 & REC_FLAT_BIT) != 0;
  const uint32_t wd = (uint32_t)r.x1 - (uint32_t)r.x0 + 1u;
  const uint32_t chunks = (wd + RASTER_CHUNK - 1u) / RASTER_CHUNK;
  const uint32_t local = it - a.olist_items[lo];
  const int jr = (int)(local / chunks), kc = (int)((local % chunks) * RASTER_CHUNK);
  const int y = (int)r.y0 + jr;
  if (y > (int)(r.y1 & 0x7fffu))
    return;
  const int xs = (int)r.x0 + kc, xe = min((int)r.x1, xs + RASTER_CHUNK - 1);
  float w0 = fold_add(fold_add(r.w0[0], r.dy[0], jr), r.dx[0], kc);
  float w1 = fold_add(fold_add(r.w0[1], r.dy[1], jr), r.dx[1], kc);
  float w2 = fold_add(fold_add(r.w0[2], r.dy[2], jr), r.dx[2], kc);
  float z = flat ? fold_add(fold_add(r.zc[0], r.zc[2], jr), r.zc[1], kc) : 0.0f;
  const uint32_t rowbase = (uint32_t)y * (uint32_t)a.width;
  for (int x = xs; x <= xe; x++) {
    if (w0 >= 0.0f && w1 >= 0.0f && w2 >= 0.0f) {
      float zz = z;
      if (!flat) {
        const float b0 = w0 * r.inv_area, b1 = w1 * r.inv_area, b2 = w2 * r.inv_area;
        zz = b0 * r.zc[0] + b1 * r.zc[1] + b2 * r.zc[2];
      }
      const uint32_t px = rowbase + (uint32_t)x;
      if (a.ordered_keep_all || zz < a.depth[px])
        push_fragment(a, px, r.order);
    }
    w0 = __fadd_rn(w0, r.dx[0]);
    w1 = __fadd_rn(w1, r.dx[1]);
    w2 = __fadd_rn(w2, r.dx[2]);
    if (flat)
      z = __fadd_rn(z, r.zc[1]);
  }
}

__device__ __forceinline__ uint32_t olist_len(const FrameArgs &a) {
  const uint32_t nl = a.ctr->olist_count;
  return nl > a.olist_cap ? a.olist_cap : nl;
}

__global__ void __launch_bounds__(256) k_oraster(FrameArgs a) {
  pdl_wait();
  const uint32_t nl = olist_len(a);
  const uint32_t total = a.ctr->olist_items;
  for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < total;
       it += gridDim.x * blockDim.x)
    oraster_item(a, it, nl);
}

/* ------------------------------------------------------------------------
 * Wireframe: mop_sw_draw_line_aa with thickness 1 (Xiaolin Wu,
 * rasterizer.c:743-871) over the triangle's edges v0-v1, v1-v2, v2-v0.  A
 * line's plots are numbered as the reference issues them: the first end
 * pixel's two plots, the second end's two, then two per column between.
 * Each plot is an item; its inputs are recomputed from the record wherever
 * it is needed, the running row `intery` of column j by fold_add (the exact
 * result of the reference's j sequential additions of the gradient).
 * ------------------------------------------------------------------------ */
struct WuLine {
  float x0, y0, z0, x1, y1, z1; /* after the steep and left-to-right swaps */
  float gradient, ye1, gap1, ye2, gap2, intery, steps;
  int xp1, xp2;
  bool steep;
};

__device__ __forceinline__ float wu_fpart(float x) { return x - floorf(x); }
__device__ __forceinline__ float wu_rfpart(float x) { return 1.0f - wu_fpart(x); }

__device__ __forceinline__ void wu_setup(float x0, float y0, float z0, float x1, float y1, float z1,
                                         WuLine &L) {
  L.steep = fabsf(y1 - y0) > fabsf(x1 - x0);
  if (L.steep) {
    float t = x0;
    x0 = y0;
    y0 = t;
    t = x1;
    x1 = y1;
    y1 = t;
  }
  if (x0 > x1) {
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
  L.x0 = x0;
  L.y0 = y0;
  L.z0 = z0;
  L.x1 = x1;
  L.y1 = y1;
  L.z1 = z1;
  const float dx = x1 - x0, dy = y1 - y0;
  L.gradient = dx < 0.001f ? 1.0f : dy / dx;
  float xe = roundf(x0);
  L.ye1 = y0 + L.gradient * (xe - x0);
  L.gap1 = wu_rfpart(x0 + 0.5f);
  L.xp1 = x86_f2i(xe);
  L.intery = L.ye1 + L.gradient;
  xe = roundf(x1);
  L.ye2 = y1 + L.gradient * (xe - x1);
  L.gap2 = wu_fpart(x1 + 0.5f);
  L.xp2 = x86_f2i(xe);
  L.steps = (float)(L.xp2 - L.xp1);
  if (L.steps < 1.0f)
    L.steps = 1.0f;
}

__device__ __forceinline__ uint32_t wu_plots(const WuLine &L) {
  const long long between = (long long)L.xp2 - (long long)L.xp1 - 1ll;
  return 4u + (between > 0 ? 2u * (uint32_t)(between < 0x3fffffffll ? between : 0x3fffffffll) : 0u);
}

/* Plot k of line L: pixel, depth and coverage. */
__device__ __forceinline__ void wu_plot(const WuLine &L, uint32_t k, int &px, int &py, float &z,
                                        float &cov) {
  int col, row;
  if (k < 4u) {
    const bool first = k < 2u;
    const float ye = first ? L.ye1 : L.ye2, gap = first ? L.gap1 : L.gap2;
    col = first ? L.xp1 : L.xp2;
    z = first ? L.z0 : L.z1;
    const int yp = x86_f2i(floorf(ye));
    row = yp + (int)(k & 1u);
    cov = (k & 1u) ? wu_fpart(ye) * gap : wu_rfpart(ye) * gap;
  } else {
    const int j = (int)((k - 4u) >> 1);
    col = L.xp1 + 1 + j;
    const float t = (float)(col - L.xp1) / L.steps;
    z = L.z0 + t * (L.z1 - L.z0);
    const float intery = fold_add(L.intery, L.gradient, j);
    row = x86_f2i(floorf(intery)) + (int)(k & 1u);
    cov = (k & 1u) ? wu_fpart(intery) : wu_rfpart(intery);
  }
  px = L.steep ? row : col;
  py = L.steep ? col : row;
}

__device__ __forceinline__ void wu_edge(const RasterRec &r, int e, WuLine &L) {
  const int f = e == 2 ? 0 : e + 1;
  wu_setup(r.w0[e], r.dx[e], r.dy[e], r.w0[f], r.dx[f], r.dy[f], L);
}

/* The wireframe plot behind item `it` (the frame's wire-item numbering):
 * its record, edge and plot. */
__device__ __forceinline__ bool wire_item(const FrameArgs &a, uint32_t it, uint32_t &rid,
                                          WuLine &L, uint32_t &k) {
  uint32_t nl = a.ctr->wire_count;
  if (nl > a.wlist_cap)
    nl = a.wlist_cap;
  if (nl == 0u)
    return false;
  uint32_t lo = 0, hi = nl;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a.wlist_items[mid] <= it)
      lo = mid;
    else
      hi = mid;
  }
  rid = a.wlist[lo];
  if (rid >= a.rec_cap)
    return false;
  const RasterRec r = a.rrec[rid];
  k = it - a.wlist_items[lo];
  for (int e = 0; e < 3; e++) {
    wu_edge(r, e, L);
    const uint32_t n = wu_plots(L);
    if (k < n)
      return true;
    k -= n;
  }
  return false;
}

/* Sort key of a fragment payload: (order, position among the record's
 * plots) for a line plot, (order, 0) for a filled record. */
__device__ __forceinline__ unsigned long long frag_key(const FrameArgs &a, uint32_t v) {
  if (!(v & FRAG_WIRE_BIT))
    return (unsigned long long)v << 32;
  const uint32_t it = v & ~FRAG_WIRE_BIT;
  uint32_t nl = a.ctr->wire_count;
  if (nl > a.wlist_cap)
    nl = a.wlist_cap;
  if (nl == 0u)
    return ~0ull;
  uint32_t lo = 0, hi = nl;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a.wlist_items[mid] <= it)
      lo = mid;
    else
      hi = mid;
  }
  const uint32_t rid = a.wlist[lo];
  if (rid >= a.rec_cap)
    return ~0ull;
  return ((unsigned long long)a.rrec[rid].order << 32) | (unsigned long long)(it - a.wlist_items[lo]);
}

/* Queues the live wireframe records of the suffix with their plot counts. */
__device__ __forceinline__ void wcount_item(const FrameArgs &a, uint32_t rid) {
  const RasterRec r = a.rrec[rid];
  if (r.x1 != (uint16_t)REC_WIRE_X1 || r.y0 == REC_REDIRECT)
    return;
  uint32_t n = 0;
  for (int e = 0; e < 3; e++) {
    WuLine L;
    wu_edge(r, e, L);
    n += wu_plots(L);
  }
  const uint32_t q = atomicAdd(&a.ctr->wire_count, 1u);
  if (q < a.wlist_cap) {
    a.wlist[q] = rid;
    a.wlist_items[q] = n;
  } else {
    atomicOr(&a.ctr->overflow, 128u);
  }
}

__global__ void __launch_bounds__(256) k_wcount(FrameArgs a) {
  pdl_wait();
  const uint32_t n = ordered_record_items(a);
  for (uint32_t rid = blockIdx.x * blockDim.x + threadIdx.x; rid < n;
       rid += gridDim.x * blockDim.x)
    wcount_item(a, rid);
}

__global__ void __launch_bounds__(1024) k_wscan(FrameArgs a) {
  pdl_wait();
  __shared__ uint32_t part[32];
  uint32_t n = a.ctr->wire_count;
  if (n > a.wlist_cap)
    n = a.wlist_cap;
  items_scan_block(a.wlist_items, n, &a.ctr->wire_items, part);
}

/* One line plot: in the framebuffer, coverage at least 0.004 and in front
 * of the opaque depth (or any depth when the suffix keeps every fragment)
 * gives a fragment. */
__device__ __forceinline__ void wplot_item(const FrameArgs &a, uint32_t it) {
  if (it >= FRAG_WIRE_BIT)
    return;
  uint32_t rid, k;
  WuLine L;
  if (!wire_item(a, it, rid, L, k))
    return;
  int x, y;
  float z, cov;
  wu_plot(L, k, x, y, z, cov);
  if (x < 0 || x >= a.width || y < 0 || y >= a.height || cov < 0.004f)
    return;
  const uint32_t px = (uint32_t)y * (uint32_t)a.width + (uint32_t)x;
  if (a.ordered_keep_all || z < a.depth[px])
    push_fragment(a, px, FRAG_WIRE_BIT | it);
}

__global__ void __launch_bounds__(256) k_wplot(FrameArgs a) {
  pdl_wait();
  const uint32_t total = a.ctr->wire_items;
  for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < total;
       it += gridDim.x * blockDim.x)
    wplot_item(a, it);
}

/* The record behind an order (triangle << 5 | fan), as shade_item finds it. */
__device__ __forceinline__ uint32_t record_of(const FrameArgs &a, uint32_t order) {
  const uint32_t t = order >> ORDER_FAN_BITS, fan = order & ((1u << ORDER_FAN_BITS) - 1u);
  if (t >= a.total_tris)
    return 0xffffffffu;
  const RasterRec r = a.rrec[t];
  if (r.y0 == REC_REDIRECT)
    return r.order + fan;
  return fan == 0u ? t : 0xffffffffu;
}

/* The composition state of one sample while its fragments are applied. */
struct OFold {
  float hdr[3];
  float depth;
  uint32_t id;
  /* a depth-write-off draw's depth is undone when the draw ends: `saved`
   * holds the depth from before it, `cur` the draw of the last fragment */
  float saved;
  uint32_t cur;
  bool cur_nw;
};

/* A fragment of draw di follows: when the draw changes, a finished
 * depth-write-off draw's depth is undone (cpu_backend.c:575-580) and a new
 * one's saved (:536-544). */
__device__ __forceinline__ void ofold_enter_draw(OFold &st, uint32_t di, const DrawRec &d) {
  if (di != st.cur) {
    if (st.cur_nw)
      st.depth = st.saved;
    st.cur = di;
    st.cur_nw = (d.flags & DF_NO_DEPTH_WRITE) != 0;
    if (st.cur_nw)
      st.saved = st.depth;
  }
}

/* Applies line plot `it` at its sample: aa_plot (rasterizer.c:687-729) on
 * the sample's HDR colour, depth and ID. */
__device__ __forceinline__ void ofold_wire(const FrameArgs &a, OFold &st, uint32_t it) {
  uint32_t rid, k;
  WuLine L;
  if (!wire_item(a, it, rid, L, k))
    return;
  const ShadeRec s = a.srec[rid];
  const uint32_t di = s.draw < a.draw_count ? s.draw : 0;
  const DrawRec &d = a.draws[di];
  ofold_enter_draw(st, di, d);
  int px, py;
  float z, cov;
  wu_plot(L, k, px, py, z, cov);
  if (!(d.flags & DF_NO_DEPTH_TEST) && z >= st.depth)
    return;
  const float inv = 1.0f - cov;
  for (int c = 0; c < 3; c++) {
    /* the line colour as the reference's byte (rasterizer.c:1226-1228) */
    const float v = s.col[c] > 1.0f ? 1.0f : s.col[c];
    const float src = (float)(uint8_t)x86_f2i(v * 255.0f) / 255.0f;
    st.hdr[c] = src * cov + st.hdr[c] * inv;
  }
  if (cov > 0.5f) {
    st.depth = z;
    st.id = d.object_id;
  }
}

/* Applies the fragment of submission order `order` at sample (x, y). */
template <bool SH>
__device__ __forceinline__ void ofold_fragment(const FrameArgs &a, OFold &st, int x, int y,
                                               uint32_t order) {
  const uint32_t rid = record_of(a, order);
  if (rid >= a.rec_cap)
    return;
  const RasterRec r = a.rrec[rid];
  const ShadeRec s = a.srec[rid];
  const uint32_t di = s.draw < a.draw_count ? s.draw : 0;
  const DrawRec &d = a.draws[di];
  ofold_enter_draw(st, di, d);
  const bool dtest = !(d.flags & DF_NO_DEPTH_TEST);
  const int jr = y - (int)r.y0, kc = x - (int)r.x0;
  if (r.y1 & REC_FLAT_BIT) { /* rasterize_filled_triangle, rasterizer.c:1000-1083 */
    const float z = fold_add(fold_add(r.zc[0], r.zc[2], jr), r.zc[1], kc);
    if (!dtest || z < st.depth) {
      float ca = d.opacity < 0.0f ? 0.0f : (d.opacity > 1.0f ? 1.0f : d.opacity);
      if (!(d.flags & DF_LIT)) /* the unlit path quantises it (rasterizer.c:1159, 1237) */
        ca = (float)(uint8_t)x86_f2i(ca * 255.0f) / 255.0f;
      if (d.blend_mode == 0 && ca >= 1.0f) {
        st.hdr[0] = s.col[0];
        st.hdr[1] = s.col[1];
        st.hdr[2] = s.col[2];
        st.depth = z;
        st.id = d.object_id;
      } else { /* blended: colour only, no depth or ID write */
        const float inv_a = 1.0f - ca;
        for (int c = 0; c < 3; c++) {
          if (d.blend_mode == 2)
            st.hdr[c] = st.hdr[c] + s.col[c] * ca;
          else if (d.blend_mode == 3)
            st.hdr[c] = st.hdr[c] * s.col[c];
          else
            st.hdr[c] = s.col[c] * ca + st.hdr[c] * inv_a;
        }
      }
    }
    return;
  }
  float w[3];
  for (int e = 0; e < 3; e++)
    w[e] = fold_add(fold_add(r.w0[e], r.dy[e], jr), r.dx[e], kc);
  const float b0 = w[0] * r.inv_area, b1 = w[1] * r.inv_area, b2 = w[2] * r.inv_area;
  const float z = b0 * r.zc[0] + b1 * r.zc[1] + b2 * r.zc[2];
  if (dtest && !(z < st.depth))
    return;
  if (s.v[0] >= a.vertex_cap || s.v[1] >= a.vertex_cap || s.v[2] >= a.vertex_cap)
    return;
  const float4 N[3] = {a.normal[s.v[0]], a.normal[s.v[1]], a.normal[s.v[2]]};
  float pc[3] = {b0 * N[0].w, b1 * N[1].w, b2 * N[2].w};
  const float ip = 1.0f / (pc[0] + pc[1] + pc[2]);
  pc[0] *= ip;
  pc[1] *= ip;
  pc[2] *= ip;
  /* edge-distance coverage (rasterizer.c:1899-1938, 1320-1361) */
  float min_d = 0.0f;
  for (int e = 0; e < 3; e++) {
    const float len = sqrtf(r.dx[e] * r.dx[e] + r.dy[e] * r.dy[e]);
    const float inv = len > 1e-6f ? 1.0f / len : 0.0f;
    const float de = w[e] * inv;
    if (e == 0 || de < min_d)
      min_d = de;
  }
  const bool legacy = !(d.flags & DF_LIT);
  if (legacy && !(min_d >= 0.0f))
    return;
  float p[3];
  if (legacy)
    shade_legacy(a, d, s.v, N, pc, p);
  else
    shade_smooth<SH>(a, d, a.lights + d.light_off, s.v, N, pc, p);
  const float op = d.opacity < 0.0f ? 0.0f : (d.opacity > 1.0f ? 1.0f : d.opacity);
  /* the legacy path blends at silhouettes only: where the sample's depth
   * so far lies clearly behind the fragment (rasterizer.c:1425-1429);
   * the multi-light path blends at every edge of a non-opaque draw
   * (rasterizer.c:2097-2100) */
  const float cov = legacy ? ((min_d < 1.0f && (st.depth - z) > 0.005f) ? min_d : 1.0f)
                           : ((min_d < 1.0f && d.blend_mode != 0) ? min_d : 1.0f);
  const float fa = op * cov;
  if (d.blend_mode == 0 && fa >= 1.0f) {
    st.hdr[0] = p[0];
    st.hdr[1] = p[1];
    st.hdr[2] = p[2];
    st.depth = z;
    st.id = d.object_id;
  } else {
    const float inv = 1.0f - fa;
    for (int c = 0; c < 3; c++) {
      if (d.blend_mode == 2)
        st.hdr[c] = st.hdr[c] + p[c] * fa;
      else if (d.blend_mode == 3)
        st.hdr[c] = st.hdr[c] * p[c];
      else
        st.hdr[c] = p[c] * fa + st.hdr[c] * inv;
    }
    if (fa > 0.5f) {
      st.depth = z;
      st.id = d.object_id;
    }
  }
}

/* Ascending heapsort of n (key, payload) pairs by key (distinct keys). */
__device__ __forceinline__ void heap_sift(ulonglong2 *h, uint32_t i, uint32_t n) {
  const ulonglong2 v = h[i];
  for (;;) {
    uint32_t c = 2u * i + 1u;
    if (c >= n)
      break;
    if (c + 1u < n && h[c + 1u].x > h[c].x)
      c++;
    if (h[c].x <= v.x)
      break;
    h[i] = h[c];
    i = c;
  }
  h[i] = v;
}

__device__ __noinline__ void heapsort_keys(ulonglong2 *h, uint32_t n) {
  if (n < 2u)
    return;
  for (uint32_t i = n / 2u; i-- > 0u;)
    heap_sift(h, i, n);
  for (uint32_t e = n - 1u; e > 0u; e--) {
    const ulonglong2 t = h[0];
    h[0] = h[e];
    h[e] = t;
    heap_sift(h, 0u, e);
  }
}

/* Each touched sample folds its fragments in submission order.  Up to
 * ORDERED_MAX_FRAGS are gathered and insertion-sorted in registers; a
 * longer list is copied with its keys into the fold's scratch and heapsorted
 * there (keys are distinct: a record covers a sample once, a line plot is
 * one item).  WIRE: the frame has line
 * plots, whose payloads sort by frag_key (a triangle's plots in the
 * reference's drawing order after the triangles before it). */
template <bool WIRE>
__device__ __forceinline__ unsigned long long ofold_key(const FrameArgs &a, uint32_t v) {
  return (WIRE && a.wire) ? frag_key(a, v) : (unsigned long long)v;
}

template <bool SH, bool WIRE>
__device__ __forceinline__ void ofold_apply(const FrameArgs &a, OFold &st, int x, int y,
                                            uint32_t v) {
  if (WIRE && a.wire && (v & FRAG_WIRE_BIT))
    ofold_wire(a, st, v & ~FRAG_WIRE_BIT);
  else
    ofold_fragment<SH>(a, st, x, y, v);
}

template <bool SH, bool WIRE>
__device__ __forceinline__ void ofold_item(const FrameArgs &a, uint32_t i) {
  const uint32_t px = a.touched[i];
  const uint32_t head = a.frag_head[px];
  uint32_t ord[ORDERED_MAX_FRAGS];
  uint32_t cnt = 0, total = 0;
  for (uint32_t node = head; node != 0xffffffffu && node < a.frag_cap; node = a.frags[node].x) {
    if (cnt < ORDERED_MAX_FRAGS)
      ord[cnt++] = a.frags[node].y;
    if (++total > a.frag_cap)
      break;
  }
  const int x = (int)(px % (uint32_t)a.width), y = (int)(px / (uint32_t)a.width);
  OFold st;
  if (a.keys[px] != KEY_EMPTY) {
    const float4 h = a.hdr[px];
    st.hdr[0] = h.x;
    st.hdr[1] = h.y;
    st.hdr[2] = h.z;
  } else if (a.sky) {
    sky_hdr(a, x, y, st.hdr);
  } else {
    st.hdr[0] = a.clear[0];
    st.hdr[1] = a.clear[1];
    st.hdr[2] = a.clear[2];
  }
  st.depth = a.depth[px];
  st.id = a.ids[px];
  st.saved = st.depth;
  st.cur = 0xffffffffu;
  st.cur_nw = false;
  if (total <= ORDERED_MAX_FRAGS) {
    if (WIRE && a.wire) { /* keys computed once: a plot's key takes a search */
      unsigned long long key[WIRE ? ORDERED_MAX_FRAGS : 1];
      for (uint32_t k = 0; k < cnt; k++)
        key[k] = frag_key(a, ord[k]);
      for (uint32_t k = 1; k < cnt; k++) {
        const uint32_t v = ord[k];
        const unsigned long long kv = key[k];
        uint32_t j = k;
        while (j > 0 && key[j - 1] > kv) {
          ord[j] = ord[j - 1];
          key[j] = key[j - 1];
          j--;
        }
        ord[j] = v;
        key[j] = kv;
      }
    } else {
      for (uint32_t k = 1; k < cnt; k++) { /* submission order */
        const uint32_t v = ord[k];
        uint32_t j = k;
        while (j > 0 && ord[j - 1] > v) {
          ord[j] = ord[j - 1];
          j--;
        }
        ord[j] = v;
      }
    }
    for (uint32_t k = 0; k < cnt; k++)
      ofold_apply<SH, WIRE>(a, st, x, y, ord[k]);
  } else {
    /* a long list: its (key, payload) pairs heapsorted in the scratch */
    const uint32_t base = atomicAdd(a.oscratch_count, total);
    if (!a.oscratch || (unsigned long long)base + total > a.oscratch_cap) {
      atomicOr(&a.ctr->overflow, 16u); /* unreachable: the scratch holds the fragment pool */
      return;
    }
    ulonglong2 *sc = a.oscratch + base;
    uint32_t m = 0;
    for (uint32_t node = head; node != 0xffffffffu && node < a.frag_cap && m < total;
         node = a.frags[node].x) {
      const uint32_t v = a.frags[node].y;
      sc[m++] = make_ulonglong2(ofold_key<WIRE>(a, v), (unsigned long long)v);
    }
    heapsort_keys(sc, m);
    for (uint32_t k = 0; k < m; k++)
      ofold_apply<SH, WIRE>(a, st, x, y, (uint32_t)sc[k].y);
  }
  if (st.cur_nw)
    st.depth = st.saved;
  /* mop_sw_hdr_resolve (rasterizer.c:2776-2803) of the composited sample */
  if (st.id == 0u)
    a.pre[px] = make_uchar4(x86_f2u8(fminf(st.hdr[0], 1.0f) * 255.0f + 0.5f),
                            x86_f2u8(fminf(st.hdr[1], 1.0f) * 255.0f + 0.5f),
                            x86_f2u8(fminf(st.hdr[2], 1.0f) * 255.0f + 0.5f), 255);
  else
    a.pre[px] = make_uchar4(u8_of(aces(st.hdr[0] * a.exposure) * 255.0f + 0.5f),
                            u8_of(aces(st.hdr[1] * a.exposure) * 255.0f + 0.5f),
                            u8_of(aces(st.hdr[2] * a.exposure) * 255.0f + 0.5f), 255);
  a.depth[px] = st.depth;
  a.ids[px] = st.id;
}

template <bool SH, bool WIRE>
__global__ void __launch_bounds__(128) k_ofold(FrameArgs a) {
  pdl_wait();
  const uint32_t n = a.ctr->touched_count;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    ofold_item<SH, WIRE>(a, i);
}

/* ========================================================================
 * Batched viewports.  One launch per stage covers every viewport of a batch
 * over one resident scene.  The stage kernels are persistent (a grid of
 * resident blocks), map each work item to (viewport, local item) through a
 * per-block prefix of the viewports' item counts, and run the same per-item
 * code as the single-viewport kernels, so every viewport's result is the
 * one its own frame would give.
 * ======================================================================== */

/* mop_mat4_multiply (math.c:182-194) on the device: running sum from 0,
 * round-to-nearest, no contraction. */
__device__ void dev_mat4_mul(const float *a, const float *b, float *c) {
  for (int col = 0; col < 4; col++)
    for (int row = 0; row < 4; row++) {
      float s = 0.0f;
      for (int k = 0; k < 4; k++)
        s = __fadd_rn(s, __fmul_rn(a[k * 4 + row], b[col * 4 + k]));
      c[col * 4 + row] = s;
    }
}

/* True when every point of the draw's bounding sphere lies outside one
 * clip plane with a margin far above the rounding of the float clip
 * transform (xform: four products, three sums), so every triangle of the
 * draw is trivially rejected by the setup (rasterizer.c:2467-2476) and the
 * draw contributes nothing.  Planes: x > w, x < -w, y > w, y < -w, and with
 * zplanes z > w, z < -w. */
__device__ bool draw_culled(const float *m, const DrawBound &bd, bool zplanes) {
  const double r = (double)bd.r;
  if (!(r >= 0.0) || !isfinite(bd.r) || !isfinite(bd.c[0]) || !isfinite(bd.c[1]) ||
      !isfinite(bd.c[2]))
    return false;
  for (int k = 0; k < 16; k++)
    if (!isfinite(m[k]))
      return false;
  const double c[3] = {(double)bd.c[0], (double)bd.c[1], (double)bd.c[2]};
  for (int axis = 0; axis < (zplanes ? 3 : 2); axis++)
    for (int sg = -1; sg <= 1; sg += 2) {
      double q[4], mag = 0.0;
      for (int j = 0; j < 4; j++) {
        const double ma = (double)m[j * 4 + axis], mw = (double)m[j * 4 + 3];
        q[j] = (double)sg * ma - mw;
        mag += (fabs(ma) + fabs(mw)) * (j < 3 ? fabs(c[j]) + r : 1.0);
      }
      const double dist = q[0] * c[0] + q[1] * c[1] + q[2] * c[2] + q[3];
      const double nrm = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
      if (dist - r * nrm > 1e-5 * mag + 1e-30)
        return true;
    }
  return false;
}

/* Block-wide (256 threads) exclusive prefix of K counters in thread order,
 * continuing the running totals s_tot (updated): off[k] is this thread's
 * offset. */
template <int K>
__device__ __forceinline__ void block_prefix(const uint32_t x[K], uint32_t off[K],
                                             uint32_t (*s_w)[K], uint32_t *s_tot) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t incl[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    incl[k] = x[k];
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl[k], o);
      if (lane >= (uint32_t)o)
        incl[k] += y;
    }
    if (lane == 31u)
      s_w[warp][k] = incl[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < K; k++) {
      uint32_t run = s_tot[k];
      for (int w = 0; w < 8; w++) {
        const uint32_t t = s_w[w][k];
        s_w[w][k] = run;
        run += t;
      }
      s_tot[k] = run;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++)
    off[k] = s_w[warp][k] + incl[k] - x[k];
  __syncthreads(); /* s_w is reused by the next call */
}

/* mvp = P * (V * M) of scene draw i in viewport vw; false when the draw has
 * no triangles or its bounding sphere is outside the frustum. */
__device__ __forceinline__ bool view_draw(const SceneDesc &sc, const ViewRec &vw, uint32_t i,
                                          float mvp[16]) {
  const DrawRec &sd = sc.draws[i];
  float vm[16];
  dev_mat4_mul(vw.view, sd.model, vm);
  dev_mat4_mul(vw.proj, vm, mvp);
  return sd.index_count / 3u > 0u && !draw_culled(mvp, sc.bounds[i], sd.depth_bias == 0.0f);
}

__device__ __forceinline__ void emit_view_draw(const SceneDesc &sc, const ViewRec &vw, uint32_t i,
                                               const float mvp[16], DrawRec *out, uint32_t pos,
                                               uint32_t vbase, uint32_t tbase) {
  DrawRec r = sc.draws[i];
  for (int k = 0; k < 16; k++)
    r.mvp[k] = mvp[k];
  r.cam_eye[0] = vw.eye[0];
  r.cam_eye[1] = vw.eye[1];
  r.cam_eye[2] = vw.eye[2];
  r.vbase = vbase;
  r.tbase = tbase;
  out[pos] = r;
}

/* Per viewport (one block of 256): the viewport's draw list in the core's
 * pass order (viewport.c:2449-2553) — the visible non-blended draws in scene
 * order, then the visible blended draws back to front by the float squared
 * distance of their translation to the eye (the core's insertion sort:
 * farthest first, ties keep scene order) — with mvp = P * (V * M), culling
 * by bounding sphere and the draws' vertex/triangle bases.  Depth ties
 * resolve as in the full frame; the first draw flagged DF_ORDERED, or the
 * first blended one, starts the viewport's ordered suffix (t_split). */
__global__ void __launch_bounds__(256) k_batch_prepare(BatchArgs b) {
  __shared__ uint32_t s_w[8][4];
  __shared__ uint32_t s_tot[4];
  __shared__ uint32_t s_bl[BATCH_MAX_BLENDED]; /* blended draws, scene order */
  __shared__ float s_bd[BATCH_MAX_BLENDED];    /* their squared eye distances */
  __shared__ uint32_t s_by[BATCH_MAX_BLENDED]; /* back-to-front position -> s_bl slot */
  __shared__ uint32_t s_split, s_nan, s_wire;
  const uint32_t v = blockIdx.x;
  const ViewRec &vw = b.views[v];
  const SceneDesc &sc = b.scenes[vw.scene];
  DrawRec *out = b.view_draws + vw.draw_off;
  if (threadIdx.x == 0) {
    s_tot[0] = s_tot[1] = s_tot[2] = s_tot[3] = 0u;
    s_split = 0xffffffffu;
    s_nan = 0u;
    s_wire = 0u;
  }
  __syncthreads();
  for (uint32_t base = 0; base < sc.nd; base += 256u) {
    const uint32_t i = base + threadIdx.x;
    float mvp[16];
    uint32_t x[4] = {0u, 0u, 0u, 0u}, off[4];
    if (i < sc.nd && view_draw(sc, vw, i, mvp)) {
      const DrawRec &sd = sc.draws[i];
      if (sd.blend_mode == 0) {
        x[0] = 1u;
        x[1] = sd.vertex_count;
        x[2] = sd.index_count / 3u;
      } else {
        x[3] = 1u;
      }
    }
    block_prefix<4>(x, off, s_w, s_tot);
    if (x[0]) {
      emit_view_draw(sc, vw, i, mvp, out, off[0], off[1], off[2]);
      if (sc.draws[i].flags & DF_ORDERED)
        atomicMin(&s_split, off[2]);
      if (sc.draws[i].flags & DF_WIRE)
        atomicOr(&s_wire, 1u);
    }
    if (x[3] && off[3] < BATCH_MAX_BLENDED) {
      const float *m = sc.draws[i].model;
      const float dx = __fsub_rn(m[12], vw.eye[0]), dy = __fsub_rn(m[13], vw.eye[1]),
                  dz = __fsub_rn(m[14], vw.eye[2]);
      const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
      s_bl[off[3]] = i;
      s_bd[off[3]] = d2;
      if (d2 != d2)
        s_nan = 1u;
    }
  }
  __syncthreads();
  const uint32_t nb = s_tot[3] < BATCH_MAX_BLENDED ? s_tot[3] : BATCH_MAX_BLENDED;
  if (!s_nan) {
    /* the stable descending order as ranks: the draws farther away, then the
     * equally far ones earlier in scene order */
    for (uint32_t j = threadIdx.x; j < nb; j += 256u) {
      const float dj = s_bd[j];
      uint32_t r = 0;
      for (uint32_t k = 0; k < nb; k++) {
        const float dk = s_bd[k];
        r += (dk > dj || (dk == dj && k < j)) ? 1u : 0u;
      }
      s_by[r] = j;
    }
  } else if (threadIdx.x == 0) {
    /* a NaN distance: the reference's insertion sort itself */
    for (uint32_t j = 0; j < nb; j++)
      s_by[j] = j;
    for (uint32_t j = 1; j < nb; j++) {
      const uint32_t key = s_by[j];
      const float kd = s_bd[key];
      int k = (int)j - 1;
      while (k >= 0 && s_bd[s_by[k]] < kd) {
        s_by[k + 1] = s_by[k];
        k--;
      }
      s_by[k + 1] = key;
    }
  }
  if (threadIdx.x == 0 && nb)
    atomicMin(&s_split, s_tot[2]); /* the first blended draw */
  __syncthreads();
  for (uint32_t base = 0; base < nb; base += 256u) {
    const uint32_t j = base + threadIdx.x;
    float mvp[16];
    uint32_t x[4] = {0u, 0u, 0u, 0u}, off[4];
    uint32_t i = 0;
    if (j < nb) {
      i = s_bl[s_by[j]];
      view_draw(sc, vw, i, mvp);
      x[0] = 1u;
      x[1] = sc.draws[i].vertex_count;
      x[2] = sc.draws[i].index_count / 3u;
    }
    block_prefix<4>(x, off, s_w, s_tot);
    if (x[0]) {
      emit_view_draw(sc, vw, i, mvp, out, off[0], off[1], off[2]);
      if (sc.draws[i].flags & DF_WIRE)
        atomicOr(&s_wire, 1u);
    }
  }
  if (threadIdx.x == 0) {
    FrameArgs a = b.tmpl;
    a.lights = sc.lights;
    a.light_total = sc.light_total;
    a.shadow_keys = sc.shadow_keys;
    a.shadow_vp = sc.shadow_vp;
    a.shadow_w = a.shadow_h = sc.shadow_size;
    a.irr = sc.irr;
    a.irr_w = sc.irr_w;
    a.irr_h = sc.irr_h;
    a.pf = sc.pf;
    a.pf_w = sc.pf_w;
    a.pf_h = sc.pf_h;
    a.pf_levels = sc.pf_levels;
    a.brdf = sc.brdf;
    a.brdf_size = sc.brdf_size;
    a.ibl_rotation = sc.ibl_rotation;
    a.ibl_intensity = sc.ibl_intensity;
    a.no_color = (int)vw.no_color;
    a.draws = out;
    a.draw_count = s_tot[0];
    a.total_vertices = s_tot[1];
    a.total_tris = s_tot[2];
    a.width = vw.width;
    a.height = vw.height;
    a.keys = b.keys + vw.sample_off;
    a.shade_list = b.shade_list + vw.sample_off;
    a.pre = b.pre + vw.sample_off;
    a.depth = b.depth + vw.sample_off;
    a.ids = b.ids + vw.sample_off;
    for (int k = 0; k < 4; k++)
      a.clear[k] = vw.clear[k];
    a.ctr = b.ctr + v;
    /* the suffix: its buffers here, its pools from k_batch_alloc */
    a.t_split = s_split;
    a.ordered_keep_all = 0;
    a.frags = nullptr;
    a.frag_cap = 0u;
    a.olist = a.olist_items = nullptr;
    a.olist_cap = 0u;
    a.wire = (int)s_wire;
    a.wlist = a.wlist_items = nullptr;
    a.wlist_cap = 0u;
    a.oscratch = b.oscratch;
    a.oscratch_count = b.oscratch_count;
    a.oscratch_cap = (uint32_t)(b.frag_pool < 0xffffffffull ? b.frag_pool : 0xffffffffull);
    if (s_wire && !b.wlist)
      atomicOr(&b.status->overflow, 256u);
    if (s_split != 0xffffffffu && b.hdr) {
      a.hdr = b.hdr + vw.sample_off;
      a.frag_head = b.frag_head + vw.sample_off;
      a.touched = b.touched + vw.sample_off;
    } else {
      if (s_split != 0xffffffffu)
        atomicOr(&b.status->overflow, 256u);
      a.hdr = nullptr;
      a.frag_head = a.touched = nullptr;
    }
    b.frames[v] = a;
  }
}

/* One block of 256: carves every viewport's vertex streams, records, clip
 * queue, large list and — for a viewport with an ordered suffix — its
 * suffix-record list and fragment pool out of the batch pools (exclusive
 * scans over the viewports).  A viewport that does not fit renders nothing this time and
 * the status tells the host how large the pools must grow. */
__global__ void __launch_bounds__(256) k_batch_alloc(BatchArgs b) {
  constexpr int NP = 7;
  __shared__ unsigned long long s_w[8][NP];
  __shared__ unsigned long long s_tot[NP];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned long long pool[NP] = {b.vertex_pool, b.rec_pool,   b.clip_pool, b.large_pool,
                                       b.olist_pool,  b.frag_pool, b.wlist_pool};
  if (threadIdx.x < NP)
    s_tot[threadIdx.x] = 0ull;
  __syncthreads();
  for (uint32_t base = 0; base < b.nv; base += 256u) {
    const uint32_t v = base + threadIdx.x;
    unsigned long long need[NP] = {0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
    if (v < b.nv) {
      const FrameArgs &a = b.frames[v];
      const unsigned long long T = a.total_tris, fan = T * b.fan_num / 8ull + 1024ull;
      need[0] = (unsigned long long)a.total_vertices + fan;
      need[1] = T + fan;
      need[2] = fan;
      need[3] = T * b.large_num / 16ull + 1024ull;
      if (a.hdr) {
        need[4] = (T - (a.t_split < T ? a.t_split : T)) + fan;
        need[5] = (unsigned long long)a.width * (unsigned long long)a.height * b.frag_num / 4ull +
                  4096ull;
        if (a.wire)
          need[6] = need[4];
      }
    }
    unsigned long long incl[NP];
    for (int k = 0; k < NP; k++) {
      incl[k] = need[k];
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl[k], o);
        if (lane >= (uint32_t)o)
          incl[k] += y;
      }
      if (lane == 31u)
        s_w[warp][k] = incl[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int k = 0; k < NP; k++) {
        unsigned long long run = s_tot[k];
        for (int w = 0; w < 8; w++) {
          const unsigned long long t = s_w[w][k];
          s_w[w][k] = run;
          run += t;
        }
        s_tot[k] = run;
      }
    }
    __syncthreads();
    if (v < b.nv) {
      unsigned long long off[NP];
      bool fits = true;
      for (int k = 0; k < NP; k++) {
        off[k] = s_w[warp][k] + incl[k] - need[k];
        if (off[k] + need[k] > pool[k]) {
          fits = false;
          atomicOr(&b.status->overflow, 1u << k);
        }
      }
      FrameArgs &a = b.frames[v];
      if (!fits) {
        a.draw_count = 0u;
        a.total_vertices = 0u;
        a.total_tris = 0u;
        a.hdr = nullptr;
        for (int k = 0; k < NP; k++) {
          off[k] = 0ull;
          need[k] = 0ull;
        }
      }
      a.clip = b.clip + off[0];
      a.world = b.world + off[0];
      a.normal = b.normal + off[0];
      a.color = b.color + off[0];
      a.vertex_cap = (uint32_t)need[0];
      a.rrec = b.rrec + off[1];
      a.srec = b.srec + off[1];
      a.rec_cap = (uint32_t)need[1];
      a.clipq = b.clipq + off[2];
      a.clip_cap = (uint32_t)need[2];
      a.large_list = b.large_list + off[3];
      a.large_items = b.large_items + off[3];
      a.large_cap = (uint32_t)need[3];
      if (a.hdr) {
        a.olist = b.olist + off[4];
        a.olist_items = b.olist_items + off[4];
        a.olist_cap = (uint32_t)need[4];
        a.frags = b.frags + off[5];
        a.frag_cap = (uint32_t)(need[5] < 0xfffffff0ull ? need[5] : 0xfffffff0ull);
        if (a.wire) {
          a.wlist = b.wlist + off[6];
          a.wlist_items = b.wlist_items + off[6];
          a.wlist_cap = (uint32_t)need[6];
        }
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    b.status->need_vertex = s_tot[0];
    b.status->need_rec = s_tot[1];
    b.status->need_clip = s_tot[2];
    b.status->need_large = s_tot[3];
    b.status->need_olist = s_tot[4];
    b.status->need_frag = s_tot[5];
    b.status->need_wlist = s_tot[6];
  }
}

enum { ST_VERTEX, ST_SETUP, ST_CLIP, ST_RSMALL, ST_RLARGE, ST_SHADE, ST_RESOLVE, ST_OCOUNT,
       ST_ORASTER, ST_OFOLD, ST_WCOUNT, ST_WPLOT };

template <int ST> __device__ __forceinline__ uint32_t stage_count(const FrameArgs &a) {
  switch (ST) {
  case ST_VERTEX:
    return a.total_vertices;
  case ST_SETUP:
    return a.total_tris;
  case ST_CLIP:
    return clip_items(a);
  case ST_RSMALL:
    return a.total_tris ? raster_small_items(a) : 0u;
  case ST_RLARGE:
    return a.total_tris ? a.ctr->large_items : 0u;
  case ST_SHADE:
    return a.ctr->shade_count;
  case ST_OCOUNT:
    return a.hdr && a.total_tris ? ordered_record_items(a) : 0u;
  case ST_ORASTER:
    return a.hdr ? a.ctr->olist_items : 0u;
  case ST_OFOLD:
    return a.hdr ? a.ctr->touched_count : 0u;
  case ST_WCOUNT:
    return a.hdr && a.wire && a.total_tris ? ordered_record_items(a) : 0u;
  case ST_WPLOT:
    return a.hdr && a.wire ? a.ctr->wire_items : 0u;
  default: /* ST_RESOLVE: chunks of 256 x RESOLVE_PER_THREAD samples */
    return ((uint32_t)a.width * (uint32_t)a.height + 256u * RESOLVE_PER_THREAD - 1u) /
           (256u * RESOLVE_PER_THREAD);
  }
}

/* s_pre[v] = items of viewports before v, s_pre[nv] = total (warp 0). */
template <int ST>
__device__ __forceinline__ uint32_t views_prefix(const FrameArgs *__restrict__ fr, uint32_t nv,
                                                 uint32_t *s_pre) {
  if (threadIdx.x < 32u) {
    const uint32_t lane = threadIdx.x;
    uint32_t run = 0;
    for (uint32_t base = 0; base < nv; base += 32u) {
      const uint32_t v = base + lane;
      const uint32_t c = v < nv ? stage_count<ST>(fr[v]) : 0u;
      uint32_t incl = c;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o)
          incl += y;
      }
      if (v < nv)
        s_pre[v] = run + incl - c;
      run += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0)
      s_pre[nv] = run;
  }
  __syncthreads();
  return s_pre[nv];
}

template <int ST, bool SH>
__global__ void __launch_bounds__(256) k_b_items(const FrameArgs *__restrict__ fr, uint32_t nv) {
  __shared__ uint32_t s_pre[MOPCUDA_MAX_VIEWS + 1];
  const uint32_t total = views_prefix<ST>(fr, nv, s_pre);
  uint32_t v = 0;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += gridDim.x * blockDim.x) {
    while (s_pre[v + 1] <= g)
      v++;
    const uint32_t i = g - s_pre[v];
    const FrameArgs &a = fr[v];
    if (ST == ST_VERTEX)
      vertex_item(a, i);
    else if (ST == ST_SETUP)
      setup_item<SH>(a, i);
    else if (ST == ST_CLIP)
      clip_item<SH>(a, i);
    else if (ST == ST_RSMALL)
      raster_small_item(a, i);
    else
      raster_large_item(a, i);
  }
}

__global__ void __launch_bounds__(256) k_b_resolve(const FrameArgs *__restrict__ fr,
                                                   uint32_t nv) {
  __shared__ uint32_t s_pre[MOPCUDA_MAX_VIEWS + 1];
  __shared__ uint32_t s_warp[8];
  __shared__ uint32_t s_base;
  const uint32_t total = views_prefix<ST_RESOLVE>(fr, nv, s_pre);
  uint32_t v = 0;
  for (uint32_t u = blockIdx.x; u < total; u += gridDim.x) {
    while (s_pre[v + 1] <= u)
      v++;
    resolve_chunk(fr[v], (u - s_pre[v]) * (256u * RESOLVE_PER_THREAD), s_warp, &s_base);
  }
}

/* shared_lights: every viewport of the launch reads one light array (one
 * scene), staged in shared memory; otherwise each reads its own. */
template <bool SH>
__global__ void __launch_bounds__(256, 4) k_b_shade(const FrameArgs *__restrict__ fr,
                                                    uint32_t nv, int shared_lights) {
  __shared__ LightRec s_lights[SHADE_SMEM_LIGHTS];
  __shared__ uint32_t s_pre[MOPCUDA_MAX_VIEWS + 1];
  const LightRec *lights = shared_lights ? stage_lights(fr[0], s_lights) : nullptr;
  const uint32_t total = views_prefix<ST_SHADE>(fr, nv, s_pre);
  uint32_t v = 0;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += gridDim.x * blockDim.x) {
    while (s_pre[v + 1] <= g)
      v++;
    const FrameArgs &a = fr[v];
    shade_item<SH>(a, g - s_pre[v], lights ? lights : a.lights);
  }
}

/* The ordered suffix of every viewport that has one, as the single-frame
 * kernels run it: queue the suffix records, scan their item counts (a block
 * per viewport), rasterise them into fragment lists, fold each touched
 * sample's list in submission order. */
__global__ void __launch_bounds__(256) k_b_ocount(const FrameArgs *__restrict__ fr, uint32_t nv) {
  __shared__ uint32_t s_pre[MOPCUDA_MAX_VIEWS + 1];
  const uint32_t total = views_prefix<ST_OCOUNT>(fr, nv, s_pre);
  uint32_t v = 0;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += gridDim.x * blockDim.x) {
    while (s_pre[v + 1] <= g)
      v++;
    ocount_item(fr[v], g - s_pre[v]);
  }
}

__global__ void __launch_bounds__(1024) k_b_oscan(const FrameArgs *__restrict__ fr) {
  __shared__ uint32_t part[32];
  const FrameArgs &a = fr[blockIdx.x];
  if (a.hdr)
    items_scan_block(a.olist_items, olist_len(a), &a.ctr->olist_items, part);
}

__global__ void __launch_bounds__(256) k_b_oraster(const FrameArgs *__restrict__ fr, uint32_t nv) {
  __shared__ uint32_t s_pre[MOPCUDA_MAX_VIEWS + 1];
  const uint32_t total = views_prefix<ST_ORASTER>(fr, nv, s_pre);
  uint32_t v = 0;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += gridDim.x * blockDim.x) {
    while (s_pre[v + 1] <= g)
      v++;
    const FrameArgs &a = fr[v];
    oraster_item(a, g - s_pre[v], olist_len(a));
  }
}

/* Wireframe records of the viewports that have them (k_wcount, k_wscan,
 * k_wplot per viewport). */
__global__ void __launch_bounds__(256) k_b_wcount(const FrameArgs *__restrict__ fr, uint32_t nv) {
  __shared__ uint32_t s_pre[MOPCUDA_MAX_VIEWS + 1];
  const uint32_t total = views_prefix<ST_WCOUNT>(fr, nv, s_pre);
  uint32_t v = 0;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += gridDim.x * blockDim.x) {
    while (s_pre[v + 1] <= g)
      v++;
    wcount_item(fr[v], g - s_pre[v]);
  }
}

__global__ void __launch_bounds__(1024) k_b_wscan(const FrameArgs *__restrict__ fr) {
  __shared__ uint32_t part[32];
  const FrameArgs &a = fr[blockIdx.x];
  if (a.hdr && a.wire) {
    uint32_t n = a.ctr->wire_count;
    if (n > a.wlist_cap)
      n = a.wlist_cap;
    items_scan_block(a.wlist_items, n, &a.ctr->wire_items, part);
  }
}

__global__ void __launch_bounds__(256) k_b_wplot(const FrameArgs *__restrict__ fr, uint32_t nv) {
  __shared__ uint32_t s_pre[MOPCUDA_MAX_VIEWS + 1];
  const uint32_t total = views_prefix<ST_WPLOT>(fr, nv, s_pre);
  uint32_t v = 0;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += gridDim.x * blockDim.x) {
    while (s_pre[v + 1] <= g)
      v++;
    wplot_item(fr[v], g - s_pre[v]);
  }
}

template <bool SH, bool WIRE>
__global__ void __launch_bounds__(128) k_b_ofold(const FrameArgs *__restrict__ fr, uint32_t nv) {
  __shared__ uint32_t s_pre[MOPCUDA_MAX_VIEWS + 1];
  const uint32_t total = views_prefix<ST_OFOLD>(fr, nv, s_pre);
  uint32_t v = 0;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += gridDim.x * blockDim.x) {
    while (s_pre[v + 1] <= g)
      v++;
    ofold_item<SH, WIRE>(fr[v], g - s_pre[v]);
  }
}

template <int SF>
__device__ __forceinline__ uint32_t post_tiles_of(const PostArgs &p) {
  const uint32_t pw = (uint32_t)(p.width / SF), ph = (uint32_t)(p.height / SF);
  return ((pw + POST_BX - 1u) / POST_BX) * ((ph + POST_BY - 1u) / POST_BY);
}

/* Post tiles of the viewports listed in views (all with ssaa SF). */
template <int SF>
__global__ void __launch_bounds__(POST_BX *POST_BY, 4) k_b_post(const PostArgs *__restrict__ posts,
                                                             const uint32_t *__restrict__ views,
                                                             uint32_t n) {
  __shared__ PostSmem<SF> sm;
  __shared__ uint32_t s_pre[MOPCUDA_MAX_VIEWS + 1];
  const uint32_t tid = threadIdx.y * POST_BX + threadIdx.x;
  if (tid < 32u) {
    uint32_t run = 0;
    for (uint32_t base = 0; base < n; base += 32u) {
      const uint32_t k = base + tid;
      const uint32_t c = k < n ? post_tiles_of<SF>(posts[views[k]]) : 0u;
      uint32_t incl = c;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (tid >= (uint32_t)o)
          incl += y;
      }
      if (k < n)
        s_pre[k] = run + incl - c;
      run += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (tid == 0)
      s_pre[n] = run;
  }
  __syncthreads();
  const uint32_t total = s_pre[n];
  uint32_t k = 0;
  for (uint32_t u = blockIdx.x; u < total; u += gridDim.x) {
    while (s_pre[k + 1] <= u)
      k++;
    const PostArgs &p = posts[views[k]];
    const uint32_t local = u - s_pre[k];
    const uint32_t tx = ((uint32_t)(p.width / SF) + POST_BX - 1u) / POST_BX;
    post_load_luts<SF>(p, sm);
    post_tile<SF>(p, sm, (int)(local % tx), (int)(local / tx));
  }
}

static int resident_blocks(const void *fn, int block) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, block, 0) != cudaSuccess) {
    cudaGetLastError();
    nb = 1;
  }
  return nb > 0 ? nb : 1;
}

void mopcuda_batch_grids(BatchLaunch &cfg) {
  const int sms = cfg.num_sms > 0 ? cfg.num_sms : 148;
  const int gm = cfg.grid_mul > 0 ? cfg.grid_mul : 1;
  auto grid = [&](const void *fn, int block) { return sms * resident_blocks(fn, block) * gm; };
  cfg.grid_vertex = grid((const void *)k_b_items<ST_VERTEX, false>, cfg.vertex_block);
  cfg.grid_setup = grid((const void *)k_b_items<ST_SETUP, false>, cfg.setup_block);
  cfg.grid_clip = grid((const void *)k_b_items<ST_CLIP, false>, 128);
  cfg.grid_rsmall = grid((const void *)k_b_items<ST_RSMALL, false>, cfg.raster_block);
  cfg.grid_rlarge = grid((const void *)k_b_items<ST_RLARGE, false>, cfg.large_block);
  cfg.grid_shade = grid((const void *)k_b_shade<false>, cfg.shade_block);
}

int mopcuda_launch_batch(const BatchArgs &b, const PostArgs *posts, const uint32_t *post_views[4],
                         const uint32_t post_count[4], const uint32_t post_tiles[4],
                         const BatchLaunch &cfg, bool shared_lights, bool shadows, bool ordered,
                         cudaStream_t s, int parts) {
  if (b.nv == 0)
    return 0;
  int launches = 0;
  const int sms = cfg.num_sms > 0 ? cfg.num_sms : 148;
  const uint32_t nv = b.nv;
  const FrameArgs *fr = b.frames;
  if (parts & BATCH_PART_MAIN) {
    k_batch_prepare<<<nv, 256, 0, s>>>(b);
    k_batch_alloc<<<1, 256, 0, s>>>(b);
    k_b_items<ST_VERTEX, false><<<cfg.grid_vertex, cfg.vertex_block, 0, s>>>(fr, nv);
    /* setup (flat colours), clipping and shading read a scene's shadow map
     * when any scene of the launch has one */
    if (shadows) {
      k_b_items<ST_SETUP, true><<<cfg.grid_setup, cfg.setup_block, 0, s>>>(fr, nv);
      k_b_items<ST_CLIP, true><<<cfg.grid_clip, 128, 0, s>>>(fr, nv);
    } else {
      k_b_items<ST_SETUP, false><<<cfg.grid_setup, cfg.setup_block, 0, s>>>(fr, nv);
      k_b_items<ST_CLIP, false><<<cfg.grid_clip, 128, 0, s>>>(fr, nv);
    }
    k_b_items<ST_RSMALL, false><<<cfg.grid_rsmall, cfg.raster_block, 0, s>>>(fr, nv);
    k_b_items<ST_RLARGE, false><<<cfg.grid_rlarge, cfg.large_block, 0, s>>>(fr, nv);
    k_b_resolve<<<sms * 8, 256, 0, s>>>(fr, nv);
    if (shadows)
      k_b_shade<true><<<cfg.grid_shade, cfg.shade_block, 0, s>>>(fr, nv, shared_lights ? 1 : 0);
    else
      k_b_shade<false><<<cfg.grid_shade, cfg.shade_block, 0, s>>>(fr, nv, shared_lights ? 1 : 0);
    launches += 9;
    if (ordered && b.hdr) {
      cudaMemsetAsync(b.frag_head, 0xff, sizeof(uint32_t) * (size_t)b.samples, s);
      k_b_ocount<<<sms * 8, 256, 0, s>>>(fr, nv);
      k_b_oscan<<<nv, 1024, 0, s>>>(fr);
      k_b_oraster<<<sms * 8, 256, 0, s>>>(fr, nv);
      launches += 4;
      if (b.wlist) { /* some viewport has wireframe draws */
        k_b_wcount<<<sms * 8, 256, 0, s>>>(fr, nv);
        k_b_wscan<<<nv, 1024, 0, s>>>(fr);
        k_b_wplot<<<sms * 8, 256, 0, s>>>(fr, nv);
        launches += 3;
        if (shadows)
          k_b_ofold<true, true><<<sms * 8, 128, 0, s>>>(fr, nv);
        else
          k_b_ofold<false, true><<<sms * 8, 128, 0, s>>>(fr, nv);
      } else if (shadows) {
        k_b_ofold<true, false><<<sms * 8, 128, 0, s>>>(fr, nv);
      } else {
        k_b_ofold<false, false><<<sms * 8, 128, 0, s>>>(fr, nv);
      }
    }
  }
  if (!(parts & BATCH_PART_POST))
    return launches;
  dim3 pb(POST_BX, POST_BY);
  for (int k = 0; k < 4; k++) {
    if (!post_count[k] || !post_tiles[k])
      continue;
    const uint32_t g = post_tiles[k] < (uint32_t)(sms * 16) ? post_tiles[k] : (uint32_t)(sms * 16);
    switch (k + 1) {
    case 1:
      k_b_post<1><<<g, pb, 0, s>>>(posts, post_views[k], post_count[k]);
      break;
    case 2:
      k_b_post<2><<<g, pb, 0, s>>>(posts, post_views[k], post_count[k]);
      break;
    case 3:
      k_b_post<3><<<g, pb, 0, s>>>(posts, post_views[k], post_count[k]);
      break;
    default:
      k_b_post<4><<<g, pb, 0, s>>>(posts, post_views[k], post_count[k]);
      break;
    }
    launches++;
  }
  return launches;
}

/* ========================================================================
 * Vertex deformation: mop_skin_apply / mop_morph_apply on the device
 * (reference src/core/viewport.c:1572-1680, 1763-1804).  One thread per
 * vertex copies the bind-pose vertex and rewrites position (and normal), in
 * the reference's operation order.
 * ======================================================================== */
__device__ __forceinline__ void copy_vertex(const uint8_t *src, uint8_t *dst, uint32_t stride) {
  const uint32_t *s = reinterpret_cast<const uint32_t *>(src);
  uint32_t *d = reinterpret_cast<uint32_t *>(dst);
  for (uint32_t k = 0; k < stride / 4u; k++)
    d[k] = s[k];
}

#define SKIN_SMEM_BONES 256

__global__ void __launch_bounds__(256) k_skin(const uint8_t *bind, uint8_t *dst, uint32_t vc,
                                              DeformLayout l, const float *bones,
                                              uint32_t bone_count) {
  __shared__ float s_b[SKIN_SMEM_BONES * 16];
  const bool in_smem = bone_count <= SKIN_SMEM_BONES;
  if (in_smem) {
    for (uint32_t i = threadIdx.x; i < bone_count * 16u; i += blockDim.x)
      s_b[i] = bones[i];
    __syncthreads();
  }
  const float *B = in_smem ? s_b : bones;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < vc; v += gridDim.x * blockDim.x) {
    const uint8_t *vert = bind + (size_t)v * l.stride;
    uint8_t *out = dst + (size_t)v * l.stride;
    copy_vertex(vert, out, l.stride);
    const uint8_t *jd = vert + l.joints_offset;
    const uint8_t j[4] = {jd[0], jd[1], jd[2], jd[3]};
    const float *wd = reinterpret_cast<const float *>(vert + l.weights_offset);
    const float w[4] = {wd[0], wd[1], wd[2], wd[3]};
    const float *pd = reinterpret_cast<const float *>(vert + l.position_offset);
    const float px = pd[0], py = pd[1], pz = pd[2];
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (int b = 0; b < 4; b++) {
      if (w[b] <= 0.0f || j[b] >= bone_count)
        continue;
      const float *m = B + 16u * j[b];
      const float rx = m[0] * px + m[4] * py + m[8] * pz + m[12];
      const float ry = m[1] * px + m[5] * py + m[9] * pz + m[13];
      const float rz = m[2] * px + m[6] * py + m[10] * pz + m[14];
      sx += w[b] * rx;
      sy += w[b] * ry;
      sz += w[b] * rz;
    }
    float *op = reinterpret_cast<float *>(out + l.position_offset);
    op[0] = sx;
    op[1] = sy;
    op[2] = sz;
    if (l.normal_offset >= 0) {
      const float *nd = reinterpret_cast<const float *>(vert + l.normal_offset);
      const float nx = nd[0], ny = nd[1], nz = nd[2];
      float snx = 0.0f, sny = 0.0f, snz = 0.0f;
      for (int b = 0; b < 4; b++) {
        if (w[b] <= 0.0f || j[b] >= bone_count)
          continue;
        const float *m = B + 16u * j[b];
        const float rx = m[0] * nx + m[4] * ny + m[8] * nz;
        const float ry = m[1] * nx + m[5] * ny + m[9] * nz;
        const float rz = m[2] * nx + m[6] * ny + m[10] * nz;
        snx += w[b] * rx;
        sny += w[b] * ry;
        snz += w[b] * rz;
      }
      const float len = sqrtf(snx * snx + sny * sny + snz * snz);
      if (len > 1e-8f) {
        snx /= len;
        sny /= len;
        snz /= len;
      }
      float *on = reinterpret_cast<float *>(out + l.normal_offset);
      on[0] = snx;
      on[1] = sny;
      on[2] = snz;
    }
  }
}

#define MORPH_SMEM_WEIGHTS 1024

__global__ void __launch_bounds__(256) k_morph(const uint8_t *bind, uint8_t *dst, uint32_t vc,
                                               DeformLayout l, const float *targets,
                                               const float *weights, uint32_t tc) {
  __shared__ float s_w[MORPH_SMEM_WEIGHTS];
  const bool in_smem = tc <= MORPH_SMEM_WEIGHTS;
  if (in_smem) {
    for (uint32_t i = threadIdx.x; i < tc; i += blockDim.x)
      s_w[i] = weights[i];
    __syncthreads();
  }
  const float *W = in_smem ? s_w : weights;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < vc; v += gridDim.x * blockDim.x) {
    const uint8_t *vert = bind + (size_t)v * l.stride;
    uint8_t *out = dst + (size_t)v * l.stride;
    copy_vertex(vert, out, l.stride);
    const float *pd = reinterpret_cast<const float *>(vert + l.position_offset);
    float p0 = pd[0], p1 = pd[1], p2 = pd[2];
    for (uint32_t t = 0; t < tc; t++) { /* targets in order, as the reference's outer loop */
      const float w = W[t];
      if (w == 0.0f)
        continue;
      const float *d = targets + ((size_t)t * vc + v) * 3u;
      p0 += w * d[0];
      p1 += w * d[1];
      p2 += w * d[2];
    }
    float *op = reinterpret_cast<float *>(out + l.position_offset);
    op[0] = p0;
    op[1] = p1;
    op[2] = p2;
  }
}

int mopcuda_launch_skin(const uint8_t *bind, uint8_t *dst, uint32_t vc, const DeformLayout &l,
                        const float *bones, uint32_t bone_count, int num_sms, cudaStream_t s) {
  if (!vc)
    return 0;
  const uint32_t g = blocks_for(vc, 256);
  const uint32_t cap = (uint32_t)num_sms * 8u;
  k_skin<<<g < cap ? g : cap, 256, 0, s>>>(bind, dst, vc, l, bones, bone_count);
  return 1;
}

int mopcuda_launch_morph(const uint8_t *bind, uint8_t *dst, uint32_t vc, const DeformLayout &l,
                         const float *targets, const float *weights, uint32_t tc, int num_sms,
                         cudaStream_t s) {
  if (!vc)
    return 0;
  const uint32_t g = blocks_for(vc, 256);
  const uint32_t cap = (uint32_t)num_sms * 8u;
  k_morph<<<g < cap ? g : cap, 256, 0, s>>>(bind, dst, vc, l, targets, weights, tc);
  return 1;
}

/* ------------------------------------------------------------------------
 * shadow pass: depth-only raster of the casters from the light
 * (mop_sw_shadow_render_mesh, rasterizer.c:357-493).  The reference keeps
 * `z < depth ? z : depth` per texel over all triangles in submission order,
 * which is the minimum whatever the order, so texels take an atomicMin of
 * depth_key(z).  The map starts at 0xffffffff (read as 1.0) and only z < 1
 * is written, as the test against a map cleared to 1.0 keeps; -0 and +0
 * share a key and compare equal after the lookup's bias anyway.
 * ------------------------------------------------------------------------ */
#define SHADOW_BLOCK 256

/* Texels [xs, xe] of row y from edge values already stepped to (xs, y).
 * The atomics' results are unused (reductions the thread does not wait on). */
__device__ __forceinline__ void shadow_walk(uint32_t *map, int size, const ShadowRec &r, int y,
                                            int xs, int xe, float w0, float w1, float w2) {
  uint32_t *row = map + (size_t)y * (size_t)size;
  bool seen = false;
  for (int x = xs; x <= xe; x++) {
    if (w0 >= 0.0f && w1 >= 0.0f && w2 >= 0.0f) {
      seen = true;
      const float b0 = w0 * r.inv_area, b1 = w1 * r.inv_area, b2 = w2 * r.inv_area;
      const float z = b0 * r.sz[0] + b1 * r.sz[1] + b2 * r.sz[2];
      if (z < 1.0f)
        atomicMin(row + x, depth_key(z));
    } else if (seen) {
      break; /* edge values are monotone along a row: coverage has ended */
    }
    w0 = __fadd_rn(w0, r.dx[0]);
    w1 = __fadd_rn(w1, r.dx[1]);
    w2 = __fadd_rn(w2, r.dx[2]);
  }
}

/* One thread per caster triangle: the reference's per-triangle front end
 * (trivial reject, w guard, divide, window map, clamped bbox, area, edges
 * flipped to positive winding, values at the bbox corner), then either the
 * whole bbox walked here (at most small_area texels) or a record queued for
 * the item-parallel walk. */
__global__ void __launch_bounds__(SHADOW_BLOCK) k_shadow_tri(ShadowArgs s) {
  const float half = (float)s.size * 0.5f;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < s.tri_total;
       t += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = s.draw_count; /* last caster with tri_off <= t */
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (s.draws[mid].tri_off <= t)
        lo = mid;
      else
        hi = mid;
    }
    const ShadowDraw &d = s.draws[lo];
    const size_t i3 = 3u * (size_t)(t - d.tri_off);
    const uint32_t i0 = d.idx[i3], i1 = d.idx[i3 + 1], i2 = d.idx[i3 + 2];
    if (i0 >= d.vertex_count || i1 >= d.vertex_count || i2 >= d.vertex_count)
      continue;
    const float *p0 = reinterpret_cast<const float *>(d.verts + (size_t)i0 * d.stride);
    const float *p1 = reinterpret_cast<const float *>(d.verts + (size_t)i1 * d.stride);
    const float *p2 = reinterpret_cast<const float *>(d.verts + (size_t)i2 * d.stride);
    const float4 c0 = xform(d.mvp, p0[0], p0[1], p0[2], 1.0f);
    const float4 c1 = xform(d.mvp, p1[0], p1[1], p1[2], 1.0f);
    const float4 c2 = xform(d.mvp, p2[0], p2[1], p2[2], 1.0f);
    if ((c0.x < -c0.w && c1.x < -c1.w && c2.x < -c2.w) ||
        (c0.x > c0.w && c1.x > c1.w && c2.x > c2.w) ||
        (c0.y < -c0.w && c1.y < -c1.w && c2.y < -c2.w) ||
        (c0.y > c0.w && c1.y > c1.w && c2.y > c2.w) ||
        (c0.z < -c0.w && c1.z < -c1.w && c2.z < -c2.w) ||
        (c0.z > c0.w && c1.z > c1.w && c2.z > c2.w))
      continue;
    if (c0.w <= 1e-6f || c1.w <= 1e-6f || c2.w <= 1e-6f)
      continue;
    const float inv0 = 1.0f / c0.w, inv1 = 1.0f / c1.w, inv2 = 1.0f / c2.w;
    const float sx0 = (c0.x * inv0 + 1.0f) * half, sy0 = (1.0f - c0.y * inv0) * half;
    const float sx1 = (c1.x * inv1 + 1.0f) * half, sy1 = (1.0f - c1.y * inv1) * half;
    const float sx2 = (c2.x * inv2 + 1.0f) * half, sy2 = (1.0f - c2.y * inv2) * half;
    ShadowRec r;
    r.sz[0] = (c0.z * inv0 + 1.0f) * 0.5f;
    r.sz[1] = (c1.z * inv1 + 1.0f) * 0.5f;
    r.sz[2] = (c2.z * inv2 + 1.0f) * 0.5f;
    /* bbox by the reference's compare-and-replace sequence (NaN keeps the
     * first operand, unlike fminf) */
    float fmin_x = sx0, fmin_y = sy0, fmax_x = sx0, fmax_y = sy0;
    if (sx1 < fmin_x)
      fmin_x = sx1;
    if (sx1 > fmax_x)
      fmax_x = sx1;
    if (sx2 < fmin_x)
      fmin_x = sx2;
    if (sx2 > fmax_x)
      fmax_x = sx2;
    if (sy1 < fmin_y)
      fmin_y = sy1;
    if (sy1 > fmax_y)
      fmax_y = sy1;
    if (sy2 < fmin_y)
      fmin_y = sy2;
    if (sy2 > fmax_y)
      fmax_y = sy2;
    int min_x = x86_f2i(floorf(fmin_x)), min_y = x86_f2i(floorf(fmin_y));
    int max_x = x86_f2i(ceilf(fmax_x)), max_y = x86_f2i(ceilf(fmax_y));
    if (min_x < 0)
      min_x = 0;
    if (min_y < 0)
      min_y = 0;
    if (max_x >= s.size)
      max_x = s.size - 1;
    if (max_y >= s.size)
      max_y = s.size - 1;
    if (min_x > max_x || min_y > max_y)
      continue;
    const float area = (sx1 - sx0) * (sy2 - sy0) - (sx2 - sx0) * (sy1 - sy0);
    if (fabsf(area) < 1e-6f)
      continue;
    r.inv_area = 1.0f / fabsf(area);
    r.dx[0] = sy1 - sy2;
    r.dy[0] = sx2 - sx1;
    r.dx[1] = sy2 - sy0;
    r.dy[1] = sx0 - sx2;
    r.dx[2] = sy0 - sy1;
    r.dy[2] = sx1 - sx0;
    const float px0 = (float)min_x + 0.5f, py0 = (float)min_y + 0.5f;
    r.w[0] = (sx2 - sx1) * (py0 - sy1) - (sy2 - sy1) * (px0 - sx1);
    r.w[1] = (sx0 - sx2) * (py0 - sy2) - (sy0 - sy2) * (px0 - sx2);
    r.w[2] = (sx1 - sx0) * (py0 - sy0) - (sy1 - sy0) * (px0 - sx0);
    if (area < 0.0f) {
      for (int k = 0; k < 3; k++) {
        r.dx[k] = -r.dx[k];
        r.dy[k] = -r.dy[k];
        r.w[k] = -r.w[k];
      }
    }
    const uint32_t bw = (uint32_t)(max_x - min_x + 1), bh = (uint32_t)(max_y - min_y + 1);
    if (bw * bh <= (uint32_t)s.small_area) {
      float w0 = r.w[0], w1 = r.w[1], w2 = r.w[2];
      for (int y = min_y; y <= max_y; y++) {
        shadow_walk(s.map, s.size, r, y, min_x, max_x, w0, w1, w2);
        w0 = __fadd_rn(w0, r.dy[0]);
        w1 = __fadd_rn(w1, r.dy[1]);
        w2 = __fadd_rn(w2, r.dy[2]);
      }
    } else {
      r.x0y0 = (uint32_t)min_x | ((uint32_t)min_y << 16);
      r.x1y1 = (uint32_t)max_x | ((uint32_t)max_y << 16);
      r.pad = 0;
      const uint32_t slot = atomicAdd(&s.ctr->recs, 1u); /* < tri_total: one per triangle */
      s.recs[slot] = r;
      s.items[slot] = bw <= (uint32_t)SHADOW_SEG ? (bh + 31u) / 32u : bh;
    }
  }
}

__global__ void __launch_bounds__(1024) k_shadow_scan(ShadowArgs s) {
  __shared__ unsigned long long part[32];
  items_scan_block(s.items, s.ctr->recs, &s.ctr->items, part);
}

/* The queued records, one warp per item, in two shapes:
 *  - narrow records (bbox at most SHADOW_SEG texels wide): an item is a band
 *    of 32 rows, one lane per row; lanes 0-2 fold one edge each to the band's
 *    first row (the long folds, once per band), every lane folds on to its
 *    own row (at most 16 + 15 predicated additions) and walks it texel by
 *    texel exactly as the reference's row loop steps;
 *  - wide records: an item is one row; lanes 0-2 fold one edge each to the
 *    row start and step along the row as the reference does, keeping the
 *    value at every 32-texel chunk start in shared memory (32 chunks at a
 *    time); each lane then walks one chunk from its start.
 * A walk ends where its coverage ends. */
__device__ __forceinline__ void shadow_span(uint32_t *row, const ShadowRec &r, int xs, int xe,
                                            float w0, float w1, float w2) {
  bool seen = false;
  for (int x = xs; x <= xe; x++) {
    if (w0 >= 0.0f && w1 >= 0.0f && w2 >= 0.0f) {
      seen = true;
      const float b0 = w0 * r.inv_area, b1 = w1 * r.inv_area, b2 = w2 * r.inv_area;
      const float z = b0 * r.sz[0] + b1 * r.sz[1] + b2 * r.sz[2];
      if (z < 1.0f)
        atomicMin(row + x, depth_key(z));
    } else if (seen) {
      break; /* edge values are monotone along a row: coverage has ended */
    }
    w0 = __fadd_rn(w0, r.dx[0]);
    w1 = __fadd_rn(w1, r.dx[1]);
    w2 = __fadd_rn(w2, r.dx[2]);
  }
}

__global__ void __launch_bounds__(SHADOW_BLOCK) k_shadow_large(ShadowArgs s) {
  __shared__ float s_cs[SHADOW_BLOCK / 32][3][32];
  const unsigned long long total = s.ctr->items;
  const uint32_t n = s.ctr->recs;
  const uint32_t lane = threadIdx.x & 31u;
  float(*cs)[32] = s_cs[threadIdx.x >> 5];
  const int k1 = lane < 16u ? (int)lane : 16, k2 = (int)lane - k1;
  const unsigned long long wpb = blockDim.x >> 5;
  for (unsigned long long it = blockIdx.x * wpb + (threadIdx.x >> 5); it < total;
       it += gridDim.x * wpb) {
    /* last record with offset <= it: a 32-way search, one candidate per lane
     * (the offsets increase strictly, so the lanes that pass form a prefix) */
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
      const uint32_t step = (hi - lo + 31u) >> 5;
      const uint32_t cand = lo + lane * step;
      const bool le = cand < hi && s.items[cand] <= it;
      const uint32_t pass = __ballot_sync(0xffffffffu, le);
      lo += (uint32_t)(31 - __clz(pass)) * step;
      hi = min(hi, lo + step);
    }
    const ShadowRec r = s.recs[lo];
    const int x0 = (int)(r.x0y0 & 0xffffu), y0 = (int)(r.x0y0 >> 16);
    const int x1 = (int)(r.x1y1 & 0xffffu), y1 = (int)(r.x1y1 >> 16);
    const int local = (int)(it - s.items[lo]);
    const float e_w = lane == 0u ? r.w[0] : (lane == 1u ? r.w[1] : r.w[2]);
    const float e_dx = lane == 0u ? r.dx[0] : (lane == 1u ? r.dx[1] : r.dx[2]);
    const float e_dy = lane == 0u ? r.dy[0] : (lane == 1u ? r.dy[1] : r.dy[2]);
    if (x1 - x0 < SHADOW_SEG) {
      const int band = local * 32;
      const float wb = lane < 3u ? fold_add(e_w, e_dy, band) : 0.0f;
      float w[3];
      for (int e = 0; e < 3; e++) {
        w[e] = __shfl_sync(0xffffffffu, wb, e);
        w[e] = fold_add(fold_add(w[e], r.dy[e], k1), r.dy[e], k2);
      }
      const int y = y0 + band + (int)lane;
      if (y <= y1)
        shadow_span(s.map + (size_t)y * (size_t)s.size, r, x0, x1, w[0], w[1], w[2]);
    } else {
      uint32_t *row = s.map + (size_t)(y0 + local) * (size_t)s.size;
      float v = lane < 3u ? fold_add(e_w, e_dy, local) : 0.0f;
      for (int xw = x0; xw <= x1; xw += 32 * RASTER_CHUNK) { /* 32 chunks per window */
        if (lane < 3u) {
          for (int c = 0; c < 32; c++) {
            cs[lane][c] = v;
#pragma unroll
            for (int k = 0; k < RASTER_CHUNK; k++)
              v = __fadd_rn(v, e_dx);
          }
        }
        __syncwarp();
        const int xs = xw + (int)lane * RASTER_CHUNK;
        if (xs <= x1)
          shadow_span(row, r, xs, min(x1, xs + RASTER_CHUNK - 1), cs[0][lane], cs[1][lane],
                      cs[2][lane]);
        __syncwarp(); /* starts read before lanes 0-2 write the next window */
      }
    }
  }
}

int mopcuda_launch_shadow(const ShadowArgs &s, cudaStream_t st) {
  if (!s.tri_total)
    return 0;
  const uint32_t cap = (uint32_t)s.num_sms * 8u;
  const uint32_t g = blocks_for(s.tri_total, SHADOW_BLOCK);
  k_shadow_tri<<<g < cap ? g : cap, SHADOW_BLOCK, 0, st>>>(s);
  k_shadow_scan<<<1, 1024, 0, st>>>(s);
  k_shadow_large<<<cap, SHADOW_BLOCK, 0, st>>>(s);
  return 3;
}
