/*
 * scene_file.cu — .mop v2 scene files loaded straight into device memory
 * (reference src/loader/mop_scene.c, include/mop/loader/mop_scene.h).
 *
 * The file is mapped read-only and checked as mop_scene_load does (magic
 * 0x4D4F5002, version 2, at most 256 sections, the table of contents inside
 * the file).  A mesh section is copied to the device as stored — quantized
 * or 48-byte raw vertices, 16- or 32-bit indices, so a quantized scene moves
 * 2.7x fewer vertex bytes over PCIe — and decoded there into a
 * MopVertex buffer and a 32-bit index buffer.  (MopQuantizedVertex is 18
 * bytes as laid out by the compiler — 3 + 2 + 2 + 2 halfwords — although the
 * reference header calls it 20.)  The decode is
 * dequantize_vertex / oct_decode (mop_scene.c:142-223) operation for
 * operation: integer-to-float conversions, divisions by 65535 / 32767 / 255,
 * one square root, all correctly rounded, so the buffers are byte-identical
 * to mop_scene_get_mesh's host arrays.
 *
 * Stricter than the reference: a mesh section whose header counts do not fit
 * its size is rejected (mop_scene_get_mesh reads past it).
 */
#include "api_internal.h"

#include <fcntl.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace {

constexpr uint32_t SCENE_MAGIC = 0x4D4F5002u;
constexpr uint32_t SCENE_VERSION = 2u;
constexpr uint32_t MAX_SECTIONS = 256u;
constexpr uint32_t SECTION_MESH = 1, SECTION_CAMERA = 2, SECTION_LIGHT = 3;
constexpr uint32_t VTX_QUANTIZED = 1;
constexpr uint32_t QVERTEX_BYTES = 18; /* sizeof(MopQuantizedVertex) */

struct TocEntry { /* MopSceneTocEntry, 24 bytes */
  uint32_t type, flags;
  uint64_t offset, size;
};
static_assert(sizeof(TocEntry) == 24, "TOC entry layout");

struct MeshHeader { /* MopMeshSectionHeader, 48 bytes */
  uint32_t vertex_count, index_count, vertex_encoding, index_size;
  float bbox_min[3], bbox_max[3];
  uint8_t pad[8];
};
static_assert(sizeof(MeshHeader) == 48, "mesh section header layout");

struct CameraSection { /* MopCameraSection, 56 bytes */
  float eye[3], target[3], up[3];
  float fov_radians, near_plane, far_plane, aspect_ratio;
  uint8_t pad[4];
};

struct LightSection { /* MopLightSection, 64 bytes */
  uint32_t type;
  float position[3], direction[3], color[4];
  float intensity, range, spot_inner_cos, spot_outer_cos;
  uint8_t pad[4];
};

uint64_t align8(uint64_t v) { return (v + 7u) & ~(uint64_t)7u; }
uint64_t align256(uint64_t v) { return (v + 255u) & ~(uint64_t)255u; }

/* dequantize_vertex + oct_decode, mop_scene.c:142-223: one thread per
 * vertex; q holds 18-byte records (9 halfwords: position x3, octahedral
 * normal x2, RGBA8, uv x2). */
__global__ void __launch_bounds__(256) k_mop_dequantize(const uint16_t *__restrict__ q,
                                                       uint32_t n, float bx0, float by0,
                                                       float bz0, float bx1, float by1,
                                                       float bz1, float *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const uint16_t *w = q + (size_t)i * 9u;
  const uint32_t p0 = w[0], p1 = w[1], p2 = w[2];
  const int16_t n0 = (int16_t)w[3], n1 = (int16_t)w[4];
  const uint32_t c0 = w[5] & 0xffu, c1 = w[5] >> 8, c2 = w[6] & 0xffu, c3 = w[6] >> 8;
  const uint32_t u0 = w[7], u1 = w[8];
  float v[12];
  v[0] = bx0 + ((float)p0 / 65535.0f) * (bx1 - bx0);
  v[1] = by0 + ((float)p1 / 65535.0f) * (by1 - by0);
  v[2] = bz0 + ((float)p2 / 65535.0f) * (bz1 - bz0);
  float ox = (float)n0 / 32767.0f, oy = (float)n1 / 32767.0f;
  float nz = 1.0f - fabsf(ox) - fabsf(oy);
  if (nz < 0.0f) {
    const float tx = (1.0f - fabsf(oy)) * (ox >= 0.0f ? 1.0f : -1.0f);
    const float ty = (1.0f - fabsf(ox)) * (oy >= 0.0f ? 1.0f : -1.0f);
    ox = tx;
    oy = ty;
  }
  float nx = ox, ny = oy;
  const float len = sqrtf(nx * nx + ny * ny + nz * nz);
  if (len > 1e-8f) {
    nx /= len;
    ny /= len;
    nz /= len;
  }
  v[3] = nx;
  v[4] = ny;
  v[5] = nz;
  v[6] = (float)c0 / 255.0f;
  v[7] = (float)c1 / 255.0f;
  v[8] = (float)c2 / 255.0f;
  v[9] = (float)c3 / 255.0f;
  v[10] = (float)u0 / 65535.0f;
  v[11] = (float)u1 / 65535.0f;
  float4 *o = reinterpret_cast<float4 *>(out + (size_t)i * 12u);
  o[0] = make_float4(v[0], v[1], v[2], v[3]);
  o[1] = make_float4(v[4], v[5], v[6], v[7]);
  o[2] = make_float4(v[8], v[9], v[10], v[11]);
}

/* 16-bit indices widened to 32 bits (mop_scene.c:460-464). */
__global__ void __launch_bounds__(256) k_mop_widen(const uint16_t *__restrict__ in, uint32_t n,
                                                  uint32_t *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    out[i] = in[i];
}

/* One mesh of a whole-file upload: where its stored bytes sit in the
 * staging copy and its decoded buffers in the slab. */
struct DecodeMesh {
  uint64_t src_v, src_i; /* staging byte offsets of the vertex / index payloads */
  uint64_t dst_v, dst_i; /* slab byte offsets (256-aligned) */
  uint32_t vc, ic, quant, idx16;
  uint32_t v_base, i_base; /* first vertex / index of the mesh in the file order */
  float bmin[3], bmax[3];
};

__device__ __forceinline__ uint32_t mesh_of(const DecodeMesh *m, uint32_t n, uint32_t g,
                                            bool by_index) {
  uint32_t lo = 0, hi = n; /* last mesh whose base <= g */
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if ((by_index ? m[mid].i_base : m[mid].v_base) <= g)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

/* Every vertex of the file: dequantized (the same arithmetic as
 * k_mop_dequantize) or copied. */
__global__ void __launch_bounds__(256) k_mop_decode_all(const uint8_t *__restrict__ stage,
                                                       uint8_t *__restrict__ slab,
                                                       const DecodeMesh *__restrict__ m,
                                                       uint32_t n, uint32_t total) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += gridDim.x * blockDim.x) {
    const DecodeMesh &d = m[mesh_of(m, n, g, false)];
    const uint32_t k = g - d.v_base;
    float *o = reinterpret_cast<float *>(slab + d.dst_v) + (size_t)k * 12u;
    if (!d.quant) {
      const float *src = reinterpret_cast<const float *>(stage + d.src_v) + (size_t)k * 12u;
      float4 *o4 = reinterpret_cast<float4 *>(o);
      o4[0] = make_float4(src[0], src[1], src[2], src[3]);
      o4[1] = make_float4(src[4], src[5], src[6], src[7]);
      o4[2] = make_float4(src[8], src[9], src[10], src[11]);
      continue;
    }
    const uint16_t *w = reinterpret_cast<const uint16_t *>(stage + d.src_v) + (size_t)k * 9u;
    const uint32_t p0 = w[0], p1 = w[1], p2 = w[2];
    const int16_t n0 = (int16_t)w[3], n1 = (int16_t)w[4];
    const uint32_t c0 = w[5] & 0xffu, c1 = w[5] >> 8, c2 = w[6] & 0xffu, c3 = w[6] >> 8;
    const uint32_t u0 = w[7], u1 = w[8];
    const float px = d.bmin[0] + ((float)p0 / 65535.0f) * (d.bmax[0] - d.bmin[0]);
    const float py = d.bmin[1] + ((float)p1 / 65535.0f) * (d.bmax[1] - d.bmin[1]);
    const float pz = d.bmin[2] + ((float)p2 / 65535.0f) * (d.bmax[2] - d.bmin[2]);
    float ox = (float)n0 / 32767.0f, oy = (float)n1 / 32767.0f;
    float nz = 1.0f - fabsf(ox) - fabsf(oy);
    if (nz < 0.0f) {
      const float tx = (1.0f - fabsf(oy)) * (ox >= 0.0f ? 1.0f : -1.0f);
      const float ty = (1.0f - fabsf(ox)) * (oy >= 0.0f ? 1.0f : -1.0f);
      ox = tx;
      oy = ty;
    }
    float nx = ox, ny = oy;
    const float len = sqrtf(nx * nx + ny * ny + nz * nz);
    if (len > 1e-8f) {
      nx /= len;
      ny /= len;
      nz /= len;
    }
    float4 *o4 = reinterpret_cast<float4 *>(o);
    o4[0] = make_float4(px, py, pz, nx);
    o4[1] = make_float4(ny, nz, (float)c0 / 255.0f, (float)c1 / 255.0f);
    o4[2] = make_float4((float)c2 / 255.0f, (float)c3 / 255.0f, (float)u0 / 65535.0f,
                        (float)u1 / 65535.0f);
  }
}

/* Every index of the file, widened to 32 bits where stored as 16. */
__global__ void __launch_bounds__(256) k_mop_indices_all(const uint8_t *__restrict__ stage,
                                                        uint8_t *__restrict__ slab,
                                                        const DecodeMesh *__restrict__ m,
                                                        uint32_t n, uint32_t total) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += gridDim.x * blockDim.x) {
    const DecodeMesh &d = m[mesh_of(m, n, g, true)];
    const uint32_t k = g - d.i_base;
    uint32_t *o = reinterpret_cast<uint32_t *>(slab + d.dst_i) + k;
    *o = d.idx16 ? (uint32_t)reinterpret_cast<const uint16_t *>(stage + d.src_i)[k]
                 : reinterpret_cast<const uint32_t *>(stage + d.src_i)[k];
  }
}

} // namespace

struct MopCudaSceneFile {
  const uint8_t *data = nullptr;
  size_t size = 0;
  uint32_t flags = 0;
  std::vector<TocEntry> toc;
};

extern "C" MopCudaSceneFile *mopcuda_scene_file_open(const char *path) {
  if (!path) {
    fail(MOPCUDA_EINVAL, "scene_file_open: no path");
    return nullptr;
  }
  const int fd = open(path, O_RDONLY);
  if (fd < 0) {
    fail(MOPCUDA_EINVAL, "scene_file_open: cannot open '%s'", path);
    return nullptr;
  }
  struct stat st;
  if (fstat(fd, &st) < 0 || st.st_size < 64) {
    close(fd);
    fail(MOPCUDA_EINVAL, "scene_file_open: '%s' is smaller than the 64-byte header", path);
    return nullptr;
  }
  const size_t size = (size_t)st.st_size;
  void *m = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
  close(fd);
  if (m == MAP_FAILED) {
    fail(MOPCUDA_EINVAL, "scene_file_open: mmap of '%s' failed", path);
    return nullptr;
  }
  const uint8_t *d = (const uint8_t *)m;
  uint32_t hdr[4];
  memcpy(hdr, d, sizeof hdr);
  const char *why = nullptr;
  if (hdr[0] != SCENE_MAGIC)
    why = "bad magic";
  else if (hdr[1] != SCENE_VERSION)
    why = "unsupported version";
  else if (hdr[2] > MAX_SECTIONS)
    why = "more than 256 sections";
  else if (64 + (uint64_t)hdr[2] * sizeof(TocEntry) > size)
    why = "table of contents beyond the file";
  if (why) {
    munmap(m, size);
    fail(MOPCUDA_EINVAL, "scene_file_open: %s in '%s'", why, path);
    return nullptr;
  }
  MopCudaSceneFile *f = new MopCudaSceneFile();
  f->data = d;
  f->size = size;
  f->flags = hdr[3];
  f->toc.resize(hdr[2]);
  if (hdr[2])
    memcpy(f->toc.data(), d + 64, hdr[2] * sizeof(TocEntry));
  return f;
}

extern "C" void mopcuda_scene_file_close(MopCudaSceneFile *f) {
  if (!f)
    return;
  munmap((void *)f->data, f->size);
  delete f;
}

static const TocEntry *nth_section(const MopCudaSceneFile *f, uint32_t type, uint32_t nth) {
  uint32_t k = 0;
  for (const TocEntry &e : f->toc)
    if (e.type == type && k++ == nth)
      return &e;
  return nullptr;
}

static uint32_t count_sections(const MopCudaSceneFile *f, uint32_t type) {
  uint32_t k = 0;
  for (const TocEntry &e : f->toc)
    k += e.type == type;
  return k;
}

extern "C" uint32_t mopcuda_scene_file_mesh_count(const MopCudaSceneFile *f) {
  return f ? count_sections(f, SECTION_MESH) : 0;
}

extern "C" uint32_t mopcuda_scene_file_light_count(const MopCudaSceneFile *f) {
  return f ? count_sections(f, SECTION_LIGHT) : 0;
}

extern "C" int mopcuda_scene_file_camera(const MopCudaSceneFile *f, float eye[3], float target[3],
                                         float up[3], float *fov_radians, float *near_plane,
                                         float *far_plane) {
  if (!f)
    return fail(MOPCUDA_EINVAL, "scene_file_camera: no file");
  const TocEntry *e = nth_section(f, SECTION_CAMERA, 0);
  if (!e || e->offset + sizeof(CameraSection) > f->size)
    return fail(MOPCUDA_EINVAL, "scene_file_camera: no camera section");
  CameraSection c;
  memcpy(&c, f->data + e->offset, sizeof c);
  if (eye)
    memcpy(eye, c.eye, sizeof c.eye);
  if (target)
    memcpy(target, c.target, sizeof c.target);
  if (up)
    memcpy(up, c.up, sizeof c.up);
  if (fov_radians)
    *fov_radians = c.fov_radians;
  if (near_plane)
    *near_plane = c.near_plane;
  if (far_plane)
    *far_plane = c.far_plane;
  return MOPCUDA_OK;
}

extern "C" int mopcuda_scene_file_light(const MopCudaSceneFile *f, uint32_t idx,
                                        MopCudaLight *out) {
  if (!f || !out)
    return fail(MOPCUDA_EINVAL, "scene_file_light: bad arguments");
  const TocEntry *e = nth_section(f, SECTION_LIGHT, idx);
  if (!e || e->offset + sizeof(LightSection) > f->size)
    return fail(MOPCUDA_EINVAL, "scene_file_light: no light section %u", idx);
  LightSection l;
  memcpy(&l, f->data + e->offset, sizeof l);
  memset(out, 0, sizeof *out);
  out->type = (int32_t)l.type;
  memcpy(out->position, l.position, sizeof l.position);
  memcpy(out->direction, l.direction, sizeof l.direction);
  memcpy(out->color, l.color, sizeof l.color);
  out->intensity = l.intensity;
  out->range = l.range;
  out->spot_inner_cos = l.spot_inner_cos;
  out->spot_outer_cos = l.spot_outer_cos;
  out->active = 1;
  return MOPCUDA_OK;
}

/* Per-mesh uploads carve their two buffers from 64 MiB device chunks: one
 * allocation serves many meshes (a cudaMalloc per buffer took most of a
 * mesh's upload).  A chunk is freed with the last buffer carved from it once
 * a newer chunk has replaced it; a mesh larger than a chunk gets an
 * allocation of its own.  Device lock held. */
constexpr size_t LOAD_CHUNK = 64ull << 20;

static BufferSlab *carve_load(MopCudaDevice *d, size_t bytes, size_t *off) {
  BufferSlab *s = nullptr;
  if (bytes > LOAD_CHUNK || !d->load_chunk || d->load_chunk_used + bytes > LOAD_CHUNK) {
    s = new BufferSlab();
    const size_t n = bytes > LOAD_CHUNK ? bytes : LOAD_CHUNK;
    if (cudaMalloc(&s->d, n) != cudaSuccess) {
      cudaGetLastError();
      delete s;
      return nullptr;
    }
    if (bytes > LOAD_CHUNK) {
      *off = 0;
      return s; /* refs come from its two buffers */
    }
    s->refs = 1; /* the device's hold while it is the current chunk */
    mc_slab_release(d->load_chunk);
    d->load_chunk = s;
    d->load_chunk_used = 0;
  }
  *off = d->load_chunk_used;
  d->load_chunk_used += bytes;
  return d->load_chunk;
}

extern "C" int mopcuda_scene_file_upload_mesh(MopCudaDevice *d, const MopCudaSceneFile *f,
                                              uint32_t idx, uint32_t flags,
                                              MopCudaBuffer **vertices, MopCudaBuffer **indices,
                                              uint32_t *vertex_count, uint32_t *index_count,
                                              float bbox_min[3], float bbox_max[3]) {
  if (!d || !f || !vertices || !indices)
    return fail(MOPCUDA_EINVAL, "scene_file_upload_mesh: bad arguments");
  const TocEntry *e = nth_section(f, SECTION_MESH, idx);
  if (!e)
    return fail(MOPCUDA_EINVAL, "scene_file_upload_mesh: no mesh section %u", idx);
  if (e->offset > f->size || e->size > f->size - e->offset || e->size < sizeof(MeshHeader))
    return fail(MOPCUDA_EINVAL, "scene_file_upload_mesh: section %u out of bounds", idx);
  MeshHeader h;
  memcpy(&h, f->data + e->offset, sizeof h);
  const bool quant = h.vertex_encoding == VTX_QUANTIZED;
  const bool idx16 = h.index_size == 2;
  const uint64_t vtx_bytes = (uint64_t)h.vertex_count * (quant ? QVERTEX_BYTES : 48u);
  const uint64_t idx_bytes = (uint64_t)h.index_count * (idx16 ? 2u : 4u);
  if (sizeof(MeshHeader) + align8(vtx_bytes) + idx_bytes > e->size)
    return fail(MOPCUDA_EINVAL, "scene_file_upload_mesh: section %u shorter than its %u vertices "
                                "and %u indices", idx, h.vertex_count, h.index_count);
  const uint8_t *payload = f->data + e->offset + sizeof(MeshHeader);
  const uint64_t payload_bytes = align8(vtx_bytes) + idx_bytes;
  const size_t out_v = (size_t)h.vertex_count * 48u, out_i = (size_t)h.index_count * 4u;

  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  /* the staging buffers are reused: finish the previous upload first */
  int rc = mc_stream_sync(d, FRAME_TIMEOUT_MS);
  if (rc)
    return rc;
  if (d->h_load.ensure(payload_bytes + 16) || d->load_stage.ensure(payload_bytes + 16))
    return MOPCUDA_ENOMEM;
  MopCudaBuffer *vb = new MopCudaBuffer(), *ib = new MopCudaBuffer();
  vb->size = out_v;
  ib->size = out_i;
  const bool shadow = (flags & MOPCUDA_LOAD_HOST_SHADOW) != 0;
  const size_t span_v = align256(out_v ? out_v : 1), span_i = align256(out_i ? out_i : 1);
  size_t off = 0;
  BufferSlab *slab = carve_load(d, span_v + span_i, &off);
  if (slab) {
    vb->slab = ib->slab = slab;
    slab->refs += 2;
    vb->d = (uint8_t *)slab->d + off;
    ib->d = (uint8_t *)slab->d + off + span_v;
  }
  if (!slab ||
      (shadow && (!(vb->h = malloc(out_v ? out_v : 16)) || !(ib->h = malloc(out_i ? out_i : 16))))) {
    if (slab) {
      mc_slab_release(slab);
      mc_slab_release(slab);
    }
    free(vb->h);
    free(ib->h);
    delete vb;
    delete ib;
    return fail(MOPCUDA_ENOMEM, "scene_file_upload_mesh: allocation of %zu + %zu bytes failed",
                out_v, out_i);
  }
  cudaStream_t st = d->stream;
  memcpy(d->h_load.p, payload, payload_bytes);
  uint8_t *stage = d->load_stage.as<uint8_t>();
  rc = MOPCUDA_OK;
  do {
    if (cudaMemcpyAsync(stage, d->h_load.p, payload_bytes, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
      break;
    const uint32_t nv = h.vertex_count, ni = h.index_count;
    if (quant && nv)
      k_mop_dequantize<<<(nv + 255u) / 256u, 256, 0, st>>>(
          reinterpret_cast<const uint16_t *>(stage), nv, h.bbox_min[0], h.bbox_min[1],
          h.bbox_min[2], h.bbox_max[0], h.bbox_max[1], h.bbox_max[2], (float *)vb->d);
    else if (nv && cudaMemcpyAsync(vb->d, stage, out_v, cudaMemcpyDeviceToDevice, st) !=
                       cudaSuccess)
      break;
    if (idx16 && ni)
      k_mop_widen<<<(ni + 255u) / 256u, 256, 0, st>>>(
          reinterpret_cast<const uint16_t *>(stage + align8(vtx_bytes)), ni, (uint32_t *)ib->d);
    else if (ni && cudaMemcpyAsync(ib->d, stage + align8(vtx_bytes), out_i,
                                   cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      break;
    d->launches += (uint64_t)((quant && nv) ? 1 : 0) + ((idx16 && ni) ? 1 : 0);
    if (cudaGetLastError() != cudaSuccess)
      break;
    if (shadow && ((out_v && cudaMemcpyAsync(vb->h, vb->d, out_v, cudaMemcpyDeviceToHost, st) !=
                                 cudaSuccess) ||
                   (out_i && cudaMemcpyAsync(ib->h, ib->d, out_i, cudaMemcpyDeviceToHost, st) !=
                                 cudaSuccess)))
      break;
    rc = mc_stream_sync(d, FRAME_TIMEOUT_MS);
    if (rc)
      break;
    *vertices = vb;
    *indices = ib;
    if (vertex_count)
      *vertex_count = nv;
    if (index_count)
      *index_count = ni;
    if (bbox_min)
      memcpy(bbox_min, h.bbox_min, sizeof h.bbox_min);
    if (bbox_max)
      memcpy(bbox_max, h.bbox_max, sizeof h.bbox_max);
    return MOPCUDA_OK;
  } while (0);
  const cudaError_t ce = cudaGetLastError();
  mc_stream_sync(d, FRAME_TIMEOUT_MS);
  mc_slab_release(slab);
  mc_slab_release(slab);
  free(vb->h);
  free(ib->h);
  delete vb;
  delete ib;
  return rc ? rc : fail(MOPCUDA_ECUDA, "scene_file_upload_mesh: %s", cudaGetErrorString(ce));
}

extern "C" int mopcuda_scene_file_upload_all(MopCudaDevice *d, const MopCudaSceneFile *f,
                                             uint32_t flags, MopCudaBuffer **vertices,
                                             MopCudaBuffer **indices, uint32_t *vertex_counts,
                                             uint32_t *index_counts) {
  if (!d || !f || !vertices || !indices)
    return fail(MOPCUDA_EINVAL, "scene_file_upload_all: bad arguments");
  /* validate every mesh section and lay out the staging copy and the slab */
  std::vector<DecodeMesh> ms;
  std::vector<const uint8_t *> payload;
  uint64_t stage_bytes = 0, slab_bytes = 0, tv = 0, ti = 0;
  for (uint32_t k = 0; k < count_sections(f, SECTION_MESH); k++) {
    const TocEntry *e = nth_section(f, SECTION_MESH, k);
    if (e->offset > f->size || e->size > f->size - e->offset || e->size < sizeof(MeshHeader))
      return fail(MOPCUDA_EINVAL, "scene_file_upload_all: section %u out of bounds", k);
    MeshHeader h;
    memcpy(&h, f->data + e->offset, sizeof h);
    DecodeMesh m;
    memset(&m, 0, sizeof m);
    m.quant = h.vertex_encoding == VTX_QUANTIZED;
    m.idx16 = h.index_size == 2;
    m.vc = h.vertex_count;
    m.ic = h.index_count;
    const uint64_t vb = (uint64_t)m.vc * (m.quant ? QVERTEX_BYTES : 48u);
    const uint64_t ib = (uint64_t)m.ic * (m.idx16 ? 2u : 4u);
    if (sizeof(MeshHeader) + align8(vb) + ib > e->size)
      return fail(MOPCUDA_EINVAL, "scene_file_upload_all: section %u shorter than its %u "
                                  "vertices and %u indices", k, m.vc, m.ic);
    memcpy(m.bmin, h.bbox_min, sizeof m.bmin);
    memcpy(m.bmax, h.bbox_max, sizeof m.bmax);
    m.src_v = stage_bytes;
    m.src_i = stage_bytes + align8(vb);
    stage_bytes += align8(align8(vb) + ib);
    m.dst_v = slab_bytes;
    slab_bytes += ((uint64_t)m.vc * 48u + 255u) & ~(uint64_t)255u;
    m.dst_i = slab_bytes;
    slab_bytes += ((uint64_t)m.ic * 4u + 255u) & ~(uint64_t)255u;
    m.v_base = (uint32_t)tv;
    m.i_base = (uint32_t)ti;
    tv += m.vc;
    ti += m.ic;
    if (tv >= (1ull << 32) || ti >= (1ull << 32))
      return fail(MOPCUDA_EINVAL, "scene_file_upload_all: more than 2^32 vertices or indices");
    ms.push_back(m);
    payload.push_back(f->data + e->offset + sizeof(MeshHeader));
  }
  const uint32_t n = (uint32_t)ms.size();
  if (!n)
    return MOPCUDA_OK;
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  int rc = mc_stream_sync(d, FRAME_TIMEOUT_MS); /* the staging buffers are reused */
  if (rc)
    return rc;
  const size_t desc_bytes = sizeof(DecodeMesh) * n;
  if (d->h_load.ensure(stage_bytes + desc_bytes + 16) ||
      d->load_stage.ensure(stage_bytes + desc_bytes + 16))
    return MOPCUDA_ENOMEM;
  BufferSlab *slab = new BufferSlab();
  if (cudaMalloc(&slab->d, slab_bytes ? slab_bytes : 256) != cudaSuccess) {
    cudaGetLastError();
    delete slab;
    return fail(MOPCUDA_ENOMEM, "scene_file_upload_all: %llu device bytes",
                (unsigned long long)slab_bytes);
  }
  uint8_t *hs = d->h_load.as<uint8_t>();
  for (uint32_t k = 0; k < n; k++) {
    const DecodeMesh &m = ms[k];
    const uint64_t vb = (uint64_t)m.vc * (m.quant ? QVERTEX_BYTES : 48u);
    const uint64_t ib = (uint64_t)m.ic * (m.idx16 ? 2u : 4u);
    memcpy(hs + m.src_v, payload[k], vb);
    memcpy(hs + m.src_i, payload[k] + align8(vb), ib);
  }
  const size_t desc_off = (size_t)align8(stage_bytes);
  memcpy(hs + desc_off, ms.data(), desc_bytes);
  cudaStream_t st = d->stream;
  uint8_t *stage = d->load_stage.as<uint8_t>();
  const uint32_t grid = (uint32_t)d->num_sms * 8u;
  bool ok = cudaMemcpyAsync(stage, hs, desc_off + desc_bytes, cudaMemcpyHostToDevice, st) ==
            cudaSuccess;
  if (ok) {
    const DecodeMesh *dm = reinterpret_cast<const DecodeMesh *>(stage + desc_off);
    if (tv)
      k_mop_decode_all<<<grid, 256, 0, st>>>(stage, (uint8_t *)slab->d, dm, n, (uint32_t)tv);
    if (ti)
      k_mop_indices_all<<<grid, 256, 0, st>>>(stage, (uint8_t *)slab->d, dm, n, (uint32_t)ti);
    d->launches += (tv ? 1u : 0u) + (ti ? 1u : 0u);
    ok = cudaGetLastError() == cudaSuccess;
  }
  const bool shadow = (flags & MOPCUDA_LOAD_HOST_SHADOW) != 0;
  std::vector<MopCudaBuffer *> made;
  for (uint32_t k = 0; ok && k < n; k++) {
    for (int which = 0; which < 2; which++) {
      MopCudaBuffer *b = new MopCudaBuffer();
      b->size = which ? (size_t)ms[k].ic * 4u : (size_t)ms[k].vc * 48u;
      b->d = (uint8_t *)slab->d + (which ? ms[k].dst_i : ms[k].dst_v);
      b->slab = slab;
      slab->refs++;
      made.push_back(b);
      if (shadow) {
        b->h = malloc(b->size ? b->size : 16);
        if (!b->h || (b->size && cudaMemcpyAsync(b->h, b->d, b->size, cudaMemcpyDeviceToHost,
                                                 st) != cudaSuccess))
          ok = false;
      }
    }
  }
  if (ok)
    rc = mc_stream_sync(d, FRAME_TIMEOUT_MS);
  if (!ok || rc) {
    const cudaError_t ce = cudaGetLastError();
    mc_stream_sync(d, FRAME_TIMEOUT_MS);
    for (MopCudaBuffer *b : made) {
      free(b->h);
      delete b;
    }
    cudaFree(slab->d);
    delete slab;
    return rc ? rc : fail(MOPCUDA_ECUDA, "scene_file_upload_all: %s", cudaGetErrorString(ce));
  }
  for (uint32_t k = 0; k < n; k++) {
    vertices[k] = made[2 * k];
    indices[k] = made[2 * k + 1];
    if (vertex_counts)
      vertex_counts[k] = ms[k].vc;
    if (index_counts)
      index_counts[k] = ms[k].ic;
  }
  return MOPCUDA_OK;
}
