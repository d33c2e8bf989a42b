/*
 * texture.cu — compressed textures and render-to-texture on the device
 * (reference src/backend/cpu/cpu_backend.c).
 *
 *   mopcuda_texture_create_ex        texture_create_ex: BC1 / BC3 / BC5
 *                                    blocks decoded to RGBA8 on the device
 *                                    (bc_decompress_to_rgba8, :855-1014;
 *                                    cpu_texture_create_ex, :1016-1056)
 *   mopcuda_framebuffer_copy_to_texture
 *                                    framebuffer_copy_to_texture: same-size
 *                                    copy or integer SSAA box (:741-790)
 *   mopcuda_framebuffer_create_from_texture
 *                                    framebuffer_create_from_texture: frames
 *                                    land in a host texture (:143-170)
 *
 * The block decode is integer arithmetic (RGB565 expansion with the
 * reference's `* 255 / 31` truncating divisions, the 1/3-2/3 and 1/2
 * palette means, the 3-bit BC4 ramps), so the decoded bytes are the CPU
 * backend's.  One thread decodes one 4x4 block and writes the texels that
 * fall inside the image, as the reference clamps the last row and column of
 * blocks.
 */
#include "api_internal.h"

#include <string.h>

namespace {

constexpr int FMT_RGBA8 = 0, FMT_BC1 = 1, FMT_BC3 = 2, FMT_BC5 = 3, FMT_BC7 = 4;

/* bc_decode_rgb565, cpu_backend.c:859-863 */
__device__ __forceinline__ void rgb565(uint32_t c, uint32_t out[3]) {
  out[0] = ((c >> 11) & 0x1Fu) * 255u / 31u;
  out[1] = ((c >> 5) & 0x3Fu) * 255u / 63u;
  out[2] = (c & 0x1Fu) * 255u / 31u;
}

/* bc1_decode_block, cpu_backend.c:866-905: the four palette entries as
 * packed RGBA8 words (R in the low byte). */
__device__ __forceinline__ void bc1_palette(const uint8_t *s, uint32_t pal[4]) {
  const uint32_t c0 = (uint32_t)s[0] | ((uint32_t)s[1] << 8);
  const uint32_t c1 = (uint32_t)s[2] | ((uint32_t)s[3] << 8);
  uint32_t a[3], b[3], p2[3], p3[3];
  rgb565(c0, a);
  rgb565(c1, b);
  uint32_t alpha3 = 255u;
  if (c0 > c1) {
    for (int i = 0; i < 3; i++) {
      p2[i] = (2u * a[i] + b[i] + 1u) / 3u;
      p3[i] = (a[i] + 2u * b[i] + 1u) / 3u;
    }
  } else {
    for (int i = 0; i < 3; i++) {
      p2[i] = (a[i] + b[i]) / 2u;
      p3[i] = 0u;
    }
    alpha3 = 0u; /* transparent black */
  }
  pal[0] = a[0] | (a[1] << 8) | (a[2] << 16) | (255u << 24);
  pal[1] = b[0] | (b[1] << 8) | (b[2] << 16) | (255u << 24);
  pal[2] = p2[0] | (p2[1] << 8) | (p2[2] << 16) | (255u << 24);
  pal[3] = p3[0] | (p3[1] << 8) | (p3[2] << 16) | (alpha3 << 24);
}

/* bc4_decode_block's palette, cpu_backend.c:908-940 */
__device__ __forceinline__ void bc4_palette(const uint8_t *s, uint32_t pal[8], uint64_t &bits) {
  const uint32_t a0 = s[0], a1 = s[1];
  bits = 0;
  for (int i = 0; i < 6; i++)
    bits |= (uint64_t)s[2 + i] << (i * 8);
  pal[0] = a0;
  pal[1] = a1;
  if (a0 > a1) {
    for (uint32_t i = 1; i <= 6; i++)
      pal[1 + i] = ((7u - i) * a0 + i * a1 + 3u) / 7u;
  } else {
    for (uint32_t i = 1; i <= 4; i++)
      pal[1 + i] = ((5u - i) * a0 + i * a1 + 2u) / 5u;
    pal[6] = 0u;
    pal[7] = 255u;
  }
}

/* One thread per 4x4 block of a BC1 / BC3 / BC5 image (w x h texels). */
__global__ void __launch_bounds__(256) k_bc_decode(const uint8_t *__restrict__ src, int w, int h,
                                                   int format, uchar4 *__restrict__ dst) {
  const int bw = (w + 3) / 4, bh = (h + 3) / 4;
  const int blk = blockIdx.x * blockDim.x + threadIdx.x;
  if (blk >= bw * bh)
    return;
  const int bx = blk % bw, by = blk / bw;
  const size_t bsize = format == FMT_BC1 ? 8u : 16u;
  const uint8_t *s = src + (size_t)blk * bsize;
  uint32_t texel[16];
  if (format == FMT_BC5) {
    /* bc5_decode_block, :960-976: (R, G) from two BC4 blocks, B 0, A 255 */
    uint32_t pr[8], pg[8];
    uint64_t br, bg;
    bc4_palette(s, pr, br);
    bc4_palette(s + 8, pg, bg);
    for (int t = 0; t < 16; t++)
      texel[t] = pr[(br >> (3 * t)) & 7u] | (pg[(bg >> (3 * t)) & 7u] << 8) | (255u << 24);
  } else {
    /* BC1: the colour block itself; BC3 (bc3_decode_block, :952-957): the
     * colour block at +8, its alpha replaced by a BC4 block at +0 */
    const uint8_t *cb = format == FMT_BC3 ? s + 8 : s;
    uint32_t pal[4];
    bc1_palette(cb, pal);
    const uint32_t lut = (uint32_t)cb[4] | ((uint32_t)cb[5] << 8) | ((uint32_t)cb[6] << 16) |
                         ((uint32_t)cb[7] << 24);
    for (int t = 0; t < 16; t++)
      texel[t] = pal[(lut >> (2 * t)) & 3u];
    if (format == FMT_BC3) {
      uint32_t pa[8];
      uint64_t ba;
      bc4_palette(s, pa, ba);
      for (int t = 0; t < 16; t++)
        texel[t] = (texel[t] & 0x00ffffffu) | (pa[(ba >> (3 * t)) & 7u] << 24);
    }
  }
  const int px = bx * 4, py = by * 4;
  for (int ty = 0; ty < 4 && py + ty < h; ty++)
    for (int tx = 0; tx < 4 && px + tx < w; tx++) {
      const uint32_t v = texel[ty * 4 + tx];
      dst[(size_t)(py + ty) * (size_t)w + (size_t)(px + tx)] =
          make_uchar4((uint8_t)v, (uint8_t)(v >> 8), (uint8_t)(v >> 16), (uint8_t)(v >> 24));
    }
}

} // namespace

extern "C" MopCudaTexture *mopcuda_texture_create_ex(MopCudaDevice *d, int w, int h, int format,
                                                    int mip_levels, const uint8_t *data,
                                                    size_t data_size) {
  (void)mip_levels; /* the CPU backend decodes level 0 only */
  if (format == FMT_RGBA8)
    return mopcuda_texture_create(d, w, h, data);
  if (!d || !data || w <= 0 || h <= 0 || w > 16384 || h > 16384) {
    fail(MOPCUDA_EINVAL, "texture_create_ex: bad arguments");
    return nullptr;
  }
  if (format == FMT_BC7) { /* no software decode in the reference either */
    fail(MOPCUDA_EUNSUPPORTED, "texture_create_ex: BC7 is not decoded (as the CPU backend)");
    return nullptr;
  }
  if (format < FMT_BC1 || format > FMT_BC7) {
    fail(MOPCUDA_EINVAL, "texture_create_ex: unknown format %d", format);
    return nullptr;
  }
  const size_t blocks = (size_t)((w + 3) / 4) * (size_t)((h + 3) / 4);
  const size_t need = blocks * (format == FMT_BC1 ? 8u : 16u);
  /* the reference reads the size the dimensions imply; a declared size
   * smaller than that is refused instead of read past */
  if (data_size && data_size < need) {
    fail(MOPCUDA_EINVAL, "texture_create_ex: %zu bytes given, BC%d %dx%d needs %zu", data_size,
         format == FMT_BC1 ? 1 : (format == FMT_BC3 ? 3 : 5), w, h, need);
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  const size_t bytes = (size_t)w * (size_t)h * 4u;
  MopCudaTexture *t = new MopCudaTexture();
  t->w = w;
  t->h = h;
  t->hcopy = malloc(bytes);
  void *blk = nullptr;
  if (!t->hcopy || cudaMalloc(&t->d, bytes) != cudaSuccess || cudaMalloc(&blk, need) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(t->d);
    free(t->hcopy);
    delete t;
    fail(MOPCUDA_ENOMEM, "texture_create_ex: allocation failed");
    return nullptr;
  }
  cudaStream_t s = d->stream;
  bool ok = cudaMemcpyAsync(blk, data, need, cudaMemcpyHostToDevice, s) == cudaSuccess;
  if (ok) {
    k_bc_decode<<<(unsigned)((blocks + 255u) / 256u), 256, 0, s>>>((const uint8_t *)blk, w, h,
                                                                   format, (uchar4 *)t->d);
    d->launches++;
    ok = cudaGetLastError() == cudaSuccess &&
         cudaMemcpyAsync(t->hcopy, t->d, bytes, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         mc_stream_sync(d, FRAME_TIMEOUT_MS) == MOPCUDA_OK;
  }
  cudaFree(blk);
  if (!ok) {
    cudaGetLastError();
    cudaFree(t->d);
    free(t->hcopy);
    delete t;
    fail(MOPCUDA_ECUDA, "texture_create_ex: upload or decode failed");
    return nullptr;
  }
  return t;
}

/* The framebuffer's post-processed colour into the texture's device copy:
 * the same size, or a whole-number SSAA factor smaller (box of sf x sf
 * samples, truncating mean), then the texture's host copy refreshed.  Called
 * with the device lock held and the frame complete. */
static int copy_out_to_texture(MopCudaDevice *d, MopCudaFramebuffer *fb, MopCudaTexture *t) {
  const int fw = fb->w, fh = fb->h, tw = t->w, th = t->h;
  cudaStream_t s = d->stream;
  if (fb->host_color) /* the core may have written through the readback pointer */
    CU_TRY(cudaMemcpyAsync(fb->out.p, fb->h_color.p, (size_t)fw * fh * 4,
                           cudaMemcpyHostToDevice, s));
  if (tw == fw && th == fh) {
    CU_TRY(cudaMemcpyAsync(t->d, fb->out.p, (size_t)fw * fh * 4, cudaMemcpyDeviceToDevice, s));
  } else {
    const int sf = fw / tw;
    d->launches += (uint64_t)mopcuda_launch_box(fb->out.as<uchar4>(), fw, fh, sf, (uchar4 *)t->d, s);
    CU_TRY(cudaGetLastError());
  }
  CU_TRY(cudaMemcpyAsync(t->hcopy, t->d, (size_t)tw * th * 4, cudaMemcpyDeviceToHost, s));
  return mc_stream_sync(d, FRAME_TIMEOUT_MS);
}

extern "C" int mopcuda_framebuffer_copy_to_texture(MopCudaDevice *d, MopCudaFramebuffer *fb,
                                                   MopCudaTexture *t) {
  if (!d || !fb || !t || t->hdr || !t->d)
    return fail(MOPCUDA_EINVAL, "framebuffer_copy_to_texture: bad arguments");
  const int fw = fb->w, fh = fb->h, tw = t->w, th = t->h;
  const bool same = tw == fw && th == fh;
  const bool boxed = tw > 0 && th > 0 && fw % tw == 0 && fh % th == 0 && fw / tw == fh / th;
  if (!same && !boxed) /* cpu_backend.c:786-789 */
    return fail(MOPCUDA_EINVAL,
                "framebuffer_copy_to_texture: unsupported size combination (fb %dx%d, tex %dx%d)",
                fw, fh, tw, th);
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->ordinal);
  int rc = mc_finish_pending(d);
  if (rc)
    return rc;
  return copy_out_to_texture(d, fb, t);
}

extern "C" MopCudaFramebuffer *mopcuda_framebuffer_create_from_texture(MopCudaDevice *d,
                                                                     MopCudaTexture *t, int w,
                                                                     int h) {
  if (!d || !t || !t->d || w <= 0 || h <= 0) {
    fail(MOPCUDA_EINVAL, "framebuffer_create_from_texture: bad arguments");
    return nullptr;
  }
  if (t->w != w || t->h != h) { /* cpu_backend.c:150-155 */
    fail(MOPCUDA_EINVAL, "framebuffer_create_from_texture: size mismatch (tex %dx%d, fb %dx%d)",
         t->w, t->h, w, h);
    return nullptr;
  }
  if (t->hdr) {
    fail(MOPCUDA_EINVAL, "framebuffer_create_from_texture: HDR target not supported");
    return nullptr;
  }
  MopCudaFramebuffer *fb = mopcuda_framebuffer_create(d, w, h);
  if (fb)
    fb->target = t;
  return fb;
}

int mc_target_update(MopCudaDevice *d, MopCudaFramebuffer *fb) {
  return fb && fb->target ? copy_out_to_texture(d, fb, fb->target) : MOPCUDA_OK;
}
