/*
 * fold.h — exact value of k sequential float additions, in O(binades).
 *
 * The reference rasteriser steps its edge functions incrementally: for each
 * pixel of a row it does `w += e_dx`, for each row `w_row += e_dy`, always
 * starting from the clamped bounding-box corner (rasterizer.c:1926-2151 and
 * 1015-1023).  Repeated round-to-nearest-even addition has no closed form in
 * general, so a pixel's coverage, depth and interpolation weights depend on
 * the exact fold  w_k = RN(w_{k-1} + d).  A GPU that evaluates pixels in
 * parallel must reproduce that fold without walking every intermediate step.
 *
 * Method.  Inside one binade [2^E, 2^(E+1)) (same sign) the representable
 * values are N*u with u = 2^(E-23) and integer N in [2^23, 2^24).  If the
 * exact sum N + d/u lies in the binade, rounding adds a fixed integer
 * increment Q = rne(d/u) — except for exact ties (d/u = M + 1/2), where the
 * result is always even, so after one tie-rounded step the increment is the
 * constant even value of {M, M+1}.  Hence: take three explicit steps
 * w1, w2, w3; when all three lie in one binade and w2, w3 keep one unit of
 * margin from its edges, Q = N3 - N2 is the increment of every later step
 * that stays inside [2^23+1, 2^24-1] (then the exact sum also stays inside
 * the binade, |exact - rounded| <= 1/2).  Jump there with integer
 * arithmetic, then continue with explicit steps into the next binade.
 * Zero, subnormal and non-finite values are stepped explicitly.  The cost is
 * about four additions per binade crossed instead of one per step.
 *
 * The same header is compiled for the device (kernels) and for the host
 * (unit test against the plain loop).
 */
#ifndef MOPCUDA_FOLD_H
#define MOPCUDA_FOLD_H

#include <stdint.h>

#if defined(__CUDACC__)
#define MOPCUDA_HD __host__ __device__ __forceinline__
#define MOPCUDA_HD_SLOW static __host__ __device__ __noinline__
#else
#define MOPCUDA_HD static inline
#define MOPCUDA_HD_SLOW static
#include <string.h>
#endif

MOPCUDA_HD uint32_t fold_bits(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}

MOPCUDA_HD float fold_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}

/* One IEEE single round-to-nearest-even addition, never contracted. */
MOPCUDA_HD float fold_fadd(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_rn(a, b);
#else
  volatile float r = a + b;
  return r;
#endif
}

#define FOLD_SERIAL_MAX 16

/* The binade-skipping path of fold_add for k > FOLD_SERIAL_MAX (kept out of
 * line: callers inline only the short serial loop). */
MOPCUDA_HD_SLOW float fold_add_long(float w, float d, int k) {
  uint32_t db = fold_bits(d);
  /* d = +-0, inf or NaN: after one addition the value is a fixed point. */
  if ((db & 0x7fffffffu) == 0u || (db & 0x7f800000u) == 0x7f800000u)
    return fold_fadd(w, d);
  while (k > 0) {
    uint32_t wb = fold_bits(w);
    if ((wb & 0x7f800000u) == 0x7f800000u) /* inf/NaN + finite d is stable */
      return w;
    if (k <= 3) {
      for (int i = 0; i < k; i++)
        w = fold_fadd(w, d);
      return w;
    }
    float w1 = fold_fadd(w, d);
    float w2 = fold_fadd(w1, d);
    float w3 = fold_fadd(w2, d);
    k -= 3;
    w = w3;
    uint32_t b1 = fold_bits(w1), b2 = fold_bits(w2), b3 = fold_bits(w3);
    uint32_t hi = b3 & 0xff800000u; /* sign + exponent */
    if ((b1 & 0xff800000u) != hi || (b2 & 0xff800000u) != hi)
      continue;
    uint32_t ex = (hi >> 23) & 0xffu;
    if (ex == 0u || ex == 0xffu)
      continue;
    int32_t n2 = (int32_t)((b2 & 0x007fffffu) | 0x00800000u);
    int32_t n3 = (int32_t)((b3 & 0x007fffffu) | 0x00800000u);
    const int32_t lo = 0x00800001, top = 0x00ffffff;
    if (n2 < lo || n3 < lo)
      continue;
    int32_t q = n3 - n2; /* steady increment of the magnitude */
    if (q == 0)
      return w3; /* the increment rounds away: w is a fixed point */
    int32_t room = q > 0 ? (top - n3) / q : (n3 - lo) / (-q);
    int32_t j = room < k ? room : k;
    if (j <= 0)
      continue;
    int32_t n = n3 + j * q; /* |j*q| < 2^24: no overflow */
    w = fold_float(hi | ((uint32_t)n & 0x007fffffu));
    k -= j;
  }
  return w;
}

/* w after k >= 0 sequential additions of d. */
MOPCUDA_HD float fold_add(float w, float d, int k) {
  if (k <= FOLD_SERIAL_MAX) {
    /* fully unrolled and predicated: no loop and no divergence on k */
#pragma unroll
    for (int i = 0; i < FOLD_SERIAL_MAX; i++)
      if (i < k)
        w = fold_fadd(w, d);
    return w;
  }
  return fold_add_long(w, d, k);
}

#endif
