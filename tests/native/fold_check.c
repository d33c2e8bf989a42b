/* Host check of fold_add (master-of-puppets_b200/csrc/fold.h) against the
 * plain serial loop it replaces.  Built and run by tests/test_fold.py. */
#include "fold.h"

#include <stdint.h>
#include <stdio.h>
#include <string.h>

static uint64_t s_state = 0x9E3779B97F4A7C15ULL;
static uint64_t rnd(void) {
  s_state ^= s_state << 13;
  s_state ^= s_state >> 7;
  s_state ^= s_state << 17;
  return s_state;
}
static float rndf(void) { /* wide range, signed, with exact-grid values */
  uint64_t r = rnd();
  int mode = (int)(r & 7);
  float mag = (float)((r >> 8) & 0xffffff) / 16777216.0f;
  int e = (int)((r >> 40) % 40) - 20;
  float v = mag;
  for (int i = 0; i < (e < 0 ? -e : e); i++)
    v = e < 0 ? v * 0.5f : v * 2.0f;
  if (mode == 0)
    v = (float)((int)((r >> 16) & 0xfff) - 2048) * 0.125f; /* coarse grid: many ties */
  if (mode == 1)
    v = (float)((int)((r >> 16) & 0xfffff) - 524288) * (1.0f / 4096.0f);
  if ((r >> 63) & 1)
    v = -v;
  return v;
}

static float serial(float w, float d, int k) {
  for (int i = 0; i < k; i++) {
    volatile float t = w + d;
    w = t;
  }
  return w;
}

/* Returns the number of mismatches over n random cases; writes the first. */
int fold_check(int n, uint64_t seed, float *bad) {
  s_state = seed | 1;
  int fails = 0;
  for (int i = 0; i < n; i++) {
    float w = rndf(), d = rndf();
    int k = (int)(rnd() % 5000);
    if (i % 7 == 0) /* screen-like: w ~ edge value, d ~ edge slope */
      d = (float)((int)(rnd() % 4001) - 2000) * (1.0f / 64.0f);
    if (i % 11 == 0) /* d exactly half an ulp of w: tie stepping */
      d = w * 5.9604645e-08f;
    if (i % 13 == 0 && w != 0.0f) { /* d = (M + 1/2) ulp(w), M of both parities */
      uint32_t wb;
      memcpy(&wb, &w, 4);
      int ex = (int)((wb >> 23) & 0xff);
      if (ex > 24 && ex < 230) {
        uint32_t ub = (uint32_t)(ex - 23) << 23; /* ulp of w's binade */
        float ulp;
        memcpy(&ulp, &ub, 4);
        d = ((float)(rnd() % 9) + 0.5f) * ulp;
        if (rnd() & 1)
          d = -d;
      }
    }
    float a = fold_add(w, d, k), b = serial(w, d, k);
    uint32_t ua, ub;
    memcpy(&ua, &a, 4);
    memcpy(&ub, &b, 4);
    if (ua != ub && !(a != a && b != b)) {
      if (fails == 0 && bad) {
        bad[0] = w;
        bad[1] = d;
        bad[2] = (float)k;
        bad[3] = a;
        bad[4] = b;
      }
      fails++;
    }
  }
  return fails;
}
