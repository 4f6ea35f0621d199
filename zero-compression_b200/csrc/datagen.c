/* datagen.c -- seeded synthetic inputs shaped like the workloads the ZB2 codec is measured on.
 *
 *   zg_text_mix : alternating 4 KiB segments.  Text: words of a 256-word vocabulary (2..10 random
 *                 lowercase letters each, Zipf s = 1.1 word frequencies) separated by a space (90 %)
 *                 or a newline (10 %).  Repeat: copies of earlier output, length geometric with mean 32,
 *                 offset uniform in [1, 65536] (never before the start of the output).
 *   zg_lz_mix   : literal runs (length geometric, mean 8; bytes drawn from a geometric distribution over
 *                 256 symbols, p = 0.05, under a seeded random permutation) alternating with matches
 *                 (length log-uniform in [4, 258], offset log-uniform in [1, block size]).
 *   zg_random   : uniform random bytes (every block of it is stored).
 *
 * The reference measures on Windows corpora that are not available; these shapes stand in for them.
 * Deterministic for a given seed on every platform (xoshiro256** seeded by splitmix64, and only
 * correctly rounded libm calls: log and exp).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { uint64_t s[4]; } zg_rng;

static uint64_t splitmix(uint64_t *x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static void rng_seed(zg_rng *r, uint64_t seed) {
  for (int i = 0; i < 4; ++i) r->s[i] = splitmix(&seed);
}
static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t rng_next(zg_rng *r) {
  const uint64_t out = rotl(r->s[1] * 5, 7) * 9, t = r->s[1] << 17;
  r->s[2] ^= r->s[0]; r->s[3] ^= r->s[1]; r->s[1] ^= r->s[2]; r->s[0] ^= r->s[3];
  r->s[2] ^= t; r->s[3] = rotl(r->s[3], 45);
  return out;
}
/* uniform in (0, 1] with 53 bits */
static double rng_unit(zg_rng *r) { return ((double)(rng_next(r) >> 11) + 1.0) * (1.0 / 9007199254740992.0); }
/* uniform integer in [lo, hi] */
static uint64_t rng_range(zg_rng *r, uint64_t lo, uint64_t hi) { return lo + rng_next(r) % (hi - lo + 1); }
/* geometric on {1, 2, ...} with the given mean */
static uint64_t rng_geometric(zg_rng *r, double mean) {
  const double q = 1.0 - 1.0 / mean;
  return 1 + (uint64_t)floor(log(rng_unit(r)) / log(q));
}
/* log-uniform integers in [lo, hi] (the bounds' logs computed once) */
typedef struct { double lo, hi, llo, lhi; } zg_logu;
static zg_logu logu(double lo, double hi) { zg_logu u = {lo, hi, log(lo), log(hi + 1.0)}; return u; }
static uint64_t rng_loguniform(zg_rng *r, const zg_logu *u) {
  const double v = exp(u->llo + (u->lhi - u->llo) * (1.0 - rng_unit(r)));
  uint64_t x = (uint64_t)floor(v);
  if (x < (uint64_t)u->lo) x = (uint64_t)u->lo;
  if (x > (uint64_t)u->hi) x = (uint64_t)u->hi;
  return x;
}
/* a 256-entry cumulative table (scaled to 2^32) with a guide: guide[g] is the first index whose bound
 * exceeds g << 20, so a draw starts its search there instead of at 0 */
typedef struct { uint64_t cdf[256]; uint8_t guide[4096]; } zg_cdf;
static void cdf_guide(zg_cdf *c) {
  int k = 0;
  for (int g = 0; g < 4096; ++g) {
    while (k < 255 && c->cdf[k] <= ((uint64_t)g << 20)) ++k;
    c->guide[g] = (uint8_t)k;
  }
}
/* the smallest index whose bound exceeds a uniform 32-bit draw */
static int pick_cdf(zg_rng *r, const zg_cdf *c) {
  const uint64_t u = rng_next(r) >> 32;
  int k = c->guide[u >> 20];
  while (u >= c->cdf[k]) ++k;
  return k;
}
static void copy_back(uint8_t *out, size_t at, size_t off, size_t len) {
  const uint8_t *src = out + at - off;
  if (off >= len) memcpy(out + at, src, len);
  else for (size_t k = 0; k < len; ++k) out[at + k] = src[k];
}

void zg_text_mix(uint8_t *out, size_t n, uint64_t seed) {
  zg_rng r;
  rng_seed(&r, seed);
  char words[256][10];
  int wlen[256];
  for (int w = 0; w < 256; ++w) {
    wlen[w] = (int)rng_range(&r, 2, 10);
    for (int k = 0; k < wlen[w]; ++k) words[w][k] = (char)('a' + rng_range(&r, 0, 25));
  }
  double z[256], zs = 0;
  for (int k = 0; k < 256; ++k) { z[k] = pow(k + 1.0, -1.1); zs += z[k]; }
  zg_cdf cdf;
  double acc = 0;
  for (int k = 0; k < 256; ++k) { acc += z[k]; cdf.cdf[k] = (uint64_t)(acc / zs * 4294967296.0); }
  cdf.cdf[255] = (uint64_t)1 << 32;
  cdf_guide(&cdf);
  const size_t SEG = 4096;
  size_t at = 0;
  for (size_t seg = 0; at < n; ++seg) {
    const size_t end = at + SEG < n ? at + SEG : n;
    if ((seg & 1) == 0 || at == 0) {
      while (at < end) {
        const int w = pick_cdf(&r, &cdf);
        for (int k = 0; k < wlen[w] && at < end; ++k) out[at++] = (uint8_t)words[w][k];
        if (at < end) out[at++] = (rng_next(&r) % 10 == 0) ? '\n' : ' ';
      }
    } else {
      while (at < end) {
        size_t len = (size_t)rng_geometric(&r, 32.0);
        const size_t maxoff = at < 65536 ? at : 65536;
        const size_t off = (size_t)rng_range(&r, 1, maxoff);
        if (len > end - at) len = end - at;
        copy_back(out, at, off, len);
        at += len;
      }
    }
  }
}

void zg_lz_mix(uint8_t *out, size_t n, uint32_t block_log, uint64_t seed) {
  zg_rng r;
  rng_seed(&r, seed);
  uint8_t perm[256];
  for (int k = 0; k < 256; ++k) perm[k] = (uint8_t)k;
  for (int k = 255; k > 0; --k) {
    const int j = (int)rng_range(&r, 0, (uint64_t)k);
    const uint8_t t = perm[k]; perm[k] = perm[j]; perm[j] = t;
  }
  /* geometric(p = 0.05) over symbol ranks 0..255, truncated at 255 and renormalised */
  double pk[256], ps = 0;
  for (int k = 0; k < 256; ++k) { pk[k] = 0.05 * pow(0.95, k); ps += pk[k]; }
  zg_cdf cdf;
  double acc = 0;
  for (int k = 0; k < 256; ++k) { acc += pk[k]; cdf.cdf[k] = (uint64_t)(acc / ps * 4294967296.0); }
  cdf.cdf[255] = (uint64_t)1 << 32;
  cdf_guide(&cdf);
  const zg_logu ulen = logu(4.0, 258.0), uoff = logu(1.0, (double)((size_t)1 << block_log));
  size_t at = 0;
  while (at < n) {
    size_t lit = (size_t)rng_geometric(&r, 8.0);
    if (lit > n - at) lit = n - at;
    for (size_t k = 0; k < lit; ++k) out[at++] = perm[pick_cdf(&r, &cdf)];
    if (at >= n) break;
    size_t len = (size_t)rng_loguniform(&r, &ulen);
    size_t off = (size_t)rng_loguniform(&r, &uoff);
    if (off > at) off = at;
    if (len > n - at) len = n - at;
    copy_back(out, at, off, len);
    at += len;
  }
}

void zg_random(uint8_t *out, size_t n, uint64_t seed) {
  zg_rng r;
  rng_seed(&r, seed);
  size_t at = 0;
  for (; at + 8 <= n; at += 8) {
    const uint64_t v = rng_next(&r);
    memcpy(out + at, &v, 8);
  }
  if (at < n) {
    const uint64_t v = rng_next(&r);
    memcpy(out + at, &v, n - at);
  }
}

/* file sizes log-uniform in [lo, hi] bytes, and a generator kind per file (0 text, 1 lz, 2 random),
 * for the many-file archive workload */
void zg_file_plan(uint64_t *sizes, uint8_t *kinds, size_t count, uint64_t lo, uint64_t hi, uint64_t seed) {
  zg_rng r;
  rng_seed(&r, seed);
  const zg_logu us = logu((double)lo, (double)hi);
  for (size_t i = 0; i < count; ++i) {
    sizes[i] = rng_loguniform(&r, &us);
    kinds[i] = (uint8_t)rng_range(&r, 0, 2);
  }
}
