/* zb2_oracle.c -- TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference CPU codec for the ZB2
 * block format (rANS streams, LZ77 parse, block payload, CRC-32).  It is the checker the CUDA path is
 * compared against; nothing in the product links it.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.
 *
 * Parity pin: every function here is checked against the reference's own code, compiled from its
 * sources into oracle/_ref/libzref.so (oracle/Makefile), and against the committed golden vectors in
 * tests/golden/ that the reference generated (tests/golden/make_golden.py).
 *
 * Citations are file:line in the reference project (rizagp/zero-compression).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ZO_NLANES 64u
#define ZO_SCALE_BITS 12u
#define ZO_SCALE (1u << ZO_SCALE_BITS)
#define ZO_LOW (1u << 23)
#define ZO_HDR 20u
#define ZO_SYM_REP 250u

static uint32_t rd32(const uint8_t *p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }
static void wr32(uint8_t *p, uint32_t v) { p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24); }

/* ---------------------------------------------------------------- CRC-32 (src/crc32.h:1-66)
 * IEEE 802.3 reflected polynomial 0xEDB88320, initial and final inversion.  Restated byte at a time. */
static uint32_t crc_tab[256];
static int crc_ready = 0;
static void crc_init(void) {
  for (uint32_t i = 0; i < 256; ++i) {
    uint32_t r = i;
    for (int k = 0; k < 8; ++k) r = (r >> 1) ^ (0xEDB88320u & (0u - (r & 1u)));
    crc_tab[i] = r;
  }
  crc_ready = 1;
}
/* crc32::update (src/crc32.h:22-38): continue a finished CRC over n more bytes */
uint32_t zo_crc32_update(uint32_t crc, const uint8_t *p, size_t n) {
  if (!crc_ready) crc_init();
  uint32_t r = ~crc;
  for (size_t i = 0; i < n; ++i) r = crc_tab[(r ^ p[i]) & 0xFFu] ^ (r >> 8);
  return ~r;
}
/* a*b in GF(2)[x] mod P, in the reflected bit order (bit 31 holds x^0) */
static uint32_t gf_mul(uint32_t a, uint32_t b) {
  uint32_t acc = 0;
  for (int i = 0; i < 32; ++i) {
    if (a & 0x80000000u) acc ^= b;
    a <<= 1;
    b = (b >> 1) ^ (0xEDB88320u & (0u - (b & 1u)));
  }
  return acc;
}
/* x^(8n) mod P by square and multiply */
static uint32_t x_pow_8n(uint64_t n) {
  uint32_t result = 0x80000000u; /* x^0 */
  uint32_t base = 0x00800000u;   /* x^8 */
  while (n) {
    if (n & 1u) result = gf_mul(result, base);
    base = gf_mul(base, base);
    n >>= 1;
  }
  return result;
}
/* crc32::combine (src/crc32.h:41-66): CRC of A||B from crc(A), crc(B), |B| */
uint32_t zo_crc32_combine(uint32_t a, uint32_t b, uint64_t len_b) {
  if (!len_b) return a;
  return gf_mul(x_pow_8n(len_b), a) ^ b;
}

/* ---------------------------------------------------------------- frequencies (src/codec.h:41-66)
 * counts -> 12-bit frequencies summing to 4096, every present symbol at least 1.  The fix-up order is
 * part of the format: while the sum is above 4096 take one from the largest frequency above 1 (lowest
 * symbol on a tie); then give any deficit to the largest frequency (lowest symbol on a tie). */
void zo_normalize(const uint32_t counts[256], uint32_t total, uint16_t freq[256]) {
  uint32_t sum = 0;
  for (int s = 0; s < 256; ++s) {
    uint32_t f = 0;
    if (counts[s]) {
      f = (uint32_t)(((uint64_t)counts[s] << ZO_SCALE_BITS) / total);
      if (!f) f = 1;
    }
    freq[s] = (uint16_t)f;
    sum += f;
  }
  for (; sum > ZO_SCALE; --sum) {
    int top = -1;
    for (int s = 0; s < 256; ++s)
      if (freq[s] > 1 && (top < 0 || freq[s] > freq[top])) top = s;
    freq[top]--;
  }
  if (sum < ZO_SCALE) {
    int top = 0;
    for (int s = 1; s < 256; ++s)
      if (freq[s] > freq[top]) top = s;
    freq[top] = (uint16_t)(freq[top] + (ZO_SCALE - sum));
  }
}

/* bit length of an offset: b with 2^b <= d < 2^(b+1) (src/codec2.h:36-40) */
static uint32_t bitlen(uint32_t d) {
  uint32_t b = 0;
  while (d >> (b + 1)) ++b;
  return b;
}

/* ---------------------------------------------------------------- one stream (src/codec.h:96-147)
 * Writes kind(u8) len(u32) body at out; returns the bytes written.  out must hold 5 + n + 800 bytes.
 * Symbol i goes to lane i % 64; each lane is coded last symbol first; raw when rANS is not smaller. */
size_t zo_encode_stream(const uint8_t *sym, uint32_t n, uint8_t *out) {
  if (n == 0) { out[0] = 0; wr32(out + 1, 0); return 5; }
  uint32_t counts[256] = {0};
  for (uint32_t i = 0; i < n; ++i) counts[sym[i]]++;
  uint16_t freq[256];
  zo_normalize(counts, n, freq);
  uint32_t cum[256], c = 0, present = 0;
  for (int s = 0; s < 256; ++s) { cum[s] = c; c += freq[s]; present += freq[s] != 0; }
  const uint32_t per_lane = (n + ZO_NLANES - 1) / ZO_NLANES;
  const size_t lane_cap = 2 * (size_t)per_lane + 16;
  uint8_t *scratch = (uint8_t *)malloc(lane_cap * ZO_NLANES);
  uint32_t lane_len[ZO_NLANES];
  size_t body = 32 + 2 * (size_t)present + 4 * ZO_NLANES;
  for (uint32_t j = 0; j < ZO_NLANES; ++j) {
    uint8_t *end = scratch + lane_cap * (j + 1), *w = end;
    uint32_t x = ZO_LOW;
    if (j < n) {
      for (int64_t i = j + (int64_t)((n - 1 - j) / ZO_NLANES) * ZO_NLANES; i >= 0; i -= ZO_NLANES) {
        const uint32_t f = freq[sym[i]];
        const uint32_t limit = f << (23 - ZO_SCALE_BITS + 8); /* RansEnc::put (src/codec.h:79-84) */
        while (x >= limit) { *--w = (uint8_t)x; x >>= 8; }
        x = ((x / f) << ZO_SCALE_BITS) + (x % f) + cum[sym[i]];
      }
    }
    w -= 4;
    wr32(w, x); /* RansEnc::flush (src/codec.h:85-89) */
    lane_len[j] = (uint32_t)(end - w);
    body += lane_len[j];
  }
  size_t at;
  if (body >= n) {
    out[0] = 0;
    wr32(out + 1, n);
    memcpy(out + 5, sym, n);
    at = 5 + n;
  } else {
    out[0] = 1;
    wr32(out + 1, (uint32_t)body);
    at = 5;
    for (int b = 0; b < 32; ++b) {
      uint8_t bits = 0;
      for (int k = 0; k < 8; ++k) bits |= (uint8_t)((freq[b * 8 + k] != 0) << k);
      out[at++] = bits;
    }
    for (int s = 0; s < 256; ++s)
      if (freq[s]) { out[at++] = (uint8_t)freq[s]; out[at++] = (uint8_t)(freq[s] >> 8); }
    for (uint32_t j = 0; j < ZO_NLANES; ++j) { wr32(out + at, lane_len[j]); at += 4; }
    for (uint32_t j = 0; j < ZO_NLANES; ++j) {
      memcpy(out + at, scratch + lane_cap * (j + 1) - lane_len[j], lane_len[j]);
      at += lane_len[j];
    }
  }
  free(scratch);
  return at;
}

/* ---------------------------------------------------------------- one stream back (src/codec.h:150-205)
 * Decodes the section at p (avail bytes readable) into n symbols; returns bytes consumed, or -1 when the
 * section is damaged (every case where the reference throws zb::Error). */
long zo_decode_stream(const uint8_t *p, size_t avail, uint32_t n, uint8_t *sym) {
  if (avail < 5) return -1;
  const uint32_t kind = p[0], len = rd32(p + 1);
  const uint8_t *body = p + 5;
  if (avail - 5 < len) return -1;
  if (kind == 0) {
    if (len != n) return -1;
    memcpy(sym, body, n);
    return 5 + (long)len;
  }
  if (kind != 1) return -1;
  if (len < 32 + 4 * ZO_NLANES) return -1;
  uint32_t present = 0;
  for (int s = 0; s < 256; ++s) present += (body[s >> 3] >> (s & 7)) & 1u;
  if (len < 32 + 2 * present + 4 * ZO_NLANES) return -1;
  uint16_t freq[256];
  uint32_t cum[256], c = 0;
  const uint8_t *fp = body + 32;
  for (int s = 0; s < 256; ++s) {
    freq[s] = 0;
    if ((body[s >> 3] >> (s & 7)) & 1u) { freq[s] = (uint16_t)(fp[0] | fp[1] << 8); fp += 2; }
    cum[s] = c;
    c += freq[s];
  }
  if (c != ZO_SCALE) return -1;
  uint8_t slot[ZO_SCALE];
  for (int s = 0; s < 256; ++s)
    for (uint32_t k = 0; k < freq[s]; ++k) slot[cum[s] + k] = (uint8_t)s;
  const uint8_t *lens = fp, *data = fp + 4 * ZO_NLANES, *body_end = body + len;
  for (uint32_t j = 0; j < ZO_NLANES; ++j) {
    const uint32_t ll = rd32(lens + 4 * j);
    if ((size_t)(body_end - data) < ll || ll < 4) return -1;
    const uint8_t *in = data + 4, *in_end = data + ll;
    uint32_t x = rd32(data);
    for (uint32_t i = j; i < n; i += ZO_NLANES) {
      const uint32_t r = x & (ZO_SCALE - 1);
      const uint8_t s = slot[r];
      sym[i] = s;
      x = freq[s] * (x >> ZO_SCALE_BITS) + r - cum[s];
      while (x < ZO_LOW) {
        if (in >= in_end) return -1;
        x = (x << 8) | *in++;
      }
    }
    data += ll;
  }
  return 5 + (long)len;
}

/* ---------------------------------------------------------------- LZ77 parse (src/codec2.h:43-81)
 * 16-bit multiplicative hash of 4 bytes, chains walked `depth` steps, the longest match kept (the
 * nearest on a tie), one position of lazy look-ahead, matches capped at 4096 bytes.
 * Writes tokens (position, length, distance); returns how many. */
uint32_t zo_parse(const uint8_t *in, uint32_t n, int depth, uint32_t *tok_i, uint32_t *tok_m, uint32_t *tok_d) {
  if (n < 4) return 0;
  int32_t *head = (int32_t *)malloc(sizeof(int32_t) << 16);
  int32_t *chain = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  for (uint32_t h = 0; h < (1u << 16); ++h) head[h] = -1;
  uint32_t next_insert = 0, nt = 0;
#define ZO_HASH(at) ((rd32(in + (at)) * 2654435761u) >> 16)
  /* the best match at position i; every position before i is in the chains first */
#define ZO_BEST(i_, m_out, d_out)                                                          \
  do {                                                                                     \
    const uint32_t qi = (i_);                                                              \
    for (; next_insert < qi; ++next_insert) {                                              \
      if (next_insert + 4 > n) continue;                                                   \
      const uint32_t h = ZO_HASH(next_insert);                                             \
      chain[next_insert] = head[h];                                                        \
      head[h] = (int32_t)next_insert;                                                      \
    }                                                                                      \
    uint32_t best = 0, bd = 0;                                                             \
    if (qi + 4 <= n) {                                                                     \
      const uint32_t lim = (n - qi) < 4096u ? (n - qi) : 4096u;                            \
      int32_t j = head[ZO_HASH(qi)];                                                       \
      for (int step = 0; step < depth && j >= 0; ++step, j = chain[j]) {                   \
        /* a candidate that differs at the byte `best` cannot be longer: skip it */        \
        const uint32_t probe = best < lim - 1 ? best : lim - 1;                            \
        if (best && in[(uint32_t)j + probe] != in[qi + probe]) continue;                   \
        uint32_t l = 0;                                                                    \
        while (l < lim && in[(uint32_t)j + l] == in[qi + l]) ++l;                          \
        if (l > best) { best = l; bd = qi - (uint32_t)j; }                                \
      }                                                                                    \
    }                                                                                      \
    (m_out) = best >= 4 ? best : 0;                                                        \
    (d_out) = bd;                                                                          \
  } while (0)
  uint32_t i = 0;
  while (i < n) {
    uint32_t m, d;
    ZO_BEST(i, m, d);
    if (!m) { ++i; continue; }
    if (i + 1 < n) {
      uint32_t m2, d2;
      ZO_BEST(i + 1, m2, d2);
      /* 8*m2 - bits(d2) - 8 > 8*m - bits(d)  (src/codec2.h:76) */
      if (m2 && (int64_t)8 * m2 - bitlen(d2) - 8 > (int64_t)8 * m - bitlen(d)) { ++i; m = m2; d = d2; }
    }
    tok_i[nt] = i; tok_m[nt] = m; tok_d[nt] = d; ++nt;
    i += m;
  }
#undef ZO_BEST
#undef ZO_HASH
  free(head);
  free(chain);
  return nt;
}

/* ---------------------------------------------------------------- tokens -> payload (src/codec2.h:84-153)
 * Groups of at most 255 tokens; a match whose source reaches into its own group's output closes the group
 * first (the default cut_below = 0).  Offsets equal to one of the last three of the group before become
 * symbols 250..252.  Returns the payload size (the caller stores the block when that is >= n).
 * out must hold n + n/2 + 1024 bytes. */
size_t zo_build_payload(const uint8_t *in, uint32_t n, const uint32_t *tok_i, const uint32_t *tok_m, const uint32_t *tok_d,
                        uint32_t nt, uint8_t *out) {
  uint8_t *lit = (uint8_t *)malloc((size_t)n + 1), *tk = (uint8_t *)malloc((size_t)nt + 1);
  uint8_t *ext = (uint8_t *)malloc(5 * (size_t)nt + 1), *sy = (uint8_t *)malloc((size_t)nt + 1);
  uint8_t *grp = (uint8_t *)malloc((size_t)nt + 1), *bits = (uint8_t *)malloc(3 * (size_t)nt + 8);
  uint32_t nl = 0, ne = 0, ng = 0, nb = 0, op = 0, gstart = 0, gcount = 0;
  uint32_t cur[3] = {1, 4, 8}, last[3] = {1, 4, 8};
  uint64_t acc = 0;
  int acc_n = 0;
  for (uint32_t t = 0; t < nt; ++t) {
    const uint32_t i = tok_i[t], m = tok_m[t], d = tok_d[t];
    if (gcount == 255) { grp[ng++] = (uint8_t)gcount; gcount = 0; gstart = op; memcpy(cur, last, sizeof cur); }
    const uint32_t src = i - d, reach = src + (m < d ? m : d);
    if (src < op && reach > gstart) {
      if (gcount) grp[ng++] = (uint8_t)gcount;
      gcount = 0; gstart = op; memcpy(cur, last, sizeof cur);
    }
    const uint32_t L = i - op;
    memcpy(lit + nl, in + op, L);
    nl += L;
    tk[t] = (uint8_t)(((L < 15 ? L : 15) << 4) | (m - 4 < 15 ? m - 4 : 15));
    if (L >= 15) { const uint32_t v = L - 15; ext[ne++] = (uint8_t)v; ext[ne++] = (uint8_t)(v >> 8); ext[ne++] = (uint8_t)(v >> 16); }
    if (m >= 19) { const uint32_t v = m - 19; ext[ne++] = (uint8_t)v; ext[ne++] = (uint8_t)(v >> 8); }
    int r = 0;
    while (r < 3 && cur[r] != d) ++r;
    if (r < 3) {
      sy[t] = (uint8_t)(ZO_SYM_REP + r);
    } else {
      const uint32_t b = bitlen(d);
      sy[t] = (uint8_t)b;
      acc |= (uint64_t)(d - (1u << b)) << acc_n;
      acc_n += (int)b;
      while (acc_n >= 8) { bits[nb++] = (uint8_t)acc; acc >>= 8; acc_n -= 8; }
    }
    last[2] = last[1]; last[1] = last[0]; last[0] = d;
    ++gcount;
    op = i + m;
  }
  if (gcount) grp[ng++] = (uint8_t)gcount;
  memcpy(lit + nl, in + op, n - op);
  nl += n - op;
  if (acc_n) bits[nb++] = (uint8_t)acc;
  wr32(out, nt); wr32(out + 4, nl); wr32(out + 8, ne); wr32(out + 12, nb); wr32(out + 16, ng);
  size_t at = ZO_HDR;
  at += zo_encode_stream(lit, nl, out + at);
  at += zo_encode_stream(tk, nt, out + at);
  at += zo_encode_stream(ext, ne, out + at);
  at += zo_encode_stream(sy, nt, out + at);
  at += zo_encode_stream(grp, ng, out + at);
  memcpy(out + at, bits, nb);
  at += nb;
  free(lit); free(tk); free(ext); free(sy); free(grp); free(bits);
  return at;
}

/* zb2::compress_block (src/codec2.h:84-153) with Params{depth}; returns the payload size (stored when >= n) */
size_t zo_compress_block(const uint8_t *in, uint32_t n, int depth, uint8_t *out) {
  const size_t cap = (size_t)n / 4 + 1;
  uint32_t *ti = (uint32_t *)malloc(cap * 4), *tm = (uint32_t *)malloc(cap * 4), *td = (uint32_t *)malloc(cap * 4);
  const uint32_t nt = zo_parse(in, n, depth, ti, tm, td);
  const size_t r = zo_build_payload(in, n, ti, tm, td, nt, out);
  free(ti); free(tm); free(td);
  return r;
}

/* ---------------------------------------------------------------- payload -> bytes (src/codec2.h:155-203)
 * Returns 0, or -1 for a damaged block (every case where the reference throws). */
int zo_decompress_block(const uint8_t *in, size_t in_len, uint8_t *out, uint32_t n) {
  if (in_len < ZO_HDR) return -1;
  const uint32_t nt = rd32(in), nl = rd32(in + 4), ne = rd32(in + 8), nb = rd32(in + 12), ng = rd32(in + 16);
  if (nl > n || nt > n || (uint64_t)ne > 5 * (uint64_t)nt || ng > nt) return -1;
  uint8_t *lit = (uint8_t *)malloc((size_t)nl + 1), *tk = (uint8_t *)malloc((size_t)nt + 1);
  uint8_t *ext = (uint8_t *)malloc((size_t)ne + 4), *sy = (uint8_t *)malloc((size_t)nt + 1), *grp = (uint8_t *)malloc((size_t)ng + 1);
  int rc = -1;
  const uint8_t *p = in + ZO_HDR, *end = in + in_len;
  long k;
  if ((k = zo_decode_stream(p, (size_t)(end - p), nl, lit)) < 0) goto done;
  p += k;
  if ((k = zo_decode_stream(p, (size_t)(end - p), nt, tk)) < 0) goto done;
  p += k;
  if ((k = zo_decode_stream(p, (size_t)(end - p), ne, ext)) < 0) goto done;
  p += k;
  if ((k = zo_decode_stream(p, (size_t)(end - p), nt, sy)) < 0) goto done;
  p += k;
  if ((k = zo_decode_stream(p, (size_t)(end - p), ng, grp)) < 0) goto done;
  p += k;
  if ((size_t)(end - p) < nb) goto done;
  {
    const uint8_t *bits = p;
    uint32_t o = 0, li = 0, ei = 0, t = 0;
    uint64_t bp = 0;
    uint32_t cur[3] = {1, 4, 8}, last[3] = {1, 4, 8};
    for (uint32_t g = 0; g < ng; ++g) {
      const uint32_t cnt = grp[g];
      if (cnt == 0 || t + cnt > nt) goto done;
      for (uint32_t q = 0; q < cnt; ++q, ++t) {
        uint32_t L = tk[t] >> 4, M = (tk[t] & 15u) + 4;
        if (L == 15) { if (ei + 3 > ne) goto done; L += (uint32_t)ext[ei] | (uint32_t)ext[ei + 1] << 8 | (uint32_t)ext[ei + 2] << 16; ei += 3; }
        if ((tk[t] & 15u) == 15) { if (ei + 2 > ne) goto done; M += (uint32_t)ext[ei] | (uint32_t)ext[ei + 1] << 8; ei += 2; }
        const uint32_t s = sy[t];
        uint32_t D;
        if (s >= ZO_SYM_REP) {
          if (s > ZO_SYM_REP + 2) goto done;
          D = cur[s - ZO_SYM_REP];
        } else {
          if (s > 19) goto done;
          uint32_t x = 0;
          for (uint32_t b = 0; b < s; ++b, ++bp) {
            if ((bp >> 3) >= nb) goto done;
            x |= (uint32_t)((bits[bp >> 3] >> (bp & 7)) & 1u) << b;
          }
          D = (1u << s) + x;
        }
        if (li + L > nl || (uint64_t)o + L + M > n || D == 0 || D > o + L) goto done;
        memcpy(out + o, lit + li, L);
        o += L; li += L;
        for (uint32_t c = 0; c < M; ++c) out[o + c] = out[o + c - D];
        o += M;
        last[2] = last[1]; last[1] = last[0]; last[0] = D;
      }
      memcpy(cur, last, sizeof cur);
    }
    if (t != nt || o + (nl - li) != n) goto done;
    memcpy(out + o, lit + li, nl - li);
    rc = 0;
  }
done:
  free(lit); free(tk); free(ext); free(sy); free(grp);
  return rc;
}

/* the CPU codec's level -> hash chain depth (src/main.cpp:45, 54) */
int zo_depth_for_level(int level) { return level <= 1 ? 8 : level >= 9 ? 256 : 32; }
