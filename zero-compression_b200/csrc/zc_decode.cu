// zc_decode.cu -- the ZB2 block decoder on sm_100a.
//
//   k_dec_streams  grid (nb, 5) x 64 threads: one CTA per (block, stream).  Locates the stream in the
//                  payload, builds the 4096-slot decode table in shared memory and runs the 64 rANS
//                  lanes side by side (src/codec.h:150-205).  Raw streams are copied.
//   k_dec_lz       one warp per block: replays the tokens group by group, 32 tokens at a time, one
//                  token per lane; a warp fence only between groups (src/codec2.h:155-203).  Stored
//                  blocks are copied here.
//   k_crc_blocks   one CTA per block: CRC-32 of each block's output (the record checksum).
//
// Damaged input can never make a kernel touch memory outside its block's buffers: every count is
// checked against the block's caps before it sizes a loop or an index, and a failing check records a
// status code in err[b] (no trap, no assert).  The host turns a nonzero status into ZC_E_DATA.
#include "zc_internal.cuh"
#include "zc_kernels.h"

namespace zc {

__device__ __forceinline__ void set_err(uint32_t* err, uint32_t b, uint32_t code) { atomicCAS(err + b, 0u, code); }

// ---------------------------------------------------------------- streams
__global__ void __launch_bounds__(64) k_dec_streams(DecArgs A) {
  const uint32_t b = blockIdx.x, s = blockIdx.y, k = threadIdx.x;
  if (A.method[b] != 1) return;
  const uint32_t raw = A.raw_len[b], clen = A.comp_len[b], B = A.B;
  __shared__ uint32_t tab[kScale];
  __shared__ uint32_t freq[256], cum[257];
  __shared__ uint32_t lstart[kLanes + 1];
  __shared__ uint32_t wsum[2];
  __shared__ uint32_t fail;
  if (raw > B) { if (k == 0 && s == 0) set_err(A.err, b, E_RAWLEN); return; }
  if (clen < kHdrBytes) { if (k == 0 && s == 0) set_err(A.err, b, E_HDR); return; }
  const uint8_t* p = A.comp + A.comp_off[b];
  const uint32_t nt = ld32(p), nl = ld32(p + 4), ne = ld32(p + 8), nob = ld32(p + 12), ng = ld32(p + 16);
  // the reference's count checks (src/codec2.h:161) and the caps every valid block respects
  if (nl > raw || nt > raw || (uint64_t)ne > 5ull * nt || ng > nt || nt > raw / 4 || ne > ext_cap(B)) {
    if (k == 0 && s == 0) set_err(A.err, b, E_COUNTS);
    return;
  }
  uint64_t pos = kHdrBytes;
  for (uint32_t t = 0; t < s; ++t) {
    if (pos + 5 > clen) { if (k == 0) set_err(A.err, b, E_STREAM); return; }
    pos += 5ull + ld32(p + pos + 1);
  }
  if (pos + 5 > clen) { if (k == 0) set_err(A.err, b, E_STREAM); return; }
  const uint32_t kind = p[pos], len = ld32(p + pos + 1);
  if (pos + 5 + len > clen) { if (k == 0) set_err(A.err, b, E_STREAM); return; }
  const uint8_t* body = p + pos + 5;
  if (s == 4 && k == 0) {
    DecMeta m;
    m.nt = nt; m.nl = nl; m.ne = ne; m.nob = nob; m.ng = ng; m.bits_off = (uint32_t)(pos + 5 + len);
    A.meta[b] = m;
    if ((uint64_t)m.bits_off + nob > clen) set_err(A.err, b, E_STREAM);
  }
  uint8_t* dest;
  uint32_t ns;
  const size_t TC = tok_cap(B), EC = ext_cap(B);
  switch (s) {
    case 0: dest = A.s_lit + (size_t)b * B; ns = nl; break;
    case 1: dest = A.s_tok + (size_t)b * TC; ns = nt; break;
    case 2: dest = A.s_ext + (size_t)b * EC; ns = ne; break;
    case 3: dest = A.s_sym + (size_t)b * TC; ns = nt; break;
    default: dest = A.s_grp + (size_t)b * TC; ns = ng; break;
  }
  if (kind == 0) {
    if (len != ns) { if (k == 0) set_err(A.err, b, E_STREAM); return; }
    for (uint32_t i = k; i < ns; i += 64) dest[i] = body[i];
    return;
  }
  if (kind != 1 || len < 32 + 4 * kLanes) { if (k == 0) set_err(A.err, b, E_STREAM); return; }
  // present bitmap -> frequency index of each symbol: thread k owns symbols 4k..4k+3
  const uint32_t bits4 = (body[k >> 1] >> ((k & 1u) * 4)) & 15u;
  const uint32_t cnt = __popc(bits4);
  const uint32_t incl = warp_incl_scan(cnt);
  if (lane_id() == 31) wsum[k >> 5] = incl;
  if (k == 0) fail = 0;
  __syncthreads();
  const uint32_t np = wsum[0] + wsum[1];
  const uint32_t idx0 = incl - cnt + (k >= 32 ? wsum[0] : 0);
  const uint32_t hdr = 32 + 2 * np + 4 * kLanes;
  if (len < hdr) { if (k == 0) set_err(A.err, b, E_STREAM); return; }
  const uint8_t* fp = body + 32;
  uint32_t f4[4], idx = idx0, fsum = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    f4[q] = 0;
    if ((bits4 >> q) & 1u) { f4[q] = (uint32_t)fp[2 * idx] | (uint32_t)fp[2 * idx + 1] << 8; ++idx; }
    fsum += f4[q];
  }
  const uint32_t fincl = warp_incl_scan(fsum);
  __syncthreads();
  if (lane_id() == 31) wsum[k >> 5] = fincl;
  __syncthreads();
  uint32_t c0 = fincl - fsum + (k >= 32 ? wsum[0] : 0);
  const uint32_t total = wsum[0] + wsum[1];
#pragma unroll
  for (int q = 0; q < 4; ++q) { freq[4 * k + q] = f4[q]; cum[4 * k + q] = c0; c0 += f4[q]; }
  if (k == 0) cum[256] = total;
  // lane lengths: each at least 4, all inside the body
  const uint8_t* lens = fp + 2 * np;
  const uint32_t ll = ld32(lens + 4 * k);
  __syncthreads();
  if (total != kScale) { if (k == 0) set_err(A.err, b, E_TABLE); return; }
  {
    uint64_t acc = ll;  // inclusive prefix of lane lengths in 64-bit (damaged lengths may be huge)
    const uint32_t l = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t t = __shfl_up_sync(kFull, acc, o);
      if (l >= (uint32_t)o) acc += t;
    }
    __shared__ uint64_t w64[2];
    if (l == 31) w64[k >> 5] = acc;
    __syncthreads();
    if (k >= 32) acc += w64[0];
    const uint64_t room = len - hdr;
    if (ll < 4 || acc > room) atomicOr(&fail, 1u);
    lstart[k] = (uint32_t)(acc - ll);
  }
  // decode table: slot -> (symbol, freq - 1, slot - cum)
  {
    const uint32_t s0 = k * 64;
    uint32_t lo = 0, hi = 256;  // last symbol with cum <= s0
    while (hi - lo > 1) { const uint32_t mid = (lo + hi) >> 1; if (cum[mid] <= s0) lo = mid; else hi = mid; }
    __syncthreads();
    uint32_t sym = lo;
    for (uint32_t sl = s0; sl < s0 + 64; ++sl) {
      while (sl >= cum[sym + 1]) ++sym;
      tab[sl] = sym | ((freq[sym] - 1u) << 8) | ((sl - cum[sym]) << 20);
    }
  }
  __syncthreads();
  if (fail) { if (k == 0) set_err(A.err, b, E_LANE); return; }
  // 64 lanes: lane k decodes symbols k, k+64, ...  The lane's bytes come through a register buffer filled
  // from aligned words, the next word loaded at least two symbols before it is needed (a symbol takes at
  // most two bytes); the words may extend up to 8 bytes past the lane, inside the input's readable slack.
  const uint8_t* in = body + hdr + lstart[k];
  uint32_t x = ld32(in);
  in += 4;
  uint32_t rem = ll - 4;  // the lane's bytes not yet taken
  const uint32_t* wp = reinterpret_cast<const uint32_t*>((uintptr_t)in & ~(uintptr_t)3);
  const uint32_t skip = (uint32_t)((uintptr_t)in & 3u);
  uint64_t buf = __ldg(wp) >> (8 * skip);
  uint32_t nbuf = 4 - skip;
  uint32_t nxt = __ldg(wp + 1);
  wp += 1;
  for (uint32_t i = k; i < ns; i += kLanes) {
    if (nbuf < 4) {
      buf |= (uint64_t)nxt << (8 * nbuf);
      nbuf += 4;
      nxt = __ldg(++wp);
    }
    const uint32_t e = tab[x & (kScale - 1)];
    dest[i] = (uint8_t)e;
    x = (((e >> 8) & 0xFFFu) + 1u) * (x >> kScaleBits) + (e >> 20);
    while (x < kRansLow) {
      if (rem == 0) { set_err(A.err, b, E_LANE); return; }
      x = (x << 8) | (uint32_t)(buf & 0xFFu);
      buf >>= 8;
      --nbuf;
      --rem;
    }
  }
}

// ---------------------------------------------------------------- LZ replay
// A chunk of at most 32 tokens of one group, as the warp's shared table: output start, match start,
// offset and literal start of each token (start[c] = the chunk's end).
struct ChunkTable {
  uint32_t start[33], ms[32], dist[32], lik[32];
};

// the byte at output position q of token k: its own literal, or a match byte, whose source is output
// from before the group or this token's own literals (src/codec2.h:1-6); an overlapping match (D < M)
// repeats the D bytes before it, so the source of match byte i is ms - D + (i mod D)
__device__ __forceinline__ uint32_t chunk_byte(const ChunkTable& T, const uint8_t* o, const uint8_t* lit, uint32_t q,
                                               uint32_t k) {
  const uint32_t opk = T.start[k], ms = T.ms[k];
  if (q < ms) return lit[T.lik[k] + (q - opk)];
  const uint32_t D = T.dist[k];
  uint32_t s = q - D;
  if (s >= ms) s = ms - D + (q - ms) % D;
  return s >= opk ? lit[T.lik[k] + (s - opk)] : o[s];
}

// all lanes fill the chunk's output [op, op_end): 4 bytes each per round, whole aligned words stored as
// words.  No byte of a group depends on another byte of the same group, so the order is free.
__device__ __forceinline__ void fill_chunk(const ChunkTable& T, uint8_t* o, const uint8_t* lit, uint32_t c,
                                          uint32_t op, uint32_t op_end) {
  const uintptr_t ob = (uintptr_t)o;
  const int64_t qa = (int64_t)(((ob + op) & ~(uintptr_t)3) - ob);
  for (int64_t q0 = qa + 4 * (int64_t)lane_id(); q0 < (int64_t)op_end; q0 += 128) {
    const uint32_t qs = (uint32_t)(q0 > (int64_t)op ? q0 : (int64_t)op);
    uint32_t lo = 0, hi = c;  // start[lo] <= qs < start[hi]
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (T.start[mid] <= qs) lo = mid; else hi = mid;
    }
    uint32_t k = lo, w = 0;
    const bool full = q0 >= (int64_t)op && q0 + 4 <= (int64_t)op_end;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t q = q0 + j;
      if (q < (int64_t)op || q >= (int64_t)op_end) continue;
      while ((uint32_t)q >= T.start[k + 1]) ++k;
      const uint32_t v = chunk_byte(T, o, lit, (uint32_t)q, k);
      if (full) w |= v << (8 * j);
      else o[q] = (uint8_t)v;
    }
    if (full) *reinterpret_cast<uint32_t*>(o + q0) = w;
  }
}
// a warp copies n bytes, coalesced (src and dst do not overlap)
__device__ inline void warp_copy(uint8_t* d, const uint8_t* s, uint32_t n) {
  const uint32_t l = lane_id();
  uint32_t i = 0;
  if ((((uintptr_t)d ^ (uintptr_t)s) & 15u) == 0) {
    const uint32_t head = (uint32_t)((16u - ((uintptr_t)d & 15u)) & 15u);
    if (l < head && l < n) d[l] = s[l];
    i = head < n ? head : n;
    for (uint32_t j = i + 16 * l; j + 16 <= n; j += 16 * 32)
      *reinterpret_cast<uint4*>(d + j) = *reinterpret_cast<const uint4*>(s + j);
    i += (n - i) & ~15u;
  }
  for (uint32_t j = i + l; j < n; j += 32) d[j] = s[j];
}

__global__ void __launch_bounds__(128) k_dec_lz(DecArgs A) {
  __shared__ ChunkTable tables[4];
  const uint32_t b = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (b >= A.nb) return;
  ChunkTable& T = tables[threadIdx.x >> 5];
  const uint32_t lane = lane_id();
  const uint32_t raw = A.raw_len[b], method = A.method[b], clen = A.comp_len[b], B = A.B;
  uint8_t* o = A.out + A.out_off[b];
  const uint8_t* p = A.comp + A.comp_off[b];
  if (raw > B) { if (lane == 0) set_err(A.err, b, E_RAWLEN); return; }
  if (method == 0) {
    if (clen != raw) { if (lane == 0) set_err(A.err, b, E_STORED); return; }
    warp_copy(o, p, raw);
    return;
  }
  if (method != 1) { if (lane == 0) set_err(A.err, b, E_METHOD); return; }
  if (A.err[b]) return;
  const DecMeta m = A.meta[b];
  const size_t TC = tok_cap(B), EC = ext_cap(B);
  const uint8_t* lit = A.s_lit + (size_t)b * B;
  const uint8_t* tok = A.s_tok + (size_t)b * TC;
  const uint8_t* sym = A.s_sym + (size_t)b * TC;
  const uint8_t* grp = A.s_grp + (size_t)b * TC;
  const uint8_t* ext = A.s_ext + (size_t)b * EC;
  const uint8_t* bits = p + m.bits_off;
  const uint64_t nbits = 8ull * m.nob;
  uint32_t t = 0, op = 0, li = 0, ei = 0;
  uint64_t bp = 0;
  uint32_t r0 = 1, r1 = 4, r2 = 8, l0 = 1, l1 = 4, l2 = 8;
  for (uint32_t g = 0; g < m.ng; ++g) {
    const uint32_t gn = grp[g];
    if (gn == 0 || t + gn > m.nt) { if (lane == 0) set_err(A.err, b, E_TOKEN); return; }
    const uint32_t tend = t + gn;
    while (t < tend) {
      const uint32_t c = min(32u, tend - t);
      const bool on = lane < c;
      const uint32_t tv = on ? tok[t + lane] : 0u, sv = on ? sym[t + lane] : 0u;
      const uint32_t fl = on && (tv >> 4) == 15u, fm = on && (tv & 15u) == 15u;
      const uint32_t nx = 3u * fl + 2u * fm;
      const uint32_t xincl = warp_incl_scan(nx);
      const uint32_t xq = ei + xincl - nx;
      bool bad = on && (uint64_t)xq + nx > m.ne;
      uint32_t L = tv >> 4, M = on ? (tv & 15u) + 4u : 0u;
      if (!bad && fl) L += (uint32_t)ext[xq] | (uint32_t)ext[xq + 1] << 8 | (uint32_t)ext[xq + 2] << 16;
      if (!bad && fm) { const uint32_t q = xq + 3u * fl; M += (uint32_t)ext[q] | (uint32_t)ext[q + 1] << 8; }
      if (on && sv > 19u && (sv < kSymRep || sv > kSymRep + 2)) bad = true;
      const uint32_t nbit = (on && sv <= 19u) ? sv : 0u;
      const uint32_t bincl = warp_incl_scan(nbit);
      const uint64_t bq = bp + bincl - nbit;
      uint32_t D = 0;
      if (on && !bad) {
        if (sv >= kSymRep) {
          D = sv == kSymRep ? r0 : sv == kSymRep + 1 ? r1 : r2;
        } else if (bq + nbit > nbits) {
          bad = true;
        } else {
          uint32_t x = 0;
          if (nbit) {
            const uint32_t j0 = (uint32_t)(bq >> 3), j1 = (uint32_t)((bq + nbit - 1) >> 3);
            uint64_t w = 0;
            for (uint32_t j = j0; j <= j1; ++j) w |= (uint64_t)bits[j] << (8 * (j - j0));
            x = (uint32_t)(w >> (bq & 7u)) & ((1u << nbit) - 1u);
          }
          D = (1u << sv) + x;
        }
      }
      const uint32_t tot = L + M;
      const uint32_t oincl = warp_incl_scan(tot), lincl = warp_incl_scan(L);
      const uint32_t opk = op + oincl - tot, lik = li + lincl - L;
      const uint32_t ms = opk + L;
      if (on && ((uint64_t)lik + L > m.nl || (uint64_t)opk + tot > raw || D == 0 || D > ms)) bad = true;
      if (__any_sync(kFull, bad)) { if (lane == 0) set_err(A.err, b, E_TOKEN); return; }
      const uint32_t op_end = op + __shfl_sync(kFull, oincl, 31);
      if (on) { T.start[lane] = opk; T.ms[lane] = ms; T.dist[lane] = D; T.lik[lane] = lik; }
      if (lane == 0) T.start[c] = op_end;
      __syncwarp();
      fill_chunk(T, o, lit, c, op, op_end);
      __syncwarp();
      op = op_end;
      li += __shfl_sync(kFull, lincl, 31);
      ei += __shfl_sync(kFull, xincl, 31);
      bp += __shfl_sync(kFull, bincl, 31);
      for (uint32_t q = c > 3u ? c - 3u : 0u; q < c; ++q) {
        const uint32_t v = __shfl_sync(kFull, D, q);
        l2 = l1; l1 = l0; l0 = v;
      }
      t += c;
    }
    r0 = l0; r1 = l1; r2 = l2;
    __syncwarp();
  }
  if (t != m.nt || op + (m.nl - li) != raw) { if (lane == 0) set_err(A.err, b, E_TOKEN); return; }
  warp_copy(o + op, lit + li, m.nl - li);
}

// ---------------------------------------------------------------- CRC of each block
__global__ void __launch_bounds__(256) k_crc_blocks(CrcArgs A) {
  const uint32_t b = blockIdx.x;
  __shared__ uint32_t t[8][256];
  __shared__ uint32_t red[8];
  if (A.err && A.err[b]) return;
  load_crc_tables(A.tables, t);
  __syncthreads();
  const uint32_t crc = cta_crc32(A.tables, t, A.base + A.offs[b], A.lens[b], red);
  if (threadIdx.x == 0) {
    A.crc[b] = crc;
    if (A.expect && A.err && A.expect[b] != crc) A.err[b] = E_CRC;
  }
}

void launch_decode(const DecArgs& A, cudaStream_t st, Stages& S) {
  if (!A.nb) return;
  S.begin("k_dec_streams", st);
  k_dec_streams<<<dim3(A.nb, 5), 64, 0, st>>>(A);
  S.end(st);
  S.begin("k_dec_lz", st);
  k_dec_lz<<<(A.nb + 3) / 4, 128, 0, st>>>(A);
  S.end(st);
}

void launch_dec_streams(const DecArgs& A, cudaStream_t st) {
  if (A.nb) k_dec_streams<<<dim3(A.nb, 5), 64, 0, st>>>(A);
}

void launch_crc(const CrcArgs& A, cudaStream_t st, Stages& S, const char* name) {
  if (!A.nb) return;
  S.begin(name, st);
  k_crc_blocks<<<A.nb, 256, 0, st>>>(A);
  S.end(st);
}

}  // namespace zc
