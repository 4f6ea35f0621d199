// zc_decode.cu -- the ZB2 block decoder's front end on sm_100a.
//
//   k_dec_locate   one thread per block: reads the payload's counts and the five stream headers that
//                  follow one another, checks them against the caps of a valid block and the payload's
//                  length, and records each stream body's offset and length (DecMeta).
//   k_dec_streams  grid (nb, 5) x 64 threads: one CTA per (block, stream).  Builds the 4096-slot decode
//                  table in shared memory and runs the 64 rANS lanes side by side (src/codec.h:150-205);
//                  raw streams are copied.
//   k_crc_blocks   one CTA per block: CRC-32 of each block (the record checksum).
// The LZ replay that follows is in zc_decode_fill.cu (k_dec_tokens, k_dec_fill).
//
// Damaged input can never make a kernel touch memory outside its block's buffers: every count is
// checked against the block's caps before it sizes a loop or an index, and a failing check records a
// status code in err[b] (no trap, no assert).  The host turns a nonzero status into ZC_E_DATA.
#include "zc_internal.cuh"
#include "zc_kernels.h"

namespace zc {

__device__ __forceinline__ void set_err(uint32_t* err, uint32_t b, uint32_t code) { atomicCAS(err + b, 0u, code); }

// ---------------------------------------------------------------- framing
// The payload (src/codec2.h:14-17): 20 bytes of counts {tokens, literals, ext bytes, offset-bit bytes,
// groups}, then the streams lit, tok, ext, sym, groups, each a u8 kind (0 raw, 1 rANS), a u32 body length
// and the body (src/codec.h:130-147), then the offset bits.  A raw body holds exactly its stream's
// symbols; a rANS body at least its presence bitmap and lane lengths.
__global__ void __launch_bounds__(256) k_dec_locate(DecArgs A) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= A.nb || A.method[b] != 1) return;  // (stored blocks and unknown methods: k_dec_fill)
  const uint32_t raw = A.raw_len[b], clen = A.comp_len[b], B = A.B;
  DecMeta m{};
  uint32_t code = 0;
  if (raw > B) {
    code = E_RAWLEN;
  } else if (clen < kHdrBytes) {
    code = E_HDR;
  } else {
    const uint8_t* p = A.comp + A.comp_off[b];
    m.nt = ld32(p); m.nl = ld32(p + 4); m.ne = ld32(p + 8); m.nob = ld32(p + 12); m.ng = ld32(p + 16);
    // the reference's count checks (src/codec2.h:161), and the caps every valid block respects
    if (m.nl > raw || m.nt > raw / 4 || (uint64_t)m.ne > 5ull * m.nt || m.ne > ext_cap(B) || m.ng > m.nt) code = E_COUNTS;
    const uint32_t want[5] = {m.nl, m.nt, m.ne, m.nt, m.ng};
    uint64_t at = kHdrBytes;
    for (uint32_t s = 0; s < 5 && !code; ++s) {
      if (at + 5 > clen) { code = E_STREAM; break; }
      const uint32_t kind = p[at], len = ld32(p + at + 1);
      at += 5;
      if (at + len > clen || (kind == 0 && len != want[s]) || (kind == 1 && len < 32 + 4 * kLanes) || kind > 1) {
        code = E_STREAM;
        break;
      }
      m.s_off[s] = (uint32_t)at;
      m.s_len[s] = len;
      m.kinds |= kind << s;
      at += len;
    }
    if (!code && at + m.nob > clen) code = E_STREAM;
    m.bits_off = (uint32_t)at;
  }
  A.meta[b] = m;
  if (code) set_err(A.err, b, code);
}

// ---------------------------------------------------------------- streams
__global__ void __launch_bounds__(64) k_dec_streams(DecArgs A) {
  const uint32_t b = blockIdx.x, s = blockIdx.y, k = threadIdx.x;
  if (A.method[b] != 1 || A.err[b]) return;  // (framing checked by k_dec_locate)
  const uint32_t B = A.B;
  __shared__ uint32_t tab[kScale];
  __shared__ uint32_t freq[256], cum[257];
  __shared__ uint32_t lstart[kLanes + 1];
  __shared__ uint32_t wsum[2];
  __shared__ uint32_t fail;
  const DecMeta& mm = A.meta[b];
  const uint32_t len = mm.s_len[s], kind = (mm.kinds >> s) & 1u;
  const uint8_t* body = A.comp + A.comp_off[b] + mm.s_off[s];
  const size_t TC = tok_cap(B), EC = ext_cap(B);
  uint8_t* dest;
  uint32_t ns;
  switch (s) {
    case 0: dest = A.s_lit + (size_t)b * B; ns = mm.nl; break;
    case 1: dest = A.s_tok + (size_t)b * TC; ns = mm.nt; break;
    case 2: dest = A.s_ext + (size_t)b * EC; ns = mm.ne; break;
    case 3: dest = A.s_sym + (size_t)b * TC; ns = mm.nt; break;
    default: dest = A.s_grp + (size_t)b * TC; ns = mm.ng; break;
  }
  if (kind == 0) {  // raw: len == ns
    for (uint32_t i = k; i < ns; i += 64) dest[i] = body[i];
    return;
  }
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

void launch_dec_streams(const DecArgs& A, cudaStream_t st, Stages& S) {
  if (!A.nb) return;
  S.begin("k_dec_locate", st);
  k_dec_locate<<<(A.nb + 255) / 256, 256, 0, st>>>(A);
  S.end(st);
  S.begin("k_dec_streams", st);
  k_dec_streams<<<dim3(A.nb, 5), 64, 0, st>>>(A);
  S.end(st);
}

void launch_crc(const CrcArgs& A, cudaStream_t st, Stages& S, const char* name) {
  if (!A.nb) return;
  S.begin(name, st);
  k_crc_blocks<<<A.nb, 256, 0, st>>>(A);
  S.end(st);
}

}  // namespace zc
