// zc_decode_fill.cu -- the ZB2 LZ replay in two kernels (src/codec2.h:155-203):
//
//   k_dec_tokens  one CTA of 1024 threads per block: every token's literal run and match length (ext
//                 bytes), offset (offset bits), output start and literal start, from block-wide scans, in
//                 parallel over the tokens; then the groups (a scan of their counts) and the recent-offset
//                 symbols (each names an earlier token's offset, src/codec2.h:180-192), resolved by pointer
//                 jumping over all tokens at once.  Every check of the reference decoder is made here; a
//                 failing one records a status and the block is not replayed.
//   k_dec_fill    one warp per block: fills the block in rounds of 128 output bytes (a 4-byte word a lane)
//                 straight through, group boundaries or not: a byte whose source lies earlier in the same
//                 round is passed along by shuffles once known; the token table is a 64-row ring in shared
//                 memory, refilled 32 tokens at a time from registers loaded one window ahead.
// Stored blocks are copied by k_dec_fill.  The rANS streams come from k_dec_streams (zc_decode.cu).
#include <algorithm>

#include "zc_internal.cuh"
#include "zc_kernels.h"

namespace zc {

namespace {

__device__ __forceinline__ void flag(uint32_t* err, uint32_t b, uint32_t code) { atomicCAS(err + b, 0u, code); }

// exclusive scan over the CTA (blockDim.x == 1024); returns the prefix, `total` gets the sum.  ws: 32 words
__device__ __forceinline__ uint32_t cta_scan(uint32_t v, uint32_t* ws, uint32_t& total) {
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint32_t inc = warp_incl_scan(v);
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  if (w == 0) {
    const uint32_t x = ws[lane];
    const uint32_t xi = warp_incl_scan(x);
    ws[lane] = xi - x;
    if (lane == 31) ws[32] = xi;
  }
  __syncthreads();
  const uint32_t r = ws[w] + inc - v;
  total = ws[32];
  __syncthreads();
  return r;
}

constexpr uint32_t kRepMark = 0x80000000u;  // a recent-offset symbol not resolved yet: kRepMark | index
constexpr uint32_t kGrpStart = 0x40000000u; // (while groups are scanned) the first token of a group

// inclusive max over the CTA in thread order (blockDim.x == 1024); `total` gets the CTA's max.  ws: 33 words
__device__ __forceinline__ uint32_t cta_max_incl(uint32_t v, uint32_t* ws, uint32_t& total) {
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= (uint32_t)o) x = max(x, y);
  }
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t z = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, z, o);
      if (lane >= (uint32_t)o) z = max(z, y);
    }
    ws[lane] = z;  // inclusive over warps
  }
  __syncthreads();
  const uint32_t r = w ? max(x, ws[w - 1]) : x;
  total = ws[31];
  __syncthreads();
  return r;
}

}  // namespace

__global__ void __launch_bounds__(1024, 2) k_dec_tokens(DecArgs A) {
  const uint32_t b = blockIdx.x, tid = threadIdx.x;
  if (A.method[b] != 1 || A.raw_len[b] > A.B || A.err[b]) return;
  __shared__ uint32_t ws[33];
  __shared__ uint32_t any_bad;
  const DecMeta m = A.meta[b];
  const uint32_t raw = A.raw_len[b], B = A.B;
  const size_t TC = tok_cap(B), EC = ext_cap(B);
  const uint8_t* tok = A.s_tok + (size_t)b * TC;
  const uint8_t* sym = A.s_sym + (size_t)b * TC;
  const uint8_t* grp = A.s_grp + (size_t)b * TC;
  const uint8_t* ext = A.s_ext + (size_t)b * EC;
  const uint8_t* bits = A.comp + A.comp_off[b] + m.bits_off;
  const uint64_t nbits = 8ull * m.nob;
  uint32_t* Ts = A.tk_start + (size_t)b * TC;
  uint32_t* Tm = A.tk_ms + (size_t)b * TC;
  uint32_t* Td = A.tk_d + (size_t)b * TC;
  uint32_t* Tl = A.tk_lik + (size_t)b * TC;
  if (tid == 0) any_bad = 0;
  __syncthreads();
  // ---- lengths, offsets and positions, 1024 tokens a tile
  uint32_t ei = 0, bp = 0, op = 0, li = 0;
  bool bad = false;
  for (uint32_t t0 = 0; t0 < m.nt; t0 += 1024) {
    const uint32_t t = t0 + tid;
    const bool on = t < m.nt;
    const uint32_t tv = on ? tok[t] : 0u, sv = on ? sym[t] : 0u;
    const uint32_t fl = on && (tv >> 4) == 15u, fm = on && (tv & 15u) == 15u;
    const uint32_t nx = 3u * fl + 2u * fm;
    const uint32_t nbit = (on && sv <= 19u) ? sv : 0u;
    if (on && sv > 19u && (sv < kSymRep || sv > kSymRep + 2)) bad = true;
    uint32_t tsum;
    const uint32_t pre = cta_scan(nx | nbit << 16, ws, tsum);  // (each part of a tile's sum fits 16 bits)
    const uint32_t xq = ei + (pre & 0xFFFFu), bq = bp + (pre >> 16);
    ei += tsum & 0xFFFFu;
    bp += tsum >> 16;
    if (on && (uint64_t)xq + nx > m.ne) bad = true;
    if (on && (uint64_t)bq + nbit > nbits) bad = true;
    uint32_t L = tv >> 4, M = on ? (tv & 15u) + 4u : 0u;
    if (!bad && fl) L += (uint32_t)ext[xq] | (uint32_t)ext[xq + 1] << 8 | (uint32_t)ext[xq + 2] << 16;
    if (!bad && fm) { const uint32_t q = xq + 3u * fl; M += (uint32_t)ext[q] | (uint32_t)ext[q + 1] << 8; }
    uint32_t D = 0;
    if (on && !bad) {
      if (sv >= kSymRep) {
        D = kRepMark | (sv - kSymRep);
      } else {
        uint32_t x = 0;
        if (nbit) {
          const uint32_t j0 = bq >> 3, j1 = (bq + nbit - 1) >> 3;
          uint64_t w = 0;
          for (uint32_t j = j0; j <= j1; ++j) w |= (uint64_t)bits[j] << (8 * (j - j0));
          x = (uint32_t)(w >> (bq & 7u)) & ((1u << nbit) - 1u);
        }
        D = (1u << sv) + x;
      }
    }
    uint32_t lsum, osum;
    const uint32_t lpre = cta_scan(L, ws, lsum);
    const uint32_t opre = cta_scan(L + M, ws, osum);
    const uint32_t opk = op + opre, lik = li + lpre;
    if (on && ((uint64_t)lik + L > m.nl || (uint64_t)opk + L + M > raw)) bad = true;
    if (on) { Ts[t] = opk; Tm[t] = opk + L; Tl[t] = lik; Td[t] = D; }
    op += osum;
    li += lsum;
  }
  if (bad) any_bad = 1;
  __syncthreads();
  // ---- groups and recent offsets (src/codec2.h:179-199).  A recent-offset symbol r of a group whose first
  //      token is gs names the offset of token gs - 1 - r (the last three offsets before the group,
  //      nearest first), or the initial 1, 4, 8 when r >= gs.  So: group starts (a scan of the group
  //      counts) flag their first tokens; a max-scan gives each token its group's start; each recent-
  //      offset token then points at the token it names, and pointer jumping resolves chains of them.
  __syncthreads();
  if (!any_bad) {
    uint32_t gbase = 0;
    for (uint32_t g0 = 0; g0 < m.ng; g0 += 1024) {
      const uint32_t g = g0 + tid;
      const uint32_t c = g < m.ng ? grp[g] : 0u;
      uint32_t tot;
      const uint32_t at = gbase + cta_scan(c, ws, tot);
      if (g < m.ng && (c == 0 || (uint64_t)at + c > m.nt)) bad = true;
      else if (g < m.ng) Td[at] |= kGrpStart;
      gbase += tot;
    }
    if (gbase != m.nt) bad = true;
  }
  if (bad) any_bad = 1;
  __syncthreads();
  if (!any_bad) {
    uint32_t carry = 0;
    for (uint32_t t0 = 0; t0 < m.nt; t0 += 1024) {
      const uint32_t t = t0 + tid;
      const bool on = t < m.nt;
      uint32_t v = on ? Td[t] : 0u;
      uint32_t tmax;
      const uint32_t gs = max(carry, cta_max_incl(on && (v & kGrpStart) ? t : 0u, ws, tmax));
      carry = max(carry, tmax);
      if (on) {
        v &= ~kGrpStart;
        if (v & kRepMark) {
          const uint32_t r = v & 3u;
          v = r < gs ? kRepMark | (gs - 1u - r) : (r - gs == 0 ? 1u : r - gs == 1 ? 4u : 8u);
        }
        Td[t] = v;
      }
    }
  }
  __syncthreads();
  if (!any_bad) {
    for (int round = 0; round < 32; ++round) {  // (a chain halves each round: at most 20 for 2^20 tokens)
      bool more = false;
      for (uint32_t t = tid; t < m.nt; t += 1024) {
        const uint32_t v = Td[t];
        if (v & kRepMark) {
          const uint32_t w = Td[v & ~kRepMark];
          Td[t] = w;
          more |= (w & kRepMark) != 0;
        }
      }
      if (!__syncthreads_or(more)) break;
    }
    for (uint32_t t = tid; t < m.nt; t += 1024) {
      const uint32_t D = Td[t];
      if ((D & kRepMark) || D == 0 || D > Tm[t]) bad = true;
    }
    if (bad) any_bad = 1;
  }
  __syncthreads();
  if (tid == 0) {
    if (any_bad || op + (m.nl - li) != raw) flag(A.err, b, E_TOKEN);
    A.meta[b].op_total = op;
    A.meta[b].li_total = li;
  }
}

namespace {

// The warp's token table: a ring of TR rows, token t in row t % TR.  start = the token's output start;
// tk = {match start, literal start - output start (mod 2^32), offset D, the reciprocal ceil(2^32 / D)
// for D >= 2 (0 for D = 1)}.  Token nt (one past the last) is the block's literal tail: it starts where
// the tokens' output ends and is literals up to the block's end; later rows start at 0xFFFFFFFF.
template <uint32_t TR>
struct FillTable {
  uint32_t start[TR];
  uint4 tk[TR];
};
// per warp, for WPL output words a lane a round: the table's rows (a round's tokens and the one carried
// in), its bytes, and the round's byte flags (which bytes are not known yet)
__host__ __device__ constexpr uint32_t fill_rows(uint32_t wpl) { return 64 * wpl; }
__host__ __device__ constexpr uint32_t fill_table_bytes(uint32_t wpl) { return 20 * fill_rows(wpl); }
__host__ __device__ constexpr uint32_t fill_flag_bytes(uint32_t wpl) { return 128 * wpl; }

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

__device__ inline void copy_bytes(uint8_t* d, const uint8_t* s, uint32_t n) {  // all lanes; no overlap
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

}  // namespace

// The replay of block b by one warp, in rounds of 128 * WPL output bytes: WPL 128-byte lines of the output
// address, lane k filling the aligned word at offset 4k of each.  Groups are not walked: a byte's value
// comes from its token's literals, from output before the round (the warp's shared-memory ring of the last
// R bytes, or global memory), or from an earlier byte of the same round.  The lanes first fill every byte
// of the first two kinds with their loads in flight together; the bytes of the third kind then read their
// sources from the round's words staged in the ring, pass after pass until all are known (each source lies
// before its byte, so this ends; the format's groups keep those chains short).
//
// A token is at least 4 bytes long, so an aligned word holds at most one token start: a line's token
// starts form a 32-bit word mask (one OR-reduction), and a lane's bytes belong to the last token starting at
// or before its word's last byte, or the one before that.  A match byte's source is ms - D + ((q - ms) mod
// D) (src/codec2.h:194-197: an overlapping match repeats its D bytes before it), the quotient from a
// multiply-high by the reciprocal, exact to one step, which a compare corrects.
template <uint32_t WPL, uint32_t TR>
__device__ __forceinline__ void fill_block(const DecArgs& A, uint32_t b, FillTable<TR>& T, uint8_t* ring,
                                           uint8_t* flags) {
  const uint32_t R = 1u << A.ring_log, rmask = R - 1u;
  const uint32_t lane = lane_id();
  const uint32_t raw = A.raw_len[b], method = A.method[b], clen = A.comp_len[b], B = A.B;
  uint8_t* o = A.out + A.out_off[b];
  const uint8_t* p = A.comp + A.comp_off[b];
  if (raw > B) { if (lane == 0) flag(A.err, b, E_RAWLEN); return; }
  if (method == 0) {
    if (clen != raw) { if (lane == 0) flag(A.err, b, E_STORED); return; }
    copy_bytes(o, p, raw);
    return;
  }
  if (method != 1) { if (lane == 0) flag(A.err, b, E_METHOD); return; }
  if (A.err[b]) return;
  const DecMeta& m = A.meta[b];
  const uint32_t nt = m.nt, op_total = m.op_total, li_total = m.li_total;
  const size_t TC = tok_cap(B);
  const uint8_t* lit = A.s_lit + (size_t)b * B;
  const uint32_t* Ts = A.tk_start + (size_t)b * TC;
  const uint32_t* Tm = A.tk_ms + (size_t)b * TC;
  const uint32_t* Td = A.tk_d + (size_t)b * TC;
  const uint32_t* Tl = A.tk_lik + (size_t)b * TC;
  const uint32_t ob = (uint32_t)(uintptr_t)o;
  // rows for tokens committed so far: [loaded - TR, loaded); row TR - 1 first holds a token "-1" (no byte
  // uses it).  The next 32 tokens wait in registers (lane k: token loaded + k), fetched one window ahead;
  // a match whose source lies beyond the ring has its first source lines brought into L2 then, and so
  // does each token's first literal line.
  uint32_t loaded = 0, ns, nm, nd, nl;
  auto fetch = [&](uint32_t base) {
    const uint32_t t = base + lane;
    ns = 0xFFFFFFFFu; nm = 0xFFFFFFFFu; nd = 1; nl = 0;
    if (t < nt) {
      ns = Ts[t]; nm = Tm[t]; nd = Td[t];
      const uint32_t lk = Tl[t];
      nl = lk - ns;
      prefetch_l2(lit + lk);
      if (nd >= R) {
        prefetch_l2(o + (nm - nd));
        prefetch_l2(o + (nm - nd) + 128);
      }
    } else if (t == nt) {
      ns = op_total; nm = raw; nl = li_total - op_total;
    }
  };
  auto commit = [&]() {
    const uint32_t t = loaded + lane;
    T.start[t % TR] = ns;
    T.tk[t % TR] = make_uint4(nm, nl, nd, nd >= 2 ? 0xFFFFFFFFu / nd + 1u : 0u);
    loaded += 32;
    fetch(loaded);
  };
  fetch(0);
  if (lane == 0) T.start[TR - 1] = 0;
  commit();
  __syncwarp();
  uint32_t before = 0;  // tokens starting before the round
  const uint32_t upto = 0xFFFFFFFFu >> (31u - lane);
  for (int32_t lb = -(int32_t)(ob & 127u); lb < (int32_t)raw; lb += 128 * WPL) {
    if (before + 32 * WPL > loaded) {  // (at most 32 tokens start in a line; the carried one keeps its row)
      do commit(); while (before + 32 * WPL > loaded);
      __syncwarp();
    }
    const int32_t rlo = lb - (int32_t)R;  // the ring holds output [lb - R, lb)
    uint32_t w[WPL], pend = 0;            // pend: bit 4h + j, byte j of word h is not known yet
    uint64_t srcs[WPL];                   // its source's offset in the round, 16 bits a byte
    uint32_t bh = before;
#pragma unroll
    for (uint32_t h = 0; h < WPL; ++h) {
      const int32_t lh = lb + 128 * (int32_t)h;
      const uint32_t ts = T.start[(bh + lane) % TR];
      const int32_t rel = (int32_t)(ts - (uint32_t)lh);
      const uint32_t mask = __reduce_or_sync(kFull, ts != 0xFFFFFFFFu && rel >= 0 && rel < 128 ? 1u << (rel >> 2) : 0u);
      const uint32_t t1 = bh + __popc(mask & upto) - 1u, t0 = t1 - 1u;  // (mod 2^32: token -1 is row TR - 1)
      const uint32_t st1 = T.start[t1 % TR], st0 = T.start[t0 % TR];
      const uint4 a1 = T.tk[t1 % TR], a0 = T.tk[t0 % TR];
      bh += __popc(mask);
      const int32_t q0 = lh + 4 * (int32_t)lane;
      w[h] = 0;
      srcs[h] = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {  // every choice a select, the load predicated
        const int32_t qi = q0 + j;
        const bool valid = qi >= 0 && qi < (int32_t)raw;
        const uint32_t q = (uint32_t)qi;
        const bool hi = q >= st1;
        const uint32_t opk = hi ? st1 : st0, ms = hi ? a1.x : a0.x, ld = hi ? a1.y : a0.y, D = hi ? a1.z : a0.z,
                       mg = hi ? a1.w : a0.w;
        const uint32_t x = q - ms;
        uint32_t r = x - __umulhi(x, mg) * D;
        r = (int32_t)r < 0 ? r + D : r;
        r = mg ? r : 0u;
        const uint32_t s = q >= ms ? ms - D + r : q;
        const bool own = s >= opk;
        const bool inr = !own && (int32_t)s >= lb;
        const uint8_t* src = own ? lit + (s + ld) : (int32_t)s >= rlo ? ring + ((ob + s) & rmask) : o + s;
        const bool take = valid && inr;
        pend |= (uint32_t)take << (4 * h + j);
        srcs[h] |= take ? (uint64_t)(s - (uint32_t)lb) << (16 * j) : 0ull;
        uint32_t v = 0;
        if (valid && !inr) v = *src;
        w[h] |= v << (8 * j);
      }
    }
    // bytes from earlier in the round: the round's words staged in their ring slots (the ring's older
    // bytes there are no longer needed: every load from the ring was made above), with a flag per byte
    // still unknown; each pass takes the bytes whose sources are known
    __syncwarp();  // (every lane's loads from the ring come before any lane's stores into it)
    if (__any_sync(kFull, pend)) {
      for (;;) {
#pragma unroll
        for (uint32_t h = 0; h < WPL; ++h) {
          const uint32_t q0 = (uint32_t)(lb + 128 * (int32_t)h + 4 * (int32_t)lane);
          *reinterpret_cast<uint32_t*>(ring + ((ob + q0) & rmask)) = w[h];
          const uint32_t f = (pend >> (4 * h)) & 15u;
          *reinterpret_cast<uint32_t*>(flags + 128 * h + 4 * lane) =
              (f & 1u) | (f & 2u) << 7 | (f & 4u) << 14 | (f & 8u) << 21;
        }
        __syncwarp();
        uint32_t left = pend;
#pragma unroll
        for (uint32_t h = 0; h < WPL; ++h) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            if (!((pend >> (4 * h + j)) & 1u)) continue;
            const uint32_t sp = (uint32_t)(srcs[h] >> (16 * j)) & 0xFFFFu;
            if (flags[sp]) continue;
            w[h] |= (uint32_t)ring[(ob + (uint32_t)lb + sp) & rmask] << (8 * j);
            left &= ~(1u << (4 * h + j));
          }
        }
        pend = left;
        __syncwarp();
        if (!__any_sync(kFull, pend)) break;
      }
    }
    // stores: the ring always whole words; the output whole words inside the block, bytes at its edges
#pragma unroll
    for (uint32_t h = 0; h < WPL; ++h) {
      const int32_t q0 = lb + 128 * (int32_t)h + 4 * (int32_t)lane;
      *reinterpret_cast<uint32_t*>(ring + ((ob + (uint32_t)q0) & rmask)) = w[h];
      if (q0 >= 0 && q0 + 4 <= (int32_t)raw) {
        *reinterpret_cast<uint32_t*>(o + q0) = w[h];
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (q0 + j >= 0 && q0 + j < (int32_t)raw) o[q0 + j] = (uint8_t)(w[h] >> (8 * j));
      }
    }
    before = bh;
    __syncwarp();
  }
}

// Fed by a device work queue: every warp takes the next block from the work counter until none is left,
// so blocks of uneven sizes (a batch of many files) balance across warps.  A CTA holds blockDim.x / 32
// warps, each with its table, a ring of 2^ring_log bytes and its byte flags in dynamic shared memory.
// The ring is read only at positions the warp has written in its current block.
template <uint32_t WPL>
__global__ void __maxnreg__(72) k_dec_fill(DecArgs A) {  // (72 registers: 28 warps an SM with 4-warp CTAs)
  constexpr uint32_t TR = fill_rows(WPL);
  extern __shared__ __align__(16) uint8_t fsm[];
  const uint32_t R = 1u << A.ring_log;
  const uint32_t wid = threadIdx.x >> 5;
  const size_t per = (size_t)fill_table_bytes(WPL) + R + fill_flag_bytes(WPL);
  uint8_t* mine = fsm + (size_t)wid * per;
  FillTable<TR>& T = *reinterpret_cast<FillTable<TR>*>(mine);
  uint8_t* ring = mine + fill_table_bytes(WPL);
  uint8_t* flags = ring + R;
  for (;;) {
    uint32_t b = 0;
    if (lane_id() == 0) b = atomicAdd(A.work, 1u);
    b = __shfl_sync(kFull, b, 0);
    if (b >= A.nb) break;
    fill_block<WPL>(A, b, T, ring, flags);
    __syncwarp();
  }
}

size_t fill_smem_bytes(uint32_t ring_log, uint32_t warps, uint32_t words) {
  return (size_t)warps * (fill_table_bytes(words) + (1u << ring_log) + fill_flag_bytes(words));
}

cudaError_t prepare_fill() {
  const int cap = (int)kMaxFillSmem;
  cudaError_t e = cudaFuncSetAttribute(k_dec_fill<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_dec_fill<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_dec_fill<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
  return e;
}

void launch_decode_fill(const DecArgs& A, cudaStream_t st, Stages& S) {
  if (!A.nb) return;
  launch_dec_streams(A, st, S);
  S.begin("k_dec_tokens", st);
  k_dec_tokens<<<A.nb, 1024, 0, st>>>(A);
  S.end(st);
  const uint32_t W = A.fill_warps;
  const size_t sm = fill_smem_bytes(A.ring_log, W, A.fill_words);
  const uint32_t grid = (A.nb + W - 1) / W;  // (as many warps as blocks; the counter balances them)
  cudaMemsetAsync(A.work, 0, sizeof(uint32_t), st);
  S.begin("k_dec_fill", st);
  if (A.fill_words == 4) k_dec_fill<4><<<grid, 32 * W, sm, st>>>(A);
  else if (A.fill_words == 2) k_dec_fill<2><<<grid, 32 * W, sm, st>>>(A);
  else k_dec_fill<1><<<grid, 32 * W, sm, st>>>(A);
  S.end(st);
}

}  // namespace zc
