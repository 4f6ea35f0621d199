// zc_decode_fill.cu -- the ZB2 LZ replay in two kernels (src/codec2.h:155-203):
//
//   k_dec_tokens  one CTA of 1024 threads per block: every token's literal run and match length (ext
//                 bytes), offset (offset bits), output start and literal start, from block-wide scans, in
//                 parallel over the tokens; then the groups (a scan of their counts) and the recent-offset
//                 symbols (each names an earlier token's offset, src/codec2.h:180-192), resolved by pointer
//                 jumping over all tokens at once.  Every check of the reference decoder is made here; a
//                 failing one records a status and the block is not replayed.
//   k_dec_fill    one warp per block: walks the groups in order and fills each group's output with all
//                 lanes (a group's matches read only output from before the group, or their own
//                 literals), the next 32 tokens' table loaded while the current ones are filled.
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

// a chunk of at most 32 tokens of one group: start[i] the output start of token i (start[c] the chunk's
// end); tk[i] = {match start, literal start - output start (mod 2^32), offset D, the reciprocal
// ceil(2^32 / D) when the match overlaps itself (D < M, D >= 2), else 0}
struct FillTable {
  uint32_t start[33];
  uint32_t pad_[3];
  uint4 tk[32];
};
constexpr uint32_t kTableBytes = (sizeof(FillTable) + 15u) & ~15u;

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Fills [op, op_end) of the chunk's tokens, 4 bytes a lane per round of 128 bytes, each lane's word
// aligned in memory.  A token is at least 4 bytes long, so an aligned word holds at most one token
// start: a round's starts form a 32-bit word mask (one OR-reduction over the window lanes `cs` of
// chunk tokens k0 .. k1-1), and a lane's bytes belong to the last token starting at or before its word,
// or the one before that.  A byte is its token's literal, or a match byte whose source is output from
// before the group or the token's own literals (an overlapping match, D < M, repeats the D bytes before
// it: match byte i comes from ms - D + (i mod D), the quotient from a multiply-high by the reciprocal,
// exact to one step, which a compare corrects).  Output from before the group is read from the warp's
// ring of the last R output bytes (shared memory, indexed by address mod R) when the round's own stores
// cannot have replaced it, else from global memory.  A round's loads are all issued before its stores.
__device__ __forceinline__ void fill_span(const FillTable& T, uint8_t* o, uint8_t* ring, uint32_t rmask,
                                          const uint8_t* lit, uint32_t op, uint32_t op_end, uint32_t cs, uint32_t k0,
                                          uint32_t k1) {
  const uint32_t lane = lane_id();
  const uint32_t ob = (uint32_t)(uintptr_t)o;
  const bool mine = lane >= k0 && lane < k1;
  uint32_t kb = 0;  // chunk tokens starting before the round
  for (int32_t base = (int32_t)op - (int32_t)((ob + op) & 3u); base < (int32_t)op_end; base += 128) {
    const int32_t rel = (int32_t)cs - base;
    const uint32_t mask = __reduce_or_sync(kFull, mine && rel >= 0 && rel < 128 ? 1u << (rel >> 2) : 0u);
    const uint32_t cnt = kb + __popc(mask & (0xFFFFFFFFu >> (31u - lane)));
    kb += __popc(mask);
    const int32_t q0 = base + 4 * (int32_t)lane;
    if (q0 >= (int32_t)op_end || q0 + 4 <= (int32_t)op) continue;
    const int32_t b1 = base + 128 < (int32_t)op_end ? base + 128 : (int32_t)op_end;
    const int32_t rlo = b1 - (int32_t)(rmask + 1);  // ring bytes at or after rlo survive this round's stores
    const uint32_t i1 = cnt - 1, i0 = cnt >= 2 ? cnt - 2 : 0;
    const uint32_t st1 = T.start[i1], st0 = T.start[i0];
    const uint4 t1 = T.tk[i1], t0 = T.tk[i0];
    const uint8_t* src[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t q = (uint32_t)(q0 + j);
      const bool h = q >= st1;
      const uint32_t opk = h ? st1 : st0, ms = h ? t1.x : t0.x, ld = h ? t1.y : t0.y, D = h ? t1.z : t0.z,
                     mg = h ? t1.w : t0.w;
      const uint8_t* p;
      if (q < ms) {
        p = lit + (q + ld);
      } else {
        uint32_t s = q - D;
        if (s >= ms) {
          const uint32_t x = q - ms;
          uint32_t r = mg ? x - __umulhi(x, mg) * D : 0u;
          if ((int32_t)r < 0) r += D;
          s = ms - D + r;
        }
        p = s >= opk ? lit + (s + ld) : (int32_t)s >= rlo ? ring + ((ob + s) & rmask) : o + s;
      }
      src[j] = (int32_t)q >= (int32_t)op && q < op_end ? p : ring;
    }
    uint32_t w = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) w |= (uint32_t)*src[j] << (8 * j);
    uint8_t* rq = ring + ((ob + (uint32_t)q0) & rmask);
    if (q0 >= (int32_t)op && q0 + 4 <= (int32_t)op_end) {
      *reinterpret_cast<uint32_t*>(o + q0) = w;
      *reinterpret_cast<uint32_t*>(rq) = w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int32_t q = q0 + j;
        if (q < (int32_t)op || q >= (int32_t)op_end) continue;
        o[q] = (uint8_t)(w >> (8 * j));
        rq[j] = (uint8_t)(w >> (8 * j));
      }
    }
  }
}

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

// The replay of block b by one warp, with the warp's table and ring.
__device__ __forceinline__ void fill_block(const DecArgs& A, uint32_t b, FillTable& T, uint8_t* ring) {
  const uint32_t R = 1u << A.ring_log;
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
  const DecMeta m = A.meta[b];
  const size_t TC = tok_cap(B);
  const uint8_t* lit = A.s_lit + (size_t)b * B;
  const uint8_t* grp = A.s_grp + (size_t)b * TC;
  const uint32_t* Ts = A.tk_start + (size_t)b * TC;
  const uint32_t* Tm = A.tk_ms + (size_t)b * TC;
  const uint32_t* Td = A.tk_d + (size_t)b * TC;
  const uint32_t* Tl = A.tk_lik + (size_t)b * TC;
  const uint32_t op_total = m.op_total, li_total = m.li_total;
  // token windows: lane k holds token w0 + k of the current window, and of the next one (prefetched;
  // a match whose source lies beyond the ring has its first source line brought into L2 then)
  uint32_t w0 = 0;
  auto load = [&](uint32_t base, uint32_t& s, uint32_t& ms, uint32_t& d, uint32_t& l) {
    const uint32_t t = base + lane;
    if (t < m.nt) {
      s = Ts[t]; ms = Tm[t]; d = Td[t]; l = Tl[t];
      if (d >= R) prefetch_l2(o + (ms - d));
    } else {
      s = op_total; ms = op_total; d = 1; l = li_total;
    }
  };
  uint32_t cs, cm, cd, cl, ns, nm, nd, nl;
  load(0, cs, cm, cd, cl);
  load(32, ns, nm, nd, nl);
  const uint32_t rmask = R - 1;
  uint32_t gc = 0;  // the group counts of groups gi0 .. gi0 + 31, lane k holding gi0 + k
  uint32_t gi0 = 0, t = 0;
  for (uint32_t g = 0; g < m.ng; ++g) {
    if ((g & 31u) == 0) { gi0 = g; gc = g + lane < m.ng ? grp[g + lane] : 0u; }
    const uint32_t gend = t + __shfl_sync(kFull, gc, g - gi0);
    while (t < gend) {
      if (t >= w0 + 32) {  // the next window becomes current; prefetch the one after
        w0 += 32;
        cs = ns; cm = nm; cd = nd; cl = nl;
        load(w0 + 32, ns, nm, nd, nl);
      }
      const uint32_t k0 = t - w0, k1 = min(gend, w0 + 32) - w0, c = k1 - k0;
      // each token's end: the next token's start (in this window or the next), or the total
      const uint32_t e_next = __shfl_sync(kFull, ns, 0);
      const uint32_t e_dn = __shfl_down_sync(kFull, cs, 1);
      const uint32_t tend = lane < 31 ? e_dn : e_next;
      if (lane >= k0 && lane < k1) {
        const uint32_t i = lane - k0;
        const uint32_t mg = cd >= 2 && cd < tend - cm ? 0xFFFFFFFFu / cd + 1u : 0u;
        T.start[i] = cs;
        T.tk[i] = make_uint4(cm, cl - cs, cd, mg);
      }
      const uint32_t op_end = __shfl_sync(kFull, tend, k1 - 1);
      const uint32_t op = __shfl_sync(kFull, cs, k0);
      if (lane == 0) T.start[c] = op_end;
      __syncwarp();
      fill_span(T, o, ring, rmask, lit, op, op_end, cs, k0, k1);
      __syncwarp();
      t += c;
    }
  }
  copy_bytes(o + op_total, lit + li_total, m.nl - li_total);
}

// Fed by a device work queue: every warp takes the next block from the work counter until none is left,
// so blocks of uneven sizes (a batch of many files) balance across warps.  A CTA holds blockDim.x / 32 warps, each
// with its table and a ring of 2^ring_log bytes in dynamic shared memory (16-byte aligned, the ring after
// the table).  The ring is read only at positions the warp has written in its current block.
__global__ void __maxnreg__(72) k_dec_fill(DecArgs A) {  // (72 registers: 28 warps an SM with 4-warp CTAs)
  extern __shared__ __align__(16) uint8_t fsm[];
  const uint32_t R = 1u << A.ring_log;
  const uint32_t wid = threadIdx.x >> 5;
  FillTable& T = *reinterpret_cast<FillTable*>(fsm + (size_t)wid * (kTableBytes + R));
  uint8_t* ring = fsm + (size_t)wid * (kTableBytes + R) + kTableBytes;
  for (;;) {
    uint32_t b = 0;
    if (lane_id() == 0) b = atomicAdd(A.work, 1u);
    b = __shfl_sync(kFull, b, 0);
    if (b >= A.nb) break;
    fill_block(A, b, T, ring);
    __syncwarp();
  }
}

size_t fill_smem_bytes(uint32_t ring_log, uint32_t warps) { return (size_t)warps * (kTableBytes + (1u << ring_log)); }

cudaError_t prepare_fill() {
  const int cap = (int)kMaxFillSmem;
  return cudaFuncSetAttribute(k_dec_fill, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
}

void launch_decode_fill(const DecArgs& A, cudaStream_t st, Stages& S) {
  if (!A.nb) return;
  launch_dec_streams(A, st, S);
  S.begin("k_dec_tokens", st);
  k_dec_tokens<<<A.nb, 1024, 0, st>>>(A);
  S.end(st);
  const uint32_t W = A.fill_warps;
  const size_t sm = fill_smem_bytes(A.ring_log, W);
  const uint32_t grid = (A.nb + W - 1) / W;  // (as many warps as blocks; the counter balances them)
  cudaMemsetAsync(A.work, 0, sizeof(uint32_t), st);
  S.begin("k_dec_fill", st);
  k_dec_fill<<<grid, 32 * W, sm, st>>>(A);
  S.end(st);
}

}  // namespace zc
