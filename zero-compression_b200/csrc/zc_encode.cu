// zc_encode.cu -- the ZB2 block encoder on sm_100a.  It writes, at each level, exactly the payload the
// reference CPU codec writes (src/codec2.h:43-153 with the depth of src/main.cpp:45, 54).
//
// The CPU parse walks hash chains: for position i, the `depth` most recent earlier positions whose
// 4-byte hash (16 bits) equals i's, the longest match kept (the nearest on a tie), one lazy step.  A
// chain is exactly the run of i's predecessors in a stable sort of the positions by hash, so:
//
//   k_sort_*       stable two-pass LSD radix sort of each block's positions by hash (8 + 8 bits), a
//                  CTA per 4096-position tile: digit counts, per-block scan, ranked scatter (warp
//                  match_any ranks, the tile reordered in shared memory, digit runs written together)
//   k_enc_match    per sorted position: its nearest candidate, then, where that does not decide it, its
//                  chain scanned (by a lane, or by a group of lanes a candidate each where the tile has few
//                  such positions), comparing at most cmp_cap bytes; a match that reaches cmp_cap, or a
//                  position that lies inside a longer match starting before it, is marked and finished
//                  only if the parse visits it
//   k_enc_parse    one CTA per block: the greedy + lazy parse as a chain 0 -> next(0) -> ..., walked
//                  per segment in parallel from the segment start, then re-walked from the true entry
//                  until it meets the first walk (rounds until no segment exit moves); a warp's walks
//                  step together and finish capped matches as a warp
//   k_enc_streams  one warp per block: group starts from a running maximum of per-token thresholds and a
//                  next-start chain, recent offsets by shuffles from each group's start, tok / ext / sym /
//                  group streams, offset bits packed by a word-segmented OR-scan, literals
//   k_enc_rans     one CTA per (block, stream): histogram, 12-bit normalisation with the reference's
//                  tie-breaks, 64 lanes coding backwards (src/codec.h:41-147)
//   k_enc_pack     one CTA per block: the payload (src/codec2.h:139-152), or "stored"
//   k_enc_scan / k_enc_emit: record sizes -> offsets, payloads packed back to back
#include "zc_internal.cuh"
#include "zc_kernels.h"

namespace zc {

// per-position match record: NONE; SAT | r (a candidate reached cmp_cap, or the position lies inside a
// longer match that starts before it; r is the position's index in the hash-sorted order, where its chain
// starts: finished on demand by the parse, which computes the chain's exact best); BELOW | r (the parse
// found that the position's match cannot win the lazy test of the position before it, and left it
// unfinished: finished like SAT if a walk needs it exactly); or the exact (length - 4) << 20 |
// (distance - 1).  Lengths are <= 4096, so an exact record has at most 0xFFC in its top 12 bits, and
// r < 2^20 - 3, so SAT | r is never NONE.
constexpr uint32_t M_NONE = 0xFFFFFFFFu;
constexpr uint32_t M_SAT = 0xFFF00000u;
constexpr uint32_t M_BELOW = 0xFFE00000u;  // capped, and known to lose the lazy test of the position before
__device__ __forceinline__ bool m_is_sat(uint32_t v) { return (v >> 20) >= 0xFFEu && v != M_NONE; }
__device__ __forceinline__ bool m_is_below(uint32_t v) { return (v >> 20) == 0xFFEu; }
__device__ __forceinline__ uint32_t m_pack(uint32_t m, uint32_t d) { return ((m - 4u) << 20) | (d - 1u); }
__device__ __forceinline__ uint32_t m_len(uint32_t v) { return (v >> 20) + 4u; }
__device__ __forceinline__ uint32_t m_dist(uint32_t v) { return (v & 0xFFFFFu) + 1u; }

// 4 bytes at byte offset x of a 4-aligned buffer, from the two aligned words around it
__device__ __forceinline__ uint32_t load4(const uint8_t* base, uint64_t x) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(base) + (x >> 2);
  return __funnelshift_r(__ldg(w), __ldg(w + 1), (uint32_t)(x & 3u) * 8u);
}
// the CPU parse's hash: 4 bytes times 2654435761, top 16 bits (src/codec2.h:47)
__device__ __forceinline__ uint32_t hash16(const uint8_t* base, uint64_t x) { return (load4(base, x) * 2654435761u) >> 16; }

// common prefix of the bytes at a and b, at most cap
__device__ __forceinline__ uint32_t lcp(const uint8_t* base, uint64_t a, uint64_t b, uint32_t cap) {
  uint32_t l = 0;
  while (l + 4 <= cap) {
    const uint32_t x = load4(base, a + l) ^ load4(base, b + l);
    if (x) return l + ((uint32_t)__ffs(x) - 1u) / 8u;
    l += 4;
  }
  if (l < cap) {
    const uint32_t x = load4(base, a + l) ^ load4(base, b + l);
    const uint32_t k = x ? ((uint32_t)__ffs(x) - 1u) / 8u : 4u;
    return l + min(k, cap - l);
  }
  return l;
}

// ---------------------------------------------------------------- 1. stable sort by hash
// Two stable LSD passes over the 16-bit hash (low byte, then high byte), each as three kernels over
// tiles of 4096 positions, every tile its own CTA: k_sort_count (the tile's digit counts), k_sort_scan
// (per block: each tile's start for each digit, digit-major), k_sort_scatter (ranks the tile's entries
// per digit in order with warp match_any, reorders the tile by digit in shared memory, and writes each
// digit's run to its place).  Pass 0 reads positions in order and hashes them; pass 1 reads pass 0's
// output.  The counts array holds tiles_per_block(B) * 256 words per block.
constexpr uint32_t kSortTile = 4096, kSortThreads = 512, kSortPer = kSortTile / kSortThreads;

__device__ __forceinline__ uint32_t sort_tiles(uint32_t B) { return (B + kSortTile - 1) / kSortTile; }

template <int PASS>
__device__ __forceinline__ void sort_load(const EncArgs& A, uint32_t b, uint32_t i, uint32_t& p, uint32_t& h) {
  if (PASS == 0) {
    p = i;
    h = hash16(A.in, A.in_off[b] + i);
  } else {
    const size_t so = (size_t)b * A.B;
    p = A.tmp_pos[so + i];
    h = A.tmp_h[so + i];
  }
}
template <int PASS>
__device__ __forceinline__ uint32_t sort_digit(uint32_t h) { return PASS == 0 ? (h & 0xFFu) : (h >> 8); }

// each thread counts 16 consecutive entries of the tile: pass 0 hashes them from three aligned 16-byte
// loads of the input (the 19 bytes it needs, inside the input's readable slack), pass 1 reads their
// 16 hashes as two 16-byte loads; per-warp histograms in shared memory, summed at the end
template <int PASS>
__global__ void __launch_bounds__(256) k_sort_count(EncArgs A) {
  const uint32_t b = blockIdx.y, t = blockIdx.x, tid = threadIdx.x, w = tid >> 5;
  __shared__ uint32_t hist[8][256];
  const uint32_t n = A.in_len[b], count = n >= 4 ? n - 3 : 0;
  const uint32_t i0 = t * kSortTile, i1 = min(i0 + kSortTile, count);
#pragma unroll
  for (int k = 0; k < 8; ++k) hist[k][tid] = 0;
  __syncthreads();
  const uint32_t i = i0 + 16 * tid;
  if (i < i1) {
    uint32_t h[16];
    if (PASS == 0) {
      const uint64_t a = A.in_off[b] + i;
      const uint4* q16 = reinterpret_cast<const uint4*>(A.in + (a & ~(uint64_t)15));
      const uint4 c0 = __ldg(q16), c1 = __ldg(q16 + 1), c2 = __ldg(q16 + 2);
      const uint32_t w12[12] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w, c2.x, c2.y, c2.z, c2.w};
      const uint32_t o = (uint32_t)(a >> 2) & 3u, sh = (uint32_t)(a & 3u) * 8u;
      uint32_t u[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) u[k] = o == 0 ? w12[k] : o == 1 ? w12[k + 1] : o == 2 ? w12[k + 2] : w12[k + 3];
      uint32_t x[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) x[k] = __funnelshift_r(u[k], u[k + 1], sh);
#pragma unroll
      for (int j = 0; j < 16; ++j) h[j] = (__funnelshift_r(x[j >> 2], x[(j >> 2) + 1], 8 * (j & 3)) * 2654435761u) >> 16;
    } else {
      const uint4* q = reinterpret_cast<const uint4*>(A.tmp_h + (size_t)b * A.B + i);
      const uint4 v0 = q[0], v1 = q[1];
      const uint32_t vw[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
#pragma unroll
      for (int j = 0; j < 16; ++j) h[j] = (vw[j >> 1] >> (16 * (j & 1))) & 0xFFFFu;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (i + j < i1) atomicAdd(&hist[w][sort_digit<PASS>(h[j])], 1u);
  }
  __syncthreads();
  uint32_t sum = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) sum += hist[k][tid];
  A.scnt[((size_t)b * sort_tiles(A.B) + t) * 256 + tid] = sum;
}

// per block: counts -> each tile's start per digit (digit-major order over the block's tiles)
__global__ void __launch_bounds__(256) k_sort_scan(EncArgs A) {
  const uint32_t b = blockIdx.x, d = threadIdx.x, lane = lane_id(), w = d >> 5;
  __shared__ uint32_t ws[8];
  const uint32_t T = sort_tiles(A.B);
  uint32_t* c = A.scnt + (size_t)b * T * 256;
  uint32_t run = 0;
  for (uint32_t t = 0; t < T; ++t) {
    const uint32_t v = c[t * 256 + d];
    c[t * 256 + d] = run;
    run += v;
  }
  const uint32_t inc = warp_incl_scan(run);
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  uint32_t base = inc - run;
  for (uint32_t k = 0; k < w; ++k) base += ws[k];
  for (uint32_t t = 0; t < T; ++t) c[t * 256 + d] += base;
}

template <int PASS>
__global__ void __launch_bounds__(kSortThreads, 4) k_sort_scatter(EncArgs A) {
  constexpr uint32_t NW = kSortThreads / 32;
  __shared__ uint32_t cw[NW][256];  // per-warp digit counts, then the warp's start within the digit
  __shared__ uint32_t st_pos[kSortTile];
  __shared__ uint16_t st_h[kSortTile];
  __shared__ uint32_t tds[256], dst[256], ws[8];
  const uint32_t b = blockIdx.y, t = blockIdx.x, tid = threadIdx.x, lane = lane_id(), w = tid >> 5;
  const uint32_t n = A.in_len[b], count = n >= 4 ? n - 3 : 0;
  const uint32_t i0 = t * kSortTile;
  if (i0 >= count) return;
  const uint32_t tn = min(kSortTile, count - i0);
  const size_t so = (size_t)b * A.B;
  for (uint32_t k = tid; k < NW * 256; k += kSortThreads) (&cw[0][0])[k] = 0;
  if (tid < 256) dst[tid] = A.scnt[((size_t)b * sort_tiles(A.B) + t) * 256 + tid];
  __syncthreads();
  // ranks: warp w holds the tile's entries [kSortPer * 32 w, kSortPer * 32 (w + 1)), 32 per round, in order
  // (all of a thread's entries are loaded first: the ranking's warp syncs would otherwise keep each load
  // behind the previous entry's ranking)
  uint32_t kp[kSortPer], kh[kSortPer], kr[kSortPer];
#pragma unroll
  for (uint32_t j = 0; j < kSortPer; ++j) {
    const uint32_t li = w * (32 * kSortPer) + j * 32 + lane;
    kp[j] = 0; kh[j] = 0;
    if (li < tn) sort_load<PASS>(A, b, i0 + li, kp[j], kh[j]);
  }
#pragma unroll
  for (uint32_t j = 0; j < kSortPer; ++j) {
    const uint32_t li = w * (32 * kSortPer) + j * 32 + lane;
    const bool on = li < tn;
    const uint32_t p = kp[j], h = kh[j];
    const uint32_t d = sort_digit<PASS>(h);
    const unsigned act = __ballot_sync(kFull, on);
    uint32_t rk = 0xFFFFFFFFu;
    if (on) {
      const unsigned peers = __match_any_sync(act, d);
      const uint32_t c = cw[w][d];
      rk = c + __popc(peers & ((1u << lane) - 1u));
      __syncwarp(act);
      if ((peers & ((1u << lane) - 1u)) == 0) cw[w][d] = c + __popc(peers);
    }
    __syncwarp();
    kp[j] = p; kh[j] = h; kr[j] = rk;
  }
  __syncthreads();
  if (tid < 256) {  // per digit: the warps' starts within it, and the tile's count
    uint32_t run = 0;
#pragma unroll
    for (uint32_t k = 0; k < NW; ++k) { const uint32_t c = cw[k][tid]; cw[k][tid] = run; run += c; }
    const uint32_t inc = warp_incl_scan(run);
    if (lane == 31) ws[w] = inc;
    tds[tid] = inc - run;  // (the warp's part; the warps before are added below)
  }
  __syncthreads();
  if (tid < 256) {
    uint32_t add = 0;
    for (uint32_t k = 0; k < w; ++k) add += ws[k];
    tds[tid] += add;
  }
  __syncthreads();
#pragma unroll
  for (uint32_t j = 0; j < kSortPer; ++j) {
    if (kr[j] == 0xFFFFFFFFu) continue;
    const uint32_t d = sort_digit<PASS>(kh[j]);
    const uint32_t at = tds[d] + cw[w][d] + kr[j];
    st_pos[at] = kp[j];
    st_h[at] = (uint16_t)kh[j];
  }
  __syncthreads();
  uint32_t* op = PASS == 0 ? A.tmp_pos : A.srt_pos;
  uint16_t* oh = PASS == 0 ? A.tmp_h : A.srt_h;
  for (uint32_t i = tid; i < tn; i += kSortThreads) {
    const uint32_t h = st_h[i], d = sort_digit<PASS>(h);
    const size_t dest = so + dst[d] + (i - tds[d]);
    op[dest] = st_pos[i];
    oh[dest] = (uint16_t)h;
  }
}

// ---------------------------------------------------------------- 2. capped matches at every position
// A position whose nearest candidate matches at least 4 bytes and also the A.match_defer bytes before them
// (1..4; 0: never) is inside a longer match; the match pass leaves it to the parse.  The mask selects those
// bytes in the little-endian word of the 4 bytes before the position.
__device__ __forceinline__ uint32_t defer_mask(uint32_t back) { return back ? 0xFFFFFFFFu << (8u * (4u - back)) : 0u; }

// the first differing byte of two 16-byte windows (16 when equal)
__device__ __forceinline__ uint32_t lcp16(const uint4& a0, const uint4& b0) {
  uint32_t x;
  if ((x = a0.x ^ b0.x)) return ((uint32_t)__ffs(x) - 1u) >> 3;
  if ((x = a0.y ^ b0.y)) return 4 + (((uint32_t)__ffs(x) - 1u) >> 3);
  if ((x = a0.z ^ b0.z)) return 8 + (((uint32_t)__ffs(x) - 1u) >> 3);
  if ((x = a0.w ^ b0.w)) return 12 + (((uint32_t)__ffs(x) - 1u) >> 3);
  return 16;
}
// the first differing byte of two 32-byte windows (32 when equal)
__device__ __forceinline__ uint32_t lcp32(const uint4& a0, const uint4& a1, const uint4& b0, const uint4& b1) {
  uint32_t x;
  if ((x = a0.x ^ b0.x)) return ((uint32_t)__ffs(x) - 1u) >> 3;
  if ((x = a0.y ^ b0.y)) return 4 + (((uint32_t)__ffs(x) - 1u) >> 3);
  if ((x = a0.z ^ b0.z)) return 8 + (((uint32_t)__ffs(x) - 1u) >> 3);
  if ((x = a0.w ^ b0.w)) return 12 + (((uint32_t)__ffs(x) - 1u) >> 3);
  if ((x = a1.x ^ b1.x)) return 16 + (((uint32_t)__ffs(x) - 1u) >> 3);
  if ((x = a1.y ^ b1.y)) return 20 + (((uint32_t)__ffs(x) - 1u) >> 3);
  if ((x = a1.z ^ b1.z)) return 24 + (((uint32_t)__ffs(x) - 1u) >> 3);
  if ((x = a1.w ^ b1.w)) return 28 + (((uint32_t)__ffs(x) - 1u) >> 3);
  return 32;
}

#ifndef ZC_MATCH_GROUP
#define ZC_MATCH_GROUP 16
#endif
constexpr uint32_t kMatchGroup = ZC_MATCH_GROUP;  // lanes per work-list entry in the match pass: 8, 16 or 32
static_assert(kMatchGroup == 8 || kMatchGroup == 16 || kMatchGroup == 32, "lanes per work-list entry");

// One CTA of 256 threads per `tile` consecutive sorted positions of a block (tile = A.match_tile, a
// multiple of 256).  The entries it needs (its own and the `depth` before them) are staged once in
// shared memory with the first WB bytes at each position (WB = 16 or 32, at least the compare cap), so
// a candidate costs a few shared loads and XORs instead of random global reads.  Pass 1 gives each
// position its nearest candidate, which decides most of them; the rest go to a work list, scanned a lane
// per entry when it fills the CTA's lanes (or chains are short), else by groups of lanes, one candidate
// a lane (one lane per entry would leave most lanes idle while a warp's longest chain finishes).
// Dynamic shared memory: (tile + depth) * (WB + 4 + 2) + 8 * tile bytes (+4).
template <uint32_t WB>
__global__ void __launch_bounds__(256) k_enc_match(EncArgs A) {
  constexpr uint32_t NV = WB / 16;  // uint4s per window
  extern __shared__ uint4 sm[];
  __shared__ uint32_t next, nwork;
  const uint32_t b = blockIdx.y, t = threadIdx.x, lane = lane_id();
  const uint32_t tile = A.match_tile;
  const uint32_t r0 = blockIdx.x * tile;
  const uint32_t n = A.in_len[b];
  if (r0 >= n) return;
  const uint32_t count = n >= 4 ? n - 3 : 0;
  const size_t so = (size_t)b * A.B;
  const uint32_t D = (uint32_t)A.depth;
  const uint32_t cap_e = tile + D;
  const uint32_t dmask = defer_mask(A.match_defer);
  uint4* win = sm;  // entry i: bytes 16 v .. 16 v + 15 at win[NV i + v]
  uint32_t* spos = reinterpret_cast<uint32_t*>(win + NV * cap_e);
  uint16_t* sh = reinterpret_cast<uint16_t*>(spos + cap_e);
  uint32_t* wl = reinterpret_cast<uint32_t*>(sh + ((cap_e + 1) & ~1u));  // work list: entry | best << 16, distance
  const uint32_t e0 = r0 > D ? r0 - D : 0, e1 = min(r0 + tile, count);
  const uint64_t base = A.in_off[b];
  // (a window may reach up to WB + 15 bytes past its position, inside the input's readable slack; bytes past
  // the block never decide a match: every compare is capped at the block's end)
  if (t == 0) { next = 0; nwork = 0; }
  for (uint32_t i = t; e0 + i < e1; i += 256) {
    const uint32_t r = e0 + i;
    const uint32_t p = A.srt_pos[so + r];
    spos[i] = p;
    sh[i] = A.srt_h[so + r];
    // the window from WB / 16 + 1 aligned 16-byte loads (a few L1 requests an entry instead of one a word:
    // the entries' positions are scattered), its words picked by selects on the word offset
    const uint64_t a = base + p;
    const uint4* c = reinterpret_cast<const uint4*>(A.in + (a & ~(uint64_t)15));
    constexpr uint32_t NC = WB / 16 + 1;
    uint32_t cw[4 * NC];
#pragma unroll
    for (uint32_t k = 0; k < NC; ++k) {
      const uint4 x = __ldg(c + k);
      cw[4 * k] = x.x; cw[4 * k + 1] = x.y; cw[4 * k + 2] = x.z; cw[4 * k + 3] = x.w;
    }
    const uint32_t o = (uint32_t)(a >> 2) & 3u, shf = (uint32_t)(a & 3u) * 8u;
    uint32_t w[WB / 4 + 1];
#pragma unroll
    for (uint32_t q = 0; q <= WB / 4; ++q) w[q] = o == 0 ? cw[q] : o == 1 ? cw[q + 1] : o == 2 ? cw[q + 2] : cw[q + 3];
    uint32_t v[WB / 4];
#pragma unroll
    for (uint32_t q = 0; q < WB / 4; ++q) v[q] = __funnelshift_r(w[q], w[q + 1], shf);
#pragma unroll
    for (uint32_t q = 0; q < NV; ++q) win[NV * i + q] = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  }
  // positions past the last hashed one (the block's final 3 bytes) have no match
  for (uint32_t r = max(r0, count) + t; r < min(r0 + tile, n); r += 256) A.minfo[so + r] = M_NONE;
  __syncthreads();
  const uint32_t tn = e1 > r0 ? e1 - r0 : 0;  // positions of this tile
  // pass 1, a thread per position: the nearest candidate decides most positions (no candidate, a chain
  // of one, or a match that reaches the cap); the others go to the work list with what it found
  for (uint32_t my = t; my < tn; my += 256) {
    const uint32_t r = r0 + my, li = r - e0;
    const uint32_t p = spos[li], h = sh[li];
    const uint32_t lim = min(kMaxMatch, n - p), cap = min(min(A.cmp_cap, WB), lim);
    uint32_t v = M_NONE;
    if (r > 0 && sh[li - 1] == h) {
      const uint32_t e = li - 1;
      const uint32_t l = min(NV == 2 ? lcp32(win[2 * e], win[2 * e + 1], win[2 * li], win[2 * li + 1])
                                     : lcp16(win[e], win[li]), cap);
      const uint32_t d = p - spos[e];
      if (l == cap) {
        v = cap < lim ? M_SAT | r : m_pack(l, d);
      } else if (r < 2 || D < 2 || sh[li - 2] != h) {
        v = l < 4 ? M_NONE : m_pack(l, d);
      } else if (dmask && l >= 4 && p >= 4 && p - d >= 4 &&
                 ((load4(A.in, base + p - 4) ^ load4(A.in, base + p - d - 4)) & dmask) == 0) {
        // the nearest candidate's match also runs match_defer bytes back, so p lies inside a longer match
        // that starts earlier: the parse rarely visits it (it lands on match starts and the position after
        // them).  It is left capped, to be finished exactly, like any capped record, if the parse comes.
        v = M_SAT | r;
      } else {
        const uint32_t w = atomicAdd(&nwork, 1u);
        wl[2 * w] = li | (l << 16);
        wl[2 * w + 1] = d;
        continue;
      }
    }
    A.minfo[so + p] = v;
  }
  __syncthreads();
  const uint32_t tw = nwork;
  if (tw >= A.match_dense || D <= 8) {
    // pass 2, a lane per work-list entry (a work list that fills the CTA, or chains of at most 8): lanes take
    // entries from a CTA counter, a warp claiming entries for all its idle lanes at once.  Per-lane state: the
    // position's entry li, its chain of kend earlier entries with the same hash (a binary search: the entries
    // are sorted by hash), the candidate k reached so far, the best length, its distance, and the position's
    // own byte at offset `best`: a candidate whose byte there differs cannot be longer and is skipped after
    // one shared byte load (the CPU parse's probe, src/codec2.h:62)
    const uint8_t* wb = reinterpret_cast<const uint8_t*>(win);
    uint32_t li = 0xFFFFFFFFu, p = 0, lim = 0, cap = 0, best = 0, bd = 0, k = 0, kend = 0, pb = 0;
    uint4 p0 = make_uint4(0, 0, 0, 0), p1 = p0;
    bool dry = false;  // the tile has no unclaimed entries left (warp-uniform)
    for (;;) {
      const bool idle = li == 0xFFFFFFFFu;
      const unsigned want = __ballot_sync(kFull, idle);
      if (want && !dry) {
        const uint32_t leader = (uint32_t)__ffs(want) - 1u;
        uint32_t got = 0;
        if (lane == leader) got = atomicAdd(&next, (uint32_t)__popc(want));
        got = __shfl_sync(kFull, got, leader);
        if (got + (uint32_t)__popc(want) >= tw) dry = true;
        if (idle) {
          const uint32_t my = got + (uint32_t)__popc(want & ((1u << lane) - 1u));
          if (my < tw) {
            const uint32_t wa = wl[2 * my];
            li = wa & 0xFFFFu;
            best = wa >> 16;
            bd = wl[2 * my + 1];
            const uint32_t r = li + e0;
            p = spos[li];
            const uint32_t h = sh[li];
            lim = min(kMaxMatch, n - p);
            cap = min(min(A.cmp_cap, WB), lim);
            p0 = win[NV * li];
            p1 = win[NV * li + NV - 1];
            k = 1;
            pb = wb[WB * li + best];
            uint32_t lo = li - min(D, r), hi = li;  // the first entry of [lo, li] with hash h
            while (lo < hi) {
              const uint32_t mid = (lo + hi) >> 1;
              if (sh[mid] < h) lo = mid + 1; else hi = mid;
            }
            kend = li - lo;
          }
        }
      }
      if (!__any_sync(kFull, li != 0xFFFFFFFFu)) break;
      if (li == 0xFFFFFFFFu) continue;
      // four candidates of this lane's chain: probes first, full compares for those that pass, in order
      bool fin = false;
      uint32_t pass = 0;
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint32_t kk = k + 1 + u;
        if (kk <= kend && (best == 0 || wb[WB * (li - kk) + best] == pb)) pass |= 1u << u;
      }
      while (pass) {
        const uint32_t u = (uint32_t)__ffs(pass) - 1u;
        pass &= pass - 1u;
        const uint32_t kk = k + 1 + u, e = li - kk;
        const uint32_t l = min(NV == 2 ? lcp32(win[2 * e], win[2 * e + 1], p0, p1) : lcp16(win[e], p0), cap);
        if (l > best) {
          best = l;
          bd = p - spos[e];
          if (best == cap) { fin = true; break; }
          pb = wb[WB * li + best];
        }
      }
      k += 4;
      if (fin || k >= kend) {
        A.minfo[so + p] = best < 4 ? M_NONE : best == cap && cap < lim ? M_SAT | (li + e0) : m_pack(best, bd);
        li = 0xFFFFFFFFu;
      }
    }
    return;
  }
  // pass 2, kMatchGroup lanes per work-list entry (a short work list: a lane each would leave most lanes
  // idle while the longest chain finishes): lane g of the group compares the chain's candidate k = kb + g
  // (kb = 2, then kMatchGroup further each round; candidate 1 was pass 1's), all from shared memory; the
  // group's longest, the nearest on a tie, replaces the best only when longer, so nearer rounds win ties
  // too, as in the CPU parse's nearest-first scan.  The chain is the run of entries before the position with
  // its hash (the entries are sorted by hash), so it ends at the first lane whose entry differs; a round
  // ends the scan when the chain ends in it or the best reaches the cap.
  constexpr uint32_t G = kMatchGroup, NG = 32 / G;
  const uint32_t gl = lane % G;
  const unsigned gmask = G == 32 ? kFull : ((1u << G) - 1u) << (lane - gl);
  for (uint32_t wi = (t >> 5) * NG + lane / G; wi < tw; wi += 8 * NG) {
    const uint32_t wa = wl[2 * wi];
    const uint32_t li = wa & 0xFFFFu, r = li + e0;
    uint32_t best = wa >> 16, bd = wl[2 * wi + 1];
    const uint32_t p = spos[li], h = sh[li];
    const uint32_t lim = min(kMaxMatch, n - p), cap = min(min(A.cmp_cap, WB), lim);
    const uint4 p0 = win[NV * li], p1 = win[NV * li + NV - 1];
    const uint32_t kmax = min(D, r);  // (li >= kmax: the tile's entries are staged from depth before it)
    for (uint32_t kb = 2; kb <= kmax; kb += G) {
      const uint32_t k = kb + gl;
      const bool on = k <= kmax && sh[li - k] == h;
      uint32_t key = 0;
      if (on) {
        const uint32_t e = li - k;
        const uint32_t l = min(NV == 2 ? lcp32(win[2 * e], win[2 * e + 1], p0, p1) : lcp16(win[e], p0), cap);
        key = (l << 8) | (G - 1u - gl);  // (l <= 32)
      }
      const uint32_t mk = __reduce_max_sync(gmask, key);
      if ((mk >> 8) > best) {
        best = mk >> 8;
        bd = p - spos[li - (kb + G - 1u - (mk & 0xFFu))];
      }
      if (best == cap || __ballot_sync(gmask, on) != gmask) break;
    }
    if (gl == 0) A.minfo[so + p] = best < 4 ? M_NONE : best == cap && cap < lim ? M_SAT | r : m_pack(best, bd);
  }
}

// ---------------------------------------------------------------- 3. the parse
struct ParseBlock {
  const uint8_t* in;
  uint64_t base;
  uint32_t n, depth;
  uint32_t* minfo;
  const uint32_t* spos;
  const uint16_t* sh;
};

// The exact match at x, all 32 lanes together (x the same in every lane).  A capped record names x's
// index r in the hash-sorted order; its chain is the entries before r with the same hash, nearest first
// (the order src/codec2.h:58-67 walks them).  Up to 32 candidates at a time: each
// lane compares its candidate's first 32 bytes; those equal for 32 bytes (when the match may be longer)
// are extended in chain order by the whole warp, 128 bytes a step.  The longest wins, the nearest on a
// tie, and a match of the whole remaining length ends the walk, as in the CPU parse.  The exact record
// replaces the capped one in minfo.
// With need > 0 the caller only needs the exact match if it is at least `need` bytes long: a candidate whose
// byte at need - 1 differs from x's is shorter and dropped after that one load, and when no candidate
// reaches need the result is NONE and minfo keeps the capped record.
__device__ uint32_t coop_exact(const ParseBlock& P, uint32_t x, uint32_t need = 0) {
  const uint32_t lane = lane_id();
  const uint32_t v = P.minfo[x];
  if (!m_is_sat(v)) return v;
  const uint32_t r = v & 0xFFFFFu, h = P.sh[r];
  const uint32_t lim = min(kMaxMatch, P.n - x);
  if (need > lim) return M_NONE;
  const uint32_t l32 = min(32u, lim);
  const uint32_t kmax = min(P.depth, r);
  const uint64_t ax = P.base + x;
  uint32_t best = 0, bd = 0;
  bool stop = false;
  for (uint32_t kb = 1; kb <= kmax && !stop; kb += 32) {
    const uint32_t k = kb + lane;
    const bool in_chain = k <= kmax && P.sh[r - k] == h;
    const unsigned chain = __ballot_sync(kFull, in_chain);
    const unsigned live = ~chain ? chain & ((1u << __ffs(~chain) - 1) - 1u) : chain;  // up to the first break
    if (live != chain || chain != kFull) stop = true;  // the chain ends in this chunk
    bool on = (live >> lane) & 1u;
    const uint32_t j = on ? P.spos[r - k] : 0u;
    if (need && on) on = __ldg(P.in + P.base + j + need - 1) == __ldg(P.in + ax + need - 1);
    uint32_t l = 0;
    if (on) {  // 16 bytes a round from independent word loads (at most two rounds)
      const uint64_t aj = P.base + j;
      for (uint32_t o = 0; o < l32; o += 16) {
        uint32_t x[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) x[q] = load4(P.in, aj + o + 4 * q) ^ load4(P.in, ax + o + 4 * q);
        uint32_t k = 16;
#pragma unroll
        for (int q = 3; q >= 0; --q) if (x[q]) k = 4 * q + (((uint32_t)__ffs(x[q]) - 1u) >> 3);
        l = min(o + k, l32);
        if (k < 16) break;
      }
    }
    // candidates shorter than 32 bytes (or the whole remaining length): the longest, nearest on a tie
    uint32_t key = on ? (l << 8) | (31u - lane) : 0u;  // (l <= 32, lanes in chain order)
    key = __reduce_max_sync(kFull, key);
    const uint32_t cl = key >> 8, cw = 31u - (key & 0xFFu);
    const uint32_t jw = __shfl_sync(kFull, j, cw);
    if (cl > best) { best = cl; bd = x - jw; }
    if (best == lim) break;
    // candidates equal for 32 bytes: extended in chain order
    unsigned ext = __ballot_sync(kFull, on && l == 32u && lim > 32u);
    while (ext) {
      // (best >= 32 < lim here) a candidate whose byte at `best` differs from x's is no longer than best:
      // all such are dropped at once, before the next one in chain order is extended
      const bool keep = ((ext >> lane) & 1u) && __ldg(P.in + P.base + j + best) == __ldg(P.in + ax + best);
      ext = __ballot_sync(kFull, keep);
      if (!ext) break;
      const uint32_t c = (uint32_t)__ffs(ext) - 1u;
      ext &= ext - 1u;
      const uint32_t jc = __shfl_sync(kFull, j, c);
      const uint64_t aj = P.base + jc;
      uint32_t len = lim;
      for (uint32_t o = 32; o < lim; o += 128) {
        const uint32_t q = o + 4 * lane;
        uint32_t diff = 0;
        if (q < lim) diff = load4(P.in, aj + q) ^ load4(P.in, ax + q);
        const uint32_t nb = q < lim ? (diff ? ((uint32_t)__ffs(diff) - 1u) >> 3 : 4u) : 0u;
        const bool miss = q < lim && (nb < 4u || q + 4 > lim);
        const unsigned mm = __ballot_sync(kFull, miss);
        if (mm) {
          const uint32_t f = (uint32_t)__ffs(mm) - 1u;
          const uint32_t qf = o + 4 * f, nf = __shfl_sync(kFull, nb, f);
          len = min(qf + nf, lim);
          break;
        }
      }
      if (len > best) {
        best = len;
        bd = x - jc;
        if (best == lim) { stop = true; break; }
      }
    }
  }
  if (best < need) {  // (warp-uniform) marked, so a later walk's lazy test skips it
    __syncwarp();
    if (lane == 0) P.minfo[x] = M_BELOW | r;
    __syncwarp();
    return M_NONE;
  }
  const uint32_t e = best < 4 ? M_NONE : m_pack(best, bd);  // (capped records match >= 4 bytes: never NONE)
  __syncwarp();
  if (lane == 0) P.minfo[x] = e;
  __syncwarp();
  return e;
}

// One step of the CPU parse (src/codec2.h:69-80) for every lane with `act` (all 32 lanes call it):
// returns the next position (p itself when !act); the token, when the step emits one, in (ti, tm, td).
// Capped records at p or p + 1 are finished first, one at a time, by the whole warp.  A position with
// no match is a literal step to the next position, so a run of them is taken at once, up to `lim` (the
// walk's end): the walk lands where the CPU parse's single steps would first leave the run or reach lim.
__device__ __forceinline__ uint32_t warp_step(const ParseBlock& P, uint32_t p, uint32_t lim, bool act, bool& tok,
                                              uint32_t& ti, uint32_t& tm, uint32_t& td) {
  uint32_t v = act ? P.minfo[p] : M_NONE;
  const bool lz = act && v != M_NONE && p + 1 < P.n;
  uint32_t v2 = lz ? P.minfo[p + 1] : M_NONE;
  unsigned s1 = __ballot_sync(kFull, act && m_is_sat(v));
  while (s1) {
    const uint32_t L = (uint32_t)__ffs(s1) - 1u;
    s1 &= s1 - 1u;
    const uint32_t e = coop_exact(P, __shfl_sync(kFull, p, L));
    if (lane_id() == L) v = e;
  }
  // the match at p + 1 replaces p's only if 8 m2 - bitlen(d2) - 8 > 8 m - bitlen(d), so (bitlen(d2) >= 0)
  // only if 8 m2 > 8 m + 8 - bitlen(d), m2 >= need; a shorter one is never needed exactly
  const uint32_t need = lz ? ((8u * m_len(v) + 8u - bitlen(m_dist(v))) >> 3) + 1u : 0u;
  if (m_is_below(v2)) v2 = M_NONE;
  unsigned s2 = __ballot_sync(kFull, lz && m_is_sat(v2));
  while (s2) {
    const uint32_t L = (uint32_t)__ffs(s2) - 1u;
    s2 &= s2 - 1u;
    const uint32_t e = coop_exact(P, __shfl_sync(kFull, p, L) + 1u, __shfl_sync(kFull, need, L));
    if (lane_id() == L) v2 = e;
  }
  tok = false;
  if (!act) return p;
  if (v == M_NONE) {
    const uint32_t* m = P.minfo;
    uint32_t q = p + 1;
    while (q + 4 <= lim) {
      const uint32_t a0 = m[q], a1 = m[q + 1], a2 = m[q + 2], a3 = m[q + 3];
      if (a0 != M_NONE) break;
      if (a1 != M_NONE) { q += 1; break; }
      if (a2 != M_NONE) { q += 2; break; }
      if (a3 != M_NONE) { q += 3; break; }
      q += 4;
    }
    while (q < lim && m[q] == M_NONE) ++q;
    return q;
  }
  uint32_t m = m_len(v), d = m_dist(v), at = p;
  if (lz && v2 != M_NONE) {
    const uint32_t m2 = m_len(v2), d2 = m_dist(v2);
    if ((int)(8 * m2) - (int)bitlen(d2) - 8 > (int)(8 * m) - (int)bitlen(d)) { at = p + 1; m = m2; d = d2; }
  }
  tok = true; ti = at; tm = m; td = d;
  return at + m;
}

// One CTA per block, 256 segments of the block, a lane each.  The parse is a chain 0 -> next(0) -> ...;
// round 0 walks every segment from its own start; each later round re-walks a segment from where the
// chain before it leaves, until that walk meets the previous one (a two-pointer merge), and rounds end
// when no segment's exit moves.  Then every segment counts and writes its tokens.  Each warp's 32 walks
// step together (warp_step), so capped matches are finished by whole warps.
__global__ void __launch_bounds__(256, 8) k_enc_parse(EncArgs A) {  // (8 CTAs an SM: latency-bound walks)
  const uint32_t b = blockIdx.x, q = threadIdx.x;
  const uint32_t n = A.in_len[b];
  const size_t so = (size_t)b * A.B;
  __shared__ uint32_t ent[256], ex[256], wsum[8];
  ParseBlock P;
  P.in = A.in; P.base = A.in_off[b]; P.n = n; P.depth = (uint32_t)A.depth;
  P.minfo = A.minfo + so; P.spos = A.srt_pos + so; P.sh = A.srt_h + so;
  const uint32_t S = max(1u, (n + 255) / 256);
  const uint32_t s = min(q * S, n), e = min(s + S, n);
  bool t; uint32_t ta, tc, td;
  // round 0: every segment walked from its own start
  {
    uint32_t p = s;
    while (__any_sync(kFull, p < e)) p = warp_step(P, p, e, p < e, t, ta, tc, td);
    ent[q] = s;
    ex[q] = s < e ? p : s;
  }
  // rounds: each segment re-walked from where the chain before it leaves, until it meets its old walk
  for (;;) {
    __syncthreads();
    const uint32_t want = q == 0 ? 0u : ex[q - 1];
    __syncthreads();
    bool changed = false;
    const uint32_t old_ent = ent[q], old_ex = ex[q];
    // mode 0: settled; 1: walk a until it leaves the segment; 2: advance the lower of a (new walk) and
    // c (old walk) until they meet or both leave
    int mode = 0;
    uint32_t a = want, c = old_ent, nx = old_ex;
    if (want != old_ent) {
      if (want >= e) nx = want;
      else mode = old_ent >= e ? 1 : 2;
    }
    while (__any_sync(kFull, mode != 0)) {
      const bool adv_a = mode == 1 || (mode == 2 && a < c);
      const uint32_t y = warp_step(P, adv_a ? a : c, e, mode != 0, t, ta, tc, td);
      if (mode == 1) {
        a = y;
        if (a >= e) { nx = a; mode = 0; }
      } else if (mode == 2) {
        if (adv_a) a = y; else c = y;
        if (a == c) { nx = old_ex; mode = 0; }
        else if (a >= e && c >= e) { nx = a; mode = 0; }
      }
    }
    if (want != old_ent) {
      ent[q] = want;
      if (nx != old_ex) { ex[q] = nx; changed = true; }
    }
    if (!__syncthreads_or(changed)) break;
  }
  // tokens: each segment's final walk writes them to its own slots (a token takes at least 4 bytes, so
  // a segment of S bytes has at most S / 4 + 1), then they move to their offsets in the block's list
  const uint32_t from = ent[q];
  const uint32_t slots = S / 4 + 2;
  uint32_t* gi = A.tk_seg + (size_t)b * 3 * seg_tok_cap(A.B) + (size_t)q * slots;
  uint32_t* gm = gi + seg_tok_cap(A.B);
  uint32_t* gd = gm + seg_tok_cap(A.B);
  uint32_t cnt = 0;
  for (uint32_t p = from; __any_sync(kFull, p < e);) {
    p = warp_step(P, p, e, p < e, t, ta, tc, td);
    if (t) { gi[cnt] = ta; gm[cnt] = tc; gd[cnt] = td; ++cnt; }
  }
  const uint32_t incl = warp_incl_scan(cnt);
  if (lane_id() == 31) wsum[q >> 5] = incl;
  __syncthreads();
  uint32_t off = incl - cnt;
  for (uint32_t k = 0; k < (q >> 5); ++k) off += wsum[k];
  const size_t to = (size_t)b * tok_cap(A.B) + off;
  for (uint32_t k = 0; k < cnt; ++k) { A.tk_i[to + k] = gi[k]; A.tk_m[to + k] = gm[k]; A.tk_d[to + k] = gd[k]; }
  if (q == 255) A.bcnt[b * 8 + 0] = off + cnt;
}

// ---------------------------------------------------------------- 4. tokens -> streams
constexpr uint32_t kWarpCopyRun = 32;

// n bytes from src, a range of the codec's input (16-byte aligned, 64 readable bytes after its end), to
// dst by the 32 lanes of a warp: 4-byte words stored aligned at dst, each built by a funnel shift from
// the two aligned input words that cover it (those may reach a few bytes past the range, into the
// input's slack, never before the input's start), four words a lane in flight.
__device__ __forceinline__ void warp_copy_in(uint8_t* dst, const uint8_t* src, uint32_t n, uint32_t lane) {
  const uint32_t head = min(n, (4u - ((uint32_t)(uintptr_t)dst & 3u)) & 3u);
  if (lane < head) dst[lane] = src[lane];
  dst += head;
  src += head;
  n -= head;
  const uint32_t nw = n >> 2, sh = (uint32_t)(uintptr_t)src & 3u;
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src - sh);
  uint32_t* d = reinterpret_cast<uint32_t*>(dst);
  if (sh) {
#pragma unroll 4
    for (uint32_t w = lane; w < nw; w += 32) d[w] = __funnelshift_r(s[w], s[w + 1], 8u * sh);
  } else {
#pragma unroll 4
    for (uint32_t w = lane; w < nw; w += 32) d[w] = s[w];
  }
  const uint32_t t = nw << 2;
  if (lane < n - t) dst[t + lane] = src[t + lane];
}

// Tokens -> streams, one warp per block, 32 tokens a round (the next 32 loaded while these are coded).
//
// Groups follow the rule of src/codec2.h:103-116: a group ends before a token whose match source starts before
// the token's own output and reaches past the group's first output byte, or once it holds 255 tokens.  Within
// a round, a group opened at token g is read by token k exactly when the output start of g lies below k's
// source reach, and the output starts rise with the token index; so each token k whose source starts before
// its output gets theta_k = how many of the round's tokens start their output below its reach (at most k),
// and a group opened at g ends at the first token with theta > g.  With P the running maximum of theta over
// the round, that is next(g) = the first k with P_k > g: a binary search over P by shuffles.  The group open
// when the round starts ends at the first token that reads it (or would be its 256th); the round's later group
// starts follow from there by next().  A token's recent-offset symbols (250..252) name the offsets of the
// three tokens before its group's first token (src/codec2.h:121-137).
//
// Offset bits (LSB first): each token's bits start at a running bit position.  The tokens are grouped by the
// 32-bit output word their bits start in (the groups are runs of lanes), an OR-scan segmented by that word
// collects each word's bits (64-bit values: a token's spill into the next word rides in the high half), and
// the last lane of each run stores its completed word.  The partly filled last word carries to the next round.
__global__ void __launch_bounds__(128) k_enc_streams(EncArgs A) {
  const uint32_t lane = lane_id();
  const uint32_t b = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (b >= A.nb) return;
  const uint32_t n = A.in_len[b], nt = A.bcnt[b * 8 + 0];
  const uint8_t* src = A.in + A.in_off[b];
  const size_t TC = tok_cap(A.B);
  const uint32_t* TI = A.tk_i + (size_t)b * TC;
  const uint32_t* TM = A.tk_m + (size_t)b * TC;
  const uint32_t* TD = A.tk_d + (size_t)b * TC;
  uint8_t* lit = A.s_lit + (size_t)b * A.B;
  uint8_t* tok = A.s_tok + (size_t)b * TC;
  uint8_t* sym = A.s_sym + (size_t)b * TC;
  uint8_t* grp = A.s_grp + (size_t)b * TC;
  uint8_t* ext = A.s_ext + (size_t)b * ext_cap(A.B);
  uint32_t* bitw = reinterpret_cast<uint32_t*>(A.s_bits + (size_t)b * bits_cap(A.B));
  const uint32_t upto = 0xFFFFFFFFu >> (31u - lane);  // lanes 0 .. lane
  uint32_t op = 0;                    // output end of the tokens coded so far
  uint32_t gpos = 0, gcnt = 0;        // the open group: its first output byte, its tokens so far
  uint32_t ra = 1, rb = 4, rc = 8;    // the open group's recent offsets
  uint32_t pa = 1, pb = 4, pc = 8;    // the offsets of the last three tokens before the round, nearest first
  uint32_t ng = 0, ei = 0, li = 0;
  uint64_t bp = 0, wbase = 0;         // bits written so far; the first bit of the word being filled
  uint32_t cw = 0;                    // that word's bits [wbase, bp)
  uint32_t ni = 0, nm = 4, nd = 1;
  if (lane < nt) { ni = TI[lane]; nm = TM[lane]; nd = TD[lane]; }
  for (uint32_t t0 = 0; t0 < nt; t0 += 32) {
    const uint32_t c = min(32u, nt - t0);
    const uint32_t q = t0 + lane;
    const bool on = lane < c;
    const uint32_t i = ni, m = nm, d = nd;
    if (q + 32 < nt) { ni = TI[q + 32]; nm = TM[q + 32]; nd = TD[q + 32]; } else { ni = 0; nm = 4; nd = 1; }
    const uint32_t endk = i + m;
    const uint32_t up = __shfl_up_sync(kFull, endk, 1);
    const uint32_t opk = lane == 0 ? op : up;
    const uint32_t L = on ? i - opk : 0u;
    const uint32_t reach = i - d + min(m, d);
    const bool back = on && i - d < opk;  // the source starts before the token's own output
    // theta: the round's tokens whose output starts below the reach (lanes past c compare as above all)
    const uint32_t key = on ? opk : 0xFFFFFFFFu;
    uint32_t below = 0;
#pragma unroll
    for (uint32_t s = 16; s; s >>= 1)
      if (__shfl_sync(kFull, key, below + s - 1) < reach) below += s;
    const uint32_t theta = back ? min(lane, below) : 0u;
    // the open group ends at the first token that reads it, or that would be its 256th
    const unsigned ends = __ballot_sync(kFull, on && ((back && reach > gpos) || gcnt + lane >= kMaxGroup));
    const uint32_t s1 = ends ? (uint32_t)__ffs(ends) - 1u : c;
    uint32_t pm = theta;  // running maximum of theta
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(kFull, pm, o);
      if (lane >= o) pm = max(pm, v);
    }
    uint32_t nx = 0;  // next(lane): the first token with pm > lane (32: none)
#pragma unroll
    for (uint32_t s = 16; s; s >>= 1)
      if (__shfl_sync(kFull, pm, nx + s - 1) <= lane) nx += s;
    if (__shfl_sync(kFull, pm, nx) <= lane) nx = 32;
    uint32_t starts = 0;  // the round's group starts (warp-uniform walk)
    for (uint32_t s = s1; s < c; s = __shfl_sync(kFull, nx, s)) starts |= 1u << s;
    // the token's group start gs (-1: the group open before the round) and its recent offsets
    const uint32_t mine = starts & upto;
    const int gs = mine ? 31 - __clz(mine) : -1;
    const uint32_t x1 = __shfl_sync(kFull, d, max(gs - 1, 0)), x2 = __shfl_sync(kFull, d, max(gs - 2, 0)),
                   x3 = __shfl_sync(kFull, d, max(gs - 3, 0));
    uint32_t r0 = ra, r1 = rb, r2 = rc;
    if (gs >= 0) {
      r0 = gs >= 1 ? x1 : pa;
      r1 = gs >= 2 ? x2 : gs == 1 ? pa : pb;
      r2 = gs >= 3 ? x3 : gs == 2 ? pa : gs == 1 ? pb : pc;
    }
    const uint32_t sv = d == r0 ? kSymRep : d == r1 ? kSymRep + 1 : d == r2 ? kSymRep + 2 : bitlen(d);
    // group counts: the open group's (when it ends in this round), then each start's that ends in it
    const uint32_t open_ends = s1 < c && gcnt + s1 > 0 ? 1u : 0u;
    if (lane == 0 && open_ends) grp[ng] = (uint8_t)(gcnt + s1);
    if (((starts >> lane) & 1u) && nx < c) grp[ng + open_ends + __popc(mine) - 1] = (uint8_t)(nx - lane);
    ng += open_ends + (starts ? (uint32_t)__popc(starts) - 1u : 0u);
    if (starts) {
      const uint32_t last = 31u - __clz(starts);
      gpos = __shfl_sync(kFull, opk, last);
      gcnt = c - last;
      ra = __shfl_sync(kFull, r0, last);
      rb = __shfl_sync(kFull, r1, last);
      rc = __shfl_sync(kFull, r2, last);
    } else {
      gcnt += c;
    }
    {  // (only a full round is followed by another)
      const uint32_t a = __shfl_sync(kFull, d, 31), bq = __shfl_sync(kFull, d, 30), cq = __shfl_sync(kFull, d, 29);
      pa = a; pb = bq; pc = cq;
    }
    if (on) {
      tok[q] = (uint8_t)((min(L, 15u) << 4) | min(m - 4u, 15u));
      sym[q] = (uint8_t)sv;
    }
    // ext bytes (src/codec2.h:120-121): L - 15 in 3 bytes when L >= 15, then m - 19 in 2 when m >= 19
    const uint32_t fl = on && L >= 15u, fm = on && m >= 19u;
    const uint32_t nx_b = 3u * fl + 2u * fm;
    const uint32_t xincl = warp_incl_scan(nx_b);
    const uint32_t xq = ei + xincl - nx_b;
    if (fl) { const uint32_t v = L - 15u; ext[xq] = (uint8_t)v; ext[xq + 1] = (uint8_t)(v >> 8); ext[xq + 2] = (uint8_t)(v >> 16); }
    if (fm) { const uint32_t v = m - 19u, y = xq + 3u * fl; ext[y] = (uint8_t)v; ext[y + 1] = (uint8_t)(v >> 8); }
    // offset bits
    const uint32_t nbit = on && sv < kSymRep ? sv : 0u;
    const uint32_t bincl = warp_incl_scan(nbit);
    const uint32_t rel = (uint32_t)(bp - wbase) + bincl - nbit;  // (bp - wbase < 32)
    const uint32_t wi = rel >> 5;
    uint64_t acc = nbit ? (uint64_t)(d - (1u << nbit)) << (rel & 31u) : 0ull;
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
      const uint64_t v = __shfl_up_sync(kFull, acc, o);
      const uint32_t vw = __shfl_up_sync(kFull, wi, o);
      if (lane >= o && vw == wi) acc |= v;
    }
    const uint32_t rel_end = (uint32_t)(bp - wbase) + __shfl_sync(kFull, bincl, 31);
    const uint32_t full = rel_end >> 5;  // words completed by this round
    const uint32_t wprev = __shfl_up_sync(kFull, wi, 1), wnext = __shfl_down_sync(kFull, wi, 1);
    const unsigned firsts = __ballot_sync(kFull, lane == 0 || wprev != wi);
    const uint32_t f = 31u - __clz(firsts & upto);  // the first lane of this lane's run
    const uint32_t spill = (uint32_t)(__shfl_sync(kFull, acc, f ? f - 1u : 0u) >> 32);
    const uint32_t word = (uint32_t)acc | (f ? spill : 0u) | (wi == 0 ? cw : 0u);
    if ((lane == 31 || wnext != wi) && wi < full) bitw[(wbase >> 5) + wi] = word;
    const uint32_t w31 = __shfl_sync(kFull, word, 31), s31 = (uint32_t)(__shfl_sync(kFull, acc, 31) >> 32);
    cw = __shfl_sync(kFull, wi, 31) == full ? w31 : s31;
    bp += __shfl_sync(kFull, bincl, 31);
    wbase += 32ull * full;
    // literals before each token: a lane copies its own short run; runs of kWarpCopyRun bytes or more
    // (a long incompressible stretch) are copied by the whole warp, one after another
    const uint32_t lincl = warp_incl_scan(L);
    const uint32_t lik = li + lincl - L;
    const bool longrun = L >= kWarpCopyRun;
    if (!longrun)
      for (uint32_t k = 0; k < L; ++k) lit[lik + k] = src[opk + k];
    for (unsigned lb = __ballot_sync(kFull, longrun); lb; lb &= lb - 1) {
      const uint32_t r = (uint32_t)__ffs(lb) - 1u;
      const uint32_t rL = __shfl_sync(kFull, L, r), rd = __shfl_sync(kFull, lik, r), rs = __shfl_sync(kFull, opk, r);
      warp_copy_in(lit + rd, src + rs, rL, lane);
    }
    li += __shfl_sync(kFull, lincl, 31);
    ei += __shfl_sync(kFull, xincl, 31);
    op = __shfl_sync(kFull, endk, c - 1);
  }
  if (gcnt) {
    if (lane == 0) grp[ng] = (uint8_t)gcnt;
    ++ng;
  }
  warp_copy_in(lit + li, src + op, n - op, lane);
  li += n - op;
  if (bp > wbase && lane == 0) bitw[wbase >> 5] = cw;
  if (lane == 0) {
    A.bcnt[b * 8 + 1] = li;
    A.bcnt[b * 8 + 2] = ei;
    A.bcnt[b * 8 + 3] = (uint32_t)((bp + 7) / 8);
    A.bcnt[b * 8 + 4] = ng;
  }
}

// ---------------------------------------------------------------- 5. rANS, per (block, stream)
__device__ __forceinline__ const uint8_t* stream_syms(const EncArgs& A, uint32_t b, uint32_t s) {
  const size_t TC = tok_cap(A.B);
  switch (s) {
    case 0: return A.s_lit + (size_t)b * A.B;
    case 1: return A.s_tok + (size_t)b * TC;
    case 2: return A.s_ext + (size_t)b * ext_cap(A.B);
    case 3: return A.s_sym + (size_t)b * TC;
    default: return A.s_grp + (size_t)b * TC;
  }
}
__device__ __forceinline__ uint32_t stream_len(const EncArgs& A, uint32_t b, uint32_t s) {
  const uint32_t* c = A.bcnt + b * 8;
  return s == 0 ? c[1] : s == 2 ? c[2] : s == 4 ? c[4] : c[0];
}

constexpr uint32_t kRansChunk = 4096;  // symbols staged per round: 64 per lane

__global__ void __launch_bounds__(64) k_enc_rans(EncArgs A) {
  const uint32_t b = blockIdx.x, s = blockIdx.y, k = threadIdx.x, g = b * 5 + s;
  const uint32_t ns = stream_len(A, b, s);
  uint32_t* info = A.sinfo + (size_t)g * 4;
  if (ns == 0) {
    if (k == 0) { info[0] = 0; info[1] = 0; info[2] = 0; info[3] = 0; }
    return;
  }
  const uint8_t* sym = stream_syms(A, b, s);
  // per symbol: fc = freq | cum << 13 | (ceil(log2 freq) - 1) << 25, rcp = ceil(2^(31 + ceil(log2 freq)) / freq)
  __shared__ uint32_t hist[256], fc[256], rcp[256], red[3];
  __shared__ __align__(16) uint8_t stage[kRansChunk];
  for (uint32_t i = k; i < 256; i += 64) hist[i] = 0;
  __syncthreads();
  for (uint32_t i = k; i < ns; i += 64) atomicAdd(&hist[sym[i]], 1u);
  __syncthreads();
  // normalisation (src/codec.h:41-66) by warp 0: lane l holds symbols 8l .. 8l+7
  if (k < 32) {
    uint32_t f[8], sum = 0, np = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint32_t c = hist[k * 8 + q];
      f[q] = c ? max(1u, (uint32_t)(((uint64_t)c << kScaleBits) / ns)) : 0u;
      sum += f[q];
      np += c != 0;
    }
    sum = warp_sum(sum);
    np = warp_sum(np);
    // too many: one from the largest frequency above 1 (the lowest symbol on a tie), repeatedly
    while (sum > kScale) {
      uint32_t bv = 0, bi = 0xFFFFFFFFu;
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (f[q] > 1 && f[q] > bv) { bv = f[q]; bi = k * 8 + q; }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const uint32_t ov = __shfl_xor_sync(kFull, bv, o), oi = __shfl_xor_sync(kFull, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if ((bi >> 3) == k) {
#pragma unroll
        for (int q = 0; q < 8; ++q) if ((uint32_t)q == (bi & 7u)) --f[q];
      }
      --sum;
    }
    if (sum < kScale) {  // too few: the deficit to the largest (the lowest symbol on a tie)
      uint32_t bv = f[0], bi = k * 8;
#pragma unroll
      for (int q = 1; q < 8; ++q)
        if (f[q] > bv) { bv = f[q]; bi = k * 8 + q; }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const uint32_t ov = __shfl_xor_sync(kFull, bv, o), oi = __shfl_xor_sync(kFull, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if ((bi >> 3) == k) {
#pragma unroll
        for (int q = 0; q < 8; ++q) if ((uint32_t)q == (bi & 7u)) f[q] += kScale - sum;
      }
    }
    uint32_t tot = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) tot += f[q];
    uint32_t c0 = warp_incl_scan(tot) - tot;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint32_t sl = f[q] > 1 ? 32u - __clz(f[q] - 1u) : 1u;  // ceil(log2 f)
      fc[k * 8 + q] = f[q] | c0 << 13 | (sl - 1u) << 25;
      rcp[k * 8 + q] = f[q] > 1 ? (uint32_t)(((1ull << (31 + sl)) + f[q] - 1u) / f[q]) : 0u;
      A.freq[(size_t)g * 256 + k * 8 + q] = (uint16_t)f[q];
      c0 += f[q];
    }
    if (k == 0) red[0] = np;
  }
  __syncthreads();
  // lane k codes symbols k, k+64, ... last first, backwards into its scratch (src/codec.h:112-128)
  const uint32_t LC = lane_cap(A.B, s);
  uint8_t* end = A.lanes + (size_t)b * lanes_per_block(A.B) + lane_base(A.B, s) + (size_t)(k + 1) * LC;
  uint8_t* ptr = end;
  // output bytes go down from the lane's (16-byte aligned) end; they are gathered four at a time, the
  // first at bits 31..24, and stored as aligned words
  uint32_t acc = 0, pend = 0;
  uint32_t x = kRansLow;
  // The stream in chunks of kRansChunk symbols (a whole number of rounds of the 64 lanes), last chunk
  // first: the CTA stages a chunk in shared memory with coalesced loads, then lane k codes its symbols
  // c0 + k + 64 j of it, j descending -- the order of the whole-stream loop, without a global load on
  // the state's dependency chain.
  const bool al4 = ((uintptr_t)sym & 3u) == 0;
  for (int32_t ch = (int32_t)((ns - 1) / kRansChunk); ch >= 0; --ch) {
    const uint32_t c0 = (uint32_t)ch * kRansChunk, cn = min(kRansChunk, ns - c0);
    __syncthreads();  // (the previous chunk is coded)
    uint32_t t0 = 0;
    if (al4) {
      const uint32_t n4 = cn >> 2;
      for (uint32_t t = k; t < n4; t += kLanes)
        reinterpret_cast<uint32_t*>(stage)[t] = reinterpret_cast<const uint32_t*>(sym + c0)[t];
      t0 = n4 << 2;
    }
    for (uint32_t t = t0 + k; t < cn; t += kLanes) stage[t] = sym[c0 + t];
    __syncthreads();
    if (k < cn) {
      // x' = (x / f) * 4096 + x % f + cum = x + cum + q * (4096 - f), with q = x / f by an exact
      // reciprocal: for x < 2^31 and s = ceil(log2 f), floor(x * ceil(2^(31+s) / f) / 2^(31+s)) = x / f
      // (the product's error is below x / 2^(31+s) < 2^-s <= 1/f, less than the gap to the next integer)
      for (int32_t t = (int32_t)(k + (cn - 1 - k) / kLanes * kLanes); t >= 0; t -= (int32_t)kLanes) {
        const uint32_t c = stage[t], e = fc[c], m = rcp[c];
        const uint32_t f = e & 0x1FFFu;
        const uint32_t xmax = f << (23 - kScaleBits + 8);
        while (x >= xmax) {
          acc |= (x & 0xFFu) << (24u - 8u * pend);
          x >>= 8;
          if (++pend == 4u) {
            ptr -= 4;
            *reinterpret_cast<uint32_t*>(ptr) = acc;
            acc = 0;
            pend = 0;
          }
        }
        const uint32_t q = f == 1 ? x : __umulhi(x, m) >> (e >> 25);
        x += ((e >> 13) & 0xFFFu) + q * (kScale - f);
      }
    }
  }
  for (uint32_t i = 0; i < pend; ++i) *--ptr = (uint8_t)(acc >> (24u - 8u * i));  // the bytes still gathered
  ptr -= 4;
  st32(ptr, x);
  const uint32_t ll = (uint32_t)(end - ptr);
  A.lanelen[(size_t)g * kLanes + k] = ll;
  const uint32_t lsum = warp_sum(ll);
  if (lane_id() == 0) red[1 + (k >> 5)] = lsum;
  __syncthreads();
  if (k == 0) {
    const uint32_t np = red[0];
    const uint32_t total = 32 + 2 * np + 4 * kLanes + red[1] + red[2];
    const uint32_t kind = total >= ns ? 0u : 1u;  // raw when rANS is not smaller (src/codec.h:130)
    info[0] = kind;
    info[1] = kind ? total : ns;
    info[2] = np;
    info[3] = ns;
  }
}

// ---------------------------------------------------------------- 6. the payload
__global__ void __launch_bounds__(256) k_enc_pack(EncArgs A) {
  const uint32_t b = blockIdx.x, tid = threadIdx.x;
  const uint32_t n = A.in_len[b];
  uint32_t* c = A.bcnt + b * 8;
  const uint32_t nob = c[3];
  uint64_t off[6];
  off[0] = kHdrBytes;
  for (uint32_t s = 0; s < 5; ++s) off[s + 1] = off[s] + 5 + A.sinfo[(size_t)(b * 5 + s) * 4 + 1];
  const uint64_t total = off[5] + nob;
  if (total >= n) {  // stored (src/codec2.h:152, src/archive.h:394)
    if (tid == 0) { c[5] = n; c[6] = 0; }
    return;
  }
  uint8_t* o = A.slab + (size_t)b * A.B;
  if (tid == 0) {
    st32(o, c[0]); st32(o + 4, c[1]); st32(o + 8, c[2]); st32(o + 12, nob); st32(o + 16, c[4]);
    c[5] = (uint32_t)total; c[6] = 1;
  }
  __shared__ uint32_t lofs[kLanes + 1];
  __shared__ uint32_t wcnt[8];
  for (uint32_t s = 0; s < 5; ++s) {
    const uint32_t g = b * 5 + s;
    const uint32_t* info = A.sinfo + (size_t)g * 4;
    const uint32_t kind = info[0], len = info[1], np = info[2], ns = info[3];
    uint8_t* d = o + off[s];
    if (tid == 0) { d[0] = (uint8_t)kind; st32(d + 1, len); }
    const uint8_t* sym = stream_syms(A, b, s);
    if (kind == 0) {
      for (uint32_t i = tid; i < ns; i += blockDim.x) d[5 + i] = sym[i];
      continue;
    }
    const uint16_t* fq = A.freq + (size_t)g * 256;
    // present bitmap, then the frequencies of the present symbols in symbol order
    const uint32_t f = fq[tid];
    const uint32_t pres = f != 0;
    const unsigned bal = __ballot_sync(kFull, pres);
    if ((tid & 7u) == 0) d[5 + (tid >> 3)] = (uint8_t)((bal >> (tid & 31u)) & 0xFFu);
    if ((tid & 31u) == 0) wcnt[tid >> 5] = __popc(bal);
    __syncthreads();
    uint32_t idx = __popc(bal & ((1u << (tid & 31u)) - 1u));
    for (uint32_t k = 0; k < (tid >> 5); ++k) idx += wcnt[k];
    if (pres) { d[5 + 32 + 2 * idx] = (uint8_t)f; d[5 + 32 + 2 * idx + 1] = (uint8_t)(f >> 8); }
    const uint32_t* ll = A.lanelen + (size_t)g * kLanes;
    if (tid < kLanes) st32(d + 5 + 32 + 2 * np + 4 * tid, ll[tid]);
    if (tid < 32) {
      const uint32_t a = ll[2 * tid], bb = ll[2 * tid + 1];
      const uint32_t inc = warp_incl_scan(a + bb);
      lofs[2 * tid] = inc - a - bb;
      lofs[2 * tid + 1] = inc - bb;
    }
    __syncthreads();
    const uint32_t data0 = 5 + 32 + 2 * np + 4 * kLanes;
    const uint32_t LC = lane_cap(A.B, s);
    const uint8_t* lb = A.lanes + (size_t)b * lanes_per_block(A.B) + lane_base(A.B, s);
    for (uint32_t jl = tid >> 5; jl < kLanes; jl += blockDim.x >> 5) {
      const uint32_t len_j = ll[jl];
      const uint8_t* srcp = lb + (size_t)(jl + 1) * LC - len_j;
      uint8_t* dst = d + data0 + lofs[jl];
      for (uint32_t i = lane_id(); i < len_j; i += 32) dst[i] = srcp[i];
    }
    __syncthreads();
  }
  const uint8_t* bits = A.s_bits + (size_t)b * bits_cap(A.B);
  for (uint32_t i = tid; i < nob; i += blockDim.x) o[off[5] + i] = bits[i];
}

// ---------------------------------------------------------------- 7. record bodies back to back
__global__ void __launch_bounds__(1024) k_enc_scan(EncArgs A) {
  const uint32_t tid = threadIdx.x, nb = A.nb;
  const uint32_t per = (nb + 1023) / 1024;
  const uint32_t b0 = min(tid * per, nb), b1 = min(b0 + per, nb);
  uint64_t sum = 0;
  for (uint32_t b = b0; b < b1; ++b) {
    const uint32_t* c = A.bcnt + b * 8;
    sum += A.rec_hdr + (c[6] ? c[5] : (A.emit_stored ? A.in_len[b] : 0u));
  }
  __shared__ uint64_t ws[32];
  uint64_t incl = sum;
  const uint32_t l = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t t = __shfl_up_sync(kFull, incl, o);
    if (l >= (uint32_t)o) incl += t;
  }
  if (l == 31) ws[tid >> 5] = incl;
  __syncthreads();
  if (tid < 32) {
    uint64_t v = ws[tid], x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t t = __shfl_up_sync(kFull, x, o);
      if (l >= (uint32_t)o) x += t;
    }
    ws[tid] = x - v;
  }
  __syncthreads();
  uint64_t off = (A.rec_base ? *A.rec_base : 0ull) + ws[tid >> 5] + incl - sum;
  for (uint32_t b = b0; b < b1; ++b) {
    const uint32_t* c = A.bcnt + b * 8;
    const uint32_t method = c[6];
    const uint32_t len = method ? c[5] : A.in_len[b];
    off += A.rec_hdr;
    A.out_off[b] = off;
    A.out_len[b] = len;
    A.out_method[b] = (uint8_t)method;
    off += method ? len : (A.emit_stored ? len : 0u);
  }
  if (tid == 1023) *A.out_total = off;
}

__global__ void __launch_bounds__(256) k_enc_emit(EncArgs A) {
  const uint32_t b = blockIdx.x;
  const uint32_t method = A.bcnt[b * 8 + 6];
  if (!method && !A.emit_stored) return;
  const uint64_t off = A.out_off[b];
  const uint32_t len = A.out_len[b];
  if (off + len > A.out_cap) return;  // (the host checks out_total against out_cap)
  const uint8_t* s = method ? A.slab + (size_t)b * A.B : A.in + A.in_off[b];
  uint8_t* d = A.out + off;
  if (A.rec_hdr && threadIdx.x < 16) {  // the record header just before the body (off >= 16 here)
    const uint32_t t = threadIdx.x, w = t >> 2, sh = 8u * (t & 3u);
    const uint32_t v = w == 0 ? A.in_len[b] : w == 1 ? len : w == 2 ? method : A.rec_crc[b];
    d[(int)t - 16] = (w == 2 && t != 8) ? 0 : (uint8_t)(v >> sh);
  }
  uint32_t i = 0;
  if ((((uintptr_t)d ^ (uintptr_t)s) & 15u) == 0) {
    const uint32_t head = min(len, (uint32_t)((16u - ((uintptr_t)d & 15u)) & 15u));
    if (threadIdx.x < head) d[threadIdx.x] = s[threadIdx.x];
    i = head;
    const uint32_t nvec = (len - i) / 16;
    for (uint32_t v = threadIdx.x; v < nvec; v += blockDim.x)
      reinterpret_cast<uint4*>(d + i)[v] = reinterpret_cast<const uint4*>(s + i)[v];
    i += nvec * 16;
  } else {
    // not co-aligned (every record of an archive): 4-byte words stored aligned at d, each built by a funnel
    // shift from the two aligned source words that cover it (those reach at most 3 bytes past the body,
    // inside the input's slack or the slab's padding)
    const uint32_t head = min(len, (uint32_t)((4u - ((uintptr_t)d & 3u)) & 3u));
    if (threadIdx.x < head) d[threadIdx.x] = s[threadIdx.x];
    i = head;
    const uint32_t nw = (len - i) >> 2, sh = (uint32_t)((uintptr_t)(s + i) & 3u);
    const uint32_t* sw = reinterpret_cast<const uint32_t*>(s + i - sh);
    uint32_t* dw = reinterpret_cast<uint32_t*>(d + i);
    if (sh == 0) {
      for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) dw[w] = sw[w];
    } else {
      for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) dw[w] = __funnelshift_r(sw[w], sw[w + 1], 8u * sh);
    }
    i += nw * 4;
  }
  for (uint32_t k = i + threadIdx.x; k < len; k += blockDim.x) d[k] = s[k];
}

size_t match_smem_bytes(uint32_t tile, uint32_t depth, uint32_t wb) {
  return (size_t)(tile + depth) * (wb + 4 + 2) + 4 + (size_t)tile * 8;  // (+ the work list)
}

cudaError_t prepare_kernels() {  // with the device current, once per context
  cudaError_t e = cudaFuncSetAttribute(k_enc_match<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)match_smem_bytes(kMaxMatchTile, 256, 32));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_enc_match<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)match_smem_bytes(kMaxMatchTile, 256, 16));
  return e == cudaSuccess ? prepare_fill() : e;
}

void launch_encode(const EncArgs& A, const CrcArgs& crc_in, cudaStream_t st, Stages& S) {
  if (!A.nb) return;
  launch_crc(crc_in, st, S, "k_crc_in");
  const dim3 sg((A.B + kSortTile - 1) / kSortTile, A.nb);
  S.begin("k_sort_count", st);
  k_sort_count<0><<<sg, 256, 0, st>>>(A);
  S.end(st);
  S.begin("k_sort_scan", st);
  k_sort_scan<<<A.nb, 256, 0, st>>>(A);
  S.end(st);
  S.begin("k_sort_scatter", st);
  k_sort_scatter<0><<<sg, kSortThreads, 0, st>>>(A);
  S.end(st);
  S.begin("k_sort_count", st);
  k_sort_count<1><<<sg, 256, 0, st>>>(A);
  S.end(st);
  S.begin("k_sort_scan", st);
  k_sort_scan<<<A.nb, 256, 0, st>>>(A);
  S.end(st);
  S.begin("k_sort_scatter", st);
  k_sort_scatter<1><<<sg, kSortThreads, 0, st>>>(A);
  S.end(st);
  S.begin("k_enc_match", st);
  const dim3 mg((A.B + A.match_tile - 1) / A.match_tile, A.nb);
  if (A.cmp_cap <= 16) k_enc_match<16><<<mg, 256, match_smem_bytes(A.match_tile, (uint32_t)A.depth, 16), st>>>(A);
  else k_enc_match<32><<<mg, 256, match_smem_bytes(A.match_tile, (uint32_t)A.depth, 32), st>>>(A);
  S.end(st);
  S.begin("k_enc_parse", st);
  k_enc_parse<<<A.nb, 256, 0, st>>>(A);
  S.end(st);
  S.begin("k_enc_streams", st);
  k_enc_streams<<<(A.nb + 3) / 4, 128, 0, st>>>(A);
  S.end(st);
  S.begin("k_enc_rans", st);
  k_enc_rans<<<dim3(A.nb, 5), 64, 0, st>>>(A);
  S.end(st);
  S.begin("k_enc_pack", st);
  k_enc_pack<<<A.nb, 256, 0, st>>>(A);
  S.end(st);
  S.begin("k_enc_scan", st);
  k_enc_scan<<<1, 1024, 0, st>>>(A);
  S.end(st);
  S.begin("k_enc_emit", st);
  k_enc_emit<<<A.nb, 256, 0, st>>>(A);
  S.end(st);
}

}  // namespace zc
