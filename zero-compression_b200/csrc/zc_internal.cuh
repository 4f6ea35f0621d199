// zc_internal.cuh -- shared definitions of the sm_100a ZB2 codec kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace zc {

// ---- format constants (src/codec.h:18-27 for the coder, src/codec2.h:23-24 for the block)
constexpr uint32_t kLanes = 64;            // interleaved rANS lanes per stream
constexpr uint32_t kScaleBits = 12;
constexpr uint32_t kScale = 1u << kScaleBits;
constexpr uint32_t kRansLow = 1u << 23;
constexpr uint32_t kHdrBytes = 20;         // u32 n_tokens, n_lits, n_ext, n_offbits, n_groups
constexpr uint32_t kSymRep = 250;          // symbols 250..252: a recent offset
constexpr uint32_t kMaxMatch = 4096;       // the CPU parse's longest match (src/codec2.h:31)
constexpr uint32_t kMaxGroup = 255;
constexpr uint32_t kMinBlockLog = 16, kMaxBlockLog = 20;
constexpr uint32_t kRecHdr = 16;           // block record header in the archive (src/archive.h:395-399)

// per-block caps a valid block respects (a block above them is damaged): every token emits >= 4 bytes,
// so tokens <= n/4; ext bytes <= n/5 (3 per >= 15 literals, 2 per >= 19 match bytes)
__host__ __device__ inline uint32_t tok_cap(uint32_t B) { return B / 4 + 16; }
__host__ __device__ inline uint32_t ext_cap(uint32_t B) { return B / 5 + 64; }

// decoder status codes per block (0 = good)
enum : uint32_t { E_HDR = 1, E_COUNTS = 2, E_STREAM = 3, E_TABLE = 4, E_LANE = 5, E_TOKEN = 6, E_METHOD = 7,
                  E_STORED = 8, E_RAWLEN = 9, E_CRC = 10 };

// ---- little-endian byte access
__device__ __forceinline__ uint32_t ld32(const uint8_t* p) {
  return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
}
__device__ __forceinline__ void st32(uint8_t* p, uint32_t v) {
  p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}
__device__ __forceinline__ uint32_t bitlen(uint32_t d) { return 31u - __clz(d); }  // d >= 1

// ---- warp helpers
constexpr unsigned kFull = 0xFFFFFFFFu;
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  const uint32_t l = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, v, o);
    if (l >= (uint32_t)o) v += t;
  }
  return v;
}
__device__ __forceinline__ uint32_t warp_sum(uint32_t v) { return __reduce_add_sync(kFull, v); }

// ---- CRC-32 (IEEE, reflected 0xEDB88320; src/crc32.h).  Linear algebra over GF(2):
// raw0(M) = the CRC register after M from a zero register, no inversions.  Leading zero bytes leave it
// unchanged, raw0(A||B) = raw0(A) * x^(8|B|) ^ raw0(B), and the standard CRC is
// crc(M) = raw0(M) ^ (0xFFFFFFFF * x^(8|M|)) ^ 0xFFFFFFFF.
struct CrcTables {
  uint32_t t[8][256];        // slice-by-8: t[k][b] = raw0 of byte b followed by k zero bytes
  uint32_t pow2[64];         // pow2[e] = x^(8 * 2^e) mod P, reflected (bit 31 = x^0)
};

__host__ __device__ inline uint32_t gf2_mul(uint32_t a, uint32_t b) {  // a*b mod P, reflected order
  uint32_t acc = 0;
  for (int i = 0; i < 32; ++i) {
    acc ^= b & (0u - (a >> 31));
    a <<= 1;
    b = (b >> 1) ^ (0xEDB88320u & (0u - (b & 1u)));
  }
  return acc;
}
// x^(8n) mod P from the power table
__device__ inline uint32_t gf2_xpow8n(const uint32_t* pow2, uint64_t n) {
  uint32_t r = 0x80000000u;
  for (int e = 0; n; ++e, n >>= 1)
    if (n & 1u) r = gf2_mul(r, pow2[e]);
  return r;
}
// raw0 register over n bytes at p (any alignment) continuing from c
__device__ inline uint32_t crc_raw_bytes(const uint32_t (*t)[256], uint32_t c, const uint8_t* p, uint32_t n) {
  uint32_t i = 0;
  const uint32_t head = (uint32_t)((8u - ((uintptr_t)p & 7u)) & 7u);
  for (; i < n && i < head; ++i) c = t[0][(c ^ p[i]) & 0xFFu] ^ (c >> 8);
  for (; i + 8 <= n; i += 8) {
    const uint2 w = *reinterpret_cast<const uint2*>(p + i);
    const uint32_t a = w.x ^ c, b = w.y;
    c = t[7][a & 0xFFu] ^ t[6][(a >> 8) & 0xFFu] ^ t[5][(a >> 16) & 0xFFu] ^ t[4][a >> 24] ^
        t[3][b & 0xFFu] ^ t[2][(b >> 8) & 0xFFu] ^ t[1][(b >> 16) & 0xFFu] ^ t[0][b >> 24];
  }
  for (; i < n; ++i) c = t[0][(c ^ p[i]) & 0xFFu] ^ (c >> 8);
  return c;
}

// Standard CRC-32 of n bytes at p, computed by all threads of the CTA (blockDim.x a multiple of 32, at
// most 1024).  The range is front-padded with zeros to nthreads * c bytes, c a power of two, so every
// thread's chunk has the same length and each level of the combining tree shifts by a table power.
// red: shared scratch of blockDim.x/32 words.  Returns the CRC on every thread.
__device__ inline uint32_t cta_crc32(const CrcTables* T, const uint32_t (*t)[256], const uint8_t* p, uint32_t n,
                                     uint32_t* red) {
  const uint32_t nthr = blockDim.x, tid = threadIdx.x;
  uint32_t e = 3;  // c = 2^e bytes per thread, at least 8
  while (((uint64_t)nthr << e) < n) ++e;
  const uint64_t c = 1ull << e, span = (uint64_t)nthr << e, pad = span - n;
  const uint64_t v0 = (uint64_t)tid * c, v1 = v0 + c;
  uint32_t r = 0;
  if (v1 > pad) {
    const uint64_t a = v0 > pad ? v0 - pad : 0, b = v1 - pad;
    r = crc_raw_bytes(t, 0, p + a, (uint32_t)(b - a));
  }
  // combine within the warp: level l joins chunks of c * 2^l bytes
  const uint32_t lane = tid & 31u;
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    const uint32_t other = __shfl_down_sync(kFull, r, 1u << l);
    if ((lane & ((2u << l) - 1u)) == 0) r = gf2_mul(r, T->pow2[e + l]) ^ other;
  }
  const uint32_t nw = nthr >> 5, w = tid >> 5;
  __syncthreads();
  if (lane == 0) red[w] = r;
  __syncthreads();
  if (w == 0) {
    r = lane < nw ? red[lane] : 0;
    for (uint32_t l = 0; (1u << l) < nw; ++l) {
      const uint32_t other = __shfl_down_sync(kFull, r, 1u << l);
      if ((lane & ((2u << l) - 1u)) == 0 && lane + (1u << l) < nw) r = gf2_mul(r, T->pow2[e + 5 + l]) ^ other;
    }
    if (lane == 0) red[0] = r ^ gf2_mul(0xFFFFFFFFu, gf2_xpow8n(T->pow2, n)) ^ 0xFFFFFFFFu;
  }
  __syncthreads();
  const uint32_t out = red[0];
  __syncthreads();
  return out;
}

// copies the slice-by-8 tables into shared memory (all threads of the CTA)
__device__ inline void load_crc_tables(const CrcTables* T, uint32_t (*s)[256]) {
  const uint32_t* src = &T->t[0][0];
  uint32_t* dst = &s[0][0];
  for (uint32_t i = threadIdx.x; i < 8 * 256; i += blockDim.x) dst[i] = src[i];
}

}  // namespace zc
