// zc_kernels.h -- argument blocks and launchers of the ZB2 kernels (host and device view).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace zc {

struct CrcTables;

// kernel launch accounting and optional per-stage timing with CUDA events on the launching stream
// (the counterpart of the reference's ZERO_PROFILE stage timer, src/gpu_codec.h:32-49, without its
// device syncs).  Implemented in zc_api.cu.
struct Stages {
  bool timing = false;
  uint64_t launches = 0;
  void* impl = nullptr;  // the context's event records
  void begin(const char* name, cudaStream_t st);  // call before a kernel launch
  void end(cudaStream_t st);                      // and after it
};

// ---- decoder
struct DecMeta {  // per block: the payload's framing (k_dec_locate) and the replay's totals (k_dec_tokens)
  uint32_t nt, nl, ne, nob, ng;  // tokens, literals, ext bytes, offset-bit bytes, groups
  uint32_t bits_off;             // where the offset bits start in the payload
  uint32_t s_off[5], s_len[5];   // each stream body's offset in the payload and its length
  uint32_t kinds;                // bit s: stream s is rANS-coded (else raw)
  uint32_t op_total, li_total;   // output and literal bytes of all tokens (the literal tail follows)
};

struct DecArgs {
  const uint8_t* comp;        // payloads
  const uint64_t* comp_off;   // per block
  const uint32_t* comp_len;
  const uint8_t* method;
  const uint32_t* raw_len;
  uint32_t nb, B;
  uint8_t* out;               // raw bytes of block b at out + out_off[b]
  const uint64_t* out_off;
  uint32_t* err;              // per block status (zeroed before)
  // scratch, per block slot b: lit at b*B, tok / sym / grp at b*tok_cap(B), ext at b*ext_cap(B)
  uint8_t *s_lit, *s_tok, *s_sym, *s_grp, *s_ext;
  DecMeta* meta;
  // the replay: per token (tok_cap(B) per block) its output start, match start, offset and literal start
  uint32_t *tk_start, *tk_ms, *tk_d, *tk_lik;
  // the fill's shape: a ring of 2^ring_log recent output bytes per warp, fill_warps warps (blocks) per CTA,
  // fill_words output words a lane a round (1, 2 or 4)
  uint32_t ring_log, fill_warps, fill_words;
  uint32_t* work;             // the fill's device work counter (zeroed by the launcher)
};

constexpr uint32_t kMinFillRingLog = 11, kMaxFillRingLog = 15, kMaxFillWarps = 8;
constexpr size_t kMaxFillSmem = 227 * 1024;
size_t fill_smem_bytes(uint32_t ring_log, uint32_t warps, uint32_t words);

struct CrcArgs {
  const uint8_t* base;
  const uint64_t* offs;
  const uint32_t* lens;
  uint32_t nb;
  uint32_t* crc;              // out, per block
  uint32_t* err;              // optional: blocks with err != 0 are skipped; with expect, a mismatch sets E_CRC
  const uint32_t* expect;     // optional
  const CrcTables* tables;
};

void launch_dec_streams(const DecArgs& A, cudaStream_t st, Stages& S);  // framing + the rANS streams
void launch_decode_fill(const DecArgs& A, cudaStream_t st, Stages& S);  // streams + token scan + fill
void launch_crc(const CrcArgs& A, cudaStream_t st, Stages& S, const char* name);

// ---- encoder
struct EncArgs {
  const uint8_t* in;          // block b: in_len[b] bytes at in + in_off[b]; 16-aligned, >= 64 readable bytes after the last
  const uint64_t* in_off;
  const uint32_t* in_len;
  uint32_t nb, B, block_log;
  int depth;                  // hash chain steps (8 / 32 / 256)
  uint32_t cmp_cap;           // bytes the all-position match pass compares before deferring to the parse
  uint32_t match_tile;        // sorted positions per match CTA: 256, 512 or 1024
  uint32_t match_dense;       // unfinished positions from which a match tile scans a lane per position
  uint32_t match_defer;       // backward bytes that mark a position as inside a longer match (0: none)
  // scratch, per block slot (capacity B positions)
  uint32_t *tmp_pos, *srt_pos, *minfo;
  uint32_t* scnt;                 // sort: per block ceil(B / 4096) * 256 tile digit counts / starts
  uint16_t *tmp_h, *srt_h;
  uint32_t *tk_i, *tk_m, *tk_d;   // tokens, tok_cap(B) per block
  uint32_t* tk_seg;               // the parse's per-segment token slots: 3 * seg_tok_cap(B) per block
  uint32_t* bcnt;                 // per block [8]: nt, nl, ne, nob, ng, payload size, method
  uint8_t *s_lit, *s_tok, *s_ext, *s_sym, *s_grp, *s_bits;
  uint8_t* lanes;                 // rANS lane scratch, lanes_per_block(B) per block
  uint16_t* freq;                 // per (block, stream) 256
  uint32_t* lanelen;              // per (block, stream) 64
  uint32_t* sinfo;                // per (block, stream) 4: kind, section body length, present symbols, symbols
  uint8_t* slab;                  // per block B bytes: the payload when it is smaller than the block
  // output
  uint8_t* out;                   // record bodies packed back to back
  uint64_t out_cap;
  uint64_t* out_off;              // per block
  uint32_t* out_len;              // per block: payload length (raw length when stored)
  uint8_t* out_method;            // per block
  uint64_t* out_total;            // device u64: bytes written to out (record mode: the end of the last record)
  int emit_stored;                // 1: copy stored blocks' raw bytes into out as well
  // archive record mode (rec_hdr = 16): every body is preceded by its block record header {u32 raw_len,
  // u32 comp_len, u8 method, 3 zero bytes, u32 crc} (src/archive.h:389-403), the first record at
  // *rec_base; rec_crc holds the blocks' CRCs (written by the first stage).  rec_hdr = 0: bodies from 0.
  uint32_t rec_hdr;
  const uint64_t* rec_base;
  const uint32_t* rec_crc;
};

// lane scratch layout per block: stream s starts at lane_base(s), each of its 64 lanes has lane_cap(s)
// bytes (rANS emits at most 2 bytes per symbol plus a 4-byte flush); every lane's end is 16-byte aligned
__host__ __device__ inline uint32_t stream_cap(uint32_t B, uint32_t s) {
  return s == 0 ? B : s == 2 ? B / 5 + 64 : B / 4 + 16;
}
__host__ __device__ inline uint32_t lane_cap(uint32_t B, uint32_t s) {  // a multiple of 16: lanes end aligned
  return (2 * ((stream_cap(B, s) + 63) / 64) + 16 + 15) & ~15u;
}
__host__ __device__ inline uint64_t lane_base(uint32_t B, uint32_t s) {
  uint64_t o = 0;
  for (uint32_t k = 0; k < s; ++k) o += 64ull * lane_cap(B, k);
  return o;
}
__host__ __device__ inline uint64_t lanes_per_block(uint32_t B) { return lane_base(B, 5); }
__host__ __device__ inline uint32_t bits_cap(uint32_t B) { return 5 * B / 8 + 64; }
// the parse's token slots per block: 256 segments of ceil(B / 256) bytes, ceil(B / 256) / 4 + 2 each
__host__ __device__ inline uint32_t seg_tok_cap(uint32_t B) { return 256 * (((B + 255) / 256) / 4 + 2); }

void launch_encode(const EncArgs& A, const CrcArgs& crc_in, cudaStream_t st, Stages& S);
constexpr uint32_t kMaxMatchTile = 1024;
size_t match_smem_bytes(uint32_t tile, uint32_t depth, uint32_t window_bytes);
cudaError_t prepare_kernels();
cudaError_t prepare_fill();  // per-kernel attributes (the sort's shared memory), the device current

}  // namespace zc
