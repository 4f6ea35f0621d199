// zref_harness.cpp -- TEST INFRASTRUCTURE ONLY.  A C-callable shim over the reference's own CPU codec,
// compiled from the reference's headers where they lie (oracle/Makefile adds -I <reference>/src).  No
// reference source is copied here: this file only calls it.  The build output goes to oracle/_ref/,
// which is never committed.  Used to pin the C restatement (oracle/zb2_oracle.c), to write the golden
// vectors, to check the CUDA codec's archives through the reference reader, and as the timed CPU
// baseline (the reference CpuCodec with all host threads).
#include "archive.h"  // reference: src/archive.h (pulls codec2.h, codec.h, crc32.h, platform.h)

#include <cstring>
#include <string>
#include <vector>

namespace {
thread_local std::string g_err;
int fail(const std::exception& e) { g_err = e.what(); return -1; }
}  // namespace

extern "C" {

const char* zref_last_error() { return g_err.c_str(); }

uint32_t zref_crc32(const uint8_t* p, size_t n) { return crc32::of(p, n); }
uint32_t zref_crc32_update(uint32_t c, const uint8_t* p, size_t n) { return crc32::update(c, p, n); }
uint32_t zref_crc32_combine(uint32_t a, uint32_t b, uint64_t len_b) { return crc32::combine(a, b, len_b); }

void zref_normalize(const uint32_t* counts, uint32_t total, uint16_t* freq) { zb::normalize(counts, total, freq); }

// zb::encode_stream (src/codec.h:96-147); returns the section size, or -1 when out is too small
long zref_encode_stream(const uint8_t* sym, uint32_t n, uint8_t* out, size_t cap) {
  std::vector<uint8_t> v;
  zb::encode_stream(sym, n, v);
  if (v.size() > cap) return -1;
  memcpy(out, v.data(), v.size());
  return (long)v.size();
}

// zb::decode_stream (src/codec.h:150-205); bytes consumed, or -1 on damage
long zref_decode_stream(const uint8_t* p, size_t avail, uint32_t n, uint8_t* sym) {
  try { return (long)zb::decode_stream(p, p + avail, n, sym); } catch (const std::exception& e) { return fail(e); }
}

// zb2::parse (src/codec2.h:43-81) with Params{depth}; returns the token count (cap exceeded: -1)
long zref_parse(const uint8_t* in, uint32_t n, int depth, uint32_t* ti, uint32_t* tm, uint32_t* td, size_t cap) {
  zb2::Params P;
  P.depth = depth;
  std::vector<zb2::RawToken> tk;
  zb2::parse(in, n, P, tk);
  if (tk.size() > cap) return -1;
  for (size_t k = 0; k < tk.size(); ++k) { ti[k] = tk[k].i; tm[k] = tk[k].m; td[k] = tk[k].d; }
  return (long)tk.size();
}

// zb2::compress_block (src/codec2.h:84-153); writes the payload, returns its size (the block is stored
// when the size is >= n, as the reference's writer decides at src/archive.h:394), -1 when cap is short
long zref_compress_block(const uint8_t* in, uint32_t n, int depth, uint8_t* out, size_t cap) {
  zb2::Params P;
  P.depth = depth;
  std::vector<uint8_t> v;
  zb2::compress_block(in, n, v, P);
  if (v.size() > cap) return -1;
  memcpy(out, v.data(), v.size());
  return (long)v.size();
}

// zb2::decompress_block (src/codec2.h:155-203); 0, or -1 on damage
int zref_decompress_block(const uint8_t* in, size_t len, uint8_t* out, uint32_t n) {
  try { zb2::decompress_block(in, len, out, n); return 0; } catch (const std::exception& e) { return fail(e); }
}

// ---- the reference CpuCodec (src/archive.h:97-136), all host threads: the timed CPU baseline.
// compress: n bytes in blocks of 2^block_log; per block method (0 stored, 1 ZB2) and payload length;
// payloads are written to out at b * out_stride.  Returns 0 or -1.
int zref_cpu_compress(const uint8_t* in, size_t n, uint32_t block_log, int depth, uint8_t* methods, uint32_t* lens,
                      uint8_t* out, size_t out_stride) {
  try {
    zero::CpuCodec c;
    c.depth = depth;
    std::vector<zero::BlockOut> outs;
    c.compress(in, n, block_log, outs);
    const size_t B = (size_t)1 << block_log;
    for (size_t b = 0; b < outs.size(); ++b) {
      const size_t len = std::min(B, n - b * B);
      const bool stored = outs[b].method == 0 || outs[b].data.size() >= len;
      methods[b] = stored ? 0 : 1;
      lens[b] = stored ? (uint32_t)len : (uint32_t)outs[b].data.size();
      if (out && !stored) {
        if (outs[b].data.size() > out_stride) throw zb::Error("payload larger than the stride");
        memcpy(out + b * out_stride, outs[b].data.data(), outs[b].data.size());
      }
    }
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

// decompress nb blocks; block b's bytes at comp + offs[b], comp_lens[b], method methods[b], raw_lens[b].
// Writes the concatenated raw bytes to out.  Returns 0 or -1.
int zref_cpu_decompress(const uint8_t* comp, const uint64_t* offs, const uint32_t* comp_lens, const uint8_t* methods,
                        const uint32_t* raw_lens, size_t nb, uint8_t* out) {
  try {
    zero::CpuCodec c;
    std::vector<zero::BlockIn> ins(nb);
    size_t total = 0;
    for (size_t b = 0; b < nb; ++b) {
      ins[b].method = methods[b];
      ins[b].raw_len = raw_lens[b];
      ins[b].data = comp + offs[b];
      ins[b].comp_len = comp_lens[b];
      total += raw_lens[b];
    }
    const uint8_t* r = c.decompress(ins);
    if (total) memcpy(out, r, total);
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

// ---- the archive entry points (src/archive.h:334-441, 724-744, 747-785) with the CPU codec
int zref_compress_archive(const char* const* inputs, int n_inputs, const char* out_path, uint32_t block_log, int level) {
  try {
    zero::Report rep;
    zero::CpuCodec c;
    c.depth = level <= 1 ? 8 : level >= 9 ? 256 : 32;  // src/main.cpp:54
    std::vector<std::string> in(inputs, inputs + n_inputs);
    zero::compress_archive(in, out_path, c, block_log, rep);
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}
int zref_extract_archive(const char* path, const char* out_dir) {
  try {
    zero::Report rep;
    zero::CpuCodec c;
    zero::extract_archive(path, out_dir, c, rep);
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}
int zref_test_archive(const char* path) {
  try {
    zero::Report rep;
    zero::CpuCodec c;
    zero::test_archive(path, c, rep);
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

unsigned zref_hardware_threads() { return zero::hardware_threads(); }

}  // extern "C"
