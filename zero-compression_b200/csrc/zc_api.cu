// zc_api.cu -- the C ABI of include/zero_cuda.h: device context, scratch sized per block size, batching
// of host calls into launches, host <-> device copies.  It replaces the reference's GpuCodec
// (src/gpu_codec.h) and the Level Zero runtime under it (src/gpu.h, src/ze_min.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/zero_cuda.h"
#include "zc_host.h"
#include "zc_internal.cuh"
#include "zc_kernels.h"

using namespace zch;

namespace {

__global__ void k_plain_blocks(uint64_t n, uint32_t B, uint32_t nb, uint64_t* off, uint32_t* len) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const uint64_t o = (uint64_t)b * B;
  off[b] = o;
  len[b] = (uint32_t)std::min<uint64_t>(B, n - o);
}

int depth_for_level(int level) { return level <= 1 ? 8 : level >= 9 ? 256 : 32; }
int level_class(int level) { return level <= 1 ? 0 : level >= 9 ? 2 : 1; }

}  // namespace

void zch::build_crc_tables(zc::CrcTables& T) {
  for (uint32_t i = 0; i < 256; ++i) {
    uint32_t r = i;
    for (int k = 0; k < 8; ++k) r = (r >> 1) ^ (0xEDB88320u & (0u - (r & 1u)));
    T.t[0][i] = r;
  }
  for (int k = 1; k < 8; ++k)
    for (uint32_t i = 0; i < 256; ++i) T.t[k][i] = (T.t[k - 1][i] >> 8) ^ T.t[0][T.t[k - 1][i] & 0xFFu];
  uint32_t p = 0x00800000u;  // x^8
  for (int e = 0; e < 64; ++e) { T.pow2[e] = p; p = zc::gf2_mul(p, p); }
}

void zc::Stages::begin(const char* name, cudaStream_t st) {
  ++launches;
  if (!timing || !impl) return;
  StageRecords* R = static_cast<StageRecords*>(impl);
  R->open_name = name;
  R->open_ev = R->get();
  cudaEventRecord(R->open_ev, st);
}
void zc::Stages::end(cudaStream_t st) {
  if (!timing || !impl) return;
  StageRecords* R = static_cast<StageRecords*>(impl);
  cudaEvent_t e = R->get();
  cudaEventRecord(e, st);
  R->pending.push_back({R->open_name, R->open_ev, e});
}

namespace zch {

int fail(zc_ctx* c, int code, const std::string& msg) {
  c->err = msg;
  return code;
}
int cuda_fail(zc_ctx* c, cudaError_t e, const char* what) {
  c->err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? ZC_E_NOMEM : ZC_E_DEVICE;
}

cudaError_t grow(DevBuf& b, size_t bytes) {
  if (bytes <= b.n && b.p) return cudaSuccess;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.n = 0;
  bytes = std::max<size_t>(bytes, 256);
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e == cudaSuccess) b.n = bytes;
  return e;
}
cudaError_t grow_host(HostBuf& b, size_t bytes) {
  if (bytes <= b.n && b.p) return cudaSuccess;
  if (b.p) cudaFreeHost(b.p);
  b.p = nullptr;
  b.n = 0;
  cudaError_t e = cudaMallocHost(&b.p, std::max<size_t>(bytes, 4096));
  if (e == cudaSuccess) b.n = std::max<size_t>(bytes, 4096);
  return e;
}
void release(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.n = 0;
}

void drop_graphs(zc_ctx* c) {
  for (GraphEntry& g : c->graph_cache) cudaGraphExecDestroy(g.exec);
  c->graph_cache.clear();
}

// Scratch is sized by capacity: a call whose buffers already fit (any block size) changes nothing and
// keeps the captured graphs; a call that needs more drops them (they name the buffers being replaced).
struct Need {
  DevBuf* b;
  size_t bytes;
};
template <size_t K>
int ensure(zc_ctx* c, Need (&need)[K]) {
  bool grows = false;
  for (const Need& x : need) grows |= !x.b->p || x.bytes > x.b->n;
  if (!grows) return ZC_OK;
  drop_graphs(c);
  for (const Need& x : need) ZC_CUDA(grow(*x.b, x.bytes));
  return ZC_OK;
}

int ensure_enc(zc_ctx* c, uint32_t nb, uint32_t block_log) {
  const size_t B = (size_t)1 << block_log, TC = zc::tok_cap((uint32_t)B), EC = zc::ext_cap((uint32_t)B);
  const size_t N = (size_t)nb * B;
  Need need[] = {
      {&c->e_tmp_pos, N * 4}, {&c->e_srt_pos, N * 4}, {&c->e_minfo, N * 4},
      {&c->e_scnt, (size_t)nb * ((B + 4095) / 4096) * 256 * 4},
      {&c->e_tk_seg, (size_t)nb * 3 * zc::seg_tok_cap((uint32_t)B) * 4},
      {&c->e_tmp_h, N * 2}, {&c->e_srt_h, N * 2},
      {&c->e_tk_i, nb * TC * 4}, {&c->e_tk_m, nb * TC * 4}, {&c->e_tk_d, nb * TC * 4},
      {&c->e_bcnt, (size_t)nb * 8 * 4}, {&c->e_lit, N}, {&c->e_tok, nb * TC}, {&c->e_ext, nb * EC},
      {&c->e_sym, nb * TC}, {&c->e_grp, nb * TC}, {&c->e_bits, (size_t)nb * zc::bits_cap((uint32_t)B)},
      {&c->e_lanes, (size_t)nb * zc::lanes_per_block((uint32_t)B)}, {&c->e_freq, (size_t)nb * 5 * 256 * 2},
      {&c->e_lanelen, (size_t)nb * 5 * 64 * 4}, {&c->e_sinfo, (size_t)nb * 5 * 4 * 4}, {&c->e_slab, N + 64}};
  return ensure(c, need);
}

int ensure_dec(zc_ctx* c, uint32_t nb, uint32_t block_log) {
  const size_t B = (size_t)1 << block_log, TC = zc::tok_cap((uint32_t)B), EC = zc::ext_cap((uint32_t)B);
  Need need[] = {
      {&c->d_lit, (size_t)nb * B}, {&c->d_tok, (size_t)nb * TC}, {&c->d_sym, (size_t)nb * TC},
      {&c->d_grp, (size_t)nb * TC}, {&c->d_ext, (size_t)nb * EC}, {&c->d_meta, (size_t)nb * sizeof(zc::DecMeta)},
      {&c->d_tks, (size_t)nb * TC * 4}, {&c->d_tkm, (size_t)nb * TC * 4}, {&c->d_tkd, (size_t)nb * TC * 4},
      {&c->d_tkl, (size_t)nb * TC * 4}};
  return ensure(c, need);
}

bool bad_block_log(uint32_t bl) { return bl < zc::kMinBlockLog || bl > zc::kMaxBlockLog; }

// blocks per encoder launch: 1 GiB of input (about 28 GiB of scratch: several waves of every stage on
// 148 SMs), and the grid's y limit
uint32_t enc_blocks_per_launch(uint32_t block_log) {
  return (uint32_t)std::min<size_t>(((size_t)1 << 30) >> block_log, 65535);
}
// blocks per decoder launch: 4 GiB of output (the fill runs one warp per block, so large launches keep
// every SM busy; about 6 bytes of scratch per output byte)
uint32_t dec_blocks_per_launch(uint32_t block_log) {
  return (uint32_t)std::min<size_t>(((size_t)4 << 30) >> block_log, 1u << 20);
}

// The test injector (src/safe_codec.h:17 has the reference's): with ZC_FAIL_AFTER=n in the environment
// when the context was opened, the (n+1)-th codec call on it fails with ZC_E_DEVICE before it launches
// anything, and so does every later call: a lost device stays lost.  Without it, nothing happens.
int gate(zc_ctx* c) {
  if (c->lost) return fail(c, ZC_E_DEVICE, "the GPU was lost earlier (device failure injected by ZC_FAIL_AFTER)");
  if (c->fail_after == 0) {
    c->lost = true;
    return fail(c, ZC_E_DEVICE, "device failure injected by ZC_FAIL_AFTER");
  }
  if (c->fail_after > 0) --c->fail_after;
  return ZC_OK;
}

int check_launch(zc_ctx* c, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, what);
  return ZC_OK;
}

// the encoder over nb device-resident blocks (offsets / lengths on the device)
int encode_device(zc_ctx* c, const uint8_t* d_in, const uint64_t* d_off, const uint32_t* d_len, uint32_t nb,
                  uint32_t block_log, int level, uint8_t* d_methods, uint32_t* d_lens, uint32_t* d_crcs,
                  uint8_t* d_out, size_t out_cap, uint64_t* d_out_offs, uint64_t* d_total, int emit_stored,
                  cudaStream_t st, const uint64_t* rec_base) {
  if (bad_block_log(block_log)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  if (rec_base && (!d_crcs || !emit_stored)) return fail(c, ZC_E_ARG, "archive records need the block CRCs");
  if (nb > enc_blocks_per_launch(block_log)) return fail(c, ZC_E_ARG, "too many blocks for one launch");
  if (int r = ensure_enc(c, nb, block_log)) return r;
  zc::EncArgs A{};
  A.in = d_in; A.in_off = d_off; A.in_len = d_len; A.nb = nb;
  A.B = 1u << block_log; A.block_log = block_log; A.depth = depth_for_level(level);
  const Shape& sh = c->shape[block_log - zc::kMinBlockLog][level_class(level)];
  A.cmp_cap = sh.cmp_cap;
  A.match_tile = sh.match_tile;
  A.match_dense = sh.match_dense;
  A.match_defer = sh.match_defer;
  A.tmp_pos = c->e_tmp_pos.as<uint32_t>(); A.srt_pos = c->e_srt_pos.as<uint32_t>();
  A.minfo = c->e_minfo.as<uint32_t>(); A.scnt = c->e_scnt.as<uint32_t>();
  A.tk_seg = c->e_tk_seg.as<uint32_t>();
  A.tmp_h = c->e_tmp_h.as<uint16_t>(); A.srt_h = c->e_srt_h.as<uint16_t>();
  A.tk_i = c->e_tk_i.as<uint32_t>(); A.tk_m = c->e_tk_m.as<uint32_t>(); A.tk_d = c->e_tk_d.as<uint32_t>();
  A.bcnt = c->e_bcnt.as<uint32_t>();
  A.s_lit = c->e_lit.as<uint8_t>(); A.s_tok = c->e_tok.as<uint8_t>(); A.s_ext = c->e_ext.as<uint8_t>();
  A.s_sym = c->e_sym.as<uint8_t>(); A.s_grp = c->e_grp.as<uint8_t>(); A.s_bits = c->e_bits.as<uint8_t>();
  A.lanes = c->e_lanes.as<uint8_t>(); A.freq = c->e_freq.as<uint16_t>(); A.lanelen = c->e_lanelen.as<uint32_t>();
  A.sinfo = c->e_sinfo.as<uint32_t>(); A.slab = c->e_slab.as<uint8_t>();
  A.out = d_out; A.out_cap = out_cap; A.out_off = d_out_offs; A.out_len = d_lens; A.out_method = d_methods;
  A.out_total = d_total; A.emit_stored = emit_stored;
  A.rec_hdr = rec_base ? 16u : 0u; A.rec_base = rec_base; A.rec_crc = d_crcs;
  zc::CrcArgs C{};
  C.base = d_in; C.offs = d_off; C.lens = d_len; C.nb = nb; C.crc = d_crcs; C.tables = c->d_crct;
  if (!d_crcs) C.nb = 0;
  zc::launch_encode(A, C, st, c->stages);
  return check_launch(c, "encoder launch");
}

int decode_device(zc_ctx* c, const uint8_t* d_comp, const uint64_t* d_comp_offs, const uint32_t* d_comp_lens,
                  const uint8_t* d_methods, const uint32_t* d_raw_lens, uint32_t nb, uint32_t block_log, uint8_t* d_out,
                  const uint64_t* d_out_offs, uint32_t* d_crcs, uint32_t* d_err, cudaStream_t st) {
  if (bad_block_log(block_log)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  if (int r = ensure_dec(c, std::max(nb, 1u), block_log)) return r;
  ZC_CUDA(cudaMemsetAsync(d_err, 0, (size_t)nb * 4, st));
  zc::DecArgs A{};
  A.comp = d_comp; A.comp_off = d_comp_offs; A.comp_len = d_comp_lens; A.method = d_methods; A.raw_len = d_raw_lens;
  A.nb = nb; A.B = 1u << block_log; A.out = d_out; A.out_off = d_out_offs; A.err = d_err;
  A.s_lit = c->d_lit.as<uint8_t>(); A.s_tok = c->d_tok.as<uint8_t>(); A.s_sym = c->d_sym.as<uint8_t>();
  A.s_grp = c->d_grp.as<uint8_t>(); A.s_ext = c->d_ext.as<uint8_t>(); A.meta = c->d_meta.as<zc::DecMeta>();
  A.tk_start = c->d_tks.as<uint32_t>(); A.tk_ms = c->d_tkm.as<uint32_t>(); A.tk_d = c->d_tkd.as<uint32_t>();
  A.tk_lik = c->d_tkl.as<uint32_t>();
  const Shape& sh = c->shape[block_log - zc::kMinBlockLog][level_class(c->level)];
  A.ring_log = sh.ring_log; A.fill_warps = sh.fill_warps; A.fill_words = sh.fill_words;
  A.work = c->work.as<uint32_t>() + 1;
  zc::launch_decode_fill(A, st, c->stages);
  if (d_crcs && nb) {
    zc::CrcArgs C{};
    C.base = d_out; C.offs = d_out_offs; C.lens = d_raw_lens; C.nb = nb; C.crc = d_crcs; C.err = d_err;
    C.tables = c->d_crct;
    zc::launch_crc(C, st, c->stages, "k_crc_out");
  }
  return check_launch(c, "decoder launch");
}

// blocks in chunk `i` of a host-pointer call: 128 MiB first (so the first kernels start early and the
// copies left exposed are short), then 512 MiB, so that a large call's copies overlap kernels
uint32_t host_chunk_blocks(uint32_t block_log, uint32_t per_launch, uint32_t i) {
  const size_t bytes = (size_t)(i == 0 ? 128 : 512) << 20;
  return std::max<uint32_t>(1, std::min<uint32_t>(per_launch, (uint32_t)(bytes >> block_log)));
}

void plain_blocks(zc_ctx* c, uint64_t n, uint32_t B, uint32_t nb, uint64_t* d_off, uint32_t* d_len, cudaStream_t st) {
  if (!nb) return;
  c->stages.begin("k_plain_blocks", st);
  k_plain_blocks<<<(nb + 255) / 256, 256, 0, st>>>(n, B, nb, d_off, d_len);
  c->stages.end(st);
}

}  // namespace zch

namespace {

// Runs `body` on stream st, through a CUDA graph when graphs are on: the first call with a given key
// captures the launches, later calls replay them.  Scratch must already be sized (a capture allocates
// nothing) and per-stage timing is off inside captures.
template <class F>
int with_graph(zc_ctx* c, int kind, const uint64_t* key, int nkey, cudaStream_t st, F body) {
  if (!c->graphs || st == nullptr) return body();
  for (GraphEntry& g : c->graph_cache) {
    if (g.kind != kind || memcmp(g.key, key, sizeof(uint64_t) * nkey) != 0) continue;
    ZC_CUDA(cudaGraphLaunch(g.exec, st));
    c->stages.launches += g.launches;
    return ZC_OK;
  }
  const bool timing = c->stages.timing;
  c->stages.timing = false;
  const uint64_t l0 = c->stages.launches;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) { c->stages.timing = timing; return cuda_fail(c, e, "cudaStreamBeginCapture"); }
  int r = body();
  e = cudaStreamEndCapture(st, &graph);
  c->stages.timing = timing;
  if (r) { if (graph) cudaGraphDestroy(graph); return r; }
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
  GraphEntry g{};
  g.kind = kind;
  memcpy(g.key, key, sizeof(uint64_t) * nkey);
  g.launches = c->stages.launches - l0;
  e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
  c->graph_cache.push_back(g);
  ZC_CUDA(cudaGraphLaunch(g.exec, st));
  return ZC_OK;
}

// Compression of host-resident blocks in chunks through the two stages: chunk i's upload (copy stream)
// overlaps chunk i-1's kernels, and chunk i-1's results come down while chunk i's kernels run.
int compress_host(zc_ctx* c, const uint8_t* host_base, const uint64_t* in_offs, const uint32_t* in_lens, uint32_t nb,
                  uint64_t plain_n, uint32_t block_log, int level, uint8_t* methods, uint32_t* comp_lens,
                  uint32_t* crcs, uint8_t* payloads, size_t payload_cap, uint64_t* pay_offs) {
  if (bad_block_log(block_log)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  const uint32_t B = 1u << block_log;
  const uint32_t per_launch = enc_blocks_per_launch(block_log);
  cudaStream_t st = c->stream, cs = c->cstream;
  uint64_t pay_at = 0;
  struct Chunk { uint32_t b0 = 0, k = 0; size_t meta_at = 0, meta_bytes = 0; };
  Chunk prev;
  bool have_prev = false;
  // the results of a finished chunk: counts first, then the payloads they size
  auto harvest = [&](zc_ctx::Stage& S, const Chunk& q) -> int {
    ZC_CUDA(cudaStreamWaitEvent(cs, S.ev_done, 0));
    uint8_t* hm = static_cast<uint8_t*>(S.h.p) + q.meta_at;
    ZC_CUDA(cudaMemcpyAsync(hm, S.meta.p, q.meta_bytes, cudaMemcpyDeviceToHost, cs));
    ZC_CUDA(cudaStreamSynchronize(cs));
    const uint64_t* h_poff = reinterpret_cast<const uint64_t*>(hm);
    const uint64_t total = h_poff[q.k];
    const uint32_t* h_plen = reinterpret_cast<const uint32_t*>(h_poff + q.k + 1);
    const uint32_t* h_crc = h_plen + q.k;
    const uint8_t* h_meth = reinterpret_cast<const uint8_t*>(h_crc + q.k);
    if (pay_at + total > payload_cap) return fail(c, ZC_E_ARG, "payload buffer too small");
    if (total) ZC_CUDA(cudaMemcpyAsync(payloads + pay_at, S.out.p, total, cudaMemcpyDeviceToHost, cs));
    for (uint32_t b = 0; b < q.k; ++b) {
      methods[q.b0 + b] = h_meth[b];
      comp_lens[q.b0 + b] = h_plen[b];
      if (crcs) crcs[q.b0 + b] = h_crc[b];
      if (pay_offs) pay_offs[q.b0 + b] = h_meth[b] ? pay_at + h_poff[b] : 0;
    }
    ZC_CUDA(cudaStreamSynchronize(cs));
    pay_at += total;
    return ZC_OK;
  };
  uint32_t it = 0;
  for (uint32_t b0 = 0; b0 < nb; b0 += prev.k, ++it) {
    zc_ctx::Stage& S = c->pipe[it & 1];
    Chunk q;
    q.b0 = b0;
    q.k = std::min(host_chunk_blocks(block_log, per_launch, it), nb - b0);
    const uint32_t k = q.k;
    // the bytes of blocks b0 .. b0+k-1 as one host span
    uint64_t lo, hi;
    if (in_offs) {
      lo = UINT64_MAX; hi = 0;
      for (uint32_t b = b0; b < b0 + k; ++b) {
        if (in_lens[b] > B) return fail(c, ZC_E_ARG, "a block is longer than the block size");
        lo = std::min(lo, in_offs[b]);
        hi = std::max(hi, in_offs[b] + in_lens[b]);
      }
      if (lo == UINT64_MAX) lo = hi = 0;
    } else {
      lo = (uint64_t)b0 * B;
      hi = std::min<uint64_t>(plain_n, (uint64_t)(b0 + k) * B);
    }
    const uint64_t span = hi - lo;
    q.meta_bytes = (size_t)k * (8 + 4 + 4 + 1) + 16;
    q.meta_at = ((size_t)k * 12 + 255) & ~(size_t)255;
    ZC_CUDA(grow(S.in, span + 64));
    ZC_CUDA(grow(S.blk, (size_t)k * 12));
    ZC_CUDA(grow(S.out, span + 64));
    ZC_CUDA(grow(S.meta, q.meta_bytes));
    ZC_CUDA(grow_host(S.h, q.meta_at + q.meta_bytes));
    uint8_t* d_in = S.in.as<uint8_t>();
    uint64_t* d_off = S.blk.as<uint64_t>();
    uint32_t* d_len = reinterpret_cast<uint32_t*>(d_off + k);
    // upload on the copy stream (the stage's last chunk was harvested, so its buffers are free)
    ZC_CUDA(cudaMemcpyAsync(d_in, host_base + lo, span, cudaMemcpyHostToDevice, cs));
    ZC_CUDA(cudaMemsetAsync(d_in + span, 0, 64, cs));
    if (in_offs) {
      uint64_t* ho = static_cast<uint64_t*>(S.h.p);
      uint32_t* hl = reinterpret_cast<uint32_t*>(ho + k);
      for (uint32_t b = 0; b < k; ++b) { ho[b] = in_offs[b0 + b] - lo; hl[b] = in_lens[b0 + b]; }
      ZC_CUDA(cudaMemcpyAsync(d_off, ho, (size_t)k * 12, cudaMemcpyHostToDevice, cs));
    }
    ZC_CUDA(cudaEventRecord(S.ev_in, cs));
    // kernels on the compute stream once the upload is in
    ZC_CUDA(cudaStreamWaitEvent(st, S.ev_in, 0));
    if (!in_offs) plain_blocks(c, span, B, k, d_off, d_len, st);
    uint8_t* m = S.meta.as<uint8_t>();
    uint64_t* d_poff = reinterpret_cast<uint64_t*>(m);
    uint64_t* d_total = d_poff + k;
    uint32_t* d_plen = reinterpret_cast<uint32_t*>(d_total + 1);
    uint32_t* d_crc = d_plen + k;
    uint8_t* d_meth = reinterpret_cast<uint8_t*>(d_crc + k);
    if (int r = encode_device(c, d_in, d_off, d_len, k, block_log, level, d_meth, d_plen, d_crc, S.out.as<uint8_t>(),
                              S.out.n, d_poff, d_total, 0, st))
      return r;
    ZC_CUDA(cudaEventRecord(S.ev_done, st));
    if (have_prev)
      if (int r = harvest(c->pipe[(it - 1) & 1], prev)) return r;
    prev = q;
    have_prev = true;
  }
  if (have_prev)
    if (int r = harvest(c->pipe[(it - 1) & 1], prev)) return r;
  return ZC_OK;
}

}  // namespace

extern "C" {

int zc_open(zc_ctx** out, int device) {
  if (!out) return ZC_E_ARG;
  *out = nullptr;
  zc_ctx* c = new zc_ctx;
  c->device = device;
  c->stages.impl = &c->records;
  if (const char* fa = getenv("ZC_FAIL_AFTER")) c->fail_after = atoll(fa);
  cudaError_t e = cudaSetDevice(device);
  cudaDeviceProp prop;
  if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, device);
  if (e == cudaSuccess && prop.major < 10) {
    c->err = "the sm_100a kernels need a Blackwell (compute 10.x) GPU";
    *out = c;
    return ZC_E_DEVICE;
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->cstream, cudaStreamNonBlocking);
  for (auto& S : c->pipe) {
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S.ev_in, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S.ev_done, cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = zc::prepare_kernels();
  if (e == cudaSuccess) e = grow(c->work, 256);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_crct, sizeof(zc::CrcTables));
  if (e == cudaSuccess) {
    zc::CrcTables T;
    build_crc_tables(T);
    e = cudaMemcpy(c->d_crct, &T, sizeof T, cudaMemcpyHostToDevice);
  }
  *out = c;
  if (e != cudaSuccess) return cuda_fail(c, e, "opening the GPU");
  char b[512];
  snprintf(b, sizeof b, "GPU %s (CUDA, %d SMs)", prop.name, prop.multiProcessorCount);
  c->name = b;
  return ZC_OK;
}

void zc_close(zc_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->cstream) cudaStreamSynchronize(c->cstream);
  drop_graphs(c);
  for (DevBuf* b : {&c->e_tmp_pos, &c->e_srt_pos, &c->e_minfo, &c->e_scnt, &c->e_tk_seg, &c->e_tmp_h, &c->e_srt_h, &c->e_tk_i,
                    &c->e_tk_m, &c->e_tk_d, &c->e_bcnt, &c->e_lit, &c->e_tok, &c->e_ext, &c->e_sym, &c->e_grp,
                    &c->e_bits, &c->e_lanes, &c->e_freq, &c->e_lanelen, &c->e_sinfo, &c->e_slab, &c->d_lit, &c->d_tok,
                    &c->d_sym, &c->d_grp, &c->d_ext, &c->d_meta, &c->d_tks, &c->d_tkm, &c->d_tkd, &c->d_tkl, &c->s_in, &c->s_blk, &c->s_out, &c->s_meta, &c->work,
                    &c->a_desc, &c->a_work})
    release(*b);
  if (c->h_meta.p) cudaFreeHost(c->h_meta.p);
  for (auto& S : c->pipe) {
    for (DevBuf* b : {&S.in, &S.blk, &S.out, &S.meta}) release(*b);
    if (S.h.p) cudaFreeHost(S.h.p);
    if (S.ev_in) cudaEventDestroy(S.ev_in);
    if (S.ev_done) cudaEventDestroy(S.ev_done);
  }
  if (c->d_crct) cudaFree(c->d_crct);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->cstream) cudaStreamDestroy(c->cstream);
  delete c;
}

const char* zc_last_error(const zc_ctx* c) { return c ? c->err.c_str() : "no context"; }
const char* zc_name(const zc_ctx* c) { return c ? c->name.c_str() : ""; }
uint64_t zc_launch_count(const zc_ctx* c) { return c ? c->stages.launches : 0; }

int zc_profile(zc_ctx* c, int on) {
  if (!c) return ZC_E_ARG;
  ZC_CUDA(cudaSetDevice(c->device));
  c->records.collect();
  c->records.totals.clear();
  c->records.order.clear();
  c->stages.timing = on != 0;
  return ZC_OK;
}

int zc_profile_stages(zc_ctx* c, uint32_t max, char* names, double* ms, uint64_t* counts, uint32_t* n_out) {
  if (!c || !n_out) return ZC_E_ARG;
  ZC_CUDA(cudaSetDevice(c->device));
  c->records.collect();
  const uint32_t n = (uint32_t)c->records.order.size();
  *n_out = n;
  for (uint32_t i = 0; i < n && i < max; ++i) {
    const std::string& k = c->records.order[i];
    const auto& v = c->records.totals[k];
    if (names) { strncpy(names + 32 * i, k.c_str(), 31); names[32 * i + 31] = 0; }
    if (ms) ms[i] = v.first;
    if (counts) counts[i] = v.second;
  }
  return ZC_OK;
}

int zc_prepare(zc_ctx* c, uint32_t block_log, int level) {
  if (!c) return ZC_E_ARG;
  ZC_GATE(c);
  if (bad_block_log(block_log)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  c->block_log = block_log;
  c->level = level;
  return ZC_OK;
}

int zc_reserve(zc_ctx* c, uint32_t block_log, uint32_t nb) {
  if (!c) return ZC_E_ARG;
  if (bad_block_log(block_log)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  if (nb > enc_blocks_per_launch(block_log) || nb > dec_blocks_per_launch(block_log))
    return fail(c, ZC_E_ARG, "too many blocks for one launch");
  ZC_CUDA(cudaSetDevice(c->device));
  if (int r = ensure_enc(c, std::max(nb, 1u), block_log)) return r;
  return ensure_dec(c, std::max(nb, 1u), block_log);
}

size_t zc_batch_bytes(const zc_ctx*, uint32_t block_log) { return (size_t)enc_blocks_per_launch(block_log) << block_log; }
size_t zc_batch_bytes_decode(const zc_ctx*, uint32_t block_log) {
  return (size_t)dec_blocks_per_launch(block_log) << block_log;
}

int zc_compress(zc_ctx* c, const uint8_t* in, size_t n, uint32_t block_log, int level, uint8_t* methods,
                uint32_t* comp_lens, uint32_t* crcs, uint8_t* payloads, size_t payload_cap, uint64_t* pay_offs) {
  if (!c) return ZC_E_ARG;
  ZC_GATE(c);
  if (bad_block_log(block_log)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  ZC_CUDA(cudaSetDevice(c->device));
  const uint64_t B = 1ull << block_log;
  const uint64_t nb = (n + B - 1) / B;
  if (nb > 0xFFFFFFFFull) return fail(c, ZC_E_ARG, "too many blocks");
  return compress_host(c, in, nullptr, nullptr, (uint32_t)nb, n, block_log, level, methods, comp_lens, crcs, payloads,
                       payload_cap, pay_offs);
}

int zc_compress_batch(zc_ctx* c, const uint8_t* in, const uint64_t* in_offs, const uint32_t* in_lens, uint32_t nb,
                      uint32_t block_log, int level, uint8_t* methods, uint32_t* comp_lens, uint32_t* crcs,
                      uint8_t* payloads, size_t payload_cap, uint64_t* pay_offs) {
  if (!c) return ZC_E_ARG;
  ZC_GATE(c);
  if (nb && (!in_offs || !in_lens)) return fail(c, ZC_E_ARG, "block offsets and lengths are required");
  ZC_CUDA(cudaSetDevice(c->device));
  return compress_host(c, in, in_offs, in_lens, nb, 0, block_log, level, methods, comp_lens, crcs, payloads,
                       payload_cap, pay_offs);
}

int zc_compress_device(zc_ctx* c, const uint8_t* d_in, const uint64_t* d_in_offs, const uint32_t* d_in_lens,
                       uint32_t nb, uint32_t block_log, int level, uint8_t* d_methods, uint32_t* d_comp_lens,
                       uint32_t* d_crcs, uint8_t* d_out, size_t out_cap, uint64_t* d_out_offs, uint64_t* d_total,
                       void* stream) {
  if (!c) return ZC_E_ARG;
  ZC_GATE(c);
  ZC_CUDA(cudaSetDevice(c->device));
  if (bad_block_log(block_log)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  if (nb > enc_blocks_per_launch(block_log)) return fail(c, ZC_E_ARG, "too many blocks for one launch");
  if (int r = ensure_enc(c, nb, block_log)) return r;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint64_t key[] = {(uint64_t)d_in, (uint64_t)d_in_offs, (uint64_t)d_in_lens, nb, block_log, (uint64_t)level,
                          (uint64_t)d_methods, (uint64_t)d_comp_lens, (uint64_t)d_crcs, (uint64_t)d_out, out_cap,
                          (uint64_t)d_out_offs, (uint64_t)d_total, (uint64_t)st};
  return with_graph(c, 0, key, (int)(sizeof key / sizeof key[0]), st, [&] {
    return encode_device(c, d_in, d_in_offs, d_in_lens, nb, block_log, level, d_methods, d_comp_lens, d_crcs, d_out,
                         out_cap, d_out_offs, d_total, 1, st);
  });
}

int zc_decompress_device(zc_ctx* c, const uint8_t* d_comp, const uint64_t* d_comp_offs, const uint32_t* d_comp_lens,
                         const uint8_t* d_methods, const uint32_t* d_raw_lens, uint32_t nb, uint32_t block_log,
                         uint8_t* d_out, const uint64_t* d_out_offs, uint32_t* d_crcs, uint32_t* d_err, void* stream) {
  if (!c) return ZC_E_ARG;
  ZC_GATE(c);
  ZC_CUDA(cudaSetDevice(c->device));
  if (nb > dec_blocks_per_launch(block_log)) return fail(c, ZC_E_ARG, "too many blocks for one launch");
  if (bad_block_log(block_log)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  if (int r = ensure_dec(c, std::max(nb, 1u), block_log)) return r;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint64_t key[] = {(uint64_t)d_comp, (uint64_t)d_comp_offs, (uint64_t)d_comp_lens, (uint64_t)d_methods,
                          (uint64_t)d_raw_lens, nb, block_log, (uint64_t)d_out, (uint64_t)d_out_offs, (uint64_t)d_crcs,
                          (uint64_t)d_err, (uint64_t)st};
  return with_graph(c, 1, key, (int)(sizeof key / sizeof key[0]), st, [&] {
    return decode_device(c, d_comp, d_comp_offs, d_comp_lens, d_methods, d_raw_lens, nb, block_log, d_out, d_out_offs,
                         d_crcs, d_err, st);
  });
}

int zc_set_graphs(zc_ctx* c, int on) {
  if (!c) return ZC_E_ARG;
  ZC_CUDA(cudaSetDevice(c->device));
  if (!on) drop_graphs(c);
  c->graphs = on != 0;
  return ZC_OK;
}

int zc_get_shape(const zc_ctx* c, uint32_t block_log, int level, zc_shape* out) {
  if (!c || !out || bad_block_log(block_log)) return ZC_E_ARG;
  const Shape& s = c->shape[block_log - zc::kMinBlockLog][level_class(level)];
  out->fill_ring_log = s.ring_log;
  out->fill_warps = s.fill_warps;
  out->match_cap = s.cmp_cap;
  out->match_tile = s.match_tile;
  out->fill_words = s.fill_words;
  out->match_dense = s.match_dense;
  out->match_defer = s.match_defer;
  return ZC_OK;
}

int zc_set_shape(zc_ctx* c, uint32_t block_log, int level, const zc_shape* in) {
  if (!c || !in) return ZC_E_ARG;
  if (bad_block_log(block_log)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  const uint32_t w = in->fill_warps;
  if (in->fill_ring_log < zc::kMinFillRingLog || in->fill_ring_log > zc::kMaxFillRingLog ||
      (w != 1 && w != 2 && w != 4 && w != 8) || in->match_cap < 8 ||
      (in->fill_words != 1 && in->fill_words != 2 && in->fill_words != 4) ||
      in->match_cap > 32 || zc::fill_smem_bytes(in->fill_ring_log, w, in->fill_words) > zc::kMaxFillSmem ||
      (in->match_tile != 256 && in->match_tile != 512 && in->match_tile != 1024) || in->match_dense > 1025 || in->match_defer > 4)
    return fail(c, ZC_E_ARG, "launch shape out of range");
  ZC_CUDA(cudaSetDevice(c->device));
  Shape& s = c->shape[block_log - zc::kMinBlockLog][level_class(level)];
  s.ring_log = in->fill_ring_log;
  s.fill_warps = w;
  s.cmp_cap = in->match_cap;
  s.match_tile = in->match_tile;
  s.fill_words = in->fill_words;
  s.match_dense = in->match_dense;
  s.match_defer = in->match_defer;
  drop_graphs(c);  // (captured launches carry the old shape)
  return ZC_OK;
}

// Times every candidate shape on the sample (whole blocks of it, up to one encoder launch) and keeps
// the fastest for (block_log, level): the match cap by the encoder's time, the fill's shape by the
// decoder's.  Each candidate runs once untimed and then `reps` times; its time is the smallest.
int zc_autotune(zc_ctx* c, const uint8_t* sample, size_t n, uint32_t block_log, int level, zc_shape* chosen) {
  if (!c || (!sample && n)) return ZC_E_ARG;
  ZC_GATE(c);
  if (bad_block_log(block_log)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  if (!n) return fail(c, ZC_E_ARG, "autotuning needs a sample");
  ZC_CUDA(cudaSetDevice(c->device));
  const uint64_t B = 1ull << block_log;
  uint32_t nb = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(n / B, 1), enc_blocks_per_launch(block_log));
  const uint64_t used = std::min<uint64_t>(n, (uint64_t)nb * B);
  nb = (uint32_t)((used + B - 1) / B);
  cudaStream_t st = c->stream;
  const size_t per_blk = 8 + 4 + 1 + 4 + 4 + 8 + 4 + 8;
  const size_t need = used + 64 + 2 * ((size_t)nb * B + 64) + (size_t)nb * per_blk + 16 * 256;  // (+ rounding)
  DevBuf tb;
  ZC_CUDA(grow(tb, need));
  uint8_t* p = tb.as<uint8_t>();
  auto take = [&](size_t bytes) { uint8_t* q = p; p += (bytes + 255) & ~(size_t)255; return q; };
  uint8_t* d_in = take(used + 64);
  uint8_t* d_comp = take((size_t)nb * B + 64);
  uint8_t* d_raw = take((size_t)nb * B + 64);
  uint64_t* d_ioff = reinterpret_cast<uint64_t*>(take((size_t)nb * 8));
  uint32_t* d_ilen = reinterpret_cast<uint32_t*>(take((size_t)nb * 4));
  uint8_t* d_meth = take(nb);
  uint32_t* d_clen = reinterpret_cast<uint32_t*>(take((size_t)nb * 4));
  uint32_t* d_crc = reinterpret_cast<uint32_t*>(take((size_t)nb * 4));
  uint64_t* d_coff = reinterpret_cast<uint64_t*>(take((size_t)nb * 8));
  uint32_t* d_err = reinterpret_cast<uint32_t*>(take((size_t)nb * 4));
  uint64_t* d_tot = reinterpret_cast<uint64_t*>(take(8));
  std::vector<uint64_t> ioff(nb);
  std::vector<uint32_t> ilen(nb);
  for (uint32_t b = 0; b < nb; ++b) {
    ioff[b] = (uint64_t)b * B;
    ilen[b] = (uint32_t)std::min<uint64_t>(B, used - ioff[b]);
  }
  int r = ZC_OK;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const bool timing = c->stages.timing;
  c->stages.timing = false;
  Shape& cur = c->shape[block_log - zc::kMinBlockLog][level_class(level)];
  const Shape saved = cur;
  const int saved_level = c->level;
  c->level = level;
  const int reps = 3;
  auto timed = [&](auto&& run, float& best_ms) -> int {
    best_ms = 1e30f;
    if (int q = run()) return q;
    for (int i = 0; i < reps; ++i) {
      cudaEventRecord(e0, st);
      if (int q = run()) return q;
      cudaEventRecord(e1, st);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) return cuda_fail(c, e, "autotune timing");
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      best_ms = std::min(best_ms, ms);
    }
    return ZC_OK;
  };
  auto encode = [&]() {
    return encode_device(c, d_in, d_ioff, d_ilen, nb, block_log, level, d_meth, d_clen, d_crc, d_comp, (size_t)nb * B,
                         d_coff, d_tot, 1, st);
  };
  auto decode = [&]() {
    return decode_device(c, d_comp, d_coff, d_clen, d_meth, d_ilen, nb, block_log, d_raw, d_ioff, nullptr, d_err, st);
  };
  do {
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_in, sample, used, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ioff, ioff.data(), (size_t)nb * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ilen, ilen.data(), (size_t)nb * 4, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) { r = cuda_fail(c, e, "autotune set-up"); break; }
    Shape best = saved;
    float best_ms = 1e30f;
    for (uint32_t cap : {12u, 16u, 24u, 32u})
      for (uint32_t tile : {256u, 512u, 1024u}) {
        if (r) break;
        cur = best;
        cur.cmp_cap = cap;
        cur.match_tile = tile;
        float ms;
        if ((r = timed(encode, ms))) break;
        if (ms < best_ms) { best_ms = ms; best.cmp_cap = cap; best.match_tile = tile; }
      }
    for (uint32_t dense : {128u, 256u, 512u, 1025u}) {  // (with the best cap and tile; 1025: never a lane each)
      if (r || dense == best.match_dense) continue;
      cur = best;
      cur.match_dense = dense;
      float ms;
      if ((r = timed(encode, ms))) break;
      if (ms < best_ms) { best_ms = ms; best.match_dense = dense; }
    }
    for (uint32_t back : {2u, 3u, 4u}) {  // (the match pass's savings against the parse's extra finishes)
      if (r || back == best.match_defer) continue;
      cur = best;
      cur.match_defer = back;
      float ms;
      if ((r = timed(encode, ms))) break;
      if (ms < best_ms) { best_ms = ms; best.match_defer = back; }
    }
    if (r) break;
    cur = best;
    if ((r = encode())) break;  // (every cap writes the same payloads)
    best_ms = 1e30f;
    for (uint32_t rl = 11; rl <= 14 && !r; ++rl)
      for (uint32_t w : {1u, 2u, 4u, 8u})
        for (uint32_t wd : {1u, 2u, 4u}) {
          if (r || zc::fill_smem_bytes(rl, w, wd) > zc::kMaxFillSmem) continue;
          Shape s = best;
          s.ring_log = rl; s.fill_warps = w; s.fill_words = wd;
          cur = s;
          float ms;
          if ((r = timed(decode, ms))) break;
          if (ms < best_ms) { best_ms = ms; best.ring_log = rl; best.fill_warps = w; best.fill_words = wd; }
        }
    if (r) break;
    cur = best;
  } while (false);
  if (r) cur = saved;
  c->level = saved_level;
  c->stages.timing = timing;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamSynchronize(st);
  release(tb);
  drop_graphs(c);
  if (!r && chosen) r = zc_get_shape(c, block_log, level, chosen);
  return r;
}

// Decompression of host-resident records in chunks through the two stages: chunk i's upload and
// kernels overlap the download of chunk i-1's raw bytes.
int zc_decompress(zc_ctx* c, const uint8_t* comp, const uint64_t* comp_offs, const uint32_t* comp_lens,
                  const uint8_t* methods, const uint32_t* raw_lens, uint32_t nb, uint8_t* out, uint32_t* crcs_out,
                  uint32_t* block_err) {
  if (!c) return ZC_E_ARG;
  ZC_GATE(c);
  ZC_CUDA(cudaSetDevice(c->device));
  uint32_t maxraw = 0;
  for (uint32_t b = 0; b < nb; ++b) maxraw = std::max(maxraw, raw_lens[b]);
  uint32_t bl = zc::kMinBlockLog;
  while (bl < zc::kMaxBlockLog && (1u << bl) < maxraw) ++bl;
  if (maxraw > (1u << zc::kMaxBlockLog)) return fail(c, ZC_E_DATA, "a block is longer than 1 MiB");
  const uint32_t per_launch = dec_blocks_per_launch(bl);
  cudaStream_t st = c->stream, cs = c->cstream;
  const size_t per_blk = 8 + 8 + 4 + 4 + 4 + 4 + 1;
  int status = ZC_OK;
  struct Chunk { uint32_t b0 = 0, k = 0; uint64_t out_at = 0, raw_total = 0; };
  Chunk prev;
  bool have_prev = false;
  // a finished chunk: its raw bytes and per-block CRCs / statuses come down on the copy stream
  auto harvest = [&](zc_ctx::Stage& S, const Chunk& q) -> int {
    uint8_t* hb = static_cast<uint8_t*>(S.h.p);
    uint32_t* h_crc = reinterpret_cast<uint32_t*>(hb + (size_t)q.k * 16 + (size_t)q.k * 8);
    uint32_t* h_err = h_crc + q.k;
    uint8_t* db = S.blk.as<uint8_t>();
    ZC_CUDA(cudaStreamWaitEvent(cs, S.ev_done, 0));
    if (q.raw_total) ZC_CUDA(cudaMemcpyAsync(out + q.out_at, S.out.p, q.raw_total, cudaMemcpyDeviceToHost, cs));
    ZC_CUDA(cudaMemcpyAsync(h_crc, db + (size_t)q.k * 24, (size_t)q.k * 8, cudaMemcpyDeviceToHost, cs));
    ZC_CUDA(cudaStreamSynchronize(cs));
    for (uint32_t b = 0; b < q.k; ++b) {
      if (crcs_out) crcs_out[q.b0 + b] = h_crc[b];
      if (block_err) block_err[q.b0 + b] = h_err[b];
      if (h_err[b] && status == ZC_OK) {
        status = ZC_E_DATA;
        char m[128];
        snprintf(m, sizeof m, "block %u damaged (GPU decoder, code %u)", q.b0 + b, h_err[b]);
        c->err = m;
      }
    }
    return ZC_OK;
  };
  uint64_t out_at = 0;
  uint32_t it = 0;
  for (uint32_t b0 = 0; b0 < nb; b0 += prev.k, ++it) {
    zc_ctx::Stage& S = c->pipe[it & 1];
    Chunk q;
    q.b0 = b0;
    q.k = std::min(host_chunk_blocks(bl, per_launch, it), nb - b0);
    q.out_at = out_at;
    const uint32_t k = q.k;
    uint64_t lo = UINT64_MAX, hi = 0, raw_total = 0, comp_sum = 0;
    for (uint32_t b = b0; b < b0 + k; ++b) {
      lo = std::min(lo, comp_offs[b]);
      hi = std::max(hi, comp_offs[b] + comp_lens[b]);
      raw_total += raw_lens[b];
      comp_sum += comp_lens[b];
    }
    if (lo == UINT64_MAX) lo = hi = 0;
    q.raw_total = raw_total;
    // one copy of the span when the blocks lie close together (an archive's records), else gathered
    const bool gather = hi - lo > comp_sum + comp_sum / 2 + 4096;
    const uint64_t span = gather ? comp_sum : hi - lo;
    ZC_CUDA(grow(S.in, span + 64));
    ZC_CUDA(grow(S.out, raw_total + 64));
    ZC_CUDA(grow(S.blk, (size_t)k * per_blk + 64));
    ZC_CUDA(grow_host(S.h, (size_t)k * per_blk + 64));
    // descriptors: comp offsets, out offsets (u64); comp lens, raw lens, crcs, errs (u32); methods (u8)
    uint8_t* hb = static_cast<uint8_t*>(S.h.p);
    uint64_t* h_coff = reinterpret_cast<uint64_t*>(hb);
    uint64_t* h_ooff = h_coff + k;
    uint32_t* h_clen = reinterpret_cast<uint32_t*>(h_ooff + k);
    uint32_t* h_rlen = h_clen + k;
    uint8_t* h_meth = reinterpret_cast<uint8_t*>(h_rlen + 3 * (size_t)k);
    uint64_t g = 0, o = 0;
    for (uint32_t b = 0; b < k; ++b) {
      const uint32_t j = b0 + b;
      h_coff[b] = gather ? g : comp_offs[j] - lo;
      g += comp_lens[j];
      h_ooff[b] = o;
      o += raw_lens[j];
      h_clen[b] = comp_lens[j];
      h_rlen[b] = raw_lens[j];
      h_meth[b] = methods[j];
    }
    uint8_t* d_in = S.in.as<uint8_t>();
    if (gather) {
      for (uint32_t b = 0; b < k; ++b)
        if (comp_lens[b0 + b])
          ZC_CUDA(cudaMemcpyAsync(d_in + h_coff[b], comp + comp_offs[b0 + b], comp_lens[b0 + b], cudaMemcpyHostToDevice, cs));
    } else if (span) {
      ZC_CUDA(cudaMemcpyAsync(d_in, comp + lo, span, cudaMemcpyHostToDevice, cs));
    }
    uint8_t* db = S.blk.as<uint8_t>();
    ZC_CUDA(cudaMemcpyAsync(db, hb, (size_t)k * per_blk, cudaMemcpyHostToDevice, cs));
    ZC_CUDA(cudaEventRecord(S.ev_in, cs));
    uint64_t* d_coff = reinterpret_cast<uint64_t*>(db);
    uint64_t* d_ooff = d_coff + k;
    uint32_t* d_clen = reinterpret_cast<uint32_t*>(d_ooff + k);
    uint32_t* d_rlen = d_clen + k;
    uint32_t* d_crc = d_rlen + k;
    uint32_t* d_err = d_crc + k;
    uint8_t* d_meth = reinterpret_cast<uint8_t*>(d_err + k);
    ZC_CUDA(cudaStreamWaitEvent(st, S.ev_in, 0));
    if (int r = decode_device(c, d_in, d_coff, d_clen, d_meth, d_rlen, k, bl, S.out.as<uint8_t>(), d_ooff, d_crc,
                              d_err, st))
      return r;
    ZC_CUDA(cudaEventRecord(S.ev_done, st));
    if (have_prev)
      if (int r = harvest(c->pipe[(it - 1) & 1], prev)) return r;
    prev = q;
    have_prev = true;
    out_at += raw_total;
  }
  if (have_prev)
    if (int r = harvest(c->pipe[(it - 1) & 1], prev)) return r;
  return status;
}

int zc_crc32(zc_ctx* c, const uint8_t* data, size_t n, uint32_t* crc) {
  if (!c || !crc) return ZC_E_ARG;
  ZC_GATE(c);
  ZC_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  const size_t piece = (size_t)1 << 20;
  const uint32_t nb = (uint32_t)((n + piece - 1) / piece);
  ZC_CUDA(grow(c->s_in, n + 64));
  ZC_CUDA(grow(c->s_blk, (size_t)nb * 16 + 64));
  ZC_CUDA(grow_host(c->h_meta, (size_t)nb * 16 + 64));
  if (n) ZC_CUDA(cudaMemcpyAsync(c->s_in.p, data, n, cudaMemcpyHostToDevice, st));
  uint64_t* d_off = c->s_blk.as<uint64_t>();
  uint32_t* d_len = reinterpret_cast<uint32_t*>(d_off + nb);
  uint32_t* d_crc = d_len + nb;
  c->stages.begin("k_plain_blocks", st);
  k_plain_blocks<<<(nb + 255) / 256 + 1, 256, 0, st>>>(n, (uint32_t)piece, nb, d_off, d_len);
  c->stages.end(st);
  zc::CrcArgs C{};
  C.base = c->s_in.as<uint8_t>(); C.offs = d_off; C.lens = d_len; C.nb = nb; C.crc = d_crc; C.tables = c->d_crct;
  zc::launch_crc(C, st, c->stages, "k_crc_in");
  if (int r = check_launch(c, "crc launch")) return r;
  uint32_t* h = static_cast<uint32_t*>(c->h_meta.p);
  ZC_CUDA(cudaMemcpyAsync(h, d_crc, (size_t)nb * 4, cudaMemcpyDeviceToHost, st));
  ZC_CUDA(cudaStreamSynchronize(st));
  uint32_t r = 0;
  for (uint32_t b = 0; b < nb; ++b) r = zc_crc32_combine(r, h[b], std::min<uint64_t>(piece, n - (uint64_t)b * piece));
  *crc = r;
  return ZC_OK;
}

uint32_t zc_crc32_combine(uint32_t a, uint32_t b, uint64_t len_b) {
  if (!len_b) return a;
  uint32_t x = 0x80000000u, base = 0x00800000u;  // x^0, x^8
  for (uint64_t n = len_b; n; n >>= 1) {
    if (n & 1u) x = zc::gf2_mul(x, base);
    base = zc::gf2_mul(base, base);
  }
  return zc::gf2_mul(x, a) ^ b;
}

}  // extern "C"
