// zc_host.h -- the device context behind the C ABI (zc_ctx) and the host-side drivers shared by the
// ABI's source files (zc_api.cu: the codec calls; zc_archive.cu: whole .zero archives).  Internal: not
// part of include/zero_cuda.h.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/zero_cuda.h"
#include "zc_kernels.h"

namespace zch {

struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  template <class T> T* as() const { return static_cast<T*>(p); }
};

struct HostBuf {  // pinned staging
  void* p = nullptr;
  size_t n = 0;
};

// per-stage CUDA-event records of one context
struct StageRecords {
  struct Rec { const char* name; cudaEvent_t a, b; };
  std::vector<cudaEvent_t> pool;
  std::vector<Rec> pending;
  const char* open_name = nullptr;
  cudaEvent_t open_ev = nullptr;
  std::map<std::string, std::pair<double, uint64_t>> totals;
  std::vector<std::string> order;
  cudaEvent_t get() {
    if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  void collect() {
    for (const Rec& r : pending) {
      float ms = 0;
      cudaEventSynchronize(r.b);
      cudaEventElapsedTime(&ms, r.a, r.b);
      auto it = totals.find(r.name);
      if (it == totals.end()) { order.push_back(r.name); it = totals.emplace(r.name, std::make_pair(0.0, (uint64_t)0)).first; }
      it->second.first += ms;
      it->second.second += 1;
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    pending.clear();
  }
  ~StageRecords() {
    for (const Rec& r : pending) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
};

// a captured launch sequence, replayed when a device entry point is called again with the same arguments
struct GraphEntry {
  int kind;
  uint64_t key[24];
  cudaGraphExec_t exec;
  uint64_t launches;  // kernels in the graph
};

// per (block size, level class) launch shapes: the fill's ring, warps per CTA and words a lane a round,
// the match pass's compare cap and tile (none of them changes a result byte)
struct Shape {
  uint32_t ring_log = 12, fill_warps = 4, cmp_cap = 16, match_tile = 1024, fill_words = 1, match_dense = 256,
           match_defer = 3;
};

}  // namespace zch

struct zc_ctx {
  int device = 0;
  zch::Shape shape[5][3];
  bool graphs = false;
  std::vector<zch::GraphEntry> graph_cache;
  cudaStream_t stream = nullptr;
  std::string err, name;
  uint32_t block_log = 18;
  int level = 5;
  zc::Stages stages;
  zch::StageRecords records;
  zc::CrcTables* d_crct = nullptr;
  // encoder scratch (sized by capacity: any block size whose blocks fit)
  zch::DevBuf e_tmp_pos, e_srt_pos, e_minfo, e_scnt, e_tk_seg, e_tmp_h, e_srt_h, e_tk_i, e_tk_m, e_tk_d, e_bcnt, e_lit, e_tok,
      e_ext, e_sym, e_grp, e_bits, e_lanes, e_freq, e_lanelen, e_sinfo, e_slab;
  // decoder scratch (likewise)
  zch::DevBuf d_lit, d_tok, d_sym, d_grp, d_ext, d_meta, d_tks, d_tkm, d_tkd, d_tkl;
  // staging for the host-pointer calls
  zch::DevBuf s_in, s_blk, s_out, s_meta;
  zch::HostBuf h_meta;
  zch::DevBuf work;  // the decoder fill's device work counter
  // whole-archive calls: descriptors (entry table, file pieces) and per-block results (the host-pointer
  // forms stream their data through the two stages below)
  zch::DevBuf a_desc, a_work;
  // the host-pointer codec calls run in chunks through two stages: a chunk's copies (on cstream) overlap
  // the other chunk's kernels (on stream)
  struct Stage {
    zch::DevBuf in, blk, out, meta;
    zch::HostBuf h;  // descriptors up, then results down
    cudaEvent_t ev_in = nullptr, ev_done = nullptr;
  } pipe[2];
  cudaStream_t cstream = nullptr;
  // the test injector of device failures: ZC_FAIL_AFTER=n at open fails the (n+1)-th codec call
  int64_t fail_after = -1;
  bool lost = false;
};

namespace zch {

int fail(zc_ctx* c, int code, const std::string& msg);
int cuda_fail(zc_ctx* c, cudaError_t e, const char* what);
cudaError_t grow(DevBuf& b, size_t bytes);
cudaError_t grow_host(HostBuf& b, size_t bytes);  // pinned
// blocks in chunk `i` of a host-pointer call: 128 MiB first, then 512 MiB (at most per_launch)
uint32_t host_chunk_blocks(uint32_t block_log, uint32_t per_launch, uint32_t i);
bool bad_block_log(uint32_t bl);
uint32_t enc_blocks_per_launch(uint32_t block_log);
uint32_t dec_blocks_per_launch(uint32_t block_log);
int check_launch(zc_ctx* c, const char* what);
// ZC_E_DEVICE when the injector fails this call (or failed an earlier one); counts the call otherwise
int gate(zc_ctx* c);
// the slice-by-8 tables and x^(8 * 2^e) powers of the CRC-32 (host copy; the context uploads one)
void build_crc_tables(zc::CrcTables& T);
// uniform blocks: block b of an n-byte span starts at b * B and holds min(B, n - b * B) bytes
void plain_blocks(zc_ctx* c, uint64_t n, uint32_t B, uint32_t nb, uint64_t* d_off, uint32_t* d_len, cudaStream_t st);
// the encoder over nb device-resident blocks.  With rec_base (a device u64) the bodies are written as
// archive block records: each preceded by its 16-byte header, the first at *rec_base, and *d_total gets
// the end of the last record; without it the bodies are packed from 0 and *d_total gets their size.
int encode_device(zc_ctx* c, const uint8_t* d_in, const uint64_t* d_off, const uint32_t* d_len, uint32_t nb,
                  uint32_t block_log, int level, uint8_t* d_methods, uint32_t* d_lens, uint32_t* d_crcs,
                  uint8_t* d_out, size_t out_cap, uint64_t* d_out_offs, uint64_t* d_total, int emit_stored,
                  cudaStream_t st, const uint64_t* rec_base = nullptr);
// the decoder over nb device-resident blocks; d_crcs (may be NULL) gets each output's CRC-32
int decode_device(zc_ctx* c, const uint8_t* d_comp, const uint64_t* d_comp_offs, const uint32_t* d_comp_lens,
                  const uint8_t* d_methods, const uint32_t* d_raw_lens, uint32_t nb, uint32_t block_log, uint8_t* d_out,
                  const uint64_t* d_out_offs, uint32_t* d_crcs, uint32_t* d_err, cudaStream_t st);

}  // namespace zch

#define ZC_GATE(c)                           \
  do {                                       \
    if (int g_ = zch::gate(c)) return g_;    \
  } while (0)

#define ZC_CUDA(call)                                  \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return zch::cuda_fail(c, e_, #call); \
  } while (0)
