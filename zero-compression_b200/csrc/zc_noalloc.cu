// zc_noalloc.cu -- zc_decompress_noalloc: the block decoder with no device allocation at all.
//
// Some callers cannot call cudaMalloc: a plugin inside a host process that hands out every byte of
// device memory itself (an admission-controlled server, a framework that owns its allocator), or a
// latency-bound path where cudaMalloc / cudaFree would synchronise the device and stall other streams.
// This entry point takes the caller's inputs and outputs and keeps its scratch (the decoded symbol
// streams and per-block counts) in one file-scope __device__ array of ZC_NOALLOC_SCRATCH_BYTES, which
// every GPU that loads the library holds until the process exits.  It opens no context: the CRC
// tables live in a second __device__ array.
#include <mutex>

#include "../../include/zero_cuda.h"
#include "zc_internal.cuh"
#include "zc_kernels.h"

namespace {

static __device__ __align__(256) uint8_t g_scratch[ZC_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) zc::CrcTables g_tables;

// per device: the device addresses of the two arrays, found once with that device current
struct Setup {
  bool ready = false;
  uint8_t* scratch = nullptr;
  zc::CrcTables* tables = nullptr;
};
constexpr int kMaxDevices = 128;
Setup g_setup[kMaxDevices];
std::mutex g_mu;

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

// the scratch one block of 2^block_log bytes needs: literals, tok / sym / groups, ext, counts
size_t scratch_per_block(uint32_t B) {
  return up256(B) + 3 * up256(zc::tok_cap(B)) + up256(zc::ext_cap(B)) + up256(sizeof(zc::DecMeta));
}

void build_tables(zc::CrcTables& T) {
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

// once per device, with that device current: host code names the arrays only through these addresses
int setup(int dev, Setup*& out) {
  if (dev < 0 || dev >= kMaxDevices) return ZC_E_DEVICE;
  std::lock_guard<std::mutex> lk(g_mu);
  Setup& s = g_setup[dev];
  if (!s.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess) return ZC_E_DEVICE;
    s.scratch = static_cast<uint8_t*>(p);
    if (cudaGetSymbolAddress(&p, g_tables) != cudaSuccess) return ZC_E_DEVICE;
    s.tables = static_cast<zc::CrcTables*>(p);
    zc::CrcTables T;
    build_tables(T);
    if (cudaMemcpyToSymbol(g_tables, &T, sizeof T) != cudaSuccess) return ZC_E_DEVICE;
    s.ready = true;
  }
  out = &s;
  return ZC_OK;
}

}  // namespace

extern "C" int zc_decompress_noalloc(const uint8_t* d_comp, const uint64_t* d_comp_offs, const uint32_t* d_comp_lens,
                                     const uint8_t* d_methods, const uint32_t* d_raw_lens, uint32_t nb,
                                     uint32_t block_log, uint8_t* d_out, const uint64_t* d_out_offs, uint32_t* d_crcs,
                                     uint32_t* d_err, void* stream) {
  if (block_log < zc::kMinBlockLog || block_log > zc::kMaxBlockLog) return ZC_E_ARG;
  const uint32_t B = 1u << block_log;
  const size_t per = scratch_per_block(B);
  if ((uint64_t)nb * per > ZC_NOALLOC_SCRATCH_BYTES) return ZC_E_ARG;  // beyond the fixed scratch
  if (!nb) return ZC_OK;
  if (!d_comp || !d_comp_offs || !d_comp_lens || !d_methods || !d_raw_lens || !d_out || !d_out_offs || !d_err)
    return ZC_E_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ZC_E_DEVICE;
  Setup* s = nullptr;
  if (int r = setup(dev, s)) return r;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the status words must start at zero; the scratch streams are written before they are read
  if (cudaMemsetAsync(d_err, 0, (size_t)nb * 4, st) != cudaSuccess) return ZC_E_DEVICE;
  uint8_t* at = s->scratch;
  zc::DecArgs A{};
  A.comp = d_comp; A.comp_off = d_comp_offs; A.comp_len = d_comp_lens; A.method = d_methods; A.raw_len = d_raw_lens;
  A.nb = nb; A.B = B; A.out = d_out; A.out_off = d_out_offs; A.err = d_err;
  A.s_lit = at; at += up256((size_t)nb * B);
  A.s_tok = at; at += up256((size_t)nb * zc::tok_cap(B));
  A.s_sym = at; at += up256((size_t)nb * zc::tok_cap(B));
  A.s_grp = at; at += up256((size_t)nb * zc::tok_cap(B));
  A.s_ext = at; at += up256((size_t)nb * zc::ext_cap(B));
  A.meta = reinterpret_cast<zc::DecMeta*>(at);
  zc::Stages stages;  // (no timing; nothing to record)
  zc::launch_decode(A, st, stages);
  if (d_crcs) {
    zc::CrcArgs C{};
    C.base = d_out; C.offs = d_out_offs; C.lens = d_raw_lens; C.nb = nb; C.crc = d_crcs; C.err = d_err;
    C.tables = s->tables;
    zc::launch_crc(C, st, stages, "k_crc_out");
  }
  return cudaGetLastError() == cudaSuccess ? ZC_OK : ZC_E_DEVICE;
}
