// zc_noalloc.cu -- zc_decompress_noalloc: the block decoder with no device allocation at all.
//
// Some callers cannot call cudaMalloc: a plugin inside a host process that hands out every byte of
// device memory itself (an admission-controlled server, a framework that owns its allocator), or a
// latency-bound path where cudaMalloc / cudaFree would synchronise the device and stall other streams.
// This entry point takes the caller's inputs and outputs and keeps its scratch (the decoded symbol
// streams, each block's framing and each token's table row) in one file-scope __device__ array of
// ZC_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library holds until the process exits.  It
// runs the same kernels as zc_decompress_device (framing, rANS streams, token scan, the queue-fed fill,
// the CRC), and opens no context: the CRC tables are a constant-initialised __device__ array, set up by
// the module load itself.
#include <mutex>

#include "../../include/zero_cuda.h"
#include "zc_internal.cuh"
#include "zc_kernels.h"

namespace {

// the CRC tables computed at compile time: the slice-by-8 tables (t[k][b] = the register after byte b and
// k zero bytes) and the powers x^(8 * 2^e) that the block CRC's combining tree shifts by
constexpr uint32_t cx_mul(uint32_t a, uint32_t b) {
  uint32_t acc = 0;
  for (int i = 0; i < 32; ++i) {
    acc ^= b & (0u - (a >> 31));
    a <<= 1;
    b = (b >> 1) ^ (0xEDB88320u & (0u - (b & 1u)));
  }
  return acc;
}
constexpr zc::CrcTables cx_tables() {
  zc::CrcTables T{};
  for (uint32_t i = 0; i < 256; ++i) {
    uint32_t r = i;
    for (int k = 0; k < 8; ++k) r = (r >> 1) ^ (0xEDB88320u & (0u - (r & 1u)));
    T.t[0][i] = r;
  }
  for (int k = 1; k < 8; ++k)
    for (uint32_t i = 0; i < 256; ++i) T.t[k][i] = (T.t[k - 1][i] >> 8) ^ T.t[0][T.t[k - 1][i] & 0xFFu];
  uint32_t p = 0x00800000u;  // x^8
  for (int e = 0; e < 64; ++e) { T.pow2[e] = p; p = cx_mul(p, p); }
  return T;
}

static __device__ __align__(256) uint8_t g_scratch[ZC_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) const zc::CrcTables g_tables = cx_tables();

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

// The scratch a call of nb blocks of B bytes takes: the fill's work counter, then per kind of buffer one
// region of nb slots: literals (B), tok / sym / group streams (tok_cap each), ext bytes (ext_cap), the
// framing records, and the four token tables (tok_cap words each).
size_t scratch_need(uint32_t nb, uint32_t B) {
  const size_t TC = zc::tok_cap(B), EC = zc::ext_cap(B);
  return 256 + up256((size_t)nb * B) + 3 * up256((size_t)nb * TC) + up256((size_t)nb * EC) +
         up256((size_t)nb * sizeof(zc::DecMeta)) + 4 * up256((size_t)nb * TC * 4);
}

// Per device: the device addresses of the two arrays, looked up with that device current.  Host code must
// not pass the arrays' names to a kernel (in host code they name host-side stand-ins); it passes these.
// The lookup is redone when the device's context changes (after a cudaDeviceReset the module, and with it
// the arrays, is loaded anew and may sit elsewhere).
struct Setup {
  void* ctx = nullptr;
  uint8_t* scratch = nullptr;
  const zc::CrcTables* tables = nullptr;
};
constexpr int kMaxDevices = 128;
Setup g_setup[kMaxDevices];
std::mutex g_mu;

void* current_context() {  // the driver's current context, through the runtime (no link to libcuda)
  using Fn = int (*)(void**);
  static Fn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    return cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess
               ? reinterpret_cast<Fn>(p)
               : nullptr;
  }();
  void* ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

int setup(int dev, Setup& out) {
  if (dev < 0 || dev >= kMaxDevices) return ZC_E_DEVICE;
  void* ctx = current_context();  // (null before the runtime has made the device's context current)
  std::lock_guard<std::mutex> lk(g_mu);
  Setup& s = g_setup[dev];
  if (!s.scratch || !ctx || ctx != s.ctx) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess) return ZC_E_DEVICE;
    s.scratch = static_cast<uint8_t*>(p);
    if (cudaGetSymbolAddress(&p, g_tables) != cudaSuccess) return ZC_E_DEVICE;
    s.tables = static_cast<const zc::CrcTables*>(p);
    s.ctx = current_context();
  }
  out = s;
  return ZC_OK;
}

}  // namespace

extern "C" int zc_decompress_noalloc(const uint8_t* d_comp, const uint64_t* d_comp_offs, const uint32_t* d_comp_lens,
                                     const uint8_t* d_methods, const uint32_t* d_raw_lens, uint32_t nb,
                                     uint32_t block_log, uint8_t* d_out, const uint64_t* d_out_offs, uint32_t* d_crcs,
                                     uint32_t* d_err, void* stream) {
  if (block_log < zc::kMinBlockLog || block_log > zc::kMaxBlockLog) return ZC_E_ARG;
  const uint32_t B = 1u << block_log;
  if (scratch_need(nb, B) > ZC_NOALLOC_SCRATCH_BYTES) return ZC_E_ARG;  // beyond the fixed scratch
  if (!nb) return ZC_OK;
  if (!d_comp || !d_comp_offs || !d_comp_lens || !d_methods || !d_raw_lens || !d_out || !d_out_offs || !d_err)
    return ZC_E_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ZC_E_DEVICE;
  Setup s;
  if (int r = setup(dev, s)) return r;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the status words and the fill's work counter must start at zero; everything else in the scratch is
  // written before it is read
  if (cudaMemsetAsync(d_err, 0, (size_t)nb * 4, st) != cudaSuccess) return ZC_E_DEVICE;
  const size_t TC = zc::tok_cap(B), EC = zc::ext_cap(B);
  uint8_t* at = s.scratch;
  zc::DecArgs A{};
  A.comp = d_comp; A.comp_off = d_comp_offs; A.comp_len = d_comp_lens; A.method = d_methods; A.raw_len = d_raw_lens;
  A.nb = nb; A.B = B; A.out = d_out; A.out_off = d_out_offs; A.err = d_err;
  A.work = reinterpret_cast<uint32_t*>(at); at += 256;
  A.s_lit = at; at += up256((size_t)nb * B);
  A.s_tok = at; at += up256((size_t)nb * TC);
  A.s_sym = at; at += up256((size_t)nb * TC);
  A.s_grp = at; at += up256((size_t)nb * TC);
  A.s_ext = at; at += up256((size_t)nb * EC);
  A.meta = reinterpret_cast<zc::DecMeta*>(at); at += up256((size_t)nb * sizeof(zc::DecMeta));
  A.tk_start = reinterpret_cast<uint32_t*>(at); at += up256((size_t)nb * TC * 4);
  A.tk_ms = reinterpret_cast<uint32_t*>(at); at += up256((size_t)nb * TC * 4);
  A.tk_d = reinterpret_cast<uint32_t*>(at); at += up256((size_t)nb * TC * 4);
  A.tk_lik = reinterpret_cast<uint32_t*>(at);
  // the fill's launch shape: the default of the context-based calls (a ring of 4 KiB per warp, 4 warps a
  // CTA, a word a lane a round)
  A.ring_log = 12;
  A.fill_warps = 4;
  A.fill_words = 1;
  zc::Stages stages;  // (no timing; nothing to record)
  zc::launch_decode_fill(A, st, stages);
  if (d_crcs) {
    zc::CrcArgs C{};
    C.base = d_out; C.offs = d_out_offs; C.lens = d_raw_lens; C.nb = nb; C.crc = d_crcs; C.err = d_err;
    C.tables = s.tables;
    zc::launch_crc(C, st, stages, "k_crc_out");
  }
  return cudaGetLastError() == cudaSuccess ? ZC_OK : ZC_E_DEVICE;
}
