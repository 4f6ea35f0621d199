// zero_cuda_codec.hpp -- zero::CudaCodec, the B200 codec behind the reference's codec interface.
//
// Header-only C++ over the C ABI of zero_cuda.h.  Include it after the reference's archive.h
// (src/archive.h:45-69 declares zero::Codec, BlockOut and BlockIn; src/codec.h declares zb::Error).
// It takes the place of zero::GpuCodec (src/gpu_codec.h:11-318):
//
//   choose_codec (src/main.cpp:36-57):   auto g = std::make_unique<zero::CudaCodec>(level);
//   SafeCodec (src/safe_codec.h:10-50):  unchanged; it catches zb::Error (damaged data: the CPU redoes the
//                                        batch and reports) and gpu::Error (device failure: CPU for good).
//
// The reference declares gpu::Error in src/gpu.h:17-19, which the CUDA build no longer includes; define
// ZERO_CUDA_DEFINE_GPU_ERROR before including this header to have it declared here.
#pragma once
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "zero_cuda.h"

#ifdef ZERO_CUDA_DEFINE_GPU_ERROR
namespace gpu {
struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};
}  // namespace gpu
#endif

namespace zero {

struct CudaCodec : Codec {
  int level = 5;  // 1 fast .. 9 thorough: the CPU codec's chain depth 8 / 32 / 256 (src/main.cpp:45)

  explicit CudaCodec(int lvl = 5, int device = 0) : level(lvl) {
    if (int rc = zc_open(&ctx_, device)) {
      const std::string m = ctx_ ? zc_last_error(ctx_) : "cannot open the GPU";
      zc_close(ctx_);
      ctx_ = nullptr;
      (void)rc;
      throw gpu::Error(m);
    }
  }
  ~CudaCodec() override { zc_close(ctx_); }
  CudaCodec(const CudaCodec&) = delete;
  CudaCodec& operator=(const CudaCodec&) = delete;

  std::string name() const override { return zc_name(ctx_); }
  size_t batch_bytes(uint32_t block_log) const override { return zc_batch_bytes(ctx_, block_log); }
  size_t batch_bytes_decode(uint32_t block_log) const override { return zc_batch_bytes_decode(ctx_, block_log); }
  void prepare(uint32_t block_log) override { check(zc_prepare(ctx_, block_log, level)); }

  // src/archive.h:60: n bytes in whole blocks (the last may be short) -> one BlockOut per block
  void compress(const uint8_t* in, size_t n, uint32_t block_log, std::vector<BlockOut>& out) override {
    const size_t B = (size_t)1 << block_log, nb = (n + B - 1) / B;
    out.assign(nb, BlockOut{});
    if (!nb) return;
    methods_.resize(nb);
    lens_.resize(nb);
    offs_.resize(nb);
    pay_.resize(n);
    check(zc_compress(ctx_, in, n, block_log, level, methods_.data(), lens_.data(), nullptr, pay_.data(), pay_.size(),
                      offs_.data()));
    for (size_t b = 0; b < nb; ++b) {
      out[b].method = methods_[b];
      if (methods_[b]) out[b].data.assign(pay_.data() + offs_[b], pay_.data() + offs_[b] + lens_[b]);
    }
  }

  // src/archive.h:61-63: the blocks' raw bytes back to back, valid through the next call and until the
  // one after (two output buffers taken in turn, as the reference's writer thread needs)
  const uint8_t* decompress(const std::vector<BlockIn>& blocks) override {
    const size_t nb = blocks.size();
    if (!nb) return nullptr;
    coffs_.resize(nb);
    clens_.resize(nb);
    raws_.resize(nb);
    methods_.resize(nb);
    // the payloads as offsets from the first one (they come from one archive read, one after the other)
    const uint8_t* base = blocks[0].data;
    for (const BlockIn& k : blocks) if (k.data && k.data < base) base = k.data;
    size_t total = 0;
    for (size_t b = 0; b < nb; ++b) {
      coffs_[b] = (uint64_t)(blocks[b].data - base);
      clens_[b] = blocks[b].comp_len;
      raws_[b] = blocks[b].raw_len;
      methods_[b] = blocks[b].method;
      total += blocks[b].raw_len;
    }
    out_at_ ^= 1;
    std::vector<uint8_t>& o = out_[out_at_];
    if (o.size() < total) o.resize(total);
    check(zc_decompress(ctx_, base, coffs_.data(), clens_.data(), methods_.data(), raws_.data(), (uint32_t)nb, o.data(),
                        nullptr, nullptr));
    return o.data();
  }

 private:
  void check(int rc) {
    if (rc == ZC_OK) return;
    if (rc == ZC_E_DATA || rc == ZC_E_ARG) throw zb::Error(zc_last_error(ctx_));
    throw gpu::Error(zc_last_error(ctx_));
  }
  zc_ctx* ctx_ = nullptr;
  std::vector<uint8_t> methods_, pay_;
  std::vector<uint32_t> lens_, clens_, raws_;
  std::vector<uint64_t> offs_, coffs_;
  std::vector<uint8_t> out_[2];
  int out_at_ = 0;
};

}  // namespace zero
