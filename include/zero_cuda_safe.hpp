// zero_cuda_safe.hpp -- zero::SafeCudaCodec: the B200 codec with the reference's CPU codec behind it.
//
// The reference wraps its GPU codec in SafeCodec (src/safe_codec.h:10-50), typed on its Level Zero
// GpuCodec; this is the same contract over zero::CudaCodec, for choose_codec (src/main.cpp:36-57):
//
//   auto s = std::make_unique<zero::SafeCudaCodec>(level);   // never throws: no GPU means the CPU from the start
//   s->set_report(&rep);
//
//   * damaged data or an impossible result (ZC_E_DATA, ZC_E_ARG -> zb::Error): this batch is done again
//     by the CPU codec, which reports what is wrong (or does better); the GPU keeps the next batches;
//   * a device failure (ZC_E_DEVICE, ZC_E_NOMEM -> gpu::Error): the CPU codec does this batch and every
//     later one -- a lost device stays lost for the process -- and the report says so once.
// Both codecs write the same bytes at a level, so an archive written across a failure is the same file.
//
// For tests, the C ABI fails a context's (n+1)-th codec call with ZC_E_DEVICE, before it launches anything,
// when the environment holds ZC_FAIL_AFTER=n at zc_open (the reference's ZERO_FAIL_GPU, src/safe_codec.h:17).
//
// Include after the reference's archive.h (it declares zero::Codec and zero::CpuCodec) and
// zero_cuda_codec.hpp.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "zero_cuda_codec.hpp"

namespace zero {

struct SafeCudaCodec : Codec {
  std::unique_ptr<CudaCodec> gpu;
  CpuCodec cpu;
  bool gpu_ok = false;
  size_t batch_cap = 0;  // when nonzero: batches of at most this many bytes (both directions)

  explicit SafeCudaCodec(int level = 5, int device = 0, Report* r = nullptr) : rep_(r) {
    cpu.depth = level <= 1 ? 8 : level >= 9 ? 256 : 32;
    try {
      gpu = std::make_unique<CudaCodec>(level, device);
      gpu_ok = true;
    } catch (const std::exception& e) {
      say(std::string("GPU unavailable (") + e.what() + "); using the CPU");
    }
  }
  void set_report(Report* r) { rep_ = r; }

  std::string name() const override { return gpu_ok ? gpu->name() : cpu.name(); }
  size_t batch_bytes(uint32_t bl) const override {
    return capped(gpu_ok ? gpu->batch_bytes(bl) : cpu.batch_bytes(bl), bl);
  }
  size_t batch_bytes_decode(uint32_t bl) const override {
    return capped(gpu_ok ? gpu->batch_bytes_decode(bl) : cpu.batch_bytes_decode(bl), bl);
  }
  void prepare(uint32_t bl) override { attempt([&] { gpu->prepare(bl); }); }
  void compress(const uint8_t* in, size_t n, uint32_t bl, std::vector<BlockOut>& out) override {
    if (!attempt([&] { gpu->compress(in, n, bl, out); })) cpu.compress(in, n, bl, out);
  }
  const uint8_t* decompress(const std::vector<BlockIn>& blocks) override {
    const uint8_t* raw = nullptr;
    if (attempt([&] { raw = gpu->decompress(blocks); })) return raw;
    return cpu.decompress(blocks);  // (a damaged block is reported from here)
  }

 private:
  Report* rep_ = nullptr;
  void say(const std::string& m) const { if (rep_) rep_->say(m); }
  size_t capped(size_t b, uint32_t bl) const {
    const size_t B = (size_t)1 << bl;
    return batch_cap && batch_cap < b ? (batch_cap > B ? batch_cap / B * B : B) : b;
  }
  template <class F> bool attempt(const F& f) {
    if (!gpu_ok) return false;
    try {
      f();
      return true;
    } catch (const zb::Error&) {
      return false;  // the data, not the device: the CPU redoes this batch
    } catch (const gpu::Error& e) {
      gpu_ok = false;
      say(std::string("GPU stopped working (") + e.what() + "); the CPU finishes the job");
      return false;
    }
  }
};

}  // namespace zero
