// dropin_zero.cpp -- TEST INFRASTRUCTURE: the drop-in check.  The reference's own archive pipeline
// (compress_archive / extract_archive / test_archive of src/archive.h, included unmodified from the
// reference tree) driven by the B200 codec through include/zero_cuda_codec.hpp, exactly where the
// reference's CLI puts its GpuCodec (src/main.cpp:36-57, 134-188).  Built by oracle/Makefile into
// oracle/_ref/zero_dropin when the reference tree is present.
//
//   zero_dropin c <file|folder>... -o <archive.zero> [--block N] [--level L]
//   zero_dropin x <archive.zero> -o <folder>
//   zero_dropin t <archive.zero>
//   zero_dropin bench <file> [--block N] [--level L]     (in memory, as src/main.cpp:205-277 measures)
//   zero_dropin c2 <file|folder>... -o <archive.zero> [--block N] [--level L]   (zc_archive_write)
//   zero_dropin t2 <archive.zero>                                             (zc_archive_extract)
//
// --safe puts zero::SafeCudaCodec (include/zero_cuda_safe.hpp) in place of the plain CudaCodec, as the
// reference's choose_codec puts SafeCodec around its GpuCodec; --batch-kib N caps its batches (so that a
// small job has several, and a failure injected with ZC_FAIL_AFTER=n can fall in the middle of a job).
#define ZERO_CUDA_DEFINE_GPU_ERROR
#include "archive.h"  // reference: src/archive.h
#include "zero_cuda_codec.hpp"
#include "zero_cuda_safe.hpp"

#include <memory>

#include <cstdio>
#include <fstream>
#include <iterator>

namespace {

int usage() {
  fprintf(stderr, "usage: zero_dropin c|x|t|bench|c2|t2 ...\n");
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) return usage();
  const std::string cmd = argv[1];
  std::vector<std::string> inputs;
  std::string out;
  uint32_t block_log = 18;
  int level = 5;
  bool safe = false;
  size_t batch_kib = 0;
  for (int i = 2; i < argc; ++i) {
    const std::string s = argv[i];
    if (s == "-o" && i + 1 < argc) out = argv[++i];
    else if (s == "--safe") safe = true;
    else if (s == "--batch-kib" && i + 1 < argc) batch_kib = (size_t)atoll(argv[++i]);
    else if (s == "--block" && i + 1 < argc) block_log = (uint32_t)atoi(argv[++i]);
    else if (s == "--level" && i + 1 < argc) level = atoi(argv[++i]);
    else inputs.push_back(s);
  }
  try {
    zero::Report rep;
    rep.log = [](const std::string& m) { fprintf(stderr, "%s\n", m.c_str()); };
    std::unique_ptr<zero::Codec> owned;
    if (safe) {
      auto sc = std::make_unique<zero::SafeCudaCodec>(level, 0, &rep);
      sc->batch_cap = batch_kib << 10;
      owned = std::move(sc);
    } else {
      owned = std::make_unique<zero::CudaCodec>(level);
    }
    zero::Codec& codec = *owned;
    if (cmd == "c") {
      const zero::CompressStats st = zero::compress_archive(inputs, out, codec, block_log, rep);
      printf("%s: %llu -> %llu bytes, %llu blocks (%llu stored), codec %.3f s\n", out.c_str(),
             (unsigned long long)st.raw, (unsigned long long)st.compressed, (unsigned long long)st.blocks,
             (unsigned long long)st.stored_blocks, st.codec_seconds);
      return 0;
    }
    if (cmd == "x") {
      const zero::ExtractStats st = zero::extract_archive(inputs.at(0), out, codec, rep);
      printf("%s: %zu files, %llu bytes, all checksums match\n", out.c_str(), st.files, (unsigned long long)st.raw);
      return 0;
    }
    if (cmd == "t") {
      const zero::ExtractStats st = zero::test_archive(inputs.at(0), codec, rep);
      printf("%s: OK, %zu files, %llu bytes in %llu blocks\n", inputs.at(0).c_str(), st.files,
             (unsigned long long)st.raw, (unsigned long long)st.blocks);
      return 0;
    }
    if (cmd == "c2" || cmd == "t2") {
      // the container on the GPU (zc_archive_write / zc_archive_extract), as `zero c` / `zero t` would call
      // it: the entries as the reference collects them (src/archive.h:170-250), the files read into one
      // solid stream in entry order (a file that shrank while read gives zeros, src/archive.h:316-318)
      zc_ctx* ctx = nullptr;
      if (zc_open(&ctx, 0) != ZC_OK) {
        const std::string m = ctx ? zc_last_error(ctx) : "zc_open failed";
        zc_close(ctx);
        throw std::runtime_error(m);
      }
      struct Closer { zc_ctx* c; ~Closer() { zc_close(c); } } closer{ctx};
      if (cmd == "t2") {
        std::ifstream f(inputs.at(0), std::ios::binary);
        std::vector<uint8_t> arch((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
        if (zc_archive_extract(ctx, arch.data(), arch.size(), nullptr, 0) != ZC_OK) throw zb::Error(zc_last_error(ctx));
        printf("%s: OK, every block and file checksum matches\n", inputs.at(0).c_str());
        return 0;
      }
      const std::vector<zero::Entry> es = zero::collect(inputs, rep);
      uint64_t total = 0;
      for (const zero::Entry& e : es) total += e.dir ? 0 : e.size;
      std::vector<uint8_t> solid(total + 1);
      std::vector<zc_entry> ze(es.size());
      size_t at = 0;
      for (size_t i = 0; i < es.size(); ++i) {
        const zero::Entry& e = es[i];
        ze[i] = zc_entry{e.name.data(), (uint32_t)e.name.size(), e.dir ? 1u : 0u, e.size, e.mtime, e.attr, 0};
        if (e.dir || !e.size) continue;
        FILE* f = zero::open_file(e.source, "rb");
        if (!f) throw zb::Error("cannot read " + e.name);
        const size_t r = fread(solid.data() + at, 1, (size_t)e.size, f);
        fclose(f);
        if (r != e.size) memset(solid.data() + at + r, 0, (size_t)e.size - r);
        at += (size_t)e.size;
      }
      std::vector<uint8_t> arch(zc_archive_bound(ze.data(), (uint32_t)ze.size(), block_log));
      uint64_t len = 0;
      if (arch.empty() || zc_archive_write(ctx, solid.data(), block_log, level, ze.data(), (uint32_t)ze.size(), arch.data(),
                                           arch.size(), &len) != ZC_OK)
        throw std::runtime_error(std::string("zc_archive_write: ") + zc_last_error(ctx));
      FILE* o = fopen(out.c_str(), "wb");
      if (!o || fwrite(arch.data(), 1, len, o) != len) throw zb::Error("writing " + out + " failed");
      fclose(o);
      printf("%s: %llu -> %llu bytes, the container written on the GPU\n", out.c_str(), (unsigned long long)total,
             (unsigned long long)len);
      return 0;
    }
    if (cmd == "bench") {
      std::ifstream f(inputs.at(0), std::ios::binary);
      std::vector<uint8_t> data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
      const size_t B = (size_t)1 << block_log;
      codec.prepare(block_log);
      const size_t batch = std::max(B, (codec.batch_bytes(block_log) / B) * B);
      std::vector<zero::BlockIn> ins;
      std::vector<std::vector<zero::BlockOut>> all;
      double t0 = zero_now();
      for (size_t off = 0; off < data.size(); off += batch) {
        std::vector<zero::BlockOut> outs;
        codec.compress(data.data() + off, std::min(batch, data.size() - off), block_log, outs);
        all.push_back(std::move(outs));
      }
      const double tc = zero_now() - t0;
      size_t pos = 0, comp = 0;
      for (auto& bo : all)
        for (zero::BlockOut& o : bo) {
          zero::BlockIn in;
          in.raw_len = (uint32_t)std::min(B, data.size() - pos);
          if (o.method == 0 || o.data.size() >= in.raw_len) { in.method = 0; in.data = data.data() + pos; in.comp_len = in.raw_len; }
          else { in.method = 1; in.data = o.data.data(); in.comp_len = (uint32_t)o.data.size(); }
          comp += in.comp_len;
          pos += in.raw_len;
          ins.push_back(in);
        }
      std::vector<uint8_t> raw(data.size());
      const size_t per = std::max<size_t>(1, codec.batch_bytes_decode(block_log) / B);
      t0 = zero_now();
      size_t o = 0;
      for (size_t i = 0; i < ins.size(); i += per) {
        std::vector<zero::BlockIn> part(ins.begin() + i, ins.begin() + std::min(ins.size(), i + per));
        const uint8_t* r = codec.decompress(part);
        size_t n = 0;
        for (const auto& k : part) n += k.raw_len;
        memcpy(raw.data() + o, r, n);
        o += n;
      }
      const double td = zero_now() - t0;
      const bool ok = raw == data;
      printf("compress %.3f s (%.0f MB/s) %zu -> %zu; decompress %.3f s (%.0f MB/s): %s\n", tc, data.size() / tc / 1e6,
             data.size(), comp, td, data.size() / td / 1e6, ok ? "identical" : "MISMATCH");
      return ok ? 0 : 1;
    }
    return usage();
  } catch (const std::exception& e) {
    fprintf(stderr, "zero_dropin: %s\n", e.what());
    return 1;
  }
}
