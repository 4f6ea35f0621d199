// zc_archive.cu -- whole .zero archives around the block codec: the container that compress_archive
// writes (src/archive.h:334-441) and read_info / read_blocks / extract_archive / test_archive read and
// check (src/archive.h:451-495, 566-635, 640-790), assembled and checked on the GPU.
//
// Writing, all queued on one stream with no host wait between the stages:
//   k_arch_head    the 24-byte header; the first record's position (24) for the encoder's scan
//   encoder        in record mode: each block's 16-byte record header and body, placed by a device scan
//                  that starts where the previous launch's records end
//   k_crc_blocks   ("k_crc_pieces") the CRCs of file pieces that do not cover a whole block
//   k_file_crcs    a warp per file: its pieces' CRCs combined in stream order (crc32::combine,
//                  src/crc32.h:60-66) and written into the entry table's CRC field
//   k_arch_tail    the table after the last record (every CTA copies a share), its CRC, the footer
// The host builds only descriptors: the entry table with zero CRC fields, and every file's span of the
// solid stream cut at block boundaries (whole blocks reuse the block CRCs the encoder computes first).
//
// Reading: the header, footer, table and block records are parsed on the host (they are a few bytes
// per block and per entry); the blocks are decoded, and the block and file CRCs computed, on the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/zero_cuda.h"
#include "zc_host.h"
#include "zc_internal.cuh"
#include "zc_kernels.h"

using namespace zch;

namespace {

constexpr uint32_t kPart = 0x80000000u;  // a piece reference naming a partial piece, not a whole block
constexpr uint64_t kArchHdr = 24, kArchFoot = 24;

struct Head {
  uint8_t b[24];
};

__global__ void k_arch_head(Head h, uint8_t* out, uint64_t* rec_end0) {
  const uint32_t t = threadIdx.x;
  if (t < 24) out[t] = h.b[t];
  if (t == 0) *rec_end0 = kArchHdr;
}

// a range's records: the first record's position for the encoder's scan; then the end of the last record
__global__ void k_range_start(uint64_t* rec_end0, uint64_t rec_base) { *rec_end0 = rec_base; }
__global__ void k_range_end(const uint64_t* rec_end, uint64_t* out_len) { *out_len = *rec_end; }

struct FileCrcArgs {
  uint32_t nf;               // files with bytes
  const uint32_t* first;     // nf + 1: file f's pieces are [first[f], first[f + 1])
  const uint32_t* ref;       // per piece: a block index, or kPart | a partial piece's index
  const uint32_t* len;       // per piece: its bytes
  const uint32_t* blk_crc;   // per block: CRC-32 of the whole block
  const uint32_t* part_crc;  // per partial piece
  const uint32_t* pos;       // per file: its CRC field's offset in the table (with table)
  const uint32_t* entry;     // per file: its entry index
  uint8_t* table;            // may be NULL: the CRCs are only reported
  uint32_t* entry_crc;       // may be NULL: per entry
  const zc::CrcTables* T;
};

// A warp per file.  Lane l combines a contiguous run of the file's pieces, then the lanes' runs are
// joined in order by a tree: crc(A || B) = crc(A) * x^(8 |B|) ^ crc(B) over GF(2).
__global__ void __launch_bounds__(256) k_file_crcs(FileCrcArgs A) {
  const uint32_t f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
  if (f >= A.nf) return;  // (uniform over the warp)
  const uint32_t p0 = A.first[f], p1 = A.first[f + 1];
  const uint32_t per = (p1 - p0 + 31u) / 32u;
  const uint32_t a = min(p0 + lane * per, p1), b = min(a + per, p1);
  const uint32_t* pow2 = A.T->pow2;
  uint32_t c = 0;
  uint64_t n = 0;
  for (uint32_t p = a; p < b; ++p) {
    const uint32_t r = A.ref[p], l = A.len[p];
    const uint32_t pc = (r & kPart) ? A.part_crc[r & ~kPart] : A.blk_crc[r];
    c = zc::gf2_mul(c, zc::gf2_xpow8n(pow2, l)) ^ pc;
    n += l;
  }
#pragma unroll
  for (uint32_t k = 0; k < 5; ++k) {
    const uint32_t oc = __shfl_down_sync(zc::kFull, c, 1u << k);
    const uint64_t on = __shfl_down_sync(zc::kFull, n, 1u << k);
    if ((lane & ((2u << k) - 1u)) == 0) {
      c = zc::gf2_mul(c, zc::gf2_xpow8n(pow2, on)) ^ oc;
      n += on;
    }
  }
  c = __shfl_sync(zc::kFull, c, 0);
  if (A.table && lane < 4) A.table[A.pos[f] + lane] = (uint8_t)(c >> (8u * lane));
  if (A.entry_crc && lane == 0) A.entry_crc[A.entry[f]] = c;
}

struct TailArgs {
  const uint64_t* rec_end;   // device: the end of the last record
  const uint8_t* table;      // the entry table, CRC fields filled
  uint32_t tl;
  uint8_t* out;
  uint64_t out_cap;
  uint64_t* out_len;         // device: the archive's length (0 if it did not fit)
  const zc::CrcTables* T;
};

// The table at the end of the records and the footer {u64 table offset, u64 table length, u32 CRC,
// "ZEND"} (src/archive.h:430-435).  Every CTA copies a share of the table; CTA 0 computes its CRC
// from the descriptor copy and writes the footer.
__global__ void __launch_bounds__(1024) k_arch_tail(TailArgs A) {
  const uint64_t end = *A.rec_end;
  const bool fits = end + A.tl + kArchFoot <= A.out_cap;
  if (fits) {
    uint8_t* d = A.out + end;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < A.tl; i += (uint64_t)gridDim.x * blockDim.x)
      d[i] = A.table[i];
  }
  if (blockIdx.x != 0) return;
  __shared__ uint32_t t[8][256];
  __shared__ uint32_t red[32];
  zc::load_crc_tables(A.T, t);
  __syncthreads();
  const uint32_t crc = zc::cta_crc32(A.T, t, A.table, A.tl, red);
  const uint32_t i = threadIdx.x;
  if (fits && i < kArchFoot) {
    const uint64_t v = i < 8 ? end : i < 16 ? (uint64_t)A.tl : crc;
    const uint32_t sh = 8u * (i & 7u);
    A.out[end + A.tl + i] = i < 20 ? (uint8_t)(v >> sh) : (uint8_t)("ZEND"[i - 20]);
  }
  if (i == 0) *A.out_len = fits ? end + A.tl + kArchFoot : 0;
}

// ---------------------------------------------------------------- host side

void put32(std::vector<uint8_t>& v, uint32_t x) {
  for (int i = 0; i < 4; ++i) v.push_back((uint8_t)(x >> (8 * i)));
}
uint32_t get32(const uint8_t* p) {
  return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
}
uint64_t get64(const uint8_t* p) { return (uint64_t)get32(p) | (uint64_t)get32(p + 4) << 32; }

// CRC-32 on the host (slice-by-8), for the table check of a read
uint32_t host_crc32(const uint8_t* p, uint64_t n) {
  static const zc::CrcTables T = [] {
    zc::CrcTables x;
    build_crc_tables(x);
    return x;
  }();
  uint32_t c = 0xFFFFFFFFu;
  for (; n >= 8; n -= 8, p += 8) {
    const uint32_t a = get32(p) ^ c, b = get32(p + 4);
    c = T.t[7][a & 0xFFu] ^ T.t[6][(a >> 8) & 0xFFu] ^ T.t[5][(a >> 16) & 0xFFu] ^ T.t[4][a >> 24] ^
        T.t[3][b & 0xFFu] ^ T.t[2][(b >> 8) & 0xFFu] ^ T.t[1][(b >> 16) & 0xFFu] ^ T.t[0][b >> 24];
  }
  for (; n; --n, ++p) c = T.t[0][(c ^ *p) & 0xFFu] ^ (c >> 8);
  return ~c;
}

// Every file's span of the solid stream cut at block boundaries.  A piece that covers a whole block is
// named by the block (its CRC is the block's); the others are partial pieces with their own CRC.
struct Pieces {
  std::vector<uint32_t> first, entry;  // per file with bytes (+1 for first)
  std::vector<uint32_t> ref, len;      // per piece
  std::vector<uint64_t> part_off;      // per partial piece: its offset in the solid stream
  std::vector<uint32_t> part_len;
};

bool cut_pieces(const zc_entry* es, uint32_t ne, uint32_t bl, uint64_t n, Pieces& P, std::string& why) {
  const uint64_t B = 1ull << bl;
  uint64_t at = 0;
  for (uint32_t i = 0; i < ne; ++i) {
    if (es[i].is_dir || !es[i].size) continue;
    const uint64_t s = at, e = at + es[i].size;
    if (e > n) { why = "the entries hold more bytes than the stream"; return false; }
    P.first.push_back((uint32_t)P.ref.size());
    P.entry.push_back(i);
    for (uint64_t b = s >> bl; b <= (e - 1) >> bl; ++b) {
      const uint64_t bs = b << bl, be = std::min(bs + B, n);
      const uint64_t ps = std::max(s, bs), pe = std::min(e, be);
      if (ps == bs && pe == be) {
        P.ref.push_back((uint32_t)b);
      } else {
        P.ref.push_back(kPart | (uint32_t)P.part_off.size());
        P.part_off.push_back(ps);
        P.part_len.push_back((uint32_t)(pe - ps));
      }
      P.len.push_back((uint32_t)(pe - ps));
      if (P.ref.size() >= 0xFFFFFFFFull || P.part_off.size() >= kPart) { why = "too many file pieces"; return false; }
    }
    at = e;
  }
  P.first.push_back((uint32_t)P.ref.size());
  return true;
}

// The pieces of every file inside the stream range [lo, hi) (lo a multiple of the block size; hi too, or
// the stream's end): blocks are numbered from the range's first, partial pieces' offsets count from lo.
bool cut_range_pieces(const zc_entry* es, uint32_t ne, uint32_t bl, uint64_t lo, uint64_t hi, Pieces& P,
                      std::string& why) {
  const uint64_t B = 1ull << bl;
  uint64_t at = 0;
  for (uint32_t i = 0; i < ne; ++i) {
    if (es[i].is_dir || !es[i].size) continue;
    const uint64_t s = std::max(at, lo), e = std::min(at + es[i].size, hi);
    at += es[i].size;
    if (e <= s) continue;
    P.first.push_back((uint32_t)P.ref.size());
    P.entry.push_back(i);
    for (uint64_t b = s >> bl; b <= (e - 1) >> bl; ++b) {
      const uint64_t bs = b << bl, be = std::min(bs + B, hi);
      const uint64_t ps = std::max(s, bs), pe = std::min(e, be);
      if (ps == bs && pe == be) {
        P.ref.push_back((uint32_t)(b - (lo >> bl)));
      } else {
        P.ref.push_back(kPart | (uint32_t)P.part_off.size());
        P.part_off.push_back(ps - lo);
        P.part_len.push_back((uint32_t)(pe - ps));
      }
      P.len.push_back((uint32_t)(pe - ps));
      if (P.ref.size() >= 0xFFFFFFFFull || P.part_off.size() >= kPart) { why = "too many file pieces"; return false; }
    }
  }
  P.first.push_back((uint32_t)P.ref.size());
  return true;
}

// Checks the entries of a write: *n gets the stream's bytes.
bool check_entries(const zc_entry* es, uint32_t ne, uint64_t* n, std::string& why) {
  if (ne && !es) { why = "no entries"; return false; }
  uint64_t sum = 0;
  for (uint32_t i = 0; i < ne; ++i) {
    if (es[i].name_len && !es[i].name) { why = "an entry has no name"; return false; }
    if (es[i].is_dir && es[i].size) { why = "a folder entry must have size 0"; return false; }
    if (sum + es[i].size < sum) { why = "the entries' sizes overflow"; return false; }
    sum += es[i].size;
  }
  *n = sum;
  return true;
}

uint64_t table_bytes(const zc_entry* es, uint32_t ne) {
  uint64_t t = 4;
  for (uint32_t i = 0; i < ne; ++i) t += 8 + (uint64_t)es[i].name_len + 24;
  return t;
}

// The entry table (src/archive.h:416-429) with zero CRC fields; pos[f] = the offset of file f's field.
void build_table(const zc_entry* es, uint32_t ne, const Pieces& P, std::vector<uint8_t>& t, std::vector<uint32_t>& pos) {
  t.reserve(table_bytes(es, ne));
  put32(t, ne);
  size_t f = 0;
  for (uint32_t i = 0; i < ne; ++i) {
    const zc_entry& e = es[i];
    t.push_back(e.is_dir ? 1 : 0);
    t.push_back(0); t.push_back(0); t.push_back(0);
    put32(t, e.name_len);
    t.insert(t.end(), reinterpret_cast<const uint8_t*>(e.name), reinterpret_cast<const uint8_t*>(e.name) + e.name_len);
    put32(t, (uint32_t)e.size);
    put32(t, (uint32_t)(e.size >> 32));
    put32(t, (uint32_t)(uint64_t)e.mtime);
    put32(t, (uint32_t)((uint64_t)e.mtime >> 32));
    put32(t, e.attr);
    if (f < P.entry.size() && P.entry[f] == i) { pos.push_back((uint32_t)t.size()); ++f; }
    put32(t, 0);
  }
}

// sections of one descriptor or result buffer, each 256-byte aligned
struct Layout {
  size_t at = 0;
  size_t put(size_t bytes) {
    const size_t o = at;
    at = (at + bytes + 255) & ~(size_t)255;
    return o;
  }
};

template <class T>
void put_section(std::vector<uint8_t>& h, size_t off, const std::vector<T>& v) {
  if (!v.empty()) memcpy(h.data() + off, v.data(), v.size() * sizeof(T));
}

// Uploads the pieces (at the given offsets of the descriptor buffer) and launches the file CRCs.
struct PieceDev {
  size_t first, entry, ref, len, part_off, part_len, pos;
};

PieceDev place_pieces(Layout& L, const Pieces& P, bool with_pos) {
  PieceDev d{};
  d.first = L.put(4 * P.first.size());
  d.entry = L.put(4 * P.entry.size());
  d.ref = L.put(4 * P.ref.size());
  d.len = L.put(4 * P.len.size());
  d.part_off = L.put(8 * P.part_off.size());
  d.part_len = L.put(4 * P.part_len.size());
  d.pos = with_pos ? L.put(4 * P.entry.size()) : 0;
  return d;
}

void fill_pieces(std::vector<uint8_t>& h, const PieceDev& d, const Pieces& P) {
  put_section(h, d.first, P.first);
  put_section(h, d.entry, P.entry);
  put_section(h, d.ref, P.ref);
  put_section(h, d.len, P.len);
  put_section(h, d.part_off, P.part_off);
  put_section(h, d.part_len, P.part_len);
}

// k_crc_pieces: the CRCs of np partial pieces (offsets from base, lengths: device arrays)
void launch_piece_crcs(zc_ctx* c, const uint8_t* base, const uint64_t* offs, const uint32_t* lens, uint32_t np,
                       uint32_t* part_crc, cudaStream_t st) {
  if (!np) return;
  zc::CrcArgs C{};
  C.base = base;
  C.offs = offs;
  C.lens = lens;
  C.nb = np;
  C.crc = part_crc;
  C.tables = c->d_crct;
  zc::launch_crc(C, st, c->stages, "k_crc_pieces");
}

// k_file_crcs: every file's CRC from its pieces' (block and partial piece CRCs already computed)
void launch_combine(zc_ctx* c, const uint8_t* D, const PieceDev& d, const Pieces& P, const uint32_t* blk_crc,
                    const uint32_t* part_crc, uint8_t* table, uint32_t* entry_crc, cudaStream_t st) {
  const uint32_t nf = (uint32_t)P.entry.size();
  if (!nf) return;
  FileCrcArgs F{};
  F.nf = nf;
  F.first = reinterpret_cast<const uint32_t*>(D + d.first);
  F.entry = reinterpret_cast<const uint32_t*>(D + d.entry);
  F.ref = reinterpret_cast<const uint32_t*>(D + d.ref);
  F.len = reinterpret_cast<const uint32_t*>(D + d.len);
  F.pos = table ? reinterpret_cast<const uint32_t*>(D + d.pos) : nullptr;
  F.blk_crc = blk_crc;
  F.part_crc = part_crc;
  F.table = table;
  F.entry_crc = entry_crc;
  F.T = c->d_crct;
  c->stages.begin("k_file_crcs", st);
  k_file_crcs<<<(nf + 7) / 8, 256, 0, st>>>(F);
  c->stages.end(st);
}

// k_crc_pieces + k_file_crcs over a solid stream resident on the device
void launch_file_crcs(zc_ctx* c, const uint8_t* d_solid, const uint8_t* D, const PieceDev& d, const Pieces& P,
                      const uint32_t* blk_crc, uint32_t* part_crc, uint8_t* table, uint32_t* entry_crc, cudaStream_t st) {
  launch_piece_crcs(c, d_solid, reinterpret_cast<const uint64_t*>(D + d.part_off),
                    reinterpret_cast<const uint32_t*>(D + d.part_len), (uint32_t)P.part_off.size(), part_crc, st);
  launch_combine(c, D, d, P, blk_crc, part_crc, table, entry_crc, st);
}

// the archive header (src/archive.h:356-361): "ZERO", version 2, block_log, 0, total raw bytes, blocks
void put_header(uint8_t* out, uint64_t n, uint64_t nb, uint32_t bl) {
  memcpy(out, "ZERO", 4);
  out[4] = 2;
  out[5] = (uint8_t)bl;
  out[6] = out[7] = 0;
  for (int i = 0; i < 8; ++i) {
    out[8 + i] = (uint8_t)(n >> (8 * i));
    out[16 + i] = (uint8_t)(nb >> (8 * i));
  }
}

int write_device(zc_ctx* c, const uint8_t* d_solid, uint32_t bl, int level, const zc_entry* es, uint32_t ne,
                 uint8_t* d_out, uint64_t out_cap, uint64_t* d_len, uint32_t* d_entry_crcs, cudaStream_t st) {
  if (bad_block_log(bl)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  std::string why;
  uint64_t n = 0;
  if (!check_entries(es, ne, &n, why)) return fail(c, ZC_E_ARG, why);
  if (n && (!d_solid || ((uintptr_t)d_solid & 15u))) return fail(c, ZC_E_ARG, "the solid stream must be 16-byte aligned");
  if (!d_out || !d_len) return fail(c, ZC_E_ARG, "no output");
  const uint64_t B = 1ull << bl, nb64 = (n + B - 1) >> bl;
  if (nb64 >= kPart) return fail(c, ZC_E_ARG, "too many blocks");
  const uint32_t nb = (uint32_t)nb64;
  Pieces P;
  if (!cut_pieces(es, ne, bl, n, P, why)) return fail(c, ZC_E_ARG, why);
  std::vector<uint8_t> table;
  std::vector<uint32_t> pos;
  build_table(es, ne, P, table, pos);
  if (table.size() >= 0xFFFFFFFFull) return fail(c, ZC_E_ARG, "the entry table is too large");
  if (out_cap < zc_archive_bound(es, ne, bl)) return fail(c, ZC_E_ARG, "the output is smaller than zc_archive_bound");
  const uint32_t per = enc_blocks_per_launch(bl), nchunk = (nb + per - 1) / per;
  // descriptors, one upload
  Layout L;
  const size_t o_tab = L.put(table.size());
  const PieceDev pd = place_pieces(L, P, true);
  std::vector<uint8_t> h(L.at);
  memcpy(h.data() + o_tab, table.data(), table.size());
  fill_pieces(h, pd, P);
  put_section(h, pd.pos, pos);
  // per-block results and per-launch block lists
  const uint32_t kmax = std::max(1u, std::min(nb, per));
  Layout W;
  const size_t o_meth = W.put(nb), o_lens = W.put(4ull * nb), o_crcs = W.put(4ull * nb), o_offs = W.put(8ull * nb);
  const size_t o_ioff = W.put(8ull * kmax), o_ilen = W.put(4ull * kmax), o_pcrc = W.put(4 * P.part_off.size());
  const size_t o_ends = W.put(8ull * (nchunk + 1));
  ZC_CUDA(grow(c->a_desc, L.at));
  ZC_CUDA(grow(c->a_work, W.at));
  uint8_t* D = c->a_desc.as<uint8_t>();
  uint8_t* X = c->a_work.as<uint8_t>();
  ZC_CUDA(cudaMemcpyAsync(D, h.data(), L.at, cudaMemcpyHostToDevice, st));
  uint64_t* ends = reinterpret_cast<uint64_t*>(X + o_ends);
  uint32_t* crcs = reinterpret_cast<uint32_t*>(X + o_crcs);
  Head hd{};
  put_header(hd.b, n, nb64, bl);
  c->stages.begin("k_arch_head", st);
  k_arch_head<<<1, 32, 0, st>>>(hd, d_out, ends);
  c->stages.end(st);
  for (uint32_t i = 0, b0 = 0; i < nchunk; ++i, b0 += per) {
    const uint32_t k = std::min(per, nb - b0);
    const uint64_t span = std::min<uint64_t>(n - (uint64_t)b0 * B, (uint64_t)k * B);
    uint64_t* ioff = reinterpret_cast<uint64_t*>(X + o_ioff);
    uint32_t* ilen = reinterpret_cast<uint32_t*>(X + o_ilen);
    plain_blocks(c, span, (uint32_t)B, k, ioff, ilen, st);
    if (int r = encode_device(c, d_solid + (uint64_t)b0 * B, ioff, ilen, k, bl, level, X + o_meth + b0,
                              reinterpret_cast<uint32_t*>(X + o_lens) + b0, crcs + b0, d_out, out_cap,
                              reinterpret_cast<uint64_t*>(X + o_offs) + b0, ends + i + 1, 1, st, ends + i))
      return r;
  }
  if (d_entry_crcs && ne) ZC_CUDA(cudaMemsetAsync(d_entry_crcs, 0, 4ull * ne, st));
  launch_file_crcs(c, d_solid, D, pd, P, crcs, reinterpret_cast<uint32_t*>(X + o_pcrc), D + o_tab, d_entry_crcs, st);
  TailArgs T{};
  T.rec_end = ends + nchunk;
  T.table = D + o_tab;
  T.tl = (uint32_t)table.size();
  T.out = d_out;
  T.out_cap = out_cap;
  T.out_len = d_len;
  T.T = c->d_crct;
  const uint32_t grid = (uint32_t)std::min<uint64_t>(592, std::max<uint64_t>(1, (table.size() + 16383) / 16384));
  c->stages.begin("k_arch_tail", st);
  k_arch_tail<<<grid, 1024, 0, st>>>(T);
  c->stages.end(st);
  return check_launch(c, "archive launch");
}

// One rank's share of a sharded archive: the block records of a range of the solid stream, from
// rec_base on, and each file's CRC over its part of the range (the rank's piece of the file CRC).
int write_range(zc_ctx* c, const uint8_t* d_range, uint64_t lo, uint64_t len, uint32_t bl, int level,
                const zc_entry* es, uint32_t ne, uint64_t rec_base, uint8_t* d_out, uint64_t out_cap,
                uint64_t* d_len, uint32_t* d_piece_crcs, cudaStream_t st) {
  if (bad_block_log(bl)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  std::string why;
  uint64_t n = 0;
  if (!check_entries(es, ne, &n, why)) return fail(c, ZC_E_ARG, why);
  const uint64_t B = 1ull << bl, hi = lo + len;
  if (lo & (B - 1) || hi > n || hi < lo || ((hi & (B - 1)) && hi != n))
    return fail(c, ZC_E_ARG, "a range must start at a block boundary and end at one or at the stream's end");
  if (len && (!d_range || ((uintptr_t)d_range & 15u))) return fail(c, ZC_E_ARG, "the range must be 16-byte aligned");
  if (!d_out || !d_len) return fail(c, ZC_E_ARG, "no output");
  const uint64_t nb64 = (len + B - 1) >> bl;
  if (nb64 >= kPart) return fail(c, ZC_E_ARG, "too many blocks");
  const uint32_t nb = (uint32_t)nb64;
  if (out_cap < rec_base || out_cap - rec_base < nb64 * zc::kRecHdr + len)
    return fail(c, ZC_E_ARG, "the output cannot hold the range's records (16 bytes + the block, each)");
  Pieces P;
  if (!cut_range_pieces(es, ne, bl, lo, hi, P, why)) return fail(c, ZC_E_ARG, why);
  const uint32_t per = enc_blocks_per_launch(bl), nchunk = (nb + per - 1) / per;
  Layout L;
  const PieceDev pd = place_pieces(L, P, false);
  std::vector<uint8_t> h(std::max<size_t>(L.at, 1));
  fill_pieces(h, pd, P);
  const uint32_t kmax = std::max(1u, std::min(nb, per));
  Layout W;
  const size_t o_meth = W.put(nb), o_lens = W.put(4ull * nb), o_crcs = W.put(4ull * nb), o_offs = W.put(8ull * nb);
  const size_t o_ioff = W.put(8ull * kmax), o_ilen = W.put(4ull * kmax), o_pcrc = W.put(4 * P.part_off.size());
  const size_t o_ends = W.put(8ull * (nchunk + 1));
  ZC_CUDA(grow(c->a_desc, std::max<size_t>(L.at, 256)));
  ZC_CUDA(grow(c->a_work, W.at));
  uint8_t* D = c->a_desc.as<uint8_t>();
  uint8_t* X = c->a_work.as<uint8_t>();
  if (L.at) ZC_CUDA(cudaMemcpyAsync(D, h.data(), L.at, cudaMemcpyHostToDevice, st));
  uint64_t* ends = reinterpret_cast<uint64_t*>(X + o_ends);
  uint32_t* crcs = reinterpret_cast<uint32_t*>(X + o_crcs);
  c->stages.begin("k_range_start", st);
  k_range_start<<<1, 1, 0, st>>>(ends, rec_base);
  c->stages.end(st);
  for (uint32_t i = 0, b0 = 0; i < nchunk; ++i, b0 += per) {
    const uint32_t k = std::min(per, nb - b0);
    const uint64_t span = std::min<uint64_t>(len - (uint64_t)b0 * B, (uint64_t)k * B);
    uint64_t* ioff = reinterpret_cast<uint64_t*>(X + o_ioff);
    uint32_t* ilen = reinterpret_cast<uint32_t*>(X + o_ilen);
    plain_blocks(c, span, (uint32_t)B, k, ioff, ilen, st);
    if (int r = encode_device(c, d_range + (uint64_t)b0 * B, ioff, ilen, k, bl, level, X + o_meth + b0,
                              reinterpret_cast<uint32_t*>(X + o_lens) + b0, crcs + b0, d_out, out_cap,
                              reinterpret_cast<uint64_t*>(X + o_offs) + b0, ends + i + 1, 1, st, ends + i))
      return r;
  }
  if (d_piece_crcs && ne) ZC_CUDA(cudaMemsetAsync(d_piece_crcs, 0, 4ull * ne, st));
  launch_file_crcs(c, d_range, D, pd, P, crcs, reinterpret_cast<uint32_t*>(X + o_pcrc), nullptr, d_piece_crcs, st);
  c->stages.begin("k_range_end", st);
  k_range_end<<<1, 1, 0, st>>>(ends + nchunk, d_len);
  c->stages.end(st);
  return check_launch(c, "archive range launch");
}

int msg_fail(char* msg, size_t cap, const std::string& why) {
  if (msg && cap) snprintf(msg, cap, "%s", why.c_str());
  return ZC_E_DATA;
}

// read_info (src/archive.h:451-495): the same checks in the same order
int parse_table(const uint8_t* a, uint64_t len, zc_archive_info* info, std::vector<zc_entry>* out, std::string& why) {
  if (!a || len < kArchHdr || memcmp(a, "ZERO", 4) != 0) { why = "not a .zero archive"; return ZC_E_DATA; }
  if (a[4] != 2) {
    why = "archive version " + std::to_string(a[4]) + ": this program reads version 2";
    return ZC_E_DATA;
  }
  zc_archive_info I{};
  I.block_log = a[5];
  I.total_raw = get64(a + 8);
  I.n_blocks = get64(a + 16);
  if (I.block_log < zc::kMinBlockLog || I.block_log > zc::kMaxBlockLog) { why = "archive damaged: block size"; return ZC_E_DATA; }
  if (len < kArchHdr + kArchFoot) { why = "archive damaged: too short"; return ZC_E_DATA; }
  const uint8_t* ft = a + len - kArchFoot;
  if (memcmp(ft + 20, "ZEND", 4) != 0) { why = "archive damaged: footer (the file was cut short?)"; return ZC_E_DATA; }
  I.table_off = get64(ft);
  I.table_len = get64(ft + 8);
  const uint32_t tc = get32(ft + 16);
  if (I.table_off < kArchHdr || I.table_off > len - kArchFoot || I.table_len != len - kArchFoot - I.table_off) {
    why = "archive damaged: table position";
    return ZC_E_DATA;
  }
  const uint8_t* p = a + I.table_off;
  const uint8_t* end = p + I.table_len;
  if (host_crc32(p, I.table_len) != tc) { why = "archive damaged: table checksum"; return ZC_E_DATA; }
  if (I.table_len < 4) { why = "archive damaged: table"; return ZC_E_DATA; }
  const uint32_t n = get32(p);
  p += 4;
  uint64_t sum = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (end - p < 8) { why = "archive damaged: entry"; return ZC_E_DATA; }
    zc_entry e{};
    e.is_dir = p[0] == 1;
    e.name_len = get32(p + 4);
    p += 8;
    if ((uint64_t)(end - p) < (uint64_t)e.name_len + 24) { why = "archive damaged: entry name"; return ZC_E_DATA; }
    e.name = reinterpret_cast<const char*>(p);
    p += e.name_len;
    e.size = get64(p);
    e.mtime = (int64_t)get64(p + 8);
    e.attr = get32(p + 16);
    e.crc = get32(p + 20);
    p += 24;
    if (!e.is_dir) sum += e.size;
    if (out) out->push_back(e);
  }
  if (sum != I.total_raw) { why = "archive damaged: sizes"; return ZC_E_DATA; }
  I.n_entries = n;
  *info = I;
  return ZC_OK;
}

// the record walk of read_blocks (src/archive.h:566-586)
int walk_blocks(const uint8_t* a, uint64_t len, const zc_archive_info& I, uint64_t* offs, uint32_t* clens,
                uint8_t* methods, uint32_t* rlens, uint32_t* crcs, std::string& why) {
  const uint64_t B = 1ull << I.block_log;
  uint64_t pos = kArchHdr;
  for (uint64_t b = 0; b < I.n_blocks; ++b) {
    if (pos > len || len - pos < zc::kRecHdr) { why = "archive damaged: block header cut"; return ZC_E_DATA; }
    const uint8_t* h = a + pos;
    pos += zc::kRecHdr;
    const uint32_t raw = get32(h), comp = get32(h + 4);
    const uint8_t method = h[8];
    if (raw > B || (method == 0 && comp != raw) || method > 1) { why = "archive damaged: block header"; return ZC_E_DATA; }
    if (pos + comp > I.table_off) { why = "archive damaged: block past the table"; return ZC_E_DATA; }
    offs[b] = pos;
    clens[b] = comp;
    methods[b] = method;
    rlens[b] = raw;
    if (crcs) crcs[b] = get32(h + 12);
    pos += comp;
  }
  return ZC_OK;
}


// the partial pieces that start in the stream range [lo, hi): indices [q0, q1) (pieces are in stream order)
void pieces_in(const Pieces& P, uint64_t lo, uint64_t hi, uint32_t& q0, uint32_t& q1) {
  q0 = (uint32_t)(std::lower_bound(P.part_off.begin(), P.part_off.end(), lo) - P.part_off.begin());
  q1 = (uint32_t)(std::lower_bound(P.part_off.begin(), P.part_off.end(), hi) - P.part_off.begin());
}

// Host-pointer archive write.  The solid stream goes up in chunks of whole blocks (128 MiB, then 512 MiB)
// through the context's two stages: a chunk's upload and the previous chunk's records coming down (copy
// stream) overlap the chunk's kernels.  Each chunk's records are written from the start of its stage
// buffer; the partial file pieces inside the chunk get their CRCs while it is resident.  At the end the
// files' CRCs are combined on the device and the host writes the table and footer after the records.
int write_host(zc_ctx* c, const uint8_t* solid, uint32_t bl, int level, zc_entry* es, uint32_t ne, uint8_t* out,
               uint64_t out_cap, uint64_t* out_len) {
  if (bad_block_log(bl)) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  std::string why;
  uint64_t n = 0;
  if (!check_entries(es, ne, &n, why)) return fail(c, ZC_E_ARG, why);
  if ((n && !solid) || !out) return fail(c, ZC_E_ARG, "no input or no output");
  if (out_cap < kArchHdr) return fail(c, ZC_E_ARG, "the output buffer is too small");
  const uint64_t B = 1ull << bl, nb64 = (n + B - 1) >> bl;
  if (nb64 >= kPart) return fail(c, ZC_E_ARG, "too many blocks");
  const uint32_t nb = (uint32_t)nb64;
  Pieces P;
  if (!cut_pieces(es, ne, bl, n, P, why)) return fail(c, ZC_E_ARG, why);
  std::vector<uint8_t> table;
  std::vector<uint32_t> pos;
  build_table(es, ne, P, table, pos);
  if (table.size() >= 0xFFFFFFFFull) return fail(c, ZC_E_ARG, "the entry table is too large");
  cudaStream_t st = c->stream, cs = c->cstream;
  Layout L;
  const PieceDev pd = place_pieces(L, P, false);
  std::vector<uint8_t> h(L.at);
  fill_pieces(h, pd, P);
  const uint32_t nq = (uint32_t)P.part_off.size();
  Layout W;
  const size_t o_crc = W.put(4ull * nb), o_pcrc = W.put(4ull * nq), o_ecrc = W.put(4ull * ne), o_zero = W.put(8);
  const size_t o_meth = W.put(nb), o_lens = W.put(4ull * nb), o_offs = W.put(8ull * nb);
  ZC_CUDA(grow(c->a_desc, L.at));
  ZC_CUDA(grow(c->a_work, W.at));
  uint8_t* D = c->a_desc.as<uint8_t>();
  uint8_t* X = c->a_work.as<uint8_t>();
  ZC_CUDA(cudaMemcpyAsync(D, h.data(), L.at, cudaMemcpyHostToDevice, st));
  ZC_CUDA(cudaMemsetAsync(X + o_zero, 0, 8, st));
  uint32_t* d_crc = reinterpret_cast<uint32_t*>(X + o_crc);
  uint32_t* d_pcrc = reinterpret_cast<uint32_t*>(X + o_pcrc);
  put_header(out, n, nb64, bl);
  uint64_t at = kArchHdr;
  const uint32_t per_launch = enc_blocks_per_launch(bl);
  struct Chunk {
    uint32_t b0 = 0, k = 0;
    size_t len_at = 0;  // where the chunk's records length lies in its stage's descriptors
  };
  Chunk prev;
  bool have_prev = false;
  // a finished chunk: its records length, then its records, come down on the copy stream
  auto harvest = [&](zc_ctx::Stage& S, const Chunk& q) -> int {
    ZC_CUDA(cudaStreamWaitEvent(cs, S.ev_done, 0));
    uint64_t* h_len = reinterpret_cast<uint64_t*>(static_cast<uint8_t*>(S.h.p) + q.len_at);
    ZC_CUDA(cudaMemcpyAsync(h_len, S.blk.as<uint8_t>() + q.len_at, 8, cudaMemcpyDeviceToHost, cs));
    ZC_CUDA(cudaStreamSynchronize(cs));
    const uint64_t rl = *h_len;
    if (rl > out_cap - at) return fail(c, ZC_E_ARG, "the output buffer is too small");
    if (rl) ZC_CUDA(cudaMemcpyAsync(out + at, S.out.p, rl, cudaMemcpyDeviceToHost, cs));
    ZC_CUDA(cudaStreamSynchronize(cs));
    at += rl;
    return ZC_OK;
  };
  uint32_t it = 0;
  for (uint32_t b0 = 0; b0 < nb; b0 += prev.k, ++it) {
    zc_ctx::Stage& S = c->pipe[it & 1];
    Chunk q;
    q.b0 = b0;
    q.k = std::min(host_chunk_blocks(bl, per_launch, it), nb - b0);
    const uint32_t k = q.k;
    const uint64_t lo = (uint64_t)b0 * B, span = std::min<uint64_t>(n - lo, (uint64_t)k * B);
    uint32_t q0, q1;
    pieces_in(P, lo, lo + span, q0, q1);
    const uint32_t kq = q1 - q0;
    // the stage's descriptors: block offsets and lengths (written by k_plain_blocks), the chunk's partial
    // pieces (offsets from the chunk's start, lengths), the records length
    Layout G;
    const size_t g_off = G.put(8ull * k), g_len = G.put(4ull * k), g_poff = G.put(8ull * kq), g_plen = G.put(4ull * kq);
    q.len_at = G.put(8);
    ZC_CUDA(grow(S.in, span + 64));
    ZC_CUDA(grow(S.out, (size_t)k * (B + zc::kRecHdr) + 64));
    ZC_CUDA(grow(S.blk, G.at));
    ZC_CUDA(grow_host(S.h, G.at));
    uint8_t* hb = static_cast<uint8_t*>(S.h.p);
    uint8_t* db = S.blk.as<uint8_t>();
    uint64_t* hpo = reinterpret_cast<uint64_t*>(hb + g_poff);
    uint32_t* hpl = reinterpret_cast<uint32_t*>(hb + g_plen);
    for (uint32_t j = 0; j < kq; ++j) {
      hpo[j] = P.part_off[q0 + j] - lo;
      hpl[j] = P.part_len[q0 + j];
    }
    // upload on the copy stream (this stage's last chunk was harvested, so its buffers are free)
    ZC_CUDA(cudaMemcpyAsync(S.in.p, solid + lo, span, cudaMemcpyHostToDevice, cs));
    ZC_CUDA(cudaMemsetAsync(S.in.as<uint8_t>() + span, 0, 64, cs));
    if (kq) ZC_CUDA(cudaMemcpyAsync(db + g_poff, hb + g_poff, q.len_at - g_poff, cudaMemcpyHostToDevice, cs));
    ZC_CUDA(cudaEventRecord(S.ev_in, cs));
    ZC_CUDA(cudaStreamWaitEvent(st, S.ev_in, 0));
    uint64_t* ioff = reinterpret_cast<uint64_t*>(db + g_off);
    uint32_t* ilen = reinterpret_cast<uint32_t*>(db + g_len);
    plain_blocks(c, span, (uint32_t)B, k, ioff, ilen, st);
    if (int r = encode_device(c, S.in.as<uint8_t>(), ioff, ilen, k, bl, level, X + o_meth + b0,
                              reinterpret_cast<uint32_t*>(X + o_lens) + b0, d_crc + b0, S.out.as<uint8_t>(), S.out.n,
                              reinterpret_cast<uint64_t*>(X + o_offs) + b0, reinterpret_cast<uint64_t*>(db + q.len_at),
                              1, st, reinterpret_cast<const uint64_t*>(X + o_zero)))
      return r;
    launch_piece_crcs(c, S.in.as<uint8_t>(), reinterpret_cast<const uint64_t*>(db + g_poff),
                      reinterpret_cast<const uint32_t*>(db + g_plen), kq, d_pcrc + q0, st);
    ZC_CUDA(cudaEventRecord(S.ev_done, st));
    if (have_prev)
      if (int r = harvest(c->pipe[(it - 1) & 1], prev)) return r;
    prev = q;
    have_prev = true;
  }
  if (have_prev)
    if (int r = harvest(c->pipe[(it - 1) & 1], prev)) return r;
  // the files' CRCs, then the table and the footer
  uint32_t* d_ecrc = reinterpret_cast<uint32_t*>(X + o_ecrc);
  if (ne) ZC_CUDA(cudaMemsetAsync(d_ecrc, 0, 4ull * ne, st));
  launch_combine(c, D, pd, P, d_crc, d_pcrc, nullptr, d_ecrc, st);
  if (int r = check_launch(c, "archive launch")) return r;
  std::vector<uint32_t> ec(ne);
  if (ne) ZC_CUDA(cudaMemcpyAsync(ec.data(), d_ecrc, 4ull * ne, cudaMemcpyDeviceToHost, st));
  ZC_CUDA(cudaStreamSynchronize(st));
  for (size_t f = 0; f < P.entry.size(); ++f)
    for (int b = 0; b < 4; ++b) table[pos[f] + b] = (uint8_t)(ec[P.entry[f]] >> (8 * b));
  for (uint32_t i = 0; i < ne; ++i) es[i].crc = ec[i];
  const uint64_t tl = table.size();
  if (tl + kArchFoot > out_cap - at) return fail(c, ZC_E_ARG, "the output buffer is too small");
  memcpy(out + at, table.data(), tl);
  uint8_t* ft = out + at + tl;
  const uint32_t tcrc = host_crc32(table.data(), tl);
  for (int i = 0; i < 8; ++i) {
    ft[i] = (uint8_t)(at >> (8 * i));
    ft[8 + i] = (uint8_t)(tl >> (8 * i));
  }
  for (int i = 0; i < 4; ++i) ft[16 + i] = (uint8_t)(tcrc >> (8 * i));
  memcpy(ft + 20, "ZEND", 4);
  *out_len = at + tl + kArchFoot;
  return ZC_OK;
}

// Host-pointer extract (out != NULL) or test.  The records go up in chunks of whole blocks through the
// two stages: a chunk's upload and the previous chunk's raw bytes coming down overlap the chunk's decode.
// Block CRCs and the partial file pieces' CRCs are computed while a chunk is resident; the files' CRCs
// are combined on the device at the end.  Checks and messages in the reader's order (src/archive.h:
// 611-634, 655-667): a damaged block, a block CRC, the stream's size, then each file's CRC.
int extract_host(zc_ctx* c, const uint8_t* arch, uint64_t len, uint8_t* out, uint64_t out_cap) {
  std::string why;
  zc_archive_info I{};
  std::vector<zc_entry> es;
  if (parse_table(arch, len, &I, &es, why)) return fail(c, ZC_E_DATA, why);
  if (I.n_blocks >= kPart) return fail(c, ZC_E_DATA, "archive damaged: block count");
  // (the walk stops at the first damaged record, so n_blocks is bounded by the records' space first)
  if (I.n_blocks > (I.table_off - kArchHdr) / zc::kRecHdr) return fail(c, ZC_E_DATA, "archive damaged: block header cut");
  const uint32_t nb = (uint32_t)I.n_blocks, bl = I.block_log;
  std::vector<uint64_t> coff(nb), ooff(nb);
  std::vector<uint32_t> clen(nb), rlen(nb), rcrc(nb);
  std::vector<uint8_t> meth(nb);
  if (walk_blocks(arch, len, I, coff.data(), clen.data(), meth.data(), rlen.data(), rcrc.data(), why))
    return fail(c, ZC_E_DATA, why);
  if (out && out_cap < I.total_raw) return fail(c, ZC_E_ARG, "the output is smaller than the archive's stream");
  uint64_t raw_sum = 0;
  for (uint32_t b = 0; b < nb; ++b) {
    ooff[b] = raw_sum;
    raw_sum += rlen[b];
  }
  const bool sizes_agree = raw_sum == I.total_raw;
  Pieces P;
  if (sizes_agree && !cut_pieces(es.data(), (uint32_t)es.size(), bl, raw_sum, P, why)) return fail(c, ZC_E_DATA, why);
  const uint32_t nq = (uint32_t)P.part_off.size(), ne = (uint32_t)es.size();
  Layout L;
  const PieceDev pd = place_pieces(L, P, false);
  std::vector<uint8_t> h(L.at);
  fill_pieces(h, pd, P);
  Layout W;
  const size_t o_crc = W.put(4ull * nb), o_err = W.put(4ull * nb), o_pcrc = W.put(4ull * nq), o_ecrc = W.put(4ull * ne);
  cudaStream_t st = c->stream, cs = c->cstream;
  ZC_CUDA(grow(c->a_desc, L.at));
  ZC_CUDA(grow(c->a_work, W.at));
  uint8_t* D = c->a_desc.as<uint8_t>();
  uint8_t* X = c->a_work.as<uint8_t>();
  ZC_CUDA(cudaMemcpyAsync(D, h.data(), L.at, cudaMemcpyHostToDevice, st));
  uint32_t* d_crc = reinterpret_cast<uint32_t*>(X + o_crc);
  uint32_t* d_err = reinterpret_cast<uint32_t*>(X + o_err);
  uint32_t* d_pcrc = reinterpret_cast<uint32_t*>(X + o_pcrc);
  const uint32_t per_launch = dec_blocks_per_launch(bl);
  struct Chunk {
    uint32_t b0 = 0, k = 0;
    uint64_t raw_at = 0, raw_total = 0;
  };
  Chunk prev;
  bool have_prev = false;
  const bool copy_out = out && sizes_agree;  // (a stream of the wrong size is refused; nothing is written)
  auto harvest = [&](zc_ctx::Stage& S, const Chunk& q) -> int {
    ZC_CUDA(cudaStreamWaitEvent(cs, S.ev_done, 0));
    if (copy_out && q.raw_total)
      ZC_CUDA(cudaMemcpyAsync(out + q.raw_at, S.out.p, q.raw_total, cudaMemcpyDeviceToHost, cs));
    ZC_CUDA(cudaStreamSynchronize(cs));
    return ZC_OK;
  };
  uint32_t it = 0;
  for (uint32_t b0 = 0; b0 < nb; b0 += prev.k, ++it) {
    zc_ctx::Stage& S = c->pipe[it & 1];
    Chunk q;
    q.b0 = b0;
    q.k = std::min(host_chunk_blocks(bl, per_launch, it), nb - b0);
    const uint32_t k = q.k;
    const uint64_t lo = coff[b0], hi = coff[b0 + k - 1] + clen[b0 + k - 1];
    q.raw_at = ooff[b0];
    q.raw_total = ooff[b0 + k - 1] + rlen[b0 + k - 1] - q.raw_at;
    uint32_t q0 = 0, q1 = 0;
    if (sizes_agree) pieces_in(P, q.raw_at, q.raw_at + q.raw_total, q0, q1);
    const uint32_t kq = q1 - q0;
    // the stage's descriptors: per block its body's offset in the chunk's span, its output offset in
    // the chunk, lengths and method; the chunk's partial pieces (offsets in its output, lengths)
    Layout G;
    const size_t g_coff = G.put(8ull * k), g_ooff = G.put(8ull * k), g_clen = G.put(4ull * k), g_rlen = G.put(4ull * k);
    const size_t g_meth = G.put(k), g_poff = G.put(8ull * kq), g_plen = G.put(4ull * kq);
    ZC_CUDA(grow(S.in, (hi - lo) + 64));
    ZC_CUDA(grow(S.out, q.raw_total + 64));
    ZC_CUDA(grow(S.blk, G.at));
    ZC_CUDA(grow_host(S.h, G.at));
    uint8_t* hb = static_cast<uint8_t*>(S.h.p);
    uint8_t* db = S.blk.as<uint8_t>();
    for (uint32_t j = 0; j < k; ++j) {
      reinterpret_cast<uint64_t*>(hb + g_coff)[j] = coff[b0 + j] - lo;
      reinterpret_cast<uint64_t*>(hb + g_ooff)[j] = ooff[b0 + j] - q.raw_at;
      reinterpret_cast<uint32_t*>(hb + g_clen)[j] = clen[b0 + j];
      reinterpret_cast<uint32_t*>(hb + g_rlen)[j] = rlen[b0 + j];
      hb[g_meth + j] = meth[b0 + j];
    }
    for (uint32_t j = 0; j < kq; ++j) {
      reinterpret_cast<uint64_t*>(hb + g_poff)[j] = P.part_off[q0 + j] - q.raw_at;
      reinterpret_cast<uint32_t*>(hb + g_plen)[j] = P.part_len[q0 + j];
    }
    if (hi > lo) ZC_CUDA(cudaMemcpyAsync(S.in.p, arch + lo, hi - lo, cudaMemcpyHostToDevice, cs));
    ZC_CUDA(cudaMemsetAsync(S.in.as<uint8_t>() + (hi - lo), 0, 64, cs));
    ZC_CUDA(cudaMemcpyAsync(db, hb, G.at, cudaMemcpyHostToDevice, cs));
    ZC_CUDA(cudaEventRecord(S.ev_in, cs));
    ZC_CUDA(cudaStreamWaitEvent(st, S.ev_in, 0));
    if (int r = decode_device(c, S.in.as<uint8_t>(), reinterpret_cast<const uint64_t*>(db + g_coff),
                              reinterpret_cast<const uint32_t*>(db + g_clen), db + g_meth,
                              reinterpret_cast<const uint32_t*>(db + g_rlen), k, bl, S.out.as<uint8_t>(),
                              reinterpret_cast<const uint64_t*>(db + g_ooff), d_crc + b0, d_err + b0, st))
      return r;
    launch_piece_crcs(c, S.out.as<uint8_t>(), reinterpret_cast<const uint64_t*>(db + g_poff),
                      reinterpret_cast<const uint32_t*>(db + g_plen), kq, d_pcrc + q0, st);
    ZC_CUDA(cudaEventRecord(S.ev_done, st));
    if (have_prev)
      if (int r = harvest(c->pipe[(it - 1) & 1], prev)) return r;
    prev = q;
    have_prev = true;
  }
  if (have_prev)
    if (int r = harvest(c->pipe[(it - 1) & 1], prev)) return r;
  uint32_t* d_ecrc = reinterpret_cast<uint32_t*>(X + o_ecrc);
  if (ne) ZC_CUDA(cudaMemsetAsync(d_ecrc, 0, 4ull * ne, st));
  if (sizes_agree) launch_combine(c, D, pd, P, d_crc, d_pcrc, nullptr, d_ecrc, st);
  if (int r = check_launch(c, "archive launch")) return r;
  std::vector<uint32_t> got(nb), err(nb), ecrc(ne);
  if (nb) {
    ZC_CUDA(cudaMemcpyAsync(got.data(), d_crc, 4ull * nb, cudaMemcpyDeviceToHost, st));
    ZC_CUDA(cudaMemcpyAsync(err.data(), d_err, 4ull * nb, cudaMemcpyDeviceToHost, st));
  }
  if (ne) ZC_CUDA(cudaMemcpyAsync(ecrc.data(), d_ecrc, 4ull * ne, cudaMemcpyDeviceToHost, st));
  ZC_CUDA(cudaStreamSynchronize(st));
  char m[512];
  for (uint32_t b = 0; b < nb; ++b) {
    if (err[b]) {
      snprintf(m, sizeof m, "block %u damaged (GPU decoder, code %u)", b, err[b]);
      return fail(c, ZC_E_DATA, m);
    }
    if (got[b] != rcrc[b]) {
      snprintf(m, sizeof m, "block %u does not match its checksum: the archive is damaged", b);
      return fail(c, ZC_E_DATA, m);
    }
  }
  if (!sizes_agree) {
    snprintf(m, sizeof m, "archive damaged: the blocks hold %llu bytes, the table %llu", (unsigned long long)raw_sum,
             (unsigned long long)I.total_raw);
    return fail(c, ZC_E_DATA, m);
  }
  for (uint32_t i = 0; i < ne; ++i) {
    if (es[i].is_dir || !es[i].size || ecrc[i] == es[i].crc) continue;
    return fail(c, ZC_E_DATA, "file " + std::string(es[i].name, es[i].name_len) + " does not match its checksum");
  }
  return ZC_OK;
}

}  // namespace

extern "C" {

uint64_t zc_archive_bound(const zc_entry* entries, uint32_t n_entries, uint32_t block_log) {
  std::string why;
  uint64_t n = 0;
  if (bad_block_log(block_log) || !check_entries(entries, n_entries, &n, why)) return 0;
  const uint64_t nb = (n + (1ull << block_log) - 1) >> block_log;
  return kArchHdr + nb * zc::kRecHdr + n + table_bytes(entries, n_entries) + kArchFoot;
}

int zc_archive_write_device(zc_ctx* c, const uint8_t* d_solid, uint32_t block_log, int level, const zc_entry* entries,
                            uint32_t n_entries, uint8_t* d_out, uint64_t out_cap, uint64_t* d_len,
                            uint32_t* d_entry_crcs, void* stream) {
  if (!c) return ZC_E_ARG;
  ZC_GATE(c);
  ZC_CUDA(cudaSetDevice(c->device));
  return write_device(c, d_solid, block_log, level, entries, n_entries, d_out, out_cap, d_len, d_entry_crcs,
                      static_cast<cudaStream_t>(stream));
}

int zc_archive_write_range(zc_ctx* c, const uint8_t* d_range, uint64_t range_off, uint64_t range_len,
                           uint32_t block_log, int level, const zc_entry* entries, uint32_t n_entries, uint64_t rec_base,
                           uint8_t* d_out, uint64_t out_cap, uint64_t* d_len, uint32_t* d_piece_crcs, void* stream) {
  if (!c) return ZC_E_ARG;
  ZC_GATE(c);
  ZC_CUDA(cudaSetDevice(c->device));
  return write_range(c, d_range, range_off, range_len, block_log, level, entries, n_entries, rec_base, d_out, out_cap,
                     d_len, d_piece_crcs, static_cast<cudaStream_t>(stream));
}

int zc_archive_write(zc_ctx* c, const uint8_t* solid, uint32_t block_log, int level, zc_entry* entries,
                     uint32_t n_entries, uint8_t* out, uint64_t out_cap, uint64_t* out_len) {
  if (!c || !out_len) return ZC_E_ARG;
  ZC_GATE(c);
  ZC_CUDA(cudaSetDevice(c->device));
  return write_host(c, solid, block_log, level, entries, n_entries, out, out_cap, out_len);
}

int zc_archive_read_table(const uint8_t* arch, uint64_t len, zc_archive_info* info, zc_entry* entries, uint32_t cap,
                          char* msg, size_t msg_cap) {
  if (!info) return ZC_E_ARG;
  std::vector<zc_entry> es;
  std::string why;
  if (parse_table(arch, len, info, &es, why)) return msg_fail(msg, msg_cap, why);
  if (entries)
    for (uint32_t i = 0; i < cap && i < es.size(); ++i) entries[i] = es[i];
  if (msg && msg_cap) msg[0] = 0;
  return ZC_OK;
}

int zc_archive_blocks(const uint8_t* arch, uint64_t len, const zc_archive_info* info, uint64_t* offs,
                      uint32_t* comp_lens, uint8_t* methods, uint32_t* raw_lens, uint32_t* crcs, char* msg,
                      size_t msg_cap) {
  if (!arch || !info || (info->n_blocks && (!offs || !comp_lens || !methods || !raw_lens))) return ZC_E_ARG;
  if (info->table_off > len) return msg_fail(msg, msg_cap, "archive damaged: table position");
  std::string why;
  if (walk_blocks(arch, len, *info, offs, comp_lens, methods, raw_lens, crcs, why)) return msg_fail(msg, msg_cap, why);
  if (msg && msg_cap) msg[0] = 0;
  return ZC_OK;
}

int zc_archive_extract(zc_ctx* c, const uint8_t* arch, uint64_t len, uint8_t* out, uint64_t out_cap) {
  if (!c) return ZC_E_ARG;
  ZC_GATE(c);
  ZC_CUDA(cudaSetDevice(c->device));
  return extract_host(c, arch, len, out, out_cap);
}

}  // extern "C"
