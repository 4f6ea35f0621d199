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

// k_crc_pieces + k_file_crcs over a solid stream on the device
void launch_file_crcs(zc_ctx* c, const uint8_t* d_solid, const uint8_t* D, const PieceDev& d, const Pieces& P,
                      const uint32_t* blk_crc, uint32_t* part_crc, uint8_t* table, uint32_t* entry_crc, cudaStream_t st) {
  if (!P.part_off.empty()) {
    zc::CrcArgs C{};
    C.base = d_solid;
    C.offs = reinterpret_cast<const uint64_t*>(D + d.part_off);
    C.lens = reinterpret_cast<const uint32_t*>(D + d.part_len);
    C.nb = (uint32_t)P.part_off.size();
    C.crc = part_crc;
    C.tables = c->d_crct;
    zc::launch_crc(C, st, c->stages, "k_crc_pieces");
  }
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
  memcpy(hd.b, "ZERO", 4);
  hd.b[4] = 2;
  hd.b[5] = (uint8_t)bl;
  for (int i = 0; i < 8; ++i) {
    hd.b[8 + i] = (uint8_t)(n >> (8 * i));
    hd.b[16 + i] = (uint8_t)(nb64 >> (8 * i));
  }
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
  ZC_CUDA(cudaSetDevice(c->device));
  return write_device(c, d_solid, block_log, level, entries, n_entries, d_out, out_cap, d_len, d_entry_crcs,
                      static_cast<cudaStream_t>(stream));
}

int zc_archive_write(zc_ctx* c, const uint8_t* solid, uint32_t block_log, int level, zc_entry* entries,
                     uint32_t n_entries, uint8_t* out, uint64_t out_cap, uint64_t* out_len) {
  if (!c || !out_len) return ZC_E_ARG;
  ZC_CUDA(cudaSetDevice(c->device));
  std::string why;
  uint64_t n = 0;
  if (!check_entries(entries, n_entries, &n, why)) return fail(c, ZC_E_ARG, why);
  if (n && !solid) return fail(c, ZC_E_ARG, "no input");
  const uint64_t bound = zc_archive_bound(entries, n_entries, block_log);
  if (!bound) return fail(c, ZC_E_ARG, "block size must be 2^16 .. 2^20 bytes");
  cudaStream_t st = c->stream;
  ZC_CUDA(grow(c->a_in, n + 64));
  const size_t ob = (bound + 255) & ~(size_t)255;
  ZC_CUDA(grow(c->a_out, ob + 256 + 4ull * n_entries));
  uint8_t* d_in = c->a_in.as<uint8_t>();
  uint8_t* d_out = c->a_out.as<uint8_t>();
  uint64_t* d_len = reinterpret_cast<uint64_t*>(d_out + ob);
  uint32_t* d_ecrc = reinterpret_cast<uint32_t*>(d_out + ob + 256);
  if (n) ZC_CUDA(cudaMemcpyAsync(d_in, solid, n, cudaMemcpyHostToDevice, st));
  ZC_CUDA(cudaMemsetAsync(d_in + n, 0, 64, st));
  if (int r = write_device(c, d_in, block_log, level, entries, n_entries, d_out, bound, d_len, d_ecrc, st)) return r;
  uint64_t len = 0;
  ZC_CUDA(cudaMemcpyAsync(&len, d_len, 8, cudaMemcpyDeviceToHost, st));
  ZC_CUDA(cudaStreamSynchronize(st));
  if (!len) return fail(c, ZC_E_DEVICE, "the archive did not fit its bound");
  *out_len = len;
  if (len > out_cap) {
    char m[128];
    snprintf(m, sizeof m, "the output buffer is too small: the archive has %llu bytes", (unsigned long long)len);
    return fail(c, ZC_E_ARG, m);
  }
  if (!out) return fail(c, ZC_E_ARG, "no output");
  std::vector<uint32_t> ec(n_entries);
  ZC_CUDA(cudaMemcpyAsync(out, d_out, len, cudaMemcpyDeviceToHost, st));
  if (n_entries) ZC_CUDA(cudaMemcpyAsync(ec.data(), d_ecrc, 4ull * n_entries, cudaMemcpyDeviceToHost, st));
  ZC_CUDA(cudaStreamSynchronize(st));
  for (uint32_t i = 0; i < n_entries; ++i) entries[i].crc = ec[i];
  return ZC_OK;
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
  ZC_CUDA(cudaSetDevice(c->device));
  std::string why;
  zc_archive_info I{};
  std::vector<zc_entry> es;
  if (parse_table(arch, len, &I, &es, why)) return fail(c, ZC_E_DATA, why);
  if (I.n_blocks >= kPart) return fail(c, ZC_E_DATA, "archive damaged: block count");
  const uint32_t nb = (uint32_t)I.n_blocks, bl = I.block_log;
  // the walk stops at the first damaged record, so n_blocks is bounded by the archive's length first
  if (I.n_blocks > (I.table_off - kArchHdr) / zc::kRecHdr) return fail(c, ZC_E_DATA, "archive damaged: block header cut");
  std::vector<uint64_t> coff(nb), ooff(nb);
  std::vector<uint32_t> clen(nb), rlen(nb), rcrc(nb);
  std::vector<uint8_t> meth(nb);
  if (walk_blocks(arch, len, I, coff.data(), clen.data(), meth.data(), rlen.data(), rcrc.data(), why))
    return fail(c, ZC_E_DATA, why);
  if (out && out_cap < I.total_raw) return fail(c, ZC_E_ARG, "the output is smaller than the archive's stream");
  uint64_t raw_sum = 0;
  for (uint32_t b = 0; b < nb; ++b) {
    coff[b] -= kArchHdr;
    ooff[b] = raw_sum;
    raw_sum += rlen[b];
  }
  const bool sizes_agree = raw_sum == I.total_raw;
  Pieces P;
  if (sizes_agree && !cut_pieces(es.data(), (uint32_t)es.size(), bl, raw_sum, P, why)) return fail(c, ZC_E_DATA, why);
  // descriptors: per block, then the pieces
  Layout L;
  const size_t o_coff = L.put(8ull * nb), o_ooff = L.put(8ull * nb), o_clen = L.put(4ull * nb), o_rlen = L.put(4ull * nb);
  const size_t o_meth = L.put(nb);
  const PieceDev pd = place_pieces(L, P, false);
  std::vector<uint8_t> h(L.at);
  put_section(h, o_coff, coff);
  put_section(h, o_ooff, ooff);
  put_section(h, o_clen, clen);
  put_section(h, o_rlen, rlen);
  put_section(h, o_meth, meth);
  fill_pieces(h, pd, P);
  Layout W;
  const size_t o_crc = W.put(4ull * nb), o_err = W.put(4ull * nb), o_pcrc = W.put(4 * P.part_off.size());
  const size_t o_ecrc = W.put(4 * es.size());
  const uint64_t span = I.table_off - kArchHdr;
  cudaStream_t st = c->stream;
  ZC_CUDA(grow(c->a_in, span + 64));
  ZC_CUDA(grow(c->a_out, raw_sum + 64));
  ZC_CUDA(grow(c->a_desc, L.at));
  ZC_CUDA(grow(c->a_work, W.at));
  uint8_t* d_in = c->a_in.as<uint8_t>();
  uint8_t* d_solid = c->a_out.as<uint8_t>();
  uint8_t* D = c->a_desc.as<uint8_t>();
  uint8_t* X = c->a_work.as<uint8_t>();
  if (span) ZC_CUDA(cudaMemcpyAsync(d_in, arch + kArchHdr, span, cudaMemcpyHostToDevice, st));
  ZC_CUDA(cudaMemsetAsync(d_in + span, 0, 64, st));
  ZC_CUDA(cudaMemcpyAsync(D, h.data(), L.at, cudaMemcpyHostToDevice, st));
  uint32_t* d_crc = reinterpret_cast<uint32_t*>(X + o_crc);
  uint32_t* d_err = reinterpret_cast<uint32_t*>(X + o_err);
  const uint32_t per = dec_blocks_per_launch(bl);
  for (uint32_t b0 = 0; b0 < nb; b0 += per) {
    const uint32_t k = std::min(per, nb - b0);
    if (int r = decode_device(c, d_in, reinterpret_cast<const uint64_t*>(D + o_coff) + b0,
                              reinterpret_cast<const uint32_t*>(D + o_clen) + b0, D + o_meth + b0,
                              reinterpret_cast<const uint32_t*>(D + o_rlen) + b0, k, bl, d_solid,
                              reinterpret_cast<const uint64_t*>(D + o_ooff) + b0, d_crc + b0, d_err + b0, st))
      return r;
  }
  uint32_t* d_ecrc = reinterpret_cast<uint32_t*>(X + o_ecrc);
  if (!es.empty()) ZC_CUDA(cudaMemsetAsync(d_ecrc, 0, 4 * es.size(), st));
  if (sizes_agree) launch_file_crcs(c, d_solid, D, pd, P, d_crc, reinterpret_cast<uint32_t*>(X + o_pcrc), nullptr, d_ecrc, st);
  if (int r = check_launch(c, "archive launch")) return r;
  std::vector<uint32_t> got(nb), err(nb), ecrc(es.size());
  if (nb) {
    ZC_CUDA(cudaMemcpyAsync(got.data(), d_crc, 4ull * nb, cudaMemcpyDeviceToHost, st));
    ZC_CUDA(cudaMemcpyAsync(err.data(), d_err, 4ull * nb, cudaMemcpyDeviceToHost, st));
  }
  if (!es.empty()) ZC_CUDA(cudaMemcpyAsync(ecrc.data(), d_ecrc, 4 * es.size(), cudaMemcpyDeviceToHost, st));
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
  for (size_t i = 0; i < es.size(); ++i) {
    if (es[i].is_dir || !es[i].size || ecrc[i] == es[i].crc) continue;
    return fail(c, ZC_E_DATA, "file " + std::string(es[i].name, es[i].name_len) + " does not match its checksum");
  }
  if (out && raw_sum) {
    ZC_CUDA(cudaMemcpyAsync(out, d_solid, raw_sum, cudaMemcpyDeviceToHost, st));
    ZC_CUDA(cudaStreamSynchronize(st));
  }
  return ZC_OK;
}

}  // extern "C"
