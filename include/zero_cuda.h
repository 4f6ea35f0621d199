/* zero_cuda.h -- C ABI of the B200 (sm_100a) ZB2 block codec.
 *
 * A drop-in for the GPU codec behind `zero c / x / t / bench`: it replaces the reference's Level Zero
 * layer (src/ze_min.h, src/gpu.h) and its GPU orchestration (src/gpu_codec.h) with CUDA kernels behind
 * plain C entry points.  The reference's callers reach the GPU codec through the virtual interface
 * zero::Codec (src/archive.h:56-69); each entry point below names the method it backs.  A C++ adapter
 * implementing zero::Codec over these calls is in include/zero_cuda_codec.hpp.
 *
 * Format: the .zero block format is unchanged (ZB2 payloads of src/codec2.h, rANS streams of
 * src/codec.h, CRC-32 of src/crc32.h).  At the same level the encoder writes exactly the bytes the
 * reference CPU codec writes (same parse: hash chains of depth 8 / 32 / 256 for levels 1 / 2-8 / 9,
 * src/main.cpp:45, 54; one lazy step; matches up to 4096 bytes).
 *
 * Errors (the reference throws; here every call returns a status):
 *   ZC_OK        success
 *   ZC_E_DATA    damaged input or an impossible result (the reference's zb::Error: retry on the CPU,
 *                which reports what is wrong -- src/safe_codec.h:36-49)
 *   ZC_E_DEVICE  the GPU failed (the reference's gpu::Error: fall back to the CPU for good)
 *   ZC_E_NOMEM   device memory could not be had
 *   ZC_E_ARG     a bad argument (block size outside 16..20, a block longer than the block size, ...)
 * zc_last_error(ctx) gives the message of the last failure on that context.
 *
 * Threading: a context is used by one host thread at a time (the reference calls its codec from one
 * thread, src/archive.h:381-413, 599-633).  Separate contexts may run on separate threads.
 */
#ifndef ZERO_CUDA_H
#define ZERO_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ZC_OK = 0, ZC_E_DATA = 1, ZC_E_DEVICE = 2, ZC_E_NOMEM = 3, ZC_E_ARG = 4 };

/* block methods, as in the block record of the archive (src/archive.h:395-398) */
enum { ZC_METHOD_STORED = 0, ZC_METHOD_ZB2 = 1 };

typedef struct zc_ctx zc_ctx;

/* Opens device `device` (replaces GpuCodec::open, src/gpu_codec.h:75-86, and gpu::Device::open,
 * src/gpu.h:140-188).  No kernel compilation at run time: the kernels are built ahead for sm_100a. */
int zc_open(zc_ctx **ctx, int device);
void zc_close(zc_ctx *ctx);

/* The message of the last error on this context ("" when none). */
const char *zc_last_error(const zc_ctx *ctx);

/* The codec's name for the user (zero::Codec::name, src/archive.h:58). */
const char *zc_name(const zc_ctx *ctx);

/* Block size and level before a job (zero::Codec::prepare, src/archive.h:68, and the level choice of
 * src/gpu_codec.h:63-70).  block_log 16..20, level 1..9.  Optional: every call below takes both. */
int zc_prepare(zc_ctx *ctx, uint32_t block_log, int level);

/* Bytes of input one compress / decompress call should hold (zero::Codec::batch_bytes and
 * batch_bytes_decode, src/archive.h:65-66). */
size_t zc_batch_bytes(const zc_ctx *ctx, uint32_t block_log);
size_t zc_batch_bytes_decode(const zc_ctx *ctx, uint32_t block_log);

/* Compresses n host bytes cut into blocks of 2^block_log (the last may be shorter): zero::Codec::compress
 * (src/archive.h:60; src/gpu_codec.h:153-229).  Per block b (nb = ceil(n / 2^block_log)):
 *   methods[b]    ZC_METHOD_ZB2, or ZC_METHOD_STORED when the payload would not be smaller than the block
 *   comp_lens[b]  the payload length (for a stored block: its raw length; nothing is written for it)
 *   crcs[b]       CRC-32 of the block's raw bytes (the record's checksum, src/archive.h:376)
 *   pay_offs[b]   where block b's payload starts in `payloads` (ZB2 payloads are packed back to back)
 * payloads must hold payload_cap bytes; n bytes always suffice.  Any of crcs / pay_offs may be NULL. */
int zc_compress(zc_ctx *ctx, const uint8_t *in, size_t n, uint32_t block_log, int level, uint8_t *methods,
                uint32_t *comp_lens, uint32_t *crcs, uint8_t *payloads, size_t payload_cap, uint64_t *pay_offs);

/* The same for nb blocks of uneven sizes from many files, in one launch per stage: block b is
 * in_lens[b] (<= 2^block_log) bytes at in + in_offs[b]. */
int zc_compress_batch(zc_ctx *ctx, const uint8_t *in, const uint64_t *in_offs, const uint32_t *in_lens, uint32_t nb,
                      uint32_t block_log, int level, uint8_t *methods, uint32_t *comp_lens, uint32_t *crcs,
                      uint8_t *payloads, size_t payload_cap, uint64_t *pay_offs);

/* Decompresses nb blocks (zero::Codec::decompress, src/archive.h:63; src/gpu_codec.h:253-315).
 * Block b is comp_lens[b] bytes at comp + comp_offs[b] with method methods[b] and raw length raw_lens[b].
 * Writes the raw bytes of all blocks back to back into out (sum of raw_lens bytes).
 * crcs_out[b] (may be NULL) gets the CRC-32 of block b's output; block_err[b] (may be NULL) a nonzero
 * code for a damaged block.  Returns ZC_E_DATA when any block is damaged. */
int zc_decompress(zc_ctx *ctx, const uint8_t *comp, const uint64_t *comp_offs, const uint32_t *comp_lens,
                  const uint8_t *methods, const uint32_t *raw_lens, uint32_t nb, uint8_t *out, uint32_t *crcs_out,
                  uint32_t *block_err);

/* ---- device-resident forms: every pointer is device memory, work is queued on `stream` (a
 * cudaStream_t; NULL for the legacy default stream) and the call returns once it is queued.  For
 * callers that keep data on the GPU, and for measuring the kernels without host copies.
 * d_in must be 16-byte aligned with at least 64 readable bytes after the last block (the match finder
 * reads whole aligned words and 16-byte groups, as the reference's kernels read words past a block:
 * kernels/zero.cl:30-31).
 *
 * zc_compress_device: nb blocks at d_in + d_in_offs[b], d_in_lens[b] bytes each.  Writes d_methods,
 * d_comp_lens, d_crcs (may be NULL) and the payloads packed into d_out (out_cap bytes) at d_out_offs[b];
 * a stored block's raw bytes are copied into d_out as well, so d_out holds every record body in order.
 * *d_total (device u64) gets the bytes written to d_out. */
int zc_compress_device(zc_ctx *ctx, const uint8_t *d_in, const uint64_t *d_in_offs, const uint32_t *d_in_lens,
                       uint32_t nb, uint32_t block_log, int level, uint8_t *d_methods, uint32_t *d_comp_lens,
                       uint32_t *d_crcs, uint8_t *d_out, size_t out_cap, uint64_t *d_out_offs, uint64_t *d_total,
                       void *stream);

/* zc_decompress_device: block b is d_comp_lens[b] bytes at d_comp + d_comp_offs[b]; its raw bytes go to
 * d_out + d_out_offs[b].  d_crcs (may be NULL) gets each output's CRC-32, d_err each block's status.
 * block_log bounds the raw lengths (a block longer than 2^block_log is damaged). */
int zc_decompress_device(zc_ctx *ctx, const uint8_t *d_comp, const uint64_t *d_comp_offs, const uint32_t *d_comp_lens,
                         const uint8_t *d_methods, const uint32_t *d_raw_lens, uint32_t nb, uint32_t block_log,
                         uint8_t *d_out, const uint64_t *d_out_offs, uint32_t *d_crcs, uint32_t *d_err, void *stream);

/* Decompression that allocates no device memory.  No counterpart in the reference: it exists for callers
 * that cannot call cudaMalloc -- a plugin in a host process that budgets all device memory itself (an
 * admission-controlled server, a framework that owns its allocator), or a latency-bound path where
 * cudaMalloc / cudaFree would synchronise the device and stall other streams.  Arguments and results are
 * those of zc_decompress_device (all device pointers, work queued on `stream`), without a context; it runs
 * the same decoder kernels.  Scratch is one fixed __device__ array of ZC_NOALLOC_SCRATCH_BYTES inside the
 * library, held by every GPU that loads the library until the process exits.  A call of nb blocks of B =
 * 2^b bytes needs 256 + nb*B + 3*nb*(B/4 + 16) + nb*(B/5 + 64) + 76*nb + 16*nb*(B/4 + 16) bytes of it
 * (each of those nine parts rounded up to a multiple of 256): at most 42 blocks of 64 KiB, 21 of 128 KiB,
 * 10 of 256 KiB, 5 of 512 KiB or 2 of 1 MiB per call; more returns ZC_E_ARG and touches nothing.
 * The first call on a device sets that device up: with the device current it looks up the array's device
 * address (and again whenever the device's context has changed, as after cudaDeviceReset); make that
 * first call before any stream capture.  Every call on a device shares the one scratch array, so calls
 * whose work overlaps on the GPU race: keep them on one stream, or order them.  d_err is cleared by the
 * call itself, and so is the one scratch word that must start at zero. */
#define ZC_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)
int zc_decompress_noalloc(const uint8_t *d_comp, const uint64_t *d_comp_offs, const uint32_t *d_comp_lens,
                          const uint8_t *d_methods, const uint32_t *d_raw_lens, uint32_t nb, uint32_t block_log,
                          uint8_t *d_out, const uint64_t *d_out_offs, uint32_t *d_crcs, uint32_t *d_err, void *stream);

/* CUDA graphs for the device-resident forms (no reference counterpart: the reference's Level Zero command
 * list replays nothing).  With on != 0, the first zc_compress_device / zc_decompress_device call with a
 * given set of arguments and a non-NULL stream captures its launches into a graph; later calls with the
 * same arguments replay it (one launch).  A batch of fixed capacity padded with zero-length blocks keeps
 * its arguments, so one graph serves every batch.  Graphs are dropped when the context's scratch grows
 * and when turned off. */
int zc_set_graphs(zc_ctx *ctx, int on);

/* Sizes the context's device scratch now for device calls of up to nb blocks of 2^block_log bytes, in both
 * directions (no reference counterpart).  Scratch is kept by capacity, so later calls that fit, of any
 * block size, allocate nothing and keep their captured graphs. */
int zc_reserve(zc_ctx *ctx, uint32_t block_log, uint32_t nb);

/* ---- launch shapes and the autotuner (no reference counterpart: the reference's kernels have fixed
 * work-group sizes, kernels/zero.cl).  A shape is kept per (block_log, level class: level 1, 2..8, 9)
 * and never changes a result byte, only speed:
 *   fill_ring_log   decoder fill: each warp keeps its last 2^fill_ring_log output bytes in shared memory
 *                   (11..15), so a match nearer than that reads shared instead of global memory
 *   fill_warps      decoder fill: blocks (warps) per CTA, 1, 2, 4 or 8; fill_warps * (2^fill_ring_log +
 *                   1408 * fill_words) bytes of shared memory per CTA, at most 227 KiB
 *   match_cap       encoder match pass: bytes compared per candidate before the match is left to the
 *                   parse to finish, 8..32
 *   match_tile      encoder match pass: sorted positions per CTA of 256 threads (256, 512 or 1024)
 *   fill_words      decoder fill: output words each lane fills per round (1, 2 or 4: rounds of 128,
 *                   256 or 512 bytes, whose loads are in flight together)
 *   match_dense     encoder match pass: a tile with at least this many positions that their nearest
 *                   candidate does not decide scans a lane per position, a tile with fewer a 16-lane group
 *                   per position, a candidate a lane (0..1025; 1025: always groups, except at level 1)
 *   match_defer     encoder match pass: a position whose nearest candidate's match also covers the
 *                   match_defer bytes before it lies inside a longer match and is left to the parse to
 *                   finish only if it lands there (0..4; 0: never; 3 by default: 2 is faster on data
 *                   with long matches, 3-4 on text-like data whose parse lands on such positions more)
 * The decoder uses the shape of the level last given to zc_prepare (5 by default).  zc_autotune times
 * the candidates on a host sample (its whole blocks, up to one encoder launch) and keeps the fastest for
 * (block_log, level); it allocates its own device buffers for the duration of the call. */
typedef struct zc_shape {
  uint32_t fill_ring_log, fill_warps, match_cap, match_tile, fill_words, match_dense, match_defer;
} zc_shape;
int zc_get_shape(const zc_ctx *ctx, uint32_t block_log, int level, zc_shape *out);
int zc_set_shape(zc_ctx *ctx, uint32_t block_log, int level, const zc_shape *shape);
int zc_autotune(zc_ctx *ctx, const uint8_t *sample, size_t n, uint32_t block_log, int level, zc_shape *chosen);

/* ---- serving: a request loop with continuous batching (no reference counterpart; the reference runs
 * one archive job at a time).  Jobs arrive from any thread; a worker thread admits them in arrival order
 * while their device memory fits in the arena (allocated at open: budget_bytes, or less when the device has
 * less free memory beside the server's own scratch, 1 GiB kept free), keeps their bytes and
 * results on the device, and each tick launches one batch of blocks taken from every admitted job of one
 * kind, block size and level, so jobs that arrive while others run share the launches.  The batches
 * have a fixed capacity (padded with empty blocks) and run as CUDA graphs.
 *
 * A job:
 *   ZC_JOB_COMPRESS  in: in_len raw bytes, cut into blocks of 2^block_log, coded at `level`.  Results per
 *                    block: out_methods, out_lens (payload or raw length), out_crcs, and the ZB2 payloads
 *                    packed into out (out_cap bytes) at out_offs (stored blocks write nothing).
 *   ZC_JOB_EXTRACT   in: nb record bodies back to back (comp_lens[b] bytes each, methods[b],
 *                    raw_lens[b]), as in zc_decompress.  Results: the raw bytes in out, out_crcs.
 *   ZC_JOB_TEST      as EXTRACT, without returning the bytes: out_crcs, and a damaged status when a block
 *                    is damaged or its CRC differs from crcs_expected[b] (src/archive.h:747-785).
 * The caller keeps every buffer of a job alive until zc_serve_wait returns for it. */
enum { ZC_JOB_COMPRESS = 0, ZC_JOB_EXTRACT = 1, ZC_JOB_TEST = 2 };
typedef struct {
  int kind;
  uint32_t block_log;
  int level;
  const uint8_t *in;
  size_t in_len;
  uint32_t nb;                     /* EXTRACT / TEST */
  const uint32_t *comp_lens;       /* EXTRACT / TEST */
  const uint8_t *methods;          /* EXTRACT / TEST */
  const uint32_t *raw_lens;        /* EXTRACT / TEST */
  const uint32_t *crcs_expected;   /* TEST */
  uint8_t *out;                    /* COMPRESS: payloads; EXTRACT: raw bytes */
  size_t out_cap;
  uint8_t *out_methods;            /* COMPRESS */
  uint32_t *out_lens;              /* COMPRESS */
  uint64_t *out_offs;              /* COMPRESS */
  uint32_t *out_crcs;              /* all kinds (may be NULL) */
} zc_job;

typedef struct zc_server zc_server;

/* Opens a server on `device`.  The codec's scratch for the largest batch of every block size is sized
 * first; then the arena for the admitted jobs' data: budget_bytes, capped by the device's free memory at
 * that point less 1 GiB (ZC_E_NOMEM below 1 MiB).  max_batch_bytes bounds one tick's input (0: the codec's
 * default). */
int zc_serve_open(zc_server **srv, int device, uint64_t budget_bytes, uint64_t max_batch_bytes);
/* Waits for every submitted job, then stops the worker and frees the device memory. */
void zc_serve_close(zc_server *srv);
/* Queues a job; *id identifies it.  ZC_E_ARG when it could never fit the budget.  The job's buffers must
 * stay valid until zc_serve_wait returns.  Page-locked buffers are faster: the input is uploaded without
 * staging, and an extract job's page-locked `out` receives its bytes by DMA, with no host copy. */
int zc_serve_submit(zc_server *srv, const zc_job *job, uint64_t *id);
/* Seconds accumulated since open: the GPU time of the batches' kernels (CUDA events around each batch's
 * graph), the worker's waits for batches in flight, its hand-out of results to jobs, and the uploader's
 * time in job uploads.  GPU time over wall time is the device's busy fraction. */
int zc_serve_times(zc_server *srv, double *gpu_s, double *wait_s, double *handout_s, double *upload_s);
/* Waits for job `id`; returns its status (ZC_OK, ZC_E_DATA for a damaged block, ...) and, when
 * latency_s is not NULL, the seconds from its submission to its completion. */
int zc_serve_wait(zc_server *srv, uint64_t id, double *latency_s);
/* Counters: jobs done, bytes (raw) processed, ticks, and device bytes in use right now. */
int zc_serve_stats(zc_server *srv, uint64_t *jobs_done, uint64_t *raw_bytes, uint64_t *ticks, uint64_t *arena_used);

/* CRC-32 of host bytes on the GPU (crc32::of, src/crc32.h:51), and CRC combination on the host
 * (crc32::combine, src/crc32.h:60-66): the CRC of A followed by B. */
int zc_crc32(zc_ctx *ctx, const uint8_t *data, size_t n, uint32_t *crc);
uint32_t zc_crc32_combine(uint32_t crc_a, uint32_t crc_b, uint64_t len_b);

/* ---- whole archives: the .zero container around the blocks, assembled on the GPU.
 * Layout (src/archive.h:334-441 writes it, 451-495 reads its table):
 *   header   "ZERO", u8 version 2, u8 block_log, u16 0, u64 total raw bytes, u64 blocks
 *   records  per block: u32 raw_len, u32 comp_len, u8 method, 3 zero bytes, u32 CRC-32 of the raw block,
 *            then comp_len bytes (the ZB2 payload, or the raw bytes when stored)
 *   table    u32 entries; per entry u8 type (1 = folder), 3 zero bytes, u32 name length, the name,
 *            u64 size, u64 mtime, u32 attributes, u32 CRC-32 of the file's bytes
 *   footer   u64 table offset, u64 table length, u32 CRC-32 of the table, "ZEND"
 * The files' bytes follow one another in entry order as one solid stream cut into blocks of
 * 2^block_log (only the last block is shorter), so a file may straddle blocks. */
typedef struct {
  const char *name;   /* the entry's '/'-separated relative name: name_len bytes, not NUL-terminated */
  uint32_t name_len;
  uint32_t is_dir;    /* 1: a folder (no bytes in the stream; its size must be 0) */
  uint64_t size;      /* the file's bytes in the solid stream */
  int64_t mtime;
  uint32_t attr;
  uint32_t crc;       /* CRC-32 of the file's bytes (0 for folders and empty files) */
} zc_entry;

typedef struct {
  uint32_t block_log;
  uint32_t n_entries;
  uint64_t total_raw;   /* bytes of the solid stream (the sum of the files' sizes) */
  uint64_t n_blocks;
  uint64_t table_off;   /* where the entry table starts: the records lie in [24, table_off) */
  uint64_t table_len;
} zc_archive_info;

/* The largest archive that zc_archive_write can produce for these entries (every block stored). */
uint64_t zc_archive_bound(const zc_entry *entries, uint32_t n_entries, uint32_t block_log);

/* Writes a whole archive of the solid stream d_solid (the files' bytes in entry order, sum of the sizes
 * bytes; 16-byte aligned with 64 readable bytes after the end, as zc_compress_device's input) into
 * d_out (out_cap >= zc_archive_bound bytes), all on the GPU: the records are placed by a device scan,
 * the files' CRCs (crc32 over each file's span, across block boundaries) are computed on the device and
 * written into the table, whose CRC and the footer follow.  *d_len (device u64) gets the archive's
 * length; d_entry_crcs (device, n_entries; may be NULL) each entry's CRC.  Work is queued on `stream`;
 * the call returns once it is queued.  At the same level, the bytes equal those compress_archive
 * (src/archive.h:334-441) writes with the reference CPU codec for the same entries. */
int zc_archive_write_device(zc_ctx *ctx, const uint8_t *d_solid, uint32_t block_log, int level,
                            const zc_entry *entries, uint32_t n_entries, uint8_t *d_out, uint64_t out_cap,
                            uint64_t *d_len, uint32_t *d_entry_crcs, void *stream);

/* One rank's share of an archive written by several GPUs, one process each (no reference counterpart: the
 * reference writes an archive from one process; the layout is compress_archive's, src/archive.h:389-403).
 * d_range holds bytes [range_off, range_off + range_len) of the solid stream (device memory, 16-byte aligned,
 * 64 readable bytes after its end); range_off is a multiple of 2^block_log, and so is the range's end unless
 * it is the stream's end.  Writes the range's block records, exactly as zc_archive_write_device writes those
 * blocks, into d_out from offset rec_base on (records only: no header, entry table or footer);
 * out_cap - rec_base must hold 16 + 2^block_log bytes per block.  *d_len (device u64) gets rec_base plus the
 * records' bytes; d_piece_crcs (device, n_entries; may be NULL) gets each entry's CRC-32 over its bytes
 * inside the range (0 when it has none; the piece's length follows from the entries' sizes).  Combining
 * the ranks' pieces in order with zc_crc32_combine gives each file's CRC.  Work is queued on `stream`. */
int zc_archive_write_range(zc_ctx *ctx, const uint8_t *d_range, uint64_t range_off, uint64_t range_len,
                           uint32_t block_log, int level, const zc_entry *entries, uint32_t n_entries,
                           uint64_t rec_base, uint8_t *d_out, uint64_t out_cap, uint64_t *d_len,
                           uint32_t *d_piece_crcs, void *stream);

/* The same from host memory into host memory (synchronous): solid holds the files' bytes in entry order;
 * *out_len gets the archive's length and entries[i].crc each entry's CRC.  The stream goes through the GPU
 * in chunks (128 MiB, then 512 MiB): a chunk's upload and the previous chunk's records coming down
 * overlap the chunk's kernels.  out_cap = zc_archive_bound is always enough. */
int zc_archive_write(zc_ctx *ctx, const uint8_t *solid, uint32_t block_log, int level, zc_entry *entries,
                     uint32_t n_entries, uint8_t *out, uint64_t out_cap, uint64_t *out_len);

/* Reads the header, footer and entry table of an archive held in host memory, arch[0 .. len), with the
 * checks of read_info (src/archive.h:451-495): the magic, version 2, the block size, the footer, the
 * table's position and CRC, every entry inside the table, and the files' sizes summing to the header's
 * total.  info gets the layout; entries (may be NULL) the first `cap` entries, their names pointing into
 * arch.  Host-only: needs no GPU and no context.  ZC_E_DATA on a damaged archive, the reason in msg
 * (msg_cap bytes, NUL-terminated; may be NULL). */
int zc_archive_read_table(const uint8_t *arch, uint64_t len, zc_archive_info *info, zc_entry *entries,
                          uint32_t cap, char *msg, size_t msg_cap);

/* Walks the block records of an archive in host memory (src/archive.h:566-586) with the same checks:
 * a raw length within the block size, a stored block's lengths equal, a known method, no body past the
 * table.  Per block b: offs[b] where its body starts in arch, comp_lens, methods, raw_lens and the
 * record's CRC in crcs (each array info->n_blocks long; crcs may be NULL).  Host-only, as above. */
int zc_archive_blocks(const uint8_t *arch, uint64_t len, const zc_archive_info *info, uint64_t *offs,
                      uint32_t *comp_lens, uint8_t *methods, uint32_t *raw_lens, uint32_t *crcs, char *msg,
                      size_t msg_cap);

/* Extracts (out != NULL: the solid stream, info.total_raw bytes, into out) or only tests (out == NULL) an
 * archive held in host memory, as read_blocks + extract_archive / test_archive do (src/archive.h:566-635,
 * 747-785): every block decoded on the GPU, each block's CRC checked against its record, each file's
 * CRC (over its span of the solid stream) computed on the GPU and checked against the table.  ZC_E_DATA
 * for the first failing check, its message in zc_last_error.  The records go through the GPU in chunks
 * that overlap their copies with the other chunk's decode, as zc_archive_write does. */
int zc_archive_extract(zc_ctx *ctx, const uint8_t *arch, uint64_t len, uint8_t *out, uint64_t out_cap);

/* Kernel launches this context has issued since it was opened (for accounting). */
uint64_t zc_launch_count(const zc_ctx *ctx);

/* Per-stage timing (the reference's ZERO_PROFILE stage times, src/gpu_codec.h:32-49): with on != 0 every
 * kernel launch is bracketed by CUDA events on its stream (no device syncs); zc_profile clears the
 * totals.  zc_profile_stages waits for the recorded events and reports, per kernel in first-launch
 * order, its name (names + 32*i, NUL-terminated), total milliseconds and launches; *n_out = stages. */
int zc_profile(zc_ctx *ctx, int on);
int zc_profile_stages(zc_ctx *ctx, uint32_t max, char *names, double *ms, uint64_t *counts, uint32_t *n_out);

#ifdef __cplusplus
}
#endif
#endif /* ZERO_CUDA_H */
