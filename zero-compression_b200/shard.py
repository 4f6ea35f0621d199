"""Sharding one archive's blocks over several GPUs (one process per GPU).

Blocks are independent (docs/how-it-works.md:3-4 in the reference), so each rank codes a contiguous range
of the solid stream's blocks with no data exchange.  Writing one archive needs a single exchange: every
rank's total record bytes (16-byte block record + body, src/archive.h:389-403), scanned across ranks to
give each rank the offset of its first record.  CRCs of files that straddle two ranks' ranges combine
with crc32::combine (src/crc32.h:60-66).  The exchange is one all-gather of one 64-bit value per rank
(torch.distributed: NCCL between GPUs, gloo on the CPU), and, for the entry table, one all-gather of each
rank's (crc, length) piece of every file.  gpu_records writes a rank's records and file pieces on its GPU
(zc_archive_write_range); records() builds them on the host from already coded blocks.
"""
import struct

REC_HDR = 16  # u32 raw_len, u32 comp_len, u8 method, 3 pad, u32 crc32 (src/archive.h:395-399)


def block_range(nb, world, rank):
    """The blocks [b0, b1) of `rank`: contiguous, sizes differing by at most one."""
    base, extra = divmod(nb, world)
    b0 = rank * base + min(rank, extra)
    return b0, b0 + base + (1 if rank < extra else 0)


def records(raw, methods, comp_lens, crcs, bodies, block_log):
    """The archive's block records for consecutive blocks of `raw` (numpy u8): each a 16-byte header and
    the body (the ZB2 payload, or the raw bytes when stored).  bodies[b] is the payload (ignored when
    stored).  Returns bytes."""
    B = 1 << block_log
    out = bytearray()
    for b in range(len(methods)):
        blk = raw[b * B:(b + 1) * B]
        stored = methods[b] == 0 or len(bodies[b]) >= blk.size
        body = blk.tobytes() if stored else bytes(bodies[b])
        out += struct.pack("<IIBBBBI", blk.size, len(body), 0 if stored else int(methods[b]), 0, 0, 0, int(crcs[b]))
        out += body
    return bytes(out)


def gpu_records(codec, stream_range, range_off, entries, block_log, level=None):
    """One rank's block records, written on its GPU by zc_archive_write_range: `stream_range` (numpy u8) is
    the solid stream's bytes [range_off, range_off + len) -- whole blocks, the last may end the stream.
    Returns (the records as bytes, per entry the (crc, length) of its piece inside the range)."""
    import numpy as np
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    n = int(stream_range.size)
    B = 1 << block_log
    nb = (n + B - 1) // B
    d_range = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
    if n:
        d_range[:n].copy_(torch.from_numpy(np.ascontiguousarray(stream_range)))
    cap = nb * (REC_HDR + B) + 64
    d_out = torch.zeros(cap, dtype=torch.uint8, device=dev)
    d_len = torch.zeros(1, dtype=torch.int64, device=dev)
    d_crc = torch.zeros(max(len(entries), 1), dtype=torch.int32, device=dev)
    codec.archive_write_range(d_range, range_off, n, entries, block_log, d_out, d_len, d_crc, level=level)
    torch.cuda.synchronize(dev)
    length = int(d_len.item())
    sizes = [0 if e.is_dir else e.size for e in entries]
    lens = [ln for _, ln in file_pieces(sizes, range_off, range_off + n)]
    crcs = [int(c) & 0xFFFFFFFF for c in d_crc.cpu().numpy()[:len(entries)]]
    return d_out[:length].cpu().numpy().tobytes(), list(zip(crcs, lens))


def place(local_bytes, group=None):
    """All ranks: (offset of this rank's records in the archive body, total body bytes of all ranks)."""
    import torch
    import torch.distributed as dist
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return 0, int(local_bytes)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    mine = torch.tensor([int(local_bytes)], dtype=torch.int64, device=dev)
    all_ = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(all_, mine, group=group)
    sizes = [int(t.item()) for t in all_]
    return sum(sizes[:rank]), sum(sizes)


def crc_combine(crc_a, crc_b, len_b):
    """CRC-32 of A followed by B (crc32::combine) through the library's host routine."""
    import zero_cuda as Z
    return int(Z.crc32_combine(crc_a & 0xFFFFFFFF, crc_b & 0xFFFFFFFF, int(len_b)))


def stream_crc(part_crcs, part_lens):
    """The CRC of consecutive parts (a file's pieces on several ranks, in rank order)."""
    crc = 0
    for c, n in zip(part_crcs, part_lens):
        crc = crc_combine(crc, c, n)
    return crc


def file_pieces(sizes, lo, hi):
    """For files of `sizes` laid end to end in the solid stream (folders have size 0): each file's part
    inside the stream range [lo, hi) as (offset in the stream, length); (0, 0) for a file outside it."""
    out, at = [], 0
    for n in sizes:
        a, b = max(at, lo), min(at + n, hi)
        out.append((a, b - a) if b > a else (0, 0))
        at += n
    return out


def gather_pieces(pieces, group=None):
    """All ranks: every rank's per-file (crc, length) pieces, in rank order (one all-gather of objects)."""
    import torch.distributed as dist
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return [pieces]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, pieces, group=group)
    return out


def entry_table(entries, crcs):
    """The entry table (src/archive.h:416-429): u32 count; per entry u8 type (1 = folder), 3 zero bytes,
    u32 name length, the name, u64 size, u64 mtime, u32 attributes, u32 CRC."""
    out = bytearray(struct.pack("<I", len(entries)))
    for e, crc in zip(entries, crcs):
        nm = e.name.encode("utf-8", "surrogateescape")
        out += struct.pack("<B3xI", 1 if e.is_dir else 0, len(nm)) + nm
        out += struct.pack("<QqII", e.size, e.mtime, e.attr, crc & 0xFFFFFFFF)
    return bytes(out)


def footer(table_off, table):
    """The footer (src/archive.h:430-435): u64 table offset, u64 table length, u32 CRC of the table, "ZEND"."""
    import zlib
    return struct.pack("<QQI", table_off, len(table), zlib.crc32(table)) + b"ZEND"


def header(total_raw, n_blocks, block_log):
    """The archive header (src/archive.h:356-361): "ZERO", version 2, block_log, 0, total raw, blocks."""
    return b"ZERO" + struct.pack("<BBH", 2, block_log, 0) + struct.pack("<QQ", total_raw, n_blocks)
