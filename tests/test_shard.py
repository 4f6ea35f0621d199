"""Multi-rank sharding on the CPU: two gloo ranks each code a contiguous block range of one solid stream;
the single exchange (rank totals, scanned) places their records, and the assembled archive body equals the
one a single rank writes.  File CRCs that straddle ranks combine to the whole file's CRC.  The coding
itself is done here by the oracle (the test's stand-in for the GPU codec: this path has no GPU)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import oracle as O
import shard


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def make_data():
    import datagen as G
    return np.concatenate([G.text_mix(300000, 3), G.lz_mix(250000, 16, 4), G.random_bytes(70000, 5)])


def code_blocks(raw, b0, b1, block_log, depth=32):
    B = 1 << block_log
    methods, lens, crcs, bodies = [], [], [], []
    for b in range(b0, b1):
        blk = raw[b * B:(b + 1) * B].tobytes()
        pay = O.Port.compress_block(blk, depth)
        stored = len(pay) >= len(blk)
        methods.append(0 if stored else 1)
        lens.append(len(blk) if stored else len(pay))
        crcs.append(O.Port.crc32(blk))
        bodies.append(b"" if stored else pay)
    return methods, lens, crcs, bodies


def rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    raw = make_data()
    bl = 16
    B = 1 << bl
    nb = (raw.size + B - 1) // B
    b0, b1 = shard.block_range(nb, world, rank)
    m, l, c, bodies = code_blocks(raw, b0, b1, bl)
    recs = shard.records(raw[b0 * B:], m, l, c, bodies, bl)
    off, total = shard.place(len(recs))
    # a "file" covering the middle of the stream: each rank's CRC of its piece
    f0, f1 = 100000, 500000
    lo, hi = max(f0, b0 * B), min(f1, min(b1 * B, raw.size))
    piece = raw[lo:hi].tobytes() if hi > lo else b""
    with open(os.path.join(out_dir, f"r{rank}.bin"), "wb") as f:
        f.write(recs)
    with open(os.path.join(out_dir, f"r{rank}.meta"), "w") as f:
        f.write(f"{off} {total} {O.Port.crc32(piece)} {len(piece)}")
    dist.barrier()
    dist.destroy_process_group()


def test_block_range_covers_all():
    for nb in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            got = [shard.block_range(nb, world, r) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == nb
            assert all(got[i][1] == got[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1


def test_two_ranks_assemble_the_single_rank_archive(tmp_path):
    world = 2
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    raw = make_data()
    bl = 16
    nb = (raw.size + (1 << bl) - 1) >> bl
    m, l, c, bodies = code_blocks(raw, 0, nb, bl)
    single = shard.records(raw, m, l, c, bodies, bl)
    body = bytearray()
    metas = []
    for r in range(world):
        with open(tmp_path / f"r{r}.meta") as f:
            off, total, crc, n = (int(x) for x in f.read().split())
        metas.append((off, total, crc, n))
        assert off == len(body)
        body += (tmp_path / f"r{r}.bin").read_bytes()
    assert all(mt[1] == len(body) for mt in metas)
    assert bytes(body) == single
    # the straddling file's CRC from its two pieces
    whole = O.Port.crc32(raw[100000:500000].tobytes())
    assert shard.stream_crc([mt[2] for mt in metas], [mt[3] for mt in metas]) == whole
    assert shard.header(raw.size, nb, bl)[:6] == b"ZERO\x02\x10"


def archive_rank_main(rank, world, port, root, out_dir):
    """One rank of a whole-archive write: its block range coded, its records placed by the scan, its
    piece of every file's CRC exchanged; rank 0 adds the header, the entry table and the footer."""
    import torch.distributed as dist
    import zero_cuda as Z
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    got = Z.collect([root])
    entries = [e for e, _ in got]
    raw = np.frombuffer(Z.read_solid(got), np.uint8)
    bl = 16
    B = 1 << bl
    nb = (raw.size + B - 1) // B
    b0, b1 = shard.block_range(nb, world, rank)
    m, l, c, bodies = code_blocks(raw, b0, b1, bl, depth=O.depth_for_level(5))
    recs = shard.records(raw[b0 * B:], m, l, c, bodies, bl)
    off, total = shard.place(len(recs))
    sizes = [0 if e.is_dir else e.size for e in entries]
    mine = [(O.Port.crc32(raw[a:a + n].tobytes()) if n else 0, n)
            for a, n in shard.file_pieces(sizes, b0 * B, min(b1 * B, raw.size))]
    everyone = shard.gather_pieces(mine)
    crcs = [shard.stream_crc([p[f][0] for p in everyone], [p[f][1] for p in everyone]) for f in range(len(entries))]
    with open(os.path.join(out_dir, f"a{rank}.bin"), "wb") as f:
        f.write(recs)
    if rank == 0:
        table = shard.entry_table(entries, crcs)
        with open(os.path.join(out_dir, "head.bin"), "wb") as f:
            f.write(shard.header(raw.size, nb, bl))
        with open(os.path.join(out_dir, "tail.bin"), "wb") as f:
            f.write(table + shard.footer(24 + total, table))
    with open(os.path.join(out_dir, f"a{rank}.off"), "w") as f:
        f.write(str(off))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_write_the_reference_archive(tmp_path):
    """Two gloo ranks write one whole archive of a folder (files straddling the ranks' block ranges):
    the bytes equal the reference's compress_archive of the same folder."""
    import datagen as G
    if not O.Ref.available():
        import pytest
        pytest.skip("oracle/_ref (built from the reference tree) is not present")
    root = tmp_path / "data"
    files = {"a.txt": G.text_mix(200000, 3).tobytes(), "m/b.lz": G.lz_mix(300000, 16, 4).tobytes(),
             "m/empty": b"", "m/z.rnd": G.random_bytes(70000, 5).tobytes(), "q": b"tiny"}
    for rel, data in files.items():
        p = root / rel
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_bytes(data)
    (root / "n").mkdir()
    for dp, dn, fn in os.walk(root):
        for x in dn + fn:
            os.utime(os.path.join(dp, x), (1700000000, 1700000000))
    os.utime(root, (1700000000, 1700000000))
    world = 2
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=archive_rank_main, args=(r, world, port, str(root), str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    parts = [(tmp_path / "head.bin").read_bytes()]
    for r in range(world):
        assert int((tmp_path / f"a{r}.off").read_text()) == sum(len(x) for x in parts) - 24
        parts.append((tmp_path / f"a{r}.bin").read_bytes())
    parts.append((tmp_path / "tail.bin").read_bytes())
    ref = tmp_path / "ref.zero"
    O.Ref.compress_archive([str(root)], str(ref), block_log=16, level=5)
    assert b"".join(parts) == ref.read_bytes()
