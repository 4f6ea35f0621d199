"""Sharded archives through the GPU writer: two gloo ranks (one process each, both on the one GPU here)
each write their contiguous block range's records with zc_archive_write_range, the one exchange (the ranks'
record totals, scanned; each rank's per-file (crc, length) pieces) goes over gloo, rank 0 adds the header,
the entry table with the combined file CRCs and the footer.  The assembled file must equal the reference's
compress_archive of the same folder byte for byte, and must extract bit-exact on the GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
import shard

pytestmark = pytest.mark.gpu


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def rank_main(rank, world, port, root, out_dir, bl, level):
    import torch
    import torch.distributed as dist
    import zero_cuda as Z
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    torch.cuda.set_device(0)
    got = Z.collect([root])
    entries = [e for e, _ in got]
    raw = np.frombuffer(Z.read_solid(got), np.uint8)
    B = 1 << bl
    nb = (raw.size + B - 1) // B
    b0, b1 = shard.block_range(nb, world, rank)
    lo, hi = b0 * B, min(b1 * B, raw.size)
    with Z.CudaCodec(level=level) as codec:
        recs, mine = shard.gpu_records(codec, raw[lo:hi], lo, entries, bl)
    off, total = shard.place(len(recs))
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


@pytest.mark.skipif(not O.Ref.available(), reason="oracle/_ref (built from the reference tree) is not present")
@pytest.mark.parametrize("bl,level,world", [(16, 5, 2), (18, 9, 2), (16, 1, 3)])
def test_ranks_write_the_reference_archive_on_the_gpu(tmp_path, bl, level, world):
    import datagen as G
    import zero_cuda as Z
    root = tmp_path / "data"
    files = {"a.txt": G.text_mix(300000, 3).tobytes(), "m/b.lz": G.lz_mix(500000, bl, 4).tobytes(),
             "m/empty": b"", "m/z.rnd": G.random_bytes(90000, 5).tobytes(), "q": b"tiny",
             "r/big.lz": G.lz_mix(700001, bl, 6).tobytes()}
    for rel, data in files.items():
        p = root / rel
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_bytes(data)
    (root / "n").mkdir()
    for dp, dn, fn in os.walk(root):
        for x in dn + fn:
            os.utime(os.path.join(dp, x), (1700000000, 1700000000))
    os.utime(root, (1700000000, 1700000000))
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=rank_main, args=(r, world, port, str(root), str(tmp_path), bl, level))
             for r in range(world)]
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
    arch = b"".join(parts)
    ref = tmp_path / "ref.zero"
    O.Ref.compress_archive([str(root)], str(ref), block_log=bl, level=level)
    assert arch == ref.read_bytes()
    with Z.CudaCodec(level=level) as codec:
        got = Z.collect([str(root)])
        assert codec.archive_extract(arch) == Z.read_solid(got)


def test_range_arguments_are_checked():
    """A range that does not start on a block boundary, or ends inside a block before the stream's end, or
    an output too small for its records, is refused before anything runs."""
    import torch
    import zero_cuda as Z
    e = Z.ArchiveEntry("f", size=300000)
    with Z.CudaCodec() as codec:
        g = torch.Generator(device="cuda").manual_seed(9)
        d = torch.randint(0, 256, (300000 + 64,), dtype=torch.uint8, device="cuda", generator=g)
        out = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
        ln = torch.zeros(1, dtype=torch.int64, device="cuda")
        for off, n, cap in ((1000, 65536, None), (0, 70000, None), (65536, 65536, 1000)):
            with pytest.raises(Z.ArgError):
                codec.archive_write_range(d, off, n, [e], 16, out, ln, out_cap=cap)
        codec.archive_write_range(d, 65536, 300000 - 65536, [e], 16, out, ln)  # up to the stream's end
        torch.cuda.synchronize()
        assert int(ln.item()) == 16 * 4 + (300000 - 65536)  # (random bytes: four stored blocks)
