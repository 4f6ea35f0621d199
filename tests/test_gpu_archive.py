"""Whole archives on the GPU (zc_archive_write / zc_archive_write_device / zc_archive_extract).  An archive
the device assembles -- records placed by the device scan, file CRCs combined across blocks, table and
footer -- must equal byte for byte the one the reference's compress_archive (src/archive.h:334-441) writes
with its CPU codec for the same files: the golden fixtures, and fresh trees through oracle/_ref when it is
present.  The extractor must return the solid stream and refuse every block or file whose CRC does not
match (src/archive.h:611-624, 655-667)."""
import os
import struct
import zlib

import numpy as np
import pytest

from conftest import load_manifest
from test_archive_host import ARCH_DIR, fix_table_crc, golden, solid_of

import oracle as O
import zero_cuda as Z

pytestmark = pytest.mark.gpu
need_ref = pytest.mark.skipif(not O.Ref.available(), reason="oracle/_ref (built from the reference tree) is not present")


@pytest.fixture(scope="module")
def codec():
    with Z.CudaCodec(level=5) as c:
        yield c


def cleared(entries):
    for e in entries:
        e.crc = 0
    return entries


def test_golden_archives_assembled_on_gpu(codec):
    for ent in load_manifest()["archives"]:
        a = golden(ent["name"])
        info, es = Z.read_table(a)
        want = [e.crc for e in es]
        solid = solid_of(es, ARCH_DIR)
        got = codec.archive_write(solid, cleared(es), info["block_log"], level=ent["level"])
        assert got == a, ent["name"]
        assert [e.crc for e in es] == want


def make_tree(root, block_log):
    """Files that start, end and straddle block boundaries: one block exactly, several blocks plus one
    byte, many tiny files sharing a block, empty files and folders, incompressible and all-zero data."""
    import datagen as G
    B = 1 << block_log
    files = {
        "a.txt": G.text_mix(3 * B + 1, 11).tobytes(),
        "exact.bin": G.lz_mix(B, 16, 12).tobytes(),
        "sub/b.lz": G.lz_mix(2 * B + B // 3, block_log, 13).tobytes(),
        "sub/empty": b"",
        "sub/deeper/c.rnd": G.random_bytes(B + 777, 14).tobytes(),
        "zeros": bytes(B // 2 + 5),
    }
    for i in range(40):
        files["tiny/t%02d" % i] = bytes((i * 7 + k) & 0xFF for k in range(1 + 37 * i % 300))
    for rel, data in files.items():
        p = root / rel
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_bytes(data)
    (root / "empty_dir").mkdir()
    for dp, dn, fn in os.walk(root):
        for x in dn + fn:
            os.utime(os.path.join(dp, x), (1700000000, 1700000000))
    os.utime(root, (1700000000, 1700000000))


@need_ref
@pytest.mark.parametrize("block,level", [(16, 1), (16, 9), (18, 5), (20, 9)])
def test_archives_equal_reference_compress_archive(codec, tmp_path, block, level):
    root = tmp_path / "data"
    make_tree(root, block)
    ref = tmp_path / "ref.zero"
    O.Ref.compress_archive([str(root)], str(ref), block_log=block, level=level)
    a = ref.read_bytes()
    info, es = Z.read_table(a)
    solid = solid_of(es, str(tmp_path))
    assert codec.archive_write(solid, cleared(es), block, level=level) == a
    assert codec.archive_extract(a) == solid
    assert codec.archive_extract(a, test=True) is None


@need_ref
def test_archive_without_bytes(codec, tmp_path):
    """Only folders and empty files: no blocks, the header, the table and the footer."""
    root = tmp_path / "data"
    (root / "d" / "e").mkdir(parents=True)
    (root / "d" / "nothing").write_bytes(b"")
    ref = tmp_path / "ref.zero"
    O.Ref.compress_archive([str(root)], str(ref), block_log=18, level=5)
    a = ref.read_bytes()
    info, es = Z.read_table(a)
    assert info["n_blocks"] == 0 and info["total_raw"] == 0
    assert codec.archive_write(b"", cleared(es), 18) == a
    assert codec.archive_extract(a) == b""


def test_device_form_equals_host_form(codec):
    import torch
    a = golden("three_files.L5")
    info, es = Z.read_table(a)
    want = [e.crc for e in es]
    solid = solid_of(es, ARCH_DIR)
    d_solid = torch.zeros(len(solid) + 64, dtype=torch.uint8, device="cuda")
    d_solid[: len(solid)] = torch.frombuffer(bytearray(solid), dtype=torch.uint8).cuda()
    cap = Z.archive_bound(es, 16)
    d_out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    d_len = torch.zeros(1, dtype=torch.int64, device="cuda")
    d_crc = torch.zeros(len(es), dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()
    codec.archive_write_device(d_solid, cleared(es), 16, d_out, d_len, d_crc, stream=s.cuda_stream, level=5)
    s.synchronize()
    n = int(d_len.item())
    assert n == len(a)
    assert d_out[:n].cpu().numpy().tobytes() == a
    assert [int(x) & 0xFFFFFFFF for x in d_crc.cpu().tolist()] == want


def table_crc_field(a, name):
    """The offset of entry `name`'s CRC field in archive a."""
    toff = struct.unpack_from("<Q", a, len(a) - 24)[0]
    p = toff + 4
    for _ in range(struct.unpack_from("<I", a, toff)[0]):
        nl = struct.unpack_from("<I", a, p + 4)[0]
        if a[p + 8:p + 8 + nl].decode() == name:
            return p + 8 + nl + 20
        p += 8 + nl + 24
    raise KeyError(name)


def test_extract_refuses_mismatched_checksums(codec):
    a = golden("three_files.L1")
    info, es = Z.read_table(a)
    rec = Z.archive_blocks(a, info)
    assert codec.archive_extract(a) == solid_of(es, ARCH_DIR)
    # a record's CRC: the block check
    b = bytearray(a)
    b[int(rec["offs"][2]) - 16 + 12] ^= 1
    with pytest.raises(Z.DataError, match="block 2 does not match its checksum"):
        codec.archive_extract(bytes(b), test=True)
    # a file's CRC in the table (the table's own CRC fixed): only the file check sees it
    b = bytearray(a)
    b[table_crc_field(a, "src/sub/b.bin")] ^= 0x80
    with pytest.raises(Z.DataError, match="file src/sub/b.bin does not match its checksum"):
        codec.archive_extract(fix_table_crc(b))
    # payload bytes: the decoder or the block CRC refuses the block
    for at in (0, 7, 100, int(rec["comp_lens"][1]) - 3):
        b = bytearray(a)
        b[int(rec["offs"][1]) + at] ^= 0x5A
        with pytest.raises(Z.DataError, match="block 1 "):
            codec.archive_extract(bytes(b), test=True)


def test_bad_entries_are_refused(codec):
    with pytest.raises(Z.ArgError):
        codec.archive_write(b"abc", [Z.ArchiveEntry("d", 3, is_dir=True)], 16)
    with pytest.raises(Z.ArgError):
        codec.archive_write(b"abc", [Z.ArchiveEntry("f", 3)], 15)


def python_archive(codec, solid, es, block_log, level):
    """The archive assembled on the host from zc_compress's per-block results (the codec's bytes are
    checked against the CPU codec elsewhere) and zlib's CRCs: the expected bytes for a large stream."""
    methods, lens, crcs, pay, offs = codec.compress_arrays(solid, block_log, level)
    B = 1 << block_log
    mv = memoryview(solid)
    parts = [b"ZERO" + bytes([2, block_log, 0, 0]) + struct.pack("<QQ", len(solid), len(methods))]
    for b in range(len(methods)):
        raw = mv[b * B:(b + 1) * B]
        body = pay[int(offs[b]):int(offs[b]) + int(lens[b])].tobytes() if methods[b] else raw
        parts.append(struct.pack("<IIB3xI", len(raw), len(body), int(methods[b]), int(crcs[b])))
        parts.append(body)
    table = [struct.pack("<I", len(es))]
    at = 0
    for e in es:
        nm = e.name.encode()
        crc = 0 if e.is_dir else zlib.crc32(mv[at:at + e.size])
        at += 0 if e.is_dir else e.size
        table.append(struct.pack("<B3xI", 1 if e.is_dir else 0, len(nm)) + nm +
                     struct.pack("<QqII", e.size, e.mtime, e.attr, crc))
    table = b"".join(table)
    head = b"".join(parts)
    return head + table + struct.pack("<QQI", len(head), len(table), zlib.crc32(table)) + b"ZEND"


def test_archive_over_several_encoder_launches(codec):
    """1 GiB + 300 KiB at block 16: the host write streams it in four chunks (128, 512, 384 MiB and the
    rest), each chunk's records coming down while the next is coded; files straddle the chunks."""
    import datagen as G
    n = (1 << 30) + 300 * 1024
    solid = np.concatenate([G.lz_mix(n - 600 * 1024, 16, 21), G.random_bytes(300 * 1024, 22),
                            G.text_mix(300 * 1024, 23)]).tobytes()
    sizes = [700 << 20, (1 << 30) - (700 << 20) + 150 * 1024, 100 * 1024, 7, 0, n]
    sizes[-1] = n - sum(sizes[:-1])
    es = [Z.ArchiveEntry("f%d" % i, s, mtime=1700000000 + i, attr=i) for i, s in enumerate(sizes)]
    es.insert(2, Z.ArchiveEntry("dir", 0, is_dir=True))
    want = python_archive(codec, solid, es, 16, 1)
    got = codec.archive_write(solid, es, 16, level=1)
    assert len(got) == len(want) and got == want
    info, back = Z.read_table(got)
    assert info["n_blocks"] == (n + 65535) >> 16 > 16384
    assert [e.crc for e in back] == [e.crc for e in es]
    # the host calls stream through two stages in 128 / 512 MiB chunks: files straddle the chunks too
    assert codec.archive_extract(got) == solid
    assert codec.archive_extract(got, test=True) is None
    # the device form: two encoder launches, the second's records placed after the first's on the device
    import torch
    d_solid = torch.zeros(n + 64, dtype=torch.uint8, device="cuda")
    d_solid[:n] = torch.frombuffer(bytearray(solid), dtype=torch.uint8).cuda()
    cap = Z.archive_bound(es, 16)
    d_out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    d_len = torch.zeros(1, dtype=torch.int64, device="cuda")
    codec.archive_write_device(d_solid, es, 16, d_out, d_len, level=1)
    torch.cuda.synchronize()
    assert int(d_len.item()) == len(got)
    assert d_out[:len(got)].cpu().numpy().tobytes() == got


@need_ref
@pytest.mark.parametrize("block,level", [(16, 9), (18, 5)])
def test_archive_write_paths_equals_compress_archive(codec, tmp_path, block, level):
    """`zero c` from Python: folders and files collected as the reference does, written on the GPU."""
    root = tmp_path / "data"
    make_tree(root, block)
    single = tmp_path / "single.bin"
    single.write_bytes(b"one file on its own" * 1000)
    ref = tmp_path / "ref.zero"
    O.Ref.compress_archive([str(root), str(single)], str(ref), block_log=block, level=level)
    got, entries = codec.archive_write_paths([str(root), str(single)], block, level=level)
    assert got == ref.read_bytes()
    assert [e.crc for e in entries] == [e.crc for e in Z.read_table(got)[1]]


@need_ref
def test_archive_extract_to_equals_extract_archive(codec, tmp_path):
    """`zero x` from Python: every CRC checked on the GPU, then the files written as extract_archive writes
    them (the same files, folders, bytes and modification times)."""
    from test_archive_host import tree_state
    for ent in load_manifest()["archives"]:
        ours, ref = tmp_path / ("ours_" + ent["name"]), tmp_path / ("ref_" + ent["name"])
        codec.archive_extract_to(golden(ent["name"]), str(ours))
        O.Ref.extract_archive(os.path.join(ARCH_DIR, ent["name"] + ".zero"), str(ref))
        assert tree_state(ours) == tree_state(ref)
