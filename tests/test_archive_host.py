"""The archive container's host side, on the CPU: the table and record readers of libzero_cuda.so
(zc_archive_read_table, zc_archive_blocks -- host-only, no GPU) against archives the reference's own
compress_archive wrote (the golden fixtures), and against the reference reader's error for every kind of
damage it detects in the header, footer, table and block records (src/archive.h:451-495, 566-586).
The blocks themselves are decoded here by the oracle."""
import os
import struct
import zlib

import numpy as np
import pytest

from conftest import GOLDEN, load_manifest

import oracle as O
import zero_cuda as Z

ARCH_DIR = os.path.join(GOLDEN, "archives", "three_files")


def golden(name):
    with open(os.path.join(ARCH_DIR, name + ".zero"), "rb") as f:
        return f.read()


def solid_of(entries, root):
    """The files' bytes in entry order (the solid stream), read from the fixture's source tree."""
    out = bytearray()
    for e in entries:
        if not e.is_dir:
            with open(os.path.join(root, e.name), "rb") as f:
                out += f.read()
    return bytes(out)


def test_golden_tables_match_the_files():
    for ent in load_manifest()["archives"]:
        a = golden(ent["name"])
        info, es = Z.read_table(a)
        assert info["block_log"] == ent["block_log"] == 16
        solid = solid_of(es, ARCH_DIR)
        assert info["total_raw"] == len(solid)
        assert info["n_blocks"] == (len(solid) + (1 << 16) - 1) >> 16
        assert info["table_off"] + info["table_len"] + 24 == len(a)
        for e in es:
            if e.is_dir:
                assert e.size == 0 and e.crc == 0 and os.path.isdir(os.path.join(ARCH_DIR, e.name))
            else:
                with open(os.path.join(ARCH_DIR, e.name), "rb") as f:
                    data = f.read()
                assert e.size == len(data) and e.crc == zlib.crc32(data)


def test_golden_records_decode_with_the_oracle():
    for ent in load_manifest()["archives"]:
        a = golden(ent["name"])
        info, es = Z.read_table(a)
        rec = Z.archive_blocks(a, info)
        solid = solid_of(es, ARCH_DIR)
        B = 1 << info["block_log"]
        out = bytearray()
        for b in range(info["n_blocks"]):
            o, cl, m, rl = int(rec["offs"][b]), int(rec["comp_lens"][b]), int(rec["methods"][b]), int(rec["raw_lens"][b])
            body = a[o:o + cl]
            raw = body if m == 0 else O.Port.decompress_block(body, rl)
            assert rl == min(B, len(solid) - b * B)
            assert int(rec["crcs"][b]) == zlib.crc32(raw)
            out += raw
        assert bytes(out) == solid


def test_bound_counts_every_part():
    es = [Z.ArchiveEntry("d", 0, is_dir=True), Z.ArchiveEntry("d/f", 100000), Z.ArchiveEntry("e", 0)]
    table = 4 + sum(8 + len(e.name) + 24 for e in es)
    assert Z.archive_bound(es, 16) == 24 + 2 * 16 + 100000 + table + 24
    assert Z.archive_bound(es, 15) == 0                              # block size out of range
    assert Z.archive_bound([Z.ArchiveEntry("d", 5, is_dir=True)], 16) == 0  # a folder with bytes


# ---- damage: each mutation of a golden archive, our reader's message and the reference reader's

def fix_table_crc(a):
    """Recomputes the footer's table CRC after an edit inside the table."""
    b = bytearray(a)
    toff, tl = struct.unpack_from("<QQ", b, len(b) - 24)
    struct.pack_into("<I", b, len(b) - 8, zlib.crc32(bytes(b[toff:toff + tl])))
    return bytes(b)


def mutate(a, what):
    b = bytearray(a)
    toff, tl = struct.unpack_from("<QQ", b, len(b) - 24)
    if what == "magic":
        b[0] = ord("X")
    elif what == "version":
        b[4] = 3
    elif what == "block_size":
        b[5] = 15
    elif what == "too_short":
        b = b[:40]
    elif what == "footer":
        b = b[:-1]
    elif what == "table_position":
        struct.pack_into("<Q", b, len(b) - 24, toff + 1)
    elif what == "table_checksum":
        b[toff + 6] ^= 1
    elif what == "entry_cut":
        struct.pack_into("<I", b, toff, 7)  # more entries than the table holds
        return fix_table_crc(b)
    elif what == "entry_name":
        struct.pack_into("<I", b, toff + 4 + 4, 10 ** 6)  # the first name runs past the table
        return fix_table_crc(b)
    elif what == "sizes":
        struct.pack_into("<Q", b, 8, struct.unpack_from("<Q", b, 8)[0] + 1)
    elif what == "rec_raw_len":
        struct.pack_into("<I", b, 24, (1 << 16) + 1)
    elif what == "rec_method":
        b[24 + 8] = 2
    elif what == "rec_stored_lens":
        b[24 + 8] = 0
    elif what == "rec_past_table":
        struct.pack_into("<I", b, 24 + 4, toff)
    elif what == "rec_count":
        struct.pack_into("<Q", b, 16, 10 ** 6)
    return bytes(b)


TABLE_DAMAGE = {
    "magic": "not a .zero archive",
    "version": "archive version 3: this program reads version 2",
    "block_size": "archive damaged: block size",
    "too_short": "archive damaged: too short",
    "footer": "archive damaged: footer (the file was cut short?)",
    "table_position": "archive damaged: table position",
    "table_checksum": "archive damaged: table checksum",
    "entry_cut": "archive damaged: entry",
    "entry_name": "archive damaged: entry name",
    "sizes": "archive damaged: sizes",
}
RECORD_DAMAGE = {
    "rec_raw_len": "archive damaged: block header",
    "rec_method": "archive damaged: block header",
    "rec_stored_lens": "archive damaged: block header",
    "rec_past_table": "archive damaged: block past the table",
    "rec_count": "archive damaged: block header cut",
}


def reference_error(a, tmp_path):
    """The reference test_archive's message for these bytes (None when it accepts them)."""
    p = tmp_path / "damaged.zero"
    p.write_bytes(a)
    try:
        O.Ref.test_archive(str(p))
        return None
    except Exception as e:  # noqa: BLE001 -- the oracle raises with the reference's message
        return str(e)


@pytest.mark.parametrize("what", sorted(TABLE_DAMAGE))
def test_table_damage(what, tmp_path):
    a = mutate(golden("three_files.L5"), what)
    with pytest.raises(Z.DataError) as ei:
        Z.read_table(a)
    assert str(ei.value) == TABLE_DAMAGE[what]
    if O.Ref.available():
        assert TABLE_DAMAGE[what] in reference_error(a, tmp_path)


@pytest.mark.parametrize("what", sorted(RECORD_DAMAGE))
def test_record_damage(what, tmp_path):
    a = mutate(golden("three_files.L5"), what)
    info, _ = Z.read_table(a)
    with pytest.raises(Z.DataError) as ei:
        Z.archive_blocks(a, info)
    assert str(ei.value) == RECORD_DAMAGE[what]
    if O.Ref.available() and what != "rec_count":  # (the reference reads past the table before failing there)
        assert RECORD_DAMAGE[what] in reference_error(a, tmp_path)


def test_reader_never_reads_outside_the_buffer():
    """Every prefix of an archive is refused cleanly (the reader bounds each access by the length)."""
    a = golden("three_files.L1")
    for n in list(range(0, 64)) + [len(a) // 2, len(a) - 25, len(a) - 1]:
        with pytest.raises(Z.DataError):
            info, _ = Z.read_table(a[:n])
            Z.archive_blocks(a[:n], info)
    # random corruption of the table and footer: a DataError or a consistent parse, never a crash
    rng = np.random.default_rng(5)
    for _ in range(200):
        b = bytearray(a)
        for _ in range(3):
            b[int(rng.integers(len(b) - 300, len(b)))] = int(rng.integers(0, 256))
        try:
            info, es = Z.read_table(bytes(b))
            Z.archive_blocks(bytes(b), info)
        except Z.DataError:
            pass


def stored_archive(files, block_log):
    """An archive written here with stored blocks only (the layout of src/archive.h:334-441):
    files = [(name, bytes or None for a folder, mtime, attr)]."""
    B = 1 << block_log
    solid = b"".join(d for _, d, _, _ in files if d is not None)
    nb = (len(solid) + B - 1) // B
    out = [b"ZERO" + bytes([2, block_log, 0, 0]) + struct.pack("<QQ", len(solid), nb)]
    for b in range(nb):
        blk = solid[b * B:(b + 1) * B]
        out.append(struct.pack("<IIB3xI", len(blk), len(blk), 0, zlib.crc32(blk)) + blk)
    table = [struct.pack("<I", len(files))]
    for name, data, mtime, attr in files:
        nm = name.encode()
        size = 0 if data is None else len(data)
        crc = 0 if data is None else zlib.crc32(data)
        table.append(struct.pack("<B3xI", 1 if data is None else 0, len(nm)) + nm + struct.pack("<QqII", size, mtime, attr, crc))
    head = b"".join(out)
    table = b"".join(table)
    return head + table + struct.pack("<QQI", len(head), len(table), zlib.crc32(table)) + b"ZEND", solid


def test_reader_fields_round_trip():
    rng = np.random.default_rng(9)
    files = [("dossier", None, 1700000000, 16),
             ("dossier/été.txt", rng.integers(0, 256, 70000, dtype=np.uint8).tobytes(), -86400, 0x20),
             ("dossier/sub", None, 0, 16),
             ("dossier/sub/empty", b"", 5, 0),
             ("dossier/sub/z", bytes(100), 2**40, 0xFFFFFFFF)]
    a, solid = stored_archive(files, 16)
    info, es = Z.read_table(a)
    assert info["total_raw"] == len(solid) and info["n_blocks"] == 2 and info["n_entries"] == len(files)
    for (name, data, mtime, attr), e in zip(files, es):
        assert e.name == name and e.is_dir == (data is None) and e.mtime == mtime and e.attr == attr
        assert e.size == (0 if data is None else len(data))
        assert e.crc == (0 if data is None else zlib.crc32(data))
    rec = Z.archive_blocks(a, info)
    assert list(rec["methods"]) == [0, 0] and list(rec["raw_lens"]) == [65536, len(solid) - 65536]
    got = b"".join(a[int(o):int(o) + int(n)] for o, n in zip(rec["offs"], rec["comp_lens"]))
    assert got == solid
    assert [int(c) for c in rec["crcs"]] == [zlib.crc32(solid[:65536]), zlib.crc32(solid[65536:])]


def test_reader_properties():
    """Random entry lists (folders, empty and non-empty files, names of any UTF-8, any mtime and
    attributes) at random block sizes: every field and block comes back as written; then random
    corruptions of each archive end in a DataError or in a parse that stays inside the buffer."""
    from hypothesis import given, settings, strategies as st, HealthCheck

    entry = st.tuples(st.text(min_size=1, max_size=12), st.one_of(st.none(), st.binary(max_size=3000)),
                      st.integers(-2**63, 2**63 - 1), st.integers(0, 2**32 - 1))

    @settings(max_examples=60, deadline=None, suppress_health_check=list(HealthCheck))
    @given(st.lists(entry, max_size=12), st.integers(16, 20), st.integers(0, 2**32 - 1))
    def check(files, block_log, seed):
        a, solid = stored_archive(files, block_log)
        info, es = Z.read_table(a)
        assert info["total_raw"] == len(solid) and info["n_entries"] == len(files)
        for (name, data, mtime, attr), e in zip(files, es):
            assert (e.name, e.is_dir, e.mtime, e.attr) == (name, data is None, mtime, attr)
            assert e.size == (0 if data is None else len(data))
        rec = Z.archive_blocks(a, info)
        assert b"".join(a[int(o):int(o) + int(n)] for o, n in zip(rec["offs"], rec["comp_lens"])) == solid
        rng = np.random.default_rng(seed)
        for _ in range(8):
            b = bytearray(a)
            for _ in range(int(rng.integers(1, 4))):
                b[int(rng.integers(0, len(b)))] = int(rng.integers(0, 256))
            try:
                i2, _ = Z.read_table(bytes(b))
                Z.archive_blocks(bytes(b), i2)
            except Z.DataError:
                pass

    check()


def test_collect_matches_the_reference(tmp_path):
    """zero_cuda.collect gives the reference's entries, in its order: byte-sorted names in every folder
    (upper case before lower case, '10' before '9', UTF-8 after ASCII), symlinks skipped, empty folders
    and files kept, a repeated input kept once; read_solid gives the bytes the reference's blocks hold."""
    if not O.Ref.available():
        pytest.skip("oracle/_ref (built from the reference tree) is not present")
    root = tmp_path / "data"
    files = {"B.txt": b"upper", "a.txt": b"lower", "été.bin": bytes(range(256)) * 300, "z/deep/file": b"x" * 70000,
             "z/empty": b"", "_": b"u", "10": b"ten", "9": b"nine"}
    for rel, data in files.items():
        p = root / rel
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_bytes(data)
    (root / "emptydir").mkdir()
    os.symlink("a.txt", root / "link")
    single = tmp_path / "single.bin"
    single.write_bytes(b"one file on its own" * 100)
    for dp, dn, fn in os.walk(root):
        for x in dn + fn:
            os.utime(os.path.join(dp, x), (1700000000, 1700000000), follow_symlinks=False)
    os.utime(root, (1700000000, 1700000000))
    inputs = [str(root), str(single), str(root) + "/"]
    ref = tmp_path / "r.zero"
    O.Ref.compress_archive(inputs, str(ref), block_log=16, level=1)
    a = ref.read_bytes()
    info, es = Z.read_table(a)
    got = Z.collect(inputs)
    assert [(e.name, e.is_dir, e.size, e.mtime, e.attr) for e, _ in got] == \
           [(e.name, e.is_dir, e.size, e.mtime, e.attr) for e in es]
    rec = Z.archive_blocks(a, info)
    out = bytearray()
    for o, cl, m, rl in zip(rec["offs"], rec["comp_lens"], rec["methods"], rec["raw_lens"]):
        body = a[int(o):int(o) + int(cl)]
        out += body if m == 0 else O.Port.decompress_block(body, int(rl))
    assert Z.read_solid(got) == bytes(out)
    with pytest.raises(FileNotFoundError):
        Z.collect([str(tmp_path / "missing")])


def tree_state(root):
    """Every path under root: (is folder, contents or None, modification time in seconds)."""
    out = {}
    for dp, dn, fn in os.walk(root):
        for x in dn + fn:
            p = os.path.join(dp, x)
            data = None
            if os.path.isfile(p):
                with open(p, "rb") as f:
                    data = f.read()
            out[os.path.relpath(p, root)] = (os.path.isdir(p), data, os.stat(p).st_mtime_ns // 10**9)
    return out


def test_write_tree_matches_reference_extract(tmp_path):
    """write_tree writes what the reference's extract_archive writes: the same files and folders, bytes
    and modification times; an unsafe name is refused with the reference's message."""
    if not O.Ref.available():
        pytest.skip("oracle/_ref (built from the reference tree) is not present")
    for ent in load_manifest()["archives"]:
        a = golden(ent["name"])
        info, es = Z.read_table(a)
        rec = Z.archive_blocks(a, info)
        solid = b"".join(a[int(o):int(o) + int(cl)] if m == 0 else O.Port.decompress_block(a[int(o):int(o) + int(cl)], int(rl))
                         for o, cl, m, rl in zip(rec["offs"], rec["comp_lens"], rec["methods"], rec["raw_lens"]))
        ours, ref = tmp_path / ("ours_" + ent["name"]), tmp_path / ("ref_" + ent["name"])
        ours.mkdir()
        Z.write_tree(es, solid, str(ours))
        O.Ref.extract_archive(os.path.join(ARCH_DIR, ent["name"] + ".zero"), str(ref))
        assert tree_state(ours) == tree_state(ref)
    bad, solid = stored_archive([("ok", b"fine", 5, 0), ("../evil", b"no", 5, 0)], 16)
    p = tmp_path / "bad.zero"
    p.write_bytes(bad)
    _, es = Z.read_table(bad)
    out = tmp_path / "bad_ours"
    out.mkdir()
    with pytest.raises(Z.DataError, match="refused: unsafe name in the archive: ../evil"):
        Z.write_tree(es, solid, str(out))
    assert not (tmp_path / "evil").exists()
    with pytest.raises(RuntimeError, match="refused: unsafe name in the archive: ../evil"):
        O.Ref.extract_archive(str(p), str(tmp_path / "bad_ref"))
