"""The C restatement of the reference codec (oracle/zb2_oracle.c) against the reference's golden vectors,
and against the reference itself (oracle/_ref/libzref.so) where that was built.  CPU only."""
import os
import random

import numpy as np
import pytest

from conftest import GOLDEN, block_input, block_payload, sha

import oracle as O

LEVELS = (1, 5, 9)


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not O.Port.available():
        O.build()


def test_golden_blocks_compress(manifest):
    for ent in manifest["blocks"]:
        data = block_input(ent)
        assert O.Port.crc32(data) == ent["crc32"]
        for lv in LEVELS:
            pay = O.Port.compress_block(data, O.depth_for_level(lv))
            want = ent["levels"][str(lv)]
            assert len(pay) == want["payload_len"], (ent["name"], lv)
            assert sha(pay) == want["sha256"], (ent["name"], lv)


def test_golden_blocks_decompress(manifest):
    for ent in manifest["blocks"]:
        data = block_input(ent)
        for lv in LEVELS:
            pay = block_payload(ent, lv)
            if pay is None:
                continue
            assert O.Port.decompress_block(pay, len(data)) == data, (ent["name"], lv)


def test_golden_streams(manifest):
    for ent in manifest["streams"]:
        with open(os.path.join(GOLDEN, "streams", ent["name"] + ".sym"), "rb") as f:
            sym = f.read()
        with open(os.path.join(GOLDEN, "streams", ent["name"] + ".sec"), "rb") as f:
            sec = f.read()
        assert O.Port.encode_stream(sym) == sec, ent["name"]
        back, used = O.Port.decode_stream(sec, len(sym))
        assert back == sym and used == len(sec)


def test_normalize_edge_cases():
    # one symbol; all 256 at count 1 (sum of mins 256); a huge count beside many tiny ones
    c = np.zeros(256, np.uint32)
    c[9] = 5
    f = O.Port.normalize(c, 5)
    assert f[9] == 4096 and f.sum() == 4096
    c = np.ones(256, np.uint32)
    assert (O.Port.normalize(c, 256) == 16).all()
    c = np.zeros(256, np.uint32)
    c[0] = 10 ** 6
    c[1:200] = 1
    f = O.Port.normalize(c, int(c.sum()))
    assert f.sum() == 4096 and (f[1:200] == 1).all()


def test_crc_combine_identity():
    rng = random.Random(3)
    for _ in range(50):
        a = rng.randbytes(rng.randrange(0, 3000))
        b = rng.randbytes(rng.randrange(0, 3000))
        assert O.Port.crc32_combine(O.Port.crc32(a), O.Port.crc32(b), len(b)) == O.Port.crc32(a + b)


def test_damaged_payloads_are_refused():
    """Random damage: the restatement never crashes, and whatever it accepts is what the reference accepts."""
    data = block_input({"name": "mixed_64k", "source": "file",
                        "sha256": [e for e in __import__("conftest").load_manifest()["blocks"]
                                   if e["name"] == "mixed_64k"][0]["sha256"]})
    pay = bytearray(O.Port.compress_block(data, 32))
    rng = random.Random(5)
    for _ in range(60):
        b = bytearray(pay)
        for _ in range(rng.randrange(1, 20)):
            b[rng.randrange(len(b))] = rng.randrange(256)
        got = O.Port.decompress_block(bytes(b), len(data))
        if O.Ref.available():
            assert got == O.Ref.decompress_block(bytes(b), len(data))


@pytest.mark.skipif(not O.Ref.available(), reason="reference shim not built here")
def test_port_matches_reference_fuzz():
    import datagen as G
    rng = random.Random(11)
    for k in range(12):
        n = rng.choice([5, 17, 100, 4097, 30000, 65536])
        kind = k % 3
        data = G.by_kind(kind, n, 16, 100 + k).tobytes()
        if k % 4 == 3:
            data = bytes(n // 2) + data[: n - n // 2]
        for depth in (8, 32, 256):
            assert O.Port.compress_block(data, depth) == O.Ref.compress_block(data, depth)
            ti, tm, td = O.Port.parse(data, depth)
            ri, rm, rd = O.Ref.parse(data, depth)
            assert np.array_equal(ti, ri) and np.array_equal(tm, rm) and np.array_equal(td, rd)
