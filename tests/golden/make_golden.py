"""Writes the golden vectors under tests/golden/ with the REFERENCE CPU codec (oracle/_ref/libzref.so, which
oracle/Makefile compiles from the reference's own sources).  Run where the reference tree exists:

    make -C oracle && python tests/golden/make_golden.py

What it writes (all committed, small):
  blocks/<case>.in            raw input of a block case (only for cases not rebuilt from the seeded generator)
  blocks/<case>.L<level>.zb2  the reference's block payload at that level (absent when the block is stored)
  streams/<case>.sym / .sec   symbols and the reference's encode_stream section for them
  archives/<case>/...         input files, and <case>.zero written by the reference's compress_archive
  manifest.json               sizes, CRC-32s and SHA-256s of everything above

Block cases follow the reference's adversarial set (tests/stress.py:27-69), scaled to one block, plus
seeded cases shaped like the measured workloads.
"""
import hashlib
import json
import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "zero-compression_b200"))
import oracle as O  # noqa: E402
import datagen as G  # noqa: E402

LEVELS = (1, 5, 9)


def sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def block_cases():
    rng = random.Random(20261203)
    c = {}
    c["one_byte"] = b"x"
    c["three_bytes"] = b"abc"
    c["four_bytes"] = b"abcd"
    c["five_bytes"] = b"abcda"
    c["abcd_x3"] = b"abcdabcdabcd"
    c["zeros_64k"] = bytes(65536)
    c["one_value_40k"] = b"\xAB" * 40000
    c["period2_50k"] = b"ab" * 25000
    c["period3_48k"] = b"abc" * 16000
    c["period7_49k"] = b"abcdefg" * 7000
    p300 = bytes(rng.randrange(256) for _ in range(300))
    c["period300_60k"] = (p300 * 200)[:60000]
    c["random_30k"] = rng.randbytes(30000)
    x = bytearray(rng.randbytes(65536))
    x[40000:52000] = x[1000:13000]
    c["far_copy_64k"] = bytes(x)
    parts = []
    while sum(map(len, parts)) < 65536:
        k = rng.randrange(5)
        n = rng.randrange(1, 6000)
        if k == 0:
            parts.append(bytes([rng.randrange(256)]) * n)
        elif k == 1:
            parts.append(rng.randbytes(n))
        elif k == 2:
            parts.append(rng.randbytes(rng.randrange(1, 9)) * (n // 8 + 1))
        elif k == 3 and parts:
            parts.append(parts[rng.randrange(len(parts))][:n])
        else:
            parts.append(b"the quick brown fox " * (n // 20 + 1))
    c["mixed_64k"] = b"".join(parts)[:65536]
    for delta in (-1, 0):
        c["hello_block16%+d" % delta] = (b"hello world " * (65536 // 12 + 1))[: 65536 + delta]
    c["long_literals_64k"] = rng.randbytes(30000) + b"0123456789" * 200 + rng.randbytes(33536)
    b = bytearray()
    for n in list(range(4, 40)) + [100, 274, 275, 1000, 4095, 4096, 5000, 9000]:
        s = rng.randbytes(8)
        b += s + s[:4] * (n // 4)
    c["every_length"] = bytes(b)
    c["runs_then_noise"] = bytes(5000) + rng.randbytes(3000) + b"\x01" * 9000 + rng.randbytes(100)
    return c


GEN_CASES = [  # (name, kind, n, block_log, seed): inputs rebuilt from the seeded generator
    ("text_mix_64k", 0, 65536, 16, 11),
    ("lz_mix_64k", 1, 65536, 16, 12),
    ("text_mix_256k", 0, 262144, 18, 13),
    ("lz_mix_256k", 1, 262144, 18, 14),
    ("lz_mix_1m", 1, 1 << 20, 20, 15),
]

STREAM_CASES = {
    "empty": b"",
    "one": b"\x07",
    "two_syms": bytes([1, 2] * 50),
    "skewed": bytes([0] * 5000 + [1] * 3 + [2]),
    "all_256": bytes(range(256)) * 3,
    "single_symbol_long": b"\x33" * 10000,
    "short_63": bytes(range(63)),
    "short_65": bytes(i % 7 for i in range(65)),
}


def gen_input(kind, n, block_log, seed):
    return G.by_kind(kind, n, block_log, seed).tobytes()


def main():
    assert O.Ref.available(), "build oracle/_ref/libzref.so first (make -C oracle)"
    os.makedirs(os.path.join(HERE, "blocks"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "streams"), exist_ok=True)
    man = {"blocks": [], "streams": [], "archives": []}

    def add_block(name, data, source):
        ent = {"name": name, "source": source, "n": len(data), "crc32": O.Ref.crc32(data), "sha256": sha(data),
               "levels": {}}
        if source == "file":
            with open(os.path.join(HERE, "blocks", name + ".in"), "wb") as f:
                f.write(data)
        for lv in LEVELS:
            pay = O.Ref.compress_block(data, O.depth_for_level(lv))
            stored = len(pay) >= len(data)
            ent["levels"][str(lv)] = {"payload_len": len(pay), "stored": stored, "sha256": sha(pay)}
            if not stored:
                with open(os.path.join(HERE, "blocks", "%s.L%d.zb2" % (name, lv)), "wb") as f:
                    f.write(pay)
        man["blocks"].append(ent)

    for name, data in block_cases().items():
        add_block(name, data, "file")
    for name, kind, n, bl, seed in GEN_CASES:
        add_block(name, gen_input(kind, n, bl, seed), {"kind": kind, "n": n, "block_log": bl, "seed": seed})

    for name, sym in STREAM_CASES.items():
        sec = O.Ref.encode_stream(sym)
        with open(os.path.join(HERE, "streams", name + ".sym"), "wb") as f:
            f.write(sym)
        with open(os.path.join(HERE, "streams", name + ".sec"), "wb") as f:
            f.write(sec)
        man["streams"].append({"name": name, "n": len(sym), "sec_len": len(sec), "sha256": sha(sec)})

    # an archive of several files straddling blocks, written by the reference's compress_archive
    arch_dir = os.path.join(HERE, "archives", "three_files")
    src = os.path.join(arch_dir, "src")
    os.makedirs(os.path.join(src, "sub"), exist_ok=True)
    files = {
        "a.txt": gen_input(0, 70000, 16, 21),
        "sub/b.bin": gen_input(1, 90000, 16, 22),
        "sub/empty": b"",
        "z.rnd": gen_input(2, 20000, 16, 23),
    }
    for rel, data in files.items():
        with open(os.path.join(src, rel), "wb") as f:
            f.write(data)
    for lv in (1, 5):
        zpath = os.path.join(arch_dir, "three_files.L%d.zero" % lv)
        O.Ref.compress_archive([src], zpath, block_log=16, level=lv)
        with open(zpath, "rb") as f:
            z = f.read()
        man["archives"].append({"name": "three_files.L%d" % lv, "block_log": 16, "level": lv, "size": len(z),
                                "sha256": sha(z),
                                "files": {rel: {"size": len(d), "crc32": O.Ref.crc32(d), "sha256": sha(d)}
                                          for rel, d in files.items()}})
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(man, f, indent=1, sort_keys=True)
    print("wrote", len(man["blocks"]), "block cases,", len(man["streams"]), "streams,", len(man["archives"]), "archives")


if __name__ == "__main__":
    main()
