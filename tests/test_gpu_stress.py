"""The reference's adversarial set at its stated sizes (tests/stress.py:27-69), on the GPU: every data set at
blocks 16 / 18 / 20 and levels 1 / 5 / 9.  The data are regenerated here from this file's own seeded
generators with the shapes and sizes that script names (8 MiB of zeros, one value, short and long periods,
4 MiB random, a far copy, 4 MiB of mixed runs, exactly a block and one byte either side at each block size,
a long literal run, matches of every length up to 70000 bytes).

Each GPU payload must equal the reference CPU codec's (libzref, compiled from the reference's sources) byte
for byte, the stored / coded choice must be the same, and the blocks must decode bit-exact through both
codecs: the GPU decoder, and the reference's CPU decoder on the GPU's payloads (stress.py:102-118)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
MiB = 1 << 20
need_ref = pytest.mark.skipif(not O.Ref.available(), reason="oracle/_ref/libzref.so (the reference) is not built")


def data_sets():
    rng = np.random.default_rng(20261204)
    rb = lambda n: rng.integers(0, 256, n, dtype=np.uint8).tobytes()
    d = {
        "empty": b"",
        "one byte": b"x",
        "three bytes": b"abc",
        "four bytes": b"abcd",
        "zeros 8 MiB": bytes(8 * MiB),
        "one value 3 MiB": b"\x5c" * (3 * MiB),
        "period 2": b"qz" * (2 * MiB),
        "period 3": b"k9#" * MiB,
        "period 7": b"period7" * (MiB // 2),
        "period 300": rb(300) * 8000,
        "random 4 MiB": rb(4 * MiB),
    }
    far = bytearray(rb(2 * MiB))
    far[MiB:MiB + MiB // 2] = far[:MiB // 2]
    d["far copy"] = bytes(far)
    parts, total = [], 0
    while total < 4 * MiB:  # long runs, short runs, noise, repeats and text side by side
        k, n = int(rng.integers(5)), int(rng.integers(1, 70000))
        if k == 0:
            p = bytes([int(rng.integers(256))]) * n
        elif k == 1:
            p = rb(n)
        elif k == 2:
            p = rb(int(rng.integers(1, 9))) * (n // 8 + 1)
        elif k == 3 and parts:
            p = parts[int(rng.integers(len(parts)))][:n]
        else:
            p = b"pack my box with five dozen jugs " * (n // 33 + 1)
        parts.append(p)
        total += len(p)
    d["mixed"] = b"".join(parts)
    for bl in (16, 18, 20):
        for delta in (-1, 0, 1):
            d["block %d %+d" % (bl, delta)] = (b"block edges " * ((1 << bl) // 12 + 1))[:(1 << bl) + delta]
    d["long literals"] = rb(200000) + b"0123456789" * 200 + rb(200000)
    ev = bytearray()
    for n in list(range(4, 40)) + [100, 274, 275, 1000, 4095, 4096, 5000, 70000]:
        s = rb(8)
        ev += s + s[:4] * (n // 4)
    d["every length"] = bytes(ev)
    return d


SETS = data_sets()


@pytest.fixture(scope="module")
def codecs():
    import zero_cuda as Z
    cs = {lv: Z.CudaCodec(level=lv) for lv in (1, 5, 9)}
    yield cs
    for c in cs.values():
        c.close()


@need_ref
@pytest.mark.parametrize("name", list(SETS))
def test_stress_set_matches_reference_codec(codecs, name):
    data = SETS[name]
    for block_log in (16, 18, 20):
        B = 1 << block_log
        nb = (len(data) + B - 1) // B
        raw_lens = [min(B, len(data) - b * B) for b in range(nb)]
        for level in (1, 5, 9):
            where = (name, block_log, level)
            methods, lens, crcs, pay, offs = codecs[level].compress_arrays(data, block_log)
            assert len(methods) == nb
            r_methods, r_lens, r_pays = O.Ref.cpu_compress(data, block_log, O.depth_for_level(level))
            assert list(methods) == list(r_methods), where
            bodies = []
            for b in range(nb):
                blk = data[b * B:(b + 1) * B]
                if methods[b]:
                    body = pay[int(offs[b]): int(offs[b]) + int(lens[b])].tobytes()
                    assert body == r_pays[b], (where, b)
                else:
                    body = blk
                assert int(crcs[b]) == O.Ref.crc32(blk), (where, b)
                bodies.append(body)
            if not nb:
                continue
            coffs = np.concatenate([[0], np.cumsum([len(x) for x in bodies])[:-1]]).astype(np.uint64)
            blob = b"".join(bodies)
            raw, dcrcs, errs = codecs[level].decompress_arrays(blob, coffs, [len(x) for x in bodies], methods, raw_lens)
            assert not errs.any() and raw.tobytes() == data, where
            assert list(dcrcs) == list(crcs), where
            back = O.Ref.cpu_decompress(np.frombuffer(blob, np.uint8), coffs, [len(x) for x in bodies], methods,
                                        raw_lens)
            assert back.tobytes() == data, where
