"""The serving loop: jobs of different kinds, sizes, block sizes and levels give the same bytes alone and
in a mix (bit-exact: integer work), extract / test round trips, admission by a memory budget."""
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu")
    import zero_cuda as Z
    import datagen as G
    return Z, G


def inputs(G):
    rng = random.Random(77)
    out = []
    for i in range(9):
        n = int(np.exp(rng.uniform(np.log(4096), np.log(3 << 20))))
        kind = i % 3
        bl = (16, 18, 20)[(i // 3) % 3]
        lv = (1, 5, 9)[i % 3]
        out.append((G.by_kind(kind, n, bl, 300 + i), bl, lv))
    out.append((np.zeros(0, np.uint8), 18, 5))  # an empty job
    return out


def result(h):
    nb = h.nb
    return (h.methods[:nb].copy(), h.lens[:nb].copy(), h.crcs[:nb].copy(),
            [h.payloads[int(o): int(o) + int(l)].tobytes() if m else b"" for m, l, o in
             zip(h.methods[:nb], h.lens[:nb], h.offs[:nb])])


def same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3])) and a[3] == b[3]


def test_compress_alone_and_in_the_mix(env):
    Z, G = env
    jobs = inputs(G)
    srv = Z.Server(budget_bytes=256 << 20)
    alone = []
    for data, bl, lv in jobs:
        alone.append(result(srv.wait(srv.compress(data, bl, lv))))
    hs = [srv.compress(data, bl, lv) for data, bl, lv in jobs]  # all in flight together
    mixed = [result(srv.wait(h)) for h in hs]
    st = srv.stats()
    srv.close()
    assert st["arena_used"] == 0
    with Z.CudaCodec() as codec:  # and the plain path agrees
        for (data, bl, lv), a, m in zip(jobs, alone, mixed):
            assert same(a, m)
            if data.size:
                meth, lens, crcs, pay, offs = codec.compress_arrays(data, bl, level=lv)
                ref = (meth, lens, crcs, [pay[int(o): int(o) + int(l)].tobytes() if mm else b""
                                          for mm, l, o in zip(meth, lens, offs)])
                assert same(a, ref)


def test_extract_and_test_jobs(env):
    Z, G = env
    jobs = [j for j in inputs(G) if j[0].size]
    srv = Z.Server(budget_bytes=512 << 20)
    comp = [srv.wait(srv.compress(d, bl, lv)) for d, bl, lv in jobs]
    hx, ht = [], []
    for (d, bl, lv), h in zip(jobs, comp):
        blob, clens, rlens = Z.record_bodies(d, h.methods[:h.nb], h.lens[:h.nb], h.payloads, h.offs[:h.nb], bl)
        hx.append(srv.extract(blob, clens, h.methods[:h.nb], rlens, bl))
        ht.append(srv.test(blob, clens, h.methods[:h.nb], rlens, h.crcs[:h.nb], bl))
    for (d, bl, lv), x, t, c in zip(jobs, hx, ht, comp):
        srv.wait(x)
        srv.wait(t)
        assert x.raw[:d.size].tobytes() == d.tobytes()
        assert np.array_equal(x.crcs[:c.nb], c.crcs[:c.nb]) and np.array_equal(t.crcs[:c.nb], c.crcs[:c.nb])
    # a damaged archive: the test job reports it, the server goes on
    d, bl, lv = jobs[1]
    c = comp[1]
    blob, clens, rlens = Z.record_bodies(d, c.methods[:c.nb], c.lens[:c.nb], c.payloads, c.offs[:c.nb], bl)
    bad = blob.copy()
    bad[len(bad) // 3: len(bad) // 3 + 40] ^= 0x5A
    t = srv.wait(srv.test(bad, clens, c.methods[:c.nb], rlens, c.crcs[:c.nb], bl), raise_on_error=False)
    assert t.status == Z.ZC_E_DATA
    x = srv.wait(srv.extract(blob, clens, c.methods[:c.nb], rlens, bl))
    assert x.raw[:d.size].tobytes() == d.tobytes()
    srv.close()


def test_admission_by_budget(env):
    Z, G = env
    srv = Z.Server(budget_bytes=6 << 20, max_batch_bytes=2 << 20)
    data = [G.lz_mix(2 << 20, 18, 900 + i) for i in range(8)]  # 16 MiB of jobs through a 6 MiB arena
    hs = [srv.compress(d, 18, 5) for d in data]
    res = [result(srv.wait(h)) for h in hs]
    assert srv.stats()["arena_used"] == 0 and srv.stats()["jobs_done"] == 8
    with pytest.raises(Z.ArgError):
        srv.compress(G.lz_mix(8 << 20, 18, 1), 18, 5)  # could never fit
    srv.close()
    with Z.CudaCodec() as codec:
        for d, r in zip(data, res):
            meth, lens, crcs, pay, offs = codec.compress_arrays(d, 18, level=5)
            assert np.array_equal(meth, r[0]) and np.array_equal(crcs, r[2])
