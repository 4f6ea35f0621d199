"""zc_decompress_noalloc, the decoder that allocates no device memory (for callers that cannot call
cudaMalloc, e.g. a plugin whose host process budgets every byte of device memory), against the regular
device entry point zc_decompress_device.  Called through the C ABI, twice in a row on different inputs,
bit-exact (integer work: the tolerance is zero).  Collected last on purpose (its name), and self-contained
so it passes alone in a fresh process as well."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ZC_E_ARG = 4
SCRATCH = 16 << 20
META_BYTES = 76  # per block: the framing record


def need(nb, block_log):
    """Scratch bytes a call of nb blocks takes (the formula of include/zero_cuda.h)."""
    up = lambda x: (x + 255) & ~255
    B = 1 << block_log
    TC, EC = B // 4 + 16, B // 5 + 64
    return 256 + up(nb * B) + 3 * up(nb * TC) + up(nb * EC) + up(nb * META_BYTES) + 4 * up(nb * TC * 4)


def limit(block_log):
    nb = 0
    while need(nb + 1, block_log) <= SCRATCH:
        nb += 1
    return nb


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu")
    import zero_cuda as Z
    lib = Z.lib()
    lib.zc_decompress_noalloc.argtypes = [C.c_void_p] * 5 + [C.c_uint32, C.c_uint32] + [C.c_void_p] * 5
    lib.zc_decompress_noalloc.restype = C.c_int
    codec = Z.CudaCodec(level=5)
    yield torch, lib, codec
    codec.close()


def make_blocks(torch, codec, data, block_log):
    """Compress with the codec; return device tensors describing the blocks as an archive holds them."""
    B = 1 << block_log
    methods, lens, _, pay, offs = codec.compress_arrays(data, block_log)
    bodies, coffs, at = [], [], 0
    for b in range(len(methods)):
        blk = data[b * B:(b + 1) * B]
        body = pay[int(offs[b]): int(offs[b]) + int(lens[b])].tobytes() if methods[b] else blk
        bodies.append(body)
        coffs.append(at)
        at += len(body)
    raw = [min(B, len(data) - b * B) for b in range(len(methods))]
    dev = torch.device("cuda", 0)
    comp = torch.zeros(at + 64, dtype=torch.uint8, device=dev)
    comp[:at] = torch.frombuffer(bytearray(b"".join(bodies)), dtype=torch.uint8).to(dev)
    t = lambda a, dt: torch.tensor(np.asarray(a).astype(dt), device=dev)
    return dict(comp=comp, coffs=t(coffs, np.int64), clens=t([len(x) for x in bodies], np.int32),
                methods=t(methods, np.uint8), raw=t(raw, np.int32),
                ooffs=t(np.concatenate([[0], np.cumsum(raw)[:-1]]), np.int64), n=len(data), nb=len(methods))


def decode_both(torch, lib, codec, blk, block_log):
    dev = torch.device("cuda", 0)
    nb, n = blk["nb"], blk["n"]
    res = []
    for which in ("device", "noalloc"):
        out = torch.full((n + 64,), 0xA5, dtype=torch.uint8, device=dev)
        crcs = torch.zeros(nb, dtype=torch.int32, device=dev)
        err = torch.full((nb,), 7, dtype=torch.int32, device=dev)
        if which == "device":
            codec.decompress_device(blk["comp"], blk["coffs"], blk["clens"], blk["methods"], blk["raw"], nb, block_log,
                                    out, blk["ooffs"], crcs, err)
        else:
            rc = lib.zc_decompress_noalloc(blk["comp"].data_ptr(), blk["coffs"].data_ptr(), blk["clens"].data_ptr(),
                                           blk["methods"].data_ptr(), blk["raw"].data_ptr(), nb, block_log,
                                           out.data_ptr(), blk["ooffs"].data_ptr(), crcs.data_ptr(), err.data_ptr(),
                                           None)
            assert rc == 0
        torch.cuda.synchronize()
        res.append((out[:n].cpu().numpy().tobytes(), crcs.cpu().numpy(), err.cpu().numpy()))
    return res


def test_noalloc_matches_device_entry_point_twice(env):
    torch, lib, codec = env
    import datagen as G
    block_log = 18
    inputs = [
        np.concatenate([G.text_mix(300000, 31), G.lz_mix(500000, 18, 32), G.random_bytes(90000, 33)]).tobytes(),
        np.concatenate([G.lz_mix(700000, 18, 34), np.zeros(40000, np.uint8), G.text_mix(123457, 35)]).tobytes(),
    ]
    for data in inputs:  # two calls in a row, different inputs: the shared scratch keeps the last call's bytes
        blk = make_blocks(torch, codec, data, block_log)
        assert need(blk["nb"], block_log) <= SCRATCH
        (o1, c1, e1), (o2, c2, e2) = decode_both(torch, lib, codec, blk, block_log)
        assert o2 == o1 == data
        assert np.array_equal(c2, c1) and np.array_equal(e2, e1) and not e1.any()


def test_noalloc_damaged_block_status_matches(env):
    torch, lib, codec = env
    import datagen as G
    block_log = 16
    data = G.lz_mix(200000, 16, 41).tobytes()
    blk = make_blocks(torch, codec, data, block_log)
    blk["comp"][30:60] ^= 0x5A  # damage inside the first payload
    (o1, c1, e1), (o2, c2, e2) = decode_both(torch, lib, codec, blk, block_log)
    assert np.array_equal(e2, e1) and e1[0] != 0
    good = [b for b in range(blk["nb"]) if e1[b] == 0]
    assert np.array_equal(c2[good], c1[good])


def test_noalloc_limits_are_the_documented_ones():
    assert [limit(bl) for bl in (16, 17, 18, 19, 20)] == [42, 21, 10, 5, 2]


@pytest.mark.parametrize("block_log", [16, 18, 20])
def test_noalloc_exactly_at_the_limit(env, block_log):
    """nb = the limit decodes; nb = the limit + 1 is refused before anything runs."""
    torch, lib, codec = env
    import datagen as G
    nb = limit(block_log)
    data = G.lz_mix(nb << block_log, block_log, 50 + block_log).tobytes()
    blk = make_blocks(torch, codec, data, block_log)
    assert blk["nb"] == nb
    (o1, c1, e1), (o2, c2, e2) = decode_both(torch, lib, codec, blk, block_log)
    assert o2 == o1 == data and np.array_equal(c2, c1) and not e2.any()
    check_refused(torch, lib, block_log, nb + 1)


def check_refused(torch, lib, block_log, nb):
    dev = torch.device("cuda", 0)
    z64 = torch.zeros(nb, dtype=torch.int64, device=dev)
    z32 = torch.zeros(nb, dtype=torch.int32, device=dev)
    out = torch.zeros(64, dtype=torch.uint8, device=dev)
    err = torch.full((nb,), 3, dtype=torch.int32, device=dev)
    rc = lib.zc_decompress_noalloc(out.data_ptr(), z64.data_ptr(), z32.data_ptr(), out.data_ptr(), z32.data_ptr(), nb,
                                   block_log, out.data_ptr(), z64.data_ptr(), None, err.data_ptr(), None)
    assert rc == ZC_E_ARG
    torch.cuda.synchronize()
    assert (err.cpu() == 3).all()  # nothing was touched
