"""GPU parity: the CUDA codec against the oracle (the C restatement of the reference CPU codec, pinned by the
reference's golden vectors).  Integer work, so every comparison is bit-exact."""
import random

import numpy as np
import pytest

from conftest import block_input, block_payload, load_manifest

import oracle as O

pytestmark = pytest.mark.gpu
LEVELS = (1, 5, 9)


@pytest.fixture(scope="module")
def codec():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu")
    if not O.Port.available():
        O.build()
    import zero_cuda as Z
    c = Z.CudaCodec(level=5)
    yield c
    c.close()


def block_log_for(n):
    bl = 16
    while (1 << bl) < n:
        bl += 1
    return bl


def cpu_blocks(data, block_log, level):
    """The oracle's per-block (method, payload) for data cut into blocks."""
    B = 1 << block_log
    out = []
    for o in range(0, len(data), B):
        blk = data[o:o + B]
        pay = O.Port.compress_block(blk, O.depth_for_level(level))
        out.append((0, None) if len(pay) >= len(blk) else (1, pay))
    return out


def test_crc32(codec):
    rng = random.Random(7)
    for n in (0, 1, 7, 8, 9, 1000, 65536, 1 << 20, (1 << 20) + 13, 3 * (1 << 20) + 5):
        d = rng.randbytes(n)
        assert codec.crc32(d) == O.Port.crc32(d), n


def test_decode_golden(codec, manifest):
    for ent in manifest["blocks"]:
        data = block_input(ent)
        for lv in LEVELS:
            pay = block_payload(ent, lv)
            if pay is None:
                continue
            raw, crcs, errs = codec.decompress_arrays(pay, [0], [len(pay)], [1], [len(data)])
            assert errs[0] == 0, (ent["name"], lv)
            assert raw.tobytes() == data, (ent["name"], lv)
            assert crcs[0] == ent["crc32"], (ent["name"], lv)


def test_encode_golden(codec, manifest):
    for ent in manifest["blocks"]:
        data = block_input(ent)
        bl = block_log_for(len(data))
        for lv in LEVELS:
            want = ent["levels"][str(lv)]
            methods, lens, crcs, pay, offs = codec.compress_arrays(data, bl, level=lv)
            assert len(methods) == 1
            assert crcs[0] == ent["crc32"]
            if want["stored"]:
                assert methods[0] == 0, (ent["name"], lv)
            else:
                assert methods[0] == 1, (ent["name"], lv)
                got = pay[int(offs[0]): int(offs[0]) + int(lens[0])].tobytes()
                assert got == block_payload(ent, lv), (ent["name"], lv)


def test_stored_block_decode(codec):
    rng = random.Random(3)
    d = rng.randbytes(70000)
    raw, crcs, errs = codec.decompress_arrays(d, [0], [len(d)], [0], [len(d)])
    assert errs[0] == 0 and raw.tobytes() == d and crcs[0] == O.Port.crc32(d)


@pytest.mark.parametrize("block_log", [16, 18, 20])
@pytest.mark.parametrize("level", LEVELS)
def test_multi_block_parity(codec, block_log, level):
    """Workload-shaped data over several blocks: payloads byte-identical to the oracle, round trip exact."""
    import datagen as G
    B = 1 << block_log
    n = 3 * B + B // 3 + 17  # a short tail block
    parts = [G.text_mix(n // 3, 100 + block_log), G.lz_mix(n // 3, block_log, 200 + level),
             G.random_bytes(n - 2 * (n // 3), 300)]
    data = np.concatenate(parts).tobytes()
    methods, lens, crcs, pay, offs = codec.compress_arrays(data, block_log, level=level)
    want = cpu_blocks(data, block_log, level)
    assert len(methods) == len(want)
    comp, coffs = [], []
    at = 0
    for b, (m, p) in enumerate(want):
        blk = data[b * B:(b + 1) * B]
        assert crcs[b] == O.Port.crc32(blk)
        assert methods[b] == m, b
        if m:
            got = pay[int(offs[b]): int(offs[b]) + int(lens[b])].tobytes()
            assert got == p, b
            comp.append(got)
        else:
            assert lens[b] == len(blk)
            comp.append(blk)
        coffs.append(at)
        at += len(comp[-1])
    raw_lens = [min(B, len(data) - b * B) for b in range(len(want))]
    raw, dcrcs, errs = codec.decompress_arrays(b"".join(comp), coffs, [len(c) for c in comp], methods, raw_lens)
    assert not errs.any()
    assert raw.tobytes() == data
    assert list(dcrcs) == list(crcs)


def test_uneven_batch(codec):
    """Blocks of uneven sizes from many files in one call (partial tails, stored blocks)."""
    import datagen as G
    rng = random.Random(9)
    files = [G.by_kind(k % 3, rng.randrange(1, 150000), 18, 40 + k).tobytes() for k in range(12)]
    files.append(b"")
    files.append(b"xyz")
    B = 1 << 17
    blob, offs, lens = bytearray(), [], []
    for f in files:
        for o in range(0, len(f), B):
            offs.append(len(blob) + o)
            lens.append(min(B, len(f) - o))
        blob += f
        blob += b"\x55" * rng.randrange(0, 7)  # gaps between files
    data = bytes(blob)
    methods, clens, crcs, pay, poffs = codec.compress_batch_arrays(data, offs, lens, 17, level=5)
    for b, (o, l) in enumerate(zip(offs, lens)):
        blk = data[o:o + l]
        p = O.Port.compress_block(blk, 32)
        if len(p) >= l:
            assert methods[b] == 0
        else:
            assert methods[b] == 1 and pay[int(poffs[b]): int(poffs[b]) + int(clens[b])].tobytes() == p
        assert crcs[b] == O.Port.crc32(blk)


def test_damaged_payloads_never_fault(codec, manifest):
    """Random damage: the GPU decoder refuses or returns bytes; where the oracle accepts, the bytes agree."""
    ent = [e for e in manifest["blocks"] if e["name"] == "mixed_64k"][0]
    data = block_input(ent)
    pay = bytearray(block_payload(ent, 5))
    rng = random.Random(21)
    refused = 0
    for _ in range(200):
        b = bytearray(pay)
        for _ in range(rng.randrange(1, 40)):
            b[rng.randrange(len(b))] = rng.randrange(256)
        if rng.random() < 0.2:
            b = b[: rng.randrange(len(b))]
        raw, crcs, errs = codec.decompress_arrays(bytes(b), [0], [len(b)], [1], [len(data)], raise_on_damage=False)
        cpu = O.Port.decompress_block(bytes(b), len(data))
        if errs[0]:
            refused += 1
        elif cpu is not None:
            assert raw.tobytes() == cpu
    assert refused > 0
    # the codec still works after the damage
    raw, _, errs = codec.decompress_arrays(bytes(pay), [0], [len(pay)], [1], [len(data)])
    assert raw.tobytes() == data


def test_reference_api_shapes(codec):
    """compress / decompress through the zero::Codec-shaped methods."""
    import zero_cuda as Z
    import datagen as G
    data = G.lz_mix(300000, 18, 5).tobytes()
    outs = codec.compress(data, 18)
    B = 1 << 18
    ins = []
    for b, o in enumerate(outs):
        blk = data[b * B:(b + 1) * B]
        ins.append(Z.BlockIn(o.method, len(blk), o.data if o.method else blk))
    assert codec.decompress(ins) == data
    assert codec.batch_bytes(18) >= B and codec.batch_bytes_decode(18) >= B
    assert "GPU" in codec.name()


def test_graph_replay_matches_direct(codec):
    """Device-resident calls captured as CUDA graphs and replayed give the same bytes as direct launches."""
    import torch
    import datagen as G
    dev = torch.device("cuda", 0)
    bl, B = 16, 1 << 16
    data = np.concatenate([G.text_mix(200000, 61), G.random_bytes(70000, 62), G.lz_mix(150000, 16, 63)])
    n, nb = data.size, (data.size + B - 1) // B
    d_in = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
    d_in[:n] = torch.from_numpy(data).to(dev)
    offs = torch.arange(nb, dtype=torch.int64, device=dev) * B
    lens = torch.clamp(n - offs, max=B).to(torch.int32)
    stream = torch.cuda.Stream(device=dev)
    res = []
    for graphs in (False, True, True):
        codec.set_graphs(graphs)
        outs = dict(m=torch.zeros(nb, dtype=torch.uint8, device=dev), l=torch.zeros(nb, dtype=torch.int32, device=dev),
                    c=torch.zeros(nb, dtype=torch.int32, device=dev), o=torch.zeros(n + 64, dtype=torch.uint8, device=dev),
                    f=torch.zeros(nb, dtype=torch.int64, device=dev), t=torch.zeros(1, dtype=torch.int64, device=dev),
                    d=torch.zeros(n + 64, dtype=torch.uint8, device=dev), dc=torch.zeros(nb, dtype=torch.int32, device=dev),
                    e=torch.zeros(nb, dtype=torch.int32, device=dev))
        for _ in range(2):  # (a second call replays the captured graph)
            codec.compress_device(d_in, offs, lens, nb, bl, outs["m"], outs["l"], outs["c"], outs["o"], outs["f"],
                                  outs["t"], stream=stream.cuda_stream)
            codec.decompress_device(outs["o"], outs["f"], outs["l"], outs["m"], lens, nb, bl, outs["d"], offs,
                                    outs["dc"], outs["e"], stream=stream.cuda_stream)
        torch.cuda.synchronize()
        assert torch.equal(outs["d"][:n], d_in[:n]) and not outs["e"].any()
        tot = int(outs["t"].item())
        res.append((outs["m"].cpu(), outs["l"].cpu(), outs["c"].cpu(), outs["o"][:tot].cpu()))
    codec.set_graphs(False)
    for r in res[1:]:
        assert all(torch.equal(a, b) for a, b in zip(res[0], r))


def test_launch_shapes_never_change_bytes(codec):
    """Every decoder fill shape (ring size, warps per CTA, words per lane) and encoder match shape (cap, tile,
    lane-or-group threshold, deferral length) gives the same bytes; the autotuner's choice too.  Data with near and far
    matches, long runs and stored blocks."""
    import datagen as G
    default = {bl: codec.get_shape(bl, 5) for bl in (16, 18)}
    try:
        for bl in (16, 18):
            B = 1 << bl
            data = np.concatenate([G.lz_mix(3 * B + 777, bl, 70 + bl), G.text_mix(B, 71), np.zeros(B // 2, np.uint8),
                                   G.random_bytes(B // 3, 72), G.lz_mix(B // 2, bl, 73)])
            ref = cpu_blocks(data.tobytes(), bl, 5)
            ref_m = [m for m, _ in ref]
            ref_p = [p for _, p in ref]
            for cap, tile, dense, defer in ((8, 256, 256, 2), (12, 1024, 0, 0), (20, 512, 1025, 3), (32, 256, 64, 4),
                                            (32, 1024, 1025, 1), (16, 1024, 0, 4), (16, 1024, 1025, 0)):
                codec.set_shape(bl, 5, match_cap=cap, match_tile=tile, match_dense=dense, match_defer=defer)
                meth, lens, crcs, pay, offs = codec.compress_arrays(data, bl, level=5)
                assert list(meth) == ref_m, (cap, tile, dense, defer)
                for b, p in enumerate(ref_p):
                    if p is not None:
                        assert pay[int(offs[b]): int(offs[b]) + int(lens[b])].tobytes() == p, (cap, tile, dense, defer, b)
            codec.prepare(bl)
            raw_lens = [min(B, data.size - o) for o in range(0, data.size, B)]
            comp = [p if p is not None else data[o:o + B].tobytes() for p, o in zip(ref_p, range(0, data.size, B))]
            coffs = np.cumsum([0] + [len(c) for c in comp[:-1]])
            for rl in (11, 13, 15):
                for w in (1, 2, 4, 8):
                    for wd in (1, 2, 4):
                        if w * ((1 << rl) + 1408 * wd) > 227 * 1024:
                            continue
                        codec.set_shape(bl, 5, fill_ring_log=rl, fill_warps=w, fill_words=wd)
                        raw, dcrcs, errs = codec.decompress_arrays(b"".join(comp), coffs, [len(c) for c in comp],
                                                                   ref_m, raw_lens)
                        assert not errs.any() and raw.tobytes() == data.tobytes(), (bl, rl, w, wd)
            chosen = codec.autotune(data, bl, 5)
            assert chosen == codec.get_shape(bl, 5)
            meth, lens, crcs, pay, offs = codec.compress_arrays(data, bl, level=5)
            assert list(meth) == ref_m
            raw, _, errs = codec.decompress_arrays(b"".join(comp), coffs, [len(c) for c in comp], ref_m, raw_lens)
            assert not errs.any() and raw.tobytes() == data.tobytes()
    finally:
        for bl, s in default.items():
            codec.set_shape(bl, 5, **s)
        codec.prepare(18)


def test_host_calls_in_chunks_match_one_device_call(codec):
    """Host-buffer calls over more than one chunk (their copies overlap the other chunk's kernels) give
    the bytes one device-resident call gives, and round-trip."""
    import torch
    import datagen as G
    dev = torch.device("cuda", 0)
    bl, B = 18, 1 << 18
    data = np.concatenate([G.lz_mix(256 << 20, bl, 81), G.lz_mix(256 << 20, bl, 82), G.text_mix((8 << 20) + 12345, 83)])
    n, nb = data.size, (data.size + B - 1) // B
    meth, lens, crcs, pay, offs = codec.compress_arrays(data, bl, level=5)
    d_in = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
    d_in[:n] = torch.from_numpy(data).to(dev)
    doffs = torch.arange(nb, dtype=torch.int64, device=dev) * B
    dlens = torch.clamp(n - doffs, max=B).to(torch.int32)
    m = torch.zeros(nb, dtype=torch.uint8, device=dev)
    l = torch.zeros(nb, dtype=torch.int32, device=dev)
    c = torch.zeros(nb, dtype=torch.int32, device=dev)
    o = torch.zeros(n + 64, dtype=torch.uint8, device=dev)
    f = torch.zeros(nb, dtype=torch.int64, device=dev)
    t = torch.zeros(1, dtype=torch.int64, device=dev)
    codec.compress_device(d_in, doffs, dlens, nb, bl, m, l, c, o, f, t)
    torch.cuda.synchronize()
    assert np.array_equal(meth, m.cpu().numpy()) and np.array_equal(lens, l.cpu().numpy().astype(np.uint32))
    assert np.array_equal(crcs, c.cpu().numpy().astype(np.uint32))
    ho, hf = o.cpu().numpy(), f.cpu().numpy()
    for b in range(nb):
        if meth[b]:
            assert pay[int(offs[b]): int(offs[b]) + int(lens[b])].tobytes() == ho[hf[b]: hf[b] + int(lens[b])].tobytes()
    comp = [pay[int(offs[b]): int(offs[b]) + int(lens[b])] if meth[b] else data[b * B:(b + 1) * B] for b in range(nb)]
    blob = np.concatenate(comp)
    coffs = np.cumsum([0] + [x.size for x in comp[:-1]])
    raw, dcrcs, errs = codec.decompress_arrays(blob, coffs, [x.size for x in comp], meth,
                                               [min(B, n - b * B) for b in range(nb)])
    assert not errs.any() and np.array_equal(raw[:n], data) and np.array_equal(dcrcs, crcs)


@pytest.mark.parametrize("block_log,level", [(20, 1), (20, 9), (16, 5)])
def test_adversarial_multi_block_parity(codec, block_log, level):
    """Long zero runs, short periods, far copies and single-byte runs across several blocks: chains of equal
    hashes at full depth, 4096-byte matches, overlapping copies.  Payloads byte-identical to the oracle."""
    import datagen as G
    rng = np.random.default_rng(5150 + block_log + level)
    far = rng.integers(0, 256, 100000, dtype=np.uint8)
    runs = np.concatenate([np.full(int(k), int(v), np.uint8) for k, v in
                           zip(rng.integers(1, 300, 2000), rng.integers(0, 4, 2000))])
    parts = [np.zeros(300000, np.uint8), np.frombuffer(b"abc" * 70000, np.uint8), far,
             rng.integers(0, 256, 50000, dtype=np.uint8), far, runs, G.lz_mix(200000, block_log, 77),
             np.frombuffer(b"\x00\x01" * 40000, np.uint8)]
    data = np.concatenate(parts).tobytes()
    B = 1 << block_log
    methods, lens, crcs, pay, offs = codec.compress_arrays(data, block_log, level=level)
    want = cpu_blocks(data, block_log, level)
    comp = []
    for b, (m, p) in enumerate(want):
        blk = data[b * B:(b + 1) * B]
        assert methods[b] == m, b
        if m:
            got = pay[int(offs[b]): int(offs[b]) + int(lens[b])].tobytes()
            assert got == p, b
            comp.append(got)
        else:
            comp.append(blk)
    coffs = np.cumsum([0] + [len(c) for c in comp[:-1]])
    raw_lens = [min(B, len(data) - b * B) for b in range(len(want))]
    raw, dcrcs, errs = codec.decompress_arrays(b"".join(comp), coffs, [len(c) for c in comp], methods, raw_lens)
    assert not errs.any() and raw.tobytes() == data and list(dcrcs) == list(crcs)
