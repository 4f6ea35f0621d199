"""The drop-in check on the GPU: the reference's own archive pipeline (src/archive.h, in oracle/_ref/zero_dropin)
runs over the B200 codec.  Archives it writes must be byte-identical to the ones the reference CPU codec
writes for the same files, pass the reference reader's CRCs, and reference-written archives must extract
bit-exact through the GPU decoder."""
import hashlib
import os
import random
import shutil
import subprocess

import pytest

from conftest import GOLDEN, load_manifest

import oracle as O

pytestmark = pytest.mark.gpu
DROPIN = os.path.join(os.path.dirname(O.HERE), "oracle", "_ref", "zero_dropin")
need = pytest.mark.skipif(not (os.path.exists(DROPIN) and O.Ref.available()),
                          reason="oracle/_ref (built from the reference tree) is not present")


def run(*args):
    return subprocess.run([DROPIN] + [str(a) for a in args], capture_output=True, text=True, timeout=600)


def tree_digest(root):
    out = {}
    for dp, dn, fn in os.walk(root):
        for f in fn:
            p = os.path.join(dp, f)
            with open(p, "rb") as fh:
                out[os.path.relpath(p, root)] = hashlib.sha256(fh.read()).hexdigest()
    return out


@pytest.fixture(scope="module")
def tree(tmp_path_factory):
    import datagen as G
    root = tmp_path_factory.mktemp("src") / "data"
    (root / "sub" / "deeper").mkdir(parents=True)
    (root / "empty_dir").mkdir()
    files = {
        "a.txt": G.text_mix(300000, 5).tobytes(),
        "sub/b.bin": G.lz_mix(700000, 18, 6).tobytes(),
        "sub/deeper/c.rnd": G.random_bytes(200000, 7).tobytes(),
        "sub/zero": b"",
        "z_tiny": b"abc",
        "zeros": bytes(300000),
    }
    for rel, data in files.items():
        with open(root / rel, "wb") as f:
            f.write(data)
    # keep the modification times equal for both writers
    for dp, dn, fn in os.walk(root):
        for x in dn + fn:
            os.utime(os.path.join(dp, x), (1700000000, 1700000000))
    os.utime(root, (1700000000, 1700000000))
    return root


@need
@pytest.mark.parametrize("block,level", [(16, 1), (18, 5), (20, 9)])
def test_archives_identical_to_cpu_codec(tree, tmp_path, block, level):
    ours, ref = tmp_path / "ours.zero", tmp_path / "ref.zero"
    r = run("c", tree, "-o", ours, "--block", block, "--level", level)
    assert r.returncode == 0, r.stderr
    O.Ref.compress_archive([str(tree)], str(ref), block_log=block, level=level)
    assert ours.read_bytes() == ref.read_bytes()
    O.Ref.test_archive(str(ours))  # the reference CPU reader: every block and file CRC
    out = tmp_path / "x"
    O.Ref.extract_archive(str(ours), str(out))
    assert tree_digest(out / "data") == tree_digest(tree)


@need
def test_reference_archives_decode_on_gpu(tree, tmp_path):
    ref = tmp_path / "ref.zero"
    O.Ref.compress_archive([str(tree)], str(ref), block_log=18, level=9)
    r = run("t", ref)
    assert r.returncode == 0 and "OK" in r.stdout, r.stderr
    r = run("x", ref, "-o", tmp_path / "x")
    assert r.returncode == 0, r.stderr
    assert tree_digest(tmp_path / "x" / "data") == tree_digest(tree)


@need
def test_golden_archives_decode_on_gpu(tmp_path):
    man = load_manifest()
    for ent in man["archives"]:
        path = os.path.join(GOLDEN, "archives", "three_files", ent["name"] + ".zero")
        r = run("t", path)
        assert r.returncode == 0, (ent["name"], r.stderr)
        out = tmp_path / ent["name"]
        r = run("x", path, "-o", out)
        assert r.returncode == 0, r.stderr
        for rel, f in ent["files"].items():
            with open(out / "src" / rel, "rb") as fh:
                assert hashlib.sha256(fh.read()).hexdigest() == f["sha256"], rel


@need
def test_damaged_archive_is_refused(tree, tmp_path):
    good = tmp_path / "good.zero"
    assert run("c", tree, "-o", good, "--block", 16).returncode == 0
    data = bytearray(good.read_bytes())
    rng = random.Random(4)
    refused = 0
    for i in range(30):
        b = bytearray(data)
        for _ in range(rng.randrange(1, 30)):
            b[rng.randrange(24, len(b) - 200)] = rng.randrange(256)
        bad = tmp_path / f"bad{i}.zero"
        bad.write_bytes(bytes(b))
        r = run("t", bad)
        txt = r.stdout + r.stderr
        assert "device" not in txt.lower() or r.returncode != 0
        refused += r.returncode != 0
    assert refused >= 25
    assert run("t", good).returncode == 0  # and the GPU still works


@need
def test_bench_entry_point(tree, tmp_path):
    r = run("bench", tree / "sub" / "b.bin", "--block", 18, "--level", 5)
    assert r.returncode == 0 and "identical" in r.stdout, r.stdout + r.stderr


@need
@pytest.mark.parametrize("block,level", [(16, 1), (18, 5), (20, 9)])
def test_container_on_gpu_equals_compress_archive(tree, tmp_path, block, level):
    """`zero c` with the whole container written on the GPU (zc_archive_write from C++, the entries as the
    reference collects them): the file equals compress_archive's with the reference CPU codec, and
    zc_archive_extract and the reference reader both check it."""
    ours, ref = tmp_path / "c2.zero", tmp_path / "ref.zero"
    r = run("c2", tree, "-o", ours, "--block", block, "--level", level)
    assert r.returncode == 0, r.stderr
    O.Ref.compress_archive([str(tree)], str(ref), block_log=block, level=level)
    assert ours.read_bytes() == ref.read_bytes()
    r = run("t2", ours)
    assert r.returncode == 0 and "OK" in r.stdout, r.stderr
    O.Ref.test_archive(str(ours))


def run_env(env, *args):
    return subprocess.run([DROPIN] + [str(a) for a in args], capture_output=True, text=True, timeout=600,
                          env=dict(os.environ, **env))


@need
@pytest.mark.parametrize("fail_after", [0, 3])
def test_safe_codec_finishes_the_job_after_a_device_failure(tree, tmp_path, fail_after):
    """SafeCudaCodec, the reference's SafeCodec contract (src/safe_codec.h:10-50) over the B200 codec.
    ZC_FAIL_AFTER=n makes the context's (n+1)-th codec call fail with ZC_E_DEVICE before it launches
    anything: that batch and every later one go to the reference's CPU codec, the report says so once,
    and the archive is still the one compress_archive writes; extraction across the same failure (the
    first batch, or one in the middle of the job) is bit-exact."""
    ours, ref = tmp_path / "safe.zero", tmp_path / "ref.zero"
    env = {"ZC_FAIL_AFTER": str(fail_after)}
    r = run_env(env, "c", tree, "-o", ours, "--block", 16, "--level", 5, "--safe", "--batch-kib", 256)
    assert r.returncode == 0, r.stderr
    assert r.stderr.count("GPU stopped working") == 1 and "ZC_FAIL_AFTER" in r.stderr, r.stderr
    O.Ref.compress_archive([str(tree)], str(ref), block_log=16, level=5)
    assert ours.read_bytes() == ref.read_bytes()
    out = tmp_path / "x"
    r = run_env(env, "x", ours, "-o", out, "--safe", "--batch-kib", 256)
    assert r.returncode == 0, r.stderr
    assert r.stderr.count("GPU stopped working") == 1, r.stderr
    assert tree_digest(out / "data") == tree_digest(tree)


@need
def test_safe_codec_without_failure_stays_on_the_gpu(tree, tmp_path):
    ours, ref = tmp_path / "safe.zero", tmp_path / "ref.zero"
    r = run_env({}, "c", tree, "-o", ours, "--block", 18, "--level", 9, "--safe", "--batch-kib", 512)
    assert r.returncode == 0 and "GPU" not in r.stderr, r.stderr
    O.Ref.compress_archive([str(tree)], str(ref), block_log=18, level=9)
    assert ours.read_bytes() == ref.read_bytes()
    r = run_env({}, "t", ours, "--safe")
    assert r.returncode == 0 and "OK" in r.stdout and "GPU" not in r.stderr, r.stderr


@need
def test_safe_codec_damaged_block_is_redone_on_the_cpu(tree, tmp_path):
    """A damaged payload is a data error, not a device failure: the GPU refuses the batch (ZC_E_DATA), the
    CPU codec decodes it again and reports the damage with the reference's own message, and the GPU is not
    given up."""
    good = tmp_path / "good.zero"
    O.Ref.compress_archive([str(tree)], str(good), block_log=16, level=5)
    data = bytearray(good.read_bytes())
    assert data[24 + 8] == 1  # block 0 is ZB2-coded (its record's method byte)
    data[24 + 16:24 + 20] = b"\xff\xff\xff\x7f"  # its token count: far above what the block can hold
    bad = tmp_path / "bad.zero"
    bad.write_bytes(bytes(data))
    with pytest.raises(RuntimeError) as cpu_err:
        O.Ref.test_archive(str(bad))
    r = run_env({}, "t", bad, "--safe")
    assert r.returncode != 0
    assert str(cpu_err.value) in r.stderr, (str(cpu_err.value), r.stderr)
    assert "GPU stopped working" not in r.stderr
