import hashlib
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for sub in ("oracle", "zero-compression_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def load_manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def block_input(ent):
    """The raw bytes of a golden block case: from its file, or rebuilt from the seeded generator."""
    if ent["source"] == "file":
        with open(os.path.join(GOLDEN, "blocks", ent["name"] + ".in"), "rb") as f:
            data = f.read()
    else:
        import datagen as G
        s = ent["source"]
        data = G.by_kind(s["kind"], s["n"], s["block_log"], s["seed"]).tobytes()
    assert sha(data) == ent["sha256"], "golden input changed: " + ent["name"]
    return data


def block_payload(ent, level):
    lv = ent["levels"][str(level)]
    if lv["stored"]:
        return None
    with open(os.path.join(GOLDEN, "blocks", "%s.L%d.zb2" % (ent["name"], level)), "rb") as f:
        pay = f.read()
    assert sha(pay) == lv["sha256"]
    return pay


@pytest.fixture(scope="session")
def manifest():
    return load_manifest()
