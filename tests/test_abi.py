"""The C ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")
SO = os.path.join(ROOT, "zero-compression_b200", "libzero_cuda.so")


def declared_symbols():
    names = set()
    for fn in os.listdir(INCLUDE):
        if not fn.endswith(".h"):
            continue
        with open(os.path.join(INCLUDE, fn)) as f:
            src = f.read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(zc_[a-z_0-9]+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def so():
    if not os.path.exists(SO):
        import __graft_entry__
        __graft_entry__.build()
    return SO


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("zc_open", "zc_close", "zc_compress", "zc_compress_batch", "zc_decompress", "zc_compress_device",
                 "zc_decompress_device", "zc_prepare", "zc_batch_bytes", "zc_batch_bytes_decode", "zc_name",
                 "zc_last_error", "zc_crc32", "zc_crc32_combine"):
        assert must in names


def test_library_exports_every_declared_symbol(so):
    lib = ctypes.CDLL(so)
    for name in sorted(declared_symbols()):
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (zc_[a-z_0-9]+)", out))
    assert declared_symbols() <= exported


def test_host_crc_combine_matches_oracle(so):
    import random
    import oracle as O
    import zero_cuda as Z
    if not O.Port.available():
        O.build()
    rng = random.Random(1)
    for _ in range(100):
        a, b, n = rng.getrandbits(32), rng.getrandbits(32), rng.randrange(0, 1 << 36)
        assert Z.crc32_combine(a, b, n) == O.Port.crc32_combine(a, b, n)



def test_library_resolves_every_symbol_at_load(so):
    """Loaded with immediate binding, and no symbol of the codec's own namespace left undefined."""
    ctypes.CDLL(so, mode=os.RTLD_NOW)
    out = subprocess.run(["nm", "-D", "--undefined-only", so], capture_output=True, text=True).stdout
    assert not re.findall(r"\b_ZN2zc\w+", out)


def test_binding_structs_match_the_header(tmp_path):
    """The ctypes structures of the binding have the header's fields at the header's offsets and sizes,
    as a C compiler lays them out (gcc on the header itself)."""
    import zero_cuda as Z
    structs = {"zc_shape": Z.Shape, "zc_archive_info": Z.ArchiveInfo, "zc_entry": Z._Entry, "zc_job": Z._Job}
    renamed = {"in_": "in"}  # (a Python keyword in the binding)
    src = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{os.path.join(INCLUDE, "zero_cuda.h")}"',
           "int main(void) {"]
    for cname, py in structs.items():
        src.append(f'  printf("{cname} (struct) %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            f = renamed.get(fname, fname)
            src.append(f'  printf("{cname} {fname} %zu %zu\\n", offsetof({cname}, {f}), sizeof((({cname} *)0)->{f}));')
    src += ["  return 0;", "}"]
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-o", str(exe), str(c)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            parts = line.split()
            got[(parts[0], parts[1])] = tuple(int(x) for x in parts[2:])
    for cname, py in structs.items():
        assert got[(cname, "(struct)")] == (ctypes.sizeof(py),), cname
        for fname, _ in py._fields_:
            field = getattr(py, fname)
            assert got[(cname, fname)] == (field.offset, field.size), (cname, fname)
