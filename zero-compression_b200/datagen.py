"""Seeded synthetic inputs for the ZB2 codec workloads (ctypes over csrc/datagen.c, built as libzgen.so).

text_mix(n, seed)            -- alternating 4 KiB text / repeat segments (Zipf word text + back copies)
lz_mix(n, block_log, seed)   -- literal runs + log-uniform matches, offsets up to the block size
random_bytes(n, seed)        -- uniform bytes (stored blocks)
file_plan(count, lo, hi, seed) -- per-file sizes (log-uniform) and generator kinds for many-file archives
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libzgen.so")
_lib = None


def _l():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            raise FileNotFoundError(f"{SO} is not built (python -c 'import __graft_entry__ as g; g.build()')")
        _lib = C.CDLL(SO)
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def text_mix(n, seed=1, out=None):
    out = np.empty(n, np.uint8) if out is None else out
    _l().zg_text_mix(_ptr(out), C.c_size_t(n), C.c_uint64(seed))
    return out


def lz_mix(n, block_log=18, seed=1, out=None):
    out = np.empty(n, np.uint8) if out is None else out
    _l().zg_lz_mix(_ptr(out), C.c_size_t(n), C.c_uint32(block_log), C.c_uint64(seed))
    return out


def random_bytes(n, seed=1, out=None):
    out = np.empty(n, np.uint8) if out is None else out
    _l().zg_random(_ptr(out), C.c_size_t(n), C.c_uint64(seed))
    return out


def file_plan(count, lo=1 << 10, hi=64 << 20, seed=1):
    sizes = np.zeros(count, np.uint64)
    kinds = np.zeros(count, np.uint8)
    _l().zg_file_plan(sizes.ctypes.data_as(C.POINTER(C.c_uint64)), _ptr(kinds), C.c_size_t(count),
                      C.c_uint64(lo), C.c_uint64(hi), C.c_uint64(seed))
    return sizes, kinds


def by_kind(kind, n, block_log, seed):
    """Generator kind 0 text mix, 1 LZ mix, 2 random."""
    if kind == 0:
        return text_mix(n, seed)
    if kind == 1:
        return lz_mix(n, block_log, seed)
    return random_bytes(n, seed)
