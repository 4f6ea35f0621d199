"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the two CPU oracles of the ZB2 block codec.

* ``Port``  -- ``oracle/liboracle.so``, the plain-C restatement of the reference CPU codec (zb2_oracle.c).
* ``Ref``   -- ``oracle/_ref/libzref.so``, the reference's own CPU codec compiled from its sources
  (src/codec.h, src/codec2.h, src/crc32.h, src/archive.h) by oracle/Makefile.  Absent when it was never
  built (it is not committed); callers check ``Ref.available()``.

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline leg of bench.py load this module; the
product path never does.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libzref.so")

_u8p = C.POINTER(C.c_uint8)
_u16p = C.POINTER(C.c_uint16)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)


def _p(a, t=_u8p):
    return a.ctypes.data_as(t)


def depth_for_level(level):
    """The CPU codec's hash chain depth for a level (src/main.cpp:45, 54)."""
    return 8 if level <= 1 else 256 if level >= 9 else 32


def payload_cap(n):
    return n + n // 2 + 4096


class _Lib:
    path = None
    prefix = None
    _lib = None

    @classmethod
    def available(cls):
        return os.path.exists(cls.path)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(cls.path):
                raise FileNotFoundError(f"{cls.path} is not built (make -C oracle)")
            cls._lib = C.CDLL(cls.path)
        return cls._lib


class Port(_Lib):
    """The C restatement."""
    path = PORT_SO

    @classmethod
    def crc32(cls, data, crc=0):
        a = np.frombuffer(bytes(data), np.uint8)
        f = cls.lib().zo_crc32_update
        f.restype = C.c_uint32
        return f(C.c_uint32(crc), _p(a), C.c_size_t(a.size))

    @classmethod
    def crc32_combine(cls, a, b, len_b):
        f = cls.lib().zo_crc32_combine
        f.restype = C.c_uint32
        return f(C.c_uint32(a), C.c_uint32(b), C.c_uint64(len_b))

    @classmethod
    def normalize(cls, counts, total):
        c = np.ascontiguousarray(counts, np.uint32)
        out = np.zeros(256, np.uint16)
        cls.lib().zo_normalize(_p(c, _u32p), C.c_uint32(total), _p(out, _u16p))
        return out

    @classmethod
    def encode_stream(cls, sym):
        a = np.frombuffer(bytes(sym), np.uint8)
        out = np.zeros(a.size + 1024, np.uint8)
        f = cls.lib().zo_encode_stream
        f.restype = C.c_size_t
        k = f(_p(a), C.c_uint32(a.size), _p(out))
        return out[:k].tobytes()

    @classmethod
    def decode_stream(cls, sec, n):
        a = np.frombuffer(bytes(sec), np.uint8)
        out = np.zeros(max(n, 1), np.uint8)
        f = cls.lib().zo_decode_stream
        f.restype = C.c_long
        k = f(_p(a), C.c_size_t(a.size), C.c_uint32(n), _p(out))
        return (None, -1) if k < 0 else (out[:n].tobytes(), k)

    @classmethod
    def parse(cls, data, depth):
        a = np.frombuffer(bytes(data), np.uint8)
        cap = a.size // 4 + 1
        ti, tm, td = (np.zeros(cap, np.uint32) for _ in range(3))
        f = cls.lib().zo_parse
        f.restype = C.c_uint32
        nt = f(_p(a), C.c_uint32(a.size), C.c_int(depth), _p(ti, _u32p), _p(tm, _u32p), _p(td, _u32p))
        return ti[:nt].copy(), tm[:nt].copy(), td[:nt].copy()

    @classmethod
    def build_payload(cls, data, ti, tm, td):
        a = np.frombuffer(bytes(data), np.uint8)
        ti, tm, td = (np.ascontiguousarray(x, np.uint32) for x in (ti, tm, td))
        out = np.zeros(payload_cap(a.size), np.uint8)
        f = cls.lib().zo_build_payload
        f.restype = C.c_size_t
        k = f(_p(a), C.c_uint32(a.size), _p(ti, _u32p), _p(tm, _u32p), _p(td, _u32p), C.c_uint32(ti.size), _p(out))
        return out[:k].tobytes()

    @classmethod
    def compress_block(cls, data, depth):
        """The payload bytes (the caller stores the block when len(payload) >= len(data))."""
        a = np.frombuffer(bytes(data), np.uint8)
        out = np.zeros(payload_cap(a.size), np.uint8)
        f = cls.lib().zo_compress_block
        f.restype = C.c_size_t
        k = f(_p(a), C.c_uint32(a.size), C.c_int(depth), _p(out))
        return out[:k].tobytes()

    @classmethod
    def decompress_block(cls, payload, n):
        a = np.frombuffer(bytes(payload), np.uint8)
        out = np.zeros(max(n, 1), np.uint8)
        f = cls.lib().zo_decompress_block
        f.restype = C.c_int
        rc = f(_p(a), C.c_size_t(a.size), _p(out), C.c_uint32(n))
        return None if rc else out[:n].tobytes()


class Ref(_Lib):
    """The reference's own CPU codec (compiled from its sources; not committed)."""
    path = REF_SO

    @classmethod
    def last_error(cls):
        f = cls.lib().zref_last_error
        f.restype = C.c_char_p
        return f().decode()

    @classmethod
    def crc32(cls, data, crc=0):
        a = np.frombuffer(bytes(data), np.uint8)
        f = cls.lib().zref_crc32_update
        f.restype = C.c_uint32
        return f(C.c_uint32(crc), _p(a), C.c_size_t(a.size))

    @classmethod
    def crc32_combine(cls, a, b, len_b):
        f = cls.lib().zref_crc32_combine
        f.restype = C.c_uint32
        return f(C.c_uint32(a), C.c_uint32(b), C.c_uint64(len_b))

    @classmethod
    def normalize(cls, counts, total):
        c = np.ascontiguousarray(counts, np.uint32)
        out = np.zeros(256, np.uint16)
        cls.lib().zref_normalize(_p(c, _u32p), C.c_uint32(total), _p(out, _u16p))
        return out

    @classmethod
    def encode_stream(cls, sym):
        a = np.frombuffer(bytes(sym), np.uint8)
        out = np.zeros(a.size + 1024, np.uint8)
        f = cls.lib().zref_encode_stream
        f.restype = C.c_long
        k = f(_p(a), C.c_uint32(a.size), _p(out), C.c_size_t(out.size))
        assert k >= 0
        return out[:k].tobytes()

    @classmethod
    def decode_stream(cls, sec, n):
        a = np.frombuffer(bytes(sec), np.uint8)
        out = np.zeros(max(n, 1), np.uint8)
        f = cls.lib().zref_decode_stream
        f.restype = C.c_long
        k = f(_p(a), C.c_size_t(a.size), C.c_uint32(n), _p(out))
        return (None, -1) if k < 0 else (out[:n].tobytes(), k)

    @classmethod
    def parse(cls, data, depth):
        a = np.frombuffer(bytes(data), np.uint8)
        cap = a.size // 4 + 1
        ti, tm, td = (np.zeros(cap, np.uint32) for _ in range(3))
        f = cls.lib().zref_parse
        f.restype = C.c_long
        nt = f(_p(a), C.c_uint32(a.size), C.c_int(depth), _p(ti, _u32p), _p(tm, _u32p), _p(td, _u32p), C.c_size_t(cap))
        assert nt >= 0
        return ti[:nt].copy(), tm[:nt].copy(), td[:nt].copy()

    @classmethod
    def compress_block(cls, data, depth):
        a = np.frombuffer(bytes(data), np.uint8)
        out = np.zeros(payload_cap(a.size), np.uint8)
        f = cls.lib().zref_compress_block
        f.restype = C.c_long
        k = f(_p(a), C.c_uint32(a.size), C.c_int(depth), _p(out), C.c_size_t(out.size))
        assert k >= 0
        return out[:k].tobytes()

    @classmethod
    def decompress_block(cls, payload, n):
        a = np.frombuffer(bytes(payload), np.uint8)
        out = np.zeros(max(n, 1), np.uint8)
        f = cls.lib().zref_decompress_block
        f.restype = C.c_int
        rc = f(_p(a), C.c_size_t(a.size), _p(out), C.c_uint32(n))
        return None if rc else out[:n].tobytes()

    @classmethod
    def cpu_compress(cls, data, block_log, depth, want_payloads=True):
        """The reference CpuCodec over all host threads: (methods, lens, payload list or None)."""
        a = np.frombuffer(data, np.uint8) if not isinstance(data, np.ndarray) else data
        B = 1 << block_log
        nb = (a.size + B - 1) // B
        methods = np.zeros(max(nb, 1), np.uint8)
        lens = np.zeros(max(nb, 1), np.uint32)
        stride = B + 8192
        out = np.zeros(nb * stride if want_payloads else 1, np.uint8)
        f = cls.lib().zref_cpu_compress
        f.restype = C.c_int
        rc = f(_p(a), C.c_size_t(a.size), C.c_uint32(block_log), C.c_int(depth), _p(methods), _p(lens, _u32p),
               _p(out) if want_payloads else None, C.c_size_t(stride))
        if rc:
            raise RuntimeError(cls.last_error())
        pays = None
        if want_payloads:
            pays = [out[b * stride: b * stride + int(lens[b])].tobytes() if methods[b] else None for b in range(nb)]
        return methods[:nb], lens[:nb], pays

    @classmethod
    def cpu_decompress(cls, comp, offs, comp_lens, methods, raw_lens):
        comp = np.ascontiguousarray(comp, np.uint8)
        offs = np.ascontiguousarray(offs, np.uint64)
        comp_lens = np.ascontiguousarray(comp_lens, np.uint32)
        methods = np.ascontiguousarray(methods, np.uint8)
        raw_lens = np.ascontiguousarray(raw_lens, np.uint32)
        out = np.zeros(max(int(raw_lens.sum()), 1), np.uint8)
        f = cls.lib().zref_cpu_decompress
        f.restype = C.c_int
        rc = f(_p(comp), _p(offs, _u64p), _p(comp_lens, _u32p), _p(methods), _p(raw_lens, _u32p),
               C.c_size_t(raw_lens.size), _p(out))
        if rc:
            raise RuntimeError(cls.last_error())
        return out[: int(raw_lens.sum())]

    @classmethod
    def compress_archive(cls, inputs, out_path, block_log=18, level=5):
        arr = (C.c_char_p * len(inputs))(*[os.fsencode(x) for x in inputs])
        f = cls.lib().zref_compress_archive
        f.restype = C.c_int
        if f(arr, C.c_int(len(inputs)), os.fsencode(out_path), C.c_uint32(block_log), C.c_int(level)):
            raise RuntimeError(cls.last_error())

    @classmethod
    def extract_archive(cls, path, out_dir):
        f = cls.lib().zref_extract_archive
        f.restype = C.c_int
        if f(os.fsencode(path), os.fsencode(out_dir)):
            raise RuntimeError(cls.last_error())

    @classmethod
    def test_archive(cls, path):
        """Raises RuntimeError with the reference's message when the archive does not check out."""
        f = cls.lib().zref_test_archive
        f.restype = C.c_int
        if f(os.fsencode(path)):
            raise RuntimeError(cls.last_error())

    @classmethod
    def hardware_threads(cls):
        f = cls.lib().zref_hardware_threads
        f.restype = C.c_uint
        return f()


def build():
    """Compile the oracles (the reference shim only where the reference tree exists)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)
