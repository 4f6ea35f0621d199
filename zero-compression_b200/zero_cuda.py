"""Python binding of the B200 ZB2 block codec (ctypes over libzero_cuda.so, the C ABI of include/zero_cuda.h).

It mirrors the reference's codec interface ``zero::Codec`` (src/archive.h:45-69):

    codec = CudaCodec(level=5)          # GpuCodec + choose_codec, src/main.cpp:36-57 / src/gpu_codec.h:63-86
    outs = codec.compress(data, 18)     # -> [BlockOut(method, data)], one per block (src/archive.h:60)
    raw = codec.decompress(blocks)      # [BlockIn(method, raw_len, data)] -> raw bytes (src/archive.h:63)
    codec.batch_bytes(18), codec.batch_bytes_decode(18), codec.prepare(18), codec.name()

Errors follow the reference's split (src/safe_codec.h:36-49): ``DataError`` for damaged input (zb::Error:
the caller may retry on a CPU codec, which reports what is wrong) and ``DeviceError`` for a failed GPU
(gpu::Error).  There is no CPU path here: without the built library or a CUDA device every call raises.
"""
import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libzero_cuda.so")

ZC_OK, ZC_E_DATA, ZC_E_DEVICE, ZC_E_NOMEM, ZC_E_ARG = 0, 1, 2, 3, 4
STORED, ZB2 = 0, 1

_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_vp = C.c_void_p


class ZcError(RuntimeError):
    code = -1


class DataError(ZcError):
    """Damaged input or an impossible result (the reference's zb::Error)."""
    code = ZC_E_DATA


class DeviceError(ZcError):
    """The GPU failed (the reference's gpu::Error)."""
    code = ZC_E_DEVICE


class NoMemError(DeviceError):
    code = ZC_E_NOMEM


class ArgError(ZcError, ValueError):
    code = ZC_E_ARG


_lib = None


def lib():
    """The loaded C library; raises when it was not built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            raise ImportError(f"{SO} is not built: run __graft_entry__.build() (make -C zero-compression_b200/csrc)")
        L = C.CDLL(SO)
        L.zc_open.argtypes = [C.POINTER(_vp), C.c_int]
        L.zc_close.argtypes = [_vp]
        L.zc_last_error.argtypes = [_vp]
        L.zc_last_error.restype = C.c_char_p
        L.zc_name.argtypes = [_vp]
        L.zc_name.restype = C.c_char_p
        L.zc_prepare.argtypes = [_vp, C.c_uint32, C.c_int]
        L.zc_batch_bytes.argtypes = [_vp, C.c_uint32]
        L.zc_batch_bytes.restype = C.c_size_t
        L.zc_batch_bytes_decode.argtypes = [_vp, C.c_uint32]
        L.zc_batch_bytes_decode.restype = C.c_size_t
        L.zc_compress.argtypes = [_vp, _vp, C.c_size_t, C.c_uint32, C.c_int, _vp, _vp, _vp, _vp, C.c_size_t, _vp]
        L.zc_compress_batch.argtypes = [_vp, _vp, _vp, _vp, C.c_uint32, C.c_uint32, C.c_int, _vp, _vp, _vp, _vp,
                                        C.c_size_t, _vp]
        L.zc_decompress.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, C.c_uint32, _vp, _vp, _vp]
        L.zc_compress_device.argtypes = [_vp, _vp, _vp, _vp, C.c_uint32, C.c_uint32, C.c_int, _vp, _vp, _vp, _vp,
                                         C.c_size_t, _vp, _vp, _vp]
        L.zc_decompress_device.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, C.c_uint32, C.c_uint32, _vp, _vp, _vp, _vp,
                                           _vp]
        L.zc_crc32.argtypes = [_vp, _vp, C.c_size_t, _u32p]
        L.zc_crc32_combine.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64]
        L.zc_crc32_combine.restype = C.c_uint32
        L.zc_launch_count.argtypes = [_vp]
        L.zc_launch_count.restype = C.c_uint64
        L.zc_profile.argtypes = [_vp, C.c_int]
        L.zc_set_graphs.argtypes = [_vp, C.c_int]
        L.zc_get_shape.argtypes = [_vp, C.c_uint32, C.c_int, C.POINTER(Shape)]
        L.zc_set_shape.argtypes = [_vp, C.c_uint32, C.c_int, C.POINTER(Shape)]
        L.zc_autotune.argtypes = [_vp, _vp, C.c_size_t, C.c_uint32, C.c_int, C.POINTER(Shape)]
        L.zc_profile_stages.argtypes = [_vp, C.c_uint32, _vp, _vp, _vp, _u32p]
        L.zc_archive_bound.argtypes = [_vp, C.c_uint32, C.c_uint32]
        L.zc_archive_bound.restype = C.c_uint64
        L.zc_archive_write_device.argtypes = [_vp, _vp, C.c_uint32, C.c_int, _vp, C.c_uint32, _vp, C.c_uint64, _vp,
                                              _vp, _vp]
        L.zc_archive_write.argtypes = [_vp, _vp, C.c_uint32, C.c_int, _vp, C.c_uint32, _vp, C.c_uint64, _u64p]
        L.zc_archive_write_range.argtypes = [_vp, _vp, C.c_uint64, C.c_uint64, C.c_uint32, C.c_int, _vp, C.c_uint32,
                                             C.c_uint64, _vp, C.c_uint64, _vp, _vp, _vp]
        L.zc_archive_read_table.argtypes = [_vp, C.c_uint64, C.POINTER(ArchiveInfo), _vp, C.c_uint32, C.c_char_p,
                                            C.c_size_t]
        L.zc_archive_blocks.argtypes = [_vp, C.c_uint64, C.POINTER(ArchiveInfo), _vp, _vp, _vp, _vp, _vp, C.c_char_p,
                                        C.c_size_t]
        L.zc_archive_extract.argtypes = [_vp, _vp, C.c_uint64, _vp, C.c_uint64]
        _lib = L
    return _lib


class Shape(C.Structure):
    """zc_shape: launch shapes kept per (block_log, level class); none of them changes a result byte."""
    _fields_ = [("fill_ring_log", C.c_uint32), ("fill_warps", C.c_uint32), ("match_cap", C.c_uint32),
                ("match_tile", C.c_uint32), ("fill_words", C.c_uint32), ("match_dense", C.c_uint32),
                ("match_defer", C.c_uint32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class ArchiveInfo(C.Structure):
    """zc_archive_info: an archive's layout, from its header, footer and table."""
    _fields_ = [("block_log", C.c_uint32), ("n_entries", C.c_uint32), ("total_raw", C.c_uint64),
                ("n_blocks", C.c_uint64), ("table_off", C.c_uint64), ("table_len", C.c_uint64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class _Entry(C.Structure):  # zc_entry
    _fields_ = [("name", C.c_void_p), ("name_len", C.c_uint32), ("is_dir", C.c_uint32), ("size", C.c_uint64),
                ("mtime", C.c_int64), ("attr", C.c_uint32), ("crc", C.c_uint32)]


@dataclass
class ArchiveEntry:
    """One entry of an archive's table (src/archive.h:139-147): a file's bytes follow the previous
    file's in the solid stream; a folder has none."""
    name: str
    size: int = 0
    mtime: int = 0
    attr: int = 0
    is_dir: bool = False
    crc: int = 0


def _c_entries(entries):
    """zc_entry array for `entries` (and the name buffers it points into, to keep alive)."""
    arr = (_Entry * max(len(entries), 1))()
    keep = []
    for i, e in enumerate(entries):
        nm = e.name.encode("utf-8", "surrogateescape") if isinstance(e.name, str) else bytes(e.name)
        buf = C.create_string_buffer(nm, max(len(nm), 1))
        keep.append(buf)
        arr[i].name = C.cast(buf, C.c_void_p)
        arr[i].name_len = len(nm)
        arr[i].is_dir = 1 if e.is_dir else 0
        arr[i].size = e.size
        arr[i].mtime = e.mtime
        arr[i].attr = e.attr
        arr[i].crc = e.crc
    return arr, keep


def collect(inputs):
    """The entries for a list of files and folders, collected as the reference's `zero c` does
    (src/archive.h:167-250): a file is one entry under its own name; a folder is itself and everything in
    it, under its name, sorted inside each folder by the UTF-8 bytes of the names; symbolic links are
    skipped; a name already taken keeps its first entry.  Modification times are whole seconds.
    Returns [(ArchiveEntry, source path)].  Raises FileNotFoundError for an input that does not exist."""
    out, seen = [], set()

    def add(e, src):
        if e.name not in seen:
            seen.add(e.name)
            out.append((e, src))

    def mtime(path):
        try:
            return int(os.stat(path).st_mtime)
        except OSError:
            return 0

    def walk(folder, rel):
        try:
            names = os.listdir(folder)
        except OSError:
            return
        for nm in sorted(names, key=os.fsencode):
            path = os.path.join(folder, nm)
            name = rel + "/" + nm
            if os.path.islink(path):
                continue
            if os.path.isdir(path):
                add(ArchiveEntry(name, 0, mtime(path), is_dir=True), path)
                walk(path, name)
            elif os.path.isfile(path):
                try:
                    size = os.path.getsize(path)
                except OSError:
                    size = 0
                add(ArchiveEntry(name, size, mtime(path)), path)

    for inp in inputs:
        path = inp if os.path.isabs(inp) else os.path.join(os.getcwd(), inp)
        while len(path) > 1 and path.endswith(os.sep):
            path = path[:-1]
        if not os.path.exists(path):
            raise FileNotFoundError("not found: " + inp)
        top = os.path.basename(path)
        if os.path.isdir(path):
            add(ArchiveEntry(top, 0, mtime(path), is_dir=True), path)
            walk(path, top)
        elif os.path.isfile(path):
            add(ArchiveEntry(top, os.path.getsize(path), mtime(path)), path)
    return out


def read_solid(collected):
    """The solid stream of collected entries: each file's bytes in entry order, exactly its recorded size
    (a file that shrank since it was collected reads as zeros past its end, as src/archive.h:316-318)."""
    parts = []
    for e, src in collected:
        if e.is_dir or not e.size:
            continue
        with open(src, "rb") as f:
            data = f.read(e.size)
        parts.append(data + bytes(e.size - len(data)))
    return b"".join(parts)


def safe_name(name):
    """A name from an archive is only ever written under the target folder (src/archive.h:511-523): not
    empty, not absolute, no backslash or colon, and no empty, '.' or '..' component."""
    if not name or name[0] == "/" or "\\" in name or ":" in name:
        return False
    return all(part not in ("", ".", "..") for part in name.split("/"))


def write_tree(entries, solid, out_dir):
    """Writes the solid stream back into files under out_dir as extract_archive does (src/archive.h:
    640-745): entries in order, folders made as needed, each file its bytes of the stream, modification
    times set (a zero time is left alone), folders' times last.  Raises DataError for an unsafe name or a
    stream whose size is not the table's."""
    _set = lambda path, t: t and os.utime(path, ns=(os.stat(path).st_atime_ns, t * 10**9))  # noqa: E731
    mv = memoryview(solid)
    pos = 0
    for e in entries:
        if not safe_name(e.name):
            raise DataError("refused: unsafe name in the archive: " + e.name)
        path = os.path.join(out_dir, *e.name.split("/"))
        if e.is_dir:
            os.makedirs(path, exist_ok=True)
            continue
        if pos + e.size > len(mv):
            raise DataError("archive damaged: the table lists more data than the blocks hold")
        os.makedirs(os.path.dirname(path) or out_dir, exist_ok=True)
        with open(path, "wb") as f:
            f.write(mv[pos:pos + e.size])
        pos += e.size
        _set(path, e.mtime)
    if pos != len(mv):
        raise DataError("archive damaged: more data than the table lists")
    for e in entries:
        if e.is_dir:
            _set(os.path.join(out_dir, *e.name.split("/")), e.mtime)


def archive_bound(entries, block_log):
    """The largest archive zc_archive_write can produce for these entries (0 for invalid ones)."""
    arr, _keep = _c_entries(entries)
    return int(lib().zc_archive_bound(arr, len(entries), block_log))


def read_table(arch):
    """An archive's header, footer and entry table, checked as read_info does (src/archive.h:451-495):
    -> (info dict, [ArchiveEntry]).  Host-only (no GPU).  Raises DataError for a damaged archive."""
    a = _as_u8(arch)
    info = ArchiveInfo()
    msg = C.create_string_buffer(512)
    rc = lib().zc_archive_read_table(_ptr(a), a.size, C.byref(info), None, 0, msg, 512)
    if rc:
        raise DataError(msg.value.decode(errors="replace")) if rc == ZC_E_DATA else ArgError("bad arguments")
    n = info.n_entries
    arr = (_Entry * max(n, 1))()
    lib().zc_archive_read_table(_ptr(a), a.size, C.byref(info), arr, n, msg, 512)
    out = []
    for i in range(n):
        e = arr[i]
        name = C.string_at(e.name, e.name_len) if e.name_len else b""
        out.append(ArchiveEntry(name.decode("utf-8", "surrogateescape"), int(e.size), int(e.mtime), int(e.attr),
                                bool(e.is_dir), int(e.crc)))
    return info.as_dict(), out


def archive_blocks(arch, info=None):
    """The block records of an archive (src/archive.h:566-586), checked as read_blocks does: a dict of
    arrays offs (where each body starts in arch), comp_lens, methods, raw_lens, crcs.  Host-only."""
    a = _as_u8(arch)
    if info is None:
        info, _ = read_table(arch)
    I = ArchiveInfo(**info)
    nb = int(I.n_blocks)
    if nb > a.size // 16:
        raise DataError("archive damaged: block header cut")
    offs = np.zeros(max(nb, 1), np.uint64)
    clens = np.zeros(max(nb, 1), np.uint32)
    methods = np.zeros(max(nb, 1), np.uint8)
    rlens = np.zeros(max(nb, 1), np.uint32)
    crcs = np.zeros(max(nb, 1), np.uint32)
    msg = C.create_string_buffer(512)
    rc = lib().zc_archive_blocks(_ptr(a), a.size, C.byref(I), _ptr(offs), _ptr(clens), _ptr(methods), _ptr(rlens),
                                 _ptr(crcs), msg, 512)
    if rc:
        raise DataError(msg.value.decode(errors="replace")) if rc == ZC_E_DATA else ArgError("bad arguments")
    return {"offs": offs[:nb], "comp_lens": clens[:nb], "methods": methods[:nb], "raw_lens": rlens[:nb],
            "crcs": crcs[:nb]}


def _ptr(a):
    return None if a is None else a.ctypes.data


def _as_u8(data):
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data.reshape(-1).view(np.uint8))
    return np.frombuffer(data, np.uint8)


@dataclass
class BlockOut:
    """One compressed block (src/archive.h:46-49): method 0 stored (the caller writes the input), 1 ZB2."""
    method: int = STORED
    data: bytes = b""


@dataclass
class BlockIn:
    """One block to decode (src/archive.h:50-55)."""
    method: int = STORED
    raw_len: int = 0
    data: bytes = b""

    @property
    def comp_len(self):
        return len(self.data)


def _raise(ctx, rc):
    msg = lib().zc_last_error(ctx).decode(errors="replace") if ctx else "zc_open failed"
    cls = {ZC_E_DATA: DataError, ZC_E_DEVICE: DeviceError, ZC_E_NOMEM: NoMemError, ZC_E_ARG: ArgError}.get(rc, ZcError)
    raise cls(msg)


class CudaCodec:
    """The GPU codec behind the reference's zero::Codec interface, on a CUDA device (sm_100a)."""

    def __init__(self, level=5, device=0):
        self.level = level
        ctx = _vp()
        rc = lib().zc_open(C.byref(ctx), device)
        self._ctx = ctx
        if rc:
            msg = lib().zc_last_error(ctx).decode(errors="replace") if ctx else "zc_open failed"
            self.close()
            raise DeviceError(msg)

    # -- lifetime
    def close(self):
        if getattr(self, "_ctx", None):
            lib().zc_close(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc:
            _raise(self._ctx, rc)

    # -- zero::Codec
    def name(self):
        return lib().zc_name(self._ctx).decode()

    def batch_bytes(self, block_log):
        return lib().zc_batch_bytes(self._ctx, block_log)

    def batch_bytes_decode(self, block_log):
        return lib().zc_batch_bytes_decode(self._ctx, block_log)

    def prepare(self, block_log):
        self._check(lib().zc_prepare(self._ctx, block_log, self.level))

    def launch_count(self):
        return lib().zc_launch_count(self._ctx)

    def set_graphs(self, on=True):
        """Capture / replay the device-resident calls as CUDA graphs (keyed by their arguments)."""
        self._check(lib().zc_set_graphs(self._ctx, 1 if on else 0))

    def get_shape(self, block_log, level):
        s = Shape()
        self._check(lib().zc_get_shape(self._ctx, block_log, level, C.byref(s)))
        return s.as_dict()

    def set_shape(self, block_log, level, **kw):
        """Sets some fields of the (block_log, level) shape; returns the new shape."""
        s = Shape(**self.get_shape(block_log, level))
        for k, v in kw.items():
            setattr(s, k, int(v))
        self._check(lib().zc_set_shape(self._ctx, block_log, level, C.byref(s)))
        return s.as_dict()

    def autotune(self, sample, block_log, level):
        """Times the candidate shapes on `sample` (numpy u8) and keeps the fastest; returns it."""
        a = np.ascontiguousarray(sample, dtype=np.uint8)
        s = Shape()
        self._check(lib().zc_autotune(self._ctx, a.ctypes.data, a.size, block_log, level, C.byref(s)))
        return s.as_dict()

    def profile(self, on=True):
        """Per-kernel CUDA-event timing on/off (clears the totals)."""
        self._check(lib().zc_profile(self._ctx, 1 if on else 0))

    def profile_stages(self):
        """{kernel: (total ms, launches)} since profile(True), in first-launch order."""
        n = C.c_uint32()
        self._check(lib().zc_profile_stages(self._ctx, 0, None, None, None, C.byref(n)))
        k = n.value
        names = C.create_string_buffer(32 * max(k, 1))
        ms = np.zeros(max(k, 1), np.float64)
        cnt = np.zeros(max(k, 1), np.uint64)
        self._check(lib().zc_profile_stages(self._ctx, k, names, _ptr(ms), _ptr(cnt), C.byref(n)))
        raw = names.raw
        return {raw[32 * i: 32 * i + 32].split(b"\0")[0].decode(): (float(ms[i]), int(cnt[i])) for i in range(k)}

    def compress_arrays(self, data, block_log, level=None, out=None):
        """n bytes in blocks of 2^block_log -> (methods, comp_lens, crcs, payloads, pay_offs) as arrays.
        out: optional preallocated (methods, comp_lens, crcs, payloads, pay_offs), e.g. in pinned memory."""
        a = _as_u8(data)
        B = 1 << block_log
        nb = (a.size + B - 1) // B
        if out is not None:
            methods, lens, crcs, pay, offs = out
        else:
            methods = np.zeros(max(nb, 1), np.uint8)
            lens = np.zeros(max(nb, 1), np.uint32)
            crcs = np.zeros(max(nb, 1), np.uint32)
            offs = np.zeros(max(nb, 1), np.uint64)
            pay = np.empty(max(a.size, 1), np.uint8)
        self._check(lib().zc_compress(self._ctx, _ptr(a), a.size, block_log, self.level if level is None else level,
                                      _ptr(methods), _ptr(lens), _ptr(crcs), _ptr(pay), pay.size, _ptr(offs)))
        return methods[:nb], lens[:nb], crcs[:nb], pay, offs[:nb]

    def compress_batch_arrays(self, data, in_offs, in_lens, block_log, level=None):
        """Blocks of uneven sizes (block b: in_lens[b] bytes at data[in_offs[b]:]) in one launch per stage."""
        a = _as_u8(data)
        offs_in = np.ascontiguousarray(in_offs, np.uint64)
        lens_in = np.ascontiguousarray(in_lens, np.uint32)
        nb = offs_in.size
        methods = np.zeros(max(nb, 1), np.uint8)
        lens = np.zeros(max(nb, 1), np.uint32)
        crcs = np.zeros(max(nb, 1), np.uint32)
        offs = np.zeros(max(nb, 1), np.uint64)
        pay = np.empty(max(int(lens_in.sum()), 1), np.uint8)
        self._check(lib().zc_compress_batch(self._ctx, _ptr(a), _ptr(offs_in), _ptr(lens_in), nb, block_log,
                                            self.level if level is None else level, _ptr(methods), _ptr(lens),
                                            _ptr(crcs), _ptr(pay), pay.size, _ptr(offs)))
        return methods[:nb], lens[:nb], crcs[:nb], pay, offs[:nb]

    def compress(self, data, block_log):
        """zero::Codec::compress: one BlockOut per block; a stored block carries no data."""
        methods, lens, _, pay, offs = self.compress_arrays(data, block_log)
        return [BlockOut(int(m), pay[int(o): int(o) + int(l)].tobytes() if m else b"")
                for m, l, o in zip(methods, lens, offs)]

    def decompress_arrays(self, comp, comp_offs, comp_lens, methods, raw_lens, raise_on_damage=True, out=None):
        """Blocks as arrays -> (raw bytes, per-block CRC-32s, per-block status).  out: optional
        preallocated output (e.g. pinned memory) of at least sum(raw_lens) bytes."""
        comp = _as_u8(comp)
        comp_offs = np.ascontiguousarray(comp_offs, np.uint64)
        comp_lens = np.ascontiguousarray(comp_lens, np.uint32)
        methods = np.ascontiguousarray(methods, np.uint8)
        raw_lens = np.ascontiguousarray(raw_lens, np.uint32)
        nb = raw_lens.size
        if out is None:
            out = np.empty(max(int(raw_lens.sum()), 1), np.uint8)
        crcs = np.zeros(max(nb, 1), np.uint32)
        errs = np.zeros(max(nb, 1), np.uint32)
        rc = lib().zc_decompress(self._ctx, _ptr(comp), _ptr(comp_offs), _ptr(comp_lens), _ptr(methods),
                                 _ptr(raw_lens), nb, _ptr(out), _ptr(crcs), _ptr(errs))
        if rc and (rc != ZC_E_DATA or raise_on_damage):
            _raise(self._ctx, rc)
        return out[: int(raw_lens.sum())], crcs[:nb], errs[:nb]

    def decompress(self, blocks):
        """zero::Codec::decompress: the blocks' raw bytes, one after the other."""
        if not blocks:
            return b""
        datas = [bytes(b.data) for b in blocks]
        comp = np.frombuffer(b"".join(datas) or b"\0", np.uint8)
        lens = np.array([len(d) for d in datas], np.uint64)
        offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
        out, _, _ = self.decompress_arrays(comp, offs, lens, [b.method for b in blocks], [b.raw_len for b in blocks])
        return out.tobytes()

    def crc32(self, data):
        a = _as_u8(data)
        v = C.c_uint32()
        self._check(lib().zc_crc32(self._ctx, _ptr(a), a.size, C.byref(v)))
        return v.value

    # -- device-resident forms (torch CUDA tensors or raw device addresses as ints; work queued on
    #    `stream`, a raw cudaStream_t handle)
    def compress_device(self, d_in, d_in_offs, d_in_lens, nb, block_log, d_methods, d_lens, d_crcs, d_out,
                        d_out_offs, d_total, stream=0, level=None, out_cap=None):
        self._check(lib().zc_compress_device(
            self._ctx, _dp(d_in), _dp(d_in_offs), _dp(d_in_lens), nb, block_log,
            self.level if level is None else level, _dp(d_methods), _dp(d_lens), _dp(d_crcs), _dp(d_out),
            out_cap if out_cap is not None else d_out.numel(), _dp(d_out_offs), _dp(d_total), stream or None))

    def decompress_device(self, d_comp, d_comp_offs, d_comp_lens, d_methods, d_raw_lens, nb, block_log, d_out,
                          d_out_offs, d_crcs, d_err, stream=0):
        self._check(lib().zc_decompress_device(
            self._ctx, _dp(d_comp), _dp(d_comp_offs), _dp(d_comp_lens), _dp(d_methods), _dp(d_raw_lens), nb,
            block_log, _dp(d_out), _dp(d_out_offs), _dp(d_crcs), _dp(d_err), stream or None))

    # -- whole archives (include/zero_cuda.h: zc_archive_*)
    def archive_write(self, solid, entries, block_log, level=None):
        """The .zero archive of `solid` (the files' bytes in entry order) with table `entries`, built on
        the GPU (compress_archive, src/archive.h:334-441) -> bytes.  Sets each entry's crc."""
        a = _as_u8(solid)
        if a.size == 0:
            a = np.zeros(1, np.uint8)
        arr, _keep = _c_entries(entries)
        cap = archive_bound(entries, block_log)
        if not cap:
            raise ArgError("invalid entries or block size")
        out = np.empty(cap, np.uint8)
        n = C.c_uint64()
        self._check(lib().zc_archive_write(self._ctx, _ptr(a), block_log, self.level if level is None else level,
                                           arr, len(entries), _ptr(out), out.size, C.byref(n)))
        for i, e in enumerate(entries):
            e.crc = int(arr[i].crc)
        return out[: n.value].tobytes()

    def archive_write_paths(self, inputs, block_log, level=None):
        """`zero c` for files and folders: the entries collected as the reference does, the files read in
        entry order, the archive written on the GPU -> (archive bytes, entries with their CRCs)."""
        got = collect(inputs)
        entries = [e for e, _ in got]
        return self.archive_write(read_solid(got), entries, block_log, level), entries

    def archive_extract_to(self, arch, out_dir):
        """`zero x`: every block and file checked on the GPU, then the files written under out_dir as the
        reference's extract_archive writes them.  Returns the entries."""
        solid = self.archive_extract(arch)
        _, entries = read_table(arch)
        os.makedirs(out_dir, exist_ok=True)
        write_tree(entries, solid, out_dir)
        return entries

    def archive_write_device(self, d_solid, entries, block_log, d_out, d_len, d_entry_crcs=None, stream=0,
                             level=None, out_cap=None):
        """zc_archive_write_device: device solid stream -> the archive in d_out, its length in d_len."""
        arr, _keep = _c_entries(entries)
        self._check(lib().zc_archive_write_device(
            self._ctx, _dp(d_solid), block_log, self.level if level is None else level, arr, len(entries),
            _dp(d_out), out_cap if out_cap is not None else d_out.numel(), _dp(d_len), _dp(d_entry_crcs),
            stream or None))

    def archive_write_range(self, d_range, range_off, range_len, entries, block_log, d_out, d_len,
                            d_piece_crcs=None, rec_base=0, stream=0, level=None, out_cap=None):
        """zc_archive_write_range: one rank's block records of the stream range [range_off, range_off +
        range_len) (in d_range) into d_out from rec_base on, *d_len = their end, d_piece_crcs[e] = entry e's
        CRC over its bytes inside the range."""
        arr, _keep = _c_entries(entries)
        self._check(lib().zc_archive_write_range(
            self._ctx, _dp(d_range), range_off, range_len, block_log, self.level if level is None else level, arr,
            len(entries), rec_base, _dp(d_out), out_cap if out_cap is not None else d_out.numel(), _dp(d_len),
            _dp(d_piece_crcs), stream or None))

    def archive_extract(self, arch, test=False):
        """Decodes and checks every block and file of an archive on the GPU (read_blocks + extract_archive /
        test_archive, src/archive.h:566-635, 747-785) -> the solid stream (None when test)."""
        a = _as_u8(arch)
        info, _ = read_table(a)
        out = None if test else np.empty(max(info["total_raw"], 1), np.uint8)
        self._check(lib().zc_archive_extract(self._ctx, _ptr(a), a.size, _ptr(out), 0 if out is None else out.size))
        return None if test else out[: info["total_raw"]].tobytes()


def _dp(x):
    """A device address: an int as given, a tensor's data pointer, None as NULL."""
    if x is None or isinstance(x, int):
        return x
    return x.data_ptr()


def crc32_combine(a, b, len_b):
    """crc32::combine (src/crc32.h:60-66) on the host."""
    return lib().zc_crc32_combine(a, b, len_b)


# ---------------------------------------------------------------- serving (include/zero_cuda.h: zc_serve_*)
JOB_COMPRESS, JOB_EXTRACT, JOB_TEST = 0, 1, 2


class _Job(C.Structure):
    _fields_ = [("kind", C.c_int), ("block_log", C.c_uint32), ("level", C.c_int), ("in_", C.c_void_p),
                ("in_len", C.c_size_t), ("nb", C.c_uint32), ("comp_lens", C.c_void_p), ("methods", C.c_void_p),
                ("raw_lens", C.c_void_p), ("crcs_expected", C.c_void_p), ("out", C.c_void_p),
                ("out_cap", C.c_size_t), ("out_methods", C.c_void_p), ("out_lens", C.c_void_p),
                ("out_offs", C.c_void_p), ("out_crcs", C.c_void_p)]


class ServeJob:
    """A submitted job: keeps its buffers alive until waited for; results are filled in place."""

    def __init__(self, kind, arrays):
        self.kind = kind
        self.arrays = arrays
        self.id = None
        self.status = None
        self.latency = None

    def __getattr__(self, name):
        arrays = self.__dict__.get("arrays", {})
        if name in arrays:
            return arrays[name]
        raise AttributeError(name)


class Server:
    """Continuous-batching request loop on one GPU: jobs admitted by free device memory (budget_bytes),
    their blocks batched with other jobs' blocks tick by tick.  pinned=True takes the jobs' result
    buffers from recycled page-locked memory (an extract job's bytes then arrive by DMA, with no host
    copy); such results are valid while their job handle lives, and the buffers are reused after."""

    def __init__(self, budget_bytes, device=0, max_batch_bytes=0, pinned=False):
        self.pinned = pinned
        self._free = {}  # pinned result buffers by size class, reused once their job handle is gone
        L = lib()
        L.zc_serve_open.argtypes = [C.POINTER(_vp), C.c_int, C.c_uint64, C.c_uint64]
        L.zc_serve_close.argtypes = [_vp]
        L.zc_serve_submit.argtypes = [_vp, C.POINTER(_Job), C.POINTER(C.c_uint64)]
        L.zc_serve_wait.argtypes = [_vp, C.c_uint64, C.POINTER(C.c_double)]
        L.zc_serve_stats.argtypes = [_vp] + [C.POINTER(C.c_uint64)] * 4
        L.zc_serve_times.argtypes = [_vp] + [C.POINTER(C.c_double)] * 4
        self._srv = _vp()
        rc = L.zc_serve_open(C.byref(self._srv), device, budget_bytes, max_batch_bytes)
        if rc:
            self._srv = None
            _raise(None, rc)

    def close(self):
        if getattr(self, "_srv", None):
            lib().zc_serve_close(self._srv)
            self._srv = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _buf(self, n, arr, key):
        if not self.pinned:
            return np.empty(n, np.uint8)
        import torch
        cls = max(1 << 16, 1 << (int(n) - 1).bit_length())
        free = self._free.setdefault(cls, [])
        t = free.pop() if free else torch.empty(cls, dtype=torch.uint8, pin_memory=True)
        arr.setdefault("_pinned", []).append((cls, t))
        return t.numpy()[:n]

    def _track(self, handle):
        """Pinned buffers go back to the free lists when the handle is collected."""
        import weakref
        for cls, t in handle.arrays.get("_pinned", []):
            weakref.finalize(handle, self._free.setdefault(cls, []).append, t)
        handle.arrays.pop("_pinned", None)
        return handle

    def _submit(self, job, handle):
        jid = C.c_uint64()
        rc = lib().zc_serve_submit(self._srv, C.byref(job), C.byref(jid))
        if rc:
            _raise(None, rc)
        handle.id = jid.value
        return handle

    def compress(self, data, block_log=18, level=5):
        a = _as_u8(data)
        B = 1 << block_log
        nb = (a.size + B - 1) // B
        arr = dict(data=a, methods=np.zeros(max(nb, 1), np.uint8),
                   lens=np.zeros(max(nb, 1), np.uint32), offs=np.zeros(max(nb, 1), np.uint64),
                   crcs=np.zeros(max(nb, 1), np.uint32))
        arr["payloads"] = self._buf(max(a.size, 1), arr, "payloads")
        j = _Job(JOB_COMPRESS, block_log, level, _ptr(a), a.size, 0, None, None, None, None, _ptr(arr["payloads"]),
                 arr["payloads"].size, _ptr(arr["methods"]), _ptr(arr["lens"]), _ptr(arr["offs"]), _ptr(arr["crcs"]))
        h = ServeJob(JOB_COMPRESS, arr)
        h.nb = nb
        return self._submit(j, self._track(h))

    def _decode(self, kind, comp, comp_lens, methods, raw_lens, block_log, crcs_expected=None):
        c = _as_u8(comp)
        cl = np.ascontiguousarray(comp_lens, np.uint32)
        me = np.ascontiguousarray(methods, np.uint8)
        rl = np.ascontiguousarray(raw_lens, np.uint32)
        nb = rl.size
        arr = dict(comp=c, comp_lens=cl, methods=me, raw_lens=rl, crcs=np.zeros(max(nb, 1), np.uint32))
        out = None
        if kind == JOB_EXTRACT:
            out = arr["raw"] = self._buf(max(int(rl.sum()), 1), arr, "raw")
        exp = None
        if crcs_expected is not None:
            exp = arr["crcs_expected"] = np.ascontiguousarray(crcs_expected, np.uint32)
        j = _Job(kind, block_log, 0, _ptr(c), c.size, nb, _ptr(cl), _ptr(me), _ptr(rl), _ptr(exp), _ptr(out),
                 0 if out is None else out.size, None, None, None, _ptr(arr["crcs"]))
        return self._submit(j, self._track(ServeJob(kind, arr)))

    def extract(self, comp, comp_lens, methods, raw_lens, block_log=18):
        """Record bodies back to back -> raw bytes (handle.raw) and CRCs (handle.crcs)."""
        return self._decode(JOB_EXTRACT, comp, comp_lens, methods, raw_lens, block_log)

    def test(self, comp, comp_lens, methods, raw_lens, crcs_expected, block_log=18):
        """Decode and check every block's CRC; status DataError on a mismatch."""
        return self._decode(JOB_TEST, comp, comp_lens, methods, raw_lens, block_log, crcs_expected)

    def wait(self, handle, raise_on_error=True):
        lat = C.c_double()
        rc = lib().zc_serve_wait(self._srv, handle.id, C.byref(lat))
        handle.status, handle.latency = rc, lat.value
        if rc and raise_on_error:
            _raise(None, rc)
        return handle

    def stats(self):
        v = [C.c_uint64() for _ in range(4)]
        lib().zc_serve_stats(self._srv, *[C.byref(x) for x in v])
        t = [C.c_double() for _ in range(4)]
        lib().zc_serve_times(self._srv, *[C.byref(x) for x in t])
        return dict(jobs_done=v[0].value, raw_bytes=v[1].value, ticks=v[2].value, arena_used=v[3].value,
                    gpu_s=t[0].value, wait_s=t[1].value, handout_s=t[2].value, upload_s=t[3].value)


def record_bodies(data, methods, lens, payloads, offs, block_log):
    """A compress result as the archive holds it: each block's payload, or its raw bytes when stored;
    returns (bodies back to back, comp_lens, raw_lens)."""
    a = _as_u8(data)
    B = 1 << block_log
    parts, clens, rlens = [], [], []
    for b in range(len(methods)):
        raw = a[b * B:(b + 1) * B]
        body = payloads[int(offs[b]): int(offs[b]) + int(lens[b])] if methods[b] else raw
        parts.append(body)
        clens.append(len(body))
        rlens.append(raw.size)
    blob = np.concatenate(parts) if parts else np.zeros(0, np.uint8)
    return blob, np.array(clens, np.uint32), np.array(rlens, np.uint32)
