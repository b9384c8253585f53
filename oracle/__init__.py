"""ORACLE — test infrastructure, not part of the product.

ctypes loaders for:
  liboracle.so          the C restatements of the reference ladders (oracle.c,
                        zstd_oracle.c, gdeflate_oracle.c) and the
                        multithreaded codec-library harness (codecs.c)
  _ref/libref_twin.so   the reference's own host twins, compiled in place
  _ref/libcudec_ref.so  the reference library (GPU), compiled in place

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this package, and only as a checker or a timed baseline.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_TWIN_LIB = os.path.join(HERE, "_ref", "libref_twin.so")
REF_GPU_LIB = os.path.join(HERE, "_ref", "libcudec_ref.so")

_U8P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_DEC = [_U8P, _U64, _U8P, _U64, ctypes.POINTER(_U64)]
_BATCH = [_U8P, _U8P, _U8P, _U8P, _U64, _U8P, _U8P, ctypes.c_int]


def build(ref=None):
    """Compile the restatement with oracle/Makefile, and the reference pieces
    when `ref` (or the CUDEC_REFERENCE environment variable) names the
    reference tree."""
    ref = ref or os.environ.get("CUDEC_REFERENCE", "")
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile"), "REF=" + ref],
                   check=True)


_libs = {}


def _load(path, funcs):
    if path not in _libs:
        if not os.path.exists(path):
            return None
        h = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
        for name, (res, args) in funcs.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _libs[path] = h
    return _libs[path]


def oracle_lib():
    h = _load(ORACLE_LIB, {
        "oracle_lz4_decode": (ctypes.c_int, _DEC),
        "oracle_snappy_decode": (ctypes.c_int, _DEC),
        "oracle_lz4f_decode": (ctypes.c_int, _DEC),
        "oracle_zstd_decode": (ctypes.c_int, _DEC),
        "oracle_zstd_decode_multi": (ctypes.c_int, _DEC),
        "oracle_xxh64": (ctypes.c_uint64, [_U8P, _U64, _U64]),
        "oracle_xxh32": (ctypes.c_uint32, [_U8P, _U64, ctypes.c_uint32]),
        "oracle_lz4_decode_batch": (ctypes.c_int, _BATCH),
        "oracle_snappy_decode_batch": (ctypes.c_int, _BATCH),
        "codec_decode_batch": (ctypes.c_int, [ctypes.c_int] + _BATCH),
        "codec_lz4_version": (ctypes.c_int, []),
        "codec_zstd_version": (ctypes.c_int, []),
        "oracle_gdeflate_decode": (ctypes.c_int, _DEC),
        "oracle_gdeflate_schedule_trace": (ctypes.c_int, [_U8P, _U64, _U8P, _U64, _U8P]),
        "oracle_tilestream_parse": (ctypes.c_int, [_U8P, _U64, _U8P, _U64, _U8P, _U8P]),
    })
    if h is None:
        raise RuntimeError("oracle/liboracle.so is not built (oracle.build())")
    return h


def ref_twin_lib():
    """The reference's host twins, or None where they were not built."""
    return _load(REF_TWIN_LIB, {
        "ref_lz4_twin_decode": (ctypes.c_int, _DEC),
        "ref_snappy_twin_decode": (ctypes.c_int, _DEC),
        "ref_zstd_twin_decode": (ctypes.c_int, _DEC),
        "ref_zstd_twin_decode_batch": (ctypes.c_int, _BATCH),
        "ref_lz4_twin_decode_batch": (ctypes.c_int, _BATCH),
        "ref_snappy_twin_decode_batch": (ctypes.c_int, _BATCH),
        "ref_gdeflate_schedule_trace": (ctypes.c_int, [_U8P, _U64, _U8P, _U64, _U8P]),
        "ref_tilestream_parse": (ctypes.c_int, [_U8P, _U64, _U8P, _U64, _U8P, _U8P]),
    })


def ref_gpu_lib():
    """The reference library (sm_100a build), or None where it was not built."""
    return _load(REF_GPU_LIB, {
        "cudec_lz4_decompress_batch": (ctypes.c_int, [ctypes.c_void_p] * 4 +
                                       [ctypes.c_size_t, ctypes.c_void_p,
                                        ctypes.c_void_p]),
        "cudec_version": (ctypes.c_int, []),
        "cudec_lz4f_decompress": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t,
                                                 ctypes.c_void_p, ctypes.c_size_t,
                                                 ctypes.c_void_p]),
    })


def _decode_one(fn, comp, cap):
    src = np.frombuffer(bytes(comp), dtype=np.uint8)
    if len(src) == 0:
        src = np.zeros(1, dtype=np.uint8)
    out = np.zeros(max(cap, 1), dtype=np.uint8)
    w = _U64(0)
    st = fn(src.ctypes.data, len(comp), out.ctypes.data, cap, ctypes.byref(w))
    return st, (out[:w.value].tobytes() if st == 0 else b"")


def xxh32(data, seed=0):
    """XXH32 from the C restatement (LZ4 frame header/block/content checks)."""
    b = np.frombuffer(bytes(data) or b"\0", dtype=np.uint8)
    return int(oracle_lib().oracle_xxh32(b.ctypes.data, len(data), seed))


def xxh64(data, seed=0):
    """XXH64 from the C restatement (Zstd content checksum)."""
    b = np.frombuffer(bytes(data) or b"\0", dtype=np.uint8)
    return int(oracle_lib().oracle_xxh64(b.ctypes.data, len(data), seed))


def lz4_decode(comp, cap):
    """(status, bytes) from the C restatement."""
    return _decode_one(oracle_lib().oracle_lz4_decode, comp, cap)


def lz4f_decode(frame, cap):
    """(status, bytes) from the C restatement of the frame ladder."""
    return _decode_one(oracle_lib().oracle_lz4f_decode, frame, cap)


def ref_lz4f_decode(frame, cap):
    """(status, bytes) from the reference library's own frame entry (GPU),
    or None where it was not built."""
    h = ref_gpu_lib()
    if h is None:
        return None
    src = np.frombuffer(bytes(frame) if frame else b"\0", dtype=np.uint8)
    out = np.zeros(max(cap, 1), dtype=np.uint8)
    w = ctypes.c_size_t(0)
    st = h.cudec_lz4f_decompress(src.ctypes.data, len(frame), out.ctypes.data, cap,
                                 ctypes.byref(w))
    return st, out[:w.value].tobytes()


def zstd_decode(frame, cap):
    """(status, bytes) from the C restatement of the Zstd frame decode."""
    return _decode_one(oracle_lib().oracle_zstd_decode, frame, cap)


def zstd_decode_multi(frames, cap):
    """(status, bytes) for a buffer of concatenated Zstd and skippable frames,
    from the C restatement."""
    return _decode_one(oracle_lib().oracle_zstd_decode_multi, frames, cap)


def ref_zstd_decode(frame, cap):
    """(status, bytes) from the reference's twin driver, or None if unbuilt."""
    h = ref_twin_lib()
    return None if h is None else _decode_one(h.ref_zstd_twin_decode, frame, cap)


def gdeflate_decode(page, cap):
    """One GDeflate page (oracle/gdeflate_oracle.c; symbol-level parity with the
    GDeflate reference decoder is unpinned)."""
    return _decode_one(oracle_lib().oracle_gdeflate_decode, page, cap)


def _schedule_trace(fn, page, ops):
    ops = np.ascontiguousarray(ops, dtype=np.uint32)
    buf = np.frombuffer(bytes(page) + b"\0", dtype=np.uint8)
    trace = np.zeros(4 * (len(ops) + 1), dtype=np.uint64)
    n = fn(buf.ctypes.data, len(page), ops.ctypes.data, len(ops), trace.ctypes.data)
    return trace[:4 * n].reshape(-1, 4)


def gdeflate_schedule_trace(page, ops):
    return _schedule_trace(oracle_lib().oracle_gdeflate_schedule_trace, page, ops)


def ref_gdeflate_schedule_trace(page, ops):
    return _schedule_trace(ref_twin_lib().ref_gdeflate_schedule_trace, page, ops)


def _tilestream(fn, stream, tiles_cap):
    buf = np.frombuffer(bytes(stream) + b"\0", dtype=np.uint8)
    tiles = np.zeros(3 * max(tiles_cap, 1), dtype=np.uint64)
    cnt, tot = _U64(), _U64()
    st = fn(buf.ctypes.data, len(stream), tiles.ctypes.data, tiles_cap, ctypes.byref(cnt),
            ctypes.byref(tot))
    if st != 0:
        return st, None, None
    return st, tiles[:3 * cnt.value].reshape(-1, 3).tolist(), tot.value


def tilestream_parse(stream, tiles_cap):
    """(status, [[src_off, src_size, dst_size], ...], total) of the envelope."""
    return _tilestream(oracle_lib().oracle_tilestream_parse, stream, tiles_cap)


def ref_tilestream_parse(stream, tiles_cap):
    return _tilestream(ref_twin_lib().ref_tilestream_parse, stream, tiles_cap)


def snappy_decode(comp, cap):
    return _decode_one(oracle_lib().oracle_snappy_decode, comp, cap)


def ref_lz4_decode(comp, cap):
    """(status, bytes) from the reference's own twin, or None if unbuilt."""
    h = ref_twin_lib()
    return None if h is None else _decode_one(h.ref_lz4_twin_decode, comp, cap)


def ref_snappy_decode(comp, cap):
    h = ref_twin_lib()
    return None if h is None else _decode_one(h.ref_snappy_twin_decode, comp, cap)


class HostBatch:
    """Chunks packed in host memory with pointer/size tables, for the batch
    drivers (restatement, reference twin, codec libraries)."""

    def __init__(self, comps, caps):
        self.n = len(comps)
        sizes = np.array([len(c) for c in comps], dtype=np.uint64)
        self.src = np.frombuffer(b"".join(comps) + b"\0", dtype=np.uint8).copy()
        offs = np.zeros(self.n, dtype=np.uint64)
        if self.n > 1:
            offs[1:] = np.cumsum(sizes[:-1])
        self.src_sizes = sizes
        self.caps = np.asarray(caps, dtype=np.uint64)
        dst_offs = np.zeros(self.n, dtype=np.uint64)
        if self.n > 1:
            dst_offs[1:] = np.cumsum(self.caps[:-1])
        self.dst = np.zeros(int(self.caps.sum()) + 1, dtype=np.uint8)
        self.src_ptrs = (offs + self.src.ctypes.data).astype(np.uint64)
        self.dst_ptrs = (dst_offs + self.dst.ctypes.data).astype(np.uint64)
        self.dst_offs = dst_offs
        self.status = np.zeros(self.n, dtype=np.int32)
        self.written = np.zeros(self.n, dtype=np.uint64)

    def args(self):
        return (self.src_ptrs.ctypes.data, self.src_sizes.ctypes.data,
                self.dst_ptrs.ctypes.data, self.caps.ctypes.data, self.n,
                self.status.ctypes.data, self.written.ctypes.data)

    def output(self, i):
        o = int(self.dst_offs[i])
        return self.dst[o:o + int(self.written[i])].tobytes()


def decode_batch(kind, batch, threads):
    """Run a batch driver: kind in {"oracle_lz4", "oracle_snappy", "ref_lz4",
    "ref_snappy", "ref_zstd", "codec_lz4", "codec_zstd"}. Returns the thread count used."""
    if kind.startswith("oracle_"):
        fn = getattr(oracle_lib(), "oracle_%s_decode_batch" % kind[7:])
        return fn(*batch.args(), threads)
    if kind.startswith("ref_"):
        h = ref_twin_lib()
        if h is None:
            raise RuntimeError("reference twins not built")
        return getattr(h, "ref_%s_twin_decode_batch" % kind[4:])(*batch.args(), threads)
    if kind.startswith("codec_"):
        code = {"codec_lz4": 0, "codec_zstd": 1}[kind]
        return oracle_lib().codec_decode_batch(code, *batch.args(), threads)
    raise ValueError(kind)
