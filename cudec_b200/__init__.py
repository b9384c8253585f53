"""cudec_b200 — B200-native batch decompression behind the iderex/cudec C ABI.

The product is the shared library `libcudec_b200.so` (C ABI in
include/cudec.h). This module is the Python mirror of that ABI over ctypes:
the same entry-point names, argument meaning and status values, used by the
tests and the benchmark. Loading fails loudly if the library has not been
built; nothing here decodes on the CPU.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcudec_b200.so")

# cudec_status (include/cudec.h)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CORRUPT_INPUT = 2
ERR_OUTPUT_TOO_SMALL = 3
ERR_CUDA = 4
ERR_NOT_IMPLEMENTED = 5
ERR_UNSUPPORTED = 6

STATUS_NAMES = {
    OK: "CUDEC_OK",
    ERR_INVALID_ARGUMENT: "CUDEC_ERR_INVALID_ARGUMENT",
    ERR_CORRUPT_INPUT: "CUDEC_ERR_CORRUPT_INPUT",
    ERR_OUTPUT_TOO_SMALL: "CUDEC_ERR_OUTPUT_TOO_SMALL",
    ERR_CUDA: "CUDEC_ERR_CUDA",
    ERR_NOT_IMPLEMENTED: "CUDEC_ERR_NOT_IMPLEMENTED",
    ERR_UNSUPPORTED: "CUDEC_ERR_UNSUPPORTED",
}

# cudec_mem_space
MEM_HOST = 0
MEM_DEVICE = 1


class ChunkResult(ctypes.Structure):
    """cudec_chunk_result: the fixed 16-byte per-chunk record."""
    _fields_ = [("status", ctypes.c_int32), ("reserved", ctypes.c_uint32),
                ("bytes_written", ctypes.c_uint64)]


assert ctypes.sizeof(ChunkResult) == 16

_P = ctypes.c_void_p
_SZ = ctypes.c_size_t

# name -> (restype, argtypes); every symbol include/cudec.h declares.
SIGNATURES = {
    "cudec_version": (ctypes.c_int, []),
    "cudec_lz4_decompress_batch": (ctypes.c_int, [_P, _P, _P, _P, _SZ, _P, _P]),
    "cudec_snappy_decompress_batch": (ctypes.c_int, [_P, _P, _P, _P, _SZ, _P, _P]),
    "cudec_zstd_workspace_bytes": (ctypes.c_size_t, [_SZ]),
    "cudec_zstd_decompress_batch": (ctypes.c_int, [_P, _P, _P, _P, _SZ, _P, _P, _SZ, _P]),
    "cudec_zstd_decompress_batch_noalloc": (ctypes.c_int, [_P, _P, _P, _P, _SZ, _P, _P]),
    "cudec_zstd_decompress_batch_multi": (ctypes.c_int, [_P, _P, _P, _P, _SZ, _P, _P, _SZ, _P]),
    "cudec_gdeflate_decompress_batch": (ctypes.c_int, [_P, _P, _P, _P, _SZ, _P, _P]),
    "cudec_gdeflate_tilestream_parse": (ctypes.c_int, [_P, _SZ, _P, _SZ, _P, _P]),
    "cudec_gdeflate_tilestream_decompress": (ctypes.c_int, [_P, _SZ, _P, _SZ, ctypes.c_int, _P]),
    "cudec_mixed_plan_create": (ctypes.c_int, [_P]),
    "cudec_mixed_plan_destroy": (ctypes.c_int, [_P]),
    "cudec_mixed_decompress": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _SZ, _P, _P]),
    "cudec_mixed_plan_tune": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _SZ, _P, _P]),
    "cudec_mixed_plan_get_tuning": (ctypes.c_int, [_P, _P]),
    "cudec_mixed_plan_get_shape": (ctypes.c_int, [_P, _P]),
    "cudec_mixed_plan_set_shape": (ctypes.c_int, [_P, _P]),
    "cudec_server_create": (ctypes.c_int, [_SZ, ctypes.c_int, ctypes.c_int, _SZ, _P]),
    "cudec_server_destroy": (ctypes.c_int, [_P]),
    "cudec_server_submit": (ctypes.c_int, [_P, _P, _SZ, _P, _P, _P, _P, _SZ, _P]),
    "cudec_server_wait": (ctypes.c_int, [_P, ctypes.c_uint64, _P, _P, _P]),
    "cudec_server_wait_for": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_double, _P, _P, _P,
                                             _P]),
    "cudec_server_release": (ctypes.c_int, [_P, ctypes.c_uint64]),
    "cudec_lz4f_decompress": (ctypes.c_int, [_P, _SZ, _P, _SZ, _P]),
    "cudec_stream_ctx_create": (ctypes.c_int, [_P]),
    "cudec_lz4_decompress_stream_ctx": (ctypes.c_int, [_P, _P, _P, _P, _P, _SZ, ctypes.c_int, _P]),
    "cudec_stream_ctx_destroy": (None, [_P]),
    "cudec_lz4_decompress_stream": (ctypes.c_int, [_P, _P, _P, _P, _SZ, ctypes.c_int, _P]),
}

_lib = None


def lib():
    """The loaded decode library (built in-tree; raises if missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libcudec_b200.so is not built: run `python -m cudec_b200.build`")
        handle = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_LOCAL)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def version():
    return lib().cudec_version()


def _batch_call(name, d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_caps, n,
                d_results, stream):
    return getattr(lib(), name)(d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_caps,
                                n, d_results, stream)


def lz4_decompress_batch(d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_caps, n,
                         d_results, stream=None):
    """cudec_lz4_decompress_batch: all pointers are device addresses (ints)."""
    return _batch_call("cudec_lz4_decompress_batch", d_src_ptrs, d_src_sizes,
                       d_dst_ptrs, d_dst_caps, n, d_results, stream)


def snappy_decompress_batch(d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_caps, n,
                            d_results, stream=None):
    """cudec_snappy_decompress_batch (same contract as the LZ4 entry)."""
    return _batch_call("cudec_snappy_decompress_batch", d_src_ptrs, d_src_sizes,
                       d_dst_ptrs, d_dst_caps, n, d_results, stream)


def zstd_workspace_bytes(n):
    return lib().cudec_zstd_workspace_bytes(n)


def zstd_decompress_batch(d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_caps, n, d_results,
                          d_workspace, workspace_bytes, stream=None):
    """cudec_zstd_decompress_batch (one Zstd frame per chunk)."""
    return lib().cudec_zstd_decompress_batch(d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_caps,
                                             n, d_results, d_workspace, workspace_bytes, stream)


def zstd_decompress_batch_multi(d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_caps, n, d_results,
                                d_workspace, workspace_bytes, stream=None):
    """cudec_zstd_decompress_batch_multi (a sequence of Zstd and skippable
    frames per chunk, outputs concatenated)."""
    return lib().cudec_zstd_decompress_batch_multi(d_src_ptrs, d_src_sizes, d_dst_ptrs,
                                                   d_dst_caps, n, d_results, d_workspace,
                                                   workspace_bytes, stream)


ZSTD_NOALLOC_MAX_CHUNKS = 64


def zstd_decompress_batch_noalloc(d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_caps, n,
                                  d_results, stream=None):
    """cudec_zstd_decompress_batch_noalloc (library-owned scratch, <= 64 chunks)."""
    return lib().cudec_zstd_decompress_batch_noalloc(d_src_ptrs, d_src_sizes, d_dst_ptrs,
                                                     d_dst_caps, n, d_results, stream)


def gdeflate_decompress_batch(d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_caps, n, d_results,
                              stream=None):
    """cudec_gdeflate_decompress_batch (one GDeflate page per chunk)."""
    return lib().cudec_gdeflate_decompress_batch(d_src_ptrs, d_src_sizes, d_dst_ptrs,
                                                 d_dst_caps, n, d_results, stream)


def tilestream_parse(stream, tiles_capacity):
    """(status, [(src_offset, src_size, dst_size)], total) from the library's
    TileStream walker."""
    import numpy as np
    buf = bytes(stream)
    tiles = np.zeros(3 * max(tiles_capacity, 1), dtype=np.uint64)
    cnt, tot = ctypes.c_size_t(), ctypes.c_size_t()
    st = lib().cudec_gdeflate_tilestream_parse(buf, len(buf), tiles.ctypes.data,
                                               tiles_capacity, ctypes.byref(cnt),
                                               ctypes.byref(tot))
    if st != OK:
        return st, None, None
    return st, tiles[:3 * cnt.value].reshape(-1, 3).tolist(), tot.value


def tilestream_decompress(stream, capacity):
    """Whole container into host memory: (status, bytes)."""
    buf = bytes(stream)
    out = ctypes.create_string_buffer(max(capacity, 1))
    written = ctypes.c_size_t()
    st = lib().cudec_gdeflate_tilestream_decompress(buf, len(buf), out, capacity, MEM_HOST,
                                                    ctypes.byref(written))
    return st, out.raw[:written.value]


BATCH_ENTRIES = {
    "lz4": lz4_decompress_batch,
    "snappy": snappy_decompress_batch,
    "gdeflate": gdeflate_decompress_batch,
}


def lz4f_decompress(frame, dst_capacity):
    """cudec_lz4f_decompress over Python bytes: returns (status, bytes)."""
    import numpy as np
    src = np.frombuffer(bytes(frame) if frame else b"\0", dtype=np.uint8)
    out = np.zeros(max(dst_capacity, 1), dtype=np.uint8)
    written = ctypes.c_size_t(0)
    st = lib().cudec_lz4f_decompress(src.ctypes.data, len(frame), out.ctypes.data,
                                      dst_capacity, ctypes.byref(written))
    return st, out[:written.value].tobytes()


class StreamContext:
    """cudec_stream_ctx: create / decode (host arrays) / destroy."""

    def __init__(self):
        h = ctypes.c_void_p()
        st = lib().cudec_stream_ctx_create(ctypes.byref(h))
        if st != OK:
            raise RuntimeError("cudec_stream_ctx_create: %s" % STATUS_NAMES.get(st, st))
        self.handle = h

    def decode(self, src_ptrs, src_sizes, dst_ptrs, dst_caps, n, space, results):
        """All arguments are host addresses of arrays (ints); returns status."""
        return lib().cudec_lz4_decompress_stream_ctx(self.handle, src_ptrs, src_sizes,
                                                     dst_ptrs, dst_caps, n, space, results)

    def close(self):
        if self.handle:
            lib().cudec_stream_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


FORMAT_LZ4, FORMAT_SNAPPY, FORMAT_ZSTD, FORMAT_GDEFLATE = 0, 1, 2, 3
FORMAT_CODES = {"lz4": FORMAT_LZ4, "snappy": FORMAT_SNAPPY, "zstd": FORMAT_ZSTD,
                "gdeflate": FORMAT_GDEFLATE}
MIXED_BUCKETS = 6
MIXED_CTA_WARPS = 8  # CUDEC_MIXED_CTA_WARPS: warps of the CTA-per-chunk decoder


class MixedPlan:
    """cudec_mixed_plan: persistent mixed-format decode with its autotuner.

    Arguments of decode/tune are device addresses (ints) of the chunk tables
    plus one format-code byte per chunk; stream is a raw cudaStream_t value.
    """

    def __init__(self):
        h = ctypes.c_void_p()
        st = lib().cudec_mixed_plan_create(ctypes.byref(h))
        if st != OK:
            raise RuntimeError("cudec_mixed_plan_create: %s" % STATUS_NAMES.get(st, st))
        self.handle = h

    def decode(self, src_ptrs, src_sizes, dst_ptrs, dst_caps, formats, n, results, stream=None):
        return lib().cudec_mixed_decompress(self.handle, src_ptrs, src_sizes, dst_ptrs,
                                            dst_caps, formats, n, results, stream)

    def tune(self, src_ptrs, src_sizes, dst_ptrs, dst_caps, formats, n, results, stream=None):
        return lib().cudec_mixed_plan_tune(self.handle, src_ptrs, src_sizes, dst_ptrs,
                                           dst_caps, formats, n, results, stream)

    def tuning(self):
        """[(parse_window, lookahead, ring_batch)] per size bucket."""
        out = (ctypes.c_uint32 * (3 * MIXED_BUCKETS))()
        st = lib().cudec_mixed_plan_get_tuning(self.handle, out)
        if st != OK:
            raise RuntimeError("cudec_mixed_plan_get_tuning: %s" % STATUS_NAMES.get(st, st))
        return [tuple(out[3 * b:3 * b + 3]) for b in range(MIXED_BUCKETS)]

    def shape(self):
        """[(warps per chunk, parse reach, lookahead, ring batch)] per bucket."""
        out = (ctypes.c_uint32 * (4 * MIXED_BUCKETS))()
        st = lib().cudec_mixed_plan_get_shape(self.handle, out)
        if st != OK:
            raise RuntimeError("cudec_mixed_plan_get_shape: %s" % STATUS_NAMES.get(st, st))
        return [tuple(out[4 * b:4 * b + 4]) for b in range(MIXED_BUCKETS)]

    def set_shape(self, shape):
        """Set [(warps, reach, lookahead, batch)] per bucket; returns the status."""
        flat = [int(v) for row in shape for v in row]
        arr = (ctypes.c_uint32 * len(flat))(*flat)
        return lib().cudec_mixed_plan_set_shape(self.handle, arr)

    def close(self):
        if self.handle:
            lib().cudec_mixed_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SERVER_MIXED, SERVER_PLAIN = 0, 1


class Server:
    """cudec_server: continuous-batching decode with a device-memory budget."""

    def __init__(self, budget_bytes, max_inflight=4, mode=SERVER_MIXED, max_chunks=4096):
        h = ctypes.c_void_p()
        st = lib().cudec_server_create(budget_bytes, max_inflight, mode, max_chunks,
                                       ctypes.byref(h))
        if st != OK:
            raise RuntimeError("cudec_server_create: %s" % STATUS_NAMES.get(st, st))
        self.handle = h
        self._keep = {}

    def submit(self, packed, offsets, sizes, caps, formats):
        """packed: numpy uint8 array (kept alive until wait); the per-chunk
        arrays are sequences of ints / format codes. Returns (status, ticket)."""
        import numpy as np
        offs = np.ascontiguousarray(offsets, dtype=np.uint64)
        szs = np.ascontiguousarray(sizes, dtype=np.uint64)
        cps = np.ascontiguousarray(caps, dtype=np.uint64)
        fms = np.ascontiguousarray([FORMAT_CODES.get(f, f) if isinstance(f, str) else f
                                    for f in formats], dtype=np.uint8)
        t = ctypes.c_uint64()
        st = lib().cudec_server_submit(self.handle, packed.ctypes.data if len(packed) else None,
                                       len(packed), offs.ctypes.data, szs.ctypes.data,
                                       cps.ctypes.data, fms.ctypes.data, len(offs),
                                       ctypes.byref(t))
        if st == OK:
            self._keep[t.value] = (packed, len(offs))
        return st, t.value

    def wait(self, ticket):
        """Returns (status, records, device output addresses, latency_ms)."""
        import numpy as np
        n = self._keep[ticket][1]
        recs = np.zeros(n, dtype=[("status", "<i4"), ("reserved", "<u4"),
                                  ("bytes_written", "<u8")])
        ptrs = np.zeros(n, dtype=np.uint64)
        lat = ctypes.c_double()
        st = lib().cudec_server_wait(self.handle, ticket, recs.ctypes.data, ptrs.ctypes.data,
                                     ctypes.byref(lat))
        return st, recs, ptrs, lat.value

    def wait_for(self, ticket, timeout_ms):
        """Bounded wait: (status, done, records, device output addresses,
        latency_ms); done False means the deadline passed first."""
        import numpy as np
        n = self._keep[ticket][1]
        recs = np.zeros(n, dtype=[("status", "<i4"), ("reserved", "<u4"),
                                  ("bytes_written", "<u8")])
        ptrs = np.zeros(n, dtype=np.uint64)
        lat = ctypes.c_double()
        done = ctypes.c_int(-1)
        st = lib().cudec_server_wait_for(self.handle, ticket, float(timeout_ms),
                                         ctypes.byref(done), recs.ctypes.data, ptrs.ctypes.data,
                                         ctypes.byref(lat))
        return st, bool(done.value == 1), recs, ptrs, lat.value

    def release(self, ticket):
        st = lib().cudec_server_release(self.handle, ticket)
        self._keep.pop(ticket, None)
        return st

    def close(self):
        if self.handle:
            lib().cudec_server_destroy(self.handle)
            self.handle = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
