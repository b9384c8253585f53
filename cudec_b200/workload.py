"""Synthetic workloads with the benchmark configurations' shapes.

Content comes from libcudec_workload.so (seeded SplitMix64 generator, see
csrc/workload.c); compression uses the codec libraries the reference pins —
liblz4's LZ4_compress_default (reached through ctypes, as the reference's
fixtures reach it) and snappy's raw-block compressor (bundled in pyarrow;
no libsnappy is installed on these hosts).

The reference measures on Silesia/enwik8, which are not available; these
seeded generators stand in for them with the distributions the benchmark
configurations name.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WORKLOAD_LIB = os.path.join(HERE, "libcudec_workload.so")


class GenParams(ctypes.Structure):
    _fields_ = [("copy_prob", ctypes.c_double), ("alphabet", ctypes.c_int),
                ("zipf_s", ctypes.c_double), ("mean_lit", ctypes.c_double),
                ("mean_match", ctypes.c_double), ("min_match", ctypes.c_uint32),
                ("max_match", ctypes.c_uint32), ("max_offset", ctypes.c_uint64),
                ("rle_prob", ctypes.c_double), ("mean_rle", ctypes.c_double),
                ("random_bytes", ctypes.c_int)]


def lz_params(copy_prob=0.5, random_bytes=False):
    """LZ4/Snappy content: 64-symbol Zipf(1.1) literals (mean run 8), copies of
    length 4-255 (geometric mean 16) at offsets uniform in 1..min(pos, 65535)."""
    return GenParams(copy_prob, 64, 1.1, 8.0, 16.0, 4, 255, 65535, 0.0, 1.0,
                     1 if random_bytes else 0)


_wl = None
_lz4 = None


def _wlib():
    global _wl
    if _wl is None:
        if not os.path.exists(WORKLOAD_LIB):
            raise RuntimeError("libcudec_workload.so is not built: run "
                               "`python -m cudec_b200.build`")
        _wl = ctypes.CDLL(WORKLOAD_LIB)
        _wl.gen_chunk.argtypes = [ctypes.c_uint64, ctypes.c_void_p,
                                  ctypes.c_uint64, ctypes.POINTER(GenParams)]
        _wl.gen_batch.argtypes = [ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.POINTER(GenParams), ctypes.c_void_p,
                                  ctypes.c_uint64, ctypes.c_int]
    return _wl


def chunk_seed(base_seed, config_id, index):
    return (base_seed ^ (config_id << 32) ^ index) & 0xFFFFFFFFFFFFFFFF


def generate(sizes, params, param_idx=None, seeds=None, threads=None):
    """Generate len(sizes) chunks into one contiguous uint8 buffer.
    Returns (buffer, offsets)."""
    sizes = np.asarray(sizes, dtype=np.uint64)
    n = len(sizes)
    offsets = np.zeros(n, dtype=np.uint64)
    if n > 1:
        offsets[1:] = np.cumsum(sizes[:-1])
    buf = np.empty(int(sizes.sum()) if n else 0, dtype=np.uint8)
    if seeds is None:
        seeds = np.arange(n, dtype=np.uint64)
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    if isinstance(params, GenParams):
        params = [params]
    parr = (GenParams * len(params))(*params)
    if param_idx is None:
        param_idx = np.zeros(n, dtype=np.int32)
    param_idx = np.ascontiguousarray(param_idx, dtype=np.int32)
    threads = threads or os.cpu_count() or 1
    _wlib().gen_batch(seeds.ctypes.data, buf.ctypes.data, offsets.ctypes.data,
                      sizes.ctypes.data, parr, param_idx.ctypes.data, n, threads)
    return buf, offsets


def _lz4lib():
    global _lz4
    if _lz4 is None:
        _lz4 = ctypes.CDLL("liblz4.so.1")
        _lz4.LZ4_compress_default.argtypes = [ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_int, ctypes.c_int]
        _lz4.LZ4_compressBound.argtypes = [ctypes.c_int]
        _lz4.LZ4_decompress_safe.argtypes = [ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_int, ctypes.c_int]
    return _lz4


def lz4_version():
    return _lz4lib().LZ4_versionNumber()


def lz4_compress(data):
    """One raw LZ4 block via liblz4 LZ4_compress_default."""
    data = np.ascontiguousarray(np.frombuffer(bytes(data), dtype=np.uint8)
                                if not isinstance(data, np.ndarray) else data)
    L = _lz4lib()
    bound = L.LZ4_compressBound(len(data))
    out = np.empty(max(bound, 1), dtype=np.uint8)
    n = L.LZ4_compress_default(data.ctypes.data, out.ctypes.data, len(data), bound)
    if n <= 0 and len(data) > 0:
        raise RuntimeError("LZ4_compress_default failed")
    return out[:n].tobytes()


def lz4_decompress_ref(comp, cap):
    """liblz4 LZ4_decompress_safe: returns bytes or None when liblz4 rejects."""
    if len(comp) == 0:
        return None
    src = np.frombuffer(comp, dtype=np.uint8)
    out = np.empty(max(cap, 1), dtype=np.uint8)
    n = _lz4lib().LZ4_decompress_safe(src.ctypes.data, out.ctypes.data,
                                      len(comp), cap)
    return None if n < 0 else out[:n].tobytes()


def snappy_codec():
    import pyarrow
    return pyarrow.Codec("snappy")


def snappy_compress(data):
    return snappy_codec().compress(bytes(data), asbytes=True)


def snappy_decompress_ref(comp, declared):
    """snappy raw decode via pyarrow: bytes or None when snappy rejects."""
    try:
        return snappy_codec().decompress(comp, decompressed_size=declared,
                                         asbytes=True)
    except Exception:  # pyarrow raises on any malformed stream
        return None


class _LZ4FPrefs(ctypes.Structure):
    # LZ4F_preferences_t (lz4frame.h): frameInfo {blockSizeID, blockMode,
    # contentChecksumFlag, frameType, contentSize, dictID, blockChecksumFlag},
    # compressionLevel, autoFlush, favorDecSpeed, reserved[3].
    _fields_ = [("blockSizeID", ctypes.c_int), ("blockMode", ctypes.c_int),
                ("contentChecksumFlag", ctypes.c_int), ("frameType", ctypes.c_int),
                ("contentSize", ctypes.c_ulonglong), ("dictID", ctypes.c_uint),
                ("blockChecksumFlag", ctypes.c_int), ("compressionLevel", ctypes.c_int),
                ("autoFlush", ctypes.c_uint), ("favorDecSpeed", ctypes.c_uint),
                ("reserved", ctypes.c_uint * 3)]


def lz4f_compress(data, block_size_id=4, independent=True, content_checksum=False,
                  block_checksum=False, content_size=False, level=0):
    """One .lz4 frame via liblz4 LZ4F_compressFrame."""
    L = _lz4lib()
    data = bytes(data)
    prefs = _LZ4FPrefs()
    prefs.blockSizeID = block_size_id
    prefs.blockMode = 1 if independent else 0
    prefs.contentChecksumFlag = 1 if content_checksum else 0
    prefs.blockChecksumFlag = 1 if block_checksum else 0
    prefs.contentSize = len(data) if content_size else 0
    prefs.compressionLevel = level
    L.LZ4F_compressFrameBound.restype = ctypes.c_size_t
    L.LZ4F_compressFrameBound.argtypes = [ctypes.c_size_t, ctypes.c_void_p]
    L.LZ4F_compressFrame.restype = ctypes.c_size_t
    L.LZ4F_compressFrame.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                     ctypes.c_size_t, ctypes.c_void_p]
    L.LZ4F_isError.restype = ctypes.c_uint
    L.LZ4F_isError.argtypes = [ctypes.c_size_t]
    bound = L.LZ4F_compressFrameBound(len(data), ctypes.byref(prefs))
    out = ctypes.create_string_buffer(bound)
    n = L.LZ4F_compressFrame(out, bound, data, len(data), ctypes.byref(prefs))
    if L.LZ4F_isError(n):
        raise RuntimeError("LZ4F_compressFrame failed")
    return out.raw[:n]



def lz4f_decompress_ref(frame, cap):
    """liblz4's frame decoder (LZ4F_decompress, checksums verified): the
    bytes of the first frame when it decodes within cap bytes, else None.
    Bytes after the frame are left unread, as the reference's frame entry
    leaves them (src/frame.cpp:340-397 stops at the end mark and the content
    checksum)."""
    L = _lz4lib()
    L.LZ4F_createDecompressionContext.restype = ctypes.c_size_t
    L.LZ4F_createDecompressionContext.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint]
    L.LZ4F_freeDecompressionContext.restype = ctypes.c_size_t
    L.LZ4F_freeDecompressionContext.argtypes = [ctypes.c_void_p]
    L.LZ4F_decompress.restype = ctypes.c_size_t
    L.LZ4F_decompress.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                  ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                  ctypes.c_void_p]
    L.LZ4F_isError.restype = ctypes.c_uint
    L.LZ4F_isError.argtypes = [ctypes.c_size_t]
    dctx = ctypes.c_void_p()
    if L.LZ4F_isError(L.LZ4F_createDecompressionContext(ctypes.byref(dctx), 100)):
        raise RuntimeError("LZ4F_createDecompressionContext failed")
    try:
        src = ctypes.create_string_buffer(bytes(frame), max(len(frame), 1))
        out = ctypes.create_string_buffer(max(cap, 1))
        sp = dp = 0
        while True:
            ssz = ctypes.c_size_t(len(frame) - sp)
            dsz = ctypes.c_size_t(cap - dp)
            r = L.LZ4F_decompress(dctx, ctypes.byref(out, dp), ctypes.byref(dsz),
                                  ctypes.byref(src, sp), ctypes.byref(ssz), None)
            if L.LZ4F_isError(r):
                return None
            sp += ssz.value
            dp += dsz.value
            if r == 0:
                return out.raw[:dp]
            if ssz.value == 0 and dsz.value == 0:
                return None  # needs input that is not there, or room that is not there
    finally:
        L.LZ4F_freeDecompressionContext(dctx)

_zstd = None


def _zstdlib():
    global _zstd
    if _zstd is None:
        _zstd = ctypes.CDLL("libzstd.so.1")
        _zstd.ZSTD_createCCtx.restype = ctypes.c_void_p
        _zstd.ZSTD_freeCCtx.argtypes = [ctypes.c_void_p]
        _zstd.ZSTD_CCtx_setParameter.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        _zstd.ZSTD_CCtx_setParameter.restype = ctypes.c_size_t
        _zstd.ZSTD_compress2.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                         ctypes.c_void_p, ctypes.c_size_t]
        _zstd.ZSTD_compress2.restype = ctypes.c_size_t
        _zstd.ZSTD_compressBound.argtypes = [ctypes.c_size_t]
        _zstd.ZSTD_compressBound.restype = ctypes.c_size_t
        _zstd.ZSTD_isError.argtypes = [ctypes.c_size_t]
        _zstd.ZSTD_isError.restype = ctypes.c_uint
        _zstd.ZSTD_decompress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                          ctypes.c_size_t]
        _zstd.ZSTD_decompress.restype = ctypes.c_size_t
    return _zstd


# ZSTD_cParameter / ZSTD_cParameter values from zstd.h (stable API)
_ZSTD_C_LEVEL = 100
_ZSTD_C_WINDOWLOG = 101
_ZSTD_C_CONTENTSIZE = 200
_ZSTD_C_CHECKSUM = 201


def zstd_version():
    return _zstdlib().ZSTD_versionNumber()


def zstd_compress(data, level=3, window_log=20, checksum=False, content_size=True):
    """One Zstd frame via libzstd ZSTD_compress2 (window log, checksum flag
    and whether the frame states its content size as given)."""
    Z = _zstdlib()
    data = bytes(data)
    cctx = Z.ZSTD_createCCtx()
    try:
        for p, v in ((_ZSTD_C_LEVEL, level), (_ZSTD_C_WINDOWLOG, window_log),
                     (_ZSTD_C_CONTENTSIZE, 1 if content_size else 0),
                     (_ZSTD_C_CHECKSUM, 1 if checksum else 0)):
            if Z.ZSTD_isError(Z.ZSTD_CCtx_setParameter(cctx, p, v)):
                raise RuntimeError("ZSTD_CCtx_setParameter(%d)" % p)
        bound = Z.ZSTD_compressBound(len(data))
        out = ctypes.create_string_buffer(bound)
        n = Z.ZSTD_compress2(cctx, out, bound, data, len(data))
        if Z.ZSTD_isError(n):
            raise RuntimeError("ZSTD_compress2 failed")
        return out.raw[:n]
    finally:
        Z.ZSTD_freeCCtx(cctx)


def zstd_decompress_ref(frame, cap):
    """libzstd ZSTD_decompress: bytes, or None when libzstd rejects."""
    Z = _zstdlib()
    out = ctypes.create_string_buffer(max(cap, 1))
    n = Z.ZSTD_decompress(out, cap, bytes(frame), len(frame))
    return None if Z.ZSTD_isError(n) else out.raw[:n]


def zstd_params(copy_prob=0.5, rle_prob=0.1):
    """Zstd content: the LZ content generator with back-references up to
    1 MiB and 10 % of events a run of one repeated byte (mean 64)."""
    return GenParams(copy_prob, 64, 1.1, 8.0, 16.0, 4, 255, 1 << 20, rle_prob, 64.0, 0)


def mixed_sizes(n, seed, median=16384, sigma=1.2, lo=256, hi=4 << 20):
    """Lognormal chunk sizes (median, sigma), clamped to [lo, hi]."""
    rng = np.random.default_rng(seed)
    s = np.exp(np.log(median) + sigma * rng.standard_normal(n))
    return np.clip(s, lo, hi).astype(np.int64)


def mixed_batch(n, seed, formats=("lz4", "snappy"), median=16384, sigma=1.2, lo=256,
                hi=4 << 20, random_frac=0.05, threads=None, weights=None, zstd_level=3):
    """The uneven mixed batch: lognormal sizes, copy probability uniform in
    0.2-0.8 per chunk, `random_frac` of the chunks uniform random bytes, the
    format of chunk i = formats[i % len(formats)], or drawn with `weights`;
    a GDeflate chunk is one page, so its size is capped at 64 KiB.
    Returns (raws, comps, fmts) with raws as numpy views of one buffer."""
    sizes = mixed_sizes(n, seed, median, sigma, lo, hi)
    rng = np.random.default_rng(seed + 1)
    probs = rng.uniform(0.2, 0.8, n)
    rand = rng.random(n) < random_frac
    if weights is None:
        fmts = [formats[i % len(formats)] for i in range(n)]
    else:
        w = np.asarray(weights, dtype=np.float64)
        fmts = [formats[k] for k in rng.choice(len(formats), size=n, p=w / w.sum())]
    # a GDeflate chunk is one page: at most 64 KiB
    sizes = np.array([min(int(s), 65536) if f == "gdeflate" else int(s)
                      for s, f in zip(sizes, fmts)], dtype=np.int64)
    params = [(zstd_params(float(p), 0.1) if f == "zstd" else
               gdeflate_params(float(p)) if f == "gdeflate" else lz_params(float(p), bool(r)))
              for p, r, f in zip(probs, rand, fmts)]
    for i, f in enumerate(fmts):
        if f == "zstd" and rand[i]:
            params[i] = lz_params(float(probs[i]), True)
    seeds = np.array([chunk_seed(seed, 2, i) for i in range(n)], dtype=np.uint64)
    buf, offs = generate(sizes, params, param_idx=np.arange(n), seeds=seeds, threads=threads)
    raws = [buf[int(o):int(o) + int(s)] for o, s in zip(offs, sizes)]
    def one(k):
        r, f = raws[k], fmts[k]
        if f == "lz4":
            return lz4_compress(r)
        if f == "snappy":
            return snappy_compress(r)
        if f == "gdeflate":
            return gdeflate_compress(r.tobytes(), 6)
        return zstd_compress(r.tobytes(), zstd_level, 20, True)

    if n >= 256:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=min(os.cpu_count() or 1, 32)) as ex:
            comps = list(ex.map(one, range(n), chunksize=64))
    else:
        comps = [one(k) for k in range(n)]
    return raws, comps, fmts


def gdeflate_params(copy_prob=0.5):
    """GDeflate content: the generator with a 256-symbol Zipf(1.3) alphabet,
    matches of 3-258 bytes and offsets up to 32 KiB."""
    return GenParams(copy_prob, 256, 1.3, 8.0, 16.0, 3, 258, 32768, 0.0, 1.0, 0)


def _gd():
    lib = _wlib()
    if not getattr(lib, "_gd_ready", False):
        for name in ("gdeflate_compress_page", "gdeflate_compress_tilestream"):
            f = getattr(lib, name)
            f.restype = ctypes.c_size_t
            f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                          ctypes.c_int, ctypes.c_uint32]
        lib._gd_ready = True
    return lib


def gdeflate_compress(data, level=12, window=32768):
    """One GDeflate page (len(data) <= 65536) from this library's own encoder."""
    data = bytes(data)
    assert len(data) <= 65536
    cap = 2 * len(data) + 4096
    out = ctypes.create_string_buffer(cap)
    n = _gd().gdeflate_compress_page(data, len(data), out, cap, level, window)
    if n == 0:
        raise RuntimeError("gdeflate_compress_page failed")
    return out.raw[:n]


def gdeflate_tilestream(data, level=12, window=32768):
    """A TileStream container of 64 KiB GDeflate pages."""
    data = bytes(data)
    cap = 2 * len(data) + 8192 + 8 * (len(data) // 65536 + 1)
    out = ctypes.create_string_buffer(cap)
    n = _gd().gdeflate_compress_tilestream(data, len(data), out, cap, level, window)
    if n == 0:
        raise RuntimeError("gdeflate_compress_tilestream failed")
    return out.raw[:n]
