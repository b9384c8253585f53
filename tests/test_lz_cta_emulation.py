"""The CTA-per-chunk LZ4/Snappy decoder's algorithm, checked on the CPU.

cudec_b200/csrc/lz_cta_kernel.cuh writes every phase of the kernel as
per-thread code between barriers; compiled for the host, the same source runs
each phase for all threads in turn (tests/native/lz_cta_emul.cpp). These
tests drive that emulation through the corpora the GPU tests use - the
reference's golden vectors, hostile shapes, sizes up to 4 MiB with
incompressible chunks, short periods and long overlapping matches, content at
the length encodings' edges, unaligned buffers and deep mutants - and require
the oracle's status, bytes and untouched tail past bytes_written. The GPU
tests run the same source as the device kernel.
"""
import ctypes
import hashlib
import json
import os
import random
import subprocess

import numpy as np
import pytest

import oracle
from cudec_b200 import workload as W
from lz_blocks import lz4_block, snappy_block, straddle_blocks

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
FMT = {"lz4": 0, "snappy": 1}
ORACLE = {"lz4": oracle.lz4_decode, "snappy": oracle.snappy_decode}
COMPRESS = {"lz4": W.lz4_compress, "snappy": W.snappy_compress}


@pytest.fixture(scope="module")
def emul():
    out_dir = os.path.join(HERE, "native", "_build")
    os.makedirs(out_dir, exist_ok=True)
    so = os.path.join(out_dir, "liblzc_emul.so")
    srcs = [os.path.join(HERE, "native", "lz_cta_emul.cpp"),
            os.path.join(ROOT, "cudec_b200", "csrc", "lz_cta_kernel.cuh"),
            os.path.join(ROOT, "cudec_b200", "csrc", "lz_ladder.cuh")]
    if not os.path.exists(so) or any(os.path.getmtime(s) > os.path.getmtime(so) for s in srcs):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-Wextra",
                        "-I" + os.path.join(ROOT, "include"),
                        "-I" + os.path.join(ROOT, "cudec_b200", "csrc"), srcs[0], "-o", so],
                       check=True)
    lib = ctypes.CDLL(so)
    lib.lzc_emulate.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
    return lib


def decode(lib, fmt, comp, cap, skew=0):
    """(status, output, bytes past the output up to the capacity)."""
    src = np.zeros(len(comp) + 64 + skew, dtype=np.uint8)
    src[32 + skew:32 + skew + len(comp)] = np.frombuffer(comp, dtype=np.uint8)
    dst = np.full(cap + 64, 0xA5, dtype=np.uint8)
    w = ctypes.c_uint64(0)
    st = lib.lzc_emulate(FMT[fmt], src.ctypes.data + 32 + skew, len(comp),
                         dst.ctypes.data + 16 + (skew * 5) % 16, cap, ctypes.byref(w))
    o = 16 + (skew * 5) % 16
    return st, dst[o:o + w.value].tobytes(), dst[o + w.value:o + cap].tobytes()


def check(lib, fmt, comps, caps, label, skew=True):
    for i, (c, cap) in enumerate(zip(comps, caps)):
        st, out, tail = decode(lib, fmt, c, cap, (i % 16) if skew else 0)
        want_st, want = ORACLE[fmt](c, cap)
        assert st == want_st, (label, i, st, want_st, len(c), cap)
        if st == 0:
            assert out == want, (label, i, "bytes differ")
            assert tail == b"\xa5" * len(tail), (label, i, "wrote past bytes_written")


def gen(sizes, probs=None, randoms=(), seed=1):
    n = len(sizes)
    probs = probs or [0.5] * n
    params = [W.lz_params(p, random_bytes=(i in randoms)) for i, p in enumerate(probs)]
    buf, offs = W.generate(sizes, params, param_idx=np.arange(n),
                           seeds=np.array([W.chunk_seed(seed, 0, i) for i in range(n)],
                                          dtype=np.uint64))
    return [buf[int(o):int(o) + int(s)].tobytes() for o, s in zip(offs, sizes)]


@pytest.mark.parametrize("fmt,fixture", [("lz4", "lz4_block.json"),
                                         ("snappy", "snappy_block.json")])
def test_golden_vectors(emul, fmt, fixture):
    for v in json.load(open(os.path.join(GOLDEN, fixture)))["vectors"]:
        st, out, _ = decode(emul, fmt, bytes.fromhex(v["input_hex"]), v["capacity"])
        assert st == v["expect_status"], v["name"]
        if st == 0:
            assert hashlib.sha256(out).hexdigest() == v["expect_sha256"], v["name"]


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_sizes_probabilities_and_incompressible(emul, fmt):
    sizes = [1, 2, 5, 12, 13, 31, 64, 100, 1000, 4095, 4096, 4097, 65535, 65536,
             65537, 100000, 262144, 1 << 20, 4 << 20]
    probs = [0.2 + 0.6 * (i % 7) / 6 for i in range(len(sizes))]
    raws = gen(sizes, probs, randoms={3, 9, 16, 18}, seed=2)
    check(emul, fmt, [COMPRESS[fmt](r) for r in raws], sizes, "sizes")


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_periods_long_matches_and_straddles(emul, fmt):
    raws = [b"ab" * 5000, b"x" + b"abc" * 7000, b"0123456789abcde" * 900,
            b"q" * 3 + b"\x00\x01" * 9000, bytes(range(7)) * 3000,
            b"\x5a" * 65536, bytes((0, 255)) * 40000, b"abc" * 300000,
            bytes(range(256)) * 4096, b"\x00" * (2 << 20)]
    check(emul, fmt, [COMPRESS[fmt](r) for r in raws], [len(r) for r in raws], "periods")
    make = lz4_block if fmt == "lz4" else snappy_block
    comps = [make(s, t) for s, t in straddle_blocks(11)]
    caps = [len(ORACLE[fmt](c, 1 << 16)[1]) for c in comps]
    check(emul, fmt, comps, caps, "straddle")


def boundary_content(rng, n):
    lits = (1, 14, 15, 16, 59, 60, 61, 268, 269, 270, 271, 524, 525, 526)
    matches = (4, 18, 19, 20, 64, 65, 272, 273, 274, 275, 528, 529, 530)
    out = bytearray(rng.randbytes(64))
    while len(out) < n:
        out += rng.randbytes(rng.choice(lits))
        m = rng.choice(matches)
        off = rng.randint(1, min(len(out), 65535))
        for _ in range(m):
            out.append(out[-off])
    return bytes(out[:n])


def mutate(c, rng):
    b = bytearray(c)
    r = rng.random()
    if r < 0.15:
        return bytes(b[:rng.randrange(len(b))])
    if r < 0.3 and len(b) > 16:
        a, z = rng.randrange(len(b) - 8), rng.randrange(len(b) - 8)
        n = rng.randint(1, 8)
        b[a:a + n] = b[z:z + n]
        return bytes(b)
    for _ in range(rng.randint(1, 3)):
        i = rng.randrange(len(b))
        k = rng.random()
        if k < 0.3:
            b[i] = 0xFF
        elif k < 0.5:
            b[i] = rng.choice((0x0F, 0xF0, 0xFF, 0x00))
        elif k < 0.7 and i + 1 < len(b):
            b[i] = rng.randrange(256)
            b[i + 1] = rng.randrange(256)
        else:
            b[i] ^= 1 << rng.randrange(8)
    return bytes(b)


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_length_edges_and_deep_mutants(emul, fmt):
    rng = random.Random(31)
    sizes = [100, 5000, 30000, 65536, 131072]
    raws = [boundary_content(rng, n) for n in sizes]
    comps = [COMPRESS[fmt](r) for r in raws]
    check(emul, fmt, comps, sizes, "edges")
    mc, mcap = [], []
    for r, c in zip(raws, comps):
        for _ in range(60):
            mc.append(mutate(c, rng))
            mcap.append(rng.choice([len(r), len(r) - 1, len(r) + 100, len(r) // 2]))
    check(emul, fmt, mc, mcap, "mutants")


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_hostile_shapes(emul, fmt):
    shapes = []
    for n in (1, 2, 15, 16, 255, 4096, 20000):
        shapes += [b"\xff" * n, b"\x00" * n, b"\xf0" + b"\xff" * n, b"\x0f\x01\x00" + b"\xff" * n,
                   b"\x1f" + b"A" + b"\x00\x00" + b"\xff" * n + b"\x10A"]
    comps, caps = [], []
    for s in shapes:
        for cap in (0, 1, 64, 70000):
            comps.append(s)
            caps.append(cap)
    check(emul, fmt, comps, caps, "hostile")
