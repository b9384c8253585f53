"""GPU parity for the LZ4 and Snappy batch entries (through the C ABI).

Every chunk's status must equal the oracle's; a successful chunk's output is
bit-exact and nothing past bytes_written is touched (destinations are
poisoned with 0xA5 and results primed with 0xFF, as the reference's
tests/gpu_fixture.cu:21,54 do). The reference's own GPU library (built from
its sources into oracle/_ref) is run on the same LZ4 inputs where present.
"""
import ctypes
import hashlib
import json
import os
import random

import numpy as np
import pytest

import oracle
from cudec_b200 import workload as W
from lz_blocks import lz4_block, snappy_block, straddle_blocks

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ORACLE = {"lz4": oracle.lz4_decode, "snappy": oracle.snappy_decode}
COMPRESS = {"lz4": W.lz4_compress, "snappy": W.snappy_compress}


def run_batch(cuda, fmt, comps, caps, **kw):
    from cudec_b200.device import DeviceBatch
    import torch
    b = DeviceBatch(comps, caps, device=cuda, **kw)
    assert b.run(fmt) == 0
    torch.cuda.synchronize()
    return b, b.results(), b.dst_host()


def check_against_oracle(fmt, b, res, dst, comps, caps, label=""):
    for i, (comp, cap) in enumerate(zip(comps, caps)):
        st, out = ORACLE[fmt](comp, cap)
        r = res[i]
        assert r["status"] == st, (label, i, int(r["status"]), st, len(comp), cap)
        assert r["reserved"] == 0
        if st == 0:
            assert r["bytes_written"] == len(out), (label, i)
            got = b.output(i, dst, len(out))
            assert got == out, (label, i, "bytes differ")
            tail = b.output(i, dst)[len(out):]
            assert tail == bytes([0xA5]) * len(tail), (label, i, "wrote past bytes_written")
        else:
            assert r["bytes_written"] == 0


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
def test_golden_vectors(cuda, fmt, fixture):
    vecs = json.load(open(os.path.join(GOLDEN, fixture)))["vectors"]
    comps = [bytes.fromhex(v["input_hex"]) for v in vecs]
    caps = [v["capacity"] for v in vecs]
    b, res, dst = run_batch(cuda, fmt, comps, caps)
    for i, v in enumerate(vecs):
        assert res[i]["status"] == v["expect_status"], v["name"]
        if v["expect_status"] == 0:
            out = b.output(i, dst, v["expect_len"])
            assert hashlib.sha256(out).hexdigest() == v["expect_sha256"], v["name"]
    check_against_oracle(fmt, b, res, dst, comps, caps, "golden")


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_seeded_sizes_and_windows(cuda, fmt):
    """Sizes from 1 B to 4 MiB: inputs spanning several 32 KiB staging windows,
    outputs far past the 64 KiB shared ring, incompressible chunks (one long
    literal run) and every copy probability."""
    sizes = [1, 2, 5, 12, 13, 31, 64, 100, 1000, 4095, 4096, 4097, 65535, 65536,
             65537, 100000, 262144, 1 << 20, 3 << 20, 4 << 20]
    probs = [0.2 + 0.6 * (i % 7) / 6 for i in range(len(sizes))]
    raws = gen(sizes, probs, randoms={3, 9, 16, 19}, seed=2)
    comps = [COMPRESS[fmt](r) for r in raws]
    caps = [len(r) for r in raws]
    b, res, dst = run_batch(cuda, fmt, comps, caps)
    check_against_oracle(fmt, b, res, dst, comps, caps, "sizes")
    assert all(res["status"] == 0)


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
@pytest.mark.parametrize("skew", [(0, 0), (1, 3), (7, 15), (13, 1)])
def test_unaligned_buffers(cuda, fmt, skew):
    raws = gen([777, 65536, 70001, 200000], seed=3)
    comps = [COMPRESS[fmt](r) for r in raws]
    caps = [len(r) + 40 for r in raws]
    b, res, dst = run_batch(cuda, fmt, comps, caps, dst_skew=skew[0], src_skew=skew[1])
    check_against_oracle(fmt, b, res, dst, comps, caps, "skew")


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_tiny_outputs_at_every_alignment(cuda, fmt):
    """Outputs shorter than a 16-byte block, and a little longer, at every
    destination misalignment: the whole output can sit inside the first
    partial block, where the aligned part of a flush is empty."""
    rng = random.Random(5)
    raws = [bytes(rng.randrange(4) + 97 for _ in range(n))
            for n in (1, 2, 3, 5, 8, 11, 12, 13, 15, 16, 17, 20, 31, 33, 47)]
    comps = [COMPRESS[fmt](r) for r in raws]
    caps = [len(r) for r in raws]
    for skew in range(16):
        b, res, dst = run_batch(cuda, fmt, comps, caps, dst_skew=skew, src_skew=(skew * 3) % 16)
        check_against_oracle(fmt, b, res, dst, comps, caps, "tiny skew %d" % skew)
        assert all(res["status"] == 0)


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_short_periods_at_every_alignment(cuda, fmt):
    """Matches whose period is shorter than a 16-byte vector, starting in the
    first vectors of the destination, for every destination misalignment."""
    raws = [b"ab" * 5000, b"x" + b"abc" * 7000, b"0123456789abcde" * 900,
            b"q" * 3 + b"\x00\x01" * 9000, bytes(range(7)) * 3000]
    comps = [COMPRESS[fmt](r) for r in raws]
    caps = [len(r) for r in raws]
    for skew in range(16):
        b, res, dst = run_batch(cuda, fmt, comps, caps, dst_skew=skew, src_skew=(skew * 7) % 16)
        check_against_oracle(fmt, b, res, dst, comps, caps, "period skew %d" % skew)
        assert all(res["status"] == 0)


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_mutants_match_oracle(cuda, fmt):
    rng = random.Random(9)
    raws = gen([50, 3000, 40000, 70000], probs=[0.3, 0.5, 0.7, 0.5], seed=4)
    comps, caps = [], []
    for r in raws:
        c = COMPRESS[fmt](r)
        for k in range(40):
            b = bytearray(c)
            if k % 3 == 0:
                b = b[:rng.randrange(max(len(b), 1))]
            else:
                for _ in range(rng.randint(1, 4)):
                    if b:
                        b[rng.randrange(len(b))] ^= 1 << rng.randrange(8)
            comps.append(bytes(b))
            caps.append(rng.choice([len(r), len(r) + 11, max(len(r) - 7, 0)]))
    b, res, dst = run_batch(cuda, fmt, comps, caps)
    check_against_oracle(fmt, b, res, dst, comps, caps, "mutants")


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_overlapping_and_long_matches(cuda, fmt):
    raws = [b"\x5a" * 65536, bytes((0, 255)) * 40000, b"abc" * 300000,
            bytes(range(256)) * 4096, b"\x00" * (2 << 20)]
    comps = [COMPRESS[fmt](r) for r in raws]
    caps = [len(r) for r in raws]
    b, res, dst = run_batch(cuda, fmt, comps, caps)
    check_against_oracle(fmt, b, res, dst, comps, caps, "overlap")
    assert all(res["status"] == 0)


def boundary_content(rng, n):
    """Random literal runs and exact repeats whose lengths sit on the length
    encodings' edges: LZ4 literal runs of 14-16, 268-271 and 524-526 bytes
    (one, two and three extension bytes, 255 in the middle), matches of
    18-20, 272-275 and 528-530 bytes, offsets anywhere back to 64 KiB."""
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


def mutate_lz(c, rng):
    """Damage aimed at the token chain: 0xFF and 15-nibble bytes (long
    extension runs), bit flips, two-byte offset changes, truncations and a
    spliced span."""
    b = bytearray(c)
    if not b:
        return bytes(b)
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
def test_walk_paths_and_deep_mutants_match_oracle(cuda, fmt):
    """The group walk's paths - the branch-free step, extension bytes of 255,
    tokens at the input window's edge, the general step - on content built
    at the length encodings' edges, intact (every chunk must decode) and
    under ~1,800 mutants at exact, short and generous capacities; status and
    bytes must equal the oracle's."""
    rng = random.Random(31)
    sizes = [100, 5000, 30000, 65536, 131072, 300000]
    raws = [boundary_content(rng, n) for n in sizes]
    comps = [COMPRESS[fmt](r) for r in raws]
    caps = [len(r) for r in raws]
    b, res, dst = run_batch(cuda, fmt, comps, caps)
    check_against_oracle(fmt, b, res, dst, comps, caps, "boundaries")
    assert all(res["status"] == 0)
    mcomps, mcaps = [], []
    for r, c in zip(raws, comps):
        for _ in range(300):
            mcomps.append(mutate_lz(c, rng))
            mcaps.append(rng.choice([len(r), len(r) - 1, len(r) + 100, len(r) // 2]))
    b, res, dst = run_batch(cuda, fmt, mcomps, mcaps)
    check_against_oracle(fmt, b, res, dst, mcomps, mcaps, "deep mutants")
    sts = {int(x) for x in res["status"]}
    assert 0 in sts and 2 in sts


def test_config1_shape_bit_exact_and_deterministic(cuda):
    """1,024 x 64 KiB LZ4 chunks (the headline workload), twice."""
    raws = gen([65536] * 1024, seed=1234)
    comps = [W.lz4_compress(r) for r in raws]
    caps = [65536] * 1024
    b, res, dst = run_batch(cuda, "lz4", comps, caps)
    assert all(res["status"] == 0) and all(res["bytes_written"] == 65536)
    for i in range(0, 1024, 37):
        assert b.output(i, dst, 65536) == raws[i]
    h1 = hashlib.sha256(dst.tobytes()).hexdigest()
    b.reset()
    import torch
    assert b.run("lz4") == 0
    torch.cuda.synchronize()
    assert hashlib.sha256(b.dst_host().tobytes()).hexdigest() == h1
    full = b.dst_host()
    assert all(b.output(i, full, 65536) == raws[i] for i in range(1024))


@pytest.mark.skipif(oracle.ref_gpu_lib() is None, reason="reference library not built")
def test_matches_reference_gpu_library(cuda):
    """Same inputs through the reference's own cudec_lz4_decompress_batch
    (compiled for sm_100a from its sources): identical records and bytes."""
    import torch
    rng = random.Random(12)
    raws = gen([100, 5000, 65536, 65536, 300000], seed=5)
    comps, caps = [], []
    for r in raws:
        c = W.lz4_compress(r)
        comps.append(c)
        caps.append(len(r))
        for _ in range(8):
            m = bytearray(c)
            m[rng.randrange(len(m))] ^= 1 << rng.randrange(8)
            comps.append(bytes(m))
            caps.append(len(r))
    b, res, dst = run_batch(cuda, "lz4", comps, caps)
    ref = oracle.ref_gpu_lib()
    b.reset()
    st = ref.cudec_lz4_decompress_batch(*[ctypes.c_void_p(a) for a in b.args()[:4]],
                                        b.n, ctypes.c_void_p(b.args()[5]), None)
    assert st == 0
    torch.cuda.synchronize()
    rres, rdst = b.results(), b.dst_host()
    assert (rres["status"] == res["status"]).all()
    assert (rres["bytes_written"] == res["bytes_written"]).all()
    for i in range(b.n):
        if res[i]["status"] == 0:
            n = int(res[i]["bytes_written"])
            assert b.output(i, dst, n) == b.output(i, rdst, n)


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_sources_straddling_a_direct_copy(cuda, fmt):
    """Short matches right after a token copied straight to the destination,
    reading back across its end, decode as the oracle does."""
    make = lz4_block if fmt == "lz4" else snappy_block
    comps = [make(s, t) for s, t in straddle_blocks(11)]
    caps = [ORACLE[fmt](c, 1 << 16)[1].__len__() for c in comps]
    assert all(ORACLE[fmt](c, cap)[0] == 0 for c, cap in zip(comps, caps))
    b, res, dst = run_batch(cuda, fmt, comps, caps)
    check_against_oracle(fmt, b, res, dst, comps, caps, "straddle")
    assert (res["status"] == 0).all()
