"""GPU parity for the Zstd batch entry (cudec_zstd_decompress_batch, through
the C ABI): the reference's fuzz seeds and libzstd frames (tests/golden/
zstd_frame.json), libzstd frames at levels 1/3/19 with and without checksum,
raw and RLE blocks, multi-block frames with matches reaching back across
blocks up to a 1 MiB window, and mutants whose status must equal the oracle's
(oracle/zstd_oracle.c, itself pinned to the reference's twin driver
tests/zstd_twin_driver.h). Destinations are poisoned; nothing past
bytes_written may change."""
import hashlib
import json
import os
import random

import numpy as np
import pytest

import oracle
from cudec_b200 import workload as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def run_batch(cuda, comps, caps, **kw):
    from cudec_b200.device import DeviceBatch
    import torch
    b = DeviceBatch(comps, caps, device=cuda, **kw)
    assert b.run("zstd") == 0
    torch.cuda.synchronize()
    return b, b.results(), b.dst_host()


def check(b, res, dst, comps, caps, label=""):
    for i, (comp, cap) in enumerate(zip(comps, caps)):
        st, out = oracle.zstd_decode(comp, cap)
        r = res[i]
        assert r["status"] == st, (label, i, int(r["status"]), st, len(comp), cap)
        assert r["reserved"] == 0
        if st == 0:
            assert r["bytes_written"] == len(out), (label, i)
            assert b.output(i, dst, len(out)) == out, (label, i, "bytes differ")
            tail = b.output(i, dst)[len(out):]
            assert tail == bytes([0xA5]) * len(tail), (label, i, "wrote past bytes_written")
        else:
            assert r["bytes_written"] == 0, (label, i)


def corpus(sizes, seed=3, copy=0.5, rle=0.1):
    buf, offs = W.generate(sizes, [W.zstd_params(copy, rle)],
                           seeds=np.arange(seed, seed + len(sizes), dtype=np.uint64))
    return [buf[int(o):int(o) + n].tobytes() for o, n in zip(offs, sizes)]


def test_golden_vectors(cuda):
    vecs = json.load(open(os.path.join(GOLDEN, "zstd_frame.json")))["vectors"]
    comps = [bytes.fromhex(v["input_hex"]) for v in vecs]
    caps = [v["capacity"] for v in vecs]
    b, res, dst = run_batch(cuda, comps, caps)
    for i, v in enumerate(vecs):
        assert res[i]["status"] == v["expect_status"], v["name"]
        if v["expect_status"] == 0:
            out = b.output(i, dst, v["expect_len"])
            assert hashlib.sha256(out).hexdigest() == v["expect_sha256"], v["name"]
    check(b, res, dst, comps, caps, "golden")


def test_libzstd_levels_and_checksums(cuda):
    raws = corpus([1, 5, 777, 4096, 131072, 131073, 300000, 1 << 20]) + [
        b"", b"\x00" * 500000, bytes(range(256)) * 900, os.urandom(0) + bytes(
            np.random.default_rng(5).integers(0, 256, 200000, dtype=np.uint8))]
    comps, caps = [], []
    for raw in raws:
        for lvl in (1, 3, 19):
            for ck in (False, True):
                comps.append(W.zstd_compress(raw, lvl, 20, ck))
                caps.append(len(raw))
    b, res, dst = run_batch(cuda, comps, caps)
    check(b, res, dst, comps, caps, "libzstd")
    assert all(int(r["status"]) == 0 for r in res)


@pytest.mark.parametrize("skew", [(0, 0), (1, 3), (7, 15)])
def test_unaligned_buffers(cuda, skew):
    raws = corpus([1000, 70000, 200000], seed=31)
    comps = [W.zstd_compress(r, 3, 20, True) for r in raws]
    caps = [len(r) + 5 for r in raws]
    b, res, dst = run_batch(cuda, comps, caps, src_skew=skew[0], dst_skew=skew[1])
    check(b, res, dst, comps, caps, "skew")


def test_capacity_edges(cuda):
    raw = corpus([50000], seed=41)[0]
    f = W.zstd_compress(raw, 3, 20, True)
    comps = [f] * 4
    caps = [len(raw), len(raw) - 1, 0, len(raw) + 4096]
    b, res, dst = run_batch(cuda, comps, caps)
    check(b, res, dst, comps, caps, "capacity")
    assert [int(r["status"]) for r in res] == [0, 3, 3, 0]


def mutate(f, rng):
    b = bytearray(f)
    r = rng.random()
    if r < 0.2:
        b = b[:rng.randrange(len(b))]
    elif r < 0.3:
        b += bytes([rng.randrange(256)])
    else:
        for _ in range(rng.randint(1, 3)):
            b[rng.randrange(len(b))] ^= 1 << rng.randrange(8)
    return bytes(b)


def test_mutants_match_oracle(cuda):
    rng = random.Random(77)
    comps, caps = [], []
    for raw in corpus([100, 5000, 70000, 150000], seed=9):
        for lvl in (1, 3, 19):
            f = W.zstd_compress(raw, lvl, 20, lvl != 3)
            for _ in range(60):
                comps.append(mutate(f, rng))
                caps.append(rng.choice([len(raw), len(raw) + 3, max(len(raw) - 2, 0)]))
    b, res, dst = run_batch(cuda, comps, caps)
    check(b, res, dst, comps, caps, "mutants")
    sts = {int(r["status"]) for r in res}
    assert 0 in sts and 2 in sts


def mutate_deep(f, rng):
    """Damage aimed past the headers: flips and byte overwrites in the last
    three quarters of the frame (where literal and sequence sections lie),
    short truncations, and a block spliced from elsewhere in the frame."""
    b = bytearray(f)
    r = rng.random()
    lo = min(len(b) - 1, max(12, len(b) // 4))
    if r < 0.15:
        b = b[:len(b) - rng.randint(1, min(16, len(b) - 1))]
    elif r < 0.3 and len(b) > 64:
        a = rng.randrange(lo, len(b) - 8)
        c = rng.randrange(lo, len(b) - 8)
        n = rng.randint(1, 8)
        b[a:a + n] = b[c:c + n]
    elif r < 0.5:
        for _ in range(rng.randint(1, 4)):
            b[rng.randrange(lo, len(b))] = rng.randrange(256)
    else:
        for _ in range(rng.randint(1, 3)):
            b[rng.randrange(lo, len(b))] ^= 1 << rng.randrange(8)
    return bytes(b)


def test_deep_mutants_match_oracle(cuda):
    """Status parity (and bytes on success) with the oracle on ~4,000 frames
    damaged inside their literal and sequence sections, at exact, short and
    generous capacities: every reject the branch-light sequence decode and
    its per-batch checks make must be the one the serial decoder makes."""
    rng = random.Random(2024)
    comps, caps = [], []
    raws = corpus([300, 2000, 9000, 33000, 130000], seed=21, copy=0.6, rle=0.15)
    for raw in raws:
        for lvl in (1, 3, 9, 19):
            f = W.zstd_compress(raw, lvl, 20, lvl == 9)
            for _ in range(200):
                comps.append(mutate_deep(f, rng))
                caps.append(rng.choice([len(raw), len(raw) - 1, len(raw) + 100, len(raw) // 2]))
    b, res, dst = run_batch(cuda, comps, caps)
    check(b, res, dst, comps, caps, "deep mutants")
    sts = {int(r["status"]) for r in res}
    assert 0 in sts and 2 in sts and 3 in sts


def test_bench_shape_bit_exact_and_deterministic(cuda):
    """The benchmark's chunk shape (1 MiB frames, 1 MiB window, 10% RLE runs)
    at a reduced count, decoded twice: identical bytes and statuses."""
    raws = corpus([1 << 20] * 12, seed=101)
    comps = [W.zstd_compress(r, 3, 20, True) for r in raws]
    caps = [len(r) for r in raws]
    b, res, dst = run_batch(cuda, comps, caps)
    check(b, res, dst, comps, caps, "bench-shape")
    import torch
    b.reset()
    assert b.run("zstd") == 0
    torch.cuda.synchronize()
    res2, dst2 = b.results(), b.dst_host()
    assert (res2 == res).all() and (dst2 == dst).all()


def test_subset_refusals(cuda):
    """Skippable frames, frames without a content size, a dictionary id and a
    window above 8 MB are UNSUPPORTED on the device as in the oracle, next to
    a frame that decodes."""
    import zstd_subset
    cases = list(zstd_subset.refused_frames().values())
    comps = [c[0] for c in cases] + [W.zstd_compress(zstd_subset.RAW, 3)]
    caps = [c[1] for c in cases] + [len(zstd_subset.RAW)]
    b, res, dst = run_batch(cuda, comps, caps)
    check(b, res, dst, comps, caps, "subset")
    assert [int(s) for s in res["status"]] == [6] * len(cases) + [0]
