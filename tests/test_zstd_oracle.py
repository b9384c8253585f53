"""Pins the Zstd oracle (oracle/zstd_oracle.c) before it checks the GPU path:
the reference's fuzz seeds (tests/golden/zstd_frame.json), libzstd on seeded
corpora (levels 1/3/19, checksum on and off, RLE-heavy content), and the
reference's own twin driver on mutants (statuses and bytes identical)."""
import hashlib
import json
import os
import random

import numpy as np
import pytest

import oracle
from cudec_b200 import workload as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def corpus(sizes, seed=3, rle=0.1):
    buf, offs = W.generate(sizes, [W.zstd_params(0.5, rle)],
                           seeds=np.arange(seed, seed + len(sizes), dtype=np.uint64))
    return [buf[int(o):int(o) + n].tobytes() for o, n in zip(offs, sizes)]


def test_zstd_oracle_matches_golden():
    vecs = json.load(open(os.path.join(GOLDEN, "zstd_frame.json")))["vectors"]
    assert len(vecs) >= 20
    for v in vecs:
        st, out = oracle.zstd_decode(bytes.fromhex(v["input_hex"]), v["capacity"])
        assert st == v["expect_status"], v["name"]
        if st == 0:
            assert hashlib.sha256(out).hexdigest() == v["expect_sha256"], v["name"]


def test_zstd_oracle_decodes_libzstd_frames():
    raws = corpus([1, 777, 131072, 300000, 1 << 20]) + [b"\x00" * 500000,
                                                        bytes(range(256)) * 900]
    for raw in raws:
        for lvl in (1, 3, 19):
            for ck in (False, True):
                f = W.zstd_compress(raw, lvl, 20, ck)
                st, out = oracle.zstd_decode(f, len(raw))
                assert st == 0 and out == raw, (len(raw), lvl, ck)
                assert W.zstd_decompress_ref(f, len(raw)) == raw
    # capacity below the declared content size
    f = W.zstd_compress(raws[2], 3)
    assert oracle.zstd_decode(f, len(raws[2]) - 1)[0] == 3


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


@pytest.mark.skipif(oracle.ref_twin_lib() is None, reason="reference twins not built here")
def test_zstd_oracle_equals_reference_twin_on_mutants():
    rng = random.Random(21)
    n = 0
    for raw in corpus([100, 5000, 70000], seed=9):
        for lvl in (1, 19):
            f = W.zstd_compress(raw, lvl, 20, lvl == 19)
            for _ in range(120):
                m = mutate(f, rng)
                cap = rng.choice([len(raw), len(raw) + 3, max(len(raw) - 2, 0)])
                assert oracle.zstd_decode(m, cap) == oracle.ref_zstd_decode(m, cap)
                n += 1
    assert n >= 700


def test_zstd_oracle_agrees_with_libzstd_on_mutants():
    """Fail-open direction: where the oracle accepts, libzstd accepts the same
    bytes."""
    rng = random.Random(22)
    for raw in corpus([3000, 40000], seed=13):
        f = W.zstd_compress(raw, 3, 20, True)
        for _ in range(150):
            m = mutate(f, rng)
            st, out = oracle.zstd_decode(m, 1 << 20)
            if st == 0:
                assert W.zstd_decompress_ref(m, 1 << 20) == out


def test_subset_refusals_match_reference():
    """Valid frames outside the subset (skippable, no content size, a
    dictionary id, a 16 MB window): the oracle and the reference twin both
    refuse them as UNSUPPORTED, while libzstd decodes those that need no
    dictionary, so the refusal is a scope line, not a malformed input."""
    import zstd_subset
    for name, (frame, cap, libzstd_ok) in zstd_subset.refused_frames().items():
        assert oracle.zstd_decode(frame, cap) == (6, b""), name
        if oracle.ref_twin_lib() is not None:
            assert oracle.ref_zstd_decode(frame, cap)[0] == 6, name
        assert (W.zstd_decompress_ref(frame, cap) is not None) == libzstd_ok, name
