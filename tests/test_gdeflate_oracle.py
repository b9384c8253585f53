"""Pins the GDeflate oracle (oracle/gdeflate_oracle.c) before it checks the
GPU decoder: its 32-lane refill schedule is trace-identical to the
reference's src/gdeflate_schedule.h (compiled from the reference's sources)
on random pages and operation lists; its TileStream walker gives the
reference walker's verdicts and tile tables on the reference's fuzz seeds
(tests/golden/tilestream.json) and on mutants; this library's encoder round-trips
through it. Symbol-level parity with the GDeflate reference decoder is
unpinned: the reference holds no decoder and no page vectors."""
import hashlib
import json
import os
import random

import numpy as np
import pytest

import oracle
from cudec_b200 import workload as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(oracle.ref_twin_lib() is None,
                               reason="reference twins not built here")


@needs_ref
def test_schedule_trace_equals_reference():
    rng = random.Random(17)
    for seed in range(60):
        words = rng.choice([0, 5, 31, 32, 33, 40, 64, 200, 700])
        page = bytes(rng.randrange(256) for _ in range(4 * words + rng.choice([0, 0, 0, 1, 3])))
        ops = []
        for _ in range(rng.randrange(50, 1500)):
            r = rng.random()
            if r < 0.45:
                ops.append(rng.choice([1, 2, 3, 5, 7, 8, 13, 15, 16, 24, 31, 32, 33, 40]))
            elif r < 0.85:
                ops.append(0)
            elif r < 0.9:
                ops.append(100)
            elif r < 0.95:
                ops.append(200)
            else:
                ops += [300, rng.randrange(0, 70)]
        a = oracle.gdeflate_schedule_trace(page, ops)
        b = oracle.ref_gdeflate_schedule_trace(page, ops)
        assert a.shape == b.shape and (a == b).all(), seed


def test_tilestream_matches_reference_seeds():
    vecs = json.load(open(os.path.join(GOLDEN, "tilestream.json")))["vectors"]
    assert len(vecs) >= 13
    for v in vecs:
        st, tiles, total = oracle.tilestream_parse(bytes.fromhex(v["input_hex"]),
                                                   v["tiles_capacity"])
        assert st == v["expect_status"], v["name"]
        if st == 0:
            assert tiles == v["expect_tiles"] and total == v["expect_total"], v["name"]


@needs_ref
def test_tilestream_mutants_match_reference():
    rng = random.Random(23)
    bases = [W.gdeflate_tilestream(bytes(rng.randrange(256) for _ in range(n)), 1)
             for n in (1, 65536, 65537, 200000)]
    for base in bases:
        for _ in range(300):
            b = bytearray(base[:64 + rng.randrange(64)] if rng.random() < 0.3 else base)
            for _ in range(rng.randint(1, 3)):
                b[rng.randrange(min(len(b), 40))] ^= 1 << rng.randrange(8)
            cap = rng.choice([0, 1, 2, 4, 8])
            assert oracle.tilestream_parse(bytes(b), cap) == oracle.ref_tilestream_parse(bytes(b), cap)


def test_gdeflate_golden_pages():
    vecs = json.load(open(os.path.join(GOLDEN, "gdeflate_page.json")))["vectors"]
    for v in vecs:
        st, out = oracle.gdeflate_decode(bytes.fromhex(v["input_hex"]), v["capacity"])
        assert st == v["expect_status"], v["name"]
        assert hashlib.sha256(out).hexdigest() == v["expect_sha256"], v["name"]


def test_encoder_round_trips_and_container():
    sizes = [1, 17, 127, 128, 5000, 65535, 65536]
    buf, offs = W.generate(sizes, [W.gdeflate_params(p) for p in (0.2, 0.5, 0.8)],
                           param_idx=np.arange(len(sizes)) % 3,
                           seeds=np.arange(100, 100 + len(sizes), dtype=np.uint64))
    for o, n in zip(offs, sizes):
        raw = buf[int(o):int(o) + n].tobytes()
        for lvl, win in ((1, 32768), (6, 65536), (12, 32768)):
            page = W.gdeflate_compress(raw, lvl, win)
            assert len(page) % 4 == 0 and len(page) >= 128
            st, out = oracle.gdeflate_decode(page, n)
            assert st == 0 and out == raw, (n, lvl)
            # capacity one short
            if n:
                assert oracle.gdeflate_decode(page, n - 1)[0] == 3
    raw = buf.tobytes()[:300000]
    ts = W.gdeflate_tilestream(raw, 6)
    st, tiles, total = oracle.tilestream_parse(ts, 8)
    assert st == 0 and total == len(raw) and len(tiles) == (len(raw) + 65535) // 65536
    got = b""
    for off, sz, dsz in tiles:
        s2, out = oracle.gdeflate_decode(ts[off:off + sz], dsz)
        assert s2 == 0 and len(out) == dsz
        got += out
    assert got == raw


def test_page_mutants_are_refused_or_decoded_deterministically():
    rng = random.Random(31)
    buf, offs = W.generate([20000], [W.gdeflate_params(0.5)], seeds=np.array([9], dtype=np.uint64))
    page = W.gdeflate_compress(buf.tobytes(), 12)
    statuses = set()
    for _ in range(400):
        b = bytearray(page)
        r = rng.random()
        if r < 0.2:
            b = b[:rng.randrange(len(b) + 1)]
        elif r < 0.3:
            b += bytes(4)
        else:
            for _ in range(rng.randint(1, 3)):
                b[rng.randrange(len(b))] ^= 1 << rng.randrange(8)
        cap = rng.choice([20000, 20001, 19999, 65536])
        a = oracle.gdeflate_decode(bytes(b), cap)
        assert a == oracle.gdeflate_decode(bytes(b), cap)
        statuses.add(a[0])
    assert statuses <= {0, 2, 3} and 2 in statuses


def test_library_tilestream_walker_matches_reference_seeds():
    """The shipped walker (cudec_gdeflate_tilestream_parse, host-only) gives
    the reference walker's verdicts and tables on its fuzz seeds."""
    import cudec_b200 as cd
    vecs = json.load(open(os.path.join(GOLDEN, "tilestream.json")))["vectors"]
    for v in vecs:
        st, tiles, total = cd.tilestream_parse(bytes.fromhex(v["input_hex"]), v["tiles_capacity"])
        assert st == v["expect_status"], v["name"]
        if st == 0:
            assert tiles == v["expect_tiles"] and total == v["expect_total"], v["name"]
    rng = random.Random(29)
    base = W.gdeflate_tilestream(bytes(rng.randrange(256) for _ in range(200000)), 1)
    for _ in range(300):
        b = bytearray(base[:64])
        b[rng.randrange(40)] ^= 1 << rng.randrange(8)
        cap = rng.choice([0, 1, 3, 4, 8])
        assert cd.tilestream_parse(bytes(b), cap) == oracle.tilestream_parse(bytes(b), cap)


def test_encoder_round_trip_sweep():
    """This library's encoder and the oracle decoder round-trip content that
    drives every part of the page format: skewed bytes (codes up to the
    15-bit limit), random bytes (stored blocks), short periods (match
    distances 1-16), long runs (258-byte matches) and text-like mixes, at
    three levels and two windows, at sizes around the page's edges."""
    rng = np.random.default_rng(61)

    def skewed(n, ratio):
        w = ratio ** np.arange(256)
        return rng.choice(256, size=n, p=w / w.sum()).astype(np.uint8).tobytes()

    def periodic(n, d):
        base = rng.integers(0, 256, d, dtype=np.uint8).tobytes()
        return (base * (n // d + 1))[:n]

    contents = []
    for n in (1, 2, 3, 258, 259, 4096, 32768, 65535, 65536):
        contents += [skewed(n, 0.7), rng.integers(0, 256, n, dtype=np.uint8).tobytes(),
                     periodic(n, 1 + n % 16), bytes([n % 251]) * n]
    mix = b"".join([skewed(3000, 0.9), periodic(5000, 7), bytes(4000), skewed(2000, 0.6)])
    contents.append(mix[:65536])
    for raw in contents:
        for lvl, win in ((1, 32768), (6, 65536), (12, 32768)):
            page = W.gdeflate_compress(raw, lvl, win)
            st, out = oracle.gdeflate_decode(page, len(raw))
            assert st == 0 and out == raw, (len(raw), lvl, win)
            if len(raw) > 0:
                assert oracle.gdeflate_decode(page, len(raw) - 1)[0] == 3, (len(raw), lvl)
