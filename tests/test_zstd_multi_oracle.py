"""Pins the multi-frame Zstd oracle (oracle_zstd_decode_multi in
oracle/zstd_oracle.c) against libzstd's ZSTD_decompress, which reads a
buffer as a sequence of Zstd and skippable frames: the same bytes on every
accepted sequence (frames without a content size and windows above 8 MB
included), the same refusals on truncated sequences, trailing bytes and
windows past libzstd's default limit, and never an accept where libzstd
refuses. The one-frame oracle (the reference's rule, pinned in
test_zstd_oracle.py) stays strict on the same inputs."""
import random

import numpy as np
import pytest

import oracle
from cudec_b200 import workload as W
from zstd_sequences import edge_cases, mutate, sequence

OK, CORRUPT, TOO_SMALL, UNSUPPORTED = 0, 2, 3, 6


def corpus(sizes, seed=3, rle=0.1):
    buf, offs = W.generate(sizes, [W.zstd_params(0.5, rle)],
                           seeds=np.arange(seed, seed + len(sizes), dtype=np.uint64))
    return [buf[int(o):int(o) + n].tobytes() for o, n in zip(offs, sizes)]


def test_sequences_match_libzstd():
    rng = random.Random(5)
    raws = corpus([0, 1, 777, 4096, 70000, 131073, 300000], seed=17) + [b"\x00" * 100000]
    for _ in range(40):
        pick = [rng.choice(raws) for _ in range(rng.randint(1, 5))]
        buf = sequence(rng, pick)
        want = b"".join(pick)
        assert W.zstd_decompress_ref(buf, len(want)) == want
        assert oracle.zstd_decode_multi(buf, len(want)) == (OK, want)
        assert oracle.zstd_decode_multi(buf, len(want) + 100) == (OK, want)
        if want:
            assert oracle.zstd_decode_multi(buf, len(want) - 1) == (TOO_SMALL, b"")
            assert W.zstd_decompress_ref(buf, len(want) - 1) is None


def test_one_frame_agrees_with_the_strict_entry():
    for raw in corpus([1, 5000, 200000], seed=23):
        f = W.zstd_compress(raw, 3, 20, True)
        assert oracle.zstd_decode_multi(f, len(raw)) == oracle.zstd_decode(f, len(raw)) == \
            (OK, raw)
        # two frames: the strict entry refuses the trailing frame, this one decodes it
        assert oracle.zstd_decode(f + f, 2 * len(raw))[0] == CORRUPT
        assert oracle.zstd_decode_multi(f + f, 2 * len(raw)) == (OK, raw + raw)


def test_edges_match_libzstd():
    raw = corpus([3000], seed=29)[0]
    f = W.zstd_compress(raw, 3, 20, True)
    for name, (buf, st, want) in edge_cases(f, raw).items():
        got = oracle.zstd_decode_multi(buf, 1 << 16)
        assert got[0] == st, name
        ref = W.zstd_decompress_ref(buf, 1 << 16)
        if st == OK:
            assert got[1] == want and ref == want, name
        else:
            assert ref is None, name


def test_wider_subset_matches_libzstd():
    """The frame-sequence reading takes what libzstd's one-shot decoder takes
    beyond the reference's subset: frames without a content size and windows
    above 8 MB (any window log up to 31); a dictionary id stays UNSUPPORTED
    and a window log above 31 is refused as libzstd refuses it. The one-frame
    reading still refuses all of them."""
    import zstd_subset
    raw = corpus([2000], seed=31)[0]
    f = W.zstd_compress(raw, 3, 20, False)
    for name, (frame, cap, libzstd_ok) in zstd_subset.refused_frames().items():
        got = oracle.zstd_decode_multi(f + frame, len(raw) + cap)
        assert oracle.zstd_decode(frame, cap)[0] == UNSUPPORTED, name
        if name == "dictionary id":
            assert got == (UNSUPPORTED, b""), name
        else:
            assert libzstd_ok, name
            want = W.zstd_decompress_ref(f + frame, len(raw) + cap)
            assert got == (OK, want), name
    # no content size, levels and checksums, alone and in sequences
    for r in corpus([1, 777, 70000, 300000], seed=33):
        for lvl in (1, 3, 19):
            for ck in (False, True):
                g = W.zstd_compress(r, lvl, 20, ck, content_size=False)
                assert g[4] >> 6 == 0 and not g[4] & 0x20  # no content size field
                assert oracle.zstd_decode(g, len(r))[0] == UNSUPPORTED
                assert oracle.zstd_decode_multi(g, len(r)) == (OK, r)
                assert oracle.zstd_decode_multi(g + f, len(r) + len(raw)) == (OK, r + raw)
                if r:
                    assert oracle.zstd_decode_multi(g, len(r) - 1)[0] == TOO_SMALL
    # a 16 MiB window (content larger than 8 MiB, no content size)
    big = corpus([12 << 20], seed=35, rle=0.05)[0]
    g = W.zstd_compress(big, 3, 24, True, content_size=False)
    wd = g[5]
    assert (1 << (10 + (wd >> 3))) > (8 << 20)
    assert oracle.zstd_decode(g, len(big))[0] == UNSUPPORTED
    assert oracle.zstd_decode_multi(g, len(big)) == (OK, big)
    assert W.zstd_decompress_ref(g, len(big)) == big
    # empty frames (one empty last raw block) by window log: up to 31 both
    # decode, above it both refuse
    magic = b"\x28\xb5\x2f\xfd"
    for exp, mant in ((14, 0), (18, 7), (21, 7), (22, 0), (31, 7)):
        fr = magic + bytes([0x00, (exp << 3) | mant]) + b"\x01\x00\x00"
        ok = 10 + exp <= 31
        assert oracle.zstd_decode_multi(fr, 64) == ((OK, b"") if ok else (UNSUPPORTED, b"")), exp
        assert (W.zstd_decompress_ref(fr, 64) == b"") == ok, exp


def test_mutated_sequences_never_accept_what_libzstd_refuses():
    rng = random.Random(33)
    raws = corpus([500, 3000, 20000], seed=37)
    n_ok = 0
    for _ in range(400):
        buf = mutate(sequence(rng, [rng.choice(raws) for _ in range(rng.randint(1, 3))]), rng)
        st, out = oracle.zstd_decode_multi(buf, 1 << 16)
        if st == OK:
            assert W.zstd_decompress_ref(buf, 1 << 16) == out
            n_ok += 1
    assert n_ok > 20


@pytest.mark.skipif(oracle.ref_twin_lib() is None, reason="reference twins not built here")
def test_single_frames_still_match_the_reference_twin():
    """On one frame with nothing after it the multi-frame reading is the
    reference's own; mutants that keep one frame agree with its twin."""
    rng = random.Random(41)
    for raw in corpus([100, 5000], seed=43):
        f = W.zstd_compress(raw, 19, 20, True)
        for _ in range(100):
            m = mutate(f, rng)
            ref = oracle.ref_zstd_decode(m, len(raw))
            got = oracle.zstd_decode_multi(m, len(raw))
            if ref[0] == OK:
                assert got == ref
