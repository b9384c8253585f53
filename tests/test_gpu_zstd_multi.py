"""GPU parity for cudec_zstd_decompress_batch_multi (chunks that hold a
sequence of Zstd and skippable frames), through the C ABI, against the
oracle's multi-frame reading (oracle_zstd_decode_multi, itself pinned to
libzstd's ZSTD_decompress): frame sequences at exact, short and generous
capacities, the edge cases around one frame, unaligned buffers, subset
refusals inside a sequence, mutated sequences, and the one-frame entry left
strict on the same chunks; frames without a content size and windows
above 8 MB, which this entry takes as libzstd's one-shot decoder does.
Destinations are poisoned; nothing past bytes_written may change."""
import json
import os
import random

import numpy as np
import pytest

import oracle
from cudec_b200 import workload as W
from zstd_sequences import edge_cases, mutate, sequence

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def corpus(sizes, seed=3):
    buf, offs = W.generate(sizes, [W.zstd_params(0.5, 0.1)],
                           seeds=np.arange(seed, seed + len(sizes), dtype=np.uint64))
    return [buf[int(o):int(o) + n].tobytes() for o, n in zip(offs, sizes)]


def run_batch(cuda, comps, caps, fmt="zstd_multi", **kw):
    from cudec_b200.device import DeviceBatch
    import torch
    b = DeviceBatch(comps, caps, device=cuda, **kw)
    assert b.run(fmt) == 0
    torch.cuda.synchronize()
    return b, b.results(), b.dst_host()


def check(b, res, dst, comps, caps, label=""):
    for i, (comp, cap) in enumerate(zip(comps, caps)):
        st, out = oracle.zstd_decode_multi(comp, cap)
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


def test_sequences(cuda):
    rng = random.Random(51)
    raws = corpus([0, 1, 777, 4096, 70000, 131073, 300000], seed=53) + [b"\x00" * 100000]
    comps, caps = [], []
    for _ in range(60):
        pick = [rng.choice(raws) for _ in range(rng.randint(1, 6))]
        buf = sequence(rng, pick)
        n = sum(len(p) for p in pick)
        for cap in (n, n + 100, max(n - 1, 0)):
            comps.append(buf)
            caps.append(cap)
    b, res, dst = run_batch(cuda, comps, caps)
    check(b, res, dst, comps, caps, "sequences")
    sts = [int(s) for s in res["status"]]
    assert sts.count(0) >= 120 and 3 in sts


def test_edge_cases(cuda):
    raw = corpus([3000], seed=59)[0]
    f = W.zstd_compress(raw, 3, 20, True)
    cases = edge_cases(f, raw)
    comps = [c[0] for c in cases.values()]
    caps = [1 << 16] * len(comps)
    b, res, dst = run_batch(cuda, comps, caps)
    check(b, res, dst, comps, caps, "edges")
    assert [int(s) for s in res["status"]] == [c[1] for c in cases.values()]


@pytest.mark.parametrize("skew", [(1, 3), (7, 15)])
def test_unaligned_buffers(cuda, skew):
    """Each frame after the first starts its output at an arbitrary offset
    inside the chunk's destination; the skews move the chunk itself too."""
    rng = random.Random(61)
    raws = corpus([1001, 33333, 70001], seed=63)
    comps = [sequence(rng, [rng.choice(raws) for _ in range(4)]) for _ in range(12)]
    caps = [len(oracle.zstd_decode_multi(c, 1 << 20)[1]) + 7 for c in comps]
    b, res, dst = run_batch(cuda, comps, caps, src_skew=skew[0], dst_skew=skew[1])
    check(b, res, dst, comps, caps, "skew")
    assert all(int(s) == 0 for s in res["status"])


def test_wider_subset(cuda):
    """Beyond the reference's subset, as libzstd's one-shot decoder: frames
    without a content size (levels 1/3/19, with and without checksums, alone
    and in sequences), a 16 MiB window, window logs at and past 31; the
    reference's other refusals next to a decodable frame. Device equals the
    oracle; the one-frame entry still refuses them."""
    import zstd_subset
    raw = corpus([2000], seed=67)[0]
    f = W.zstd_compress(raw, 3, 20, False)
    cases = zstd_subset.refused_frames()
    comps = [f + c[0] for c in cases.values()] + [c[0] + f for c in cases.values()]
    caps = [len(raw) + c[1] for c in cases.values()] * 2
    for r in corpus([1, 777, 70000, 300000], seed=69):
        for lvl in (1, 3, 19):
            for ck in (False, True):
                g = W.zstd_compress(r, lvl, 20, ck, content_size=False)
                comps += [g, g + f, g]
                caps += [len(r), len(r) + len(raw), max(len(r) - 1, 0)]
    big = corpus([12 << 20], seed=71)[0]
    comps.append(W.zstd_compress(big, 3, 24, True, content_size=False))
    caps.append(len(big))
    magic = b"\x28\xb5\x2f\xfd"
    for exp in (18, 21, 22, 31):
        comps.append(magic + bytes([0x00, exp << 3]) + b"\x01\x00\x00")
        caps.append(64)
    b, res, dst = run_batch(cuda, comps, caps)
    check(b, res, dst, comps, caps, "wide")
    sts = [int(x) for x in res["status"]]
    want = [6 if name == "dictionary id" else 0 for name in cases]
    assert sts[:2 * len(cases)] == want * 2
    assert sts[-5:] == [0, 0, 0, 6, 6]
    b1, r1, _ = run_batch(cuda, comps, caps, fmt="zstd")
    assert all(int(x) != 0 for x in r1["status"][2 * len(cases):])


def test_mutated_sequences(cuda):
    rng = random.Random(71)
    raws = corpus([500, 3000, 20000, 90000], seed=73)
    comps, caps = [], []
    for _ in range(1500):
        buf = mutate(sequence(rng, [rng.choice(raws) for _ in range(rng.randint(1, 3))]), rng)
        comps.append(buf)
        caps.append(rng.choice([1 << 16, 1 << 18]))
    b, res, dst = run_batch(cuda, comps, caps)
    check(b, res, dst, comps, caps, "mutants")
    sts = {int(s) for s in res["status"]}
    assert 0 in sts and 2 in sts


def test_one_frame_chunks_agree_with_the_strict_entry(cuda):
    """On the golden vectors the two entries agree wherever the strict one
    accepts; a skippable frame alone is UNSUPPORTED there and zero bytes
    here, and two frames are CORRUPT there and both decoded here."""
    vecs = json.load(open(os.path.join(GOLDEN, "zstd_frame.json")))["vectors"]
    comps = [bytes.fromhex(v["input_hex"]) for v in vecs]
    caps = [v["capacity"] for v in vecs]
    raw = corpus([40000], seed=79)[0]
    f = W.zstd_compress(raw, 3, 20, True)
    comps += [f + f, b"\x5a\x2a\x4d\x18" + bytes(4)]
    caps += [2 * len(raw), 64]
    b1, r1, d1 = run_batch(cuda, comps, caps, fmt="zstd")
    b2, r2, d2 = run_batch(cuda, comps, caps)
    check(b2, r2, d2, comps, caps, "golden-multi")
    for i in range(len(vecs)):
        if int(r1[i]["status"]) == 0:
            assert int(r2[i]["status"]) == 0
            n = int(r1[i]["bytes_written"])
            assert b1.output(i, d1, n) == b2.output(i, d2, n)
    k = len(vecs)
    assert [int(r1[k]["status"]), int(r1[k + 1]["status"])] == [2, 6]
    assert [int(r2[k]["status"]), int(r2[k + 1]["status"])] == [0, 0]
    assert int(r2[k]["bytes_written"]) == 2 * len(raw)
