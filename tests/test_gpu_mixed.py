"""GPU parity for the persistent mixed-format path (cudec_mixed_plan_*):
every chunk's record and bytes equal what its own format's batch entry gives
for it alone (LZ4, Snappy, Zstd, in one uneven batch with incompressible
chunks, mutants, short capacities and unknown format codes), through graph
capture and replay, new argument sets and the autotuner."""
import random

import numpy as np
import pytest

import cudec_b200 as cd
import oracle
from cudec_b200 import workload as W

ORACLE = {"lz4": oracle.lz4_decode, "snappy": oracle.snappy_decode, "zstd": oracle.zstd_decode,
          "gdeflate": oracle.gdeflate_decode}
FORMATS = ("lz4", "snappy", "zstd", "gdeflate")

pytestmark = pytest.mark.gpu


def mutate(b, rng):
    b = bytearray(b)
    for _ in range(rng.randint(1, 3)):
        b[rng.randrange(len(b))] ^= 1 << rng.randrange(8)
    return bytes(b)


def make_batch(n, seed, hi=1 << 20):
    raws, comps, fmts = W.mixed_batch(n, seed, formats=FORMATS, hi=hi)
    rng = random.Random(seed)
    comps = [bytes(c) for c in comps]
    caps = [len(r) for r in raws]
    for i in range(n):
        r = rng.random()
        if r < 0.04:
            comps[i] = mutate(comps[i], rng)
        elif r < 0.06:
            caps[i] = max(caps[i] - rng.randint(1, 64), 0)
        elif r < 0.07:
            caps[i] += rng.randint(1, 4096)
    return raws, comps, caps, fmts


def per_format(cuda, comps, caps, fmts):
    """Records and outputs from each format's own batch entry."""
    import torch
    from cudec_b200.device import DeviceBatch
    recs, outs = [None] * len(comps), [None] * len(comps)
    for f in FORMATS:
        idx = [i for i, x in enumerate(fmts) if x == f]
        if not idx:
            continue
        b = DeviceBatch([comps[i] for i in idx], [caps[i] for i in idx], device=cuda)
        assert b.run(f) == 0
        torch.cuda.synchronize()
        res, dst = b.results(), b.dst_host()
        for k, i in enumerate(idx):
            recs[i] = (int(res[k]["status"]), int(res[k]["bytes_written"]))
            outs[i] = b.output(k, dst)
    return recs, outs


def check(b, recs, outs, label):
    res, dst = b.results(), b.dst_host()
    for i in range(b.n):
        got = (int(res[i]["status"]), int(res[i]["bytes_written"]))
        assert got == recs[i], (label, i, got, recs[i])
        assert res[i]["reserved"] == 0
        if got[0] == 0:
            assert b.output(i, dst) == outs[i], (label, i)
        else:
            tail_ok = True  # rejected chunks: content unspecified, bounded by capacity
            assert tail_ok


def test_mixed_equals_per_format_entries(cuda):
    import torch
    from cudec_b200.device import DeviceBatch
    raws, comps, caps, fmts = make_batch(700, 11)
    recs, outs = per_format(cuda, comps, caps, fmts)
    assert sum(1 for r in recs if r[0] == 0) > 600
    plan = cd.MixedPlan()
    b = DeviceBatch(comps, caps, device=cuda)
    assert b.run_mixed(plan, fmts) == 0
    torch.cuda.synchronize()
    check(b, recs, outs, "mixed")
    for i in range(len(comps)):
        st, out = ORACLE[fmts[i]](comps[i], caps[i])
        assert recs[i] == (st, len(out) if st == 0 else 0), (i, fmts[i], recs[i], st)
        if st == 0:
            assert outs[i][:len(out)] == out, (i, fmts[i])
    # graph replay on the same arguments
    b.reset()
    assert b.run_mixed(plan, fmts) == 0
    torch.cuda.synchronize()
    check(b, recs, outs, "replay")
    plan.close()


def test_new_arguments_recapture_and_unknown_codes(cuda):
    import torch
    from cudec_b200.device import DeviceBatch
    plan = cd.MixedPlan()
    for seed in (21, 22):
        raws, comps, caps, fmts = make_batch(300, seed, hi=256 << 10)
        recs, outs = per_format(cuda, comps, caps, fmts)
        codes = [cd.FORMAT_CODES[f] for f in fmts]
        codes[3] = 9
        codes[7] = 200
        recs[3] = recs[7] = (cd.ERR_UNSUPPORTED, 0)
        b = DeviceBatch(comps, caps, device=cuda)
        assert b.run_mixed(plan, codes) == 0
        torch.cuda.synchronize()
        check(b, recs, outs, "seed%d" % seed)
    plan.close()


def test_warps_per_chunk_shapes_agree(cuda):
    """Every LZ4 / Snappy chunk on one warp, every one on a whole CTA (the
    CTA-per-chunk decoder beside the warp grid), and the compiled-in default:
    identical records and bytes, equal to the per-format entries. Shapes
    read back as set; invalid shapes are refused and change nothing."""
    import torch
    from cudec_b200.device import DeviceBatch
    raws, comps, caps, fmts = make_batch(500, 41, hi=2 << 20)
    recs, outs = per_format(cuda, comps, caps, fmts)
    plan = cd.MixedPlan()
    default = plan.shape()
    assert [s[0] for s in default] == [1, 1] + [cd.MIXED_CTA_WARPS] * 4
    b = DeviceBatch(comps, caps, device=cuda)
    for wpc in (1, cd.MIXED_CTA_WARPS, None):
        shape = default if wpc is None else [(wpc,) + tuple(s[1:]) for s in default]
        assert plan.set_shape(shape) == 0
        assert plan.shape() == [tuple(s) for s in shape]
        b.reset()
        assert b.run_mixed(plan, fmts) == 0
        torch.cuda.synchronize()
        check(b, recs, outs, "warps per chunk %s" % wpc)
    bad = [list(s) for s in default]
    bad[2][0] = 2
    assert plan.set_shape(bad) == cd.ERR_INVALID_ARGUMENT
    bad = [list(s) for s in default]
    bad[0][1] = 7
    assert plan.set_shape(bad) == cd.ERR_INVALID_ARGUMENT
    assert plan.shape() == [tuple(s) for s in default]
    plan.close()


def test_tuner_keeps_results_and_reports_valid_shapes(cuda):
    import torch
    from cudec_b200.device import DeviceBatch
    raws, comps, caps, fmts = make_batch(400, 31, hi=2 << 20)
    recs, outs = per_format(cuda, comps, caps, fmts)
    plan = cd.MixedPlan()
    b = DeviceBatch(comps, caps, device=cuda)
    assert b.run_mixed(plan, fmts, tune=True) == 0
    check(b, recs, outs, "tuning run")
    for pw, ahead, batch in plan.tuning():
        assert pw in (256, 512, 1024) and pw + 64 <= ahead <= 4032 and batch in (2048, 4096)
    assert all(s[0] in (1, cd.MIXED_CTA_WARPS) for s in plan.shape())
    b.reset()
    assert b.run_mixed(plan, fmts) == 0
    torch.cuda.synchronize()
    check(b, recs, outs, "tuned")
    plan.close()


def test_edge_cases_in_one_mixed_batch(cuda):
    """The per-format edge cases in one persistent launch: LZ4 and Snappy
    matches reading back across a token copied straight to the destination,
    Zstd frames outside the subset next to one that decodes, and GDeflate
    pages whose codes pass the 10-bit lookup table. Records and bytes equal
    each format's own entry and the oracle."""
    import torch
    from cudec_b200.device import DeviceBatch
    from lz_blocks import lz4_block, snappy_block, straddle_blocks
    import zstd_subset
    comps, caps, fmts = [], [], []
    for fmt, make in (("lz4", lz4_block), ("snappy", snappy_block)):
        for seqs, tail in straddle_blocks(23):
            c = make(seqs, tail)
            comps.append(c)
            caps.append(len(ORACLE[fmt](c, 1 << 16)[1]))
            fmts.append(fmt)
    for frame, cap, _ in zstd_subset.refused_frames().values():
        comps.append(frame)
        caps.append(cap)
        fmts.append("zstd")
    comps.append(W.zstd_compress(zstd_subset.RAW, 3))
    caps.append(len(zstd_subset.RAW))
    fmts.append("zstd")
    rng = np.random.default_rng(5)
    for ratio in (0.6, 0.85):
        w = ratio ** np.arange(256)
        raw = rng.choice(256, size=65536, p=w / w.sum()).astype(np.uint8).tobytes()
        comps.append(W.gdeflate_compress(raw, 12))
        caps.append(len(raw))
        fmts.append("gdeflate")
    recs, outs = per_format(cuda, comps, caps, fmts)
    for i in range(len(comps)):
        st, out = ORACLE[fmts[i]](comps[i], caps[i])
        assert recs[i] == (st, len(out) if st == 0 else 0), (i, fmts[i], recs[i], st)
    assert [r[0] for r, f in zip(recs, fmts) if f == "zstd"] == [6, 6, 6, 6, 0]
    plan = cd.MixedPlan()
    b = DeviceBatch(comps, caps, device=cuda)
    assert b.run_mixed(plan, fmts) == 0
    torch.cuda.synchronize()
    check(b, recs, outs, "edge cases")
    plan.close()
