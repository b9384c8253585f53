"""Determinism across launch geometries and stream splits (the reference's
tests/determinism_gpu.cu: geometries x runs plus a three-stream split).

One batch - the headline shape at reduced count, uneven sizes, incompressible
chunks and mutants - must give identical records and bytes on every run and
every path: the batch entry run five times, the batch split into three
sub-batches decoded concurrently on three streams, and the persistent mixed
plan under its default shapes and under the shapes its autotuner picks.
"""
import hashlib
import random

import numpy as np
import pytest

import cudec_b200 as cd
import oracle
from cudec_b200 import workload as W

pytestmark = pytest.mark.gpu


def build_batch(fmt):
    rng = random.Random(7)
    sizes = [65536] * 96 + [rng.randint(1, 300000) for _ in range(96)]
    probs = [rng.uniform(0.2, 0.8) for _ in sizes]
    params = [W.lz_params(p, random_bytes=(i % 17 == 0)) for i, p in enumerate(probs)]
    buf, offs = W.generate(sizes, params, param_idx=np.arange(len(sizes)))
    raws = [buf[int(o):int(o) + s].tobytes() for o, s in zip(offs, sizes)]
    comp = W.lz4_compress if fmt == "lz4" else W.snappy_compress
    comps = [comp(r) for r in raws]
    caps = [len(r) for r in raws]
    for i in range(0, len(comps), 5):
        m = bytearray(comps[i])
        m[rng.randrange(len(m))] ^= 1 << rng.randrange(8)
        comps[i] = bytes(m)
    return comps, caps


def snapshot(b):
    res, dst = b.results(), b.dst_host()
    outs = [b.output(i, dst, int(res[i]["bytes_written"])) for i in range(b.n)]
    return [(int(r["status"]), int(r["bytes_written"])) for r in res], \
        hashlib.sha256(b"".join(outs)).hexdigest()


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_runs_streams_and_plans_agree(cuda, fmt):
    import torch
    from cudec_b200.device import DeviceBatch
    comps, caps = build_batch(fmt)
    ref = {"lz4": oracle.lz4_decode, "snappy": oracle.snappy_decode}[fmt]
    want = [ref(c, cap) for c, cap in zip(comps, caps)]
    want_recs = [(st, len(out) if st == 0 else 0) for st, out in want]
    want_hash = hashlib.sha256(b"".join(out for st, out in want if st == 0)).hexdigest()
    b = DeviceBatch(comps, caps, device=cuda)
    for _ in range(5):
        b.reset()
        assert b.run(fmt) == 0
        torch.cuda.synchronize()
        assert snapshot(b) == (want_recs, want_hash)
    # three sub-batches, three streams, launched back to back
    parts = [(0, 61), (61, 130), (130, len(comps))]
    subs = [DeviceBatch(comps[a:z], caps[a:z], device=cuda) for a, z in parts]
    streams = [torch.cuda.Stream(cuda) for _ in parts]
    torch.cuda.synchronize()
    for sb, st in zip(subs, streams):
        assert sb.run(fmt, st) == 0
    torch.cuda.synchronize()
    recs, outs = [], []
    for sb in subs:
        res, dst = sb.results(), sb.dst_host()
        recs += [(int(r["status"]), int(r["bytes_written"])) for r in res]
        outs += [sb.output(i, dst, int(res[i]["bytes_written"])) for i in range(sb.n)]
    assert (recs, hashlib.sha256(b"".join(outs)).hexdigest()) == (want_recs, want_hash)
    # the persistent mixed plan: default shapes, then the tuned ones
    plan = cd.MixedPlan()
    fmts = [fmt] * len(comps)
    for tune in (False, True, False):
        b.reset()
        assert b.run_mixed(plan, fmts, tune=tune) == 0
        torch.cuda.synchronize()
        assert snapshot(b) == (want_recs, want_hash), ("mixed", tune, plan.tuning())
    plan.close()
