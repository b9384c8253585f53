"""GPU tests of the continuous-batching server (cudec_server_*): requests
decoded while others are in flight give exactly the records and bytes they
give alone, and both equal the oracle; the device-memory budget admits
requests only when they fit; the plain (per-format, one slot) path agrees."""
import ctypes
import threading
import random
import time

import numpy as np
import pytest

import cudec_b200 as cd
import oracle
from cudec_b200 import workload as W
from cudec_b200.device import read_device

pytestmark = pytest.mark.gpu

ORACLE = {"lz4": oracle.lz4_decode, "snappy": oracle.snappy_decode, "zstd": oracle.zstd_decode,
          "gdeflate": oracle.gdeflate_decode}


def make_requests(k, seed, max_n=300, hi=256 << 10):
    rng = random.Random(seed)
    reqs = []
    for i in range(k):
        n = int(round(np.exp(rng.uniform(0, np.log(max_n)))))
        raws, comps, fmts = W.mixed_batch(n, seed * 1000 + i,
                                          formats=("lz4", "snappy", "zstd", "gdeflate"),
                                          median=32768, sigma=1.0, lo=512, hi=hi)
        caps = [len(r) for r in raws]
        if n > 3:
            caps[1] = max(caps[1] - 7, 0)  # a short capacity in most requests
        sizes = [len(c) for c in comps]
        offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
        packed = np.frombuffer(b"".join(bytes(c) for c in comps), dtype=np.uint8).copy()
        reqs.append(dict(packed=packed, offs=offs, sizes=sizes, caps=caps, fmts=fmts,
                         comps=[bytes(c) for c in comps]))
    return reqs


def collect(srv, ticket, req):
    st, recs, ptrs, lat = srv.wait(ticket)
    assert st == 0
    outs = [read_device(int(p), int(r["bytes_written"])) for p, r in zip(ptrs, recs)]
    assert srv.release(ticket) == 0
    return [(int(r["status"]), int(r["bytes_written"])) for r in recs], outs, lat


def run_together(srv, reqs, jitter=True):
    tickets = [None] * len(reqs)

    def submitter():
        rng = random.Random(5)
        for i, r in enumerate(reqs):
            st, t = srv.submit(r["packed"], r["offs"], r["sizes"], r["caps"], r["fmts"])
            assert st == 0
            tickets[i] = t
            if jitter:
                time.sleep(rng.uniform(0, 0.002))

    th = threading.Thread(target=submitter)
    th.start()
    out = []
    for i in range(len(reqs)):
        while tickets[i] is None:
            time.sleep(0.0005)
        out.append(collect(srv, tickets[i], reqs[i]))
    th.join()
    return out


def test_results_in_the_mix_equal_alone_and_oracle(cuda):
    reqs = make_requests(24, 7)
    mix = cd.Server(512 << 20, max_inflight=4)
    together = run_together(mix, reqs)
    mix.close()
    alone_srv = cd.Server(512 << 20, max_inflight=1)
    for r, (recs, outs, _) in zip(reqs, together):
        st, t = alone_srv.submit(r["packed"], r["offs"], r["sizes"], r["caps"], r["fmts"])
        assert st == 0
        recs1, outs1, _ = collect(alone_srv, t, r)
        assert recs1 == recs and outs1 == outs
        for i, (c, cap, f) in enumerate(zip(r["comps"], r["caps"], r["fmts"])):
            ost, oout = ORACLE[f](c, cap)
            assert recs[i] == (ost, len(oout) if ost == 0 else 0), (i, f)
            if ost == 0:
                assert outs[i] == oout
    alone_srv.close()


def test_budget_admission_and_oversize_reject(cuda):
    reqs = make_requests(10, 8, max_n=120)
    foot = max(256 * 2 + 49 * len(r["sizes"]) + len(r["packed"]) +
               sum((c + 15) // 16 * 16 for c in r["caps"]) + 1024 for r in reqs)
    srv = cd.Server(foot, max_inflight=4)  # roughly one request at a time fits
    got = run_together(srv, reqs, jitter=False)
    for r, (recs, outs, _) in zip(reqs, got):
        for i, (c, cap, f) in enumerate(zip(r["comps"], r["caps"], r["fmts"])):
            ost, oout = ORACLE[f](c, cap)
            assert recs[i][0] == ost
            if ost == 0:
                assert outs[i] == oout
    big = dict(reqs[0])
    st, _ = srv.submit(big["packed"], big["offs"], big["sizes"],
                       [foot] * len(big["sizes"]), big["fmts"])
    assert st == cd.ERR_INVALID_ARGUMENT
    srv.close()


def test_plain_mode_agrees(cuda):
    reqs = make_requests(8, 9)
    a = cd.Server(512 << 20, max_inflight=1, mode=cd.SERVER_PLAIN)
    b = cd.Server(512 << 20, max_inflight=2)
    ra = run_together(a, reqs, jitter=False)
    rb = run_together(b, reqs, jitter=False)
    for (x, xo, _), (y, yo, _) in zip(ra, rb):
        assert x == y and xo == yo
    a.close()
    b.close()


def test_bounded_wait(cuda):
    """cudec_server_wait_for: a deadline that passes first reports not done
    and writes nothing; a later bounded wait returns the request's records,
    which equal the oracle's; bad arguments are refused."""
    import numpy as np
    reqs = make_requests(3, 11)
    srv = cd.Server(512 << 20, max_inflight=1)
    tickets = []
    for r in reqs:
        st, t = srv.submit(r["packed"], r["offs"], r["sizes"], r["caps"], r["fmts"])
        assert st == 0
        tickets.append(t)
    for r, t in zip(reqs, tickets):
        st, done, recs, ptrs, lat = srv.wait_for(t, 0.0)
        assert st == 0
        if not done:  # nothing written on a missed deadline
            assert (recs["status"] == 0).all() and (recs["bytes_written"] == 0).all()
            assert (ptrs == 0).all()
        st, done, recs, ptrs, lat = srv.wait_for(t, 120000.0)
        assert st == 0 and done and lat >= 0
        for i, (c, cap, f) in enumerate(zip(r["comps"], r["caps"], r["fmts"])):
            ost, oout = ORACLE[f](c, cap)
            assert (int(recs[i]["status"]), int(recs[i]["bytes_written"])) == \
                (ost, len(oout) if ost == 0 else 0), (i, f)
        assert srv.release(t) == 0
    done = ctypes.c_int(0)
    assert cd.lib().cudec_server_wait_for(srv.handle, 12345, 1.0, ctypes.byref(done), None,
                                          None, None) == cd.ERR_INVALID_ARGUMENT
    assert cd.lib().cudec_server_wait_for(srv.handle, 1, -1.0, ctypes.byref(done), None,
                                          None, None) == cd.ERR_INVALID_ARGUMENT
    srv.close()
