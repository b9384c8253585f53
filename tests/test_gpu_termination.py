"""Termination on the device, behind a host-side deadline.

The oracle tests prove the ladders terminate on the host; these drive the
same hostile shapes - the reference's fuzz seeds and adversarial blocks
(tests/golden), runs of 0xFF extension bytes, zero offsets, truncations and
seeded mutants of real blocks - through the batch entries on the GPU. A
decode that never finished would not return a bad status: it would hold the
launch and every stream behind it. So the launch is fenced with an event and
polled against a wall-clock deadline (the reference's
tests/termination_gpu.cu:150-165): on expiry the test reports which batch
did not finish and ends the process, which releases the launch (waiting on
the stream here would inherit the hang being reported). No case is expected
to come near the deadline; statuses and bytes are also checked against the
oracle.
"""
import json
import os
import random
import sys
import time

import pytest

import oracle
from cudec_b200 import workload as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DEADLINE_S = 60.0
ORACLE = {"lz4": oracle.lz4_decode, "snappy": oracle.snappy_decode}
COMPRESS = {"lz4": W.lz4_compress, "snappy": W.snappy_compress}


def decode_with_watchdog(cuda, fmt, comps, caps, label):
    """Submit on a private stream, record an event, poll it until the
    deadline; returns the batch once the event has completed."""
    import torch
    from cudec_b200.device import DeviceBatch
    b = DeviceBatch(comps, caps, device=cuda)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream(cuda)
    done = torch.cuda.Event()
    assert b.run(fmt, stream) == 0
    done.record(stream)
    t0 = time.monotonic()
    while not done.query():
        if time.monotonic() - t0 > DEADLINE_S:
            sys.stderr.write("FATAL: %s batch (%s, %d chunks) did not finish within %.0f s: "
                             "a non-terminating decode\n" % (label, fmt, len(comps), DEADLINE_S))
            sys.stderr.flush()
            os._exit(70)
        time.sleep(0.001)
    return b


def hostile_shapes(fmt, rng):
    """Inputs aimed at the token loop: long 0xFF runs (extension bytes that
    never end, or end past the input), tokens that claim huge lengths, zero
    and far offsets, all-zero and all-0xFF streams, every truncation of a
    short block."""
    shapes = []
    for n in (1, 2, 15, 16, 255, 4096, 65536):
        shapes.append(b"\xff" * n)
        shapes.append(b"\x00" * n)
        shapes.append(b"\xf0" + b"\xff" * n)
        shapes.append(b"\x0f\x01\x00" + b"\xff" * n)
        shapes.append(b"\x1f" + b"A" + b"\x00\x00" + b"\xff" * n + b"\x10A")
    raw = bytes(rng.randrange(4) + 65 for _ in range(3000))
    c = COMPRESS[fmt](raw)
    shapes += [c[:k] for k in range(0, min(len(c), 300))]
    return shapes


@pytest.mark.parametrize("fmt", ["lz4", "snappy"])
def test_hostile_corpus_terminates_and_matches_oracle(cuda, fmt):
    rng = random.Random(99)
    fixture = "lz4_block.json" if fmt == "lz4" else "snappy_block.json"
    vecs = json.load(open(os.path.join(GOLDEN, fixture)))["vectors"]
    comps = [bytes.fromhex(v["input_hex"]) for v in vecs]
    caps = [v["capacity"] for v in vecs]
    for s in hostile_shapes(fmt, rng):
        for cap in (0, 1, 64, 70000):
            comps.append(s)
            caps.append(cap)
    base = [W.lz_params(p) for p in (0.2, 0.5, 0.8)]
    buf, offs = W.generate([65536] * 3, base, param_idx=[0, 1, 2])
    for k in range(3):
        c = COMPRESS[fmt](buf[int(offs[k]):int(offs[k]) + 65536])
        for _ in range(400):
            m = bytearray(c)
            for _ in range(rng.randint(1, 4)):
                m[rng.randrange(len(m))] = rng.choice((0xFF, 0xF0, 0x0F, 0x00, rng.randrange(256)))
            comps.append(bytes(m))
            caps.append(rng.choice((65536, 65535, 32768, 1 << 20)))
    b = decode_with_watchdog(cuda, fmt, comps, caps, "hostile")
    res, dst = b.results(), b.dst_host()
    for i, (comp, cap) in enumerate(zip(comps, caps)):
        st, out = ORACLE[fmt](comp, cap)
        assert res[i]["status"] == st, (i, int(res[i]["status"]), st)
        if st == 0:
            assert res[i]["bytes_written"] == len(out) and b.output(i, dst, len(out)) == out, i
        else:
            assert res[i]["bytes_written"] == 0
