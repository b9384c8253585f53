"""GPU parity for the GDeflate page decoder (cudec_gdeflate_decompress_batch)
and the TileStream entry: every page's status and bytes equal the oracle's
(oracle/gdeflate_oracle.c, whose refill schedule and envelope walker are
pinned to the reference's headers), on this library's golden pages, encoder
output across levels, sizes and content (stored, static and dynamic blocks),
mutants, short capacities and unaligned buffers; nothing past bytes_written
is touched."""
import hashlib
import json
import os
import random

import numpy as np
import pytest

import cudec_b200 as cd
import oracle
from cudec_b200 import workload as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def run(cuda, comps, caps, **kw):
    import torch
    from cudec_b200.device import DeviceBatch
    b = DeviceBatch(comps, caps, device=cuda, **kw)
    assert b.run("gdeflate") == 0
    torch.cuda.synchronize()
    return b, b.results(), b.dst_host()


def check(b, res, dst, comps, caps, label):
    for i, (c, cap) in enumerate(zip(comps, caps)):
        st, out = oracle.gdeflate_decode(c, cap)
        r = res[i]
        assert r["status"] == st, (label, i, int(r["status"]), st, len(c), cap)
        assert r["reserved"] == 0
        if st == 0:
            assert r["bytes_written"] == len(out)
            assert b.output(i, dst, len(out)) == out, (label, i)
            tail = b.output(i, dst)[len(out):]
            assert tail == bytes([0xA5]) * len(tail), (label, i)
        else:
            assert r["bytes_written"] == 0


def pages(seed=5):
    sizes = [1, 31, 32, 33, 1000, 4096, 30000, 65535, 65536, 65536]
    probs = [0.5, 0.2, 0.8, 0.5, 0.5, 0.3, 0.6, 0.5, 0.7, 0.5]
    buf, offs = W.generate(sizes, [W.gdeflate_params(p) for p in probs],
                           param_idx=np.arange(len(sizes)),
                           seeds=np.arange(seed, seed + len(sizes), dtype=np.uint64))
    raws = [buf[int(o):int(o) + n].tobytes() for o, n in zip(offs, sizes)]
    raws += [b"", b"\x00" * 65536, bytes(range(256)) * 256, os.urandom(0) +
             bytes(np.random.default_rng(seed).integers(0, 256, 65536, dtype=np.uint8)),
             b"ab" * 20000]
    return raws


def test_golden_pages(cuda):
    vecs = json.load(open(os.path.join(GOLDEN, "gdeflate_page.json")))["vectors"]
    comps = [bytes.fromhex(v["input_hex"]) for v in vecs]
    caps = [v["capacity"] for v in vecs]
    b, res, dst = run(cuda, comps, caps)
    for i, v in enumerate(vecs):
        assert res[i]["status"] == 0, v["name"]
        assert hashlib.sha256(b.output(i, dst, v["expect_len"])).hexdigest() == v["expect_sha256"]
    check(b, res, dst, comps, caps, "golden")


def test_encoder_output_levels_and_content(cuda):
    raws = pages()
    comps, caps = [], []
    for raw in raws:
        for lvl, win in ((1, 32768), (6, 65536), (12, 32768)):
            comps.append(W.gdeflate_compress(raw, lvl, win))
            caps.append(len(raw))
    b, res, dst = run(cuda, comps, caps)
    check(b, res, dst, comps, caps, "levels")
    assert (res["status"] == 0).all()


@pytest.mark.parametrize("skew", [(0, 0), (1, 3), (2, 15), (3, 7)])
def test_unaligned_and_capacity_edges(cuda, skew):
    raws = pages(9)[:8]
    comps = [W.gdeflate_compress(r, 6) for r in raws]
    caps = [len(r) for r in raws]
    caps[2] = max(caps[2] - 1, 0)
    caps[4] = caps[4] + 100
    caps[6] = 0
    b, res, dst = run(cuda, comps, caps, src_skew=skew[0], dst_skew=skew[1])
    check(b, res, dst, comps, caps, "skew")


def test_mutants_match_oracle(cuda):
    rng = random.Random(41)
    comps, caps = [], []
    for raw in pages(13)[3:10]:
        page = W.gdeflate_compress(raw, 12)
        for _ in range(60):
            m = bytearray(page)
            r = rng.random()
            if r < 0.15:
                m = m[:rng.randrange(len(m) + 1)]
            elif r < 0.25:
                m += bytes(4 * rng.randint(1, 3))
            else:
                for _ in range(rng.randint(1, 4)):
                    m[rng.randrange(len(m))] ^= 1 << rng.randrange(8)
            comps.append(bytes(m))
            caps.append(rng.choice([len(raw), len(raw) + 17, max(len(raw) - 3, 0), 65536]))
    b, res, dst = run(cuda, comps, caps)
    check(b, res, dst, comps, caps, "mutants")
    sts = {int(x) for x in res["status"]}
    assert 0 in sts and 2 in sts


def skewed_pages(seed):
    """Bytes drawn from geometric distributions over all 256 values: most
    symbols are rare, so the dynamic codes reach the 15-bit limit and the
    decoder's path for codes longer than its lookup table is exercised."""
    rng = np.random.default_rng(seed)
    out = []
    for ratio in (0.55, 0.7, 0.8, 0.9):
        w = ratio ** np.arange(256)
        out.append(rng.choice(256, size=65536, p=w / w.sum()).astype(np.uint8).tobytes())
    return out


def test_long_codes_and_their_mutants_match_oracle(cuda):
    """Pages whose Huffman codes run past the 10-bit lookup table, at three
    encoder levels, intact and under mutants; status and bytes must equal
    the oracle's."""
    rng = random.Random(77)
    comps, caps = [], []
    for raw in skewed_pages(3):
        for lvl in (1, 6, 12):
            page = W.gdeflate_compress(raw, lvl)
            comps.append(page)
            caps.append(len(raw))
            for _ in range(40):
                m = bytearray(page)
                for _ in range(rng.randint(1, 3)):
                    m[rng.randrange(len(m))] ^= 1 << rng.randrange(8)
                comps.append(bytes(m))
                caps.append(rng.choice([len(raw), len(raw) - 5, 65536]))
    b, res, dst = run(cuda, comps, caps)
    check(b, res, dst, comps, caps, "long codes")
    intact = [int(res[i]["status"]) for i in range(0, len(comps), 41)]
    assert intact == [0] * len(intact)


def test_tilestream_container(cuda):
    raw = b"".join(pages(17))
    ts = W.gdeflate_tilestream(raw, 6)
    st, out = cd.tilestream_decompress(ts, len(raw))
    assert st == 0 and out == raw
    assert cd.tilestream_decompress(ts, len(raw) - 1)[0] == cd.ERR_OUTPUT_TOO_SMALL
    bad = bytearray(ts)
    bad[1] ^= 1
    assert cd.tilestream_decompress(bytes(bad), len(raw))[0] == cd.ERR_CORRUPT_INPUT
    # a tile whose page produces more than its declared size: the page's
    # capacity is that size; fewer bytes than declared: corrupt
    one = W.gdeflate_tilestream(raw[:1000], 6)
    for declared, want in ((999, cd.ERR_OUTPUT_TOO_SMALL), (1001, cd.ERR_CORRUPT_INPUT)):
        m = bytearray(one)
        m[4:8] = (1 | (declared << 2)).to_bytes(4, "little")
        assert cd.tilestream_decompress(bytes(m), 2000)[0] == want
