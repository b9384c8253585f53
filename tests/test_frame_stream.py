"""LZ4 frame entry and pinned streaming context.

CPU: the oracle's frame ladder against liblz4 frames and crafted negatives;
argument rules of the frame and stream entries (they make no CUDA call).
GPU: cudec_lz4f_decompress against the oracle and the reference library's
own frame entry; the stream context against the batch path, fresh vs reused,
both memory spaces, several waves, and the poison latch (a host-side
allocation failure, no GPU fault) as in the reference's
tests/stream_twin.cu:392-450.
"""
import ctypes
import random
import struct

import numpy as np
import pytest

import cudec_b200 as cd
import oracle
from cudec_b200 import workload as W


def raw_data(n, seed=1, p=0.5):
    buf, _ = W.generate([n], W.lz_params(p), seeds=np.array([seed], dtype=np.uint64))
    return buf.tobytes()


FRAME_OPTS = [dict(), dict(content_checksum=True), dict(block_checksum=True),
              dict(content_size=True), dict(block_size_id=5, content_checksum=True),
              dict(block_size_id=6, block_checksum=True, content_size=True),
              dict(block_size_id=7)]


def frames():
    out = []
    for i, kw in enumerate(FRAME_OPTS):
        for n in (0, 1, 5000, 70000, 300000):
            d = raw_data(n, seed=10 * i + 1) if n else b""
            out.append((d, W.lz4f_compress(d, **kw), kw))
    # incompressible content gives uncompressed (raw) blocks
    rnd = np.random.default_rng(3).integers(0, 256, 200000, dtype=np.uint8).tobytes()
    out.append((rnd, W.lz4f_compress(rnd, content_checksum=True), {"raw": True}))
    return out


def negatives(data, frame):
    """Crafted frame negatives (the reference's tests/frame_host_negative.cpp
    shapes): each entry (name, bytes, capacity)."""
    f = bytearray(frame)
    neg = [("empty", b"", 100), ("short", frame[:6], 100),
           ("bad-magic", b"\x05" + frame[1:], len(data))]
    g = bytearray(f); g[4] ^= 0x40; neg.append(("version", bytes(g), len(data)))
    g = bytearray(f); g[4] |= 0x02; neg.append(("reserved-flg", bytes(g), len(data)))
    g = bytearray(f); g[5] |= 0x80; neg.append(("reserved-bd", bytes(g), len(data)))
    g = bytearray(f); g[5] = (g[5] & 0x8F) | 0x30; neg.append(("bmax-small", bytes(g), len(data)))
    g = bytearray(f); g[-5] ^= 1; neg.append(("flip-late", bytes(g), len(data)))
    g = bytearray(f); g[6] ^= 0xFF; neg.append(("header-checksum", bytes(g), len(data)))
    neg.append(("truncated", frame[:len(frame) // 2], len(data)))
    neg.append(("no-end-mark", frame[:-4] if len(frame) > 11 else frame[:7], len(data)))
    neg.append(("capacity-short", frame, max(len(data) - 1, 0)))
    return neg


def test_oracle_frame_decodes_liblz4_frames():
    for d, fr, kw in frames():
        st, out = oracle.lz4f_decode(fr, len(d))
        assert st == 0 and out == d, kw
    # block-linked (liblz4's default) and dictionary frames are out of subset
    big = raw_data(300000)  # one-block frames are written independent anyway
    assert oracle.lz4f_decode(W.lz4f_compress(big, independent=False), len(big))[0] == 6


def test_oracle_frame_negatives_fail_closed():
    d = raw_data(70000, seed=4)
    fr = W.lz4f_compress(d, content_checksum=True, block_checksum=True, content_size=True)
    for name, body, cap in negatives(d, fr):
        st, out = oracle.lz4f_decode(body, cap)
        assert st != 0, name
        assert out == b""


def test_frame_and_stream_argument_rules_without_gpu():
    lib = cd.lib()
    w = ctypes.c_size_t(7)
    buf = ctypes.create_string_buffer(64)
    assert lib.cudec_lz4f_decompress(None, 10, buf, 64, ctypes.byref(w)) == cd.ERR_INVALID_ARGUMENT
    assert w.value == 0
    assert lib.cudec_lz4f_decompress(buf, 10, buf, 64, None) == cd.ERR_INVALID_ARGUMENT
    assert lib.cudec_lz4f_decompress(buf, 10, None, 64, ctypes.byref(w)) == cd.ERR_INVALID_ARGUMENT
    assert lib.cudec_stream_ctx_create(None) == cd.ERR_INVALID_ARGUMENT
    lib.cudec_stream_ctx_destroy(None)
    arr = (ctypes.c_uint64 * 4)(ctypes.addressof(buf), 0, 0, 0)
    sizes = (ctypes.c_uint64 * 4)(4, 0, 0, 0)
    caps = (ctypes.c_uint64 * 4)(64, 0, 0, 0)
    dsts = (ctypes.c_uint64 * 4)(ctypes.addressof(buf), 0, 0, 0)
    res = (cd.ChunkResult * 4)()
    one = lib.cudec_lz4_decompress_stream
    assert one(None, sizes, dsts, caps, 1, 0, res) == cd.ERR_INVALID_ARGUMENT
    assert one(arr, sizes, dsts, caps, 0, 0, res) == cd.ERR_INVALID_ARGUMENT
    assert one(arr, sizes, dsts, caps, 1, 7, res) == cd.ERR_INVALID_ARGUMENT
    assert one(arr, sizes, dsts, caps, 2**64 - 1, 0, res) == cd.ERR_INVALID_ARGUMENT
    sizes[1] = 5   # NULL source with a non-zero size
    assert one(arr, sizes, dsts, caps, 2, 0, res) == cd.ERR_INVALID_ARGUMENT
    sizes[1] = 0
    caps[1] = 9    # NULL destination with a non-zero capacity
    assert one(arr, sizes, dsts, caps, 2, 0, res) == cd.ERR_INVALID_ARGUMENT
    assert lib.cudec_lz4_decompress_stream_ctx(None, arr, sizes, dsts, caps, 1, 0, res) \
        == cd.ERR_INVALID_ARGUMENT


# ------------------------------------------------------------------ GPU ---

@pytest.mark.gpu
def test_frame_entry_matches_oracle_and_reference(cuda):
    have_ref = oracle.ref_gpu_lib() is not None
    for d, fr, kw in frames():
        st, out = cd.lz4f_decompress(fr, len(d) + 13)
        assert st == 0 and out == d, kw
        if have_ref:
            assert oracle.ref_lz4f_decode(fr, len(d) + 13) == (st, out)
    d = raw_data(70000, seed=4)
    fr = W.lz4f_compress(d, content_checksum=True, block_checksum=True, content_size=True)
    cases = negatives(d, fr)
    rng = random.Random(5)
    for k in range(60):
        g = bytearray(fr)
        for _ in range(rng.randint(1, 3)):
            g[rng.randrange(len(g))] ^= 1 << rng.randrange(8)
        cases.append(("mutant%d" % k, bytes(g), len(d)))
    big = raw_data(300000, seed=8)
    cases.append(("linked", W.lz4f_compress(big, independent=False), len(big)))
    for name, body, cap in cases:
        want = oracle.lz4f_decode(body, cap)
        got = cd.lz4f_decompress(body, cap)
        assert got[0] == want[0], (name, got[0], want[0])
        assert got[1] == want[1], name
        if have_ref:
            assert oracle.ref_lz4f_decode(body, cap)[0] == got[0], name


def block_offsets(fr):
    """(offset, length) of each block's data in an .lz4 frame with block
    checksums (the 4-byte checksum follows each block)."""
    flg = fr[4]
    pos = 4 + 2 + (8 if flg & 8 else 0) + 1
    out = []
    while True:
        bs = int.from_bytes(fr[pos:pos + 4], "little")
        pos += 4
        if bs == 0:
            return out
        n = bs & 0x7FFFFFFF
        out.append((pos, n))
        pos += n + 4


@pytest.mark.gpu
def test_frame_block_checksums_checked_in_parallel(cuda):
    """Frames large enough for the block checksums to be verified on host
    threads while the blocks decode: a good frame decodes; a bad checksum in
    any block (first, middle, last, a stored block) is CORRUPT_INPUT, also
    when the capacity is too small (the checksum outranks it), exactly as
    the oracle's in-order walk decides."""
    d = raw_data(12 << 20, seed=21)
    noise = np.random.default_rng(2).integers(0, 256, 200000, dtype=np.uint8).tobytes()
    d = d[:3 << 20] + noise + d[3 << 20:]  # an incompressible run: stored blocks
    fr = W.lz4f_compress(d, block_size_id=4, content_checksum=True, block_checksum=True)
    blocks = block_offsets(fr)
    assert len(blocks) > 150
    stored = [i for i, (o, n) in enumerate(blocks)
              if int.from_bytes(fr[o - 4:o], "little") >> 31]
    assert stored
    st, out = cd.lz4f_decompress(fr, len(d))
    assert st == 0 and out == d
    for k in (0, len(blocks) // 2, len(blocks) - 1, stored[0]):
        o, n = blocks[k]
        g = bytearray(fr)
        g[o + n] ^= 0x40  # the block's checksum
        for cap in (len(d), len(d) - 1):
            want = oracle.lz4f_decode(bytes(g), cap)
            assert want[0] == cd.ERR_CORRUPT_INPUT
            assert cd.lz4f_decompress(bytes(g), cap)[0] == want[0], (k, cap)


def host_arrays(comps, caps, space, device=None):
    """Host pointer tables for the stream entry; destinations host or device."""
    import torch
    n = len(comps)
    srcs = [np.frombuffer(c if c else b"\0", dtype=np.uint8).copy() for c in comps]
    src_ptrs = np.array([s.ctypes.data for s in srcs], dtype=np.uint64)
    sizes = np.array([len(c) for c in comps], dtype=np.uint64)
    capa = np.array(caps, dtype=np.uint64)
    if space == cd.MEM_HOST:
        dsts = [np.full(max(c, 1), 0xA5, dtype=np.uint8) for c in caps]
        dst_ptrs = np.array([x.ctypes.data for x in dsts], dtype=np.uint64)
    else:
        dsts = [torch.full((max(c, 1),), 0xA5, dtype=torch.uint8, device=device) for c in caps]
        dst_ptrs = np.array([x.data_ptr() for x in dsts], dtype=np.uint64)
    res = np.zeros(n, dtype=[("status", "<i4"), ("reserved", "<u4"), ("bytes_written", "<u8")])
    return srcs, src_ptrs, sizes, capa, dsts, dst_ptrs, res


def run_stream(ctx, comps, caps, space, device=None):
    srcs, sp, sz, cp, dsts, dp, res = host_arrays(comps, caps, space, device)
    st = ctx.decode(sp.ctypes.data, sz.ctypes.data, dp.ctypes.data, cp.ctypes.data,
                    len(comps), space, res.ctypes.data)
    outs = []
    for i, x in enumerate(dsts):
        h = x if space == cd.MEM_HOST else x.cpu().numpy()
        outs.append(h.tobytes())
    return st, res, outs


@pytest.mark.gpu
@pytest.mark.parametrize("space", [0, 1])
def test_stream_context_matches_oracle_fresh_and_reused(cuda, space):
    rng = random.Random(7)
    raws = [raw_data(n, seed=i + 3) for i, n in enumerate([1, 100, 5000, 65536, 70000, 200000])]
    comps = [W.lz4_compress(r) for r in raws]
    caps = [len(r) + 9 for r in raws]
    # a corrupt neighbour must not disturb the others
    bad = bytearray(comps[3]); bad[len(bad) // 2] ^= 0x55
    comps.append(bytes(bad)); caps.append(65536)
    ctx = cd.StreamContext()
    for rep in range(3):
        st, res, outs = run_stream(ctx, comps, caps, space, cuda)
        want_st = [oracle.lz4_decode(c, k) for c, k in zip(comps, caps)]
        first_bad = next((w[0] for w in want_st if w[0] != 0), 0)
        assert st == first_bad
        for i, (ws, wb) in enumerate(want_st):
            assert res[i]["status"] == ws
            if ws == 0:
                assert res[i]["bytes_written"] == len(wb)
                assert outs[i][:len(wb)] == wb
                assert outs[i][len(wb):] == b"\xa5" * (len(outs[i]) - len(wb))
        # the reused context (same inputs again) is bit-identical, and so is
        # a fresh one
        st2, res2, outs2 = run_stream(ctx, comps, caps, space, cuda)
        fresh = cd.StreamContext()
        st3, res3, outs3 = run_stream(fresh, comps, caps, space, cuda)
        fresh.close()
        assert st2 == st3 == st
        ok = [i for i, w in enumerate(want_st) if w[0] == 0]
        assert all(outs2[i] == outs[i] and outs3[i] == outs[i] for i in ok)
        # grow the staging between repetitions
        comps.append(W.lz4_compress(raw_data(300000 + rep, seed=99 + rep)))
        caps.append(300000 + rep)
    ctx.close()


@pytest.mark.gpu
def test_stream_many_waves_and_one_shot(cuda):
    n = 9000  # more than one 4096-chunk wave
    raws = [raw_data(200 + (i % 50), seed=i) for i in range(n)]
    comps = [W.lz4_compress(r) for r in raws]
    caps = [len(r) for r in raws]
    srcs, sp, sz, cp, dsts, dp, res = host_arrays(comps, caps, cd.MEM_HOST)
    st = cd.lib().cudec_lz4_decompress_stream(sp.ctypes.data, sz.ctypes.data, dp.ctypes.data,
                                              cp.ctypes.data, n, cd.MEM_HOST, res.ctypes.data)
    assert st == 0
    assert all(dsts[i][:len(raws[i])].tobytes() == raws[i] for i in range(n))


@pytest.mark.gpu
def test_stream_host_output_large_waves(cuda):
    """Host output in waves large enough for the copy to the caller's
    buffers to be split over host threads (uneven chunk sizes, some corrupt
    chunks and capacities too small among them): every chunk's bytes and
    record equal the oracle's, exactly bytes_written bytes land, the rest of
    each destination keeps its fill, and the aggregate is the first non-OK
    chunk in index order."""
    rng = random.Random(31)
    n = 700
    raws = [raw_data(rng.choice([100, 5000, 65536, 200000]), seed=500 + i) for i in range(n)]
    comps = [W.lz4_compress(r) for r in raws]
    caps = [len(r) + rng.choice([0, 0, 0, 7]) for r in raws]
    for i in rng.sample(range(n), 12):  # corrupt a few: a bad offset, or a capacity too small
        if i % 2:
            caps[i] = max(len(raws[i]) - 1, 0)
        else:
            c = bytearray(comps[i])
            c[len(c) // 2] ^= 0xFF
            comps[i] = bytes(c)
    ctx = cd.StreamContext()
    st, res, outs = run_stream(ctx, comps, caps, cd.MEM_HOST)
    first = None
    for i in range(n):
        want_st, want = oracle.lz4_decode(comps[i], caps[i])
        assert int(res[i]["status"]) == want_st, i
        if want_st == 0:
            assert int(res[i]["bytes_written"]) == len(want)
            assert outs[i][:len(want)] == want, i
            assert outs[i][len(want):] == bytes([0xA5]) * (len(outs[i]) - len(want)), i
        else:
            assert int(res[i]["bytes_written"]) == 0
            first = i if first is None else first
    assert first is not None and st == int(res[first]["status"])
    ctx.close()


@pytest.mark.gpu
def test_stream_host_output_one_buffer(cuda):
    """Destinations back to back in one host buffer (the shape that lets a
    full wave go to the caller in one copy): every chunk full; then one chunk
    with spare capacity and one corrupt chunk, which take the staged path.
    Bytes and records equal the oracle's, and nothing past bytes_written
    changes."""
    n = 300
    raws = [raw_data(20000 + 37 * i, seed=900 + i) for i in range(n)]
    base_comps = [W.lz4_compress(r) for r in raws]
    for case in ("full", "mixed"):
        comps = list(base_comps)
        caps = [len(r) for r in raws]
        if case == "mixed":
            caps[17] += 9
            c = bytearray(comps[200])
            c[len(c) // 2] ^= 0xFF
            comps[200] = bytes(c)
        offs = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
        buf = np.full(int(offs[-1]), 0xA5, dtype=np.uint8)
        srcs = [np.frombuffer(c, dtype=np.uint8).copy() for c in comps]
        sp = np.array([x.ctypes.data for x in srcs], dtype=np.uint64)
        sz = np.array([len(c) for c in comps], dtype=np.uint64)
        cp = np.array(caps, dtype=np.uint64)
        dp = np.array([buf.ctypes.data + int(o) for o in offs[:-1]], dtype=np.uint64)
        res = np.zeros(n, dtype=[("status", "<i4"), ("reserved", "<u4"), ("bytes_written", "<u8")])
        ctx = cd.StreamContext()
        st = ctx.decode(sp.ctypes.data, sz.ctypes.data, dp.ctypes.data, cp.ctypes.data, n,
                        cd.MEM_HOST, res.ctypes.data)
        ctx.close()
        first = None
        for i in range(n):
            want_st, want = oracle.lz4_decode(comps[i], caps[i])
            assert int(res[i]["status"]) == want_st, (case, i)
            seg = buf[offs[i]:offs[i + 1]].tobytes()
            if want_st == 0:
                assert seg[:len(want)] == want, (case, i)
                assert seg[len(want):] == bytes([0xA5]) * (len(seg) - len(want)), (case, i)
            else:
                assert seg == bytes([0xA5]) * len(seg), (case, i)
                first = i if first is None else first
        assert st == (0 if first is None else int(res[first]["status"])), case
        assert (first is None) == (case == "full")


@pytest.mark.gpu
@pytest.mark.parametrize("packed", [True, False])
def test_stream_pageable_sources_staged_by_threads(cuda, packed):
    """Pageable source chunks of more than 4 MiB a wave, packed back to back
    in one buffer or scattered: the call stages them on host threads; bytes
    and records equal the oracle's."""
    import torch
    n = 400
    raws = [raw_data(30000 + 101 * i, seed=1300 + i) for i in range(n)]
    comps = [W.lz4_compress(r) for r in raws]
    caps = [len(r) for r in raws]
    if packed:
        buf = np.frombuffer(b"".join(comps), dtype=np.uint8).copy()
        offs = np.concatenate([[0], np.cumsum([len(c) for c in comps])[:-1]]).astype(np.uint64)
        sp = (offs + np.uint64(buf.ctypes.data)).astype(np.uint64)
    else:
        srcs = [np.frombuffer(c, dtype=np.uint8).copy() for c in comps]
        sp = np.array([x.ctypes.data for x in srcs], dtype=np.uint64)
    assert sum(len(c) for c in comps) > (4 << 20)
    sz = np.array([len(c) for c in comps], dtype=np.uint64)
    cp = np.array(caps, dtype=np.uint64)
    dsts = [torch.full((c,), 0xA5, dtype=torch.uint8, device=cuda) for c in caps]
    dp = np.array([x.data_ptr() for x in dsts], dtype=np.uint64)
    res = np.zeros(n, dtype=[("status", "<i4"), ("reserved", "<u4"), ("bytes_written", "<u8")])
    ctx = cd.StreamContext()
    st = ctx.decode(sp.ctypes.data, sz.ctypes.data, dp.ctypes.data, cp.ctypes.data, n,
                    cd.MEM_DEVICE, res.ctypes.data)
    ctx.close()
    assert st == 0
    for i in range(n):
        assert int(res[i]["status"]) == 0 and int(res[i]["bytes_written"]) == caps[i]
        assert dsts[i].cpu().numpy().tobytes() == raws[i], i


@pytest.mark.gpu
def test_stream_poison_latch_on_allocation_failure(cuda):
    """An impossible host-output staging size makes the grow allocation fail
    on the host side: CUDA status, every record defined, context poisoned,
    later decodes refused without touching the device."""
    ctx = cd.StreamContext()
    comp = W.lz4_compress(raw_data(1000))
    src = np.frombuffer(comp, dtype=np.uint8).copy()
    dst = np.zeros(4096, dtype=np.uint8)
    sp = np.array([src.ctypes.data], dtype=np.uint64)
    sz = np.array([len(comp)], dtype=np.uint64)
    dp = np.array([dst.ctypes.data], dtype=np.uint64)
    cp = np.array([1 << 60], dtype=np.uint64)
    res = np.zeros(1, dtype=[("status", "<i4"), ("reserved", "<u4"), ("bytes_written", "<u8")])
    res["status"] = 77
    assert ctx.decode(sp.ctypes.data, sz.ctypes.data, dp.ctypes.data, cp.ctypes.data, 1,
                      cd.MEM_HOST, res.ctypes.data) == cd.ERR_CUDA
    assert res[0]["status"] == cd.ERR_CUDA and res[0]["bytes_written"] == 0
    cp[0] = 1000
    res["status"] = 77
    assert ctx.decode(sp.ctypes.data, sz.ctypes.data, dp.ctypes.data, cp.ctypes.data, 1,
                      cd.MEM_HOST, res.ctypes.data) == cd.ERR_CUDA
    assert res[0]["status"] == cd.ERR_CUDA
    ctx.close()
    # a fresh context is unaffected
    ctx2 = cd.StreamContext()
    assert ctx2.decode(sp.ctypes.data, sz.ctypes.data, dp.ctypes.data, cp.ctypes.data, 1,
                       cd.MEM_HOST, res.ctypes.data) == 0
    ctx2.close()


def _pinned_pages(nbytes):
    """A page-aligned numpy buffer of whole pages, page-locked and mapped
    with cudaHostRegister (portable | mapped); unregister when done."""
    import torch
    page = 4096
    pages = (nbytes + page - 1) // page
    raw = np.zeros(pages * page + page, dtype=np.uint8)
    off = (-raw.ctypes.data) % page
    buf = raw[off:off + pages * page]
    rc = torch.cuda.cudart().cudaHostRegister(buf.ctypes.data, buf.nbytes, 3)
    assert int(rc) == 0
    return raw, buf


def _unpin(buf):
    import torch
    assert int(torch.cuda.cudart().cudaHostUnregister(buf.ctypes.data)) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("space", [0, 1])
def test_stream_reads_page_locked_sources_in_place(cuda, space):
    """Chunks in page-locked host memory are read by the device in place:
    packed in one torch pinned buffer, and scattered over two registered
    allocations at odd offsets with the last chunk ending on the final byte
    of its allocation. A batch with one pageable chunk is staged as before.
    Every variant matches the oracle."""
    import torch
    probe = cd.lib().cdb_stream_reads_in_place
    probe.restype = ctypes.c_int
    probe.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
    raws = [raw_data(n, seed=40 + i) for i, n in enumerate([1, 777, 4096, 65536, 3, 100000])]
    comps = [W.lz4_compress(r) for r in raws]
    caps = [len(r) + 5 for r in raws]
    bad = bytearray(comps[3]); bad[len(bad) // 3] ^= 0x21
    comps.insert(0, bytes(bad)); caps.insert(0, 65536)
    comps.insert(4, b""); caps.insert(4, 0)
    n = len(comps)
    want = [oracle.lz4_decode(c, k) for c, k in zip(comps, caps)]
    sizes = np.array([len(c) for c in comps], dtype=np.uint64)

    def check(src_ptrs, expect_in_place, keep):
        assert probe(src_ptrs.ctypes.data, sizes.ctypes.data, n) == int(expect_in_place)
        _, _, _, capa, dsts, dp, res = host_arrays(comps, caps, space, cuda)
        ctx = cd.StreamContext()
        st = ctx.decode(src_ptrs.ctypes.data, sizes.ctypes.data, dp.ctypes.data,
                        capa.ctypes.data, n, space, res.ctypes.data)
        ctx.close()
        assert st == next(w[0] for w in want if w[0] != 0)
        for i, (ws, wb) in enumerate(want):
            assert res[i]["status"] == ws, i
            if ws == 0:
                got = dsts[i] if space == cd.MEM_HOST else dsts[i].cpu().numpy()
                assert res[i]["bytes_written"] == len(wb)
                assert got.tobytes()[:len(wb)] == wb

    # packed in one pinned tensor
    blob = b"".join(comps)
    pinned = torch.empty(len(blob) + 1, dtype=torch.uint8).pin_memory()
    pinned.numpy()[:len(blob)] = np.frombuffer(blob, dtype=np.uint8)
    offs = np.concatenate([[0], np.cumsum(sizes[:-1])]).astype(np.uint64)
    check(offs + np.uint64(pinned.data_ptr()), True, pinned)

    # scattered over two registered allocations, odd offsets, tail at the end
    half = n // 2
    need_a = sum(len(c) + 3 for c in comps[:half]) + 16
    need_b = sum(len(c) + 3 for c in comps[half:]) + 4096
    raw_a, a = _pinned_pages(need_a)
    raw_b, b = _pinned_pages(need_b)
    try:
        ptrs = []
        pos = 1
        for c in comps[:half]:
            a[pos:pos + len(c)] = np.frombuffer(c, dtype=np.uint8)
            ptrs.append(a.ctypes.data + pos)
            pos += len(c) + 3
        # the second allocation is filled from its end backwards
        pos = b.nbytes
        tail = []
        for c in reversed(comps[half:]):
            if c:
                pos -= len(c)
                b[pos:pos + len(c)] = np.frombuffer(c, dtype=np.uint8)
            tail.append(b.ctypes.data + pos)
            if c:
                pos -= 5
        ptrs += list(reversed(tail))
        scattered = np.array(ptrs, dtype=np.uint64)
        check(scattered, True, (a, b))
        # one pageable chunk: staged path, same results
        loose = np.frombuffer(comps[2], dtype=np.uint8).copy()
        mixed = scattered.copy()
        mixed[2] = loose.ctypes.data  # comps[2] sits in the first allocation
        check(mixed, False, loose)
    finally:
        _unpin(a)
        _unpin(b)
