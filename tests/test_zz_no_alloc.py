"""cudec_zstd_decompress_batch_noalloc: the Zstd batch kernel with its
literal slots in a library-owned static device array (no counterpart in the
reference). Collected last on purpose: it must give the same records and
bytes as cudec_zstd_decompress_batch (caller workspace) whether it runs alone
or after every other test, and on two calls in a row (the second reuses the
static slots the first left behind)."""
import ctypes

import numpy as np
import pytest

import cudec_b200 as cd
from cudec_b200 import workload as W


def test_noalloc_rejects_oversize_and_bad_args_synchronously():
    buf = (ctypes.c_uint8 * 4096)()
    a = (ctypes.addressof(buf) + 15) & ~15
    z = cd.zstd_decompress_batch_noalloc
    assert cd.ZSTD_NOALLOC_MAX_CHUNKS == 64
    assert z(a, a, a, a, cd.ZSTD_NOALLOC_MAX_CHUNKS + 1, a, None) == cd.ERR_INVALID_ARGUMENT
    assert z(a, a, a, a, 1 << 40, a, None) == cd.ERR_INVALID_ARGUMENT
    assert z(a, a, a, a, 0, a, None) == cd.ERR_INVALID_ARGUMENT
    assert z(None, a, a, a, 4, a, None) == cd.ERR_INVALID_ARGUMENT
    assert z(a, a, a, a, 4, a + 8, None) == cd.ERR_INVALID_ARGUMENT


def _frames():
    sizes = [1, 900, 30000, 131072, 140000, 400000, 1 << 20]
    buf, offs = W.generate(sizes, [W.zstd_params(0.5, 0.1)],
                           seeds=np.arange(500, 500 + len(sizes), dtype=np.uint64))
    raws = [buf[int(o):int(o) + n].tobytes() for o, n in zip(offs, sizes)]
    comps, caps = [], []
    for k, raw in enumerate(raws):
        for lvl in (1, 3, 19):
            comps.append(W.zstd_compress(raw, lvl, 20, lvl != 3))
            caps.append(len(raw))
    comps.append(comps[-1][:-7])          # truncated: corrupt
    caps.append(caps[-1])
    comps.append(comps[5])                # capacity one short: too small
    caps.append(caps[5] - 1)
    comps.append(b"\x50\x2a\x4d\x18" + bytes(12))   # skippable frame: unsupported
    caps.append(64)
    return comps, caps


@pytest.mark.gpu
@pytest.mark.parametrize("count", [64, 25])
def test_noalloc_equals_workspace_entry_twice_in_a_row(cuda, count):
    import torch
    from cudec_b200.device import DeviceBatch
    comps, caps = _frames()
    comps = (comps * 3)[:count]
    caps = (caps * 3)[:count]
    ref = DeviceBatch(comps, caps, device=cuda)
    assert ref.run("zstd") == 0
    torch.cuda.synchronize()
    want_res, want_dst = ref.results().copy(), ref.dst_host().copy()
    sts = set(int(s) for s in want_res["status"])
    assert 0 in sts and 2 in sts and 3 in sts and 6 in sts

    b = DeviceBatch(comps, caps, device=cuda)
    s = torch.cuda.current_stream(b.device).cuda_stream
    for _ in range(2):
        b.reset()
        assert cd.zstd_decompress_batch_noalloc(*b.args(), s) == 0
        torch.cuda.synchronize()
        got_res, got_dst = b.results(), b.dst_host()
        assert (got_res == want_res).all()
        for i in range(count):
            assert b.output(i, got_dst) == ref.output(i, want_dst), i
