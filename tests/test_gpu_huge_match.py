"""A match longer than 2^32 bytes, decoded on the device (the reference's
tests/huge_match_gpu.cu). Opt-in: it allocates 4 GiB and one warp walks all
of it, so it runs only with CUDEC_RUN_HUGE=1 (and -m gpu).

One valid LZ4 block: three literals "ABC", one match of 2^32 + 4096 bytes at
offset 3, a five-byte literal tail. The output is "ABC" repeating, so byte i
is "ABC"[i % 3] up to the tail; 2^32 mod 3 == 1, so a copy whose index or
phase were truncated to 32 bits shifts the pattern at the 4 GiB mark, and a
window astride that mark (plus the head and the tail) carries the verdict.
The block's shape is first ruled on by liblz4 at a small match length.
"""
import os

import numpy as np
import pytest

from cudec_b200 import workload as W

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("CUDEC_RUN_HUGE") != "1",
                                 reason="opt-in (CUDEC_RUN_HUGE=1): 4 GiB, one chunk")]

SEED, TAIL = b"ABC", b"wxyz."


def make_block(match_len):
    enc = match_len - 4
    out = bytearray([(3 << 4) | min(enc, 15)]) + SEED + b"\x03\x00"
    if enc >= 15:
        rest = enc - 15
        out += b"\xff" * (rest // 255) + bytes([rest % 255])
    out += bytes([len(TAIL) << 4]) + TAIL
    return bytes(out)


def expected(match_len, lo, hi):
    copied = 3 + match_len
    return bytes(SEED[i % 3] if i < copied else TAIL[i - copied] for i in range(lo, hi))


def test_match_longer_than_2_pow_32(cuda):
    import torch
    small = 4096
    assert W.lz4_decompress_ref(make_block(small), 3 + small + 5) == expected(small, 0, 3 + small + 5)
    ml = (1 << 32) + 4096
    blk = make_block(ml)
    total = 3 + ml + 5
    src = torch.from_numpy(np.frombuffer(blk, dtype=np.uint8).copy()).to(cuda)
    dst = torch.full((total + 64,), 0xA5, dtype=torch.uint8, device=cuda)
    tab = lambda v: torch.tensor([v], dtype=torch.int64, device=cuda)
    srcp, sizes, dstp, caps = tab(src.data_ptr()), tab(len(blk)), tab(dst.data_ptr()), tab(total)
    res = torch.zeros(16, dtype=torch.uint8, device=cuda)
    import cudec_b200 as cd
    s = torch.cuda.current_stream(cuda).cuda_stream
    assert cd.BATCH_ENTRIES["lz4"](srcp.data_ptr(), sizes.data_ptr(), dstp.data_ptr(),
                                   caps.data_ptr(), 1, res.data_ptr(), s) == 0
    torch.cuda.synchronize()
    rec = res.cpu().numpy().view(np.int64)
    assert int(res.cpu().numpy()[:4].view(np.int32)[0]) == 0
    assert int(rec[1]) == total
    mark = 1 << 32
    for lo, hi in ((0, 64), (mark - 32, mark + 32), (total - 64, total)):
        assert dst[lo:hi].cpu().numpy().tobytes() == expected(ml, lo, hi), (lo, hi)
    assert dst[total:total + 64].cpu().numpy().tobytes() == b"\xa5" * 64
