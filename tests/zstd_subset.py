"""Zstd frames that are valid but outside the decoded subset: the reference
refuses each with CUDEC_ERR_UNSUPPORTED (src/zstd_frame.h:12-18, 203-300;
its extension ladder, docs/MASTERPLAN.md:1282-1303, keeps them refused)."""
from cudec_b200 import workload as W

RAW = bytes(range(256)) * 64


def refused_frames():
    """name -> (frame, capacity, libzstd decodes it without a dictionary)."""
    base = W.zstd_compress(RAW, 3)
    assert base[4] == 0x60  # single segment, 2-byte content size, no dictionary
    magic = b"\x28\xb5\x2f\xfd"
    return {
        # skippable frame (magic 0x184D2A5A), 8 bytes of user data
        "skippable": (b"\x5a\x2a\x4d\x18" + (8).to_bytes(4, "little") + bytes(8), 64, True),
        # libzstd told not to write the content size
        "no content size": (W.zstd_compress(RAW, 3, 20, False, content_size=False),
                            len(RAW), True),
        # the same frame with a 1-byte dictionary id (descriptor bits 0-1)
        "dictionary id": (base[:4] + bytes([0x61, 0x07]) + base[5:], len(RAW), False),
        # multi-segment, 4-byte content size 0, window 2^24 = 16 MB, one
        # empty last raw block
        "16 MB window": (magic + bytes([0x80, 0x70]) + bytes(4) + b"\x01\x00\x00", 64, True),
    }
