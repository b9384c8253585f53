"""The LZ4 frame oracle (oracle/oracle.c, the reference's frame ladder
src/frame.cpp:282-397) against liblz4's own frame decoder on seeded mutants of
liblz4 frames, in both directions: a frame the oracle accepts decodes to the
same bytes in liblz4, and a frame liblz4 refuses is refused by the oracle.
Frames carry every combination of block checksums, content checksum and
content size, at two block sizes. Bytes after a frame are ignored by both,
as the reference's frame entry ignores them (src/frame.cpp:340-397)."""
import random

import numpy as np

import oracle
from cudec_b200 import workload as W


def frames():
    rng = np.random.default_rng(4)
    raw = bytes(rng.integers(0, 6, 150000, dtype=np.uint8)) + bytes(rng.integers(0, 256, 3000,
                                                                                dtype=np.uint8))
    out = []
    for bsid in (4, 5):
        for bc in (False, True):
            for cc in (False, True):
                for cs in (False, True):
                    out.append(W.lz4f_compress(raw, block_size_id=bsid, block_checksum=bc,
                                               content_checksum=cc, content_size=cs))
    return raw, out


def mutants(frame, rng, k):
    for _ in range(k):
        m = bytearray(frame)
        r = rng.random()
        if r < 0.15:
            m = m[:rng.randrange(len(m))]
        elif r < 0.2:
            m += bytes(rng.randrange(256) for _ in range(rng.randint(1, 8)))
        elif r < 0.35:  # the header and the first block's size field
            for _ in range(rng.randint(1, 2)):
                m[rng.randrange(min(len(m), 20))] ^= 1 << rng.randrange(8)
        else:
            for _ in range(rng.randint(1, 3)):
                m[rng.randrange(len(m))] ^= 1 << rng.randrange(8)
        yield bytes(m)


def test_frame_oracle_vs_liblz4_both_directions():
    raw, frs = frames()
    rng = random.Random(12)
    accepted = refused = stricter = 0
    for fr in frs:
        assert oracle.lz4f_decode(fr, len(raw)) == (0, raw)
        assert W.lz4f_decompress_ref(fr, len(raw)) == raw
        for m in mutants(fr, rng, 40):
            cap = len(raw) + 64
            st, out = oracle.lz4f_decode(m, cap)
            lib = W.lz4f_decompress_ref(m, cap)
            if st == 0:
                accepted += 1
                assert lib == out, "oracle accepted a frame liblz4 decodes differently"
            if lib is None:
                refused += 1
                assert st != 0, "liblz4 refused a frame the oracle accepted"
            elif st != 0:
                stricter += 1
    assert accepted > 0 and refused > 0
    # the reference ladder may be stricter than liblz4, never looser
    assert stricter <= refused
