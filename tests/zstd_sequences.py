"""Chunks that hold a sequence of Zstd and skippable frames, for the
multi-frame entry's tests (the chunk shape libzstd's ZSTD_decompress reads;
RFC 8878 section 3.1.2 for the skippable frame)."""
from cudec_b200 import workload as W


def skippable(n, nibble=0xA, fill=0x5C):
    """A skippable frame: magic 0x184D2A5<nibble>, 4-byte size, n bytes."""
    return (0x184D2A50 | nibble).to_bytes(4, "little") + n.to_bytes(4, "little") + \
        bytes([fill]) * n


def sequence(rng, raws):
    """Frames of `raws` at random levels and checksum flags, with skippable
    frames (0 to 40 bytes of payload, any of the 16 magics) between them."""
    parts = []
    for raw in raws:
        if rng.random() < 0.5:
            parts.append(skippable(rng.randrange(41), rng.randrange(16)))
        parts.append(W.zstd_compress(raw, rng.choice([1, 3, 19]), 20, rng.random() < 0.5))
    if rng.random() < 0.5:
        parts.append(skippable(rng.randrange(41), rng.randrange(16)))
    return b"".join(parts)


def mutate(b, rng):
    """Truncation, one appended byte, or one to three bit flips."""
    b = bytearray(b)
    r = rng.random()
    if r < 0.2:
        b = b[:rng.randrange(len(b))]
    elif r < 0.3:
        b += bytes([rng.randrange(256)])
    else:
        for _ in range(rng.randint(1, 3)):
            b[rng.randrange(len(b))] ^= 1 << rng.randrange(8)
    return bytes(b)


def edge_cases(frame, raw):
    """name -> (chunk, expected status, expected bytes or None), around one
    valid frame and its content."""
    return {
        "empty": (b"", 0, b""),
        "skippable only": (skippable(8), 0, b""),
        "empty skippable": (skippable(0), 0, b""),
        "skippable then frame": (skippable(3) + frame, 0, raw),
        "frame then 1 byte": (frame + b"\x28", 2, None),
        "frame then 3 bytes": (frame + b"\x28\xb5\x2f", 2, None),
        "frame then a bare magic": (frame + b"\x28\xb5\x2f\xfd", 2, None),
        "frame then a bare skippable magic": (frame + b"\x50\x2a\x4d\x18", 2, None),
        "skippable past the end": (skippable(8)[:-1], 2, None),
        "skippable size past the end": (frame + skippable(100)[:50], 2, None),
        "unknown magic after a frame": (frame + b"\x00\x01\x02\x03\x04\x05", 2, None),
        "truncated second frame": (frame + frame[:-1], 2, None),
    }

