"""Hand-built LZ4 and raw Snappy blocks for the GPU tests: a token-level
writer for each format, and blocks whose short matches read back across the
end of a token long enough to be copied straight to the destination."""
import random


def lz4_block(seqs, tail):
    """An LZ4 block from (literals, offset, match length) sequences and a
    final literal run."""
    out = bytearray()

    def ext(n):
        while n >= 255:
            out.append(255)
            n -= 255
        out.append(n)

    for lit, off, ml in seqs:
        out.append((min(len(lit), 15) << 4) | min(ml - 4, 15))
        if len(lit) >= 15:
            ext(len(lit) - 15)
        out += lit
        out += off.to_bytes(2, "little")
        if ml - 4 >= 15:
            ext(ml - 4 - 15)
    out.append(min(len(tail), 15) << 4)
    if len(tail) >= 15:
        ext(len(tail) - 15)
    out += tail
    return bytes(out)


def snappy_block(seqs, tail):
    """A raw Snappy block from the same sequences (copies split at 64)."""
    body = bytearray()
    total = 0

    def literal(b):
        n = len(b) - 1
        if n < 60:
            body.append(n << 2)
        else:
            nb = (n.bit_length() + 7) // 8
            body.append((59 + nb) << 2)
            body.extend(n.to_bytes(nb, "little"))
        body.extend(b)

    for lit, off, ml in seqs:
        if lit:
            literal(lit)
        total += len(lit) + ml
        while ml:
            k = min(ml, 64)
            body.append(((k - 1) << 2) | 2)
            body.extend(off.to_bytes(2, "little"))
            ml -= k
    literal(tail)
    total += len(tail)
    pre = bytearray()
    while True:
        b = total & 0x7F
        total >>= 7
        pre.append(b | (0x80 if total else 0))
        if not total:
            break
    return bytes(pre + body)


def straddle_blocks(seed):
    """Blocks in which tokens longer than the ring path (copied straight to
    the destination) are followed by short tokens whose match sources start
    before the long token's end and reach past it: sources split between the
    destination and the ring, with periods below and above 16 bytes."""
    rng = random.Random(seed)
    blocks = []
    for _ in range(24):
        seqs = [(bytes(rng.randrange(256) for _ in range(64)), 0, 0)]
        seqs[0] = (seqs[0][0], 7, 9)
        pos = 64 + 9
        for _ in range(rng.randint(1, 4)):
            if rng.random() < 0.5:  # a long literal run, short match
                lit = bytes(rng.randrange(256) for _ in range(rng.randint(257, 700)))
                off, ml = rng.randint(1, 60), 4
            else:  # a long match
                lit = bytes(rng.randrange(256) for _ in range(rng.randint(0, 3)))
                off, ml = rng.randint(1, 60), rng.randint(260, 600)
            seqs.append((lit, min(off, pos + len(lit)), ml))
            pos += len(lit) + ml
            for _ in range(rng.randint(1, 5)):
                lit = bytes(rng.randrange(256) for _ in range(rng.randint(0, 12)))
                off = min(rng.randint(1, 48), pos + len(lit))
                ml = rng.randint(4, 40)
                seqs.append((lit, off, ml))
                pos += len(lit) + ml
        blocks.append((seqs, bytes(rng.randrange(256) for _ in range(16))))
    return blocks

