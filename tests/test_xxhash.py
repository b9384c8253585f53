"""The oracle's XXH32 (LZ4 frame checksums, src/xxhash32.h in the reference)
and XXH64 (Zstd content checksum, src/xxhash64.h) against an independent
Python restatement of the public xxHash specification, over every length up
to 1,100 bytes (all stripe and tail paths) and several seeds, plus the
specification's published digests of the empty input."""
import random

import oracle

M32, M64 = (1 << 32) - 1, (1 << 64) - 1
Q1, Q2, Q3, Q4, Q5 = 2654435761, 2246822519, 3266489917, 668265263, 374761393
R1, R2, R3, R4, R5 = (11400714785074694791, 14029467366897019727, 1609587929392839161,
                      9650029242287828579, 2870177450012600261)


def rotl32(x, r):
    return ((x << r) | (x >> (32 - r))) & M32


def rotl64(x, r):
    return ((x << r) | (x >> (64 - r))) & M64


def xxh32(b, seed=0):
    n, i = len(b), 0
    if n >= 16:
        v = [(seed + Q1 + Q2) & M32, (seed + Q2) & M32, seed & M32, (seed - Q1) & M32]
        while i + 16 <= n:
            for j in range(4):
                w = int.from_bytes(b[i + 4 * j:i + 4 * j + 4], "little")
                v[j] = (rotl32((v[j] + w * Q2) & M32, 13) * Q1) & M32
            i += 16
        h = (rotl32(v[0], 1) + rotl32(v[1], 7) + rotl32(v[2], 12) + rotl32(v[3], 18)) & M32
    else:
        h = (seed + Q5) & M32
    h = (h + n) & M32
    while i + 4 <= n:
        h = (rotl32((h + int.from_bytes(b[i:i + 4], "little") * Q3) & M32, 17) * Q4) & M32
        i += 4
    while i < n:
        h = (rotl32((h + b[i] * Q5) & M32, 11) * Q1) & M32
        i += 1
    h ^= h >> 15
    h = (h * Q2) & M32
    h ^= h >> 13
    h = (h * Q3) & M32
    return h ^ (h >> 16)


def _round(acc, lane):
    return (rotl64((acc + lane * R2) & M64, 31) * R1) & M64


def xxh64(b, seed=0):
    n, i = len(b), 0
    if n >= 32:
        v = [(seed + R1 + R2) & M64, (seed + R2) & M64, seed & M64, (seed - R1) & M64]
        while i + 32 <= n:
            for j in range(4):
                v[j] = _round(v[j], int.from_bytes(b[i + 8 * j:i + 8 * j + 8], "little"))
            i += 32
        h = (rotl64(v[0], 1) + rotl64(v[1], 7) + rotl64(v[2], 12) + rotl64(v[3], 18)) & M64
        for j in range(4):
            h = (((h ^ _round(0, v[j])) * R1) + R4) & M64
    else:
        h = (seed + R5) & M64
    h = (h + n) & M64
    while i + 8 <= n:
        h ^= _round(0, int.from_bytes(b[i:i + 8], "little"))
        h = (rotl64(h, 27) * R1 + R4) & M64
        i += 8
    if i + 4 <= n:
        h ^= (int.from_bytes(b[i:i + 4], "little") * R1) & M64
        h = (rotl64(h, 23) * R2 + R3) & M64
        i += 4
    while i < n:
        h ^= (b[i] * R5) & M64
        h = (rotl64(h, 11) * R1) & M64
        i += 1
    h ^= h >> 33
    h = (h * R2) & M64
    h ^= h >> 29
    h = (h * R3) & M64
    return h ^ (h >> 32)


def test_published_empty_digests():
    assert xxh32(b"") == 0x02CC5D05 == oracle.xxh32(b"")
    assert xxh64(b"") == 0xEF46DB3751D8E999 == oracle.xxh64(b"")


def test_length_sweep_and_seeds():
    rng = random.Random(9)
    data = bytes(rng.randrange(256) for _ in range(1100))
    for seed in (0, 1, 0x9E3779B1, M32):
        for n in range(0, 1101):
            b = data[:n]
            assert oracle.xxh32(b, seed) == xxh32(b, seed), (n, seed)
    for seed in (0, 1, 0x9E3779B97F4A7C15, M64):
        for n in range(0, 1101):
            b = data[:n]
            assert oracle.xxh64(b, seed) == xxh64(b, seed), (n, seed)
