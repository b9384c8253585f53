// XXH32 (seed 0 by default), written from the published xxHash specification
// (xxhash.com, "xxHash fast digest algorithm", 32-bit variant): four 32-bit
// accumulators over 16-byte stripes, then the 4-byte and 1-byte tails and the
// final avalanche. Used for the LZ4 frame's header, block and content
// checksums (lz4 frame format, "Header Checksum" / "Block checksum" /
// "Content checksum"). Host-only.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>

namespace cdb {

constexpr uint32_t kXxhP1 = 0x9E3779B1u;
constexpr uint32_t kXxhP2 = 0x85EBCA77u;
constexpr uint32_t kXxhP3 = 0xC2B2AE3Du;
constexpr uint32_t kXxhP4 = 0x27D4EB2Fu;
constexpr uint32_t kXxhP5 = 0x165667B1u;

inline uint32_t xxh_rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

inline uint32_t xxh_read32(const unsigned char* p) {
    uint32_t v;
    std::memcpy(&v, p, 4);  // little-endian hosts
    return v;
}

inline uint32_t xxh32(const void* data, size_t len, uint32_t seed = 0) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    const unsigned char* const end = p + len;
    uint32_t h;
    if (len >= 16) {
        uint32_t a = seed + kXxhP1 + kXxhP2, b = seed + kXxhP2, c = seed,
                 d = seed - kXxhP1;
        const unsigned char* const limit = end - 16;
        do {
            a = xxh_rotl(a + xxh_read32(p) * kXxhP2, 13) * kXxhP1;
            b = xxh_rotl(b + xxh_read32(p + 4) * kXxhP2, 13) * kXxhP1;
            c = xxh_rotl(c + xxh_read32(p + 8) * kXxhP2, 13) * kXxhP1;
            d = xxh_rotl(d + xxh_read32(p + 12) * kXxhP2, 13) * kXxhP1;
            p += 16;
        } while (p <= limit);
        h = xxh_rotl(a, 1) + xxh_rotl(b, 7) + xxh_rotl(c, 12) + xxh_rotl(d, 18);
    } else {
        h = seed + kXxhP5;
    }
    h += static_cast<uint32_t>(len);
    while (p + 4 <= end) {
        h = xxh_rotl(h + xxh_read32(p) * kXxhP3, 17) * kXxhP4;
        p += 4;
    }
    while (p < end) {
        h = xxh_rotl(h + (*p) * kXxhP5, 11) * kXxhP1;
        ++p;
    }
    h ^= h >> 15;
    h *= kXxhP2;
    h ^= h >> 13;
    h *= kXxhP3;
    h ^= h >> 16;
    return h;
}

}  // namespace cdb
