// ORACLE — test infrastructure, not part of the product.
//
// extern "C" shims over the reference's own host decoders, compiled from the
// reference's sources where they lie (see oracle/Makefile) into
// oracle/_ref/libref_twin.so. Nothing of the reference is copied here: this
// file only includes its headers and exposes plain-pointer entry points so the
// Python tests can call them through ctypes.
//
//   tests/lz4_twin.h:41-86      cudec_test::Lz4TwinDecode over src/lz4_block.h
//   tests/snappy_twin.h:140-160 cudec_test::SnappyTwinDecode over
//                               src/snappy_block.h
//   tests/zstd_twin_driver.h:178-390 cudec_twin::DecodeFrame over
//                               src/zstd_*.h
//
// The batch shims run those same functions over a std::thread pool; they are
// the "reference CPU implementation" timed by `bench.py --impl reference`.
#include "lz4_twin.h"
#include "snappy_twin.h"
#include "zstd_twin_driver.h"

#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

extern "C" {

int ref_lz4_twin_decode(const uint8_t* src, uint64_t n, uint8_t* dst,
                        uint64_t cap, uint64_t* written) {
    cudec_test::Lz4TwinResult r = cudec_test::Lz4TwinDecode(src, n, cap);
    *written = 0;
    if (r.status != CUDEC_OK) return r.status;
    if (r.size) std::memcpy(dst, r.bytes.get(), r.size);
    *written = r.size;
    return CUDEC_OK;
}

int ref_snappy_twin_decode(const uint8_t* src, uint64_t n, uint8_t* dst,
                           uint64_t cap, uint64_t* written) {
    std::vector<unsigned char> out;
    cudec_test::SnappyTwinObserver obs;
    cudec_status st = cudec_test::SnappyTwinDecode(src, n, cap, &out, &obs);
    *written = 0;
    if (st != CUDEC_OK) return st;
    if (!out.empty()) std::memcpy(dst, out.data(), out.size());
    *written = out.size();
    return CUDEC_OK;
}

int ref_zstd_twin_decode(const uint8_t* src, uint64_t n, uint8_t* dst,
                         uint64_t cap, uint64_t* written) {
    cudec_twin::Bytes frame(src, src + n);
    cudec_twin::Run run = cudec_twin::DecodeFrame(frame, cap);
    *written = 0;
    if (!run.ok) return run.status;
    if (!run.output.empty()) std::memcpy(dst, run.output.data(), run.output.size());
    *written = run.output.size();
    return CUDEC_OK;
}

typedef int (*ref_fn)(const uint8_t*, uint64_t, uint8_t*, uint64_t, uint64_t*);

static int ref_batch(ref_fn fn, const uint8_t* const* src,
                     const uint64_t* sizes, uint8_t* const* dst,
                     const uint64_t* caps, uint64_t n, int32_t* status,
                     uint64_t* written, int threads) {
    if (threads < 1) threads = 1;
    std::atomic<uint64_t> cursor{0};
    auto work = [&]() {
        for (;;) {
            uint64_t i = cursor.fetch_add(1);
            if (i >= n) break;
            uint64_t w = 0;
            status[i] = fn(src[i], sizes[i], dst[i], caps[i], &w);
            written[i] = w;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; t++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return threads;
}

int ref_lz4_twin_decode_batch(const uint8_t* const* src, const uint64_t* sizes,
                              uint8_t* const* dst, const uint64_t* caps,
                              uint64_t n, int32_t* status, uint64_t* written,
                              int threads) {
    return ref_batch(ref_lz4_twin_decode, src, sizes, dst, caps, n, status,
                     written, threads);
}

int ref_zstd_twin_decode_batch(const uint8_t* const* src, const uint64_t* sizes,
                               uint8_t* const* dst, const uint64_t* caps,
                               uint64_t n, int32_t* status, uint64_t* written,
                               int threads) {
    return ref_batch(ref_zstd_twin_decode, src, sizes, dst, caps, n, status,
                     written, threads);
}

int ref_snappy_twin_decode_batch(const uint8_t* const* src,
                                 const uint64_t* sizes, uint8_t* const* dst,
                                 const uint64_t* caps, uint64_t n,
                                 int32_t* status, uint64_t* written,
                                 int threads) {
    return ref_batch(ref_snappy_twin_decode, src, sizes, dst, caps, n, status,
                     written, threads);
}

}  // extern "C"
