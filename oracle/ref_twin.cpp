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
#include "gdeflate_schedule.h"
#include "tilestream.h"

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


// The reference's GDeflate refill schedule (src/gdeflate_schedule.h) run over
// an operation list, recording the state after each op: the same encoding as
// oracle_gdeflate_schedule_trace (0 advance, 1..64 pop, 100 reset, 200
// ensure, 300 remove of the next slot's width).
int ref_gdeflate_schedule_trace(const uint8_t* page, uint64_t bytes, const uint32_t* ops,
                                uint64_t n_ops, uint64_t* trace) {
    using namespace cudec_detail;
    GDeflateSchedule s;
    const bool ok = GDeflateInit(s, page, bytes);
    trace[0] = s.cursor;
    trace[1] = s.idx;
    trace[2] = s.failed ? 1 : 0;
    trace[3] = ok ? 1 : 0;
    uint64_t t = 4, i = 0;
    while (i < n_ops) {
        const uint32_t op = ops[i++];
        uint64_t v = 0;
        if (op == 0) GDeflateAdvance(s, page);
        else if (op <= 64) v = GDeflatePop(s, op);
        else if (op == 100) GDeflateReset(s);
        else if (op == 200) GDeflateEnsure(s, page);
        else if (op == 300 && i < n_ops) GDeflateRemove(s, ops[i++]);
        trace[t++] = s.cursor;
        trace[t++] = s.idx;
        trace[t++] = s.failed ? 1 : 0;
        trace[t++] = v;
    }
    return static_cast<int>(t / 4);
}

// The reference's TileStream envelope walker (src/tilestream.h); tiles gets
// three words per tile (src offset, src size, dst size).
int ref_tilestream_parse(const uint8_t* st, uint64_t size, uint64_t* tiles, uint64_t tiles_cap,
                         uint64_t* count, uint64_t* total) {
    using namespace cudec_detail;
    std::vector<TileStreamTile> t(tiles_cap ? tiles_cap : 1);
    TileStreamInfo info{};
    const cudec_status st_ = TileStreamParse(st, size, t.data(), tiles_cap, &info);
    if (st_ == CUDEC_OK) {
        for (uint64_t k = 0; k < info.tile_count; ++k) {
            tiles[3 * k] = t[k].src_off;
            tiles[3 * k + 1] = t[k].src_size;
            tiles[3 * k + 2] = t[k].dst_size;
        }
        *count = info.tile_count;
        *total = info.total_uncompressed;
    }
    return st_;
}

}  // extern "C"
