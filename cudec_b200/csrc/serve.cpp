// Continuous-batching decode server (one device).
//
// Requests (a packed host buffer of compressed chunks plus per-chunk offsets,
// sizes, output capacities and format codes) arrive at any time from any
// thread. A worker thread admits them in arrival order as soon as an
// in-flight slot and enough of the device-memory budget are free, so work
// that arrives while other requests are on the GPU starts immediately and
// overlaps with them on the device. Each slot owns a stream and a mixed
// plan; a request costs one table upload, one input DMA straight from the
// caller's buffer, one persistent mixed launch (sized to the request) and a
// 16-byte-per-chunk result readback. Outputs stay resident in the server's
// device arena until the caller releases the request.
//
// The "plain" mode is the comparison path: one slot (a FIFO queue), and each
// request decoded by the per-format batch entries, one launch per format.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cudec.h"
#include "host_util.h"
#include "mixed.h"

namespace {

using Clock = std::chrono::steady_clock;

constexpr size_t kAlign = 256;

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// First-fit allocator over [0, size) of the device arena, coalescing frees.
class Arena {
   public:
    void init(size_t size) { free_[0] = size; }
    bool alloc(size_t bytes, size_t* off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes;
            const size_t at = it->first + bytes;
            free_.erase(it);
            if (rest) free_[at] = rest;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        auto it = free_.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }

   private:
    std::map<size_t, size_t> free_;
};

struct Request {
    uint64_t ticket = 0;
    const uint8_t* input = nullptr;
    size_t input_bytes = 0, n = 0;
    std::vector<size_t> offs, sizes, caps;
    std::vector<uint8_t> fmts;
    std::vector<uint32_t> perm;   // table row -> chunk index
    std::vector<uint8_t> refused; // plain mode: rows of an unknown format
    std::vector<size_t> out_off;  // per chunk, within the request's block
    size_t tables_bytes = 0, footprint = 0, block = 0;
    enum { kPending, kRunning, kDone } state = kPending;
    cudec_status status = CUDEC_OK;
    std::vector<cudec_chunk_result> results;
    Clock::time_point t_submit, t_done;
};

struct Slot {
    cudaStream_t s = nullptr;
    cudaEvent_t done = nullptr;
    cudec_mixed_plan* plan = nullptr;
    cdb::PinnedBuf stage, res;
    cdb::DevBuf zstd_ws;
    Request* req = nullptr;
    bool signalled = false;
};

}  // namespace

struct cudec_server {
    int mode = CUDEC_SERVER_MIXED;
    size_t budget = 0, max_chunks = 0;
    void* arena_base = nullptr;
    Arena arena;
    std::vector<std::unique_ptr<Slot>> slots;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread worker;
    int dev = -1;

    void run();
    cudaError_t launch(Slot& sl, Request& r);
    void finish(Slot& sl, cudaError_t err);
    ~cudec_server();
};

namespace {

void CUDART_CB on_slot_done(void* p) {
    auto* pair = static_cast<std::pair<cudec_server*, Slot*>*>(p);
    {
        std::lock_guard<std::mutex> lk(pair->first->mu);
        pair->second->signalled = true;
    }
    pair->first->cv.notify_all();
    delete pair;
}

}  // namespace

cudaError_t cudec_server::launch(Slot& sl, Request& r) {
    uint8_t* dbase = static_cast<uint8_t*>(arena_base) + r.block;
    const size_t n = r.n;
    // Table block: src ptrs, sizes, dst ptrs, caps (8 bytes each), results
    // (16), formats (1); then the input, then the outputs.
    cudaError_t e = sl.stage.ensure(r.tables_bytes);
    if (e != cudaSuccess) return e;
    uint8_t* h = static_cast<uint8_t*>(sl.stage.p);
    auto* src_ptrs = reinterpret_cast<uint64_t*>(h);
    auto* sizes = reinterpret_cast<uint64_t*>(h + 8 * n);
    auto* dst_ptrs = reinterpret_cast<uint64_t*>(h + 16 * n);
    auto* caps = reinterpret_cast<uint64_t*>(h + 24 * n);
    uint8_t* fmts = h + 48 * n;
    const size_t in_at = r.tables_bytes;
    const size_t out_at = align_up(in_at + r.input_bytes, kAlign);
    for (size_t j = 0; j < n; ++j) {
        const uint32_t i = r.perm[j];
        src_ptrs[j] = reinterpret_cast<uint64_t>(dbase + in_at + r.offs[i]);
        sizes[j] = r.sizes[i];
        dst_ptrs[j] = reinterpret_cast<uint64_t>(dbase + out_at + r.out_off[i]);
        caps[j] = r.caps[i];
        fmts[j] = r.fmts[i];
    }
    e = cudaMemcpyAsync(dbase, h, r.tables_bytes, cudaMemcpyHostToDevice, sl.s);
    if (e != cudaSuccess) return e;
    if (r.input_bytes) {
        e = cudaMemcpyAsync(dbase + in_at, r.input, r.input_bytes, cudaMemcpyHostToDevice, sl.s);
        if (e != cudaSuccess) return e;
    }
    auto* d_src = reinterpret_cast<const void* const*>(dbase);
    auto* d_sizes = reinterpret_cast<const size_t*>(dbase + 8 * n);
    auto* d_dst = reinterpret_cast<void* const*>(dbase + 16 * n);
    auto* d_caps = reinterpret_cast<const size_t*>(dbase + 24 * n);
    auto* d_res = reinterpret_cast<cudec_chunk_result*>(dbase + 32 * n);
    auto* d_fmts = reinterpret_cast<const uint8_t*>(dbase + 48 * n);
    if (mode == CUDEC_SERVER_MIXED) {
        e = cdb::mixed_launch(sl.plan, d_src, d_sizes, d_dst, d_caps, d_fmts, n, d_res, sl.s);
        if (e != cudaSuccess) return e;
    } else {
        // Rows are grouped by format: one batch launch per format present.
        r.refused.assign(n, 0);
        size_t j = 0;
        while (j < n) {
            size_t k = j;
            while (k < n && fmts[k] == fmts[j]) ++k;
            const cudec_stream_t cs = reinterpret_cast<cudec_stream_t>(sl.s);
            cudec_status st = CUDEC_OK;
            if (fmts[j] == CUDEC_FORMAT_LZ4)
                st = cudec_lz4_decompress_batch(d_src + j, d_sizes + j, d_dst + j, d_caps + j,
                                                k - j, d_res + j, cs);
            else if (fmts[j] == CUDEC_FORMAT_SNAPPY)
                st = cudec_snappy_decompress_batch(d_src + j, d_sizes + j, d_dst + j, d_caps + j,
                                                   k - j, d_res + j, cs);
            else if (fmts[j] == CUDEC_FORMAT_GDEFLATE)
                st = cudec_gdeflate_decompress_batch(d_src + j, d_sizes + j, d_dst + j,
                                                     d_caps + j, k - j, d_res + j, cs);
            else if (fmts[j] == CUDEC_FORMAT_ZSTD)
                st = cudec_zstd_decompress_batch(d_src + j, d_sizes + j, d_dst + j, d_caps + j,
                                                 k - j, d_res + j, sl.zstd_ws.p, sl.zstd_ws.cap,
                                                 cs);
            else
                st = CUDEC_ERR_UNSUPPORTED;  // recorded below for these rows
            if (st == CUDEC_ERR_UNSUPPORTED) {
                for (size_t q = j; q < k; ++q) r.refused[q] = 1;
            } else if (st != CUDEC_OK) {
                return cudaErrorLaunchFailure;
            }
            j = k;
        }
    }
    e = sl.res.ensure(16 * n);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(sl.res.p, d_res, 16 * n, cudaMemcpyDeviceToHost, sl.s);
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(sl.done, sl.s);
    if (e != cudaSuccess) return e;
    auto* pair = new (std::nothrow) std::pair<cudec_server*, Slot*>(this, &sl);
    if (pair == nullptr) return cudaErrorMemoryAllocation;
    e = cudaLaunchHostFunc(sl.s, on_slot_done, pair);
    if (e != cudaSuccess) delete pair;
    return e;
}

void cudec_server::finish(Slot& sl, cudaError_t err) {
    Request& r = *sl.req;
    r.results.assign(r.n, cudec_chunk_result{CUDEC_ERR_CUDA, 0, 0});
    if (err == cudaSuccess) {
        const auto* res = static_cast<const cudec_chunk_result*>(sl.res.p);
        for (size_t j = 0; j < r.n; ++j) {
            cudec_chunk_result x = res[j];
            if (!r.refused.empty() && r.refused[j]) x = cudec_chunk_result{CUDEC_ERR_UNSUPPORTED, 0, 0};
            r.results[r.perm[j]] = x;
        }
        r.status = CUDEC_OK;
    } else {
        r.status = CUDEC_ERR_CUDA;
    }
    r.t_done = Clock::now();
    r.state = Request::kDone;
    sl.req = nullptr;
    sl.signalled = false;
}

void cudec_server::run() {
    (void)cudaSetDevice(dev);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        bool progressed = false;
        for (auto& sp : slots) {
            Slot& sl = *sp;
            if (sl.req == nullptr) continue;
            const cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) continue;
            if (!sl.signalled && q == cudaSuccess) continue;  // the host callback is still queued
            finish(sl, q);
            progressed = true;
        }
        while (!pending.empty()) {
            Slot* free_slot = nullptr;
            for (auto& sp : slots)
                if (sp->req == nullptr) {
                    free_slot = sp.get();
                    break;
                }
            if (free_slot == nullptr) break;
            Request* r = pending.front();
            size_t off = 0;
            if (!arena.alloc(r->footprint, &off)) break;  // FIFO: wait for memory
            pending.pop_front();
            r->block = off;
            r->state = Request::kRunning;
            free_slot->req = r;
            lk.unlock();
            const cudaError_t e = launch(*free_slot, *r);
            lk.lock();
            if (e != cudaSuccess) {
                (void)cudaStreamSynchronize(free_slot->s);
                (void)cudaGetLastError();
                finish(*free_slot, e);
            }
            progressed = true;
        }
        if (progressed) cv.notify_all();
        bool busy = false;
        for (auto& sp : slots) busy = busy || sp->req != nullptr;
        if (stop && pending.empty() && !busy) break;
        if (!progressed) cv.wait_for(lk, std::chrono::microseconds(busy ? 200 : 5000));
    }
}

cudec_server::~cudec_server() {
    if (worker.joinable()) {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        worker.join();
    }
    for (auto& sp : slots) {
        Slot& sl = *sp;
        if (sl.s) (void)cudaStreamSynchronize(sl.s);
        if (sl.plan) (void)cudec_mixed_plan_destroy(sl.plan);
        if (sl.done) (void)cudaEventDestroy(sl.done);
        if (sl.s) (void)cudaStreamDestroy(sl.s);
    }
    if (arena_base) (void)cudaFree(arena_base);
}

extern "C" {

cudec_status cudec_server_create(size_t device_budget_bytes, int max_inflight, int mode,
                                 size_t max_chunks_per_request, cudec_server** out_server) {
    if (out_server == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    *out_server = nullptr;
    if (device_budget_bytes == 0 || max_chunks_per_request == 0 ||
        max_chunks_per_request > 0xFFFFFFFFull ||
        (mode != CUDEC_SERVER_MIXED && mode != CUDEC_SERVER_PLAIN) || max_inflight < 1 ||
        max_inflight > 64 || (mode == CUDEC_SERVER_PLAIN && max_inflight != 1))
        return CUDEC_ERR_INVALID_ARGUMENT;
    (void)cudaGetLastError();
    std::unique_ptr<cudec_server> s(new (std::nothrow) cudec_server());
    if (!s) return CUDEC_ERR_CUDA;
    s->mode = mode;
    s->budget = device_budget_bytes;
    s->max_chunks = max_chunks_per_request;
    if (cudaGetDevice(&s->dev) != cudaSuccess) return CUDEC_ERR_CUDA;
    if (cudaMalloc(&s->arena_base, device_budget_bytes) != cudaSuccess) {
        (void)cudaGetLastError();
        return CUDEC_ERR_CUDA;
    }
    s->arena.init(device_budget_bytes);
    for (int i = 0; i < max_inflight; ++i) {
        auto sl = std::make_unique<Slot>();
        bool ok = cudaStreamCreateWithFlags(&sl->s, cudaStreamNonBlocking) == cudaSuccess;
        ok = ok && cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming) == cudaSuccess;
        if (ok && mode == CUDEC_SERVER_MIXED) {
            ok = cudec_mixed_plan_create(&sl->plan) == CUDEC_OK;
            ok = ok && cdb::mixed_reserve(sl->plan, max_chunks_per_request) == cudaSuccess;
        }
        if (ok && mode == CUDEC_SERVER_PLAIN)
            ok = sl->zstd_ws.ensure(cudec_zstd_workspace_bytes(max_chunks_per_request)) ==
                 cudaSuccess;
        // Staging sized for the largest request up front: growing pinned
        // memory later would synchronize the device under other slots' work.
        ok = ok && sl->stage.ensure(align_up(49 * max_chunks_per_request, kAlign)) == cudaSuccess;
        ok = ok && sl->res.ensure(16 * max_chunks_per_request) == cudaSuccess;
        s->slots.push_back(std::move(sl));
        if (!ok) {
            (void)cudaGetLastError();
            return CUDEC_ERR_CUDA;
        }
    }
    s->worker = std::thread([p = s.get()] { p->run(); });
    *out_server = s.release();
    return CUDEC_OK;
}

cudec_status cudec_server_destroy(cudec_server* server) {
    if (server == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    delete server;
    return CUDEC_OK;
}

cudec_status cudec_server_submit(cudec_server* server, const void* h_input, size_t input_bytes,
                                 const size_t* h_offsets, const size_t* h_sizes,
                                 const size_t* h_dst_caps, const uint8_t* h_formats,
                                 size_t chunk_count, uint64_t* out_ticket) {
    if (server == nullptr || out_ticket == nullptr || h_offsets == nullptr ||
        h_sizes == nullptr || h_dst_caps == nullptr || h_formats == nullptr ||
        chunk_count == 0 || chunk_count > server->max_chunks ||
        (h_input == nullptr && input_bytes != 0))
        return CUDEC_ERR_INVALID_ARGUMENT;
    auto r = std::make_unique<Request>();
    const size_t n = chunk_count;
    r->input = static_cast<const uint8_t*>(h_input);
    r->input_bytes = input_bytes;
    r->n = n;
    r->offs.assign(h_offsets, h_offsets + n);
    r->sizes.assign(h_sizes, h_sizes + n);
    r->caps.assign(h_dst_caps, h_dst_caps + n);
    r->fmts.assign(h_formats, h_formats + n);
    r->out_off.resize(n);
    size_t out_total = 0;
    for (size_t i = 0; i < n; ++i) {
        if (r->offs[i] > input_bytes || r->sizes[i] > input_bytes - r->offs[i])
            return CUDEC_ERR_INVALID_ARGUMENT;
        r->out_off[i] = out_total;
        const size_t c = align_up(r->caps[i], 16);
        if (c < r->caps[i] || out_total + c < out_total) return CUDEC_ERR_INVALID_ARGUMENT;
        out_total += c;
    }
    r->perm.resize(n);
    for (size_t i = 0; i < n; ++i) r->perm[i] = static_cast<uint32_t>(i);
    if (server->mode == CUDEC_SERVER_PLAIN)
        std::stable_sort(r->perm.begin(), r->perm.end(),
                         [&](uint32_t a, uint32_t b) { return r->fmts[a] < r->fmts[b]; });
    r->tables_bytes = align_up(49 * n, kAlign);
    const size_t in_end = align_up(r->tables_bytes + input_bytes, kAlign);
    if (in_end < input_bytes || in_end + out_total < in_end) return CUDEC_ERR_INVALID_ARGUMENT;
    r->footprint = align_up(in_end + out_total, kAlign);
    if (r->footprint > server->budget) return CUDEC_ERR_INVALID_ARGUMENT;
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(server->mu);
        r->ticket = server->next_ticket++;
        *out_ticket = r->ticket;
        server->pending.push_back(r.get());
        server->reqs.emplace(r->ticket, std::move(r));
    }
    server->cv.notify_all();
    return CUDEC_OK;
}

}  // extern "C"

namespace {

// The wait of both entries; timeout_ms < 0 waits for good. *done = whether
// the request completed within the time (nothing is written otherwise).
cudec_status wait_request(cudec_server* server, uint64_t ticket, double timeout_ms, int* done,
                          cudec_chunk_result* h_results, void** h_dst_ptrs,
                          double* out_latency_ms) {
    std::unique_lock<std::mutex> lk(server->mu);
    auto it = server->reqs.find(ticket);
    if (it == server->reqs.end()) return CUDEC_ERR_INVALID_ARGUMENT;
    Request& r = *it->second;
    const auto finished = [&] { return r.state == Request::kDone; };
    if (timeout_ms < 0) {
        server->cv.wait(lk, finished);
    } else if (!server->cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                                    finished)) {
        *done = 0;
        return CUDEC_OK;
    }
    *done = 1;
    if (h_results) std::memcpy(h_results, r.results.data(), r.n * sizeof(cudec_chunk_result));
    if (h_dst_ptrs) {
        uint8_t* out = static_cast<uint8_t*>(server->arena_base) + r.block +
                       align_up(r.tables_bytes + r.input_bytes, kAlign);
        for (size_t i = 0; i < r.n; ++i) h_dst_ptrs[i] = out + r.out_off[i];
    }
    if (out_latency_ms)
        *out_latency_ms =
            std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count();
    return r.status;
}

}  // namespace

extern "C" {

cudec_status cudec_server_wait(cudec_server* server, uint64_t ticket,
                               cudec_chunk_result* h_results, void** h_dst_ptrs,
                               double* out_latency_ms) {
    if (server == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    int done = 0;
    return wait_request(server, ticket, -1.0, &done, h_results, h_dst_ptrs, out_latency_ms);
}

cudec_status cudec_server_wait_for(cudec_server* server, uint64_t ticket, double timeout_ms,
                                   int* out_done, cudec_chunk_result* h_results,
                                   void** h_dst_ptrs, double* out_latency_ms) {
    if (server == nullptr || out_done == nullptr || !(timeout_ms >= 0.0))
        return CUDEC_ERR_INVALID_ARGUMENT;
    *out_done = 0;
    return wait_request(server, ticket, timeout_ms, out_done, h_results, h_dst_ptrs,
                        out_latency_ms);
}

cudec_status cudec_server_release(cudec_server* server, uint64_t ticket) {
    if (server == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(server->mu);
        auto it = server->reqs.find(ticket);
        if (it == server->reqs.end() || it->second->state != Request::kDone)
            return CUDEC_ERR_INVALID_ARGUMENT;
        server->arena.release(it->second->block, it->second->footprint);
        server->reqs.erase(it);
    }
    server->cv.notify_all();
    return CUDEC_OK;
}

}  // extern "C"
