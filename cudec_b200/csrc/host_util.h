// Host-side CUDA resource owners for the synchronous entry points (frame and
// stream decode). Every owner releases on scope exit, so no early return can
// leak device or pinned memory; nothing here throws.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace cdb {

// Per-device stream-ordered memory pool that keeps freed blocks cached
// across calls (the device's default pool trims to zero at every
// synchronize, which would turn each frame decode into fresh driver
// allocations). Returns nullptr when pools are unavailable.
cudaMemPool_t device_pool(int dev);

// Stream-ordered device allocation from device_pool(), freed on the owning
// stream at scope exit.
struct AsyncBuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    cudaError_t alloc(size_t bytes, cudaStream_t stream);
    ~AsyncBuf();
    AsyncBuf() = default;
    AsyncBuf(const AsyncBuf&) = delete;
    AsyncBuf& operator=(const AsyncBuf&) = delete;
};

struct StreamOwner {
    cudaStream_t s = nullptr;
    cudaError_t create() { return cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking); }
    ~StreamOwner() {
        if (s) {
            (void)cudaStreamSynchronize(s);
            (void)cudaStreamDestroy(s);
        }
    }
};

struct EventOwner {
    cudaEvent_t e = nullptr;
    cudaError_t create() { return cudaEventCreateWithFlags(&e, cudaEventDisableTiming); }
    ~EventOwner() {
        if (e) (void)cudaEventDestroy(e);
    }
};

// Grow-only device buffer (keeps its high-water size).
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) (void)cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 1);
        if (e == cudaSuccess) cap = bytes;
        return e;
    }
    ~DevBuf() {
        if (p) (void)cudaFree(p);
    }
};

// Grow-only pinned host buffer.
struct PinnedBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) (void)cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaHostAlloc(&p, bytes ? bytes : 1, cudaHostAllocDefault);
        if (e == cudaSuccess) cap = bytes;
        return e;
    }
    ~PinnedBuf() {
        if (p) (void)cudaFreeHost(p);
    }
};

}  // namespace cdb
