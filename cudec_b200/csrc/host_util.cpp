// Host resource helpers: the per-device memory pool and stream-ordered buffers.
#include "host_util.h"

#include <atomic>
#include <cstdint>
#include <mutex>

namespace cdb {

namespace {
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxPoolDevices];
bool g_pool_tried[kMaxPoolDevices];
}  // namespace

cudaMemPool_t device_pool(int dev) {
    if (dev < 0 || dev >= kMaxPoolDevices) return nullptr;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pool_tried[dev]) {
        g_pool_tried[dev] = true;
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
            // Keep up to 1 GiB of freed blocks cached between calls.
            uint64_t keep = 1ull << 30;
            (void)cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            g_pools[dev] = pool;
        } else {
            (void)cudaGetLastError();
        }
    }
    return g_pools[dev];
}

cudaError_t AsyncBuf::alloc(size_t bytes, cudaStream_t stream) {
    s = stream;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool = device_pool(dev);
    if (pool) return cudaMallocFromPoolAsync(&p, bytes ? bytes : 1, pool, stream);
    return cudaMallocAsync(&p, bytes ? bytes : 1, stream);
}

AsyncBuf::~AsyncBuf() {
    if (p) (void)cudaFreeAsync(p, s);
}

}  // namespace cdb
