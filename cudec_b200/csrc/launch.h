// Internal (non-ABI) declarations shared by the library's translation units.
#pragma once

#include <cstddef>
#include <cstdint>

#include "cudec.h"

namespace cdb {

// One chunk per warp slot and at most INT32_MAX warps: the largest batch any
// entry maps onto a launch (same bound as iderex/cudec src/batch_limits.h:28).
constexpr size_t kMaxBatchChunks = static_cast<size_t>(INT32_MAX) * 32;

// Synchronous argument rules of every batch entry: non-NULL arrays, 16-byte
// aligned results, 0 < n <= kMaxBatchChunks. Makes no CUDA call.
cudec_status validate_batch(const void* const* src, const size_t* src_sizes,
                            void* const* dst, const size_t* caps, size_t n,
                            const cudec_chunk_result* results);

// Multiprocessor count of `dev`, cached; 0 on failure.
int device_sm_count(int dev);

}  // namespace cdb
