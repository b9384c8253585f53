// Library-internal entry points of the mixed-format plan (csrc/mixed.cu) for
// the serving loop: launches without graph capture on a caller-chosen stream.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "cudec.h"

namespace cdb {

// Grow the plan's order buffer to hold max_chunks (may allocate; call before
// concurrent use).
cudaError_t mixed_reserve(cudec_mixed_plan* plan, size_t max_chunks);

// Enqueue one mixed decode (order kernels + persistent kernel) on `stream`
// without a graph. The plan's workspace must not be used by another launch
// in flight at the same time. Requires chunk_count <= the reserved count.
cudaError_t mixed_launch(cudec_mixed_plan* plan, const void* const* d_src_ptrs,
                         const size_t* d_src_sizes, void* const* d_dst_ptrs,
                         const size_t* d_dst_capacities, const uint8_t* d_formats,
                         size_t chunk_count, cudec_chunk_result* d_results, cudaStream_t stream);

}  // namespace cdb
