/* cudec-b200: batch decompression for NVIDIA B200 (sm_100a).
 *
 * Public C ABI. Binary-compatible with the iderex/cudec interface
 * (include/cudec.h of that project): the same status values, the same
 * 16-byte per-chunk result record, the same entry-point signatures and the
 * same synchronous/asynchronous split. A caller built against that header
 * links against this library unchanged. Entry points that the reference does
 * not ship carry the same contract shape and say so where they are declared.
 *
 * Nothing here needs CUDA headers. No entry point throws or longjmps across
 * this boundary, and no output is reported that was not fully validated.
 */
#ifndef CUDEC_H
#define CUDEC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUDEC_VERSION_MAJOR 0
#define CUDEC_VERSION_MINOR 1
#define CUDEC_VERSION_PATCH 0

/* Runtime library version, major * 10000 + minor * 100 + patch.
 * Replaces: src/version.c:3-6 (declared include/cudec.h:26). */
int cudec_version(void);

/* Replaces: include/cudec.h:28-43. Values are fixed by the ABI. */
typedef enum cudec_status {
    CUDEC_OK = 0,
    CUDEC_ERR_INVALID_ARGUMENT = 1,
    CUDEC_ERR_CORRUPT_INPUT = 2,
    CUDEC_ERR_OUTPUT_TOO_SMALL = 3,
    CUDEC_ERR_CUDA = 4,
    /* Kept at this value for exhaustive switches; no entry point returns it. */
    CUDEC_ERR_NOT_IMPLEMENTED = 5,
    /* Valid input outside the decoded subset (e.g. an LZ4 frame in
     * block-linked mode, or one carrying a dictionary id). */
    CUDEC_ERR_UNSUPPORTED = 6
} cudec_status;

/* Same representation as cudaStream_t (a pointer to CUstream_st). NULL is
 * the legacy default stream. Replaces: include/cudec.h:49. */
typedef struct CUstream_st* cudec_stream_t;

/* Per-chunk outcome written by the device into caller memory.
 * Replaces: include/cudec.h:53-78 (layout pinned below). */
typedef struct cudec_chunk_result {
    int32_t status;         /* a cudec_status value */
    uint32_t reserved;      /* always written as zero */
    uint64_t bytes_written; /* decoded bytes when status == CUDEC_OK, else 0 */
} cudec_chunk_result;

#if defined(__cplusplus) && __cplusplus >= 201103L
static_assert(sizeof(cudec_chunk_result) == 16 &&
                  offsetof(cudec_chunk_result, bytes_written) == 8,
              "cudec_chunk_result is a fixed 16-byte record");
#elif defined(__STDC_VERSION__) && __STDC_VERSION__ >= 201112L
_Static_assert(sizeof(cudec_chunk_result) == 16 &&
                   offsetof(cudec_chunk_result, bytes_written) == 8,
               "cudec_chunk_result is a fixed 16-byte record");
#else
typedef char cudec_chunk_result_size_check
    [(sizeof(cudec_chunk_result) == 16 &&
      offsetof(cudec_chunk_result, bytes_written) == 8) ? 1 : -1];
#endif

/* ---------------------------------------------------------------------
 * Batch block decode (device memory in, device memory out, asynchronous)
 *
 * Every array argument is a device array of chunk_count entries and every
 * pointer held in them is a device pointer. d_results must be 16-byte
 * aligned. Synchronous return: argument validation and launch submission
 * only. Per-chunk outcomes land in d_results once `stream` reaches the end of
 * the launch. A chunk that decodes reports CUDEC_OK and bytes_written, and
 * exactly dst[0, bytes_written) was written. A chunk that does not reports
 * CUDEC_ERR_CORRUPT_INPUT or CUDEC_ERR_OUTPUT_TOO_SMALL with bytes_written 0;
 * its destination is then unspecified (never beyond its capacity).
 *
 * Validation failures return CUDEC_ERR_INVALID_ARGUMENT, launch nothing and
 * make no CUDA call (the thread's pending CUDA error is left as it was): a
 * NULL array, a misaligned d_results, chunk_count == 0, or chunk_count above
 * the launch limit (2^31-1 warps of 32 chunks; rejected, never truncated).
 * A call that passes validation consumes the pending CUDA error, so the
 * returned status describes this submission alone. The library allocates
 * nothing on this path. Thread-safe for distinct streams.
 * ------------------------------------------------------------------- */

/* LZ4 block format (one raw LZ4 block per chunk).
 * Replaces: include/cudec.h:102-108, src/batch.cu:6-31. */
cudec_status cudec_lz4_decompress_batch(const void* const* d_src_ptrs,
                                        const size_t* d_src_sizes,
                                        void* const* d_dst_ptrs,
                                        const size_t* d_dst_capacities,
                                        size_t chunk_count,
                                        cudec_chunk_result* d_results,
                                        cudec_stream_t stream);

/* Raw Snappy block format (varint length preamble + elements; no framing).
 * Not shipped by the reference: its design record commits this exact
 * signature with "no deltas" from the LZ4 entry (docs/MASTERPLAN.md:720-740);
 * the per-chunk rules follow src/snappy_block.h:58-436. The declared length
 * above the chunk's capacity is CUDEC_ERR_OUTPUT_TOO_SMALL; every other
 * inconsistency, including under- or over-production of the declared length,
 * is CUDEC_ERR_CORRUPT_INPUT. */
cudec_status cudec_snappy_decompress_batch(const void* const* d_src_ptrs,
                                           const size_t* d_src_sizes,
                                           void* const* d_dst_ptrs,
                                           const size_t* d_dst_capacities,
                                           size_t chunk_count,
                                           cudec_chunk_result* d_results,
                                           cudec_stream_t stream);

/* Zstd frames (RFC 8878), one frame per chunk, in the reference's v1 subset
 * (docs/MASTERPLAN.md:1208-1251; ladder src/zstd_frame.h:196-409 and the
 * units it drives, status mapping tests/zstd_twin_driver.h:178-390). Not
 * shipped by the reference as a kernel; same contract shape as the LZ4 entry
 * plus a caller-owned device workspace, so the call still allocates nothing.
 * Statuses: skippable frames, a dictionary id, no content size, a window above
 * 8 MB -> CUDEC_ERR_UNSUPPORTED; content size above the capacity or output
 * past it -> CUDEC_ERR_OUTPUT_TOO_SMALL; any other inconsistency (headers,
 * literals, tables, sequences, repeat offsets, window, content size,
 * checksum, trailing bytes) -> CUDEC_ERR_CORRUPT_INPUT. d_workspace must hold
 * cudec_zstd_workspace_bytes(chunk_count) bytes (a NULL or short workspace is
 * CUDEC_ERR_INVALID_ARGUMENT); it may be reused once the launch completes. */
size_t cudec_zstd_workspace_bytes(size_t chunk_count);

cudec_status cudec_zstd_decompress_batch(const void* const* d_src_ptrs,
                                         const size_t* d_src_sizes,
                                         void* const* d_dst_ptrs,
                                         const size_t* d_dst_capacities,
                                         size_t chunk_count,
                                         cudec_chunk_result* d_results,
                                         void* d_workspace,
                                         size_t workspace_bytes,
                                         cudec_stream_t stream);

/* Zstd chunks that hold a sequence of frames, read the way libzstd's
 * one-shot ZSTD_decompress reads a buffer: the reference's subset ladder
 * (docs/MASTERPLAN.md:1286-1296), which the reference leaves untaken, up to
 * that decoder's limits; no counterpart in its ABI. Skippable frames (magic
 * 0x184D2A50-0x184D2A5F, then a 4-byte little-endian size) are skipped, and
 * each Zstd frame decodes into the output right after the previous frame's
 * bytes. Beyond cudec_zstd_decompress_batch's subset a frame may omit its
 * content size (its output is bounded by the capacity alone) and may declare
 * any window up to a window log of 31; a dictionary id, or a larger window
 * log, is CUDEC_ERR_UNSUPPORTED. The chunk keeps one 16-byte record:
 * bytes_written is the sum over its frames, and the status is the first
 * failing frame's (then bytes_written is 0 and the output is undefined). An
 * empty chunk decodes to zero bytes; fewer than 4 bytes left after a frame,
 * or a skippable frame that runs past the chunk, is CUDEC_ERR_CORRUPT_INPUT.
 * Workspace and every argument rule as cudec_zstd_decompress_batch; the
 * one-frame entry above is unchanged. */
cudec_status cudec_zstd_decompress_batch_multi(const void* const* d_src_ptrs,
                                               const size_t* d_src_sizes,
                                               void* const* d_dst_ptrs,
                                               const size_t* d_dst_capacities,
                                               size_t chunk_count,
                                               cudec_chunk_result* d_results,
                                               void* d_workspace,
                                               size_t workspace_bytes,
                                               cudec_stream_t stream);

/* Allocation-free Zstd batch entry, for callers that cannot allocate device
 * memory. No counterpart in the reference. Same statuses and records as
 * cudec_zstd_decompress_batch, but the per-frame literal slots come from a
 * static device array inside the library (8 MiB), so a call takes at most
 * CUDEC_ZSTD_NOALLOC_MAX_CHUNKS chunks: a larger chunk_count is
 * CUDEC_ERR_INVALID_ARGUMENT, returned before any CUDA call. The array is
 * shared by every call on a device: calls whose launches overlap in time
 * (different streams or host threads) race on it; calls queued on one stream
 * are ordered and safe. The first call on a device looks up the array's
 * device address (once per device, with that device current), so make that
 * first call before any stream capture. The address is kept for the life of
 * the process: after cudaDeviceReset on a device, this entry must not be
 * called on it again until the library is reloaded. */
#define CUDEC_ZSTD_NOALLOC_MAX_CHUNKS 64

cudec_status cudec_zstd_decompress_batch_noalloc(const void* const* d_src_ptrs,
                                                 const size_t* d_src_sizes,
                                                 void* const* d_dst_ptrs,
                                                 const size_t* d_dst_capacities,
                                                 size_t chunk_count,
                                                 cudec_chunk_result* d_results,
                                                 cudec_stream_t stream);

/* ---------------------------------------------------------------------
 * GDeflate (no decoder in the reference; its 32-lane refill schedule and
 * TileStream envelope are src/gdeflate_schedule.h and src/tilestream.h). One
 * page per chunk, at most 64 KiB out; the page format's open points are
 * decided as documented with the decoder. Statuses: OUTPUT_TOO_SMALL when a
 * page produces more than the capacity, CORRUPT_INPUT for every malformed
 * page (including one that would produce more than 64 KiB or does not end
 * exactly at its last word). */
cudec_status cudec_gdeflate_decompress_batch(const void* const* d_src_ptrs,
                                             const size_t* d_src_sizes,
                                             void* const* d_dst_ptrs,
                                             const size_t* d_dst_capacities,
                                             size_t chunk_count,
                                             cudec_chunk_result* d_results,
                                             cudec_stream_t stream);

/* One validated tile of a TileStream container. */
typedef struct cudec_tile {
    uint64_t src_offset; /* from the start of the stream */
    uint64_t src_size;
    uint64_t dst_size;
} cudec_tile;

/* The TileStream envelope walker (src/tilestream.h:117-261): host memory,
 * no device work. INVALID_ARGUMENT for NULL arguments or a tile array smaller
 * than the declared count; CORRUPT_INPUT for everything the bytes get wrong. */
cudec_status cudec_gdeflate_tilestream_parse(const void* h_stream, size_t stream_size,
                                             cudec_tile* tiles, size_t tiles_capacity,
                                             size_t* out_tile_count, size_t* out_total);

/* ---------------------------------------------------------------------
 * Mixed-format persistent batch decode (no counterpart in the reference; the
 * design record's batching direction). One launch decodes LZ4 blocks, raw
 * Snappy blocks, Zstd frames and GDeflate pages in any mix, with per-chunk
 * statuses and bytes
 * identical to the per-format entries. A plan (bound to the device current at
 * creation) owns the device workspace (work counter, a largest-first chunk
 * order, Zstd literal slots), the decode shape per size bucket and a CUDA
 * graph of the launch sequence, captured once per argument set and replayed.
 * d_formats holds one cudec_format code per chunk; an unknown code is
 * CUDEC_ERR_UNSUPPORTED for that chunk. chunk_count <= 2^32 - 1. Calls on one
 * plan are serialised on its private stream and ordered after `stream`. */
typedef enum cudec_format {
    CUDEC_FORMAT_LZ4 = 0,
    CUDEC_FORMAT_SNAPPY = 1,
    CUDEC_FORMAT_ZSTD = 2,
    CUDEC_FORMAT_GDEFLATE = 3
} cudec_format;

/* Size buckets of the tuned decode shape, by output capacity: < 4 KiB,
 * < 16 KiB, < 64 KiB, < 256 KiB, < 1 MiB, larger. */
#define CUDEC_MIXED_BUCKETS 6

/* Warps of the CTA-per-chunk LZ4 / Snappy decoder (the whole-CTA value of a
 * decode shape's warps per chunk). */
#define CUDEC_MIXED_CTA_WARPS 8

typedef struct cudec_mixed_plan cudec_mixed_plan;

cudec_status cudec_mixed_plan_create(cudec_mixed_plan** out_plan);
cudec_status cudec_mixed_plan_destroy(cudec_mixed_plan* plan);

cudec_status cudec_mixed_decompress(cudec_mixed_plan* plan,
                                    const void* const* d_src_ptrs,
                                    const size_t* d_src_sizes,
                                    void* const* d_dst_ptrs,
                                    const size_t* d_dst_capacities,
                                    const uint8_t* d_formats,
                                    size_t chunk_count,
                                    cudec_chunk_result* d_results,
                                    cudec_stream_t stream);

/* Autotuner: decodes the given batch once per candidate shape (parse reach,
 * input lookahead, ring batch), bucket by bucket, timing each on the device,
 * and keeps the fastest per bucket; then, per bucket, times its LZ4 and
 * Snappy chunks under that one-warp shape against a whole CTA per chunk and
 * keeps the faster. Synchronous; destinations and results receive the
 * normal decode. */
cudec_status cudec_mixed_plan_tune(cudec_mixed_plan* plan,
                                   const void* const* d_src_ptrs,
                                   const size_t* d_src_sizes,
                                   void* const* d_dst_ptrs,
                                   const size_t* d_dst_capacities,
                                   const uint8_t* d_formats,
                                   size_t chunk_count,
                                   cudec_chunk_result* d_results,
                                   cudec_stream_t stream);

/* out_params[3*b .. 3*b+2] = parse reach, lookahead, ring batch of bucket b. */
cudec_status cudec_mixed_plan_get_tuning(const cudec_mixed_plan* plan,
                                         uint32_t* out_params);

/* The whole decode shape, 4 values per bucket b: out_shape[4*b] = warps per
 * LZ4 / Snappy chunk (1: one warp; CUDEC_MIXED_CTA_WARPS: a whole CTA runs
 * the CTA-per-chunk decoder), then parse reach, lookahead and ring batch of
 * the one-warp decoder. A plan starts from a compiled-in table (one warp per
 * LZ4 / Snappy chunk below 16 KiB, a whole CTA from 16 KiB up);
 * cudec_mixed_plan_tune measures one on
 * the caller's chunks. A caller can save the shape and set it on later
 * plans, so the decode shape is fixed across runs; set_shape refuses
 * (INVALID_ARGUMENT, nothing changed) a warps value other than 1 or
 * CUDEC_MIXED_CTA_WARPS, or an out-of-range one-warp shape. Any shape
 * decodes identically; it only moves time. */
cudec_status cudec_mixed_plan_get_shape(const cudec_mixed_plan* plan, uint32_t* out_shape);
cudec_status cudec_mixed_plan_set_shape(cudec_mixed_plan* plan, const uint32_t* shape);

/* ---------------------------------------------------------------------
 * Continuous-batching decode server (no counterpart in the reference). A
 * server owns a device arena of `device_budget_bytes` and `max_inflight`
 * slots (a stream and a mixed plan each). Requests are admitted in arrival
 * order as soon as a slot and enough of the budget are free, so requests
 * that arrive while others run overlap with them on the device. A request's
 * footprint (tables, compressed input, 16-byte-aligned outputs) must fit the
 * whole budget. Outputs stay in the arena until the request is released.
 * CUDEC_SERVER_PLAIN (requires max_inflight == 1) decodes each request with
 * the per-format batch entries in arrival order: the comparison path. */
#define CUDEC_SERVER_MIXED 0
#define CUDEC_SERVER_PLAIN 1

typedef struct cudec_server cudec_server;

cudec_status cudec_server_create(size_t device_budget_bytes, int max_inflight, int mode,
                                 size_t max_chunks_per_request, cudec_server** out_server);
/* Waits for admitted work; requests still queued are decoded first. */
cudec_status cudec_server_destroy(cudec_server* server);

/* h_input holds the compressed chunks (chunk i at h_offsets[i], h_sizes[i]
 * bytes) and must stay valid until cudec_server_wait returns for the ticket;
 * the per-chunk arrays are copied. Returns at once with a ticket. */
cudec_status cudec_server_submit(cudec_server* server, const void* h_input, size_t input_bytes,
                                 const size_t* h_offsets, const size_t* h_sizes,
                                 const size_t* h_dst_caps, const uint8_t* h_formats,
                                 size_t chunk_count, uint64_t* out_ticket);

/* Blocks until the request is decoded. h_results (chunk_count records) and
 * h_dst_ptrs (device addresses of the outputs) may be NULL; *out_latency_ms =
 * submit to completion. Returns CUDEC_ERR_CUDA if the request's device work
 * failed, else CUDEC_OK (per-chunk statuses in the records). */
cudec_status cudec_server_wait(cudec_server* server, uint64_t ticket,
                               cudec_chunk_result* h_results, void** h_dst_ptrs,
                               double* out_latency_ms);

/* The same with a deadline: waits at most timeout_ms (>= 0) milliseconds.
 * If the request completed, *out_done = 1 and the outputs are as for
 * cudec_server_wait; otherwise *out_done = 0, CUDEC_OK is returned and
 * nothing else is written (wait again later). A negative or NaN timeout or a
 * NULL out_done is CUDEC_ERR_INVALID_ARGUMENT. No counterpart in the
 * reference. */
cudec_status cudec_server_wait_for(cudec_server* server, uint64_t ticket, double timeout_ms,
                                   int* out_done, cudec_chunk_result* h_results,
                                   void** h_dst_ptrs, double* out_latency_ms);

/* Returns the request's device memory to the budget (after wait). */
cudec_status cudec_server_release(cudec_server* server, uint64_t ticket);

/* ---------------------------------------------------------------------
 * LZ4 frame (.lz4 container), host memory in and out, synchronous.
 * Replaces: include/cudec.h:130-132, src/frame.cpp:401-422.
 *
 * Decodes block-INDEPENDENT frames; verifies the header, block and content
 * checksums and the declared content size when present. Returns
 * CUDEC_ERR_UNSUPPORTED for a valid frame outside that subset (block-linked
 * mode, a dictionary id), CUDEC_ERR_CORRUPT_INPUT for a malformed frame or a
 * checksum / content-size mismatch, CUDEC_ERR_OUTPUT_TOO_SMALL when
 * dst_capacity is short, CUDEC_ERR_CUDA on a device or host resource failure,
 * and CUDEC_ERR_INVALID_ARGUMENT for a NULL frame or bytes_written, or a NULL
 * dst with a non-zero capacity. On any error *bytes_written is 0.
 * ------------------------------------------------------------------- */
cudec_status cudec_lz4f_decompress(const void* frame, size_t frame_size,
                                   void* dst, size_t dst_capacity,
                                   size_t* bytes_written);

/* Memory space of the streaming decoder's destinations.
 * Replaces: include/cudec.h:135-138. */
typedef enum cudec_mem_space {
    CUDEC_MEM_HOST = 0,   /* host destinations; output is copied back */
    CUDEC_MEM_DEVICE = 1  /* device destinations; output stays in HBM */
} cudec_mem_space;

/* GDeflate TileStream container, synchronous: parse, one page-batch launch
 * over every tile; each tile must produce exactly its size (else
 * CORRUPT_INPUT; the first failing tile's status otherwise). dst is host or
 * device memory per dst_space. */
cudec_status cudec_gdeflate_tilestream_decompress(const void* h_stream, size_t stream_size,
                                                  void* dst, size_t dst_capacity,
                                                  cudec_mem_space dst_space,
                                                  size_t* out_written);

/* ---------------------------------------------------------------------
 * Streaming batch LZ4 block decode from HOST-resident chunks.
 * Replaces: include/cudec.h:140-218, src/stream.cpp:492-593.
 *
 * A context owns a CUDA stream and grow-only pinned/device staging (sized to
 * the largest batch so far); create it once per thread and reuse it. It is
 * not thread-safe. Decoding is synchronous: every destination and result is
 * final on return. Argument arrays are host arrays of chunk_count entries;
 * dst_ptrs are host or device pointers per dst_space; exactly bytes_written
 * bytes are written per successful chunk, in both spaces.
 *
 * A NULL ctx or array, a NULL source with a non-zero size, a NULL
 * destination with a non-zero capacity, an unknown dst_space, chunk_count ==
 * 0 or above the launch limit: CUDEC_ERR_INVALID_ARGUMENT, nothing decoded,
 * the context not poisoned, h_results untouched. Otherwise every record is
 * defined on return; the aggregate is CUDEC_OK iff every chunk decoded, else
 * CUDEC_ERR_CUDA if a device/host resource failure happened, else the first
 * non-OK chunk's status in index order. A CUDA fault poisons the context:
 * every later decode returns CUDEC_ERR_CUDA without touching the device;
 * only destroy is valid on it. Nothing throws across this boundary.
 * ------------------------------------------------------------------- */
typedef struct cudec_stream_ctx cudec_stream_ctx;

cudec_status cudec_stream_ctx_create(cudec_stream_ctx** out_ctx);

cudec_status cudec_lz4_decompress_stream_ctx(
    cudec_stream_ctx* ctx, const void* const* h_src_ptrs,
    const size_t* h_src_sizes, void* const* dst_ptrs, const size_t* dst_caps,
    size_t chunk_count, cudec_mem_space dst_space,
    cudec_chunk_result* h_results);

/* NULL-safe; valid on a poisoned context. */
void cudec_stream_ctx_destroy(cudec_stream_ctx* ctx);

/* One-shot: create, one decode, destroy (pays the staging every call). */
cudec_status cudec_lz4_decompress_stream(const void* const* h_src_ptrs,
                                         const size_t* h_src_sizes,
                                         void* const* dst_ptrs,
                                         const size_t* dst_caps,
                                         size_t chunk_count,
                                         cudec_mem_space dst_space,
                                         cudec_chunk_result* h_results);

#ifdef __cplusplus
}
#endif

#endif /* CUDEC_H */
