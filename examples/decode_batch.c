/* Decode a batch of LZ4 blocks and a batch of raw Snappy blocks on the GPU
 * through the batch entry points, from plain C99 and the CUDA runtime.
 *
 *   decode_batch          (no arguments; exit status 0 when every chunk
 *                          reports what is printed as expected)
 *
 * The blocks are written out below field by field. Three things a first-time
 * caller has to get right:
 *   - every array passed to a batch entry is DEVICE memory, and the pointers
 *     stored in the source and destination arrays are device pointers too:
 *     the host builds the pointer tables and copies them up;
 *   - the call is asynchronous on the stream: its return value covers
 *     argument validation and submission only, and each chunk's outcome is
 *     in its cudec_chunk_result once the stream has been synchronised;
 *   - chunks are independent: a corrupt chunk or one whose capacity is too
 *     small gets its own status (with bytes_written 0) and the others decode.
 */
#include "cudec.h"

#include <cuda_runtime.h>

#include <stdio.h>
#include <string.h>

/* One LZ4 block: a 3-byte literal run "abc", a 13-byte match at offset 3
 * (it overlaps its own output, so it repeats "abc"), then the 5-byte literal
 * run every LZ4 block ends with.
 *   0x39        token: 3 literals, match length 9 + 4
 *   'a' 'b' 'c' the literals
 *   03 00       offset 3, little endian
 *   0x50        token: 5 literals, no match
 *   "-end\n"    the literals */
static const unsigned char kLz4Block[] = {0x39, 'a', 'b', 'c', 0x03, 0x00,
                                          0x50, '-', 'e', 'n', 'd', '\n'};

/* The same block with offset 16: the match would read before the start of
 * the output, which the format forbids. */
static const unsigned char kLz4BadOffset[] = {0x39, 'a', 'b', 'c', 0x10, 0x00,
                                              0x50, '-', 'e', 'n', 'd', '\n'};

/* The same text as a raw Snappy block.
 *   21          varint preamble: 21 bytes of output
 *   0x08        literal tag, length 2 + 1
 *   'a' 'b' 'c'
 *   0x32 03 00  copy with a 2-byte offset: length 12 + 1, offset 3
 *   0x10        literal tag, length 4 + 1
 *   "-end\n" */
static const unsigned char kSnappyBlock[] = {21,   0x08, 'a', 'b', 'c', 0x32, 0x03,
                                             0x00, 0x10, '-', 'e', 'n', 'd', '\n'};

static const char kText[] = "abcabcabcabcabca-end\n"; /* 21 bytes */

static const char* status_name(int s) {
    switch (s) {
    case CUDEC_OK: return "OK";
    case CUDEC_ERR_INVALID_ARGUMENT: return "INVALID_ARGUMENT";
    case CUDEC_ERR_CORRUPT_INPUT: return "CORRUPT_INPUT";
    case CUDEC_ERR_OUTPUT_TOO_SMALL: return "OUTPUT_TOO_SMALL";
    case CUDEC_ERR_CUDA: return "CUDA";
    case CUDEC_ERR_UNSUPPORTED: return "UNSUPPORTED";
    default: return "?";
    }
}

#define MAX_CHUNKS 4
#define SLOT 64 /* bytes per source and per destination slot */

/* Uploads the n blocks, decodes them with `entry` into destinations of the
 * given capacities, and checks each chunk's status (and, for OK, its bytes)
 * against `expect`. Returns the number of mismatches, or -1 on a CUDA or
 * submission failure. */
typedef cudec_status (*batch_entry)(const void* const*, const size_t*, void* const*,
                                    const size_t*, size_t, cudec_chunk_result*,
                                    cudec_stream_t);

static int run_batch(const char* label, batch_entry entry, const unsigned char* const* blocks,
                     const size_t* block_sizes, const size_t* caps, const int* expect,
                     size_t n) {
    unsigned char* d_src = NULL;
    unsigned char* d_dst = NULL;
    void* d_tables = NULL;
    cudec_chunk_result* d_results = NULL;
    const void* h_src_ptrs[MAX_CHUNKS];
    void* h_dst_ptrs[MAX_CHUNKS];
    cudec_chunk_result h_results[MAX_CHUNKS];
    unsigned char out[MAX_CHUNKS][SLOT];
    cudaStream_t stream;
    int bad = 0;
    size_t i;

    if (cudaStreamCreate(&stream) != cudaSuccess) return -1;
    /* sources and destinations: one slot of SLOT bytes per chunk */
    if (cudaMalloc((void**)&d_src, n * SLOT) != cudaSuccess ||
        cudaMalloc((void**)&d_dst, n * SLOT) != cudaSuccess ||
        /* four tables of n entries: sources, sizes, destinations, capacities */
        cudaMalloc(&d_tables, 4 * n * sizeof(void*)) != cudaSuccess ||
        /* cudaMalloc memory is 256-byte aligned, so the records are 16-byte
         * aligned as the entry requires */
        cudaMalloc((void**)&d_results, n * sizeof(cudec_chunk_result)) != cudaSuccess) {
        bad = -1;
        goto done;
    }
    for (i = 0; i < n; ++i) {
        if (cudaMemcpy(d_src + i * SLOT, blocks[i], block_sizes[i], cudaMemcpyHostToDevice) !=
            cudaSuccess) {
            bad = -1;
            goto done;
        }
        h_src_ptrs[i] = d_src + i * SLOT;
        h_dst_ptrs[i] = d_dst + i * SLOT;
    }
    {
        const void** t_src = (const void**)d_tables;
        size_t* t_sizes = (size_t*)(t_src + n);
        void** t_dst = (void**)(t_sizes + n);
        size_t* t_caps = (size_t*)(t_dst + n);
        cudec_status st;
        if (cudaMemcpy(t_src, h_src_ptrs, n * sizeof(void*), cudaMemcpyHostToDevice) !=
                cudaSuccess ||
            cudaMemcpy(t_sizes, block_sizes, n * sizeof(size_t), cudaMemcpyHostToDevice) !=
                cudaSuccess ||
            cudaMemcpy(t_dst, h_dst_ptrs, n * sizeof(void*), cudaMemcpyHostToDevice) !=
                cudaSuccess ||
            cudaMemcpy(t_caps, caps, n * sizeof(size_t), cudaMemcpyHostToDevice) !=
                cudaSuccess) {
            bad = -1;
            goto done;
        }
        st = entry(t_src, t_sizes, t_dst, t_caps, n, d_results, stream);
        if (st != CUDEC_OK) {
            fprintf(stderr, "%s: submission failed: %s\n", label, status_name(st));
            bad = -1;
            goto done;
        }
    }
    /* the outcomes exist once the stream reaches the end of the launch */
    if (cudaStreamSynchronize(stream) != cudaSuccess ||
        cudaMemcpy(h_results, d_results, n * sizeof(cudec_chunk_result),
                   cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(out, d_dst, n * SLOT, cudaMemcpyDeviceToHost) != cudaSuccess) {
        bad = -1;
        goto done;
    }
    for (i = 0; i < n; ++i) {
        const cudec_chunk_result* r = &h_results[i];
        int ok = r->status == expect[i] && r->reserved == 0;
        if (r->status == CUDEC_OK)
            ok = ok && r->bytes_written == sizeof kText - 1 &&
                 memcmp(out[i], kText, sizeof kText - 1) == 0;
        else
            ok = ok && r->bytes_written == 0;
        printf("%s chunk %u: capacity %2u -> %-16s %2llu bytes", label, (unsigned)i,
               (unsigned)caps[i], status_name(r->status), (unsigned long long)r->bytes_written);
        if (r->status == CUDEC_OK) printf("  \"%.*s\\n\"", (int)r->bytes_written - 1, out[i]);
        printf("%s\n", ok ? "" : "  <- unexpected");
        bad += !ok;
    }

done:
    cudaFree(d_results);
    cudaFree(d_tables);
    cudaFree(d_dst);
    cudaFree(d_src);
    cudaStreamDestroy(stream);
    return bad;
}

int main(void) {
    /* LZ4: a good block, a match that reaches before the output, and the
     * good block with 15 bytes of room (its 13-byte match does not fit). */
    const unsigned char* lz4_blocks[3] = {kLz4Block, kLz4BadOffset, kLz4Block};
    const size_t lz4_sizes[3] = {sizeof kLz4Block, sizeof kLz4BadOffset, sizeof kLz4Block};
    const size_t lz4_caps[3] = {SLOT, SLOT, 15};
    const int lz4_expect[3] = {CUDEC_OK, CUDEC_ERR_CORRUPT_INPUT, CUDEC_ERR_OUTPUT_TOO_SMALL};
    /* Snappy: a good block, and the same block when its declared 21 bytes do
     * not fit a 20-byte destination. */
    const unsigned char* snappy_blocks[2] = {kSnappyBlock, kSnappyBlock};
    const size_t snappy_sizes[2] = {sizeof kSnappyBlock, sizeof kSnappyBlock};
    const size_t snappy_caps[2] = {SLOT, 20};
    const int snappy_expect[2] = {CUDEC_OK, CUDEC_ERR_OUTPUT_TOO_SMALL};
    int a, b;

    printf("cudec %d\n", cudec_version());
    a = run_batch("lz4   ", cudec_lz4_decompress_batch, lz4_blocks, lz4_sizes, lz4_caps,
                  lz4_expect, 3);
    b = run_batch("snappy", cudec_snappy_decompress_batch, snappy_blocks, snappy_sizes,
                  snappy_caps, snappy_expect, 2);
    if (a < 0 || b < 0) {
        fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(cudaGetLastError()));
        return 2;
    }
    if (a + b) return 1;
    printf("all chunks as expected\n");
    return 0;
}
