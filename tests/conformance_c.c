/* ABI conformance from plain C: include/cudec.h compiles as C99 (its record
 * layout check then takes the negative-array-size form) and as C11
 * (_Static_assert), every public entry point resolves with C linkage, and
 * each entry's documented synchronous rejects hold for a C caller. The
 * reference pins the same properties in tests/conformance_c.c (version
 * encoding, the batch reject classes, the frame and stream argument rules).
 *
 * Every call below is a reject that the header documents as returning before
 * any CUDA call, or a host-only parse, so the program runs on a machine with
 * no GPU. The pointers are host memory and are never dereferenced by the
 * library. Exit status 0 and a final PASS line mean every check held. */
#include "cudec.h"

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

static int failures = 0;

#define CHECK(cond)                                                           \
    do {                                                                      \
        if (!(cond)) {                                                        \
            fprintf(stderr, "FAIL %s:%d: %s\n", __FILE__, __LINE__, #cond);   \
            ++failures;                                                       \
        }                                                                     \
    } while (0)

typedef cudec_status (*batch_fn)(const void* const*, const size_t*, void* const*,
                                 const size_t*, size_t, cudec_chunk_result*,
                                 cudec_stream_t);

/* The reject classes every batch entry shares: a NULL array, NULL or
 * misaligned results, an empty batch, a count above the launch limit. */
static void batch_rejects(const char* name, batch_fn fn, cudec_chunk_result* aligned) {
    const void* srcs[4] = {0, 0, 0, 0};
    size_t sizes[4] = {0, 0, 0, 0};
    void* dsts[4] = {0, 0, 0, 0};
    size_t caps[4] = {0, 0, 0, 0};
    cudec_chunk_result* misaligned = (cudec_chunk_result*)((unsigned char*)aligned + 8);
    int before = failures;
    CHECK(fn(0, sizes, dsts, caps, 4, aligned, 0) == CUDEC_ERR_INVALID_ARGUMENT);
    CHECK(fn(srcs, 0, dsts, caps, 4, aligned, 0) == CUDEC_ERR_INVALID_ARGUMENT);
    CHECK(fn(srcs, sizes, 0, caps, 4, aligned, 0) == CUDEC_ERR_INVALID_ARGUMENT);
    CHECK(fn(srcs, sizes, dsts, 0, 4, aligned, 0) == CUDEC_ERR_INVALID_ARGUMENT);
    CHECK(fn(srcs, sizes, dsts, caps, 4, 0, 0) == CUDEC_ERR_INVALID_ARGUMENT);
    CHECK(fn(srcs, sizes, dsts, caps, 4, misaligned, 0) == CUDEC_ERR_INVALID_ARGUMENT);
    CHECK(fn(srcs, sizes, dsts, caps, 0, aligned, 0) == CUDEC_ERR_INVALID_ARGUMENT);
    CHECK(fn(srcs, sizes, dsts, caps, SIZE_MAX, aligned, 0) == CUDEC_ERR_INVALID_ARGUMENT);
    if (failures != before) fprintf(stderr, "  (in %s)\n", name);
}

int main(void) {
    /* 16-byte aligned host storage standing in for device arrays. */
    static uint64_t storage[64];
    cudec_chunk_result* aligned = (cudec_chunk_result*)storage;
    const void* srcs[4] = {0, 0, 0, 0};
    size_t sizes[4] = {0, 0, 0, 0};
    void* dsts[4] = {0, 0, 0, 0};
    size_t caps[4] = {0, 0, 0, 0};
    uint8_t formats[4] = {0, 0, 0, 0};

    /* version: the macros' encoding, and this release's number */
    CHECK(cudec_version() == CUDEC_VERSION_MAJOR * 10000 + CUDEC_VERSION_MINOR * 100 +
                                 CUDEC_VERSION_PATCH);
    CHECK(cudec_version() == 100);

    /* the result record and the enum values are fixed by the ABI */
    CHECK(sizeof(cudec_chunk_result) == 16);
    CHECK(offsetof(cudec_chunk_result, status) == 0);
    CHECK(offsetof(cudec_chunk_result, reserved) == 4);
    CHECK(offsetof(cudec_chunk_result, bytes_written) == 8);
    CHECK(sizeof(cudec_tile) == 24);
    CHECK(CUDEC_OK == 0 && CUDEC_ERR_INVALID_ARGUMENT == 1 && CUDEC_ERR_CORRUPT_INPUT == 2 &&
          CUDEC_ERR_OUTPUT_TOO_SMALL == 3 && CUDEC_ERR_CUDA == 4 &&
          CUDEC_ERR_NOT_IMPLEMENTED == 5 && CUDEC_ERR_UNSUPPORTED == 6);
    CHECK(CUDEC_MEM_HOST == 0 && CUDEC_MEM_DEVICE == 1);
    CHECK(CUDEC_FORMAT_LZ4 == 0 && CUDEC_FORMAT_SNAPPY == 1 && CUDEC_FORMAT_ZSTD == 2 &&
          CUDEC_FORMAT_GDEFLATE == 3);

    /* batch entries */
    batch_rejects("cudec_lz4_decompress_batch", cudec_lz4_decompress_batch, aligned);
    batch_rejects("cudec_snappy_decompress_batch", cudec_snappy_decompress_batch, aligned);
    batch_rejects("cudec_gdeflate_decompress_batch", cudec_gdeflate_decompress_batch, aligned);
    batch_rejects("cudec_zstd_decompress_batch_noalloc", cudec_zstd_decompress_batch_noalloc,
                  aligned);

    /* Zstd: the workspace rule, and the allocation-free entry's chunk limit */
    {
        const size_t ws = cudec_zstd_workspace_bytes(4);
        CHECK(ws > 0);
        CHECK(cudec_zstd_workspace_bytes(64) >= ws);
        CHECK(cudec_zstd_decompress_batch(srcs, sizes, dsts, caps, 4, aligned, 0, ws, 0) ==
              CUDEC_ERR_INVALID_ARGUMENT); /* NULL workspace */
        CHECK(cudec_zstd_decompress_batch(srcs, sizes, dsts, caps, 4, aligned, storage, ws - 1,
                                          0) == CUDEC_ERR_INVALID_ARGUMENT); /* short */
        CHECK(cudec_zstd_decompress_batch(0, sizes, dsts, caps, 4, aligned, storage, ws, 0) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_zstd_decompress_batch(srcs, sizes, dsts, caps, 0, aligned, storage, ws, 0) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_zstd_decompress_batch_noalloc(srcs, sizes, dsts, caps,
                                                  CUDEC_ZSTD_NOALLOC_MAX_CHUNKS + 1, aligned,
                                                  0) == CUDEC_ERR_INVALID_ARGUMENT);
        /* the multi-frame entry keeps every argument rule */
        CHECK(cudec_zstd_decompress_batch_multi(srcs, sizes, dsts, caps, 4, aligned, 0, ws, 0) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_zstd_decompress_batch_multi(srcs, sizes, dsts, caps, 4, aligned, storage,
                                                ws - 1, 0) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_zstd_decompress_batch_multi(
                  srcs, sizes, dsts, caps, 4, (cudec_chunk_result*)((unsigned char*)aligned + 8),
                  storage, ws, 0) == CUDEC_ERR_INVALID_ARGUMENT); /* misaligned records */
        CHECK(cudec_zstd_decompress_batch_multi(srcs, sizes, dsts, caps, 0, aligned, storage, ws,
                                                0) == CUDEC_ERR_INVALID_ARGUMENT);
    }

    /* GDeflate TileStream: the envelope walker is host-only */
    {
        cudec_tile tiles[4];
        size_t count = 7, total = 7, written = 7;
        const unsigned char junk[3] = {1, 2, 3};
        unsigned char out[8];
        CHECK(cudec_gdeflate_tilestream_parse(0, 0, tiles, 4, &count, &total) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_gdeflate_tilestream_parse(junk, sizeof junk, tiles, 4, &count, &total) ==
              CUDEC_ERR_CORRUPT_INPUT);
        CHECK(cudec_gdeflate_tilestream_decompress(0, 0, out, sizeof out, CUDEC_MEM_HOST,
                                                   &written) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(written == 0);
        CHECK(cudec_gdeflate_tilestream_decompress(junk, sizeof junk, out, sizeof out,
                                                   (cudec_mem_space)5, &written) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_gdeflate_tilestream_decompress(junk, sizeof junk, out, sizeof out,
                                                   CUDEC_MEM_HOST, &written) ==
              CUDEC_ERR_CORRUPT_INPUT);
        CHECK(written == 0);
    }

    /* mixed plan: every entry refuses a NULL plan */
    {
        uint32_t params[3 * CUDEC_MIXED_BUCKETS];
        CHECK(cudec_mixed_plan_create(0) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_mixed_plan_destroy(0) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_mixed_decompress(0, srcs, sizes, dsts, caps, formats, 4, aligned, 0) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_mixed_plan_tune(0, srcs, sizes, dsts, caps, formats, 4, aligned, 0) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_mixed_plan_get_tuning(0, params) == CUDEC_ERR_INVALID_ARGUMENT);
    }

    /* server: argument rules of create, and a NULL server everywhere else */
    {
        cudec_server* srv = 0;
        uint64_t ticket = 0;
        double ms = 0;
        size_t offs[1] = {0};
        CHECK(cudec_server_create(0, 4, CUDEC_SERVER_MIXED, 4096, &srv) ==
              CUDEC_ERR_INVALID_ARGUMENT); /* no budget */
        CHECK(cudec_server_create(1 << 20, 0, CUDEC_SERVER_MIXED, 4096, &srv) ==
              CUDEC_ERR_INVALID_ARGUMENT); /* no slots */
        CHECK(cudec_server_create(1 << 20, 2, CUDEC_SERVER_PLAIN, 4096, &srv) ==
              CUDEC_ERR_INVALID_ARGUMENT); /* plain mode is one slot */
        CHECK(cudec_server_create(1 << 20, 4, 7, 4096, &srv) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_server_create(1 << 20, 4, CUDEC_SERVER_MIXED, 0, &srv) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_server_create(1 << 20, 4, CUDEC_SERVER_MIXED, 4096, 0) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(srv == 0);
        CHECK(cudec_server_submit(0, storage, 8, offs, sizes, caps, formats, 1, &ticket) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_server_wait(0, 1, 0, 0, &ms) == CUDEC_ERR_INVALID_ARGUMENT);
        {
            int done = 7;
            CHECK(cudec_server_wait_for(0, 1, 5.0, &done, 0, 0, &ms) ==
                  CUDEC_ERR_INVALID_ARGUMENT);
        }
        CHECK(cudec_server_release(0, 1) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_server_destroy(0) == CUDEC_ERR_INVALID_ARGUMENT);
    }

    /* LZ4 frame entry */
    {
        size_t written = 123;
        unsigned char byte = 0;
        CHECK(cudec_lz4f_decompress(0, 0, &byte, 1, &written) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(written == 0);
        CHECK(cudec_lz4f_decompress(&byte, 1, &byte, 1, 0) == CUDEC_ERR_INVALID_ARGUMENT);
        written = 123;
        CHECK(cudec_lz4f_decompress(&byte, 1, 0, 1, &written) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(written == 0);
    }

    /* streaming entries; the records stay untouched on a reject */
    {
        cudec_chunk_result res[1];
        memset(res, 0x5a, sizeof res);
        CHECK(cudec_lz4_decompress_stream(0, sizes, dsts, caps, 1, CUDEC_MEM_DEVICE, res) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_lz4_decompress_stream(srcs, sizes, dsts, caps, 0, CUDEC_MEM_DEVICE, res) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_lz4_decompress_stream(srcs, sizes, dsts, caps, 1, (cudec_mem_space)7, res) ==
              CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_stream_ctx_create(0) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_lz4_decompress_stream_ctx(0, srcs, sizes, dsts, caps, 1, CUDEC_MEM_DEVICE,
                                              res) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(cudec_lz4_decompress_stream_ctx(0, srcs, sizes, dsts, caps, 0, CUDEC_MEM_HOST,
                                              res) == CUDEC_ERR_INVALID_ARGUMENT);
        CHECK(res[0].status == 0x5a5a5a5a && res[0].bytes_written == 0x5a5a5a5a5a5a5a5aull);
        cudec_stream_ctx_destroy(0); /* NULL-safe */
    }

    if (failures) {
        fprintf(stderr, "%d check(s) failed\n", failures);
        return 1;
    }
    printf("PASS: every public entry point called from C\n");
    return 0;
}
