/* Decode one .lz4 frame file with the GPU frame entry point, from plain C99.
 *
 *   decode_frame <input.lz4> <output>
 *
 * cudec_lz4f_decompress takes host memory in and out and is synchronous: it
 * stages the frame's blocks on the device, decodes them in one launch,
 * verifies the checksums the frame carries and copies the result back. When
 * the frame states no content size the caller does not know how large the
 * output is, so this program starts from a guess and doubles the buffer on
 * CUDEC_ERR_OUTPUT_TOO_SMALL. Exit status: 0 decoded and written, 1 usage or
 * file error, 2 the frame was refused (the status is printed).
 */
#include "cudec.h"

#include <stdio.h>
#include <stdlib.h>

static const char* status_name(cudec_status s) {
    switch (s) {
    case CUDEC_OK: return "OK";
    case CUDEC_ERR_INVALID_ARGUMENT: return "INVALID_ARGUMENT";
    case CUDEC_ERR_CORRUPT_INPUT: return "CORRUPT_INPUT";
    case CUDEC_ERR_OUTPUT_TOO_SMALL: return "OUTPUT_TOO_SMALL";
    case CUDEC_ERR_CUDA: return "CUDA";
    case CUDEC_ERR_NOT_IMPLEMENTED: return "NOT_IMPLEMENTED";
    case CUDEC_ERR_UNSUPPORTED: return "UNSUPPORTED";
    }
    return "?";
}

static unsigned char* read_file(const char* path, size_t* size) {
    FILE* f = fopen(path, "rb");
    unsigned char* buf = NULL;
    long n;
    if (f == NULL) return NULL;
    if (fseek(f, 0, SEEK_END) == 0 && (n = ftell(f)) >= 0 && fseek(f, 0, SEEK_SET) == 0) {
        buf = (unsigned char*)malloc(n > 0 ? (size_t)n : 1);
        if (buf != NULL && fread(buf, 1, (size_t)n, f) != (size_t)n) {
            free(buf);
            buf = NULL;
        }
        *size = (size_t)n;
    }
    fclose(f);
    return buf;
}

int main(int argc, char** argv) {
    /* the largest output this program is willing to allocate */
    const size_t kLimit = (size_t)1 << 32;
    unsigned char* frame;
    unsigned char* out = NULL;
    size_t frame_size = 0, capacity, written = 0;
    cudec_status st = CUDEC_ERR_OUTPUT_TOO_SMALL;
    FILE* f;

    if (argc != 3) {
        fprintf(stderr, "usage: %s <input.lz4> <output>\n", argv[0]);
        return 1;
    }
    frame = read_file(argv[1], &frame_size);
    if (frame == NULL) {
        fprintf(stderr, "%s: cannot read\n", argv[1]);
        return 1;
    }
    /* start from 4x the frame (at least 64 KiB) and double while too small */
    capacity = frame_size < 16384 ? 65536 : 4 * frame_size;
    while (st == CUDEC_ERR_OUTPUT_TOO_SMALL && capacity <= kLimit) {
        unsigned char* grown = (unsigned char*)realloc(out, capacity);
        if (grown == NULL) break;
        out = grown;
        st = cudec_lz4f_decompress(frame, frame_size, out, capacity, &written);
        if (st == CUDEC_ERR_OUTPUT_TOO_SMALL) capacity *= 2;
    }
    free(frame);
    if (st != CUDEC_OK) {
        fprintf(stderr, "%s: %s (cudec_status %d)\n", argv[1], status_name(st), (int)st);
        free(out);
        return 2;
    }
    f = fopen(argv[2], "wb");
    if (f == NULL || fwrite(out, 1, written, f) != written) {
        fprintf(stderr, "%s: cannot write\n", argv[2]);
        if (f != NULL) fclose(f);
        free(out);
        return 1;
    }
    fclose(f);
    free(out);
    printf("%s -> %s, %llu bytes\n", argv[1], argv[2], (unsigned long long)written);
    return 0;
}
