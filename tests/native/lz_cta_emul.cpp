// Host emulation of the CTA-per-chunk LZ decoder (cudec_b200/csrc/
// lz_cta_kernel.cuh): the kernel's phases run for every thread in turn, so
// the CPU tests can check the decoder's algorithm (tiling, segment exits,
// candidate and tile chases, counts, checks, grouped execution, whole-CTA
// copies) against the oracle without a GPU. Test infrastructure only.
#include <cstdint>
#include <cstring>
#include <memory>

#include "lz_cta_kernel.cuh"

namespace {

template <class F>
int run(const uint8_t* src, uint64_t S, uint8_t* dst, uint64_t cap, uint64_t* written) {
    std::unique_ptr<cdb::lzc::Shm<F>> shm(new cdb::lzc::Shm<F>());
    std::memset(shm.get(), 0x5C, sizeof(cdb::lzc::Shm<F>));  // stale state must not matter
    cdb::lzc::Chunk<F> ch{*shm, src, S, dst, cap, 0};
    *written = 0;
    const int st = ch.run(written);
    if (st != CUDEC_OK) *written = 0;
    return st;
}

}  // namespace

// fmt 0 = LZ4, 1 = Snappy. src must have 16 readable bytes before src and
// after src + S, dst 4 before dst; dst receives the output.
extern "C" int lzc_emulate(int fmt, const uint8_t* src, uint64_t S, uint8_t* dst, uint64_t cap,
                           uint64_t* written) {
    return fmt == 0 ? run<cdb::lzc::Lz4F>(src, S, dst, cap, written)
                    : run<cdb::lzc::SnappyF>(src, S, dst, cap, written);
}

extern "C" uint64_t lzc_shm_bytes(int fmt) {
    return fmt == 0 ? sizeof(cdb::lzc::Shm<cdb::lzc::Lz4F>)
                    : sizeof(cdb::lzc::Shm<cdb::lzc::SnappyF>);
}
