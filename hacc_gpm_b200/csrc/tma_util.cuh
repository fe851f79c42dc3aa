// tma_util.cuh — TMA (cp.async.bulk.tensor) and mbarrier helpers for the
// persistent FFT passes.  Plain (non-multicast) loads and stores only.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace hgpm {

constexpr int kTmaThreads = 256;
constexpr unsigned kMaxPolls = 1u << 22;

// Rows per TMA box: the largest divisor d of n with d <= 256 (a box
// dimension) whose box of ct complex columns is a whole number of 128-byte
// lines (d * ct * 8 % 128 == 0), so every box's shared-memory destination,
// b * d * ct * 8 bytes into a 1024-aligned tile, is 128-byte aligned.
constexpr int box_rows(int n, int ct, int d = 256) {
    return d <= 1 ? 1 : ((n % d == 0 && (d * ct * 8) % 128 == 0) ? d : box_rows(n, ct, d - 1));
}

template <int NG> struct TmaCfg {
    static constexpr int CT = NG <= 256 ? 16 : (NG <= 512 ? 8 : 4);  // complex columns per tile
    // rows per TMA box (384 -> 2 x 192, 1000 -> 5 x 200)
    static constexpr int RB = box_rows(NG, CT);
    static_assert(NG % RB == 0 && RB <= 256 && (RB * CT * 8) % 128 == 0, "TMA box rows");
    static constexpr int NBOX = NG / RB;
    static constexpr int TILE_BYTES = NG * CT * 8;
    static constexpr int SMEM = 2 * TILE_BYTES + 1024;               // + alignment slack
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// bounded wait: false after kMaxPolls unsuccessful polls
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (unsigned i = 0; i < kMaxPolls; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_store_4d(const CUtensorMap* tm, int c0, int c1, int c2, int c3, const void* src) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                     reinterpret_cast<uint64_t>(tm)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// tile t -> (column chunk, plane, component)
struct TileIdx {
    int chunk, plane, comp;
};
__device__ __forceinline__ TileIdx tile_of(int t, int nchunks, int nplanes) {
    TileIdx r;
    r.chunk = t % nchunks;
    const int rest = t / nchunks;
    r.plane = rest % nplanes;
    r.comp = rest / nplanes;
    return r;
}

}  // namespace hgpm
