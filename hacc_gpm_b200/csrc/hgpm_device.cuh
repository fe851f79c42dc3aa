// hgpm_device.cuh — device-side shared definitions of the PM step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hgpm {

constexpr int kThreads = 256;            // threads per CTA for all pass kernels
// int64 fixed-point density: value * 2^31.  Each CIC weight (times the
// particle mass) is rounded to 2^-24, the FP32 resolution of a unit weight,
// and stored shifted by kQShift, so a unit weight is 2^24 in a 32-bit
// shared-memory window and 2^31 in the int64 grid.
constexpr double kFixScale = 2147483648.0;
constexpr double kFixInv = 1.0 / 2147483648.0;
constexpr float kQ24F = 16777216.0f;
constexpr int kQShift = 7;

// Particle positions are a packed cell (10 bits per axis, ng <= 1024) plus
// an FP32 offset in [0, 1) per axis.
__host__ __device__ __forceinline__ uint32_t pack_cell(int ix, int iy, int iz) {
    return ((uint32_t)ix << 20) | ((uint32_t)iy << 10) | (uint32_t)iz;
}
__host__ __device__ __forceinline__ int cell_x(uint32_t c) { return (int)(c >> 20); }
__host__ __device__ __forceinline__ int cell_y(uint32_t c) { return (int)((c >> 10) & 1023u); }
__host__ __device__ __forceinline__ int cell_z(uint32_t c) { return (int)(c & 1023u); }

// Particle state, structure of arrays (coalesced 4-byte streams).
struct ParticleSoA {
    uint32_t* cell;
    float* ox;
    float* oy;
    float* oz;
    float* vx;
    float* vy;
    float* vz;
};

__host__ __device__ __forceinline__ ParticleSoA offset_soa(ParticleSoA p, size_t off) {
    return ParticleSoA{p.cell + off, p.ox + off, p.oy + off, p.oz + off, p.vx + off, p.vy + off, p.vz + off};
}

// Slots of a batched launch: the boxes of one size class live in slabs with a
// fixed element stride per buffer, so slot s of a kernel's first buffer starts
// s*s0 elements after slot 0 (second buffer: s*s1; the per-block window
// records of the deposit and kick: s*s2).  `active` (may be null: every slot
// runs) lets idle slots' CTAs return at once.  A single-box launch passes
// Slots{} and has one slot.
struct Slots {
    const int* active = nullptr;
    size_t s0 = 0, s1 = 0, s2 = 0;
};
__device__ __forceinline__ bool slot_idle(const Slots& b, int slot) { return b.active && !b.active[slot]; }

// Blocks whose CIC window is wider than a kernel's shared-memory window:
// the windowed kernel queues them (cnt[slot], items[slot * nblocks + i]) and
// a one-particle-per-thread pass handles their particles.
struct SpillList {
    int* cnt = nullptr;
    int* items = nullptr;
    int nblocks = 0;
    // blocks whose window exceeds the float4 kick's cap, counted by the
    // deposit (over[slot]); the kick reads it to choose its path
    int* over = nullptr;
    // work counter of a persistent windowed kernel (next block to take)
    int* next = nullptr;
};

// Per-slot kick parameters of a batched step: row `slot` of a table of
// float4 (dtf = float(deltaT*fscal), pf_a, pf_b, ndrift) indexed by the
// slot's step counter.  sched == null: the launch's own scalars apply.
struct KickSched {
    const float4* sched = nullptr;
    const int* step = nullptr;
    int pitch = 0;
};

// Signed mode index as get_kmodes maps it (src/haccgpm.hpp:255-274).
__host__ __device__ __forceinline__ int signed_mode(int i, int n) { return i > n / 2 - 1 ? i - n : i; }

// Internal particle order: Lagrangian blocks of B^3 particles stored
// contiguously (block-major, then x, y, z inside the block), so that one CTA
// owns a compact patch of space.  The C-ABI exchanges particles in the
// reference's lattice order q = (qx*np + qy)*np + qz (get_index).
__host__ __device__ __forceinline__ int block_side(int np, int ng) {
    return (np % 16 == 0 && ng <= np) ? 16 : 8;
}
__host__ __device__ __forceinline__ size_t lattice_of_internal(size_t p, int np, int B) {
    const size_t B3 = (size_t)B * B * B;
    const size_t blk = p / B3;
    const int l = (int)(p % B3);
    const int nb = np / B;
    const int bz = (int)(blk % nb), by = (int)((blk / nb) % nb), bx = (int)(blk / ((size_t)nb * nb));
    const int lz = l % B, ly = (l / B) % B, lx = l / (B * B);
    return ((size_t)(bx * B + lx) * np + (by * B + ly)) * np + (bz * B + lz);
}

}  // namespace hgpm
