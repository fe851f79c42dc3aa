// particles.cu — particle-side kernels of the PM step: state conversion,
// drift, deterministic fixed-point CIC deposit, fused CIC gather + kick +
// drift(s), and the small per-size table kernels.
//
// Positions are a packed int32 cell (10 bits per axis) plus an FP32 offset
// in [0, 1) per axis; the offset equals the reference's `x - (int)x`
// (cic_pm.cu:52-58) bit for bit when a state is loaded.
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <stdint.h>
#include <math.h>

#include <map>
#include <mutex>
#include <utility>

#include "hgpm_device.cuh"
#include "hgpm_internal.h"
#include "multi_class.h"

namespace hgpm {

__device__ __forceinline__ int wrap_axis(int i, int ng) {
    if ((unsigned)i >= (unsigned)ng) {
        i %= ng;
        if (i < 0) i += ng;
    }
    return i;
}

// One axis of UpdatePosKernel (update_positions_pm.cu:9-14):
// x <- x + v*pf wrapped periodically, done on (cell, offset).
__device__ __forceinline__ void drift_axis(int& i, float& o, float v, float pf, int ng) {
    float d = fmaf(v, pf, o);
    float fl = floorf(d);
    d -= fl;
    if (d >= 1.f) {
        d -= 1.f;
        fl += 1.f;
    }
    o = d;
    i = wrap_axis(i + (int)fl, ng);
}

__device__ __forceinline__ void split_axis(float x, int ng, int& i, float& o) {
    float fl = floorf(x);
    o = x - fl;
    if (o >= 1.f) {
        o -= 1.f;
        fl += 1.f;
    }
    i = wrap_axis((int)fl, ng);
}

// State conversion between the reference layout (float3, lattice order) and
// the internal SoA in Lagrangian-block order (hgpm_device.cuh).
__global__ void load_state_kernel(const float* __restrict__ x, const float* __restrict__ v, ParticleSoA p,
                                  int np_side, int B, int ng) {
    const size_t n = (size_t)np_side * np_side * np_side;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t q = lattice_of_internal(i, np_side, B);
    int ix, iy, iz;
    float ox, oy, oz;
    split_axis(x[3 * q + 0], ng, ix, ox);
    split_axis(x[3 * q + 1], ng, iy, oy);
    split_axis(x[3 * q + 2], ng, iz, oz);
    p.cell[i] = pack_cell(ix, iy, iz);
    p.ox[i] = ox;
    p.oy[i] = oy;
    p.oz[i] = oz;
    p.vx[i] = v[3 * q + 0];
    p.vy[i] = v[3 * q + 1];
    p.vz[i] = v[3 * q + 2];
}

// x = cell + offset in float; a sum that rounds up to ng is stored as 0, so
// positions stay in [0, ng) as the reference's fmod keeps them.
__device__ __forceinline__ float join_axis(int cell, float o, float fng) {
    const float x = (float)cell + o;
    return x >= fng ? x - fng : x;
}

__global__ void store_state_kernel(ParticleSoA p, float* __restrict__ x, float* __restrict__ v, int np_side, int B,
                                   int ng) {
    const size_t n = (size_t)np_side * np_side * np_side;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t q = lattice_of_internal(i, np_side, B);
    const uint32_t c = p.cell[i];
    const float fng = (float)ng;
    x[3 * q + 0] = join_axis(cell_x(c), p.ox[i], fng);
    x[3 * q + 1] = join_axis(cell_y(c), p.oy[i], fng);
    x[3 * q + 2] = join_axis(cell_z(c), p.oz[i], fng);
    v[3 * q + 0] = p.vx[i];
    v[3 * q + 1] = p.vy[i];
    v[3 * q + 2] = p.vz[i];
}

__global__ void drift_kernel(ParticleSoA p, size_t n, int ng, float pf) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t c = p.cell[i];
    int ix = cell_x(c), iy = cell_y(c), iz = cell_z(c);
    float ox = p.ox[i], oy = p.oy[i], oz = p.oz[i];
    drift_axis(ix, ox, p.vx[i], pf, ng);
    drift_axis(iy, oy, p.vy[i], pf, ng);
    drift_axis(iz, oz, p.vz[i], pf, ng);
    p.cell[i] = pack_cell(ix, iy, iz);
    p.ox[i] = ox;
    p.oy[i] = oy;
    p.oz[i] = oz;
}

// CICKernel (cic_pm.cu:46-87) with float weights ((w_x*w_y)*w_z)*mass, each
// rounded to a 2^-31 fixed-point integer and added with integer atomics, so
// the density is independent of particle, thread and CTA order (bit-exact
// run to run).  One CTA owns one Lagrangian block of B^3 particles: it finds
// the bounding box of their cells, accumulates the block's CIC weights in a
// shared-memory window over that box, and flushes the window's non-zero cells
// to the global int64 accumulator with one coalesced red.add per cell.
// Inside the window each cell is a (hi, lo) pair of 32-bit words updated with
// native 32-bit shared atomics (win_add).  A thread walks its particles along
// Lagrangian x, so particle k's upper-x corners are merged in registers with
// particle k+1's lower-x corners whenever their cells line up (about 4
// instead of 8 shared atomics per particle).  A block whose particles spread
// over more than cap_cells cells is queued for deposit_spill_kernel (a wider
// window, one CTA per SM; wider still, per-corner global atomics).
__device__ __forceinline__ int nearest_image(int d, int ng) {
    if (d < -(ng >> 1)) d += ng;
    else if (d >= (ng >> 1)) d -= ng;
    return d;
}

// n / d for n, d < 2^16 with m = floor((2^32 - 1) / d) + 1 (exact in that range)
__device__ __forceinline__ unsigned div_magic(unsigned d) { return 0xffffffffu / d + 1u; }
__device__ __forceinline__ unsigned div_by(unsigned n, unsigned m) { return __umulhi(n, m); }

// Window cell i (z fastest, then y, then x) -> global linear cell index.
struct WinMap {
    int wy, wz, gx0, gy0, gz0, ng;
    unsigned mz, my;
    __device__ __forceinline__ WinMap(int wy_, int wz_, int gx0_, int gy0_, int gz0_, int ng_)
        : wy(wy_), wz(wz_), gx0(gx0_), gy0(gy0_), gz0(gz0_), ng(ng_) {
        mz = div_magic((unsigned)wz_);
        my = div_magic((unsigned)wy_);
    }
    // 32-bit: ng^3 <= 2^30
    __device__ __forceinline__ unsigned global(int i) const {
        const int row = (int)div_by((unsigned)i, mz);
        const int cz = i - row * wz;
        const int cx = (int)div_by((unsigned)row, my);
        const int cy = row - cx * wy;
        int gx = gx0 + cx, gy = gy0 + cy, gz = gz0 + cz;
        gx = gx >= ng ? gx - ng : (gx < 0 ? gx + ng : gx);
        gy = gy >= ng ? gy - ng : (gy < 0 ? gy + ng : gy);
        gz = gz >= ng ? gz - ng : (gz < 0 ? gz + ng : gz);
        return ((unsigned)gx * (unsigned)ng + (unsigned)gy) * (unsigned)ng + (unsigned)gz;
    }
};

// Bounding box of a Lagrangian block's cells relative to the block's
// lattice origin (o0x, o0y, o0z), plus one cell for the CIC upper corners:
// window origin (l0) and extent (w) per axis.  Every thread of the CTA calls
// it (two barriers); bb is 6 ints of shared memory.
template <int NT, int PPT>
__device__ __forceinline__ void block_window(const uint32_t* __restrict__ cell, size_t p0, int o0x, int o0y, int o0z,
                                             int ng, int* bb, int l0[3], int w[3]) {
    const int tid = threadIdx.x;
    if (tid < 3) bb[tid] = 0x7fffffff;
    else if (tid < 6) bb[tid] = -0x7fffffff;
    __syncthreads();
    int mn[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, mx[3] = {-0x7fffffff, -0x7fffffff, -0x7fffffff};
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const uint32_t c = __ldg(&cell[p0 + tid + k * NT]);
        const int rx = nearest_image(cell_x(c) - o0x, ng);
        const int ry = nearest_image(cell_y(c) - o0y, ng);
        const int rz = nearest_image(cell_z(c) - o0z, ng);
        mn[0] = min(mn[0], rx); mx[0] = max(mx[0], rx);
        mn[1] = min(mn[1], ry); mx[1] = max(mx[1], ry);
        mn[2] = min(mn[2], rz); mx[2] = max(mx[2], rz);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        mn[a] = __reduce_min_sync(0xffffffffu, mn[a]);
        mx[a] = __reduce_max_sync(0xffffffffu, mx[a]);
    }
    if ((tid & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            atomicMin(&bb[a], mn[a]);
            atomicMax(&bb[3 + a], mx[a]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        l0[a] = bb[a];
        w[a] = bb[3 + a] - bb[a] + 2;
    }
}

__device__ __forceinline__ int wrap_once(int g, int ng) { return g >= ng ? g - ng : (g < 0 ? g + ng : g); }

// Window-relative coordinate of a cell along one axis: (g - origin) mod ng
// for an origin already wrapped into [0, ng); exact for windows narrower
// than the grid.
__device__ __forceinline__ int win_rel(int g, int origin, int ng) {
    const int d = g - origin;
    return d < 0 ? d + ng : d;
}

// Per-block window record (origin l0 relative to the block's lattice corner,
// extent w), written by the deposit for the kick of the same positions.
constexpr int kWinRec = 8;
// Window cap of the float4 kick (kick_win4_kernel): 110.6 KB, two 512-thread
// CTAs per SM.  The deposit counts the blocks above it.
constexpr int kWin4Cap = 6912;

// 8 corner weights ((w_x w_y) w_z) * mass rounded to 2^-24, index (a*2+b)*2+c
// for corner (+a, +b, +c).  Q32: every value < 2^32 (mass < 256).  The x
// weights are scaled by 2^24 first: a power-of-two factor commutes with
// every rounding of the products while they stay normal, and a weight whose
// products leave the normal range (below 2^-126) rounds to 0 either way, so
// the integers are those of scaling the finished product.
template <bool Q32>
__device__ __forceinline__ void cic_q24(float dx, float dy, float dz, float mass, unsigned long long q[8]) {
    const float wx[2] = {__fmul_rn(1.f - dx, kQ24F), __fmul_rn(dx, kQ24F)}, wy[2] = {1.f - dy, dy},
                wz[2] = {1.f - dz, dz};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                float mul = __fmul_rn(__fmul_rn(wx[a], wy[b]), wz[cc]);
                if (mass != 1.f) mul = __fmul_rn(mul, mass);  // exact when mass is 1 (ng = np)
                q[(a * 2 + b) * 2 + cc] = Q32 ? (unsigned long long)__float2uint_rn(mul)
                                              : (unsigned long long)__float2ull_rn(mul);
            }
}

// The same weights on the int64 grid's 2^31 scale.  SMALL (mass <= 1): each
// value, and the sum of two (the x-chain merges an upper-x weight < 1 with a
// lower-x weight <= 1), is below 2^32.
template <bool SMALL>
__device__ __forceinline__ void cic_fixed(float dx, float dy, float dz, float mass, unsigned long long q[8]) {
    cic_q24<SMALL>(dx, dy, dz, mass, q);
#pragma unroll
    for (int j = 0; j < 8; ++j) q[j] <<= kQShift;
}

// Window cell update.  SMALL (every contribution < 2^32): the low and high
// 16-bit halves go to two u32 accumulators with return-free atomics; a CTA
// makes at most B^3*8 <= 32768 contributions to a cell, so neither half can
// overflow and hi*2^16 + lo is the exact 64-bit sum.  Otherwise: (hi, lo)
// 32-bit words with an explicit carry from the returned old value.
template <bool SMALL>
__device__ __forceinline__ void win_add(unsigned* __restrict__ w0, unsigned* __restrict__ w1, int w,
                                        unsigned long long v) {
    if (SMALL) {
        atomicAdd(&w0[w], (unsigned)v & 0xffffu);
        atomicAdd(&w1[w], (unsigned)v >> 16);
    } else {
        const unsigned lo = (unsigned)v;
        const unsigned old = atomicAdd(&w0[w], lo);
        const unsigned hi = (unsigned)(v >> 32) + ((old + lo < old) ? 1u : 0u);
        if (hi) atomicAdd(&w1[w], hi);
    }
}

template <bool SMALL>
__device__ __forceinline__ unsigned long long win_value(const unsigned* __restrict__ w0, const unsigned* __restrict__ w1,
                                                        int i) {
    return SMALL ? ((unsigned long long)w1[i] << 16) + w0[i] : ((unsigned long long)w1[i] << 32) | w0[i];
}

// NT threads; thread t owns the x-run of PPT particles at (y, z) = t % B^2,
// x in [(t / B^2) * PPT, +PPT), so its consecutive particles are x-adjacent.
template <int B, bool SMALL, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) deposit_tiled_kernel(ParticleSoA p, int np_side, int ng, float mass,
                                                                 unsigned long long* __restrict__ rho, int cap_cells,
                                                                 int* __restrict__ blkwin, SpillList spill, Slots sl) {
    constexpr int B3 = B * B * B, BB = B * B;
    constexpr int PPT = B3 / NT;
    extern __shared__ unsigned long long win[];
    __shared__ int bb[6];
    if (slot_idle(sl, blockIdx.y)) return;
    const int tid = threadIdx.x;
    const int nb = np_side / B;
    const int blk = blockIdx.x;
    // this block's particles: 32-bit indices from here on
    p = offset_soa(p, (size_t)blockIdx.y * sl.s0 + (size_t)blk * B3);
    rho += (size_t)blockIdx.y * sl.s1;
    const int bz = blk % nb, by = (blk / nb) % nb, bx = blk / (nb * nb);
    const int ox = (int)((long long)bx * B * ng / np_side);
    const int oy = (int)((long long)by * B * ng / np_side);
    const int oz = (int)((long long)bz * B * ng / np_side);
    int l0[3], w[3];
    block_window<NT, PPT>(p.cell, 0, ox, oy, oz, ng, bb, l0, w);
    if (blkwin && tid < 6) blkwin[(size_t)blockIdx.y * sl.s2 + (size_t)blk * kWinRec + tid] = tid < 3 ? l0[tid] : w[tid - 3];
    const int wx = w[0], wy = w[1], wz = w[2];
    // window origin in grid coordinates, wrapped into [0, ng)
    const int gx0 = wrap_once(ox + l0[0], ng), gy0 = wrap_once(oy + l0[1], ng), gz0 = wrap_once(oz + l0[2], ng);
    const long long vol = (long long)wx * wy * wz;
    if (tid == 0 && spill.over && vol > kWin4Cap) atomicAdd(&spill.over[blockIdx.y], 1);
    if (vol <= cap_cells) {
        unsigned* w0 = reinterpret_cast<unsigned*>(win);
        unsigned* w1 = w0 + cap_cells;
        for (int i = tid; i < vol; i += NT) {
            w0[i] = 0u;
            w1[i] = 0u;
        }
        __syncthreads();
        const int syz = wy * wz;
        const int off[4] = {0, 1, wz, wz + 1};  // (b, c) corner offsets in the window
        unsigned long long pend[4] = {0ull, 0ull, 0ull, 0ull};
        int pw = -1;  // window index of the pending (upper-x) face; -1: none
        const int i0 = (tid / BB) * PPT * BB + tid % BB;  // the thread's first particle
        // next particle's cell and offsets are loaded one iteration ahead
        uint32_t nc = __ldg(&p.cell[i0]);
        float nx = __ldg(&p.ox[i0]), ny = __ldg(&p.oy[i0]), nz = __ldg(&p.oz[i0]);
#pragma unroll 1
        for (int k = 0; k < PPT; ++k) {
            const uint32_t c = nc;
            const float cx = nx, cy = ny, cz = nz;
            if (k + 1 < PPT) {
                const int nidx = i0 + (k + 1) * BB;
                nc = __ldg(&p.cell[nidx]);
                nx = __ldg(&p.ox[nidx]);
                ny = __ldg(&p.oy[nidx]);
                nz = __ldg(&p.oz[nidx]);
            }
            unsigned long long q[8];
            cic_fixed<SMALL>(cx, cy, cz, mass, q);
            const int cw = (win_rel(cell_x(c), gx0, ng) * wy + win_rel(cell_y(c), gy0, ng)) * wz +
                           win_rel(cell_z(c), gz0, ng);
            if (pw == cw) {
#pragma unroll
                for (int j = 0; j < 4; ++j) q[j] += pend[j];
            } else if (pw >= 0) {
#pragma unroll
                for (int j = 0; j < 4; ++j) win_add<SMALL>(w0, w1, pw + off[j], pend[j]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) win_add<SMALL>(w0, w1, cw + off[j], q[j]);
#pragma unroll
            for (int j = 0; j < 4; ++j) pend[j] = q[4 + j];
            pw = cw + syz;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) win_add<SMALL>(w0, w1, pw + off[j], pend[j]);
        __syncthreads();
        const WinMap map(wy, wz, gx0, gy0, gz0, ng);
        for (int i = tid; i < vol; i += NT) {
            const unsigned long long v = win_value<SMALL>(w0, w1, i);
            if (v != 0ull) atomicAdd(&rho[map.global(i)], v);
        }
    } else if (tid == 0) {
        // too wide for the window: queued (whole) for deposit_spill_kernel
        const int slot = blockIdx.y;
        spill.items[(size_t)slot * spill.nblocks + atomicAdd(&spill.cnt[slot], 1)] = blk * 4;
    }
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// deposit_tiled_kernel with one 32-bit word per window cell: the weights are
// added as 2^-24 integers (cic_q24) with one shared atomic per corner instead
// of two 16-bit halves.  A corner adds at most mass * 2^24, so a cell can wrap
// only where the block puts 256 units of weight x mass into it (256 times the
// mean density from one block, in dense cores late in a run).  Before the
// flush the CTA compares the 64-bit sum of its window with the sum of every
// value it added; a block that wrapped is queued, like a block too wide for the
// window, for deposit_spill_kernel, whose 16-bit-split window is exact.  Needs
// mass <= 64 (two merged corners below 2^32).  CHAIN: the x-chain merge of
// deposit_tiled_kernel; otherwise each particle adds its 8 corners.
template <int B, int NT, int MINB, bool CHAIN, int PF = 1>
__global__ void __launch_bounds__(NT, MINB) deposit_w32_kernel(ParticleSoA p, int np_side, int ng, float mass,
                                                               unsigned long long* __restrict__ rho, int cap_cells,
                                                               int* __restrict__ blkwin, SpillList spill, Slots sl) {
    constexpr int B3 = B * B * B, BB = B * B;
    constexpr int PPT = B3 / NT;
    static_assert(NT % BB == 0 && B3 % NT == 0, "a thread owns one x-run of PPT particles");
    extern __shared__ unsigned long long win[];
    __shared__ int bb[6];
    __shared__ long long wsum[NT / 32];
    if (slot_idle(sl, blockIdx.y)) return;
    const int tid = threadIdx.x;
    const int nb = np_side / B;
    const int blk = blockIdx.x;
    p = offset_soa(p, (size_t)blockIdx.y * sl.s0 + (size_t)blk * B3);
    rho += (size_t)blockIdx.y * sl.s1;
    const int bz = blk % nb, by = (blk / nb) % nb, bx = blk / (nb * nb);
    const int ox = (int)((long long)bx * B * ng / np_side);
    const int oy = (int)((long long)by * B * ng / np_side);
    const int oz = (int)((long long)bz * B * ng / np_side);
    int l0[3], w[3];
    block_window<NT, PPT>(p.cell, 0, ox, oy, oz, ng, bb, l0, w);
    if (blkwin && tid < 6) blkwin[(size_t)blockIdx.y * sl.s2 + (size_t)blk * kWinRec + tid] = tid < 3 ? l0[tid] : w[tid - 3];
    const int wy = w[1], wz = w[2];
    const int gx0 = wrap_once(ox + l0[0], ng), gy0 = wrap_once(oy + l0[1], ng), gz0 = wrap_once(oz + l0[2], ng);
    const long long vol = (long long)w[0] * wy * wz;
    if (tid == 0 && spill.over && vol > kWin4Cap) atomicAdd(&spill.over[blockIdx.y], 1);
    if (vol > cap_cells) {
        if (tid == 0) spill.items[(size_t)blockIdx.y * spill.nblocks + atomicAdd(&spill.cnt[blockIdx.y], 1)] = blk * 4;
        return;
    }
    unsigned* w0 = reinterpret_cast<unsigned*>(win);
    for (int i = tid; i < vol; i += NT) w0[i] = 0u;
    __syncthreads();
    const int syz = wy * wz;
    const int off[4] = {0, 1, wz, wz + 1};  // (b, c) corner offsets in the window
    unsigned long long added = 0ull;        // every value this thread adds
    unsigned pend[4] = {0u, 0u, 0u, 0u};
    int pw = -1;  // window index of the pending (upper-x) face; -1: none
    const int i0 = (tid / BB) * PPT * BB + tid % BB;
    // the particles PF ahead are in flight in a register ring (PF = 1: the
    // next one; PF > 1 unrolls the run so the ring indices are static)
    uint32_t rc[PF];
    float rx[PF], ry[PF], rz[PF];
#pragma unroll
    for (int k = 0; k < PF; ++k) {
        if (k < PPT) {
            const int idx = i0 + k * BB;
            rc[k] = __ldg(&p.cell[idx]);
            rx[k] = __ldg(&p.ox[idx]);
            ry[k] = __ldg(&p.oy[idx]);
            rz[k] = __ldg(&p.oz[idx]);
        }
    }
#pragma unroll(PF > 1 ? PPT : 1)
    for (int k = 0; k < PPT; ++k) {
        const int r = PF > 1 ? k % PF : 0;
        const uint32_t c = rc[r];
        const float cx = rx[r], cy = ry[r], cz = rz[r];
        if (k + PF < PPT) {
            const int nidx = i0 + (k + PF) * BB;
            rc[r] = __ldg(&p.cell[nidx]);
            rx[r] = __ldg(&p.ox[nidx]);
            ry[r] = __ldg(&p.oy[nidx]);
            rz[r] = __ldg(&p.oz[nidx]);
        }
        unsigned long long q64[8];
        cic_q24<true>(cx, cy, cz, mass, q64);
        unsigned q[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            q[j] = (unsigned)q64[j];
            added += q64[j];
        }
        const int cw = (win_rel(cell_x(c), gx0, ng) * wy + win_rel(cell_y(c), gy0, ng)) * wz +
                       win_rel(cell_z(c), gz0, ng);
        if (CHAIN) {
            if (pw == cw) {
#pragma unroll
                for (int j = 0; j < 4; ++j) q[j] += pend[j];
            } else if (pw >= 0) {
#pragma unroll
                for (int j = 0; j < 4; ++j) atomicAdd(&w0[pw + off[j]], pend[j]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) atomicAdd(&w0[cw + off[j]], q[j]);
#pragma unroll
            for (int j = 0; j < 4; ++j) pend[j] = q[4 + j];
            pw = cw + syz;
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) atomicAdd(&w0[cw + (j >> 2) * syz + off[j & 3]], q[j]);
        }
    }
    if (CHAIN) {
#pragma unroll
        for (int j = 0; j < 4; ++j) atomicAdd(&w0[pw + off[j]], pend[j]);
    }
    __syncthreads();
    // wrap check: the window's 64-bit sum equals the sum of the added values
    // unless a cell wrapped (a wrap only lowers it)
    long long d = -(long long)added;
    for (int i = tid; i < vol; i += NT) d += (long long)w0[i];
    d = warp_sum_ll(d);
    if ((tid & 31) == 0) wsum[tid >> 5] = d;
    __syncthreads();
    long long tot = 0;
#pragma unroll
    for (int k = 0; k < NT / 32; ++k) tot += wsum[k];
    if (tot != 0) {
        if (tid == 0) spill.items[(size_t)blockIdx.y * spill.nblocks + atomicAdd(&spill.cnt[blockIdx.y], 1)] = blk * 4;
        return;
    }
    const WinMap map(wy, wz, gx0, gy0, gz0, ng);
    for (int i = tid; i < vol; i += NT) {
        const unsigned v = w0[i];
        if (v != 0u) atomicAdd(&rho[map.global(i)], (unsigned long long)v << kQShift);
    }
}

// Column deposit: 32-bit windows (as deposit_w32_kernel) with one thread per
// (y, z) column of the block, which walks the column's B particles along x
// with the next PF in flight in a register ring.  A block whose window is
// wider than the cap but whose two x-halves (x < B/2, x >= B/2) each fit is
// deposited as two halves, one after the other, each with its own window,
// wrap check and flush; only blocks whose halves do not fit either (or that
// wrap) go to deposit_spill_kernel.
// Adds the column range [k0, k0 + len) into the window.  RET: each atomic
// returns the cell's old value, and *wrapped records whether any old value
// had its top bit set: an add of v < 2^30 (mass <= 64) can wrap only a cell
// already at 2^32 - v > 2^31, so every wrap is caught (a cell that passes
// 2^31 without wrapping, 128 units of weight x mass from one block, is sent
// to the exact pass too); otherwise the sum of the added values is returned
// for the caller's window-sum check.
// CHAIN: a particle's 4 upper-x corners are held in registers and merged
// into the next particle's lower-x corners when its cell is the next in x (the
// column walks Lagrangian x), saving 4 shared atomics; merged values stay
// below 2^31 (mass <= 64), so the wrap argument above holds.
template <int B, int PF, bool RET, bool CHAIN = false>
__device__ __forceinline__ unsigned long long column_adds(const ParticleSoA& p, int i0, int k0, int len, float mass,
                                                          unsigned* __restrict__ w0, int gx0, int gy0, int gz0,
                                                          int wy, int wz, int ng, bool* wrapped) {
    constexpr int BB = B * B;
    const int syz = wy * wz;
    unsigned long long added = 0ull;
    unsigned acc = 0u;  // OR of the returned old values (RET)
    unsigned pend[4] = {0u, 0u, 0u, 0u};  // CHAIN: pending upper-x corners at window cell pw
    int pw = -1;
    auto add = [&](int w, unsigned v) {
        if (RET) acc |= atomicAdd(&w0[w], v);
        else atomicAdd(&w0[w], v);
    };
    uint32_t rc[PF];
    float rx[PF], ry[PF], rz[PF];
#pragma unroll
    for (int j = 0; j < PF; ++j) {
        if (j < len) {
            const int idx = i0 + (k0 + j) * BB;
            rc[j] = __ldg(&p.cell[idx]);
            rx[j] = __ldg(&p.ox[idx]);
            ry[j] = __ldg(&p.oy[idx]);
            rz[j] = __ldg(&p.oz[idx]);
        }
    }
#pragma unroll
    for (int j = 0; j < B; ++j) {
        if (j < len) {
            const int r = j % PF;
            const uint32_t c = rc[r];
            const float cx = rx[r], cy = ry[r], cz = rz[r];
            if (j + PF < len) {
                const int idx = i0 + (k0 + j + PF) * BB;
                rc[r] = __ldg(&p.cell[idx]);
                rx[r] = __ldg(&p.ox[idx]);
                ry[r] = __ldg(&p.oy[idx]);
                rz[r] = __ldg(&p.oz[idx]);
            }
            unsigned long long q[8];
            cic_q24<true>(cx, cy, cz, mass, q);
            const int cw = (win_rel(cell_x(c), gx0, ng) * wy + win_rel(cell_y(c), gy0, ng)) * wz +
                           win_rel(cell_z(c), gz0, ng);
            unsigned v[8];
#pragma unroll
            for (int m = 0; m < 8; ++m) v[m] = (unsigned)q[m];
            if (!RET) {
                // a particle's 8 values sum to about mass * 2^24 (< 2^31 for mass <= 64)
                unsigned psum = 0u;
#pragma unroll
                for (int m = 0; m < 8; ++m) psum += v[m];
                added += psum;
            }
            if (CHAIN) {
                if (cw == pw) {
#pragma unroll
                    for (int m = 0; m < 4; ++m) v[m] += pend[m];
                } else if (pw >= 0) {
#pragma unroll
                    for (int b = 0; b < 2; ++b)
#pragma unroll
                        for (int cc = 0; cc < 2; ++cc) add(pw + b * wz + cc, pend[b * 2 + cc]);
                }
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int cc = 0; cc < 2; ++cc) add(cw + b * wz + cc, v[b * 2 + cc]);
#pragma unroll
                for (int m = 0; m < 4; ++m) pend[m] = v[4 + m];
                pw = cw + syz;
            } else {
#pragma unroll
                for (int a = 0; a < 2; ++a)
#pragma unroll
                    for (int b = 0; b < 2; ++b)
#pragma unroll
                        for (int cc = 0; cc < 2; ++cc) add(cw + a * syz + b * wz + cc, v[(a * 2 + b) * 2 + cc]);
            }
        }
    }
    if (CHAIN && pw >= 0) {
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) add(pw + b * wz + cc, pend[b * 2 + cc]);
    }
    if (RET) *wrapped = (acc >> 31) != 0u;
    return added;
}

// Zero the window, add the column range [k0, k0 + len), check for wraps and
// flush; returns false (nothing left in the grid) if a cell wrapped.  Called
// by every thread of the CTA.  CHK, how a wrap is found:
//   0  before the flush, the window's 64-bit sum against the sum of the
//      values added (a wrapped cell changes it by a multiple of 2^32);
//   1  from the atomics' returned values (column_adds with RET);
//   2  the same two sums, the window's taken while flushing; a wrapped window
//      (in practice never at the workloads' densities) is taken back out of
//      the grid by adding the negated values, so the grid's integers are
//      those of the other checks.
template <int B, int PF, int CHK, bool CHAIN = false>
__device__ __forceinline__ bool column_pass(const ParticleSoA& p, int i0, int k0, int len, float mass,
                                            unsigned* __restrict__ w0, long long* wsum, const int* box, int ox,
                                            int oy, int oz, int ng, unsigned long long* __restrict__ rho) {
    constexpr int NT = B * B;
    constexpr bool RET = CHK == 1;
    const int tid = threadIdx.x;
    const int wx = box[3] - box[0] + 2, wy = box[4] - box[1] + 2, wz = box[5] - box[2] + 2;
    const int gx0 = wrap_once(ox + box[0], ng), gy0 = wrap_once(oy + box[1], ng), gz0 = wrap_once(oz + box[2], ng);
    const int vol = wx * wy * wz;
    for (int i = tid; i < vol; i += NT) w0[i] = 0u;
    __syncthreads();
    bool wrapped = false;
    const unsigned long long added =
        column_adds<B, PF, RET, CHAIN>(p, i0, k0, len, mass, w0, gx0, gy0, gz0, wy, wz, ng, &wrapped);
    long long tot = 0;
    if (CHK == 2) {
        __syncthreads();
        const WinMap map(wy, wz, gx0, gy0, gz0, ng);
        long long d = -(long long)added;
        for (int i = tid; i < vol; i += NT) {
            const unsigned v = w0[i];
            if (v != 0u) {
                d += v;
                atomicAdd(&rho[map.global(i)], (unsigned long long)v << kQShift);
            }
        }
        d = warp_sum_ll(d);
        if ((tid & 31) == 0) wsum[tid >> 5] = d;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < NT / 32; ++k) tot += wsum[k];
        if (tot != 0) {
            for (int i = tid; i < vol; i += NT) {
                const unsigned v = w0[i];
                if (v != 0u) atomicAdd(&rho[map.global(i)], 0ull - ((unsigned long long)v << kQShift));
            }
        }
        __syncthreads();  // the window and wsum are reused by the next pass
        return tot == 0;
    }
    if (RET) {
        tot = __syncthreads_or(wrapped) ? 1 : 0;
    } else {
        __syncthreads();
        long long d = -(long long)added;
        for (int i = tid; i < vol; i += NT) d += (long long)w0[i];
        d = warp_sum_ll(d);
        if ((tid & 31) == 0) wsum[tid >> 5] = d;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < NT / 32; ++k) tot += wsum[k];
    }
    if (tot == 0) {
        const WinMap map(wy, wz, gx0, gy0, gz0, ng);
        for (int i = tid; i < vol; i += NT) {
            const unsigned v = w0[i];
            if (v != 0u) atomicAdd(&rho[map.global(i)], (unsigned long long)v << kQShift);
        }
    }
    __syncthreads();  // the window is reused by the next pass
    return tot == 0;
}

// Block blk of one box: p, rho, recs (window records, may be null), the
// box's spill queue (items, cnt) and wide-window counter (over, may be
// null).  The single-class kernel below and the multi-class deposit run it.
template <int B, int PF, int CHK, bool CHAIN = false>
__device__ __forceinline__ void deposit_col_body(ParticleSoA p, int np_side, int ng, float mass,
                                                 unsigned long long* __restrict__ rho, int cap_cells,
                                                 int* __restrict__ recs, int* __restrict__ items, int* cnt,
                                                 int* over, int blk) {
    constexpr int B3 = B * B * B, NT = B * B;
    extern __shared__ unsigned long long win[];
    __shared__ int bb[18];  // (min xyz, max xyz) of the block, then of each x-half
    __shared__ long long wsum[NT / 32];
    const int tid = threadIdx.x;
    const int nb = np_side / B;
    p = offset_soa(p, (size_t)blk * B3);
    const int bz = blk % nb, by = (blk / nb) % nb, bx = blk / (nb * nb);
    const int ox = (int)((long long)bx * B * ng / np_side);
    const int oy = (int)((long long)by * B * ng / np_side);
    const int oz = (int)((long long)bz * B * ng / np_side);
    if (tid < 18) bb[tid] = (tid % 6) < 3 ? 0x7fffffff : -0x7fffffff;
    __syncthreads();
    {
        // bounding boxes of the two x-halves of the thread's column
        int mn[2][3], mx[2][3];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                mn[h][a] = 0x7fffffff;
                mx[h][a] = -0x7fffffff;
            }
#pragma unroll
        for (int k = 0; k < B; ++k) {
            const int h = k >= B / 2;
            const uint32_t c = __ldg(&p.cell[tid + k * NT]);
            const int r[3] = {nearest_image(cell_x(c) - ox, ng), nearest_image(cell_y(c) - oy, ng),
                              nearest_image(cell_z(c) - oz, ng)};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                mn[h][a] = min(mn[h][a], r[a]);
                mx[h][a] = max(mx[h][a], r[a]);
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                mn[h][a] = __reduce_min_sync(0xffffffffu, mn[h][a]);
                mx[h][a] = __reduce_max_sync(0xffffffffu, mx[h][a]);
            }
        if ((tid & 31) == 0) {
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    atomicMin(&bb[6 + 6 * h + a], mn[h][a]);
                    atomicMax(&bb[9 + 6 * h + a], mx[h][a]);
                    atomicMin(&bb[a], mn[h][a]);
                    atomicMax(&bb[3 + a], mx[h][a]);
                }
        }
    }
    __syncthreads();
    const int wx = bb[3] - bb[0] + 2, wy = bb[4] - bb[1] + 2, wz = bb[5] - bb[2] + 2;
    if (recs && tid < 6) {
        const int rec = tid < 3 ? bb[tid] : bb[tid] - bb[tid - 3] + 2;
        recs[(size_t)blk * kWinRec + tid] = rec;
    }
    const long long vol = (long long)wx * wy * wz;
    if (tid == 0 && over && vol > kWin4Cap) atomicAdd(over, 1);
    unsigned* w0 = reinterpret_cast<unsigned*>(win);
    // queued part: 0 the whole block, 2 its upper x-half (the lower half
    // flushed); at most one item per block
    int queue = -1;
    if (vol <= cap_cells) {
        if (!column_pass<B, PF, CHK, CHAIN>(p, tid, 0, B, mass, w0, wsum, bb, ox, oy, oz, ng, rho)) queue = 0;
    } else {
        auto hvol = [&](int h) {
            const int* q = bb + 6 + 6 * h;
            return (long long)(q[3] - q[0] + 2) * (q[4] - q[1] + 2) * (q[5] - q[2] + 2);
        };
        if (hvol(0) <= cap_cells && hvol(1) <= cap_cells) {
            if (!column_pass<B, PF, CHK, CHAIN>(p, tid, 0, B / 2, mass, w0, wsum, bb + 6, ox, oy, oz, ng, rho)) queue = 0;
            else if (!column_pass<B, PF, CHK, CHAIN>(p, tid, B / 2, B / 2, mass, w0, wsum, bb + 12, ox, oy, oz, ng, rho))
                queue = 2;
        } else {
            queue = 0;
        }
    }
    if (queue >= 0 && tid == 0) items[atomicAdd(cnt, 1)] = blk * 4 + queue;
}

template <int B, int MINB, int PF, int CHK = 0, bool CHAIN = false>
__global__ void __launch_bounds__(B * B, MINB) deposit_col_kernel(ParticleSoA p, int np_side, int ng, float mass,
                                                                  unsigned long long* __restrict__ rho, int cap_cells,
                                                                  int* __restrict__ blkwin, SpillList spill, Slots sl) {
    const int slot = blockIdx.y;
    if (slot_idle(sl, slot)) return;
    deposit_col_body<B, PF, CHK, CHAIN>(offset_soa(p, (size_t)slot * sl.s0), np_side, ng, mass, rho + (size_t)slot * sl.s1,
                                 cap_cells, blkwin ? blkwin + (size_t)slot * sl.s2 : nullptr,
                                 spill.items + (size_t)slot * spill.nblocks, spill.cnt + slot,
                                 spill.over ? spill.over + slot : nullptr, blockIdx.x);
}

// The 8 fixed-point corner weights of one particle added straight to the
// int64 grid (blocks too wide for a shared-memory window).
template <bool SMALL>
__device__ __forceinline__ void deposit_global(unsigned long long* __restrict__ rho, uint32_t c, float dx, float dy,
                                               float dz, float mass, int ng) {
    unsigned long long q[8];
    cic_fixed<SMALL>(dx, dy, dz, mass, q);
    const int ix = cell_x(c), iy = cell_y(c), iz = cell_z(c);
    const int ix1 = ix + 1 == ng ? 0 : ix + 1;
    const int iy1 = iy + 1 == ng ? 0 : iy + 1;
    const int iz1 = iz + 1 == ng ? 0 : iz + 1;
    const size_t sx[2] = {(size_t)ix * ng * ng, (size_t)ix1 * ng * ng};
    const size_t sy[2] = {(size_t)iy * ng, (size_t)iy1 * ng};
    const size_t sz[2] = {(size_t)iz, (size_t)iz1};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) atomicAdd(&rho[sx[a] + sy[b] + sz[cc]], q[(a * 2 + b) * 2 + cc]);
}

// Direct deposit: one CTA per Lagrangian block records the block's window
// (for the windowed kick, as the windowed deposits do), then every particle
// adds its 8 fixed-point weights straight to the int64 grid.  Where a window
// would hold about one contribution per cell (more cells than particles per
// axis: each particle's corners are mostly its own) this skips the window's
// zeroing and flush; the sums are the same integers (bit-identical grids).
template <int B, bool SMALL, int NT>
__global__ void __launch_bounds__(NT) deposit_direct_kernel(ParticleSoA p, int np_side, int ng, float mass,
                                                            unsigned long long* __restrict__ rho, int cap_cells,
                                                            int* __restrict__ blkwin, SpillList spill, Slots sl) {
    constexpr int B3 = B * B * B;
    constexpr int PPT = B3 / NT;
    static_assert(B3 % NT == 0, "whole particles per thread");
    (void)cap_cells;
    __shared__ int bb[6];
    if (slot_idle(sl, blockIdx.y)) return;
    const int tid = threadIdx.x;
    const int nb = np_side / B;
    const int blk = blockIdx.x;
    p = offset_soa(p, (size_t)blockIdx.y * sl.s0 + (size_t)blk * B3);
    rho += (size_t)blockIdx.y * sl.s1;
    const int bz = blk % nb, by = (blk / nb) % nb, bx = blk / (nb * nb);
    const int ox = (int)((long long)bx * B * ng / np_side);
    const int oy = (int)((long long)by * B * ng / np_side);
    const int oz = (int)((long long)bz * B * ng / np_side);
    int l0[3], w[3];
    block_window<NT, PPT>(p.cell, 0, ox, oy, oz, ng, bb, l0, w);
    if (blkwin && tid < 6) blkwin[(size_t)blockIdx.y * sl.s2 + (size_t)blk * kWinRec + tid] = tid < 3 ? l0[tid] : w[tid - 3];
    if (tid == 0 && spill.over && (long long)w[0] * w[1] * w[2] > kWin4Cap) atomicAdd(&spill.over[blockIdx.y], 1);
#pragma unroll 2
    for (int k = 0; k < PPT; ++k) {
        const int i = tid + k * NT;
        deposit_global<SMALL>(rho, __ldg(&p.cell[i]), __ldg(&p.ox[i]), __ldg(&p.oy[i]), __ldg(&p.oz[i]), mass, ng);
    }
}

// Blocks queued by deposit_tiled_kernel (window wider than its own): a
// persistent grid of one CTA per SM with a kBigCap-cell window (216 KB) takes
// them from the queue one at a time.  A thread walks PPT x-adjacent particles
// (the x-chain of deposit_tiled_kernel).  Windows wider still add straight to
// the global grid.
constexpr int kBigCap = 27648;

// The queue of one box (p, rho, recs, items: that box's; cnt items), items
// cta, cta + ncta, ...  Run by the single-class kernel below and by the
// multi-class spill pass.
template <int B, bool SMALL, int NT>
__device__ __forceinline__ void deposit_spill_body(ParticleSoA p, int np_side, int ng, float mass,
                                                   unsigned long long* __restrict__ rho,
                                                   const int* __restrict__ recs, const int* __restrict__ items,
                                                   int cnt, int cta, int ncta) {
    constexpr int B3 = B * B * B, PPT = B3 / NT, BB = B * B;
    extern __shared__ unsigned long long win[];
    unsigned* w0 = reinterpret_cast<unsigned*>(win);
    unsigned* w1 = w0 + kBigCap;
    const int tid = threadIdx.x;
    const int g = tid / BB, r = tid % BB;  // x group and (y, z) of the thread's chain
    const int nb = np_side / B;
    for (int t = cta; t < cnt; t += ncta) {
        // item = block * 4 + part: 0 the whole block, 2 its upper x-half only
        const int item = __ldg(&items[t]);
        const int blk = item >> 2;
        const int xlo = (item & 3) == 2 ? B / 2 : 0;
        const int* rec = recs + (size_t)blk * kWinRec;
        const int wx = __ldg(&rec[3]), wy = __ldg(&rec[4]), wz = __ldg(&rec[5]);
        const int bz = blk % nb, by = (blk / nb) % nb, bx = blk / (nb * nb);
        const int gx0 = wrap_once((int)((long long)bx * B * ng / np_side) + __ldg(&rec[0]), ng);
        const int gy0 = wrap_once((int)((long long)by * B * ng / np_side) + __ldg(&rec[1]), ng);
        const int gz0 = wrap_once((int)((long long)bz * B * ng / np_side) + __ldg(&rec[2]), ng);
        const long long vol = (long long)wx * wy * wz;
        const ParticleSoA pb = offset_soa(p, (size_t)blk * B3);
        if (vol <= kBigCap) {
            for (int i = tid; i < vol; i += NT) {
                w0[i] = 0u;
                w1[i] = 0u;
            }
            __syncthreads();
            const int syz = wy * wz;
            const int off[4] = {0, 1, wz, wz + 1};
            unsigned long long pend[4] = {0ull, 0ull, 0ull, 0ull};
            int pw = -1;
#pragma unroll
            for (int k = 0; k < PPT; ++k) {
                const int i = (g * PPT + k) * BB + r;
                const uint32_t c = __ldg(&pb.cell[i]);
                unsigned long long q[8];
                cic_fixed<SMALL>(__ldg(&pb.ox[i]), __ldg(&pb.oy[i]), __ldg(&pb.oz[i]), mass, q);
                if (g * PPT + k < xlo) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) q[j] = 0ull;  // outside the queued part
                }
                const int cw = (win_rel(cell_x(c), gx0, ng) * wy + win_rel(cell_y(c), gy0, ng)) * wz +
                               win_rel(cell_z(c), gz0, ng);
                if (pw == cw) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) q[j] += pend[j];
                } else if (pw >= 0) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) win_add<SMALL>(w0, w1, pw + off[j], pend[j]);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) win_add<SMALL>(w0, w1, cw + off[j], q[j]);
#pragma unroll
                for (int j = 0; j < 4; ++j) pend[j] = q[4 + j];
                pw = cw + syz;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) win_add<SMALL>(w0, w1, pw + off[j], pend[j]);
            __syncthreads();
            const WinMap map(wy, wz, gx0, gy0, gz0, ng);
            for (int i = tid; i < vol; i += NT) {
                const unsigned long long v = win_value<SMALL>(w0, w1, i);
                if (v != 0ull) atomicAdd(&rho[map.global(i)], v);
            }
            __syncthreads();
        } else {
#pragma unroll
            for (int k = 0; k < PPT; ++k) {
                const int i = (g * PPT + k) * BB + r;
                if (g * PPT + k >= xlo)
                    deposit_global<SMALL>(rho, __ldg(&pb.cell[i]), __ldg(&pb.ox[i]), __ldg(&pb.oy[i]),
                                          __ldg(&pb.oz[i]), mass, ng);
            }
        }
    }
}

template <int B, bool SMALL, int NT>
__global__ void __launch_bounds__(NT, 1) deposit_spill_kernel(ParticleSoA p, int np_side, int ng, float mass,
                                                              unsigned long long* __restrict__ rho,
                                                              const int* __restrict__ blkwin, SpillList spill,
                                                              Slots sl) {
    const int slot = blockIdx.y;
    if (slot_idle(sl, slot)) return;
    const int cnt = __ldg(&spill.cnt[slot]);
    if ((int)blockIdx.x >= cnt) return;
    deposit_spill_body<B, SMALL, NT>(offset_soa(p, (size_t)slot * sl.s0), np_side, ng, mass,
                                     rho + (size_t)slot * sl.s1, blkwin + (size_t)slot * sl.s2,
                                     spill.items + (size_t)slot * spill.nblocks, cnt, blockIdx.x, gridDim.x);
}

// ICICKernel (icic_pm.cu:72-127) fused with up to two UpdatePosKernel drifts
// (update_positions_pm.cu:3-20): v += sum_8 float(w*deltaT*fscal) F[corner],
// then x += v*pf_a (, then x += v*pf_b).  The force grid is float4
// (F_x, F_y, F_z, 0) per cell, so a corner is one 16-byte load.
struct PState {
    uint32_t c;
    float dx, dy, dz, vx, vy, vz;
};

__device__ __forceinline__ PState load_p(const ParticleSoA& p, size_t i) {
    return PState{p.cell[i], p.ox[i], p.oy[i], p.oz[i], p.vx[i], p.vy[i], p.vz[i]};
}

__device__ __forceinline__ void finish_p(ParticleSoA& p, size_t i, const PState& s, float3 dv, float pf_a, float pf_b,
                                         int ndrift, int ng) {
    const float vx = s.vx + dv.x, vy = s.vy + dv.y, vz = s.vz + dv.z;
    p.vx[i] = vx;
    p.vy[i] = vy;
    p.vz[i] = vz;
    if (ndrift > 0) {
        int ix = cell_x(s.c), iy = cell_y(s.c), iz = cell_z(s.c);
        float ox = s.dx, oy = s.dy, oz = s.dz;
        drift_axis(ix, ox, vx, pf_a, ng);
        drift_axis(iy, oy, vy, pf_a, ng);
        drift_axis(iz, oz, vz, pf_a, ng);
        if (ndrift > 1) {
            drift_axis(ix, ox, vx, pf_b, ng);
            drift_axis(iy, oy, vy, pf_b, ng);
            drift_axis(iz, oz, vz, pf_b, ng);
        }
        p.cell[i] = pack_cell(ix, iy, iz);
        p.ox[i] = ox;
        p.oy[i] = oy;
        p.oz[i] = oz;
    }
}

// The 8 CIC weights of a particle, the kick factor deltaT*fscal folded into
// the x weight (FP32; the reference forms float(w*deltaT*fscal) in double, a
// <= 1 ulp difference), in the reference's ((w_x w_y) w_z) order.
struct KickWeights {
    float wx[2], wy[2], wz[2];
    __device__ __forceinline__ KickWeights(const PState& c, float dtf) {
        wx[0] = (1.f - c.dx) * dtf;
        wx[1] = c.dx * dtf;
        wy[0] = 1.f - c.dy;
        wy[1] = c.dy;
        wz[0] = 1.f - c.dz;
        wz[1] = c.dz;
    }
};

// Fill a float4 window of wx*wy*wz cells whose origin (gx0, gy0, gz0) is
// wrapped into [0, ng), row by row: a warp takes an (x, y) row, lanes walk z,
// RU rows in flight per warp, the row start formed once.
template <int NT, int RU>
__device__ __forceinline__ void fill_win4(float4* __restrict__ win4, const float4* __restrict__ f, int wx, int wy,
                                          int wz, int gx0, int gy0, int gz0, int ng) {
    constexpr int NW = NT / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nrows = wx * wy;
    const unsigned my = div_magic((unsigned)wy);
    for (int z0 = 0; z0 < wz; z0 += 32) {
        const int z = z0 + lane;
        const int gz = wrap_once(gz0 + z, ng);
        for (int r0 = warp; r0 < nrows; r0 += RU * NW) {
            float4 v[RU];
#pragma unroll
            for (int u = 0; u < RU; ++u) {
                const int r = r0 + u * NW;
                if (r < nrows && z < wz) {
                    const int cx = (int)div_by((unsigned)r, my), cy = r - cx * wy;
                    v[u] = __ldg(&f[((size_t)wrap_once(gx0 + cx, ng) * ng + wrap_once(gy0 + cy, ng)) * ng + gz]);
                }
            }
#pragma unroll
            for (int u = 0; u < RU; ++u) {
                const int r = r0 + u * NW;
                if (r < nrows && z < wz) win4[r * wz + z] = v[u];
            }
        }
    }
}

__device__ __forceinline__ float3 gather_win4(const float4* __restrict__ win4, int j0, int syz, int wz,
                                              const KickWeights& w) {
    float3 dv = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const float wab = __fmul_rn(w.wx[a], w.wy[b]);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const float4 f = win4[j0 + a * syz + b * wz + cc];
                const float mul = __fmul_rn(wab, w.wz[cc]);
                dv.x = fmaf(mul, f.x, dv.x);
                dv.y = fmaf(mul, f.y, dv.y);
                dv.z = fmaf(mul, f.z, dv.z);
            }
        }
    return dv;
}

__device__ __forceinline__ float3 gather_global(const float4* __restrict__ f, const PState& c, const KickWeights& w,
                                                int ng) {
    const int ix = cell_x(c.c), iy = cell_y(c.c), iz = cell_z(c.c);
    const int ix1 = ix + 1 == ng ? 0 : ix + 1;
    const int iy1 = iy + 1 == ng ? 0 : iy + 1;
    const int iz1 = iz + 1 == ng ? 0 : iz + 1;
    const size_t sx[2] = {(size_t)ix * ng * ng, (size_t)ix1 * ng * ng};
    const size_t sy[2] = {(size_t)iy * ng, (size_t)iy1 * ng};
    const size_t sz[2] = {(size_t)iz, (size_t)iz1};
    float4 g[8];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) g[(a * 2 + b) * 2 + cc] = __ldg(&f[sx[a] + sy[b] + sz[cc]]);
    float3 dv = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const float wab = __fmul_rn(w.wx[a], w.wy[b]);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const float4 v = g[(a * 2 + b) * 2 + cc];
                const float mul = __fmul_rn(wab, w.wz[cc]);
                dv.x = fmaf(mul, v.x, dv.x);
                dv.y = fmaf(mul, v.y, dv.y);
                dv.z = fmaf(mul, v.z, dv.z);
            }
        }
    return dv;
}

// Per-slot kick scalars: the launch's own, or the slot's row of a batched
// step's schedule.
__device__ __forceinline__ void kick_scalars(const KickSched& ks, int slot, double deltaT, double fscal, float& dtf,
                                             float& pf_a, float& pf_b, int& ndrift) {
    dtf = (float)(deltaT * fscal);
    if (ks.sched) {
        const float4 q = ks.sched[(size_t)slot * ks.pitch + ks.step[slot]];
        dtf = q.x;
        pf_a = q.y;
        pf_b = q.z;
        ndrift = (int)q.w;
    }
}

// The whole box goes through kick_spill_kernel: forced (variant 1), or most
// blocks' windows exceed kWin4Cap (counted by the deposit of these positions).
__device__ __forceinline__ bool kick_flat_mode(int force_flat, int have_rec, const SpillList& spill, int slot) {
    return force_flat || (have_rec && spill.over && spill.over[slot] * 2 > spill.nblocks);
}

// Windowed kick: persistent CTAs take Lagrangian blocks from a per-slot
// counter; the block's force window (from the deposit's record when the
// positions are the ones it deposited, else measured here and recorded) is
// staged as float4, so each corner is one 16-byte shared load; the kick and
// both drifts stay in registers.  Blocks whose window exceeds kWin4Cap cells
// are queued for kick_spill_kernel.
template <int B, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) kick_win4_kernel(ParticleSoA p, int np_side, int ng,
                                                                  const float4* __restrict__ f, double deltaT,
                                                                  double fscal, float pf_a, float pf_b, int ndrift,
                                                                  int* __restrict__ blkwin, int have_rec,
                                                                  int force_flat, SpillList spill, Slots sl,
                                                                  KickSched ks) {
    constexpr int B3 = B * B * B, PPT = B3 / NT;
    extern __shared__ float4 win4[];
    __shared__ int bb[6];
    __shared__ int next_blk;
    const int slot = blockIdx.y;
    if (slot_idle(sl, slot) || kick_flat_mode(force_flat, have_rec, spill, slot)) return;
    p = offset_soa(p, (size_t)slot * sl.s0);
    f += (size_t)slot * sl.s1;
    float dtf;
    kick_scalars(ks, slot, deltaT, fscal, dtf, pf_a, pf_b, ndrift);
    const int tid = threadIdx.x;
    const int nb = np_side / B;
    for (;;) {
        if (tid == 0) next_blk = atomicAdd(&spill.next[slot], 1);
        __syncthreads();
        const int blk = next_blk;
        __syncthreads();  // everyone has read next_blk before thread 0 takes another
        if (blk >= nb * nb * nb) break;
        const int bz = blk % nb, by = (blk / nb) % nb, bx = blk / (nb * nb);
        const int ox0 = (int)((long long)bx * B * ng / np_side);
        const int oy0 = (int)((long long)by * B * ng / np_side);
        const int oz0 = (int)((long long)bz * B * ng / np_side);
        const size_t p0 = (size_t)blk * B3;
        int* rec = blkwin + (size_t)slot * sl.s2 + (size_t)blk * kWinRec;
        int l0[3], w[3];
        if (have_rec) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                l0[a] = rec[a];
                w[a] = rec[3 + a];
            }
        } else {
            block_window<NT, PPT>(p.cell, p0, ox0, oy0, oz0, ng, bb, l0, w);
            if (tid < 6) rec[tid] = tid < 3 ? l0[tid] : w[tid - 3];
        }
        const int wy = w[1], wz = w[2];
        if (w[0] * wy * wz > kWin4Cap) {
            if (tid == 0) spill.items[(size_t)slot * spill.nblocks + atomicAdd(&spill.cnt[slot], 1)] = blk;
            continue;
        }
        const int gx0 = wrap_once(ox0 + l0[0], ng), gy0 = wrap_once(oy0 + l0[1], ng);
        const int gz0 = wrap_once(oz0 + l0[2], ng);
        fill_win4<NT, 4>(win4, f, w[0], wy, wz, gx0, gy0, gz0, ng);
        __syncthreads();
        const int syz = wy * wz;
        PState n1 = load_p(p, p0 + tid);
        PState n2 = PPT > 1 ? load_p(p, p0 + tid + NT) : n1;
#pragma unroll 1
        for (int k = 0; k < PPT; ++k) {
            const size_t i = p0 + tid + k * NT;
            const PState cur = n1;
            n1 = n2;
            if (k + 2 < PPT) n2 = load_p(p, i + 2 * NT);
            const int j0 = (win_rel(cell_x(cur.c), gx0, ng) * wy + win_rel(cell_y(cur.c), gy0, ng)) * wz +
                           win_rel(cell_z(cur.c), gz0, ng);
            finish_p(p, i, cur, gather_win4(win4, j0, syz, wz, KickWeights(cur, dtf)), pf_a, pf_b, ndrift, ng);
        }
        __syncthreads();  // the window is refilled for the next block
    }
}

// Queued blocks (or, in flat mode, every block), one particle per thread over
// a persistent grid that walks (block, 256-particle part) work items; the
// corners are gathered from the global float4 force grid.  (A larger shared
// window per block, one CTA per SM, was slower here: late in a run the
// bounding boxes are mostly empty cells, so filling them costs more than the
// gathers.)
template <int B>
__global__ void __launch_bounds__(256) kick_spill_kernel(ParticleSoA p, int ng, const float4* __restrict__ f,
                                                         double deltaT, double fscal, float pf_a, float pf_b,
                                                         int ndrift, int have_rec, int force_flat, SpillList spill,
                                                         Slots sl, KickSched ks) {
    constexpr int B3 = B * B * B, SUB = B3 / 256;
    const int slot = blockIdx.y;
    if (slot_idle(sl, slot)) return;
    const bool all = kick_flat_mode(force_flat, have_rec, spill, slot);
    const int n = (all ? spill.nblocks : __ldg(&spill.cnt[slot])) * SUB;
    if ((int)blockIdx.x >= n) return;
    p = offset_soa(p, (size_t)slot * sl.s0);
    f += (size_t)slot * sl.s1;
    float dtf;
    kick_scalars(ks, slot, deltaT, fscal, dtf, pf_a, pf_b, ndrift);
    const int* items = spill.items + (size_t)slot * spill.nblocks;
    auto index = [&](int w) {
        const int blk = all ? w / SUB : __ldg(&items[w / SUB]);
        return (size_t)blk * B3 + (w % SUB) * 256 + threadIdx.x;
    };
    // the next item's particle is loaded while this one's corners are gathered
    size_t inext = index(blockIdx.x);
    PState next = load_p(p, inext);
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const size_t i = inext;
        const PState cur = next;
        if (w + (int)gridDim.x < n) {
            inext = index(w + gridDim.x);
            next = load_p(p, inext);
        }
        finish_p(p, i, cur, gather_global(f, cur, KickWeights(cur, dtf), ng), pf_a, pf_b, ndrift, ng);
    }
}

// Flat kick over every block with NT threads per CTA: a unit is NT / B^2
// consecutive Lagrangian x-planes of a block, so the force-grid planes that
// neighbouring x-planes share are gathered by warps of the same SM and meet
// in its L1 (kick_spill_kernel's 256-thread items put neighbouring planes on
// different SMs); a CTA takes runs of R consecutive units, the next particle
// always loaded one unit ahead.  Arithmetic as kick_spill_kernel, bit for
// bit.
template <int B, int NT, int R = 1>
__global__ void __launch_bounds__(NT, 1024 / NT) kick_flat_nt_kernel(ParticleSoA p, int ng, const float4* __restrict__ f,
                                                                   double deltaT, double fscal, float pf_a, float pf_b,
                                                                   int ndrift, int nblocks, Slots sl, KickSched ks) {
    constexpr int B3 = B * B * B, SUB = B3 / NT;
    const int slot = blockIdx.y;
    if (slot_idle(sl, slot)) return;
    const int n = nblocks * SUB;  // units of NT particles; a CTA takes runs of R consecutive units
    if ((int)blockIdx.x * R >= n) return;
    p = offset_soa(p, (size_t)slot * sl.s0);
    f += (size_t)slot * sl.s1;
    float dtf;
    kick_scalars(ks, slot, deltaT, fscal, dtf, pf_a, pf_b, ndrift);
    auto index = [&](int u) { return (size_t)(u / SUB) * B3 + (u % SUB) * NT + threadIdx.x; };
    auto unit = [&](int k) { return ((int)blockIdx.x + (k / R) * (int)gridDim.x) * R + k % R; };
    int k = 0;
    size_t inext = index(unit(0));
    PState next = load_p(p, inext);
    for (;;) {
        const size_t i = inext;
        const PState cur = next;
        const int un = unit(k + 1);
        const bool more = un < n;
        if (more) {
            inext = index(un);
            next = load_p(p, inext);
        }
        finish_p(p, i, cur, gather_global(f, cur, KickWeights(cur, dtf), ng), pf_a, pf_b, ndrift, ng);
        if (!more) break;
        ++k;
    }
}

// v += sum over the 8 CIC corners of w * F, each corner's force formed from
// the gathered potential: P[a][b][t] = phi(x_a, y_b, z_{t-1}) on the inner
// columns, X[e][b][cc] and Y[a][e][cc] the x and y faces (e = 0: x-1 / y-1,
// e = 1: x+2 / y+2); F_d = 0.5f * (phi(-e_d) - phi(+e_d)) as gradient_kernel
// forms it.
__device__ __forceinline__ float3 phi_corner_kick(const float (&P)[2][2][4], const float (&X)[2][2][2],
                                                  const float (&Y)[2][2][2], const KickWeights& w) {
    float3 dv = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const float wab = __fmul_rn(w.wx[a], w.wy[b]);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const float lo_x = a == 0 ? X[0][b][cc] : P[0][b][1 + cc];
                const float hi_x = a == 0 ? P[1][b][1 + cc] : X[1][b][cc];
                const float lo_y = b == 0 ? Y[a][0][cc] : P[a][0][1 + cc];
                const float hi_y = b == 0 ? P[a][1][1 + cc] : Y[a][1][cc];
                const float fx = 0.5f * (lo_x - hi_x);
                const float fy = 0.5f * (lo_y - hi_y);
                const float fz = 0.5f * (P[a][b][cc] - P[a][b][cc + 2]);
                const float mul = __fmul_rn(wab, w.wz[cc]);
                dv.x = fmaf(mul, fx, dv.x);
                dv.y = fmaf(mul, fy, dv.y);
                dv.z = fmaf(mul, fz, dv.z);
            }
        }
    return dv;
}

// The CIC-weighted force of a particle gathered from the real potential phi
// instead of the float4 force grid: each corner's force is formed from phi as
// gradient_kernel forms it, F_d = 0.5f * (phi(c - e_d) - phi(c + e_d)), and
// accumulated in gather_global's order, so the result is bit-identical to
// gradient_kernel followed by gather_global.  The 8 corners need phi on the
// 32 points of the 4^3 cube around the cell without its edges and corners:
// the four inner z columns (z-1 .. z+2) and the x and y faces.  4 bytes per
// point from a 4-byte grid instead of 16 bytes per corner from a 16-byte
// grid, and no force grid to write.
__device__ __forceinline__ float3 gather_phi(const float* __restrict__ phi, const PState& c, const KickWeights& w,
                                             int ng) {
    const int ix = cell_x(c.c), iy = cell_y(c.c), iz = cell_z(c.c);
    const int xm = ix == 0 ? ng - 1 : ix - 1, x1 = ix + 1 == ng ? 0 : ix + 1, x2 = x1 + 1 == ng ? 0 : x1 + 1;
    const int ym = iy == 0 ? ng - 1 : iy - 1, y1 = iy + 1 == ng ? 0 : iy + 1, y2 = y1 + 1 == ng ? 0 : y1 + 1;
    const int zm = iz == 0 ? ng - 1 : iz - 1, z1 = iz + 1 == ng ? 0 : iz + 1, z2 = z1 + 1 == ng ? 0 : z1 + 1;
    // 32-bit cell indices (ng^3 <= 2^30)
    const unsigned sx[4] = {(unsigned)(xm * ng), (unsigned)(ix * ng), (unsigned)(x1 * ng), (unsigned)(x2 * ng)};
    const unsigned sy[4] = {(unsigned)ym, (unsigned)iy, (unsigned)y1, (unsigned)y2};
    auto row = [&](int a, int b) { return (sx[a] + sy[b]) * (unsigned)ng; };
    const unsigned sz[4] = {(unsigned)zm, (unsigned)iz, (unsigned)z1, (unsigned)z2};
    // P[a][b][t]: phi(x_a, y_b, z_{t-1}) on the inner columns; X[e][b][cc],
    // Y[a][e][cc]: the x and y faces (e = 0: x-1 / y-1, e = 1: x+2 / y+2)
    float P[2][2][4], X[2][2][2], Y[2][2][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int t = 0; t < 4; ++t) P[a][b][t] = __ldg(&phi[row(1 + a, 1 + b) + sz[t]]);
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                X[e][b][cc] = __ldg(&phi[row(3 * e, 1 + b) + sz[1 + cc]]);
                Y[b][e][cc] = __ldg(&phi[row(1 + b, 3 * e) + sz[1 + cc]]);
            }
    return phi_corner_kick(P, X, Y, w);
}

// The paired potential (zpass_c2r_kernel with PAIR): cell z holds
// (phi(z), phi(z+1)), so the 4 z values of an inner column are two 8-byte
// loads and the 2 of a face column one: 16 loads instead of 32, the same
// values, the same forces (bit-identical to gather_phi).
__device__ __forceinline__ float3 gather_phi2(const float2* __restrict__ phi2, const PState& c, const KickWeights& w,
                                              int ng) {
    const int ix = cell_x(c.c), iy = cell_y(c.c), iz = cell_z(c.c);
    const int xm = ix == 0 ? ng - 1 : ix - 1, x1 = ix + 1 == ng ? 0 : ix + 1, x2 = x1 + 1 == ng ? 0 : x1 + 1;
    const int ym = iy == 0 ? ng - 1 : iy - 1, y1 = iy + 1 == ng ? 0 : iy + 1, y2 = y1 + 1 == ng ? 0 : y1 + 1;
    const int zm = iz == 0 ? ng - 1 : iz - 1, z1 = iz + 1 == ng ? 0 : iz + 1;
    // 32-bit cell indices (ng^3 <= 2^30): one wide multiply-add per address
    const unsigned sx[4] = {(unsigned)(xm * ng), (unsigned)(ix * ng), (unsigned)(x1 * ng), (unsigned)(x2 * ng)};
    const unsigned sy[4] = {(unsigned)ym, (unsigned)iy, (unsigned)y1, (unsigned)y2};
    auto row = [&](int a, int b) { return (sx[a] + sy[b]) * (unsigned)ng; };
    float P[2][2][4], X[2][2][2], Y[2][2][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const unsigned r = row(1 + a, 1 + b);
            const float2 lo = __ldg(&phi2[r + zm]);  // z-1, z
            const float2 hi = __ldg(&phi2[r + z1]);  // z+1, z+2
            P[a][b][0] = lo.x;
            P[a][b][1] = lo.y;
            P[a][b][2] = hi.x;
            P[a][b][3] = hi.y;
        }
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const float2 xf = __ldg(&phi2[row(3 * e, 1 + b) + iz]);
            const float2 yf = __ldg(&phi2[row(1 + b, 3 * e) + iz]);
            X[e][b][0] = xf.x;
            X[e][b][1] = xf.y;
            Y[b][e][0] = yf.x;
            Y[b][e][1] = yf.y;
        }
    return phi_corner_kick(P, X, Y, w);
}


// kick_flat_nt_kernel gathering from the real potential (gather_phi), or with
// PAIR from the paired potential (gather_phi2; phi then holds ng^3 pairs).
template <int B, int NT, int R = 1, bool PAIR = false>
__global__ void __launch_bounds__(NT, 1024 / NT) kick_phi_kernel(ParticleSoA p, int ng, const float* __restrict__ phi,
                                                               double deltaT, double fscal, float pf_a, float pf_b,
                                                               int ndrift, int nblocks, Slots sl, KickSched ks) {
    constexpr int B3 = B * B * B, SUB = B3 / NT;
    const int slot = blockIdx.y;
    if (slot_idle(sl, slot)) return;
    const int n = nblocks * SUB;
    if ((int)blockIdx.x * R >= n) return;
    p = offset_soa(p, (size_t)slot * sl.s0);
    phi += (size_t)slot * sl.s1;
    float dtf;
    kick_scalars(ks, slot, deltaT, fscal, dtf, pf_a, pf_b, ndrift);
    const float2* phi2 = reinterpret_cast<const float2*>(phi);
    auto index = [&](int u) { return (size_t)(u / SUB) * B3 + (u % SUB) * NT + threadIdx.x; };
    auto unit = [&](int k) { return ((int)blockIdx.x + (k / R) * (int)gridDim.x) * R + k % R; };
    int k = 0;
    size_t inext = index(unit(0));
    PState next = load_p(p, inext);
    for (;;) {
        const size_t i = inext;
        const PState cur = next;
        const int un = unit(k + 1);
        const bool more = un < n;
        if (more) {
            inext = index(un);
            next = load_p(p, inext);
        }
        const KickWeights w(cur, dtf);
        finish_p(p, i, cur, PAIR ? gather_phi2(phi2, cur, w, ng) : gather_phi(phi, cur, w, ng), pf_a, pf_b, ndrift,
                 ng);
        if (!more) break;
        ++k;
    }
}

__global__ void density_kernel(const unsigned long long* __restrict__ rho64, float* __restrict__ rho, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rho[i] = (float)((double)(long long)rho64[i] * kFixInv);
}

// Reference-rounded k-space tables (computed with the same float expressions
// as the reference so the device math library rounds them identically):
//   cosq[i] = cos(float(i) * float(2pi/ng)) - 1   (calcGreens.hpp:15-17, cos of a float)
//   sk[i]   = sinf(float(signed(i) * (2pi/ng)))    (kspace_solver.cu:3-5, 61-64)
//   pkw[i]  = [sinf(k/2)/(k/2)]^-4 as float         (filter_power.cu:3-32), 1 at k = 0
__global__ void ktables_kernel(int ng, double* __restrict__ cosq, float* __restrict__ sk, float* __restrict__ pkw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ng) return;
    const float df = (float)((2 * M_PI) / ((float)ng));
    const float arg = (float)i * df;
    const double c = cos(arg);
    cosq[i] = c - 1.0;
    const double d = (2 * M_PI) / ((double)ng);
    float km = (float)signed_mode(i, ng);
    km = (float)((double)km * d);
    sk[i] = sinf(km);
    float f = sinf(0.5f * km) / (0.5 * km);
    f = f * f;
    f = __frcp_rn(f * f);
    if (km == 0.f) f = 1.0f;
    pkw[i] = f;
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): counter = (cell, 0, 0,
// 0), key = (seed, 0x4850474D); two 53-bit uniforms -> one Box-Muller normal.
__device__ __forceinline__ void philox_round(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3, uint32_t k0,
                                             uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t hi0 = __umulhi(M0, c0), lo0 = M0 * c0;
    const uint32_t hi1 = __umulhi(M1, c2), lo1 = M1 * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
}

__device__ __forceinline__ double philox_normal(uint64_t ctr, uint32_t seed) {
    uint32_t c0 = (uint32_t)ctr, c1 = (uint32_t)(ctr >> 32), c2 = 0u, c3 = 0u;
    uint32_t k0 = seed, k1 = 0x4850474Du;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        philox_round(c0, c1, c2, c3, k0, k1);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    const double u1 = ((double)(((uint64_t)(c0 >> 5) << 26) | (uint64_t)(c1 >> 6)) + 0.5) * (1.0 / 9007199254740992.0);
    const double u2 = ((double)(((uint64_t)(c2 >> 5) << 26) | (uint64_t)(c3 >> 6)) + 0.5) * (1.0 / 9007199254740992.0);
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

__global__ void noise_kernel(float* __restrict__ out, size_t n, uint32_t seed) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = (float)philox_normal((uint64_t)i, seed);
}

// The reference's white noise (GenerateRealRandom, rng_initializer.cu:38-49),
// drawn through cuRAND's device API: the default generator state seeded with
// (seed, subsequence = the cell's linear index, offset 0), one
// curand_normal_double per cell, stored as float.  T threads (a power of two)
// draw cells t, t + T, t + 2T, ...: a thread seeds its first cell with
// curand_init and reaches each next one with skipahead_sequence(T).
// Subsequence skips compose, so every cell gets exactly the state
// curand_init(seed, cell, 0) gives it, for one jump per cell instead of
// curand_init's skip over the whole cell index.
__global__ void noise_curand_kernel(float* __restrict__ out, int n, int seed, int T) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T || t >= n) return;
    curandState base;
    curand_init(seed, t, 0, &base);
    for (int c = t; c < n; c += T) {
        curandState st = base;
        out[c] = (float)curand_normal_double(&st);
        if (c + T < n) skipahead_sequence((unsigned long long)T, &base);
    }
}

// placeParticles (place_particles_initializer.cu:23-65): lattice point q of
// particle idx (get_index with np), x = q*(ng/np) + delta*s (wrapped),
// v = velmul * s.  The position is formed in FP64 and split into cell + offset.
__global__ void place_kernel(const float* __restrict__ s, size_t scomp, ParticleSoA p, int np_side, int B, int ng,
                             float delta_f, float velmul) {
    const size_t n = (size_t)np_side * np_side * np_side;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t q = lattice_of_internal(i, np_side, B);
    const int qx = (int)(q / ((size_t)np_side * np_side));
    const int qy = (int)((q / np_side) % np_side);
    const int qz = (int)(q % np_side);
    const float r = (float)ng / (float)np_side;
    const float sxv = s[q], syv = s[scomp + q], szv = s[2 * scomp + q];
    const float dsx = delta_f * sxv, dsy = delta_f * syv, dsz = delta_f * szv;
    int ix, iy, iz;
    float ox, oy, oz;
    {
        const double X = (double)((float)qx * r) + (double)dsx;
        const double fl = floor(X);
        ix = wrap_axis((int)fl, ng);
        ox = (float)(X - fl);
        if (ox >= 1.f) { ox = 0.f; ix = wrap_axis(ix + 1, ng); }
    }
    {
        const double X = (double)((float)qy * r) + (double)dsy;
        const double fl = floor(X);
        iy = wrap_axis((int)fl, ng);
        oy = (float)(X - fl);
        if (oy >= 1.f) { oy = 0.f; iy = wrap_axis(iy + 1, ng); }
    }
    {
        const double X = (double)((float)qz * r) + (double)dsz;
        const double fl = floor(X);
        iz = wrap_axis((int)fl, ng);
        oz = (float)(X - fl);
        if (oz >= 1.f) { oz = 0.f; iz = wrap_axis(iz + 1, ng); }
    }
    p.cell[i] = pack_cell(ix, iy, iz);
    p.ox[i] = ox;
    p.oy[i] = oy;
    p.oz[i] = oz;
    p.vx[i] = velmul * sxv;
    p.vy[i] = velmul * syv;
    p.vz[i] = velmul * szv;
}

// ---------------------------------------------------------------------------
static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

cudaError_t smem_attr_once(const void* func, int bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, int> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> g(mu);
    int& have = done[{dev, func}];
    if (have >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) have = bytes;
    return e;
}

int blocks_per_sm_once(const void* func, int threads, int smem) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, int> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> g(mu);
    auto it = done.find({dev, func});
    if (it != done.end()) return it->second;
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem) != cudaSuccess) per_sm = 1;
    if (per_sm < 1) per_sm = 1;
    done[{dev, func}] = per_sm;
    return per_sm;
}

cudaError_t launch_load_state(const float* x, const float* v, const ParticleSoA& p, int np_side, int B, int ng,
                              cudaStream_t s) {
    const size_t n = (size_t)np_side * np_side * np_side;
    load_state_kernel<<<nblk(n, 256), 256, 0, s>>>(x, v, p, np_side, B, ng);
    return cudaGetLastError();
}
cudaError_t launch_store_state(const ParticleSoA& p, float* x, float* v, int np_side, int B, int ng,
                               cudaStream_t s) {
    const size_t n = (size_t)np_side * np_side * np_side;
    store_state_kernel<<<nblk(n, 256), 256, 0, s>>>(p, x, v, np_side, B, ng);
    return cudaGetLastError();
}
cudaError_t launch_drift(const ParticleSoA& p, size_t n, int ng, float pf, cudaStream_t s) {
    drift_kernel<<<nblk(n, 256), 256, 0, s>>>(p, n, ng, pf);
    return cudaGetLastError();
}

// CIC of the particles folded `fold` times for P(k): foldParticles
// (fold_particles_power.cu:3-27) maps x to 2x mod ng per axis, applied fold
// times to the power spectrum's copy of the positions (power.cu:194-199).
// Done here exactly on the packed form (cell, offset): doubling a float is
// exact and so is taking 1 off an offset in [1, 2).  The folded positions
// spread a Lagrangian block over the whole grid, so the weights (the
// deposit's fixed point) go straight to the int64 grid; P(k) only.
template <bool SMALL>
__global__ void deposit_folded_kernel(ParticleSoA p, size_t n, int ng, int fold, float mass,
                                      unsigned long long* __restrict__ rho) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t c = __ldg(&p.cell[i]);
    int cx = cell_x(c), cy = cell_y(c), cz = cell_z(c);
    float ox = __ldg(&p.ox[i]), oy = __ldg(&p.oy[i]), oz = __ldg(&p.oz[i]);
    for (int f = 0; f < fold; ++f) {
        ox *= 2.f;
        oy *= 2.f;
        oz *= 2.f;
        cx *= 2;
        cy *= 2;
        cz *= 2;
        if (ox >= 1.f) { ox -= 1.f; ++cx; }
        if (oy >= 1.f) { oy -= 1.f; ++cy; }
        if (oz >= 1.f) { oz -= 1.f; ++cz; }
        cx %= ng;
        cy %= ng;
        cz %= ng;
    }
    deposit_global<SMALL>(rho, pack_cell(cx, cy, cz), ox, oy, oz, mass, ng);
}

cudaError_t launch_deposit_folded(const ParticleSoA& p, size_t n, int ng, int fold, float mass,
                                  unsigned long long* rho, cudaStream_t s) {
    if (fold < 0) return cudaErrorInvalidValue;
    if (mass <= 1.0f)
        deposit_folded_kernel<true><<<nblk(n, 256), 256, 0, s>>>(p, n, ng, fold, mass, rho);
    else
        deposit_folded_kernel<false><<<nblk(n, 256), 256, 0, s>>>(p, n, ng, fold, mass, rho);
    return cudaGetLastError();
}
int window_records(int np_side, int ng) {
    const int nb = np_side / block_side(np_side, ng);
    return nb * nb * nb * kWinRec;
}

int deposit_cap_cells(int np_side, int ng) {
    const int B = block_side(np_side, ng);
    const int r = (B * ng + np_side - 1) / np_side + 6;  // block region + margin
    int cap = r * r * r;
    if (cap < 4096) cap = 4096;
    if (cap > 9216) cap = 9216;  // 72 KB: three CTAs per SM
    return cap & ~3;             // a multiple of 4: the windows are zeroed and read as uint4
}

static int num_sms() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = n > 0 ? n : 148;
    }
    return cached[dev];
}

// Windowed deposit configurations.  The kernels share one signature; a
// configuration is (kernel, threads per CTA, window cells, bytes per window
// cell).
using DepositFn = void (*)(ParticleSoA, int, int, float, unsigned long long*, int, int*, SpillList, Slots);
struct DepositCfg {
    DepositFn fn;
    int nt, cap, cell_bytes;
};

constexpr int kDepositCands = 12;

// Candidates per block side; index = HGPM_DEPOSIT (or the tuned choice).
//   16^3 blocks: 0-2 (lo, hi) 16-bit-split windows (deposit_tiled_kernel) with
//   256 / 512 / 1024 threads; 3-4 32-bit windows (deposit_w32_kernel), 512
//   threads x-chained, 256 threads with a 4-deep load ring; 5-8 column
//   kernels (deposit_col_kernel, 256 threads, x-half split): 4 CTAs per SM
//   with a 4- or 2-deep ring, 3 CTAs per SM with 18432-cell windows, and 4
//   CTAs per SM detecting wraps from the atomics' returned values; 9 direct
//   (deposit_direct_kernel: no window, every weight to the int64 grid); 10
//   the column kernel with the wrap check folded into the flush; 11 the
//   default column kernel with the x-chain merge (column_adds CHAIN).
//   8^3 blocks: 0 split window, 1 32-bit window (256 threads, 13312 cells),
//   2 column kernel (64 threads, 4096 cells), 3 32-bit window (512 threads,
//   kBigCap cells), 4 column kernel with returned-value wrap detection, 5
//   direct, 6 column kernel with the check in the flush, 7 column kernel with
//   returned-value wraps and the x-chain merge.
// The 32-bit windows need mass <= 64; otherwise the split window of the same
// thread count runs.
template <int B, bool SMALL>
static int deposit_candidates(int cap_default, bool w32, DepositCfg* out) {
    int n = 0;
    if constexpr (B == 16) {
        out[n++] = {deposit_tiled_kernel<B, SMALL, 256, 3>, 256, cap_default, 8};
        out[n++] = {deposit_tiled_kernel<B, SMALL, 512, 2>, 512, 13824, 8};
        out[n++] = {deposit_tiled_kernel<B, SMALL, 1024, 1>, 1024, kBigCap, 8};
        if (w32) {
            out[n++] = {deposit_w32_kernel<B, 512, 2, true>, 512, 13824, 4};
            out[n++] = {deposit_w32_kernel<B, 256, 4, true, 4>, 256, 13312, 4};
            out[n++] = {deposit_col_kernel<B, 4, 4>, 256, 13312, 4};
            out[n++] = {deposit_col_kernel<B, 4, 2>, 256, 13312, 4};
            out[n++] = {deposit_col_kernel<B, 3, 4>, 256, 18432, 4};
            out[n++] = {deposit_col_kernel<B, 4, 4, 1>, 256, 13312, 4};
        } else {
            // the split window with the same threads per CTA
            const int same_nt[6] = {1, 0, 0, 0, 0, 0};
            for (int i = 0; i < 6; ++i) out[n + i] = out[same_nt[i]];
            n += 6;
        }
        out[n++] = {deposit_direct_kernel<B, SMALL, 512>, 512, 0, 0};
        out[n++] = w32 ? DepositCfg{deposit_col_kernel<B, 4, 4, 2>, 256, 13312, 4} : out[0];
        out[n++] = w32 ? DepositCfg{deposit_col_kernel<B, 4, 4, 1, true>, 256, 13312, 4} : out[0];
    } else {
        out[n++] = {deposit_tiled_kernel<B, SMALL, 256, 3>, 256, cap_default, 8};
        if (w32) {
            out[n++] = {deposit_w32_kernel<B, 256, 4, true, 2>, 256, 13312, 4};
            out[n++] = {deposit_col_kernel<B, 12, 4>, B * B, 4096, 4};
            out[n++] = {deposit_w32_kernel<B, 512, 2, true, 1>, 512, kBigCap, 4};
            out[n++] = {deposit_col_kernel<B, 12, 4, 1>, B * B, 4096, 4};
        } else {
            for (int i = 0; i < 4; ++i) out[n++] = out[0];
        }
        out[n++] = {deposit_direct_kernel<B, SMALL, 256>, 256, 0, 0};
        out[n++] = w32 ? DepositCfg{deposit_col_kernel<B, 12, 4, 2>, B * B, 4096, 4} : out[0];
        out[n++] = w32 ? DepositCfg{deposit_col_kernel<B, 12, 4, 1, true>, B * B, 4096, 4} : out[0];
    }
    return n;
}

// Default candidate (measured mid-run): 16^3 blocks the column kernel with
// returned-value wrap detection (1.41 ms at 512^3, against 1.46 with the
// window-sum check and 2.22 for the split window with 512 threads); 8^3
// blocks with more cells than particles per axis (their windows span twice
// the block) the 32-bit 256-thread kernel with 13312-cell windows (6.9 ms
// for 512^3 particles on a 1024^3 grid, against 8.3-11.8 for the other
// windows), otherwise the column kernel.
template <int B>
static int deposit_default_choice(int np_side, int ng) {
    if (B == 16) return 8;
    return ng > np_side ? 1 : 2;
}

template <int B, bool SMALL>
static cudaError_t deposit_impl(const ParticleSoA& p, int np_side, int ng, float mass, unsigned long long* rho,
                                int cap, int* blkwin, const SpillList& spill, const Slots& sl, int nslots,
                                int choice, cudaStream_t s) {
    DepositCfg cands[kDepositCands];
    const int ncand = deposit_candidates<B, SMALL>(cap, mass <= 64.0f, cands);
    const int mode = choice >= 0 && choice < ncand ? choice : deposit_default_choice<B>(np_side, ng);
    const DepositCfg& cfg = cands[mode];
    const DepositFn k = cfg.fn;
    const int nt = cfg.nt;
    cap = cfg.cap;
    const int smem = cap * cfg.cell_bytes;
    cudaError_t e = smem_attr_once((const void*)k, smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(spill.cnt, 0, sizeof(int) * nslots, s);
    if (e == cudaSuccess && spill.over) e = cudaMemsetAsync(spill.over, 0, sizeof(int) * nslots, s);
    if (e != cudaSuccess) return e;
    const int nb = np_side / B;
    k<<<dim3(nb * nb * nb, nslots), nt, smem, s>>>(p, np_side, ng, mass, rho, cap, blkwin, spill, sl);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    constexpr int NTS = B * B * B >= 1024 ? 1024 : B * B * B;
    auto ks = deposit_spill_kernel<B, SMALL, NTS>;
    e = smem_attr_once((const void*)ks, kBigCap * 8);
    if (e != cudaSuccess) return e;
    const int per_slot = num_sms() / nslots > 1 ? num_sms() / nslots : 1;  // about one CTA per SM in all
    ks<<<dim3(per_slot, nslots), NTS, kBigCap * 8, s>>>(p, np_side, ng, mass, rho, blkwin, spill, sl);
    return cudaGetLastError();
}

int deposit_candidates(int np_side, int ng) { return block_side(np_side, ng) == 16 ? kDepositCands : 8; }

int deposit_default(int np_side, int ng) {
    return block_side(np_side, ng) == 16 ? deposit_default_choice<16>(np_side, ng)
                                         : deposit_default_choice<8>(np_side, ng);
}

cudaError_t launch_deposit(const ParticleSoA& p, int np_side, int ng, float mass, unsigned long long* rho,
                           int* blkwin, const SpillList& spill, cudaStream_t s, const Slots& sl, int nslots,
                           int choice) {
    if (!blkwin || !spill.cnt || !spill.items) return cudaErrorInvalidValue;
    const int B = block_side(np_side, ng);
    const int cap = deposit_cap_cells(np_side, ng);
    // SMALL needs every window add (a weight, or two merged x-chain weights,
    // each < mass*2^31) below 2^32: mass <= 1
    const bool small = mass <= 1.0f;
    if (B == 16) return small ? deposit_impl<16, true>(p, np_side, ng, mass, rho, cap, blkwin, spill, sl, nslots, choice, s)
                              : deposit_impl<16, false>(p, np_side, ng, mass, rho, cap, blkwin, spill, sl, nslots, choice, s);
    return small ? deposit_impl<8, true>(p, np_side, ng, mass, rho, cap, blkwin, spill, sl, nslots, choice, s)
                 : deposit_impl<8, false>(p, np_side, ng, mass, rho, cap, blkwin, spill, sl, nslots, choice, s);
}
// Kick candidates per block side; all run the same FP32 arithmetic in the
// same order (bit-identical).  16^3 blocks: 0-2 flat 1024-thread CTAs taking
// a block as four four-plane units in runs of 4 / 2 / 1 (kick_flat_nt_kernel;
// measured at 512^3 mid-run 2.03 / 2.04 / 2.08 ms), 3 flat 256-thread items
// (kick_spill_kernel, 2.25 ms), 4 windowed (kick_win4_kernel + the flat
// kernel for the queued blocks).  8^3 blocks: 0 flat 256-thread items, 1-2
// flat 512-thread CTAs (a whole block per unit) in runs of 1 / 2, 3 flat
// 256-thread CTAs in runs of 4, 4 windowed.  Both: 5-6 the flat schedules of
// 0 / 1 gathering the real potential, 7 the paired potential.
constexpr int kKickCands = 8;
constexpr int kKickWindowed = 4;
// candidates 5 and 6 gather from the real potential (kick_phi_kernel), 7 from
// the paired potential: the step then needs no force grid (kick_uses_phi)
constexpr int kKickPhiFirst = 5;
constexpr int kKickPhi2 = 7;

int kick_candidates(int np_side, int ng) {
    (void)np_side;
    (void)ng;
    return kKickCands;
}

bool kick_uses_phi(int choice) { return choice >= kKickPhiFirst && choice < kKickCands; }
bool kick_uses_phi2(int choice) { return choice == kKickPhi2; }

// Measured mid-run, kick plus the z inverse phase that makes what it
// gathers: 512^3 particles on 512^3 cells (16^3 blocks) 2.51 ms for the
// paired potential, 2.73 for the real one, 2.78 for the force grid with its
// gradient kernel; 512^3 on 1024^3 (8^3 blocks) 7.5 / 9.7 / 12.2 ms for the
// real potential / the paired one / the force grid.
int kick_default(int np_side, int ng) { return block_side(np_side, ng) == 16 ? kKickPhi2 : kKickPhiFirst; }

int kick_kernels(int choice, int np_side, int ng) {
    (void)np_side;
    (void)ng;
    return choice == kKickWindowed ? 2 : 1;
}

template <int B, int NT, int R>
static cudaError_t kick_flat_launch(const ParticleSoA& p, int np_side, int ng, const float4* f, double deltaT,
                                    double fscal, float pf_a, float pf_b, int ndrift, const Slots& sl,
                                    const KickSched& ks, int nslots, cudaStream_t s) {
    const int nblocks = (np_side / B) * (np_side / B) * (np_side / B);
    auto kf = kick_flat_nt_kernel<B, NT, R>;
    const int grid = num_sms() * blocks_per_sm_once((const void*)kf, NT, 0);
    kf<<<dim3(grid, nslots), NT, 0, s>>>(p, ng, f, deltaT, fscal, pf_a, pf_b, ndrift, nblocks, sl, ks);
    return cudaGetLastError();
}

template <int B, int NT, int R, bool PAIR = false>
static cudaError_t kick_phi_launch(const ParticleSoA& p, int np_side, int ng, const float* phi, double deltaT,
                                   double fscal, float pf_a, float pf_b, int ndrift, const Slots& sl,
                                   const KickSched& ks, int nslots, cudaStream_t s) {
    const int nblocks = (np_side / B) * (np_side / B) * (np_side / B);
    auto kf = kick_phi_kernel<B, NT, R, PAIR>;
    const int grid = num_sms() * blocks_per_sm_once((const void*)kf, NT, 0);
    kf<<<dim3(grid, nslots), NT, 0, s>>>(p, ng, phi, deltaT, fscal, pf_a, pf_b, ndrift, nblocks, sl, ks);
    return cudaGetLastError();
}

template <int B>
static cudaError_t kick_impl(const ParticleSoA& p, int np_side, int ng, const float4* f, const float* phi,
                             double deltaT, double fscal, float pf_a, float pf_b, int ndrift, int choice, int* blkwin,
                             bool have_rec, const SpillList& spill, const Slots& sl, const KickSched& ks, int nslots,
                             cudaStream_t s) {
    if (kick_uses_phi(choice)) {
        if constexpr (B == 16) {
            if (choice == 5) return kick_phi_launch<B, 1024, 4>(p, np_side, ng, phi, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
            if (choice == 7) return kick_phi_launch<B, 1024, 4, true>(p, np_side, ng, phi, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
            return kick_phi_launch<B, 1024, 2>(p, np_side, ng, phi, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
        } else {
            if (choice == 5) return kick_phi_launch<B, 512, 1>(p, np_side, ng, phi, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
            if (choice == 7) return kick_phi_launch<B, 512, 1, true>(p, np_side, ng, phi, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
            return kick_phi_launch<B, 512, 2>(p, np_side, ng, phi, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
        }
    }
    constexpr int NT = 512;
    auto ksp = kick_spill_kernel<B>;
    // persistent grid of exactly the resident CTAs (no second round)
    const int sp_grid = num_sms() * blocks_per_sm_once((const void*)ksp, 256, 0);
    if (choice != kKickWindowed) {
        if constexpr (B == 16) {
            if (choice == 0) return kick_flat_launch<B, 1024, 4>(p, np_side, ng, f, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
            if (choice == 1) return kick_flat_launch<B, 1024, 2>(p, np_side, ng, f, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
            if (choice == 2) return kick_flat_launch<B, 1024, 1>(p, np_side, ng, f, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
        } else {
            if (choice == 1) return kick_flat_launch<B, 512, 1>(p, np_side, ng, f, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
            if (choice == 2) return kick_flat_launch<B, 512, 2>(p, np_side, ng, f, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
            if (choice == 3) return kick_flat_launch<B, 256, 4>(p, np_side, ng, f, deltaT, fscal, pf_a, pf_b, ndrift, sl, ks, nslots, s);
        }
        ksp<<<dim3(sp_grid, nslots), 256, 0, s>>>(p, ng, f, deltaT, fscal, pf_a, pf_b, ndrift, 0, 1, spill, sl, ks);
        return cudaGetLastError();
    }
    auto k = kick_win4_kernel<B, NT>;
    const int smem = kWin4Cap * 16;
    cudaError_t e = smem_attr_once((const void*)k, smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(spill.cnt, 0, sizeof(int) * nslots, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(spill.next, 0, sizeof(int) * nslots, s);
    if (e != cudaSuccess) return e;
    const int nb = np_side / B;
    // persistent: about two CTAs per SM over all slots, blocks taken in order
    // from a per-slot counter
    int per_slot = 2 * num_sms() / nslots;
    if (per_slot < 1) per_slot = 1;
    if (per_slot > nb * nb * nb) per_slot = nb * nb * nb;
    k<<<dim3(per_slot, nslots), NT, smem, s>>>(p, np_side, ng, f, deltaT, fscal, pf_a, pf_b, ndrift, blkwin,
                                                 have_rec ? 1 : 0, 0, spill, sl, ks);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    ksp<<<dim3(sp_grid, nslots), 256, 0, s>>>(p, ng, f, deltaT, fscal, pf_a, pf_b, ndrift, have_rec ? 1 : 0, 0, spill,
                                               sl, ks);
    return cudaGetLastError();
}

cudaError_t launch_kick_drift(const ParticleSoA& p, int np_side, int ng, const float4* f, double deltaT,
                              double fscal, float pf_a, float pf_b, int ndrift, int choice, int* blkwin,
                              bool have_rec, const SpillList& spill, cudaStream_t s, const Slots& sl,
                              const KickSched& ks, int nslots, const float* phi) {
    if (!spill.cnt || !spill.items || !spill.next || !blkwin) return cudaErrorInvalidValue;
    if (choice < 0 || choice >= kKickCands) choice = 0;
    if (kick_uses_phi(choice) && !phi) choice = 0;
    if (block_side(np_side, ng) == 16)
        return kick_impl<16>(p, np_side, ng, f, phi, deltaT, fscal, pf_a, pf_b, ndrift, choice, blkwin, have_rec,
                             spill, sl, ks, nslots, s);
    return kick_impl<8>(p, np_side, ng, f, phi, deltaT, fscal, pf_a, pf_b, ndrift, choice, blkwin, have_rec, spill,
                        sl, ks, nslots, s);
}
__global__ void slots_advance_kernel(int* __restrict__ active, int* __restrict__ step,
                                     const int* __restrict__ nsteps, int nslots) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nslots || !active[k]) return;
    const int st = step[k] + 1;
    step[k] = st;
    if (st >= nsteps[k]) active[k] = 0;
}

cudaError_t launch_slots_advance(int* active, int* step, const int* nsteps, int nslots, cudaStream_t s) {
    slots_advance_kernel<<<nblk(nslots, 128), 128, 0, s>>>(active, step, nsteps, nslots);
    return cudaGetLastError();
}

cudaError_t launch_density(const unsigned long long* rho64, float* rho, size_t n, cudaStream_t s) {
    density_kernel<<<nblk(n, 256), 256, 0, s>>>(rho64, rho, n);
    return cudaGetLastError();
}
cudaError_t launch_ktables(int ng, double* cosq, float* sk, float* pkw, cudaStream_t s) {
    ktables_kernel<<<nblk(ng, 128), 128, 0, s>>>(ng, cosq, sk, pkw);
    return cudaGetLastError();
}
cudaError_t launch_noise(float* out, size_t n, int seed, int kind, cudaStream_t s) {
    if (kind == 0) {
        if (n > 0x7fffffffu) return cudaErrorInvalidValue;  // the reference's int cell index
        // threads T, a power of two (which thread draws a cell does not change
        // the cell's state): about n / 64, so a thread's one curand_init is
        // shared by ~64 cells that each cost one skip, but at least
        // min(n, 32768) so that small grids still spread over the GPU (at
        // least 32)
        const size_t target = n / 64 > (n < 32768 ? n : 32768) ? n / 64 : (n < 32768 ? n : 32768);
        size_t T = 32;
        while (T * 2 <= target) T *= 2;
        noise_curand_kernel<<<nblk(T, 256), 256, 0, s>>>(out, (int)n, seed, (int)T);
    } else {
        noise_kernel<<<nblk(n, 256), 256, 0, s>>>(out, n, (uint32_t)seed);
    }
    return cudaGetLastError();
}
cudaError_t launch_place(const float* sgrid, size_t scomp, const ParticleSoA& p, int np_side, int ng, float delta_f,
                         float velmul, cudaStream_t s) {
    const size_t n = (size_t)np_side * np_side * np_side;
    place_kernel<<<nblk(n, 256), 256, 0, s>>>(sgrid, scomp, p, np_side, block_side(np_side, ng), ng, delta_f, velmul);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Multi-class step (multi_class.h): the particle phases, each one launch over
// every class and slot, running the single-class kernels' device bodies.
// ---------------------------------------------------------------------------
namespace {

constexpr int kMCDepCap = 13312;  // the column deposit's window (52 KB)

// global unit u -> (class k, slot, local unit); false for an idle slot
__device__ __forceinline__ bool mc_find(const MCTable& t, int u, int& k, int& slot, int& lu) {
    k = 0;
    while (k + 1 < t.n && u >= t.u0[k + 1]) ++k;
    const int per = (t.u0[k + 1] - t.u0[k]) / t.c[k].nslots;
    const int r = u - t.u0[k];
    slot = r / per;
    lu = r - slot * per;
    return !t.c[k].active || t.c[k].active[slot];
}

__global__ void mc_prep_kernel(const __grid_constant__ MCTable t) {
    for (int k = 0; k < t.n; ++k) {
        const MCClass& c = t.c[k];
        for (int i = threadIdx.x; i < c.nslots; i += blockDim.x) {
            c.spill.cnt[i] = 0;
            if (c.spill.over) c.spill.over[i] = 0;
        }
    }
}

// deposit_col_kernel<16, 4, 4, 1> over the blocks of every slot of every
// class, one CTA per block (a persistent grid walking the blocks took 8 %
// longer: blocks' windows differ in size across classes)
__global__ void __launch_bounds__(256, 4) mc_deposit_kernel(const __grid_constant__ MCTable t) {
    int k, slot, blk;
    if (!mc_find(t, blockIdx.x, k, slot, blk)) return;
    const MCClass& c = t.c[k];
    deposit_col_body<16, 4, 1>(offset_soa(c.p, (size_t)slot * c.part_stride), c.np, c.ng, c.mass,
                               c.rho64 + (size_t)slot * c.ncell, kMCDepCap, c.blkwin + (size_t)slot * c.win_stride,
                               c.spill.items + (size_t)slot * c.spill.nblocks, c.spill.cnt + slot,
                               c.spill.over ? c.spill.over + slot : nullptr, blk);
}

// deposit_spill_kernel over every slot's queue: blockIdx.y = global slot
__global__ void __launch_bounds__(1024, 1) mc_spill_kernel(const __grid_constant__ MCTable t) {
    int k = 0, slot = blockIdx.y;
    while (k < t.n && slot >= t.c[k].nslots) slot -= t.c[k++].nslots;
    if (k >= t.n) return;
    const MCClass& c = t.c[k];
    if (c.active && !c.active[slot]) return;
    const int cnt = c.spill.cnt[slot];
    if ((int)blockIdx.x >= cnt) return;
    deposit_spill_body<16, true, 1024>(offset_soa(c.p, (size_t)slot * c.part_stride), c.np, c.ng, c.mass,
                                       c.rho64 + (size_t)slot * c.ncell, c.blkwin + (size_t)slot * c.win_stride,
                                       c.spill.items + (size_t)slot * c.spill.nblocks, cnt, blockIdx.x, gridDim.x);
}

// kick_phi_kernel's arithmetic (the paired potential) over units of 1024
// particles (a quarter of a 16^3 block: four Lagrangian x-planes) of every
// slot of every class; the slot's scalars come from its schedule row.  The
// next unit's particle is loaded before the current one is finished.
__global__ void __launch_bounds__(1024, 1) mc_kick_kernel(const __grid_constant__ MCTable t) {
    constexpr int B3 = 4096, SUB = 4;
    int u = blockIdx.x, k = 0, slot = 0, lu = 0;
    // first unit of an active slot at or after u (u = total: none)
    auto next_active = [&](int v) {
        for (; v < t.u0[t.n]; v += gridDim.x)
            if (mc_find(t, v, k, slot, lu)) break;
        return v;
    };
    auto index = [&]() { return (size_t)(lu / SUB) * B3 + (lu % SUB) * 1024 + threadIdx.x; };
    u = next_active(u);
    if (u >= t.u0[t.n]) return;
    PState next = load_p(offset_soa(t.c[k].p, (size_t)slot * t.c[k].part_stride), index());
    while (u < t.u0[t.n]) {
        const MCClass& c = t.c[k];
        const int cslot = slot;
        const size_t i = index();
        const PState cur = next;
        u = next_active(u + gridDim.x);
        if (u < t.u0[t.n]) next = load_p(offset_soa(t.c[k].p, (size_t)slot * t.c[k].part_stride), index());
        ParticleSoA p = offset_soa(c.p, (size_t)cslot * c.part_stride);
        const float2* phi2 = reinterpret_cast<const float2*>(c.force + (size_t)cslot * c.force_elems);
        float dtf, pf_a = 0.f, pf_b = 0.f;
        int ndrift = 0;
        kick_scalars(KickSched{c.sched, c.step, c.pitch}, cslot, 0.0, 0.0, dtf, pf_a, pf_b, ndrift);
        finish_p(p, i, cur, gather_phi2(phi2, cur, KickWeights(cur, dtf), c.ng), pf_a, pf_b, ndrift, c.ng);
    }
}

__global__ void mc_advance_kernel(const __grid_constant__ MCTable t) {
    for (int k = 0; k < t.n; ++k) {
        const MCClass& c = t.c[k];
        for (int i = threadIdx.x; i < c.nslots; i += blockDim.x) {
            if (!c.active[i]) continue;
            const int st = c.step[i] + 1;
            c.step[i] = st;
            if (st >= c.nsteps[i]) c.active[i] = 0;
        }
    }
}

cudaError_t mc_persistent(const void* kern, MCTable& t, int threads, int smem, cudaStream_t s) {
    if (t.u0[t.n] == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (e != cudaSuccess) return e;
    int grid = num_sms() * (per_sm > 0 ? per_sm : 1);
    if (grid > t.u0[t.n]) grid = t.u0[t.n];
    void* args[] = {&t};
    return cudaLaunchKernel(kern, dim3(grid), dim3(threads), args, smem, s);
}

}  // namespace

bool mc_class_supported(int ng, int np) {
    if (block_side(np, ng) != 16 || ng > np) return false;
    switch (ng) {
#define X(n) case n:
        HGPM_MC_SIZES(X)
#undef X
        return true;
        default:
            return false;
    }
}

cudaError_t mc_step(const MCTable& base, cudaStream_t s) {
    if (base.n < 1 || base.n > kMaxMC) return cudaErrorInvalidValue;
    int nslots = 0;
    for (int k = 0; k < base.n; ++k) {
        if (!mc_class_supported(base.c[k].ng, base.c[k].np) || base.c[k].nslots < 1) return cudaErrorInvalidValue;
        nslots += base.c[k].nslots;
    }
    void* pargs[] = {const_cast<MCTable*>(&base)};
    cudaError_t e = cudaLaunchKernel((const void*)mc_prep_kernel, dim3(1), dim3(256), pargs, 0, s);
    if (e != cudaSuccess) return e;
    // deposit: one unit per Lagrangian block
    MCTable td = base;
    td.u0[0] = 0;
    for (int k = 0; k < base.n; ++k) td.u0[k + 1] = td.u0[k] + base.c[k].nblocks * base.c[k].nslots;
    e = smem_attr_once((const void*)mc_deposit_kernel, kMCDepCap * 4);
    if (e != cudaSuccess) return e;
    {
        void* dargs[] = {&td};
        e = cudaLaunchKernel((const void*)mc_deposit_kernel, dim3(td.u0[td.n]), dim3(256), dargs, kMCDepCap * 4, s);
        if (e != cudaSuccess) return e;
    }
    {
        const int per = num_sms() / nslots > 1 ? num_sms() / nslots : 1;
        auto ks = mc_spill_kernel;
        e = smem_attr_once((const void*)ks, kBigCap * 8);
        if (e != cudaSuccess) return e;
        ks<<<dim3(per, nslots), 1024, kBigCap * 8, s>>>(base);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    e = mc_launch_fft_passes(base, s);
    if (e != cudaSuccess) return e;
    // kick: four units per block
    MCTable tk = base;
    tk.u0[0] = 0;
    for (int k = 0; k < base.n; ++k) tk.u0[k + 1] = tk.u0[k] + base.c[k].nblocks * 4 * base.c[k].nslots;
    e = mc_persistent((const void*)mc_kick_kernel, tk, 1024, 0, s);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernel((const void*)mc_advance_kernel, dim3(1), dim3(256), pargs, 0, s);
}

}  // namespace hgpm

// ===========================================================================
// Allocation-free CIC density
//
// Some callers cannot allocate device memory at all: code that runs inside a
// host framework which owns every device allocation (a memory pool with a
// fixed budget, or a plugin host that forbids its plugins to call
// cudaMalloc), and code that must not allocate after start-up so that a long
// run cannot fail later on an out-of-memory error.  For them,
// hgpm_cic_density_noalloc computes the same deterministic density as
// hgpm_deposit + hgpm_get_density from device positions into a device
// density, and takes its int64 accumulation grid from this file-scope
// device array instead of from an allocation.
// ===========================================================================
#define HGPM_NOALLOC_MAX_NG 128
static __device__ __align__(256) unsigned long long g_noalloc_acc[HGPM_NOALLOC_MAX_NG * HGPM_NOALLOC_MAX_NG *
                                                                   HGPM_NOALLOC_MAX_NG];

namespace hgpm {

__global__ void noalloc_zero_kernel(unsigned long long* __restrict__ acc, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) acc[i] = 0ull;
}

// One thread per particle: the same cell/offset split as load_state_kernel and
// the same fixed-point corner weights as the tiled deposit, added with
// integer atomics (so the result is bit-identical to the tiled deposit).
template <bool SMALL>
__global__ void noalloc_deposit_kernel(const float* __restrict__ x, size_t n, int ng, float mass,
                                       unsigned long long* __restrict__ acc) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int ix, iy, iz;
    float dx, dy, dz;
    split_axis(x[3 * i + 0], ng, ix, dx);
    split_axis(x[3 * i + 1], ng, iy, dy);
    split_axis(x[3 * i + 2], ng, iz, dz);
    unsigned long long q[8];
    cic_fixed<SMALL>(dx, dy, dz, mass, q);
    const int ix1 = ix + 1 == ng ? 0 : ix + 1;
    const int iy1 = iy + 1 == ng ? 0 : iy + 1;
    const int iz1 = iz + 1 == ng ? 0 : iz + 1;
    const size_t sx[2] = {(size_t)ix * ng * ng, (size_t)ix1 * ng * ng};
    const size_t sy[2] = {(size_t)iy * ng, (size_t)iy1 * ng};
    const size_t sz[2] = {(size_t)iz, (size_t)iz1};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) atomicAdd(&acc[sx[a] + sy[b] + sz[cc]], q[(a * 2 + b) * 2 + cc]);
}

}  // namespace hgpm

#include <cstdio>
#include <mutex>

#include "../../include/hgpm_c.h"

// Device address of g_noalloc_acc, looked up once per device (with that device
// current); in host code the array's name is only a host-side stand-in.
static unsigned long long* g_noalloc_ptr[64];
static std::mutex g_noalloc_mu;

extern "C" int hgpm_cic_density_noalloc(const float* x_dev, int np_side, int ng, float* rho_dev, void* stream) {
    if (!x_dev || !rho_dev || np_side <= 0 || ng <= 0) return HGPM_ERR_ARG;
    if (ng > HGPM_NOALLOC_MAX_NG) {
        fprintf(stderr,
                "hgpm_cic_density_noalloc: ng = %d exceeds the %d^3-cell limit of the built-in accumulation "
                "grid; use hgpm_deposit on a context instead\n",
                ng, HGPM_NOALLOC_MAX_NG);
        return HGPM_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HGPM_ERR_CUDA;
    unsigned long long* acc;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_acc);
            if (e != cudaSuccess || !p) {
                fprintf(stderr, "hgpm_cic_density_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
                return HGPM_ERR_CUDA;
            }
            g_noalloc_ptr[dev] = static_cast<unsigned long long*>(p);
        }
        acc = g_noalloc_ptr[dev];
    }
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t ncell = (size_t)ng * ng * ng;
    const size_t n = (size_t)np_side * np_side * np_side;
    const float gp = (float)ng / (float)np_side;  // pm_actions.cpp:229-230
    const float mass = gp * gp * gp;
    hgpm::noalloc_zero_kernel<<<(unsigned)((ncell + 255) / 256), 256, 0, s>>>(acc, ncell);
    if (mass <= 1.0f)
        hgpm::noalloc_deposit_kernel<true><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x_dev, n, ng, mass, acc);
    else
        hgpm::noalloc_deposit_kernel<false><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x_dev, n, ng, mass, acc);
    if (hgpm::launch_density(acc, rho_dev, ncell, s) != cudaSuccess) return HGPM_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? HGPM_OK : HGPM_ERR_CUDA;
}
