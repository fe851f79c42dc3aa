// particles.cu — particle-side kernels of the PM step: state conversion,
// drift, deterministic fixed-point CIC deposit, fused CIC gather + kick +
// drift(s), and the small per-size table kernels.
//
// Positions are a packed int32 cell (10 bits per axis) plus an FP32 offset
// in [0, 1) per axis; the offset equals the reference's `x - (int)x`
// (cic_pm.cu:52-58) bit for bit when a state is loaded.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "hgpm_device.cuh"
#include "hgpm_internal.h"

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

__global__ void store_state_kernel(ParticleSoA p, float* __restrict__ x, float* __restrict__ v, int np_side, int B) {
    const size_t n = (size_t)np_side * np_side * np_side;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t q = lattice_of_internal(i, np_side, B);
    const uint32_t c = p.cell[i];
    x[3 * q + 0] = (float)cell_x(c) + p.ox[i];
    x[3 * q + 1] = (float)cell_y(c) + p.oy[i];
    x[3 * q + 2] = (float)cell_z(c) + p.oz[i];
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
// rounded to a 2^-32 fixed-point int64 and added with integer atomics, so the
// density is independent of particle, thread and CTA order (bit-exact run to
// run).  One CTA owns one Lagrangian block of B^3 particles: it finds the
// bounding box of their cells, accumulates the block's CIC weights in a
// shared-memory int64 window over that box, and flushes the window's non-zero
// cells to the global accumulator with one coalesced red.add per cell.  A
// block whose particles spread over more than cap_cells cells falls back to
// per-corner global atomics.
__device__ __forceinline__ int nearest_image(int d, int ng) {
    if (d < -(ng >> 1)) d += ng;
    else if (d >= (ng >> 1)) d -= ng;
    return d;
}

__device__ __forceinline__ void cic_fixed(float dx, float dy, float dz, float mass, long long q[8]) {
    const float wx[2] = {1.f - dx, dx}, wy[2] = {1.f - dy, dy}, wz[2] = {1.f - dz, dz};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const float mul = __fmul_rn(__fmul_rn(__fmul_rn(wx[a], wy[b]), wz[cc]), mass);
                q[(a * 2 + b) * 2 + cc] = __float2ll_rn(mul * kFixScaleF);
            }
}

template <int B>
__global__ void __launch_bounds__(256) deposit_tiled_kernel(ParticleSoA p, int np_side, int ng, float mass,
                                                            unsigned long long* __restrict__ rho, int cap_cells) {
    constexpr int B3 = B * B * B;
    constexpr int PPT = B3 / 256;
    extern __shared__ unsigned long long win[];
    __shared__ int bb[6];
    const int tid = threadIdx.x;
    const int nb = np_side / B;
    const int blk = blockIdx.x;
    const int bz = blk % nb, by = (blk / nb) % nb, bx = blk / (nb * nb);
    const int ox = (int)((long long)bx * B * ng / np_side);
    const int oy = (int)((long long)by * B * ng / np_side);
    const int oz = (int)((long long)bz * B * ng / np_side);
    if (tid < 3) bb[tid] = 0x7fffffff;
    else if (tid < 6) bb[tid] = -0x7fffffff;
    __syncthreads();
    const size_t p0 = (size_t)blk * B3;
    int rx[PPT], ry[PPT], rz[PPT];
    int mn[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, mx[3] = {-0x7fffffff, -0x7fffffff, -0x7fffffff};
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const uint32_t c = __ldg(&p.cell[p0 + tid + k * 256]);
        rx[k] = nearest_image(cell_x(c) - ox, ng);
        ry[k] = nearest_image(cell_y(c) - oy, ng);
        rz[k] = nearest_image(cell_z(c) - oz, ng);
        mn[0] = min(mn[0], rx[k]); mx[0] = max(mx[0], rx[k]);
        mn[1] = min(mn[1], ry[k]); mx[1] = max(mx[1], ry[k]);
        mn[2] = min(mn[2], rz[k]); mx[2] = max(mx[2], rz[k]);
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
    const int lx0 = bb[0], ly0 = bb[1], lz0 = bb[2];
    const int wx = bb[3] - lx0 + 2, wy = bb[4] - ly0 + 2, wz = bb[5] - lz0 + 2;
    const long long vol = (long long)wx * wy * wz;
    if (vol <= cap_cells) {
        for (int i = tid; i < vol; i += 256) win[i] = 0ull;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            const size_t idx = p0 + tid + k * 256;
            long long q[8];
            cic_fixed(__ldg(&p.ox[idx]), __ldg(&p.oy[idx]), __ldg(&p.oz[idx]), mass, q);
            const int a0 = rx[k] - lx0, b0 = ry[k] - ly0, c0 = rz[k] - lz0;
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int cc = 0; cc < 2; ++cc)
                        atomicAdd(&win[((a0 + a) * wy + (b0 + b)) * wz + (c0 + cc)],
                                  (unsigned long long)q[(a * 2 + b) * 2 + cc]);
        }
        __syncthreads();
        const int gx0 = ox + lx0, gy0 = oy + ly0, gz0 = oz + lz0;
        for (int i = tid; i < vol; i += 256) {
            const unsigned long long v = win[i];
            if (v == 0ull) continue;
            const int cz = i % wz, cy = (i / wz) % wy, cx = i / (wz * wy);
            const int gx = wrap_axis(gx0 + cx, ng), gy = wrap_axis(gy0 + cy, ng), gz = wrap_axis(gz0 + cz, ng);
            atomicAdd(&rho[((size_t)gx * ng + gy) * ng + gz], v);
        }
    } else {
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            const size_t idx = p0 + tid + k * 256;
            long long q[8];
            cic_fixed(__ldg(&p.ox[idx]), __ldg(&p.oy[idx]), __ldg(&p.oz[idx]), mass, q);
            const int ix = wrap_axis(ox + rx[k], ng), iy = wrap_axis(oy + ry[k], ng), iz = wrap_axis(oz + rz[k], ng);
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
                    for (int cc = 0; cc < 2; ++cc)
                        atomicAdd(&rho[sx[a] + sy[b] + sz[cc]], (unsigned long long)q[(a * 2 + b) * 2 + cc]);
        }
    }
}

// ICICKernel (icic_pm.cu:72-127) fused with up to two UpdatePosKernel drifts:
// v += sum_8 float(w*deltaT*fscal) * F[corner]; then x += v*pf_a (, v*pf_b).
__global__ void kick_drift_kernel(ParticleSoA p, size_t n, int ng, const float* __restrict__ fx,
                                  const float* __restrict__ fy, const float* __restrict__ fz, double deltaT,
                                  double fscal, float pf_a, float pf_b, int ndrift) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t c = p.cell[i];
    float ox = p.ox[i], oy = p.oy[i], oz = p.oz[i];
    int ix = cell_x(c), iy = cell_y(c), iz = cell_z(c);
    const int ix1 = ix + 1 == ng ? 0 : ix + 1;
    const int iy1 = iy + 1 == ng ? 0 : iy + 1;
    const int iz1 = iz + 1 == ng ? 0 : iz + 1;
    const uint32_t sx[2] = {(uint32_t)ix * ng * ng, (uint32_t)ix1 * ng * ng};
    const uint32_t sy[2] = {(uint32_t)iy * ng, (uint32_t)iy1 * ng};
    const uint32_t sz[2] = {(uint32_t)iz, (uint32_t)iz1};
    const float wx[2] = {1.f - ox, ox}, wy[2] = {1.f - oy, oy}, wz[2] = {1.f - oz, oz};
    float dvx = 0.f, dvy = 0.f, dvz = 0.f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const uint32_t idx = sx[a] + sy[b] + sz[cc];
                const float w = __fmul_rn(__fmul_rn(wx[a], wy[b]), wz[cc]);
                const float mul = (float)(((double)w * deltaT) * fscal);
                dvx = fmaf(mul, __ldg(&fx[idx]), dvx);
                dvy = fmaf(mul, __ldg(&fy[idx]), dvy);
                dvz = fmaf(mul, __ldg(&fz[idx]), dvz);
            }
    const float vx = p.vx[i] + dvx, vy = p.vy[i] + dvy, vz = p.vz[i] + dvz;
    p.vx[i] = vx;
    p.vy[i] = vy;
    p.vz[i] = vz;
    if (ndrift > 0) {
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

cudaError_t launch_load_state(const float* x, const float* v, const ParticleSoA& p, int np_side, int B, int ng,
                              cudaStream_t s) {
    const size_t n = (size_t)np_side * np_side * np_side;
    load_state_kernel<<<nblk(n, 256), 256, 0, s>>>(x, v, p, np_side, B, ng);
    return cudaGetLastError();
}
cudaError_t launch_store_state(const ParticleSoA& p, float* x, float* v, int np_side, int B, cudaStream_t s) {
    const size_t n = (size_t)np_side * np_side * np_side;
    store_state_kernel<<<nblk(n, 256), 256, 0, s>>>(p, x, v, np_side, B);
    return cudaGetLastError();
}
cudaError_t launch_drift(const ParticleSoA& p, size_t n, int ng, float pf, cudaStream_t s) {
    drift_kernel<<<nblk(n, 256), 256, 0, s>>>(p, n, ng, pf);
    return cudaGetLastError();
}
int deposit_cap_cells(int np_side, int ng) {
    const int B = block_side(np_side, ng);
    const int r = (B * ng + np_side - 1) / np_side + 6;  // block region + margin
    int cap = r * r * r;
    if (cap < 4096) cap = 4096;
    if (cap > 12288) cap = 12288;  // 96 KB of int64: two CTAs per SM
    return cap;
}

cudaError_t launch_deposit(const ParticleSoA& p, int np_side, int ng, float mass, unsigned long long* rho,
                           cudaStream_t s) {
    const int B = block_side(np_side, ng);
    const int cap = deposit_cap_cells(np_side, ng);
    const int nblocks = (np_side / B) * (np_side / B) * (np_side / B);
    const int smem = cap * 8;
    if (B == 16) {
        auto k = deposit_tiled_kernel<16>;
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        k<<<nblocks, 256, smem, s>>>(p, np_side, ng, mass, rho, cap);
    } else {
        auto k = deposit_tiled_kernel<8>;
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        k<<<nblocks, 256, smem, s>>>(p, np_side, ng, mass, rho, cap);
    }
    return cudaGetLastError();
}
cudaError_t launch_kick_drift(const ParticleSoA& p, size_t n, int ng, const float* fx, const float* fy,
                              const float* fz, double deltaT, double fscal, float pf_a, float pf_b, int ndrift,
                              cudaStream_t s) {
    kick_drift_kernel<<<nblk(n, 256), 256, 0, s>>>(p, n, ng, fx, fy, fz, deltaT, fscal, pf_a, pf_b, ndrift);
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
cudaError_t launch_noise(float* out, size_t n, uint32_t seed, cudaStream_t s) {
    noise_kernel<<<nblk(n, 256), 256, 0, s>>>(out, n, seed);
    return cudaGetLastError();
}
cudaError_t launch_place(const float* sgrid, size_t scomp, const ParticleSoA& p, int np_side, int ng, float delta_f,
                         float velmul, cudaStream_t s) {
    const size_t n = (size_t)np_side * np_side * np_side;
    place_kernel<<<nblk(n, 256), 256, 0, s>>>(sgrid, scomp, p, np_side, block_side(np_side, ng), ng, delta_f, velmul);
    return cudaGetLastError();
}

}  // namespace hgpm
