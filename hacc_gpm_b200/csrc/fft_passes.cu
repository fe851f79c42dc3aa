// fft_passes.cu — the 3D R2C/C2R FFT passes of the PM step and the x pass
// fused with k-space operators.
//
// Layouts (row-major, z fastest, as get_index in src/haccgpm.hpp:423-429):
//   real grid      float  [ng][ng][ng]
//   half spectrum  float2 [ng][ng][zs]   kz in [0, ng/2], zs = padded row
// The forward 3D transform is: z pass (R2C along contiguous rows) ->
// y pass (strided, in place) -> x pass (strided).  The inverse runs the
// passes in reverse order with a C2R z pass.  The step never materialises
// the forward x output: the x pass is fused with the Green's function and
// gradient (Poisson), with the IC displacement operator, or with P(k)
// binning, all of which act on one x-line tile while it is in shared memory.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include <map>
#include <mutex>

#include "fft_engine.cuh"
#include "hgpm_device.cuh"
#include "hgpm_internal.h"
#include "kspace_ops.cuh"
#include "multi_class.h"

namespace hgpm {

extern __shared__ float4 hgpm_smem[];

// ---------------------------------------------------------------------------
// per-size tile configuration
// ---------------------------------------------------------------------------
template <int NG> struct Cfg {
    static constexpr int M = NG / 2;                       // complex length of z lines
    static constexpr int L = M >= 512 ? 8 : (M >= 256 ? 16 : (M >= 96 ? 32 : 64));  // z lines per CTA
    static constexpr int CS = NG >= 768 ? 8 : 16;          // strided-pass columns per CTA
    static constexpr int CX = NG >= 768 ? 4 : (NG >= 384 ? 8 : 16);  // fused x-pass columns
    static constexpr int ZSMEM = M * (L + 1) * 8;
    static constexpr int SSMEM = NG * CS * 8;
    static constexpr int XSMEM = 2 * NG * CX * 8;
    // threads per CTA of the strided and fused x passes: 512 halves the
    // per-thread register staging so two CTAs (32 warps) fit per SM
    static constexpr int NTS = NG >= 128 ? 512 : 256;
    static constexpr int NTX = NG >= 128 ? 512 : 256;
};

// ---------------------------------------------------------------------------
// tile load/store between global strided lines and shared [N][C]
// ---------------------------------------------------------------------------
// Rows e in [0, N) at g + e*rs; columns [0, nvalid) valid (nvalid may be < C).
// All of a thread's global loads are issued before any shared store
// (register staging) so each CTA keeps its whole tile in flight.  CG: loads
// from L2 (ld.global.cg), for data other CTAs of the same kernel wrote.
template <int N, int C, int NT = kThreads, bool CG = false>
__device__ __forceinline__ void load_tile(float2* __restrict__ tile, const float2* __restrict__ g,
                                          size_t rs, int nvalid) {
    constexpr int TPR = C / 2;  // float4 (two complex) per row chunk
    constexpr int TOT = N * TPR;
    constexpr int PER = (TOT + NT - 1) / NT;
    float4 v[PER];
    if (nvalid >= C) {
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int i = threadIdx.x + t * NT;
            if ((TOT % NT) == 0 || i < TOT) {
                const int e = i / TPR, c = 2 * (i % TPR);
                const float4* src = reinterpret_cast<const float4*>(g + (size_t)e * rs + c);
                v[t] = CG ? __ldcg(src) : __ldcs(src);
            }
        }
    } else {
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int i = threadIdx.x + t * NT;
            v[t] = make_float4(0.f, 0.f, 0.f, 0.f);
            if ((TOT % NT) == 0 || i < TOT) {
                const int e = i / TPR, c = 2 * (i % TPR);
                const float2* src = g + (size_t)e * rs + c;
                if (c + 1 < nvalid) {
                    v[t] = CG ? __ldcg(reinterpret_cast<const float4*>(src)) : *reinterpret_cast<const float4*>(src);
                } else if (c < nvalid) {
                    const float2 s = CG ? __ldcg(src) : src[0];
                    v[t] = make_float4(s.x, s.y, 0.f, 0.f);
                }
            }
        }
    }
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int i = threadIdx.x + t * NT;
        if ((TOT % NT) == 0 || i < TOT) {
            const int e = i / TPR, c = 2 * (i % TPR);
            *reinterpret_cast<float4*>(&tile[e * C + c]) = v[t];
        }
    }
}

// WB: write-back stores (kept in L2 for a read later in the same kernel)
// instead of streaming ones.
template <int N, int C, int NT = kThreads, bool WB = false>
__device__ __forceinline__ void store_tile(const float2* __restrict__ tile, float2* __restrict__ g,
                                           size_t rs, int nvalid) {
    constexpr int TPR = C / 2;
    constexpr int TOT = N * TPR;
    constexpr int PER = (TOT + NT - 1) / NT;
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int i = threadIdx.x + t * NT;
        if ((TOT % NT) == 0 || i < TOT) {
            const int e = i / TPR, c = 2 * (i % TPR);
            float2* dst = g + (size_t)e * rs + c;
            const float4 v = *reinterpret_cast<const float4*>(&tile[e * C + c]);
            if (c + 1 < nvalid) {
                if (WB) *reinterpret_cast<float4*>(dst) = v;
                else __stcs(reinterpret_cast<float4*>(dst), v);
            } else if (c < nvalid) {
                dst[0] = make_float2(v.x, v.y);
            }
        }
    }
}

// store_tile with a per-column operator applied on the way out:
// g[e][c] = op.comp(d, 0, iy, col0 + c, tile[e][c]) (components d >= 1 of the
// fused x pass, whose factor depends on the plane and column only).
template <int N, int C, int NT, class Op>
__device__ __forceinline__ void store_tile_comp(const float2* __restrict__ tile, float2* __restrict__ g, size_t rs,
                                                int nvalid, const Op& op, int d, int iy, int col0) {
    constexpr int TPR = C / 2;
    constexpr int TOT = N * TPR;
    constexpr int PER = (TOT + NT - 1) / NT;
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int i = threadIdx.x + t * NT;
        if ((TOT % NT) == 0 || i < TOT) {
            const int e = i / TPR, c = 2 * (i % TPR);
            float2* dst = g + (size_t)e * rs + c;
            const float4 v = *reinterpret_cast<const float4*>(&tile[e * C + c]);
            const float2 a = op.comp(d, 0, iy, col0 + c, make_float2(v.x, v.y));
            const float2 b = op.comp(d, 0, iy, col0 + c + 1, make_float2(v.z, v.w));
            if (c + 1 < nvalid) {
                __stcs(reinterpret_cast<float4*>(dst), make_float4(a.x, a.y, b.x, b.y));
            } else if (c < nvalid) {
                dst[0] = a;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// z pass, forward R2C.  FIX: input is the int64 fixed-point density
// (value * 2^32); it is converted to float delta = rho - mean in FP64 and the
// accumulator is zeroed for the next deposit.  Otherwise input is float.
// ---------------------------------------------------------------------------
// The CTA's work (line group bx of one box) as a device function: the
// single-class kernel below and the multi-class pass (mc_zfwd_kernel) run
// the same code.
template <int NG, bool FIX, int L = Cfg<NG>::L>
__device__ __forceinline__ void zpass_r2c_body(void* __restrict__ in_, float2* __restrict__ out, int nlines, int zs,
                                               double mean, const float2* __restrict__ tw, int bx) {
    constexpr int M = NG / 2, ES = L + 1;
    float2* buf = reinterpret_cast<float2*>(hgpm_smem);
    const int line0 = bx * L;
    constexpr int TOT = L * M;
    constexpr int PER = (TOT + kThreads - 1) / kThreads;
    if (FIX) {
        ulonglong2 q[PER];
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int i = threadIdx.x + t * kThreads;
            const int l = i / M, m = i % M;
            q[t] = make_ulonglong2(0ull, 0ull);
            if (((TOT % kThreads) == 0 || i < TOT) && line0 + l < nlines)
                q[t] = __ldcs(reinterpret_cast<const ulonglong2*>(reinterpret_cast<unsigned long long*>(in_) +
                                                                  (size_t)(line0 + l) * NG) + m);
        }
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int i = threadIdx.x + t * kThreads;
            const int l = i / M, m = i % M;
            if (((TOT % kThreads) == 0 || i < TOT)) {
                if (line0 + l < nlines)
                    __stcs(reinterpret_cast<ulonglong2*>(reinterpret_cast<unsigned long long*>(in_) +
                                                         (size_t)(line0 + l) * NG) + m, make_ulonglong2(0ull, 0ull));
                buf[m * ES + l] = make_float2((float)((double)(long long)q[t].x * kFixInv - mean),
                                              (float)((double)(long long)q[t].y * kFixInv - mean));
            }
        }
    } else {
        float2 z[PER];
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int i = threadIdx.x + t * kThreads;
            const int l = i / M, m = i % M;
            z[t] = make_float2(0.f, 0.f);
            if (((TOT % kThreads) == 0 || i < TOT) && line0 + l < nlines)
                z[t] = reinterpret_cast<const float2*>(reinterpret_cast<const float*>(in_) + (size_t)(line0 + l) * NG)[m];
        }
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int i = threadIdx.x + t * kThreads;
            if ((TOT % kThreads) == 0 || i < TOT) buf[(i % M) * ES + i / M] = z[t];
        }
    }
    __syncthreads();
    fft_tile<M, L, ES, false, kThreads, 2>(buf, tw);
    constexpr int H = M / 2 + 1;
    for (int i = threadIdx.x; i < L * H; i += kThreads) {
        const int l = i / H, k = i % H;
        const int line = line0 + l;
        if (line >= nlines) continue;
        const float2 zk = buf[k * ES + l];
        const float2 zm = buf[((M - k) % M) * ES + l];
        const float2 w = __ldg(&tw[k]);
        // E = (Zk + conj Zm)/2, O = -i (Zk - conj Zm)/2, X[k] = E + w O,
        // X[M-k] = conj(E - w O)
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        const float2 wo = cmul(w, o);
        float2* dst = out + (size_t)line * zs;
        dst[k] = cadd(e, wo);
        if (k != M - k) {
            const float2 xm = csub(e, wo);
            dst[M - k] = make_float2(xm.x, -xm.y);
        }
    }
}

// The single-class kernel: zpass_r2c_body's code with the slot prologue
// written out (as a kernel with its own restrict-qualified parameters it
// compiles without the body's 76 bytes of spills at 512^3).
template <int NG, bool FIX>
__global__ void __launch_bounds__(kThreads, 4) zpass_r2c_kernel(void* __restrict__ in_, float2* __restrict__ out,
                                                             int nlines, int zs, double mean,
                                                             const float2* __restrict__ tw, Slots sl) {
    constexpr int M = NG / 2, L = Cfg<NG>::L, ES = L + 1;
    float2* buf = reinterpret_cast<float2*>(hgpm_smem);
    if (slot_idle(sl, blockIdx.y)) return;
    // slot stride s0 counts input elements (int64 when FIX, float otherwise)
    in_ = FIX ? (void*)(reinterpret_cast<unsigned long long*>(in_) + (size_t)blockIdx.y * sl.s0)
              : (void*)(reinterpret_cast<float*>(in_) + (size_t)blockIdx.y * sl.s0);
    out += (size_t)blockIdx.y * sl.s1;
    const int line0 = blockIdx.x * L;
    constexpr int TOT = L * M;
    constexpr int PER = (TOT + kThreads - 1) / kThreads;
    if (FIX) {
        ulonglong2 q[PER];
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int i = threadIdx.x + t * kThreads;
            const int l = i / M, m = i % M;
            q[t] = make_ulonglong2(0ull, 0ull);
            if (((TOT % kThreads) == 0 || i < TOT) && line0 + l < nlines)
                q[t] = __ldcs(reinterpret_cast<const ulonglong2*>(reinterpret_cast<unsigned long long*>(in_) +
                                                                  (size_t)(line0 + l) * NG) + m);
        }
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int i = threadIdx.x + t * kThreads;
            const int l = i / M, m = i % M;
            if (((TOT % kThreads) == 0 || i < TOT)) {
                if (line0 + l < nlines)
                    __stcs(reinterpret_cast<ulonglong2*>(reinterpret_cast<unsigned long long*>(in_) +
                                                         (size_t)(line0 + l) * NG) + m, make_ulonglong2(0ull, 0ull));
                buf[m * ES + l] = make_float2((float)((double)(long long)q[t].x * kFixInv - mean),
                                              (float)((double)(long long)q[t].y * kFixInv - mean));
            }
        }
    } else {
        float2 z[PER];
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int i = threadIdx.x + t * kThreads;
            const int l = i / M, m = i % M;
            z[t] = make_float2(0.f, 0.f);
            if (((TOT % kThreads) == 0 || i < TOT) && line0 + l < nlines)
                z[t] = reinterpret_cast<const float2*>(reinterpret_cast<const float*>(in_) + (size_t)(line0 + l) * NG)[m];
        }
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int i = threadIdx.x + t * kThreads;
            if ((TOT % kThreads) == 0 || i < TOT) buf[(i % M) * ES + i / M] = z[t];
        }
    }
    __syncthreads();
    fft_tile<M, L, ES, false, kThreads, 2>(buf, tw);
    constexpr int H = M / 2 + 1;
    for (int i = threadIdx.x; i < L * H; i += kThreads) {
        const int l = i / H, k = i % H;
        const int line = line0 + l;
        if (line >= nlines) continue;
        const float2 zk = buf[k * ES + l];
        const float2 zm = buf[((M - k) % M) * ES + l];
        const float2 w = __ldg(&tw[k]);
        // E = (Zk + conj Zm)/2, O = -i (Zk - conj Zm)/2, X[k] = E + w O,
        // X[M-k] = conj(E - w O)
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        const float2 wo = cmul(w, o);
        float2* dst = out + (size_t)line * zs;
        dst[k] = cadd(e, wo);
        if (k != M - k) {
            const float2 xm = csub(e, wo);
            dst[M - k] = make_float2(xm.x, -xm.y);
        }
    }
}

// ---------------------------------------------------------------------------
// z pass, inverse C2R, ncomp components, unnormalised * scale;
// blockIdx.y = slot * ncomp + component.
// X[0] and X[ng/2] are taken as real (Hermitian extension), which makes the
// result equal to the real part of the reference's full C2C inverse.
// ---------------------------------------------------------------------------
// PAIR: out holds nlines * NG pairs, cell z of a line (phi(z), phi(z+1 mod
// NG)) (the paired potential the pair-gathering kick reads).
// CG: the spectrum is read from L2 (written earlier in the same kernel).
template <int NG, bool PAIR = false, bool CG = false>
__device__ __forceinline__ void zpass_c2r_body(const float2* __restrict__ in, float* __restrict__ out, int nlines,
                                               int zs, float scale, const float2* __restrict__ tw, int bx) {
    constexpr int M = NG / 2, L = Cfg<NG>::L, ES = L + 1;
    float2* buf = reinterpret_cast<float2*>(hgpm_smem);
    const int line0 = bx * L;
    constexpr int H = M / 2 + 1;
    constexpr int TOT = L * H;
    constexpr int PER = (TOT + kThreads - 1) / kThreads;
    // register-staged: every (X[k], X[M-k]) pair of the thread is in flight
    // before the first use
    float2 rk[PER], rm[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int i = threadIdx.x + t * kThreads;
        const int l = i / H, k = i % H;
        rk[t] = make_float2(0.f, 0.f);
        rm[t] = make_float2(0.f, 0.f);
        if (i < TOT && line0 + l < nlines) {
            const float2* src = in + (size_t)(line0 + l) * zs;
            rk[t] = CG ? __ldcg(&src[k]) : __ldcs(&src[k]);
            rm[t] = CG ? __ldcg(&src[M - k]) : __ldcs(&src[M - k]);
        }
    }
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int i = threadIdx.x + t * kThreads;
        if (i >= TOT) break;
        const int l = i / H, k = i % H;
        float2 xk = rk[t], xm = rm[t];
        if (k == 0) {
            xk.y = 0.f;
            xm.y = 0.f;
        }
        const float2 w = __ldg(&tw[k]);
        // S = X[k] + conj X[M-k], D = X[k] - conj X[M-k], T = i conj(w) D
        // Z[k] = S + T, Z[M-k] = conj(S - T)
        const float2 s = make_float2(xk.x + xm.x, xk.y - xm.y);
        const float2 d = make_float2(xk.x - xm.x, xk.y + xm.y);
        const float2 cd = cmulc(d, w);                  // conj(w) * d
        const float2 tt = make_float2(-cd.y, cd.x);     // i * conj(w) * d
        buf[k * ES + l] = cadd(s, tt);
        if (k != 0 && k != M - k) {
            const float2 zm = csub(s, tt);
            buf[(M - k) * ES + l] = make_float2(zm.x, -zm.y);
        }
    }
    __syncthreads();
    fft_tile<M, L, ES, true, kThreads, 2>(buf, tw);
    for (int i = threadIdx.x; i < L * M; i += kThreads) {
        const int l = i / M, m = i % M;
        const int line = line0 + l;
        if (line >= nlines) continue;
        const float2 z = buf[m * ES + l];
        if (PAIR) {
            // cells 2m and 2m+1: (phi(2m), phi(2m+1)), (phi(2m+1), phi(2m+2))
            const float nx = buf[(m + 1 == M ? 0 : m + 1) * ES + l].x * scale;
            reinterpret_cast<float4*>(out + (size_t)line * NG * 2)[m] =
                make_float4(z.x * scale, z.y * scale, z.y * scale, nx);
        } else {
            reinterpret_cast<float2*>(out + (size_t)line * NG)[m] = make_float2(z.x * scale, z.y * scale);
        }
    }
}

template <int NG>
__global__ void __launch_bounds__(kThreads) zpass_c2r_pair_kernel(const float2* __restrict__ in,
                                                                  float* __restrict__ out, int nlines, int zs,
                                                                  const float2* __restrict__ tw) {
    zpass_c2r_body<NG, true>(in, out, nlines, zs, 1.0f, tw, blockIdx.x);
}

template <int NG>
__global__ void __launch_bounds__(kThreads) zpass_c2r_kernel(const float2* __restrict__ in, float* __restrict__ out,
                                                             int nlines, int zs, size_t in_cs, size_t out_cs,
                                                             float scale, const float2* __restrict__ tw, int ncomp,
                                                             Slots sl) {
    const int slot = blockIdx.y / ncomp, comp = blockIdx.y % ncomp;
    if (slot_idle(sl, slot)) return;
    in += (size_t)slot * sl.s0 + (size_t)comp * in_cs;
    out += (size_t)slot * sl.s1 + (size_t)comp * out_cs;
    zpass_c2r_body<NG>(in, out, nlines, zs, scale, tw, blockIdx.x);
}

// ---------------------------------------------------------------------------
// z and y passes of the x planes with a thread-block cluster per plane.
//
// A cluster of kPlaneCTAs CTAs works on one x plane at a time, planes
// cid, cid + G, cid + 2G, ... (G clusters, as many as are resident at once).
// Forward (zy_fwd_kernel): the R2C z pass of a plane's L-line tiles (int64
// density in and zeroed, as zpass_r2c_kernel<NG,1>; every kPlaneCTAs-th tile
// per CTA), the cluster barrier (release / acquire at cluster scope) that
// makes the plane's half spectrum visible to every CTA of the cluster, then
// the y transform of the plane's PlaneCfg-column tiles in place.  The plane
// (ng x zs complex, 1.1 MB at 512^3) was written microseconds earlier by
// write-back stores and is read back from L2 (.cg loads), so DRAM sees the
// z pass's traffic and one write of the spectrum instead of the y pass's
// extra read and write.  Each CTA interleaves the next plane's z tiles
// (DRAM-bound) with the current plane's y tiles (L2 and shared memory), one
// barrier per plane.  Inverse (yz_inv_pair_kernel), the same pipeline with
// the roles swapped: the y inverse of the next plane's columns (DRAM in,
// write-back stores) interleaved with the C2R z pass of the current plane's
// lines into the paired potential (as zpass_c2r_pair_kernel<NG>).  Every
// transform runs the same stages in the same order as the separate passes,
// so the results are bit-identical to theirs.
// ---------------------------------------------------------------------------
constexpr int kPlaneCTAs = 8;
template <int NG> struct PlaneCfg {
    static constexpr int CY = NG >= 768 ? 4 : 8;  // y columns per tile
    static constexpr int L = Cfg<NG>::L;
    static constexpr int ZT = NG / L;                                  // z tiles per plane
    static constexpr int YT = (NG / 2 + 1 + CY - 1) / CY;             // y tiles per plane
    static constexpr int SMEM = Cfg<NG>::ZSMEM > NG * CY * 8 ? Cfg<NG>::ZSMEM : NG * CY * 8;
    static_assert(NG % L == 0 && ZT >= kPlaneCTAs, "a plane holds whole z tiles, one or more per CTA");
};

// Every thread of every CTA of the cluster arrives; the writes before it
// are visible to the reads after it in every CTA of the cluster.  A
// hardware barrier over CTAs the cluster launch co-schedules: no polling.
__device__ __forceinline__ void plane_cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// The R2C z pass of lines [line0, line0 + L) of the int64 density: the
// arithmetic of zpass_r2c_kernel<NG, true>, the half spectrum written with
// write-back stores.  Returns synchronised (the tile may be reused).
template <int NG>
__device__ __forceinline__ void zr2c_fix_tile(unsigned long long* __restrict__ in, float2* __restrict__ out, int line0,
                                              int zs, double mean, const float2* __restrict__ tw, float2* buf) {
    constexpr int M = NG / 2, L = Cfg<NG>::L, ES = L + 1;
    constexpr int TOT = L * M;
    constexpr int PER = (TOT + kThreads - 1) / kThreads;
    static_assert(TOT % kThreads == 0, "whole tiles");
    ulonglong2 q[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int i = threadIdx.x + t * kThreads;
        const int l = i / M, m = i % M;
        q[t] = __ldcs(reinterpret_cast<const ulonglong2*>(in + (size_t)(line0 + l) * NG) + m);
    }
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int i = threadIdx.x + t * kThreads;
        const int l = i / M, m = i % M;
        __stcs(reinterpret_cast<ulonglong2*>(in + (size_t)(line0 + l) * NG) + m, make_ulonglong2(0ull, 0ull));
        buf[m * ES + l] = make_float2((float)((double)(long long)q[t].x * kFixInv - mean),
                                      (float)((double)(long long)q[t].y * kFixInv - mean));
    }
    __syncthreads();
    fft_tile<M, L, ES, false, kThreads, 2>(buf, tw);
    constexpr int H = M / 2 + 1;
    for (int i = threadIdx.x; i < L * H; i += kThreads) {
        const int l = i / H, k = i % H;
        const float2 zk = buf[k * ES + l];
        const float2 zm = buf[((M - k) % M) * ES + l];
        const float2 w = __ldg(&tw[k]);
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        const float2 wo = cmul(w, o);
        float2* dst = out + (size_t)(line0 + l) * zs;
        dst[k] = cadd(e, wo);
        if (k != M - k) {
            const float2 xm = csub(e, wo);
            dst[M - k] = make_float2(xm.x, -xm.y);
        }
    }
    __syncthreads();
}

// One y-column tile (columns [c0, c0 + CY)) of plane g transformed in place.
// CG: read from L2 (the plane was written earlier in the same kernel); WB:
// written back through L2 (read later in the same kernel).
template <int NG, bool INV, bool CG, bool WB>
__device__ __forceinline__ void plane_y_tile(float2* __restrict__ g, int c0, int zs, const float2* __restrict__ tw,
                                             float2* buf) {
    constexpr int CY = PlaneCfg<NG>::CY, H = NG / 2 + 1;
    load_tile<NG, CY, kThreads, CG>(buf, g + c0, zs, H - c0);
    __syncthreads();
    fft_tile<NG, CY, CY, INV, kThreads>(buf, tw);
    store_tile<NG, CY, kThreads, WB>(buf, g + c0, zs, H - c0);
    __syncthreads();
}

template <int NG, int MINB>
__global__ void __cluster_dims__(kPlaneCTAs, 1, 1) __launch_bounds__(kThreads, MINB)
    zy_fwd_kernel(unsigned long long* __restrict__ rho, float2* __restrict__ spec, int zs, double mean,
                  const float2* __restrict__ tw) {
    using P = PlaneCfg<NG>;
    constexpr int TMAX = P::ZT > P::YT ? P::ZT : P::YT;
    float2* buf = reinterpret_cast<float2*>(hgpm_smem);
    const int nclu = gridDim.x / kPlaneCTAs, cid = blockIdx.x / kPlaneCTAs, r = blockIdx.x % kPlaneCTAs;
    for (int t = r; t < P::ZT; t += kPlaneCTAs) zr2c_fix_tile<NG>(rho, spec, cid * NG + t * P::L, zs, mean, tw, buf);
    plane_cluster_sync();
    for (int x = cid; x < NG; x += nclu) {
        const int xn = x + nclu;
        float2* g = spec + (size_t)x * NG * zs;
        for (int t = r; t < TMAX; t += kPlaneCTAs) {
            if (xn < NG && t < P::ZT) zr2c_fix_tile<NG>(rho, spec, xn * NG + t * P::L, zs, mean, tw, buf);
            if (t < P::YT) plane_y_tile<NG, false, true, false>(g, t * P::CY, zs, tw, buf);
        }
        plane_cluster_sync();
    }
}

template <int NG, int MINB>
__global__ void __cluster_dims__(kPlaneCTAs, 1, 1) __launch_bounds__(kThreads, MINB)
    yz_inv_pair_kernel(float2* __restrict__ spec, float* __restrict__ out, int zs, const float2* __restrict__ tw) {
    using P = PlaneCfg<NG>;
    constexpr int TMAX = P::ZT > P::YT ? P::ZT : P::YT;
    float2* buf = reinterpret_cast<float2*>(hgpm_smem);
    const int nclu = gridDim.x / kPlaneCTAs, cid = blockIdx.x / kPlaneCTAs, r = blockIdx.x % kPlaneCTAs;
    for (int t = r; t < P::YT; t += kPlaneCTAs)
        plane_y_tile<NG, true, false, true>(spec + (size_t)cid * NG * zs, t * P::CY, zs, tw, buf);
    plane_cluster_sync();
    for (int x = cid; x < NG; x += nclu) {
        const int xn = x + nclu;
        for (int t = r; t < TMAX; t += kPlaneCTAs) {
            if (xn < NG && t < P::YT)
                plane_y_tile<NG, true, false, true>(spec + (size_t)xn * NG * zs, t * P::CY, zs, tw, buf);
            if (t < P::ZT) {
                zpass_c2r_body<NG, true, true>(spec, out, NG * NG, zs, 1.0f, tw, x * P::ZT + t);
                __syncthreads();
            }
        }
        plane_cluster_sync();
    }
}

// ---------------------------------------------------------------------------
// z pass of a complex-to-complex transform of a caller's [ng][ng][ng] grid
// (forward_fft / backward_fft on a cufftComplex grid, ffts.cu:244-294,
// 397-445), in place: a CTA transforms CZ<NG> contiguous z lines, staged
// transposed in shared memory ([m][l], padded) so each stage's butterflies
// read conflict-free columns.
template <int NG> struct CZ {
    static constexpr int L = NG >= 1024 ? 8 : (NG >= 512 ? 16 : (NG >= 128 ? 32 : 64));
    static constexpr int SMEM = NG * (L + 1) * 8;
};

template <int NG, bool INV>
__global__ void __launch_bounds__(kThreads) zpass_c2c_kernel(float2* __restrict__ data, int nlines,
                                                             const float2* __restrict__ tw) {
    constexpr int L = CZ<NG>::L, ES = L + 1;
    float2* buf = reinterpret_cast<float2*>(hgpm_smem);
    const int line0 = blockIdx.x * L;
    for (int i = threadIdx.x; i < L * NG; i += kThreads) {
        const int l = i / NG, m = i % NG;
        buf[m * ES + l] = line0 + l < nlines ? data[(size_t)(line0 + l) * NG + m] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_tile<NG, L, ES, INV, kThreads>(buf, tw);
    for (int i = threadIdx.x; i < L * NG; i += kThreads) {
        const int l = i / NG, m = i % NG;
        if (line0 + l < nlines) data[(size_t)(line0 + l) * NG + m] = buf[m * ES + l];
    }
}

// ---------------------------------------------------------------------------
// strided pass (y or x lines), in place,
// blockIdx = (column chunk, plane, slot * ncomp + comp)
// ---------------------------------------------------------------------------
// Column chunk bx of plane by of one component of one box, NT threads.
template <int NG, bool INV, int NT, int C = Cfg<NG>::CS>
__device__ __forceinline__ void strided_body(float2* __restrict__ data, int ncols, size_t rs, size_t ps,
                                             const float2* __restrict__ tw, int bx, int by) {
    float2* tile = reinterpret_cast<float2*>(hgpm_smem);
    const int col0 = bx * C;
    float2* g = data + (size_t)by * ps + col0;
    const int nvalid = ncols - col0;
    load_tile<NG, C, NT>(tile, g, rs, nvalid);
    __syncthreads();
    fft_tile<NG, C, C, INV, NT>(tile, tw);
    store_tile<NG, C, NT>(tile, g, rs, nvalid);
}

template <int NG, bool INV>
__global__ void __launch_bounds__(Cfg<NG>::NTS, 2) strided_kernel(float2* __restrict__ data, int ncols, size_t rs,
                                                               size_t ps, size_t cs, const float2* __restrict__ tw,
                                                               int ncomp, Slots sl) {
    const int slot = blockIdx.z / ncomp, comp = blockIdx.z % ncomp;
    if (slot_idle(sl, slot)) return;
    strided_body<NG, INV, Cfg<NG>::NTS>(data + (size_t)slot * sl.s0 + (size_t)comp * cs, ncols, rs, ps, tw,
                                        blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// x pass fused with a k-space operator producing 3 components:
//   forward x FFT of the (z,y)-transformed tile -> t = op.pre(k, rho_k) ->
//   out[0] = IFFT_x(op.comp(0, k, t));  T = IFFT_x(t) ->
//   out[1] = op.comp(1, ky, kz, T), out[2] = op.comp(2, ky, kz, T).
// The y and z components' operators (e.g. -i sin(k_y)) are constant along an
// x line, so they commute with the inverse x transform: two inverse FFTs per
// tile instead of three.
// plane = ky index, rows = kx index, columns = kz index; blockIdx.z = slot.
// ---------------------------------------------------------------------------
// One-output x pass on a loaded tile: forward x FFT, pre() in registers,
// inverse x FFT, the same stages and arithmetic as xpotential_tma_kernel (bit
// for bit).
template <int NG, int NT, class Op, int C = Cfg<NG>::CX>
__device__ __forceinline__ void xone_after_load(float2* __restrict__ tile, float2* __restrict__ out, size_t rs,
                                                int nvalid, const float2* __restrict__ tw, const Op& op, int iy,
                                                int col0) {
    fft_tile_fwd_op_inv<NG, C, C, NT, 1, true>(tile, tw,
                                              [&](int ix, int c, float2 v) { return op.pre(ix, iy, col0 + c, v); });
    store_tile<NG, C, NT>(tile, out, rs, nvalid);
}

// The one-output x pass of column chunk bx (C columns) of plane (ky) by of
// one box.
template <int NG, int NT, class Op, int C = Cfg<NG>::CX>
__device__ __forceinline__ void xone_body(const float2* __restrict__ in, float2* __restrict__ out, int ncols,
                                          size_t rs, size_t ps, const float2* __restrict__ tw, const Op& op, int bx,
                                          int by) {
    float2* tile = reinterpret_cast<float2*>(hgpm_smem);
    const int col0 = bx * C;
    const size_t off = (size_t)by * ps + col0;
    const int nvalid = ncols - col0;
    load_tile<NG, C, NT>(tile, in + off, rs, nvalid);
    __syncthreads();
    xone_after_load<NG, NT, Op, C>(tile, out + off, rs, nvalid, tw, op, by, col0);
}

// The Poisson x pass with twice the columns per CTA (one tile in shared
// memory, 2 CTAs of 512 threads per SM): more columns in flight per SM for
// the long lines (1024^3: 8 columns of 1024 points against 4).  Columns stay
// within the grid side (the Green's function indexes its table by column).
template <int NG> struct XW {
    static constexpr int C = 2 * Cfg<NG>::CX <= NG ? 2 * Cfg<NG>::CX : Cfg<NG>::CX;
};
template <int NG>
__global__ void __launch_bounds__(512, 2) xpot_wide_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                                           int ncols, size_t rs, size_t ps,
                                                           const float2* __restrict__ tw, PotentialOp op) {
    xone_body<NG, 512, PotentialOp, XW<NG>::C>(in, out, ncols, rs, ps, tw, op, blockIdx.x, blockIdx.y);
}

template <int NG, class Op>
__global__ void __launch_bounds__(Cfg<NG>::NTX) xfused_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                                              int ncols, size_t rs, size_t ps, size_t out_cs,
                                                              const float2* __restrict__ tw, Op op, Slots sl) {
    constexpr int C = Cfg<NG>::CX, NT = Cfg<NG>::NTX;
    float2* tile = reinterpret_cast<float2*>(hgpm_smem);
    float2* work = tile + NG * C;
    if (slot_idle(sl, blockIdx.z)) return;
    in += (size_t)blockIdx.z * sl.s0;
    out += (size_t)blockIdx.z * sl.s1;
    const int col0 = blockIdx.x * C;
    const int iy = blockIdx.y;
    const size_t off = (size_t)iy * ps + col0;
    const int nvalid = ncols - col0;
    load_tile<NG, C, NT>(tile, in + off, rs, nvalid);
    __syncthreads();
    if constexpr (Op::kOut == 1) {
        xone_after_load<NG, NT>(tile, out + off, rs, nvalid, tw, op, iy, col0);
        return;
    }
    // the three-output IC pass, whose registers are tight, reads every
    // twiddle from the table
    fft_tile<NG, C, C, false, NT, 1, false>(tile, tw);
    for (int i = threadIdx.x; i < NG * C; i += NT) {
        const int ix = i / C, c = i % C;
        tile[i] = op.pre(ix, iy, col0 + c, tile[i]);
    }
    // (fft_tile ended with a barrier; pre() only touches the thread's own cells)
    for (int i = threadIdx.x; i < NG * C; i += NT) {
        const int ix = i / C, c = i % C;
        work[i] = op.comp(0, ix, iy, col0 + c, tile[i]);
    }
    __syncthreads();
    fft_tile<NG, C, C, true, NT, 1, false>(work, tw);
    store_tile<NG, C, NT>(work, out + off, rs, nvalid);
    // (no thread writes tile between the barrier above and this transform)
    fft_tile<NG, C, C, true, NT, 1, false>(tile, tw);
    store_tile_comp<NG, C, NT>(tile, out + out_cs + off, rs, nvalid, op, 1, iy, col0);
    store_tile_comp<NG, C, NT>(tile, out + 2 * out_cs + off, rs, nvalid, op, 2, iy, col0);
}

// ---------------------------------------------------------------------------
// Force grid from the potential phi (real, [ng][ng][ng], z fastest):
// F_d(x) = (phi(x - e_d) - phi(x + e_d)) / 2, periodic, written as float4
// (F_x, F_y, F_z, 0) per cell.  With the unnormalised transforms used here
// this is exactly the reference's -i sin(k_d) G rho_k followed by the inverse
// FFT (kspace_solver.cu:55-90, solver.cpp:144-170): the central difference
// multiplies mode k by -i sin(2 pi k_d / ng), it is real, so it commutes with
// taking the real part, and it annihilates the Nyquist mode of its own axis
// as the reference's real part does.  blockIdx.y = slot.
// ---------------------------------------------------------------------------
// 256-bit (8 x f32) global accesses, sm_100: 32-byte aligned addresses.
struct F8 {
    float v[8];
};
__device__ __forceinline__ F8 ldg8(const float* p) {
    F8 r;
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]), "=f"(r.v[5]), "=f"(r.v[6]),
                   "=f"(r.v[7])
                 : "l"(p));
    return r;
}
// two float4 cells, streaming (evict-first)
__device__ __forceinline__ void stcs8(float4* p, float4 a, float4 b) {
    asm volatile("st.global.cs.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(a.x), "f"(a.y), "f"(a.z),
                 "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w)
                 : "memory");
}

// A thread makes 8 z-consecutive cells at XR consecutive x: 256-bit loads of
// phi and of its y neighbours, the x neighbours carried from the previous x
// (one new row per x), 256-bit stores of two cells each (whole sectors).
template <int XR, int MINB = 1, int U = 1>
__global__ void __launch_bounds__(256, MINB) gradient_kernel(const float* __restrict__ phi, float4* __restrict__ f, int ng,
                                                       Slots sl) {
    if (slot_idle(sl, blockIdx.y)) return;
    phi += (size_t)blockIdx.y * sl.s0;
    f += (size_t)blockIdx.y * sl.s1;
    const int n8 = ng / 8;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    // the launcher makes (ng / XR) ng^2 / 8 a whole number of warps, so this
    // exit takes whole warps and the shuffles below see all 32 lanes
    if (q >= (size_t)(ng / XR) * ng * n8) return;
    const int z0 = (int)(q % n8) * 8;
    const int r = (int)(q / n8);
    const int y = r % ng;
    int x = (r / ng) * XR;
    const int ym = y == 0 ? ng - 1 : y - 1, yp = y + 1 == ng ? 0 : y + 1;
    const size_t plane = (size_t)ng * ng;
    const size_t oy = (size_t)y * ng + z0, oym = (size_t)ym * ng + z0, oyp = (size_t)yp * ng + z0;
    const int lane = threadIdx.x & 31;
    F8 a = ldg8(phi + (size_t)(x == 0 ? ng - 1 : x - 1) * plane + oy);
    F8 c = ldg8(phi + (size_t)x * plane + oy);
#pragma unroll U
    for (int k = 0; k < XR; ++k, ++x) {
        const size_t px = (size_t)x * plane;
        const F8 b = ldg8(phi + (size_t)(x + 1 == ng ? 0 : x + 1) * plane + oy);
        const F8 d = ldg8(phi + px + oym);
        const F8 e = ldg8(phi + px + oyp);
        // the z neighbours of the run's ends are the adjacent lanes' end cells
        // (same row); the warp's end lanes and the row's periodic wrap load them
        float zm = __shfl_up_sync(0xffffffffu, c.v[7], 1);
        float zp = __shfl_down_sync(0xffffffffu, c.v[0], 1);
        if (lane == 0 || z0 == 0) zm = __ldg(phi + px + oy - z0 + (z0 == 0 ? ng - 1 : z0 - 1));
        if (lane == 31 || z0 + 8 == ng) zp = __ldg(phi + px + oy - z0 + (z0 + 8 == ng ? 0 : z0 + 8));
        float4 o[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const float lo = m == 0 ? zm : c.v[m - 1];
            const float hi = m == 7 ? zp : c.v[m + 1];
            o[m] = make_float4(0.5f * (a.v[m] - b.v[m]), 0.5f * (d.v[m] - e.v[m]), 0.5f * (lo - hi), 0.f);
        }
        float4* dst = f + px + oy;
#pragma unroll
        for (int m = 0; m < 8; m += 2) stcs8(dst + m, o[m], o[m + 1]);
        a = c;
        c = b;
    }
}
// ---------------------------------------------------------------------------
// x pass fused with P(k): forward x FFT, |delta|^2 * scale * CIC window, and
// deterministic per-warp FP64 shell sums.  Persistent CTAs take tiles
// blockIdx.x, +gridDim.x, ... and write one partial histogram each.
// ---------------------------------------------------------------------------
template <int NG>
__global__ void __launch_bounds__(kThreads) xpk_kernel(const float2* __restrict__ in, int ncols, size_t rs,
                                                       size_t ps, int nchunks, const float2* __restrict__ tw,
                                                       PkArgs a, double* __restrict__ part_sum,
                                                       unsigned long long* __restrict__ part_cnt) {
    constexpr int C = Cfg<NG>::CX;
    constexpr int M = NG / 2;
    constexpr int NW = kThreads / 32;
    float2* tile = reinterpret_cast<float2*>(hgpm_smem);
    double* hs = reinterpret_cast<double*>(tile + NG * C);
    unsigned long long* hc = reinterpret_cast<unsigned long long*>(hs + NW * a.nbins);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int i = threadIdx.x; i < NW * a.nbins; i += kThreads) {
        hs[i] = 0.0;
        hc[i] = 0ull;
    }
    const int ntiles = nchunks * NG;
    for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x) {
        const int chunk = tile_id % nchunks, iy = tile_id / nchunks;
        const int col0 = chunk * C;
        const int nvalid = ncols - col0;
        __syncthreads();
        load_tile<NG, C>(tile, in + (size_t)iy * ps + col0, rs, nvalid);
        __syncthreads();
        fft_tile<NG, C, C, false, kThreads>(tile, tw);
        // each warp walks its own cells in a fixed order
        for (int base = warp * 32; base < NG * C; base += kThreads) {
            const int i = base + lane;
            int bin = -1;
            double val = 0.0;
            int wgt = 0;
            if (i < NG * C) {
                const int ix = i / C, c = i % C, iz = col0 + c;
                const bool dc = (ix == 0 && iy == 0 && iz == 0);
                const bool corner = (ix == M && iy == M && iz == M);
                if (c < nvalid && !dc && !corner) {
                    const float kx = __ldg(&a.kf[ix]), ky = __ldg(&a.kf[iy]), kz = __ldg(&a.kf[iz]);
                    const float s2 = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
                    const float kmag = __fsqrt_rn(s2);
                    double fb;
                    if (a.log_bins) {
                        fb = log((double)kmag / a.min_k) / a.bin_delta;
                    } else {
                        fb = ((double)kmag - a.min_k) / a.bin_delta;
                    }
                    // (int) truncates, as calc_power_bins does (bin_power.cu:12-13):
                    // a mode just below minK lands in bin 0; further below
                    // the reference indexes before the array, here it is dropped
                    const int b = (int)fb;
                    if (b >= 0 && b < a.nbins) {
                        const float2 v = tile[i];
                        wgt = (iz == 0 || iz == M) ? 1 : 2;
                        const double p = ((double)v.x * v.x + (double)v.y * v.y) * a.scale *
                                         __ldg(&a.filt[ix]) * __ldg(&a.filt[iy]) * __ldg(&a.filt[iz]);
                        val = p * wgt;
                        bin = b;
                    }
                }
            }
            const unsigned grp = __match_any_sync(0xffffffffu, bin);
            const int leader = __ffs(grp) - 1;
            double s = 0.0;
            unsigned long long n = 0;
            unsigned m = grp;
            while (m) {
                const int src = __ffs(m) - 1;
                m &= m - 1;
                const double vv = __shfl_sync(grp, val, src);
                const int ww = __shfl_sync(grp, wgt, src);
                s += vv;
                n += (unsigned long long)ww;
            }
            if (lane == leader && bin >= 0) {
                hs[warp * a.nbins + bin] += s;
                hc[warp * a.nbins + bin] += n;
            }
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < a.nbins; b += kThreads) {
        double s = 0.0;
        unsigned long long n = 0;
        for (int w = 0; w < NW; ++w) {
            s += hs[w * a.nbins + b];
            n += hc[w * a.nbins + b];
        }
        part_sum[(size_t)blockIdx.x * a.nbins + b] = s;
        part_cnt[(size_t)blockIdx.x * a.nbins + b] = n;
    }
}

// Bin b's partial sums: one warp per bin, lane l adding partials l, l + 32,
// ... in order, then the 32 lane sums combined by a fixed shuffle tree (a
// fixed order: deterministic run to run).
__global__ void pk_reduce_kernel(const double* __restrict__ part_sum, const unsigned long long* __restrict__ part_cnt,
                                 int nparts, int nbins, double* __restrict__ sum, unsigned long long* __restrict__ cnt) {
    const int b = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (b >= nbins) return;  // whole warps
    double s = 0.0;
    unsigned long long n = 0;
    for (int p = lane; p < nparts; p += 32) {
        s += part_sum[(size_t)p * nbins + b];
        n += part_cnt[(size_t)p * nbins + b];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        n += __shfl_down_sync(0xffffffffu, n, o);
    }
    if (lane == 0) {
        sum[b] = s;
        cnt[b] = n;
    }
}

// ---------------------------------------------------------------------------
// host launchers (dispatch on the grid side)
// ---------------------------------------------------------------------------
template <class K>
static cudaError_t ensure_smem(K kernel, int bytes) {
    return smem_attr_once((const void*)kernel, bytes);
}

static inline unsigned cdiv(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

template <int NG>
static cudaError_t zfwd_impl(void* in, bool fixed, float2* out, int nlines, int zs, double mean,
                             const float2* tw, cudaStream_t s, const Slots& sl, int nslots) {
    using G = Cfg<NG>;
    const dim3 grid(cdiv(nlines, G::L), nslots);
    if (fixed) {
        auto k = zpass_r2c_kernel<NG, true>;
        cudaError_t e = ensure_smem(k, G::ZSMEM);
        if (e != cudaSuccess) return e;
        k<<<grid, kThreads, G::ZSMEM, s>>>(in, out, nlines, zs, mean, tw, sl);
    } else {
        auto k = zpass_r2c_kernel<NG, false>;
        cudaError_t e = ensure_smem(k, G::ZSMEM);
        if (e != cudaSuccess) return e;
        k<<<grid, kThreads, G::ZSMEM, s>>>(in, out, nlines, zs, mean, tw, sl);
    }
    return cudaGetLastError();
}

template <int NG>
static cudaError_t zinv_impl(const float2* in, float* out, int nlines, int zs, size_t in_cs, size_t out_cs,
                             int ncomp, float scale, const float2* tw, cudaStream_t s, const Slots& sl, int nslots) {
    using G = Cfg<NG>;
    auto k = zpass_c2r_kernel<NG>;
    cudaError_t e = ensure_smem(k, G::ZSMEM);
    if (e != cudaSuccess) return e;
    dim3 grid(cdiv(nlines, G::L), ncomp * nslots);
    k<<<grid, kThreads, G::ZSMEM, s>>>(in, out, nlines, zs, in_cs, out_cs, scale, tw, ncomp, sl);
    return cudaGetLastError();
}

// Clusters of `func` (kPlaneCTAs CTAs of kThreads threads, smem bytes each)
// resident at once on the current device, queried once per (device,
// kernel); 0 if the query fails.
static int plane_clusters_once(const void* func, int smem) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, int> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> g(mu);
    auto it = done.find({dev, func});
    if (it != done.end()) return it->second;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kPlaneCTAs, 1, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, func, &cfg) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    done[{dev, func}] = n;
    return n;
}

template <int NG, int MINB>
static cudaError_t plane_impl(bool inv, void* a, float2* spec, int zs, double mean, const float2* tw, cudaStream_t s) {
    constexpr int SMEM = PlaneCfg<NG>::SMEM;
    const void* fn = inv ? (const void*)yz_inv_pair_kernel<NG, MINB> : (const void*)zy_fwd_kernel<NG, MINB>;
    cudaError_t e = smem_attr_once(fn, SMEM);
    if (e != cudaSuccess) return e;
    int nclu = plane_clusters_once(fn, SMEM);
    if (nclu < 1 || nclu > NG) nclu = NG;  // one plane per cluster
    if (inv)
        yz_inv_pair_kernel<NG, MINB><<<nclu * kPlaneCTAs, kThreads, SMEM, s>>>(spec, reinterpret_cast<float*>(a), zs, tw);
    else
        zy_fwd_kernel<NG, MINB><<<nclu * kPlaneCTAs, kThreads, SMEM, s>>>(reinterpret_cast<unsigned long long*>(a), spec,
                                                                          zs, mean, tw);
    return cudaGetLastError();
}

template <int NG>
static cudaError_t zinv_pair_impl(const float2* in, float* out, int nlines, int zs, const float2* tw, cudaStream_t s) {
    using G = Cfg<NG>;
    auto k = zpass_c2r_pair_kernel<NG>;
    cudaError_t e = ensure_smem(k, G::ZSMEM);
    if (e != cudaSuccess) return e;
    k<<<cdiv(nlines, G::L), kThreads, G::ZSMEM, s>>>(in, out, nlines, zs, tw);
    return cudaGetLastError();
}

template <int NG>
static cudaError_t strided_impl(bool inv, float2* data, int ncols, size_t rs, size_t ps, int nplanes, size_t cs,
                                int ncomp, const float2* tw, cudaStream_t s, const Slots& sl, int nslots) {
    using G = Cfg<NG>;
    dim3 grid(cdiv(ncols, G::CS), nplanes, ncomp * nslots);
    if (inv) {
        auto k = strided_kernel<NG, true>;
        cudaError_t e = ensure_smem(k, G::SSMEM);
        if (e != cudaSuccess) return e;
        k<<<grid, G::NTS, G::SSMEM, s>>>(data, ncols, rs, ps, cs, tw, ncomp, sl);
    } else {
        auto k = strided_kernel<NG, false>;
        cudaError_t e = ensure_smem(k, G::SSMEM);
        if (e != cudaSuccess) return e;
        k<<<grid, G::NTS, G::SSMEM, s>>>(data, ncols, rs, ps, cs, tw, ncomp, sl);
    }
    return cudaGetLastError();
}

template <int NG, class Op>
static cudaError_t xfused_impl(const float2* in, float2* out, int ncols, size_t rs, size_t ps, int nplanes,
                               size_t out_cs, const float2* tw, const Op& op, cudaStream_t s, const Slots& sl = Slots{},
                               int nslots = 1) {
    using G = Cfg<NG>;
    auto k = xfused_kernel<NG, Op>;
    cudaError_t e = ensure_smem(k, G::XSMEM);
    if (e != cudaSuccess) return e;
    dim3 grid(cdiv(ncols, G::CX), nplanes, nslots);
    k<<<grid, G::NTX, G::XSMEM, s>>>(in, out, ncols, rs, ps, out_cs, tw, op, sl);
    return cudaGetLastError();
}

template <int NG>
static cudaError_t xpk_impl(const float2* in, int ncols, size_t rs, size_t ps, const float2* tw, const PkArgs& a,
                            double* part_sum, unsigned long long* part_cnt, int nparts, double* sum,
                            unsigned long long* cnt, cudaStream_t s) {
    using G = Cfg<NG>;
    constexpr int NW = kThreads / 32;
    const int smem = NG * G::CX * 8 + NW * a.nbins * 16;
    auto k = xpk_kernel<NG>;
    cudaError_t e = smem_attr_once((const void*)k, smem);
    if (e != cudaSuccess) return e;
    const int nchunks = cdiv(ncols, G::CX);
    k<<<nparts, kThreads, smem, s>>>(in, ncols, rs, ps, nchunks, tw, a, part_sum, part_cnt);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    pk_reduce_kernel<<<cdiv((size_t)a.nbins * 32, 256), 256, 0, s>>>(part_sum, part_cnt, nparts, a.nbins, sum, cnt);
    return cudaGetLastError();
}

bool fft_size_supported(int ng) {
    switch (ng) {
#define X(n) case n:
        HGPM_SIZES(X)
#undef X
        return true;
        default:
            return false;
    }
}

cudaError_t launch_zfwd(int ng, void* in, bool fixed, float2* out, int nlines, int zs, double mean,
                        const float2* tw, cudaStream_t s, const Slots& sl, int nslots) {
    switch (ng) {
#define X(n) \
    case n: return zfwd_impl<n>(in, fixed, out, nlines, zs, mean, tw, s, sl, nslots);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

bool plane_fft_supported(int ng) {
    switch (ng) {
#define X(n) \
    case n:  \
        return true;
        HGPM_PLANE_SIZES(X)
#undef X
    }
    return false;
}

static cudaError_t launch_plane(int ng, bool inv, void* a, float2* spec, int zs, double mean,
                                const float2* tw, cudaStream_t s) {
    switch (ng) {
#define X(n)                                                                          \
    case n:                                                                           \
        return plane_impl<n, 3>(inv, a, spec, zs, mean, tw, s);
        HGPM_PLANE_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_zy_fwd(int ng, unsigned long long* rho, float2* spec, int zs, double mean, const float2* tw,
                          cudaStream_t s) {
    return launch_plane(ng, false, rho, spec, zs, mean, tw, s);
}

cudaError_t launch_yz_inv_pair(int ng, float2* spec, float* out, int zs, const float2* tw, cudaStream_t s) {
    return launch_plane(ng, true, out, spec, zs, 0.0, tw, s);
}

cudaError_t launch_zinv(int ng, const float2* in, float* out, int nlines, int zs, size_t in_cs, size_t out_cs,
                        int ncomp, float scale, const float2* tw, cudaStream_t s, const Slots& sl, int nslots) {
    switch (ng) {
#define X(n) \
    case n: return zinv_impl<n>(in, out, nlines, zs, in_cs, out_cs, ncomp, scale, tw, s, sl, nslots);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

template <int NG>
static cudaError_t c2c_impl(float2* data, bool inv, const float2* tw, cudaStream_t s) {
    constexpr int L = CZ<NG>::L;
    const int nlines = NG * NG;
    auto kz = inv ? zpass_c2c_kernel<NG, true> : zpass_c2c_kernel<NG, false>;
    cudaError_t e = ensure_smem(kz, CZ<NG>::SMEM);
    if (e != cudaSuccess) return e;
    kz<<<cdiv(nlines, L), kThreads, CZ<NG>::SMEM, s>>>(data, nlines, tw);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // y lines (stride ng, planes x at ng^2), then x lines (stride ng^2,
    // planes y at ng); the z index is the contiguous column in both
    e = strided_impl<NG>(inv, data, NG, (size_t)NG, (size_t)NG * NG, NG, 0, 1, tw, s, Slots{}, 1);
    if (e != cudaSuccess) return e;
    return strided_impl<NG>(inv, data, NG, (size_t)NG * NG, (size_t)NG, NG, 0, 1, tw, s, Slots{}, 1);
}

cudaError_t launch_fft_c2c(int ng, float2* data, bool inv, const float2* tw, cudaStream_t s) {
    switch (ng) {
#define X(n) \
    case n: return c2c_impl<n>(data, inv, tw, s);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_zinv_pair(int ng, const float2* in, float* out, int zs, const float2* tw, cudaStream_t s) {
    switch (ng) {
#define X(n) \
    case n: return zinv_pair_impl<n>(in, out, n * n, zs, tw, s);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_strided(int ng, bool inv, float2* data, int ncols, size_t rs, size_t ps, int nplanes, size_t cs,
                           int ncomp, const float2* tw, cudaStream_t s, const Slots& sl, int nslots) {
    switch (ng) {
#define X(n) \
    case n: return strided_impl<n>(inv, data, ncols, rs, ps, nplanes, cs, ncomp, tw, s, sl, nslots);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_gradient(int ng, const float* phi, float4* f, cudaStream_t s, const Slots& sl, int nslots) {
    if (!fft_size_supported(ng)) return cudaErrorInvalidValue;
    // eight x per thread from 64^3 (the thread count, ng^3 / 64, is then a
    // whole number of warps for ng a multiple of 16); one on smaller grids,
    // which need every thread they can get (ng^3 / 8 threads, ng a multiple
    // of 8).  Measured at 512^3: x runs of 4, 8 or 16 within 1 %, 0.04 ms
    // faster than one x per thread.
#define GV(XR, MB, U)                                                                      \
    {                                                                                      \
        const size_t nq = (size_t)(ng / XR) * ng * (ng / 8);                               \
        gradient_kernel<XR, MB, U><<<dim3(cdiv(nq, 256), nslots), 256, 0, s>>>(phi, f, ng, sl); \
    }
    if (ng % 16 == 0 && ng >= 64) GV(8, 3, 2)
    else GV(1, 1, 1)
#undef GV
    return cudaGetLastError();
}

cudaError_t launch_xpotential(int ng, const float2* in, float2* out, int ncols, size_t rs, size_t ps, int nplanes,
                              const float2* tw, const double* cosq, double coeff, cudaStream_t s, const Slots& sl,
                              int nslots) {
    PotentialOp op{cosq, coeff};
    switch (ng) {
#define X(n) \
    case n: return xfused_impl<n, PotentialOp>(in, out, ncols, rs, ps, nplanes, 0, tw, op, s, sl, nslots);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

template <int NG>
static cudaError_t xpot_wide_impl(const float2* in, float2* out, int ncols, size_t rs, size_t ps, int nplanes,
                                  const float2* tw, const PotentialOp& op, cudaStream_t s) {
    constexpr int C = XW<NG>::C, SMEM = NG * C * 8;
    auto k = xpot_wide_kernel<NG>;
    cudaError_t e = ensure_smem(k, SMEM);
    if (e != cudaSuccess) return e;
    k<<<dim3(cdiv(ncols, C), nplanes), 512, SMEM, s>>>(in, out, ncols, rs, ps, tw, op);
    return cudaGetLastError();
}

cudaError_t launch_xpotential_wide(int ng, const float2* in, float2* out, int ncols, size_t rs, size_t ps, int nplanes,
                                   const float2* tw, const double* cosq, double coeff, cudaStream_t s) {
    PotentialOp op{cosq, coeff};
    switch (ng) {
#define X(n) \
    case n: return xpot_wide_impl<n>(in, out, ncols, rs, ps, nplanes, tw, op, s);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_xic(int n, const float2* in, float2* out, int ncols, size_t rs, size_t ps, int nplanes,
                       size_t out_cs, const float2* tw, const double* table, int nbins, double k_delta,
                       double pkscale, double inv_delta, const float* kf, int* err, cudaStream_t s) {
    ICOp op{table, nbins, k_delta, pkscale, inv_delta, kf, err, n / 2};
    switch (n) {
#define X(m) \
    case m: return xfused_impl<m, ICOp>(in, out, ncols, rs, ps, nplanes, out_cs, tw, op, s);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_xpk(int ng, const float2* in, int ncols, size_t rs, size_t ps, const float2* tw, const PkArgs& a,
                       double* part_sum, unsigned long long* part_cnt, int nparts, double* sum,
                       unsigned long long* cnt, cudaStream_t s) {
    switch (ng) {
#define X(n) \
    case n: return xpk_impl<n>(in, ncols, rs, ps, tw, a, part_sum, part_cnt, nparts, sum, cnt, s);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

int pk_max_bins() { return 1024; }

}  // namespace hgpm

// ===========================================================================
// Multi-class FFT passes (multi_class.h): one launch per pass over the work
// units of every class and slot, one CTA per unit.  The body is the one the
// single-class kernel runs (the z passes with 256 threads, the y and x passes
// with 512, for every size: a butterfly's arithmetic does not depend on which
// thread does it).
// ===========================================================================
namespace hgpm {

namespace {

// Threads and minimum CTAs per SM of each pass.  z passes: 256 threads, 3
// CTAs per SM (80 registers; the forward pass with half-height tiles from
// 192 up, MCCols::ZL, which bounds its register staging: 0.283 against
// 0.326 ms per ensemble step at 2 CTAs of 128 registers; the inverse 0.156
// against 0.184).  y and x passes: 512 x 2 (62 / 64 registers;
// the single-class configuration at 128^3 and above; 256 x 2 at 101 / 104
// registers measured the same at the 96-box ensemble).
constexpr int kMCYX = 512;
template <int PASS> constexpr int mc_threads() { return PASS == 0 || PASS == 4 ? 256 : kMCYX; }
template <int PASS> constexpr int mc_minb() { return PASS == 0 || PASS == 4 ? 3 : 2; }

// Columns per y / x tile.  Up to 128 a plane's ng/2 + 1 columns are split
// into the fewest even-width tiles that keep a stage at about two radix-8
// butterflies per thread (NG C <= 8192): the Nyquist column gets no tile of
// its own, which left most of a last tile empty (at 64: 33 columns in tiles
// of 16 or 32).  Larger sides keep the single-class widths.
template <int NG> struct MCCols {
    static constexpr int NC = NG / 2 + 1;
    static constexpr int TILES = ((NC + 1) / 2 * 2 * NG + 8191) / 8192;
    static constexpr int EVEN = ((NC + TILES - 1) / TILES + 1) / 2 * 2;
    static constexpr int Y = NG <= 128 ? EVEN : Cfg<NG>::CS;
    static constexpr int X = NG <= 128 ? EVEN : XW<NG>::C;
    // z lines per forward z tile: half the single-class count from 192 up,
    // which bounds the pass's register staging by the smaller sides'
    static constexpr int ZL = NG >= 192 ? Cfg<NG>::L / 2 : Cfg<NG>::L;
};

// One unit of each pass for one grid side.
template <int NG>
__device__ __forceinline__ void mc_zfwd_unit(const MCClass& c, int slot, int lu) {
    zpass_r2c_body<NG, true, MCCols<NG>::ZL>(c.rho64 + (size_t)slot * c.ncell, c.spec + (size_t)slot * c.spec_elems,
                                             NG * NG, c.zs, c.mean, c.tw, lu);
}
template <int NG, bool INV>
__device__ __forceinline__ void mc_ypass_unit(const MCClass& c, int slot, int lu) {
    float2* data = INV ? c.fspec + (size_t)slot * 3 * c.spec_elems : c.spec + (size_t)slot * c.spec_elems;
    constexpr int ncols = NG / 2 + 1, nch = (ncols + MCCols<NG>::Y - 1) / MCCols<NG>::Y;
    strided_body<NG, INV, kMCYX, MCCols<NG>::Y>(data, ncols, (size_t)c.zs, (size_t)NG * c.zs, c.tw, lu % nch,
                                                 lu / nch);
}
template <int NG>
__device__ __forceinline__ void mc_xpot_unit(const MCClass& c, int slot, int lu) {
    constexpr int ncols = NG / 2 + 1, nch = (ncols + MCCols<NG>::X - 1) / MCCols<NG>::X;
    const PotentialOp op{c.cosq, 0.5 / ((double)NG * NG * NG)};
    xone_body<NG, kMCYX, PotentialOp, MCCols<NG>::X>(c.spec + (size_t)slot * c.spec_elems, c.fspec + (size_t)slot * 3 * c.spec_elems, ncols,
                       (size_t)NG * c.zs, (size_t)c.zs, c.tw, op, lu % nch, lu / nch);
}
template <int NG>
__device__ __forceinline__ void mc_zinv_unit(const MCClass& c, int slot, int lu) {
    zpass_c2r_body<NG, true>(c.fspec + (size_t)slot * 3 * c.spec_elems, c.force + (size_t)slot * c.force_elems,
                             NG * NG, c.zs, 1.0f, c.tw, lu);
}

// PASS: 0 z forward, 1 y forward, 2 x with the Green's function, 3 y
// inverse, 4 z inverse.  One CTA per unit: CTA u of the launch is unit u -
// u0[k] of class k (slot (u - u0[k]) / per[k]).  (A persistent grid whose CTAs
// each serve one class ran 1.7-2.2x slower at the 96-box ensemble: CTAs
// shared out by points per unit starve the small sides, whose tiles cost
// nearly as much as large ones; the block scheduler balances by itself.)
template <int PASS>
__global__ void __launch_bounds__(mc_threads<PASS>(), mc_minb<PASS>()) mc_fft_kernel(const __grid_constant__ MCTable t) {
    const int u = blockIdx.x;
    int k = 0;
    while (k + 1 < t.n && u >= t.u0[k + 1]) ++k;
    const MCClass& c = t.c[k];
    const int r = u - t.u0[k], slot = r / t.per[k], lu = r - slot * t.per[k];
    if (c.active && !c.active[slot]) return;
    switch (c.ng) {
#define X(n)                                                     \
    case n:                                                      \
        if (PASS == 0) mc_zfwd_unit<n>(c, slot, lu);             \
        else if (PASS == 1) mc_ypass_unit<n, false>(c, slot, lu); \
        else if (PASS == 2) mc_xpot_unit<n>(c, slot, lu);        \
        else if (PASS == 3) mc_ypass_unit<n, true>(c, slot, lu); \
        else mc_zinv_unit<n>(c, slot, lu);                       \
        break;
        HGPM_MC_SIZES(X)
#undef X
    }
}

// Per-size unit counts and shared memory of the passes (host).
struct MCPassGeom {
    int zfunits, zunits, yunits, xunits;  // per slot (z forward, z inverse, y, x)
    int zsmem, ysmem, xsmem;
};
MCPassGeom mc_geom(int ng) {
    switch (ng) {
#define X(n)                                                                                            \
    case n: {                                                                                           \
        const int ncols = n / 2 + 1;                                                                    \
        return MCPassGeom{(n * n + MCCols<n>::ZL - 1) / MCCols<n>::ZL, (n * n + Cfg<n>::L - 1) / Cfg<n>::L,  \
                          (ncols + MCCols<n>::Y - 1) / MCCols<n>::Y * n,                                 \
                          (ncols + MCCols<n>::X - 1) / MCCols<n>::X * n, Cfg<n>::ZSMEM,                   \
                          n * MCCols<n>::Y * 8, n * MCCols<n>::X * 8};                                   \
    }
        HGPM_MC_SIZES(X)
#undef X
    }
    return MCPassGeom{0, 0, 0, 0, 0, 0, 0};
}

// One launch of `kern` (`threads` per CTA, `smem` bytes), one CTA per unit
// of every class's slots.
cudaError_t mc_launch(const void* kern, MCTable t, const int* units, int threads, int smem, cudaStream_t s) {
    t.u0[0] = 0;
    for (int k = 0; k < t.n; ++k) {
        t.per[k] = units[k];
        t.u0[k + 1] = t.u0[k] + units[k] * t.c[k].nslots;
    }
    if (t.u0[t.n] == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    void* args[] = {&t};
    return cudaLaunchKernel(kern, dim3(t.u0[t.n]), dim3(threads), args, smem, s);
}

}  // namespace

cudaError_t mc_launch_fft_passes(const MCTable& base, cudaStream_t s) {
    int zf[kMaxMC], zu[kMaxMC], yu[kMaxMC], xu[kMaxMC];
    int zs = 0, ys = 0, xs = 0;
    for (int k = 0; k < base.n; ++k) {
        const MCPassGeom g = mc_geom(base.c[k].ng);
        if (!g.zunits) return cudaErrorInvalidValue;
        zf[k] = g.zfunits;
        zu[k] = g.zunits;
        yu[k] = g.yunits;
        xu[k] = g.xunits;
        zs = g.zsmem > zs ? g.zsmem : zs;
        ys = g.ysmem > ys ? g.ysmem : ys;
        xs = g.xsmem > xs ? g.xsmem : xs;
    }
    cudaError_t e = mc_launch((const void*)mc_fft_kernel<0>, base, zf, mc_threads<0>(), zs, s);
    if (e == cudaSuccess) e = mc_launch((const void*)mc_fft_kernel<1>, base, yu, mc_threads<1>(), ys, s);
    if (e == cudaSuccess) e = mc_launch((const void*)mc_fft_kernel<2>, base, xu, mc_threads<2>(), xs, s);
    if (e == cudaSuccess) e = mc_launch((const void*)mc_fft_kernel<3>, base, yu, mc_threads<3>(), ys, s);
    if (e == cudaSuccess) e = mc_launch((const void*)mc_fft_kernel<4>, base, zu, mc_threads<4>(), zs, s);
    return e;
}

}  // namespace hgpm
