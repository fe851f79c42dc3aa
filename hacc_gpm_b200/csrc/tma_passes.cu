// tma_passes.cu — strided FFT passes (y lines, and x lines for the plain
// transforms) as persistent kernels fed by TMA.
//
// Each CTA walks tiles t = blockIdx.x, +gridDim.x, ...; a tile is NG rows
// (the FFT axis) by CT contiguous complex columns of one plane of one
// component.  Thread 0 issues cp.async.bulk.tensor loads of the NEXT tile
// into the other shared-memory buffer (completion on an mbarrier with a
// transaction count) while all threads transform the current tile; the
// result goes back with a cp.async.bulk.tensor store.  The tensor map's
// inner extent is the valid half-spectrum width (ng/2 + 1 complex), so the
// ragged last column chunk is zero-filled on load and clipped on store.
// No multicast is used anywhere.  Every mbarrier wait is bounded: on time-out
// the CTA records an error, waits (bounded) for its own copies and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_engine.cuh"
#include "hgpm_device.cuh"
#include "hgpm_internal.h"
#include "kspace_ops.cuh"
#include "tma_util.cuh"

namespace hgpm {

// ISX = false: lines along y (tensor dim 1), plane = x (dim 2).
// ISX = true : lines along x (tensor dim 2), plane = y (dim 1).
template <int NG, bool ISX>
__device__ __forceinline__ void issue_tile_load(const CUtensorMap* tm, float2* buf, uint64_t* bar, const TileIdx& ti) {
    using G = TmaCfg<NG>;
    mbar_expect_tx(bar, G::TILE_BYTES);
    const int c0 = 2 * G::CT * ti.chunk;
#pragma unroll
    for (int b = 0; b < G::NBOX; ++b) {
        float2* dst = buf + (size_t)b * G::RB * G::CT;
        if (ISX) tma_load_4d(dst, tm, c0, ti.plane, b * G::RB, ti.comp, bar);
        else tma_load_4d(dst, tm, c0, b * G::RB, ti.plane, ti.comp, bar);
    }
}

template <int NG, bool ISX>
__device__ __forceinline__ void issue_tile_store(const CUtensorMap* tm, const float2* buf, const TileIdx& ti) {
    using G = TmaCfg<NG>;
    const int c0 = 2 * G::CT * ti.chunk;
#pragma unroll
    for (int b = 0; b < G::NBOX; ++b) {
        const float2* src = buf + (size_t)b * G::RB * G::CT;
        if (ISX) tma_store_4d(tm, c0, ti.plane, b * G::RB, ti.comp, src);
        else tma_store_4d(tm, c0, b * G::RB, ti.plane, ti.comp, src);
    }
    bulk_commit();
}

template <int NG, bool INV, bool ISX>
__global__ void __launch_bounds__(kTmaThreads, 2) strided_tma_kernel(const __grid_constant__ CUtensorMap tm, int nchunks,
                                                                  int nplanes, int ncomp, const float2* __restrict__ tw,
                                                                  int* __restrict__ err) {
    using G = TmaCfg<NG>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float2* buf[2] = {reinterpret_cast<float2*>(base), reinterpret_cast<float2*>(base + G::TILE_BYTES)};
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int failed;
    const int ntiles = nchunks * nplanes * ncomp;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        failed = 0;
        fence_async_shared();
    }
    __syncthreads();
    int t = blockIdx.x;
    if (threadIdx.x == 0 && t < ntiles) issue_tile_load<NG, ISX>(&tm, buf[0], &bar[0], tile_of(t, nchunks, nplanes));
    int j = 0;
    bool next_in_flight = false;
    for (; t < ntiles; t += gridDim.x, ++j) {
        const int cur = j & 1;
        const int tn = t + gridDim.x;
        if (threadIdx.x == 0) {
            next_in_flight = false;
            if (tn < ntiles) {
                // the other buffer was stored from in the previous iteration
                bulk_wait_read_all();
                issue_tile_load<NG, ISX>(&tm, buf[cur ^ 1], &bar[cur ^ 1], tile_of(tn, nchunks, nplanes));
                next_in_flight = true;
            }
            if (!mbar_wait_bounded(&bar[cur], (j >> 1) & 1)) failed = 1;
        }
        __syncthreads();
        if (failed) break;
        fft_tile<NG, G::CT, G::CT, INV, kTmaThreads>(buf[cur], tw);
        fence_async_shared();
        __syncthreads();
        if (threadIdx.x == 0) issue_tile_store<NG, ISX>(&tm, buf[cur], tile_of(t, nchunks, nplanes));
    }
    if (threadIdx.x == 0) {
        if (failed) {
            atomicExch(err, 1);
            // the current load never completed; also drain the prefetched one
            mbar_wait_bounded(&bar[j & 1], (j >> 1) & 1);
            if (next_in_flight) mbar_wait_bounded(&bar[(j + 1) & 1], ((j + 1) >> 1) & 1);
        }
        bulk_wait_all();
    }
}

// ---------------------------------------------------------------------------
// x pass fused with the Green's function, persistent and TMA-fed: the next
// x-line tile (all kx of one ky, CT kz columns) streams in while the current
// one is transformed forward, multiplied by G (calcGreens.hpp:11-25, as
// PotentialOp::pre) and transformed back; the potential's x-inverted spectrum
// leaves with coalesced streaming stores.
template <int NG, int CT, int NT>
__device__ __forceinline__ void store_rows(const float2* __restrict__ tile, float2* __restrict__ g, size_t rs,
                                           int nvalid) {
    constexpr int TPR = CT / 2;
    constexpr int TOT = NG * TPR;
#pragma unroll 4
    for (int i = threadIdx.x; i < TOT; i += NT) {
        const int e = i / TPR, c = 2 * (i % TPR);
        const float4 v = *reinterpret_cast<const float4*>(&tile[e * CT + c]);
        float2* dst = g + (size_t)e * rs + c;
        if (c + 1 < nvalid) __stcs(reinterpret_cast<float4*>(dst), v);
        else if (c < nvalid) dst[0] = make_float2(v.x, v.y);
    }
}

template <int NG, int NT>
__global__ void __launch_bounds__(NT, 768 / NT) xpotential_tma_kernel(const __grid_constant__ CUtensorMap tm,
                                                                       float2* __restrict__ out, int ncols, int zs,
                                                                       int nchunks, const float2* __restrict__ tw,
                                                                       const double* __restrict__ cosq_g,
                                                                       double coeff, int* __restrict__ err) {
    using G = TmaCfg<NG>;
    constexpr int CT = G::CT;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float2* in[2] = {reinterpret_cast<float2*>(base), reinterpret_cast<float2*>(base + G::TILE_BYTES)};
    double* cosq = reinterpret_cast<double*>(base + 2 * G::TILE_BYTES);
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int failed;
    const int ntiles = nchunks * NG;
    for (int i = threadIdx.x; i < NG; i += NT) cosq[i] = cosq_g[i];
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        failed = 0;
        fence_async_shared();
    }
    __syncthreads();
    int t = blockIdx.x;
    if (threadIdx.x == 0 && t < ntiles) issue_tile_load<NG, true>(&tm, in[0], &bar[0], tile_of(t, nchunks, NG));
    int j = 0;
    bool next_in_flight = false;
    const size_t rs = (size_t)NG * zs;
    for (; t < ntiles; t += gridDim.x, ++j) {
        const int cur = j & 1;
        const int tn = t + gridDim.x;
        if (threadIdx.x == 0) {
            next_in_flight = false;
            if (tn < ntiles) {
                issue_tile_load<NG, true>(&tm, in[cur ^ 1], &bar[cur ^ 1], tile_of(tn, nchunks, NG));
                next_in_flight = true;
            }
            if (!mbar_wait_bounded(&bar[cur], (j >> 1) & 1)) failed = 1;
        }
        __syncthreads();
        if (failed) break;
        const TileIdx ti = tile_of(t, nchunks, NG);
        const int iy = ti.plane, col0 = ti.chunk * CT;
        float2* tile = in[cur];
        // forward x FFT, t = G rho_k (PotentialOp::pre with the table in
        // shared memory, in registers between the two transforms), the
        // potential's inverse x FFT; the gradient is taken in real space
        // (gradient_kernel)
        const double cy = cosq[iy];
        fft_tile_fwd_op_inv<NG, CT, CT, NT, 1, true>(tile, tw, [&](int ix, int c, float2 v) {
            const int iz = col0 + c;
            if (iz >= ncols) return make_float2(0.f, 0.f);
            const double sum = cosq[ix] + cy + cosq[iz];
            const float g = (sum == 0.0) ? 0.f : (float)(coeff / sum);
            return make_float2(__fmul_rn(v.x, g), __fmul_rn(v.y, g));  // as PotentialOp::pre
        });
        store_rows<NG, CT, NT>(tile, out + (size_t)iy * zs + col0, rs, ncols - col0);
        // the next TMA load into this buffer follows generic-proxy writes
        fence_async_shared();
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (failed) {
            atomicExch(err, 1);
            mbar_wait_bounded(&bar[j & 1], (j >> 1) & 1);
            if (next_in_flight) mbar_wait_bounded(&bar[(j + 1) & 1], ((j + 1) >> 1) & 1);
        }
    }
}

// ---------------------------------------------------------------------------
// The time-out path of the passes' bounded waits, for tests: thread 0 arms an
// mbarrier for a 16-byte copy that is never issued, polls it `polls` times
// as the passes do, and on time-out sets the error flag and returns (no
// fault, nothing left in flight).
__global__ void wait_timeout_probe_kernel(int* __restrict__ err, unsigned polls) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    fence_async_shared();
    mbar_expect_tx(&bar, 16u);
    bool done = false;
    for (unsigned i = 0; i < polls && !done; ++i) done = mbar_try_wait(&bar, 0);
    if (!done) atomicExch(err, 1);
}

cudaError_t launch_wait_timeout_probe(int* err, unsigned polls, cudaStream_t s) {
    wait_timeout_probe_kernel<<<1, 32, 0, s>>>(err, polls);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static bool encode_fn() {
    if (g_encode) return true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
        return false;
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    return true;
}

// Tensor map over a half-spectrum buffer: dims (2*ncols floats, ng, ng, ncomp),
// row stride zs complex, component stride cs complex.
cudaError_t make_spec_map(CUtensorMap* tm, float2* data, int ng, int ncols, int zs, size_t cs, int ncomp,
                                 int ct, int rb, bool isx) {
    if (!encode_fn()) return cudaErrorNotSupported;
    cuuint64_t dims[4] = {(cuuint64_t)(2 * ncols), (cuuint64_t)ng, (cuuint64_t)ng, (cuuint64_t)ncomp};
    cuuint64_t strides[3] = {(cuuint64_t)zs * 8, (cuuint64_t)ng * zs * 8, (cuuint64_t)(cs ? cs : (size_t)ng * ng * zs) * 8};
    cuuint32_t box[4] = {(cuuint32_t)(2 * ct), isx ? 1u : (cuuint32_t)rb, isx ? (cuuint32_t)rb : 1u, 1u};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = g_encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, data, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

static int g_num_sms = 0;

template <int NG>
static cudaError_t tma_impl(bool inv, bool isx, float2* data, int ncols, int zs, size_t cs, int ncomp,
                            const float2* tw, int* err, cudaStream_t s) {
    using G = TmaCfg<NG>;
    CUtensorMap tm;
    cudaError_t e = make_spec_map(&tm, data, NG, ncols, zs, cs, ncomp, G::CT, G::RB, isx);
    if (e != cudaSuccess) return e;
    if (!g_num_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    }
    const int nchunks = (ncols + G::CT - 1) / G::CT;
    const int ntiles = nchunks * NG * ncomp;
    // persistent grid: exactly the CTAs that are resident at once (no tail wave)
#define HGPM_TMA_LAUNCH(I, X)                                                                       \
    {                                                                                               \
        auto k = strided_tma_kernel<NG, I, X>;                                                      \
        e = smem_attr_once((const void*)k, G::SMEM);                                                \
        if (e != cudaSuccess) return e;                                                             \
        int grid = g_num_sms * blocks_per_sm_once((const void*)k, kTmaThreads, G::SMEM);           \
        if (grid > ntiles) grid = ntiles;                                                           \
        k<<<grid, kTmaThreads, G::SMEM, s>>>(tm, nchunks, NG, ncomp, tw, err);                      \
    }
    if (inv) {
        if (isx) HGPM_TMA_LAUNCH(true, true) else HGPM_TMA_LAUNCH(true, false)
    } else {
        if (isx) HGPM_TMA_LAUNCH(false, true) else HGPM_TMA_LAUNCH(false, false)
    }
#undef HGPM_TMA_LAUNCH
    return cudaGetLastError();
}

template <int NG>
static cudaError_t xpotential_tma_impl(float2* in, float2* out, int ncols, int zs, const float2* tw,
                                       const double* cosq, double coeff, int* err, cudaStream_t s) {
    using G = TmaCfg<NG>;
    constexpr int NT = 256;  // three CTAs per SM (0.55 ms at 512^3 against 0.60 with two of 512)
    CUtensorMap tm;
    cudaError_t e = make_spec_map(&tm, in, NG, ncols, zs, 0, 1, G::CT, G::RB, true);
    if (e != cudaSuccess) return e;
    if (!g_num_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    }
    constexpr int SMEM = 2 * G::TILE_BYTES + NG * 8 + 1024;
    const int nchunks = (ncols + G::CT - 1) / G::CT;
    const int ntiles = nchunks * NG;
    auto k = xpotential_tma_kernel<NG, NT>;
    e = smem_attr_once((const void*)k, SMEM);
    if (e != cudaSuccess) return e;
    int grid = g_num_sms * blocks_per_sm_once((const void*)k, NT, SMEM);
    if (grid > ntiles) grid = ntiles;
    k<<<grid, NT, SMEM, s>>>(tm, out, ncols, zs, nchunks, tw, cosq, coeff, err);
    return cudaGetLastError();
}

cudaError_t launch_xpotential_tma(int ng, float2* in, float2* out, int ncols, int zs, const float2* tw,
                                  const double* cosq, double coeff, int* err, cudaStream_t s) {
    switch (ng) {
#define X(n) \
    case n: return xpotential_tma_impl<n>(in, out, ncols, zs, tw, cosq, coeff, err, s);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_strided_tma(int ng, bool inv, bool isx, float2* data, int ncols, int zs, size_t cs, int ncomp,
                               const float2* tw, int* err, cudaStream_t s) {
    switch (ng) {
#define X(n) \
    case n: return tma_impl<n>(inv, isx, data, ncols, zs, cs, ncomp, tw, err, s);
        HGPM_SIZES(X)
#undef X
    }
    return cudaErrorInvalidValue;
}

}  // namespace hgpm
