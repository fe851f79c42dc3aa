// fft_engine.cuh — shared-memory tile FFT for the PM step.
//
// A tile is C independent complex lines of length N held in shared memory as
//   buf[e * ES + c]      e in [0, N) element, c in [0, C) line, ES >= C
// i.e. lines are columns with unit stride between lines.  Every pass kernel
// (z R2C/C2R lines, y and x strided lines) stages its data into this layout
// and calls fft_tile<>.  The transform is a Stockham autosort mixed-radix
// FFT (radices 2, 3, 4, 5, 8): each stage reads R values per butterfly into
// registers, synchronises, twiddles, does the radix-R DFT in registers and
// writes back in place in Stockham order.  Threads are mapped line-fastest
// so a half-warp touches 16 consecutive lines of one element (conflict-free
// 64-bit shared accesses).
//
// Twiddles come from a per-length table tw[m] = exp(-2 pi i m / L) computed
// on the host in double precision (no device transcendental functions);
// a transform of length N may use a table of length N*TWS (stride TWS).
#pragma once
#include <cuda_runtime.h>

namespace hgpm {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 rot90(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// ---- radix-R DFTs in registers (forward: exp(-2 pi i r m / R)) ----------
template <int R, bool INV> struct Dft;

template <bool INV> struct Dft<2, INV> {
    static __device__ __forceinline__ void run(float2* v) {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <bool INV> struct Dft<3, INV> {
    static __device__ __forceinline__ void run(float2* v) {
        const float s3 = 0.86602540378443864676f;  // sqrt(3)/2
        float2 t1 = cadd(v[1], v[2]);
        float2 t2 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
        float2 d = csub(v[1], v[2]);
        float2 t3 = make_float2(s3 * d.x, s3 * d.y);
        float2 rt3 = rot90<INV>(t3);  // -i*t3 forward, +i*t3 inverse
        v[0] = cadd(v[0], t1);
        v[1] = cadd(t2, rt3);
        v[2] = csub(t2, rt3);
    }
};

template <bool INV> struct Dft<4, INV> {
    static __device__ __forceinline__ void run(float2* v) {
        float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        float2 b0 = cadd(v[1], v[3]), b1 = rot90<INV>(csub(v[1], v[3]));
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1);
        v[3] = csub(a1, b1);
    }
};

// Radix 5 from the DFT definition: with t1 = v1 + v4, t2 = v2 + v3,
// t3 = v1 - v4, t4 = v2 - v3, c_k = cos(2 pi k/5), s_k = sin(2 pi k/5),
//   X0 = v0 + t1 + t2,
//   X1, X4 = a1 -+ i b1,  a1 = v0 + c1 t1 + c2 t2,  b1 = s1 t3 + s2 t4,
//   X2, X3 = a2 -+ i b2,  a2 = v0 + c2 t1 + c1 t2,  b2 = s2 t3 - s1 t4
// (forward, exp(-2 pi i jk/5); the inverse flips the sign of i).
template <bool INV> struct Dft<5, INV> {
    static __device__ __forceinline__ void run(float2* v) {
        const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
        const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
        const float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        const float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        const float2 a1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
        const float2 a2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
        const float2 b1 = rot90<INV>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
        const float2 b2 = rot90<INV>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
        v[0] = cadd(v[0], cadd(t1, t2));
        v[1] = cadd(a1, b1);
        v[4] = csub(a1, b1);
        v[2] = cadd(a2, b2);
        v[3] = csub(a2, b2);
    }
};

template <bool INV> struct Dft<8, INV> {
    static __device__ __forceinline__ void run(float2* v) {
        const float h = 0.70710678118654752440f;  // 1/sqrt(2)
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4, INV>::run(e);
        Dft<4, INV>::run(o);
        // o[m] *= w8^m, w8 = exp(-+ i pi/4)
        float2 o1 = INV ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                        : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
        float2 o2 = rot90<INV>(o[2]);
        float2 o3 = INV ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                        : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
};

// ---- one Stockham stage -------------------------------------------------
// NS = product of the radices of the previous stages.  TP: radix-4/8
// twiddles beyond the loaded powers formed as products (fewer loads, more
// registers; a pass whose registers are capped keeps TP false).
// Twiddles and radix-R DFT of butterfly k (k = j % NS) of a stage, in place
// on the R values of the butterfly.
template <int N, int NS, int R, bool INV, int TWS, bool TP>
__device__ __forceinline__ void stage_butterfly(float2* v, int k, const float2* __restrict__ tw) {
    if (NS > 1) {
        const int m = k * (N / (NS * R));  // twiddle r is tw[r * m]
        if (TP && (R == 8 || R == 4)) {
            // powers 1, 2 (and 4) from the table, the rest as products
            // (one extra rounding each): fewer loads per butterfly
            float2 w[R];
            w[1] = __ldg(&tw[TWS * m]);
            w[2] = __ldg(&tw[TWS * 2 * m]);
            w[3] = cmul(w[1], w[2]);
            if (R == 8) {
                w[4] = __ldg(&tw[TWS * 4 * m]);
                w[5] = cmul(w[1], w[4]);
                w[6] = cmul(w[2], w[4]);
                w[7] = cmul(w[3], w[4]);
            }
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = INV ? cmulc(v[r], w[r]) : cmul(v[r], w[r]);
        } else {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const float2 w = __ldg(&tw[TWS * (r * m)]);
                v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
            }
        }
    }
    Dft<R, INV>::run(v);
}

template <int N, int C, int ES, int NS, int R, bool INV, int NT, int TWS, bool TP>
__device__ __forceinline__ void fft_stage(float2* __restrict__ buf, const float2* __restrict__ tw) {
    constexpr int NB = N / R;        // butterflies per line
    constexpr int TOT = NB * C;      // butterflies in the tile
    constexpr int PER = (TOT + NT - 1) / NT;
    float2 v[PER][R];
    const int tid = threadIdx.x;
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int b = tid + t * NT;
        if ((TOT % NT) == 0 || b < TOT) {
            const int c = b % C, j = b / C;
#pragma unroll
            for (int r = 0; r < R; ++r) v[t][r] = buf[(j + r * NB) * ES + c];
        }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int b = tid + t * NT;
        if ((TOT % NT) == 0 || b < TOT) {
            const int c = b % C, j = b / C;
            const int k = j % NS;
            stage_butterfly<N, NS, R, INV, TWS, TP>(v[t], k, tw);
            const int base = (j / NS) * NS * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[(base + r * NS) * ES + c] = v[t][r];
        }
    }
    __syncthreads();
}

// The last stage of a forward transform, a per-mode operator and the first
// stage of the inverse transform in one pass.  With the forward radices
// R_1..R_L, the last forward stage (NS = N / R_L) leaves butterfly j's outputs
// at modes j + r N / R_L, which are exactly the inputs of butterfly j of an
// inverse stage of radix R_L with NS = 1; the inverse then runs the radices in
// reverse order.  So the operator is applied in registers and the tile makes
// one shared-memory round trip instead of three.  op(e, c, v): mode e of line
// c.
template <int N, int C, int ES, int R, int NT, int TWS, bool TP, class F>
__device__ __forceinline__ void fft_turn_stage(float2* __restrict__ buf, const float2* __restrict__ tw, const F& op) {
    constexpr int NB = N / R, NS = N / R;
    constexpr int TOT = NB * C;
    constexpr int PER = (TOT + NT - 1) / NT;
    float2 v[PER][R];
    const int tid = threadIdx.x;
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int b = tid + t * NT;
        if ((TOT % NT) == 0 || b < TOT) {
            const int c = b % C, j = b / C;
#pragma unroll
            for (int r = 0; r < R; ++r) v[t][r] = buf[(j + r * NB) * ES + c];
        }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int b = tid + t * NT;
        if ((TOT % NT) == 0 || b < TOT) {
            const int c = b % C, j = b / C;
            stage_butterfly<N, NS, R, false, TWS, TP>(v[t], j, tw);
#pragma unroll
            for (int r = 0; r < R; ++r) v[t][r] = op(j + r * NS, c, v[t][r]);
            stage_butterfly<N, 1, R, true, TWS, TP>(v[t], 0, tw);
#pragma unroll
            for (int r = 0; r < R; ++r) buf[(j * R + r) * ES + c] = v[t][r];
        }
    }
    __syncthreads();
}

template <int... Rs> struct RSeq {};

template <int N, int C, int ES, bool INV, int NT, int TWS, bool TP, int NS>
__device__ __forceinline__ void fft_stages(float2*, const float2*, RSeq<>) {}

template <int N, int C, int ES, bool INV, int NT, int TWS, bool TP, int NS, int R, int... Rs>
__device__ __forceinline__ void fft_stages(float2* buf, const float2* tw, RSeq<R, Rs...>) {
    fft_stage<N, C, ES, NS, R, INV, NT, TWS, TP>(buf, tw);
    fft_stages<N, C, ES, INV, NT, TWS, TP, NS * R>(buf, tw, RSeq<Rs...>{});
}

// Radix plans for the supported lengths (2^a 3^b 5^c, 8..1024; the grid
// sides and their halves, the z passes' complex lengths).
template <int N> struct Plan;
template <> struct Plan<8> { using type = RSeq<8>; };
template <> struct Plan<12> { using type = RSeq<3, 4>; };
template <> struct Plan<16> { using type = RSeq<4, 4>; };
template <> struct Plan<24> { using type = RSeq<3, 8>; };
template <> struct Plan<32> { using type = RSeq<8, 4>; };
template <> struct Plan<48> { using type = RSeq<3, 4, 4>; };
template <> struct Plan<64> { using type = RSeq<8, 8>; };
template <> struct Plan<96> { using type = RSeq<3, 8, 4>; };
template <> struct Plan<128> { using type = RSeq<8, 4, 4>; };
template <> struct Plan<192> { using type = RSeq<3, 8, 8>; };
template <> struct Plan<256> { using type = RSeq<8, 8, 4>; };
template <> struct Plan<384> { using type = RSeq<3, 8, 4, 4>; };
template <> struct Plan<512> { using type = RSeq<8, 8, 8>; };
template <> struct Plan<768> { using type = RSeq<3, 8, 8, 4>; };
template <> struct Plan<1024> { using type = RSeq<8, 8, 4, 4>; };
template <> struct Plan<20> { using type = RSeq<5, 4>; };
template <> struct Plan<40> { using type = RSeq<5, 8>; };
template <> struct Plan<60> { using type = RSeq<3, 5, 4>; };
template <> struct Plan<80> { using type = RSeq<5, 4, 4>; };
template <> struct Plan<100> { using type = RSeq<5, 5, 4>; };
template <> struct Plan<120> { using type = RSeq<3, 5, 8>; };
template <> struct Plan<160> { using type = RSeq<5, 8, 4>; };
template <> struct Plan<200> { using type = RSeq<5, 5, 8>; };
template <> struct Plan<240> { using type = RSeq<3, 5, 4, 4>; };
template <> struct Plan<320> { using type = RSeq<5, 8, 8>; };
template <> struct Plan<400> { using type = RSeq<5, 5, 4, 4>; };
template <> struct Plan<480> { using type = RSeq<3, 5, 8, 4>; };
template <> struct Plan<500> { using type = RSeq<5, 5, 5, 4>; };
template <> struct Plan<640> { using type = RSeq<5, 8, 4, 4>; };
template <> struct Plan<800> { using type = RSeq<5, 5, 8, 4>; };
template <> struct Plan<960> { using type = RSeq<3, 5, 8, 8>; };
template <> struct Plan<1000> { using type = RSeq<5, 5, 5, 8>; };

// Radix sequence helpers: all but the last radix, the last radix, reversal.
template <int R, class S> struct SeqCons;
template <int R, int... Ts> struct SeqCons<R, RSeq<Ts...>> { using type = RSeq<R, Ts...>; };
template <class S> struct SeqInit;
template <int R> struct SeqInit<RSeq<R>> { using type = RSeq<>; };
template <int R, int R2, int... Rs> struct SeqInit<RSeq<R, R2, Rs...>> {
    using type = typename SeqCons<R, typename SeqInit<RSeq<R2, Rs...>>::type>::type;
};
template <class S> struct SeqLast;
template <int R> struct SeqLast<RSeq<R>> { static constexpr int value = R; };
template <int R, int R2, int... Rs> struct SeqLast<RSeq<R, R2, Rs...>> {
    static constexpr int value = SeqLast<RSeq<R2, Rs...>>::value;
};
template <class S, class Acc = RSeq<>> struct SeqRev;
template <int... As> struct SeqRev<RSeq<>, RSeq<As...>> { using type = RSeq<As...>; };
template <int R, int... Rs, int... As> struct SeqRev<RSeq<R, Rs...>, RSeq<As...>> {
    using type = typename SeqRev<RSeq<Rs...>, RSeq<R, As...>>::type;
};

// Transform all C lines of the tile (natural order in, natural order out).
// Caller must __syncthreads() after filling the tile; returns synchronised.
template <int N, int C, int ES, bool INV, int NT, int TWS = 1, bool TP = true>
__device__ __forceinline__ void fft_tile(float2* buf, const float2* __restrict__ tw) {
    fft_stages<N, C, ES, INV, NT, TWS, TP, 1>(buf, tw, typename Plan<N>::type{});
}

// Forward transform, op(e, c, v) on every mode e of every line c, inverse
// transform (radices in reverse order), with the last forward and first
// inverse stages fused around op (fft_turn_stage).  Natural order in and out;
// caller synchronises after filling the tile; returns synchronised.
template <int N, int C, int ES, int NT, int TWS, bool TP, class F>
__device__ __forceinline__ void fft_tile_fwd_op_inv(float2* buf, const float2* __restrict__ tw, const F& op) {
    using P = typename Plan<N>::type;
    using Init = typename SeqInit<P>::type;
    constexpr int RL = SeqLast<P>::value;
    fft_stages<N, C, ES, false, NT, TWS, TP, 1>(buf, tw, Init{});
    fft_turn_stage<N, C, ES, RL, NT, TWS, TP>(buf, tw, op);
    fft_stages<N, C, ES, true, NT, TWS, TP, RL>(buf, tw, typename SeqRev<Init>::type{});
}

}  // namespace hgpm
