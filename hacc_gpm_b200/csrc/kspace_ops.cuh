// kspace_ops.cuh — k-space operators applied by the fused x passes:
// pre() once per mode on the forward-transformed x line, comp(d) per output
// component before the inverse x transform.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace hgpm {

// ---------------------------------------------------------------------------
// k-space operators
// ---------------------------------------------------------------------------
// Green's function of calcGreens (calcGreens.hpp:11-25): the x pass forms
// the potential's spectrum t = G rho_k and transforms it back along x (one
// output).  cosq[i] = cos(k_i) - 1 (double) is tabulated once per grid side;
// G is formed in double from the sum of the (non-positive) cosq terms, so
// there is no cancellation near k = 0.  The gradient of kspace_solve_gradient
// (kspace_solver.cu:55-90), -i sin(k_d) t, is applied in real space after
// the inverse transform (gradient_kernel: the central difference
// (phi(x - e_d) - phi(x + e_d)) / 2 multiplies mode k by exactly
// -i sin(2 pi k_d / ng)).
struct PotentialOp {
    static constexpr int kOut = 1;
    const double* cosq;  // cos(k_i) - 1, one entry per grid index
    double coeff;        // 0.5 / ng^3
    __device__ __forceinline__ float2 pre(int ix, int iy, int iz, float2 v) const {
        const double s = __ldg(&cosq[ix]) + __ldg(&cosq[iy]) + __ldg(&cosq[iz]);
        const float g = (s == 0.0) ? 0.f : (float)(coeff / s);
        // explicit roundings: the product is never contracted into the
        // butterfly arithmetic around it, so every kernel that applies this
        // operator between its transforms gets the same bits
        return make_float2(__fmul_rn(v.x, g), __fmul_rn(v.y, g));
    }
    __device__ __forceinline__ float2 comp(int, int, int, int, float2 t) const { return t; }
};

// Zel'dovich displacement (initializer.cpp:10-117): ScaleAmplitudes by
// sqrt(P(|k|) n^3/rl^3) from the .ipk table (interpolation_initializer.cu:3-30),
// then transformDensityField (transform_density_field_initializer.cu:72-112):
// s_d = (Im k_d, -Re k_d) / (k^2 delta).
struct ICOp {
    static constexpr int kOut = 3;  // the x pass stores all three components
    const double* table;
    int nbins;
    double k_delta;
    double pkscale;    // n^3 / rl^3
    double inv_delta;  // 1 / delta
    const float* kf;   // float(signed(i) * 2 pi / rl)
    int* err;          // set when |k| runs past the table
    __device__ __forceinline__ float2 pre(int ix, int iy, int iz, float2 v) const {
        const float kx = __ldg(&kf[ix]), ky = __ldg(&kf[iy]), kz = __ldg(&kf[iz]);
        const float k2f = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
        double y = 0.0;
        if (!(ix == 0 && iy == 0 && iz == 0)) {
            const double my_k = (double)__fsqrt_rn(k2f);
            const int left = (int)(my_k / k_delta);
            const int right = left + 1;
            if (right >= nbins) {
                atomicExch(err, 1);
            } else if (left == 0) {
                y = __ldg(&table[right]) * pkscale;
            } else {
                const double ly1 = log(__ldg(&table[left]));
                const double lx1 = log(k_delta * (double)left);
                const double ly2 = log(__ldg(&table[right]));
                const double lx2 = log(k_delta * (double)right);
                const double lx = log(my_k);
                y = exp(ly1 + ((ly2 - ly1) / (lx2 - lx1)) * (lx - lx1)) * pkscale;
            }
        }
        const double sc = sqrt(y);
        v.x = (float)((double)v.x * sc);
        v.y = (float)((double)v.y * sc);
        const double k2 = (double)k2f;
        const double mul = inv_delta * (k2 == 0.0 ? 0.0 : 1.0 / k2);
        v.x = (float)((double)v.x * mul);
        v.y = (float)((double)v.y * mul);
        return v;
    }
    int nyq;           // n / 2
    __device__ __forceinline__ float2 comp(int d, int ix, int iy, int iz, float2 t) const {
        const int id = d == 0 ? ix : (d == 1 ? iy : iz);
        if (id == nyq) return make_float2(0.f, 0.f);
        const float kd = __ldg(&kf[id]);
        return make_float2(t.y * kd, -t.x * kd);
    }
};

}  // namespace hgpm
