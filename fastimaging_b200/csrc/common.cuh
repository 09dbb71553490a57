// Shared device/host helpers of the B200 imager and source finder.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/stpgpu.h"

namespace stpgpu {

// Error carrying status + message through the host orchestration.
struct Error {
    stpgpu_status status;
    std::string msg;
};

#define STPGPU_CUDA_TRY(expr)                                                                                        \
    do {                                                                                                             \
        cudaError_t _e = (expr);                                                                                     \
        if (_e != cudaSuccess) {                                                                                     \
            throw ::stpgpu::Error { _e == cudaErrorMemoryAllocation ? STPGPU_ERR_OOM : STPGPU_ERR_CUDA,              \
                std::string(#expr) + ": " + cudaGetErrorString(_e) };                                                \
        }                                                                                                            \
    } while (0)

// Kernel launches of the current API call (reported in the call's info).
inline thread_local int g_launches = 0;
#define STPGPU_CHECK_LAUNCH()                                                                                        \
    do {                                                                                                             \
        ++::stpgpu::g_launches;                                                                                      \
        STPGPU_CUDA_TRY(cudaGetLastError());                                                                         \
    } while (0)

inline void fail(stpgpu_status s, const std::string& m) { throw Error { s, m }; }

constexpr int kTopHat = 0, kTriangle = 1, kSinc = 2, kGaussian = 3, kGaussianSinc = 4, kPSWF = 5;

// __grdsf, src/stp/convolution/conv_func.cpp:112-182 (one element).
__host__ __device__ inline double grdsf(double nu)
{
    const double p0[5] = { 8.203343e-2, -3.644705e-1, 6.278660e-1, -5.335581e-1, 2.312756e-1 };
    const double p1[5] = { 4.028559e-3, -3.697768e-2, 1.021332e-1, -1.201436e-1, 6.412774e-2 };
    const double q0[3] = { 1.0000000e0, 8.212018e-1, 2.078043e-1 };
    const double q1[3] = { 1.0000000e0, 9.599102e-1, 2.918724e-1 };
    nu = fabs(nu);
    const double* p;
    const double* q;
    double nuend;
    if (nu >= 0.0 && nu < 0.75) {
        p = p0;
        q = q0;
        nuend = 0.75;
    } else if (nu >= 0.75 && nu <= 1.0) {
        p = p1;
        q = q1;
        nuend = 1.0;
    } else {
        p = p0;
        q = q0;
        nuend = 0.0;
    }
    const double d = nu * nu - nuend * nuend;
    double top = p[0], bot = q[0], dk = 1.0;
    for (int k = 1; k < 5; k++) {
        dk *= d;
        top += p[k] * dk;
        if (k < 3)
            bot += q[k] * dk;
    }
    return bot > 0.0 ? top / bot : 0.0;
}

// Kernel functors as ImageVisibilities builds them (src/stp/imager/imager.cpp:25-64),
// src/stp/convolution/conv_func.cpp:11-196; `trunc` is the functor argument
// (truncation radius, or half_base_width for TopHat/Triangle).
__host__ __device__ inline double kernel_value(int kf, double trunc, double r)
{
    const double pi = 3.141592653589793238462643383279502884;
    switch (kf) {
    case kTopHat:
        return fabs(r) < trunc ? 1.0 : 0.0;
    case kTriangle: {
        double v = 1.0 - fabs(r) / trunc;
        return v > 0.0 ? v : 0.0;
    }
    case kSinc: {
        double x = r * (pi / 1.0);
        if (x == 0.0)
            x = 1.0e-20;
        double v = sin(x) / x;
        return (trunc > 0.0 && fabs(r) > trunc) ? 0.0 : v;
    }
    case kGaussian: {
        double v = exp((-1.0 / (1.0 * 1.0)) * (r * r));
        return (trunc > 0.0 && fabs(r) > trunc) ? 0.0 : v;
    }
    case kGaussianSinc: {
        const double wg = 2.52, ws = 1.55;
        double g = exp((-1.0 / (wg * wg)) * (r * r));
        double x = r * (pi / ws);
        if (x == 0.0)
            x = 1.0e-20;
        double v = g * (sin(x) / x);
        return (trunc > 0.0 && fabs(r) > trunc) ? 0.0 : v;
    }
    case kPSWF: {
        double nu = r / trunc;
        double v = grdsf(nu) * (1 - nu * nu);
        return (trunc > 0.0 && fabs(r) > trunc) ? 0.0 : v;
    }
    }
    return 0.0;
}

// Analytic grid-correction functions, conv_func.cpp:18-22,37-41,62-67,85-89,106-110,199-202.
// TopHat/Triangle/GaussianSinc return the radius itself (the reference's
// release-build behaviour of `assert(false); return radius;`).
__host__ __device__ inline double gcf_value(int kf, double r)
{
    const double pi = 3.141592653589793238462643383279502884;
    switch (kf) {
    case kSinc:
        return fabs(r) < 1.0 ? 1.0 : 0.0;
    case kGaussian: {
        double t = r * pi / (1.0 * 2);
        return exp(-1.0 * (t * t));
    }
    case kPSWF:
        return grdsf(r);
    default:
        return r;
    }
}

// Bessel function of the first kind, order 1, as the reference evaluates it
// for its discrete Hankel transform (besselj1, src/stp/gridder/aw_projection.cpp:490-508):
// the published rational approximation (Hart's coefficients, as tabulated in
// Numerical Recipes' bessj1; about 1e-8 absolute accuracy) for x < 8, and
// the asymptotic form sqrt(2/(pi x)) (P cos(x - 3pi/4) - z Q sin(x - 3pi/4)),
// z = 8/x, above.  The coefficients must be the reference's for identical
// W-kernels.  Arguments are >= 0 on this path.
__host__ __device__ inline double besselj1_ref(double x)
{
    if (x < 8.0) {
        const double num[6] = { 72362614232.0, -7895059235.0, 242396853.1, -2972611.439, 15704.48260, -30.16036606 };
        const double den[6] = { 144725228442.0, 2300535178.0, 18583304.74, 99447.43394, 376.9991397, 1.0 };
        const double xx = x * x;
        double p = num[5], q = den[5];
        for (int k = 4; k >= 0; k--) {
            p = num[k] + xx * p;
            q = den[k] + xx * q;
        }
        return (x * p) / q;
    }
    const double a[5] = { 1.0, 0.183105e-2, -0.3516396496e-4, 0.2457520174e-5, -0.240337019e-6 };
    const double b[5] = { 0.04687499995, -0.2002690873e-3, 0.8449199096e-5, -0.88228987e-6, 0.105787412e-6 };
    const double z = 8.0 / x;
    const double zz = z * z;
    const double y = x - 2.356194491;
    double p = a[4], q = b[4];
    for (int k = 3; k >= 0; k--) {
        p = a[k] + zz * p;
        q = b[k] + zz * q;
    }
    return sqrt(0.636619772 / x) * (cos(y) * p - z * sin(y) * q);
}

// Maximum radius (in pixels) beyond which every functor is exactly zero.
__host__ __device__ inline double kernel_zero_beyond(int kf, double trunc) { return trunc; }

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

} // namespace stpgpu
