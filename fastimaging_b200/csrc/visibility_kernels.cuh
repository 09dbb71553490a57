// Model visibilities of a point-source sky (stp/visibility/visibility.cpp:15-40):
//   vis(k) = sum_s flux_s * n_s * exp(-2 pi i * (uvw(k) . -(l_s, m_s, n_s - 1))),
//   n_s = sqrt(1 - l_s^2 - m_s^2),
// accumulated over the sources in sky-model order.  FP64 throughout.
#pragma once

#include "common.cuh"

namespace stpgpu {

constexpr int VIS_THREADS = 256;
constexpr int VIS_SRC_CHUNK = 512;

// One thread per visibility; the sky model is staged through shared memory
// in chunks.  subtract != 0: out = in - model (residual visibilities,
// reduce.cpp:113-122), else out = model.  vis arrays are interleaved complex;
// vin may alias out (each thread reads its element before writing it).
__global__ void __launch_bounds__(VIS_THREADS) k_model_vis(const double* __restrict__ sky, int n_src,
    const double* __restrict__ uvw, int64_t n, const double* vin, int subtract, double* out)
{
    __shared__ double s_l[VIS_SRC_CHUNK], s_m[VIS_SRC_CHUNK], s_f[VIS_SRC_CHUNK], s_n[VIS_SRC_CHUNK];
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    double u = 0.0, v = 0.0, w = 0.0;
    if (k < n) {
        u = uvw[k];
        v = uvw[n + k];
        w = uvw[2 * n + k];
    }
    const double two_pi = 2.0 * 3.141592653589793238462643383279502884;
    double re = 0.0, im = 0.0;
    for (int c0 = 0; c0 < n_src; c0 += VIS_SRC_CHUNK) {
        const int cn = min(VIS_SRC_CHUNK, n_src - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < cn; t += blockDim.x) {
            const double l = sky[c0 + t], m = sky[n_src + c0 + t];
            s_l[t] = l;
            s_m[t] = m;
            s_f[t] = sky[2 * n_src + c0 + t];
            s_n[t] = sqrt(1.0 - l * l - m * m);
        }
        __syncthreads();
        if (k < n) {
            for (int t = 0; t < cn; t++) {
                // dist_uvw * src_offset with src_offset = -(l, m, n - 1)
                const double dot = __dadd_rn(__dadd_rn(__dmul_rn(u, -s_l[t]), __dmul_rn(v, -s_m[t])),
                    __dmul_rn(w, -(s_n[t] - 1.0)));
                // exp(cx(0, -2 pi) * dot) = cos(theta) + i sin(theta), theta = -2 pi * dot
                double sn, cs;
                sincos(__dmul_rn(-two_pi, dot), &sn, &cs);
                const double a = __dmul_rn(s_f[t], s_n[t]);
                re = __dadd_rn(re, __dmul_rn(a, cs));
                im = __dadd_rn(im, __dmul_rn(a, sn));
            }
        }
    }
    if (k < n) {
        if (subtract) {
            out[2 * k] = vin[2 * k] - re;
            out[2 * k + 1] = vin[2 * k + 1] - im;
        } else {
            out[2 * k] = re;
            out[2 * k + 1] = im;
        }
    }
}

} // namespace stpgpu
