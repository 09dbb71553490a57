// CPU oracle for the FastImaging snapshot imager + source finder hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, loop by loop, the algorithms
// of the reference C++ library (SKA-ScienceDataProcessor/FastImaging, `src/stp/`)
// so that the CUDA product can be checked against it.  It is imported only by
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, always as
// the checker, never as the product path.
//
// Every function cites the reference file:line it follows.  FFTs are not done
// here: oracle/stp_oracle.py orchestrates these loops around scipy.fft.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum KernelFunction { kTopHat = 0, kTriangle = 1, kSinc = 2, kGaussian = 3, kGaussianSinc = 4, kPSWF = 5 };

// stp/convolution/conv_func.cpp:112-182 (__grdsf), one element.
double grdsf_one(double nu)
{
    static const double p[2][5] = { { 8.203343e-2, -3.644705e-1, 6.278660e-1, -5.335581e-1, 2.312756e-1 },
        { 4.028559e-3, -3.697768e-2, 1.021332e-1, -1.201436e-1, 6.412774e-2 } };
    static const double q[2][3] = { { 1.0000000e0, 8.212018e-1, 2.078043e-1 }, { 1.0000000e0, 9.599102e-1, 2.918724e-1 } };
    nu = std::fabs(nu);
    int part;
    double nuend;
    if (nu >= 0.0 && nu < 0.75) {
        part = 0;
        nuend = 0.75;
    } else if (nu >= 0.75 && nu <= 1.0) {
        part = 1;
        nuend = 1.0;
    } else {
        part = 0;
        nuend = 0.0;
    }
    double top = p[part][0];
    double bot = q[part][0];
    const double delnusq = std::pow(nu, 2) - std::pow(nuend, 2);
    for (int k = 1; k < 5; k++)
        top += p[part][k] * std::pow(delnusq, k);
    for (int k = 1; k < 3; k++)
        bot += q[part][k] * std::pow(delnusq, k);
    return (bot > 0.0) ? top / bot : 0.0;
}

// Kernel functors, stp/convolution/conv_func.cpp:11-196.  The functors are
// built by ImageVisibilities (stp/imager/imager.cpp:25-64) with
// trunc/half_base_width = kernel_support and default width normalisations
// (GaussianSinc 2.52 / 1.55, stp/convolution/conv_func.h:216-217).
double kernel_value(int kf, double trunc, double r)
{
    switch (kf) {
    case kTopHat: // conv_func.cpp:25-34
        return (std::fabs(r) < trunc) ? 1.0 : 0.0;
    case kTriangle: // conv_func.cpp:11-15
        return std::max(1.0 - std::fabs(r) / trunc, 0.0);
    case kSinc: { // conv_func.cpp:44-59, width_normalization 1.0
        double x = r * (M_PI / 1.0);
        if (x == 0.0)
            x = 1.0e-20;
        double v = std::sin(x) / x;
        if (trunc > 0.0 && std::fabs(r) > trunc)
            v = 0.0;
        return v;
    }
    case kGaussian: { // conv_func.cpp:71-82, width_normalization 1.0
        double v = std::exp((-1.0 / (1.0 * 1.0)) * (r * r));
        if (trunc > 0.0 && std::fabs(r) > trunc)
            v = 0.0;
        return v;
    }
    case kGaussianSinc: { // conv_func.cpp:92-103
        const double wg = 2.52, ws = 1.55;
        double g = std::exp((-1.0 / (wg * wg)) * (r * r));
        double x = r * (M_PI / ws);
        if (x == 0.0)
            x = 1.0e-20;
        double s = std::sin(x) / x;
        double v = g * s;
        if (trunc > 0.0 && std::fabs(r) > trunc)
            v = 0.0;
        return v;
    }
    case kPSWF: { // conv_func.cpp:185-196
        double nu = r / trunc;
        double v = grdsf_one(nu) * (1 - std::pow(nu, 2));
        if (trunc > 0.0 && std::fabs(r) > trunc)
            v = 0.0;
        return v;
    }
    }
    return 0.0;
}

// Analytic grid-correction functions, conv_func.cpp:18-22,37-41,62-67,85-89,106-110,199-202.
// TopHat/Triangle/GaussianSinc assert(false) and return the radius itself in
// release builds; that behaviour is kept.
double gcf_value(int kf, double r)
{
    switch (kf) {
    case kSinc:
        return (std::fabs(r) < 1.0) ? 1.0 : 0.0;
    case kGaussian:
        return std::exp(-1.0 * std::pow(r * M_PI / (1.0 * 2), 2));
    case kPSWF:
        return grdsf_one(r);
    default:
        return r;
    }
}

// Armadillo accu() on a dense vector: two interleaved accumulators.
double accu(const double* x, size_t n)
{
    double a1 = 0.0, a2 = 0.0;
    size_t i = 0;
    for (; i + 1 < n; i += 2) {
        a1 += x[i];
        a2 += x[i + 1];
    }
    if (i < n)
        a1 += x[i];
    return a1 + a2;
}

inline int64_t idx2(int64_t r, int64_t c, int64_t nrows) { return c * nrows + r; }

} // namespace

extern "C" {

// ---------------------------------------------------------------- kernels

void orc_kernel_eval(int kf, double trunc, const double* r, double* out, int64_t n)
{
    for (int64_t i = 0; i < n; i++)
        out[i] = kernel_value(kf, trunc, r[i]);
}

void orc_gcf_eval(int kf, const double* r, double* out, int64_t n)
{
    for (int64_t i = 0; i < n; i++)
        out[i] = gcf_value(kf, r[i]);
}

// make_1D_kernel, stp/convolution/conv_func.h:319-337.
void orc_make_1d_kernel(int kf, double trunc, int support, double offset, int oversampling, int pad, int normalize, double* out)
{
    const int local_pad = pad ? 1 : 0;
    const int array_size = 2 * (support + local_pad) * oversampling + 1;
    const int centre_idx = (support + local_pad) * oversampling;
    for (int i = 0; i < array_size; i++) {
        double d = (double(i) - centre_idx) / oversampling;
        out[i] = kernel_value(kf, trunc, d - offset);
    }
    if (normalize) {
        double s = accu(out, array_size);
        for (int i = 0; i < array_size; i++)
            out[i] = out[i] / s;
    }
}

// make_kernel_array, stp/convolution/conv_func.h:279-303.  Column-major
// array_size x array_size: result(r, c) = y[r] * x[c].
void orc_make_kernel_array(int kf, double trunc, int support, double off_x, double off_y, int oversampling, int pad, int normalize,
    double* out)
{
    const int local_pad = pad ? 1 : 0;
    const int n = 2 * (support + local_pad) * oversampling + 1;
    const int centre_idx = (support + local_pad) * oversampling;
    std::vector<double> xk(n), yk(n);
    for (int i = 0; i < n; i++) {
        double d = (double(i) - centre_idx) / oversampling;
        xk[i] = kernel_value(kf, trunc, d - off_x);
        yk[i] = kernel_value(kf, trunc, d - off_y);
    }
    for (int c = 0; c < n; c++)
        for (int r = 0; r < n; r++)
            out[idx2(r, c, n)] = yk[r] * xk[c];
    if (normalize) {
        double s = accu(out, size_t(n) * n);
        for (int i = 0; i < n * n; i++)
            out[i] = out[i] / s;
    }
}

// populate_kernel_cache, stp/gridder/gridder.h:73-105, as the table of 1-D
// kernels k1d[(os/2)*2+1][2S+1]; the 2-D cache entry (cp_y, cp_x)(r, c) is
// k1d[cp_y][r] * k1d[cp_x][c] (an exact product, so this table is lossless).
void orc_kernel_table_1d(int kf, double trunc, int support, int oversampling, double* out)
{
    const int half = oversampling / 2;
    const int cache_size = half * 2 + 1;
    const int ksize = 2 * support + 1;
    for (int i = 0; i < cache_size; i++) {
        double offset = (double(i) - half) / oversampling;
        orc_make_1d_kernel(kf, trunc, support, offset, 1, 0, 1, out + size_t(i) * ksize);
    }
}

// calculate_oversampled_kernel_indices, stp/gridder/gridder.cpp:219-241.
void orc_oversampled_indices(const double* frac, int64_t n, int oversampling, int32_t* out)
{
    const int range_max = oversampling / 2;
    const int range_min = -range_max;
    for (int64_t i = 0; i < n; i++) {
        int v = int(std::rint(frac[i] * oversampling));
        if (v > range_max)
            v = range_max;
        else if (v < range_min)
            v = range_min;
        out[i] = v;
    }
}

// ---------------------------------------------------------------- gridder prepass

// convolve_to_grid steps before the gridding loop, stp/gridder/gridder.h:259-423
// (W-plane sort :311-367, half-plane conversion :369-375 with
// stp/gridder/gridder.cpp:11-66, rint split :378-386, bounds check :387 with
// gridder.cpp:202-217, uv shift :399-413, sampling total :417-423, oversampled
// indices :504 with gridder.cpp:219-241).
//
// uv: n x 2 column-major (pixels); vis: 2n interleaved; in place on copies
// owned by the caller.  Outputs per visibility: good (0/1/2), kc (n x 2),
// cp (n x 2; already + os/2), frac (n x 2).  When use_wproj, the arrays are
// permuted into |w| order first (sort_index is not stable in Armadillo; a
// stable sort is used here, so equal |w| keep input order).
// Returns sample_grid_total.
double orc_grid_prepass(int64_t n, double* uv, double* vis, double* weights, double* w, int use_wproj, int conv_support,
    int image_size, int kernel_exact, int oversampling, int shift_uv, int halfplane, int32_t* good, int32_t* kc,
    int32_t* cp, double* frac)
{
    if (use_wproj) {
        std::vector<int64_t> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return std::fabs(w[a]) < std::fabs(w[b]); });
        std::vector<double> tuv(2 * n), tvis(2 * n), tw(n), tww(n);
        for (int64_t i = 0; i < n; i++) {
            int64_t s = order[i];
            tuv[i] = uv[s];
            tuv[n + i] = uv[n + s];
            tvis[2 * i] = vis[2 * s];
            tvis[2 * i + 1] = vis[2 * s + 1];
            tw[i] = w[s];
            tww[i] = weights[s];
        }
        std::memcpy(uv, tuv.data(), sizeof(double) * 2 * n);
        std::memcpy(vis, tvis.data(), sizeof(double) * 2 * n);
        std::memcpy(w, tw.data(), sizeof(double) * n);
        std::memcpy(weights, tww.data(), sizeof(double) * n);
    }
    for (int64_t i = 0; i < n; i++)
        good[i] = 1;
    if (halfplane) {
        for (int64_t i = 0; i < n; i++) {
            double v = uv[n + i];
            if (v < 0.0) {
                if (v > -(conv_support + 1))
                    good[i] = 2;
                uv[i] *= -1;
                uv[n + i] *= -1;
                if (use_wproj)
                    w[i] *= -1;
                vis[2 * i + 1] = -vis[2 * i + 1];
            } else {
                if (v < (conv_support + 1))
                    good[i] = 2;
            }
        }
    }
    const int half_image_size = image_size / 2;
    for (int64_t i = 0; i < n; i++) {
        for (int d = 0; d < 2; d++) {
            double x = uv[d * n + i];
            int val = int(std::rint(x));
            frac[d * n + i] = x - val;
            kc[d * n + i] = val + half_image_size;
        }
    }
    for (int64_t i = 0; i < n; i++) {
        int kx = kc[i], ky = kc[n + i];
        if ((kx - conv_support) <= 0 || (ky - conv_support) <= 0 || (kx + conv_support) >= image_size
            || (ky + conv_support) >= image_size)
            good[i] = 0;
    }
    if (shift_uv) {
        for (int64_t i = 0; i < 2 * n; i++) {
            if (kc[i] < half_image_size)
                kc[i] += half_image_size;
            else
                kc[i] -= half_image_size;
        }
    }
    double total = 0.0;
    for (int64_t i = 0; i < n; i++)
        if (good[i] != 0)
            total += weights[i];
    total *= 2.0;
    if (!kernel_exact) {
        orc_oversampled_indices(frac, 2 * n, oversampling, cp);
        for (int64_t i = 0; i < 2 * n; i++)
            cp[i] += oversampling / 2;
    } else {
        for (int64_t i = 0; i < 2 * n; i++)
            cp[i] = 0;
    }
    return total;
}

// average_w_planes, stp/gridder/gridder.cpp:68-146 (w already |w|).
void orc_average_w_planes(const double* absw, const int32_t* good, int64_t n, int num_wplanes, int median, double* w_avg,
    int64_t* firstidx)
{
    uint64_t num_gvis = 0;
    for (int64_t i = 0; i < n; i++)
        if (good[i] != 0)
            num_gvis++;
    uint64_t begin = 0;
    for (int idx = 0; idx < num_wplanes; idx++) {
        uint64_t plane_size = uint64_t(std::ceil(double(num_gvis - begin) / (num_wplanes - idx)));
        if (median) {
            uint64_t idx_mid = 0;
            uint64_t middle = plane_size / 2;
            if ((begin + plane_size) > num_gvis)
                middle = (num_gvis - begin) / 2;
            uint64_t k, counter = 0;
            for (k = begin; (counter < plane_size) && (k < uint64_t(n)); k++) {
                if (good[k] != 0) {
                    if (counter == middle)
                        idx_mid = k;
                    counter++;
                }
            }
            if (counter > 0) {
                if ((plane_size % 2) == 0)
                    w_avg[idx] = (absw[idx_mid - 1] + absw[idx_mid]) / 2.0;
                else
                    w_avg[idx] = absw[idx_mid];
            } else
                w_avg[idx] = 0.0;
            firstidx[idx] = int64_t(begin);
            begin = k;
        } else {
            double sum = 0;
            uint64_t k, counter = 0;
            for (k = begin; (counter < plane_size) && (k < uint64_t(n)); k++) {
                if (good[k] != 0) {
                    sum += absw[k];
                    counter++;
                }
            }
            firstidx[idx] = int64_t(begin);
            begin = k;
            w_avg[idx] = counter > 0 ? sum / counter : 0.0;
        }
    }
}

// WideFieldImaging::generate_image_domain_convolution_kernel with
// combine_2d_kernel_value, stp/gridder/aw_projection.cpp:50-111,455-474.
// out: arr x arr complex (interleaved), column-major, zero outside the
// filled region.
void orc_wkernel_image_domain(double w_value, const double* aa, int kernel_size, int oversampling, double cell_size_rad,
    double scaling_factor, double* out)
{
    const int64_t arr = int64_t(kernel_size) * oversampling;
    const int half = kernel_size / 2;
    const double scaled_cell = cell_size_rad * scaling_factor;
    std::memset(out, 0, sizeof(double) * 2 * arr * arr);
    auto value = [&](int px, int py, double& re, double& im) {
        double dx = double(px) * scaled_cell, dy = double(py) * scaled_cell;
        double r2 = dx * dx + dy * dy;
        double a = aa[half + px] * aa[half + py];
        if (r2 >= 1.0) {
            re = a;
            im = 0.0;
        } else {
            double nn = std::sqrt(1.0 - r2);
            double ph = (-2.0 * M_PI) * w_value * (nn - 1.0);
            // (exp(i ph) / n) * aa_x * aa_y, evaluated as the complex expression
            double er = std::cos(ph) / nn, ei = std::sin(ph) / nn;
            re = er * aa[half + px];
            im = ei * aa[half + px];
            re = re * aa[half + py];
            im = im * aa[half + py];
        }
    };
    auto put = [&](int64_t r, int64_t c, double re, double im) {
        out[2 * idx2(r, c, arr)] = re;
        out[2 * idx2(r, c, arr) + 1] = im;
    };
    for (int i = 1; i < half; i++) {
        double re, im;
        value(i, 0, re, im);
        put(i, 0, re, im);
        put(arr - i, 0, re, im);
        put(0, i, re, im);
        put(0, arr - i, re, im);
    }
    put(0, 0, aa[half] * aa[half], 0.0);
    for (int j = 1; j < half; j++)
        for (int i = 1; i < half; i++) {
            double re, im;
            value(i, j, re, im);
            put(i, j, re, im);
            put(arr - i, j, re, im);
            put(i, arr - j, re, im);
            put(arr - i, arr - j, re, im);
        }
}

// Truncation of the W-kernel, stp/gridder/aw_projection.cpp:197-209.
// conv: arr x arr complex column-major (forward c2c FFT of the image-domain kernel).
int orc_wkernel_truncate(const double* conv, int64_t arr, int max_support, int oversampling, double kernel_trunc_perc,
    int current_support)
{
    if (!(kernel_trunc_perc > 0.0))
        return current_support;
    const double trunc_at = kernel_trunc_perc / 100.0;
    const double min_value = std::hypot(conv[0], conv[1]) * trunc_at;
    unsigned i = std::min(unsigned(max_support * oversampling), unsigned(arr >> 1));
    while (i > 0) {
        if (std::hypot(conv[2 * i], conv[2 * i + 1]) > min_value)
            break;
        i -= oversampling;
    }
    return int(std::min(unsigned(i / oversampling), unsigned(max_support)));
}

// generate_kernel_cache, non-Hankel branch, stp/gridder/aw_projection.cpp:366-452.
// out: [(os/2*2+1)^2] kernels, entry (y, x) at ((y*cs + x) * K*K), each
// K x K complex column-major (row = v offset, column = u offset).
void orc_wkernel_cache(const double* conv, int64_t arr, int support, int oversampling, double* out)
{
    const int64_t ctr = arr / 2;
    const int64_t os = oversampling;
    const int64_t half_os = os / 2;
    const int64_t cs = half_os * 2 + 1;
    const int64_t K = 2 * support + 1;
    const int64_t khalf = arr / 2;
    const int64_t oconv = ctr - support * os + half_os;
    std::vector<double> tmp(2 * K * K);
    for (int64_t x = 0; x < cs; x++) {
        for (int64_t y = 0; y < cs; y++) {
            int64_t xx = oconv - x;
            double ksum = 0.0;
            for (int64_t ty = 0; ty < K; ty++, xx += os) {
                int64_t cx = (xx + khalf) % arr;
                int64_t yy = oconv - y;
                for (int64_t tx = 0; tx < K; tx++, yy += os) {
                    int64_t cy = (yy + khalf) % arr;
                    const double* v = conv + 2 * idx2(cx, cy, arr);
                    tmp[2 * idx2(tx, ty, K)] = v[0];
                    tmp[2 * idx2(tx, ty, K) + 1] = v[1];
                    ksum += v[0];
                }
            }
            ksum = 1 / ksum;
            double* dst = out + 2 * (y * cs + x) * K * K;
            for (int64_t e = 0; e < 2 * K * K; e++)
                dst[e] = tmp[e] * ksum;
        }
    }
}

// ---------------------------------------------------------------- gridding loop

// The oversampled gridder (serial form stp/gridder/gridder.h:596-678; the TBB
// form :767-934 adds to each cell in the same visibility order, so both give
// the same bits) and the exact gridder (:943-994).
//
// kmode 0: separable real kernel from the 1-D table k1d (non-W-proj,
//          oversampled); 1: exact kernel (make_kernel_array per visibility);
//          2: complex W-kernel cache wk (orc_wkernel_cache layout), with
//          conj(kernel) where w < 0.
// Grids are image_rows x image_size complex, column-major, interleaved.
// Processes visibilities [vi_begin, vi_end).  threads > 1 uses the reference's
// TBB decomposition (one task per kernel-column residue mod K).
void orc_grid_accumulate(int kmode, int kf, double trunc, const double* k1d, const double* wk, int support,
    int image_size, int image_rows, int oversampling, int64_t n, int64_t vi_begin, int64_t vi_end, const double* vis,
    const double* weights, const double* w, const int32_t* good, const int32_t* kc, const int32_t* cp, const double* frac,
    int generate_beam, double* vis_grid, double* sampling_grid, int threads)
{
    const int K = 2 * support + 1;
    auto tap = [&](int64_t vi, int gv, int i, int j, double& kr, double& ki, const double* exact) {
        if (kmode == 0) {
            int cpx = cp[vi], cpy = cp[n + vi];
            if (gv && oversampling > 1) {
                cpx = oversampling - cpx;
                cpy = oversampling - cpy;
            }
            kr = k1d[size_t(cpy) * K + i] * k1d[size_t(cpx) * K + j];
            ki = 0.0;
        } else if (kmode == 1) {
            kr = exact[idx2(i, j, K)];
            ki = 0.0;
        } else {
            int cpx = cp[vi], cpy = cp[n + vi];
            if (gv && oversampling > 1) {
                cpx = oversampling - cpx;
                cpy = oversampling - cpy;
            }
            const int cs = (oversampling / 2) * 2 + 1;
            const double* kk = wk + 2 * (size_t(cpy * cs + cpx) * K * K + idx2(i, j, K));
            kr = kk[0];
            ki = kk[1];
            double wv = gv ? -w[vi] : w[vi];
            if (wv < 0.0)
                ki = -ki;
        }
    };
    auto one_vis = [&](int64_t vi, int col_residue) {
        const int gvis = good[vi];
        if (gvis == 0)
            return;
        std::vector<double> exact;
        for (int gv = 0; gv < gvis; gv++) {
            int gc_x = kc[vi], gc_y = kc[n + vi];
            double vr = vis[2 * vi], vim = vis[2 * vi + 1];
            if (gv) {
                gc_x = -kc[vi] + image_size;
                gc_y = -kc[n + vi] + image_size;
                vim = -vim;
            }
            if (kmode == 1) {
                exact.resize(size_t(K) * K);
                double fx = frac[vi], fy = frac[n + vi];
                if (gv) {
                    fx *= -1;
                    fy *= -1;
                }
                orc_make_kernel_array(kf, trunc, support, fx, fy, 1, 0, 1, exact.data());
            }
            const double wt = weights[vi];
            for (int j = 0; j < K; j++) {
                int grid_col = gc_x - support + j;
                if (grid_col < 0)
                    grid_col += image_size;
                if (grid_col >= image_size)
                    grid_col -= image_size;
                if (col_residue >= 0 && (grid_col % K) != col_residue)
                    continue;
                int grid_row = gc_y - support;
                for (int i = 0; i < K; ++i, ++grid_row) {
                    int row = grid_row;
                    if (row < 0) {
                        if (kmode == 1)
                            row += image_size; // exact path wraps (gridder.h:978-979)
                        else
                            continue; // oversampled path skips (gridder.h:662-663)
                    }
                    if (row >= image_size)
                        row -= image_size;
                    if (row < image_rows) {
                        double kr, ki;
                        tap(vi, gv, i, j, kr, ki, exact.data());
                        kr = kr * wt;
                        ki = ki * wt;
                        double* g = vis_grid + 2 * idx2(row, grid_col, image_rows);
                        g[0] += vr * kr - vim * ki;
                        g[1] += vr * ki + vim * kr;
                        if (generate_beam) {
                            double* s = sampling_grid + 2 * idx2(row, grid_col, image_rows);
                            s[0] += kr;
                            s[1] += ki;
                        }
                    }
                    if (kmode != 1)
                        grid_row = row; // the oversampled path rewrites grid_row in place
                }
            }
        }
    };
    if (threads <= 1 || kmode == 1) {
        for (int64_t vi = vi_begin; vi < vi_end; vi++)
            one_vis(vi, -1);
    } else {
#ifdef _OPENMP
#pragma omp parallel for schedule(static, 1) num_threads(threads)
#endif
        for (int r = 0; r < K; r++)
            for (int64_t vi = vi_begin; vi < vi_end; vi++)
                one_vis(vi, r);
    }
}

// normalise_image_beam_result_1D, non-FFTSHIFT branch, stp/imager/imager.h:97-150.
// img: padded x padded real column-major; out: image_size^2.
void orc_normalise(const double* img, int64_t padded, int64_t image_size, double normalization_factor, const double* gcf,
    int grid_correction, double* out, int threads)
{
    const int64_t hp = padded / 2;
    const int64_t hs = image_size / 2;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : 1)
#endif
    for (int64_t j = 0; j < image_size; j++) {
        int64_t orig_j = (j < hs) ? j : padded + j - image_size;
        int64_t jj = (j < hs) ? j + hp : hp + j - image_size;
        for (int64_t i = 0; i < image_size; i++) {
            int64_t orig_i = (i < hs) ? i : padded - hs + (i - hs);
            int64_t ii = (i < hs) ? hp + i : hp - hs + (i - hs);
            double v = img[idx2(orig_i, orig_j, padded)];
            out[idx2(i, j, image_size)]
                = grid_correction ? v * normalization_factor / (gcf[ii] * gcf[jj]) : v * normalization_factor;
        }
    }
}

// ---------------------------------------------------------------- statistics

// mat_mean_and_stddev, stp/common/matrix_math.cpp:457-499 (one TBB range:
// 4-way unrolled body, remainder loop).
void orc_mean_std(const double* x, int64_t n, double* mean, double* sigma)
{
    if (n < 1) {
        *mean = 0.0;
        *sigma = 0.0;
        return;
    }
    double d1 = 0.0, d2 = 0.0;
    int64_t i = 0, rend = n;
    if (rend - i > 8) {
        rend -= 4;
        for (; i < rend; i += 4) {
            double a = x[i], b = x[i + 1], c = x[i + 2], d = x[i + 3];
            d1 += a + b + c + d;
            d2 += a * a + b * b + c * c + d * d;
        }
        rend += 4;
    }
    for (; i < rend; i++) {
        d1 += x[i];
        d2 += x[i] * x[i];
    }
    *mean = d1 / double(n);
    *sigma = std::sqrt(d2 / double(n) - (*mean) * (*mean));
}

// mat_median_exact, stp/common/matrix_math.cpp:20-48.
double orc_median_exact(const double* x, int64_t n)
{
    std::vector<double> a(x, x + n);
    size_t k = size_t(n / 2);
    std::nth_element(a.begin(), a.begin() + k, a.end());
    if (n & 1)
        return a[k];
    double v1 = a[k];
    double v2 = *std::max_element(a.begin(), a.begin() + k);
    return (v1 + v2) / 2;
}

// mat_median_binapprox, stp/common/matrix_math.cpp:334-455.
void orc_median_binapprox(const double* x, int64_t n, double* mean_out, double* sigma_out, double* median_out)
{
    const int N = 1000;
    double mean, sigma;
    orc_mean_std(x, n, &mean, &sigma);
    *mean_out = mean;
    *sigma_out = sigma;
    if ((sigma * 2) < 0.0001) {
        *median_out = orc_median_exact(x, n);
        return;
    }
    const double scalefactor = double(N) / (2 * sigma);
    const double leftend = mean - sigma;
    std::vector<uint64_t> bins(N + 1, 0);
    uint64_t bottom = 0;
    for (int64_t i = 0; i < n; i++) {
        const int bin = int((x[i] - leftend) * scalefactor);
        if (bin < 0)
            bottom++;
        else if (bin <= N)
            bins[bin]++;
    }
    bool ok = false;
    double median = 0.0;
    if (n & 1) {
        uint64_t k = (uint64_t(n) + 1) / 2, count = bottom;
        for (int i = 0; i < N + 1; i++) {
            count += bins[i];
            if (count >= k) {
                median = double(i + 0.5) / scalefactor + leftend;
                ok = true;
                break;
            }
        }
    } else {
        uint64_t k = uint64_t(n) / 2, count = bottom;
        for (int i = 0; i < N + 1; i++) {
            count += bins[i];
            if (count >= k) {
                int j = i;
                while (count == k) {
                    j++;
                    count += bins[j];
                    if (j == N)
                        break;
                }
                median = double(i + j + 1) / (2 * scalefactor) + leftend;
                ok = true;
                break;
            }
        }
    }
    if (!ok)
        median = orc_median_exact(x, n);
    *median_out = median;
}

// mat_binmedian, stp/common/matrix_math.cpp:50-332 (successive binning, then
// nth_element on the surviving bin).
void orc_median_binmedian(const double* x, int64_t n, double* mean_out, double* sigma_out, double* median_out)
{
    const int N = 1000;
    double mean, sigma;
    orc_mean_std(x, n, &mean, &sigma);
    *mean_out = mean;
    *sigma_out = sigma;
    if ((sigma * 2) < 0.0001) {
        *median_out = orc_median_exact(x, n);
        return;
    }
    double scalefactor = double(N) / (2 * sigma);
    double leftend = mean - sigma;
    double rightend = mean + sigma;
    std::vector<uint64_t> bins(N + 1, 0);
    uint64_t bottom = 0;
    auto binning = [&]() {
        std::fill(bins.begin(), bins.end(), 0);
        bottom = 0;
        for (int64_t i = 0; i < n; i++) {
            const int bin = int((x[i] - leftend) * scalefactor);
            if (bin < 0)
                bottom++;
            else if (bin <= N)
                bins[bin]++;
        }
    };
    binning();
    uint64_t k = uint64_t(n) / 2 + 1;
    uint64_t oldmedbinsize = n, medbinsize = n;
    double oldscalefactor = 0.0, oldleftend = 0.0;
    int right_medbin = -1, left_medbin = -1;
    while (true) {
        bool found = false;
        uint64_t count = bottom;
        k = uint64_t(n) / 2 + 1;
        int i;
        for (i = 0; i < N + 1; ++i) {
            count += bins[i];
            if (count >= k) {
                right_medbin = i;
                left_medbin = i;
                k = k - (count - bins[i]);
                medbinsize = bins[i];
                found = true;
                break;
            }
        }
        if (!(n & 1)) {
            if (found && k == 1) {
                if (i > 0) {
                    i--;
                    while (bins[i] == 0) {
                        i--;
                        if (i < 0)
                            break;
                    }
                    if (i >= 0) {
                        k += bins[i];
                        medbinsize += bins[i];
                        left_medbin = i;
                    } else
                        found = false;
                } else
                    found = false;
            }
        }
        if (found) {
            oldscalefactor = scalefactor;
            oldleftend = leftend;
            leftend = double(left_medbin) / oldscalefactor + oldleftend;
            rightend = double(right_medbin + 1) / oldscalefactor + oldleftend;
            scalefactor = double(N) / (rightend - leftend);
        } else {
            if (right_medbin == -1) {
                *median_out = orc_median_exact(x, n);
                return;
            }
            break;
        }
        if ((medbinsize < 100) || (medbinsize < uint64_t(n) / 10) || ((rightend - leftend) < 0.0001)
            || (oldmedbinsize == medbinsize)) {
            oldmedbinsize = medbinsize;
            break;
        }
        oldmedbinsize = medbinsize;
        binning();
    }
    std::vector<double> aux;
    aux.reserve(oldmedbinsize);
    for (int64_t i = 0; i < n; i++) {
        const int bin = int((x[i] - oldleftend) * oldscalefactor);
        if (bin >= left_medbin && bin <= right_medbin)
            aux.push_back(x[i]);
    }
    auto nth = aux.begin() + (k - 1);
    std::nth_element(aux.begin(), nth, aux.end());
    double median;
    if (n & 1)
        median = *nth;
    else {
        double v1 = *nth;
        double v2 = *std::max_element(aux.begin(), nth);
        median = (v1 + v2) / 2;
    }
    *median_out = median;
}

// estimate_rms, stp/sourcefind/sourcefind.cpp:22-154.  The reference compares
// |x - median| with the thresholds through the integer bits of IEEE doubles;
// for non-negative finite numbers that is the same as comparing the doubles.
double orc_estimate_rms(const double* x, int64_t n, double num_sigma, int iters, double mean, double sigma, double median)
{
    double m = mean - median;
    double s = sigma;
    double d1 = m * double(n), d2 = (s * s + m * m) * double(n);
    uint64_t valid = uint64_t(n);
    double prev_upper = std::numeric_limits<double>::max();
    for (int it = 0; it < iters; it++) {
        const double upper = num_sigma * s;
        double r1 = 0.0, r2 = 0.0;
        uint64_t rem = 0;
        for (int64_t j = 0; j < n; j++) {
            const double v = x[j] - median;
            const double a = std::fabs(v);
            if (a > upper && !(a > prev_upper)) {
                r1 += v;
                r2 += v * v;
                rem++;
            }
        }
        if (rem == 0)
            break;
        valid -= rem;
        d1 -= r1;
        d2 -= r2;
        s = std::sqrt(d2 / double(valid) - (d1 / double(valid)) * (d1 / double(valid)));
        prev_upper = upper;
    }
    return s;
}

// ---------------------------------------------------------------- connected components

namespace {
inline uint32_t find_root(const uint32_t* P, uint32_t i)
{
    uint32_t root = i;
    while (P[root] < root)
        root = P[root];
    return root;
}
inline void set_root(uint32_t* P, uint32_t i, uint32_t root)
{
    while (P[i] < i) {
        uint32_t j = P[i];
        P[i] = root;
        i = j;
    }
    P[i] = root;
}
inline uint32_t set_union(uint32_t* P, uint32_t i, uint32_t j)
{
    uint32_t root = find_root(P, i);
    if (i != j) {
        uint32_t rootj = find_root(P, j);
        if (root > rootj)
            root = rootj;
        set_root(P, j, root);
    }
    set_root(P, i, root);
    return root;
}
} // namespace

// labeling_8con / labeling_4con, non-FFTSHIFT build, stp/common/ccl.h:107-484
// and :505-773, with the TBB column slices processed one after another (one
// legal interleaving of the parallel scan).  Slices start at multiples of
// slice_cols; the reference's static_partitioner gives T slices of cols/T
// columns for T threads.  Outputs the provisional label map L (rows x cols,
// column-major), the flattened equivalence tables Pp / Pn (length
// cols*rows/2 each) and the label counts.
void orc_ccl(const double* I, int rows, int cols, double thr_pos, double thr_neg, int find_negative, int conn4,
    int slice_cols, int32_t* L, uint32_t* Pp, uint32_t* Pn, uint32_t* n_pos, uint32_t* n_neg)
{
    const size_t cshift = cols / 2, rshift = rows / 2;
    std::memset(L, 0, sizeof(int32_t) * size_t(rows) * cols);
    const size_t Plength = size_t(cols) * rows / 2;
    std::memset(Pp, 0, sizeof(uint32_t) * Plength);
    std::memset(Pn, 0, sizeof(uint32_t) * Plength);
    if (slice_cols < 1)
        slice_cols = 1;
    struct Slice {
        uint32_t col_start, lstart, lp, ln;
    };
    std::vector<Slice> slices;
    for (int cs = 0; cs < cols; cs += slice_cols) {
        const int ce = std::min(cols, cs + slice_cols);
        const uint32_t lstart = uint32_t(cs) * uint32_t(rows / 2);
        Pp[lstart] = 0;
        Pn[lstart] = 0;
        uint32_t lp = lstart + 1, ln = lstart + 1;
        for (uint32_t c_i = cs; c_i < uint32_t(ce); ++c_i) {
            const uint32_t mc = c_i >= cshift ? c_i - cshift : c_i + cshift;
            const uint32_t mcp = (mc == 0) ? cols - 1 : mc - 1;
            int32_t* Lc = L + size_t(mc) * rows;
            int32_t* Lp = L + size_t(mcp) * rows;
            const double* Ic = I + size_t(mc) * rows;
            const bool left_ok = !(c_i == uint32_t(cs));
            for (uint32_t r = 0; r < uint32_t(rows); r++) {
                const double val = Ic[r];
                const bool pos = val > thr_pos;
                const bool neg = !pos && find_negative && (val < thr_neg);
                if (!pos && !neg)
                    continue;
                const uint32_t rp = (r == 0) ? r : r - 1;
                const uint32_t rn = (r == uint32_t(rows) - 1) ? r : r + 1;
                const int32_t top = Lc[rp], left = Lp[r], topleft = Lp[rp], bottomleft = Lp[rn];
                auto is = [&](int32_t v) { return pos ? v > 0 : v < 0; };
                uint32_t* P = pos ? Pp : Pn;
                const int sgn = pos ? 1 : -1;
                const bool T_left = left_ok && is(left);
                const bool T_top = (r == rshift || r == 0) ? false : is(top);
                int32_t& cur = Lc[r];
                if (conn4) {
                    if (T_left) {
                        cur = T_top ? sgn * int32_t(set_union(P, sgn * top, sgn * left)) : left;
                    } else if (T_top) {
                        cur = top;
                    } else {
                        uint32_t& lu = pos ? lp : ln;
                        cur = sgn * int32_t(lu);
                        P[lu] = lu;
                        lu++;
                    }
                } else {
                    const bool T_topleft = (r == rshift || r == 0) ? false : (left_ok && is(topleft));
                    const bool T_bottomleft = (r == rshift - 1 || r == uint32_t(rows) - 1) ? false : (left_ok && is(bottomleft));
                    if (T_left) {
                        cur = left;
                    } else if (T_bottomleft) {
                        if (T_topleft)
                            cur = sgn * int32_t(set_union(P, sgn * topleft, sgn * bottomleft));
                        else if (T_top)
                            cur = sgn * int32_t(set_union(P, sgn * top, sgn * bottomleft));
                        else
                            cur = bottomleft;
                    } else if (T_topleft) {
                        cur = topleft;
                    } else if (T_top) {
                        cur = top;
                    } else {
                        uint32_t& lu = pos ? lp : ln;
                        cur = sgn * int32_t(lu);
                        P[lu] = lu;
                        lu++;
                    }
                }
            }
            // Row border merge (rows 0 and rows-1), ccl.h:308-342 / :660-683.
            {
                int32_t& cur = Lc[0];
                const int32_t top = Lc[rows - 1];
                const int32_t topleft = Lp[rows - 1];
                if (cur > 0) {
                    if (top > 0)
                        cur = int32_t(set_union(Pp, cur, top));
                    if (!conn4 && topleft > 0 && top != topleft)
                        cur = int32_t(set_union(Pp, cur, topleft));
                } else if (find_negative && cur < 0) {
                    if (top < 0)
                        cur = -int32_t(set_union(Pn, -cur, -top));
                    if (!conn4 && topleft < 0 && top != topleft)
                        cur = -int32_t(set_union(Pn, -cur, -topleft));
                }
            }
        }
        slices.push_back({ uint32_t(cs), lstart, lp, ln });
    }
    // Column border merging, ccl.h:355-448 (8-conn) / :695-745 (4-conn).
    for (const Slice& s : slices) {
        const uint32_t c_i = s.col_start;
        const uint32_t mc = c_i >= cshift ? c_i - cshift : c_i + cshift;
        const uint32_t mcp = (mc == 0) ? cols - 1 : mc - 1;
        int32_t* Lc = L + size_t(mc) * rows;
        int32_t* Lp = L + size_t(mcp) * rows;
        const bool left_ok = c_i != 0;
        for (uint32_t r = 0; r < uint32_t(rows); r++) {
            int32_t& cur = Lc[r];
            const int32_t cp = cur;
            if (cp == 0)
                continue;
            const bool pos = cp > 0;
            if (!pos && !find_negative)
                continue;
            auto is = [&](int32_t v) { return pos ? v > 0 : v < 0; };
            uint32_t* P = pos ? Pp : Pn;
            const int sgn = pos ? 1 : -1;
            const uint32_t rp = (r == 0) ? rows - 1 : (r == rshift ? r : r - 1);
            const uint32_t rn = (r == uint32_t(rows) - 1) ? 0 : (r == rshift - 1 ? r : r + 1);
            const int32_t topleft = Lp[rp], left = Lp[r], bottomleft = Lp[rn];
            const bool T_left = left_ok && is(left);
            if (conn4) {
                if (T_left)
                    cur = sgn * int32_t(set_union(P, sgn * cp, sgn * left));
            } else {
                const bool T_topleft = (r == rshift) ? false : (left_ok && is(topleft));
                const bool T_bottomleft = (r == rshift - 1) ? false : (left_ok && is(bottomleft));
                if (T_topleft)
                    cur = sgn * int32_t(set_union(P, sgn * cp, sgn * topleft));
                if (T_left)
                    cur = sgn * int32_t(set_union(P, sgn * cp, sgn * left));
                if (T_bottomleft)
                    cur = sgn * int32_t(set_union(P, sgn * cp, sgn * bottomleft));
            }
        }
    }
    // Analysis (flatten), ccl.h:452-480.
    uint32_t k = 1;
    for (const Slice& s : slices)
        for (uint32_t i = s.lstart + 1; i < s.lp; ++i) {
            if (Pp[i] < i)
                Pp[i] = Pp[Pp[i]];
            else
                Pp[i] = k++;
        }
    *n_pos = k - 1;
    k = 1;
    if (find_negative)
        for (const Slice& s : slices)
            for (uint32_t i = s.lstart + 1; i < s.ln; ++i) {
                if (Pn[i] < i)
                    Pn[i] = Pn[Pn[i]];
                else
                    Pn[i] = k++;
            }
    *n_neg = k - 1;
}

// _label_detection_islands after the CCL call, stp/sourcefind/sourcefind.cpp:323-628
// (single thread: final labels + extrema :342-378, detection filter
// :417-436, moments / counts :457-569, normalisation :591-628).
// ext_val/ext_idx/moments (5 per label)/numsamples/valid for positive labels
// then negative labels (arrays sized n_pos and n_neg).
void orc_label_analysis(const double* data, int rows, int cols, int32_t* L, const uint32_t* Pp, const uint32_t* Pn,
    uint32_t n_pos, uint32_t n_neg, double det_pos, double det_neg, int generate_labelmap, double* ext_val_pos,
    int64_t* ext_idx_pos, double* moments_pos, int32_t* nsamp_pos, int32_t* valid_pos, double* ext_val_neg,
    int64_t* ext_idx_neg, double* moments_neg, int32_t* nsamp_neg, int32_t* valid_neg)
{
    const int64_t total = int64_t(rows) * cols;
    for (uint32_t l = 0; l < n_pos; l++) {
        ext_val_pos[l] = det_pos;
        ext_idx_pos[l] = -1;
    }
    for (uint32_t l = 0; l < n_neg; l++) {
        ext_val_neg[l] = det_neg;
        ext_idx_neg[l] = -1;
    }
    for (int64_t i = 0; i < total; i++) {
        const int32_t t = L[i];
        if (t == 0)
            continue;
        if (t > 0) {
            int32_t l = int32_t(Pp[t]);
            if (l > 0) {
                L[i] = l;
                l--;
                if (data[i] > ext_val_pos[l]) {
                    ext_val_pos[l] = data[i];
                    ext_idx_pos[l] = i;
                }
            }
        } else {
            int32_t l = int32_t(Pn[-t]);
            if (l > 0) {
                L[i] = -l;
                l--;
                if (data[i] < ext_val_neg[l]) {
                    ext_val_neg[l] = data[i];
                    ext_idx_neg[l] = i;
                }
            }
        }
    }
    for (uint32_t l = 0; l < n_pos; l++)
        valid_pos[l] = ext_val_pos[l] > det_pos ? 1 : 0;
    for (uint32_t l = 0; l < n_neg; l++)
        valid_neg[l] = ext_val_neg[l] < det_neg ? 1 : 0;
    std::vector<double> mp(6 * size_t(n_pos), 0.0), mn(6 * size_t(n_neg), 0.0);
    for (uint32_t l = 0; l < n_pos; l++)
        nsamp_pos[l] = 0;
    for (uint32_t l = 0; l < n_neg; l++)
        nsamp_neg[l] = 0;
    const int h_shift = cols / 2, v_shift = rows / 2;
    int64_t li = 0;
    for (int c = 0; c < cols; c++) {
        for (int r = 0; r < rows; r++, li++) {
            const int32_t label = L[li];
            if (label == 0)
                continue;
            int idx;
            if (label > 0) {
                idx = label - 1;
                if (!valid_pos[idx]) {
                    if (generate_labelmap)
                        L[li] = 0;
                    continue;
                }
            } else {
                idx = -label - 1;
                if (!valid_neg[idx]) {
                    if (generate_labelmap)
                        L[li] = 0;
                    continue;
                }
            }
            const double val = data[li];
            const double y = r < v_shift ? double(r + v_shift) : double(r - v_shift);
            const double x = c < h_shift ? double(c + h_shift) : double(c - h_shift);
            const double xb = x * val, yb = y * val;
            double* m = label > 0 ? &mp[6 * size_t(idx)] : &mn[6 * size_t(idx)];
            (label > 0 ? nsamp_pos : nsamp_neg)[idx]++;
            m[0] += xb;
            m[1] += yb;
            m[2] += xb * x;
            m[3] += yb * y;
            m[4] += xb * y;
            m[5] += val;
        }
    }
    auto norm = [](const double* a, double* out) {
        const double xb = a[0] / a[5], yb = a[1] / a[5];
        out[0] = xb;
        out[1] = yb;
        out[2] = a[2] / a[5] - xb * xb;
        out[3] = a[3] / a[5] - yb * yb;
        out[4] = a[4] / a[5] - xb * yb;
    };
    for (uint32_t l = 0; l < n_pos; l++) {
        if (valid_pos[l])
            norm(&mp[6 * size_t(l)], moments_pos + 5 * size_t(l));
        else
            for (int q = 0; q < 5; q++)
                moments_pos[5 * size_t(l) + q] = 0.0;
    }
    for (uint32_t l = 0; l < n_neg; l++) {
        if (valid_neg[l])
            norm(&mn[6 * size_t(l)], moments_neg + 5 * size_t(l));
        else
            for (int q = 0; q < 5; q++)
                moments_neg[5 * size_t(l) + q] = 0.0;
    }
}

int orc_num_threads()
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

} // extern "C"
