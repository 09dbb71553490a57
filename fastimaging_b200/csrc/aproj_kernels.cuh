// A-projection: W-kernels per W-plane AND time step.  Each visibility is
// assigned to a time step by its local hour angle; each (plane, step) pair
// gets its own kernel: the plane's image-domain W-screen times the inverse
// primary beam (a spherical-harmonic expansion, rotated by the step's
// parallactic angle), 2-D FFT, truncation and the oversampled kernel cache.
// The reference builds this with ENABLE_APROJECTION (experimental):
//   average_lha_planes           src/stp/gridder/gridder.cpp:148-200
//   generate_a_kernel            src/stp/gridder/gridder.cpp:243-275
//   parangle                     src/stp/gridder/aw_projection.cpp:599-608
//   generate_convolution_kernel_aproj  aw_projection.cpp:290-364
//   per-step loop and the rotated-kernel option (aproj_opt)
//                                src/stp/gridder/gridder.h:507-520,686-745
//   rotate_matrix                src/stp/common/matrix_math.cpp:610-733
// The gridder itself is unchanged: a visibility's item carries the combined
// index plane * T + step, and the kernel tables are laid out over P * T.
#pragma once

#include "imager_kernels.cuh"

namespace stpgpu {

constexpr double kApPi = 3.141592653589793238462643383279502884;

// Time-step boundaries: linspace(min - step/2, max + step/2, T + 1) with
// step = (max - min) / T over every visibility's hour angle (Armadillo's
// linspace: start + i * delta, the last point = end).
__global__ void __launch_bounds__(1024) k_lha_intervals(const double* lha, int64_t n, int T, double* iv)
{
    __shared__ double smin[1024], smax[1024];
    double lo = n > 0 ? lha[0] : 0.0, hi = lo;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        lo = fmin(lo, lha[i]);
        hi = fmax(hi, lha[i]);
    }
    smin[threadIdx.x] = lo;
    smax[threadIdx.x] = hi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
            smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double mn = smin[0], mx = smax[0];
        const double step = (mx - mn) / T;
        const double start = mn - step / 2, end = mx + step / 2;
        const double delta = (end - start) / double(T);
        for (int i = 0; i < T; i++)
            iv[i] = start + double(i) * delta;
        iv[T] = end;
    }
}

// Time step of each good visibility (input order): the first boundary
// iv[k] (k >= 1) with lha <= iv[k] closes its interval k - 1.
template <typename R>
__global__ void k_lha_steps(const double* lha, const Item<R>* items, int64_t n, int T, const double* iv, uint8_t* ts_of)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int sel = 0;
    if (items[i].good) {
        const double t = lha[i];
        int k = 1;
        double v = iv[1];
        while (t > v) {
            k++;
            if (k < T + 1)
                v = iv[k];
            else
                break;
        }
        sel = min(k - 1, T - 1);
    }
    ts_of[i] = uint8_t(sel);
}

// Mean hour angle of the good visibilities of each step (0 when empty); one
// block per step, fixed-order reduction.
template <typename R>
__global__ void __launch_bounds__(256) k_lha_means(const double* lha, const Item<R>* items, const uint8_t* ts_of,
    int64_t n, double* mean)
{
    const int ts = blockIdx.x;
    __shared__ double ssum[256];
    __shared__ unsigned long long scnt[256];
    double s = 0.0;
    unsigned long long c = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
        if (items[i].good && ts_of[i] == ts) {
            s += lha[i];
            c++;
        }
    ssum[threadIdx.x] = s;
    scnt[threadIdx.x] = c;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            ssum[threadIdx.x] += ssum[threadIdx.x + h];
            scnt[threadIdx.x] += scnt[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        mean[ts] = scnt[0] ? ssum[0] / double(scnt[0]) : 0.0;
}

// Parallactic angle of each step's mean hour angle (hours), with the
// reference's formula (the pointing RA stands where an observatory latitude
// would).
__global__ void k_parangle(const double* lha_mean, int T, double dec_rad, double ra_rad, double* angle)
{
    const int t = threadIdx.x;
    if (t >= T)
        return;
    const double ha = lha_mean[t] * (15.0 * kApPi / 180.0);
    const double s = cos(ra_rad) * sin(ha);
    const double c = sin(ra_rad) * cos(dec_rad) - cos(ra_rad) * sin(dec_rad) * cos(ha);
    angle[t] = atan2(s, c);
}

// |Y_l^m(theta, phi)| of the orthonormal real spherical harmonics
// (m > 0: sqrt2 K P_l^m(cos theta) cos(m phi); m < 0: sqrt2 K P_l^|m| sin(|m| phi);
// m = 0: K P_l^0, K = sqrt((2l+1)/(4 pi) (l-|m|)!/(l+|m|)!)), the associated
// Legendre function from the upward recurrence in l (the sign convention
// drops out of the magnitude).
__device__ __host__ inline double sh_abs(int l, int m, double phi, double theta)
{
    const int am = m < 0 ? -m : m;
    const double x = cos(theta), s = fabs(sin(theta));
    double pmm = 1.0, f = 1.0;
    for (int i = 1; i <= am; i++) {
        pmm *= f * s;
        f += 2.0;
    }
    double p = pmm;
    if (l > am) {
        double pm2 = pmm, pm1 = x * (2.0 * am + 1.0) * pmm;
        p = pm1;
        for (int ll = am + 2; ll <= l; ll++) {
            p = ((2.0 * ll - 1.0) * x * pm1 - (ll + am - 1.0) * pm2) / double(ll - am);
            pm2 = pm1;
            pm1 = p;
        }
    }
    double ratio = 1.0;
    for (int k = l - am + 1; k <= l + am; k++)
        ratio /= double(k);
    double v = sqrt((2.0 * l + 1.0) / (4.0 * kApPi) * ratio) * p;
    if (m > 0)
        v *= 1.4142135623730950488 * cos(double(m) * phi);
    else if (m < 0)
        v *= 1.4142135623730950488 * sin(double(am) * phi);
    return fabs(v);
}

// Inverse primary beam on the workarea, one map per angle:
// A[a][row][col] = 1 / sum_m |Y_deg^m(phi + angle[a], theta) c_m| with row,
// col = centre + (j, i) and theta = |(j, i)| fov / workarea,
// phi = atan(i / j) (pi/2 on j = 0).
__global__ void k_aproj_beam(int nA, int wa, double fov, const double* coefs, int deg, const double* angle, double* A)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(nA) * wa * wa)
        return;
    const int a = int(t / (int64_t(wa) * wa));
    const int rem = int(t % (int64_t(wa) * wa));
    const int row = rem / wa, col = rem % wa;
    const int c = wa / 2;
    const int j = row - c, i = col - c;
    const double j_rad = double(j) * fov / double(wa);
    const double i_rad = double(i) * fov / double(wa);
    const double theta = sqrt(j_rad * j_rad + i_rad * i_rad);
    const double phi = j != 0 ? atan(i_rad / j_rad) : kApPi / 2.0;
    const double rot = angle ? angle[a] : 0.0;
    double sum = 0.0;
    for (int m = -deg; m <= deg; m++)
        sum += fabs(sh_abs(deg, m, phi + rot, theta) * coefs[deg + m]);
    A[t] = 1.0 / sum;
}

// W-screen x inverse beam for images g = p * nA + a (arr x arr, row-major,
// row = u offset, column = v offset, zero outside the filled corners; the
// caller clears the buffer): tmp(i, j) = comb(i, j) * A(half + i, half + j)
// for |offsets| < half (aw_projection.cpp:305-345 with the W-screen of
// :50-111).
__global__ void k_aproj_screen(WkParams q, int P, int nA, const double* A, double2* buf)
{
    const int half = q.half, arr = q.arr, span = 2 * half - 1;
    const int64_t per = int64_t(span) * span;
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(P) * nA * per)
        return;
    const int g = int(t / per);
    const int rem = int(t % per);
    const int ao = rem / span - (half - 1), bo = rem % span - (half - 1);
    const int p = g / nA, a = g % nA;
    const double w = q.w_avg[p];
    const int ai = ao < 0 ? -ao : ao, bi = bo < 0 ? -bo : bo;
    double2 v;
    if (ai == 0 && bi == 0)
        v = make_double2(q.aa[half] * q.aa[half], 0.0);
    else if (bi == 0)
        v = wk_value(q, w, ai, 0);
    else if (ai == 0)
        v = wk_value(q, w, bi, 0); // output(0, i) holds value(i, 0)
    else
        v = wk_value(q, w, ai, bi);
    const int wa = 2 * half;
    const double m = A[(int64_t(a) * wa + (half + ao)) * wa + (half + bo)];
    const int r = ao < 0 ? ao + arr : ao, c = bo < 0 ? bo + arr : bo;
    buf[int64_t(g) * arr * arr + int64_t(r) * arr + c] = make_double2(v.x * m, v.y * m);
}

// Truncated support of each transformed image (aw_projection.cpp:350-363):
// the last u offset i = k * os, i <= min(max_support * os, arr / 2), on the
// u axis whose magnitude exceeds trunc% of the centre; out[g * rep + r] for
// r < rep (the rotated-kernel option shares one support per plane).
__global__ void k_aproj_support(const double2* buf, int G, int arr, int os, int max_support, double trunc_perc,
    int rep, int* out)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G)
        return;
    const double2* conv = buf + int64_t(g) * arr * arr;
    int S = max_support;
    if (trunc_perc > 0.0) {
        const double minv = hypot(conv[0].x, conv[0].y) * (trunc_perc / 100.0);
        unsigned i = min(unsigned(max_support * os), unsigned(arr / 2));
        while (i > 0) {
            const double2 v = conv[int64_t(i) * arr];
            if (hypot(v.x, v.y) > minv)
                break;
            i -= unsigned(os);
        }
        S = int(min(i / unsigned(os), unsigned(max_support)));
    }
    for (int r = 0; r < rep; r++)
        out[g * rep + r] = S;
}

// rotate_matrix of an fftshift-ed kernel, shifted back: dst = fftshift(
// rotate(fftshift(src), angle, fill = fftshift(src)(0, 0))), one thread per
// output sample; bilinear interpolation with the reference's edge rules
// (positions below -1e-7 step to the previous sample, positions within 1e-7
// of the last sample use it alone).
__global__ void k_aproj_rotate(const double2* src, int64_t src_stride, double2* dst, int64_t dst_stride, int G,
    int arr, const double* angles, int step)
{
    const double angle = angles[step];
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(G) * arr * arr)
        return;
    const int g = int(t / (int64_t(arr) * arr));
    const int rem = int(t % (int64_t(arr) * arr));
    const int ro = rem / arr, co = rem % arr; // output sample (unshifted)
    const int h = arr / 2;
    const double2* in = src + g * src_stride;
    auto S = [&](int row, int col) { return in[int64_t((row + h) % arr) * arr + (col + h) % arr]; };
    const int j = (ro + h) % arr, i = (co + h) % arr; // shifted output row j, column i
    const double cosa = cos(angle), sina = sin(angle);
    const double centre = double(arr) / 2 - 0.5;
    // products rounded, then added left to right (no fused multiply-add), so
    // that the truncations below see the same positions as the host code
    const double cj = __dmul_rn(cosa, double(j) - centre), si = __dmul_rn(sina, double(i) - centre);
    const double sj = __dmul_rn(sina, double(j) - centre), ci = __dmul_rn(cosa, double(i) - centre);
    const double vpos = __dadd_rn(__dadd_rn(cj, si), centre);
    const double hpos = __dadd_rn(__dadd_rn(-sj, ci), centre);
    constexpr double tol = 10e-8;
    int top = int(vpos), bottom = top + 1, left = int(hpos), right = left + 1;
    if (vpos < -tol) {
        top -= 1;
    } else {
        const int rv = int(round(vpos));
        if (rv == arr - 1 && (vpos - double(rv)) < tol) {
            top = rv;
            bottom = top;
        }
    }
    if (hpos < -tol) {
        left -= 1;
    } else {
        const int rh = int(round(hpos));
        if (rh == arr - 1 && (hpos - double(rh)) < tol) {
            left = rh;
            right = left;
        }
    }
    double2 v;
    if (top >= 0 && bottom < arr && left >= 0 && right < arr) {
        const double2 tl = S(top, left), tr = S(top, right), bl = S(bottom, left), br = S(bottom, right);
        const double hd = hpos - double(left), vd = vpos - double(top);
        const double2 tb = make_double2(tl.x + hd * (tr.x - tl.x), tl.y + hd * (tr.y - tl.y));
        const double2 bb = make_double2(bl.x + hd * (br.x - bl.x), bl.y + hd * (br.y - bl.y));
        v = make_double2(tb.x + vd * (bb.x - tb.x), tb.y + vd * (bb.y - tb.y));
    } else {
        v = S(0, 0);
    }
    dst[g * dst_stride + int64_t(ro) * arr + co] = v;
}

// Kernel tables of combined plane pt (blockIdx.x) and oversampled offset pair
// (cy, cx) (blockIdx.y): tap (i, j) = conv(du, dv) / sum Re over the K x K
// taps, du = (j - S) os + os/2 - cx, dv = (i - S) os + os/2 - cy (mod arr),
// as generate_kernel_cache reads the FFT (aw_projection.cpp:415-448; the sum
// runs u-outer, v-inner).  Table pt starts at off[pt] = sum over q < pt of
// cs^2 K_q^2.
template <typename R>
__global__ void __launch_bounds__(256) k_aproj_expand(const double2* conv_base, int arr, const int* support, int cs,
    int os, typename Cplx<R>::T* out, uint32_t* off)
{
    const int pt = blockIdx.x;
    const int pair = blockIdx.y;
    const int cy = pair / cs, cx = pair % cs;
    uint32_t base = 0;
    for (int q = 0; q < pt; q++) {
        const uint32_t Kq = uint32_t(2 * support[q] + 1);
        base += uint32_t(cs) * uint32_t(cs) * Kq * Kq;
    }
    if (pair == 0 && threadIdx.x == 0)
        off[pt] = base;
    const int S = support[pt];
    const int K = 2 * S + 1;
    const double2* conv = conv_base + int64_t(pt) * arr * arr;
    auto at = [&](int i, int j) {
        int du = (j - S) * os + os / 2 - cx, dv = (i - S) * os + os / 2 - cy;
        du = ((du % arr) + arr) % arr;
        dv = ((dv % arr) + arr) % arr;
        return conv[int64_t(du) * arr + dv];
    };
    __shared__ double red[256];
    double ks = 0.0;
    for (int t = threadIdx.x; t < K * K; t += blockDim.x) {
        const int j = t / K, i = t % K; // u outer, v inner
        ks += at(i, j).x;
    }
    red[threadIdx.x] = ks;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    const double inv = 1 / red[0];
    typename Cplx<R>::T* dst = out + base + uint32_t(pair) * uint32_t(K * K);
    for (int t = threadIdx.x; t < K * K; t += blockDim.x) {
        const int i = t / K, j = t % K;
        const double2 v = at(i, j);
        typename Cplx<R>::T o;
        o.x = R(v.x * inv);
        o.y = R(v.y * inv);
        dst[t] = o;
    }
}

} // namespace stpgpu
