"""CPU oracle for the FastImaging snapshot imager and source finder.

TEST INFRASTRUCTURE ONLY: the checker that the CUDA product is compared with.
Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  It is never on the product path.

The loops live in ``stp_oracle.cpp`` (built into ``liboracle.so``); this
module orchestrates them the way the reference's ``stp::image_visibilities``
(``src/stp/imager/imager.h:233-376``), ``stp::convolve_to_grid``
(``src/stp/gridder/gridder.h:240-997``) and ``stp::SourceFindImage``
(``src/stp/sourcefind/sourcefind.cpp:156-292``) do, with ``scipy.fft`` in place
of FFTW 3.3.5 (unnormalised transforms with FFTW's sign conventions).

Parity pins: the restatement is checked against every inline known answer of
the reference's own gtest suite (tests/golden/reference_pins.json, generated
from the reference test sources by tests/golden/make_reference_pins.py).  The
reference's NPZ golden images (the ``test-data`` submodule) are not in the
reference tree, so whole-imager parity against the original binary is
unpinned; the imager is pinned through the gridder/kernel/conv unit pins.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
import threading
from dataclasses import dataclass, field

import numpy as np
import scipy.fft

HERE = os.path.dirname(os.path.abspath(__file__))

# Enum values, same order as src/stp/types.h:32-89.
TopHat, Triangle, Sinc, Gaussian, GaussianSinc, PSWF = range(6)
ZEROMEDIAN, BINMEDIAN, BINAPPROX, NTHELEMENT = range(4)
LINEAR, CUBIC, COSINE = range(3)

_lib_lock = threading.Lock()
_libs: dict = {}

_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i64p = ctypes.POINTER(ctypes.c_int64)


def _build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(fast: bool = False):
    """Load (building on first use) the oracle shared library."""
    name = "liboracle_fast.so" if fast else "liboracle.so"
    with _lib_lock:
        if name in _libs:
            return _libs[name]
        path = os.path.join(HERE, name)
        src = os.path.join(HERE, "stp_oracle.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            _build()
        L = ctypes.CDLL(path)
        L.orc_grid_prepass.restype = ctypes.c_double
        L.orc_median_exact.restype = ctypes.c_double
        L.orc_estimate_rms.restype = ctypes.c_double
        L.orc_wkernel_truncate.restype = ctypes.c_int
        L.orc_num_threads.restype = ctypes.c_int
        _libs[name] = L
        return L


def _d(a):
    return a.ctypes.data_as(_dp)


def _i32(a):
    return a.ctypes.data_as(_i32p)


def _u32(a):
    return a.ctypes.data_as(_u32p)


def _i64(a):
    return a.ctypes.data_as(_i64p)


def arc_sec_to_rad(v):
    """gridder.h:20."""
    return (v / 3600.0) * (math.pi / 180.0)


# ------------------------------------------------------------------ kernels

def kernel_eval(kf, trunc, r):
    r = np.ascontiguousarray(r, dtype=np.float64)
    out = np.empty_like(r)
    lib().orc_kernel_eval(ctypes.c_int(kf), ctypes.c_double(trunc), _d(r), _d(out), ctypes.c_int64(r.size))
    return out


def gcf_eval(kf, r):
    r = np.ascontiguousarray(r, dtype=np.float64)
    out = np.empty_like(r)
    lib().orc_gcf_eval(ctypes.c_int(kf), _d(r), _d(out), ctypes.c_int64(r.size))
    return out


def make_1d_kernel(kf, trunc, support, offset, oversampling=1, pad=False, normalize=True):
    n = 2 * (support + (1 if pad else 0)) * oversampling + 1
    out = np.empty(n)
    lib().orc_make_1d_kernel(ctypes.c_int(kf), ctypes.c_double(trunc), ctypes.c_int(support), ctypes.c_double(offset),
                             ctypes.c_int(oversampling), ctypes.c_int(int(pad)), ctypes.c_int(int(normalize)), _d(out))
    return out


def make_kernel_array(kf, trunc, support, offset, oversampling=1, pad=False, normalize=True):
    n = 2 * (support + (1 if pad else 0)) * oversampling + 1
    out = np.empty(n * n)
    lib().orc_make_kernel_array(ctypes.c_int(kf), ctypes.c_double(trunc), ctypes.c_int(support),
                                ctypes.c_double(offset[0]), ctypes.c_double(offset[1]), ctypes.c_int(oversampling),
                                ctypes.c_int(int(pad)), ctypes.c_int(int(normalize)), _d(out))
    return out.reshape((n, n), order="F")


def kernel_table_1d(kf, trunc, support, oversampling):
    cs = (oversampling // 2) * 2 + 1
    out = np.empty(cs * (2 * support + 1))
    lib().orc_kernel_table_1d(ctypes.c_int(kf), ctypes.c_double(trunc), ctypes.c_int(support),
                              ctypes.c_int(oversampling), _d(out))
    return out.reshape(cs, 2 * support + 1)


def populate_kernel_cache(kf, trunc, support, oversampling):
    """gridder.h:73-105 as a dict {(cp_y, cp_x): K x K matrix}."""
    t = kernel_table_1d(kf, trunc, support, oversampling)
    cs = t.shape[0]
    return {(y, x): np.outer(t[y], t[x]) for y in range(cs) for x in range(cs)}


def oversampled_indices(frac, oversampling):
    frac = np.ascontiguousarray(frac, dtype=np.float64)
    out = np.empty(frac.shape, dtype=np.int32)
    lib().orc_oversampled_indices(_d(frac), ctypes.c_int64(frac.size), ctypes.c_int(oversampling), _i32(out))
    return out


def img_dom_kernel(kf, trunc, n, analytic_gcf):
    """ImgDomKernel, conv_func.h:351-412 (normalize=false)."""
    centre = n // 2
    lin = np.arange(n, dtype=np.float64) - centre
    if analytic_gcf:
        return gcf_eval(kf, lin / centre)
    k1 = kernel_eval(kf, trunc, lin)
    s = float(np.sum(k1))
    if s > 0.0:
        k1 = k1 / s
    arr = np.zeros(n)
    arr[:centre] = k1[centre:centre + centre]
    arr[n - centre:n - centre + centre] = k1[:centre]
    # FFTW_R2HC real parts r_0..r_{n/2}
    re = scipy.fft.rfft(arr).real
    aa = np.zeros(n)
    half = n // 2
    aa[half:half + half] = re[:half]
    aa[half - np.arange(1, half + 1)] = re[1:half + 1]
    return aa


# ------------------------------------------------------------------ gridder

@dataclass
class WProj:
    num_wplanes: int = 0
    max_wpconv_support: int = 0
    undersampling_opt: int = 1
    kernel_trunc_perc: float = 0.0
    wplanes_median: bool = False
    hankel_opt: bool = False
    hankel_proj_slice: bool = False
    interp_type: int = LINEAR

    @property
    def enabled(self):
        return self.num_wplanes > 0


@dataclass
class GridResult:
    vis_grid: np.ndarray
    sampling_grid: np.ndarray
    sample_grid_total: float
    plane_supports: list = field(default_factory=list)
    plane_w: list = field(default_factory=list)


def _wkernel_workarea(image_size, kernel_size, undersampling_opt):
    """gridder.h:467-483."""
    u = int(2 ** (undersampling_opt - 1)) if undersampling_opt > 0 else 0
    wa = 2
    if u > 0:
        while (wa // u) < kernel_size:
            wa *= 2
    else:
        while wa < image_size:
            wa *= 2
    return wa


def wkernel_plane(w_value, aa, workarea, oversampling, cell_size_arcsec, scaling, max_support, trunc_perc,
                  current_support):
    """One W-plane: aw_projection.cpp:173-210 then :366-452.

    Returns (support, cache[cs*cs, K, K] complex, column-major K x K)."""
    L = lib()
    arr = workarea * oversampling
    comb = np.empty(2 * arr * arr)
    aa = np.ascontiguousarray(aa, dtype=np.float64)
    L.orc_wkernel_image_domain(ctypes.c_double(w_value), _d(aa), ctypes.c_int(workarea), ctypes.c_int(oversampling),
                               ctypes.c_double(arc_sec_to_rad(cell_size_arcsec)), ctypes.c_double(scaling), _d(comb))
    M = comb.view(np.complex128).reshape((arr, arr), order="F")
    conv = scipy.fft.fft2(M)
    convF = np.asfortranarray(conv).reshape(-1, order="F").view(np.float64).copy()
    support = L.orc_wkernel_truncate(_d(convF), ctypes.c_int64(arr), ctypes.c_int(max_support),
                                     ctypes.c_int(oversampling), ctypes.c_double(trunc_perc),
                                     ctypes.c_int(current_support))
    cs = (oversampling // 2) * 2 + 1
    K = 2 * support + 1
    cache = np.empty(2 * cs * cs * K * K)
    L.orc_wkernel_cache(_d(convF), ctypes.c_int64(arr), ctypes.c_int(support), ctypes.c_int(oversampling), _d(cache))
    return support, cache


def besselj1(x):
    """The reference's order-1 Bessel function (besselj1,
    aw_projection.cpp:490-508): a rational approximation for x < 8 and the
    asymptotic form with z = 8/x above (the published Hart coefficients of
    Numerical Recipes' bessj1, about 1e-8 absolute accuracy), Horner-evaluated
    in the reference's order.  x >= 0."""
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    lo = x < 8.0
    xl = x[lo]
    xx = xl * xl
    num = (72362614232.0, -7895059235.0, 242396853.1, -2972611.439, 15704.48260, -30.16036606)
    den = (144725228442.0, 2300535178.0, 18583304.74, 99447.43394, 376.9991397, 1.0)
    p = np.full_like(xl, num[5])
    q = np.full_like(xl, den[5])
    for k in range(4, -1, -1):
        p = num[k] + xx * p
        q = den[k] + xx * q
    out[lo] = (xl * p) / q
    xh = x[~lo]
    a = (1.0, 0.183105e-2, -0.3516396496e-4, 0.2457520174e-5, -0.240337019e-6)
    b = (0.04687499995, -0.2002690873e-3, 0.8449199096e-5, -0.88228987e-6, 0.105787412e-6)
    z = 8.0 / xh
    zz = z * z
    y = xh - 2.356194491
    p = np.full_like(xh, a[4])
    q = np.full_like(xh, b[4])
    for k in range(3, -1, -1):
        p = a[k] + zz * p
        q = b[k] + zz * q
    out[~lo] = np.sqrt(0.636619772 / xh) * (np.cos(y) * p - z * np.sin(y) * q)
    return out


def dht_matrix(n, j1=None):
    """Discrete Hankel transform matrix, stored transposed: D[j, i] is the
    weight of radial sample j in output i (WideFieldImaging::dht,
    aw_projection.cpp:532-596).  Sample j covers the annulus [rn_{j-1}, rn_j]
    with rn_j = j + 1/2 (rn_{n-1} = n - 1); output i is the order-0 Hankel
    transform at k_i = pi i / n of the piecewise-constant profile:
    D[j, 0] = pi (rn_j^2 - rn_{j-1}^2), D[j, i] = F_i(j) - F_i(j-1) with
    F_i(j) = (2 pi / k_i) rn_j J1(k_i rn_j).  J1 is the reference's rational
    approximation (besselj1 above) unless another function is given."""
    if j1 is None:
        j1 = besselj1

    idx = np.arange(n, dtype=np.float64)
    k = (np.pi / n) * idx
    rn = idx + 0.5
    rn[n - 1] = n - 1
    D = np.empty((n, n))
    area = np.pi * rn * rn
    D[0, 0] = area[0]
    D[1:, 0] = area[1:] - area[:-1]
    kn = (2.0 * np.pi) / k[1:]
    F = kn[None, :] * rn[:, None] * j1(k[None, 1:] * rn[:, None])
    D[0, 1:] = F[0]
    D[1:, 1:] = F[1:] - F[:-1]
    return D


def spline_coefficients(y, cubic):
    """tk::spline over unit-spaced nodes x_i = i (aw_projection.h:154-160 ->
    spline.h set_points with the default natural boundary, f'' = 0 at both
    ends).  Returns (a, b, c) with f(x_k + t) = ((a_k t + b_k) t + c_k) t + y_k
    for k < n-1 and the end segment k = n-1 extrapolating (a = 0, b = b_{n-1},
    c = f'(x_{n-1})); linear: a = b = 0, c_k = y_{k+1} - y_k, c_{n-1} = c_{n-2}."""
    from scipy.linalg import solve_banded

    y = np.asarray(y, dtype=np.float64)
    n = y.size
    a = np.zeros(n)
    b = np.zeros(n)
    c = np.zeros(n)
    if not cubic:
        c[:-1] = y[1:] - y[:-1]
        c[-1] = c[-2]
        return a, b, c
    ab = np.zeros((3, n))
    ab[0, 2:] = 1.0 / 3.0   # A(i, i+1), rows 1..n-2
    ab[1, :] = 4.0 / 3.0    # A(i, i)
    ab[2, :-2] = 1.0 / 3.0  # A(i, i-1), rows 1..n-2
    ab[1, 0] = 2.0          # 2 b_0 = f''(x_0) = 0
    ab[0, 1] = 0.0
    ab[1, n - 1] = 2.0      # 2 b_{n-1} = 0
    ab[2, n - 2] = 0.0
    rhs = np.zeros(n)
    rhs[1:-1] = (y[2:] - y[1:-1]) - (y[1:-1] - y[:-2])
    b = solve_banded((1, 1), ab, rhs)
    a[:-1] = 1.0 / 3.0 * (b[1:] - b[:-1])
    c[:-1] = (y[1:] - y[:-1]) - 1.0 / 3.0 * (2.0 * b[:-1] + b[1:])
    a[-1] = 0.0
    c[-1] = 3.0 * a[-2] + 2.0 * b[-2] + c[-2]
    return a, b, c


def hankel_wkernel_plane(w_value, aa, workarea, oversampling, cell_size_arcsec, scaling, max_support, trunc_perc,
                         current_support, proj_slice=False, interp_type=LINEAR):
    """One W-plane with hankel_opt: generate_convolution_kernel_wproj's
    Hankel branch (aw_projection.cpp:211-287), RadialInterpolate
    (aw_projection.h:126-214) and the Hankel branch of generate_kernel_cache
    (aw_projection.cpp:378-412).  Same return layout as wkernel_plane."""
    os_ = int(oversampling)
    arr = workarea * os_
    half = workarea // 2
    scaled = arc_sec_to_rad(cell_size_arcsec) * scaling
    aa = np.asarray(aa, dtype=np.float64)

    def value(px, py):  # combine_2d_kernel_value, aw_projection.cpp:455-474
        dx = px * scaled
        dy = py * scaled
        r2 = dx * dx + dy * dy
        a = aa[half + px] * aa[half + py]
        with np.errstate(invalid="ignore"):
            nn = np.sqrt(1.0 - np.minimum(r2, 1.0))
            v = (np.exp(1j * ((-2.0 * np.pi) * w_value * (nn - 1.0))) / np.where(nn > 0, nn, 1.0)) * a
        return np.where(r2 >= 1.0, a + 0j, v)

    if not proj_slice:
        j = np.arange(half)
        dx = j * scaled
        r2 = dx * dx
        with np.errstate(invalid="ignore"):
            nn = np.sqrt(1.0 - np.minimum(r2, 1.0))
            tmp = np.exp(1j * ((-2.0 * np.pi) * w_value * (nn - 1.0))) / np.where(nn > 0, nn, 1.0)
        tmp = np.where(r2 >= 1.0, 1.0 + 0j, tmp)
        radial = tmp * aa[half + j]
        n = arr // 2
        D = dht_matrix(n)
        Y = D[:half, :].T @ radial
    else:
        # projection onto one axis (generate_projected_image_domain_kernel, aw_projection.cpp:113-170)
        ii, jj = np.meshgrid(np.arange(half), np.arange(half), indexing="ij")
        V = value(ii, jj)  # V[i, j] = value(i, j)
        P = np.empty(half, dtype=np.complex128)
        P[0] = 2.0 * V[1:, 0].sum() + aa[half] * aa[half]
        P[1:] = V[1:, 0] + 2.0 * V[1:, 1:].sum(axis=0)
        out = np.zeros(arr, dtype=np.complex128)
        out[:half] = P
        out[arr - np.arange(1, half)] = P[1:]
        Y = np.fft.fft(out)
        n = arr
    # truncation (aw_projection.h:135-148)
    S = int(current_support)
    if trunc_perc > 0.0:
        minv = abs(Y[0]) * (trunc_perc / 100.0)
        t = int(max_support) * os_
        while t > os_:
            if abs(Y[t]) > minv:
                break
            t -= os_
        S = min(int(math.ceil(float(t) * (1.0 / os_))), int(max_support))
    cubic = interp_type == CUBIC
    ar, br, cr = spline_coefficients(Y.real, cubic)
    ai, bi, ci = spline_coefficients(Y.imag, cubic)
    ko = (S * 2 + 2) * os_ // 2
    size = ko + ko * (ko - 1) // 2
    hq = np.empty(size, dtype=np.complex128)
    i = 0
    for row in range(ko):  # half quadrant, row `row` holds columns row..ko-1
        for col in range(row, ko):
            if col == 0:
                x = float(row)
            elif row == 0:
                x = float(col)
            else:
                x = math.sqrt(float(row * row + col * col))
            k = min(int(x), n - 1)
            t = x - k
            hq[i] = complex(((ar[k] * t + br[k]) * t + cr[k]) * t + Y.real[k],
                            ((ai[k] * t + bi[k]) * t + ci[k]) * t + Y.imag[k])
            i += 1
    cs = (os_ // 2) * 2 + 1
    K = 2 * S + 1
    cache = np.empty((cs * cs, K * K), dtype=np.complex128)
    for x in range(cs):
        for y in range(cs):
            tmp = np.empty((K, K), dtype=np.complex128)  # tmp[tx, ty]
            ksum = 0.0
            for ty in range(K):
                cx = (ty - S) * os_ + os_ // 2 - x
                dcx = abs(cx)
                for tx in range(K):
                    cy = (tx - S) * os_ + os_ // 2 - y
                    dcy = abs(cy)
                    if dcx > dcy:
                        vi = dcy * ko - ((dcy * (dcy + 1)) >> 1) + dcx
                    else:
                        vi = dcx * ko - ((dcx * (dcx + 1)) >> 1) + dcy
                    tmp[tx, ty] = hq[vi]
                    ksum += hq[vi].real
            cache[y * cs + x] = (tmp / ksum).reshape(-1, order="F")
    return S, cache.reshape(-1).view(np.float64).copy()


@dataclass
class AProj:
    """stp::A_ProjectionPars (types.h:255-316): num_timesteps > 0 enables it."""
    num_timesteps: int = 0
    obs_dec: float = 0.0
    obs_ra: float = 0.0
    aproj_opt: bool = False
    lha: np.ndarray | None = None
    pbeam_coefs: list | None = None

    @property
    def enabled(self):
        return self.num_timesteps > 0


def _linspace(start, end, num):
    """arma::linspace: start + i * delta for i < num - 1, the last point = end."""
    delta = (end - start) / float(num - 1)
    out = start + np.arange(num, dtype=np.float64) * delta
    out[num - 1] = end
    return out


def average_lha_planes(lha, good, num_timesteps):
    """gridder.cpp:148-200.  lha in the gridder's (|w|-sorted) order; returns
    (mean hour angle per step, step of each visibility; 0 where not good)."""
    lha = np.asarray(lha, dtype=np.float64)
    T = int(num_timesteps)
    lo, hi = float(lha.min()), float(lha.max())
    step = (hi - lo) / T
    iv = _linspace(lo - step / 2, hi + step / 2, T + 1)
    ts = np.zeros(lha.size, dtype=np.int64)
    planes = np.zeros(T)
    count = np.zeros(T, dtype=np.int64)
    for i in np.nonzero(np.asarray(good) != 0)[0]:
        t = lha[i]
        k = 1
        v = iv[1]
        while t > v:
            k += 1
            if k < T + 1:
                v = iv[k]
            else:
                break
        sel = k - 1
        ts[i] = sel
        planes[sel] += t
        count[sel] += 1
    planes = np.where(count > 0, planes / np.maximum(count, 1), 0.0)
    return planes, ts


def parangle(ha, dec_rad, ra_rad):
    """aw_projection.cpp:599-608 (the pointing RA where a latitude would stand)."""
    h = ha * (15.0 * math.pi / 180.0)
    s_ = math.cos(ra_rad) * math.sin(h)
    c_ = math.sin(ra_rad) * math.cos(dec_rad) - math.cos(ra_rad) * math.sin(dec_rad) * math.cos(h)
    return math.atan2(s_, c_)


def sh_abs(l, m, phi, theta):
    """|real spherical harmonic Y_l^m(theta, phi)| (orthonormal; the
    reference's sh::EvalSH from google/spherical-harmonics, un-vendored
    submodule, restated from the definition): sqrt2 K |P_l^|m|(cos theta)|
    |cos(m phi)| for m > 0, |sin(|m| phi)| for m < 0, K |P_l^0| for m = 0."""
    phi = np.asarray(phi, dtype=np.float64)
    theta = np.asarray(theta, dtype=np.float64)
    am = abs(m)
    x = np.cos(theta)
    sn = np.abs(np.sin(theta))
    pmm = np.ones_like(x)
    f = 1.0
    for _ in range(am):
        pmm = pmm * (f * sn)
        f += 2.0
    p = pmm
    if l > am:
        pm2 = pmm
        pm1 = x * (2.0 * am + 1.0) * pmm
        p = pm1
        for ll in range(am + 2, l + 1):
            p = ((2.0 * ll - 1.0) * x * pm1 - (ll + am - 1.0) * pm2) / float(ll - am)
            pm2, pm1 = pm1, p
    ratio = 1.0
    for k in range(l - am + 1, l + am + 1):
        ratio /= float(k)
    v = math.sqrt((2.0 * l + 1.0) / (4.0 * math.pi) * ratio) * p
    if m > 0:
        v = v * (math.sqrt(2.0) * np.cos(float(m) * phi))
    elif m < 0:
        v = v * (math.sqrt(2.0) * np.sin(float(am) * phi))
    return np.abs(v)


def generate_a_kernel(coefs, fov, workarea, rot_angle=0.0):
    """gridder.cpp:243-275: A[j + c, i + c] = 1 / sum_m |Y_deg^m(phi + rot,
    theta) c_m| with theta = |(j, i)| fov / workarea, phi = atan(i / j)
    (pi/2 for j = 0)."""
    coefs = np.asarray(coefs, dtype=np.float64)
    deg = int((coefs.size - 1) // 2)
    c = workarea // 2
    j = np.arange(-c, c, dtype=np.float64)[:, None]
    i = np.arange(-c, c, dtype=np.float64)[None, :]
    j_rad = j * fov / float(workarea)
    i_rad = i * fov / float(workarea)
    theta = np.sqrt(j_rad * j_rad + i_rad * i_rad)
    with np.errstate(divide="ignore", invalid="ignore"):
        phi = np.where(j != 0, np.arctan(i_rad / np.where(j != 0, j_rad, 1.0)), math.pi / 2.0)
    acc = np.zeros((workarea, workarea))
    for m in range(-deg, deg + 1):
        acc = acc + np.abs(sh_abs(deg, m, phi + rot_angle, theta) * coefs[deg + m])
    return 1.0 / acc


def rotate_matrix_cx(m, angle, cval):
    """matrix_math.cpp:715-733 (complex rotate_matrix, out_size = in_size):
    bilinear rotation about (n/2 - 0.5, n/2 - 0.5) with the reference's edge
    rules; samples that fall outside take cval."""
    n = m.shape[1]
    tol = 10e-8
    cosa = math.cos(angle)
    sina = math.sin(angle)
    ctr = float(n) / 2 - 0.5
    idx = np.arange(n, dtype=np.float64)
    sa = sina * (idx - ctr)
    ca = cosa * (idx - ctr)
    V = (ca[:, None] + sa[None, :]) + ctr   # out(j, i): row j, column i
    H = (-sa[:, None] + ca[None, :]) + ctr
    top = V.astype(np.int64)
    left = H.astype(np.int64)
    bottom = top + 1
    right = left + 1

    def cround(x):
        return np.where(x >= 0, np.floor(x + 0.5), np.ceil(x - 0.5)).astype(np.int64)

    negv = V < -tol
    top = np.where(negv, top - 1, top)
    rv = cround(V)
    edge = (~negv) & (rv == n - 1) & ((V - rv) < tol)
    top = np.where(edge, rv, top)
    bottom = np.where(edge, rv, bottom)
    negh = H < -tol
    left = np.where(negh, left - 1, left)
    rh = cround(H)
    edgeh = (~negh) & (rh == n - 1) & ((H - rh) < tol)
    left = np.where(edgeh, rh, left)
    right = np.where(edgeh, rh, right)
    ok = (top >= 0) & (bottom < n) & (left >= 0) & (right < n)
    t_, b_ = np.clip(top, 0, n - 1), np.clip(bottom, 0, n - 1)
    l_, r_ = np.clip(left, 0, n - 1), np.clip(right, 0, n - 1)
    tl, tr, bl, br = m[t_, l_], m[t_, r_], m[b_, l_], m[b_, r_]
    hd = H - left
    vd = V - top
    tb = tl + hd * (tr - tl)
    bb = bl + hd * (br - bl)
    out = tb + vd * (bb - tb)
    return np.where(ok, out, cval)


def _aproj_conv(comb, A, workarea, oversampling):
    """generate_convolution_kernel_aproj before the truncation
    (aw_projection.cpp:290-348): the W-screen times the beam on the
    workarea's corners, then the forward 2-D FFT."""
    arr = workarea * oversampling
    half = workarea // 2
    rows = np.concatenate([np.arange(0, half), np.arange(arr - half, arr)])
    offs = np.concatenate([np.arange(0, half), np.arange(-half, 0)])
    tmp = np.zeros((arr, arr), dtype=np.complex128)
    tmp[np.ix_(rows, rows)] = comb[np.ix_(rows, rows)] * A[np.ix_(half + offs, half + offs)]
    return scipy.fft.fft2(tmp)


def _conv_truncate_and_cache(conv, arr, max_support, oversampling, trunc_perc, current):
    L = lib()
    convF = np.asfortranarray(conv).reshape(-1, order="F").view(np.float64).copy()
    support = L.orc_wkernel_truncate(_d(convF), ctypes.c_int64(arr), ctypes.c_int(max_support),
                                     ctypes.c_int(oversampling), ctypes.c_double(trunc_perc), ctypes.c_int(current))
    return support, convF


def _conv_cache(convF, arr, support, oversampling):
    L = lib()
    cs = (oversampling // 2) * 2 + 1
    K = 2 * support + 1
    cache = np.empty(2 * cs * cs * K * K)
    L.orc_wkernel_cache(_d(convF), ctypes.c_int64(arr), ctypes.c_int(support), ctypes.c_int(oversampling), _d(cache))
    return cache


def convolve_to_grid(kf, support, image_size, uv, vis, weights, kernel_exact=True, oversampling=1, shift_uv=True,
                     halfplane=True, generate_beam=True, wproj: WProj | None = None, w=None, cell_size=0.0,
                     analytic_gcf=True, threads=1, fast=False, trunc=None, aproj: AProj | None = None):
    """stp::convolve_to_grid, gridder.h:240-997.  uv in pixels (n x 2).

    ``trunc`` is the kernel functor's own parameter (truncation radius or
    half_base_width); ImageVisibilities builds the functor with
    trunc = kernel_support (imager.cpp:25-64), the default here."""
    L = lib(fast)
    trunc = float(support) if trunc is None else float(trunc)
    wproj = wproj or WProj()
    n = int(np.asarray(vis).size)
    uvc = np.asfortranarray(np.asarray(uv, dtype=np.float64).reshape(n, 2)).reshape(-1, order="F").copy()
    visc = np.ascontiguousarray(np.asarray(vis, dtype=np.complex128).reshape(-1)).view(np.float64).copy()
    wts = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1)).copy()
    use_wproj = wproj.enabled
    wc = np.zeros(n) if w is None else np.ascontiguousarray(np.asarray(w, dtype=np.float64).reshape(-1)).copy()
    conv_support = support
    if use_wproj:
        conv_support = int(wproj.max_wpconv_support)
        kernel_exact = False
    if kernel_exact:
        oversampling = 1
    else:
        oversampling = (oversampling >> 1) << 1
        if oversampling == 0:
            oversampling = 1
    good = np.empty(n, dtype=np.int32)
    kc = np.empty(2 * n, dtype=np.int32)
    cp = np.empty(2 * n, dtype=np.int32)
    frac = np.empty(2 * n)
    total = L.orc_grid_prepass(ctypes.c_int64(n), _d(uvc), _d(visc), _d(wts), _d(wc), ctypes.c_int(int(use_wproj)),
                               ctypes.c_int(conv_support), ctypes.c_int(image_size), ctypes.c_int(int(kernel_exact)),
                               ctypes.c_int(oversampling), ctypes.c_int(int(shift_uv)), ctypes.c_int(int(halfplane)),
                               _i32(good), _i32(kc), _i32(cp), _d(frac))
    image_rows = image_size // 2 + 1 if halfplane else image_size
    vg = np.zeros(2 * image_rows * image_size)
    sg = np.zeros(2 * image_rows * image_size) if generate_beam else np.zeros(2)
    empty = np.zeros(1)
    res = GridResult(None, None, total)

    def accumulate(kmode, k1d, wk, sup, b, e):
        L.orc_grid_accumulate(ctypes.c_int(kmode), ctypes.c_int(kf), ctypes.c_double(trunc), _d(k1d), _d(wk),
                              ctypes.c_int(sup), ctypes.c_int(image_size), ctypes.c_int(image_rows),
                              ctypes.c_int(oversampling), ctypes.c_int64(n), ctypes.c_int64(b), ctypes.c_int64(e),
                              _d(visc), _d(wts), _d(wc), _i32(good), _i32(kc), _i32(cp), _d(frac),
                              ctypes.c_int(int(generate_beam)), _d(vg), _d(sg), ctypes.c_int(threads))

    if kernel_exact:
        accumulate(1, empty, empty, support, 0, n)
    elif not use_wproj:
        k1d = np.ascontiguousarray(kernel_table_1d(kf, trunc, support, oversampling)).reshape(-1)
        accumulate(0, k1d, empty, support, 0, n)
    else:
        nplanes = int(wproj.num_wplanes)
        w_avg = np.empty(nplanes)
        first = np.empty(nplanes, dtype=np.int64)
        absw = np.abs(wc)
        L.orc_average_w_planes(_d(absw), _i32(good), ctypes.c_int64(n), ctypes.c_int(nplanes),
                               ctypes.c_int(int(wproj.wplanes_median)), _d(w_avg), _i64(first))
        kernel_size = 2 * conv_support + 1
        workarea = _wkernel_workarea(image_size, kernel_size, wproj.undersampling_opt)
        scaling = float(image_size) / float(workarea)
        aa = img_dom_kernel(kf, trunc, workarea, analytic_gcf)
        cur = int(wproj.max_wpconv_support)
        if aproj is not None and aproj.enabled:
            # A-projection (gridder.h:507-520,686-745): per plane and time step
            order = np.argsort(np.abs(np.ascontiguousarray(np.asarray(w, dtype=np.float64).reshape(-1))),
                               kind="stable")
            slha = np.asarray(aproj.lha, dtype=np.float64).reshape(-1)[order]
            T = int(aproj.num_timesteps)
            lha_planes, ts_of = average_lha_planes(slha, good, T)
            dec = (aproj.obs_dec * math.pi) / 180.0
            ra = (aproj.obs_ra * math.pi) / 180.0
            fov = arc_sec_to_rad(cell_size) * float(image_size)
            arr = workarea * oversampling
            angles = [parangle(float(lha_planes[t]), dec, ra) for t in range(T)]
            A0 = generate_a_kernel(aproj.pbeam_coefs, fov, workarea) if aproj.aproj_opt else None
            good_all = good.copy()
            for p in range(nplanes):
                b = int(first[p])
                e = n if p == nplanes - 1 else int(first[p + 1])
                comb = np.empty(2 * arr * arr)
                L.orc_wkernel_image_domain(ctypes.c_double(float(w_avg[p])), _d(np.ascontiguousarray(aa)),
                                           ctypes.c_int(workarea), ctypes.c_int(oversampling),
                                           ctypes.c_double(arc_sec_to_rad(cell_size)), ctypes.c_double(scaling),
                                           _d(comb))
                M = comb.view(np.complex128).reshape((arr, arr), order="F")
                if aproj.aproj_opt:
                    conv = _aproj_conv(M, A0, workarea, oversampling)
                    cur, _ = _conv_truncate_and_cache(conv, arr, int(wproj.max_wpconv_support), oversampling,
                                                      float(wproj.kernel_trunc_perc), cur)
                for t in range(T):
                    if aproj.aproj_opt:
                        sh = np.fft.fftshift(conv)
                        conv = np.fft.fftshift(rotate_matrix_cx(sh, angles[t], sh[0, 0]))
                        convF = np.asfortranarray(conv).reshape(-1, order="F").view(np.float64).copy()
                    else:
                        A = generate_a_kernel(aproj.pbeam_coefs, fov, workarea, angles[t])
                        conv = _aproj_conv(M, A, workarea, oversampling)
                        cur, convF = _conv_truncate_and_cache(conv, arr, int(wproj.max_wpconv_support),
                                                              oversampling, float(wproj.kernel_trunc_perc), cur)
                    cache = _conv_cache(convF, arr, cur, oversampling)
                    res.plane_supports.append(cur)
                    res.plane_w.append(float(w_avg[p]))
                    good[:] = np.where(ts_of == t, good_all, 0)
                    accumulate(2, empty, cache, cur, b, e)
            good[:] = good_all
            nplanes = 0
        for p in range(nplanes):
            b = int(first[p])
            e = n if p == nplanes - 1 else int(first[p + 1])
            if wproj.hankel_opt:
                cur, cache = hankel_wkernel_plane(float(w_avg[p]), aa, workarea, oversampling, cell_size, scaling,
                                                  int(wproj.max_wpconv_support), float(wproj.kernel_trunc_perc), cur,
                                                  bool(wproj.hankel_proj_slice), int(wproj.interp_type))
            else:
                cur, cache = wkernel_plane(float(w_avg[p]), aa, workarea, oversampling, cell_size, scaling,
                                           int(wproj.max_wpconv_support), float(wproj.kernel_trunc_perc), cur)
            res.plane_supports.append(cur)
            res.plane_w.append(float(w_avg[p]))
            accumulate(2, empty, cache, cur, b, e)
    res.vis_grid = vg.view(np.complex128).reshape((image_rows, image_size), order="F")
    res.sampling_grid = (sg.view(np.complex128).reshape((image_rows, image_size), order="F") if generate_beam
                         else np.zeros((0, 0), dtype=np.complex128))
    return res


def convolve_to_grid_functor(kf, trunc, support, image_size, uv, vis, weights, kernel_exact, oversampling, shift_uv,
                             halfplane, generate_beam):
    """convolve_to_grid with an explicitly parameterised functor (the
    reference unit tests build e.g. TopHat(half_base_width) themselves)."""
    return convolve_to_grid(kf, support, image_size, uv, vis, weights, kernel_exact, oversampling, shift_uv, halfplane,
                            generate_beam, trunc=trunc)


make_kernel_array_functor = make_kernel_array


def populate_kernel_cache_functor(kf, trunc, support, oversampling):
    t = kernel_table_1d(kf, trunc, support, oversampling)
    cs = t.shape[0]
    return {(y, x): np.outer(t[y], t[x]) for y in range(cs) for x in range(cs)}


def c2r(grid, n, threads=1):
    """fft_fftw_c2r, fft.cpp:45-135: unnormalised backward 2-D c2r of a
    (n/2+1) x n column-major half-plane grid into an n x n column-major image."""
    X = np.asarray(grid).T  # axis 0 = columns (slow FFTW dim), axis 1 = half axis
    Y = scipy.fft.irfft2(X, s=(n, n), norm="forward", workers=threads)
    return np.asfortranarray(Y.T)


def normalise(img, padded, image_size, normalization_factor, gcf, grid_correction, threads=1, fast=False):
    out = np.empty(image_size * image_size)
    imgF = np.asfortranarray(img, dtype=np.float64)
    g = np.ascontiguousarray(gcf if gcf is not None else np.ones(padded), dtype=np.float64)
    lib(fast).orc_normalise(_d(imgF.reshape(-1, order="F")), ctypes.c_int64(padded), ctypes.c_int64(image_size),
                            ctypes.c_double(normalization_factor), _d(g), ctypes.c_int(int(grid_correction)), _d(out),
                            ctypes.c_int(threads))
    return out.reshape((image_size, image_size), order="F")


def image_visibilities(vis, weights, uvw, image_size, cell_size, padding_factor=1.0, kernel_func=PSWF,
                       kernel_support=3, kernel_exact=True, oversampling=8, generate_beam=False,
                       gridding_correction=True, analytic_gcf=False, num_wplanes=0, wplanes_median=False,
                       max_wpconv_support=0, undersampling_opt=1, kernel_trunc_perc=0.0, hankel_opt=False,
                       hankel_proj_slice=False, interp_type=LINEAR, aproj_numtimesteps=0, obs_dec=0.0, obs_ra=0.0,
                       aproj_opt=False, aproj_mask_perc=0.0, lha=None, pbeam_coefs=None, threads=1, fast=False,
                       return_grid=False):
    """stp_python.image_visibilities_wrapper (stp-python/stp_python.cpp:17-140)
    -> ImageVisibilities (stp/imager/imager.cpp:12-68) -> image_visibilities
    (stp/imager/imager.h:233-376).  Returns (image, beam)."""
    image_size = int(image_size)
    while image_size % 4:
        image_size += 1
    padded = int(float(image_size) * padding_factor)
    while padded % 4:
        padded += 1
    uvw = np.asarray(uvw, dtype=np.float64).reshape(-1, 3)
    inv = arc_sec_to_rad(cell_size) * float(padded)
    uv = np.empty((uvw.shape[0], 2))
    uv[:, 0] = uvw[:, 0] * inv
    uv[:, 1] = uvw[:, 1] * inv
    wp = WProj(num_wplanes, max_wpconv_support, undersampling_opt, kernel_trunc_perc, wplanes_median, hankel_opt,
               hankel_proj_slice, interp_type)
    ap = AProj(int(aproj_numtimesteps), float(obs_dec), float(obs_ra), bool(aproj_opt), lha, pbeam_coefs)
    g = convolve_to_grid(kernel_func, kernel_support, padded, uv, vis, weights, kernel_exact, oversampling, True,
                         True, generate_beam, wp, uvw[:, 2], cell_size, analytic_gcf, threads, fast, aproj=ap)
    img = c2r(g.vis_grid, padded, threads)
    beam = c2r(g.sampling_grid, padded, threads) if generate_beam else None
    out_img = np.zeros((0, 0))
    out_beam = np.zeros((0, 0))
    if g.sample_grid_total > 0.0:
        nf = 1.0 / g.sample_grid_total
        gcf = img_dom_kernel(kernel_func, float(kernel_support), padded, analytic_gcf) if gridding_correction else None
        out_img = normalise(img, padded, image_size, nf, gcf, gridding_correction, threads, fast)
        if generate_beam:
            out_beam = normalise(beam, padded, image_size, nf, gcf, gridding_correction, threads, fast)
    if return_grid:
        return out_img, out_beam, g
    return out_img, out_beam


# ------------------------------------------------------------------ source finder

def mean_std(x):
    x = np.asfortranarray(x, dtype=np.float64).reshape(-1, order="F")
    m = ctypes.c_double()
    s = ctypes.c_double()
    lib().orc_mean_std(_d(x), ctypes.c_int64(x.size), ctypes.byref(m), ctypes.byref(s))
    return m.value, s.value


def median_exact(x):
    x = np.asfortranarray(x, dtype=np.float64).reshape(-1, order="F")
    return lib().orc_median_exact(_d(x), ctypes.c_int64(x.size))


def median_binapprox(x):
    x = np.asfortranarray(x, dtype=np.float64).reshape(-1, order="F")
    m, s, md = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    lib().orc_median_binapprox(_d(x), ctypes.c_int64(x.size), ctypes.byref(m), ctypes.byref(s), ctypes.byref(md))
    return m.value, s.value, md.value


def median_binmedian(x):
    x = np.asfortranarray(x, dtype=np.float64).reshape(-1, order="F")
    m, s, md = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    lib().orc_median_binmedian(_d(x), ctypes.c_int64(x.size), ctypes.byref(m), ctypes.byref(s), ctypes.byref(md))
    return m.value, s.value, md.value


def estimate_rms(x, num_sigma, iters, mean, sigma, median):
    x = np.asfortranarray(x, dtype=np.float64).reshape(-1, order="F")
    return lib().orc_estimate_rms(_d(x), ctypes.c_int64(x.size), ctypes.c_double(num_sigma), ctypes.c_int(iters),
                                  ctypes.c_double(mean), ctypes.c_double(sigma), ctypes.c_double(median))


def default_slice_cols(cols):
    """Column-slice width of the reference's TBB scan on an 8-thread host:
    static_partitioner over blocked_range(0, cols, max(cols/32, 2))."""
    return max(2, cols // 8)


def ccl(data, thr_pos, thr_neg, find_negative=True, conn4=False, slice_cols=0):
    data = np.asfortranarray(data, dtype=np.float64)
    rows, cols = data.shape
    if slice_cols <= 0:
        slice_cols = default_slice_cols(cols)
    L = np.zeros(rows * cols, dtype=np.int32)
    plen = cols * rows // 2
    Pp = np.zeros(plen, dtype=np.uint32)
    Pn = np.zeros(plen, dtype=np.uint32)
    npos, nneg = ctypes.c_uint32(), ctypes.c_uint32()
    lib().orc_ccl(_d(data.reshape(-1, order="F")), ctypes.c_int(rows), ctypes.c_int(cols), ctypes.c_double(thr_pos),
                  ctypes.c_double(thr_neg), ctypes.c_int(int(find_negative)), ctypes.c_int(int(conn4)),
                  ctypes.c_int(slice_cols), _i32(L), _u32(Pp), _u32(Pn), ctypes.byref(npos), ctypes.byref(nneg))
    return L, Pp, Pn, npos.value, nneg.value


@dataclass
class Gaussian2dParams:
    """fitting.h:90-150 (fields as bound by stp_python.cpp:224-235)."""
    amplitude: float = 0.0
    x_centre: float = 0.0
    y_centre: float = 0.0
    semimajor: float = 0.0
    semiminor: float = 0.0
    theta: float = 0.0

    def convert_to_constrained_parameters(self):
        """fitting.cpp:32-57."""
        half_pi = math.pi / 2.0
        self.semimajor = math.fabs(self.semimajor)
        self.semiminor = math.fabs(self.semiminor)
        if self.semimajor < self.semiminor:
            self.semimajor, self.semiminor = self.semiminor, self.semimajor
            self.theta += half_pi
        t = math.fmod(self.theta, math.pi)
        if t <= -half_pi:
            t += math.pi
        elif t > half_pi:
            t -= math.pi
        self.theta = t


def _csqrt(x):
    return math.sqrt(x) if x >= 0 else float("nan")


def _clog(x):
    if x > 0:
        return math.log(x)
    return float("-inf") if x == 0 else float("nan")


def moments_fit(sign, extremum_val, x_bar, y_bar, xx_bar, yy_bar, xy_bar, rms_est, analysis_n_sigma):
    """IslandParams::estimate_moments_fit, sourcefind.cpp:691-717."""
    w1 = (xx_bar + yy_bar) / 2.0
    w2 = _csqrt(((xx_bar - yy_bar) * (xx_bar - yy_bar) / 4) + xy_bar * xy_bar)
    tmaj = w1 + w2
    tmin = w1 - w2
    thr = analysis_n_sigma * rms_est
    ratio = sign * extremum_val / thr
    with np.errstate(all="ignore"):
        scale = 1.0 - _clog(ratio) / (ratio - 1.0) if ratio != 1.0 else float("nan")
        smaj = _csqrt(tmaj / scale) if scale != 0 else float("inf")
        smin = _csqrt(tmin / scale) if scale != 0 else float("inf")
        den = xx_bar - yy_bar
        arg = 2.0 * xy_bar / den if den != 0 else math.copysign(float("inf"), 2.0 * xy_bar) if xy_bar != 0 else float("nan")
        theta = 0.5 * math.atan(arg) if not math.isnan(arg) else float("nan")
    if theta * xy_bar < 0.0:
        theta += math.pi / 2.0
    g = Gaussian2dParams(extremum_val, x_bar, y_bar, smaj, smin, theta)
    g.convert_to_constrained_parameters()
    return g


@dataclass
class SourceFindResult:
    islands: list
    label_map: np.ndarray
    bg_level: float
    rms_est: float
    n_pos: int
    n_neg: int
    label_valid_pos: np.ndarray
    label_valid_neg: np.ndarray


def source_find(image, detection_n_sigma, analysis_n_sigma, rms_est=0.0, find_negative_sources=True,
                sigma_clip_iters=5, median_method=BINAPPROX, gaussian_fitting=False, ccl_4connectivity=False,
                generate_labelmap=True, source_min_area=5, slice_cols=0):
    """SourceFindImage ctor, sourcefind.cpp:156-292 (+ the python tuple layout,
    stp_python.cpp:142-179).  Islands: (sign, extremum_val, x_idx, y_idx,
    num_samples, moments_fit, leastsq_fit, ceres_report)."""
    data = np.asfortranarray(image, dtype=np.float64)
    rows, cols = data.shape
    mean = sigma = None
    if median_method == ZEROMEDIAN:
        median = 0.0
    elif median_method == BINAPPROX:
        mean, sigma, median = median_binapprox(data)
    elif median_method == BINMEDIAN:
        mean, sigma, median = median_binmedian(data)
    elif median_method == NTHELEMENT:
        median = median_exact(data)
    else:
        raise ValueError("median_method")
    bg = median
    if abs(rms_est) > 0.0:
        rms = rms_est
    else:
        if mean is None:
            mean, sigma = mean_std(data)
        rms = estimate_rms(data, 3.0, sigma_clip_iters, mean, sigma, median)
    a_pos = bg + analysis_n_sigma * rms
    a_neg = bg - analysis_n_sigma * rms
    d_pos = bg + detection_n_sigma * rms
    d_neg = bg - detection_n_sigma * rms
    L, Pp, Pn, npos, nneg = ccl(data, a_pos, a_neg, find_negative_sources, ccl_4connectivity, slice_cols)
    ev_p = np.empty(npos)
    ei_p = np.empty(npos, dtype=np.int64)
    mo_p = np.empty(5 * npos)
    ns_p = np.empty(npos, dtype=np.int32)
    va_p = np.empty(npos, dtype=np.int32)
    ev_n = np.empty(nneg)
    ei_n = np.empty(nneg, dtype=np.int64)
    mo_n = np.empty(5 * nneg)
    ns_n = np.empty(nneg, dtype=np.int32)
    va_n = np.empty(nneg, dtype=np.int32)
    dataflat = data.reshape(-1, order="F")
    lib().orc_label_analysis(_d(dataflat), ctypes.c_int(rows), ctypes.c_int(cols), _i32(L), _u32(Pp), _u32(Pn),
                             ctypes.c_uint32(npos), ctypes.c_uint32(nneg), ctypes.c_double(d_pos),
                             ctypes.c_double(d_neg), ctypes.c_int(int(generate_labelmap)), _d(ev_p), _i64(ei_p),
                             _d(mo_p), _i32(ns_p), _i32(va_p), _d(ev_n), _i64(ei_n), _d(mo_n), _i32(ns_n), _i32(va_n))
    islands = []
    vs, hs = rows // 2, cols // 2
    for sign, n_l, ev, ei, mo, ns, va in ((1, npos, ev_p, ei_p, mo_p, ns_p, va_p), (-1, nneg, ev_n, ei_n, mo_n, ns_n, va_n)):
        for i in range(n_l):
            if not va[i]:
                continue
            r, c = int(ei[i] % rows), int(ei[i] // rows)
            y = r + vs if r < vs else r - vs
            x = c + hs if c < hs else c - hs
            if ns[i] >= source_min_area:
                m = mo[5 * i:5 * i + 5]
                g = moments_fit(sign, float(ev[i]), m[0], m[1], m[2], m[3], m[4], rms, analysis_n_sigma)
                fit = Gaussian2dParams()
                if gaussian_fitting:
                    fit = leastsq_fit_gaussian_2d(dataflat, L, rows, cols, sign * (i + 1), int(ns[i]), float(ev[i]), g)
                islands.append((sign, float(ev[i]), x, y, int(ns[i]), g, fit, ""))
    return SourceFindResult(islands, L.reshape((rows, cols), order="F"), bg, rms, npos, nneg, va_p, va_n)


def visibilities_for_point_source(uvw, l, m, flux):
    """visibility.cpp:15-28: flux * n * exp(cx(0, -2 pi) * (dist_uvw * -(l, m, n - 1)))."""
    src_n = math.sqrt(1 - l * l - m * m)
    off = -np.array([l, m, src_n - 1.0])
    uvw = np.asarray(uvw, dtype=np.float64).reshape(-1, 3)
    dot = (uvw[:, 0] * off[0] + uvw[:, 1] * off[1]) + uvw[:, 2] * off[2]
    theta = (-2.0 * math.pi) * dot
    return flux * src_n * (np.cos(theta) + 1j * np.sin(theta))


def generate_visibilities_from_local_skymodel(skymodel, uvw):
    """visibility.cpp:30-40: model visibilities summed over the sky-model rows in order."""
    uvw = np.asarray(uvw, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(uvw.shape[0], dtype=np.complex128)
    for l, m, f in np.asarray(skymodel, dtype=np.float64).reshape(-1, 3):
        out += visibilities_for_point_source(uvw, l, m, f)
    return out


FIT_MAX_ITER = 100


def _gauss_terms(p):
    """a, b, c of GaussianResidual (fitting.h:183-210) and their derivatives in (sx, sy, theta)."""
    ct, st, s2t, c2t = math.cos(p[5]), math.sin(p[5]), math.sin(2.0 * p[5]), math.cos(2.0 * p[5])
    ct2, st2 = ct * ct, st * st
    ix2, iy2 = 1.0 / (p[3] * p[3]), 1.0 / (p[4] * p[4])
    ix3, iy3 = ix2 / p[3], iy2 / p[4]
    return dict(a=0.5 * (ct2 * ix2 + st2 * iy2), b=0.5 * (s2t * ix2 - s2t * iy2), c=0.5 * (st2 * ix2 + ct2 * iy2),
                dsx=(-ct2 * ix3, -s2t * ix3, -st2 * ix3), dsy=(-st2 * iy3, s2t * iy3, -ct2 * iy3),
                dt=(0.5 * s2t * (iy2 - ix2), c2t * (ix2 - iy2), 0.5 * s2t * (ix2 - iy2)))


def gauss_fit_lm(vals, xs, ys, p0):
    """Least-squares 2-D Gaussian (the residual of fitting.h:183-210) by Levenberg-Marquardt with analytic
    derivatives; the algorithm the GPU runs (the reference uses Ceres, sourcefind.cpp:719-866).
    Returns (params, iterations)."""
    p = np.array(p0, dtype=np.float64)

    def evaluate(q, normal):
        g = _gauss_terms(q)
        dx, dy = xs - q[1], ys - q[2]
        ex = np.exp(-(g["a"] * dx * dx + g["b"] * dx * dy + g["c"] * dy * dy))
        r = q[0] * ex - vals
        cost = float(np.dot(r, r))
        if not normal:
            return cost, None, None
        ae = q[0] * ex
        J = np.empty((vals.size, 6))
        J[:, 0] = ex
        J[:, 1] = ae * (2.0 * g["a"] * dx + g["b"] * dy)
        J[:, 2] = ae * (g["b"] * dx + 2.0 * g["c"] * dy)
        for k, key in ((3, "dsx"), (4, "dsy"), (5, "dt")):
            da, db, dc = g[key]
            J[:, k] = -ae * (da * dx * dx + db * dx * dy + dc * dy * dy)
        return cost, J.T @ J, J.T @ r

    cost, JtJ, Jtr = evaluate(p, True)
    lam = 1e-3
    it = 0
    while it < FIT_MAX_ITER:
        it += 1
        M = JtJ.copy()
        dg = np.diag(JtJ)
        M[np.diag_indices(6)] += lam * np.maximum(dg, 1e-12 * dg.max() + 1e-300)
        ok = True
        try:
            Lc = np.linalg.cholesky(M)
            d = np.linalg.solve(Lc.T, np.linalg.solve(Lc, -Jtr))
            q = p + d
            ok = q[3] != 0.0 and q[4] != 0.0
        except np.linalg.LinAlgError:
            ok = False
        if ok:
            cnew, _, _ = evaluate(q, False)
            ok = cnew == cnew and cnew < cost
        if ok:
            step = float(np.max(np.abs(d) / (np.abs(p) + 1e-10)))
            small = (cost - cnew) <= 1e-12 * cost or step <= 1e-10
            p = q
            cost, JtJ, Jtr = evaluate(p, True)
            lam = max(lam * 0.1, 1e-15)
            if small:
                break
        else:
            lam *= 10.0
            if lam > 1e16:
                break
    return p, it


def leastsq_fit_gaussian_2d(dataflat, L, rows, cols, label, num_samples, extremum_val, moments):
    """IslandParams::leastsq_fit_gaussian_2d (sourcefind.cpp:719-866) with the LM minimiser above: pixels of the
    island in display coordinates, start at the moments fit (unset widths 1.0), result constrained
    (fitting.cpp:32-57); islands of one or two pixels keep (extremum, 0, ...)."""
    if num_samples < 3:
        return Gaussian2dParams(extremum_val, 0.0, 0.0, 0.0, 0.0, 0.0)
    m = np.nonzero(L == label)[0]
    r, c = m % rows, m // rows
    vs, hs = rows // 2, cols // 2
    ys = np.where(r < vs, r + vs, r - vs).astype(np.float64)
    xs = np.where(c < hs, c + hs, c - hs).astype(np.float64)
    g = moments
    p0 = [g.amplitude, g.x_centre, g.y_centre, g.semimajor if g.semimajor > 0 else 1.0,
          g.semiminor if g.semiminor > 0 else 1.0, g.theta]
    p, _ = gauss_fit_lm(dataflat[m], xs, ys, p0)
    out = Gaussian2dParams(*[float(v) for v in p])
    out.convert_to_constrained_parameters()
    return out
