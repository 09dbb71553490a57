"""The oracle's Hankel-transform W-kernels (hankel_opt): the discrete Hankel
transform is exact for profiles that are constant on its annuli, the spline
follows the natural cubic / linear interpolant, and the projection-slice
variant reproduces the central row of the 2-D FFT W-kernel (projection-slice
theorem)."""
import math

import numpy as np
import scipy.fft
from scipy.interpolate import CubicSpline
from scipy.special import j1

from oracle import stp_oracle as orc


def test_besselj1_approximation():
    """The reference's rational J1 (aw_projection.cpp:490-508) stays within its
    published accuracy of the exact Bessel function on both branches, and is
    continuous enough at the branch point x = 8."""
    x = np.concatenate([np.linspace(0.0, 8.0, 2001)[:-1], np.linspace(8.0, 400.0, 4001)])
    assert np.max(np.abs(orc.besselj1(x) - j1(x))) < 2e-8
    assert abs(orc.besselj1(np.array([8.0 - 1e-12]))[0] - orc.besselj1(np.array([8.0]))[0]) < 2e-8
    assert orc.besselj1(np.array([0.0]))[0] == 0.0


def test_dht_is_exact_for_a_disc():
    n = 64
    D = orc.dht_matrix(n, j1=j1)
    m = 10
    f = np.zeros(n)
    f[:m + 1] = 1.0  # 1 on the annuli j <= m, i.e. a disc of radius m + 1/2
    Y = D.T @ f
    R = m + 0.5
    k = np.pi * np.arange(1, n) / n
    assert math.isclose(Y[0], math.pi * R * R, rel_tol=1e-13)
    assert np.allclose(Y[1:], 2 * np.pi * R * j1(k * R) / k, rtol=1e-12, atol=1e-12)


def test_spline_matches_natural_cubic_and_linear():
    rng = np.random.default_rng(7)
    y = rng.normal(size=40)
    x = np.arange(40.0)
    q = np.sort(rng.uniform(0, 39, 200))
    cs = CubicSpline(x, y, bc_type="natural")
    for cubic, ref in ((True, cs(q)), (False, np.interp(q, x, y))):
        a, b, c = orc.spline_coefficients(y, cubic)
        k = np.minimum(q.astype(int), 39)
        t = q - k
        got = ((a[k] * t + b[k]) * t + c[k]) * t + y[k]
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)
    # beyond the last node the end segment extrapolates linearly with the end slope
    a, b, c = orc.spline_coefficients(y, True)
    assert a[-1] == 0.0 and abs(b[-1]) < 1e-15
    assert math.isclose(c[-1], cs(39.0, 1), rel_tol=1e-10, abs_tol=1e-12)


def _planes(w, proj_slice, interp, trunc=0.0):
    workarea, os_, cell, max_sup = 64, 8, 2.0, 8
    aa = orc.img_dom_kernel(orc.GaussianSinc, 3.0, workarea, False)
    scaling = 512.0 / workarea
    return orc.hankel_wkernel_plane(w, aa, workarea, os_, cell, scaling, max_sup, trunc, max_sup, proj_slice, interp)


def test_projection_slice_reproduces_the_fft_kernel_axis():
    w = 300.0
    workarea, os_, cell, max_sup = 64, 8, 2.0, 8
    aa = orc.img_dom_kernel(orc.GaussianSinc, 3.0, workarea, False)
    scaling = 512.0 / workarea
    S_f, cache_f = orc.wkernel_plane(w, aa, workarea, os_, cell, scaling, max_sup, 0.0, max_sup)
    S_h, cache_h = orc.hankel_wkernel_plane(w, aa, workarea, os_, cell, scaling, max_sup, 0.0, max_sup, True,
                                            orc.CUBIC)
    assert S_f == S_h == max_sup
    K = 2 * max_sup + 1
    cs = os_ + 1
    f = cache_f.view(np.complex128).reshape(cs * cs, K * K)
    h = cache_h.view(np.complex128).reshape(cs * cs, K * K)
    # the sub-kernel of the centred offset (os/2, os/2), column-major K x K: its centre row and column lie on
    # the uv axes, where the Hankel kernel samples the 1-D transform at integer radii (no interpolation);
    # the two caches are normalised by different sums, so compare shapes
    c = (os_ // 2) * cs + os_ // 2
    F = f[c].reshape(K, K, order="F")
    H = h[c].reshape(K, K, order="F")
    row_f, row_h = F[max_sup, :], H[max_sup, :]
    scale = row_f[max_sup] / row_h[max_sup]
    assert np.allclose(row_h * scale, row_f, rtol=0, atol=1e-12 * abs(row_f[max_sup]))


def test_hankel_kernels_match_fft_kernel_for_a_radial_taper():
    # with a Gaussian taper aa(x) aa(y) = aa(r) aa(0) the image-domain kernel is radially symmetric, so both
    # Hankel variants must reproduce the 2-D FFT kernel: the projection slice up to the cubic interpolation
    # between radii, the discrete Hankel transform up to its annulus discretisation
    workarea, os_, cell, max_sup = 64, 8, 2.0, 8
    x = np.arange(workarea) - workarea // 2
    for sigma in (4.0, 8.0):
        aa = np.exp(-(x / sigma) ** 2)
        for w in (0.0, 300.0):
            _, cf = orc.wkernel_plane(w, aa, workarea, os_, cell, 512.0 / workarea, max_sup, 0.0, max_sup)
            f = cf.view(np.complex128)
            for proj_slice, interp, tol in ((True, orc.CUBIC, 1e-4), (False, orc.CUBIC, 2e-2),
                                            (False, orc.LINEAR, 2e-2)):
                _, ch = orc.hankel_wkernel_plane(w, aa, workarea, os_, cell, 512.0 / workarea, max_sup, 0.0,
                                                 max_sup, proj_slice, interp)
                h = ch.view(np.complex128)
                assert np.max(np.abs(f - h)) < tol * np.max(np.abs(f)), (sigma, w, proj_slice, interp)


def test_truncation_shrinks_support_with_w():
    s_small, _ = _planes(0.0, False, orc.LINEAR, trunc=1.0)
    s_large, _ = _planes(1500.0, False, orc.LINEAR, trunc=1.0)
    assert 1 <= s_small <= s_large <= 8


def test_fft_kernel_slice_identity_directly():
    # projection-slice theorem on the oracle's own image-domain kernel: the 1-D FFT of the projection equals
    # row 0 of the 2-D FFT
    w = 500.0
    workarea, os_, cell = 32, 4, 2.0
    arr = workarea * os_
    aa = orc.img_dom_kernel(orc.PSWF, 3.0, workarea, False)
    comb = np.empty(2 * arr * arr)
    L = orc.lib()
    L.orc_wkernel_image_domain(orc.ctypes.c_double(w), orc._d(np.ascontiguousarray(aa)), orc.ctypes.c_int(workarea),
                               orc.ctypes.c_int(os_), orc.ctypes.c_double(orc.arc_sec_to_rad(cell)),
                               orc.ctypes.c_double(256.0 / workarea), orc._d(comb))
    M = comb.view(np.complex128).reshape((arr, arr), order="F")
    conv = scipy.fft.fft2(M)
    proj = M.sum(axis=1)
    assert np.allclose(np.fft.fft(proj), conv[:, 0], rtol=0, atol=1e-12 * np.max(np.abs(conv)))
