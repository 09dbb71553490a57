"""The oracle's A-projection pieces: spherical-harmonic magnitudes against
scipy, the time-step assignment, the kernel rotation, and the whole
A-projected imager reducing to W-projection for a constant beam at zero
parallactic angle."""
import math

import numpy as np
from scipy.special import sph_harm_y

from fastimaging_b200.synthetic import make_snapshot
from oracle import stp_oracle as orc


def test_sh_magnitudes_match_scipy():
    rng = np.random.default_rng(11)
    theta = rng.uniform(0, math.pi, 50)
    phi = rng.uniform(-math.pi, math.pi, 50)
    for l in range(0, 7):
        for m in range(-l, l + 1):
            y = sph_harm_y(l, abs(m), theta, phi)
            if m > 0:
                ref = math.sqrt(2) * np.abs(y.real)
            elif m < 0:
                ref = math.sqrt(2) * np.abs(y.imag)
            else:
                ref = np.abs(y.real)
            assert np.allclose(orc.sh_abs(l, m, phi, theta), ref, rtol=1e-11, atol=1e-14), (l, m)


def test_time_steps_and_means():
    lha = np.arange(10.0)
    good = np.ones(10, dtype=np.int32)
    good[3] = 0
    means, ts = orc.average_lha_planes(lha, good, 2)
    # boundaries linspace(-2.25, 11.25, 3) = (-2.25, 4.5, 11.25)
    assert list(ts[[0, 1, 2, 4, 5, 9]]) == [0, 0, 0, 0, 1, 1]
    assert math.isclose(means[0], (0 + 1 + 2 + 4) / 4) and math.isclose(means[1], 7.0)


def test_parangle_zero_at_transit():
    assert orc.parangle(0.0, math.radians(-30.0), math.radians(30.0)) == 0.0


def test_rotation_quarter_turn_and_identity():
    rng = np.random.default_rng(3)
    n = 16
    m = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    assert np.array_equal(orc.rotate_matrix_cx(m, 0.0, 0.0), m)
    r = orc.rotate_matrix_cx(m, math.pi / 2, 0.0)
    j, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    assert np.allclose(r, m[i, n - 1 - j], atol=1e-12)


def test_constant_beam_at_transit_equals_wprojection():
    s = make_snapshot(51, 3000, 128, 2.0, n_src=3, w_range=(-800.0, 800.0))
    kw = dict(kernel_func=orc.GaussianSinc, kernel_support=3, kernel_exact=False, oversampling=4,
              num_wplanes=3, max_wpconv_support=6, kernel_trunc_perc=1.0)
    ref, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 128, s.cell_size, **kw)
    lha = np.zeros(s.vis.size)
    for opt in (False, True):
        img, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 128, s.cell_size, aproj_numtimesteps=2,
                                        obs_dec=-30.0, obs_ra=30.0, aproj_opt=opt, lha=lha, pbeam_coefs=[2.5],
                                        **kw)
        assert np.max(np.abs(img - ref)) < 1e-12 * np.max(np.abs(ref)), opt
