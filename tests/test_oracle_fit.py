"""The least-squares Gaussian fit of the oracle (the Levenberg-Marquardt
minimiser that stands in for the reference's Ceres call) recovers known
parameters of a noiseless island and lowers the cost of a noisy one."""
import math

import numpy as np

from oracle import stp_oracle as orc


def _island(p, half=8):
    g = orc._gauss_terms(p)
    ys, xs = np.mgrid[int(p[2]) - half:int(p[2]) + half + 1, int(p[1]) - half:int(p[1]) + half + 1]
    xs = xs.ravel().astype(float)
    ys = ys.ravel().astype(float)
    dx, dy = xs - p[1], ys - p[2]
    vals = p[0] * np.exp(-(g["a"] * dx * dx + g["b"] * dx * dy + g["c"] * dy * dy))
    keep = vals > 0.05 * p[0]
    return vals[keep], xs[keep], ys[keep]


def test_recovers_noiseless_gaussian():
    truth = np.array([5.0, 100.3, 200.7, 3.0, 1.5, 0.4])
    vals, xs, ys = _island(truth)
    p, it = orc.gauss_fit_lm(vals, xs, ys, [4.0, 100.0, 201.0, 2.5, 1.8, 0.2])
    assert it < orc.FIT_MAX_ITER
    assert np.allclose(p, truth, rtol=1e-7, atol=1e-7)


def test_noisy_island_lowers_cost():
    rng = np.random.default_rng(3)
    truth = np.array([8.0, 50.2, 60.9, 2.2, 2.0, -0.7])
    vals, xs, ys = _island(truth)
    vals = vals + rng.normal(0, 0.05, vals.size)
    p0 = np.array([7.0, 50.0, 61.0, 2.0, 2.0, 0.0])

    def cost(p):
        g = orc._gauss_terms(p)
        dx, dy = xs - p[1], ys - p[2]
        r = p[0] * np.exp(-(g["a"] * dx * dx + g["b"] * dx * dy + g["c"] * dy * dy)) - vals
        return float(r @ r)

    p, _ = orc.gauss_fit_lm(vals, xs, ys, p0)
    assert cost(p) < cost(p0)
    assert abs(p[0] - truth[0]) < 0.1 and math.hypot(p[1] - truth[1], p[2] - truth[2]) < 0.05
