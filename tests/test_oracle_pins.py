"""Pin the CPU oracle to the reference's own inline known answers.

Every case below comes from tests/golden/reference_pins.json, which
tests/golden/make_reference_pins.py extracts from the reference gtest sources
(src/test/...).  Tolerance: the reference's fptolerance for double builds,
1e-10 (src/stp/types.h:26).
"""
import numpy as np
import pytest

from oracle import stp_oracle as orc

TOL = 1e-10
KF = {"TopHat": orc.TopHat, "Triangle": orc.Triangle, "Sinc": orc.Sinc, "Gaussian": orc.Gaussian,
      "GaussianSinc": orc.GaussianSinc, "PSWF": orc.PSWF}


def _grid(case, kernel_exact=None):
    uv = np.array(case["uv"], dtype=np.float64)
    vis = np.array([complex(a, b) for a, b in case["vis"]])
    w = np.array(case["weights"], dtype=np.float64)
    ke = case["kernel_exact"] if kernel_exact is None else kernel_exact
    return orc.convolve_to_grid(KF[case["kernel"]], case["support"], case["image_size"], uv, vis, w, ke,
                                case["oversampling"], case["shift_uv"], case["halfplane"], True, w=None)


@pytest.mark.parametrize("name", ["SmallPillbox", "MultiPixelPillbox", "MultipleComplexVis", "NearbyComplexVis",
                                  "SinglePixelOverlapPillbox"])
def test_gridder_pins(pins, name, monkeypatch):
    case = next(c for c in pins["gridder"] if c["name"] == name)
    # TopHat's half_base_width is the functor argument in these tests, not the
    # support; the oracle's functor takes it as `trunc`.
    res = _grid_hbw(case)
    exp = np.array(case["expect_vis_grid_real"])
    assert np.max(np.abs(res.vis_grid.real - exp)) < TOL
    if case["expect_sampling_real"] is not None:
        assert np.max(np.abs(res.sampling_grid.real - np.array(case["expect_sampling_real"]))) < TOL


def _grid_hbw(case, kernel_exact=None, halfplane=None, shift=None):
    """convolve_to_grid with the functor built from half_base_width."""
    uv = np.array(case["uv"], dtype=np.float64)
    vis = np.array([complex(a, b) for a, b in case["vis"]])
    w = np.array(case["weights"], dtype=np.float64)
    ke = case["kernel_exact"] if kernel_exact is None else kernel_exact
    return orc.convolve_to_grid_functor(KF[case["kernel"]], case["hbw"], case["support"], case["image_size"], uv, vis,
                                        w, ke, case["oversampling"],
                                        case["shift_uv"] if shift is None else shift,
                                        case["halfplane"] if halfplane is None else halfplane, True)


def test_gridder_halfplane_shifted(pins):
    case = next(c for c in pins["gridder"] if c["name"] == "HalfPlaneShiftedGridding")
    over = _grid_hbw(case, kernel_exact=False)
    exact = _grid_hbw(case, kernel_exact=True)
    roll = case["roll_cols"]
    beam_over = np.roll(over.vis_grid, roll, axis=1)
    beam_exact = np.roll(exact.vis_grid, roll, axis=1)
    exp = np.array(case["expect_vis_grid_real"])
    # the reference asserts sums; the element-wise match is stronger and holds
    assert abs(np.sum(beam_over.real - beam_exact.real)) < TOL
    assert np.max(np.abs(beam_over.real - exp)) < TOL
    assert np.sum(np.roll(over.sampling_grid, roll, axis=1).real) - 2 * 2 < TOL


def test_gridder_natural_weighting(pins):
    case = next(c for c in pins["gridder"] if c["name"] == "SampleWeightingNatural")
    res = _grid_hbw(case)
    s = res.sampling_grid
    exp = np.array(case["expect_sampling_normalised"])
    assert np.max(np.abs(s / s.sum() - exp)) < TOL
    assert np.max(np.abs(res.vis_grid / s.sum() - exp * case["natural_weighted_sum"])) < TOL


def test_gridder_zero_weighting():
    """gridder_test_SampleWeighting.cpp zero_weighting: zero weights give zero grids."""
    uv = np.array([[-2.0, 0.0], [-2.0, 0.0]])
    vis = np.full(2, 42.123 + 0j)
    w = np.zeros(2)
    for ke, os_ in ((True, 1), (False, 5)):
        r = orc.convolve_to_grid_functor(orc.TopHat, 0.5, 1, 8, uv, vis, w, ke, os_, False, False, True)
        assert np.max(np.abs(r.vis_grid)) < TOL


def test_gridder_bounds_checking():
    """gridder_test_BoundsChecking.cpp: an out-of-bounds kernel centre is dropped."""
    bad = orc.convolve_to_grid_functor(orc.TopHat, 1.5, 2, 8, np.array([[-3.0, 0.0]]), np.ones(1, complex), np.ones(1),
                                       True, 1, True, True, True)
    assert bad.vis_grid.real.sum() == 0 and bad.sampling_grid.real.sum() == 0
    good = orc.convolve_to_grid_functor(orc.TopHat, 1.5, 2, 8, np.array([[0.0, 0.0]]), np.ones(1, complex), np.ones(1),
                                        True, 1, True, True, True)
    mixed = orc.convolve_to_grid_functor(orc.TopHat, 1.5, 2, 8, np.array([[-3.0, 0.0], [0.0, 0.0]]),
                                         np.ones(2, complex), np.ones(2), True, 1, True, True, True)
    assert np.array_equal(good.vis_grid, mixed.vis_grid)
    assert np.array_equal(good.sampling_grid, mixed.sampling_grid)


def test_gridder_triangle_uv_location():
    """gridder_test_Triangle.cpp: exact gridding places the normalised kernel at the uv location."""
    off = (0.1, -0.15)
    uv = np.array([[1.0 + off[0], 0.0 + off[1]]])
    r = orc.convolve_to_grid_functor(orc.Triangle, 2.0, 2, 8, uv, np.ones(1, complex), np.ones(1), True, 1, False,
                                     False, True)
    k = orc.make_kernel_array_functor(orc.Triangle, 2.0, 2, off, 1, False, True)
    sub = r.vis_grid.real[8 // 2 - 2:8 // 2 + 3, 8 // 2 + 1 - 2:8 // 2 + 1 + 3]
    assert np.max(np.abs(sub - k / k.sum())) < TOL


def test_gridder_oversampled_sum():
    """gridder_test_OversampledGridding.cpp: total sampling weight equals the visibility count."""
    uv = np.array([[1.0, 0.0], [1.3, 0.0], [0.01, -1.32]])
    r = orc.convolve_to_grid_functor(orc.Triangle, 2.0, 2, 8, uv, np.ones(3, complex), np.ones(3), False, 9, False,
                                     False, True)
    assert r.sampling_grid.real.sum() - 3 < TOL


def test_oversampled_index_pins(pins):
    p = pins["oversampled_indices"]
    io = np.array(p["io_pairs"])
    assert np.array_equal(orc.oversampled_indices(io[:, 0], p["oversampling"]), io[:, 1].astype(np.int32))
    assert np.array_equal(orc.oversampled_indices(-io[:, 0], p["oversampling"]), -io[:, 1].astype(np.int32))
    e = p["edge_case"]
    assert orc.oversampled_indices(np.array([e["offset"]]), e["oversampling"])[0] == e["expected"]
    assert np.array_equal(orc.oversampled_indices(np.array([0.3, 0.3]), 5), np.array([2, 2], np.int32))


def test_make_kernel_array_pins(pins):
    for c in pins["make_kernel_array"]:
        k = orc.make_kernel_array_functor(KF[c["kernel"]], c["hbw"], c["support"], c["offset"], c["oversampling"],
                                          False, False)
        assert np.max(np.abs(k - np.array(c["expected"]))) < TOL, c


def test_kernel_caching():
    """gridder_test_KernelCaching.cpp: the cache entry picked by the
    oversampled index equals the exact kernel at the aligned offset."""
    os_ = 5
    cache = orc.populate_kernel_cache_functor(orc.Triangle, 2.5, 3, os_)
    for step in (-0.4, 0.2, 0.0, 0.2, 0.4):
        exact = orc.make_kernel_array_functor(orc.Triangle, 2.5, 3, (step, 0.0), 1, False, True)
        idx = orc.oversampled_indices(np.array([step, 0.0]), os_)
        cached = cache[(idx[1] + os_ // 2, idx[0] + os_ // 2)]
        assert np.max(np.abs(exact - cached)) < TOL
        for sub in np.linspace(-0.099999, 0.099999, 15):
            if abs(sub) > 0:
                j = orc.oversampled_indices(np.array([step + sub, 0.0]), os_)
                assert np.array_equal(j, idx)


def test_conv_pins(pins):
    for c in pins["conv"]:
        if c["kernel"] == "GaussianSinc":
            out = orc.kernel_eval(orc.GaussianSinc, c["trunc"], np.array(c["input"]))
        else:
            out = orc.kernel_eval(KF[c["kernel"]], c["trunc"], np.array(c["input"]))
        assert np.max(np.abs(out - np.array(c["output"]))) < TOL, c["kernel"]


@pytest.mark.parametrize("idx", range(12))
def test_labeling_pins(pins, idx):
    """sourcefind_test_Labeling.cpp: exact label maps, positive and inverted."""
    c = pins["labeling"][idx]
    img = np.array(c["img"], dtype=np.float64)
    exp = np.array(c["expected_map"], dtype=np.int32)
    for sgn in (1, -1):
        data = np.fft.fftshift(sgn * img)  # the test feeds the shifted image
        r = orc.source_find(data, c["detection_n_sigma"], c["analysis_n_sigma"], c["rms_est"], True, 5, orc.ZEROMEDIAN,
                            False, c["conn4"], c["generate_labelmap"], c["source_min_area"])
        got = np.fft.fftshift(r.label_map)
        assert len(r.islands) == c["expected_total_islands"], (c["name"], sgn)
        assert np.array_equal(got, sgn * exp), (c["name"], sgn, got)


def test_labeling_slice_dependence(pins):
    """8CCL_ImageCornerObjs holds only when column 4 starts a TBB slice: one
    slice (a 1-thread run) leaves the two centre pixels unjoined."""
    c = next(x for x in pins["labeling"] if x["name"] == "8CCL_ImageCornerObjs")
    data = np.fft.fftshift(np.array(c["img"], dtype=np.float64))
    one = orc.source_find(data, 4, 3, 1.0, True, 5, orc.ZEROMEDIAN, False, False, False, 1, slice_cols=8)
    two = orc.source_find(data, 4, 3, 1.0, True, 5, orc.ZEROMEDIAN, False, False, False, 1, slice_cols=2)
    assert len(one.islands) == c["expected_total_islands"] + 1
    assert len(two.islands) == c["expected_total_islands"]


def _pattern(p):
    if "data" in p:
        return np.array(p["data"], dtype=np.float64)
    d = np.full((20, 20), 100.0)
    d[:, 0:10] = -100.0
    if p["fill"] == "halves_extremes":
        d[0, 19] = 200.0
        d[19, 0] = -200.0
    return d


def test_median_patterns(pins):
    """matrixmath_test_median_funcs.cpp: binmedian == exact median (1e-12),
    binapprox within sigma/800-style tolerance."""
    for p in pins["median_patterns"]:
        d = _pattern(p)
        ref = float(np.median(d))
        assert abs(orc.median_binmedian(d)[2] - ref) < 1e-12, p["name"]
        assert abs(orc.median_exact(d) - ref) < 1e-12, p["name"]
        if "fill" in p:
            assert abs(orc.median_binapprox(d)[2] - ref) < 100.0 / 800.0, p["name"]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_median_noise(seed):
    """matrixmath_test_median_funcs.cpp noise cases, re-expressed with numpy's
    RNG (Armadillo's generator is not available)."""
    rng = np.random.default_rng(seed)
    for sigma, mean in ((1.0, 0.0), (0.5, 0.0), (1e-4, 0.0), (1e10, 0.0), (1.0, -25.0)):
        d = rng.normal(mean, sigma, size=(128, 128))
        ref = float(np.median(d))
        assert abs(orc.median_binmedian(d)[2] - ref) <= 1e-12 * max(1.0, abs(ref))
        assert abs(orc.median_exact(d) - ref) <= 1e-12 * max(1.0, abs(ref))
        assert abs(orc.median_binapprox(d)[2] - ref) < sigma / 800.0 + 1e-12 * abs(mean)


def test_mean_std_and_rms():
    """sourcefind_test_RmsEstimation.cpp: the clipped RMS of Gaussian noise is
    within 5% of the true sigma; matrixmath stat funcs: mean/std match numpy."""
    rng = np.random.default_rng(7)
    d = rng.normal(0.0, 1.0, size=(256, 256))
    m, s = orc.mean_std(d)
    assert abs(m - d.mean()) < 1e-12 and abs(s - d.std()) < 1e-12
    mm, ss, med = orc.median_binapprox(d)
    rms = orc.estimate_rms(d, 3.0, 5, mm, ss, med)
    assert abs(rms - 1.0) < 0.05
