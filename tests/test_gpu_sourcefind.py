"""GPU parity of the source finder through the C ABI: labels bit-exact to the
oracle (and to the reference's own expected label maps), statistics within
1e-10 relative."""
import numpy as np
import pytest

from fastimaging_b200 import capi
from fastimaging_b200.synthetic import make_snapshot
from oracle import stp_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("idx", range(12))
def test_labeling_reference_maps(ctx, pins, idx):
    c = pins["labeling"][idx]
    img = np.array(c["img"], dtype=np.float64)
    exp = np.array(c["expected_map"], dtype=np.int32)
    for sgn in (1, -1):
        data = np.fft.fftshift(sgn * img)
        isl, lab, info = ctx.source_find(data, c["detection_n_sigma"], c["analysis_n_sigma"], c["rms_est"], True, 5,
                                         capi.ZEROMEDIAN, False, c["conn4"], c["generate_labelmap"],
                                         c["source_min_area"])
        assert len(isl) == c["expected_total_islands"], (c["name"], sgn)
        assert np.array_equal(np.fft.fftshift(lab), sgn * exp), (c["name"], sgn)


def _compare(isl, ref, lab, rl, rtol=1e-9):
    assert np.array_equal(lab, rl)
    assert len(isl) == len(ref.islands)
    for a, b in zip(isl, ref.islands):
        sign, val, x, y, ns, mom, _, _ = b
        assert a.sign == sign and a.extremum_x_idx == x and a.extremum_y_idx == y and a.num_samples == ns
        assert a.extremum_val == val
        got = np.array(a.moments_fit[:])
        want = np.array([mom.amplitude, mom.x_centre, mom.y_centre, mom.semimajor, mom.semiminor, mom.theta])
        ok = np.isclose(got, want, rtol=rtol, atol=1e-9) | (np.isnan(got) & np.isnan(want))
        assert ok.all(), (got, want)


@pytest.mark.parametrize("conn4", [False, True])
@pytest.mark.parametrize("slice_cols", [0, 1, 64])
def test_labels_injected_thresholds(ctx, conn4, slice_cols):
    """Thresholds fixed (ZEROMEDIAN + given rms): labels must be bit-exact."""
    rng = np.random.default_rng(5)
    img = rng.normal(size=(256, 256))
    img[100:110, 30:38] += 8.0
    img[0:3, :] += 4.0  # structures across the shifted-topology seams
    img[:, 127:130] -= 5.0
    ref = orc.source_find(img, 4.0, 2.5, 1.0, True, 5, orc.ZEROMEDIAN, False, conn4, True, 3, slice_cols)
    isl, lab, info = ctx.source_find(img, 4.0, 2.5, 1.0, True, 5, capi.ZEROMEDIAN, False, conn4, True, 3, slice_cols)
    assert info.n_labels_pos == ref.n_pos and info.n_labels_neg == ref.n_neg
    _compare(isl, ref, lab, ref.label_map)


@pytest.mark.parametrize("method", [capi.BINAPPROX, capi.BINMEDIAN, capi.NTHELEMENT, capi.ZEROMEDIAN])
def test_source_find_end_to_end(ctx, method):
    """Median + sigma-clip RMS estimated on the device; bg and rms match the
    oracle to 1e-10 relative, labels bit-exact (no pixel lies within rounding
    distance of a threshold, checked)."""
    s = make_snapshot(7, 20000, 256, 2.0, n_src=6, flux=(2.0, 8.0), noise_sigma=0.3, n_extended=2)
    img, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, kernel_func=5, kernel_exact=False,
                                    oversampling=8, analytic_gcf=True)
    ref = orc.source_find(img, 5.0, 3.0, 0.0, True, 5, method, False, False, True, 5)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 0.0, True, 5, method, False, False, True, 5)
    assert abs(info.bg_level - ref.bg_level) <= 1e-10 * max(1e-300, abs(ref.rms_est))
    assert abs(info.rms_est - ref.rms_est) <= 1e-10 * abs(ref.rms_est)
    thr = [ref.bg_level + k * ref.rms_est for k in (3.0, -3.0, 5.0, -5.0)]
    near = min(float(np.min(np.abs(img - t))) for t in thr)
    if near < 1e-9 * ref.rms_est:
        pytest.skip("a pixel sits on a threshold")
    _compare(isl, ref, lab, ref.label_map)


def test_source_find_float32_input(ctx):
    rng = np.random.default_rng(9)
    img = rng.normal(size=(128, 192)).astype(np.float32)
    img[40:44, 50:55] += 9
    ref = orc.source_find(img.astype(np.float64), 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True, 5)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, False, False, True, 5)
    assert abs(info.rms_est - ref.rms_est) <= 1e-10 * ref.rms_est
    _compare(isl, ref, lab, ref.label_map)


def test_source_find_float32_extremum_ties(ctx):
    """Single-precision images take the one-pass extremum (value and first memory index in one 64-bit key):
    equal maxima / minima inside one island resolve to the first pixel in memory order, as in the
    reference's serial scan."""
    rng = np.random.default_rng(10)
    img = (0.5 * rng.normal(size=(160, 128))).astype(np.float32)
    img[30:35, 40:46] += 6.0
    img[31, 41] = img[33, 44] = np.float32(12.5)   # tied maxima, (31, 41) first in memory (column-major)
    img[100:104, 20:25] -= 6.0
    img[102, 21] = img[100, 23] = np.float32(-11.0)  # tied minima
    img = np.asfortranarray(img)
    ref = orc.source_find(img.astype(np.float64), 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True, 5)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, False, False, True, 5)
    _compare(isl, ref, lab, ref.label_map)
    got = {(i.sign, i.extremum_x_idx, i.extremum_y_idx) for i in isl}
    assert len(got) == len(isl) >= 2


def test_source_find_no_labelmap_cleanup(ctx):
    rng = np.random.default_rng(13)
    img = rng.normal(size=(64, 64))
    img[10:12, 10:12] += 10
    ref = orc.source_find(img, 5.0, 3.0, 1.0, False, 5, orc.ZEROMEDIAN, False, False, False, 1)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 1.0, False, 5, capi.ZEROMEDIAN, False, False, False, 1)
    _compare(isl, ref, lab, ref.label_map)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_crowded_field(ctx, dtype):
    """About a thousand bright islands (tens of thousands of valid pixels): each island's entries are
    ordered by one warp, and the island records come back in two reads; labels and islands as the
    oracle's."""
    rng = np.random.default_rng(9)
    img = rng.normal(size=(384, 384))
    for r in range(2, 384 - 10, 12):
        for c in range(2, 384 - 10, 12):
            img[r:r + 8, c:c + 8] += 6.0 + rng.uniform(0, 4)
    img = img.astype(dtype)
    ref = orc.source_find(img.astype(np.float64), 4.0, 2.5, 1.0, True, 5, orc.ZEROMEDIAN, False, False, True, 3, 0)
    assert sum(i[4] for i in ref.islands) > 8192 and len(ref.islands) > 512
    for _ in range(2):
        isl, lab, info = ctx.source_find(img, 4.0, 2.5, 1.0, True, 5, capi.ZEROMEDIAN, False, False, True, 3, 0)
        assert info.n_labels_pos == ref.n_pos and info.n_labels_neg == ref.n_neg
        _compare(isl, ref, lab, ref.label_map)


@pytest.mark.parametrize("step", [44, 36])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_medium_field_one_block_sort(ctx, step, dtype):
    """Between 2048 and 8192 valid island pixels (about 5.2k and 7.8k here) in 64-pixel islands; labels
    and islands as the oracle's."""
    rng = np.random.default_rng(10)
    img = rng.normal(size=(384, 384))
    for r in range(2, 384 - 10, step):
        for c in range(2, 384 - 10, step):
            img[r:r + 8, c:c + 8] += 6.0 + rng.uniform(0, 4)
    img = img.astype(dtype)
    ref = orc.source_find(img.astype(np.float64), 4.0, 2.5, 1.0, True, 5, orc.ZEROMEDIAN, False, False, True, 3, 0)
    assert 2048 < sum(i[4] for i in ref.islands) <= 8192
    isl, lab, info = ctx.source_find(img, 4.0, 2.5, 1.0, True, 5, capi.ZEROMEDIAN, False, False, True, 3, 0)
    assert info.n_labels_pos == ref.n_pos and info.n_labels_neg == ref.n_neg
    _compare(isl, ref, lab, ref.label_map)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_large_islands(ctx, dtype):
    """One island of 1600 pixels (ordered by one block) and one of 22500 (beyond the one-block
    limit of 16384: the multi-block sort of every entry), beside small ones; labels and islands as
    the oracle's."""
    rng = np.random.default_rng(12)
    img = rng.normal(size=(384, 384))
    img[20:60, 20:60] += 9.0
    img[200:350, 180:330] += 9.0
    img[100:104, 300:304] -= 9.0
    img = img.astype(dtype)
    ref = orc.source_find(img.astype(np.float64), 4.0, 2.5, 1.0, True, 5, orc.ZEROMEDIAN, False, False, True, 3, 0)
    assert max(i[4] for i in ref.islands) > 16384
    isl, lab, info = ctx.source_find(img, 4.0, 2.5, 1.0, True, 5, capi.ZEROMEDIAN, False, False, True, 3, 0)
    assert info.n_labels_pos == ref.n_pos and info.n_labels_neg == ref.n_neg
    _compare(isl, ref, lab, ref.label_map)


@pytest.mark.parametrize("shape", [(130, 98), (98, 130)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_rows_not_multiple_of_four(ctx, shape, dtype):
    """Row counts of 2 mod 4 take the one-key-per-thread class and label passes; labels and islands as the
    oracle's, with fixed and with estimated thresholds."""
    rng = np.random.default_rng(21)
    img = rng.normal(size=shape)
    img[10:18, 20:27] += 9.0
    img[0:2, :] += 4.5  # across the shifted-topology seams
    img[:, shape[1] // 2 - 1:shape[1] // 2 + 1] -= 5.0
    img = img.astype(dtype)
    ref = orc.source_find(img.astype(np.float64), 4.0, 2.5, 1.0, True, 5, orc.ZEROMEDIAN, False, False, True, 3, 0)
    isl, lab, info = ctx.source_find(img, 4.0, 2.5, 1.0, True, 5, capi.ZEROMEDIAN, False, False, True, 3, 0)
    assert info.n_labels_pos == ref.n_pos and info.n_labels_neg == ref.n_neg
    _compare(isl, ref, lab, ref.label_map)
    ref = orc.source_find(img.astype(np.float64), 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True, 5)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, False, False, True, 5)
    assert np.array_equal(lab, ref.label_map) and len(isl) == len(ref.islands)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_binned_median_falls_back_to_exact(ctx, dtype):
    """sigma * 2 < 1e-4: the binned median is not defined and the exact median is taken (the device flags
    it and the call runs the exact path); labels, islands and statistics as the oracle's."""
    rng = np.random.default_rng(4)
    img = (1e-6 * rng.normal(size=(128, 96))).astype(dtype)  # zero mean: no cancellation in sum x^2 / n - mean^2
    img[40:44, 50:53] = dtype(2e-5)
    ref = orc.source_find(img.astype(np.float64), 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True, 5)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, False, False, True, 5)
    assert info.sigma * 2 < 1e-4
    assert info.bg_level == ref.bg_level
    assert np.isclose(info.rms_est, ref.rms_est, rtol=1e-9, atol=0)
    assert np.array_equal(lab, ref.label_map) and len(isl) == len(ref.islands)


def _clip_image(kind, dtype):
    rng = np.random.default_rng(23)
    shape = (516, 388)  # 200208 pixels: not a multiple of 32 (the band mask's partial last word)
    if kind == "gauss":  # thresholds settle in the band, the clip ends early
        x = rng.normal(size=shape)
    elif kind == "laplace":  # thresholds stay in the band for eight passes
        x = rng.laplace(size=shape)
    elif kind == "skew":  # the third threshold falls below the band: full passes again
        x = np.where(rng.random(shape) < 0.3, rng.exponential(4.0, size=shape), rng.normal(size=shape))
    else:  # uniform: nothing beyond three sigma, the first pass ends the clip
        x = rng.uniform(-1.0, 1.0, size=shape)
    return np.asfortranarray(x.astype(dtype))


@pytest.mark.parametrize("kind", ["gauss", "laplace", "skew", "uniform"])
@pytest.mark.parametrize("iters", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("method", ["NTHELEMENT", "BINAPPROX"])
def test_sigma_clip_iterations(ctx, kind, iters, dtype, method):
    """The estimated RMS after 1-8 sigma-clip passes (sourcefind.cpp:280-301) within 1e-10 of the oracle's,
    labels bit-exact, through the fused statistics kernel: after a full pass, the passes whose threshold stays
    above the band's lower edge visit only the listed band samples; the skewed image's thresholds leave the
    band, so full passes come again."""
    img = _clip_image(kind, dtype)
    x = img.astype(np.float64)
    ref = orc.source_find(x, 5.0, 3.0, 0.0, True, iters, getattr(orc, method), False, False, True, 5)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 0.0, True, iters, getattr(capi, method), False, False, True, 5)
    assert abs(info.rms_est - ref.rms_est) <= 1e-10 * abs(ref.rms_est)
    assert abs(info.bg_level - ref.bg_level) <= 1e-12 * max(1.0, abs(ref.bg_level))
    assert np.array_equal(lab, ref.label_map) and len(isl) == len(ref.islands)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("case", ["two_level", "offset"])
def test_binned_median_cases(ctx, case, dtype):
    """The binned median (matrix_math.cpp:334-455) through the fused statistics kernel: a two-level image
    whose cumulative count equals the rank at the lower level's bin, so the even-count walk crosses empty bins
    to the upper level's bin; a large offset (mean 3e4 sigma), where the single-precision bin screen defers
    most samples to double precision.  Labels and islands as the oracle's; bg_level exact for the two-level
    image.  With the offset, sigma = sqrt(sum x^2 / n - mean^2) cancels 9e8 against 9e8 (the reference's
    formula, matrix_math.cpp:457-499), and the clip's d^2 sums inherit it, so the oracle's sequential sums and
    the device's tree sums agree only to that conditioning: bg_level within 1e-10 relative, rms within 1e-4
    (measured 1e-5 and 2e-6)."""
    rng = np.random.default_rng(31)
    if case == "two_level":
        img = np.empty((512, 384))
        img[: img.shape[0] // 2] = -1.0
        img[img.shape[0] // 2:] = 1.0
        img[300:303, 100:103] = 40.0  # in the upper half: the lower half's count is exactly the rank
        img[301, 101] = 41.0
    else:
        img = 3.0e4 + rng.normal(size=(512, 384))
        img[300:304, 60:63] += 15.0
    img = np.asfortranarray(img.astype(dtype))
    x = img.astype(np.float64)
    ref = orc.source_find(x, 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True, 5)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, False, False, True, 5)
    if case == "two_level":
        assert info.bg_level == ref.bg_level
        assert abs(info.rms_est - ref.rms_est) <= 1e-10 * abs(ref.rms_est)
    else:
        assert abs(info.bg_level - ref.bg_level) <= 1e-10 * abs(ref.bg_level)
        assert abs(info.rms_est - ref.rms_est) <= 1e-4 * abs(ref.rms_est)
    assert np.array_equal(lab, ref.label_map) and len(isl) == len(ref.islands)


@pytest.mark.parametrize("method", ["ZEROMEDIAN", "BINAPPROX", "BINMEDIAN", "NTHELEMENT"])
@pytest.mark.parametrize("rms_est", [0.0, 1.5])
def test_stats_fused_and_pass_kernels_agree(ctx, monkeypatch, method, rms_est):
    """Each median method, with the rms estimated or given: the fused statistics kernel and the pass kernels
    (STPGPU_SF_STATS=passes) give the oracle's labels and islands and the same statistics."""
    img = _clip_image("laplace", np.float64)
    img[100:104, 200:203] += 30.0
    ref = orc.source_find(img, 5.0, 3.0, rms_est, True, 5, getattr(orc, method), False, False, True, 5)
    got = []
    for mode in ("fused", "passes"):
        if mode == "passes":
            monkeypatch.setenv("STPGPU_SF_STATS", "passes")
        isl, lab, info = ctx.source_find(img, 5.0, 3.0, rms_est, True, 5, getattr(capi, method), False, False, True,
                                         5)
        monkeypatch.delenv("STPGPU_SF_STATS", raising=False)
        assert np.array_equal(lab, ref.label_map) and len(isl) == len(ref.islands), mode
        assert abs(info.rms_est - ref.rms_est) <= 1e-10 * abs(ref.rms_est), mode
        got.append((info.bg_level, info.rms_est))
    assert np.allclose(got[0], got[1], rtol=1e-12, atol=0)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_repeated_device_calls_replay_graph_with_new_data(dtype):
    """Identical device-pointer calls: the second captures the first attempt into a CUDA graph, later ones
    replay it.  New pixel values written into the same device buffer between calls must be what the replay
    reads: every call's labels and islands equal the oracle's for that call's image."""
    import torch

    fresh = capi.Context(0)
    rng = np.random.default_rng(41)
    rows, cols = 512, 384
    dimg = torch.empty(rows * cols, dtype=torch.float64 if dtype == np.float64 else torch.float32, device="cuda")
    lab = torch.empty(rows * cols, dtype=torch.int32, device="cuda")
    try:
        for call in range(5):
            img = rng.normal(size=(rows, cols))
            for _ in range(4 + call):
                r, c = rng.integers(0, rows - 6), rng.integers(0, cols - 6)
                img[r:r + 4, c:c + 3] += rng.choice([-9.0, 9.0])
            img = np.asfortranarray(img.astype(dtype))
            dimg.copy_(torch.from_numpy(img.reshape(-1, order="F").copy()))
            torch.cuda.synchronize()
            isl, _, info = fresh.source_find(dimg, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, False, False, True, 5,
                                             device_ptrs=True, rows=rows, cols=cols, label_out=lab)
            torch.cuda.synchronize()
            got = lab.cpu().numpy().reshape((rows, cols), order="F")
            ref = orc.source_find(img.astype(np.float64), 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True,
                                  5)
            assert np.array_equal(got, ref.label_map), f"call {call}"
            assert abs(info.rms_est - ref.rms_est) <= 1e-10 * abs(ref.rms_est)
            _compare(isl, ref, got, ref.label_map)
    finally:
        fresh.close()


def test_foreground_beyond_first_capacity():
    """A 512^2 image with a low analysis threshold has about 200 k foreground pixels, beyond the
    label-analysis capacity a fresh context starts with (n / 16 entries, at least 131072): the first call runs
    that stage again with larger buffers, the second uses the remembered capacity; both match the oracle."""
    fresh = capi.Context(0)
    rng = np.random.default_rng(17)
    img = rng.normal(size=(512, 512))
    ref = orc.source_find(img, 3.0, 0.3, 1.0, True, 5, orc.ZEROMEDIAN, False, False, True, 3, 0)
    try:
        for _ in range(2):
            isl, lab, info = fresh.source_find(img, 3.0, 0.3, 1.0, True, 5, capi.ZEROMEDIAN, False, False, True, 3,
                                               0)
            assert info.n_labels_pos == ref.n_pos and info.n_labels_neg == ref.n_neg
            _compare(isl, ref, lab, ref.label_map)
    finally:
        fresh.close()


def test_source_find_rejects(ctx):
    with pytest.raises(capi.StpGpuError):
        ctx.source_find(np.zeros((7, 8)), 5, 3)


@pytest.mark.parametrize("min_area", [5, 1])
def test_gaussian_fit_matches_oracle(ctx, min_area):
    """Least-squares 2-D Gaussian per island (sourcefind.cpp:719-866; Levenberg-Marquardt on both sides in
    place of Ceres): the GPU fit agrees with the oracle's, and recovers the injected extended sources."""
    from fastimaging_b200.synthetic import make_snapshot

    s = make_snapshot(81, 30000, 256, 2.0, n_src=5, flux=(4.0, 9.0), noise_sigma=0.05, n_extended=3)
    img, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, kernel_func=capi.GaussianSinc,
                                       kernel_exact=False, oversampling=8)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, True, False, True, min_area)
    ref = orc.source_find(img, 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, True, False, True, min_area)
    assert len(isl) == len(ref.islands) > 0
    fitted = 0
    for a, b in zip(isl, ref.islands):
        f = b[6]
        want = np.array([f.amplitude, f.x_centre, f.y_centre, f.semimajor, f.semiminor, f.theta])
        got = np.array(a.leastsq_fit[:])
        assert np.allclose(got, want, rtol=1e-6, atol=1e-6), (got, want)
        if a.num_samples >= 3:
            assert a.fit_iterations > 0
            assert got[3] >= got[4] and -np.pi / 2 <= got[5] <= np.pi / 2
            fitted += 1
        else:
            assert got[0] == a.extremum_val and not got[1:].any()
    assert fitted > 0
