"""The stp_python drop-in module on the GPU against the oracle, called the
way the reference's Python tests and pipelines call its binding
(src/stp-python/stp_python.cpp:17-173)."""
import numpy as np
import pytest

from fastimaging_b200.synthetic import make_snapshot
from oracle import stp_oracle as orc

pytestmark = pytest.mark.gpu
stp_python = pytest.importorskip("fastimaging_b200.stp_python")


def _peak_rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("image_size,padding,beam", [(256, 1.0, False), (254, 1.0, True), (192, 1.5, False)])
def test_image_visibilities_wrapper_matches_oracle(image_size, padding, beam):
    s = make_snapshot(21, 4000, 256, 2.0, n_src=3, noise_sigma=0.1)
    kw = dict(padding_factor=padding, kernel_support=3, kernel_exact=False, kernel_oversampling=8,
              generate_beam=beam, gridding_correction=True, analytic_gcf=False)
    img, bm = stp_python.image_visibilities_wrapper(s.vis, s.weights, s.uvw, image_size, s.cell_size,
                                                    kernel_func=stp_python.KernelFunction.GaussianSinc, **kw)
    okw = dict(kw)
    okw["oversampling"] = okw.pop("kernel_oversampling")
    ref, rbeam = orc.image_visibilities(s.vis, s.weights, s.uvw, image_size, s.cell_size, kernel_func=orc.GaussianSinc,
                                        **okw)
    size = image_size + (-image_size) % 4
    assert img.shape == (size, size) and img.flags.f_contiguous and img.dtype == np.float64
    assert _peak_rel(img, ref) < 1e-10
    if beam:
        assert bm.shape == (size, size)
        assert _peak_rel(bm, rbeam) < 1e-10
    else:
        assert bm.shape == (0, 0)


def test_image_visibilities_wrapper_wproj_and_c_order_inputs():
    s = make_snapshot(22, 3000, 256, 2.0, n_src=3, w_range=(-400.0, 400.0))
    kw = dict(kernel_support=3, kernel_exact=False, kernel_oversampling=8, num_wplanes=4, max_wpconv_support=8,
              kernel_trunc_perc=1.0)
    uvw_c = np.ascontiguousarray(s.uvw)  # C order: coerced to F order as forcecast does
    img, _ = stp_python.image_visibilities_wrapper(s.vis, s.weights, uvw_c, 256, s.cell_size,
                                                   kernel_func=stp_python.KernelFunction.GaussianSinc, **kw)
    okw = dict(kw)
    okw["oversampling"] = okw.pop("kernel_oversampling")
    ref, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, kernel_func=orc.GaussianSinc, **okw)
    assert _peak_rel(img, ref) < 1e-10


def test_image_visibilities_wrapper_empty_result():
    s = make_snapshot(23, 100, 64, 1.0, n_src=1)
    uvw = s.uvw.copy()
    uvw[:, :2] *= 1e6  # every visibility out of bounds: sample total 0 -> empty matrices
    img, bm = stp_python.image_visibilities_wrapper(s.vis, s.weights, uvw, 64, s.cell_size)
    assert img.shape == (0, 0) and bm.shape == (0, 0)


def test_image_visibilities_wrapper_aprojection_and_hankel():
    s = make_snapshot(24, 3000, 128, 10.0, n_src=2, w_range=(-500.0, 500.0))
    # A-projection without W-projection is an error (imager.h:279-280)
    with pytest.raises(RuntimeError):
        stp_python.image_visibilities_wrapper(s.vis, s.weights, s.uvw, 128, s.cell_size, aproj_numtimesteps=2)
    lha = np.linspace(-2.0, 2.0, s.vis.size)
    kw = dict(kernel_func=stp_python.KernelFunction.GaussianSinc, kernel_exact=False, kernel_oversampling=4,
              num_wplanes=2, max_wpconv_support=6, kernel_trunc_perc=1.0)
    img, _ = stp_python.image_visibilities_wrapper(s.vis, s.weights, s.uvw, 128, s.cell_size, aproj_numtimesteps=2,
                                                   obs_dec=-30.0, obs_ra=10.0, lha=lha,
                                                   pbeam_coefs=np.array([0.2, 1.0, 0.4]), **kw)
    ref, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 128, s.cell_size, kernel_func=orc.GaussianSinc,
                                    kernel_exact=False, oversampling=4, num_wplanes=2, max_wpconv_support=6,
                                    kernel_trunc_perc=1.0, aproj_numtimesteps=2, obs_dec=-30.0, obs_ra=10.0, lha=lha,
                                    pbeam_coefs=[0.2, 1.0, 0.4])
    assert np.max(np.abs(img - ref)) < 1e-10 * np.max(np.abs(ref))
    img, _ = stp_python.image_visibilities_wrapper(s.vis, s.weights, s.uvw, 128, s.cell_size, hankel_opt=True,
                                                   interp_type=stp_python.InterpType.CUBIC, **kw)
    ref, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 128, s.cell_size, kernel_func=orc.GaussianSinc,
                                    kernel_exact=False, oversampling=4, num_wplanes=2, max_wpconv_support=6,
                                    kernel_trunc_perc=1.0, hankel_opt=True, interp_type=orc.CUBIC)
    assert np.max(np.abs(img - ref)) < 1e-10 * np.max(np.abs(ref))


def test_source_find_wrapper_matches_oracle():
    s = make_snapshot(25, 20000, 256, 2.0, n_src=6, flux=(3.0, 8.0), noise_sigma=0.1)
    img, _ = stp_python.image_visibilities_wrapper(s.vis, s.weights, s.uvw, 256, s.cell_size,
                                                   kernel_func=stp_python.KernelFunction.GaussianSinc,
                                                   kernel_exact=False)
    got = stp_python.source_find_wrapper(img, 5.0, 3.0)
    ref = orc.source_find(img, 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True, 5)
    assert len(got) == len(ref.islands) > 0
    for a, b in zip(got, ref.islands):
        assert a[:5] == b[:5]
        m, r = a[5], b[5]
        for f in ("amplitude", "x_centre", "y_centre", "semimajor", "semiminor", "theta"):
            assert np.isclose(getattr(m, f), getattr(r, f), rtol=1e-9, atol=1e-9), f
        assert a[6].amplitude == 0.0 and a[7] == ""
