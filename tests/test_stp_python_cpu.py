"""The stp_python drop-in module: interface checks that need no GPU
(names, enum values, defaults, Gaussian2dParams), mirroring the reference's
binding src/stp-python/stp_python.cpp:181-284."""
import numpy as np
import pytest

stp_python = pytest.importorskip("fastimaging_b200.stp_python")


def test_enums_match_reference_values():
    assert [int(getattr(stp_python.KernelFunction, n)) for n in
            ("TopHat", "Triangle", "Sinc", "Gaussian", "GaussianSinc", "PSWF")] == list(range(6))
    assert [int(getattr(stp_python.MedianMethod, n)) for n in
            ("ZEROMEDIAN", "BINMEDIAN", "BINAPPROX", "NTHELEMENT")] == list(range(4))
    for n in ("FFTW_ESTIMATE_FFT", "FFTW_MEASURE_FFT", "FFTW_PATIENT_FFT", "FFTW_WISDOM_FFT",
              "FFTW_WISDOM_INPLACE_FFT"):
        assert hasattr(stp_python.FFTRoutine, n)
    for n in ("LINEAR", "COSINE", "CUBIC"):
        assert hasattr(stp_python.InterpType, n)
    for n in ("AutoDiff", "AutoDiff_SingleResBlk", "AnalyticDiff", "AnalyticDiff_SingleResBlk"):
        assert hasattr(stp_python.CeresDiffMethod, n)
    for n in ("LinearSearch_BFGS", "LinearSearch_LBFGS", "TrustRegion_DenseQR"):
        assert hasattr(stp_python.CeresSolverType, n)


def test_gaussian2dparams():
    g = stp_python.Gaussian2dParams()
    assert (g.amplitude, g.x_centre, g.y_centre, g.semimajor, g.semiminor, g.theta) == (0.0,) * 6
    g.amplitude = 2.5
    assert repr(g).startswith("Gaussian2dParams=[2.500000, 0.000000")


def _defaults(fn):
    """{argument: default text or None} parsed from the pybind11 signature line."""
    sig = fn.__doc__.split("\n")[0]
    body = sig[sig.index("(") + 1:sig.rindex(")")]
    parts, depth, cur = [], 0, ""
    for ch in body:
        if ch in "[(<":
            depth += 1
        elif ch in "])>":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    out = {}
    for p in parts:
        name = p.split(":")[0].strip()
        out[name] = p.split(" = ", 1)[1].strip() if " = " in p else None
    return out


def test_signatures_and_defaults():
    d = _defaults(stp_python.image_visibilities_wrapper)
    assert list(d) == ["vis", "snr_weights", "uvw_lambda", "image_size", "cell_size", "padding_factor", "kernel_func",
                       "kernel_support", "kernel_exact", "kernel_oversampling", "generate_beam", "gridding_correction",
                       "analytic_gcf", "r_fft", "fft_wisdom_filename", "num_wplanes", "wplanes_median",
                       "max_wpconv_support", "hankel_opt", "hankel_proj_slice", "undersampling_opt",
                       "kernel_trunc_perc", "interp_type", "aproj_numtimesteps", "obs_dec", "obs_ra", "aproj_opt",
                       "aproj_mask_perc", "lha", "pbeam_coefs"]
    assert d["vis"] is None and d["cell_size"] is None
    assert (d["padding_factor"], d["kernel_support"], d["kernel_exact"], d["kernel_oversampling"]) == \
        ("1.0", "3", "True", "8")
    assert "PSWF" in d["kernel_func"] and "FFTW_ESTIMATE_FFT" in d["r_fft"] and "LINEAR" in d["interp_type"]
    assert (d["generate_beam"], d["gridding_correction"], d["analytic_gcf"], d["num_wplanes"],
            d["undersampling_opt"], d["kernel_trunc_perc"]) == ("False", "True", "False", "0", "1", "0.0")
    d = _defaults(stp_python.source_find_wrapper)
    assert list(d) == ["image_data", "detection_n_sigma", "analysis_n_sigma", "rms_est", "find_negative_sources",
                       "sigma_clip_iters", "median_method", "gaussian_fitting", "ccl_4connectivity",
                       "generate_labelmap", "source_min_area", "ceres_diffmethod", "ceres_solvertype"]
    assert (d["rms_est"], d["find_negative_sources"], d["sigma_clip_iters"], d["gaussian_fitting"],
            d["ccl_4connectivity"], d["generate_labelmap"], d["source_min_area"]) == \
        ("0.0", "True", "5", "False", "False", "True", "5")
    assert "BINAPPROX" in d["median_method"] and "AutoDiff_SingleResBlk" in d["ceres_diffmethod"]
    assert "LinearSearch_BFGS" in d["ceres_solvertype"]


def test_no_device_raises_runtime_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError):
        stp_python.image_visibilities_wrapper(np.zeros(4, complex), np.ones(4), np.zeros((4, 3)), 64, 1.0)
