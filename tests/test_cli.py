"""Command-line drivers (src/reduce/*.cpp): configuration keys and defaults,
size rounding, island JSON layout; end to end on the GPU."""
import json
import os

import numpy as np
import pytest

from fastimaging_b200 import capi, cli

CONFIG = {
    "imager_settings": {"image_size_pix": 254, "cell_size_arcsec": 2.0, "padding_factor": 1.0,
                        "kernel_function": "GaussianSinc", "kernel_support": 3, "kernel_exact": False,
                        "oversampling": 8, "generate_beam": False, "gridding_correction": True, "analytic_gcf": False,
                        "fft_routine": "FFTW_ESTIMATE_FFT", "fft_wisdom_filename": ""},
    "wprojection_settings": {"num_wplanes": 0},
    "sourcefind_settings": {"sourcefind_detection": 5.0, "sourcefind_analysis": 3.0, "find_negative_sources": True,
                            "rms_estimation": 0.0, "sigma_clip_iters": 5, "median_method": "BINAPPROX",
                            "gaussian_fitting": False, "ccl_4connectivity": False, "generate_labelmap": True,
                            "source_min_area": 5, "ceres_diffmethod": "AutoDiff_SingleResBlk",
                            "ceres_solvertype": "LinearSearch_BFGS"},
}


def test_config_keys_and_defaults(tmp_path):
    p = tmp_path / "c.json"
    p.write_text(json.dumps(CONFIG))
    cfg = cli.load_config(str(p))
    assert cfg["image_size"] == 254 and cfg["kernel_func"] == capi.GaussianSinc and cfg["oversampling"] == 8
    assert cfg["median_method"] == capi.BINAPPROX and cfg["detection_n_sigma"] == 5.0
    cli.set_image_sizes(cfg)
    assert cfg["image_size"] == 256 and cfg["padded_image_size"] == 256
    p.write_text(json.dumps({"imager_settings": {"image_size_pix": 64, "cell_size_arcsec": 1.0}}))
    d = cli.load_config(str(p))
    # ConfigurationFile / ImagerPars defaults
    assert d["kernel_func"] == capi.PSWF and d["kernel_exact"] and not d["gridding_correction"]
    assert d["median_method"] == capi.BINMEDIAN and d["gaussian_fitting"] and not d["generate_labelmap"]
    assert d["source_min_area"] == 5 and d["sigma_clip_iters"] == 5 and d["num_wplanes"] == 0
    p.write_text(json.dumps({"imager_settings": {"kernel_function": "Bessel"}}))
    with pytest.raises(ValueError):
        cli.load_config(str(p))
    # Hankel and A-projection settings (load_json_config.cpp: wprojection_settings, aprojection_settings)
    p.write_text(json.dumps({"wprojection_settings": {"num_wplanes": 4, "hankel_opt": True, "hankel_proj_slice": True,
                                                      "interp_type": "cubic"},
                             "aprojection_settings": {"aproj_numtimesteps": 3, "obs_dec": -30.0, "obs_ra": 20.0,
                                                      "pbeam_coefs": [0.5, 1.0, 0.5], "aproj_opt": True}}))
    h = cli.load_config(str(p))
    assert h["hankel_opt"] and h["hankel_proj_slice"] and h["interp_type"] == capi.CUBIC
    assert h["aproj_numtimesteps"] == 3 and h["pbeam_coefs"] == [0.5, 1.0, 0.5] and h["aproj_opt"]
    assert h["obs_dec"] == -30.0 and h["obs_ra"] == 20.0
    empty = tmp_path / "e.json"
    empty.write_text("")
    with pytest.raises(RuntimeError):
        cli.load_config(str(empty))


def test_island_json_layout():
    isl = capi.Island()
    isl.sign, isl.extremum_val, isl.extremum_x_idx, isl.extremum_y_idx = -1, -7.5, 10, 20
    isl.moments_fit[:] = [1, 2, 3, 4, 5, 0.5]
    isl.leastsq_fit[:] = [6, 7, 8, 9, 10, 0.25]
    d = cli.islands_json([isl], False)
    assert d == {"Islands": [{"sign": -1, "val": -7.5, "x_idx": 10, "y_idx": 20,
                              "MomentsFit": {"amplitude": 1.0, "x_centre": 2.0, "y_centre": 3.0, "semimajor": 4.0,
                                             "semiminor": 5.0, "theta": 0.5}}]}
    assert cli.islands_json([isl], True)["Islands"][0]["GaussianFit"]["theta"] == 0.25


def test_run_sourcefind_passes_area_and_labelmap_swapped():
    cfg = dict(detection_n_sigma=5.0, analysis_n_sigma=3.0, rms_est=0.0, find_negative_sources=True,
               sigma_clip_iters=5, median_method=capi.BINAPPROX, gaussian_fitting=False, ccl_4connectivity=False,
               generate_labelmap=False, source_min_area=7)
    assert cli._sf_args(cfg)[-2:] == (False, 7)
    assert cli._sf_args(cfg, swapped=True)[-2:] == (True, 0)


@pytest.mark.gpu
def test_reduce_end_to_end(tmp_path):
    from fastimaging_b200.synthetic import make_snapshot

    s = make_snapshot(91, 20000, 256, 2.0, n_src=5, flux=(3.0, 8.0), noise_sigma=0.05)
    npz = tmp_path / "in.npz"
    sky = s.sources.copy()
    np.savez(npz, uvw_lambda=s.uvw, vis=s.vis, snr_weights=s.weights, skymodel=sky)
    cfgp = tmp_path / "c.json"
    cfgp.write_text(json.dumps(CONFIG))
    out_json, out_npz = tmp_path / "o.json", tmp_path / "o.npz"
    assert cli.main(["reduce", str(cfgp), str(npz), "-s", str(out_json), "-o", str(out_npz)]) == 0
    got = json.loads(out_json.read_text())["Islands"]
    ctx = capi.Context(0)
    try:
        img, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, 2.0, kernel_func=capi.GaussianSinc,
                                           kernel_support=3, kernel_exact=False, oversampling=8,
                                           gridding_correction=True, analytic_gcf=False)
        isl, lab, _ = ctx.source_find(img, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, False, False, True, 5)
    finally:
        ctx.close()
    assert len(got) == len(isl) > 0
    for a, b in zip(got, isl):
        assert (a["sign"], a["x_idx"], a["y_idx"]) == (b.sign, b.extremum_x_idx, b.extremum_y_idx)
        assert a["val"] == pytest.approx(b.extremum_val, rel=1e-12)
    assert np.array_equal(np.load(out_npz)["label_map"], lab)
    # residual imaging: the model of the sky removes the sources
    out_img = tmp_path / "img.npz"
    assert cli.main(["run_imager", str(cfgp), str(npz), "-o", str(out_img), "-d"]) == 0
    res = np.load(out_img)["image"]
    assert res.shape == (256, 256) and np.max(np.abs(res)) < 0.2 * np.max(np.abs(img))
