"""Command-line drivers with the reference's interface (src/reduce/reduce.cpp,
run_imager.cpp, run_sourcefind.cpp): a JSON configuration with the
reference's keys (src/auxiliary/load_json_config.h) and NPZ data with its
array names, run on the GPU through the C ABI.

    python -m fastimaging_b200.cli reduce         CONFIG.json INPUT.npz [-s OUT.json] [-o OUT.npz] [-d] [-l] [-n] [-b]
    python -m fastimaging_b200.cli run_imager     CONFIG.json INPUT.npz [-o OUT.npz] [-d] [-l] [-b]
    python -m fastimaging_b200.cli run_sourcefind CONFIG.json INPUT.npz [-s OUT.json] [-o OUT.npz] [-l] [-n] [-b]

Input NPZ arrays: uvw_lambda (n x 3), vis (n, complex), snr_weights (n),
skymodel (k x 3: l, m, flux; with -d the model visibilities are subtracted),
lha (n, hours; read when aprojection_settings enable A-projection);
run_sourcefind reads image.  Outputs: islands as JSON
({"Islands": [{"sign", "val", "x_idx", "y_idx", "MomentsFit", "GaussianFit"}]},
save_json_sf_output.cpp), label_map / image and beam as NPZ.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import capi

KERNELS = {"TopHat": capi.TopHat, "Triangle": capi.Triangle, "Sinc": capi.Sinc, "Gaussian": capi.Gaussian,
           "GaussianSinc": capi.GaussianSinc, "PSWF": capi.PSWF}
MEDIANS = {"ZEROMEDIAN": capi.ZEROMEDIAN, "BINMEDIAN": capi.BINMEDIAN, "BINAPPROX": capi.BINAPPROX,
           "NTHELEMENT": capi.NTHELEMENT}
FFT_ROUTINES = ("FFTW_ESTIMATE_FFT", "FFTW_MEASURE_FFT", "FFTW_PATIENT_FFT", "FFTW_WISDOM_FFT", "FFTW_WISDOM_INPLACE_FFT")
INTERP = ("linear", "cosine", "cubic")
DIFF_METHODS = ("AutoDiff", "AutoDiff_SingleResBlk", "AnalyticDiff", "AnalyticDiff_SingleResBlk")
SOLVERS = ("LinearSearch_BFGS", "LinearSearch_LBFGS", "TrustRegion_DenseQR")


def load_config(path):
    """ConfigurationFile (src/auxiliary/load_json_config.h): the sections imager_settings,
    wprojection_settings, aprojection_settings and sourcefind_settings, with the reference's defaults for
    missing keys.  Unknown enum strings raise ValueError (the reference asserts)."""
    with open(path) as f:
        text = f.read()
    if not text.strip():
        raise RuntimeError("Failed to read configuration file: " + path)
    doc = json.loads(text)

    def pick(table, name, what):
        if name not in table:
            raise ValueError(f"unknown {what}: {name}")
        return table[name] if isinstance(table, dict) else table.index(name)

    im = doc.get("imager_settings", {})
    cfg = dict(image_size=0, cell_size=0.0, padding_factor=1.0, kernel_func=capi.PSWF, kernel_support=0,
               kernel_exact=True, oversampling=0, generate_beam=False, gridding_correction=False, analytic_gcf=False,
               fft_routine="FFTW_ESTIMATE_FFT", fft_wisdom_filename="")
    if "image_size_pix" in im:
        cfg["image_size"] = int(im["image_size_pix"])
    if "cell_size_arcsec" in im:
        cfg["cell_size"] = float(im["cell_size_arcsec"])
    if "padding_factor" in im:
        cfg["padding_factor"] = float(im["padding_factor"])
    if "kernel_function" in im:
        cfg["kernel_func"] = pick(KERNELS, im["kernel_function"], "kernel_function")
    for key, name, cast in (("kernel_support", "kernel_support", int), ("kernel_exact", "kernel_exact", bool),
                            ("oversampling", "oversampling", int), ("generate_beam", "generate_beam", bool),
                            ("gridding_correction", "gridding_correction", bool),
                            ("analytic_gcf", "analytic_gcf", bool)):
        if key in im:
            cfg[name] = cast(im[key])
    if "fft_routine" in im:
        pick(FFT_ROUTINES, im["fft_routine"], "fft_routine")
        cfg["fft_routine"] = im["fft_routine"]
    if "fft_wisdom_filename" in im:
        cfg["fft_wisdom_filename"] = im["fft_wisdom_filename"]

    wp = doc.get("wprojection_settings", {})
    cfg.update(num_wplanes=int(wp.get("num_wplanes", 0)), wplanes_median=bool(wp.get("wplanes_median", False)),
               max_wpconv_support=int(wp.get("max_wpconv_support", 0)), hankel_opt=bool(wp.get("hankel_opt", False)),
               undersampling_opt=int(wp.get("undersampling_opt", 1)),
               kernel_trunc_perc=float(wp.get("kernel_trunc_perc", 0.0)))
    cfg["hankel_proj_slice"] = bool(wp.get("hankel_proj_slice", False))
    cfg["interp_type"] = capi.LINEAR
    if "interp_type" in wp:
        pick(INTERP, wp["interp_type"], "interp_type")
        cfg["interp_type"] = {"linear": capi.LINEAR, "cosine": capi.COSINE, "cubic": capi.CUBIC}[wp["interp_type"]]
    ap = doc.get("aprojection_settings", {})
    cfg.update(aproj_numtimesteps=int(ap.get("aproj_numtimesteps", 0)), obs_dec=float(ap.get("obs_dec", 0.0)),
               obs_ra=float(ap.get("obs_ra", 0.0)), aproj_opt=bool(ap.get("aproj_opt", False)),
               aproj_mask_perc=float(ap.get("aproj_mask_perc", 0.0)),
               pbeam_coefs=[float(v) for v in ap.get("pbeam_coefs", [])])

    sf = doc.get("sourcefind_settings", {})
    cfg.update(detection_n_sigma=float(sf.get("sourcefind_detection", 0.0)),
               analysis_n_sigma=float(sf.get("sourcefind_analysis", 0.0)),
               find_negative_sources=bool(sf.get("find_negative_sources", True)),
               rms_est=float(sf.get("rms_estimation", 0.0)), sigma_clip_iters=int(sf.get("sigma_clip_iters", 5)),
               median_method=pick(MEDIANS, sf.get("median_method", "BINMEDIAN"), "median_method"),
               gaussian_fitting=bool(sf.get("gaussian_fitting", True)),
               ccl_4connectivity=bool(sf.get("ccl_4connectivity", False)),
               generate_labelmap=bool(sf.get("generate_labelmap", False)),
               source_min_area=int(sf.get("source_min_area", 5)))
    pick(DIFF_METHODS, sf.get("ceres_diffmethod", "AutoDiff_SingleResBlk"), "ceres_diffmethod")
    pick(SOLVERS, sf.get("ceres_solvertype", "LinearSearch_BFGS"), "ceres_solvertype")
    return cfg


def set_image_sizes(cfg, log=None):
    """set_image_sizes (src/reduce/common_functions.cpp:49-78): image and padded sizes up to multiples of 4."""
    size = cfg["image_size"]
    while size % 4:
        size += 1
    if size != cfg["image_size"] and log:
        log(f"Image size must be a multiple of four: set to {size} pixels.")
    cfg["image_size"] = size
    padded = int(float(size) * cfg["padding_factor"])
    p0 = padded
    while padded % 4:
        padded += 1
    if padded != p0 and log:
        log(f"Padded image size must be a multiple of four: set to {padded} pixels.")
    cfg["padded_image_size"] = padded
    return cfg


def islands_json(islands, gaussian_fitting):
    """save_json_sourcefind_output (src/auxiliary/save_json_sf_output.cpp:8-49)."""
    names = ("amplitude", "x_centre", "y_centre", "semimajor", "semiminor", "theta")
    out = []
    for i in islands:
        d = {"sign": int(i.sign), "val": float(i.extremum_val), "x_idx": int(i.extremum_x_idx),
             "y_idx": int(i.extremum_y_idx), "MomentsFit": dict(zip(names, map(float, i.moments_fit[:])))}
        if gaussian_fitting:
            d["GaussianFit"] = dict(zip(names, map(float, i.leastsq_fit[:])))
        out.append(d)
    return {"Islands": out}


def _imager_kw(cfg):
    keys = ("padding_factor", "kernel_func", "kernel_support", "kernel_exact", "oversampling", "generate_beam",
            "gridding_correction", "analytic_gcf", "num_wplanes", "wplanes_median", "max_wpconv_support",
            "undersampling_opt", "kernel_trunc_perc", "hankel_opt", "hankel_proj_slice", "interp_type",
            "aproj_numtimesteps", "padded_image_size")
    kw = {k: cfg[k] for k in keys}
    if cfg["aproj_numtimesteps"] > 0:
        kw.update({k: cfg[k] for k in ("obs_dec", "obs_ra", "aproj_opt", "aproj_mask_perc", "pbeam_coefs")})
    return kw


def _sf_args(cfg, swapped=False):
    """SourceFindImage arguments in order.  swapped: pass source_min_area where generate_labelmap goes and
    vice versa, as run_sourcefind.cpp:103-105 does (the standalone source-finder tool of the reference)."""
    gl, area = cfg["generate_labelmap"], cfg["source_min_area"]
    if swapped:
        gl, area = bool(area), int(gl)
    return (cfg["detection_n_sigma"], cfg["analysis_n_sigma"], cfg["rms_est"], cfg["find_negative_sources"],
            cfg["sigma_clip_iters"], cfg["median_method"], cfg["gaussian_fitting"], cfg["ccl_4connectivity"], gl, area)


def _parser(prog, desc, sf_out, img_diff):
    p = argparse.ArgumentParser(prog=prog, description=desc)
    p.add_argument("input_file_json")
    p.add_argument("input_file_npz")
    if sf_out:
        p.add_argument("-s", "--output-file-json", default=None, help="output JSON file for detected islands")
    p.add_argument("-o", "--output-file-npz", default=None, help="output NPZ file")
    if img_diff:
        p.add_argument("-d", "--diff", action="store_true",
                       help="image the residual visibilities: input vis minus the model of 'skymodel'")
    p.add_argument("-l", "--log", action="count", default=0, help="log to stdout")
    if sf_out:
        p.add_argument("-n", "--no-src", action="store_true", help="do not log the detected islands")
    p.add_argument("-b", "--no-bench", action="store_true", help="do not log timings")
    return p


def _run_imager(ctx, cfg, npz, diff, log):
    uvw = np.asarray(npz["uvw_lambda"], dtype=np.float64)
    vis = np.asarray(npz["vis"]).reshape(-1).astype(np.complex128)
    w = np.asarray(npz["snr_weights"], dtype=np.float64).reshape(-1)
    if diff:
        vis = ctx.model_visibilities(np.asarray(npz["skymodel"], dtype=np.float64), uvw, vis=vis)
        log("Use residual visibilities - input visibilities subtracted from model visibilities")
    kw = _imager_kw(cfg)
    if cfg["aproj_numtimesteps"] > 0:
        kw["lha"] = np.asarray(npz["lha"], dtype=np.float64).reshape(-1)  # reduce.cpp:107-111
    t0 = time.perf_counter()
    img, beam, info = ctx.image_visibilities(vis, w, uvw, cfg["image_size"], cfg["cell_size"], **kw)
    return img, beam, info, time.perf_counter() - t0


def _log_islands(islands, log):
    log(f"Number of detected sources: {len(islands)}")
    for k, i in enumerate(islands):
        log(f"Island {k}: sign={i.sign} val={i.extremum_val:.6g} x_idx={i.extremum_x_idx} y_idx={i.extremum_y_idx} "
            f"num_samples={i.num_samples}")


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] not in ("reduce", "run_imager", "run_sourcefind"):
        print(__doc__)
        return 2
    cmd = argv.pop(0)
    descs = {"reduce": "Slow Transients Pipeline run (imager + source finder) on the GPU",
             "run_imager": "Imager run on the GPU", "run_sourcefind": "Source finder run on the GPU"}
    p = _parser(cmd, descs[cmd], cmd != "run_imager", cmd != "run_sourcefind")
    a = p.parse_args(argv)
    log = print if a.log else (lambda *_: None)
    cfg = load_config(a.input_file_json)
    npz = np.load(a.input_file_npz)
    ctx = capi.Context(0)
    try:
        if cmd == "run_sourcefind":
            image = np.asfortranarray(np.asarray(npz["image"], dtype=np.float64))
            t0 = time.perf_counter()
            islands, labels, _ = ctx.source_find(image, *_sf_args(cfg, swapped=True))
            t_sf = time.perf_counter() - t0
            t_img = None
        else:
            set_image_sizes(cfg, log)
            img, beam, info, t_img = _run_imager(ctx, cfg, npz, a.diff, log)
            if cmd == "run_imager":
                if a.output_file_npz:
                    np.savez(a.output_file_npz, image=img, beam=beam)
                if not a.no_bench:
                    log(f"imager: {1e3 * t_img:.2f} ms")
                return 0
            t0 = time.perf_counter()
            islands, labels, _ = ctx.source_find(img, *_sf_args(cfg))
            t_sf = time.perf_counter() - t0
        if a.output_file_json:
            with open(a.output_file_json, "w") as f:
                json.dump(islands_json(islands, cfg["gaussian_fitting"]), f)
        if a.output_file_npz:
            np.savez(a.output_file_npz, label_map=labels)
        if not a.no_src:
            _log_islands(islands, log)
        else:
            log(f"Number of detected sources: {len(islands)}")
        if not a.no_bench:
            if t_img is not None:
                log(f"imager: {1e3 * t_img:.2f} ms")
            log(f"source find: {1e3 * t_sf:.2f} ms")
        return 0
    finally:
        ctx.close()


if __name__ == "__main__":
    sys.exit(main())
