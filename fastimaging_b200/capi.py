"""ctypes binding of the C ABI in include/stpgpu.h (libstpgpu.so).

This is the boundary every Python caller goes through; there is no CPU
fallback: if the library or a CUDA device is missing the calls raise.
"""
from __future__ import annotations

import ctypes
import os
import threading
from dataclasses import dataclass

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libstpgpu.so")

# enums (src/stp/types.h:32-89)
TopHat, Triangle, Sinc, Gaussian, GaussianSinc, PSWF = range(6)
ZEROMEDIAN, BINMEDIAN, BINAPPROX, NTHELEMENT = range(4)
LINEAR, CUBIC, COSINE = range(3)  # InterpType of the Hankel-transform W-kernels
FP64, FP32, FP32C = 0, 1, 2
C128, C64 = 0, 1
F64, F32 = 0, 1

STATUS = {0: "OK", 1: "INVALID_ARG", 2: "UNSUPPORTED", 3: "CUDA", 4: "CUFFT", 5: "OOM", 6: "CAPACITY", 7: "DEVICE",
          8: "TIMEOUT", 9: "NO_DEVICE"}


class StpGpuError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"stpgpu {STATUS.get(status, status)}: {msg}")
        self.status = status


class ImagerPars(ctypes.Structure):
    _fields_ = [("image_size", ctypes.c_int32), ("padded_image_size", ctypes.c_int32), ("cell_size", ctypes.c_double),
                ("padding_factor", ctypes.c_double), ("kernel_function", ctypes.c_int32),
                ("kernel_support", ctypes.c_int32), ("kernel_exact", ctypes.c_int32), ("oversampling", ctypes.c_int32),
                ("generate_beam", ctypes.c_int32), ("gridding_correction", ctypes.c_int32),
                ("analytic_gcf", ctypes.c_int32), ("r_fft", ctypes.c_int32)]


class WProjPars(ctypes.Structure):
    _fields_ = [("num_wplanes", ctypes.c_int32), ("max_wpconv_support", ctypes.c_int32),
                ("undersampling_opt", ctypes.c_int32), ("kernel_trunc_perc", ctypes.c_double),
                ("hankel_opt", ctypes.c_int32), ("hankel_proj_slice", ctypes.c_int32), ("interp_type", ctypes.c_int32),
                ("wplanes_median", ctypes.c_int32)]


class AProjPars(ctypes.Structure):
    _fields_ = [("num_timesteps", ctypes.c_int32), ("obs_dec", ctypes.c_double), ("obs_ra", ctypes.c_double),
                ("aproj_opt", ctypes.c_int32), ("aproj_mask_perc", ctypes.c_double), ("lha", ctypes.c_void_p),
                ("pbeam_coefs", ctypes.c_void_p), ("n_pbeam_coefs", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class ImagerInfo(ctypes.Structure):
    _fields_ = [("sample_grid_total", ctypes.c_double), ("n_good_vis", ctypes.c_int64),
                ("n_grid_items", ctypes.c_int64), ("padded_image_size", ctypes.c_int32),
                ("image_size", ctypes.c_int32), ("num_wplanes", ctypes.c_int32),
                ("max_plane_support", ctypes.c_int32), ("device_ms", ctypes.c_double),
                ("phase_ms", ctypes.c_double * 4), ("n_launches", ctypes.c_int32), ("flags", ctypes.c_int32)]


class Island(ctypes.Structure):
    _fields_ = [("label_idx", ctypes.c_int32), ("sign", ctypes.c_int32), ("extremum_val", ctypes.c_double),
                ("extremum_y_idx", ctypes.c_int32), ("extremum_x_idx", ctypes.c_int32),
                ("num_samples", ctypes.c_int32), ("bbox_top", ctypes.c_int32), ("bbox_bottom", ctypes.c_int32),
                ("bbox_left", ctypes.c_int32), ("bbox_right", ctypes.c_int32),
                ("moments_fit", ctypes.c_double * 6), ("leastsq_fit", ctypes.c_double * 6),
                ("fit_iterations", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class SfPars(ctypes.Structure):
    _fields_ = [("detection_n_sigma", ctypes.c_double), ("analysis_n_sigma", ctypes.c_double),
                ("rms_est", ctypes.c_double), ("find_negative_sources", ctypes.c_int32),
                ("sigma_clip_iters", ctypes.c_int32), ("median_method", ctypes.c_int32),
                ("gaussian_fitting", ctypes.c_int32), ("ccl_4connectivity", ctypes.c_int32),
                ("generate_labelmap", ctypes.c_int32), ("source_min_area", ctypes.c_int32),
                ("ccl_slice_cols", ctypes.c_int32)]


class SfInfo(ctypes.Structure):
    _fields_ = [("bg_level", ctypes.c_double), ("rms_est", ctypes.c_double), ("mean", ctypes.c_double),
                ("sigma", ctypes.c_double), ("n_labels_pos", ctypes.c_int32), ("n_labels_neg", ctypes.c_int32),
                ("n_valid_labels", ctypes.c_int32), ("n_islands", ctypes.c_int32), ("device_ms", ctypes.c_double)]


class Snapshot(ctypes.Structure):
    _fields_ = [("vis", ctypes.c_void_p), ("vis_dtype", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("weights", ctypes.c_void_p), ("uvw", ctypes.c_void_p), ("n_vis", ctypes.c_int64),
                ("pars", ImagerPars), ("wproj", WProjPars), ("image", ctypes.c_void_p)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("device_ms", ctypes.c_double), ("graph", ctypes.c_int32), ("gridder_launches", ctypes.c_int32),
                ("tuned_classes", ctypes.c_int32), ("n_launches", ctypes.c_int32)]


def imager_pars(image_size, cell_size, padding_factor=1.0, kernel_func=PSWF, kernel_support=3, kernel_exact=True,
                oversampling=8, generate_beam=False, gridding_correction=True, analytic_gcf=False, num_wplanes=0,
                wplanes_median=False, max_wpconv_support=0, undersampling_opt=1, kernel_trunc_perc=0.0,
                padded_image_size=0, hankel_opt=False, hankel_proj_slice=False, interp_type=LINEAR, **_):
    """(ImagerPars, WProjPars) from image_visibilities-style keywords."""
    ip = ImagerPars(int(image_size), int(padded_image_size), float(cell_size), float(padding_factor),
                    int(kernel_func), int(kernel_support), int(bool(kernel_exact)), int(oversampling),
                    int(bool(generate_beam)), int(bool(gridding_correction)), int(bool(analytic_gcf)), 0)
    wp = WProjPars(int(num_wplanes), int(max_wpconv_support), int(undersampling_opt), float(kernel_trunc_perc),
                   int(bool(hankel_opt)), int(bool(hankel_proj_slice)), int(interp_type), int(bool(wplanes_median)))
    return ip, wp


class ServerPars(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("slots", ctypes.c_int32), ("hbm_budget_bytes", ctypes.c_int64),
                ("precision", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class Request(ctypes.Structure):
    _fields_ = [("vis", ctypes.c_void_p), ("vis_dtype", ctypes.c_int32), ("out_dtype", ctypes.c_int32),
                ("weights", ctypes.c_void_p), ("uvw", ctypes.c_void_p), ("n_vis", ctypes.c_int64),
                ("pars", ImagerPars), ("wproj", WProjPars), ("image", ctypes.c_void_p),
                ("find_sources", ctypes.c_int32), ("island_capacity", ctypes.c_int32), ("sf", SfPars),
                ("label_map", ctypes.c_void_p), ("islands", ctypes.c_void_p)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("n_islands", ctypes.c_int32), ("est_bytes", ctypes.c_int64),
                ("submit_ms", ctypes.c_double), ("admit_ms", ctypes.c_double), ("done_ms", ctypes.c_double),
                ("imager", ImagerInfo), ("sf", SfInfo), ("error", ctypes.c_char * 160)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("in_flight", ctypes.c_int64), ("queued", ctypes.c_int64), ("peak_in_flight", ctypes.c_int64),
                ("peak_admitted_bytes", ctypes.c_int64), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("throughput_rps", ctypes.c_double)]


EXPORTED = ["stpgpu_abi_version", "stpgpu_create", "stpgpu_destroy", "stpgpu_last_error", "stpgpu_stream",
            "stpgpu_set_timing", "stpgpu_trim", "stpgpu_image_visibilities", "stpgpu_image_visibilities_ex", "stpgpu_convolve_to_grid",
            "stpgpu_source_find", "stpgpu_source_find_ex", "stpgpu_model_visibilities", "stpgpu_image_batch", "stpgpu_server_create",
            "stpgpu_server_destroy", "stpgpu_server_submit", "stpgpu_server_prepare", "stpgpu_server_wait", "stpgpu_server_stats_get",
            "stpgpu_label_noalloc"]
NOALLOC_MAX_PIXELS = 1024 * 1024

_lock = threading.Lock()
_lib = None


def load():
    """Load libstpgpu.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built; run `python -m fastimaging_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.stpgpu_abi_version.restype = ctypes.c_int
        L.stpgpu_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
        L.stpgpu_destroy.argtypes = [vp]
        L.stpgpu_last_error.argtypes = [vp]
        L.stpgpu_last_error.restype = ctypes.c_char_p
        L.stpgpu_stream.argtypes = [vp]
        L.stpgpu_stream.restype = vp
        L.stpgpu_trim.argtypes = [vp]
        L.stpgpu_set_timing.argtypes = [vp, ctypes.c_int]
        L.stpgpu_image_visibilities.argtypes = [vp, vp, vp, vp, ctypes.c_int64, ctypes.POINTER(ImagerPars),
                                                ctypes.POINTER(WProjPars), ctypes.POINTER(AProjPars), vp, vp,
                                                ctypes.POINTER(ImagerInfo)]
        L.stpgpu_image_visibilities_ex.argtypes = [vp, vp, ctypes.c_int, vp, vp, ctypes.c_int64,
                                                   ctypes.POINTER(ImagerPars), ctypes.POINTER(WProjPars),
                                                   ctypes.POINTER(AProjPars), ctypes.c_int, vp, vp, ctypes.c_int,
                                                   ctypes.c_int, ctypes.POINTER(ImagerInfo)]
        L.stpgpu_convolve_to_grid.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, vp, vp, vp,
                                              ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.POINTER(WProjPars), vp, ctypes.c_double,
                                              ctypes.c_int, vp, vp, ctypes.POINTER(ctypes.c_double)]
        L.stpgpu_source_find.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(SfPars), vp, vp,
                                         ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(SfInfo)]
        L.stpgpu_source_find_ex.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.POINTER(SfPars), vp, ctypes.c_int, vp, ctypes.c_int32,
                                            ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(SfInfo)]
        L.stpgpu_model_visibilities.argtypes = [vp, vp, ctypes.c_int32, vp, ctypes.c_int64, vp, vp, ctypes.c_int]
        L.stpgpu_image_batch.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp,
                                         ctypes.POINTER(BatchInfo)]
        L.stpgpu_server_create.argtypes = [ctypes.POINTER(ServerPars), ctypes.POINTER(vp)]
        L.stpgpu_server_destroy.argtypes = [vp]
        L.stpgpu_server_submit.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_int64)]
        L.stpgpu_server_prepare.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(Result)]
        L.stpgpu_server_wait.argtypes = [vp, ctypes.c_int64, ctypes.c_double, ctypes.POINTER(Result)]
        L.stpgpu_server_stats_get.argtypes = [vp, ctypes.POINTER(ServerStats)]
        L.stpgpu_label_noalloc.argtypes = [ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                           ctypes.c_char_p, ctypes.c_size_t]
        _lib = L
        return L


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):  # torch tensor
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)


class Context:
    """One device + stream + cached buffers/plans (stpgpu_context)."""

    def __init__(self, device: int = 0):
        self.L = load()
        self.h = ctypes.c_void_p()
        st = self.L.stpgpu_create(int(device), ctypes.byref(self.h))
        if st != 0:
            raise StpGpuError(st, "stpgpu_create failed")

    def close(self):
        if self.h:
            self.L.stpgpu_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            raise StpGpuError(st, self.L.stpgpu_last_error(self.h).decode())

    def set_timing(self, enable=True):
        self._check(self.L.stpgpu_set_timing(self.h, int(bool(enable))))

    @property
    def stream(self):
        return self.L.stpgpu_stream(self.h)

    # ------------------------------------------------------------ imager
    def image_visibilities(self, vis, weights, uvw, image_size, cell_size, padding_factor=1.0, kernel_func=PSWF,
                           kernel_support=3, kernel_exact=True, oversampling=8, generate_beam=False,
                           gridding_correction=True, analytic_gcf=False, num_wplanes=0, wplanes_median=False,
                           max_wpconv_support=0, undersampling_opt=1, kernel_trunc_perc=0.0, hankel_opt=False,
                           hankel_proj_slice=False, interp_type=LINEAR, aproj_numtimesteps=0, obs_dec=0.0,
                           obs_ra=0.0, aproj_opt=False, aproj_mask_perc=0.0, lha=None, pbeam_coefs=None,
                           precision=FP64, out_dtype=F64, padded_image_size=0, device_ptrs=False, image_out=None,
                           beam_out=None):
        """stp::image_visibilities semantics (sizes used as given).

        Host mode: numpy inputs (vis complex128/complex64 (n,), weights (n,),
        uvw (n, 3)); returns (image, beam, info) as F-ordered arrays.
        Device mode: torch CUDA tensors; uvw must be (3, n) contiguous (the
        column-major n x 3 layout); outputs written into image_out/beam_out.
        A-projection (aproj_numtimesteps > 0): lha (n,) local hour angles in
        hours (a CUDA tensor in device mode), pbeam_coefs the beam's
        spherical-harmonic coefficients (host).
        """
        ip = ImagerPars(int(image_size), int(padded_image_size), float(cell_size), float(padding_factor),
                        int(kernel_func), int(kernel_support), int(bool(kernel_exact)), int(oversampling),
                        int(bool(generate_beam)), int(bool(gridding_correction)), int(bool(analytic_gcf)), 0)
        wp = WProjPars(int(num_wplanes), int(max_wpconv_support), int(undersampling_opt), float(kernel_trunc_perc),
                       int(bool(hankel_opt)), int(bool(hankel_proj_slice)), int(interp_type),
                       int(bool(wplanes_median)))
        coefs = np.ascontiguousarray(np.asarray(pbeam_coefs if pbeam_coefs is not None else [], dtype=np.float64))
        if lha is not None and not hasattr(lha, "data_ptr"):
            lha = np.ascontiguousarray(np.asarray(lha, dtype=np.float64).reshape(-1))
        ap = AProjPars(int(aproj_numtimesteps), float(obs_dec), float(obs_ra), int(bool(aproj_opt)),
                       float(aproj_mask_perc), _ptr(lha) if lha is not None else None,
                       _ptr(coefs) if coefs.size else None, int(coefs.size), 0)
        info = ImagerInfo()
        if device_ptrs:
            n = int(weights.numel())
            vdt = C64 if str(vis.dtype).endswith("complex64") else C128
            self._check(self.L.stpgpu_image_visibilities_ex(self.h, _ptr(vis), vdt, _ptr(weights), _ptr(uvw), n,
                                                            ctypes.byref(ip), ctypes.byref(wp), ctypes.byref(ap),
                                                            int(precision), _ptr(image_out), _ptr(beam_out),
                                                            int(out_dtype), 1, ctypes.byref(info)))
            return image_out, beam_out, info
        vis = np.ascontiguousarray(vis)
        if vis.dtype not in (np.complex128, np.complex64):
            vis = vis.astype(np.complex128)
        vdt = C64 if vis.dtype == np.complex64 else C128
        n = vis.size
        w = np.ascontiguousarray(weights, dtype=np.float64).reshape(-1)
        uvwF = np.asfortranarray(np.asarray(uvw, dtype=np.float64).reshape(n, 3))
        odt = np.float32 if out_dtype == F32 else np.float64
        img = np.empty((image_size, image_size), dtype=odt, order="F")
        beam = np.empty((image_size, image_size), dtype=odt, order="F") if generate_beam else None
        self._check(self.L.stpgpu_image_visibilities_ex(self.h, _ptr(vis), vdt, _ptr(w), _ptr(uvwF), n,
                                                        ctypes.byref(ip), ctypes.byref(wp), ctypes.byref(ap),
                                                        int(precision), _ptr(img), _ptr(beam), int(out_dtype), 0,
                                                        ctypes.byref(info)))
        if info.image_size == 0:
            return np.zeros((0, 0)), np.zeros((0, 0)), info
        return img, (beam if beam is not None else np.zeros((0, 0))), info

    def model_visibilities(self, skymodel, uvw, vis=None):
        """stp::generate_visibilities_from_local_skymodel on the GPU (host arrays): skymodel (n_src, 3) rows
        (l, m, flux), uvw (n, 3).  With vis: returns vis - model (residual visibilities)."""
        sky = np.asfortranarray(np.asarray(skymodel, dtype=np.float64).reshape(-1, 3))
        uvwF = np.asfortranarray(np.asarray(uvw, dtype=np.float64).reshape(-1, 3))
        n = uvwF.shape[0]
        out = np.empty(n, dtype=np.complex128)
        vin = None if vis is None else np.ascontiguousarray(vis, dtype=np.complex128).reshape(-1)
        self._check(self.L.stpgpu_model_visibilities(self.h, _ptr(sky), sky.shape[0], _ptr(uvwF), n, _ptr(vin),
                                                     _ptr(out), 0))
        return out

    def image_batch(self, snapshots, precision=FP32C, out_dtype=F32, device_ptrs=True):
        """stpgpu_image_batch over a list of dicts, one per snapshot:
        vis, weights, uvw, image (torch CUDA tensors when device_ptrs, uvw
        (3, n) contiguous; numpy arrays otherwise, uvw (n, 3)), plus the
        image_visibilities keywords (image_size, cell_size, kernel_func, ...).
        Returns (images, infos, batch_info); images are the given outputs
        (device) or new F-ordered arrays (host)."""
        n = len(snapshots)
        arr = (Snapshot * n)()
        keep, outs = [], []
        odt = np.float32 if out_dtype == F32 else np.float64
        for i, sd in enumerate(snapshots):
            ip, wp = imager_pars(**{k: v for k, v in sd.items() if k not in ("vis", "weights", "uvw", "image")})
            if device_ptrs:
                vis, w, uvw, img = sd["vis"], sd["weights"], sd["uvw"], sd["image"]
                nv = int(w.numel())
                vdt = C64 if str(vis.dtype).endswith("complex64") else C128
            else:
                vis = np.ascontiguousarray(sd["vis"])
                if vis.dtype not in (np.complex128, np.complex64):
                    vis = vis.astype(np.complex128)
                vdt = C64 if vis.dtype == np.complex64 else C128
                nv = vis.size
                w = np.ascontiguousarray(sd["weights"], dtype=np.float64).reshape(-1)
                uvw = np.asfortranarray(np.asarray(sd["uvw"], dtype=np.float64).reshape(nv, 3))
                img = sd.get("image")
                if img is None:
                    img = np.empty((int(sd["image_size"]), int(sd["image_size"])), dtype=odt, order="F")
            keep += [vis, w, uvw, img]
            outs.append(img)
            arr[i] = Snapshot(_ptr(vis), vdt, 0, _ptr(w), _ptr(uvw), nv, ip, wp, _ptr(img))
        infos = (ImagerInfo * n)()
        bi = BatchInfo()
        self._check(self.L.stpgpu_image_batch(self.h, arr, n, int(precision), int(out_dtype), int(bool(device_ptrs)),
                                               infos, ctypes.byref(bi)))
        return outs, list(infos), bi

    def convolve_to_grid(self, kernel_func, kernel_trunc, support, image_size, uv, vis, weights, kernel_exact=True,
                         oversampling=1, shift_uv=True, halfplane=True, generate_beam=True, num_wplanes=0,
                         max_wpconv_support=0, undersampling_opt=1, kernel_trunc_perc=0.0, wplanes_median=False,
                         w=None, cell_size=0.0, analytic_gcf=True):
        vis = np.ascontiguousarray(vis, dtype=np.complex128).reshape(-1)
        n = vis.size
        uvF = np.asfortranarray(np.asarray(uv, dtype=np.float64).reshape(n, 2))
        wts = np.ascontiguousarray(weights, dtype=np.float64).reshape(-1)
        ww = None if w is None else np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
        rows = image_size // 2 + 1 if halfplane else image_size
        vg = np.empty((rows, image_size), dtype=np.complex128, order="F")
        sg = np.empty((rows, image_size), dtype=np.complex128, order="F") if generate_beam else None
        wp = WProjPars(int(num_wplanes), int(max_wpconv_support), int(undersampling_opt), float(kernel_trunc_perc), 0,
                       0, 0, int(bool(wplanes_median)))
        tot = ctypes.c_double()
        self._check(self.L.stpgpu_convolve_to_grid(self.h, int(kernel_func), float(kernel_trunc), int(support),
                                                   int(image_size), _ptr(uvF), _ptr(vis), _ptr(wts), n,
                                                   int(bool(kernel_exact)), int(oversampling), int(bool(shift_uv)),
                                                   int(bool(halfplane)), int(bool(generate_beam)), ctypes.byref(wp),
                                                   _ptr(ww), float(cell_size), int(bool(analytic_gcf)), _ptr(vg),
                                                   _ptr(sg), ctypes.byref(tot)))
        return vg, (sg if sg is not None else np.zeros((0, 0), np.complex128)), tot.value

    # ------------------------------------------------------------ source finder
    def source_find(self, image, detection_n_sigma, analysis_n_sigma, rms_est=0.0, find_negative_sources=True,
                    sigma_clip_iters=5, median_method=BINAPPROX, gaussian_fitting=False, ccl_4connectivity=False,
                    generate_labelmap=True, source_min_area=5, ccl_slice_cols=0, want_labels=True,
                    device_ptrs=False, rows=None, cols=None, label_out=None, capacity=4096):
        p = SfPars(float(detection_n_sigma), float(analysis_n_sigma), float(rms_est), int(bool(find_negative_sources)),
                   int(sigma_clip_iters), int(median_method), int(bool(gaussian_fitting)),
                   int(bool(ccl_4connectivity)), int(bool(generate_labelmap)), int(source_min_area),
                   int(ccl_slice_cols))
        info = SfInfo()
        nis = ctypes.c_int32()
        if device_ptrs:
            dt = F32 if str(image.dtype).endswith("float32") else F64
            r, c = int(rows), int(cols)
            labels = label_out
        else:
            img = np.asfortranarray(image)
            if img.dtype not in (np.float64, np.float32):
                img = img.astype(np.float64)
            dt = F32 if img.dtype == np.float32 else F64
            r, c = img.shape
            labels = np.empty((r, c), dtype=np.int32, order="F") if want_labels else None
        while True:
            buf = (Island * max(1, capacity))()
            st = self.L.stpgpu_source_find_ex(self.h, _ptr(image) if device_ptrs else _ptr(img), dt, r, c,
                                              ctypes.byref(p), _ptr(labels), int(bool(device_ptrs)), buf,
                                              int(capacity), ctypes.byref(nis), ctypes.byref(info))
            if st == 6:
                capacity = nis.value
                continue
            self._check(st)
            break
        islands = [buf[i] for i in range(nis.value)]
        return islands, labels, info


def label_noalloc(device, stream, image_ptr, image_dtype, rows, cols, thresh_pos, thresh_neg, find_negative_sources=True,
                  ccl_4connectivity=False, ccl_slice_cols=0, label_ptr=None):
    """Allocation-free labelling (stpgpu_label_noalloc): device image in, device
    int32 label map out (both raw device addresses).  Returns (n_pos, n_neg)."""
    L = load()
    npos, nneg = ctypes.c_int32(), ctypes.c_int32()
    msg = ctypes.create_string_buffer(256)
    st = L.stpgpu_label_noalloc(int(device), ctypes.c_void_p(stream or 0), ctypes.c_void_p(image_ptr),
                                int(image_dtype), int(rows), int(cols), float(thresh_pos), float(thresh_neg),
                                int(bool(find_negative_sources)), int(bool(ccl_4connectivity)), int(ccl_slice_cols),
                                ctypes.c_void_p(label_ptr), ctypes.byref(npos), ctypes.byref(nneg), msg, len(msg))
    if st != 0:
        raise StpGpuError(st, msg.value.decode(errors="replace"))
    return npos.value, nneg.value


class Server:
    """Request loop over one GPU (stpgpu_server_*): submit imaging (+ source
    finding) requests from host buffers, wait for their results."""

    def __init__(self, device=0, slots=4, hbm_budget_bytes=32 << 30, precision=FP32C):
        self.L = load()
        self.h = ctypes.c_void_p()
        st = self.L.stpgpu_server_create(ctypes.byref(ServerPars(int(device), int(slots), int(hbm_budget_bytes),
                                                                    int(precision), 0)), ctypes.byref(self.h))
        if st != 0:
            raise StpGpuError(st, "server create")
        self._keep = {}

    def submit(self, vis, weights, uvw, find_sources=False, out_dtype=F32, sf=None, want_labels=False,
               island_capacity=4096, want_image=True, **imager_kw):
        """imager_kw: image_size, cell_size and the image_visibilities keywords.
        sf: dict of source_find keywords (detection_n_sigma, analysis_n_sigma, ...).
        Inputs: numpy arrays (uvw (n, 3)), or page-locked torch CPU tensors
        (vis complex (n,), weights (n,), uvw (3, n) contiguous).  Returns a ticket."""
        req, keep = self._request(vis, weights, uvw, find_sources, out_dtype, sf, want_labels, island_capacity,
                                  want_image, imager_kw)
        t = ctypes.c_int64()
        st = self.L.stpgpu_server_submit(self.h, ctypes.byref(req), ctypes.byref(t))
        if st != 0:
            raise StpGpuError(st, "submit")
        self._keep[t.value] = keep
        return t.value

    def prepare(self, vis, weights, uvw, find_sources=False, out_dtype=F32, sf=None, want_labels=False,
                island_capacity=4096, want_image=True, **imager_kw):
        """Run a request (the arguments of submit) once on every slot while
        admission is held, so that requests of its size class admitted later
        allocate, plan and tune nothing.  -> Result of the last slot."""
        req, _keep = self._request(vis, weights, uvw, find_sources, out_dtype, sf, want_labels, island_capacity,
                                    want_image, imager_kw)
        res = Result()
        st = self.L.stpgpu_server_prepare(self.h, ctypes.byref(req), ctypes.byref(res))
        if st != 0:
            raise StpGpuError(st, res.error.decode(errors="replace"))
        return res

    @staticmethod
    def _request(vis, weights, uvw, find_sources, out_dtype, sf, want_labels, island_capacity, want_image,
                 imager_kw):
        if hasattr(vis, "data_ptr"):
            n = int(weights.numel())
            vdt = C64 if str(vis.dtype).endswith("complex64") else C128
            w, uvwF = weights, uvw
        else:
            vis = np.ascontiguousarray(vis)
            if vis.dtype not in (np.complex128, np.complex64):
                vis = vis.astype(np.complex128)
            vdt = C64 if vis.dtype == np.complex64 else C128
            n = vis.size
            w = np.ascontiguousarray(weights, dtype=np.float64).reshape(-1)
            uvwF = np.asfortranarray(np.asarray(uvw, dtype=np.float64).reshape(n, 3))
        ip, wp = imager_pars(**imager_kw)
        size = int(imager_kw["image_size"])
        img = (np.empty((size, size), dtype=np.float32 if out_dtype == F32 else np.float64, order="F")
               if (want_image or not find_sources) else None)
        sfd = dict(detection_n_sigma=5.0, analysis_n_sigma=3.0, rms_est=0.0, find_negative_sources=True,
                   sigma_clip_iters=5, median_method=BINAPPROX, gaussian_fitting=False, ccl_4connectivity=False,
                   generate_labelmap=True, source_min_area=5, ccl_slice_cols=0)
        sfd.update(sf or {})
        sp = SfPars(float(sfd["detection_n_sigma"]), float(sfd["analysis_n_sigma"]), float(sfd["rms_est"]),
                    int(bool(sfd["find_negative_sources"])), int(sfd["sigma_clip_iters"]), int(sfd["median_method"]),
                    int(bool(sfd["gaussian_fitting"])), int(bool(sfd["ccl_4connectivity"])),
                    int(bool(sfd["generate_labelmap"])), int(sfd["source_min_area"]), int(sfd["ccl_slice_cols"]))
        labels = np.empty((size, size), dtype=np.int32, order="F") if (find_sources and want_labels) else None
        isl = (Island * max(1, int(island_capacity)))()
        req = Request(_ptr(vis), vdt, int(out_dtype), _ptr(w), _ptr(uvwF), n,
                      ip, wp, _ptr(img), int(bool(find_sources)), int(island_capacity), sp, _ptr(labels),
                      ctypes.cast(isl, ctypes.c_void_p))
        return req, (vis, w, uvwF, img, labels, isl, req)

    def wait(self, ticket, timeout_s=-1.0):
        """-> (image, label_map or None, [Island], Result); raises on failure."""
        res = Result()
        st = self.L.stpgpu_server_wait(self.h, int(ticket), float(timeout_s), ctypes.byref(res))
        if st == 8:
            raise StpGpuError(st, "not done")
        vis, w, uvwF, img, labels, isl, req = self._keep.pop(int(ticket))
        if st != 0:
            raise StpGpuError(st, res.error.decode(errors="replace"))
        islands = [isl[i] for i in range(min(res.n_islands, len(isl)))] if req.find_sources else []
        if res.imager.image_size == 0 and img is not None:
            img = np.zeros((0, 0))
        return img, labels, islands, res

    def stats(self):
        s = ServerStats()
        self.L.stpgpu_server_stats_get(self.h, ctypes.byref(s))
        return s

    def close(self):
        if self.h:
            self.L.stpgpu_server_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
