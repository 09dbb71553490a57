"""GPU parity at the sizes of the benchmark workloads, through the C ABI,
against the CPU oracle (FP64).

* plain imager, 2048^2, 100k visibilities, Gaussian-Sinc S=3 os=8: FP64 within
  1e-10 of the oracle's peak, compensated FP32 within 1e-5;
* W-projection imager, 4096^2, 1M visibilities, |w| <= 2000, 32 planes,
  W-kernel support <= 16: FP64 within 1e-10, compensated FP32 within 1e-5;
* precision study, 8192^2, 4M complex64 visibilities concentrated in uv, PSWF
  S=4 os=16 with the analytic correction: compensated FP32 within 1e-5 of the
  FP64 oracle (max-abs/peak; RMS reported), FP64 within 1e-10;
* source finding on images of the serving workload (2048^2, 4096^2, 8192^2;
  50 point and 5 extended sources): label maps bit-exact to the oracle's,
  island tuples equal (extremum bit-exact, moments within 1e-9 relative).

Tolerances: 1e-10 peak-relative for FP64 and 1e-5 for FP32 forms, the
reference's fptolerance (src/stp/types.h:23-27)."""
import os

import numpy as np
import pytest

from fastimaging_b200 import capi
from fastimaging_b200 import synthetic as syn
from oracle import stp_oracle as orc

pytestmark = pytest.mark.gpu
TOL64 = 1e-10
TOL32 = 1e-5
THREADS = max(1, len(os.sched_getaffinity(0)))


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def errors(img, ref):
    d = np.abs(np.asarray(img, dtype=np.float64) - ref)
    peak = float(np.max(np.abs(ref)))
    return float(d.max()) / peak, float(np.sqrt(np.mean(d * d)) / np.sqrt(np.mean(ref * ref)))


def _oracle_image(s, kw):
    img, _ = orc.image_visibilities(s.vis.astype(np.complex128), s.weights, s.uvw, s.image_size, s.cell_size,
                                    threads=THREADS, **kw)
    return img


@pytest.fixture(scope="module")
def config1():
    s = syn.config1()
    return s, _oracle_image(s, syn.CONFIG1_IMAGER)


@pytest.fixture(scope="module")
def config2():
    s = syn.config2()
    return s, _oracle_image(s, syn.CONFIG2_IMAGER)


@pytest.fixture(scope="module")
def config3():
    s = syn.config3()
    return s, _oracle_image(s, syn.CONFIG3_IMAGER)


@pytest.mark.parametrize("precision,tol", [(capi.FP64, TOL64), (capi.FP32C, TOL32)])
def test_config1_plain_imager(ctx, config1, precision, tol):
    s, ref = config1
    img, _, info = ctx.image_visibilities(s.vis, s.weights, s.uvw, s.image_size, s.cell_size, precision=precision,
                                          **syn.CONFIG1_IMAGER)
    peak, rms = errors(img, ref)
    print(f"config1 precision {precision}: max-abs/peak {peak:.3e} rms {rms:.3e}")
    assert info.image_size == 2048
    assert peak <= tol


@pytest.mark.parametrize("precision,tol", [(capi.FP64, TOL64), (capi.FP32C, TOL32)])
def test_config2_wproj_imager(ctx, config2, precision, tol):
    s, ref = config2
    img, _, info = ctx.image_visibilities(s.vis, s.weights, s.uvw, s.image_size, s.cell_size, precision=precision,
                                          **syn.CONFIG2_IMAGER)
    peak, rms = errors(img, ref)
    print(f"config2 precision {precision}: max-abs/peak {peak:.3e} rms {rms:.3e}, "
          f"max plane support {info.max_plane_support}")
    assert info.num_wplanes == 32
    assert peak <= tol
    # Gaussian-Sinc with the DFT correction: 1/gcf_min^2 = 890, the FP32 c2r suffices
    assert precision != capi.FP32C or info.flags & 1 == 0


@pytest.mark.parametrize("precision,tol", [(capi.FP32C, TOL32), (capi.FP64, TOL64)])
def test_config3_precision(ctx, config3, precision, tol):
    s, ref = config3
    img, _, info = ctx.image_visibilities(s.vis, s.weights, s.uvw, s.image_size, s.cell_size, precision=precision,
                                          out_dtype=capi.F32 if precision != capi.FP64 else capi.F64,
                                          **syn.CONFIG3_IMAGER)
    peak, rms = errors(img, ref)
    print(f"config3 precision {precision}: max-abs/peak {peak:.3e} rms {rms:.3e} flags {info.flags}")
    assert peak <= tol
    if precision == capi.FP32C:
        # analytic PSWF correction: 1/gcf(1)^2 = 6.2e4 > 4096, double-precision c2r
        assert info.flags & 1


def _serving_image(size, seed):
    """An image of the serving workload: a snapshot with 50 point sources and 5
    extended Gaussians (sigma 2-6 px), W-projection with 16 planes, imaged by
    the oracle (FP64)."""
    s = syn.make_snapshot(seed, 300_000, size, 1.0, n_src=50, flux=(0.5, 10.0), noise_sigma=0.05,
                          w_range=(-500.0, 500.0), n_extended=5)
    kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, gridding_correction=True,
              analytic_gcf=False, num_wplanes=16, max_wpconv_support=16, undersampling_opt=1, kernel_trunc_perc=1.0)
    return _oracle_image(s, kw)


def _compare_islands(isl, ref, rtol=1e-9):
    assert len(isl) == len(ref.islands)
    for a, b in zip(isl, ref.islands):
        sign, val, x, y, ns, mom, _, _ = b
        assert (a.sign, a.extremum_x_idx, a.extremum_y_idx, a.num_samples) == (sign, x, y, ns)
        assert a.extremum_val == val
        got = np.array(a.moments_fit[:])
        want = np.array([mom.amplitude, mom.x_centre, mom.y_centre, mom.semimajor, mom.semiminor, mom.theta])
        ok = np.isclose(got, want, rtol=rtol, atol=1e-9) | (np.isnan(got) & np.isnan(want))
        assert ok.all(), (got, want)


@pytest.mark.parametrize("size,seed", [(2048, 51), (4096, 52), (8192, 53)])
def test_serving_sizes_source_find(ctx, size, seed):
    """5-sigma detection, 3-sigma analysis, BINAPPROX, 8-connectivity, negative
    sources, minimum area 5: labels bit-exact, islands equal."""
    img = _serving_image(size, seed)
    ref = orc.source_find(img, 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True, 5)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, False, False, True, 5)
    print(f"serving {size}^2: {len(ref.islands)} islands, {ref.n_pos}+{ref.n_neg} labels")
    assert abs(info.rms_est - ref.rms_est) <= 1e-10 * abs(ref.rms_est)
    assert info.n_labels_pos == ref.n_pos and info.n_labels_neg == ref.n_neg
    assert np.array_equal(lab, ref.label_map)
    _compare_islands(isl, ref)
    assert len(isl) >= 20


def test_serving_size_source_find_float32(ctx):
    """The bench's single-precision source-finder input (4096^2): the oracle
    labels the same single-precision pixel values, promoted."""
    img = _serving_image(4096, 54).astype(np.float32)
    ref = orc.source_find(img.astype(np.float64), 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True, 5)
    isl, lab, info = ctx.source_find(img, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, False, False, True, 5)
    assert np.array_equal(lab, ref.label_map)
    _compare_islands(isl, ref)
