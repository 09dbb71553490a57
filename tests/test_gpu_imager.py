"""GPU parity of the imager through the C ABI, against the CPU oracle.

Tolerances: FP64 path within 1e-10 peak-relative error of the oracle (the
reference's fptolerance for double builds, src/stp/types.h:26); FP32 and
compensated FP32 within 1e-5 peak-relative of the FP64 oracle.
"""
import numpy as np
import pytest

from fastimaging_b200 import capi
from fastimaging_b200.synthetic import make_snapshot
from oracle import stp_oracle as orc

pytestmark = pytest.mark.gpu
TOL64 = 1e-10
TOL32 = 1e-5


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def peak_rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


KF = {"TopHat": 0, "Triangle": 1, "Sinc": 2, "Gaussian": 3, "GaussianSinc": 4, "PSWF": 5}


@pytest.mark.parametrize("name", ["SmallPillbox", "MultiPixelPillbox", "MultipleComplexVis", "NearbyComplexVis",
                                  "SinglePixelOverlapPillbox"])
def test_gridder_reference_pins(ctx, pins, name):
    c = next(x for x in pins["gridder"] if x["name"] == name)
    vis = np.array([complex(a, b) for a, b in c["vis"]])
    vg, sg, tot = ctx.convolve_to_grid(KF[c["kernel"]], c["hbw"], c["support"], c["image_size"], np.array(c["uv"]),
                                       vis, np.array(c["weights"]), c["kernel_exact"], c["oversampling"],
                                       c["shift_uv"], c["halfplane"], True)
    assert np.max(np.abs(vg.real - np.array(c["expect_vis_grid_real"]))) < TOL64
    if c["expect_sampling_real"] is not None:
        assert np.max(np.abs(sg.real - np.array(c["expect_sampling_real"]))) < TOL64


def test_gridder_halfplane_shifted_pin(ctx, pins):
    c = next(x for x in pins["gridder"] if x["name"] == "HalfPlaneShiftedGridding")
    vis = np.ones(2, complex)
    for exact in (False, True):
        vg, sg, tot = ctx.convolve_to_grid(0, c["hbw"], c["support"], 8, np.array(c["uv"]), vis, np.ones(2), exact,
                                           c["oversampling"], True, True, True)
        assert np.max(np.abs(np.roll(vg, 4, axis=1).real - np.array(c["expect_vis_grid_real"]))) < TOL64


@pytest.mark.parametrize("mode", ["oversampled", "exact", "fullplane_noshift", "exact_fullplane"])
@pytest.mark.parametrize("kf", [4, 5, 1])
def test_gridder_random_vs_oracle(ctx, mode, kf):
    rng = np.random.default_rng(11 + kf)
    N, n, S = 64, 300, 3
    uv = rng.uniform(-N / 2 + 1, N / 2 - 1, size=(n, 2))
    uv[:20, 1] = rng.uniform(-S - 1.2, S + 1.2, size=20)  # near v = 0: mirrored duplicates
    vis = rng.normal(size=n) + 1j * rng.normal(size=n)
    w = rng.uniform(0.5, 2.0, size=n)
    exact = mode.startswith("exact")
    half = mode in ("oversampled", "exact")
    shift = half
    g, s, t = ctx.convolve_to_grid(kf, float(S), S, N, uv, vis, w, exact, 8, shift, half, True)
    r = orc.convolve_to_grid(kf, S, N, uv, vis, w, exact, 8, shift, half, True)
    assert abs(t - r.sample_grid_total) <= 1e-12 * abs(r.sample_grid_total)
    assert peak_rel(g, r.vis_grid) < 1e-12
    assert peak_rel(s, r.sampling_grid) < 1e-12


def _imager_case(seed, N, n, **kw):
    return make_snapshot(seed, n, N, 2.0, n_src=4, flux=(1.0, 5.0), noise_sigma=0.05, **kw)


@pytest.mark.parametrize("kf,exact,analytic", [(4, False, False), (5, False, True), (5, False, False),
                                                (4, True, False), (2, False, False), (3, False, True)])
def test_imager_fp64_vs_oracle(ctx, kf, exact, analytic):
    s = _imager_case(5 + kf, 256, 3000)
    kw = dict(kernel_func=kf, kernel_support=3, kernel_exact=exact, oversampling=8, gridding_correction=True,
              analytic_gcf=analytic, generate_beam=True)
    img, beam, info = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
    ri, rb = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, oversampling=8, **{
        k: v for k, v in kw.items() if k != "oversampling"})
    assert info.image_size == 256
    assert peak_rel(img, ri) < TOL64
    assert peak_rel(beam, rb) < TOL64


def test_imager_padding_crop(ctx):
    s = _imager_case(21, 192, 2500)
    kw = dict(kernel_func=5, kernel_support=3, kernel_exact=False, oversampling=8, analytic_gcf=True)
    img, _, info = ctx.image_visibilities(s.vis, s.weights, s.uvw, 192, s.cell_size, padding_factor=1.5, **kw)
    ri, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 192, s.cell_size, padding_factor=1.5, **kw)
    assert info.padded_image_size == 288
    assert peak_rel(img, ri) < TOL64


@pytest.mark.parametrize("median", [False, True])
def test_imager_wproj_fp64_vs_oracle(ctx, median):
    s = _imager_case(31, 256, 6000, w_range=(-800.0, 800.0))
    kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, analytic_gcf=False,
              num_wplanes=6, max_wpconv_support=8, undersampling_opt=1, kernel_trunc_perc=1.0,
              wplanes_median=median)
    img, _, info = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
    ri, _, g = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, return_grid=True, **kw)
    assert info.max_plane_support == max(g.plane_supports)
    assert peak_rel(img, ri) < TOL64


@pytest.mark.parametrize("case", ["out_of_grid", "planes_beyond_items", "many_planes", "outlier_then_again"])
def test_imager_wproj_planes_without_sort(case):
    """The W-planes found without sorting |w| (k_wsel_*) where every visibility is in the grid, and the
    sorting path it falls back to otherwise: visibilities outside the grid (the reference's begin rule then
    counts them), more planes than visibilities (empty planes), 300 planes over 3000 visibilities, and a
    size class whose previous call fell back.  FP64 image within 1e-10 of the oracle, plane supports equal."""
    fresh = capi.Context(0)
    try:
        n, planes = {"out_of_grid": (6000, 6), "planes_beyond_items": (40, 64), "many_planes": (3000, 300),
                     "outlier_then_again": (6000, 8)}[case]
        s = _imager_case(57, 256, n, w_range=(-700.0, 700.0))
        uvw = np.array(s.uvw, order="F")
        if case == "out_of_grid":
            uvw[::97, 0] += 1.0e7  # about 1 % outside the grid
        kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, analytic_gcf=False,
                  num_wplanes=planes, max_wpconv_support=8, undersampling_opt=1, kernel_trunc_perc=1.0)
        calls = [uvw]
        if case == "outlier_then_again":
            bad = uvw.copy()
            bad[::50, 0] += 1.0e7
            calls = [uvw, bad, bad, uvw]
        for u in calls:
            img, _, info = fresh.image_visibilities(s.vis, s.weights, u, 256, s.cell_size, **kw)
            ri, _, g = orc.image_visibilities(s.vis, s.weights, u, 256, s.cell_size, return_grid=True, **kw)
            assert info.max_plane_support == max(g.plane_supports)
            assert peak_rel(img, ri) < TOL64
    finally:
        fresh.close()


def test_imager_wproj_untruncated(ctx):
    s = _imager_case(33, 128, 3000, w_range=(-3000.0, 3000.0))
    kw = dict(kernel_func=5, kernel_support=3, kernel_exact=False, oversampling=4, analytic_gcf=True,
              num_wplanes=4, max_wpconv_support=5, kernel_trunc_perc=0.0)
    img, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 128, s.cell_size, **kw)
    ri, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 128, s.cell_size, **kw)
    assert peak_rel(img, ri) < TOL64


@pytest.mark.parametrize("trunc", [0.0, 1.0])
def test_imager_wproj_large_support(ctx, trunc):
    """W-kernel supports above 32 (the reference's W-projection configurations use up to 127): tables and tile
    lists sized from the measured supports."""
    s = _imager_case(37, 256, 1500, w_range=(-4000.0, 4000.0))
    kw = dict(kernel_func=5, kernel_support=3, kernel_exact=False, oversampling=4, analytic_gcf=True,
              num_wplanes=3, max_wpconv_support=40, kernel_trunc_perc=trunc)
    img, _, info = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
    ri, _, g = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, return_grid=True, **kw)
    assert info.max_plane_support == max(g.plane_supports)
    if trunc == 0.0:
        assert info.max_plane_support == 40
    assert peak_rel(img, ri) < TOL64


@pytest.mark.parametrize("proj_slice,interp", [(False, capi.LINEAR), (False, capi.CUBIC), (True, capi.LINEAR),
                                               (True, capi.CUBIC), (False, capi.COSINE)])
def test_imager_hankel_fp64_vs_oracle(ctx, proj_slice, interp):
    """Hankel-transform W-kernels (hankel_opt): discrete Hankel transform or projection slice, linear or
    cubic radial interpolation, truncated at 1 %."""
    s = _imager_case(35, 256, 5000, w_range=(-1500.0, 1500.0))
    kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, analytic_gcf=False,
              num_wplanes=5, max_wpconv_support=8, undersampling_opt=1, kernel_trunc_perc=1.0, hankel_opt=True,
              hankel_proj_slice=proj_slice, interp_type=interp)
    img, _, info = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
    ri, _, g = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, return_grid=True, **kw)
    assert info.max_plane_support == max(g.plane_supports)
    assert peak_rel(img, ri) < TOL64


def test_imager_hankel_large_support_and_fp32c(ctx):
    s = _imager_case(36, 256, 2000, w_range=(-4000.0, 4000.0))
    kw = dict(kernel_func=5, kernel_support=3, kernel_exact=False, oversampling=4, analytic_gcf=False,
              num_wplanes=3, max_wpconv_support=40, kernel_trunc_perc=0.0, hankel_opt=True, interp_type=capi.CUBIC)
    ri, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
    img, _, info = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
    assert info.max_plane_support == 40
    assert peak_rel(img, ri) < TOL64
    img32, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, precision=capi.FP32C,
                                         out_dtype=capi.F32, **kw)
    # 81 x 81 untruncated W-kernels in single precision: rounding the oracle's own kernel tables to FP32
    # alone moves this image by 6.6e-6 of its peak (9.5e-6 for the FFT W-kernels of the same case), so the
    # FP32 gridder + FP32 FFT are held to 1e-4 here; the small-support case below keeps 1e-5
    assert peak_rel(img32.astype(np.float64), ri) < 1e-4


def test_imager_hankel_fp32c_vs_oracle(ctx):
    s = _imager_case(38, 256, 5000, w_range=(-1500.0, 1500.0))
    kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, analytic_gcf=False,
              num_wplanes=5, max_wpconv_support=8, kernel_trunc_perc=1.0, hankel_opt=True,
              hankel_proj_slice=True, interp_type=capi.CUBIC)
    ri, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
    img32, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, precision=capi.FP32C,
                                         out_dtype=capi.F32, **kw)
    assert peak_rel(img32.astype(np.float64), ri) < 1e-5


def _aproj_case(seed):
    s = make_snapshot(seed, 4000, 256, 20.0, n_src=4, flux=(1.0, 5.0), noise_sigma=0.05, w_range=(-600.0, 600.0))
    lha = np.random.default_rng(seed).uniform(-3.0, 2.0, s.vis.size)
    kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=4, analytic_gcf=False,
              num_wplanes=3, max_wpconv_support=8, kernel_trunc_perc=1.0, aproj_numtimesteps=3, obs_dec=-40.0,
              obs_ra=25.0, lha=lha, pbeam_coefs=[0.3, 0.8, 1.0, 0.5, 0.2])
    return s, kw


@pytest.mark.parametrize("opt", [False, True])
def test_imager_aproj_fp64_vs_oracle(ctx, opt):
    """A-projection: kernels per W-plane and hour-angle step, the beam rotated per step (or, with aproj_opt,
    the convolution kernel rotated step after step)."""
    s, kw = _aproj_case(61)
    kw["aproj_opt"] = opt
    img, _, info = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
    ri, _, g = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, return_grid=True, **kw)
    assert info.max_plane_support == max(g.plane_supports)
    assert peak_rel(img, ri) < TOL64
    # the beam changed the image (against plain W-projection)
    wkw = {k: v for k, v in kw.items() if k not in ("aproj_numtimesteps", "obs_dec", "obs_ra", "lha", "pbeam_coefs",
                                                    "aproj_opt")}
    wimg, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **wkw)
    assert peak_rel(img, wimg) > 1e-6


def test_imager_aproj_device_pointers_and_fp32c(ctx):
    import torch

    s, kw = _aproj_case(62)
    ri, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
    dkw = dict(kw, lha=torch.from_numpy(kw["lha"]).cuda())
    out = torch.empty(256 * 256, dtype=torch.float64, device="cuda")
    ctx.image_visibilities(torch.from_numpy(s.vis).cuda(), torch.from_numpy(s.weights).cuda(),
                           torch.from_numpy(np.ascontiguousarray(s.uvw.T)).cuda(), 256, s.cell_size,
                           device_ptrs=True, image_out=out, **dkw)
    torch.cuda.synchronize()
    assert peak_rel(out.cpu().numpy().reshape(256, 256).T, ri) < TOL64
    img32, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, precision=capi.FP32C,
                                         out_dtype=capi.F32, **kw)
    assert peak_rel(img32.astype(np.float64), ri) < 1e-5


@pytest.mark.parametrize("pattern", ["short_runs", "long_run", "all_equal", "oversized_bucket", "outlier"])
def test_imager_wproj_near_tied_w(ctx, pattern):
    """|w| values that are equal in the 24-bit sort key but distinct in double
    (or exactly equal): the W-plane boundaries must follow the exact stable
    double order of the reference's sort.  Short runs are re-sorted after the
    24-bit key sort; long runs of distinct values (200 of them, or 5000 within
    one part in 1e6) take the 64-bit sort; exactly equal values keep index
    order; one |w| 10^4 times the others (the key's scale) leaves the rest
    resolved to 2^-19 of their own size."""
    s = _imager_case(35, 256, 6000 if pattern == "oversized_bucket" else 4000, w_range=(-600.0, 600.0))
    uvw = np.array(s.uvw, order="F")
    w = uvw[:, 2]
    rng = np.random.default_rng(7)
    nplanes = 6
    if pattern == "short_runs":
        for k in range(0, w.size - 1, 2):  # |w| of the pair one double step apart
            w[k + 1] = np.copysign(np.nextafter(abs(w[k]), np.inf), w[k + 1])
    elif pattern == "outlier":
        w[17] = 6.0e6
    elif pattern == "oversized_bucket":
        # 5000 distinct |w| within one part in 1e6: runs of hundreds per single-precision key
        mags = 300.0 * (1.0 + rng.permutation(5000) * 1e-10)
        w[:5000] = np.where(rng.random(5000) < 0.5, mags, -mags)
    else:
        # a cluster placed across the first plane boundary
        aw = np.sort(np.abs(w))
        base = aw[w.size // nplanes]
        idx = rng.choice(w.size, size=200 if pattern == "long_run" else 300, replace=False)
        for j, k in enumerate(idx):
            mag = base * (1.0 + j * 1e-15) if pattern == "long_run" else base
            w[k] = mag if rng.random() < 0.5 else -mag
    kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, analytic_gcf=False,
              num_wplanes=nplanes, max_wpconv_support=8, undersampling_opt=1, kernel_trunc_perc=1.0)
    img, _, info = ctx.image_visibilities(s.vis, s.weights, uvw, 256, s.cell_size, **kw)
    ri, _, g = orc.image_visibilities(s.vis, s.weights, uvw, 256, s.cell_size, return_grid=True, **kw)
    assert info.max_plane_support == max(g.plane_supports)
    assert peak_rel(img, ri) < TOL64


@pytest.mark.parametrize("precision", [capi.FP32, capi.FP32C])
def test_imager_fp32_vs_fp64_oracle(ctx, precision):
    s = _imager_case(41, 512, 20000, w_range=(-500.0, 500.0))
    kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, analytic_gcf=False,
              num_wplanes=4, max_wpconv_support=8, kernel_trunc_perc=1.0)
    img, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 512, s.cell_size, precision=precision,
                                       out_dtype=capi.F32, **kw)
    ri, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, 512, s.cell_size, **kw)
    assert peak_rel(img.astype(np.float64), ri) < TOL32


def test_imager_empty_and_out_of_bounds(ctx):
    """No good visibilities -> the reference returns empty matrices (imager.h:355)."""
    uvw = np.asfortranarray(np.array([[1e9, 1e9, 0.0], [-1e9, 0.0, 0.0]]))
    img, beam, info = ctx.image_visibilities(np.ones(2, complex), np.ones(2), uvw, 64, 1.0, kernel_exact=False,
                                             oversampling=8)
    assert info.image_size == 0 and img.size == 0
    img, beam, info = ctx.image_visibilities(np.zeros(0, complex), np.zeros(0), np.zeros((0, 3)), 64, 1.0,
                                             kernel_exact=False, oversampling=8)
    assert info.image_size == 0


def test_imager_rejects_unsupported(ctx):
    s = _imager_case(1, 64, 100)
    with pytest.raises(capi.StpGpuError) as e:
        ctx.image_visibilities(s.vis, s.weights, s.uvw, 64, 1.0, num_wplanes=2, max_wpconv_support=4,
                               kernel_exact=False, hankel_opt=True, interp_type=7)
    assert e.value.status == 1
    # A-projection needs W-projection, no Hankel option, hour angles and beam coefficients (imager.h:274-283)
    lha = np.zeros(s.vis.size)
    for extra in (dict(), dict(num_wplanes=2, max_wpconv_support=4, hankel_opt=True, pbeam_coefs=[1.0], lha=lha),
                  dict(num_wplanes=2, max_wpconv_support=4, lha=lha)):
        with pytest.raises(capi.StpGpuError) as e:
            ctx.image_visibilities(s.vis, s.weights, s.uvw, 64, 1.0, aproj_numtimesteps=2, kernel_exact=False,
                                   **extra)
        assert e.value.status == 1
    with pytest.raises(capi.StpGpuError) as e:
        ctx.image_visibilities(s.vis, s.weights, s.uvw, 64, -1.0)
    assert e.value.status == 1


def test_imager_repeatable(ctx):
    """Two calls on the same context give the same image (cached buffers reused)."""
    s = _imager_case(3, 256, 4000)
    a, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, kernel_exact=False)
    b, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, kernel_exact=False)
    assert peak_rel(a, b) < 1e-13


def test_repeated_device_calls_replay_graph_with_new_data(ctx):
    """Device-pointer calls that repeat the previous call are replayed from a
    captured CUDA graph: the replay must read the buffers' current contents."""
    import torch

    s = _imager_case(51, 256, 5000, w_range=(-300.0, 300.0))
    s2 = _imager_case(52, 256, 5000, w_range=(-300.0, 300.0))
    kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, analytic_gcf=False,
              num_wplanes=4, max_wpconv_support=8, kernel_trunc_perc=1.0)
    c2 = capi.Context(0)
    try:
        dv = torch.from_numpy(s.vis).cuda()
        dw = torch.from_numpy(s.weights).cuda()
        duvw = torch.from_numpy(np.ascontiguousarray(s.uvw.T)).cuda()
        out = torch.empty(256 * 256, dtype=torch.float64, device="cuda")
        ref1, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
        ref2, _, _ = ctx.image_visibilities(s2.vis, s2.weights, s2.uvw, 256, s2.cell_size, **kw)
        for call in range(5):
            if call == 3:  # new data in the same buffers
                dv.copy_(torch.from_numpy(s2.vis))
                dw.copy_(torch.from_numpy(s2.weights))
                duvw.copy_(torch.from_numpy(np.ascontiguousarray(s2.uvw.T)))
            out.fill_(-1.0)
            _, _, info = c2.image_visibilities(dv, dw, duvw, 256, s.cell_size, device_ptrs=True, image_out=out, **kw)
            got = out.cpu().numpy().reshape(256, 256).T
            ref = ref1 if call < 3 else ref2
            assert info.image_size == 256
            assert peak_rel(got, ref) < 1e-12, call
            # every call, replays included, reports the kernels of ours it ran
            assert info.n_launches > 5, call
    finally:
        c2.close()


@pytest.mark.parametrize("layout", ["32", "16", "32c", "16c", "32t", "16t", "8t", "32r", "16r", "8r"])
@pytest.mark.parametrize("wproj", [False, True])
def test_imager_every_gridder_layout_vs_oracle(layout, wproj, monkeypatch):
    """Each tile width and gridder form the autotuner may pick gives the oracle's image (FP64 1e-10,
    FP32C 1e-5); the image spans the grid edges (items near the uv origin wrap after the shift)."""
    monkeypatch.setenv("STPGPU_GRIDDER_LAYOUT", layout)
    s = _imager_case(61, 256, 8000, w_range=(-600.0, 600.0) if wproj else (0.0, 0.0))
    kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, analytic_gcf=False,
              generate_beam=not wproj)
    if wproj:
        kw.update(num_wplanes=5, max_wpconv_support=8, kernel_trunc_perc=1.0)
    ref, rbeam = orc.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
    c = capi.Context(0)
    try:
        img, beam, _ = c.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, **kw)
        assert peak_rel(img, ref) < TOL64
        if not wproj:
            assert peak_rel(beam, rbeam) < TOL64
        img32, _, _ = c.image_visibilities(s.vis, s.weights, s.uvw, 256, s.cell_size, precision=capi.FP32C,
                                           out_dtype=capi.F32, **kw)
        assert peak_rel(img32.astype(np.float64), ref) < TOL32
    finally:
        c.close()
