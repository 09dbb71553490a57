"""Serving loop (stpgpu_server_*): requests that run concurrently on the GPU
must give the same result as when each runs alone; admission keeps the
working sets in flight within the HBM budget."""
import numpy as np
import pytest

from fastimaging_b200 import capi
from fastimaging_b200.synthetic import make_snapshot

pytestmark = pytest.mark.gpu


def peak_rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _requests():
    out = []
    for k in range(8):
        size = 256 if k % 2 == 0 else 512
        wproj = k % 3 == 0
        s = make_snapshot(60 + k, 3000 + 700 * k, size, 2.0, n_src=4, flux=(3.0, 9.0), noise_sigma=0.05,
                          n_extended=1, w_range=(-200.0, 200.0) if wproj else (0.0, 0.0))
        kw = dict(image_size=size, cell_size=s.cell_size, kernel_func=capi.GaussianSinc if k % 2 else capi.PSWF,
                  kernel_support=3, kernel_exact=False, oversampling=8)
        if wproj:
            kw.update(num_wplanes=4, max_wpconv_support=8, kernel_trunc_perc=1.0)
        out.append((s, kw))
    return out


def _run(server, reqs, sequential, out_dtype):
    results = []
    if sequential:
        for s, kw in reqs:
            t = server.submit(s.vis, s.weights, s.uvw, find_sources=True, want_labels=True, out_dtype=out_dtype, **kw)
            results.append(server.wait(t))
    else:
        tickets = [server.submit(s.vis, s.weights, s.uvw, find_sources=True, want_labels=True, out_dtype=out_dtype,
                                 **kw) for s, kw in reqs]
        results = [server.wait(t) for t in tickets]
    return results


def _same_islands(a, b):
    """Islands of two FP64 images that differ only in the gridder's summation
    order (~1e-15 relative): identical pixels and extrema; the moment fit of a
    near-circular island (theta from atan of a near 0/0 ratio) may move by
    ~1e-8, so it is compared to 1e-6."""
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert (x.sign, x.extremum_x_idx, x.extremum_y_idx, x.num_samples) == \
            (y.sign, y.extremum_x_idx, y.extremum_y_idx, y.num_samples)
        assert np.isclose(x.extremum_val, y.extremum_val, rtol=1e-12, atol=0)
        assert np.allclose(x.moments_fit[:], y.moments_fit[:], rtol=1e-6, atol=1e-6)


def test_fp64_requests_same_alone_and_in_the_mix():
    reqs = _requests()
    alone = capi.Server(slots=1, precision=capi.FP64)
    try:
        ref = _run(alone, reqs, True, capi.F64)
    finally:
        alone.close()
    mix = capi.Server(slots=4, precision=capi.FP64)
    try:
        got = _run(mix, reqs, False, capi.F64)
        st = mix.stats()
    finally:
        mix.close()
    assert st.completed == len(reqs) and st.failed == 0
    assert st.peak_in_flight > 1  # the requests did overlap
    ctx = capi.Context(0)
    try:
        for (s, kw), (img, lab, isl, res), (rimg, rlab, risl, rres) in zip(reqs, got, ref):
            assert res.status == 0 and res.imager.image_size == kw["image_size"]
            # FP64 images: equal up to the gridder's summation order
            assert peak_rel(img, rimg) < 1e-12
            # the detection pipeline on equal images gives identical labels
            assert np.array_equal(lab, rlab)
            assert res.sf.n_labels_pos == rres.sf.n_labels_pos
            _same_islands(isl, risl)
            assert len(isl) > 0
        # and the served image is the single-call image
        s, kw = reqs[1]
        single, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, kw["image_size"], kw["cell_size"],
                                              **{k: v for k, v in kw.items() if k not in ("image_size", "cell_size")})
        assert peak_rel(got[1][0], single) < 1e-12
    finally:
        ctx.close()


def test_fp32c_requests_same_alone_and_in_the_mix():
    reqs = _requests()[:5]
    alone = capi.Server(slots=1, precision=capi.FP32C)
    try:
        ref = _run(alone, reqs, True, capi.F32)
    finally:
        alone.close()
    mix = capi.Server(slots=3, precision=capi.FP32C)
    try:
        got = _run(mix, reqs, False, capi.F32)
    finally:
        mix.close()
    for (img, _, isl, res), (rimg, _, risl, _) in zip(got, ref):
        assert res.status == 0
        assert peak_rel(img.astype(np.float64), rimg.astype(np.float64)) < 1e-6


def test_admission_keeps_in_flight_within_budget():
    reqs = _requests()
    probe = capi.Server(slots=1, precision=capi.FP32C)
    try:
        s, kw = reqs[1]
        t = probe.submit(s.vis, s.weights, s.uvw, find_sources=True, **kw)
        est = probe.wait(t)[3].est_bytes
    finally:
        probe.close()
    budget = int(est * 2.5)
    srv = capi.Server(slots=4, hbm_budget_bytes=budget, precision=capi.FP32C)
    try:
        tickets = [srv.submit(s.vis, s.weights, s.uvw, find_sources=True, **kw) for s, kw in reqs]
        res = [srv.wait(t)[3] for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    assert all(r.status == 0 for r in res)
    assert st.completed == len(reqs)
    assert st.peak_admitted_bytes <= budget
    assert 1 <= st.peak_in_flight <= 4
    assert st.queued == 0 and st.in_flight == 0
    assert st.p99_ms >= st.p50_ms > 0
    # first-in first-out admission
    admits = [r.admit_ms for r in res]
    assert admits == sorted(admits)


def test_request_larger_than_budget_is_rejected():
    s, kw = _requests()[1]
    srv = capi.Server(slots=1, hbm_budget_bytes=1 << 20, precision=capi.FP32C)
    try:
        with pytest.raises(capi.StpGpuError) as e:
            srv.submit(s.vis, s.weights, s.uvw, **kw)
        assert e.value.status == 5
    finally:
        srv.close()


def test_prepare_warms_every_slot_and_is_not_counted():
    reqs = _requests()
    srv = capi.Server(slots=3, precision=capi.FP64)
    try:
        # a request in flight while prepare holds admission
        s0, kw0 = reqs[0]
        t0 = srv.submit(s0.vis, s0.weights, s0.uvw, find_sources=True, out_dtype=capi.F64, **kw0)
        s, kw = reqs[3]
        res = srv.prepare(s.vis, s.weights, s.uvw, find_sources=True, out_dtype=capi.F64, **kw)
        assert res.status == 0 and res.imager.image_size == kw["image_size"]
        img, _, isl, r = srv.wait(t0)
        assert r.status == 0
        t = srv.submit(s.vis, s.weights, s.uvw, find_sources=True, out_dtype=capi.F64, **kw)
        _, _, isl3, r3 = srv.wait(t)
        st = srv.stats()
    finally:
        srv.close()
    assert st.submitted == 2 and st.completed == 2
    # the prepared request's outcome is the served one's
    assert r3.n_islands == res.n_islands and r3.sf.n_labels_pos == res.sf.n_labels_pos
    assert r3.imager.n_good_vis == res.imager.n_good_vis
