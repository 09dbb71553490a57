"""Model visibilities (stp::generate_visibilities_from_local_skymodel,
src/stp/visibility/visibility.cpp:15-40).  The reference's expected-model
NPZ is not available, so the oracle is checked against the published
point-source formula, and the GPU against the oracle with the reference
test's tolerance (absolute 1e-11, visibility_test_ModelGeneration.cpp:15)."""
import math

import numpy as np
import pytest

from fastimaging_b200 import capi
from fastimaging_b200.synthetic import point_source_vis
from oracle import stp_oracle as orc

TOL = 1e-11


def _case(seed, n_vis, n_src):
    rng = np.random.default_rng(seed)
    uvw = np.asfortranarray(np.column_stack([rng.uniform(-2e4, 2e4, n_vis), rng.uniform(-2e4, 2e4, n_vis),
                                             rng.uniform(-500, 500, n_vis)]))
    sky = np.column_stack([rng.uniform(-0.02, 0.02, n_src), rng.uniform(-0.02, 0.02, n_src),
                           rng.uniform(0.5, 10.0, n_src)])
    return uvw, sky


def test_oracle_matches_point_source_formula():
    uvw, sky = _case(1, 2000, 7)
    got = orc.generate_visibilities_from_local_skymodel(sky, uvw)
    ref = point_source_vis(uvw[:, 0], uvw[:, 1], uvw[:, 2], sky)
    assert np.max(np.abs(got - ref)) < TOL


def test_oracle_single_source_at_phase_centre():
    uvw, _ = _case(2, 100, 1)
    got = orc.generate_visibilities_from_local_skymodel(np.array([[0.0, 0.0, 3.5]]), uvw)
    assert np.allclose(got, 3.5 + 0j, atol=1e-15)


@pytest.mark.gpu
def test_gpu_model_visibilities_match_oracle():
    ctx = capi.Context(0)
    try:
        for seed, n_vis, n_src in ((3, 50_000, 20), (4, 1000, 600), (5, 7, 1)):
            uvw, sky = _case(seed, n_vis, n_src)
            ref = orc.generate_visibilities_from_local_skymodel(sky, uvw)
            got = ctx.model_visibilities(sky, uvw)
            assert np.max(np.abs(got - ref)) < TOL, (seed, np.max(np.abs(got - ref)))
            vis = ref * 1.5 + 0.25j
            res = ctx.model_visibilities(sky, uvw, vis=vis)
            assert np.max(np.abs(res - (vis - ref))) < TOL
        uvw, _ = _case(6, 100, 1)
        assert np.array_equal(ctx.model_visibilities(np.zeros((0, 3)), uvw), np.zeros(100, complex))
    finally:
        ctx.close()


@pytest.mark.gpu
def test_gpu_residual_in_place_on_device():
    import torch

    uvw, sky = _case(7, 20_000, 12)
    ref = orc.generate_visibilities_from_local_skymodel(sky, uvw)
    vis = np.exp(1j * np.linspace(0, 3, uvw.shape[0])) + ref
    ctx = capi.Context(0)
    try:
        dv = torch.from_numpy(vis.copy()).cuda()
        dsky = torch.from_numpy(np.asfortranarray(sky).T.copy()).cuda()  # (3, n_src): column-major n_src x 3
        duvw = torch.from_numpy(np.ascontiguousarray(uvw.T)).cuda()
        import ctypes

        st = ctx.L.stpgpu_model_visibilities(ctx.h, ctypes.c_void_p(dsky.data_ptr()), sky.shape[0],
                                             ctypes.c_void_p(duvw.data_ptr()), uvw.shape[0],
                                             ctypes.c_void_p(dv.data_ptr()), ctypes.c_void_p(dv.data_ptr()), 1)
        assert st == 0
        got = dv.cpu().numpy()
        assert np.max(np.abs(got - (vis - ref))) < TOL
    finally:
        ctx.close()
