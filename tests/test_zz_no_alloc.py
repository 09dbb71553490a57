"""Allocation-free labelling entry point (stpgpu_label_noalloc) against the
labelling of the regular source-finder entry point (stpgpu_source_find with
no label-map clean-up), through the C ABI.  Labels are integers: the check is
bit-exact, on two calls in a row for each case."""
import numpy as np
import pytest

from fastimaging_b200 import capi

pytestmark = pytest.mark.gpu

RMS = 1.0
ANALYSIS_N_SIGMA = 3.0


def _image(seed, rows, cols, dtype):
    rng = np.random.default_rng(seed)
    img = rng.normal(size=(rows, cols))
    for _ in range(12):
        r, c = rng.integers(0, rows - 6), rng.integers(0, cols - 6)
        img[r:r + 5, c:c + 4] += rng.choice([-8.0, 8.0])
    # components touching the row/column edges exercise the wrap links
    img[0:2, 40:44] += 9.0
    img[rows - 2:rows, 40:44] += 9.0
    return np.asfortranarray(img.astype(dtype))


@pytest.mark.parametrize("dtype,conn4,find_neg", [(np.float64, False, True), (np.float32, False, True),
                                                  (np.float64, True, True), (np.float64, False, False)])
def test_label_noalloc_matches_source_find(dtype, conn4, find_neg):
    import torch

    rows, cols = 384, 512
    img = _image(7, rows, cols, dtype)
    ctx = capi.Context(0)
    try:
        _, ref_labels, info = ctx.source_find(img, 5.0, ANALYSIS_N_SIGMA, RMS, find_neg, 5, capi.ZEROMEDIAN, False,
                                              conn4, False, 1)
    finally:
        ctx.close()
    # thresholds as the source finder forms them: bg + n_sigma * rms, bg = 0
    tp = 0.0 + ANALYSIS_N_SIGMA * RMS
    tn = 0.0 - ANALYSIS_N_SIGMA * RMS
    d_img = torch.from_numpy(np.ascontiguousarray(img.T)).cuda()  # column-major storage
    d_lab = torch.full((cols, rows), 12345, dtype=torch.int32, device="cuda")
    dt = capi.F32 if dtype == np.float32 else capi.F64
    torch.cuda.synchronize()
    for call in range(2):
        free0 = torch.cuda.mem_get_info()[0]
        npos, nneg = capi.label_noalloc(0, 0, d_img.data_ptr(), dt, rows, cols, tp, tn, find_neg, conn4, 0,
                                        d_lab.data_ptr())
        free1 = torch.cuda.mem_get_info()[0]
        got = d_lab.cpu().numpy().T
        assert np.array_equal(got, ref_labels), f"call {call}: label maps differ"
        assert (npos, nneg) == (info.n_labels_pos, info.n_labels_neg)
        if call == 1:
            assert free1 == free0, "device memory changed across an allocation-free call"
        d_lab.fill_(-7)
        torch.cuda.synchronize()
    assert info.n_labels_pos > 0 and (info.n_labels_neg > 0) == find_neg


def test_label_noalloc_rejects_beyond_maximum():
    with pytest.raises(capi.StpGpuError) as e:
        capi.label_noalloc(0, 0, 1, capi.F64, 2048, 1024, 3.0, -3.0, label_ptr=1)
    assert e.value.status == 1
    assert "maximum" in str(e.value)
    with pytest.raises(capi.StpGpuError):
        capi.label_noalloc(0, 0, 1, capi.F64, 7, 8, 3.0, -3.0, label_ptr=1)
