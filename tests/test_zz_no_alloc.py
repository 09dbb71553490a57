"""Allocation-free labelling entry point (stpgpu_label_noalloc), through the
C ABI, against the CPU oracle's labelling (the source finder with no label-map
clean-up) and against the regular source-finder entry point
(stpgpu_source_find).  Labels are integers: the check is bit-exact, on two
calls in a row for each case.  Cases cover row counts that are multiples of
four (16 keys a thread in the class pass) and rows = 2 mod 4 (the
per-key class pass and the padded chunk tail)."""
import numpy as np
import pytest

from fastimaging_b200 import capi
from oracle import stp_oracle as orc

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


@pytest.mark.parametrize("rows,cols,dtype,conn4,find_neg", [
    (384, 512, np.float64, False, True), (384, 512, np.float32, False, True),
    (384, 512, np.float64, True, True), (384, 512, np.float64, False, False),
    (130, 98, np.float64, False, True), (130, 98, np.float32, False, True)])
def test_label_noalloc_matches_source_find(rows, cols, dtype, conn4, find_neg):
    import torch

    img = _image(7, rows, cols, dtype)
    # the checker: the oracle's labels before the detection filter, from the
    # same (single-precision images: promoted) pixel values
    ref = orc.source_find(img.astype(np.float64), 5.0, ANALYSIS_N_SIGMA, RMS, find_neg, 5, orc.ZEROMEDIAN, False,
                          conn4, False, 1)
    ctx = capi.Context(0)
    try:
        _, sf_labels, info = ctx.source_find(img, 5.0, ANALYSIS_N_SIGMA, RMS, find_neg, 5, capi.ZEROMEDIAN, False,
                                             conn4, False, 1)
    finally:
        ctx.close()
    assert np.array_equal(sf_labels, ref.label_map), "source finder and oracle label maps differ"
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
        assert np.array_equal(got, ref.label_map), f"call {call}: label map differs from the oracle's"
        assert (npos, nneg) == (ref.n_pos, ref.n_neg)
        assert (npos, nneg) == (info.n_labels_pos, info.n_labels_neg)
        if call == 1:
            assert free1 == free0, "device memory changed across an allocation-free call"
        d_lab.fill_(-7)
        torch.cuda.synchronize()
    assert info.n_labels_pos > 0 and (info.n_labels_neg > 0) == find_neg


def test_label_noalloc_rejects_beyond_maximum():
    """Sizes beyond the maximum, and odd sizes, are refused before any launch.
    The buffers passed are real device buffers of the stated sizes, so the
    call stays in bounds even if the validation were to let it through."""
    import torch

    img = torch.zeros((1024, 2048), dtype=torch.float64, device="cuda")
    lab = torch.zeros((1024, 2048), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(capi.StpGpuError) as e:
        capi.label_noalloc(0, 0, img.data_ptr(), capi.F64, 2048, 1024, 3.0, -3.0, label_ptr=lab.data_ptr())
    assert e.value.status == 1
    assert "maximum" in str(e.value)
    small = torch.zeros((8, 7), dtype=torch.float64, device="cuda")
    small_lab = torch.zeros((8, 7), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(capi.StpGpuError):
        capi.label_noalloc(0, 0, small.data_ptr(), capi.F64, 7, 8, 3.0, -3.0, label_ptr=small_lab.data_ptr())
