"""CPU-side checks of the drop-in boundary: the C-ABI library loads and
exports every symbol include/stpgpu.h declares (no compute without a GPU)."""
import ctypes
import os
import re

import pytest

from fastimaging_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "stpgpu.h")) as f:
        txt = f.read()
    return sorted(set(re.findall(r"STPGPU_API[^;(]*?\b(stpgpu_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = _declared()
    assert "stpgpu_image_visibilities" in names and "stpgpu_source_find" in names
    assert set(names) == set(capi.EXPORTED)


def test_library_exports_all_symbols():
    if not os.path.exists(capi.LIB_PATH):
        pytest.skip("libstpgpu.so not built")
    L = ctypes.CDLL(capi.LIB_PATH)
    for name in _declared():
        assert hasattr(L, name), name
    assert L.stpgpu_abi_version() == 2


def test_struct_sizes_match_header():
    # field layout mirrors include/stpgpu.h (checked against the C compiler)
    import subprocess
    import tempfile

    src = r"""
#include <stdio.h>
#include "stpgpu.h"
int main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(stpgpu_imager_pars), sizeof(stpgpu_wproj_pars),
 sizeof(stpgpu_aproj_pars), sizeof(stpgpu_imager_info), sizeof(stpgpu_island), sizeof(stpgpu_sf_pars),
 sizeof(stpgpu_sf_info), sizeof(stpgpu_snapshot), sizeof(stpgpu_batch_info), sizeof(stpgpu_server_pars),
 sizeof(stpgpu_request), sizeof(stpgpu_result), sizeof(stpgpu_server_stats));return 0;}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        with open(c, "w") as f:
            f.write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    sizes = [int(x) for x in out]
    py = [ctypes.sizeof(t) for t in (capi.ImagerPars, capi.WProjPars, capi.AProjPars, capi.ImagerInfo, capi.Island,
                                     capi.SfPars, capi.SfInfo, capi.Snapshot, capi.BatchInfo,
                                     capi.ServerPars, capi.Request, capi.Result, capi.ServerStats)]
    assert sizes == py


def test_no_device_is_reported_not_faked():
    """Without a GPU the library must refuse (no CPU fallback)."""
    if not os.path.exists(capi.LIB_PATH):
        pytest.skip("libstpgpu.so not built")
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(capi.StpGpuError) as e:
        capi.Context(0)
    assert e.value.status == 9
