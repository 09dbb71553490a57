"""The C++ drop-in (include/stpgpu_stp.hpp): stp::image_visibilities /
stp::ImageVisibilities (src/stp/imager/imager.h:233-411) and
stp::SourceFindImage (src/stp/sourcefind/sourcefind.h:143-201) with the
reference's signatures, compiled against Armadillo-shaped test containers
(tests/cpp/arma_shim.h; Armadillo is not installed) and the library.

CPU: the driver compiles and links, for double and for single-precision
(USE_FLOAT) real_t.  GPU: the driver images a snapshot through the class and
the template entry points and runs the source finder on the image; the image
is compared with the CPU oracle at the FP64 tolerance (1e-10 peak-relative,
src/stp/types.h:26), the label map bit-exact, the islands equal."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "fastimaging_b200")


def _compile(out, use_float=False):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(ROOT, "tests", "cpp"), os.path.join(ROOT, "tests", "cpp", "adapter_main.cpp"), "-o", out,
           "-L", LIBDIR, "-lstpgpu", "-Wl,-rpath," + LIBDIR]
    if use_float:
        cmd.insert(1, "-DUSE_FLOAT")
    subprocess.run(cmd, check=True, capture_output=True, text=True)


@pytest.mark.parametrize("use_float", [False, True])
def test_adapter_compiles_and_links(tmp_path, use_float):
    if not os.path.exists(os.path.join(LIBDIR, "libstpgpu.so")):
        pytest.skip("libstpgpu.so not built")
    exe = str(tmp_path / "adapter_main")
    _compile(exe, use_float)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_adapter_matches_oracle(tmp_path):
    from fastimaging_b200.synthetic import make_snapshot
    from oracle import stp_oracle as orc

    exe = str(tmp_path / "adapter_main")
    _compile(exe)
    N = 512
    s = make_snapshot(61, 30000, N, 2.0, n_src=6, flux=(2.0, 8.0), noise_sigma=0.1, w_range=(-400.0, 400.0))
    kf, support, os_, exact, analytic, planes, wsup, trunc = 4, 3, 8, 0, 0, 8, 8, 1.0
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.array([s.vis.size], dtype=np.int64).tofile(f)
        np.array([N, kf, support, os_, exact, analytic, planes, wsup], dtype=np.int32).tofile(f)
        np.array([s.cell_size, trunc], dtype=np.float64).tofile(f)
        np.ascontiguousarray(s.vis, dtype=np.complex128).tofile(f)
        np.ascontiguousarray(s.weights, dtype=np.float64).tofile(f)
        np.asfortranarray(s.uvw).reshape(-1, order="F").tofile(f)
    prefix = str(tmp_path / "out")
    r = subprocess.run([exe, str(inp), prefix], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "error path ok" in r.stdout
    kw = dict(kernel_func=kf, kernel_support=support, kernel_exact=False, oversampling=os_, gridding_correction=True,
              analytic_gcf=False, num_wplanes=planes, max_wpconv_support=wsup, kernel_trunc_perc=trunc)
    ref_img, ref_beam = orc.image_visibilities(s.vis, s.weights, s.uvw, N, s.cell_size, generate_beam=True, **kw)
    img = np.fromfile(prefix + "_image.bin", dtype=np.float64).reshape((N, N), order="F")
    beam = np.fromfile(prefix + "_beam.bin", dtype=np.float64).reshape((N, N), order="F")
    img_gs = np.fromfile(prefix + "_image_gs.bin", dtype=np.float64).reshape((N, N), order="F")
    peak = np.max(np.abs(ref_img))
    assert np.max(np.abs(img - ref_img)) / peak < 1e-10
    assert np.max(np.abs(img_gs - ref_img)) / peak < 1e-10
    assert np.max(np.abs(beam - ref_beam)) / np.max(np.abs(ref_beam)) < 1e-10
    ref = orc.source_find(img, 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True, 5)
    labels = np.fromfile(prefix + "_labels.bin", dtype=np.int32).reshape((N, N), order="F")
    assert np.array_equal(labels, ref.label_map)
    with open(prefix + "_islands.txt") as f:
        bg, rms = (float(x) for x in f.readline().split())
        rows = [line.split() for line in f if line.strip()]
    assert abs(rms - ref.rms_est) <= 1e-10 * abs(ref.rms_est)
    assert len(rows) == len(ref.islands) and len(rows) > 0
    for row, isl in zip(rows, ref.islands):
        sign, val, x, y, ns, mom, _, _ = isl
        assert (int(row[1]), int(row[3]), int(row[4]), int(row[5])) == (sign, x, y, ns)
        assert float(row[2]) == val
        got = np.array([float(v) for v in row[6:12]])
        want = np.array([mom.amplitude, mom.x_centre, mom.y_centre, mom.semimajor, mom.semiminor, mom.theta])
        assert np.allclose(got, want, rtol=1e-9, atol=1e-9)
