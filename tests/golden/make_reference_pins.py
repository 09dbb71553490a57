"""Extract the reference's inline known answers into tests/golden/reference_pins.json.

Reads the reference gtest sources as text (never compiles or runs them) and
records the literal expected matrices/values with the parameters of each test.
Run in a container that has the reference tree:

    python tests/golden/make_reference_pins.py <path of the FastImaging source tree>

The JSON is committed; nothing on the GPU side reads the reference tree.
"""
from __future__ import annotations

import json
import math
import os
import re
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_pins.json")


def _block_after(text, start):
    """Balanced {...} block starting at the first '{' at/after start."""
    i = text.index("{", start)
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i:j + 1], j + 1
    raise ValueError("unbalanced")


def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def _non_fftshift(text):
    """Keep the '#ifndef FFTSHIFT' branches (the reference's default build)."""
    out = []
    lines = text.split("\n")
    state = []
    for ln in lines:
        s = ln.strip()
        if s.startswith("#ifndef FFTSHIFT"):
            state.append("keep")
            continue
        if s.startswith("#ifdef FFTSHIFT"):
            state.append("drop")
            continue
        if s.startswith("#else") and state:
            state[-1] = "drop" if state[-1] == "keep" else "keep"
            continue
        if s.startswith("#endif") and state:
            state.pop()
            continue
        if state and state[-1] == "drop":
            continue
        out.append(ln)
    return "\n".join(out)


def _eval_matrix(block, symbols):
    expr = block.replace("{", "[").replace("}", "]")
    expr = expr.replace("arma::datum::pi", "pi").replace("real_t", "").replace("cx_real_t", "")
    ns = {"pi": math.pi, "exp": math.exp, "pow": math.pow, "__builtins__": {}}
    ns.update(symbols)
    return eval(expr, ns)  # noqa: S307 - literal matrices from test sources


def matrix(text, name, symbols, occurrence=0):
    pat = re.compile(r"\b" + re.escape(name) + r"\s*=\s*\{")
    ms = list(pat.finditer(text))
    blk, _ = _block_after(text, ms[occurrence].start())
    return _eval_matrix(blk, symbols)


def load(ref, rel):
    with open(os.path.join(ref, "src", "test", rel)) as f:
        return _non_fftshift(_strip_comments(f.read()))


def main(ref):
    pins = {"source": "SKA-ScienceDataProcessor/FastImaging src/test (inline known answers)"}

    # --- gridder (convolve_to_grid) unit tests
    g = []
    t = load(ref, "gridder/gridder_test_SmallPillbox.cpp")
    g.append(dict(name="SmallPillbox", file="gridder/gridder_test_SmallPillbox.cpp", kernel="TopHat", hbw=0.55,
                  support=1, image_size=8, kernel_exact=True, oversampling=1, shift_uv=False, halfplane=False,
                  uv=[[-1.5, 0.5]], vis=[[1, 0]], weights=[1.0],
                  expect_vis_grid_real=matrix(t, "expected_result", {"v": 0.25}), expect_sampling_real=None))
    t = load(ref, "gridder/gridder_test_MultiPixelPillbox.cpp")
    e = matrix(t, "expected_result", {"v": 1.0 / 9.0})
    g.append(dict(name="MultiPixelPillbox", file="gridder/gridder_test_MultiPixelPillbox.cpp", kernel="TopHat",
                  hbw=1.1, support=1, image_size=8, kernel_exact=True, oversampling=1, shift_uv=False,
                  halfplane=False, uv=[[-2.0, 0.0]], vis=[[1, 0]], weights=[1.0], expect_vis_grid_real=e,
                  expect_sampling_real=e))
    t = load(ref, "gridder/gridder_test_MultipleComplexVis.cpp")
    e = matrix(t, "expected_result", {"v": 1.0 / 9.0})
    g.append(dict(name="MultipleComplexVis", file="gridder/gridder_test_MultipleComplexVis.cpp", kernel="TopHat",
                  hbw=1.1, support=1, image_size=8, kernel_exact=True, oversampling=1, shift_uv=False,
                  halfplane=False, uv=[[-2.0, 1.0], [1.0, -1.0]], vis=[[1, 0], [1, 0]], weights=[1.0, 1.0],
                  expect_vis_grid_real=e, expect_sampling_real=e))
    t = load(ref, "gridder/gridder_test_NearbyComplexVis.cpp")
    e = matrix(t, "expected_vis_grid", {"v": 1.0 / 9.0})
    g.append(dict(name="NearbyComplexVis", file="gridder/gridder_test_NearbyComplexVis.cpp", kernel="TopHat",
                  hbw=1.1, support=2, image_size=8, kernel_exact=True, oversampling=1, shift_uv=False,
                  halfplane=False, uv=[[-1.0, 1.0], [0.0, -1.0]], vis=[[1, 0], [1, 0]], weights=[1.0, 1.0],
                  expect_vis_grid_real=e, expect_sampling_real=e))
    t = load(ref, "gridder/gridder_test_SinglePixelOverlapPillbox.cpp")
    e = matrix(t, "expected_result", {})
    amp = 42.123
    g.append(dict(name="SinglePixelOverlapPillbox", file="gridder/gridder_test_SinglePixelOverlapPillbox.cpp",
                  kernel="TopHat", hbw=0.5, support=1, image_size=8, kernel_exact=True, oversampling=1,
                  shift_uv=False, halfplane=False, uv=[[-2.0, 0.0], [-2.0, 0.0]], vis=[[amp, 0], [amp, 0]],
                  weights=[1.0, 1.0], expect_vis_grid_real=[[x * 2 * amp for x in r] for r in e],
                  expect_sampling_real=[[x * 2 for x in r] for r in e]))
    t = load(ref, "gridder/gridder_test_HalfPlaneShiftedGridding.cpp")
    g.append(dict(name="HalfPlaneShiftedGridding", file="gridder/gridder_test_HalfPlaneShiftedGridding.cpp",
                  kernel="TopHat", hbw=1.1, support=1, image_size=8, kernel_exact=False, oversampling=9,
                  shift_uv=True, halfplane=True, uv=[[-2.0, 0.0], [0.0, -2.0]], vis=[[1, 0], [1, 0]],
                  weights=[1.0, 1.0], roll_cols=4,
                  expect_vis_grid_real=matrix(t, "expected_result", {"v": 1.0 / 9.0}), expect_sampling_real=None,
                  also_exact=True))
    t = load(ref, "gridder/gridder_test_SampleWeighting.cpp")
    g.append(dict(name="SampleWeightingNatural", file="gridder/gridder_test_SampleWeighting.cpp", kernel="TopHat",
                  hbw=0.5, support=1, image_size=8, kernel_exact=True, oversampling=1, shift_uv=False,
                  halfplane=False, uv=[[-2.0, 0.0], [-2.0, 0.0]], vis=[[1.5, 0], [3.0, 0]], weights=[2.0, 3.0],
                  expect_sampling_normalised=matrix(t, "expected_sample_locations", {}),
                  natural_weighted_sum=(1.5 * 2.0 + 3.0 * 3.0) / 5.0))
    pins["gridder"] = g

    # --- oversampled index maths
    t = load(ref, "gridder/gridder_test_FractionalCoordToOversampledIndexMath.cpp")
    pins["oversampled_indices"] = dict(oversampling=5, io_pairs=matrix(t, "io_pairs", {}),
                                       edge_case=dict(oversampling=7, offset=0.5, expected=3))

    # --- kernel generation (make_kernel_array)
    k = []
    for rel, kernel, hbw, support, os_ in (
            ("kernel/kernel_test_OversampledPillbox.cpp", "TopHat", 0.7, 1, 3),
            ("kernel/kernel_test_OversampledPillboxSmall.cpp", "TopHat", 0.25, 1, 5),
            ("kernel/kernel_test_RegularSamplingPillbox.cpp", "TopHat", 1.1, 2, 1),
            ("kernel/kernel_test_RegularSamplingTriangle.cpp", "Triangle", 1.5, 2, 1)):
        t = load(ref, rel)
        sym = {"kv1": 1.0 - 1.0 / 1.5, "kv1sq": (1.0 - 1.0 / 1.5) ** 2, "kv_half": 1.0 - 0.5 / 1.5}
        offsets = re.findall(r"offset_index\s*=\s*(?:arma::mat)?\s*\{([^}]*)\}", t)
        for occ, off in enumerate(offsets):
            off = [float(x) for x in off.split(",")]
            k.append(dict(file=rel, kernel=kernel, hbw=hbw, support=support, oversampling=os_, offset=off,
                          expected=matrix(t, "expected_results", sym, occ)))
    pins["make_kernel_array"] = k

    # --- convolution functor values
    c = []
    t = load(ref, "conv/conv_test_pswf.cpp")
    c.append(dict(kernel="PSWF", trunc=3.0, input=matrix(t, "input", {}), output=matrix(t, "output", {})))
    t = load(ref, "conv/conv_test_sinc.cpp")
    c.append(dict(kernel="Sinc", trunc=3.0, input=matrix(t, "input", {}), output=matrix(t, "output", {})))
    t = load(ref, "conv/conv_test_tophat.cpp")
    c.append(dict(kernel="TopHat", trunc=3.0, input=matrix(t, "input", {}), output=matrix(t, "output", {})))
    t = load(ref, "conv/conv_test_triangle.cpp")
    c.append(dict(kernel="Triangle", trunc=2.0, input=matrix(t, "input", {}), output=matrix(t, "output", {})))
    t = load(ref, "conv/conv_test_gaussian.cpp")
    c.append(dict(kernel="Gaussian", trunc=3.0, input=matrix(t, "input", {}), output=matrix(t, "output", {})))
    t = load(ref, "conv/conv_test_gaussiansinc.cpp")
    sym = {"width_normalization_sinc": 1.55, "width_normalization_gaussian": 2.52}
    c.append(dict(kernel="GaussianSinc", trunc=5.0, input=matrix(t, "input", sym), output=matrix(t, "output", sym)))
    pins["conv"] = c

    # --- CCL label maps (non-FFTSHIFT expectations)
    t = load(ref, "sourcefind/sourcefind_test_Labeling.cpp")
    labs = []
    for m in re.finditer(r"TEST_F\(SourceFindLabeling,\s*(\w+)\)", t):
        body, _ = _block_after(t, m.end())
        sym = {"S": 10.0, "n": 0.0, "I": -10.0}
        img = matrix(body, "img", sym)
        exp = matrix(body, "expected_map", sym)
        conn4 = "ccl_4connectivity = true" in body
        tot = int(re.search(r"expected_total_islands\s*=\s*(\d+)", body).group(1))
        labs.append(dict(name=m.group(1), conn4=conn4, img=img, expected_map=exp, expected_total_islands=tot,
                         detection_n_sigma=4.0, analysis_n_sigma=3.0, rms_est=1.0, median_method="ZEROMEDIAN",
                         source_min_area=1, generate_labelmap=False, fftshift_input=True))
    pins["labeling"] = labs

    # --- median hand patterns (binmedian / binapprox vs exact median)
    pins["median_patterns"] = [
        dict(name="BinMedianSpecificPattern1", data=[[1, 30, 60], [1, 30, 60], [1, 30, 60]]),
        dict(name="BinMedianSpecificPattern2", data=[[1, 1, 60], [1, 1, 60], [1, 60, 60]]),
        dict(name="BinMedianSpecificPattern3", data=[[1, 1, 1], [1, 1, 1], [1, 1, 60]]),
        dict(name="Pattern4_20x20_halves", fill="halves"),
        dict(name="Pattern5_20x20_halves_extremes", fill="halves_extremes"),
    ]
    with open(OUT, "w") as f:
        json.dump(pins, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_reference_pins.py <path of the FastImaging source tree>")
    main(sys.argv[1])
