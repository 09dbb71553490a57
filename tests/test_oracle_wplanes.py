"""The W-plane rule behind the GPU's sort-free planes (k_wsel_plan): when every
visibility is good, the oracle's average_w_planes (gridder.cpp:68-146) starts
plane p at sorted rank G_p = p * (n // P) + min(p, n % P), the closed form of
its ceil((n - begin) / (P - p)) recurrence; and the plane of a visibility is
the number of plane-start visibilities at or before it in the stable |w|
order, with the plane mean equal to the oracle's within rounding."""
import ctypes

import numpy as np
import pytest

from oracle import stp_oracle as orc


def _oracle_planes(absw_sorted, P):
    n = absw_sorted.size
    good = np.ones(n, dtype=np.int32)
    w_avg = np.empty(P)
    first = np.empty(P, dtype=np.int64)
    orc.lib().orc_average_w_planes(orc._d(np.ascontiguousarray(absw_sorted)), orc._i32(good), ctypes.c_int64(n),
                                   ctypes.c_int(P), ctypes.c_int(0), orc._d(w_avg), orc._i64(first))
    return first, w_avg


@pytest.mark.parametrize("n,P", [(1, 1), (7, 3), (10, 3), (11, 3), (40, 64), (1000, 32), (999983, 32), (3000, 300),
                                 (6000, 7)])
def test_plane_starts_closed_form(n, P):
    rng = np.random.default_rng(n + P)
    absw = np.sort(rng.uniform(0.0, 2000.0, size=n))
    first, _ = _oracle_planes(absw, P)
    q, r = divmod(n, P)
    closed = np.array([p * q + min(p, r) for p in range(P)], dtype=np.int64)
    assert np.array_equal(first, closed)


@pytest.mark.parametrize("ties", [False, True])
def test_planes_from_start_items(ties):
    """Plane by counting start items at or before (|w| bits, index), means from
    per-plane sums relative to the plane's smallest |w| (the GPU sums those
    offsets in exact fixed point): equal to the sorted assignment."""
    rng = np.random.default_rng(3)
    n, P = 20000, 24
    absw = rng.uniform(0.0, 700.0, size=n)
    if ties:
        absw[rng.integers(0, n, size=4000)] = absw[5]  # one |w| shared by ~4000 visibilities
    order = np.lexsort((np.arange(n), absw.view(np.uint64)))  # stable |w| order
    first, w_avg = _oracle_planes(absw[order], P)
    plane_sorted = np.searchsorted(first, np.arange(n), side="right") - 1
    plane_of = np.empty(n, dtype=np.int64)
    plane_of[order] = plane_sorted
    # start items: the visibility at each plane's first rank
    starts = [(absw[order[g]].view(np.uint64), order[g]) for g in first[1:]]
    keys = list(zip(absw.view(np.uint64), np.arange(n)))
    got = np.array([sum(1 for s in starts if s <= k) for k in keys])
    assert np.array_equal(got, plane_of)
    for p in range(P):
        members = absw[plane_of == p]
        lo = members.min()
        mean = lo + np.sum(members - lo) / members.size
        assert abs(mean - w_avg[p]) <= 1e-13 * max(1.0, abs(w_avg[p]))
