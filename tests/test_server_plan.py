"""The request server's chunk planner (xs_plan_chunks), on the CPU: chunks
tile the grid in whole 256-point tiles, respect the work and line bounds,
carry every line that can reach them, and depend only on the request."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_cross_b200 import capi


def exact_pairs(nu, f0, df, start, points, cut):
    f = f0 + np.arange(start, start + points) * df
    lo = np.searchsorted(f, nu - cut, "left")
    hi = np.searchsorted(f, nu + cut, "right")
    return int((hi - lo).sum())


def lines(n, lo, hi, seed):
    return np.sort(np.random.default_rng(seed).uniform(lo, hi, n))


def check_plan(p, nu, f0, df, npoints, cut, max_pairs, max_lines):
    st, pt = p["start"], p["points"]
    assert st[0] == 0 and np.all(st[1:] == st[:-1] + pt[:-1])
    assert st[-1] + pt[-1] == npoints
    assert np.all(st % 256 == 0) and np.all(pt[:-1] % 256 == 0) and np.all(pt > 0)
    for k in range(len(st)):
        single = pt[k] <= 256
        assert single or p["pairs"][k] <= max_pairs
        n_k = int(p["l1"][k] - p["l0"][k])
        assert single or max_lines == 0 or n_k <= max_lines
        # every line whose window reaches the chunk is in its slice
        a = f0 + st[k] * df
        b = f0 + (st[k] + pt[k] - 1) * df
        need = np.nonzero((nu >= a - cut) & (nu <= b + cut))[0]
        if need.size:
            assert p["l0"][k] <= need[0] and p["l1"][k] >= need[-1] + 1


@pytest.mark.parametrize("max_pairs", [3e6, 5e7, 1e12])
def test_plan_tiles_and_bounds(built_libs, max_pairs):
    nu = lines(60000, 900.0, 2100.0, 5)
    f0, df, npoints, cut = 1000.0, 0.01, 100_000, 25.0
    p = capi.plan_chunks(nu, f0, df, npoints, cut, max_pairs)
    check_plan(p, nu, f0, df, npoints, cut, max_pairs, 0)
    if max_pairs == 1e12:
        assert len(p["start"]) == 1
    else:
        assert len(p["start"]) > 1


def test_plan_estimate_matches_exact_count(built_libs):
    nu = lines(40000, 0.0, 3000.0, 6)
    f0, df, npoints, cut = 500.0, 0.05, 30000, 25.0
    p = capi.plan_chunks(nu, f0, df, npoints, cut, 2e7)
    for k in range(len(p["start"])):
        ex = exact_pairs(nu, f0, df, int(p["start"][k]), int(p["points"][k]), cut)
        # the estimate is the window-overlap length / df: within one point per line
        n_k = int(p["l1"][k] - p["l0"][k])
        assert abs(p["pairs"][k] - ex) <= n_k + 1


def test_plan_line_bound(built_libs):
    nu = lines(200000, 0.0, 1000.0, 7)
    p = capi.plan_chunks(nu, 100.0, 0.01, 50000, 25.0, 1e15, max_lines=20000)
    check_plan(p, nu, 100.0, 0.01, 50000, 25.0, 1e15, 20000)
    assert len(p["start"]) > 1


def test_plan_is_deterministic(built_libs):
    nu = lines(50000, 0.0, 5000.0, 8)
    a = capi.plan_chunks(nu, 1000.0, 0.02, 120000, 25.0, 1e7)
    b = capi.plan_chunks(nu, 1000.0, 0.02, 120000, 25.0, 1e7)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_plan_edges(built_libs):
    # fewer points than a tile, no lines, lines all out of reach
    p = capi.plan_chunks(np.array([]), 0.0, 0.1, 100, 25.0, 1e9)
    assert list(p["start"]) == [0] and list(p["points"]) == [100] and p["pairs"][0] == 0.0
    nu = np.array([5000.0, 6000.0])
    p = capi.plan_chunks(nu, 0.0, 0.1, 1000, 25.0, 1e9)
    assert p["l1"][0] == p["l0"][0] and p["pairs"][0] == 0.0
    with pytest.raises(capi.XsError):
        capi.plan_chunks(np.array([2.0, 1.0]), 0.0, 0.1, 1000, 25.0, 1e9)
