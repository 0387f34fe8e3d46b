"""Partition functions on the device (xs_partition_sum) and the server's
per-temperature Q(T) from a molecule's states."""
from __future__ import annotations

import math

import numpy as np
import pytest

from gpu_cross_b200 import capi, synth

pytestmark = pytest.mark.gpu

C2 = 6.6260693e-27 * 2.99792458e10 / 1.380658e-16  # exomol_functions.cpp:49-53


def states(n, seed):
    rng = np.random.default_rng(seed)
    e = np.sort(rng.uniform(0.0, 8000.0, n))
    g = (np.where(rng.random(n) < 0.5, 1, 3) * (2 * rng.integers(0, 61, n) + 1)).astype(np.int32)
    return e, g


def test_partition_sum_vs_exact_sum(cuda):
    e, g = states(20000, 5)
    temps = np.array([200.0, 296.0, 1000.0, 3000.0])
    q = capi.partition_sum(e, g, temps)
    for t, qt in zip(temps, q):
        want = math.fsum(float(gi) * math.exp(-(C2 / t) * ei) for ei, gi in zip(e, g))
        assert qt == pytest.approx(want, rel=1e-13)
    assert np.array_equal(q, capi.partition_sum(e, g, temps))


def test_server_computes_and_caches_q(cuda):
    lines = synth.random_lines(20000, 900.0, 1100.0, 1500.0, 1e-6, 1e2, seed=31)
    e, g = states(5000, 6)
    srv = capi.Server(0, lanes=1)
    try:
        mid = srv.add_molecule(lines, 18.02)
        with pytest.raises(capi.XsError):
            srv.submit(mid, capi.VOIGT, capi.FP64, 800.0, -1.0, 1.0, 950.0, 0.01, 5000)
        srv.add_states(mid, e, g)
        q = float(capi.partition_sum(e, g, [800.0])[0])
        a, _ = srv.wait(srv.submit(mid, capi.VOIGT, capi.FP64, 800.0, -1.0, 1.0, 950.0, 0.01, 5000),
                        5000)
        b, _ = srv.wait(srv.submit(mid, capi.VOIGT, capi.FP64, 800.0, q, 1.0, 950.0, 0.01, 5000), 5000)
        c, _ = srv.wait(srv.submit(mid, capi.VOIGT, capi.FP64, 800.0, 0.0, 1.0, 950.0, 0.01, 5000),
                        5000)
    finally:
        srv.close()
    assert np.array_equal(a, b) and np.array_equal(a, c) and np.abs(a).max() > 0
