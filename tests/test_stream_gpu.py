"""Streamed line lists (xs_stream_execute): FP64 centres, FP32 S(T) and FP32
gamma(T, P) in pinned host memory, copied chunk by chunk while earlier chunks
are evaluated.  Checked against the oracle on an equivalent line list (E'' = 0,
g = 1, n = 0 and A chosen so that step one gives back the stored S), against
one engine call over the same list, and for determinism."""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

import oracle
from gpu_cross_b200 import capi, synth
from helpers import assert_fp64_parity, assert_mixed_parity

pytestmark = pytest.mark.gpu

T, P_BAR, MASS = 2000.0, 1.0, 17.03


def equivalent_lines(nu, s32, g32, q):
    """A line list whose reference step one reproduces S = s32 and
    gamma(T, P) = g32: E'' = 0, g = 1, n = 0, gamma = g32, and
    A = S nu^2 Q / (cmcoef ISQRTPI (1 - exp(-beta nu)))."""
    cmcoef = 1.0 / (8.0 * math.acos(-1.0) * 2.99792458e10)
    beta = 6.6260693e-27 * 2.99792458e10 / (1.380658e-16 * T)
    s = s32.astype(np.float64)
    aif = s * nu * nu * q / (cmcoef * 0.564189584 * (1.0 - np.exp(-beta * nu)))
    n = nu.size
    return synth.LineList(nu.copy(), np.zeros(n), aif, np.ones(n, np.int32), g32.astype(np.float64),
                          np.zeros(n))


@pytest.fixture(scope="module")
def streamed():
    nu, s, g, kept, _ = synth.stream_workload(300_000, temperature=T, p_bar=P_BAR, seed=77)
    # a narrow band keeps the oracle quick: 1000-1060 cm-1 of the list
    a, b = np.searchsorted(nu, [1000.0, 1060.0])
    return nu[a:b].copy(), s[a:b].copy(), g[a:b].copy()


def run_stream(eng, nu, s, g, grid, prec, chunk):
    dev = torch.device("cuda:0")
    h_nu = torch.from_numpy(nu).pin_memory()
    h_s = torch.from_numpy(s).pin_memory()
    h_g = torch.from_numpy(g).pin_memory()
    fr = torch.as_tensor(grid.freq(), device=dev)
    out = torch.zeros(grid.npoints, dtype=torch.float64, device=dev)
    opts = capi.make_options(capi.VOIGT, grid.dfreq, MASS, precision=prec)
    cond = capi.make_condition(T, synth.partition_poly(T), 1.0, 1.0, 25.0)
    st = eng.stream_execute(opts, cond, h_nu.data_ptr(), h_s.data_ptr(), h_g.data_ptr(), nu.size,
                            capi.make_grid(fr), out.data_ptr(), chunk)
    return out.cpu().numpy(), st


def test_stream_fp64_vs_oracle_and_engine(cuda, streamed):
    nu, s, g = streamed
    grid = synth.Grid(990.0, 1070.0, 8000)
    q = synth.partition_poly(T)
    eng = capi.Engine(0)
    try:
        got, st = run_stream(eng, nu, s, g, grid, capi.FP64, chunk=200)
        assert st["chunks"] == (nu.size + 199) // 200 and st["chunks"] > 3
        # grid check, step one, step two, the core pass (+ the split
        # reduction) per chunk that reaches the grid
        assert 0 < st["kernels"] <= 5 * st["chunks"]
        again, _ = run_stream(eng, nu, s, g, grid, capi.FP64, chunk=200)
        assert np.array_equal(got, again)
        eq = equivalent_lines(nu, s, g, q)
        cond = dict(temperature=T, partition=q, mean_mass=MASS, pressure=1.0, ref_temp=296.0)
        ref = oracle.gpu_convention(oracle.VOIGT, grid.freq(), np.zeros(grid.npoints), eq, cond,
                                    grid.dfreq, cut=25.0)
        assert_fp64_parity(got, ref)
        whole, _ = run_stream(eng, nu, s, g, grid, capi.FP64, chunk=nu.size)
        assert_fp64_parity(got, whole)
        mixed, _ = run_stream(eng, nu, s, g, grid, capi.MIXED, chunk=200)
        assert_mixed_parity(mixed, ref)
    finally:
        eng.close()


def test_stream_rejects_bad_input(cuda, streamed):
    nu, s, g = streamed
    grid = synth.Grid(990.0, 1070.0, 8000)
    eng = capi.Engine(0)
    try:
        with pytest.raises(capi.XsError) as ei:
            run_stream(eng, nu[::-1].copy(), s, g, grid, capi.FP64, chunk=1000)
        assert ei.value.code == capi.XS_ERR_UNSORTED
        with pytest.raises(capi.XsError):
            run_stream(eng, nu, s, g, grid, capi.FP64, chunk=0)
    finally:
        eng.close()
