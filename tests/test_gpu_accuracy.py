"""The error statement of mixed-precision results (xs_engine_accuracy),
through the C ABI: the stated a-priori bound must hold for the true error
against the FP64 oracle at every point above 1e-6 of the peak and for the
band integral, and the sampled FP64 re-evaluation must report the errors the
oracle gives on the same rows."""
import numpy as np
import pytest

import oracle
from gpu_cross_b200 import capi, synth

from helpers import to_device

pytestmark = pytest.mark.gpu


def _rows(start, points, k):
    """The engine's sampled rows: k evenly spaced rows of 32 points."""
    out = []
    for i in range(k):
        mid = points * (2 * i + 1) // (2 * k)
        r0 = start + mid - 16
        r0 = min(r0, start + points - 32)
        out.append(max(r0, start))
    return out


def _true_errors(got, ref):
    peak = np.abs(ref).max()
    big = np.abs(ref) > 1e-6 * peak
    rel = float(np.max(np.abs(got[big] - ref[big]) / np.abs(ref[big])))
    integ = abs(float(got.sum()) - float(ref.sum())) / abs(float(ref.sum()))
    return rel, integ


def _sampled_errors(got, ref, rows, end):
    idx = np.concatenate([np.arange(r, min(r + 32, end)) for r in rows])
    g, r = got[idx], ref[idx]
    peak = np.abs(r).max()
    big = np.abs(r) > 1e-6 * peak
    rel = float(np.max(np.abs(g[big] - r[big]) / np.abs(r[big])))
    integ = abs(float((g - r).sum())) / abs(float(r.sum()))
    return rel, integ


CASES = [
    # (seed, n, nu range, grid points, T, P atm, C, conditions)
    ("doppler-dominated", 11, 4000, (1000.0, 1100.0), 12000, [(300.0, 1e-3), (2100.0, 1e-3)], 2),
    ("pressure-dominated", 12, 4000, (1000.0, 1100.0), 12000, [(300.0, 10.0), (2100.0, 10.0)], 2),
    ("sweep grid, 8 conditions", 13, 20000, (500.0, 8000.0), 75000,
     [(t, p) for t in (300.0, 900.0, 1500.0, 2100.0) for p in (1e-3, 1.0)], 8),
    ("single condition", 14, 6000, (2000.0, 2100.0), 12000, [(1000.0, 1.0)], 1),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_error_statement_bounds_the_true_error(cuda, case):
    import torch

    _, seed, n, (lo, hi), npts, tp, C = case
    lines = synth.random_lines(n, lo, hi, 2500.0, 1e-6, 1e2, seed=seed, pressure_atm=1.0)
    grid = synth.Grid(lo - 10.0, hi + 10.0, npts)
    fr = grid.freq()
    d = to_device(lines, cuda)
    dfr = torch.as_tensor(fr, device=cuda)
    conds = [capi.make_condition(t, synth.partition_poly(t), 1.0, p, 25.0) for t, p in tp]
    eng = capi.Engine(0)
    try:
        eng.set_stream(torch.cuda.current_stream(cuda).cuda_stream)
        out = torch.zeros((len(conds), npts), dtype=torch.float64, device=cuda)
        opts = capi.make_options(capi.VOIGT, grid.dfreq, 17.03, precision=capi.MIXED,
                                 conditions_per_warp=C, check_rows=8)
        eng.execute(opts, conds, capi.make_lines(d), capi.make_grid(dfr), out.data_ptr(), npts)
        acc = eng.accuracy()
        got = out.cpu().numpy()
        f64 = torch.zeros_like(out)
        eng.execute(capi.make_options(capi.VOIGT, grid.dfreq, 17.03, precision=capi.FP64),
                    conds, capi.make_lines(d), capi.make_grid(dfr), f64.data_ptr(), npts)
        acc64 = eng.accuracy()
    finally:
        eng.close()
    assert acc["bound_rel"] == pytest.approx(1024 * 2.0 ** -24)
    assert acc["sampled_rows"] == 8 and acc["conditions"] == len(conds)
    assert acc64["bound_rel"] <= 1e-12 and acc64["sampled_rows"] == 0
    assert acc64["sampled_max_rel"] == -1.0
    rows = _rows(0, npts, 8)
    worst_rel, worst_int, worst_srel, worst_sint = 0.0, 0.0, 0.0, 0.0
    for k, (t, p) in enumerate(tp):
        scaled = synth.LineList(lines.nu, lines.energies, lines.aif, lines.gns, lines.gamma * p,
                                lines.n)
        cond = dict(temperature=t, partition=synth.partition_poly(t), mean_mass=17.03,
                    pressure=1.0, ref_temp=296.0, cut=25.0)
        ref = oracle.gpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), scaled, cond, grid.dfreq)
        rel, integ = _true_errors(got[k], ref)
        # the stated bound holds for every point and for the integral
        assert rel <= acc["bound_rel"], (k, rel)
        assert integ <= acc["bound_rel"], (k, integ)
        srel, sint = _sampled_errors(got[k], ref, rows, npts)
        worst_rel, worst_int = max(worst_rel, rel), max(worst_int, integ)
        worst_srel, worst_sint = max(worst_srel, srel), max(worst_sint, sint)
        assert np.max(np.abs(f64.cpu().numpy()[k] - ref)) <= 1e-10 * np.abs(ref).max()
    # the measured figures are the oracle's on the sampled rows (the FP64
    # re-evaluation differs from the oracle by summation order only)
    assert acc["sampled_max_rel"] == pytest.approx(worst_srel, rel=1e-3, abs=1e-10)
    assert acc["sampled_integrated_rel"] == pytest.approx(worst_sint, rel=1e-3, abs=1e-10)
    assert acc["sampled_max_rel"] <= acc["bound_rel"]


def test_error_statement_of_a_graph_replay_and_cpu_convention(cuda):
    import torch

    lines = synth.random_lines(3000, 1000.0, 1100.0, 2500.0, 1e-6, 1e2, seed=15, pressure_atm=0.3)
    grid = synth.Grid(990.0, 1110.0, 12000)
    fr = grid.freq()
    d = to_device(lines, cuda)
    dfr = torch.as_tensor(fr, device=cuda)
    cond = capi.make_condition(800.0, synth.partition_poly(800.0), 1.0, 1.0, -1.0)
    eng = capi.Engine(0)
    try:
        eng.set_stream(torch.cuda.current_stream(cuda).cuda_stream)
        out = torch.zeros_like(dfr)
        opts = capi.make_options(capi.VOIGT, grid.dfreq, 17.03, convention=capi.CONV_CPU,
                                 precision=capi.MIXED, cpu_threads=4, check_rows=4)
        g = eng.capture(opts, [cond], capi.make_lines(d), capi.make_grid(dfr), out.data_ptr(),
                        zero_out=True)
        g.launch(torch.cuda.current_stream(cuda).cuda_stream)
        acc = eng.accuracy()
        got = out.cpu().numpy()
        g.close()
    finally:
        eng.close()
    c = dict(temperature=800.0, partition=synth.partition_poly(800.0), mean_mass=17.03,
             pressure=1.0, ref_temp=296.0)
    ref = oracle.cpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), lines, c, grid.dfreq,
                                nthreads=4)
    rel, integ = _true_errors(got, ref)
    assert rel <= acc["bound_rel"] and integ <= acc["bound_rel"]
    srel, sint = _sampled_errors(got, ref, _rows(0, len(fr), 4), len(fr))
    assert acc["sampled_rows"] == 4
    assert acc["sampled_max_rel"] == pytest.approx(srel, rel=1e-3, abs=1e-10)
    assert acc["sampled_integrated_rel"] == pytest.approx(sint, rel=1e-3, abs=1e-10)
