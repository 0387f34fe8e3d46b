"""Parity of the CUDA path with the oracle and with the reference's own code.

Tier 1: FP64, reference GPU convention  vs oracle GPU restatement and vs the
        reference's cross_kernal.cu compiled for sm_100a: <= 1e-10 relative
        (points above 1e-6 of the peak; <= 1e-10 of the peak elsewhere).
Tier 2: FP64, reference CPU convention  vs the reference's own OpenMPManager
        and its restatement: same bound.
Tier 3: mixed precision vs FP64: <= 1e-4 relative above 1e-6 of the peak,
        integrated cross-section within 1e-6.
All calls go through the C ABI.
"""
import numpy as np
import pytest

import oracle
from gpu_cross_b200 import capi, synth

from helpers import (assert_fp64_parity, assert_mixed_parity, parity_errors, run_engine,
                     small_voigt_case, to_device)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine(cuda):
    e = capi.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("pressure", [0.1, 1.0, 10.0])
def test_voigt_gpu_convention_vs_oracle(engine, cuda, pressure):
    lines, grid, cond = small_voigt_case(pressure_atm=pressure)
    cond = dict(cond, pressure=pressure)
    fr = grid.freq()
    z = np.zeros_like(fr)
    ref = oracle.gpu_convention(oracle.VOIGT, fr, z, lines, cond, grid.dfreq)
    got = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda)
    assert_fp64_parity(got, ref)


@pytest.mark.parametrize("P", [1, 2, 4, 8])
def test_voigt_shapes_agree(engine, cuda, P):
    lines, grid, cond = small_voigt_case(seed=11, n=1500)
    fr = grid.freq()
    ref = oracle.gpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    for W in (4, 8):
        got = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, P=P, W=W)
        assert_fp64_parity(got, ref)
        # the mixed kernel at this shape (P = 2, 4, 8: reciprocals shared
        # between two lines or two row pairs)
        mix = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, P=P, W=W,
                         precision=capi.MIXED)
        assert_mixed_parity(mix, ref)


@pytest.mark.parametrize("S", [1, 3, 64])
def test_line_splits_vs_oracle(engine, cuda, S):
    """A tile's lines split over S warps (partial sums added in split order)
    give the oracle's result, and the same bits on every run."""
    lines, grid, cond = small_voigt_case(seed=12, n=4000)
    fr = grid.freq()
    ref = oracle.gpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    got = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, S=S)
    assert_fp64_parity(got, ref)
    again = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, S=S)
    assert np.array_equal(got, again)
    mix = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, S=S,
                     precision=capi.MIXED)
    assert_mixed_parity(mix, ref)
    dl = synth.exomol_like(2000, 3000, seed=13, nu_max=2000.0)
    dg = synth.Grid(0.0, 2000.0, 20000)
    dc = dict(temperature=296.0, partition=2844.0, mean_mass=30.01, pressure=1.0, ref_temp=296.0)
    dref = oracle.gpu_convention(oracle.DOPPLER, dg.freq(), np.zeros(dg.npoints), dl, dc, dg.dfreq)
    dgot = run_engine(engine, capi.DOPPLER, dl, dg.freq(), dc, dg.dfreq, cuda, S=S)
    assert_fp64_parity(dgot, dref)


def test_line_splits_multi_condition(engine, cuda):
    lines = synth.random_lines(3000, 1000.0, 1100.0, 2500.0, 1e-6, 1e2, seed=52, pressure_atm=1.0)
    grid = synth.Grid(990.0, 1110.0, 1200)
    base = dict(mean_mass=17.03, pressure=1.0, ref_temp=296.0)
    conds = [dict(base, temperature=t, partition=synth.partition_poly(t), gamma_scale=p, cut=25.0)
             for t in (300.0, 2100.0) for p in (1e-3, 10.0)]
    fr = grid.freq()
    one = run_engine(engine, capi.VOIGT, lines, fr, base, grid.dfreq, cuda, conds=conds, C=2, S=1,
                     precision=capi.MIXED)
    five = run_engine(engine, capi.VOIGT, lines, fr, base, grid.dfreq, cuda, conds=conds, C=2, S=5,
                      precision=capi.MIXED)
    f64 = run_engine(engine, capi.VOIGT, lines, fr, base, grid.dfreq, cuda, conds=conds, S=1)
    for k in range(len(conds)):
        assert_mixed_parity(one[k], f64[k])
        assert_mixed_parity(five[k], f64[k])


@pytest.mark.parametrize("C", [1, 4, 8])
def test_multi_condition_mixed_wide_and_narrow_lines(engine, cuda, C):
    """Lines at 10-60 cm-1 have Doppler widths of a few 1e-5 cm-1, so the
    25 cm-1 cut reaches x ~ 1e6: their shared region-I reciprocals need the
    scaled products ("wide" lines); lines at 2000 cm-1 take the unscaled ones.
    Mixed against FP64 for both in one call."""
    low = synth.random_lines(1500, 10.0, 60.0, 2500.0, 1e-6, 1e2, seed=54, pressure_atm=1.0)
    high = synth.random_lines(1500, 2000.0, 2050.0, 2500.0, 1e-6, 1e2, seed=55, pressure_atm=1.0)
    lines = synth.LineList(*(np.concatenate([getattr(low, f), getattr(high, f)])
                             for f in ("nu", "energies", "aif", "gns", "gamma", "n")))
    grid = synth.Grid(0.0, 2100.0, 210000)
    base = dict(mean_mass=17.03, pressure=1.0, ref_temp=296.0)
    conds = [dict(base, temperature=t, partition=synth.partition_poly(t), gamma_scale=p, cut=25.0)
             for t in (300.0, 2100.0) for p in (1e-3, 0.1, 1.0, 10.0)][:C]
    fr = grid.freq()
    f64 = run_engine(engine, capi.VOIGT, lines, fr, base, grid.dfreq, cuda, conds=conds)
    mix = run_engine(engine, capi.VOIGT, lines, fr, base, grid.dfreq, cuda, conds=conds, C=C,
                     precision=capi.MIXED)
    for k in range(len(conds)):
        assert_mixed_parity(mix[k], f64[k])


@pytest.mark.parametrize("C", [2, 4, 8])
def test_multi_condition_mixed_cpu_convention(engine, cuda, C):
    """Mixed multi-condition tiles in the CPU convention (sqrt(ln 2) Doppler
    widths, rounded windows, the OpenMPManager's line coverage) against the
    oracle's OpenMPManager restatement, per condition."""
    lines = synth.random_lines(3000, 1000.0, 1100.0, 2500.0, 1e-6, 1e2, seed=53, pressure_atm=1.0)
    grid = synth.Grid(990.0, 1110.0, 1200)
    base = dict(mean_mass=17.03, pressure=1.0, ref_temp=296.0)
    conds = [dict(base, temperature=t, partition=synth.partition_poly(t), gamma_scale=p)
             for t in (300.0, 700.0, 1500.0, 2100.0) for p in (1e-3, 10.0)]
    fr = grid.freq()
    mix = run_engine(engine, capi.VOIGT, lines, fr, base, grid.dfreq, cuda, conds=conds, C=C,
                     convention=capi.CONV_CPU, cpu_threads=3, precision=capi.MIXED)
    for k, c in enumerate(conds):
        scaled = synth.LineList(lines.nu, lines.energies, lines.aif, lines.gns,
                                lines.gamma * c["gamma_scale"], lines.n)
        ref = oracle.cpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), scaled,
                                    dict(c, pressure=1.0), grid.dfreq, nthreads=3)
        assert_mixed_parity(mix[k], ref)


@pytest.mark.parametrize("threads", [1, 3, 8])
def test_voigt_cpu_convention_vs_reference_openmp(engine, cuda, threads):
    lines, grid, cond = small_voigt_case(seed=3)
    fr = grid.freq()
    z = np.zeros_like(fr)
    ref = oracle.ref_cpu(oracle.VOIGT, fr, z, lines, cond, grid.dfreq, nthreads=threads)
    got = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda,
                     convention=capi.CONV_CPU, cpu_threads=threads)
    assert_fp64_parity(got, ref)


def test_doppler_gpu_convention_vs_oracle(engine, cuda):
    lines = synth.exomol_like(2000, 4000, seed=5, nu_max=3000.0)
    grid = synth.Grid(0.0, 3000.0, 300000)
    cond = dict(temperature=296.0, partition=2844.0, mean_mass=30.01, pressure=1.0)
    fr = grid.freq()
    ref = oracle.gpu_convention(oracle.DOPPLER, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    got = run_engine(engine, capi.DOPPLER, lines, fr, cond, grid.dfreq, cuda)
    assert_fp64_parity(got, ref)


@pytest.mark.parametrize("threads", [1, 4])
def test_doppler_cpu_convention_vs_reference_openmp(engine, cuda, threads):
    lines = synth.exomol_like(2000, 3000, seed=6, nu_max=2000.0)
    grid = synth.Grid(0.0, 2000.0, 200000)
    cond = dict(temperature=296.0, partition=2844.0, mean_mass=30.01, pressure=1.0)
    fr = grid.freq()
    ref = oracle.ref_cpu(oracle.DOPPLER, fr, np.zeros_like(fr), lines, cond, grid.dfreq,
                         nthreads=threads)
    got = run_engine(engine, capi.DOPPLER, lines, fr, cond, grid.dfreq, cuda,
                     convention=capi.CONV_CPU, cpu_threads=threads)
    assert_fp64_parity(got, ref)


@pytest.mark.parametrize("profile, convention, threads, pieces",
                         [(capi.DOPPLER, capi.CONV_GPU, 1, 4), (capi.DOPPLER, capi.CONV_CPU, 3, 7),
                          (capi.VOIGT, capi.CONV_CPU, 4, 5)])
def test_execute_host_matches_execute(engine, cuda, profile, convention, threads, pieces):
    """xs_engine_execute_host (host lines copied in slices that overlap step
    one) against xs_engine_execute on the same lines already on the device:
    bit-identical, including the CPU convention's coverage rule (the lines
    past the threads' blocks are copied but not evaluated)."""
    import torch

    lines = synth.exomol_like(2003, 3000, seed=6, nu_max=2000.0)
    grid = synth.Grid(0.0, 2000.0, 200000)
    cond = dict(temperature=296.0, partition=2844.0, mean_mass=30.01, pressure=1.0)
    fr = grid.freq()
    want = run_engine(engine, profile, lines, fr, cond, grid.dfreq, cuda, convention=convention,
                      cpu_threads=threads)
    host = {k: v.cpu().pin_memory() for k, v in to_device(lines, cuda).items()}
    dev = {k: torch.empty_like(v, device=cuda) for k, v in host.items()}
    dfr = torch.as_tensor(fr, device=cuda)
    out = torch.zeros((1, len(fr)), dtype=torch.float64, device=cuda)
    out_host = torch.full((1, len(fr)), -1.0, dtype=torch.float64).pin_memory()
    opts = capi.make_options(profile, grid.dfreq, cond["mean_mass"], convention=convention,
                             cpu_threads=threads)
    cc = [capi.make_condition(cond["temperature"], cond["partition"], 1.0, 1.0, -1.0)]
    engine.set_stream(torch.cuda.current_stream(cuda).cuda_stream)
    engine.execute_host(opts, cc, capi.make_lines(host), capi.make_lines(dev), capi.make_grid(dfr),
                        out.data_ptr(), len(fr), out_host.data_ptr(), pieces=pieces)
    engine.sync()
    for k in host:
        assert torch.equal(dev[k].cpu(), host[k])
    np.testing.assert_array_equal(out.cpu().numpy()[0], want[0] if want.ndim == 2 else want)
    np.testing.assert_array_equal(out_host.numpy()[0], want[0] if want.ndim == 2 else want)


def test_gaussian_vs_oracle(engine, cuda):
    lines, grid, cond = small_voigt_case(seed=9, n=2000)
    fr = grid.freq()
    hw = 0.05
    ref = oracle.gpu_convention(oracle.GAUSSIAN, fr, np.zeros_like(fr), lines,
                                dict(cond, half_width=hw), grid.dfreq)
    got = run_engine(engine, capi.GAUSSIAN, lines, fr, cond, grid.dfreq, cuda, half_width=hw)
    assert_fp64_parity(got, ref)


def test_chunk_accumulates_into_slice(engine, cuda):
    """ExecuteCrossSection(N, N_ener, start_idx) adds into [start, start+N)
    only, on top of what the grid holds (cross_kernal.cu:994)."""
    lines, grid, cond = small_voigt_case(seed=4, n=800)
    fr = grid.freq()
    rng = np.random.default_rng(1)
    init = rng.uniform(0, 1e-22, len(fr))
    start, pts = 2500, 4000
    ref = oracle.gpu_convention(oracle.VOIGT, fr, init, lines, cond, grid.dfreq, points=pts,
                                start_idx=start)
    got = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, start_idx=start,
                     points=pts, intens0=init)
    assert np.array_equal(got[:start], init[:start])
    assert np.array_equal(got[start + pts:], init[start + pts:])
    assert_fp64_parity(got, ref)


def test_mixed_precision_vs_fp64(engine, cuda):
    lines, grid, cond = small_voigt_case(seed=21, n=4000)
    fr = grid.freq()
    f64 = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda)
    mix = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, precision=capi.MIXED)
    assert_mixed_parity(mix, f64)


@pytest.mark.parametrize("p_bar", [1e-3, 1e-1, 10.0])
def test_mixed_precision_pressure_regimes(engine, cuda, p_bar):
    lines = synth.random_lines(3000, 1000.0, 1100.0, 2500.0, 1e-6, 1e2, seed=31,
                               pressure_atm=p_bar * synth.BAR_TO_ATM)
    grid = synth.Grid(990.0, 1110.0, 12000)
    for t in (300.0, 2100.0):
        cond = dict(temperature=t, partition=synth.partition_poly(t), mean_mass=17.03,
                    pressure=1.0, cut=25.0)
        fr = grid.freq()
        f64 = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda)
        mix = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda,
                         precision=capi.MIXED)
        assert_mixed_parity(mix, f64)


def test_multi_condition_batch_matches_single_runs(engine, cuda):
    """A batch of conditions gives each condition's single-run result (the
    multi-condition tiles sum in another fixed order: FP64 rounding only)."""
    lines, grid, cond = small_voigt_case(seed=41, n=1500)
    fr = grid.freq()
    conds = [dict(cond, temperature=t, partition=synth.partition_poly(t), gamma_scale=p, cut=25.0)
             for t in (300.0, 1200.0) for p in (0.01, 1.0, 5.0)]
    batch = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, conds=conds)
    again = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, conds=conds)
    assert np.array_equal(batch, again)  # deterministic
    for k, c in enumerate(conds):
        single = run_engine(engine, capi.VOIGT, lines, fr, c, grid.dfreq, cuda)
        assert_fp64_parity(batch[k], single, rel=1e-12)


@pytest.mark.parametrize("C", [2, 4])
def test_multi_condition_tiles_vs_oracle(engine, cuda, C):
    """Forced multi-condition tiles: FP64 against the oracle per condition,
    mixed against FP64, across Doppler- and pressure-dominated conditions."""
    lines = synth.random_lines(2500, 1000.0, 1100.0, 2500.0, 1e-6, 1e2, seed=51, pressure_atm=1.0)
    grid = synth.Grid(990.0, 1110.0, 1200)  # 0.1 cm-1, as in the sweep
    base = dict(mean_mass=17.03, pressure=1.0, ref_temp=296.0)
    conds = [dict(base, temperature=t, partition=synth.partition_poly(t), gamma_scale=p, cut=25.0)
             for t in (300.0, 2100.0) for p in (1e-3, 10.0)]
    fr = grid.freq()
    f64 = run_engine(engine, capi.VOIGT, lines, fr, base, grid.dfreq, cuda, conds=conds, C=C)
    mix = run_engine(engine, capi.VOIGT, lines, fr, base, grid.dfreq, cuda, conds=conds, C=C,
                     precision=capi.MIXED)
    for k, c in enumerate(conds):
        scaled = synth.LineList(lines.nu, lines.energies, lines.aif, lines.gns,
                                lines.gamma * c["gamma_scale"], lines.n)
        ref = oracle.gpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), scaled,
                                    dict(c, pressure=1.0), grid.dfreq)
        assert_fp64_parity(f64[k], ref)
        assert_mixed_parity(mix[k], f64[k])


@pytest.mark.parametrize("C", [1, 2, 4])
def test_multi_condition_mixed_edges(engine, cuda, C):
    """Mixed single- and multi-condition tiles against FP64 where the region
    intervals are clipped or replaced: lines centred beyond both grid ends, a grid
    chunk that starts inside the grid, and a grid fine enough (1e-6 cm-1)
    that the cores span more than 2^15 points and lines 20 cm-1 away lie
    more than 2^24 points from the grid's first point (pair-by-pair
    classification, offsets from the FP64 centre)."""
    base = dict(mean_mass=17.03, pressure=1.0, ref_temp=296.0)
    conds = [dict(base, temperature=t, partition=synth.partition_poly(t), gamma_scale=p, cut=25.0)
             for t in (300.0, 2100.0) for p in (1e-3, 1.0)]
    # 0.1 cm-1 grid; lines on both sides of it and across both ends
    lines = synth.random_lines(2000, 960.0, 1140.0, 2500.0, 1e-6, 1e2, seed=61, pressure_atm=1.0)
    grid = synth.Grid(990.0, 1110.0, 1200)
    fr = grid.freq()
    for start, points in ((0, None), (317, 611)):
        f64 = run_engine(engine, capi.VOIGT, lines, fr, base, grid.dfreq, cuda, conds=conds, C=C,
                         start_idx=start, points=points)
        mix = run_engine(engine, capi.VOIGT, lines, fr, base, grid.dfreq, cuda, conds=conds, C=C,
                         start_idx=start, points=points, precision=capi.MIXED)
        for k in range(len(conds)):
            assert_mixed_parity(mix[k], f64[k])
    # 1e-6 cm-1 grid over 0.05 cm-1: cores of +-0.2 cm-1 (2e5 points); the
    # lines at 1020 cm-1 reach it through the 25 cm-1 cut from 2e7 points away
    near = synth.random_lines(60, 999.98, 1000.07, 2500.0, 1e-3, 1e2, seed=62, pressure_atm=1.0)
    far = synth.random_lines(20, 1020.0, 1020.5, 2500.0, 1e-3, 1e2, seed=63, pressure_atm=1.0)
    both = synth.LineList(*(np.concatenate([getattr(near, f), getattr(far, f)])
                            for f in ("nu", "energies", "aif", "gns", "gamma", "n")))
    fine = synth.Grid(1000.0, 1000.05, 50001)
    ff = fine.freq()
    f64 = run_engine(engine, capi.VOIGT, both, ff, base, fine.dfreq, cuda, conds=conds, C=C)
    mix = run_engine(engine, capi.VOIGT, both, ff, base, fine.dfreq, cuda, conds=conds, C=C,
                     precision=capi.MIXED)
    for k in range(len(conds)):
        assert_mixed_parity(mix[k], f64[k])


@pytest.mark.parametrize("profile,precision,C", [
    (capi.VOIGT, capi.FP64, 0), (capi.VOIGT, capi.FP64, 2), (capi.VOIGT, capi.MIXED, 1),
    (capi.VOIGT, capi.MIXED, 8), (capi.DOPPLER, capi.FP64, 0), (capi.GAUSSIAN, capi.FP64, 0)])
def test_empty_and_outside_lines(engine, cuda, profile, precision, C):
    """No lines, and lines whose windows miss the grid (beyond it on either
    side): every kernel path leaves the grid exactly zero."""
    lines, grid, cond = small_voigt_case(seed=2, n=100)
    fr = grid.freq()
    conds = None
    if C > 1:
        conds = [dict(cond, temperature=t, partition=synth.partition_poly(t), gamma_scale=g)
                 for t in (500.0, 1500.0) for g in ((0.01, 1.0, 10.0, 100.0) if C == 8 else (1.0,))]
    kw = dict(precision=precision, conds=conds, C=C)
    got = run_engine(engine, profile, lines.slice(0, 0), fr, cond, grid.dfreq, cuda, **kw)
    assert not np.asarray(got).any()
    above = synth.random_lines(100, 5000.0, 5100.0, 2500.0, 1e-6, 1e2, seed=2)
    below = synth.random_lines(100, 100.0, 200.0, 2500.0, 1e-6, 1e2, seed=3)
    for far in (above, below):
        got = run_engine(engine, profile, far, fr, cond, grid.dfreq, cuda, **kw)
        assert not np.asarray(got).any()


def test_unsorted_lines_are_reported(engine, cuda):
    lines, grid, cond = small_voigt_case(seed=2, n=200)
    rev = synth.LineList(*(a[::-1].copy() for a in (lines.nu, lines.energies, lines.aif,
                                                      lines.gns, lines.gamma, lines.n)))
    with pytest.raises(capi.XsError) as ei:
        run_engine(engine, capi.VOIGT, rev, grid.freq(), cond, grid.dfreq, cuda)
    assert ei.value.code == capi.XS_ERR_UNSORTED


@pytest.mark.parametrize("C", [1, 2])
def test_unreachable_core_is_reported_in_mixed(engine, cuda, C):
    """A grid so fine (5e-10 cm-1) that a line's core reaches it from 4e7
    grid points away: the mixed core pass finds lines by the grid index of
    their centre within a bounded reach, so the engine reports
    XS_ERR_UNSUPPORTED instead of leaving those pairs out; FP64 computes it."""
    grid = synth.Grid(1000.0, 1000.0 + 1000 * 5e-10, 1000)
    line = synth.random_lines(1, 999.98, 999.98 + 1e-9, 100.0, 1.0, 1.0001, seed=5)
    conds = [dict(temperature=2000.0, partition=synth.partition_poly(2000.0), mean_mass=17.03,
                  pressure=1.0, cut=25.0, gamma_scale=s) for s in (1e-4, 2e-4)]
    f64 = run_engine(engine, capi.VOIGT, line, grid.freq(), conds[0], grid.dfreq, cuda,
                     conds=conds, C=C if C > 1 else 0)
    assert np.all(f64 > 0.0)
    with pytest.raises(capi.XsError) as ei:
        run_engine(engine, capi.VOIGT, line, grid.freq(), conds[0], grid.dfreq, cuda,
                   conds=conds, C=C if C > 1 else 1, precision=capi.MIXED)
    assert ei.value.code == capi.XS_ERR_UNSUPPORTED


def test_bad_arguments_rejected(engine, cuda):
    lines, grid, cond = small_voigt_case(seed=2, n=10)
    with pytest.raises(capi.XsError) as ei:
        run_engine(engine, capi.PSUEDO_VOIGT, lines, grid.freq(), cond, grid.dfreq, cuda)
    assert ei.value.code == capi.XS_ERR_UNSUPPORTED
    with pytest.raises(capi.XsError):
        run_engine(engine, capi.VOIGT, lines, grid.freq(), cond, grid.dfreq, cuda, P=3)


def test_device_erf_saturates_where_pairs_are_skipped(cuda):
    """Doppler/Gaussian pairs whose erf arguments are both beyond 6 on one
    side are skipped as exact zeros: the device erf must return exactly +-1
    there."""
    import torch

    x = torch.linspace(6.0, 40.0, 2_000_001, dtype=torch.float64, device=cuda)
    assert bool((torch.erf(x) == 1.0).all())
    assert bool((torch.erf(-x) == -1.0).all())


# --- against the reference's own kernels (cross_kernal.cu for sm_100a) -------

def test_voigt_vs_reference_gpu_kernels(engine, cuda):
    lines, grid, cond = small_voigt_case(seed=13)
    fr = grid.freq()
    ref, _ = oracle.ref_gpu(oracle.VOIGT, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    got = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda)
    assert_fp64_parity(got, ref)
    # and the oracle restatement of those kernels agrees with them
    orc = oracle.gpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    assert_fp64_parity(orc, ref)


def test_doppler_vs_reference_gpu_kernels(engine, cuda):
    lines = synth.exomol_like(2000, 4000, seed=15, nu_max=3000.0)
    grid = synth.Grid(0.0, 3000.0, 300000)
    cond = dict(temperature=296.0, partition=2844.0, mean_mass=30.01, pressure=1.0)
    fr = grid.freq()
    ref, _ = oracle.ref_gpu(oracle.DOPPLER, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    got = run_engine(engine, capi.DOPPLER, lines, fr, cond, grid.dfreq, cuda)
    assert_fp64_parity(got, ref)


# --- launcher level (cross_kernal.cuh drop-in) -------------------------------

def test_launcher_level_voigt(cuda):
    import torch

    lines, grid, cond = small_voigt_case(seed=17, n=1200)
    fr = grid.freq()
    d = to_device(lines, cuda)
    dfr = torch.as_tensor(fr, device=cuda)
    out = torch.zeros_like(dfr)
    c = capi.CrossSectionData()
    c.halfwidth = 0.1
    c.mean_mass = cond["mean_mass"]
    c.temperature = cond["temperature"]
    c.pressure = cond["pressure"]
    c.partition = cond["partition"]
    c.ref_temp = cond["ref_temp"]
    c.dfreq = grid.dfreq
    c.beta = 6.6260693e-27 * 2.99792458e10 / (1.380658e-16 * cond["temperature"])
    c.cmcoef = 1.0 / (8.0 * np.arccos(-1.0) * 2.99792458e10)
    L = capi.lib()
    capi.check(L.xs_copy_intensity_info(c))
    torch.cuda.synchronize()
    capi.check(L.xs_execute_two_step_kernal_voigt_block(
        dfr.data_ptr(), out.data_ptr(), d["energies"].data_ptr(), d["nu"].data_ptr(),
        d["gns"].data_ptr(), d["aif"].data_ptr(), d["gamma"].data_ptr(), d["n"].data_ptr(),
        len(fr), len(lines), 0))
    capi.check(L.xs_launcher_sync())
    ref = oracle.gpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    assert_fp64_parity(out.cpu().numpy(), ref)
    # inputs are left as uploaded (the reference overwrote E'' and gamma)
    assert np.array_equal(d["energies"].cpu().numpy(), lines.energies)


# --- manager level (BaseManager over host buffers) ---------------------------

def _manager_run(kind, profile, lines, grid, cond, threads=1, chunks=1, precision=capi.FP64):
    m = capi.Manager(kind, profile, 0, threads, 4_000_000_000)
    m.set_precision(precision)
    fr = grid.freq()
    intens = np.zeros_like(fr)
    m.InitializeVectors(len(fr))
    m.TransferFreq(fr, intens, len(fr))
    m.InitializeConstants(0.1, cond["temperature"], cond["partition"], grid.dfreq,
                          cond["mean_mass"], cond["pressure"], cond.get("ref_temp", 296.0))
    n = len(lines)
    per = (n + chunks - 1) // chunks
    cut = min(25.0 * cond["pressure"], 100.0) if profile == capi.VOIGT else 100.0
    for k in range(chunks):
        part = lines.slice(k * per, min(n, (k + 1) * per))
        if len(part) == 0:
            continue
        m.TransferVectors(len(part), part.energies, part.nu, part.aif, part.gns,
                          part.gamma if profile == capi.VOIGT else None,
                          part.n if profile == capi.VOIGT else None)
        # BaseProfile::PerformCrossSection (BaseProfile.cpp:55-57)
        ib = int(max(round((part.nu.min() - cut - fr[0]) / grid.dfreq), 0.0))
        ie = int(min(round((part.nu.max() + cut - fr[0]) / grid.dfreq), float(len(fr))))
        m.ExecuteCrossSection(ie - ib, len(part), ib)
    out_f = np.zeros_like(fr)
    out = np.zeros_like(fr)
    m.TransferResults(out_f, out, len(fr))
    m.close()
    return out, out_f


def test_gpumanager_chunked_vs_oracle(cuda):
    lines, grid, cond = small_voigt_case(seed=19, n=3000)
    got, got_f = _manager_run(0, capi.VOIGT, lines, grid, cond, chunks=3)
    fr = grid.freq()
    assert np.array_equal(got_f, fr)
    # chunks cut off wings at chunk edges exactly as the reference's chunked
    # run does; compare chunk by chunk through the oracle
    per = 1000
    ref = np.zeros_like(fr)
    for k in range(3):
        part = lines.slice(k * per, (k + 1) * per)
        ib = int(max(round((part.nu[0] - 25.0 - fr[0]) / grid.dfreq), 0.0))
        ie = int(min(round((part.nu[-1] + 25.0 - fr[0]) / grid.dfreq), float(len(fr))))
        ref = oracle.gpu_convention(oracle.VOIGT, fr, ref, part, cond, grid.dfreq,
                                    points=ie - ib, start_idx=ib)
    assert_fp64_parity(got, ref)


def test_openmpmanager_semantics_on_gpu_vs_reference(cuda):
    lines, grid, cond = small_voigt_case(seed=23, n=2500)
    got, _ = _manager_run(1, capi.VOIGT, lines, grid, cond, threads=4)
    fr = grid.freq()
    ref = oracle.ref_cpu(oracle.VOIGT, fr, np.zeros_like(fr), lines, cond, grid.dfreq, nthreads=4)
    assert_fp64_parity(got, ref)


def test_manager_sorts_unsorted_chunk(cuda):
    lines, grid, cond = small_voigt_case(seed=29, n=800)
    rng = np.random.default_rng(0)
    perm = rng.permutation(len(lines))
    shuffled = synth.LineList(*(a[perm].copy() for a in (lines.nu, lines.energies, lines.aif,
                                                           lines.gns, lines.gamma, lines.n)))
    a, _ = _manager_run(0, capi.VOIGT, lines, grid, cond)
    b, _ = _manager_run(0, capi.VOIGT, shuffled, grid, cond)
    assert_fp64_parity(b, a, rel=1e-13)


def test_graph_replay_matches_execute(engine, cuda):
    """A captured sweep replays to the same grids as a direct execute, and
    the step timings are readable both ways."""
    import torch

    lines, grid, cond = small_voigt_case(seed=43, n=1500)
    fr = grid.freq()
    d = to_device(lines, cuda)
    dfr = torch.as_tensor(fr, device=cuda)
    conds = [capi.make_condition(t, synth.partition_poly(t), 1.0, p, 25.0)
             for t in (500.0, 1500.0) for p in (0.1, 2.0)]
    opts = capi.make_options(capi.VOIGT, grid.dfreq, 17.03, precision=capi.MIXED)
    stream = torch.cuda.current_stream(cuda)
    engine.set_stream(stream.cuda_stream)
    direct = torch.zeros((len(conds), len(fr)), dtype=torch.float64, device=cuda)
    engine.execute(opts, conds, capi.make_lines(d), capi.make_grid(dfr), direct.data_ptr(), len(fr))
    engine.sync()
    prep_ms, step_ms = engine.last_stats()
    assert prep_ms > 0 and step_ms > 0
    replay = torch.full_like(direct, 7.0)
    g = engine.capture(opts, conds, capi.make_lines(d), capi.make_grid(dfr), replay.data_ptr(),
                       len(fr), zero_out=True)
    try:
        for _ in range(2):  # zero_out makes every replay start from 0
            g.launch(stream.cuda_stream)
            engine.sync()
            assert torch.equal(replay, direct)
            assert engine.last_stats()[1] > 0
        # grid check, step one, step two, the core pass (+ the split reduction)
        assert g.kernel_count() in (4, 5)
    finally:
        g.close()
    one = capi.make_options(capi.VOIGT, grid.dfreq, 17.03, precision=capi.MIXED, line_splits=1)
    two = capi.make_options(capi.VOIGT, grid.dfreq, 17.03, precision=capi.MIXED, line_splits=2)
    f64 = capi.make_options(capi.VOIGT, grid.dfreq, 17.03, line_splits=1, conditions_per_warp=1)
    for o, kernels in ((one, 4), (two, 5), (f64, 3)):
        g = engine.capture(o, conds, capi.make_lines(d), capi.make_grid(dfr), replay.data_ptr(), len(fr),
                           zero_out=True)
        try:
            assert g.kernel_count() == kernels
        finally:
            g.close()


def test_autotune_picks_a_shape_later_calls_use(engine, cuda, tmp_path):
    import torch

    lines, grid, cond = small_voigt_case(seed=21, n=2000)
    fr = grid.freq()
    dev = to_device(lines, cuda)
    dfr = torch.as_tensor(fr, device=cuda)
    out = torch.zeros(len(fr), dtype=torch.float64, device=cuda)
    opts = capi.make_options(capi.VOIGT, grid.dfreq, cond["mean_mass"], precision=capi.MIXED)
    cc = [capi.make_condition(cond["temperature"], cond["partition"], 1.0, 1.0, -1.0)]
    engine.set_stream(torch.cuda.current_stream(cuda).cuda_stream)
    capi.lib().xs_tune_clear()
    best = engine.autotune(opts, cc, capi.make_lines(dev), capi.make_grid(dfr), out.data_ptr())
    assert best["candidates"] >= 8 and best["ms"] > 0
    assert best["points_per_thread"] in (1, 2, 4, 8) and best["warps_per_block"] in (4, 8)
    auto = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, precision=capi.MIXED)
    explicit = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, precision=capi.MIXED,
                          P=best["points_per_thread"], W=best["warps_per_block"],
                          C=best["conditions_per_warp"])
    assert np.array_equal(auto, explicit)
    path = str(tmp_path / "shapes.txt").encode()
    capi.check(capi.lib().xs_tune_save(path))
    capi.lib().xs_tune_clear()
    capi.check(capi.lib().xs_tune_load(path))
    again = run_engine(engine, capi.VOIGT, lines, fr, cond, grid.dfreq, cuda, precision=capi.MIXED)
    assert np.array_equal(auto, again)
    capi.lib().xs_tune_clear()
