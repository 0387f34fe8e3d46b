"""The allocation-free entry point (xs_execute_noalloc) against the regular
engine entry point (xs_engine_execute), through the C ABI.

xs_execute_noalloc serves callers that cannot let the library allocate device
memory (a host whose own pool already holds the device's memory, or a
latency-critical loop that cannot take cudaMalloc's synchronisation); it runs
the same kernels with a fixed scratch array compiled into the library.  This
file is collected last so that a stop-at-first-failure run has already run
every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from gpu_cross_b200 import capi, synth

from helpers import FP64_REL, MIXED_REL, parity_errors, to_device

pytestmark = pytest.mark.gpu


def _call_noalloc(opts, cond, lines, grid, out, stream):
    rc = capi.lib().xs_execute_noalloc(ctypes.byref(opts), ctypes.byref(cond), ctypes.byref(lines),
                                       ctypes.byref(grid), out.data_ptr(), stream)
    capi.check(rc)


def _case(seed, n, temperature, p_atm):
    lines = synth.random_lines(n, 1000.0, 1100.0, 2500.0, 1e-6, 1e2, seed=seed,
                               pressure_atm=p_atm)
    grid = synth.Grid(990.0, 1110.0, 12000)
    cond = capi.make_condition(temperature, synth.partition_poly(temperature), 1.0, 1.0, 25.0)
    return lines, grid, cond


@pytest.mark.parametrize("precision,bound", [(capi.FP64, FP64_REL), (capi.MIXED, MIXED_REL)])
def test_noalloc_matches_engine_two_calls_in_a_row(cuda, precision, bound):
    import torch

    stream = torch.cuda.current_stream(cuda)
    eng = capi.Engine(0)
    eng.set_stream(stream.cuda_stream)
    try:
        cases = []
        for seed, n, t, p in ((101, 5000, 1000.0, 1.0), (202, 3000, 400.0, 0.2)):
            lines, grid, cond = _case(seed, n, t, p)
            d = to_device(lines, cuda)
            fr = torch.as_tensor(grid.freq(), device=cuda)
            opts = capi.make_options(capi.VOIGT, grid.dfreq, 17.03, precision=precision)
            L = capi.make_lines(d)
            G = capi.make_grid(fr)
            ref = torch.zeros_like(fr)
            eng.execute(opts, [cond], L, G, ref.data_ptr())
            eng.sync()
            cases.append((d, fr, opts, cond, L, G, ref))
        # Two consecutive no-alloc calls with different inputs: the second
        # must not see anything the first left in the shared scratch array.
        outs = []
        for d, fr, opts, cond, L, G, ref in cases:
            got = torch.zeros_like(fr)
            _call_noalloc(opts, cond, L, G, got, stream.cuda_stream)
            outs.append(got)
        for (d, fr, opts, cond, L, G, ref), got in zip(cases, outs):
            r, a, _ = parity_errors(got.cpu().numpy(), ref.cpu().numpy())
            assert r <= bound and a <= bound, (r, a)
    finally:
        eng.close()


# (profile, convention, precision): the other branches of the entry point --
# the erf profiles and the CPU convention, whose line coverage rule trims the
# list and whose mixed core pass runs without line splits.
OTHER_BRANCHES = [
    (capi.DOPPLER, capi.CONV_GPU, capi.FP64),
    (capi.DOPPLER, capi.CONV_CPU, capi.FP64),
    (capi.GAUSSIAN, capi.CONV_GPU, capi.FP64),
    (capi.VOIGT, capi.CONV_CPU, capi.FP64),
    (capi.VOIGT, capi.CONV_CPU, capi.MIXED),
]


@pytest.mark.parametrize("profile,convention,precision", OTHER_BRANCHES)
def test_noalloc_other_branches_match_engine(cuda, profile, convention, precision):
    import torch

    stream = torch.cuda.current_stream(cuda)
    eng = capi.Engine(0)
    eng.set_stream(stream.cuda_stream)
    bound = MIXED_REL if precision == capi.MIXED else FP64_REL
    try:
        cases = []
        for seed, n, t, p in ((303, 4000, 800.0, 1.0), (404, 2500, 1500.0, 0.3)):
            lines, grid, cond = _case(seed, n, t, p)
            d = to_device(lines, cuda)
            fr = torch.as_tensor(grid.freq(), device=cuda)
            opts = capi.make_options(profile, grid.dfreq, 17.03, convention=convention,
                                     precision=precision, cpu_threads=3, half_width=0.05)
            L = capi.make_lines(d)
            G = capi.make_grid(fr)
            ref = torch.zeros_like(fr)
            eng.execute(opts, [cond], L, G, ref.data_ptr())
            eng.sync()
            cases.append((d, fr, opts, cond, L, G, ref))  # d keeps the line arrays alive
        outs = []
        for d, fr, opts, cond, L, G, ref in cases:
            got = torch.zeros_like(fr)
            _call_noalloc(opts, cond, L, G, got, stream.cuda_stream)
            outs.append(got)
        for (d, fr, opts, cond, L, G, ref), got in zip(cases, outs):
            want = ref.cpu().numpy()
            assert np.abs(want).max() > 0.0
            r, a, _ = parity_errors(got.cpu().numpy(), want)
            assert r <= bound and a <= bound, (r, a)
    finally:
        eng.close()


def test_noalloc_rejects_oversize_before_device_work(cuda):
    import torch

    lines, grid, cond = _case(7, 100, 1000.0, 1.0)
    d = to_device(lines, cuda)
    fr = torch.as_tensor(grid.freq(), device=cuda)
    out = torch.zeros_like(fr)
    opts = capi.make_options(capi.VOIGT, grid.dfreq, 17.03)
    too_many = capi.make_lines(d, count=10_000_000)  # never read: rejected on size
    with pytest.raises(capi.XsError) as ei:
        _call_noalloc(opts, cond, too_many, capi.make_grid(fr), out,
                      torch.cuda.current_stream(cuda).cuda_stream)
    assert ei.value.code == capi.XS_ERR_INVALID
    assert "fixed array" in str(ei.value)
    assert not out.any()
