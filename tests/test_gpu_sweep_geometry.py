"""The timed launch shapes on the benchmark geometry, through the C ABI.

* The 40-condition sweep (T 300..2100 K x P {1e-3, 0.1, 1, 10} bar) on the
  sweep's own grid -- 500-8000 cm-1 at 0.1 cm-1, 7.5e4 points, cut 25 -- with
  1e5 lines from the sweep's generator, at 8 conditions per warp and 4 or 8
  warps per block (the shapes the autotuner picks for the benchmark):
  mixed against the engine's FP64 for all 40 conditions (<= 1e-4 relative
  above 1e-6 of the peak, integrated within 1e-6), and FP64 and mixed against
  the oracle for the four corner conditions (FP64 <= 1e-10).
* The single-point configuration reduced to 1e5 lines (grid 500-8000 cm-1 at
  0.01 cm-1, 7.5e5 points, T 1000 K, P 1 bar): the engine's FP64 against the
  reference's own cross_kernal.cu (cross_kernal.cu:924-997) built for sm_100a,
  over the same line chunks and grid slices as BaseProfile feeds it
  (BaseProfile.cpp:55-57, MAX-POINTS 80000), <= 1e-10; and mixed against
  FP64.
"""
import numpy as np
import pytest

import oracle
from gpu_cross_b200 import capi, synth

from helpers import assert_fp64_parity, assert_mixed_parity, to_device

pytestmark = pytest.mark.gpu

N_LINES = 100_000


@pytest.fixture(scope="module")
def sweep(cuda):
    import torch

    lines, grid, conds, common = synth.voigt_sweep_workload(N_LINES, 75_000)
    fr = grid.freq()
    d = to_device(lines, cuda)
    dfr = torch.as_tensor(fr, device=cuda)
    cc = [capi.make_condition(c["temperature"], c["partition"], 1.0, c["pressure_atm"], c["cut"])
          for c in conds]
    return lines, grid, conds, common, fr, d, dfr, cc


def _run(eng, cuda, sweep, precision, C, W):
    import torch

    lines, grid, conds, common, fr, d, dfr, cc = sweep
    out = torch.zeros((len(conds), len(fr)), dtype=torch.float64, device=cuda)
    opts = capi.make_options(capi.VOIGT, grid.dfreq, common["mean_mass"], precision=precision,
                             ref_temp=common["ref_temp"], warps_per_block=W, conditions_per_warp=C)
    eng.set_stream(torch.cuda.current_stream(cuda).cuda_stream)
    eng.execute(opts, cc, capi.make_lines(d), capi.make_grid(dfr), out.data_ptr(), len(fr))
    eng.sync()
    return out.cpu().numpy()


CORNERS = [0, 3, 36, 39]  # (300 K, 1e-3 bar), (300 K, 10 bar), (2100 K, 1e-3 bar), (2100 K, 10 bar)


@pytest.mark.parametrize("W", [4, 8])
def test_sweep_eight_conditions_per_warp(cuda, sweep, W):
    lines, grid, conds, common, fr, d, dfr, cc = sweep
    eng = capi.Engine(0)
    try:
        f64 = _run(eng, cuda, sweep, capi.FP64, 2, 4)
        mix = _run(eng, cuda, sweep, capi.MIXED, 8, W)
        again = _run(eng, cuda, sweep, capi.MIXED, 8, W)
    finally:
        eng.close()
    assert np.array_equal(mix, again)  # fixed summation order
    for k in range(len(conds)):
        assert np.abs(f64[k]).max() > 0.0
        assert_mixed_parity(mix[k], f64[k])
    for k in CORNERS:
        c = conds[k]
        scaled = synth.LineList(lines.nu, lines.energies, lines.aif, lines.gns,
                                lines.gamma * c["pressure_atm"], lines.n)
        cond = dict(temperature=c["temperature"], partition=c["partition"],
                    mean_mass=common["mean_mass"], pressure=1.0, ref_temp=common["ref_temp"],
                    cut=c["cut"])
        ref = oracle.gpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), scaled, cond, grid.dfreq)
        assert_fp64_parity(f64[k], ref)
        assert_mixed_parity(mix[k], ref)


def test_single_point_reduced_vs_reference_kernel(cuda):
    import torch

    lines, grid, cond = synth.voigt_single_workload(N_LINES, 750_000)
    fr = grid.freq()
    c = dict(temperature=cond["temperature"], partition=cond["partition"],
             mean_mass=cond["mean_mass"], pressure=1.0, ref_temp=cond["ref_temp"])
    # BaseProfile's chunking: equal consecutive line chunks, each over the
    # grid slice its lines reach, at most MAX-POINTS (80000) points
    span_pts = (lines.nu[-1] - lines.nu[0]) / grid.dfreq + 2 * 25.0 / grid.dfreq
    chunks = max(1, int(np.ceil(span_pts / 80000.0)))
    ref, _ = oracle.ref_gpu(oracle.VOIGT, fr, np.zeros_like(fr), lines, c, grid.dfreq,
                            chunks=chunks)

    d = to_device(lines, cuda)
    dfr = torch.as_tensor(fr, device=cuda)
    eng = capi.Engine(0)
    outs = {}
    try:
        eng.set_stream(torch.cuda.current_stream(cuda).cuda_stream)
        cc = [capi.make_condition(cond["temperature"], cond["partition"], 1.0, 1.0, -1.0)]
        for prec in (capi.FP64, capi.MIXED):
            out = torch.zeros_like(dfr)
            opts = capi.make_options(capi.VOIGT, grid.dfreq, cond["mean_mass"], precision=prec,
                                     ref_temp=cond["ref_temp"])
            n = len(lines)
            per = (n + chunks - 1) // chunks
            for k in range(chunks):
                a, b = k * per, min(n, (k + 1) * per)
                if b <= a:
                    break
                ib = int(max(np.round((lines.nu[a] - 25.0 - fr[0]) / grid.dfreq), 0.0))
                ie = int(min(np.round((lines.nu[b - 1] + 25.0 - fr[0]) / grid.dfreq), float(len(fr))))
                if chunks == 1:
                    ib, ie = 0, len(fr)
                if ie <= ib:
                    continue
                dk = {key: v[a:b] for key, v in d.items()}
                eng.execute(opts, cc, capi.make_lines(dk), capi.make_grid(dfr, ib, ie - ib),
                            out.data_ptr())
            eng.sync()
            outs[prec] = out.cpu().numpy()
    finally:
        eng.close()
    assert chunks > 1
    assert_fp64_parity(outs[capi.FP64], ref)
    assert_mixed_parity(outs[capi.MIXED], outs[capi.FP64])


@pytest.mark.parametrize("precision, C, pieces", [(capi.MIXED, 8, 8), (capi.FP64, 2, 5), (capi.MIXED, 1, 3)])
def test_execute_host_matches_execute(cuda, sweep, precision, C, pieces):
    """xs_engine_execute_host (pinned host lines copied in slices that overlap
    step one, result copied back) gives the bit-identical result of
    xs_engine_execute on the same lines already on the device."""
    import torch

    lines, grid, conds, common, fr, d, dfr, cc = sweep
    if C == 1:
        cc = cc[:1]
    nc = len(cc)
    opts = capi.make_options(capi.VOIGT, grid.dfreq, common["mean_mass"], precision=precision,
                             ref_temp=common["ref_temp"], warps_per_block=4, conditions_per_warp=C)
    stream = torch.cuda.current_stream(cuda)
    eng = capi.Engine(cuda.index)
    try:
        eng.set_stream(stream.cuda_stream)
        want = torch.zeros((nc, len(fr)), dtype=torch.float64, device=cuda)
        eng.execute(opts, cc, capi.make_lines(d), capi.make_grid(dfr), want.data_ptr(), len(fr))
        eng.sync()
        host = {k: torch.from_numpy(np.ascontiguousarray(getattr(lines, k))).pin_memory()
                for k in ("nu", "energies", "aif", "gns", "gamma", "n")}
        dev = {k: torch.empty_like(v, device=cuda) for k, v in host.items()}  # filled by the call
        out = torch.zeros_like(want)
        out_host = torch.full((nc, len(fr)), -1.0, dtype=torch.float64).pin_memory()
        eng.execute_host(opts, cc, capi.make_lines(host), capi.make_lines(dev), capi.make_grid(dfr),
                         out.data_ptr(), len(fr), out_host.data_ptr(), pieces=pieces)
        eng.sync()
    finally:
        eng.close()
    for k in host:
        assert torch.equal(dev[k].cpu(), host[k])
    np.testing.assert_array_equal(out.cpu().numpy(), want.cpu().numpy())
    np.testing.assert_array_equal(out_host.numpy(), want.cpu().numpy())
