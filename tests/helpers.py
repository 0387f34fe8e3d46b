"""Shared helpers for the parity tests: run the engine on torch CUDA buffers
and compare against the oracle with the tolerances of the accuracy tiers."""
from __future__ import annotations

import numpy as np

from gpu_cross_b200 import capi, synth

# Tier 1/2: plain FP64 vs the reference backends.
FP64_REL = 1e-10
# Tier 3: mixed precision vs FP64, on points above 1e-6 of the peak, and the
# integrated cross-section.
MIXED_REL = 1e-4
MIXED_INTEGRATED = 1e-6
PEAK_FLOOR = 1e-6


def parity_errors(got: np.ndarray, ref: np.ndarray, floor: float = PEAK_FLOOR):
    """(max relative error on points above floor*peak,
        max absolute error elsewhere / peak,
        relative error of the integral)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    peak = float(np.max(np.abs(ref))) if ref.size else 0.0
    if peak == 0.0:
        return 0.0, float(np.max(np.abs(got))) if got.size else 0.0, 0.0
    big = np.abs(ref) > floor * peak
    rel = float(np.max(np.abs(got[big] - ref[big]) / np.abs(ref[big]))) if big.any() else 0.0
    small = ~big
    ab = float(np.max(np.abs(got[small] - ref[small])) / peak) if small.any() else 0.0
    integ = abs(float(np.sum(got)) - float(np.sum(ref))) / abs(float(np.sum(ref)))
    return rel, ab, integ


def assert_fp64_parity(got, ref, rel=FP64_REL):
    r, a, _ = parity_errors(got, ref)
    assert r <= rel and a <= rel, f"FP64 parity: rel {r:.3e} abs/peak {a:.3e} (bound {rel})"


def assert_mixed_parity(got, ref):
    r, a, i = parity_errors(got, ref)
    assert r <= MIXED_REL, f"mixed: max rel {r:.3e} > {MIXED_REL}"
    assert i <= MIXED_INTEGRATED, f"mixed: integrated rel {i:.3e} > {MIXED_INTEGRATED}"
    assert a <= MIXED_REL, f"mixed: abs/peak below the floor {a:.3e}"


def to_device(lines, device):
    import torch

    return dict(
        nu=torch.as_tensor(np.ascontiguousarray(lines.nu), device=device),
        energies=torch.as_tensor(np.ascontiguousarray(lines.energies), device=device),
        aif=torch.as_tensor(np.ascontiguousarray(lines.aif), device=device),
        gns=torch.as_tensor(np.ascontiguousarray(lines.gns, dtype=np.int32), device=device),
        gamma=torch.as_tensor(np.ascontiguousarray(lines.gamma), device=device),
        n=torch.as_tensor(np.ascontiguousarray(lines.n), device=device),
    )


def run_engine(engine: capi.Engine, profile: int, lines, freq: np.ndarray, cond: dict, dfreq: float,
               device, convention=capi.CONV_GPU, precision=capi.FP64, cpu_threads=1,
               start_idx=0, points=None, intens0=None, half_width=0.1, P=0, W=0,
               conds: list[dict] | None = None, C=0, S=0):
    """Run the engine once; returns the grid(s) as numpy."""
    import torch

    dev = to_device(lines, device)
    fr = torch.as_tensor(np.ascontiguousarray(freq), device=device)
    clist = conds if conds is not None else [cond]
    npts = len(freq)
    out = torch.zeros((len(clist), npts), dtype=torch.float64, device=device)
    if intens0 is not None:
        out[:] = torch.as_tensor(intens0, device=device)
    opts = capi.make_options(profile, dfreq, cond["mean_mass"], convention=convention,
                             precision=precision, cpu_threads=cpu_threads,
                             ref_temp=cond.get("ref_temp", 296.0), half_width=half_width,
                             points_per_thread=P, warps_per_block=W, conditions_per_warp=C,
                             line_splits=S)
    cc = [capi.make_condition(c["temperature"], c["partition"], c.get("pressure", 1.0),
                              c.get("gamma_scale", 1.0), c.get("cut", -1.0)) for c in clist]
    grid = capi.make_grid(fr, start_idx, points)
    engine.set_stream(torch.cuda.current_stream(device).cuda_stream)
    engine.execute(opts, cc, capi.make_lines(dev), grid, int(out.data_ptr()), npts)
    engine.sync()
    res = out.cpu().numpy()
    return res if conds is not None else res[0]


def small_voigt_case(seed=7, n=3000, nu_lo=1000.0, nu_hi=1100.0, pressure_atm=1.0):
    lines = synth.random_lines(n, nu_lo, nu_hi, 2500.0, 1e-6, 1e2, seed=seed,
                               pressure_atm=pressure_atm)
    grid = synth.Grid(nu_lo - 10.0, nu_hi + 10.0, int(round((nu_hi - nu_lo + 20.0) / 0.01)))
    cond = dict(temperature=1000.0, partition=synth.partition_poly(1000.0), mean_mass=17.03,
                pressure=1.0, ref_temp=296.0)
    return lines, grid, cond
