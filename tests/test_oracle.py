"""The oracle, pinned against the reference (CPU-only tests).

* the CPU-convention restatement is bit-identical to the reference's own
  OpenMPManager: against the committed golden fixtures and, where the
  reference build is present, against it live;
* the GPU-convention restatement matches the golden fixtures made by the
  reference's own kernels on a B200;
* known-answer properties: Doppler bins telescope to 2 per line, the Voigt
  integral, the Humlicek W4 error envelope against scipy's Faddeeva function.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from gpu_cross_b200 import synth

from helpers import assert_fp64_parity

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(path):
    z = np.load(path)
    lines = synth.LineList(z["nu"], z["energies"], z["aif"], z["gns"], z["gamma"], z["n"])
    g = z["grid"]
    grid = synth.Grid(float(g[0]), float(g[1]), int(g[2]))
    cond = dict(temperature=float(z["temperature"]), partition=float(z["partition"]),
                mean_mass=float(z["mean_mass"]), pressure=float(z["pressure"]),
                ref_temp=float(z["ref_temp"]))
    return z, lines, grid, cond, int(z["profile"])


CPU_FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.cpu.npz")))
GPU_FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.gpu.npz")))


def test_fixtures_present():
    assert len(CPU_FIXTURES) >= 4


@pytest.mark.parametrize("path", CPU_FIXTURES, ids=os.path.basename)
def test_cpu_convention_bit_identical_to_reference_fixture(built_libs, path):
    z, lines, grid, cond, prof = _load(path)
    fr = grid.freq()
    for thr in (1, 4):
        got = oracle.cpu_convention(prof, fr, np.zeros_like(fr), lines, cond, grid.dfreq,
                                    nthreads=thr)
        assert np.array_equal(got, z[f"ref_cpu_t{thr}"]), f"threads={thr}"


@pytest.mark.parametrize("path", GPU_FIXTURES, ids=os.path.basename)
def test_gpu_convention_matches_reference_kernels_fixture(built_libs, path):
    z, lines, grid, cond, prof = _load(path)
    fr = grid.freq()
    got = oracle.gpu_convention(prof, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    assert_fp64_parity(got, z["ref_gpu"])


@pytest.mark.skipif(not os.path.exists(oracle.LIB_REF_CPU), reason="reference CPU build absent")
@pytest.mark.parametrize("profile", [oracle.VOIGT, oracle.DOPPLER])
@pytest.mark.parametrize("threads", [1, 2, 5])
@pytest.mark.parametrize("chunk", [None, (3000, 2000)])
def test_cpu_convention_bit_identical_to_live_reference(built_libs, profile, threads, chunk):
    lines = synth.random_lines(900, 1000.0, 1040.0, 2500.0, 1e-6, 1e2, seed=77 + threads,
                               pressure_atm=0.5)
    grid = synth.Grid(990.0, 1050.0, 6000)
    cond = dict(temperature=800.0, partition=synth.partition_poly(800.0), mean_mass=18.02,
                pressure=0.5, ref_temp=296.0)
    fr = grid.freq()
    init = np.zeros_like(fr)
    kw = {} if chunk is None else dict(start_idx=chunk[0], points=chunk[1])
    ref = oracle.ref_cpu(profile, fr, init, lines, cond, grid.dfreq, nthreads=threads, **kw)
    got = oracle.cpu_convention(profile, fr, init, lines, cond, grid.dfreq, nthreads=threads, **kw)
    assert np.array_equal(got, ref)


def test_doppler_bins_telescope_to_two_per_line(built_libs):
    """sum_j [erf(g(d_j + h)) - erf(g(d_j - h))] telescopes to 2 for a line
    whose window lies inside the grid (h = df/2)."""
    lines = synth.exomol_like(500, 400, seed=8, nu_max=900.0)
    keep = (lines.nu > 200.0) & (lines.nu < 800.0)
    lines = synth.LineList(*(a[keep] for a in (lines.nu, lines.energies, lines.aif, lines.gns,
                                               lines.gamma, lines.n)))
    grid = synth.Grid(0.0, 1000.0, 100000)
    cond = dict(temperature=296.0, partition=2844.0, mean_mass=30.01, pressure=1.0)
    fr = grid.freq()
    sig = oracle.gpu_convention(oracle.DOPPLER, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    s = np.zeros(len(lines))
    lib = oracle.oracle_lib()
    import ctypes
    c = oracle._consts(cond, grid.dfreq)
    nu, e, a, g, _, _ = oracle._arrs(lines)
    lib.oracle_gpu_doppler_stepone(ctypes.byref(c), ctypes.c_long(len(nu)), oracle._p(e),
                                   oracle._p(nu), oracle._p(a), oracle._p(g, oracle._i),
                                   oracle._p(s))
    assert np.isclose(sig.sum(), 2.0 * s.sum(), rtol=1e-12)


def test_voigt_integral_is_the_line_intensity(built_libs):
    """The profile integrates to sqrt(pi) (ISQRTPI is folded into S), minus
    the Lorentz wings beyond the cut (about (2/pi) gamma / cut)."""
    lines = synth.random_lines(50, 1045.0, 1055.0, 1000.0, 1e-3, 1e-1, seed=9, pressure_atm=1.0)
    grid = synth.Grid(1000.0, 1100.0, 100000)
    cond = dict(temperature=1000.0, partition=synth.partition_poly(1000.0), mean_mass=17.03,
                pressure=1.0, ref_temp=296.0)
    fr = grid.freq()
    sig = oracle.gpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    s = np.zeros(len(lines))
    gl = np.zeros(len(lines))
    lib = oracle.oracle_lib()
    import ctypes
    c = oracle._consts(cond, grid.dfreq)
    nu, e, a, g, gm, n = oracle._arrs(lines)
    lib.oracle_gpu_voigt_stepone(ctypes.byref(c), ctypes.c_long(len(nu)), oracle._p(e),
                                 oracle._p(nu), oracle._p(a), oracle._p(g, oracle._i),
                                 oracle._p(gm), oracle._p(n), oracle._p(s), oracle._p(gl))
    # fraction of a Lorentzian of HWHM gl inside +-25: (2/pi) atan(25/gl)
    expect = np.sum(s * np.sqrt(np.pi) * (2.0 / np.pi) * np.arctan(25.0 / gl))
    assert np.isclose(sig.sum() * grid.dfreq, expect, rtol=2e-4)


def test_humlicek_w4_error_envelope():
    """W4 approximates Re w(z) to about 1e-4 relative; bound it against
    scipy's Faddeeva function over all four regions."""
    scipy_special = pytest.importorskip("scipy.special")
    lib = oracle.oracle_lib()
    xs = np.concatenate([np.linspace(0, 20, 401), np.geomspace(20, 1e4, 60)])
    ys = np.concatenate([[1e-6, 1e-4, 1e-3, 1e-2], np.geomspace(0.03, 200, 40)])
    worst = 0.0
    for y in ys:
        for x in xs:
            ref = scipy_special.wofz(x + 1j * y)
            got = lib.oracle_humlic(float(x), float(y))
            err = abs(got - ref.real) / abs(ref)
            worst = max(worst, err)
    assert worst < 2e-4, worst


def test_humlicek_regions_cover_their_boundaries():
    lib = oracle.oracle_lib()
    for x, y in [(15.0, 0.0), (14.999999, 1e-6), (5.5, 0.0), (5.4999, 1e-3), (1.0, 0.019),
                 (1.0, 0.0191), (0.0, 0.0)]:
        v = lib.oracle_humlic(x, y)
        assert np.isfinite(v) and v >= -1e-6
