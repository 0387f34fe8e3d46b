"""Host-side logic on the CPU: grid construction, window/pair counting used by
the benchmark, the OpenMPManager line-coverage rule and the workload
generators."""
import math

import numpy as np

import bench
from gpu_cross_b200 import synth


def test_grid_is_built_like_baseprofile():
    # BaseProfile.cpp:10,19 -- df = (end - start) / Npoints (not Npoints - 1)
    g = synth.Grid(500.0, 8000.0, 750000)
    assert g.dfreq == (8000.0 - 500.0) / 750000.0
    f = g.freq()
    i = 123457
    assert f[i] == 500.0 + float(i) * g.dfreq
    assert f[-1] < 8000.0


def test_pairs_gpu_window_matches_bruteforce():
    rng = np.random.default_rng(0)
    nu = np.sort(rng.uniform(10.0, 20.0, 200))
    f = synth.Grid(0.0, 30.0, 3000).freq()
    brute = sum(int(np.sum((nu_i - f >= -2.5) & (nu_i - f <= 2.5))) for nu_i in nu)
    assert bench.pairs_gpu_window(nu, f, 2.5) == brute


def test_pairs_cpu_window_matches_openmp_rule():
    rng = np.random.default_rng(1)
    nu = rng.uniform(1.0, 29.0, 300)
    f0, df, npts, cut = 0.0, 0.01, 3000, 2.5
    brute = 0
    for x in nu:
        ib = max(round((x - cut - f0) / df), 0)
        ie = min(round((x + cut - f0) / df), npts)
        brute += max(ie - ib, 0)
    assert bench.pairs_cpu_window(nu, f0, df, npts, cut) == brute


def _covered(n, threads):
    # OpenMPManager.cpp:186-188: int for_block = std::ceil(float(N)/float(threads))
    fb = int(math.ceil(np.float32(n) / np.float32(threads)))
    return min(threads * fb, n)


def test_openmp_line_coverage_rule():
    assert _covered(1000, 3) == 1000
    # beyond 2^24 the float division can drop the last lines
    n = (1 << 24) + 1  # float(n) rounds down to 2^24
    assert _covered(n, 8) == 1 << 24


def test_sweep_conditions():
    conds = synth.sweep_conditions()
    assert len(conds) == 40
    ts = sorted({c["temperature"] for c in conds})
    ps = sorted({round(c["pressure_atm"] / synth.BAR_TO_ATM, 6) for c in conds})
    assert ts[0] == 300.0 and ts[-1] == 2100.0 and len(ts) == 10
    assert ps == [1e-3, 0.1, 1.0, 10.0]
    assert all(c["cut"] == 25.0 for c in conds)


def test_generators_are_seeded_and_sorted():
    a = synth.random_lines(1000, 500.0, 8000.0, 2500.0, 1e-6, 1e2, seed=1003)
    b = synth.random_lines(1000, 500.0, 8000.0, 2500.0, 1e-6, 1e2, seed=1003)
    assert np.array_equal(a.nu, b.nu) and np.array_equal(a.gns, b.gns)
    assert np.all(np.diff(a.nu) >= 0)
    assert a.gns.dtype == np.int32 and a.gns.min() >= 1
    x = synth.exomol_like(2000, 5000, seed=1001)
    assert np.all(np.diff(x.nu) >= 0) and x.nu.min() > 0 and x.nu.max() <= 10000.0


def test_partition_poly_monotone():
    t = np.linspace(200, 3000, 50)
    q = np.array([synth.partition_poly(v) for v in t])
    assert np.all(np.diff(q) > 0)
