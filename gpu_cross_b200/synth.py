"""Seeded synthetic line lists and grids for the cross-section workloads.

No line list of the reference's samples (ExoMol BT2 water, HITRAN NH3) ships
with it, and none can be fetched, so every workload is synthetic.  Each
generator uses numpy's PCG64 seeded with ``1000 + workload number`` by
default, so a workload is reproducible from its name alone.

Arrays follow the reference's host layout (BaseProfile.h:97-102): ``nu``,
``energies`` (lower-state energy E''), ``aif`` (Einstein A), ``gns`` (int32
upper-state degeneracy), ``gamma`` (Lorentz HWHM, already multiplied by the
pressure in atm, as the readers do: ExomolStateReader.cpp:17-26,
HITRANStateReader.cpp:218) and ``n`` (temperature exponent).  Lines are
sorted by ``nu``, as the reference requires of its input files.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

BAR_TO_ATM = 0.986923


@dataclasses.dataclass
class LineList:
    nu: np.ndarray
    energies: np.ndarray
    aif: np.ndarray
    gns: np.ndarray
    gamma: np.ndarray
    n: np.ndarray

    def __len__(self) -> int:
        return int(self.nu.shape[0])

    def slice(self, a: int, b: int) -> "LineList":
        return LineList(*(getattr(self, f.name)[a:b] for f in dataclasses.fields(self)))

    def sorted(self) -> "LineList":
        order = np.argsort(self.nu, kind="stable")
        return LineList(*(np.ascontiguousarray(getattr(self, f.name)[order])
                          for f in dataclasses.fields(self)))


@dataclasses.dataclass
class Grid:
    """Uniform grid built as BaseProfile does: df = (end - start) / npoints,
    freq[i] = start + i * df (BaseProfile.cpp:7-21)."""

    start: float
    end: float
    npoints: int

    @property
    def dfreq(self) -> float:
        return (self.end - self.start) / float(self.npoints)

    def freq(self) -> np.ndarray:
        i = np.arange(self.npoints, dtype=np.float64)
        # start + i*df with one rounding per operation (no fused multiply-add),
        # as the reference's host loop computes it.
        return np.add(self.start, np.multiply(i, self.dfreq))


def partition_poly(t: float) -> float:
    """Fixed 4th-order polynomial Q(T) used by the single-point and sweep
    workloads (the reference takes Q as an input; it has no polynomial)."""
    return 13.2 + 2.914 * t + 7.37e-3 * t ** 2 - 1.2e-6 * t ** 3 + 2.1e-10 * t ** 4


def random_lines(n: int, nu_lo: float, nu_hi: float, e_mean: float, a_lo: float, a_hi: float,
                 seed: int, gamma_lo: float = 0.03, gamma_hi: float = 0.1,
                 n_lo: float = 0.4, n_hi: float = 0.8, pressure_atm: float = 1.0) -> LineList:
    """nu ~ U(nu_lo, nu_hi) sorted, E'' ~ Exp(e_mean), A ~ logU(a_lo, a_hi),
    g = g_ns (2J+1) with g_ns in {1, 3} and J ~ U{0..60},
    gamma = U(gamma_lo, gamma_hi) * pressure_atm, n ~ U(n_lo, n_hi)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nu = np.sort(rng.uniform(nu_lo, nu_hi, n))
    e = rng.exponential(e_mean, n)
    aif = np.exp(rng.uniform(math.log(a_lo), math.log(a_hi), n))
    j = rng.integers(0, 61, n)
    gns_ns = np.where(rng.random(n) < 0.5, 1, 3)
    gns = (gns_ns * (2 * j + 1)).astype(np.int32)
    gamma = rng.uniform(gamma_lo, gamma_hi, n) * pressure_atm
    nexp = rng.uniform(n_lo, n_hi, n)
    return LineList(nu.astype(np.float64), e, aif, gns, gamma, nexp)


def exomol_like(n_states: int = 20000, n_trans: int = 1_000_000, seed: int = 1001,
                nu_max: float = 10000.0) -> LineList:
    """ExoMol-style list: states E ~ U(0, 8000), J ~ U{0..60},
    g_tot = g_ns (2J+1), g_ns in {1, 3}; transitions are (upper, lower) state
    pairs with 0 < nu = E' - E'' <= nu_max, A ~ logU(1e-6, 1e2).  As in
    ExomolStateReader::ReadNextState (ExomolStateReader.cpp:156-160):
    nu = E[f] - E[i], E'' = E[i], g = g_tot[f]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    energy = rng.uniform(0.0, 8000.0, n_states)
    jq = rng.integers(0, 61, n_states)
    g_tot = (np.where(rng.random(n_states) < 0.5, 1, 3) * (2 * jq + 1)).astype(np.int32)
    up = np.empty(0, dtype=np.int64)
    lo = np.empty(0, dtype=np.int64)
    while up.shape[0] < n_trans:
        m = 2 * (n_trans - up.shape[0]) + 16
        a = rng.integers(0, n_states, m)
        b = rng.integers(0, n_states, m)
        d = energy[a] - energy[b]
        ok = (d > 0.0) & (d <= nu_max)
        up = np.concatenate([up, a[ok]])
        lo = np.concatenate([lo, b[ok]])
    up, lo = up[:n_trans], lo[:n_trans]
    nu = energy[up] - energy[lo]
    aif = np.exp(rng.uniform(math.log(1e-6), math.log(1e2), n_trans))
    gamma = np.full(n_trans, 0.05)
    nexp = np.full(n_trans, 0.5)
    ll = LineList(nu, energy[lo], aif, g_tot[up], gamma, nexp)
    return ll.sorted()


# Workload descriptions (sizes of the reference-style configurations).
def doppler_exomol_workload(scale: float = 1.0):
    """Plain Doppler: 20k states, 1e6 transitions, M = 30.01, T = 296 K,
    Q = 2844.0, grid 0-10000 cm-1 at 0.01 (1e6 points), cut 25."""
    n_trans = max(1, int(1_000_000 * scale))
    lines = exomol_like(20000, n_trans, seed=1001)
    grid = Grid(0.0, 10000.0, 1_000_000)
    cond = dict(temperature=296.0, partition=2844.0, mean_mass=30.01, pressure=1.0, cut=25.0)
    return lines, grid, cond


def voigt_single_workload(n_lines: int = 10_000_000, grid_points: int = 750_000):
    """Voigt single point: nu ~ U(500, 8000), E'' ~ Exp(2500),
    A ~ logU(1e-6, 1e2), gamma_ref ~ U(0.03, 0.1) per atm, n ~ U(0.4, 0.8),
    T = 1000 K, P = 1 bar, M = 17.03, Q = partition_poly(T),
    grid 500-8000 at 0.01 (7.5e5 points), cut 25."""
    lines = random_lines(n_lines, 500.0, 8000.0, 2500.0, 1e-6, 1e2, seed=1002,
                         pressure_atm=BAR_TO_ATM)
    grid = Grid(500.0, 8000.0, grid_points)
    cond = dict(temperature=1000.0, partition=partition_poly(1000.0), mean_mass=17.03,
                pressure=1.0, cut=25.0, ref_temp=296.0)
    return lines, grid, cond


SWEEP_T = tuple(300.0 + 200.0 * k for k in range(10))
SWEEP_P_BAR = (1e-3, 1e-1, 1.0, 10.0)


def sweep_conditions(cut: float = 25.0):
    """The 40 (T, P) points: T in {300, 500, ..., 2100} K x P in
    {1e-3, 1e-1, 1, 10} bar; Q = partition_poly(T)."""
    out = []
    for t in SWEEP_T:
        for p in SWEEP_P_BAR:
            out.append(dict(temperature=t, pressure_atm=p * BAR_TO_ATM,
                            partition=partition_poly(t), cut=cut))
    return out


def voigt_sweep_workload(n_lines: int = 10_000_000, grid_points: int = 75_000):
    """Batched Voigt sweep: the single-point line list with gamma_ref per atm
    (pressure applied per condition), grid 500-8000 at 0.1 (7.5e4 points)."""
    lines = random_lines(n_lines, 500.0, 8000.0, 2500.0, 1e-6, 1e2, seed=1003,
                         pressure_atm=1.0)
    grid = Grid(500.0, 8000.0, grid_points)
    return lines, grid, sweep_conditions(), dict(mean_mass=17.03, ref_temp=296.0)


# Serving: three resident molecules and a seeded Poisson request stream.
SERVE_MOLECULES = ((1_000_000, 18.02), (10_000_000, 30.01), (100_000_000, 16.04))


def serving_molecules(scale: float = 1.0):
    """[(LineList, mass)] for the three served molecules: 1e6, 1e7 and 1e8
    lines (times scale) with nu ~ U(0, 12000) and the single-point list's
    other statistics; gamma per atm at 296 K."""
    out = []
    for k, (n, mass) in enumerate(SERVE_MOLECULES):
        m = max(1000, int(n * scale))
        out.append((random_lines(m, 0.0, 12000.0, 2500.0, 1e-6, 1e2, seed=1005 + 10 * k,
                                 pressure_atm=1.0), mass))
    return out


def serving_trace(rate: float = 200.0, duration_s: float = 10.0, seed: int = 1005,
                  n_molecules: int = 3):
    """Poisson arrivals (mean `rate` per second) over duration_s; each request:
    molecule uniform, T ~ U(200, 3000) K, P ~ logU(1e-5, 100) bar,
    Doppler or Voigt (1/2 each), span ~ U(100, 5000) cm-1 inside 0-12000,
    resolution df ~ logU(0.01, 1) cm-1, cut 25 cm-1, Q = partition_poly(T)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration_s:
            break
        span = rng.uniform(100.0, 5000.0)
        df = math.exp(rng.uniform(math.log(0.01), math.log(1.0)))
        f0 = rng.uniform(0.0, 12000.0 - span)
        temp = rng.uniform(200.0, 3000.0)
        p_bar = math.exp(rng.uniform(math.log(1e-5), math.log(100.0)))
        out.append(dict(t=t, molecule=int(rng.integers(0, n_molecules)),
                        voigt=bool(rng.random() < 0.5), temperature=temp,
                        partition=partition_poly(temp), pressure=p_bar * BAR_TO_ATM,
                        f0=f0, df=df, npoints=max(1, int(round(span / df))), cut=25.0))
    return out


# Streamed list: intensities precomputed at the condition (GPU-convention
# constants, GPUManager.cpp:28-39 and cross_kernal.cu:775-779).
_PLANCK, _VELLGT, _BOLTZ = 6.6260693e-27, 2.99792458e10, 1.380658e-16
_ISQRTPI = 0.564189584


def intensity_gpu(nu, energies, aif, gns, temperature, partition):
    """S(T) = cmcoef A g ISQRTPI exp(-beta E'') (1 - exp(-beta nu)) / (nu^2 Q)
    with the reference GPU path's constants (nu = 0 -> 1e-6)."""
    cmcoef = 1.0 / (8.0 * math.acos(-1.0) * _VELLGT)
    beta = _PLANCK * _VELLGT / (_BOLTZ * temperature)
    nu_if = np.where(nu == 0.0, 1e-6, nu)
    return (cmcoef * aif * gns * _ISQRTPI * np.exp(-beta * energies) * (1.0 - np.exp(-beta * nu_if))
            / (nu_if * nu_if * partition))


def stream_workload(n_lines: int = 500_000_000, temperature: float = 2000.0, p_bar: float = 1.0,
                    seed: int = 1004, prefilter: float = 1e-30, block: int = 10_000_000):
    """The streamed configuration: nu ~ U(100, 12000) (sorted, built from
    cumulative exponential gaps), E'' ~ Exp(4000), A ~ logU(1e-8, 1e3),
    g = g_ns (2J+1), gamma_ref ~ U(0.03, 0.1) per atm, n ~ U(0.4, 0.8); stored
    as FP64 centres, FP32 S(T) and FP32 gamma(T, P) for T = 2000 K, P = 1 bar,
    Q = partition_poly(T); lines with S < prefilter are dropped.
    Returns (nu, s, gamma_t, kept, generated)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    q = partition_poly(temperature)
    p_atm = p_bar * BAR_TO_ATM
    gaps_total = 0.0
    nus, ss, gs = [], [], []
    # centres: cumulative exponential gaps, scaled once the total is known
    gaps = []
    for b0 in range(0, n_lines, block):
        g = rng.exponential(1.0, min(block, n_lines - b0))
        gaps.append(g)
        gaps_total += float(g.sum())
    scale = (12000.0 - 100.0) / gaps_total
    run = 0.0
    kept = 0
    for g in gaps:
        c = np.cumsum(g)
        nu = 100.0 + (run + c) * scale
        run += float(c[-1])
        m = nu.size
        e = rng.exponential(4000.0, m)
        aif = np.exp(rng.uniform(math.log(1e-8), math.log(1e3), m))
        j = rng.integers(0, 61, m)
        gns = np.where(rng.random(m) < 0.5, 1.0, 3.0) * (2 * j + 1)
        gam = rng.uniform(0.03, 0.1, m) * p_atm
        nexp = rng.uniform(0.4, 0.8, m)
        s = intensity_gpu(nu, e, aif, gns, temperature, q)
        gl = gam * np.power(296.0 / temperature, nexp)
        keep = s >= prefilter
        kept += int(keep.sum())
        nus.append(nu[keep])
        ss.append(s[keep].astype(np.float32))
        gs.append(gl[keep].astype(np.float32))
    return np.concatenate(nus), np.concatenate(ss), np.concatenate(gs), kept, n_lines
