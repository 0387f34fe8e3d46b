"""End to end on the B200: xsec_cross (the reference's main program on the
C++ host layer) reads each synthetic case's .inp, ExoMol/HITRAN files and
.bz2 streams, chunks the lines, computes on the GPU and prints the
spectrum.  The default backend (HybridManager, the reference's CPU
arithmetic) must print what the reference's own main program printed
(tests/golden/e2e_*.spec.xz); the GPU-convention backends must match the
oracle's restatement of the reference GPU kernels; mixed precision must meet
its accuracy bounds."""
from __future__ import annotations

import re

import numpy as np
import pytest

import e2e_cases
import oracle
from helpers import MIXED_INTEGRATED, MIXED_REL, PEAK_FLOOR
from test_host_layer import PRINT_REL, case_lines, cli, load_golden

pytestmark = pytest.mark.gpu

CASES = sorted(e2e_cases.CASES)


def run_cli(workdir, *args):
    p = cli(["--input", "case.inp", *args], workdir)
    assert p.returncode == 0, p.stderr[-2000:]
    fr, iv = e2e_cases.parse_spectrum(p.stdout)
    return fr, iv, p.stderr


@pytest.mark.parametrize("name", CASES)
def test_cli_prints_the_reference_programs_spectrum(cuda, tmp_path, name):
    lines, cond, grid, prof, thr = case_lines(name, tmp_path)
    _, want = load_golden(name)
    fr, got, log = run_cli(tmp_path)
    assert len(got) == grid.npoints
    np.testing.assert_allclose(fr, grid.freq(), rtol=0, atol=5e-7)
    peak = np.abs(want).max()
    err = np.abs(got - want)
    assert np.all(err <= PRINT_REL * np.abs(want) + 1e-12 * peak), float((err / peak).max())
    if name == "exomol_voigt":
        # MAX-POINTS 3000 over a 20000-point grid: several chunks
        assert "in 1 chunks" not in log


def chunks_of(log):
    """(lines, ib, ie) of every chunk the profile evaluated, from its log."""
    out = []
    for m in re.finditer(r"chunk \d+: (\d+) lines, points \[(-?\d+), (-?\d+)\)", log):
        out.append(tuple(int(v) for v in m.groups()))
    return out


@pytest.mark.parametrize("backend", ["gpu", "multigpu"])
@pytest.mark.parametrize("name", CASES)
def test_cli_gpu_convention_backends(cuda, tmp_path, name, backend):
    """GpuManager arithmetic through the profile's chunks: each chunk covers
    the grid points [ib, ie) (BaseProfile.cpp:55-60), so a window point that
    rounds outside its chunk is not evaluated -- as in the reference."""
    lines, cond, grid, prof, _ = case_lines(name, tmp_path)
    _, got, log = run_cli(tmp_path, "--backend", backend)
    want = np.zeros(grid.npoints)
    k = 0
    chunks = chunks_of(log)
    assert chunks and sum(c[0] for c in chunks) == len(lines)
    for n, ib, ie in chunks:
        if ie > ib:
            want = oracle.gpu_convention(prof, grid.freq(), want, lines.slice(k, k + n), cond,
                                         grid.dfreq, points=ie - ib, start_idx=ib)
        k += n
    peak = np.abs(want).max()
    err = np.abs(got - want)
    # one rounding of the printed value on top of the engine's <= 1e-10
    assert np.all(err <= (PRINT_REL + 1e-10) * np.abs(want) + 1e-12 * peak), \
        float((err / peak).max())


@pytest.mark.parametrize("name", ["exomol_voigt", "hitran_voigt"])
def test_cli_mixed_precision(cuda, tmp_path, name):
    case_lines(name, tmp_path)
    _, want = load_golden(name)
    _, got, _ = run_cli(tmp_path, "--precision", "mixed")
    peak = np.abs(want).max()
    big = np.abs(want) > PEAK_FLOOR * peak
    rel = np.abs(got[big] - want[big]) / np.abs(want[big])
    assert rel.max() <= MIXED_REL
    assert abs(got.sum() - want.sum()) / want.sum() <= MIXED_INTEGRATED
    assert np.abs(got[~big] - want[~big]).max(initial=0.0) <= MIXED_REL * peak


def test_cli_openmp_backend_equals_hybrid(cuda, tmp_path):
    case_lines("hitran_voigt", tmp_path)
    _, a, _ = run_cli(tmp_path)
    _, b, _ = run_cli(tmp_path, "--backend", "openmp")
    np.testing.assert_array_equal(a, b)


def read_binary_spectrum(path):
    raw = open(path, "rb").read()
    assert raw[:8] == b"XSECBIN1"
    n = int(np.frombuffer(raw[8:16], dtype="<i8")[0])
    body = np.frombuffer(raw[16:], dtype="<f8")
    assert body.size == 2 * n
    return body[:n], body[n:]


@pytest.mark.parametrize("name", ["exomol_doppler", "hitran_voigt"])
def test_cli_binary_output_keeps_fp64(cuda, tmp_path, name):
    """--format binary writes every bit of the grid and the cross-section:
    the GPU-convention backend against the oracle at the FP64 bound (the
    text output holds nine digits), and the same values as the text."""
    lines, cond, grid, prof, _ = case_lines(name, tmp_path)
    p = cli(["--input", "case.inp", "--backend", "gpu", "--format", "binary", "--output",
             "spec.bin"], tmp_path)
    assert p.returncode == 0, p.stderr[-2000:]
    fr, got = read_binary_spectrum(tmp_path / "spec.bin")
    np.testing.assert_allclose(fr, grid.freq(), rtol=1e-15, atol=0)
    want = np.zeros(grid.npoints)
    k = 0
    for n, ib, ie in chunks_of(p.stderr):
        if ie > ib:
            want = oracle.gpu_convention(prof, grid.freq(), want, lines.slice(k, k + n), cond,
                                         grid.dfreq, points=ie - ib, start_idx=ib)
        k += n
    peak = np.abs(want).max()
    big = np.abs(want) > PEAK_FLOOR * peak
    assert np.max(np.abs(got[big] - want[big]) / np.abs(want[big])) <= 1e-10
    assert np.max(np.abs(got[~big] - want[~big]), initial=0.0) <= 1e-10 * peak
    _, text, _ = run_cli(tmp_path, "--backend", "gpu")
    assert np.all(np.abs(text - got) <= PRINT_REL * np.abs(got) + 1e-300)
