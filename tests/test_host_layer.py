"""The C++ host layer (include/xsec/xsec.h) through its program, xsec_cross,
on the CPU: .inp parsing (Input.cpp:98-182), the ExoMol and HITRAN readers,
and -- against the reference's own main program -- the whole read/filter
path: the golden spectra made by oracle/_ref/ref_main are reproduced by the
C oracle fed with the lines our readers return.  Computing a spectrum needs
the GPU; without one the program fails loudly."""
from __future__ import annotations

import bz2
import json
import lzma
import math
import os
import subprocess

import numpy as np
import pytest

import e2e_cases
import oracle
from gpu_cross_b200 import build, synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cli(args, cwd, stdin=None):
    return subprocess.run([build.CLI, *args], cwd=cwd, capture_output=True, text=True,
                          input=stdin, timeout=300)


def settings(text, tmp_path):
    p = cli(["--settings"], tmp_path, stdin=text)
    assert p.returncode == 0, p.stderr
    out = {}
    for ln in p.stdout.splitlines():
        k, _, v = ln.partition(" ")
        out.setdefault(k, []).append(v)
    return out


def list_lines(tmp_path, inp="case.inp"):
    p = cli(["--input", inp, "--list-lines"], tmp_path)
    assert p.returncode == 0, p.stderr
    rows = [ln.split() for ln in p.stdout.splitlines()]
    part = [r for r in rows if r[0] == "partition"]
    arr = np.array([[float(x) for x in r] for r in rows if r[0] != "partition"])
    return part[0], arr


# ---------------------------------------------------------------------------
def test_cli_built(built_libs):
    assert os.path.exists(build.CLI) and os.path.exists(build.LIB_HOST)


def test_inp_keywords(built_libs, tmp_path):
    text = "\n".join([
        "EXOMOL", "TEMPERATURE 1000.0", "PRESSURE 0.986923", "PARTITION -1.725235E+03",
        "N-POINTS 3000001", "NU-RANGE 0.0 30000.0", "PROFILE VOIGT", "MEAN-MASS 18.01528",
        "HITRAN-MIXTURE 0.0", "  ", "STATE-FILE  water.states  ", "BROADENERS ", "  h2.broad",
        "END", "TRANS-FILES", " a.trans", " b.trans.bz2", "END", "NUM-THREADS 8", "MEMORY 4",
        "MAX-POINTS 12345", "GAMMA-AIR 0.07", "N-AIR 0.5", "HALF-WIDTH 0.2", "SOMETHING ELSE",
        ""])
    s = settings(text, tmp_path)
    assert s["file-type"] == ["EXOMOL"] and s["profile"] == ["VOIGT"]
    assert float(s["temperature"][0]) == 1000.0
    assert float(s["pressure"][0]) == 0.986923
    assert float(s["partition"][0]) == -1725.235
    assert s["n-points"] == ["3000001"] and s["nu-range"] == ["0 30000"]
    assert float(s["mean-mass"][0]) == 18.01528
    # "HITRAN-MIXTURE" is not the reference's keyword (HITRAN-MIXTURE-AIR):
    # ignored, the default 1.0 stays (Input.cpp:130)
    assert float(s["hitran-mixture-air"][0]) == 1.0
    assert s["state-file"] == ["water.states"]
    assert s["trans-file"] == ["a.trans", "b.trans.bz2"] and s["broadener"] == ["h2.broad"]
    assert s["num-threads"] == ["8"] and s["memory"] == ["4000000000"]
    assert s["max-points"] == ["12345"]
    assert float(s["gamma-air"][0]) == 0.07 and float(s["n-air"][0]) == 0.5
    assert float(s["half-width"][0]) == 0.2


def test_inp_defaults_and_profiles(built_libs, tmp_path):
    s = settings("HITRAN\nTRANS-FILES\nx.par\nEND\n", tmp_path)
    # Input::Input and ReadInputII defaults (Input.cpp:2-15, 112-114)
    assert float(s["partition"][0]) == -1.0 and s["num-threads"] == ["1"]
    assert s["memory"] == ["1000000000"] and s["max-points"] == ["80000"]
    assert float(s["pressure"][0]) == 1.0 and float(s["temperature"][0]) == 296.0
    assert s["nu-range"] == ["0 100"] and s["n-points"] == ["1000"]
    for word, want in [("DOPPLER", "DOPPLER"), ("GAUSSIAN", "GAUSSIAN"), ("VOIGT", "VOIGT"),
                       ("LORENTZ", "PSUEDO_VOIGT")]:
        s = settings(f"HITRAN\nPROFILE {word}\n", tmp_path)
        assert s["profile"] == [want]


@pytest.mark.parametrize("text, msg", [
    ("XSEC\n", "not supported"),
    ("EXOMOL\nTEMPERATURE\n", "needs a value"),
    ("EXOMOL\nNU-RANGE 10\n", "needs a value"),
    ("EXOMOL\nNU-RANGE 10 5\n", "ascending"),
    ("", "empty"),
])
def test_inp_errors(built_libs, tmp_path, text, msg):
    p = cli(["--settings"], tmp_path, stdin=text)
    assert p.returncode == 1 and msg in p.stderr


# ---------------------------------------------------------------------------
def _write_inp(tmp_path, kind, body):
    (tmp_path / "case.inp").write_text(kind + "\n" + body)


def test_exomol_reader_matches_restatement(built_libs, tmp_path):
    files = e2e_cases.write_exomol(str(tmp_path), 77, n_states=300, n_trans=3000)
    _write_inp(tmp_path, "EXOMOL", "PROFILE VOIGT\nPRESSURE 2.0\nTEMPERATURE 700\n"
               "STATE-FILE mol.states\nBROADENERS\nmol.broad\nEND\nTRANS-FILES\n"
               + "\n".join(files["trans"]) + "\nEND\n")
    part, got = list_lines(tmp_path)
    # restatement: nu = E' - E'', gns = g', E'', A, gamma = a1(J'', J') * P
    st = np.loadtxt(tmp_path / "mol.states")
    E, g, J = st[:, 1], st[:, 2], st[:, 3].astype(int)
    broad = {}
    for ln in (tmp_path / "mol.broad").read_text().splitlines():
        t = ln.split()
        key = (t[0], int(t[3]), int(t[4]) if t[0] == "a1" else -1)
        broad[key] = (float(t[1]), float(t[2]))
    recs = []
    for fn in files["trans_plain"]:
        recs += [ln.split() for ln in (tmp_path / fn).read_text().splitlines()]
    assert got.shape == (len(recs), 6)
    f = np.array([int(r[0]) - 1 for r in recs])
    i = np.array([int(r[1]) - 1 for r in recs])
    a = np.array([float(r[2]) for r in recs])
    np.testing.assert_array_equal(got[:, 0], E[f] - E[i])
    np.testing.assert_array_equal(got[:, 1], g[f])
    np.testing.assert_array_equal(got[:, 2], E[i])
    np.testing.assert_array_equal(got[:, 3], a)
    gam = np.array([broad[("a1", J[ii], J[ff])][0] * 2.0 for ii, ff in zip(i, f)])
    nn = np.array([broad[("a1", J[ii], J[ff])][1] for ii, ff in zip(i, f)])
    np.testing.assert_array_equal(got[:, 4], gam)
    np.testing.assert_array_equal(got[:, 5], nn)
    # partition sum over the states (exomol_functions.cpp:44-62)
    beta = 6.6260693e-27 * 2.99792458e10 / (1.380658e-16 * 700.0)
    q = 0.0
    for k in range(len(E)):
        q += g[k] * math.exp(-beta * E[k])
    assert float(part[1]) == pytest.approx(q, rel=1e-15)


def test_exomol_bz2_stream_split_inside_a_record(built_libs, tmp_path):
    """Two bzip2 streams whose boundary falls inside a 37-byte record read
    the same lines as the plain file."""
    e2e_cases.write_exomol(str(tmp_path), 78, n_states=200, n_trans=2000, bz2_split_record=37 * 50 + 11)
    common = "PROFILE DOPPLER\nSTATE-FILE mol.states\nTRANS-FILES\n"
    _write_inp(tmp_path, "EXOMOL", common + "mol_b.trans.bz2\nEND\n")
    _, a = list_lines(tmp_path)
    (tmp_path / "plain.inp").write_text("EXOMOL\n" + common + "mol_b.trans\nEND\n")
    _, b = list_lines(tmp_path, "plain.inp")
    assert a.shape[0] > 500
    np.testing.assert_array_equal(a, b)


def test_exomol_broadening_fallbacks(built_libs, tmp_path):
    (tmp_path / "s.states").write_text("1 0.0 1 0\n2 100.0 3 1\n3 250.0 5 2\n4 400.0 7 3\n")
    (tmp_path / "t.trans").write_text("2 1 1.0E-01\n3 1 2.0E-01\n\n4 2 3.0E-01\n4 3 4.0E-01 399.9\n")
    (tmp_path / "b.broad").write_text("a1 0.0700 0.610 0 1\na0 0.0500 0.450 1\n")
    _write_inp(tmp_path, "EXOMOL", "PROFILE VOIGT\nPRESSURE 0.5\nGAMMA-AIR 0.09\nN-AIR 0.33\n"
               "STATE-FILE s.states\nBROADENERS\nb.broad\nEND\nTRANS-FILES\nt.trans\nEND\n")
    _, got = list_lines(tmp_path)
    want = [
        (100.0, 3, 0.0, 0.1, 0.07 * 0.5, 0.61),   # a1 (J''=0, J'=1)
        (250.0, 5, 0.0, 0.2, 0.09 * 0.5, 0.33),   # no a1 (0, 2), no a0 for J''=0: defaults
        (300.0, 7, 100.0, 0.3, 0.05 * 0.5, 0.45),  # a0 J''=1
        (150.0, 7, 250.0, 0.4, 0.09 * 0.5, 0.33),  # extra column ignored; defaults
    ]
    np.testing.assert_allclose(got, np.array(want), rtol=1e-15, atol=0)


def test_exomol_bad_state_id_is_an_error(built_libs, tmp_path):
    (tmp_path / "s.states").write_text("1 0.0 1 0\n2 100.0 3 1\n")
    (tmp_path / "t.trans").write_text("2 1 1.0E-01\n5 1 2.0E-01\n")
    _write_inp(tmp_path, "EXOMOL", "PROFILE DOPPLER\nSTATE-FILE s.states\nTRANS-FILES\nt.trans\nEND\n")
    p = cli(["--input", "case.inp", "--list-lines"], tmp_path)
    assert p.returncode == 1 and "outside the state file" in p.stderr


def test_hitran_reader_fields(built_libs, tmp_path):
    recs = [e2e_cases.hitran_record(11, 1, 100.25, 3.5e-21, 0.125, 0.0734, 0.402, 512.125, 0.76,
                                    42.0, 1.0),
            e2e_cases.hitran_record(11, 1, 101.5, 2.0e-22, 0.0, 0.05, 0.3, 200.0, 0.5, 6.0, 1.0)]
    (tmp_path / "m.par").write_text("".join(recs) + "\n")
    _write_inp(tmp_path, "HITRAN", "PROFILE VOIGT\nPRESSURE 2.0\nTEMPERATURE 296.0\n"
               "PARTITION 512.0\nHITRAN-MIXTURE-AIR 0.25\nTRANS-FILES\nm.par\nEND\n")
    part, got = list_lines(tmp_path)
    assert float(part[1]) == 512.0
    assert got.shape == (2, 6)
    np.testing.assert_array_equal(got[0], [100.25, 42, 512.125, 0.125,
                                           (0.0734 * 0.25 + 0.402 * 0.75) * 2.0, 0.76])
    # A == 0: gns*A rebuilt from S(296 K) with Q(296) (HITRANStateReader.cpp:222-233)
    beta = 6.6260693e-27 * 2.99792458e10 / (1.380658e-16 * 296.0)
    nu, E = 101.5, 200.0
    a = 2.0e-22 * 8.0 * math.acos(-1.0) * 2.99792458e10 * 512.0 * nu * nu / (
        math.exp(-beta * E) * (1.0 - math.exp(-beta * nu)))
    assert got[1, 1] == 1 and got[1, 3] == pytest.approx(a, rel=1e-15)


def test_hitran_without_einstein_a_needs_q296(built_libs, tmp_path):
    rec = e2e_cases.hitran_record(11, 1, 101.5, 2.0e-22, 0.0, 0.05, 0.3, 200.0, 0.5, 6.0, 1.0)
    (tmp_path / "m.par").write_text(rec)
    _write_inp(tmp_path, "HITRAN", "PROFILE DOPPLER\nTEMPERATURE 500\nPARTITION 900\n"
               "TRANS-FILES\nm.par\nEND\n")
    p = cli(["--input", "case.inp", "--list-lines"], tmp_path)
    assert p.returncode == 1 and "Q(296 K)" in p.stderr


def test_hitran_partition_required(built_libs, tmp_path):
    (tmp_path / "m.par").write_text(e2e_cases.hitran_record(11, 1, 100.0, 1e-21, 1.0, 0.05, 0.3,
                                                            10.0, 0.5, 6.0, 1.0))
    _write_inp(tmp_path, "HITRAN", "PROFILE DOPPLER\nTRANS-FILES\nm.par\nEND\n")
    p = cli(["--input", "case.inp", "--list-lines"], tmp_path)
    assert "partition unavailable" in p.stdout and "TIPS" in p.stdout


# ---------------------------------------------------------------------------
def load_golden(name):
    meta = json.load(open(os.path.join(GOLDEN, "e2e_golden.json")))[name]
    with open(os.path.join(GOLDEN, f"e2e_{name}.spec.xz"), "rb") as f:
        vals = np.array([float(x) for x in lzma.decompress(f.read()).split()])
    assert len(vals) == meta["npoints"]
    return meta, vals


def case_lines(name, workdir):
    """Writes the case, checks its inputs against the golden's hash, and
    returns (lines kept by the window filter, condition, grid, profile,
    threads) from our readers."""
    kind, _, st = e2e_cases.CASES[name]
    meta, _ = load_golden(name)
    _, digest = e2e_cases.make_case(name, str(workdir))
    assert digest == meta["inputs_sha256"], (
        "generated inputs differ from the golden's; rerun tests/golden/make_e2e_golden.py")
    part, L = list_lines(workdir)
    voigt = st["PROFILE"] == "VOIGT"
    T, P = float(st["TEMPERATURE"]), float(st["PRESSURE"])
    lo, hi = map(float, st["NU-RANGE"].split())
    cut = min(25.0 * P, 100.0) if voigt else 100.0
    L = L[(L[:, 0] >= lo - cut) & (L[:, 0] <= hi + cut)]
    lines = synth.LineList(L[:, 0].copy(), L[:, 2].copy(), L[:, 3].copy(), L[:, 1].astype(np.int32),
                           L[:, 4].copy(), L[:, 5].copy())
    cond = dict(temperature=T, partition=float(part[1]), mean_mass=float(st["MEAN-MASS"]),
                pressure=P, ref_temp=500.0 if (kind == "EXOMOL" and voigt) else 296.0)
    grid = synth.Grid(lo, hi, int(st["N-POINTS"]))
    return lines, cond, grid, (oracle.VOIGT if voigt else oracle.DOPPLER), int(st.get("NUM-THREADS", 1))


# Printed with 9 significant digits ("%13.8E"): two correctly rounded
# printings of values that agree to 1e-12 differ by at most one unit in the
# last digit.
PRINT_REL = 1.01e-8


@pytest.mark.parametrize("name", sorted(e2e_cases.CASES))
def test_reference_main_is_reproduced_by_our_readers(built_libs, tmp_path, name):
    """ref_main's spectrum == C oracle (CPU convention) over the lines our
    readers return: pins the readers, the window filter and the .inp path
    against the reference program itself."""
    lines, cond, grid, prof, thr = case_lines(name, tmp_path)
    _, want = load_golden(name)
    got = oracle.cpu_convention(prof, grid.freq(), np.zeros(grid.npoints), lines, cond, grid.dfreq,
                                nthreads=thr)
    peak = np.abs(want).max()
    assert peak > 0
    err = np.abs(got - want)
    assert np.all(err <= PRINT_REL * np.abs(want) + 1e-12 * peak), float((err / peak).max())


def test_compute_without_gpu_fails_loudly(built_libs, tmp_path):
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("checks the behaviour on a machine without a GPU")
    except ImportError:
        pass
    e2e_cases.make_case("hitran_voigt", str(tmp_path))
    p = cli(["--input", "case.inp"], tmp_path)
    assert p.returncode == 1 and "device" in p.stderr.lower()
    assert "E+" not in p.stdout and "E-" not in p.stdout


# ---------------------------------------------------------------------------
REF_SIDE_MANAGER = r'''
#include <cstdio>
#include "xsec/xsec.h"
// A manager written against the reference's BaseManager.h:6-33: it defines
// the reference's pure virtuals only, not SetPrecision.
class RefSideManager : public BaseManager {
public:
    RefSideManager() : BaseManager(VOIGT) {}
    void InitializeVectors(int) {}
    void InitializeConstants(double, double, double, double, double, double, double) {}
    void TransferVectors(size_t, double*, double*, double*, int*, double*, double*) {}
    void TransferFreq(double*, double*, int) {}
    void ExecuteCrossSection(int, int, int) {}
    void TransferResults(double*, double*, int) {}
    void Cleanup() {}
};
int main() {
    RefSideManager m;
    BaseManager* b = &m;
    b->SetPrecision(XS_FP64);
    try {
        b->SetPrecision(XS_MIXED);
    } catch (const xs_error& e) {
        std::printf("mixed refused: %d\n", e.code());
        return 0;
    }
    return 1;
}
'''


def test_reference_side_manager_subclass_compiles(built_libs, tmp_path):
    """BaseManager::SetPrecision is not pure: a subclass with only the
    reference's virtuals compiles, accepts FP64 and refuses MIXED."""
    src = tmp_path / "ref_side.cpp"
    src.write_text(REF_SIDE_MANAGER)
    exe = tmp_path / "ref_side"
    libdir = os.path.dirname(build.LIB_HOST)
    subprocess.run(["g++", "-std=c++11", "-I", build.INCLUDE, str(src), "-o", str(exe), "-L", libdir,
                    "-lxsec_host", "-lxsec_b200", f"-Wl,-rpath,{libdir}"], check=True, timeout=120)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "mixed refused" in p.stdout
