"""Seeded synthetic input files for the end-to-end cases: ExoMol
(.states, .trans, multi-stream .trans.bz2, .broad), HITRAN 160-character
.par records, and the .inp keyword files that point at them.

The same generator feeds the reference's own main program (oracle/_ref/
ref_main, in tests/golden/make_e2e_golden.py) and xsec_cross, so the
committed golden spectra pin the whole path: .inp parsing, the readers, the
window filter and chunking of the profiles, and the managers.  Each fixture
stores a hash of the files it was made from; a test that regenerates
different files fails instead of comparing against a stale spectrum.

Shapes follow what the reference reads:
  .states   "id E g J ..." (exomol_functions.cpp:24-35)
  .trans    "%12d %12d %10.4E" records of 37 bytes, ascending nu
            (ExomolStateReader.cpp:145, read_compress_trans.c:34)
  .broad    "a0 gamma n J''" and "a1 gamma n J'' J'" (ExomolStateReader.cpp:52-63)
  .par      HITRAN 2004 records, field widths of HITRANStateReader.cpp:4
"""
from __future__ import annotations

import bz2
import hashlib
import os

import numpy as np

# J takes one digit so that the reference's broadener keys ("a1" + J'' + J'
# concatenated) cannot collide; every (J'', J') pair has an a1 entry because
# the reference's a0 fallback never matches.
J_MAX = 9


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def write_exomol(dirname, seed, n_states=700, n_trans=16000, e_max=6000.0, nu_lo=300.0,
                 nu_hi=3300.0, split_nu=1800.0, bz2_split_record=None):
    """States, a broadener file and two transition files: <split_nu as plain
    text, >=split_nu as a .bz2 made of two bzip2 streams.  Returns the file
    names (relative to dirname)."""
    rng = _rng(seed)
    e = np.sort(rng.uniform(0.0, e_max, n_states))
    e[0] = 0.0
    g = rng.choice(np.array([1, 3, 5, 6, 10, 15]), n_states)
    J = rng.integers(0, J_MAX + 1, n_states)
    with open(os.path.join(dirname, "mol.states"), "w") as f:
        for k in range(n_states):
            # two trailing quantum-number columns the readers ignore
            f.write("%12d %12.6f %6d %7d %4d %4d\n" % (k + 1, e[k], g[k], J[k], k % 3, k % 7))
    with open(os.path.join(dirname, "mol.broad"), "w") as f:
        for ji in range(J_MAX + 1):
            f.write("a0 %6.4f %5.3f %3d\n" % (0.05 + 0.001 * ji, 0.5 - 0.01 * ji, ji))
        for ji in range(J_MAX + 1):
            for jf in range(J_MAX + 1):
                gam = 0.02 + 0.004 * ji + 0.0015 * jf + 0.002 * rng.random()
                nn = 0.3 + 0.04 * abs(ji - jf) + 0.05 * rng.random()
                f.write("a1 %6.4f %5.3f %3d %3d\n" % (gam, nn, ji, jf))
    # transitions: random (upper, lower) pairs with nu in range
    up = rng.integers(1, n_states, 4 * n_trans)
    lo = (rng.random(4 * n_trans) * up).astype(np.int64)
    nu = e[up] - e[lo]
    keep = (nu >= nu_lo) & (nu <= nu_hi)
    up, lo, nu = up[keep][:n_trans], lo[keep][:n_trans], nu[keep][:n_trans]
    order = np.argsort(nu, kind="stable")
    up, lo, nu = up[order], lo[order], nu[order]
    a = 10.0 ** rng.uniform(-4.0, 2.0, up.size)
    recs = ["%12d %12d %10.4E\n" % (u + 1, l + 1, x) for u, l, x in zip(up, lo, a)]
    assert all(len(r) == 37 for r in recs)
    cut = int(np.searchsorted(nu, split_nu))
    with open(os.path.join(dirname, "mol_a.trans"), "w") as f:
        f.writelines(recs[:cut])
    body = "".join(recs[cut:]).encode()
    mid = (len(recs[cut:]) // 2) * 37 if bz2_split_record is None else bz2_split_record
    with open(os.path.join(dirname, "mol_b.trans.bz2"), "wb") as f:
        f.write(bz2.compress(body[:mid]))
        f.write(bz2.compress(body[mid:]))
    with open(os.path.join(dirname, "mol_b.trans"), "w") as f:
        f.write(body.decode())
    return dict(states="mol.states", broad="mol.broad", trans=["mol_a.trans", "mol_b.trans.bz2"],
                trans_plain=["mol_a.trans", "mol_b.trans"])


def hitran_record(mol, iso, nu, S, A, gair, gself, E, nair, gup, glo):
    # gamma_air is F5.4 (".0734": no leading zero)
    rec = ("%2d%1d%12.6f%10.3E%10.3E%s%5.3f%10.4f%4.2f%8.5f" %
           (mol, iso, nu, S, A, ("%6.4f" % gair)[1:], gself, E, nair, -0.001))
    rec += " " * 60 + "345560" + " 2 2 2 2 2 2" + " " + "%7.1f%7.1f" % (gup, glo)
    assert len(rec) == 160, len(rec)
    return rec + "\n"


def write_hitran(dirname, seed, n=6000, nu_lo=5.0, nu_hi=1700.0):
    rng = _rng(seed)
    nu = np.sort(rng.uniform(nu_lo, nu_hi, n))
    E = rng.exponential(900.0, n)
    A = 10.0 ** rng.uniform(-5.0, 1.5, n)
    S = 10.0 ** rng.uniform(-26.0, -19.0, n)
    gair = rng.uniform(0.02, 0.12, n)
    gself = rng.uniform(0.1, 0.5, n)
    nair = rng.uniform(0.3, 0.9, n)
    gup = rng.choice(np.array([3.0, 6.0, 12.0, 24.0, 42.0]), n)
    with open(os.path.join(dirname, "mol.par"), "w") as f:
        for k in range(n):
            f.write(hitran_record(11, 1, nu[k], S[k], A[k], gair[k], gself[k], E[k], nair[k],
                                  gup[k], 1.0))
    return dict(par="mol.par")


def inp_text(kind, settings, files):
    lines = [kind]
    for k, v in settings.items():
        lines.append("%s %s" % (k, v))
    if kind == "EXOMOL":
        lines.append("STATE-FILE %s" % files["states"])
        if "broad" in files:
            lines += ["BROADENERS", "  " + files["broad"], "END"]
    lines += ["TRANS-FILES"] + [" " + t for t in files["trans"]] + ["END", ""]
    return "\n".join(lines)


# name: (file kind, generator seed, .inp settings)
CASES = {
    "exomol_voigt": ("EXOMOL", 2101, {
        "TEMPERATURE": "1000.0", "PRESSURE": "0.5", "PARTITION": "-1", "MEAN-MASS": "18.01528",
        "PROFILE": "VOIGT", "NU-RANGE": "1000.0 3000.0", "N-POINTS": "20000",
        "NUM-THREADS": "3", "MAX-POINTS": "3000"}),
    "exomol_doppler": ("EXOMOL", 2102, {
        "TEMPERATURE": "3000.0", "PRESSURE": "1.0", "PARTITION": "-1", "MEAN-MASS": "2.016",
        "PROFILE": "DOPPLER", "NU-RANGE": "1000.0 1400.0", "N-POINTS": "20000",
        "NUM-THREADS": "2"}),
    "hitran_voigt": ("HITRAN", 2103, {
        "TEMPERATURE": "296.0", "PRESSURE": "1.0", "PARTITION": "512.5", "MEAN-MASS": "17.031",
        "HITRAN-MIXTURE-AIR": "0.7", "PROFILE": "VOIGT", "NU-RANGE": "0.0 1500.0",
        "N-POINTS": "15000", "NUM-THREADS": "4"}),
    "hitran_doppler": ("HITRAN", 2104, {
        "TEMPERATURE": "2500.0", "PRESSURE": "0.1", "PARTITION": "2250.0", "MEAN-MASS": "2.016",
        "PROFILE": "DOPPLER", "NU-RANGE": "1200.0 1500.0", "N-POINTS": "30000"}),
}


def make_case(name, dirname):
    """Writes the case's data files and case.inp into dirname; returns
    (path of case.inp, sha256 over every file written)."""
    kind, seed, settings = CASES[name]
    if kind == "EXOMOL":
        files = write_exomol(dirname, seed)
        if settings["PROFILE"] == "DOPPLER":
            files = dict(files)
            files.pop("broad")
    else:
        files = write_hitran(dirname, seed)
        files["trans"] = [files["par"]]
    inp = os.path.join(dirname, "case.inp")
    with open(inp, "w") as f:
        f.write(inp_text(kind, settings, files))
    h = hashlib.sha256()
    for fn in sorted(os.listdir(dirname)):
        with open(os.path.join(dirname, fn), "rb") as f:
            h.update(fn.encode())
            h.update(f.read())
    return inp, h.hexdigest()


def parse_spectrum(text):
    """(freq, intens) from "%12.6f %13.8E" lines; other lines are skipped."""
    fr, iv = [], []
    for ln in text.splitlines():
        t = ln.split()
        if len(t) != 2 or "E" not in t[1] or "." not in t[0]:
            continue
        try:
            a, b = float(t[0]), float(t[1])
        except ValueError:
            continue
        fr.append(a)
        iv.append(b)
    return np.array(fr), np.array(iv)
