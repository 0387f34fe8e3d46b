"""Generates the end-to-end golden spectra of tests/golden/ by running the
reference's own main program (oracle/_ref/ref_main, built from the reference
sources by oracle/Makefile) on the synthetic cases of tests/e2e_cases.py.

  python tests/golden/make_e2e_golden.py [outdir]

For each case: the input files and case.inp are written to a scratch
directory, `ref_main < case.inp` runs there, and the "%13.8E" column of its
spectrum is stored, one value per line, xz-compressed, as
e2e_<case>.spec.xz; e2e_golden.json records the number of points and the
sha256 of the input files.

Two properties of the reference program are handled here:
  * it exits with SIGSEGV after printing everything (in its teardown), so the
    run is accepted when the full spectrum and the timer table came out, and
    stdout is unbuffered (stdbuf -o0) so nothing is lost;
  * OpenMPManager adds into a grid it never clears (OpenMPManager.cpp:23,
    125), so allocations of 64 KiB and more are forced onto fresh, zeroed
    pages (MALLOC_MMAP_THRESHOLD_).
"""
from __future__ import annotations

import json
import lzma
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import e2e_cases  # noqa: E402

REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "ref_main")


def run_reference(name: str, workdir: str):
    inp, digest = e2e_cases.make_case(name, workdir)
    env = dict(os.environ, MALLOC_MMAP_THRESHOLD_="65536")
    with open(inp) as f:
        p = subprocess.run(["stdbuf", "-o0", REF_MAIN], stdin=f, cwd=workdir, capture_output=True,
                           text=True, env=env, timeout=600)
    freq, intens = e2e_cases.parse_spectrum(p.stdout)
    npoints = int(e2e_cases.CASES[name][2]["N-POINTS"])
    if len(intens) != npoints or "Timer Data" not in p.stdout:
        raise RuntimeError(f"{name}: reference run incomplete (rc {p.returncode}, "
                           f"{len(intens)} of {npoints} points)\n{p.stdout[-2000:]}")
    return freq, intens, digest, p.stdout


def main(outdir: str = HERE):
    if not os.path.exists(REF_MAIN):
        raise SystemExit("oracle/_ref/ref_main is missing: run make -C oracle ref_main")
    meta = {}
    for name in e2e_cases.CASES:
        with tempfile.TemporaryDirectory() as d:
            _, _, digest, out = run_reference(name, d)
        col = [ln.split()[1] for ln in out.splitlines()
               if len(ln.split()) == 2 and "E" in ln.split()[1] and "." in ln.split()[0]]
        path = os.path.join(outdir, f"e2e_{name}.spec.xz")
        with open(path, "wb") as f:
            f.write(lzma.compress(("\n".join(col) + "\n").encode(), preset=9))
        meta[name] = {"npoints": len(col), "inputs_sha256": digest}
        print("wrote", path)
    with open(os.path.join(outdir, "e2e_golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    out = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out, exist_ok=True)
    main(out)
