"""Generates the golden fixtures of tests/golden/ from the reference itself.

  python tests/golden/make_golden.py cpu   # reference OpenMPManager (oracle/_ref/libref_cpu.so)
  python tests/golden/make_golden.py gpu   # reference cross_kernal.cu kernels (needs a B200)

Each fixture is a small seeded case: the inputs (line list, grid, constants)
and the grid the reference produced, stored as .npz.  The CPU fixtures are
made in the build container (the reference tree is there); the GPU fixtures
on a B200 from the prebuilt oracle/_ref/libref_gpu.so.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from gpu_cross_b200 import synth  # noqa: E402

CASES = {
    # name: (profile, builder)
    "voigt_p1": ("voigt", dict(seed=501, n=1500, nu=(1000.0, 1060.0), grid=(990.0, 1070.0, 8000),
                               T=1000.0, M=17.03, P=1.0, p_atm=1.0)),
    "voigt_p0.1_coldT": ("voigt", dict(seed=502, n=1200, nu=(2000.0, 2050.0),
                                        grid=(1995.0, 2055.0, 6000), T=300.0, M=17.03, P=0.1,
                                        p_atm=0.1)),
    "voigt_p10_hotT": ("voigt", dict(seed=503, n=1000, nu=(500.0, 560.0), grid=(480.0, 580.0, 10000),
                                      T=2100.0, M=17.03, P=10.0, p_atm=10.0)),
    "doppler_exomol": ("doppler", dict(seed=504, n=3000, nu_max=2000.0, grid=(0.0, 2000.0, 200000),
                                       T=296.0, M=30.01, P=1.0)),
}


def build_case(kind, p):
    if kind == "voigt":
        lines = synth.random_lines(p["n"], p["nu"][0], p["nu"][1], 2500.0, 1e-6, 1e2, seed=p["seed"],
                                   pressure_atm=p["p_atm"])
        cond = dict(temperature=p["T"], partition=synth.partition_poly(p["T"]), mean_mass=p["M"],
                    pressure=p["P"], ref_temp=296.0)
    else:
        lines = synth.exomol_like(2000, p["n"], seed=p["seed"], nu_max=p["nu_max"])
        cond = dict(temperature=p["T"], partition=2844.0, mean_mass=p["M"], pressure=p["P"],
                    ref_temp=296.0)
    grid = synth.Grid(*p["grid"])
    return lines, grid, cond


def main(which: str, outdir: str = HERE):
    for name, (kind, p) in CASES.items():
        lines, grid, cond = build_case(kind, p)
        fr = grid.freq()
        z = np.zeros_like(fr)
        prof = oracle.VOIGT if kind == "voigt" else oracle.DOPPLER
        out = {}
        if which == "cpu":
            for thr in (1, 4):
                out[f"ref_cpu_t{thr}"] = oracle.ref_cpu(prof, fr, z, lines, cond, grid.dfreq,
                                                        nthreads=thr)
            path = os.path.join(outdir, f"{name}.cpu.npz")
        else:
            out["ref_gpu"], _ = oracle.ref_gpu(prof, fr, z, lines, cond, grid.dfreq)
            path = os.path.join(outdir, f"{name}.gpu.npz")
        np.savez_compressed(path, nu=lines.nu, energies=lines.energies, aif=lines.aif,
                            gns=lines.gns, gamma=lines.gamma, n=lines.n, grid=np.array(p["grid"]),
                            temperature=cond["temperature"], partition=cond["partition"],
                            mean_mass=cond["mean_mass"], pressure=cond["pressure"],
                            ref_temp=cond["ref_temp"], profile=prof, **out)
        print("wrote", path)


if __name__ == "__main__":
    out = sys.argv[2] if len(sys.argv) > 2 else HERE
    os.makedirs(out, exist_ok=True)
    main(sys.argv[1] if len(sys.argv) > 1 else "cpu", out)
