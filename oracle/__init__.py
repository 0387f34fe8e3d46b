"""ctypes access to the test-only checkers built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs -- never by gpu_cross_b200.

  liboracle.so    C restatement of both reference backends (xsec_oracle.c)
  libref_cpu.so   the reference's own OpenMPManager (compiled from its sources)
  libref_gpu.so   the reference's own cross_kernal.cu for sm_100a
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "lib", "liboracle.so")
LIB_REF_CPU = os.path.join(HERE, "_ref", "libref_cpu.so")
LIB_REF_GPU = os.path.join(HERE, "_ref", "libref_gpu.so")

GAUSSIAN, DOPPLER, VOIGT = 0, 1, 2

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)


class Consts(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in
                ("half_width", "temperature", "partition", "dfreq", "mean_mass",
                 "pressure", "ref_temp")]


def build(ref: bool = True) -> None:
    """Build liboracle.so, and the reference checkers when the reference
    tree is present."""
    targets = ["oracle"]
    # the reference tree sits beside the repository checkout unless REF says
    # otherwise (the same rule as the Makefile's)
    ref_dir = os.environ.get("REF", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
    if ref and os.path.isdir(ref_dir):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, *targets], check=True)


_libs: dict[str, ctypes.CDLL] = {}


def _load(path: str) -> ctypes.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run make -C oracle)")
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def oracle_lib() -> ctypes.CDLL:
    lib = _load(LIB_ORACLE)
    lib.oracle_humlic.restype = ctypes.c_double
    lib.oracle_humlic.argtypes = [ctypes.c_double, ctypes.c_double]
    return lib


def _p(a: np.ndarray | None, kind=_d):
    if a is None:
        return None
    return a.ctypes.data_as(kind)


def _consts(cond: dict, dfreq: float) -> Consts:
    return Consts(half_width=cond.get("half_width", 0.1), temperature=cond["temperature"],
                  partition=cond["partition"], dfreq=dfreq, mean_mass=cond["mean_mass"],
                  pressure=cond.get("pressure", 1.0), ref_temp=cond.get("ref_temp", 296.0))


def _arrs(lines):
    nu = np.ascontiguousarray(lines.nu, dtype=np.float64)
    e = np.ascontiguousarray(lines.energies, dtype=np.float64)
    a = np.ascontiguousarray(lines.aif, dtype=np.float64)
    g = np.ascontiguousarray(lines.gns, dtype=np.int32)
    gm = np.ascontiguousarray(lines.gamma, dtype=np.float64)
    n = np.ascontiguousarray(lines.n, dtype=np.float64)
    return nu, e, a, g, gm, n


def gpu_convention(profile: int, freq: np.ndarray, intens: np.ndarray, lines, cond: dict,
                   dfreq: float, points: int | None = None, start_idx: int = 0,
                   cut: float | None = None) -> np.ndarray:
    """The reference GpuManager path (cross_kernal.cu block kernels), restated
    in C.  Returns a new grid = intens + contributions.  cut: window half
    width in place of the reference rule (Voigt and Doppler)."""
    lib = oracle_lib()
    if cut is not None:
        lib.oracle_set_cut(ctypes.c_double(cut))
        try:
            return gpu_convention(profile, freq, intens, lines, cond, dfreq, points, start_idx)
        finally:
            lib.oracle_set_cut(ctypes.c_double(-1.0))
    out = np.array(intens, dtype=np.float64, copy=True)
    fr = np.ascontiguousarray(freq, dtype=np.float64)
    pts = len(fr) - start_idx if points is None else points
    c = _consts(cond, dfreq)
    nu, e, a, g, gm, n = _arrs(lines)
    nl = ctypes.c_long(len(nu))
    if profile == VOIGT:
        lib.oracle_gpu_voigt(ctypes.byref(c), _p(fr), _p(out), pts, start_idx, nl, _p(e), _p(nu),
                             _p(a), _p(g, _i), _p(gm), _p(n))
    elif profile == DOPPLER:
        lib.oracle_gpu_doppler(ctypes.byref(c), _p(fr), _p(out), pts, start_idx, nl, _p(e), _p(nu),
                               _p(a), _p(g, _i))
    else:
        lib.oracle_gpu_gaussian(ctypes.byref(c), _p(fr), _p(out), pts, start_idx, nl, _p(e),
                                _p(nu), _p(a), _p(g, _i))
    return out


def cpu_convention(profile: int, freq: np.ndarray, intens: np.ndarray, lines, cond: dict,
                   dfreq: float, nthreads: int = 1, points: int | None = None,
                   start_idx: int = 0) -> np.ndarray:
    """The reference OpenMPManager path, restated in C."""
    lib = oracle_lib()
    out = np.array(intens, dtype=np.float64, copy=True)
    fr = np.ascontiguousarray(freq, dtype=np.float64)
    pts = len(fr) - start_idx if points is None else points
    c = _consts(cond, dfreq)
    nu, e, a, g, gm, n = _arrs(lines)
    nl = ctypes.c_long(len(nu))
    if profile == VOIGT:
        lib.oracle_cpu_voigt(ctypes.byref(c), nthreads, len(fr), _p(fr), _p(out), pts, start_idx,
                             nl, _p(e), _p(nu), _p(a), _p(g, _i), _p(gm), _p(n))
    elif profile == DOPPLER:
        lib.oracle_cpu_doppler(ctypes.byref(c), nthreads, len(fr), _p(fr), _p(out), pts,
                               start_idx, nl, _p(e), _p(nu), _p(a), _p(g, _i))
    else:
        raise ValueError("the reference CPU backend implements DOPPLER and VOIGT only")
    return out


def ref_cpu(profile: int, freq: np.ndarray, intens: np.ndarray, lines, cond: dict, dfreq: float,
            nthreads: int = 1, points: int | None = None, start_idx: int = 0) -> np.ndarray:
    """Run the reference's own OpenMPManager (compiled from its sources)."""
    lib = _load(LIB_REF_CPU)
    lib.ref_cpu_run.restype = ctypes.c_int
    out = np.array(intens, dtype=np.float64, copy=True)
    fr = np.array(freq, dtype=np.float64, copy=True)
    pts = len(fr) - start_idx if points is None else points
    nu, e, a, g, gm, n = _arrs(lines)
    c = _consts(cond, dfreq)
    if profile != VOIGT:
        # DopplerProfile passes NULL gamma/n (BaseProfile.cpp:3); the
        # OpenMPManager only allocates them for VOIGT (OpenMPManager.cpp:48).
        gm = n = None
    rc = lib.ref_cpu_run(ctypes.c_int(profile), ctypes.c_int(nthreads), ctypes.c_int(len(fr)),
                         _p(fr), _p(out), ctypes.c_long(len(nu)), _p(e), _p(nu), _p(a),
                         _p(g, _i), _p(gm), _p(n), ctypes.c_double(c.half_width),
                         ctypes.c_double(c.temperature), ctypes.c_double(c.partition),
                         ctypes.c_double(c.dfreq), ctypes.c_double(c.mean_mass),
                         ctypes.c_double(c.pressure), ctypes.c_double(c.ref_temp),
                         ctypes.c_int(pts), ctypes.c_int(start_idx), ctypes.c_int(1))
    if rc != 0:
        raise RuntimeError(f"ref_cpu_run failed with {rc}")
    return out


def ref_gpu(profile: int, freq: np.ndarray, intens: np.ndarray, lines, cond: dict, dfreq: float,
            points: int | None = None, start_idx: int = 0, chunks: int = 1):
    """Run the reference's own GPU kernels (needs a GPU).  Returns
    (grid, kernel_ms)."""
    lib = _load(LIB_REF_GPU)
    lib.ref_gpu_run.restype = ctypes.c_int
    out = np.array(intens, dtype=np.float64, copy=True)
    fr = np.array(freq, dtype=np.float64, copy=True)
    pts = len(fr) - start_idx if points is None else points
    nu, e, a, g, gm, n = _arrs(lines)
    c = _consts(cond, dfreq)
    ms = ctypes.c_float(0.0)
    rc = lib.ref_gpu_run(ctypes.c_int(profile), ctypes.c_int(len(fr)), _p(fr), _p(out),
                         ctypes.c_long(len(nu)), _p(e), _p(nu), _p(a), _p(g, _i), _p(gm), _p(n),
                         ctypes.c_double(c.half_width), ctypes.c_double(c.temperature),
                         ctypes.c_double(c.partition), ctypes.c_double(c.dfreq),
                         ctypes.c_double(c.mean_mass), ctypes.c_double(c.pressure),
                         ctypes.c_double(c.ref_temp), ctypes.c_int(pts), ctypes.c_int(start_idx),
                         ctypes.c_int(chunks), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"ref_gpu_run failed with {rc}")
    return out, float(ms.value)
