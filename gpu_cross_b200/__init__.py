"""gpu_cross_b200 -- B200-native molecular absorption cross-section engine.

sigma(f) = sum over lines of S_i(T) x profile_i(f - nu_i; T, P), truncated at a
cutoff, on a uniform wavenumber grid, computed by hand-written sm_100a kernels
behind a C ABI (include/xsec_b200.h).  The C++ host classes that mirror the
reference's BaseManager / GpuManager / OpenMPManager / BaseProfile API live in
include/xsec/ and gpu_cross_b200/csrc/host/.

Python is used for tests, benchmarks and fixtures only: ``capi`` binds the
C ABI with ctypes, ``synth`` makes the seeded synthetic workloads.
"""
from . import build, capi, synth  # noqa: F401

__all__ = ["build", "capi", "synth"]
