"""ctypes binding of the C ABI (include/xsec_b200.h) for tests and bench.py.

The library is built in-tree by gpu_cross_b200.build; loading fails loudly
when it is missing -- there is no CPU fallback anywhere in this package.
Device buffers are torch CUDA tensors passed by data pointer.
"""
from __future__ import annotations

import ctypes
import os
import re

from . import build as _build

XS_OK = 0
XS_ERR_INVALID, XS_ERR_CUDA, XS_ERR_NOMEM, XS_ERR_UNSORTED, XS_ERR_GRID = 1, 2, 3, 4, 5
XS_ERR_STATE, XS_ERR_NODEVICE, XS_ERR_TIMEOUT, XS_ERR_UNSUPPORTED = 6, 7, 8, 9
POLICY_LEAST_WORK, POLICY_ROUND_ROBIN, POLICY_DEADLINE = 0, 1, 2

GAUSSIAN, DOPPLER, VOIGT, PSUEDO_VOIGT = 0, 1, 2, 3
CONV_GPU, CONV_CPU = 0, 1
FP64, MIXED = 0, 1


class XsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"xsec_b200 error {code}: {msg}")
        self.code = code


class CrossSectionData(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in
                ("halfwidth", "mean_mass", "temperature", "pressure", "beta", "partition", "ln2",
                 "ref_temp", "cmcoef", "dfreq")]


class Condition(ctypes.Structure):
    _fields_ = [("temperature", ctypes.c_double), ("partition", ctypes.c_double),
                ("pressure", ctypes.c_double), ("gamma_scale", ctypes.c_double),
                ("cut", ctypes.c_double)]


class Options(ctypes.Structure):
    _fields_ = [("profile", ctypes.c_int), ("convention", ctypes.c_int),
                ("precision", ctypes.c_int), ("cpu_threads", ctypes.c_int),
                ("mean_mass", ctypes.c_double), ("ref_temp", ctypes.c_double),
                ("half_width", ctypes.c_double), ("dfreq", ctypes.c_double),
                ("points_per_thread", ctypes.c_int), ("warps_per_block", ctypes.c_int),
                ("conditions_per_warp", ctypes.c_int), ("line_splits", ctypes.c_int),
                ("check_rows", ctypes.c_int)]


class Accuracy(ctypes.Structure):
    _fields_ = [("bound_rel", ctypes.c_double), ("sampled_max_rel", ctypes.c_double),
                ("sampled_integrated_rel", ctypes.c_double), ("sampled_rows", ctypes.c_int),
                ("conditions", ctypes.c_int)]


class Lines(ctypes.Structure):
    _fields_ = [("nu", ctypes.c_void_p), ("energies", ctypes.c_void_p), ("aif", ctypes.c_void_p),
                ("gns", ctypes.c_void_p), ("gamma", ctypes.c_void_p), ("n", ctypes.c_void_p),
                ("count", ctypes.c_size_t)]


class GridC(ctypes.Structure):
    _fields_ = [("freq", ctypes.c_void_p), ("npoints_total", ctypes.c_int),
                ("start_idx", ctypes.c_int), ("points", ctypes.c_int)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device_budget", ctypes.c_size_t), ("host_budget", ctypes.c_size_t),
                ("lanes", ctypes.c_int), ("depth", ctypes.c_int), ("chunk_pairs", ctypes.c_double),
                ("chunk_lines", ctypes.c_size_t), ("policy", ctypes.c_int),
                ("tcache_bytes", ctypes.c_longlong)]


class Request(ctypes.Structure):
    _fields_ = [("molecule", ctypes.c_int), ("profile", ctypes.c_int), ("precision", ctypes.c_int),
                ("temperature", ctypes.c_double), ("partition", ctypes.c_double),
                ("pressure", ctypes.c_double), ("cut", ctypes.c_double), ("f0", ctypes.c_double),
                ("df", ctypes.c_double), ("npoints", ctypes.c_int)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("latency_ms", ctypes.c_double),
                ("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double), ("chunks", ctypes.c_int),
                ("line_evals", ctypes.c_double), ("lines", ctypes.c_size_t),
                ("err_bound", ctypes.c_double), ("tcache_chunks", ctypes.c_int)]


class TuneResult(ctypes.Structure):
    _fields_ = [("points_per_thread", ctypes.c_int), ("warps_per_block", ctypes.c_int),
                ("conditions_per_warp", ctypes.c_int), ("ms", ctypes.c_double),
                ("candidates", ctypes.c_int)]


class StreamStats(ctypes.Structure):
    _fields_ = [("total_ms", ctypes.c_double), ("copy_span_ms", ctypes.c_double),
                ("h2d_bytes", ctypes.c_double), ("chunks", ctypes.c_int), ("kernels", ctypes.c_int)]


_VP = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_SZ = ctypes.c_size_t

# name -> (restype, argtypes)
_SIGS = {
    "xs_last_error": (ctypes.c_char_p, []),
    "xs_version": (ctypes.c_char_p, []),
    "xs_device_available": (_I, []),
    "xs_device_count": (_I, [ctypes.POINTER(ctypes.c_int)]),
    "xs_copy_intensity_info": (_I, [ctypes.POINTER(CrossSectionData)]),
    "xs_execute_two_step_kernal_voigt_block": (_I, [_VP] * 8 + [_I, _I, _I]),
    "xs_execute_two_step_kernal_doppler_block": (_I, [_VP] * 6 + [_I, _I, _I]),
    "xs_execute_two_step_kernal_block": (_I, [_VP] * 6 + [_I, _I, _I]),
    "xs_launcher_sync": (_I, []),
    "xs_engine_create": (_I, [_I, ctypes.POINTER(_VP)]),
    "xs_engine_destroy": (_I, [_VP]),
    "xs_engine_set_stream": (_I, [_VP, _VP]),
    "xs_engine_sync": (_I, [_VP]),
    "xs_engine_scratch_bytes": (_I, [_VP, ctypes.POINTER(_SZ)]),
    "xs_scratch_bytes_needed": (_SZ, [ctypes.POINTER(Options), _I, _SZ]),
    "xs_engine_execute": (_I, [_VP, ctypes.POINTER(Options), ctypes.POINTER(Condition), _I,
                               ctypes.POINTER(Lines), ctypes.POINTER(GridC), _VP, _SZ]),
    "xs_engine_execute_host": (_I, [_VP, ctypes.POINTER(Options), ctypes.POINTER(Condition), _I,
                                    ctypes.POINTER(Lines), ctypes.POINTER(Lines), ctypes.POINTER(GridC), _VP,
                                    _SZ, _VP, _I]),
    "xs_engine_last_stats": (_I, [_VP, ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "xs_engine_accuracy": (_I, [_VP, _VP]),
    "xs_error_bound": (_D, [_I, _I]),
    "xs_engine_capture": (_I, [_VP, ctypes.POINTER(Options), ctypes.POINTER(Condition), _I,
                               ctypes.POINTER(Lines), ctypes.POINTER(GridC), _VP, _SZ, _I,
                               ctypes.POINTER(_VP)]),
    "xs_graph_launch": (_I, [_VP, _VP]),
    "xs_graph_kernel_count": (_I, [_VP, ctypes.POINTER(ctypes.c_int)]),
    "xs_graph_destroy": (_I, [_VP]),
    "xs_measure_peaks": (_I, [_I, ctypes.POINTER(_D), ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "xs_execute_noalloc": (_I, [ctypes.POINTER(Options), ctypes.POINTER(Condition),
                                ctypes.POINTER(Lines), ctypes.POINTER(GridC), _VP, _VP]),
    "xs_engine_autotune": (_I, [_VP, ctypes.POINTER(Options), ctypes.POINTER(Condition), _I,
                                ctypes.POINTER(Lines), ctypes.POINTER(GridC), _VP, _SZ,
                                ctypes.POINTER(TuneResult)]),
    "xs_tune_save": (_I, [ctypes.c_char_p]),
    "xs_tune_load": (_I, [ctypes.c_char_p]),
    "xs_tune_clear": (_I, []),
    "xs_stream_execute": (_I, [_VP, ctypes.POINTER(Options), ctypes.POINTER(Condition), _VP, _VP,
                               _VP, _SZ, ctypes.POINTER(GridC), _VP, _SZ,
                               ctypes.POINTER(StreamStats)]),
    "xs_manager_create": (_I, [_I, _I, _I, _I, _SZ, ctypes.POINTER(_VP)]),
    "xs_manager_destroy": (_I, [_VP]),
    "xs_manager_set_precision": (_I, [_VP, _I]),
    "xs_manager_initialize_vectors": (_I, [_VP, _I]),
    "xs_manager_initialize_constants": (_I, [_VP] + [_D] * 7),
    "xs_manager_transfer_vectors": (_I, [_VP, _SZ] + [_VP] * 6),
    "xs_manager_transfer_freq": (_I, [_VP, _VP, _VP, _I]),
    "xs_manager_execute_cross_section": (_I, [_VP, _I, _I, _I]),
    "xs_manager_transfer_results": (_I, [_VP, _VP, _VP, _I]),
    "xs_manager_cleanup": (_I, [_VP]),
    "xs_manager_ready_for_work": (_I, [_VP, ctypes.POINTER(_I)]),
    "xs_manager_get_ntrans": (_I, [_VP, ctypes.POINTER(_SZ)]),
    "xs_server_create": (_I, [_I, ctypes.POINTER(ServerConfig), ctypes.POINTER(_VP)]),
    "xs_server_destroy": (_I, [_VP]),
    "xs_server_add_molecule": (_I, [_VP] + [_VP] * 6 + [_SZ, _D, _D, ctypes.POINTER(_I)]),
    "xs_server_add_states": (_I, [_VP, _I, _VP, _VP, _SZ]),
    "xs_partition_sum": (_I, [_I, _VP, _VP, _SZ, _VP, _I, _VP]),
    "xs_server_submit": (_I, [_VP, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_ulonglong)]),
    "xs_server_wait": (_I, [_VP, ctypes.c_ulonglong, _VP, _I, ctypes.POINTER(RequestInfo), _I]),
    "xs_server_pending": (_I, [_VP, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "xs_plan_chunks": (_I, [_VP, _SZ, _D, _D, _I, _D, _D, _SZ, _I, _VP, _VP, _VP, _VP, _VP,
                            ctypes.POINTER(_I)]),
    "xs_split_grid": (_I, [_VP, _SZ, _D, _D, _I, _D, _I, _I, ctypes.POINTER(_I), ctypes.POINTER(_I),
                           ctypes.POINTER(_SZ), ctypes.POINTER(_SZ), ctypes.POINTER(_D)]),
}

_lib: ctypes.CDLL | None = None


def library_path() -> str:
    return _build.LIB_CUDA


def declared_functions() -> list[str]:
    """Function names declared in include/xsec_b200.h."""
    hdr = os.path.join(_build.INCLUDE, "xsec_b200.h")
    text = open(hdr).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(xs_[a-z0-9_]+)\s*\(", text)))


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = library_path()
        if not os.path.exists(path):
            raise ImportError(f"{path} is not built; run python -m gpu_cross_b200.build "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(path)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != XS_OK:
        msg = lib().xs_last_error()
        raise XsError(rc, msg.decode() if msg else "")


def device_available() -> bool:
    return bool(lib().xs_device_available())


def _ptr(t) -> int | None:
    if t is None:
        return None
    return int(t.data_ptr())


class Engine:
    """One engine handle (device scratch, stream, timing events)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        check(lib().xs_engine_create(device, ctypes.byref(h)))
        self.h = h
        self.device = device

    def close(self) -> None:
        if self.h:
            lib().xs_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int | None) -> None:
        check(lib().xs_engine_set_stream(self.h, stream_handle))

    def sync(self) -> None:
        check(lib().xs_engine_sync(self.h))

    def scratch_bytes(self) -> int:
        v = ctypes.c_size_t()
        check(lib().xs_engine_scratch_bytes(self.h, ctypes.byref(v)))
        return int(v.value)

    def execute(self, opts: Options, conds: list[Condition], lines: Lines, grid: GridC, out_ptr: int,
                out_stride: int = 0) -> None:
        arr = (Condition * len(conds))(*conds)
        check(lib().xs_engine_execute(self.h, ctypes.byref(opts), arr, len(conds),
                                      ctypes.byref(lines), ctypes.byref(grid), out_ptr, out_stride))

    def execute_host(self, opts: Options, conds: list[Condition], host_lines: Lines, dev_lines: Lines,
                     grid: GridC, out_ptr: int, out_stride: int = 0, host_out_ptr: int | None = None,
                     pieces: int = 8) -> None:
        """xs_engine_execute_host: lines from (pinned) host arrays, copied in
        `pieces` slices that overlap step one; the result span copied to
        host_out_ptr.  Asynchronous: sync() before reading it."""
        arr = (Condition * len(conds))(*conds)
        check(lib().xs_engine_execute_host(self.h, ctypes.byref(opts), arr, len(conds),
                                           ctypes.byref(host_lines), ctypes.byref(dev_lines),
                                           ctypes.byref(grid), out_ptr, out_stride, host_out_ptr, pieces))

    def accuracy(self) -> dict:
        """xs_engine_accuracy: the error statement of the last execute."""
        a = Accuracy()
        check(lib().xs_engine_accuracy(self.h, ctypes.byref(a)))
        return {k: getattr(a, k) for k, _ in Accuracy._fields_}

    def autotune(self, opts: Options, conds: list[Condition], lines: Lines, grid: GridC, out_ptr: int,
                 out_stride: int = 0) -> dict:
        arr = (Condition * len(conds))(*conds)
        r = TuneResult()
        check(lib().xs_engine_autotune(self.h, ctypes.byref(opts), arr, len(conds), ctypes.byref(lines),
                                       ctypes.byref(grid), out_ptr, out_stride, ctypes.byref(r)))
        return {k: getattr(r, k) for k, _ in TuneResult._fields_}

    def stream_execute(self, opts: Options, cond: Condition, h_nu: int, h_s: int, h_gamma: int,
                       n: int, grid: GridC, out_ptr: int, chunk_lines: int) -> dict:
        """xs_stream_execute over host arrays given by address (f64 centres,
        f32 intensities, f32 Lorentz widths; pinned for overlapped copies)."""
        st = StreamStats()
        check(lib().xs_stream_execute(self.h, ctypes.byref(opts), ctypes.byref(cond), h_nu, h_s,
                                      h_gamma, n, ctypes.byref(grid), out_ptr, chunk_lines,
                                      ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in StreamStats._fields_}

    def capture(self, opts: Options, conds: list[Condition], lines: Lines, grid: GridC, out_ptr: int,
                out_stride: int = 0, zero_out: bool = True) -> "Graph":
        arr = (Condition * len(conds))(*conds)
        h = ctypes.c_void_p()
        check(lib().xs_engine_capture(self.h, ctypes.byref(opts), arr, len(conds),
                                      ctypes.byref(lines), ctypes.byref(grid), out_ptr, out_stride,
                                      1 if zero_out else 0, ctypes.byref(h)))
        return Graph(h)

    def last_stats(self) -> tuple[float, float]:
        a, b = ctypes.c_double(), ctypes.c_double()
        check(lib().xs_engine_last_stats(self.h, ctypes.byref(a), ctypes.byref(b)))
        return float(a.value), float(b.value)


class Graph:
    """A captured sweep (xs_engine_capture)."""

    def __init__(self, h):
        self.h = h

    def launch(self, stream_handle: int | None = None) -> None:
        check(lib().xs_graph_launch(self.h, stream_handle))

    def kernel_count(self) -> int:
        """Kernel launches one replay makes."""
        k = ctypes.c_int()
        check(lib().xs_graph_kernel_count(self.h, ctypes.byref(k)))
        return int(k.value)

    def close(self) -> None:
        if self.h:
            lib().xs_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def measure_peaks(device: int = 0) -> dict:
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    check(lib().xs_measure_peaks(device, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
    return dict(fp32_tflops=a.value, fp64_tflops=b.value, rcp32_tops=c.value)


def make_lines(dev: dict, count: int | None = None) -> Lines:
    """dev: dict of torch CUDA tensors nu, energies, aif, gns, gamma, n."""
    n = int(dev["nu"].numel()) if count is None else count
    return Lines(_ptr(dev["nu"]), _ptr(dev["energies"]), _ptr(dev["aif"]), _ptr(dev["gns"]),
                 _ptr(dev.get("gamma")), _ptr(dev.get("n")), n)


def make_grid(freq, start_idx: int = 0, points: int | None = None) -> GridC:
    total = int(freq.numel())
    pts = total - start_idx if points is None else points
    return GridC(_ptr(freq), total, start_idx, pts)


def make_options(profile: int, dfreq: float, mean_mass: float, convention: int = CONV_GPU,
                 precision: int = FP64, cpu_threads: int = 1, ref_temp: float = 296.0,
                 half_width: float = 0.1, points_per_thread: int = 0,
                 warps_per_block: int = 0, conditions_per_warp: int = 0,
                 line_splits: int = 0, check_rows: int = 0) -> Options:
    return Options(profile, convention, precision, cpu_threads, mean_mass, ref_temp, half_width,
                   dfreq, points_per_thread, warps_per_block, conditions_per_warp, line_splits,
                   check_rows)


def make_condition(temperature: float, partition: float, pressure: float = 1.0,
                   gamma_scale: float = 1.0, cut: float = -1.0) -> Condition:
    return Condition(temperature, partition, pressure, gamma_scale, cut)


class Manager:
    """The BaseManager interface (BaseManager.h:22-30) over host numpy
    arrays.  kind 0 = GpuManager, 1 = OpenMPManager (computed on the GPU)."""

    def __init__(self, kind: int, profile: int, gpu_id: int = 0, num_threads: int = 1,
                 total_memory: int = 1_000_000_000):
        h = ctypes.c_void_p()
        check(lib().xs_manager_create(kind, profile, gpu_id, num_threads, total_memory,
                                      ctypes.byref(h)))
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().xs_manager_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _np(a):
        return None if a is None else a.ctypes.data

    def set_precision(self, p: int) -> None:
        check(lib().xs_manager_set_precision(self.h, p))

    def InitializeVectors(self, npoints: int) -> None:
        check(lib().xs_manager_initialize_vectors(self.h, npoints))

    def InitializeConstants(self, half_width, temperature, partition, dfreq, meanmass,
                            pressure=10.0, ref_temp=296.0) -> None:
        check(lib().xs_manager_initialize_constants(self.h, half_width, temperature, partition,
                                                    dfreq, meanmass, pressure, ref_temp))

    def TransferVectors(self, nener, energies, nu, aif, gns, gamma=None, n=None) -> None:
        check(lib().xs_manager_transfer_vectors(self.h, nener, self._np(energies), self._np(nu),
                                                self._np(aif), self._np(gns), self._np(gamma),
                                                self._np(n)))

    def TransferFreq(self, freq, intens, n) -> None:
        check(lib().xs_manager_transfer_freq(self.h, self._np(freq), self._np(intens), n))

    def ExecuteCrossSection(self, n, n_ener, start_idx) -> None:
        check(lib().xs_manager_execute_cross_section(self.h, n, n_ener, start_idx))

    def TransferResults(self, freq, intens, n) -> None:
        check(lib().xs_manager_transfer_results(self.h, self._np(freq), self._np(intens), n))

    def Cleanup(self) -> None:
        check(lib().xs_manager_cleanup(self.h))

    def ReadyForWork(self) -> bool:
        v = ctypes.c_int()
        check(lib().xs_manager_ready_for_work(self.h, ctypes.byref(v)))
        return bool(v.value)

    def GetNtrans(self) -> int:
        v = ctypes.c_size_t()
        check(lib().xs_manager_get_ntrans(self.h, ctypes.byref(v)))
        return int(v.value)


# ---------------------------------------------------------------------------
def plan_chunks(nu, f0: float, df: float, npoints: int, cut: float, max_pairs: float,
                max_lines: int = 0):
    """The server's chunk planner on a host nu array (no device needed).
    Returns a dict of numpy arrays: start, points, l0, l1, pairs."""
    import numpy as np

    nu = np.ascontiguousarray(nu, dtype=np.float64)
    cap = npoints // 256 + 2
    out = dict(start=np.zeros(cap, np.int32), points=np.zeros(cap, np.int32),
               l0=np.zeros(cap, np.uint64), l1=np.zeros(cap, np.uint64), pairs=np.zeros(cap))
    n = ctypes.c_int()
    check(lib().xs_plan_chunks(nu.ctypes.data if nu.size else None, nu.size, f0, df, npoints, cut,
                               max_pairs, max_lines, cap, out["start"].ctypes.data,
                               out["points"].ctypes.data, out["l0"].ctypes.data,
                               out["l1"].ctypes.data, out["pairs"].ctypes.data, ctypes.byref(n)))
    return {k: v[:n.value] for k, v in out.items()}


def split_grid(nu, f0: float, df: float, npoints: int, cut: float, nranks: int, rank: int):
    """Rank `rank`'s share of a grid-range split (xs_split_grid) on a host nu
    array: dict(start, points, l0, l1, pairs)."""
    import numpy as np

    nu = np.ascontiguousarray(nu, dtype=np.float64)
    st, pt = ctypes.c_int(), ctypes.c_int()
    a, b = ctypes.c_size_t(), ctypes.c_size_t()
    pr = ctypes.c_double()
    check(lib().xs_split_grid(nu.ctypes.data if nu.size else None, nu.size, f0, df, npoints, cut,
                              nranks, rank, ctypes.byref(st), ctypes.byref(pt), ctypes.byref(a),
                              ctypes.byref(b), ctypes.byref(pr)))
    return dict(start=st.value, points=pt.value, l0=a.value, l1=b.value, pairs=pr.value)


class Server:
    """A request server (xs_server_*): resident molecules, submit/wait."""

    def __init__(self, device: int = 0, device_budget: int = 0, host_budget: int = 0,
                 lanes: int = 0, depth: int = 0, chunk_pairs: float = 0.0, chunk_lines: int = 0,
                 policy: int = 0, tcache_bytes: int = 0):
        cfg = ServerConfig(device_budget, host_budget, lanes, depth, chunk_pairs, chunk_lines, policy,
                           tcache_bytes)
        h = ctypes.c_void_p()
        check(lib().xs_server_create(device, ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().xs_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_molecule(self, lines, mean_mass: float, ref_temp: float = 296.0) -> int:
        """lines: a synth.LineList (host numpy arrays, nu ascending, gamma per atm)."""
        import numpy as np

        arrs = [np.ascontiguousarray(lines.nu, np.float64),
                np.ascontiguousarray(lines.energies, np.float64),
                np.ascontiguousarray(lines.aif, np.float64),
                np.ascontiguousarray(lines.gns, np.int32),
                np.ascontiguousarray(lines.gamma, np.float64),
                np.ascontiguousarray(lines.n, np.float64)]
        mid = ctypes.c_int()
        check(lib().xs_server_add_molecule(self.h, *[a.ctypes.data for a in arrs], arrs[0].size,
                                           mean_mass, ref_temp, ctypes.byref(mid)))
        return mid.value

    def add_states(self, molecule: int, energies, gns) -> None:
        import numpy as np

        e = np.ascontiguousarray(energies, np.float64)
        g = np.ascontiguousarray(gns, np.int32)
        check(lib().xs_server_add_states(self.h, molecule, e.ctypes.data, g.ctypes.data, e.size))

    def submit(self, molecule: int, profile: int, precision: int, temperature: float,
               partition: float, pressure: float, f0: float, df: float, npoints: int,
               cut: float = -1.0) -> int:
        r = Request(molecule, profile, precision, temperature, partition, pressure, cut, f0, df,
                    npoints)
        rid = ctypes.c_ulonglong()
        check(lib().xs_server_submit(self.h, ctypes.byref(r), ctypes.byref(rid)))
        return rid.value

    def wait(self, rid: int, npoints: int, timeout_ms: int = -1):
        """(result as numpy float64[npoints], info dict)."""
        import numpy as np

        out = np.empty(npoints, np.float64)
        info = RequestInfo()
        check(lib().xs_server_wait(self.h, rid, out.ctypes.data, npoints, ctypes.byref(info),
                                   timeout_ms))
        return out, {k: getattr(info, k) for k, _ in RequestInfo._fields_}

    def pending(self):
        q, a = ctypes.c_int(), ctypes.c_int()
        check(lib().xs_server_pending(self.h, ctypes.byref(q), ctypes.byref(a)))
        return q.value, a.value


def partition_sum(energies, gns, temperatures, device: int = 0):
    """xs_partition_sum: Q(T) for each temperature from a state list."""
    import numpy as np

    e = np.ascontiguousarray(energies, np.float64)
    g = np.ascontiguousarray(gns, np.int32)
    t = np.ascontiguousarray(np.atleast_1d(temperatures), np.float64)
    q = np.empty(t.size)
    check(lib().xs_partition_sum(device, e.ctypes.data if e.size else None,
                                 g.ctypes.data if g.size else None, e.size, t.ctypes.data, t.size,
                                 q.ctypes.data))
    return q
