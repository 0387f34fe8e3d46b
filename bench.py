"""Benchmark of the cross-section hot path on B200.

Default workload (one "step"): the batched Voigt sweep -- 1e7 seeded lines,
grid 500-8000 cm-1 at 0.1 cm-1 (7.5e4 points), the 40 (T, P) conditions
T in {300..2100 K} x P in {1e-3, 0.1, 1, 10} bar, cut 25 cm-1 -- evaluated in
mixed precision by one CUDA-graph replay (grid check, step one for all 40
conditions, persistent step two).  Inputs stay resident in HBM; the per-step
working set (1e7 lines x 40 conditions of records, ~19 GB) is far larger
than L2, so no flush is needed between steps.

metric: Voigt line-evals/s = pairs (line, grid point) inside the reference
window, summed over the 40 conditions, per second of device time.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Under torchrun each rank runs its own 40-condition batch (temperatures shifted
by rank) with no data-path collective (weak scaling); rank 0 prints one JSON
line.  --impl reference times the reference's own OpenMPManager (compiled from
its sources into oracle/_ref/) on the host cores on a bounded sample of the
same workload.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# algorithmic FLOPs of one Voigt region-I pair: offset, x^2, the real
# rational's numerator and denominator, the scale and the accumulate, with the
# per-line terms hoisted (the reciprocal runs on the XU pipe, not counted)
FLOPS_PER_PAIR = 14
# XU-pipe reciprocals per region-I pair: two pairs of line-evals share one
RCP_PER_PAIR = 0.5


def hbm_view(traffic_bytes, ms):
    """Step two's DRAM traffic per launch over its time, against the
    measured copy bandwidth of this pool's B200s (MEASURED_PEAKS.json)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = None
    if os.path.exists(path):
        try:
            peak = float(json.load(open(path))["hbm_gbs"])
        except (OSError, ValueError, KeyError):
            peak = None
    if not traffic_bytes or not ms:
        return {"peak_gbs": peak, "achieved_gbs": None, "frac": None}
    gbs = traffic_bytes / (ms * 1e-3) / 1e9
    return {"peak_gbs": peak, "achieved_gbs": gbs, "frac": gbs / peak if peak else None,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peak else None}


METRIC = "Voigt line-evals/s & p99 request latency: mixed-precision batched vs plain FP64"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------------------
# workload
# --------------------------------------------------------------------------
def sweep_workload(n_lines: int, grid_points: int, rank: int = 0, workload: str = "sweep",
                   pbar: float = 1.0):
    from gpu_cross_b200 import synth

    if workload == "single":
        # Voigt single point: T = 1000 K, P = 1 bar, grid 500-8000 at 0.01
        lines, grid, cond = synth.voigt_single_workload(n_lines, grid_points)
        conds = [dict(temperature=cond["temperature"], partition=cond["partition"],
                      pressure_atm=pbar, cut=25.0)]
        common = dict(mean_mass=cond["mean_mass"], ref_temp=cond["ref_temp"])
    else:
        lines, grid, conds, common = synth.voigt_sweep_workload(n_lines, grid_points)
    if rank:
        conds = [dict(c, temperature=c["temperature"] + 10.0 * rank,
                      partition=synth.partition_poly(c["temperature"] + 10.0 * rank))
                 for c in conds]
    return lines, grid, conds, common


def pairs_gpu_window(nu: np.ndarray, freq: np.ndarray, cut: float) -> int:
    """Pairs with -cut <= nu - f <= cut (the reference GPU window)."""
    lo = np.searchsorted(freq, nu - cut, side="left")
    hi = np.searchsorted(freq, nu + cut, side="right")
    return int(np.sum(hi - lo))


def region_histogram(lines, grid, conds, common, stride: int = 50) -> dict:
    """Share of the window's (line, point) pairs in each W4 region, from every
    stride-th line: region I |x| + y >= 15, II >= 5.5, III y >= 0.195|x| - 0.176,
    IV the rest, with x = (nu - f) / (nu dpw) and y = gamma(T, P) / (nu dpw)
    as the GPU convention computes them (counted per line from the half-widths
    of each region in grid points)."""
    kb, c, na = 1.380658e-16, 2.99792458e10, 6.0221412927e23
    nu = lines.nu[::stride]
    gam, nex = lines.gamma[::stride], lines.n[::stride]
    fr = grid.freq()
    f0, df, npts = fr[0], grid.dfreq, grid.npoints

    def count(h):  # grid points with |nu - f| < h
        lo = np.clip(np.floor((nu - h - f0) / df) + 1, 0, npts)
        hi = np.clip(np.ceil((nu + h - f0) / df) - 1, -1, npts - 1)
        return np.maximum(hi - lo + 1, 0).sum()

    tot = {"I": 0.0, "II": 0.0, "III": 0.0, "IV": 0.0}
    for cd in conds:
        t = cd["temperature"]
        g = 1.0 / (nu * np.sqrt(2.0 * kb * t * na / common["mean_mass"]) / c)
        y = gam * cd["pressure_atm"] * (common["ref_temp"] / t) ** nex * g
        win = pairs_gpu_window(nu, fr, cd["cut"])
        n15 = count(np.maximum(15.0 - y, 0.0) / g)
        n55 = count(np.maximum(5.5 - y, 0.0) / g)
        # region III: |x| <= (y + 0.176) / 0.195 inside |x| < 5.5 - y
        n3 = count(np.clip(np.minimum(5.5 - y, (y + 0.176) / 0.195), 0.0, None) / g)
        tot["I"] += win - n15
        tot["II"] += n15 - n55
        tot["III"] += n3
        tot["IV"] += n55 - n3
    s = sum(tot.values())
    return {k: v / s for k, v in tot.items()} if s > 0 else tot


def pairs_cpu_window(nu: np.ndarray, f0: float, df: float, npts: int, cut: float) -> int:
    """Pairs of the reference OpenMPManager window
    [round((nu-cut-f0)/df), round((nu+cut-f0)/df)) clamped to the grid."""
    ib = np.clip(np.round((nu - cut - f0) / df), 0, npts)
    ie = np.clip(np.round((nu + cut - f0) / df), 0, npts)
    return int(np.sum(np.maximum(ie - ib, 0)))


def pairs_doppler_evaluated(nu: np.ndarray, freq: np.ndarray, cut: float, temperature: float,
                            mass: float) -> int:
    """Pairs the Doppler kernel actually evaluates: the reference window
    narrowed to the span where the two erf arguments are not both beyond 6
    on one side (those pairs add exactly 0 in FP64 and are skipped), with the
    margins step one uses."""
    kb, c, na = 1.380658e-16, 2.99792458e10, 6.0221412927e23
    dpw = np.sqrt(2.0 * kb * temperature * na / mass) / c
    f0, df, n = freq[0], freq[1] - freq[0], len(freq)
    lo = np.searchsorted(freq, nu - cut, side="left")
    hi = np.searchsorted(freq, nu + cut, side="right")
    w = 6.0 * dpw * (1.0 + 1e-6)
    m = 0.5 * df * (1.0 + 1e-6) + 2.0 * df
    alo = np.clip(np.floor((nu * (1.0 - w) - m - f0) / df), 0, n)
    ahi = np.clip(np.ceil((nu * (1.0 + w) + m - f0) / df) + 1.0, 0, n)
    return int(np.sum(np.maximum(np.minimum(hi, ahi) - np.maximum(lo, alo), 0)))


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
               "-lms", "200"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        loaded = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------
# reference CPU (OpenMPManager compiled from the reference sources)
# --------------------------------------------------------------------------
def _reference_cpu_slice(lines, cond, common, n: int):
    """The middle n lines of the list, with gamma scaled to the condition's
    pressure (the reference takes gamma per unit pressure as uploaded)."""
    mid = len(lines) // 2
    a = max(0, mid - n // 2)
    part = lines.slice(a, a + n)
    part.gamma = part.gamma * cond["pressure_atm"]
    return part


def reference_cpu_run(part, grid, cond, common, threads):
    """One run of the reference OpenMPManager over `part` on the whole grid;
    returns (pairs of its window, seconds)."""
    import oracle

    fr = grid.freq()
    c = dict(temperature=cond["temperature"], partition=cond["partition"],
             mean_mass=common["mean_mass"], pressure=1.0, ref_temp=common["ref_temp"])
    z = np.zeros_like(fr)
    t = time.perf_counter()
    oracle.ref_cpu(oracle.VOIGT, fr, z, part, c, grid.dfreq, nthreads=threads)
    dt = time.perf_counter() - t
    return pairs_cpu_window(part.nu, fr[0], grid.dfreq, len(fr), 25.0), dt


def reference_cpu_calibrate(lines, grid, cond, common, target_s: float, threads: int) -> int:
    """Line count of a middle slice that the reference OpenMPManager takes
    about target_s seconds for."""
    n = 20000
    _, dt = reference_cpu_run(_reference_cpu_slice(lines, cond, common, n), grid, cond, common, threads)
    while dt < 1.0 and n < len(lines):
        n = min(len(lines), n * 4)
        _, dt = reference_cpu_run(_reference_cpu_slice(lines, cond, common, n), grid, cond, common,
                                  threads)
    return int(min(len(lines), max(n, n * target_s / max(dt, 1e-3))))


def reference_cpu_describe(part, cond, threads, pairs, dt) -> str:
    return (f"reference OpenMPManager (g++ -O3, no -march), {threads} threads, one condition "
            f"(T={cond['temperature']:.0f} K, P={cond['pressure_atm'] / 0.986923:.3g} bar), "
            f"{len(part)} lines nu {part.nu[0]:.1f}-{part.nu[-1]:.1f} cm-1 of the 1e7-line list, "
            f"{pairs:.3e} pairs in {dt:.2f} s")


def reference_cpu_sample(lines, grid, cond, common, target_s: float = 12.0, threads=None):
    """Time the reference OpenMPManager on a nu-slice of the line list sized
    for about target_s seconds; returns (pairs/s, threads, description)."""
    threads = threads or os.cpu_count() or 1
    n = reference_cpu_calibrate(lines, grid, cond, common, target_s, threads)
    part = _reference_cpu_slice(lines, cond, common, n)
    pairs, dt = reference_cpu_run(part, grid, cond, common, threads)
    return pairs / dt, threads, reference_cpu_describe(part, cond, threads, pairs, dt)


def reference_gpu_sample(lines, grid, cond, common, n_lines: int = 400_000, device=None):
    """Time the reference's own step-one/step-two kernels (cross_kernal.cu for
    sm_100a, oracle/_ref/libref_gpu.so) on a contiguous slice of the list for
    one condition, chunked at 80000 grid points as BaseProfile does, and
    compare their spectrum with the engine's plain-FP64 result for the same
    slice and chunks (the FP64 parity tier, <= 1e-10 relative above 1e-6 of
    the peak)."""
    import torch

    import oracle
    from gpu_cross_b200 import capi

    fr = grid.freq()
    mid = len(lines) // 2
    part = lines.slice(mid - n_lines // 2, mid + n_lines // 2)
    part.gamma = part.gamma * cond["pressure_atm"]
    c = dict(temperature=cond["temperature"], partition=cond["partition"],
             mean_mass=common["mean_mass"], pressure=1.0, ref_temp=common["ref_temp"])
    span_pts = (part.nu[-1] - part.nu[0]) / grid.dfreq + 2 * 25.0 / grid.dfreq
    chunks = max(1, int(np.ceil(span_pts / 80000.0)))
    z = np.zeros_like(fr)
    ref_out, ms = oracle.ref_gpu(oracle.VOIGT, fr, z, part, c, grid.dfreq, chunks=chunks)
    pairs = pairs_gpu_window(part.nu, fr, 25.0)

    # the engine, FP64 and the GPU convention, over the same line chunks and
    # grid slices (BaseProfile.cpp:55-57, as the harness applies it)
    dev = device or torch.device("cuda", 0)
    keys = ("nu", "energies", "aif", "gns", "gamma", "n")
    d = {k: torch.as_tensor(np.ascontiguousarray(getattr(part, k)), device=dev) for k in keys}
    dfr = torch.as_tensor(fr, device=dev)
    out = torch.zeros_like(dfr)
    eng = capi.Engine(dev.index)
    try:
        eng.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        opts = capi.make_options(capi.VOIGT, grid.dfreq, common["mean_mass"], precision=capi.FP64,
                                 ref_temp=common["ref_temp"])
        cc = [capi.make_condition(cond["temperature"], cond["partition"], 1.0, 1.0, -1.0)]
        n = len(part)
        per = (n + chunks - 1) // chunks
        for k in range(chunks):
            a, b = k * per, min(n, (k + 1) * per)
            if b <= a:
                break
            ib, npts = 0, len(fr)
            if chunks > 1:
                ib = int(max(np.round((part.nu[a] - 25.0 - fr[0]) / grid.dfreq), 0.0))
                ie = int(min(np.round((part.nu[b - 1] + 25.0 - fr[0]) / grid.dfreq), float(len(fr))))
                npts = ie - ib
                if npts <= 0:
                    continue
            dk = {key: v[a:b] for key, v in d.items()}
            eng.execute(opts, cc, capi.make_lines(dk), capi.make_grid(dfr, ib, npts), out.data_ptr())
        eng.sync()
    finally:
        eng.close()
    ours = out.cpu().numpy()
    peak = np.abs(ref_out).max()
    big = np.abs(ref_out) > 1e-6 * peak
    rel = float(np.max(np.abs(ours[big] - ref_out[big]) / np.abs(ref_out[big]))) if big.any() else 0.0
    small_abs = float(np.max(np.abs(ours[~big] - ref_out[~big])) / peak) if (~big).any() else 0.0
    return {"value": pairs / (ms * 1e-3), "unit": "line-evals/s", "kernel_ms": ms,
            "fp64_vs_reference_kernel_max_rel": rel,
            "fp64_vs_reference_kernel_max_abs_below_floor": small_abs,
            "sample": f"reference cross_kernal.cu (FP64, sm_100a) step one + step two, one condition "
                      f"(T={cond['temperature']:.0f} K), {len(part)} lines nu {part.nu[0]:.1f}-"
                      f"{part.nu[-1]:.1f} cm-1, {chunks} chunk(s), {pairs:.3e} pairs; its spectrum "
                      f"against the engine's FP64 result on the same slice and chunks"}


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def run_ours(args, rank, world, dist):
    import torch

    from gpu_cross_b200 import capi

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    lines, grid, conds, common = sweep_workload(args.lines, args.points, rank, args.workload,
                                                args.pbar)
    if args.conds < len(conds):
        step = len(conds) / float(args.conds)
        conds = [conds[int(k * step)] for k in range(args.conds)]
    fr = grid.freq()
    npts = len(fr)
    nc = len(conds)
    pairs_per_cond = pairs_gpu_window(lines.nu, fr, 25.0)
    pairs_step = pairs_per_cond * nc
    log(f"[bench] rank {rank}: {len(lines)} lines, {npts} points, {nc} conditions, "
        f"{pairs_step:.3e} line-evals per step")

    keys = ("nu", "energies", "aif", "gns", "gamma", "n")
    host = {k: torch.from_numpy(np.ascontiguousarray(getattr(lines, k))).pin_memory() for k in keys}
    d = {k: host[k].to(dev, non_blocking=False) for k in keys}
    dfr = torch.as_tensor(fr, device=dev)
    out = torch.zeros((nc, npts), dtype=torch.float64, device=dev)
    out_f64 = torch.zeros_like(out) if not args.no_fp64 else None
    stream = torch.cuda.current_stream(dev)

    eng = capi.Engine(dev.index)
    eng.set_stream(stream.cuda_stream)
    cc = [capi.make_condition(c["temperature"], c["partition"], 1.0, c["pressure_atm"], c["cut"])
          for c in conds]
    L = capi.make_lines(d)
    G = capi.make_grid(dfr)
    o_mix = capi.make_options(capi.VOIGT, grid.dfreq, common["mean_mass"], precision=capi.MIXED,
                              ref_temp=common["ref_temp"], points_per_thread=args.P,
                              warps_per_block=args.W, conditions_per_warp=args.C,
                              line_splits=args.S)
    o_f64 = capi.make_options(capi.VOIGT, grid.dfreq, common["mean_mass"], precision=capi.FP64,
                              ref_temp=common["ref_temp"], conditions_per_warp=args.C64,
                              line_splits=args.S)
    tuned = None
    if not (args.P or args.W or args.C or args.C64) and not args.no_tune:
        # launch shapes measured on this workload (outside the timed region)
        tuned = {"mixed": eng.autotune(o_mix, cc, L, G, out.data_ptr(), npts)}
        if out_f64 is not None:
            tuned["fp64"] = eng.autotune(o_f64, cc, L, G, out_f64.data_ptr(), npts)
            out_f64.zero_()
        out.zero_()
        log(f"[bench] autotuned: {tuned}")
    g_mix = eng.capture(o_mix, cc, L, G, out.data_ptr(), npts, zero_out=True)
    mix_kernels = g_mix.kernel_count()  # kernels one replay (one step) launches
    eng2 = g_f64 = None
    if not args.no_fp64:
        eng2 = capi.Engine(dev.index)
        eng2.set_stream(stream.cuda_stream)
        g_f64 = eng2.capture(o_f64, cc, L, G, out_f64.data_ptr(), npts, zero_out=True)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(v: float) -> float:
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # peaks of this GPU (roofline denominators of the FP32/FP64 pipes)
    peaks = capi.measure_peaks(dev.index)

    # warm-up
    for _ in range(args.warmup):
        g_mix.launch(stream.cuda_stream)
    if g_f64 is not None:
        g_f64.launch(stream.cuda_stream)
    torch.cuda.synchronize(dev)

    # accuracy of the mixed result against the FP64 sweep (same inputs)
    g_mix.launch(stream.cuda_stream)
    torch.cuda.synchronize(dev)
    a = out.cpu().numpy()
    b = out_f64.cpu().numpy() if out_f64 is not None else a
    rel_max, integ_max = 0.0, 0.0
    for k in range(nc if out_f64 is not None else 0):
        peak = np.abs(b[k]).max()
        big = np.abs(b[k]) > 1e-6 * peak
        rel_max = max(rel_max, float(np.max(np.abs(a[k][big] - b[k][big]) / np.abs(b[k][big]))))
        integ_max = max(integ_max, abs(a[k].sum() - b[k].sum()) / abs(b[k].sum()))

    # timed region: K mixed sweeps
    gpu_uuid = None
    try:
        gpu_uuid = str(torch.cuda.get_device_properties(dev).uuid)
        if not gpu_uuid.startswith("GPU-"):
            gpu_uuid = "GPU-" + gpu_uuid
    except Exception:
        gpu_uuid = None
    clocks = ClockSampler(gpu_uuid)
    clocks.start()
    time.sleep(0.3)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    step2 = []
    prep = []
    e0.record(stream)
    for _ in range(args.steps):
        g_mix.launch(stream.cuda_stream)
        p_ms, s_ms = eng.last_stats()
        prep.append(p_ms)
        step2.append(s_ms)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_total = e0.elapsed_time(e1)
    barrier()
    clk = clocks.stop()
    ms_total = max_over_ranks(ms_total)
    ms_step = ms_total / args.steps
    value = pairs_step * world / (ms_step * 1e-3)

    # plain FP64 sweep, same workload
    f64_ms = []
    for _ in range(max(2, args.steps // 3) if g_f64 is not None else 0):
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        g_f64.launch(stream.cuda_stream)
        t1.record(stream)
        torch.cuda.synchronize(dev)
        f64_ms.append(t0.elapsed_time(t1))
    f64_step = max_over_ranks(float(np.mean(f64_ms))) if f64_ms else float("nan")
    f64_value = pairs_step * world / (f64_step * 1e-3) if f64_ms else None

    # end-to-end through xs_engine_execute_host: pinned host lines -> device
    # in 16 slices whose copies overlap step one, sweep, result -> pinned host
    out_host = torch.empty((nc, npts), dtype=torch.float64).pin_memory()
    h2d = sum(int(host[k].numel() * host[k].element_size()) for k in keys)
    d2h = int(out.numel() * out.element_size())
    e2e_steps = 0 if args.no_e2e else max(2, args.steps // 2)
    L_host = capi.make_lines(host)
    barrier()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(e2e_steps):
        out.zero_()
        eng.execute_host(o_mix, cc, L_host, L, G, out.data_ptr(), npts, out_host.data_ptr(), pieces=16)
    s1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(s0.elapsed_time(s1) / e2e_steps) if e2e_steps else float("nan")
    e2e_value = pairs_step * world / (e2e_ms * 1e-3) if e2e_steps else None

    # error statement of the mixed result: the a-priori bound and a sampled
    # FP64 re-evaluation of 8 rows per condition (one execute outside the
    # timed region)
    shape = (tuned or {}).get("mixed") or {}
    o_chk = capi.make_options(capi.VOIGT, grid.dfreq, common["mean_mass"], precision=capi.MIXED,
                              ref_temp=common["ref_temp"],
                              points_per_thread=shape.get("points_per_thread", args.P),
                              warps_per_block=shape.get("warps_per_block", args.W),
                              conditions_per_warp=shape.get("conditions_per_warp", args.C),
                              line_splits=args.S, check_rows=8)  # the timed launch shape
    out.zero_()
    eng.execute(o_chk, cc, L, G, out.data_ptr(), npts)
    error_statement = eng.accuracy()
    error_statement["how"] = ("bound_rel: a-priori bound (every grid point and the band integral); "
                              "sampled_*: FP64 re-evaluation of 8 evenly spaced 32-point rows per "
                              "condition in the same call, worst over conditions")

    step2_ms = float(np.mean(step2))
    achieved = pairs_step * FLOPS_PER_PAIR / (step2_ms * 1e-3) / 1e12
    traffic = xu_pct = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            tj = json.load(open(tpath))
            traffic = tj.get("steptwo_mixed_sweep_bytes_per_launch")
            xu_pct = tj.get("steptwo_mixed_sweep_xu_pipe_pct")
        except (OSError, ValueError):
            traffic = None
    if args.workload != "sweep" or grid.npoints != 75_000:
        traffic = xu_pct = None  # measured on the sweep's grid and conditions only
    elif traffic:
        traffic = traffic * lines.nu.size / 1e7  # step two's reads grow with the line count
    regions = region_histogram(lines, grid, conds, common) if args.workload == "sweep" else None

    # the reference's own GPU kernels (cross_kernal.cu built for sm_100a) on a
    # bounded sample: one condition, a nu-slice of the list, chunked the way
    # BaseProfile feeds GpuManager (MAX-POINTS 80000 per chunk)
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        try:
            ref_gpu = reference_gpu_sample(lines, grid, conds[min(26, len(conds) - 1)], common,
                                           device=dev)
        except Exception as exc:
            ref_gpu = {"value": None, "sample": f"not run: {exc}"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            rate, thr, desc = reference_cpu_sample(lines, grid, conds[min(26, len(conds) - 1)], common,
                                                   target_s=args.cpu_seconds)
            cpu = {"value": rate, "unit": "line-evals/s", "cores": thr, "kind": "reference",
                   "sample": desc}
        except Exception as exc:  # the reference build is test infrastructure
            cpu = {"value": None, "unit": "line-evals/s", "cores": 0, "kind": "reference",
                   "sample": f"not run: {exc}"}

    for gobj in (g_mix, g_f64):
        if gobj is not None:
            gobj.close()
    eng.close()
    if eng2 is not None:
        eng2.close()
    del d, out, out_f64, out_host
    torch.cuda.empty_cache()

    serving = None
    if rank == 0 and world == 1 and not args.no_serve:
        try:
            serving = run_serving(args, dev.index)
        except Exception as exc:
            serving = {"error": f"{type(exc).__name__}: {exc}"}

    if rank != 0:
        return None
    return {
        "metric": METRIC,
        "value": value,
        "unit": "line-evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 profile / f64 offsets+intensities+tile sums",
        "data": "synthetic (seeded; no line list ships with the reference)",
        "config": {
            "workload": (("voigt_sweep_40tp: 1e7 lines, nu U(500,8000), grid 500-8000 cm-1 at 0.1 "
                          "(7.5e4 points), T 300-2100 K x P {1e-3,0.1,1,10} bar, cut 25 cm-1")
                         if args.workload == "sweep" else
                         ("voigt_single: 1e7 lines, nu U(500,8000), grid 500-8000 cm-1 at 0.01 "
                          "(7.5e5 points), T 1000 K, P 1 bar, cut 25 cm-1"))
                        + ", mixed precision, one CUDA-graph replay per step",
            "lines": len(lines), "grid_points": npts, "conditions": nc,
            "line_evals_per_step": pairs_step,
            "parallelism": f"{world} rank(s), independent (T,P) batches, no collective",
            "l2": "inputs larger than L2 (per-step records > 0.6 GB), no flush",
            "launch_shape": tuned if tuned else {"points_per_thread": args.P or "default",
                                                 "warps_per_block": args.W or "default",
                                                 "conditions_per_warp": args.C or "auto"},
        },
        "accuracy_vs_fp64": {"max_rel_above_1e-6_peak": rel_max, "max_integrated_rel": integ_max},
        "error_statement": error_statement,
        "grid_points_per_s": npts * nc * world / (ms_step * 1e-3),
        "fp64": {"value": f64_value, "ms_per_step": f64_step, "unit": "line-evals/s",
                 "grid_points_per_s": npts * nc * world / (f64_step * 1e-3) if f64_ms else None},
        "speedup_mixed_vs_fp64": value / f64_value if f64_value else None,
        "kernel_ms": {"steptwo_mean": step2_ms, "prep_mean": float(np.mean(prep))},
        "roofline": {
            "bound": "fp32", "achieved": achieved, "peak": peaks["fp32_tflops"],
            "unit": "TFLOP/s", "frac": achieved / peaks["fp32_tflops"], "traffic": traffic,
            "peak_source": "measured (in-repo FP32 FMA probe, xs_measure_peaks, burst)",
            "flops_per_pair": FLOPS_PER_PAIR,
            "other_peaks": peaks,
            "region_share": regions,
            "xu_pipe_pct_ncu": xu_pct if args.workload == "sweep" else None,
            "mufu_view": {
                "achieved_rcp_per_s": pairs_step * RCP_PER_PAIR / (step2_ms * 1e-3),
                "peak_rcp_per_s": peaks.get("rcp32_tops", 0.0) * 1e12,
                "rcp_per_pair": RCP_PER_PAIR,
                "note": "reciprocals on the XU pipe: one per two region-I line-evals (shared)"},
            "hbm_view": hbm_view(traffic, step2_ms),
        },
        "cpu_baseline": cpu,
        "reference_gpu_kernel": ref_gpu,
        "e2e": {"value": e2e_value, "unit": "line-evals/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "grid_points_per_s": npts * nc * world / (e2e_ms * 1e-3) if e2e_steps else None},
        "serving": serving,
        "gpu_launches": mix_kernels * args.steps,
        "clocks": clk,
        "when": datetime.datetime.now(datetime.timezone.utc).isoformat(),
    }


def run_doppler(args, rank, world, dist):
    """Plain Doppler in FP64 (configuration 1): ExoMol-style list of 20k states
    and 1e6 transitions, T = 296 K, Q = 2844, M = 30.01, grid 0-10000 cm-1 at
    0.01 (1e6 points), cut 25 -- and the reference's own cut of 100 beside it,
    the one its unmodified OpenMPManager (the CPU baseline) uses."""
    import torch

    import oracle
    from gpu_cross_b200 import capi, synth

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    lines, grid, cond = synth.doppler_exomol_workload()
    fr = grid.freq()
    keys = ("nu", "energies", "aif", "gns")
    host = {k: torch.from_numpy(np.ascontiguousarray(getattr(lines, k))).pin_memory() for k in keys}
    d = {k: host[k].to(dev) for k in keys}
    dfr = torch.as_tensor(fr, device=dev)
    out = torch.zeros(grid.npoints, dtype=torch.float64, device=dev)
    out_host = torch.empty(grid.npoints, dtype=torch.float64).pin_memory()
    stream = torch.cuda.current_stream(dev)
    eng = capi.Engine(dev.index)
    eng.set_stream(stream.cuda_stream)
    L = capi.make_lines(d)
    G = capi.make_grid(dfr)
    opts = capi.make_options(capi.DOPPLER, grid.dfreq, cond["mean_mass"])
    res = {}
    for cut in (25.0, 100.0):
        cc = [capi.make_condition(cond["temperature"], cond["partition"], 1.0, 1.0, cut)]
        pairs = pairs_gpu_window(lines.nu, fr, cut)
        g = eng.capture(opts, cc, L, G, out.data_ptr(), grid.npoints, zero_out=True)
        for _ in range(args.warmup):
            g.launch(stream.cuda_stream)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            g.launch(stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / args.steps
        # end to end: lines from pinned host, the pass, the grid back
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(2):
            for k in keys:
                d[k].copy_(host[k], non_blocking=True)
            g.launch(stream.cuda_stream)
            out_host.copy_(out, non_blocking=True)
        s1.record(stream)
        torch.cuda.synchronize(dev)
        res[cut] = dict(pairs=pairs, ms=ms, e2e_ms=s0.elapsed_time(s1) / 2, kernels=g.kernel_count(),
                        evaluated=pairs_doppler_evaluated(lines.nu, fr, cut, cond["temperature"],
                                                          cond["mean_mass"]))
        g.close()
    eng.close()
    # the reference OpenMPManager (unmodified: cut 100) on a slice, and the
    # oracle check of the GPU result on the same slice
    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        c = dict(temperature=cond["temperature"], partition=cond["partition"],
                 mean_mass=cond["mean_mass"], pressure=1.0, ref_temp=296.0)
        n = 20000
        while True:
            part = lines.slice(len(lines) // 2 - n // 2, len(lines) // 2 + n // 2)
            t = time.perf_counter()
            oracle.ref_cpu(oracle.DOPPLER, fr, np.zeros_like(fr), part, c, grid.dfreq, nthreads=threads)
            dt = time.perf_counter() - t
            if dt > args.cpu_seconds / 4 or n >= len(lines):
                break
            n = min(len(lines), n * 4)
        pairs_cpu = pairs_cpu_window(part.nu, fr[0], grid.dfreq, len(fr), 100.0)
        cpu = {"value": pairs_cpu / dt, "unit": "line-evals/s", "cores": threads, "kind": "reference",
               "sample": (f"reference OpenMPManager Doppler (unmodified, cut 100), {threads} threads, "
                          f"{len(part)} of the 1e6 lines, {pairs_cpu:.3e} pairs in {dt:.2f} s")}
    v25 = res[25.0]["pairs"] * world / (res[25.0]["ms"] * 1e-3)
    if rank != 0:
        return None
    return {
        "metric": METRIC,
        "value": v25,
        "unit": "line-evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": res[25.0]["ms"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": ("doppler_exomol_1e6: 20k states, 1e6 transitions nu 0-10000, "
                                "T 296 K, Q 2844, M 30.01, grid 0-10000 at 0.01 (1e6 points), cut 25, FP64"),
                   "lines": len(lines), "grid_points": grid.npoints,
                   "line_evals_per_step": res[25.0]["pairs"]},
        "evaluated_pairs_per_s": res[25.0]["evaluated"] * world / (res[25.0]["ms"] * 1e-3),
        "evaluated_pairs_per_step": res[25.0]["evaluated"],
        "grid_points_per_s": grid.npoints * world / (res[25.0]["ms"] * 1e-3),
        "cut_100": {"value": res[100.0]["pairs"] * world / (res[100.0]["ms"] * 1e-3),
                    "ms_per_step": res[100.0]["ms"], "line_evals_per_step": res[100.0]["pairs"],
                    "evaluated_pairs_per_s": res[100.0]["evaluated"] * world / (res[100.0]["ms"] * 1e-3)},
        "cpu_baseline": cpu,
        "e2e": {"value": res[25.0]["pairs"] * world / (res[25.0]["e2e_ms"] * 1e-3),
                "unit": "line-evals/s", "ms_per_step": res[25.0]["e2e_ms"],
                "h2d_bytes_per_step": int(sum(host[k].numel() * host[k].element_size() for k in keys)),
                "d2h_bytes_per_step": int(grid.npoints * 8)},
        "note": ("pairs beyond ~6 Doppler widths add exactly 0 in FP64 and are skipped, so the "
                 "line-evals/s counts the reference window, most of which needs no work"),
        "gpu_launches": res[25.0]["kernels"] * args.steps,
        "when": datetime.datetime.now(datetime.timezone.utc).isoformat(),
    }


def run_stream(args, rank, world, dist):
    """The streamed configuration: 5e8 lines (after the 1e-30 intensity
    pre-filter) held in pinned host memory as FP64 centres + FP32 S(T) and
    gamma(T, P), one Voigt pass per step over grid 100-12000 cm-1 at 0.01
    (1.19e6 points), T = 2000 K, P = 1 bar, cut 25; chunks copied on a second
    stream while earlier chunks are evaluated (xs_stream_execute)."""
    import torch

    from gpu_cross_b200 import capi, synth

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    nu, s, g, kept, generated = synth.stream_workload(args.lines, seed=1004 + rank)
    grid = synth.Grid(100.0, 12000.0, 1_190_000)
    fr = grid.freq()
    log(f"[stream] rank {rank}: {kept:.4g} of {generated:.4g} lines kept, generated in "
        f"{time.perf_counter() - t0:.1f} s")
    pairs = 0
    for b0 in range(0, nu.size, 20_000_000):
        pairs += pairs_gpu_window(nu[b0:b0 + 20_000_000], fr, 25.0)
    h_nu = torch.from_numpy(nu).pin_memory()
    h_s = torch.from_numpy(s).pin_memory()
    h_g = torch.from_numpy(g).pin_memory()
    del nu, s, g
    dfr = torch.as_tensor(fr, device=dev)
    out = torch.zeros(grid.npoints, dtype=torch.float64, device=dev)
    out_host = torch.empty(grid.npoints, dtype=torch.float64).pin_memory()
    eng = capi.Engine(dev.index)
    stream = torch.cuda.current_stream(dev)
    eng.set_stream(stream.cuda_stream)
    cond = capi.make_condition(2000.0, synth.partition_poly(2000.0), 1.0, 1.0, 25.0)
    G = capi.make_grid(dfr)

    def one(prec):
        out.zero_()
        opts = capi.make_options(capi.VOIGT, grid.dfreq, 17.03, precision=prec)
        return eng.stream_execute(opts, cond, h_nu.data_ptr(), h_s.data_ptr(), h_g.data_ptr(),
                                  h_nu.numel(), G, out.data_ptr(), args.chunk_lines)

    for _ in range(args.warmup):
        one(capi.MIXED)
    clocks = ClockSampler(None)
    clocks.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    st_list = [one(capi.MIXED) for _ in range(args.steps)]
    clk = clocks.stop()
    ms = float(np.mean([st["total_ms"] for st in st_list]))
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    copy_ms = float(np.mean([st["copy_span_ms"] for st in st_list]))
    h2d = st_list[0]["h2d_bytes"]
    mixed_out = out.cpu().numpy()
    f64 = one(capi.FP64)
    f64_out = out.cpu().numpy()
    peak = np.abs(f64_out).max()
    big = np.abs(f64_out) > 1e-6 * peak
    rel = float(np.max(np.abs(mixed_out[big] - f64_out[big]) / np.abs(f64_out[big])))
    integ = abs(mixed_out.sum() - f64_out.sum()) / abs(f64_out.sum())
    # end to end: the pass plus the result read back to pinned host memory
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(2):
        one(capi.MIXED)
        out_host.copy_(out, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = e0.elapsed_time(e1) / 2
    eng.close()
    value = pairs * world / (ms * 1e-3)
    if rank != 0:
        return None
    return {
        "metric": METRIC,
        "value": value,
        "unit": "line-evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 profile / f64 offsets+tile sums; f32 S and gamma as stored",
        "data": "synthetic (seeded)",
        "config": {
            "workload": ("voigt_stream_5e8: nu U(100,12000), E'' Exp(4000), A logU(1e-8,1e3), "
                         "T 2000 K, P 1 bar, grid 0.01 (1.19e6 points), cut 25, S >= 1e-30 kept; "
                         "lines in pinned host memory, chunks copied while earlier chunks run"),
            "lines_generated": generated, "lines_kept": kept, "grid_points": grid.npoints,
            "line_evals_per_step": pairs, "chunk_lines": args.chunk_lines,
            "inputs": "host-resident by design: value includes the host-to-device copies",
        },
        "accuracy_vs_fp64": {"max_rel_above_1e-6_peak": rel, "max_integrated_rel": integ},
        "fp64": {"ms_per_step": f64["total_ms"], "value": pairs / (f64["total_ms"] * 1e-3),
                 "unit": "line-evals/s"},
        "grid_points_per_s": grid.npoints * world / (ms * 1e-3),
        "h2d": {"bytes_per_step": h2d, "copy_span_ms": copy_ms,
                "gb_per_s_over_copy_span": h2d / (copy_ms * 1e-3) / 1e9},
        "e2e": {"value": pairs * world / (e2e_ms * 1e-3), "unit": "line-evals/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(grid.npoints * 8),
                "ms_per_step": e2e_ms},
        "gpu_launches": int(sum(st["kernels"] for st in st_list)),
        "clocks": clk,
        "when": datetime.datetime.now(datetime.timezone.utc).isoformat(),
    }


def run_serving(args, dev_index: int):
    """The request server under a seeded Poisson stream (three resident
    molecules of 1e6, 1e7 and 1e8 lines), once with every request in mixed
    precision and once in plain FP64.  Latency is the server's own: submit to
    result in pinned host memory."""
    import queue

    from gpu_cross_b200 import capi, synth

    t0 = time.perf_counter()
    mols = synth.serving_molecules(args.serve_scale)
    trace = synth.serving_trace(rate=args.serve_rate, duration_s=args.serve_seconds)
    log(f"[serve] {len(mols)} molecules ({sum(len(l) for l, _ in mols):.3e} lines) and "
        f"{len(trace)} requests generated in {time.perf_counter() - t0:.1f} s")
    srv = capi.Server(dev_index, policy=args.serve_policy, lanes=args.serve_lanes, depth=args.serve_depth,
                      chunk_pairs=args.serve_chunk_pairs)
    try:
        mids = [srv.add_molecule(l, m) for l, m in mols]
        del mols

        def submit(r, prec):
            return srv.submit(mids[r["molecule"]], capi.VOIGT if r["voigt"] else capi.DOPPLER, prec,
                              r["temperature"], r["partition"], r["pressure"], r["f0"], r["df"],
                              r["npoints"], cut=r["cut"])

        def stream(prec):
            q: queue.Queue = queue.Queue()
            infos = []
            done_at = []

            def waiter():
                while True:
                    item = q.get()
                    if item is None:
                        return
                    rid, n = item
                    _, info = srv.wait(rid, n)
                    infos.append(info)
                    done_at.append(time.perf_counter())

            th = threading.Thread(target=waiter)
            th.start()
            late = []
            start = time.perf_counter()
            for r in trace:
                dt = r["t"] - (time.perf_counter() - start)
                if dt > 0:
                    time.sleep(dt)
                late.append(time.perf_counter() - start - r["t"])
                q.put((submit(r, prec), r["npoints"]))
            q.put(None)
            th.join()
            span = max(done_at) - start
            lat = np.array([i["latency_ms"] for i in infos])
            evals = float(sum(i["line_evals"] for i in infos))
            vo = np.array([r["voigt"] for r in trace])
            return {
                "requests": len(infos), "seconds": span,
                "requests_per_s": len(infos) / span,
                "line_evals_per_s": evals / span,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "max_ms": float(lat.max()), "mean_ms": float(lat.mean()),
                "p99_ms_voigt": float(np.percentile(lat[vo], 99)) if vo.any() else None,
                "p99_ms_doppler": float(np.percentile(lat[~vo], 99)) if (~vo).any() else None,
                "queue_p99_ms": float(np.percentile([i["queue_ms"] for i in infos], 99)),
                "submit_late_p99_ms": float(np.percentile(late, 99) * 1e3),
                "chunks": int(sum(i["chunks"] for i in infos)),
                "chunks_from_tcache": int(sum(i["tcache_chunks"] for i in infos)),
            }

        # warm-up: the first requests of the trace, one at a time
        for r in trace[:16]:
            srv.wait(submit(r, capi.MIXED), r["npoints"])
            srv.wait(submit(r, capi.FP64), r["npoints"])
        res = {"mixed": stream(capi.MIXED), "fp64": stream(capi.FP64)}

        # A lower bound on the mixed stream's p99: a request's latency is at
        # least its latency alone on an idle server, so the k-th largest
        # latency is at least the k-th largest alone latency.  The requests
        # with the most estimated work are timed alone, one at a time (the
        # rest count as 0, which keeps the bound a bound).
        dens = [n * args.serve_scale / 12000.0 for n, _ in synth.SERVE_MOLECULES]
        # (Doppler pairs beyond a few Doppler widths are skipped: counted at 1/10)
        est = [dens[r["molecule"]] * r["npoints"] * 2.0 * r["cut"] * (1.0 if r["voigt"] else 0.1)
               for r in trace]
        heavy = sorted(range(len(trace)), key=lambda k: -est[k])[:args.serve_alone]
        alone = []
        for k in heavy:
            r = trace[k]
            _, info = srv.wait(submit(r, capi.MIXED), r["npoints"])
            alone.append(info["latency_ms"])
        padded = np.zeros(len(trace))
        padded[:len(alone)] = alone
        res["mixed"]["p99_lower_bound_ms"] = float(np.percentile(padded, 99))
        res["mixed"]["alone_ms_largest"] = sorted(alone, reverse=True)[:25]
        res["mixed"]["alone_how"] = (f"the {len(alone)} requests with the most estimated work "
                                     "(window-overlap pairs) timed alone on the idle server")
    finally:
        srv.close()
    res["config"] = (f"{len(trace)} requests, Poisson {args.serve_rate:g}/s over "
                     f"{args.serve_seconds:g} s (seed 1005); molecules "
                     f"{'/'.join(f'{n * args.serve_scale:.0e}' for n, _ in synth.SERVE_MOLECULES)} "
                     "lines (M 18.02/30.01/16.04), T U(200,3000) K, P logU(1e-5,100) bar, "
                     "Doppler/Voigt 1:1, span U(100,5000) cm-1, df logU(0.01,1) cm-1, cut 25; "
                     f"chunk order {['least remaining work', 'round robin', 'earliest deadline'][args.serve_policy]}")
    res["line_evals"] = "window-overlap count (line, point) pairs inside +/-25 cm-1"
    return res


def run_extra_configs(args, rank, world, dist) -> dict:
    """The other configurations as extra keys of the default run, each with
    its own timing: "single" (1e7 lines, 7.5e5 points, T 1000 K, P 1 bar;
    mixed and plain FP64), "doppler" (the ExoMol-style 1e6-line list, FP64,
    cut 25 and the reference's 100) and "stream" (5e8 lines generated, those
    with S >= 1e-30 kept in pinned host memory, 3 timed passes)."""
    import copy

    out = {}
    a = copy.copy(args)
    a.steps, a.warmup = min(args.steps, 10), 3
    a.no_serve = a.no_ref_gpu = True
    a.no_tune = False
    a.P = a.W = a.C = a.C64 = a.S = 0
    a.no_cpu = True
    try:
        a1 = copy.copy(a)
        a1.workload, a1.points, a1.lines = "single", 750_000, 10_000_000
        r = run_ours(a1, rank, world, dist)
        if r is not None:
            out["single"] = {k: r.get(k) for k in (
                "value", "unit", "ms_per_step", "grid_points_per_s", "fp64", "speedup_mixed_vs_fp64",
                "accuracy_vs_fp64", "error_statement", "kernel_ms", "e2e", "gpu_launches")}
            out["single"]["config"] = r["config"]["workload"]
            out["single"]["launch_shape"] = r["config"]["launch_shape"]
            out["single"]["roofline_frac"] = r["roofline"]["frac"]
    except Exception as exc:
        out["single"] = {"error": f"{type(exc).__name__}: {exc}"}
    try:
        a2 = copy.copy(a)
        a2.workload = "doppler"
        a2.no_cpu = args.no_cpu
        a2.cpu_seconds = min(args.cpu_seconds, 6.0)
        r = run_doppler(a2, rank, world, dist)
        if r is not None:
            out["doppler"] = {k: r.get(k) for k in (
                "value", "unit", "ms_per_step", "line_evals_per_step", "evaluated_pairs_per_s",
                "evaluated_pairs_per_step", "grid_points_per_s", "cut_100", "cpu_baseline", "e2e",
                "note", "gpu_launches")}
            out["doppler"]["config"] = r["config"]["workload"]
    except Exception as exc:
        out["doppler"] = {"error": f"{type(exc).__name__}: {exc}"}
    try:
        a3 = copy.copy(a)
        a3.workload, a3.lines, a3.steps = "stream", 500_000_000, 3
        r = run_stream(a3, rank, world, dist)
        if r is not None:
            out["stream"] = {k: r.get(k) for k in (
                "value", "unit", "ms_per_step", "grid_points_per_s", "fp64", "accuracy_vs_fp64", "h2d",
                "e2e", "gpu_launches")}
            out["stream"]["config"] = r["config"]["workload"]
            out["stream"]["lines_kept"] = r["config"]["lines_kept"]
    except Exception as exc:
        out["stream"] = {"error": f"{type(exc).__name__}: {exc}"}
    return out


def run_reference(args, rank, world):
    """The reference's own OpenMPManager on the host cores; rank 0 only.  A
    step is one bounded sample of the sweep workload: one of its conditions
    (T = 1500 K, P = 1 bar) over a middle slice of the 1e7-line list on the
    full 7.5e4-point grid, the slice sized so that warm-up and timed steps
    together take about --ref-seconds.  ms_per_step is the measured time of
    that sample; value is its line-evals/s."""
    if rank != 0:
        return None
    lines, grid, conds, common = sweep_workload(args.lines, args.points, 0)
    cond = conds[min(26, len(conds) - 1)]
    threads = os.cpu_count() or 1
    per_step = max(1.0, min(args.cpu_seconds, args.ref_seconds / max(1, args.steps + args.warmup)))
    n = reference_cpu_calibrate(lines, grid, cond, common, per_step, threads)
    part = _reference_cpu_slice(lines, cond, common, n)
    for _ in range(args.warmup):
        reference_cpu_run(part, grid, cond, common, threads)
    times = []
    pairs = 0
    for _ in range(args.steps):
        pairs, dt = reference_cpu_run(part, grid, cond, common, threads)
        times.append(dt)
    ms = float(np.mean(times)) * 1e3
    v = pairs / (ms * 1e-3)
    desc = reference_cpu_describe(part, cond, threads, pairs, ms * 1e-3)
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "line-evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": (f"voigt_sweep_40tp sample: one of the 40 conditions (T "
                                f"{cond['temperature']:.0f} K, P {cond['pressure_atm'] / 0.986923:.3g} bar), "
                                f"{len(part)} of the 1e7 lines (middle nu slice), grid 500-8000 cm-1 at "
                                f"0.1 (7.5e4 points), cut 25 cm-1"),
                   "lines": len(part), "grid_points": grid.npoints, "conditions": 1,
                   "line_evals_per_step": pairs,
                   "full_workload": {"lines": len(lines), "conditions": len(conds)}},
        "cpu_baseline": {"value": v, "unit": "line-evals/s", "cores": threads, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": v, "unit": "line-evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--lines", type=int, default=10_000_000)
    ap.add_argument("--points", type=int, default=0, help="grid points (default per workload)")
    ap.add_argument("--workload", choices=["sweep", "single", "stream", "doppler"], default="sweep")
    ap.add_argument("--chunk-lines", type=int, default=10_000_000, help="stream workload")
    ap.add_argument("--pbar", type=float, default=1.0,
                    help="single workload: pressure factor on the 1-bar Lorentz widths")
    ap.add_argument("--P", type=int, default=0)
    ap.add_argument("--W", type=int, default=0)
    ap.add_argument("--C", type=int, default=0, help="conditions per warp (mixed)")
    ap.add_argument("--C64", type=int, default=0, help="conditions per warp (FP64)")
    ap.add_argument("--S", type=int, default=0, help="line splits per tile (0 = automatic)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--conds", type=int, default=40, help="subset of the 40 conditions (profiling)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-seconds", type=float, default=100.0,
                    help="--impl reference: seconds of reference CPU work over warm-up + steps")
    ap.add_argument("--no-serve", action="store_true", help="skip the request-server stream")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes, no autotuning")
    ap.add_argument("--no-extra", action="store_true",
                    help="default run: leave out the single-point and Doppler configurations")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--serve-policy", type=int, default=0,
                    help="server chunk order: 0 least remaining work, 1 round robin, 2 earliest deadline")
    ap.add_argument("--serve-lanes", type=int, default=0, help="server streams (0: the server's default)")
    ap.add_argument("--serve-depth", type=int, default=0, help="chunks in flight per stream (0: default)")
    ap.add_argument("--serve-chunk-pairs", type=float, default=0.0,
                    help="target line-evals per served chunk (0: the server's default)")
    ap.add_argument("--serve-alone", type=int, default=40,
                    help="heaviest requests timed alone for the p99 lower bound")
    ap.add_argument("--serve-scale", type=float, default=1.0,
                    help="scale of the served molecules' line counts (1 = 1e6/1e7/1e8)")
    args = ap.parse_args()
    if not args.points:
        args.points = 750_000 if args.workload == "single" else 75_000
    if args.workload == "stream" and args.lines == 10_000_000:
        args.lines = 500_000_000
    if args.warmup < 3 and args.impl == "ours":
        log("[bench] warm-up raised to 3")
        args.warmup = 3

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    dist = None
    if world > 1 and args.impl == "ours":
        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist

    if args.impl == "reference":
        res = run_reference(args, rank, world)
    elif args.workload == "stream":
        res = run_stream(args, rank, world, dist)
    elif args.workload == "doppler":
        res = run_doppler(args, rank, world, dist)
    else:
        res = run_ours(args, rank, world, dist)
        if args.workload == "sweep" and world == 1 and not args.no_extra:
            extra = run_extra_configs(args, rank, world, dist)
            if res is not None:
                res.update(extra)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if res is not None and rank == 0:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
