"""The request server on the B200: results against the oracle, the same
result alone and in a mix of concurrent requests, admission under a small
memory budget, and request errors."""
from __future__ import annotations

import ctypes
import threading

import numpy as np
import pytest

import oracle
from gpu_cross_b200 import capi, synth
from helpers import FP64_REL, assert_fp64_parity, assert_mixed_parity

pytestmark = pytest.mark.gpu

MASS = 18.02


@pytest.fixture(scope="module")
def molecule():
    # gamma per atm (the server scales it by the request's pressure)
    return synth.random_lines(60000, 800.0, 1400.0, 1500.0, 1e-6, 1e2, seed=4242)


def oracle_for(lines, prof, T, Q, P, f0, df, n, cut):
    g = synth.Grid(f0, f0 + n * df, n)
    # the server's grid is f0 + i*df; build the same values for the oracle
    fr = np.add(f0, np.multiply(np.arange(n, dtype=np.float64), df))
    scaled = synth.LineList(lines.nu, lines.energies, lines.aif, lines.gns, lines.gamma * P, lines.n)
    cond = dict(temperature=T, partition=Q, mean_mass=MASS, pressure=P, ref_temp=296.0)
    return oracle.gpu_convention(prof, fr, np.zeros(n), scaled, cond, df, cut=cut), g


def subset(lines, lo, hi):
    a, b = np.searchsorted(lines.nu, [lo, hi])
    return lines.slice(int(a), int(b))


@pytest.mark.parametrize("prof, prec", [(capi.VOIGT, capi.FP64), (capi.VOIGT, capi.MIXED),
                                        (capi.DOPPLER, capi.FP64)])
def test_server_matches_oracle(cuda, molecule, prof, prec):
    T, Q, P, f0, df, n, cut = 900.0, 1234.5, 2.0, 1000.0, 0.01, 12000, 25.0
    # small chunks: the request runs as many chunks (Doppler work is counted
    # over the few Doppler widths where pairs are not exactly zero)
    srv = capi.Server(0, lanes=2, chunk_pairs=2e6 if prof == capi.VOIGT else 2e3)
    try:
        mid = srv.add_molecule(molecule, MASS)
        rid = srv.submit(mid, prof, prec, T, Q, P, f0, df, n, cut=cut)
        got, info = srv.wait(rid, n)
    finally:
        srv.close()
    assert info["status"] == 0 and info["chunks"] > 3
    want, _ = oracle_for(subset(molecule, f0 - 30, f0 + n * df + 30), prof, T, Q, P, f0, df, n, cut)
    if prec == capi.FP64:
        assert_fp64_parity(got, want, FP64_REL)
        assert info["err_bound"] <= 1e-12
    else:
        assert_mixed_parity(got, want)
        # the request's error statement bounds its true error against FP64
        assert info["err_bound"] == pytest.approx(1024 * 2.0 ** -24)
        peak = np.abs(want).max()
        big = np.abs(want) > 1e-6 * peak
        assert np.max(np.abs(got[big] - want[big]) / np.abs(want[big])) <= info["err_bound"]
        assert abs(got.sum() - want.sum()) / want.sum() <= info["err_bound"]


def random_requests(mid, rng, k):
    reqs = []
    for _ in range(k):
        prof = capi.VOIGT if rng.random() < 0.5 else capi.DOPPLER
        df = float(10 ** rng.uniform(-2, -1))
        f0 = float(rng.uniform(800, 1300))
        n = int(rng.uniform(50, 400) / df)
        reqs.append(dict(molecule=mid, profile=prof, precision=capi.MIXED if rng.random() < 0.5
                         else capi.FP64, temperature=float(rng.uniform(200, 3000)),
                         partition=float(rng.uniform(100, 5000)),
                         pressure=float(10 ** rng.uniform(-3, 1.5)), f0=f0, df=df, npoints=n,
                         cut=25.0))
    return reqs


@pytest.mark.parametrize("policy", [capi.POLICY_LEAST_WORK, capi.POLICY_ROUND_ROBIN, capi.POLICY_DEADLINE])
def test_same_result_alone_and_in_a_mix(cuda, molecule, policy):
    rng = np.random.default_rng(77)
    srv = capi.Server(0, lanes=4, depth=2, chunk_pairs=5e7, policy=policy)
    try:
        mid = srv.add_molecule(molecule, MASS)
        reqs = random_requests(mid, rng, 24)
        alone = []
        for r in reqs:
            rid = srv.submit(**r)
            alone.append(srv.wait(rid, r["npoints"])[0])
        # the same requests at once, from three threads, in another order
        order = rng.permutation(len(reqs))
        ids = {}
        lock = threading.Lock()

        def feed(part):
            for i in part:
                rid = srv.submit(**reqs[i])
                with lock:
                    ids[i] = rid

        threads = [threading.Thread(target=feed, args=(order[j::3],)) for j in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        q, a = srv.pending()
        mixed = {}
        for i in range(len(reqs)):
            mixed[i], info = srv.wait(ids[i], reqs[i]["npoints"])
            assert info["status"] == 0
    finally:
        srv.close()
    for i in range(len(reqs)):
        np.testing.assert_array_equal(alone[i], mixed[i])
    # and two of them against the oracle
    for i in (0, 1):
        r = reqs[i]
        want, _ = oracle_for(subset(molecule, r["f0"] - 30, r["f0"] + r["npoints"] * r["df"] + 30),
                             r["profile"], r["temperature"], r["partition"], r["pressure"], r["f0"],
                             r["df"], r["npoints"], 25.0)
        if r["precision"] == capi.FP64:
            assert_fp64_parity(alone[i], want, FP64_REL)
        else:
            assert_mixed_parity(alone[i], want)


@pytest.mark.parametrize("prof, prec", [(capi.VOIGT, capi.FP64), (capi.VOIGT, capi.MIXED),
                                        (capi.DOPPLER, capi.FP64)])
def test_per_temperature_cache(cuda, molecule, prof, prec):
    """Requests with one (molecule, profile, T, Q) key: the second makes the
    cache and fills it, the third reads it on every chunk, and all three
    results are bit-identical to a server without caches."""
    n = 30000
    base = dict(profile=prof, precision=prec, temperature=1234.0, partition=2345.5, f0=1000.0, df=0.01,
                npoints=n, cut=25.0)
    pressures = (0.3, 1.7, 0.3)

    def run(tcache_bytes):
        srv = capi.Server(0, lanes=2, chunk_pairs=2e7 if prof == capi.VOIGT else 2e4,
                          tcache_bytes=tcache_bytes)
        try:
            mid = srv.add_molecule(molecule, MASS)
            return [srv.wait(srv.submit(molecule=mid, pressure=P, **base), n) for P in pressures]
        finally:
            srv.close()

    cached, plain = run(0), run(-1)
    infos = [info for _, info in cached]
    assert all(info["status"] == 0 for info in infos) and infos[0]["chunks"] > 3
    assert infos[0]["tcache_chunks"] == 0 and infos[1]["tcache_chunks"] == 0
    assert infos[2]["tcache_chunks"] == infos[2]["chunks"]
    assert all(info["tcache_chunks"] == 0 for _, info in plain)
    for (got, _), (want, _) in zip(cached, plain):
        np.testing.assert_array_equal(got, want)
    # a different pressure changes a Voigt result: the cache key does not hold it
    if prof == capi.VOIGT:
        assert not np.array_equal(cached[0][0], cached[1][0])


def server_resident_bytes(lanes, chunk_lines):
    """What xs_server_create reserves: per lane the largest Voigt scratch
    for chunk_lines lines, 64 MiB for line-split parts, plus 4 MiB."""
    need = 0
    for prec in (capi.FP64, capi.MIXED):
        o = capi.make_options(capi.VOIGT, 0.01, MASS, precision=prec)
        need = max(need, capi.lib().xs_scratch_bytes_needed(ctypes.byref(o), 1, chunk_lines))
    need = (need + 255) // 256 * 256 + (64 << 20)
    return lanes * (need + (4 << 20))


def test_admission_under_a_small_budget(cuda, molecule):
    """A budget with room for two requests' grids at a time: six requests
    queue, all complete with the results of an unconstrained server, and a
    request larger than the budget is refused."""
    n, lanes, cl = 40000, 1, 1 << 16
    req_bytes = 2 * ((8 * n + 511) // 512 * 512)
    budget = server_resident_bytes(lanes, cl) + molecule.nu.size * 44 + 2 * req_bytes + 4096
    args = [(1000.0 + 50 * k, 900.0, 1.0, 1000.0 + k, 0.005, n) for k in range(6)]
    srv = capi.Server(0, lanes=lanes, chunk_lines=cl, device_budget=budget, chunk_pairs=1e8)
    try:
        mid = srv.add_molecule(molecule, MASS)
        ids = [srv.submit(mid, capi.VOIGT, capi.MIXED, T, Q, P, f0, df, npts, cut=25.0)
               for (T, Q, P, f0, df, npts) in args]
        outs = [srv.wait(i, n) for i in ids]
        assert all(info["status"] == 0 for _, info in outs)
        with pytest.raises(capi.XsError) as ei:
            srv.submit(mid, capi.VOIGT, capi.MIXED, 1000.0, 900.0, 1.0, 1000.0, 0.001, 4 * n)
        assert ei.value.code == capi.XS_ERR_NOMEM
    finally:
        srv.close()
    free = capi.Server(0, lanes=lanes, chunk_lines=cl, chunk_pairs=1e8)
    try:
        mid = free.add_molecule(molecule, MASS)
        for (T, Q, P, f0, df, npts), (got, _) in zip(args, outs):
            want, _ = free.wait(free.submit(mid, capi.VOIGT, capi.MIXED, T, Q, P, f0, df, npts,
                                            cut=25.0), n)
            np.testing.assert_array_equal(got, want)
    finally:
        free.close()


def test_request_errors(cuda, molecule):
    srv = capi.Server(0, lanes=1)
    try:
        mid = srv.add_molecule(molecule, MASS)
        for bad in (dict(molecule=mid + 1), dict(temperature=-1.0), dict(df=0.0), dict(npoints=0),
                    dict(profile=capi.GAUSSIAN)):
            kw = dict(molecule=mid, profile=capi.VOIGT, precision=capi.FP64, temperature=1000.0,
                      partition=100.0, pressure=1.0, f0=1000.0, df=0.01, npoints=1000)
            kw.update(bad)
            with pytest.raises(capi.XsError):
                srv.submit(**kw)
        with pytest.raises(capi.XsError):
            srv.wait(123456, 10)
        unsorted = synth.LineList(*(np.ascontiguousarray(a[::-1]) for a in
                                    (molecule.nu[:10], molecule.energies[:10], molecule.aif[:10],
                                     molecule.gns[:10], molecule.gamma[:10], molecule.n[:10])))
        with pytest.raises(capi.XsError) as ei:
            srv.add_molecule(unsorted, MASS)
        assert ei.value.code == capi.XS_ERR_UNSORTED
    finally:
        srv.close()
