"""Serving workload and driver: seeded mixed STEM requests through the continuous-batching
scheduler (``totem_server_*``), with per-request latency percentiles and aggregate throughput.

The workload follows the serving configuration of the hot path (windows of several sizes,
probe counts log-uniform, slice counts uniform, Lobato / Peng half and half, SrTiO3 supercells
sized to the potential grid), scaled by the arguments so that a run takes seconds to minutes.
The comparator is the same requests served one at a time through the blocking ``totem_stem_run``
(the reference's calling pattern: one MEX call per request), with the same arrival times.

    python -m totem_b200.serving --requests 64 --sizes 256 512 --max-probes 1024
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import replace

import numpy as np

from . import capi, request, specimen

STEP = 8
SAMPLING = 0.0625  # Angstrom per pixel


def _grid(n: int, rmax: int) -> int:
    need = n + (rmax - 1) * STEP
    return 1 << (need - 1).bit_length()


def _base(n: int, flag: str, rmax: int, smax: int, what: str = "srtio3"):
    """A supercell filling the potential grid of an n^2 window and an rmax^2 scan, ``smax`` slices
    thick: SrTiO3 [001] (2 slices per 3.905 Angstrom cell) or Si [001] (4 per 5.431 Angstrom)."""
    p = _grid(n, rmax)
    if what == "si":
        cells = max(1, int(p * SAMPLING // 5.431))
        st = specimen.si_001(cells, cells, (smax + 3) // 4)
        return request.build_stem_on_structure(st, n=n, sampling=SAMPLING, step=STEP, raster=(rmax, rmax), p=p,
                                               flag=flag, native_slicing=True, engine_optics=True)
    cells = max(1, int(p * SAMPLING // 3.905))
    return request.build_srtio3_stem(cells=(cells, cells, (smax + 1) // 2), n=n, sampling=SAMPLING, step=STEP,
                                     raster=(rmax, rmax), p=p, flag=flag, native_slicing=True, engine_optics=True)


def derive(base, rows: int, cols: int, slices: int, mid_layer=()):
    """A request on ``base``'s specimen and grid with a rows x cols scan centred on the grid and
    the first ``slices`` slices."""
    n = base.height
    p = base.p_height
    br = (p - (n + (rows - 1) * STEP)) // 2
    bc = (p - (n + (cols - 1) * STEP)) // 2
    keep = int(np.sum(base.series_n[:slices]))
    keep_i = int(np.sum(base.series_n_i[:slices])) if len(base.series_n_i) else 0
    return replace(base, hight_red=rows, width_red=cols, beginrow=br, begincol=bc,
                   series_n=base.series_n[:slices].copy(), ele_n=base.ele_n[:keep],
                   series_n_i=base.series_n_i[:slices].copy(), ele_n_i=base.ele_n_i[:keep_i],
                   mid_layer=np.asarray(mid_layer, dtype=np.int32))


def make_workload(count: int = 64, seed: int = 0, sizes=(256, 512), max_probes: int = 1024,
                  slices=(20, 100), specimens=("srtio3",)):
    """``count`` seeded requests: window from ``sizes``, probes log-uniform in [1, max_probes],
    slices uniform in ``slices``, Peng / Lobato half and half, a mid-layer detector on a third,
    the supercell drawn from ``specimens`` ("srtio3", "si") when there is more than one."""
    rng = np.random.default_rng(seed)
    rmax = int(math.ceil(math.sqrt(max_probes)))
    bases = {}
    reqs = []
    for _ in range(count):
        n = int(rng.choice(sizes))
        flag = "p" if rng.random() < 0.5 else "l"
        what = str(rng.choice(specimens)) if len(specimens) > 1 else specimens[0]
        if (n, flag, what) not in bases:
            bases[(n, flag, what)] = _base(n, flag, rmax, slices[1], what)
        probes = int(round(math.exp(rng.uniform(0.0, math.log(max_probes)))))
        rows = min(rmax, int(math.ceil(math.sqrt(probes))))
        cols = min(rmax, max(1, int(math.ceil(probes / rows))))
        s = int(rng.integers(slices[0], slices[1] + 1))
        mid = (s // 2,) if rng.random() < 1 / 3 else ()
        reqs.append(derive(bases[(n, flag, what)], rows, cols, s, mid))
    return reqs


def poisson_arrivals(count: int, rate_hz: float, seed: int = 0) -> np.ndarray:
    if rate_hz <= 0:
        return np.zeros(count)
    rng = np.random.default_rng(seed + 1)
    return np.cumsum(rng.exponential(1.0 / rate_hz, size=count)) - 0.0


def serve(reqs, arrivals, policy: int = capi.SCHED_SHORTEST, **server_kw):
    """Submit each request at its arrival time (seconds from start); wait for all.

    Returns (results, latencies_ms, makespan_s)."""
    with capi.Server(policy=policy, **server_kw) as srv:
        t0 = time.perf_counter()
        tickets = []
        for req, at in zip(reqs, arrivals):
            dt = at - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            tickets.append(srv.submit(req))
        results = [srv.wait(t) for t in tickets]
        makespan = time.perf_counter() - t0
        infos = [srv.info(t) for t in tickets]
        lat = np.array([i.latency_ms for i in infos])
        serve.last_phases = {k: float(np.mean([getattr(i, k) for i in infos]))
                             for k in ("queued_ms", "prepare_ms", "run_ms")}
        serve.last_stats = srv.stats()
    return results, lat, makespan


def serve_one_at_a_time(reqs, arrivals):
    """The blocking comparator: each request through ``totem_stem_run`` after the previous one,
    starting no earlier than its arrival.  Returns (results, latencies_ms, makespan_s)."""
    t0 = time.perf_counter()
    results, lat = [], []
    for req, at in zip(reqs, arrivals):
        dt = at - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        results.append(capi.stem_run(req))
        lat.append((time.perf_counter() - t0 - at) * 1e3)
    return results, np.array(lat), time.perf_counter() - t0


def summary(name, reqs, lat, makespan):
    ps = sum(r.probe_slices for r in reqs)
    return {"mode": name, "requests": len(reqs), "probe_slices": int(ps),
            "probe_slices_per_s": ps / makespan, "makespan_s": makespan,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean())}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--sizes", type=int, nargs="+", default=[256, 512])
    ap.add_argument("--max-probes", type=int, default=1024)
    ap.add_argument("--slices", type=int, nargs=2, default=[20, 100])
    ap.add_argument("--rate", type=float, default=0.0,
                    help="Poisson arrival rate (requests/s); 0 = --load times the server's burst capacity")
    ap.add_argument("--load", type=float, default=0.85, help="offered load as a fraction of burst capacity")
    ap.add_argument("--policy", default="shortest", choices=["fifo", "shortest"])
    ap.add_argument("--wave-mib", type=int, default=0, help="wave memory of the server (0 = its default)")
    ap.add_argument("--chunk-mib", type=int, default=0, help="probes a request may start per tick (0 = default)")
    ap.add_argument("--prep-threads", type=int, default=0, help="server preparation threads (0 = its default)")
    ap.add_argument("--compare", action="store_true", help="also serve one request at a time")
    ap.add_argument("--burst-only", action="store_true", help="skip the Poisson-arrival runs")
    ap.add_argument("--specimens", nargs="+", default=["srtio3"], choices=["srtio3", "si"])
    ap.add_argument("--capacity-sample", type=int, default=0,
                    help="measure the burst capacity on the first K requests only (0 = all of them)")
    ap.add_argument("--check-alone", type=int, default=0,
                    help="compare K seeded requests of the Poisson run with the same request alone")
    ap.add_argument("--mixed-windows", action="store_true", help="one persistent launch for 256^2..1024^2 windows")
    ns = ap.parse_args(argv)
    policy = capi.SCHED_SHORTEST if ns.policy == "shortest" else capi.SCHED_FIFO
    t0 = time.perf_counter()
    reqs = make_workload(ns.requests, ns.seed, tuple(ns.sizes), ns.max_probes, tuple(ns.slices), tuple(ns.specimens))
    print(json.dumps({"workload_built_s": time.perf_counter() - t0, "requests": len(reqs),
                      "probe_slices": int(sum(r.probe_slices for r in reqs))}), flush=True)
    kw = {"wave_bytes": ns.wave_mib << 20} if ns.wave_mib else {}
    if ns.mixed_windows:
        kw["mixed_windows"] = True
    if ns.chunk_mib:
        kw["chunk_bytes"] = ns.chunk_mib << 20
    if ns.prep_threads:
        kw["prep_threads"] = ns.prep_threads
    # warm-up (kernels, pools) on a few requests, then the burst capacity
    serve(reqs[:4], np.zeros(4), policy, **kw)
    cap = reqs[:ns.capacity_sample] if ns.capacity_sample else reqs
    res_b, lat_b, mk_b = serve(cap, np.zeros(len(cap)), policy, **kw)
    out = [dict(summary("burst" if cap is reqs else f"burst (first {len(cap)})", cap, lat_b, mk_b),
                phases_mean=serve.last_phases, server=serve.last_stats)]
    if ns.compare:
        _, lat_sb, mk_sb = serve_one_at_a_time(reqs, np.zeros(len(reqs)))
        out.append(summary("one-at-a-time burst", reqs, lat_sb, mk_sb))
    if ns.burst_only:
        for o in out:
            print(json.dumps(o), flush=True)
        return out
    # offered load: a fraction of the burst capacity in probe*slices/s, in requests of this mix
    capacity = sum(r.probe_slices for r in cap) / mk_b
    rate = ns.rate or ns.load * capacity / np.mean([r.probe_slices for r in reqs])
    arr = poisson_arrivals(len(reqs), rate, ns.seed)
    res_p, lat_p, mk_p = serve(reqs, arr, policy, **kw)
    out.append(dict(summary("poisson", reqs, lat_p, mk_p), rate_hz=rate, phases_mean=serve.last_phases,
                    server=serve.last_stats))
    sizes = sorted({r.height for r in reqs})
    out[-1]["by_window"] = {str(n): {"requests": int(sum(r.height == n for r in reqs)),
                                     "p50_ms": float(np.percentile([l for r, l in zip(reqs, lat_p) if r.height == n], 50)),
                                     "p99_ms": float(np.percentile([l for r, l in zip(reqs, lat_p) if r.height == n], 99))}
                            for n in sizes}
    if ns.check_alone:
        rng = np.random.default_rng(ns.seed + 2)
        idx = sorted(rng.choice(len(reqs), size=min(ns.check_alone, len(reqs)), replace=False).tolist())
        same = [bool(np.array_equal(res_p[i][0], capi.stem_run(reqs[i])[0])) for i in idx]
        out[-1]["alone_vs_mix"] = {"checked": idx, "bit_identical": same}
    if ns.compare:
        res_s, lat_s, mk_s = serve_one_at_a_time(reqs, arr)
        out.append(dict(summary("one-at-a-time", reqs, lat_s, mk_s), rate_hz=rate))
        same = all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) for a, b in zip(res_p, res_s))
        out[-1]["results_identical_to_served"] = bool(same)
    for o in out:
        print(json.dumps(o), flush=True)
    return out


if __name__ == "__main__":
    main()
