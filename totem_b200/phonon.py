"""Frozen-phonon STEM: detector images summed over thermally displaced configurations.

The reference loops over configurations in MATLAB, one blocking STEM call each, and accumulates
``myresul = myresul + myresultemp`` (ToTEM_submit_v1.m:847-929, displacements from
randshiftpos.m); the images are divided by the configuration count only when displayed or
written (:954, :999).  Here every configuration is a request of the serving scheduler, so the
configurations run batched: their probe groups share the slice-loop launches, and the
transmission of one configuration is built while others propagate.  The sum is formed on the
host in configuration order, so it is the same whichever configuration finishes first.

    python -m totem_b200.phonon --configs 4 --raster 32 --window 1024
"""
from __future__ import annotations

import argparse
import json
import time
from dataclasses import replace

import numpy as np

from . import capi


def frozen_phonon(configs, server: "capi.Server | None" = None, wave_bytes: int = 4 << 30):
    """Sum of the detector images (result, mid-layer) over ``configs`` (a sequence of requests of
    identical geometry, e.g. ``shard.PhononConfigurations``).  Configurations are submitted as
    they are built, so host-side specimen building overlaps the device work.  Without a
    ``server`` one is made with ``wave_bytes`` of probe waves in flight (large: configurations
    are throughput work, not latency-bound requests)."""
    own = server is None
    srv = server or capi.Server(wave_bytes=wave_bytes, chunk_bytes=wave_bytes)
    try:
        tickets = [srv.submit(configs[i]) for i in range(len(configs))]
        res = mid = None
        for t in tickets:
            r, m = srv.wait(t)
            res = r.copy() if res is None else res + r
            mid = m.copy() if mid is None else mid + m
        return res, mid
    finally:
        if own:
            srv.close()


def frozen_phonon_sequential(configs):
    """The comparator: one blocking ``totem_stem_run`` per configuration, summed in order."""
    res = mid = None
    for i in range(len(configs)):
        r, m = capi.stem_run(configs[i])
        res = r if res is None else res + r
        mid = m if mid is None else mid + m
    return res, mid


def main(argv=None):
    from . import request
    from .shard import PhononConfigurations
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--configs", type=int, default=4)
    ap.add_argument("--raster", type=int, default=32)
    ap.add_argument("--window", type=int, default=1024)
    ap.add_argument("--cells", type=int, nargs=3, default=[8, 8, 50])
    ap.add_argument("--wave-gib", type=int, default=4)
    ap.add_argument("--plain-sample", type=int, default=8,
                    help="probes of one configuration timed through the per-probe cuFFT path (0 = skip)")
    ap.add_argument("--no-sequential", action="store_true",
                    help="skip the one-call-per-configuration comparator")
    ns = ap.parse_args(argv)

    def builder(phonon_seed, first=None):
        return request.build_srtio3_stem(cells=tuple(ns.cells), n=ns.window, raster=(ns.raster, ns.raster),
                                         phonon_seed=phonon_seed, engine_optics=True, optics_from=first)
    t0 = time.perf_counter()
    configs = [builder(0)]
    configs += [builder(s, configs[0]) for s in range(1, ns.configs)]
    t_build = time.perf_counter() - t0
    ps = sum(c.probe_slices for c in configs)
    frozen_phonon(configs[:1])  # warm-up
    with capi.Server(wave_bytes=ns.wave_gib << 30, chunk_bytes=ns.wave_gib << 30) as srv:
        t0 = time.perf_counter()
        res_b, mid_b = frozen_phonon(configs, srv)
        t_b = time.perf_counter() - t0
        stats = srv.stats()
    res_s = mid_s = None
    t_s = float("nan")
    if not ns.no_sequential:
        t0 = time.perf_counter()
        res_s, mid_s = frozen_phonon_sequential(configs)
        t_s = time.perf_counter() - t0
    plain = None
    if ns.plain_sample:
        # the reference's structure: one probe at a time through cuFFT (batch = 1), on a sample
        sub = replace(configs[0], hight_red=1, width_red=ns.plain_sample)
        sess = capi.Session()
        sess.upload(sub)
        sess.run(path=capi.PATH_PLAIN, batch=1)
        t0 = time.perf_counter()
        sess.run(path=capi.PATH_PLAIN, batch=1, skip_transmission=True)
        sess.download()
        plain = sub.probe_slices / (time.perf_counter() - t0)
        sess.close()
    out = {"workload": f"SrTiO3 {ns.cells} frozen phonon, {ns.configs} configurations, "
                       f"{ns.raster}x{ns.raster} probes, window {ns.window}^2",
           "probe_slices": int(ps), "host_build_s": t_build,
           "batched_probe_slices_per_s": ps / t_b, "sequential_probe_slices_per_s": ps / t_s,
           "identical": (None if res_s is None else
                         bool(np.array_equal(res_b, res_s) and np.array_equal(mid_b, mid_s))),
           "wave_gib": ns.wave_gib, "server": stats,
           "plain_per_probe_probe_slices_per_s": plain,
           "plain_sample": f"{ns.plain_sample} probes of configuration 0, batch 1, transmission built beforehand"}
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
