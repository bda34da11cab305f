"""Autotuner for the fused slice loop: picks the row-pass register cap, the column-pass variant and
the batch size for each window size on the GPU it runs on, by measurement.

    python -m totem_b200.tune [--sizes 256 512 1024 2048] [--out totem_b200/data/tuning.jsonl]

For every window size it builds a SrTiO3 STEM request with that window (20 slices, enough probes
for two of the largest batches), keeps it resident in a session and times the slice loop (CUDA
events around the device work, transmission excluded, best of ``--reps`` runs after a warm-up) for

  * the column-pass variants (TotemRunOptions.col_variant: 1 default, 2 propagator in shared
    memory, 3 lower register cap, 5 8-column tiles, 6 32-column tiles where they exist),
  * the row-pass variants (row_variant: 1 default, 3 / 4 / 5 resident 128-thread CTAs per SM),
  * batches of 1, 2 and 4 GiB of probe waves,

by coordinate descent (column variant, then row variant, then batch, then the column variant
once more).  Each size's choice goes into the table as one JSON line; the engine reads it for runs
that leave those options at 0 (``totem_load_tuning``).  Entries of other GPUs and sizes are kept.

The reference has no counterpart: it sizes its batch from half the free memory
(cuda_source_lobato.cu:1250-1260) and uses fixed cuFFT plans.
"""
from __future__ import annotations

import argparse
import json
import os
import time

from . import capi, request

COL_VARIANTS = (1, 2, 3, 5, 6)
ROW_VARIANTS = (1, 3, 4, 5)
BATCH_MIB = (1024, 2048, 4096)


def col_variants(n: int):
    return [v for v in COL_VARIANTS if not (v == 6 and n > 512) and not (v == 5 and n > 2048)]


def row_variants(n: int):
    out = [1]
    if n >= 1024:
        out.append(3)
    if n >= 512:
        out.append(4)
    if 512 <= n <= 1024:
        out.append(5)
    return out


def workload(n: int, slices: int = 20):
    """SrTiO3 [001] with an n x n window: probes for two batches of the largest size tried."""
    probes = max(64, 2 * (max(BATCH_MIB) << 20) // (n * n * 8))
    r = 1
    while r * r < probes:
        r *= 2
    return request.build_srtio3_stem(cells=(8, 8, (slices + 1) // 2), n=n, raster=(r, r))


class Timer:
    """Slice-loop time per probe*slice (microseconds) of a resident request."""

    def __init__(self, req, device: int = 0, reps: int = 3):
        self.req, self.reps = req, reps
        self.sess = capi.Session(device=device)
        self.sess.upload(req)
        self.sess.run(row_variant=1, col_variant=1, batch=1)  # transmission
        self.cache = {}

    def __call__(self, rv: int, cv: int, batch_mib: int) -> float:
        key = (rv, cv, batch_mib)
        if key not in self.cache:
            n = self.req.height
            batch = max(1, (batch_mib << 20) // (n * n * 8))
            best = float("inf")
            for i in range(self.reps + 1):
                self.sess.run(skip_transmission=True, row_variant=rv, col_variant=cv, batch=batch)
                t = self.sess.timing()
                if i:  # the first run of a shape is the warm-up (and is captured for graph replay next)
                    best = min(best, t.slice_loop_ms)
            self.cache[key] = 1e3 * best / self.req.probe_slices
        return self.cache[key]

    def close(self):
        self.sess.close()


def tune_size(n: int, device: int = 0, reps: int = 3, log=print):
    req = workload(n)
    tm = Timer(req, device, reps)
    try:
        default = tm(1, 1, 4096)
        rv, cv, bm = 1, 1, 4096
        for stage in ("col", "row", "batch", "col"):
            if stage == "col":
                cv = min(col_variants(n), key=lambda v: tm(rv, v, bm))
            elif stage == "row":
                rv = min(row_variants(n), key=lambda v: tm(v, cv, bm))
            else:
                bm = min(BATCH_MIB, key=lambda b: tm(rv, cv, b))
        best = tm(rv, cv, bm)
        log(f"n={n}: row {rv} col {cv} batch {bm} MiB: {best:.4f} us per probe*slice "
            f"(default {default:.4f}; {len(tm.cache)} shapes timed)")
        return {"n": n, "row_variant": rv, "col_variant": cv, "batch_mib": bm, "us_per_probe_slice": best,
                "default_us_per_probe_slice": default,
                "workload": f"SrTiO3 [001], {req.depth} probes x {req.slices} slices, window {n}^2, "
                            f"potential {req.p_height}^2",
                "timed": {f"r{k[0]}c{k[1]}b{k[2]}": v for k, v in sorted(tm.cache.items())}}
    finally:
        tm.close()


def device_name(device: int = 0) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def merge(path: str, device: str, entries):
    """Replace this device's entries of the sizes tuned, keep every other line."""
    sizes = {e["n"] for e in entries}
    keep = []
    if os.path.exists(path):
        for line in open(path):
            if line.strip():
                d = json.loads(line)
                if not (d.get("device") == device and d.get("n") in sizes):
                    keep.append(d)
    when = time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())
    rows = keep + [dict({"device": device}, **e, when=when) for e in entries]
    rows.sort(key=lambda d: (d["device"], d["n"]))
    with open(path, "w") as f:
        for d in rows:
            f.write(json.dumps(d) + "\n")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--sizes", type=int, nargs="+", default=[256, 512, 1024, 2048])
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=capi.TUNING_FILE)
    ns = ap.parse_args(argv)
    capi.load_tuning(None)  # time the shapes themselves, not an older table's
    entries = [tune_size(n, ns.device, ns.reps) for n in ns.sizes]
    merge(ns.out, device_name(ns.device), entries)
    print(f"wrote {ns.out}")
    return entries


if __name__ == "__main__":
    main()
