"""Transmission build time of the two builders for separable grids: the direct per-species sums
(O(atoms x pixels)) and Gaussian gridding + FFT (O(atoms + pixels log pixels)), on SrTiO3 [001]
supercells that fill the potential grid (the serving workload's specimens), through a resident
session.  Prints one JSON line per grid with both times, the speed-up and the relative L2
difference of the two transmission stacks (on the first ``--check-slices`` slices).

    python -m totem_b200.txbuild --grids 1024 2048 4096 --slices 20

``--correction`` adds Peng-extended correction rows (a neutral row for every atom, an ionic row for
every second, two correction planes, values per element as in ToTem) and ``--per-atom`` also times the per-atom kernel, which every
kind of row takes when the reciprocal grid is not the separable meshgrid (forced here by a relative
change of 1e-12 in every other row of kx).
"""
from __future__ import annotations

import argparse
import json
from dataclasses import replace

import numpy as np

from . import capi, request

SAMPLING = 0.0625  # Angstrom per pixel


def grid_filling_request(p: int, slices: int, flag: str = request.PENG):
    cells = max(1, int(p * SAMPLING // 3.905))
    return request.build_srtio3_stem(cells=(cells, cells, (slices + 1) // 2), n=64, raster=(1, 1), p=p,
                                     sampling=SAMPLING, flag=flag, native_slicing=True)


def build_ms(req, mode: int, reps: int) -> tuple[float, int]:
    """Median device time of ``reps`` transmission builds (after one warm-up) and launches."""
    with capi.tx_builder(mode):
        s = capi.Session()
        try:
            s.upload(req, stem=False)
            s.run(what=1)
            times = []
            for _ in range(reps):
                s.run(what=1)
                times.append(s.timing().transmission_ms)
            return float(np.median(times)), s.timing().kernel_launches
        finally:
            s.close()


def off_meshgrid(req):
    """The request with kx changed by a relative 1e-12 in every other row: no longer separable."""
    kx = req.kx.copy()
    kx[1::2] *= 1.0 + 1e-12
    return replace(req, kx=kx)


def stacks(req, mode: int):
    with capi.tx_builder(mode):
        return capi.transmission_run(req)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--grids", type=int, nargs="+", default=[1024, 2048, 4096])
    ap.add_argument("--slices", type=int, default=20)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--check-slices", type=int, default=2)
    ap.add_argument("--flag", default=request.PENG)
    ap.add_argument("--correction", action="store_true", help="add Peng-extended correction rows")
    ap.add_argument("--per-atom", action="store_true", help="also time the per-atom kernel (off the meshgrid)")
    ns = ap.parse_args(argv)
    out = []
    for p in ns.grids:
        req = grid_filling_request(p, ns.slices, ns.flag)
        if ns.correction:
            req = request.with_correction(req, every=1, per_element=True)
        atoms = int(np.sum(req.series_n) + np.sum(req.series_n_i))
        corr_rows = 0 if req.series_n_corr is None else int(np.sum(req.series_n_corr) + np.sum(req.series_n_i_corr))
        d_ms, d_l = build_ms(req, capi.TX_DIRECT, ns.reps)
        g_ms, g_l = build_ms(req, capi.TX_GRIDDING, ns.reps)
        a_ms, _ = build_ms(req, capi.TX_AUTO, 1)
        r_ms = build_ms(off_meshgrid(req), capi.TX_AUTO, 1)[0] if ns.per_atom else None
        small = replace(req, series_n=req.series_n[:ns.check_slices],
                        ele_n=req.ele_n[:int(np.sum(req.series_n[:ns.check_slices]))])
        diff = None
        if ns.check_slices > 0 and not ns.correction:
            td, tg = stacks(small, capi.TX_DIRECT), stacks(small, capi.TX_GRIDDING)
            diff = float(np.linalg.norm(tg - td) / np.linalg.norm(td))
        line = {"grid": p, "slices": req.slices, "atoms": atoms, "atoms_per_slice": atoms / req.slices,
                "correction_rows": corr_rows, "per_atom_ms": r_ms,
                "direct_ms": d_ms, "gridding_ms": g_ms, "auto_ms": a_ms, "speedup": d_ms / g_ms,
                "direct_launches": d_l, "gridding_launches": g_l,
                "rel_l2_gridding_vs_direct": diff, "check_slices": ns.check_slices}
        print(json.dumps(line), flush=True)
        out.append(line)
    return out


if __name__ == "__main__":
    main()
