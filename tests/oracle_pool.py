"""Test helper: the oracle's potential for chosen slices, computed in parallel over atoms.

``stem_oracle.potential_fourier`` sums one atom row at a time over the whole potential grid, which
takes ~15 s per SrTiO3 slice at 1024^2 and ~1 min at 2048^2 on one core.  The parity tests at the
headline sizes need a few such slices, so the atoms of each slice are split into chunks, every
chunk is summed by ``potential_fourier`` in a spawned worker, and the chunks of a slice are added
(the oracle's own sum, in another association order: FP64 rounding only).  The reciprocal grids
are handed to each worker once, at start-up.
"""
from __future__ import annotations

import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor
from dataclasses import replace

import numpy as np

_GRIDS = {}


def _init(kx, ky, s2):
    _GRIDS["kx"], _GRIDS["ky"], _GRIDS["s2"] = kx, ky, s2


def _chunk(sub):
    from oracle import stem_oracle as so
    sub = replace(sub, kx=_GRIDS["kx"], ky=_GRIDS["ky"], s2=_GRIDS["s2"])
    return so.potential_fourier(sub, chunk=2)[0]


def slice_rows(req, k):
    """(neutral rows, ionic rows, neutral absorptive rows, ionic absorptive rows) of slice ``k``."""
    sn, si = req.padded_series()
    bn = np.concatenate([[0], np.cumsum(sn)]).astype(int)
    bi = np.concatenate([[0], np.cumsum(si)]).astype(int)
    n = slice(bn[k], bn[k + 1])
    i = slice(bi[k], bi[k + 1])
    return (req.ele_n[n], req.ele_n_i[i] if len(req.ele_n_i) else req.ele_n_i,
            None if req.absorp_n is None else req.absorp_n[n],
            None if req.absorp_n_i is None else req.absorp_n_i[i])


def distinct_slices(req):
    """Groups of slices whose coefficient rows are identical (a perfect crystal repeats its
    planes), as lists of slice indices in order of first appearance."""
    groups = {}
    for k in range(req.slices):
        key = b"".join(np.ascontiguousarray(a).tobytes() if a is not None else b"-" for a in slice_rows(req, k))
        groups.setdefault(key, []).append(k)
    return list(groups.values())


def potential_slices(req, slices, workers: int | None = None, atoms_per_task: int = 8) -> np.ndarray:
    """V_k(g) (FP64, before aperture / ifftshift / IFFT) for every k in ``slices``."""
    if req.corr_info_matrix is not None and len(req.corr_info_matrix):
        raise NotImplementedError("correction rows are not split by this helper")
    workers = workers or min(16, len(os.sched_getaffinity(0)))
    slim = replace(req, probe=np.zeros((1, 2, 2), complex), aper=np.zeros((0, 2, 2)), aper2=np.zeros((0, 2, 2)),
                   prop=np.zeros((2, 2), complex), kx=None, ky=None, s2=None)
    tasks, owner = [], []
    for j, k in enumerate(slices):
        rn, ri, an, ai = slice_rows(req, k)
        for lo in range(0, max(len(rn), 1), atoms_per_task):
            hi = min(lo + atoms_per_task, len(rn))
            if hi <= lo:
                break
            tasks.append(replace(slim, ele_n=rn[lo:hi], series_n=np.array([hi - lo], float),
                                 ele_n_i=ri[:0], series_n_i=np.array([0.0]),
                                 absorp_n=None if an is None else an[lo:hi], absorp_n_i=None))
            owner.append(j)
        for lo in range(0, len(ri), atoms_per_task):
            hi = min(lo + atoms_per_task, len(ri))
            tasks.append(replace(slim, ele_n=rn[:0], series_n=np.array([0.0]), ele_n_i=ri[lo:hi],
                                 series_n_i=np.array([hi - lo], float), absorp_n=None,
                                 absorp_n_i=None if ai is None else ai[lo:hi]))
            owner.append(j)
    out = np.zeros((len(slices), req.p_height, req.p_width), dtype=np.complex128)
    ctx = mp.get_context("spawn")
    with ProcessPoolExecutor(workers, mp_context=ctx, initializer=_init, initargs=(req.kx, req.ky, req.s2)) as ex:
        for j, v in zip(owner, ex.map(_chunk, tasks, chunksize=1)):
            out[j] += v
    return out
