"""Spreading STEM work over ranks (one process per GPU) and collecting the detector images.

The work units of the path are independent: scan positions, defocus-spread probes and
frozen-phonon configurations.  Two ways to use several GPUs:

  * ``stem_sharded``: one request, its scan rows cut into contiguous bands, one band per rank.
    Each rank builds its own transmission from the atom list (no bulk data crosses NVLink) and
    the per-rank images (A x positions doubles) are gathered once at the end.
  * ``configurations_summed``: frozen-phonon configurations dealt round-robin to the ranks,
    summed locally and reduced once (``all_reduce``).

``compute(req) -> (result, mid)`` does one request on the local device; the default is the
engine, through a session on the rank's own GPU (``LOCAL_RANK``).  Collectives go through ``torch.distributed`` (NCCL on GPUs, gloo
on CPU) and are only used for the final gather / reduction.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np


def _dist():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist, dist.get_rank(), dist.get_world_size()
    return None, 0, 1


def row_bands(rows: int, world: int):
    """Contiguous, balanced ranges of scan rows, one per rank (empty ranges when rows < world)."""
    edges = np.linspace(0, rows, world + 1).round().astype(int)
    return [(int(edges[i]), int(edges[i + 1])) for i in range(world)]


def band_request(req, r0: int, r1: int):
    """The sub-request scanning rows r0 .. r1-1 of ``req`` (window placement unchanged)."""
    return replace(req, beginrow=req.beginrow + r0 * req.step, hight_red=r1 - r0)


def local_device() -> int:
    """This rank's GPU: ``LOCAL_RANK`` as set by ``torchrun`` (one process per GPU), or -1 outside
    a launcher (the engine then picks the GPU with the most free memory)."""
    import os
    v = os.environ.get("LOCAL_RANK")
    return int(v) if v not in (None, "") else -1


_SESSIONS = {}


def _default_compute(req):
    """One request on this rank's own GPU through a session kept per device.  A session pinned to
    ``LOCAL_RANK`` keeps ranks off each other's GPUs: the one-shot ``totem_stem_run`` would pick
    the GPU with the most free memory, which several ranks can agree on."""
    from . import capi
    dev = local_device()
    s = _SESSIONS.get(dev)
    if s is None:
        s = _SESSIONS[dev] = capi.Session(device=dev)
    s.upload(req)
    s.run()
    res, mid, _ = s.download()
    return res, mid


def stem_sharded(req, compute=None, group=None):
    """Detector images of ``req`` computed with its scan rows spread over the ranks.

    Returns ``(result, mid)`` in the MEX layouts (``result[a*depth + pos]``,
    ``mid[(l*A + a)*depth + pos]``) on every rank.
    """
    compute = compute or _default_compute
    dist, rank, world = _dist()
    bands = row_bands(req.hight_red, world)
    r0, r1 = bands[rank]
    A, L, W = req.aper_num, len(req.mid_layer), req.width_red
    if r1 > r0:
        res, mid = compute(band_request(req, r0, r1))
        res = np.asarray(res).reshape(A, (r1 - r0) * W)
        mid = np.asarray(mid).reshape(L, A, (r1 - r0) * W)
    else:
        res, mid = np.zeros((A, 0)), np.zeros((L, A, 0))
    if dist is None:
        parts = [(res, mid)]
    else:
        parts = [None] * world
        dist.all_gather_object(parts, (res, mid), group=group)
    full = np.concatenate([p[0] for p in parts], axis=1)
    full_mid = np.concatenate([p[1] for p in parts], axis=2)
    return full.reshape(-1), full_mid.reshape(-1)


def configurations_summed(requests, compute=None, group=None):
    """Sum of the detector images of several requests (frozen-phonon configurations), with the
    requests dealt round-robin to the ranks.  ``requests`` is a sequence (or a callable
    ``i -> request`` together with ``len``-able range) of requests of identical shape."""
    compute = compute or _default_compute
    dist, rank, world = _dist()
    mine = [i for i in range(len(requests)) if i % world == rank]
    acc = None
    for i in mine:
        r = requests[i]
        res, mid = compute(r)
        res, mid = np.asarray(res, dtype=np.float64), np.asarray(mid, dtype=np.float64)
        acc = (res, mid) if acc is None else (acc[0] + res, acc[1] + mid)
    if acc is None:
        r0 = requests[0]
        acc = (np.zeros(r0.aper_num * r0.depth), np.zeros(r0.aper_num * r0.depth * len(r0.mid_layer)))
    if dist is None:
        return acc
    import torch
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.concatenate(acc)).to(dev)
    dist.all_reduce(t, group=group)
    out = t.cpu().numpy()
    n = len(acc[0])
    return out[:n], out[n:]


class PhononConfigurations:
    """Frozen-phonon requests of one structure, configuration ``i`` seeded with ``seed0 + i``.

    Built lazily, so every rank builds only the configurations it runs.
    """

    def __init__(self, builder, count: int, seed0: int = 0):
        self.builder, self.count, self.seed0 = builder, count, seed0

    def __len__(self):
        return self.count

    def __getitem__(self, i):
        return self.builder(phonon_seed=self.seed0 + i)
