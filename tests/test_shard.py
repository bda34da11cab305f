"""Multi-rank host logic on CPU: world size 2 over gloo, the FP64 oracle as each rank's compute.

The sharded images must equal the single-process images exactly (each position is computed by
exactly one rank with the same arithmetic), and phonon configurations summed over ranks must equal
the serial sum.
"""
import os
import socket
from functools import partial

import numpy as np
import pytest
import torch.multiprocessing as mp

from totem_b200 import request, shard


def _oracle_compute(req):
    from oracle import stem_oracle as so
    return so.stem(req)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, what, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        if what == "bands":
            req = request.build_small_stem(raster=(5, 3), slices=3, mid_layer=(2,))
            res, mid = shard.stem_sharded(req, compute=_oracle_compute)
        elif what == "pinning":
            # the default compute: a session on this rank's GPU (LOCAL_RANK), with the engine's
            # session replaced by a recorder so that no device is needed
            os.environ["LOCAL_RANK"] = str(rank)
            from totem_b200 import capi
            capi.Session = _RecordingSession
            req = request.build_small_stem(raster=(4, 3), slices=2, mid_layer=())
            res, mid = shard.stem_sharded(req)
            res = np.asarray(_RecordingSession.devices, dtype=float)
        else:
            confs = shard.PhononConfigurations(partial(_small_phonon), 3)
            res, mid = shard.configurations_summed(confs, compute=_oracle_compute)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), res=res, mid=mid)
    finally:
        dist.destroy_process_group()


class _RecordingSession:
    """Stands in for ``capi.Session``: records the device each session was opened on and returns
    zero images of the right size."""
    devices = []

    def __init__(self, device=-1, stream=None):
        _RecordingSession.devices.append(device)

    def upload(self, req, stem=True):
        self.req = req

    def run(self, **kw):
        pass

    def download(self, want_transmission=False):
        r = self.req
        return np.zeros(r.aper_num * r.depth), np.zeros(r.aper_num * r.depth * len(r.mid_layer)), None


def _small_phonon(phonon_seed):
    return request.build_srtio3_stem(cells=(2, 2, 2), n=64, p=128, sampling=0.25, step=6, raster=(2, 2),
                                     phonon_seed=phonon_seed, detectors=((30.0, 120.0), (0.0, 15.0)), mid_layer=(1,))


def _run(what, tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, what, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    return [np.load(tmp_path / f"r{r}.npz") for r in range(2)]


def test_row_bands_cover_all_rows():
    for rows in (1, 2, 7, 64):
        for world in (1, 2, 3, 8):
            b = shard.row_bands(rows, world)
            assert b[0][0] == 0 and b[-1][1] == rows
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))


def test_band_request_places_windows_like_the_full_request():
    req = request.build_small_stem(raster=(5, 3))
    sub = shard.band_request(req, 2, 4)
    r, c = request.window_origins(req)
    rs, cs = request.window_origins(sub)
    assert np.array_equal(rs, r[2 * 3:4 * 3]) and np.array_equal(cs, c[2 * 3:4 * 3])


@pytest.mark.timeout(600)
def test_sharded_scan_equals_single_process(tmp_path):
    outs = _run("bands", tmp_path)
    req = request.build_small_stem(raster=(5, 3), slices=3, mid_layer=(2,))
    ref_res, ref_mid = _oracle_compute(req)
    for o in outs:
        assert np.array_equal(o["res"], ref_res) and np.array_equal(o["mid"], ref_mid)


@pytest.mark.timeout(600)
def test_phonon_configurations_summed_over_ranks(tmp_path):
    outs = _run("phonon", tmp_path)
    ref = [_oracle_compute(_small_phonon(i)) for i in range(3)]
    ref_res = sum(r[0] for r in ref)
    ref_mid = sum(r[1] for r in ref)
    for o in outs:
        assert np.allclose(o["res"], ref_res, rtol=1e-13) and np.allclose(o["mid"], ref_mid, rtol=1e-13)


@pytest.mark.timeout(600)
def test_sharded_default_compute_pins_the_rank_gpu(tmp_path):
    outs = _run("pinning", tmp_path)
    # each rank opened exactly one session, on the GPU of its LOCAL_RANK
    assert [list(o["res"]) for o in outs] == [[0.0], [1.0]]


def test_local_device_reads_local_rank(monkeypatch):
    monkeypatch.setenv("LOCAL_RANK", "3")
    assert shard.local_device() == 3
    monkeypatch.delenv("LOCAL_RANK")
    assert shard.local_device() == -1
