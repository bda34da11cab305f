"""The serving scheduler (``totem_server_*``) on the device.

Requests of different window sizes, slice counts, mid layers, defocus series and
parameterisations run together through continuous batching.  Each result must equal the same
request run alone through ``totem_stem_run`` bit for bit (same kernels, same fixed summation
order), and match the FP64 oracle within the parity tolerance.
"""
from dataclasses import replace

import numpy as np
import pytest

from oracle import stem_oracle as so
from tests.conftest import rel_l2
from totem_b200 import capi, request

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _mix():
    return [
        request.build_small_stem(),                                                   # n 64, mid layers
        request.build_small_stem(flag="l", raster=(2, 5), slices=4, mid_layer=()),
        request.build_small_stem(n=128, p=256, raster=(2, 3), step=17, slices=5, sampling=0.1, mid_layer=(2,)),
        request.build_small_stem(focal_steps=3, mid_layer=(5, 2, 5, 99)),              # w_num 3, gfsf weights
        request.build_small_stem(n=256, p=512, raster=(1, 2), step=30, slices=3, sampling=0.1, mid_layer=(1, 3)),
        request.build_small_stem(raster=(1, 1), slices=1, mid_layer=(1,)),           # one probe, one slice
    ]


def _oracle_check(req, res, mid):
    T = so.transmission(req)
    ref_res, ref_mid = so.stem(req, T)
    assert rel_l2(res, ref_res) < TOL
    if len(req.mid_layer) and np.linalg.norm(ref_mid):
        assert rel_l2(mid, ref_mid) < TOL


@pytest.mark.parametrize("policy", [capi.SCHED_FIFO, capi.SCHED_SHORTEST])
def test_mixed_requests_equal_alone(engine_lib, policy):
    reqs = _mix()
    alone = [capi.stem_run(r) for r in reqs]
    with capi.Server(device=0, policy=policy) as srv:
        tickets = [srv.submit(r) for r in reqs]
        got = [srv.wait(t) for t in tickets]
        infos = [srv.info(t) for t in tickets]
    for (r0, m0), (r1, m1) in zip(alone, got):
        assert np.array_equal(r0, r1)
        assert np.array_equal(m0, m1)
    for i in infos:
        assert i.state == capi.REQ_DONE and i.status == capi.OK
        assert i.latency_ms >= i.run_ms >= 0
    _oracle_check(reqs[0], *got[0])
    _oracle_check(reqs[3], *got[3])


def test_small_wave_budget_splits_requests(engine_lib):
    # room for 5 probes of 64^2 (plus partial sums): requests run in many probe groups
    reqs = [request.build_small_stem(raster=(4, 5)), request.build_small_stem(flag="l", raster=(3, 3))]
    alone = [capi.stem_run(r) for r in reqs]
    with capi.Server(device=0, wave_bytes=5 * (64 * 64 * 8 + 4096), chunk_bytes=2 * 64 * 64 * 8) as srv:
        tickets = [srv.submit(r) for r in reqs]
        got = [srv.wait(t) for t in tickets]
    for (r0, m0), (r1, m1) in zip(alone, got):
        assert np.array_equal(r0, r1) and np.array_equal(m0, m1)


def test_submit_rejects_invalid_requests(engine_lib):
    req = request.build_small_stem()
    with capi.Server(device=0) as srv:
        with pytest.raises(capi.TotemError) as e:
            srv.submit(replace(req, begincol=req.p_width - req.width + 1))
        assert e.value.code == capi.ERR_INVALID_ARG
        # a valid request still runs on the same server afterwards
        t = srv.submit(req)
        res, mid = srv.wait(t)
    r0, m0 = capi.stem_run(req)
    assert np.array_equal(res, r0) and np.array_equal(mid, m0)


def test_many_requests_in_flight(engine_lib):
    rng = np.random.default_rng(3)
    reqs = [request.build_small_stem(raster=(int(rng.integers(1, 4)), int(rng.integers(1, 4))),
                                     slices=int(rng.integers(1, 7)), mid_layer=(2,), seed=int(rng.integers(0, 5)))
            for _ in range(24)]
    with capi.Server(device=0) as srv:
        tickets = [srv.submit(r) for r in reqs]
        got = [srv.wait(t) for t in tickets]
    for r, (res, mid) in zip(reqs, got):
        r0, m0 = capi.stem_run(r)
        assert np.array_equal(res, r0) and np.array_equal(mid, m0)


def test_mixed_window_sizes_in_one_launch_equal_alone(engine_lib):
    # 256^2, 512^2 and 1024^2 windows running at the same ticks go through one persistent
    # row-pass and one column-pass launch (mixed_windows); each result must still equal the
    # request alone bit for bit, with mid layers, defocus series and both parameterisations
    reqs = [
        request.build_small_stem(n=256, p=512, raster=(2, 2), step=30, slices=6, sampling=0.1, mid_layer=(2, 5)),
        request.build_small_stem(n=512, p=1024, raster=(1, 3), step=64, slices=5, sampling=0.05, cells=4,
                                 mid_layer=(3,), flag="l"),
        request.build_small_stem(n=1024, p=1024, raster=(1, 1), step=0, slices=4, sampling=0.05, cells=4,
                                 mid_layer=()),
        request.build_small_stem(n=256, p=512, raster=(1, 2), step=40, slices=3, sampling=0.1, focal_steps=3,
                                 mid_layer=(1,)),
        request.build_small_stem(raster=(2, 2), slices=4, mid_layer=(2,)),  # 64^2: its own launches
    ]
    alone = [capi.stem_run(r) for r in reqs]
    with capi.Server(device=0, mixed_windows=True) as srv:
        tickets = [srv.submit(r) for r in reqs]
        got = [srv.wait(t) for t in tickets]
        stats = srv.stats()
    for i, ((r0, m0), (r1, m1)) in enumerate(zip(alone, got)):
        assert np.array_equal(r0, r1), i
        assert np.array_equal(m0, m1), i
    assert stats["requests_done"] == len(reqs)
    _oracle_check(reqs[0], *got[0])
