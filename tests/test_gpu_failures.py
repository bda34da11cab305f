"""Failure handling, with failures injected on the host (``totem_inject_failures``; no GPU fault):

* a device allocation that fails (as if the device were full) makes the call return
  TOTEM_ERR_OOM, and the same session and the one-shot entry point work again afterwards;
* a server whose preparation of some requests fails (a worker failure) fails exactly those
  requests, with their status and message, and serves every other request, bit-identical to the
  request alone; the server keeps serving afterwards.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from totem_b200 import capi, request

pytestmark = pytest.mark.gpu


def test_allocation_failure_then_recovery(engine_lib):
    req = request.build_small_stem(raster=(2, 3))
    ref = capi.stem_run(req)
    try:
        capi.inject_failures(alloc_after=0)
        s = capi.Session(device=0)
        with pytest.raises(capi.TotemError) as e:
            s.upload(req)
        assert e.value.code == capi.ERR_OOM and "injected" in str(e.value)
        s.upload(req)  # the failure fired once: the same session uploads now
        s.run()
        res, mid, _ = s.download()
        s.close()
        assert np.array_equal(res, ref[0]) and np.array_equal(mid, ref[1])
    finally:
        capi.inject_failures()
    # The one-shot entry point keeps a process-wide default session whose buffers only grow, so
    # whether a request allocates depends on what ran before it in the process: it is checked in
    # a fresh process, where its third device allocation fails.
    out = subprocess.run([sys.executable, "-c", _ONE_SHOT], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", "")))
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().splitlines()[-1] == "ok", out.stdout


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# fails cleanly with TOTEM_ERR_OOM, then serves the same request twice with equal results
_ONE_SHOT = """
import numpy as np
from totem_b200 import capi, request
big = request.build_small_stem(n=128, p=256, raster=(2, 2), step=17, sampling=0.1)
capi.inject_failures(alloc_after=2)
try:
    capi.stem_run(big)
    raise SystemExit("no failure")
except capi.TotemError as e:
    assert e.code == capi.ERR_OOM, e
capi.inject_failures()
r2 = capi.stem_run(big)
r3 = capi.stem_run(big)
assert np.array_equal(r2[0], r3[0])
print("ok")
"""


def test_server_fails_only_the_requests_whose_preparation_failed(engine_lib):
    reqs = [request.build_small_stem(raster=(2, 2), seed=i, mid_layer=(2,)) for i in range(6)]
    alone = [capi.stem_run(r) for r in reqs]
    try:
        capi.inject_failures(prepare_every=3)  # the 3rd and 6th preparations fail
        with capi.Server(device=0, policy=capi.SCHED_FIFO) as srv:
            tickets = [srv.submit(r) for r in reqs]
            outcomes = []
            for t in tickets:
                try:
                    outcomes.append(srv.wait(t))
                except capi.TotemError as e:
                    outcomes.append(e)
            infos = [srv.info(t) for t in tickets]
            capi.inject_failures()
            again = srv.wait(srv.submit(reqs[0]))  # the server keeps serving
    finally:
        capi.inject_failures()
    failed = [i for i, o in enumerate(outcomes) if isinstance(o, capi.TotemError)]
    assert len(failed) == 2
    for i in failed:
        assert outcomes[i].code == capi.ERR_STATE and "injected" in str(outcomes[i])
        assert infos[i].state == capi.REQ_FAILED and infos[i].status == capi.ERR_STATE
    for i, o in enumerate(outcomes):
        if i not in failed:
            assert infos[i].state == capi.REQ_DONE
            assert np.array_equal(o[0], alone[i][0]) and np.array_equal(o[1], alone[i][1])
    assert np.array_equal(again[0], alone[0][0])
