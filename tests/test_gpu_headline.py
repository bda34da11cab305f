"""Parity at the headline sizes, engine vs the FP64 oracle.

1. SrTiO3 [001] STEM-ADF exactly as the benchmark runs it: 8x8x50 cells, 100 slices, Peng,
   300 kV, 64x64 probes at 8 px on a 1024^2 potential, 512^2 windows, ADF and BF detectors.
   The whole transmission stack (all 100 slices) is compared with the oracle's; a perfect crystal
   repeats its two planes, so the oracle evaluates each distinct slice once and the stack is
   assembled from those.  The detector images of 16 probes (the four raster corners and 12
   seeded positions) are compared with the oracle's slice loop run on the oracle's transmission.
2. One frozen-phonon configuration of the frozen-phonon workload: the same specimen with seeded
   Gaussian displacements (seed 0; every slice differs), 128x128 probes, 1024^2 windows on a
   2048^2 potential.  Three slices of the transmission (first, middle, last) are compared with
   the oracle's; the images of 6 probes (corners and 2 seeded positions) with the oracle's slice
   loop run on the engine's transmission stack.

Reference semantics: cuda_STEM_CPU_Mcore_lobato_peng.m:55-77 (slice loop and detectors),
GetPotential4AllSlice_multicore_lotabo_peng.m:25-100, 187-190 (Peng potential, transmission).
Tolerance: relative L2 <= 1e-4 on each slice of T and on each detector's image over the probes
checked.  With TOTEM_REPORT_DIR set the errors are written there as JSON.
"""
import json
import os

import numpy as np
import pytest

from oracle import stem_oracle as so
from tests import oracle_pool
from tests.conftest import rel_l2
from totem_b200 import capi, request

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _device_to_host(ptr: int, shape, dtype=np.complex64) -> np.ndarray:
    """Copy a device buffer (the engine's transmission stack) into a new host array."""
    from cuda.bindings import runtime as rt
    out = np.empty(shape, dtype=dtype)
    (err,) = rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess, err
    return out


def _probe_sample(req, extra: int, seed: int):
    r, c = req.hight_red, req.width_red
    corners = [0, c - 1, (r - 1) * c, r * c - 1]
    rng = np.random.default_rng(seed)
    rest = rng.choice(np.setdiff1d(np.arange(req.depth), corners), size=extra, replace=False)
    return sorted(set(corners) | set(int(p) for p in rest))


def _report(name, payload):
    print(name, json.dumps(payload))
    out = os.environ.get("TOTEM_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, f"{name}.json"), "w") as f:
            json.dump(payload, f, indent=1)


def _engine_run(req):
    s = capi.Session(device=0)
    s.upload(req)
    s.run()
    res, mid, _ = s.download()
    T = _device_to_host(s.transmission_ptr(), (req.slices, req.p_height, req.p_width))
    s.close()
    return res.reshape(req.aper_num, req.depth), T


def _image_errors(req, res, T_for_oracle, probes):
    ref, _ = so.stem(req, T_for_oracle, items=probes)
    ref = ref.reshape(req.aper_num, req.depth)
    return [rel_l2(res[a, probes], ref[a, probes]) for a in range(req.aper_num)]


def test_stem_adf_headline_vs_oracle(engine_lib):
    req = request.build_srtio3_stem()  # the benchmark's stem-adf request
    assert (req.depth, req.slices, req.height, req.p_height) == (4096, 100, 512, 1024)
    res, T_eng = _engine_run(req)

    groups = oracle_pool.distinct_slices(req)
    V = oracle_pool.potential_slices(req, [g[0] for g in groups])
    T_distinct = so.transmission(req, V)
    T_ref = np.empty((req.slices, req.p_height, req.p_width), dtype=np.complex128)
    for g, t in zip(groups, T_distinct):
        T_ref[g] = t
    t_err = [rel_l2(T_eng[k], T_ref[k]) for k in range(req.slices)]

    probes = _probe_sample(req, 12, seed=2)
    img_err = _image_errors(req, res, T_ref, probes)
    _report("parity_stem_adf_headline", {
        "workload": "SrTiO3 [001] 8x8x50 cells, 100 slices, Peng 300 kV, 64x64 probes, 512^2 window, 1024^2 potential",
        "distinct_slices": len(groups), "transmission_rel_l2_max": max(t_err),
        "transmission_rel_l2_mean": float(np.mean(t_err)), "probes_checked": probes,
        "image_rel_l2": {"ADF 60-200 mrad": img_err[0], "BF 0-10 mrad": img_err[1]}})
    assert max(t_err) < TOL, max(t_err)
    for a, e in enumerate(img_err):
        assert e < TOL, (a, e)


def test_frozen_phonon_1024_window_vs_oracle(engine_lib):
    req = request.build_srtio3_stem(n=1024, raster=(128, 128), phonon_seed=0)
    assert (req.depth, req.slices, req.height, req.p_height) == (16384, 100, 1024, 2048)
    res, T_eng = _engine_run(req)

    checked = [0, req.slices // 2, req.slices - 1]
    V = oracle_pool.potential_slices(req, checked)
    T_ref = so.transmission(req, V)
    t_err = [rel_l2(T_eng[k], T_ref[j]) for j, k in enumerate(checked)]

    probes = _probe_sample(req, 2, seed=3)
    img_err = _image_errors(req, res, T_eng, probes)
    _report("parity_frozen_phonon_1024", {
        "workload": "SrTiO3 [001] 8x8x50 cells, frozen-phonon configuration seed 0, 100 slices, Peng 300 kV, "
                    "128x128 probes, 1024^2 window, 2048^2 potential",
        "transmission_slices_checked": checked, "transmission_rel_l2": t_err, "probes_checked": probes,
        "image_rel_l2": {"ADF 60-200 mrad": img_err[0], "BF 0-10 mrad": img_err[1]},
        "note": "images: the oracle's FP64 slice loop on the engine's transmission stack"})
    assert max(t_err) < TOL, t_err
    for a, e in enumerate(img_err):
        assert e < TOL, (a, e)
