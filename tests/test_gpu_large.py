"""2048^2 windows: the slice loop's and the HRTEM imaging kernels' largest size (three-stage
transforms), against the FP64 oracle.  The oracle's potential sum at 2048^2 takes minutes, so the
oracle propagates the engine's own transmission (whose builders are checked against the oracle
at smaller sizes and against each other at 1024^2); these tests isolate the 2048 slice loop,
detectors and imaging.  Tolerance: relative L2 <= 1e-4."""
import numpy as np
import pytest

from oracle import stem_oracle as so
from tests.conftest import rel_l2
from totem_b200 import capi, request

pytestmark = pytest.mark.gpu
TOL = 1e-4


def test_stem_2048_window(engine_lib):
    # one scan position, three defocus-spread probes (three items per batch)
    req = request.build_small_stem(n=2048, p=2048, raster=(1, 1), step=0, slices=4, sampling=0.05, cells=6,
                                   mid_layer=(2,), focal_steps=3)
    T = capi.transmission_run(req)
    ref_res, ref_mid = so.stem(req, T)
    res, mid = capi.stem_run(req)
    A, D = req.aper_num, req.depth
    for a in range(A):
        assert rel_l2(res.reshape(A, D)[a], ref_res.reshape(A, D)[a]) < TOL, a
        assert rel_l2(mid.reshape(A, D)[a], ref_mid.reshape(A, D)[a]) < TOL, a


def test_hrtem_2048(engine_lib):
    req, hs = request.build_si_hrtem_001(cells=(4, 4, 1), p=2048, slices=4)
    T = capi.transmission_run(req)
    ex, img = capi.hrtem_run(req, hs)
    rex = so.hrtem_exit_wave(T, hs.prop)
    rimg = so.hrtem_image(rex, np.fft.fftshift(hs.tf, axes=(-2, -1)), np.ones(rex.shape), hs.weights)
    assert rel_l2(ex, rex) < TOL
    assert rel_l2(img, rimg) < TOL
