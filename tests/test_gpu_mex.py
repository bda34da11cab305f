"""ToTem's own MEX shim (waveCuda.cpp, unchanged, built by ``oracle/build_ref.py`` against a
stand-in mex.h and linked to this repo's libraries) called with 41 MATLAB-layout arrays, as
cuda_stem.m:97-106 calls it; its outputs against the FP64 oracle.  Skipped where the MEX builds
were not made (they need the reference's waveCuda.cpp at build time)."""
import numpy as np
import pytest

from oracle import stem_oracle as so
from tests import mex_driver
from tests.conftest import rel_l2
from totem_b200 import request

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _lib(param, transmission):
    lib = mex_driver.mex_library(param, transmission)
    if lib is None:
        pytest.skip("MEX builds of the reference shim not present (oracle/build_ref.py)")
    return lib


@pytest.mark.parametrize("param", ["p", "l"])
def test_mex_stem_vs_oracle(engine_lib, param):
    req = request.build_small_stem(flag=param, raster=(3, 3), slices=5, mid_layer=(4, 2))
    lib = _lib(param, False)
    call = mex_driver.MexCall(lib, req)
    n0 = lib.mex_stub_error_count()
    res, mid, _, _ = call.call()
    call.close()
    assert lib.mex_stub_error_count() == n0
    ref_res, ref_mid = so.stem(req, so.transmission(req))
    A, D, L = req.aper_num, req.depth, len(req.mid_layer)
    for a in range(A):  # plhs[0]: Depth x aper_num, column-major -> [a * Depth + pos]
        assert rel_l2(res[a * D:(a + 1) * D], ref_res[a * D:(a + 1) * D]) < TOL
    m, rm = mid.reshape(L, A, D), ref_mid.reshape(L, A, D)
    for l in range(L):
        for a in range(A):
            assert rel_l2(m[l, a], rm[l, a]) < TOL, (l, a)


@pytest.mark.parametrize("param", ["p", "l"])
def test_mex_transmission_vs_oracle(engine_lib, param):
    req = request.build_small_stem(flag=param, slices=4)
    lib = _lib(param, True)
    call = mex_driver.MexCall(lib, req, transmission=True)
    _, _, px, py = call.call()
    call.close()
    t = (px + 1j * py).reshape(req.slices, req.p_height, req.p_width)
    assert rel_l2(t, so.transmission(req)) < TOL
