"""The drop-in boundary, literally: ToTem's own MEX shim (waveCuda.cpp with waveCuda.h, unchanged,
read from the reference tree) compiled against a stand-in mex.h and linked, with no undefined
symbols allowed, to each of this repo's four myProjectfun libraries (``oracle/build_ref.py``).
Without a GPU these tests check the link, the shim's own argument-count errors
(waveCuda.cpp:7-16) and that a full 41-argument call returns cleanly with outputs of the sizes
MATLAB would get (waveCuda.cpp:85-92).  tests/test_gpu_mex.py checks the numbers on a GPU.
"""
import ctypes as C
import os

import numpy as np
import pytest

from tests import mex_driver
from totem_b200 import request

FLAVOURS = [("p", False), ("l", False), ("p", True), ("l", True)]


@pytest.fixture(scope="module")
def mex_built():
    from oracle import build_ref
    from totem_b200 import build
    build.build()
    built = build_ref.build()
    if built is None and not all(os.path.exists(build_ref.mex_path(n)) for n in build_ref.FLAVOURS):
        pytest.skip("the reference's waveCuda.cpp is not present and no MEX builds were made beforehand")
    return True


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.parametrize("param,transmission", FLAVOURS)
def test_mex_build_loads_and_exports_mexfunction(mex_built, param, transmission):
    lib = mex_driver.mex_library(param, transmission)
    assert lib is not None
    assert hasattr(lib, "mexFunction")
    # the shim's myProjectfun reference is bound to this repo's library of the same flavour
    from totem_b200 import capi
    shim = C.CDLL(os.path.join(capi.LIB_DIR, capi.SHIM_LIBS[(param, transmission)]))
    assert hasattr(shim, capi.MYPROJECTFUN_MANGLED)


def test_argument_count_errors_come_from_the_shim(mex_built):
    lib = mex_driver.mex_library("p", False)
    req = request.build_small_stem(raster=(1, 2), slices=2)
    call = mex_driver.MexCall(lib, req)
    n0 = lib.mex_stub_error_count()
    outs = call.call(nlhs=4, nrhs=40)
    assert lib.mex_stub_error_count() == n0 + 1
    assert b"Invalid number of input arguments" in lib.mex_stub_last_error()
    assert all(o is None for o in outs)
    call.call(nlhs=3, nrhs=41)
    assert lib.mex_stub_error_count() == n0 + 2
    assert b"Invalid number of outputs" in lib.mex_stub_last_error()
    call.close()


@pytest.mark.skipif(_has_gpu(), reason="checks the behaviour without a CUDA device")
@pytest.mark.parametrize("param,transmission", FLAVOURS)
def test_full_call_without_a_device_returns_matlab_sized_outputs(mex_built, param, transmission):
    lib = mex_driver.mex_library(param, transmission)
    req = request.build_small_stem(flag=param, raster=(2, 3), slices=3, mid_layer=(1, 3))
    call = mex_driver.MexCall(lib, req, transmission=transmission)
    n0 = lib.mex_stub_error_count()
    res, mid, px, py = call.call()
    call.close()
    assert lib.mex_stub_error_count() == n0  # the argument checks passed
    depth = 0 if transmission else req.depth
    aper = 0 if transmission else req.aper_num
    layers = 0 if transmission else len(req.mid_layer)
    assert res.size == depth * aper and mid.size == depth * aper * layers
    assert px.size == py.size == req.p_height * req.p_width * req.slices
    # no device: the engine reports the failure on stderr and leaves MATLAB's zeroed outputs
    assert not np.any(res) and not np.any(px)
