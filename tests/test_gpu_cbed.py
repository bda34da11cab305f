"""CBED on the device (totem_session_cbed / totem_cbed_run) against the FP64 oracle's restatement of
ToTem's CBED loop (ToTEM_submit_v1.m:1478-1492): one probe position, defocus-spread probes, the
whole diffraction pattern.  Tolerance: relative L2 <= 1e-4, as for every image."""
import numpy as np
import pytest

from oracle import stem_oracle as so
from tests.conftest import rel_l2
from totem_b200 import capi, request

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.mark.parametrize("n,p,sampling,path", [(128, 256, 0.1, capi.PATH_FUSED), (400, 448, 0.05, capi.PATH_FUSED),
                                              (80, 176, 0.2, capi.PATH_PLAIN)])
def test_cbed_vs_oracle(engine_lib, n, p, sampling, path):
    req = request.build_small_stem(n=n, p=p, raster=(1, 1), step=0, slices=5, sampling=sampling,
                                   focal_steps=3, mid_layer=(), cells=4 if n == 400 else None)
    s = capi.Session()
    s.upload(req)
    pat = s.cbed()
    assert s.timing().slice_path == path
    again = s.cbed()
    s.close()
    np.testing.assert_array_equal(pat, again)
    np.testing.assert_array_equal(capi.cbed_run(req), pat)
    assert rel_l2(pat, so.cbed(req)) < TOL


def test_cbed_takes_one_position(engine_lib):
    req = request.build_small_stem(raster=(2, 2))
    with pytest.raises(capi.TotemError) as e:
        capi.cbed_run(req)
    assert e.value.code == capi.ERR_INVALID_ARG
