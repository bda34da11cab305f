"""The engine on the specimen the reference itself saved (``allresul.mat``: ToTem's slicing of a
791-atom SrTiO3 block, 41 slices of 0.823175 Angstrom; fixture from
tests/golden/make_reference_fixtures.py) against the FP64 oracle: STEM with Peng and Lobato
rows, and Peng rows spread over neighbouring slices (multiceng = 1,
CalAllEquilent20210223_lobato_peng.m:23-74)."""
import os

import numpy as np
import pytest

from oracle import stem_oracle as so
from tests.conftest import rel_l2
from totem_b200 import capi, request

pytestmark = pytest.mark.gpu
TOL = 1e-4
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("flag,multiceng", [("p", 0), ("l", 0), ("p", 1)])
def test_reference_specimen_stem_vs_oracle(engine_lib, flag, multiceng):
    d = np.load(os.path.join(GOLDEN, "allresul_srtio3.npz"))
    # 0.15 Angstrom pixels: the 2/3 band limit is 44 mrad at 300 kV, so the annular detector is
    # 20-40 mrad (a 60-200 mrad ADF would see nothing on this grid)
    req = request.build_stem_from_table(d["atoms"], float(d["eachthick"]), d["slicethick"], flag=flag,
                                        multiceng=multiceng, mid_layer=(20, 41),
                                        detectors=((20.0, 40.0), (0.0, 10.0)))
    res, mid = capi.stem_run(req)
    T = so.transmission(req)
    ref_res, ref_mid = so.stem(req, T)
    A, D, L = req.aper_num, req.depth, len(req.mid_layer)
    for a in range(A):
        assert rel_l2(res[a * D:(a + 1) * D], ref_res[a * D:(a + 1) * D]) < TOL, a
    m, rm = mid.reshape(L, A, D), ref_mid.reshape(L, A, D)
    for l in range(L):
        for a in range(A):
            assert rel_l2(m[l, a], rm[l, a]) < TOL, (l, a)
    t = capi.transmission_run(req)
    assert rel_l2(t, T) < TOL
