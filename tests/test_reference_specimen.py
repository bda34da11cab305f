"""Inputs the reference itself produced, fed through this repo's specimen preparation.

``tests/golden/allresul_srtio3.npz`` is ToTem's saved slicing of a 791-atom SrTiO3 block
(``allresul.mat``, written by slicingdisplay.m:250-254 and loaded by the STEM simulation at
ToTEM_submit_v1.m:764-766); ``pydata_grid.npz`` holds the reciprocal axes of ToTem's
``pydata.mat``.  Generated by ``tests/golden/make_reference_fixtures.py``.
"""
import os

import numpy as np
import pytest

from totem_b200 import capi, optics, request, specimen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _allresul():
    d = np.load(os.path.join(GOLDEN, "allresul_srtio3.npz"))
    return d["atoms"], float(d["eachthick"]), d["slicethick"]


def test_reference_specimen_fixture():
    atoms, eachthick, slicethick = _allresul()
    assert atoms.shape == (791, 8)
    z, counts = np.unique(atoms[:, 0], return_counts=True)
    assert list(z) == [8, 22, 38] and list(counts) == [450, 125, 216]
    assert abs(eachthick - 0.823175) < 1e-12 and len(slicethick) == 41
    # the slice tops are (0:40) * eachthick, which is what Structure.slicethick produces
    st = specimen.Structure(atoms, (0, 0, 0), eachthick, len(slicethick))
    assert np.array_equal(st.slicethick, slicethick)


@pytest.mark.parametrize("flag,multiceng", [("p", 0), ("p", 1), ("p", 2), ("l", 0)])
def test_reference_specimen_slicing_numpy_equals_library(flag, multiceng):
    atoms, eachthick, slicethick = _allresul()
    nuc, ion = specimen.potential_params(atoms, flag)
    a = specimen.slice_rows(nuc, ion, eachthick, slicethick, multiceng, flag)
    b = capi.slice_rows(nuc, ion, eachthick, slicethick, multiceng, flag)
    np.testing.assert_array_equal(a[2], b[2])  # per-slice counts
    np.testing.assert_array_equal(a[3], b[3])
    for x, y in zip(a[:2], b[:2]):
        # multi-slice weights are differences of erf values near one: SciPy's and the C library's
        # erf may differ in the last bit
        np.testing.assert_allclose(np.asarray(x), np.asarray(y), rtol=1e-12, atol=1e-13)
    ele_n, _, series_n, _ = a
    assert len(series_n) == 41 and int(series_n.sum()) == len(ele_n)
    if multiceng == 0:
        # every atom in exactly one slice, with its full projected potential (weight 1)
        assert len(ele_n) == 791
        occ = ele_n[:, 2]
        np.testing.assert_allclose(occ, 1.0, rtol=0, atol=1e-12)
    else:
        # spread over neighbouring slices: per atom the erf weights add up to its occupancy
        assert len(ele_n) > 791


def test_reference_specimen_request_builds():
    atoms, eachthick, slicethick = _allresul()
    req = request.build_stem_from_table(atoms, eachthick, slicethick)
    assert req.slices == 41 and req.p_height == 256 and req.depth == 9
    request.validate(req)


def test_reciprocal_axes_match_the_reference_meshgrid():
    d = np.load(os.path.join(GOLDEN, "pydata_grid.npz"))
    u, v, dx_nm = d["u_axis"], d["v_axis"], float(d["sampling_nm"])
    n = len(u)
    kx, ky, _ = optics.reciprocal_grids(n, n, dx_nm * 10.0)  # Angstrom and 1/Angstrom here
    np.testing.assert_allclose(kx[0] * 10.0, u, rtol=0, atol=1e-12)
    np.testing.assert_allclose(ky[:, 0] * 10.0, v, rtol=0, atol=1e-12)
