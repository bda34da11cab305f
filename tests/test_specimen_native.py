"""Specimen preparation in the library (``totem_slice_rows``, ``totem_fold_debye_waller``,
``totem_frozen_phonon``; host code, no GPU) against the NumPy restatement in
``totem_b200.specimen`` of CalAllEquilent20210223_lobato_peng.m, CommonPart_forsimulation and
randshiftpos.m.

Slicing must match to ~1e-13 (the erf of the C library and of SciPy may differ in the last bit,
and the weights are differences of erf values near one) and the Debye-Waller fold exactly; the
phonon deviates come from a different generator
than NumPy's, so they are checked by their statistics, their slab bound and their seeding.
"""
import numpy as np
import pytest

from totem_b200 import build, capi, specimen


@pytest.fixture(scope="module")
def lib():
    build.build()
    return capi.load()


def _tables(flag, seed=0, ionic=True):
    """SrTiO3 with thermal displacements (atoms off the slice planes) and, optionally, a third of
    the O partly ionised (so both tables are filled)."""
    st = specimen.srtio3_001(4, 4, 5, dw={38: 0.6, 22: 0.45, 8: 0.6})
    x = st.atoms.copy()
    if ionic:
        o = np.flatnonzero(x[:, 0] == 8)[::3]
        x[o, 4] = -2
        x[o, 5] = 0.4
    nuc, ion = specimen.potential_params(x, flag)
    rng = np.random.default_rng(seed)
    nuc = specimen.frozen_phonon(nuc, st.slice_dz, st.slicethick, rng)
    if len(ion):
        ion = specimen.frozen_phonon(ion, st.slice_dz, st.slicethick, rng)
    return st, nuc, ion


@pytest.mark.parametrize("flag,dbmode", [("p", 0), ("l", 0), ("l", 1)])
@pytest.mark.parametrize("multiceng", [0, 1, 2])
def test_slice_rows_match_numpy(lib, flag, dbmode, multiceng):
    st, nuc, ion = _tables(flag)
    assert len(nuc) and len(ion)
    ref = specimen.slice_rows(nuc, ion, st.slice_dz, st.slicethick, multiceng, flag, dbmode)
    got = capi.slice_rows(nuc, ion, st.slice_dz, st.slicethick, multiceng, flag, dbmode)
    for r, g in zip(ref, got):
        assert r.shape == g.shape
        np.testing.assert_allclose(g, r, rtol=1e-12, atol=1e-13)  # erf differences near 1 cancel
    if multiceng:
        # atoms near a boundary are spread over neighbouring slices with weights summing to one
        assert len(got[0]) > len(nuc)


def test_slice_rows_single_kind_and_counting(lib):
    st, nuc, _ = _tables("p", ionic=False)
    ref = specimen.slice_rows(nuc, np.zeros((0, 28)), st.slice_dz, st.slicethick, 1, "p")
    got = capi.slice_rows(nuc, np.zeros((0, 28)), st.slice_dz, st.slicethick, 1, "p")
    assert len(got[1]) == 0 and len(got[3]) == 0 and len(ref[3]) == 0
    np.testing.assert_allclose(got[0], ref[0], rtol=1e-12, atol=1e-13)
    np.testing.assert_array_equal(got[2], ref[2])
    # a buffer smaller than the rows is an error, with the totals reported
    import ctypes as C
    n = np.ascontiguousarray(nuc)
    st_t = np.ascontiguousarray(st.slicethick)
    small = np.zeros((3, 13))
    rn, ri = C.c_longlong(0), C.c_longlong(0)
    rc = lib.totem_slice_rows(capi.PARAM_PENG, n.ctypes.data_as(capi._dp), len(n), None, 0, st.slice_dz,
                              st_t.ctypes.data_as(capi._dp), len(st_t), 1, 0, small.ctypes.data_as(capi._dp), 3,
                              None, 0, None, None, C.byref(rn), C.byref(ri))
    assert rc == capi.ERR_INVALID_ARG and rn.value == len(ref[0])


@pytest.mark.parametrize("flag", ["p", "l"])
def test_fold_debye_waller_matches_numpy(lib, flag):
    _, nuc, ion = _tables(flag)
    ra, rb = specimen.fold_debye_waller(nuc, ion, flag)
    ga, gb = capi.fold_debye_waller(nuc, ion, flag)
    np.testing.assert_array_equal(ga, ra)
    np.testing.assert_array_equal(gb, rb)


def test_frozen_phonon_seeded_statistics(lib):
    st = specimen.srtio3_001(24, 24, 10, dw={38: 0.6, 22: 0.45, 8: 0.6})
    nuc, _ = specimen.potential_params(st.atoms, "p")
    a = capi.frozen_phonon(nuc, st.slice_dz, st.slicethick, seed=7)
    b = capi.frozen_phonon(nuc, st.slice_dz, st.slicethick, seed=7)
    c = capi.frozen_phonon(nuc, st.slice_dz, st.slicethick, seed=8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    np.testing.assert_array_equal(np.delete(a, [1, 2, 3], axis=1), np.delete(nuc, [1, 2, 3], axis=1))
    lo, hi = st.slicethick[0], st.slicethick[-1] + st.slice_dz
    assert np.all((a[:, 3] >= lo) & (a[:, 3] < hi))
    sig = np.sqrt(nuc[:, 4] / 8 / np.pi ** 2)
    d = (a[:, 1:3] - nuc[:, 1:3]) / sig[:, None]   # re-draws depend on z only: x and y stay normal
    assert abs(d.mean()) < 0.02 and abs(d.std() - 1) < 0.02
    # the same statistics as the NumPy restatement (a different stream)
    ref = specimen.frozen_phonon(nuc, st.slice_dz, st.slicethick, np.random.default_rng(7))
    dr = (ref[:, 1:3] - nuc[:, 1:3]) / sig[:, None]
    assert abs(d.std() - dr.std()) < 0.03


def test_frozen_phonon_unplaceable_atom_is_an_error(lib):
    t = np.zeros((1, 16))
    t[0, 3] = 100.0   # far outside the slab, with no displacement to bring it in
    with pytest.raises(capi.TotemError):
        capi.frozen_phonon(t, 2.0, np.array([0.0, 2.0]), seed=1)


def test_request_builder_native_slicing(lib):
    from totem_b200 import request
    a = request.build_srtio3_stem(cells=(4, 4, 3), n=64, raster=(2, 2), p=128, phonon_seed=3)
    b = request.build_srtio3_stem(cells=(4, 4, 3), n=64, raster=(2, 2), p=128, phonon_seed=3, native_slicing=True)
    np.testing.assert_array_equal(a.series_n, b.series_n)
    np.testing.assert_allclose(b.ele_n, a.ele_n, rtol=1e-12, atol=1e-13)
