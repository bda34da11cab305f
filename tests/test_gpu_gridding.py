"""The gridding transmission builder (Gaussian gridding + FFT, ``TOTEM_TX_GRIDDING``) against the
FP64 oracle and against the direct per-species sums, through the C ABI.

Tolerances: relative L2 <= 1e-4 against the oracle (the engine's accuracy target); against the
direct FP32 builder <= 5e-6 on the transmission stack (both are FP32; the gridding error itself
is ~1e-7 of the structure factor).
"""
from dataclasses import replace

import numpy as np
import pytest

from oracle import stem_oracle as so
from tests.conftest import rel_l2
from totem_b200 import capi, request

pytestmark = pytest.mark.gpu
TOL = 1e-4
TOL_DIRECT = 5e-6


def _both(req, scratch_bytes=0):
    with capi.tx_builder(capi.TX_DIRECT):
        direct = capi.transmission_run(req)
    with capi.tx_builder(capi.TX_GRIDDING, scratch_bytes):
        grid = capi.transmission_run(req)
    return direct, grid


@pytest.mark.parametrize("flag,p", [("p", 128), ("l", 128), ("p", 256)])
def test_gridding_vs_oracle(engine_lib, flag, p):
    # from 256 on, the row pass skips fine rows no atom touched
    req = request.build_small_stem(flag=flag, p=p)
    direct, grid = _both(req)
    ref = so.transmission(req)
    assert rel_l2(grid, ref) < TOL, rel_l2(grid, ref)
    assert rel_l2(grid, direct) < TOL_DIRECT, rel_l2(grid, direct)
    assert not np.array_equal(grid, direct)  # the gridding path ran


def test_gridding_rectangular_grid(engine_lib):
    # 128 rows x 256 columns: separate axis tables and transform lengths per direction
    from totem_b200 import optics, specimen
    st = specimen.center_in_field(specimen.srtio3_001(6, 3, 2), 256 * 0.2, 128 * 0.2)
    req = request.specimen_request(st, "p", 200.0, 0.2, 128)
    kx, ky, s2 = optics.reciprocal_grids(128, 256, 0.2)
    req = replace(req, kx=kx, ky=ky, s2=s2, p_height=128, p_width=256, aper_true=np.ones((128, 256)),
                  parameter=optics.potential_parameter(128, 256, 0.2))
    direct, grid = _both(req)
    ref = so.transmission(req)
    assert grid.shape == (req.slices, 128, 256)
    assert rel_l2(grid, ref) < TOL, rel_l2(grid, ref)
    assert rel_l2(grid, direct) < TOL_DIRECT


def test_gridding_ionic_absorptive_and_vacuum_slices(engine_lib):
    req = request.with_absorption(request.with_ionic_oxygen(request.build_small_stem(flag="p")))
    req = request.without_slice_atoms(req, [0, 3])
    direct, grid = _both(req)
    ref = so.transmission(req)
    assert rel_l2(grid, ref) < TOL, rel_l2(grid, ref)
    assert rel_l2(grid, direct) < TOL_DIRECT
    assert np.all(grid[0] == 1.0) and np.all(grid[3] == 1.0)  # V = 0 exactly in vacuum slices


@pytest.mark.parametrize("per_element", [False, True])
def test_correction_rows_both_builders(engine_lib, per_element):
    # Peng-extended correction rows (per-pixel planes) summed by species in either builder: the
    # structure factor of each group of identical correction rows times its amplitude, Debye-Waller
    # envelope and plane(s); and on a non-separable grid by the per-atom kernel
    # per_element: few distinct rows per slice, summed by species; otherwise nearly every row is
    # distinct and the rows are added by the per-atom kernel
    req = request.with_correction(request.build_small_stem(flag="p"), every=1 if per_element else 4,
                                  per_element=per_element)
    ref = so.transmission(req)
    assert rel_l2(ref, so.transmission(replace(req, corr_info_matrix=None))) > 10 * TOL  # rows matter
    direct, grid = _both(req)
    assert rel_l2(direct, ref) < TOL, rel_l2(direct, ref)
    assert rel_l2(grid, ref) < TOL, rel_l2(grid, ref)
    res, mid = capi.stem_run(req)
    ref_res, _ = so.stem(req, ref)
    assert rel_l2(res, ref_res) < TOL


def test_gridding_batches_split_slices(engine_lib):
    # scratch for one job: every slice's species run in separate batches, later ones adding to
    # what the earlier ones wrote; equal to the unsplit build up to FP32 rounding
    req = request.with_ionic_oxygen(request.build_small_stem(flag="p"))
    one_job = req.p_height * req.p_width * 64 + 8 * req.p_height  # four planes and the row flags
    _, whole = _both(req)
    _, split = _both(req, scratch_bytes=one_job)
    _, three = _both(req, scratch_bytes=3 * one_job)
    assert rel_l2(split, whole) < 1e-6 and rel_l2(three, whole) < 1e-6
    assert rel_l2(split, so.transmission(req)) < TOL


def test_gridding_is_deterministic(engine_lib):
    req = request.build_small_stem(flag="l")
    _, a = _both(req)
    _, b = _both(req)
    assert np.array_equal(a, b)  # fixed-point spreading: no dependence on atomic order


def test_gridding_scratch_reuse_across_grids(engine_lib):
    # the kernels leave the work memory cleared for the next build; builds of other grid sizes
    # and batch splits in between must not change a result by a bit
    a = request.build_small_stem(flag="p", p=256)
    b = request.with_ionic_oxygen(request.build_small_stem(flag="p", p=128))
    _, ta = _both(a)
    _, tb = _both(b, scratch_bytes=b.p_height * b.p_width * 64)
    for req, ref, scratch in ((a, ta, 0), (b, tb, 0), (a, ta, 3 * a.p_height * a.p_width * 64), (b, tb, 0)):
        _, t = _both(req, scratch_bytes=scratch)
        if scratch == 0 and req is a:
            assert np.array_equal(t, ref)
        else:
            assert rel_l2(t, ref) < 1e-6
    assert rel_l2(ta, so.transmission(a)) < TOL


def test_gridding_needs_uniform_axes(engine_lib):
    # separable but non-uniform reciprocal axes: the gridding request falls back to the direct sums
    req = request.build_small_stem(flag="p")
    kx = req.kx.copy()
    kx[:, 5] += 1e-3 * (kx[0, 1] - kx[0, 0])
    req = replace(req, kx=kx)
    direct, grid = _both(req)
    assert np.array_equal(grid, direct)
    assert rel_l2(grid, so.transmission(req)) < TOL


def test_gridding_stem_vs_direct_1024(engine_lib):
    # SrTiO3 filling a 1024^2 potential (16 x 16 cells, 10 slices): transmission and ADF/BF images
    req = request.build_srtio3_stem(cells=(16, 16, 5), n=256, raster=(3, 3), p=1024)
    direct, grid = _both(req)
    assert rel_l2(grid, direct) < TOL_DIRECT, rel_l2(grid, direct)
    with capi.tx_builder(capi.TX_DIRECT):
        rd, _ = capi.stem_run(req)
    with capi.tx_builder(capi.TX_GRIDDING):
        rg, _ = capi.stem_run(req)
    A, D = req.aper_num, req.depth
    for a in range(A):
        assert rel_l2(rg.reshape(A, D)[a], rd.reshape(A, D)[a]) < 1e-5



def test_correction_rows_on_a_non_separable_grid(engine_lib):
    # a reciprocal grid that is not a meshgrid (kx depending on the row) takes the per-atom kernel
    # for every kind of row, the correction rows included
    req = request.with_correction(request.build_small_stem(flag="p", slices=3))
    kx = req.kx.copy()
    kx[1::2] *= 1.0 + 1e-9  # breaks the separable layout, changes the physics negligibly
    bent = replace(req, kx=kx)
    s = capi.Session()
    s.upload(bent)
    s.run(what=1)
    assert s.timing().tx_builder == capi.TX_ROWS
    t = s.download(want_transmission=True)[2]
    s.close()
    assert rel_l2(t, so.transmission(bent)) < TOL
