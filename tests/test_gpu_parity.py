"""CUDA engine vs the FP64 oracle, through the C ABI (``totem_stem_run`` / sessions /
``myProjectfun``).

Tolerance: relative L2 <= 1e-4 on every detector image and on the transmission stack -- the
accuracy target of the FP32 engine against FP64.
"""
import numpy as np
import pytest

from oracle import stem_oracle as so
from tests.conftest import rel_l2
from totem_b200 import capi, request

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _check(req, res, mid, tol=TOL, T=None):
    if T is None:
        T = so.transmission(req)
    ref_res, ref_mid = so.stem(req, T)
    A, D, L = req.aper_num, req.depth, len(req.mid_layer)
    r, rr = res.reshape(A, D), ref_res.reshape(A, D)
    for a in range(A):
        assert rel_l2(r[a], rr[a]) < tol, (a, rel_l2(r[a], rr[a]))
    if L:
        m, rm = mid.reshape(L, A, D), ref_mid.reshape(L, A, D)
        for l in range(L):
            for a in range(A):
                if np.linalg.norm(rm[l, a]) == 0:
                    assert np.all(m[l, a] == 0)
                else:
                    assert rel_l2(m[l, a], rm[l, a]) < tol, (l, a, rel_l2(m[l, a], rm[l, a]))


@pytest.mark.parametrize("flag", ["p", "l"])
@pytest.mark.parametrize("path", [capi.PATH_FUSED, capi.PATH_PLAIN])
def test_stem_small_vs_oracle(engine_lib, flag, path):
    req = request.build_small_stem(flag=flag)
    res, mid = capi.stem_run(req, path=path)
    _check(req, res, mid)


@pytest.mark.parametrize("n,p", [(128, 256), (256, 512)])
def test_stem_window_sizes(engine_lib, n, p):
    req = request.build_small_stem(n=n, p=p, raster=(2, 2), step=17, slices=4, sampling=0.1, mid_layer=(1, 4))
    res, mid = capi.stem_run(req)
    _check(req, res, mid)


@pytest.mark.parametrize("n,p,raster,step", [(512, 1024, (2, 2), 64), (1024, 1024, (1, 1), 0)])
def test_stem_large_windows(engine_lib, n, p, raster, step):
    req = request.build_small_stem(n=n, p=p, raster=raster, step=step, slices=3, sampling=0.05, cells=4,
                                   mid_layer=(2,))
    for path in (capi.PATH_FUSED, capi.PATH_PLAIN):
        res, mid = capi.stem_run(req, path=path)
        _check(req, res, mid)


def test_transmission_vs_oracle(engine_lib):
    req = request.build_small_stem(flag="l")
    t = capi.transmission_run(req)
    ref = so.transmission(req)
    assert rel_l2(t, ref) < TOL
    # the *P MEX flavour through the reference's own entry-point signature
    t2 = capi.call_myprojectfun(req, transmission=True)
    assert rel_l2(t2, ref) < TOL


def test_myprojectfun_stem_abi(engine_lib):
    req = request.build_small_stem(flag="p", mid_layer=(3,))
    res, mid = capi.call_myprojectfun(req, transmission=False)
    _check(req, res, mid)


def test_defocus_spread_and_unsorted_layers(engine_lib):
    # w_num > 1 with gfsf weights; mid layers unsorted, repeated and out of range
    req = request.build_small_stem(focal_steps=3, mid_layer=(5, 2, 5, 99, 6))
    res, mid = capi.stem_run(req)
    _check(req, res, mid)


def test_absorptive_and_ionic_rows(engine_lib):
    # a third of the atoms as partly ionic O (O2-), plus absorptive rows on everything
    req = request.with_absorption(request.with_ionic_oxygen(request.build_small_stem(flag="p")))
    res, mid = capi.stem_run(req)
    _check(req, res, mid)


def test_session_reuse_and_batches(engine_lib):
    req = request.build_small_stem(raster=(4, 5))
    s = capi.Session()
    s.upload(req)
    outs = []
    for b, cv in ((1, 0), (3, 2), (7, 3), (0, 0), (2, 1)):
        s.run(batch=b, col_variant=cv)
        res, mid, _ = s.download()
        outs.append((res, mid))
    for r, m in outs[1:]:
        assert np.array_equal(r, outs[0][0]) and np.array_equal(m, outs[0][1])  # batch-composition invariance
    _check(req, *outs[0])
    t = s.timing()
    assert t.kernel_launches > 0 and t.total_ms > 0
    # wider column tiles regroup the FP64 detector sums: equal to rounding, not bit for bit
    for cv in (5, 6):
        s.run(batch=5, col_variant=cv)
        res, mid, _ = s.download()
        np.testing.assert_allclose(res, outs[0][0], rtol=1e-12, atol=0)
        np.testing.assert_allclose(mid, outs[0][1], rtol=1e-12, atol=0)
    s.close()


def test_repeated_runs_replay_as_graph(engine_lib):
    # the second run with the same shapes is captured into a CUDA graph and later runs replay it;
    # every run must equal the direct (ungraphed) run bit for bit, also after the inputs change
    req = request.build_small_stem(raster=(3, 5), mid_layer=(2, 5))
    capi.set_slice_graphs(False)
    try:
        s0 = capi.Session()
        s0.upload(req)
        s0.run()
        ref = s0.download()[:2]
        s0.close()
    finally:
        capi.set_slice_graphs(True)
    s = capi.Session()
    s.upload(req)
    for i in range(4):
        s.run(skip_transmission=i > 0)
        res, mid, _ = s.download()
        assert np.array_equal(res, ref[0]) and np.array_equal(mid, ref[1]), i
        assert s.timing().kernel_launches > 0
    # new probe contents in the same buffers: the replayed graph reads them
    from dataclasses import replace
    req2 = replace(req, probe=req.probe * np.exp(0.3j))
    s.upload(req2)
    s.run()
    s.run(skip_transmission=True)
    res2, mid2, _ = s.download()
    r2, m2 = capi.stem_run(req2)
    np.testing.assert_allclose(res2, r2, rtol=1e-12)
    np.testing.assert_allclose(mid2, m2, rtol=1e-12)
    s.close()
    _check(req, *ref)


def test_invalid_window_rejected(engine_lib):
    req = request.build_small_stem()
    from dataclasses import replace
    bad = replace(req, begincol=req.p_width - req.width + 1)
    with pytest.raises(capi.TotemError) as e:
        capi.stem_run(bad)
    assert e.value.code == capi.ERR_INVALID_ARG


def test_path_used_is_reported_and_fused_only_refuses_cufft(engine_lib):
    # an 80^2 window on a 176^2 grid: no hand-written transform of these lengths, so the fused
    # request runs on cuFFT, says so in its timing, and TOTEM_PATH_FUSED_ONLY refuses it
    odd = request.build_small_stem(n=80, p=176, raster=(2, 2), step=5, slices=3, mid_layer=(2,))
    s = capi.Session()
    s.upload(odd)
    s.run(path=capi.PATH_FUSED)
    res, mid, _ = s.download()
    t = s.timing()
    assert (t.slice_path, t.tx_fft_path) == (capi.PATH_PLAIN, capi.PATH_PLAIN)
    assert t.tx_builder in (capi.TX_DIRECT, capi.TX_GRIDDING)
    _check(odd, res, mid)
    with pytest.raises(capi.TotemError) as e:
        s.run(path=capi.PATH_FUSED_ONLY)
    assert e.value.code == capi.ERR_UNSUPPORTED and "FUSED_ONLY" in str(e.value)
    s.close()
    ok = request.build_small_stem()
    s = capi.Session()
    s.upload(ok)
    s.run(path=capi.PATH_FUSED_ONLY)
    res, mid, _ = s.download()
    t = s.timing()
    assert (t.slice_path, t.tx_fft_path) == (capi.PATH_FUSED, capi.PATH_FUSED)
    _check(ok, res, mid)
    s.run(path=capi.PATH_PLAIN)
    assert s.timing().slice_path == capi.PATH_PLAIN
    s.close()


@pytest.mark.parametrize("n,p,variant,focal", [(64, 128, 0, 1), (64, 128, 5, 3), (128, 256, 2, 1), (128, 256, 6, 1),
                                                (256, 512, 0, 3)])
def test_zero_band_skip_changes_nothing(engine_lib, n, p, variant, focal):
    # The propagator is zero beyond 2/3 of Nyquist, so about a third of the wave's columns are
    # zero after every column pass; skipping them (reads, transforms, writes, detector partials)
    # must give the same numbers as computing them.
    req = request.build_small_stem(n=n, p=p, raster=(2, 3), step=9, slices=5, sampling=0.1, mid_layer=(2, 5),
                                   focal_steps=focal)
    outs = {}
    for skip in (False, True):
        capi.set_band_skip(skip)
        try:
            s = capi.Session()
            s.upload(req)
            s.run(col_variant=variant)
            outs[skip] = s.download()[:2]
            s.close()
        finally:
            capi.set_band_skip(True)
    for a, b in zip(outs[False], outs[True]):
        np.testing.assert_array_equal(a, b)
    _check(req, *outs[True])


def test_zero_band_skip_hrtem_and_server(engine_lib):
    # HRTEM's propagator is cut at 1/2 of Nyquist: half of the columns are skipped; the kept
    # spectrum of the last pass is stored whole.  The server applies the same skip per group.
    req, hs = request.build_si_hrtem_001(cells=(2, 2, 2), p=128, slices=6)
    capi.set_band_skip(False)
    try:
        ex0, img0 = capi.hrtem_run(req, hs)
        stem = request.build_small_stem(raster=(3, 3), mid_layer=(3,))
        r0, m0 = capi.stem_run(stem)
    finally:
        capi.set_band_skip(True)
    ex1, img1 = capi.hrtem_run(req, hs)
    np.testing.assert_array_equal(ex0, ex1)
    np.testing.assert_array_equal(img0, img1)
    with capi.Server() as srv:
        t = srv.submit(stem)
        r1, m1 = srv.wait(t)
    np.testing.assert_array_equal(r0, r1)
    np.testing.assert_array_equal(m0, m1)


# Mixed-radix windows (2^a x 3, 5, 7, 9, 25): window, potential grid, raster, step, slices.  The
# grids that are not powers of two take cuFFT for the transmission FFT; the slice loop is fused.
MR_CASES = [(96, 128, (2, 3), 5, 5), (160, 192, (2, 2), 9, 4), (192, 256, (2, 2), 17, 4), (288, 320, (2, 2), 9, 3),
            (320, 512, (2, 2), 33, 3), (384, 512, (2, 1), 40, 3), (400, 448, (2, 2), 17, 3), (448, 512, (1, 2), 30, 3),
            (576, 640, (2, 1), 33, 3), (640, 768, (1, 2), 64, 2), (768, 1024, (2, 2), 64, 2), (800, 832, (1, 1), 0, 2),
            (1152, 1152, (1, 1), 0, 2), (1280, 1280, (1, 1), 0, 2), (1536, 1536, (1, 1), 0, 2),
            (1600, 1600, (1, 1), 0, 2)]


@pytest.mark.parametrize("n,p,raster,step,slices", MR_CASES)
def test_mixed_radix_windows_vs_oracle(engine_lib, n, p, raster, step, slices):
    # four unit cells across, inside the field of every grid
    req = request.build_small_stem(n=n, p=p, raster=raster, step=step, slices=slices, sampling=max(0.05, 20.0 / p),
                                   cells=4, mid_layer=(1,))
    s = capi.Session()
    s.upload(req)
    s.run(path=capi.PATH_FUSED)
    res, mid, _ = s.download()
    t = s.timing()
    assert t.slice_path == capi.PATH_FUSED
    assert (t.row_variant, t.col_variant) == (1, 1)
    s.run(path=capi.PATH_FUSED, col_variant=5, row_variant=4)  # shapes other than the default: ignored
    assert (s.timing().row_variant, s.timing().col_variant) == (1, 1)
    r2, m2, _ = s.download()
    np.testing.assert_array_equal(res, r2)
    np.testing.assert_array_equal(mid, m2)
    s.close()
    # above 1024^2 grids the oracle's own transmission takes minutes: the slice loop is checked
    # on the engine's transmission (checked against the oracle on the smaller grids)
    _check(req, res, mid, T=capi.transmission_run(req) if p > 1024 else None)


@pytest.mark.parametrize("n,p", [(288, 320), (400, 448), (1600, 1600)])
def test_mixed_radix_zero_band_skip_and_server(engine_lib, n, p):
    # CTA-wide barriers (transform groups of 12, 20 and 80 threads), the zero-band skip on and
    # off, and the same request served by the continuous-batching server next to a 64^2 one
    raster, step = ((2, 2), 9) if n < 1600 else ((1, 1), 0)
    req = request.build_small_stem(n=n, p=p, raster=raster, step=step, slices=3, sampling=max(0.05, 20.0 / p),
                                   cells=4, mid_layer=(2,), focal_steps=3 if n < 1600 else 1)
    outs = {}
    for skip in (False, True):
        capi.set_band_skip(skip)
        try:
            outs[skip] = capi.stem_run(req)
        finally:
            capi.set_band_skip(True)
    for a, b in zip(outs[False], outs[True]):
        np.testing.assert_array_equal(a, b)
    with capi.Server() as srv:
        t1 = srv.submit(req)
        t2 = srv.submit(request.build_small_stem())
        r1, m1 = srv.wait(t1)
        srv.wait(t2)
    np.testing.assert_array_equal(r1, outs[True][0])
    np.testing.assert_array_equal(m1, outs[True][1])
    _check(req, *outs[True], T=capi.transmission_run(req) if p > 1024 else None)


@pytest.mark.parametrize("p", [320, 400, 576])
def test_mixed_radix_potential_grid_transmission(engine_lib, p):
    # mixed-radix potential grids take the fused transmission FFT (TOTEM_PATH_FUSED_ONLY accepts them)
    req = request.build_small_stem(n=64, p=p, raster=(2, 2), step=9, slices=3, sampling=max(0.05, 20.0 / p),
                                   cells=4, mid_layer=(2,))
    s = capi.Session()
    s.upload(req)
    s.run(path=capi.PATH_FUSED_ONLY)
    t = s.timing()
    assert (t.slice_path, t.tx_fft_path) == (capi.PATH_FUSED, capi.PATH_FUSED)
    res, mid, _ = s.download()
    s.close()
    ref_t = so.transmission(req)
    assert rel_l2(capi.transmission_run(req), ref_t) < TOL
    _check(req, res, mid, T=ref_t)


@pytest.mark.parametrize("p_w,fused", [(160, False), (256, True)])
def test_non_square_potential_grid(engine_lib, p_w, fused):
    # A 192 x p_w potential grid: the fused transmission FFT needs the rows of all slices to make
    # whole row tiles of p_w (20 rows for 160: 3 x 192 rows do not) and p_w whole column tiles of
    # 192; otherwise the request runs the transmission FFT on cuFFT.  Both match the oracle.
    from dataclasses import replace
    from totem_b200 import optics
    req = request.build_small_stem(n=64, p=192, raster=(2, 2), step=9, slices=3, sampling=0.1, mid_layer=(2,))
    kx, ky, s2 = optics.reciprocal_grids(192, p_w, 0.1)
    req = replace(req, p_width=p_w, kx=kx, ky=ky, s2=s2, aper_true=np.ones((192, p_w)),
                  parameter=optics.potential_parameter(192, p_w, 0.1))
    s = capi.Session()
    s.upload(req)
    s.run()
    t = s.timing()
    assert t.slice_path == capi.PATH_FUSED
    assert t.tx_fft_path == (capi.PATH_FUSED if fused else capi.PATH_PLAIN)
    res, mid, _ = s.download()
    s.close()
    ref_t = so.transmission(req)
    assert rel_l2(capi.transmission_run(req), ref_t) < TOL
    _check(req, res, mid, T=ref_t)
