"""Host-side request preparation: scattering tables, parameter rows, slicing, frozen phonons,
probe, propagator, detectors and window placement."""
import math

import numpy as np
import pytest

from totem_b200 import optics, request, specimen


def test_tables_parsed_from_reference_files():
    t = specimen.tables()
    assert t["lobato"].shape == (103, 10) and t["peng"].shape == (98, 10)
    assert t["peng_ion"].shape[1] == 12
    # O (Z=8) Peng row as printed in ABSFpara.m
    assert np.allclose(t["peng"][7], [0.0365, 0.1729, 0.5805, 0.8814, 0.3121, 0.0652, 0.6184, 2.9449, 9.6298, 28.2194])
    assert np.allclose(specimen.ion_params(8, -2)[:2], [0.0421, 0.210])


def test_srtio3_slices_hold_sro_and_tio2_planes():
    st = specimen.srtio3_001(8, 8, 2)
    nuc, ion = specimen.potential_params(st.atoms, "p")
    assert nuc.shape == (8 * 8 * 2 * 5, 16) and ion.shape == (0, 28)
    ele_n, ele_n_i, sn, sni = specimen.slice_rows(nuc, ion, st.slice_dz, st.slicethick, 0, "p")
    assert list(sn) == [128, 192, 128, 192] and len(sni) == 0
    assert ele_n.shape == (640, 13)
    z_first = np.unique(nuc[:128, 0])  # rows keep the atom order of the table within a slice
    assert set(z_first) <= {8, 38, 22}
    # Peng rows: x y occ a1 b1 .. a5 b5 with the table's interleaving
    o = specimen.element_params(8, "p")
    row = ele_n[np.argmin(np.abs(ele_n[:, 3] - o[0]))]
    assert np.allclose(row[3:13:2], o[:5]) and np.allclose(row[4:13:2], o[5:])


def test_lobato_rows_carry_debye_waller_column():
    st = specimen.si_001(1, 1, 1, dw={14: 0.5})
    nuc, ion = specimen.potential_params(st.atoms, "l")
    ele_n, _, sn, _ = specimen.slice_rows(nuc, ion, st.slice_dz, st.slicethick, 0, "l", dbmode=1)
    assert ele_n.shape[1] == 14 and np.allclose(ele_n[:, 13], 0.5)
    ele_n0, _, _, _ = specimen.slice_rows(nuc, ion, st.slice_dz, st.slicethick, 0, "l", dbmode=0)
    assert np.allclose(ele_n0[:, 13], 0.0)
    assert sum(sn) == len(st.atoms)


def test_partly_ionic_atoms_use_25_column_rows():
    x = np.array([[8, 1.0, 1.0, 0.2, -2, 0.4, 0.0, 1.0], [38, 2.0, 2.0, 0.3, 0, 0.0, 0.0, 1.0]])
    nuc, ion = specimen.potential_params(x, "p")
    assert nuc.shape == (1, 16) and ion.shape == (1, 28)
    ele_n, ele_n_i, sn, sni = specimen.slice_rows(nuc, ion, 1.0, [0.0], 0, "p")
    assert ele_n_i.shape == (1, 25) and sni[0] == 1
    assert ele_n_i[0, 3] == pytest.approx(0.4) and ele_n_i[0, 14] == pytest.approx(0.6)


def test_debye_waller_folds_into_peng_b():
    x = np.array([[8, 1.0, 1.0, 0.2, 0, 0, 0.7, 1.0]])
    nuc, ion = specimen.potential_params(x, "p")
    f, _ = specimen.fold_debye_waller(nuc, ion, "p")
    assert np.allclose(f[0, 7:16:2], nuc[0, 7:16:2] + 0.7)
    same, _ = specimen.fold_debye_waller(nuc, ion, "l")
    assert np.array_equal(same, nuc)


def test_multislice_spreading_weights():
    # an atom near a slice boundary contributes to both slices with erf weights
    # (CalAllEquilent20210223_lobato_peng.m:213-226)
    x = np.array([[8, 1.0, 1.0, 0.98, 0, 0, 0, 1.0]])
    nuc, ion = specimen.potential_params(x, "p")
    ele_n, _, sn, _ = specimen.slice_rows(nuc, ion, 1.0, [0.0, 1.0, 2.0], 1, "p")
    assert list(sn) == [1, 1, 0]
    w0 = ele_n[0, 3:13:2] / nuc[0, 6:16:2]
    w1 = ele_n[1, 3:13:2] / nuc[0, 6:16:2]
    assert np.all(w0 > 0.4) and np.all(w1 > 0) and np.all(w0 + w1 < 1.0 + 1e-12)


def test_frozen_phonon_is_seeded_and_has_the_requested_rms():
    st = specimen.srtio3_001(6, 6, 6, dw={38: specimen.b_from_rms(0.089), 22: specimen.b_from_rms(0.075),
                                          8: specimen.b_from_rms(0.088)})
    nuc, _ = specimen.potential_params(st.atoms, "p")
    a = specimen.frozen_phonon(nuc, st.slice_dz, st.slicethick, np.random.default_rng(3))
    b = specimen.frozen_phonon(nuc, st.slice_dz, st.slicethick, np.random.default_rng(3))
    c = specimen.frozen_phonon(nuc, st.slice_dz, st.slicethick, np.random.default_rng(4))
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    d = (a - nuc)[:, 1:3]
    for z, rms in ((38, 0.089), (22, 0.075), (8, 0.088)):
        sel = nuc[:, 0] == z
        assert np.std(d[sel]) == pytest.approx(rms, rel=0.1)
    lo, hi = st.slicethick[0], st.slicethick[-1] + st.slice_dz
    assert np.all((a[:, 3] >= lo) & (a[:, 3] < hi))


def test_probe_is_normalised_and_centred():
    spec = optics.ProbeSpec(kv=300, semi_angle_mrad=25, aberrations=optics.Aberrations(Cs=-5e3))
    probe, gfsf = optics.stem_probes(spec, 256, 0.0625)
    assert probe.shape == (1, 256, 256) and np.allclose(gfsf, [1.0])
    assert np.sum(np.abs(probe[0]) ** 2) == pytest.approx(1.0, rel=1e-12)
    assert np.unravel_index(np.argmax(np.abs(probe[0])), probe[0].shape) == (128, 128)


def test_focal_spread_weights_sum_to_about_one():
    delta, w = optics.gaussian_focal_weights(11, 4.0, optics.wavelength_nm(200), 2.0)
    assert len(w) == 11 and delta > 0
    assert w.sum() == pytest.approx(1.0, abs=0.05)
    assert np.allclose(w, w[::-1])


def test_propagator_band_limit_and_phase():
    n, dx, kv, dz = 64, 0.2, 200.0, 1.5
    h = np.fft.fftshift(optics.propagator(n, dx, kv, dz, "2/3"))
    px = optics.centered_freqs(n, dx)
    p2 = px[None, :] ** 2 + px[:, None] ** 2
    inside = p2 <= 1 / (9 * dx * dx)
    assert np.all(h[~inside] == 0) and np.allclose(np.abs(h[inside]), 1)
    lam = optics.wavelength_nm(kv) * 10
    assert np.allclose(np.angle(h[inside] * np.exp(1j * math.pi * lam * dz * p2[inside])), 0, atol=1e-9)
    h2 = np.fft.fftshift(optics.propagator(n, dx, kv, dz, "1/2"))
    assert np.count_nonzero(h2) < np.count_nonzero(h)


def test_annular_detectors():
    a = optics.annular_detectors(128, 0.1, 300, [(60, 200), (0, 10)])
    assert a.shape == (2, 128, 128) and set(np.unique(a)) <= {0.0, 1.0}
    assert a[1, 64, 64] == 1 and a[0, 64, 64] == 0
    q = optics.segmented_detectors(128, 0.1, 300, [(10, 30, 0)])
    assert q.shape == (4, 128, 128) and np.allclose(q.sum(0), optics.annular_detectors(128, 0.1, 300, [(10, 30)])[0])


def test_window_origins_follow_the_reference_scan_order():
    req = request.build_small_stem(raster=(3, 4), step=5)
    r, c = request.window_origins(req)
    assert r[0] == req.beginrow and c[0] == req.begincol
    assert r[4] == req.beginrow + 5 and c[4] == req.begincol  # pos = 4 -> second scan row
    assert c[3] == req.begincol + 15
    request.validate(req)
    from dataclasses import replace
    with pytest.raises(ValueError):
        request.validate(replace(req, begincol=req.p_width))


def test_config_workload_shape():
    req = request.build_srtio3_stem(cells=(8, 8, 50))
    assert req.slices == 100 and req.depth == 4096 and req.height == 512 and req.p_height == 1024
    assert len(req.ele_n) == 16000 and req.probe_slices == 409600
    request.validate(req)
