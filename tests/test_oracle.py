"""The FP64 oracle pinned against physics and against its committed golden fixtures.

The reference ships no tests or golden vectors and its CPU path (MATLAB) cannot run here, so the
oracle is pinned by closed-form physics and invariants:
  * electron wavelength and interaction constant against Kirkland's published values;
  * the projected potential of one Peng atom against its analytic real-space form;
  * vacuum transmission and flux conservation of the slice loop;
  * Peng vs Lobato scattering factors (two independent fits of the same physics);
  * regression fixtures in tests/golden (see make_golden.py).
"""
import math
import os
from dataclasses import replace

import numpy as np
import pytest

from oracle import stem_oracle as so
from tests.conftest import rel_l2
from totem_b200 import optics, request, specimen

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_wavelength_and_sigma_match_published_values():
    # Kirkland, Advanced Computing in Electron Microscopy, table 5.2
    assert optics.wavelength_nm(200.0) * 10 == pytest.approx(0.025079, rel=2e-4)
    assert optics.wavelength_nm(300.0) * 10 == pytest.approx(0.019687, rel=2e-4)
    # sigma in rad / (kV * Angstrom): the engine applies sigma / 1000 per volt
    assert optics.interaction_sigma(200.0) / 1000 == pytest.approx(7.2884e-4, rel=1e-3)
    assert optics.interaction_sigma(300.0) / 1000 == pytest.approx(6.5262e-4, rel=1e-3)


def _single_atom_request(flag, z, p=256, sampling=0.05):
    x = np.zeros((1, 8))
    x[0] = [z, p * sampling / 2, p * sampling / 2, 0.1, 0, 0, 0, 1]
    st = specimen.Structure(x, (0, 0, 1.0), 1.0, 1)
    nuc, ion = specimen.potential_params(x, flag)
    ele_n, ele_n_i, sn, sni = specimen.slice_rows(nuc, ion, 1.0, st.slicethick, 0, flag)
    kx, ky, s2 = optics.reciprocal_grids(p, p, sampling)
    return request.StemRequest(
        param=flag, probe=np.zeros((1, 2, 2), complex), aper=np.zeros((1, 2, 2)), aper2=np.zeros((1, 2, 2)),
        ele_n=ele_n, series_n=sn, ele_n_i=ele_n_i, series_n_i=np.zeros(1), kx=kx, ky=ky, s2=s2,
        prop=np.ones((2, 2), complex), gfsf=np.ones(1), p_height=p, p_width=p, step=0, beginrow=0, begincol=0,
        width_red=1, hight_red=0, sigma=optics.interaction_sigma(200.0),
        parameter=optics.potential_parameter(p, p, sampling), aper_true=np.ones((p, p)))


def _real_potential(req):
    vg = so.potential_fourier(req)[0]
    n = req.p_height * req.p_width
    return np.fft.ifft2(np.fft.ifftshift(vg)) * n


@pytest.mark.parametrize("z", [8, 14, 38])
def test_single_peng_atom_matches_analytic_projected_potential(z):
    # f(s) = sum a_i exp(-b_i s^2), s = g/2, has the projected potential
    #   v(r) = C sum a_i (4 pi / b_i) exp(-4 pi^2 r^2 / b_i),  C = 2 pi hbar^2 / (e m) in V A^2,
    # whose integral over the plane is C f(0).  A 0.02 A grid resolves the narrowest Gaussian
    # (f at the Nyquist frequency < 1e-4 of f(0)), so the sampled potential must match point-wise.
    p, dx = 512, 0.02
    req = _single_atom_request("p", z, p, dx)
    v = _real_potential(req)
    c = p // 2
    prm = specimen.element_params(z, "p")
    a, b = prm[:5], prm[5:]
    const = 2 * math.pi * optics.H_BAR ** 2 / (optics.E_CHARGE * optics.M_ELECTRON * 1e-20)
    assert v.real.sum() * dx * dx == pytest.approx(const * a.sum(), rel=1e-6)
    r = np.arange(0, 60) * dx
    analytic = const * np.array([np.sum(a * 4 * math.pi / b * np.exp(-4 * math.pi ** 2 * rr ** 2 / b)) for rr in r])
    got = v.real[c, c:c + 60]
    assert np.max(np.abs(got - analytic) / analytic) < 1e-3
    # radially symmetric: along rows and columns, both directions
    assert np.allclose(v.real[c, c + 1:c + 60], v.real[c + 1:c + 60, c], rtol=1e-9)
    assert np.allclose(v.real[c, c + 1:c + 60], v.real[c, c - 1:c - 60:-1], rtol=1e-9)


def test_lobato_and_peng_agree():
    s = np.linspace(0.0, 1.5, 50)
    g2 = 4 * s * s
    for z in (8, 14, 22, 38):
        pp = specimen.element_params(z, "p")
        pl = specimen.element_params(z, "l")
        fp = sum(pp[i] * np.exp(-pp[5 + i] * s * s) for i in range(5))
        fl = sum(pl[i] * (2 + pl[5 + i] * g2) / (1 + pl[5 + i] * g2) ** 2 for i in range(5))
        assert np.max(np.abs(fp - fl) / fl) < 0.05, z


def test_vacuum_transmission_is_one_and_flux_is_conserved():
    req = request.build_small_stem(slices=3, mid_layer=(1,))
    A = req.aper_num
    empty = replace(req, ele_n=req.ele_n[:0], series_n=np.zeros(req.slices),
                    aper=np.ones((1, req.height, req.width)), aper2=np.ones((1, req.height, req.width)))
    T = so.transmission(empty)
    assert np.abs(T - 1).max() == 0.0
    res, mid = so.stem(empty, T)
    n2 = req.height * req.width
    # a unit-norm probe inside the propagator's band limit keeps sum |FFT psi|^2 = N^2
    assert np.allclose(res, n2, rtol=1e-10) and np.allclose(mid, n2, rtol=1e-10)
    assert A >= 1


def test_specimen_scatters_but_conserves_flux_to_the_band_limit():
    req = request.build_small_stem(slices=4)
    ones = replace(req, aper=np.ones((1, req.height, req.width)), aper2=np.ones((1, req.height, req.width)),
                   mid_layer=np.zeros(0, dtype=np.int32))
    res, _ = so.stem(ones)
    n2 = req.height * req.width
    # a pure phase object only loses what it scatters past 2/3 of Nyquist; |T| != 1 only through
    # the Nyquist row/column of V(g), a tiny amount
    assert np.all(res < 1.01 * n2) and np.all(res > 0.9 * n2)


def test_detector_images_are_linear_in_gfsf():
    req = request.build_small_stem(focal_steps=3, mid_layer=(2,))
    T = so.transmission(req)
    res, mid = so.stem(req, T)
    res2, mid2 = so.stem(replace(req, gfsf=2.0 * req.gfsf), T)
    assert np.allclose(res2, 2 * res, rtol=1e-12) and np.allclose(mid2, 2 * mid, rtol=1e-12)


@pytest.mark.parametrize("name", ["peng_small", "lobato_spread"])
def test_golden_fixture(name):
    path = os.path.join(GOLDEN, f"{name}.npz")
    g = np.load(path)
    from tests.golden.make_golden import CASES, build_case
    req = build_case(CASES[name])
    # the inputs the oracle sees are still the ones the fixture was made from
    for key in ("probe", "ele_n", "prop", "aper"):
        assert np.allclose(getattr(req, key), g[key], rtol=0, atol=1e-12), key
    T = so.transmission(req)
    assert rel_l2(T, g["T"]) < 1e-12
    res, mid = so.stem(req, T)
    assert rel_l2(res, g["result"]) < 1e-12
    if len(g["mid"]):
        assert rel_l2(mid, g["mid"]) < 1e-12


def test_focal_spread_steps_must_be_odd():
    from totem_b200 import optics
    with pytest.raises(ValueError):
        optics.gaussian_focal_weights(2, 4.0, 0.0025, 1.0)
    d, w = optics.gaussian_focal_weights(3, 4.0, 0.0025, 1.0)
    assert len(w) == 3 and d > 0


def test_cbed_in_vacuum_is_the_probe_spectrum():
    # With T = 1 every slice only multiplies the spectrum by the unit-modulus propagator inside its
    # band, and the probes (20 mrad aperture) lie inside it: the CBED pattern is
    # sum_n gfsf_n |fftshift(fft2(probe_n))|^2 (ToTEM_submit_v1.m:1478-1492), whose sum is
    # N^2 sum_n gfsf_n |probe_n|^2 (Parseval).
    req = request.build_small_stem(n=64, p=128, raster=(1, 1), slices=4, focal_steps=3)
    T = np.ones((req.slices, req.p_height, req.p_width), dtype=np.complex128)
    pat = so.cbed(req, T)
    ref = sum(g * np.abs(np.fft.fftshift(np.fft.fft2(p))) ** 2 for g, p in zip(req.gfsf, req.probe))
    assert rel_l2(pat, ref) < 1e-12
    norm = sum(g * np.sum(np.abs(p) ** 2) for g, p in zip(req.gfsf, req.probe))
    assert abs(pat.sum() / (req.height * req.width * norm) - 1.0) < 1e-12
    # zero frequency at the centre: the untilted bright-field disc is centred on (N/2, N/2)
    r, c = np.indices(pat.shape)
    assert abs((r * pat).sum() / pat.sum() - req.height // 2) < 0.5
    assert abs((c * pat).sum() / pat.sum() - req.width // 2) < 0.5
