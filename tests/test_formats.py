"""Output files and DPC / IDPC post-processing (host only)."""
import numpy as np

from totem_b200 import formats


def test_exit_wave_round_trip_and_layout(tmp_path):
    rng = np.random.default_rng(0)
    psi = rng.normal(size=(6, 4)) + 1j * rng.normal(size=(6, 4))
    p = tmp_path / "HRTEM_exitwave.dat"
    formats.write_exit_wave_dat(str(p), psi)
    raw = np.fromfile(p, dtype=np.float32)
    # column 0, row 0 then column 0, row 1: re, im interleaved down the column
    assert np.isclose(raw[0], psi[0, 0].real) and np.isclose(raw[1], psi[0, 0].imag)
    assert np.isclose(raw[2], psi[1, 0].real) and np.isclose(raw[3], psi[1, 0].imag)
    back = formats.read_exit_wave_dat(str(p), 6, 4)
    assert np.allclose(back, psi, rtol=1e-6, atol=1e-6)


def test_stem_dat_scan_order(tmp_path):
    result = np.arange(2 * 6, dtype=np.float64)  # 2 detectors x (2 rows x 3 columns)
    paths = formats.write_stem_dat(str(tmp_path), "run", result, 2, 6, 97.6, [(60, 200), (0, 10)], scale=0.5)
    assert paths[0].endswith("run_STEM_97.6slice_Dect_60_200.dat")
    assert np.array_equal(formats.read_f32(paths[1], (6,)), (result[6:] * 0.5).astype(np.float32))
    img = formats.stem_images(result, 2, 2, 3)
    assert img[1, 1, 0] == result[6 + 3]


def test_idpc_integrates_a_gradient():
    h, w, pitch = 32, 48, 0.4
    y, x = np.mgrid[0:h, 0:w]
    phi = np.cos(2 * np.pi * 3 * x / w) + 0.5 * np.sin(2 * np.pi * 2 * y / h)
    kx, ky = np.meshgrid(np.fft.fftfreq(w, d=pitch), np.fft.fftfreq(h, d=pitch))
    F = np.fft.fft2(phi)
    px = np.real(np.fft.ifft2(2j * np.pi * kx * F))
    py = np.real(np.fft.ifft2(2j * np.pi * ky * F))
    p = formats.idpc(px, py, pitch)
    assert np.allclose(p - p.mean(), phi - phi.mean(), atol=1e-10)


def test_ddpc_and_idpc_files(tmp_path):
    rng = np.random.default_rng(1)
    q = [rng.random((8, 8)) for _ in range(4)]
    out = formats.write_idpc_dat(str(tmp_path), "run", q, 100, 195.25, (10, 40), 0.5)
    px, py = formats.ddpc(*q)
    assert np.allclose(formats.read_f32(out["DDPCx"], (8, 8)), px.astype(np.float32))
    assert np.allclose(formats.read_f32(out["DDPCy"], (8, 8)), py.astype(np.float32))
    assert out["IDPC"].endswith("run_IDPC_195.25slice_Dect_10_40.dat")
