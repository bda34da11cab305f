"""HRTEM on the device: exit wave and TCC image against the FP64 CPU oracle (small grids), the
bfloat16 transmission trial, and the precision sweep of the Si [110] 520-slice case against an
FP64 re-run of the same propagation."""
import json
import os

import numpy as np
import pytest

from oracle import stem_oracle as so
from tests.conftest import rel_l2
from totem_b200 import capi, request

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _oracle(req, hs):
    T = so.transmission(req)
    ex = so.hrtem_exit_wave(T, hs.prop)
    img = None
    if hs.tf is not None:
        img = so.hrtem_image(ex, np.fft.fftshift(hs.tf, axes=(-2, -1)), np.ones(ex.shape), hs.weights)
    return ex, img


@pytest.mark.parametrize("case", ["si001", "si110"])
def test_hrtem_vs_oracle(engine_lib, case):
    if case == "si001":
        req, hs = request.build_si_hrtem_001(cells=(4, 4, 2), p=128, slices=8)
    else:
        req, hs = request.build_si_hrtem_110(repeats=6, p=256, sampling=0.08)
    ex, img = capi.hrtem_run(req, hs)
    rex, rimg = _oracle(req, hs)
    assert rel_l2(ex, rex) < TOL
    assert rel_l2(img, rimg) < TOL


@pytest.mark.parametrize("p,path", [(192, capi.PATH_FUSED), (400, capi.PATH_FUSED), (200, capi.PATH_PLAIN),
                                    (250, capi.PATH_PLAIN)])
def test_hrtem_grid_edges_vs_oracle(engine_lib, p, path):
    # the reference's HRTEM grid is the potential grid, round(extent / sampling) made even: mixed-radix
    # edges run the fused passes, every other edge cuFFT, and the session says which ran
    req, hs = request.build_si_hrtem_001(cells=(3, 3, 2), p=p, slices=6)
    s = capi.Session()
    s.upload(req, stem=False)
    ex, img = s.hrtem(hs)
    assert s.timing().slice_path == path
    if path == capi.PATH_PLAIN:
        with pytest.raises(capi.TotemError) as e:
            s.hrtem(hs, t_storage=capi.T_BF16)
        assert e.value.code == capi.ERR_UNSUPPORTED
    s.close()
    rex, rimg = _oracle(req, hs)
    assert rel_l2(ex, rex) < TOL
    assert rel_l2(img, rimg) < TOL


def test_hrtem_session_matches_one_shot_and_bf16_trial(engine_lib):
    req, hs = request.build_si_hrtem_001(cells=(4, 4, 4), p=256, slices=16)
    ex1, img1 = capi.hrtem_run(req, hs)
    s = capi.Session()
    s.upload(req, stem=False)
    ex2, img2 = s.hrtem(hs)
    assert np.array_equal(ex1, ex2) and np.array_equal(img1, img2)
    exb, imgb = s.hrtem(hs, t_storage=capi.T_BF16)
    s.close()
    # bfloat16 keeps ~3 significant digits of T: a visible but bounded change of the result
    e_b = rel_l2(exb, ex1)
    assert 1e-6 < e_b < 2e-2, e_b
    assert rel_l2(imgb, img1) < 2e-2


def test_stem_bf16_transmission_trial(engine_lib):
    req = request.build_small_stem(mid_layer=())
    r32, _ = capi.stem_run(req)
    s = capi.Session()
    s.upload(req)
    s.run(t_storage=capi.T_BF16)
    rb, _, _ = s.download()
    s.close()
    e = rel_l2(rb, r32)
    assert 0 < e < 1e-2, e


def test_precision_sweep_si110_520(engine_lib):
    """Si [110], 200 nm (520 slices), 1024^2, 11 defoci: FP32 and FP32 + bfloat16 T against FP64."""
    import torch
    from oracle.hrtem_fp64 import device_complex64, hrtem_fp64
    req, hs = request.build_si_hrtem_110()
    s = capi.Session(device=0)
    s.upload(req, stem=False)
    ex32, img32 = s.hrtem(hs)
    exb, imgb = s.hrtem(hs, t_storage=capi.T_BF16)
    T = device_complex64(s.transmission_ptr(), (req.slices, req.p_height, req.p_width))
    ex64, img64 = hrtem_fp64(T, hs.prop, hs.tf, hs.weights)
    torch.cuda.synchronize()
    del T
    s.close()

    def phase_rms(a, b):
        m = np.abs(b) > 1e-3 * np.abs(b).max()
        return float(np.sqrt(np.mean(np.angle(a[m] * np.conj(b[m])) ** 2)))
    rep = {"workload": "Si [110] 200 nm, 520 slices, 1024^2, 200 kV Lobato, 11 defoci (4 nm rms)",
           "reference": "FP64 propagation (complex128 FFTs) of the same complex64 transmission",
           "fp32": {"image_rel_l2": rel_l2(img32, img64), "exit_rel_l2": rel_l2(ex32, ex64),
                    "exit_phase_rms_rad": phase_rms(ex32, ex64)},
           "fp32_bf16_t": {"image_rel_l2": rel_l2(imgb, img64), "exit_rel_l2": rel_l2(exb, ex64),
                           "exit_phase_rms_rad": phase_rms(exb, ex64)}}
    out = os.environ.get("TOTEM_REPORT_DIR")
    if out:
        with open(os.path.join(out, "precision_si110_520.json"), "w") as f:
            json.dump(rep, f, indent=1)
    print(json.dumps(rep))
    assert rep["fp32"]["image_rel_l2"] < 1e-3
    assert rep["fp32_bf16_t"]["image_rel_l2"] < 0.2


def test_config1_full_size_vs_cpu_oracle(engine_lib):
    """Si [001] 4x4x20 cells, 256^2, 80 slices, Lobato 200 kV, image at Cs 1.2 mm / -50 nm /
    20 mrad: parity at full size and the GPU and CPU-oracle times of one simulation."""
    import time
    req, hs = request.build_si_hrtem_001()
    capi.hrtem_run(req, hs)  # warm-up
    gpu = []
    for _ in range(3):
        t0 = time.perf_counter()
        ex, img = capi.hrtem_run(req, hs)
        gpu.append(time.perf_counter() - t0)
    t0 = time.perf_counter()
    rex, rimg = _oracle(req, hs)
    cpu_s = time.perf_counter() - t0
    rep = {"workload": "Si [001] 4x4x20 cells, 256^2, 80 slices, Lobato 200 kV, Cs 1.2 mm, df -50 nm, 20 mrad",
           "gpu_s_median": float(np.median(gpu)), "cpu_oracle_s": cpu_s, "cpu_threads": 1,
           "exit_rel_l2": rel_l2(ex, rex), "image_rel_l2": rel_l2(img, rimg),
           "note": "GPU time is the whole totem_hrtem_run call from host arrays (upload, transmission, "
                   "80 slices, exit wave, image, download)"}
    out = os.environ.get("TOTEM_REPORT_DIR")
    if out:
        with open(os.path.join(out, "hrtem_si001_config1.json"), "w") as f:
            json.dump(rep, f, indent=1)
    print(json.dumps(rep))
    assert rep["exit_rel_l2"] < TOL and rep["image_rel_l2"] < TOL
