"""ToTem's output files and the DPC / IDPC post-processing of segmented-detector images.

Restated from ToTEM_submit_v1.m (the GUI's result writers, :942-1161, and HRTEMsimulation's
exit-wave dump, :1355-1362), so images computed here can replace the MATLAB ones in users'
downstream scripts:

* every ``.dat`` is raw float32 without a header.  STEM images are written in scan order
  (``fwrite(midimg(:,:,j))`` of the column-major W x H array, i.e. ``result[a*Depth + pos]``);
  HRTEM, CBED and the DPC / IDPC images are written transposed (``fwrite(img.')``), which is
  the row-major order of the image;
* the HRTEM exit wave (``HRTEM_exitwave.dat``, "complex 8") interleaves real and imaginary parts
  down each column: for every column c, for every row r: Re psi(r, c), Im psi(r, c);
* DDPC: px = bb - dd, py = cc - aa from the four quadrants (aa, bb, cc, dd) of a ring; IDPC:
  p = real(ifft2(ifftshift((fftshift(fft2(px)) kx + fftshift(fft2(py)) ky) / (2 pi i k^2))))
  with the zero frequency set to mean(px) + mean(py), on the scan grid (pitch = step x sampling).
"""
from __future__ import annotations

import os

import numpy as np


def write_f32(path: str, arr) -> None:
    """Raw float32 in C order (the layout of ``fwrite(..., 'float')`` of the transposed array)."""
    np.ascontiguousarray(np.asarray(arr, dtype=np.float32)).tofile(path)


def read_f32(path: str, shape) -> np.ndarray:
    return np.fromfile(path, dtype=np.float32).reshape(shape)


# ----------------------------------------------------------------------------------------------
# STEM
# ----------------------------------------------------------------------------------------------

def stem_images(result, aper_num: int, hight_red: int, width_red: int, scale: float = 1.0) -> np.ndarray:
    """Detector images [A][scan row][scan column] from ``result[a*Depth + pos]`` (pos = row *
    width_red + column), times ``scale`` (the reference divides by probesx^2 * allvib)."""
    return np.asarray(result, dtype=np.float64).reshape(aper_num, hight_red, width_red) * scale


def stem_dat_name(name: str, thickness, detector) -> str:
    """``<name>_STEM_<thickness>slice_Dect_<inner>_<outer>.dat`` (ToTEM_submit_v1.m:975-980)."""
    return f"{name}_STEM_{_num2str(thickness)}slice_Dect_{int(round(detector[0]))}_{int(round(detector[1]))}.dat"


def write_stem_dat(folder: str, name: str, result, aper_num: int, depth: int, thickness, detectors,
                   scale: float = 1.0):
    """One ``.dat`` per detector, in scan order, as the reference writes them.  Returns the paths."""
    r = np.asarray(result, dtype=np.float64).reshape(aper_num, depth) * scale
    paths = []
    for a in range(aper_num):
        p = os.path.join(folder, stem_dat_name(name, thickness, detectors[a]))
        write_f32(p, r[a])
        paths.append(p)
    return paths


# ----------------------------------------------------------------------------------------------
# HRTEM
# ----------------------------------------------------------------------------------------------

def write_hrtem_dat(path: str, image, allvib: int = 1) -> None:
    """``fwrite(myresul.'/allvib, 'float')``: the image row by row."""
    write_f32(path, np.asarray(image) / allvib)


def write_exit_wave_dat(path: str, psi) -> None:
    """``HRTEM_exitwave.dat``: real and imaginary parts interleaved down each column."""
    psi = np.asarray(psi)
    a = np.empty((psi.shape[1], psi.shape[0], 2), dtype=np.float32)  # [column][row][re, im]
    a[..., 0] = psi.real.T
    a[..., 1] = psi.imag.T
    a.tofile(path)


def read_exit_wave_dat(path: str, rows: int, cols: int) -> np.ndarray:
    a = np.fromfile(path, dtype=np.float32).reshape(cols, rows, 2)
    return (a[..., 0] + 1j * a[..., 1]).T.astype(np.complex128)


# ----------------------------------------------------------------------------------------------
# DPC / IDPC
# ----------------------------------------------------------------------------------------------

def ddpc(aa, bb, cc, dd):
    """Differential DPC vectors from the four quadrant images of one ring."""
    return np.asarray(bb) - np.asarray(dd), np.asarray(cc) - np.asarray(aa)


def idpc(px, py, pitch_a: float) -> np.ndarray:
    """Integrated DPC: the field whose gradient is (px, py), by division in Fourier space;
    ``pitch_a`` is the scan pitch (step x sampling) in Angstrom."""
    px = np.asarray(px, dtype=np.float64)
    py = np.asarray(py, dtype=np.float64)
    h, w = px.shape
    kx, ky = np.meshgrid(np.arange(-w / 2, w / 2) / (w * pitch_a), np.arange(-h / 2, h / 2) / (h * pitch_a))
    k2 = kx ** 2 + ky ** 2
    num = np.fft.fftshift(np.fft.fft2(px)) * kx + np.fft.fftshift(np.fft.fft2(py)) * ky
    with np.errstate(divide="ignore", invalid="ignore"):
        p = num / (2 * np.pi * 1j * k2)
    p[h // 2, w // 2] = px.mean() + py.mean()
    return np.real(np.fft.ifft2(np.fft.ifftshift(p)))


def write_idpc_dat(folder: str, name: str, quadrants, slice_index: int, thickness, detector, pitch_a: float):
    """The reference's aa/bb/cc/dd, DDPCx/DDPCy and IDPC files of one ring (ToTEM_submit_v1.m
    :1040-1160); ``quadrants`` = (aa, bb, cc, dd) images [scan row][scan column]."""
    aa, bb, cc, dd = quadrants
    px, py = ddpc(aa, bb, cc, dd)
    p = idpc(px, py, pitch_a)
    tag = f"slice_Dect_{int(round(detector[0]))}_{int(round(detector[1]))}.dat"
    out = {}
    for key, img in (("aa", aa), ("bb", bb), ("cc", cc), ("dd", dd), ("DDPCx", px), ("DDPCy", py)):
        out[key] = os.path.join(folder, f"{name}_{key}_{slice_index}{tag}")
        write_f32(out[key], img)
    out["IDPC"] = os.path.join(folder, f"{name}_IDPC_{_num2str(thickness)}{tag}")
    write_f32(out["IDPC"], p)
    return out


def _num2str(x) -> str:
    """MATLAB num2str for the thickness in file names: integers without a decimal point, other
    values with up to 4 decimals (num2str's default precision), trailing zeros dropped."""
    x = float(x)
    if x == int(x):
        return str(int(x))
    return f"{x:.4f}".rstrip("0").rstrip(".")
