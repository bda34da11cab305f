"""Electron-optical inputs of a STEM/HRTEM request: constants, grids, propagator, detectors, probe.

Everything here restates the reference's host-side MATLAB (``ToTEM_submit_v1.m``) in NumPy FP64.
These arrays are the *inputs* of the multislice engine; they are formed on the host exactly like
the reference forms them before it calls the MEX entry point (``cuda_stem.m``).

Units follow the reference: lengths in Angstrom unless a name says ``_nm``; reciprocal
coordinates in 1/Angstrom; voltage in kV at the API surface.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Physical constants exactly as the reference writes them (ToTEM_submit_v1.m:1509-1513).
H_PLANCK = 6.6255916e-34
H_BAR = H_PLANCK / 2.0 / math.pi
E_CHARGE = 1.602102e-19
M_ELECTRON = 9.1093807e-31
C_LIGHT = 2.9979251e8


def wavelength_nm(kv: float) -> float:
    """Relativistic electron wavelength in nm (ToTEM_submit_v1.m:789)."""
    v = kv * 1000.0
    return 1.0e9 * H_PLANCK * C_LIGHT / math.sqrt(
        E_CHARGE * v * (2 * M_ELECTRON * C_LIGHT * C_LIGHT + E_CHARGE * v))


def interaction_sigma(kv: float) -> float:
    """Interaction constant sigma in 1/(kV*Angstrom) (ToTEM_submit_v1.m:1520).

    The engine applies ``exp(i * V * sigma / 1000)`` (cuda_source_lobato.cu:955, p_exp_sigma).
    """
    v = kv * 1000.0
    lam_a = wavelength_nm(kv) * 10.0
    mc2 = M_ELECTRON * C_LIGHT * C_LIGHT
    return 2 * math.pi / (lam_a * v / 1000.0) * (mc2 + E_CHARGE * v) / (2 * mc2 + E_CHARGE * v)


def potential_parameter(p_rows: int, p_cols: int, sampling: float) -> float:
    """The scale ``PARAMETER`` of the Fourier-space potential (ToTEM_submit_v1.m:1519)."""
    return (2 * math.pi * H_BAR * H_BAR / (E_CHARGE * M_ELECTRON * 1.0e-10 * 1.0e-10)
            / (p_rows * p_cols * sampling * sampling))


def centered_freqs(n: int, sampling: float) -> np.ndarray:
    """(-n/2 .. n/2-1) / (n * sampling): the reference's centred reciprocal axis."""
    return np.arange(-(n // 2), n - n // 2, dtype=np.float64) / (n * sampling)


def reciprocal_grids(p_rows: int, p_cols: int, sampling: float):
    """kx, ky, s^2 on the potential ("green") grid (ToTEM_submit_v1.m:1534-1538).

    ``kx`` varies along columns, ``ky`` along rows; ``s = g/2`` is Peng's variable.
    Arrays are (p_rows, p_cols), C order -- the layout the MEX receives after the
    MATLAB transposes in cuda_stem.m:50-52.
    """
    gx, gy = np.meshgrid(centered_freqs(p_cols, sampling), centered_freqs(p_rows, sampling))
    s2 = (gx / 2) ** 2 + (gy / 2) ** 2
    return gx, gy, s2


def propagator(n: int, sampling: float, kv: float, dz: float, limit: str = "2/3",
               tilt_mrad: float = 0.0, tilt_deg: float = 0.0) -> np.ndarray:
    """Fresnel propagator ``psf_fft`` in natural FFT order (ToTEM_submit_v1.m:1558-1564).

    ``limit='2/3'`` zeroes |k|^2 > 1/(9 dx^2) as the STEM path does; ``limit='1/2'``
    zeroes |k|^2 > 1/(16 dx^2) as the HRTEM path does (ToTEM_submit_v1.m:1330-1333).
    """
    lam_nm = wavelength_nm(kv)
    tilt = tilt_mrad * 1e-3
    phit = -tilt_deg
    tiltx = tilt / lam_nm * math.cos(phit / 180 * math.pi)
    tilty = tilt / lam_nm * math.sin(phit / 180 * math.pi)
    px, py = np.meshgrid(centered_freqs(n, sampling), centered_freqs(n, sampling))
    p2 = (px + tiltx * 0.1) ** 2 + (py + tilty * 0.1) ** 2
    psf = np.exp(-1j * math.pi * lam_nm * 10 * dz * p2)
    cut = 1.0 / (9 * sampling * sampling) if limit == "2/3" else 1.0 / (16 * sampling * sampling)
    psf[p2 > cut] = 0
    return np.fft.ifftshift(psf)


def annular_detectors(n: int, sampling: float, kv: float, ranges_mrad) -> np.ndarray:
    """0/1 annular masks, centred (not shifted) (ToTEM_submit_v1.m:1570-1583).

    ``ranges_mrad`` is a list of ``(inner, outer)`` semi-angles.  Returns (A, n, n).
    """
    lam_a = wavelength_nm(kv) * 10
    px, py = np.meshgrid(centered_freqs(n, sampling), centered_freqs(n, sampling))
    p2 = px ** 2 + py ** 2
    out = np.zeros((len(ranges_mrad), n, n))
    for i, rng in enumerate(ranges_mrad):
        lo, hi = min(rng) * 1e-3 / lam_a, max(rng) * 1e-3 / lam_a
        out[i][(p2 >= lo * lo) & (p2 <= hi * hi)] = 1.0
    return out


def segmented_detectors(n: int, sampling: float, kv: float, rows) -> np.ndarray:
    """Quadrant (DPC/IDPC) masks, four per ``(inner, outer, rotation_deg)`` row.

    Restates ``makeAPER`` (ToTEM_submit_v1.m:1170-1214).
    """
    lam_a = wavelength_nm(kv) * 10
    px, py = np.meshgrid(centered_freqs(n, sampling), centered_freqs(n, sampling))
    p2 = px ** 2 + py ** 2
    theta = np.arctan2(py, px)
    masks = []
    for lo_mrad, hi_mrad, rot in rows:
        lo, hi = lo_mrad * 1e-3 / lam_a, hi_mrad * 1e-3 / lam_a
        ring = ((p2 >= lo * lo) & (p2 <= hi * hi)).astype(np.float64)
        if rot > 180:
            rot -= 180
        if -180 <= rot < -90:
            d = rot
        elif -90 <= rot < 0:
            d = rot - 90
        elif 0 <= rot < 90:
            d = rot - 180
        else:
            d = rot - 270
        q = []
        for k in range(3):
            a0 = (d + 90 * k) * math.pi / 180
            a1 = (d + 90 * (k + 1)) * math.pi / 180
            q.append(((theta >= a0) & (theta < a1)).astype(np.float64))
        q.append(1 - q[0] - q[1] - q[2])
        masks.extend(ring * m for m in q)
    return np.array(masks)


# ----------------------------------------------------------------------------------------------
# Probe formation: aberration function, partial-coherence envelopes, focal spread.
# ----------------------------------------------------------------------------------------------

@dataclass
class Aberrations:
    """Aberration coefficients in the reference's GUI units, already converted to nm.

    Field names follow ``readtccfromhandles_newTEM`` (ToTEM_submit_v1.m:2189-2259): the
    magnitudes are in nm and the angles in degrees *as entered* (the reference negates them).
    """
    focus: float = 0.0      # C1, nm
    A1: float = 0.0
    phiA1: float = 0.0
    A2: float = 0.0
    phiA2: float = 0.0
    B2: float = 0.0
    phiB2: float = 0.0
    Cs: float = 0.0         # C3, nm (1 um = 1000 nm)
    A3: float = 0.0
    phiA3: float = 0.0
    S3: float = 0.0
    phiS3: float = 0.0
    A4: float = 0.0
    phiA4: float = 0.0
    D4: float = 0.0
    phiD4: float = 0.0
    B4: float = 0.0
    phiB4: float = 0.0
    A5: float = 0.0
    phiA5: float = 0.0
    C5: float = 0.0
    S5: float = 0.0
    phiS5: float = 0.0
    D5: float = 0.0
    phiD5: float = 0.0

    def xy(self, name: str):
        mag = getattr(self, name)
        ang = -getattr(self, "phi" + name)
        return mag * math.cos(ang / 180 * math.pi), mag * math.sin(ang / 180 * math.pi)


def _residual_w(ab: Aberrations, u, v, lam):
    """W of all aberrations except C1/A1 (WholeTCC_residual_newTEM, ToTEM_submit_v1.m:2263-2299)."""
    wu = u * lam
    wv = v * lam
    om = wu + 1j * wv
    omc = wu - 1j * wv
    A2x, A2y = ab.xy("A2")
    B2x, B2y = ab.xy("B2")
    A3x, A3y = ab.xy("A3")
    S3x, S3y = ab.xy("S3")
    A4x, A4y = ab.xy("A4")
    D4x, D4y = ab.xy("D4")
    B4x, B4y = ab.xy("B4")
    A5x, A5y = ab.xy("A5")
    S5x, S5y = ab.xy("S5")
    D5x, D5y = ab.xy("D5")
    C3 = ab.Cs
    C5 = ab.C5
    W = (np.real((A2x / 3 + 1j * A2y / 3) * omc ** 3)
         + np.real((B2x + 1j * B2y) * om ** 2 * omc)
         + np.real((A3x / 4 + 1j * A3y / 4) * omc ** 4)
         + np.real(omc * om ** 3 * (S3x + 1j * S3y))
         + np.real(C3 * om ** 2 * omc ** 2) / 4
         + np.real((A4x / 5 + 1j * A4y / 5) * omc ** 5)
         + np.real((D4x + 1j * D4y) * om ** 4 * omc)
         + np.real((B4x + 1j * B4y) * om ** 3 * omc ** 2)
         + np.real((A5x / 6 + 1j * A5y / 6) * omc ** 6)
         + np.real(om ** 4 * omc ** 2 * (S5x + 1j * S5y))
         + np.real(C5 * om ** 3 * omc ** 3) / 6
         + np.real((D5x + 1j * D5y) * om ** 5 * omc))
    return W


def _gradient_w(ab: Aberrations, u, v, lam):
    """Gradient of W without the C1 term (ToTEM_submit_v1.m:2336-2369, the ``flag==2`` branch).

    The reference's expressions are kept as written, including their asymmetries.
    """
    A1x, A1y = ab.xy("A1")
    A2x, A2y = ab.xy("A2")
    B2x, B2y = ab.xy("B2")
    A3x, A3y = ab.xy("A3")
    S3x, S3y = ab.xy("S3")
    A4x, A4y = ab.xy("A4")
    D4x, D4y = ab.xy("D4")
    B4x, B4y = ab.xy("B4")
    A5x, A5y = ab.xy("A5")
    S5x, S5y = ab.xy("S5")
    D5x, D5y = ab.xy("D5")
    C3, C5 = ab.Cs, ab.C5
    L = lam
    r2 = u * u + v * v
    gu = (L * (A1x * u + A1y * v)
          + A2x * L ** 2 / 3 * (3 * u * u - 3 * v * v) + A2y * L ** 2 / 3 * 6 * u * v
          + B2x * (3 * u ** 2 + v ** 2) * L ** 2 - B2y * L ** 2 * 2 * u * v
          + 0.25 * L ** 3 * (A3x * (4 * u ** 3 - 12 * u * v * v) + A3y * (12 * u * u * v - 4 * v ** 3))
          + L ** 3 * (2 * u * (S3x * (u * u - v * v) - S3y * 2 * u * v) + r2 * (2 * S3x * u - 2 * S3y * v))
          + C3 * L ** 3 * r2 * u
          + 0.2 * L ** 4 * (A4x * (5 * u ** 4 + 5 * v ** 4 - 30 * u ** 2 * v ** 2) + A4y * (20 * u ** 3 * v - 20 * u * v ** 3))
          + L ** 4 * ((2 * u) * (D4x * (u ** 3 - 3 * u * v ** 2) - D4y * (3 * u ** 2 * v - v ** 3))
                      + r2 * (D4x * (3 * u ** 2 - 3 * v ** 2) - D4y * 6 * u * v))
          + L ** 4 * (2 * r2 * 2 * u * (B4x * u - B4y * v) + r2 ** 2 * B4x)
          + L ** 5 / 6 * (A5x * (4 * u ** 3 - 14 * v) * (u ** 2 - v ** 2) + A5x * (u ** 4 + v ** 4 - 14 * u * v) * 2 * u
                          - A5y * 2 * v * (3 * u ** 4 + 3 * v ** 4 - 10 * u ** 2 * v ** 2)
                          - A5y * 2 * v * u * (12 * u ** 3 - 20 * u * v ** 2))
          + L ** 5 * (2 * r2 * 2 * u * (S5x * (u ** 2 - v ** 2) - 2 * u * v * S5y) + r2 ** 2 * (2 * S5x * u - 2 * v * S5y))
          + L ** 5 / 6 * C5 * 3 * r2 ** 2 * 2 * u
          + L ** 5 * (2 * u * (D5x * (u ** 4 + v ** 4 - 6 * u ** 2 * v ** 2) - D5y * 4 * u * v * (u ** 2 - v ** 2))
                      + r2 * (D5x * (4 * u ** 3 - 12 * u * v ** 2) - D5y * (12 * u ** 2 * v - 4 * v ** 3))))
    gv = (L * (A1y * u - A1x * v)
          - A3x * L ** 2 / 3 * 6 * u * v + A3y * L ** 2 / 3 * (-3 * v ** 2 + 3 * u ** 2)
          + B2x * L * L * 2 * u * v - B2y * L * L * (u ** 2 + 3 * v ** 2)
          + 0.25 * L ** 3 * (A3x * (4 * v ** 3 - 12 * u * u * v) + A3y * (4 * u ** 3 - 12 * u * v * v))
          + L ** 3 * (2 * v * (S3x * (u * u - v * v) - S3y * 2 * u * v) + r2 * (-2 * S3x * v - 2 * S3y * u))
          + C3 * L ** 3 * r2 * v
          + 0.2 * L ** 4 * (A4x * (20 * u * v ** 3 - 20 * u ** 3 * v) + A4y * (5 * v ** 4 + 5 * u ** 4 - 30 * u ** 2 * v ** 2))
          + L ** 4 * ((2 * v) * (D4x * (u ** 3 - 3 * u * v ** 2) - D4y * (3 * u ** 2 * v - v ** 3))
                      + r2 * (-D4x * 6 * u * v - D4y * (3 * u ** 2 - 3 * v ** 2)))
          + L ** 4 * (2 * r2 * 2 * v * (B4x * u - B4y * v) - r2 ** 2 * B4y)
          + L ** 5 / 6 * (A5x * (4 * v ** 3 - 14 * u) * (u ** 2 - v ** 2) + A5x * (u ** 4 + v ** 4 - 14 * u * v) * (-2 * v)
                          - A5y * 2 * u * (3 * u ** 4 + 3 * v ** 4 - 10 * u ** 2 * v ** 2)
                          - A5y * 2 * v * u * (12 * v ** 3 - 20 * u ** 2 * v))
          + L ** 5 * (2 * r2 * 2 * v * (S5x * (u ** 2 - v ** 2) - 2 * u * v * S5y) + r2 ** 2 * (-2 * S5x * v - 2 * u * S5y))
          + L ** 5 / 6 * C5 * 3 * r2 ** 2 * 2 * v
          + L ** 5 * (2 * v * (D5x * (u ** 4 + v ** 4 - 6 * u ** 2 * v ** 2) - D5y * 4 * u * v * (u ** 2 - v ** 2))
                      + r2 * (D5x * (4 * v ** 3 - 12 * u ** 2 * v) - D5y * (4 * u ** 3 - 12 * u * v ** 2))))
    return gu, gv


def gaussian_focal_weights(mtotal: int, rms_nm: float, lam_nm: float, gmax: float):
    """Defocus step and Gaussian weights ``gfsf`` (Gaussian_focal, ToTEM_submit_v1.m:610-646).

    Returns ``(delta_nm, weights)``.  ``mtotal`` must be odd; ``mtotal == 1`` gives ``(0, [1])``.
    """
    if mtotal < 1 or mtotal % 2 == 0:
        raise ValueError("the number of focal-spread steps must be odd (Gaussian_focal's -M..M)")
    M = (mtotal - 1) // 2
    if M == 0:
        return 0.0, np.array([1.0])

    def weights(delta):
        a = np.arange(-M, M + 1) * delta
        return delta * np.exp(-a * a / (2 * rms_nm * rms_nm)) / (math.sqrt(2 * math.pi) * rms_nm)

    uu = np.arange(0.0, gmax + 1e-12, 0.01)
    fixed = np.exp(-0.5 * (math.pi * rms_nm * lam_nm) ** 2 * uu ** 4)
    cands = np.arange(0.5 * rms_nm, 2.0 * rms_nm + 1e-9, 0.1)
    errs = []
    for d in cands:
        g = weights(d)
        phase = np.exp(-1j * math.pi * lam_nm * np.arange(-M, M + 1)[:, None] * d * uu[None, :] ** 2)
        errs.append(np.max(np.abs(fixed - np.real(g @ phase))))
    errs = np.asarray(errs)
    delta = float(cands[np.flatnonzero(errs == errs.min())[0]])
    return delta, weights(delta)


@dataclass
class ProbeSpec:
    kv: float = 300.0
    semi_angle_mrad: float = 25.0      # objective / probe-forming aperture (edit_Ape)
    aberrations: Aberrations = field(default_factory=Aberrations)
    convergence_mrad: float = 0.0      # spatial-coherence semi-angle alpha (edit_Con)
    focal_spread_nm: float = 0.0       # defocus-spread rms (edit_Spr)
    focal_steps: int = 1               # mtotal


def tcc_stack(spec: ProbeSpec, n: int, sampling_a: float, with_gradient: bool = True, engine: bool = False):
    """Per-defocus transfer functions (WholeTCC2D_newTEM, ToTEM_submit_v1.m:2305-2406).

    ``with_gradient`` selects the spatial envelope with the full aberration gradient
    (the reference forces ``flag = 2`` at :2333 for both STEM and HRTEM).  ``engine`` evaluates
    the stack on the GPU (``totem_tcc_stack``, FP64) instead of in NumPy.
    Returns ``(tcc[m, n, n], gfsf[m])`` on the centred grid.
    """
    lam = wavelength_nm(spec.kv)
    samp_nm = sampling_a * 0.1
    gmax = spec.semi_angle_mrad * 0.1  # tccpara.gmax (ToTEM_submit_v1.m:2166)
    delta, gfsf = gaussian_focal_weights(spec.focal_steps, spec.focal_spread_nm, lam, gmax)
    if engine:
        from . import capi
        tcc = capi.tcc_stack(spec.aberrations, lam, n, sampling_a, spec.convergence_mrad, with_gradient,
                             spec.focal_steps, delta)
        return tcc, np.asarray(gfsf, dtype=np.float64)
    half = int(math.floor((n + 1) / 2 + 0.5))  # MATLAB round((n+1)/2)
    ax = np.arange(-half + 1, n - half + 1, dtype=np.float64) / (samp_nm * n)
    U, V = np.meshgrid(ax, ax)
    ab = spec.aberrations
    A1x, A1y = ab.xy("A1")
    wu, wv = U * lam, V * lam
    W = (np.real((A1x + 1j * A1y) * (wu - 1j * wv) ** 2) / 2
         + np.real(ab.focus * (wu + 1j * wv) * (wu - 1j * wv)) / 2
         + _residual_w(ab, U, V, lam))
    if with_gradient:
        gu0, gv0 = _gradient_w(ab, U, V, lam)
    else:
        gu0 = gv0 = 0.0
    alpha = spec.convergence_mrad * 1e-3
    out = []
    mt = spec.focal_steps
    for m in range(1, mt + 1):
        gu = gu0 + ab.focus * lam * U
        gv = gv0 + ab.focus * lam * V
        es = np.exp(-alpha * alpha * math.pi * math.pi / lam / lam * (gu ** 2 + gv ** 2))
        chi = 2 * math.pi * W / lam
        ef = np.exp(-1j * math.pi * (m - (mt + 1) / 2) * delta * (U ** 2 + V ** 2) * lam)
        out.append(es * ef * np.exp(-1j * chi))
    return np.array(out), np.asarray(gfsf, dtype=np.float64)


def aperture_mask(n: int, sampling_nm: float, k_outer: float) -> np.ndarray:
    """Hard circular aperture ``myaperture(ones, dk, dk, 0, k_outer, 0, 0, 1)`` (ToTEM_submit_v1.m:727-748)."""
    # MATLAB: uu = -round((n-1)/2) : round(n/2)-1, with round() taking halves away from zero
    uu = np.arange(-int(math.floor((n - 1) / 2 + 0.5)), int(math.floor(n / 2 + 0.5)), dtype=np.float64)
    dk = 1.0 / (sampling_nm * n)
    X, Y = np.meshgrid(uu * dk, uu * dk)
    r = np.sqrt(X * X + Y * Y)
    m = np.ones((n, n))
    m[(r < 0) | (r > k_outer)] = 0
    return m


def stem_probes(spec: ProbeSpec, n: int, sampling_a: float, engine: bool = False):
    """Normalised STEM probes, one per focal-spread step (ToTEM_submit_v1.m:800-818).

    Returns ``(probe[m, n, n] complex128, gfsf[m])``; each probe is centred (fftshift-ed) and
    has unit L2 norm.  ``engine``: transfer functions on the GPU (``tcc_stack``).
    """
    lam = wavelength_nm(spec.kv)
    tcc, gfsf = tcc_stack(spec, n, sampling_a, with_gradient=True, engine=engine)
    ap = aperture_mask(n, sampling_a * 0.1, spec.semi_angle_mrad * 0.1 * 0.01 / lam)
    probes = []
    for t in tcc:
        w = np.fft.ifft2(np.fft.ifftshift(ap * t))
        norm = math.sqrt(float(np.sum(np.abs(w) ** 2)))
        probes.append(np.fft.fftshift(w) / norm)
    return np.array(probes), gfsf
