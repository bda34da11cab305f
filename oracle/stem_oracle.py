"""FP64 CPU oracle for the STEM multislice hot path -- TEST INFRASTRUCTURE ONLY.

This module restates the reference's own CPU path (MATLAB, not runnable here) in NumPy/SciPy
FP64.  It is the checker the CUDA engine is compared against; nothing in the product imports it.
Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may call it.

Sources restated (file:line in the reference tree):

  * potential, Peng and Lobato, neutral and ionic rows, absorptive rows:
      GetPotential4AllSlice_multicore_lotabo_peng.m:25-182
  * Peng-extended correction potential:
      GetPotential4AllSlice_multicore_lotabo_peng_corr.m:13-60
  * transmission exp(i sigma V / 1000) after ifft2(ifftshift(V .* APERTURE)) * N^2:
      GetPotential4AllSlice_multicore_lotabo_peng.m:187-190
  * STEM slice loop, mid-slice and exit detectors:
      cuda_STEM_CPU_Mcore_lobato_peng.m:50-97
  * gfsf-weighted sum over defocus-spread probes: same file :62-77 (``gfsf(nn) .* ...``)

Decisions where the reference's two implementations disagree (each noted where applied):

  1. Ion rows are read at their own per-slice offsets.  The MATLAB loop indexes ion rows with
     the neutral offsets ``beg1`` (GetPotential4AllSlice_multicore_lotabo_peng.m:61,141), which
     is wrong whenever both kinds exist; the CUDA code uses the right offsets
     (cuda_source_lobato.cu:760-766).
  2. A detector weight multiplies |psi|^2 linearly, as the CUDA code does
     (cuda_source_lobato.cu:460, ``powf(hypotf(..), 2) * aper``).  The MATLAB path squares the
     weight (``abs(mywave.*APER).^2``); the two agree for the 0/1 masks ToTem builds.
  3. Mid-slice outputs follow the MATLAB rule (``find(midslice==k, 1)``, any order) and the
     gfsf sum is taken per layer.  The CUDA code needs a sorted list and its
     ``accumulate_result2`` (cuda_source_lobato.cu:1001-1015) strides the probe index by
     ``aper_num*depth*layer_len`` while the data are laid out with stride ``aper_num*depth``; the
     two agree whenever ``w_num == 1`` or ``layer_len <= 1``.
  4. The exit-wave detector uses ``ifftshift(aper)``; the ``aper2`` argument is used for the
     mid-slice detectors only, as the CUDA code does (cuda_source_lobato.cu:1342-1356, 1421).

Parity of this oracle is pinned against golden fixtures produced by this very code and by the
physics invariants in ``tests/test_oracle.py``; the reference publishes no golden vectors, its
MATLAB path cannot run here (no MATLAB runtime) and its CUDA engine is not run (it frees
uninitialised device pointers and races in its potential kernels), so at the FFT boundary the
oracle is *parity unpinned*.

HRTEM (``hrtem_exit_wave``, ``hrtem_image``) restates ToTEM_submit_v1.m:1320-1369; the incident
wave may be given (a tilted plane wave), the default is the plane wave of ones.
"""
from __future__ import annotations

import math
import os
from concurrent.futures import ProcessPoolExecutor
import multiprocessing as mp

import numpy as np
import scipy.fft as sfft


# ----------------------------------------------------------------------------------------------
# Potential
# ----------------------------------------------------------------------------------------------

def _peng(c, s2):
    """sum_i a_i exp(-b_i s^2) for rows ``c`` = [a1 b1 .. a5 b5] (broadcast over atoms)."""
    out = 0.0
    for i in range(5):
        out = out + c[:, 2 * i, None, None] * np.exp(-s2[None] * c[:, 2 * i + 1, None, None])
    return out


def _lobato(c, g2):
    """sum_i a_i (2 + b_i g^2) / (1 + b_i g^2)^2 (GetPotential4AllSlice...:111-118)."""
    out = 0.0
    for i in range(5):
        a = c[:, 2 * i, None, None]
        b = c[:, 2 * i + 1, None, None]
        out = out + a * (2 + b * g2[None]) / (1 + b * g2[None]) ** 2
    return out


def _phase(rows, kx, ky):
    return np.exp(-2j * math.pi * (kx[None] * rows[:, 0, None, None] + ky[None] * rows[:, 1, None, None]))


def _absorptive(ab, s2):
    return _peng(ab, s2)


def potential_fourier(req, chunk: int = 8) -> np.ndarray:
    """V_k(g) for every slice, before the aperture / ifftshift / IFFT (FP64)."""
    S = req.slices
    series_n, series_n_i = req.padded_series()
    kx, ky, s2 = req.kx, req.ky, req.s2
    g2 = 4 * s2
    lob = req.param == "l"
    out = np.zeros((S, req.p_height, req.p_width), dtype=np.complex128)
    beg_n = np.concatenate([[0], np.cumsum(series_n)]).astype(int)
    beg_i = np.concatenate([[0], np.cumsum(series_n_i)]).astype(int)
    for k in range(S):
        # neutral / single-kind rows (GetPotential4AllSlice...:29-57, 104-136)
        for a0 in range(beg_n[k], beg_n[k + 1], chunk):
            a1 = min(a0 + chunk, beg_n[k + 1])
            rows = req.ele_n[a0:a1]
            if lob:
                f = _lobato(rows[:, 3:13], g2) * np.exp(-s2[None] * rows[:, 13, None, None])
            else:
                f = _peng(rows[:, 3:13], s2)
            f = f.astype(np.complex128)
            if req.absorp_n is not None:
                f = f + 1j * _absorptive(req.absorp_n[a0:a1], s2)
            out[k] += req.parameter * np.sum(rows[:, 2, None, None] * f * _phase(rows, kx, ky), axis=0)
        # partly ionic rows (GetPotential4AllSlice...:59-98, 138-182), decision 1 above
        for a0 in range(beg_i[k], beg_i[k + 1], chunk):
            a1 = min(a0 + chunk, beg_i[k + 1])
            rows = req.ele_n_i[a0:a1]
            if lob:
                f = (rows[:, 3, None, None] * _lobato(rows[:, 4:14], g2)
                     + rows[:, 14, None, None] * _lobato(rows[:, 15:25], g2))
                f = f * np.exp(-s2[None] * rows[:, 25, None, None])
            else:
                f = (rows[:, 3, None, None] * _peng(rows[:, 4:14], s2)
                     + rows[:, 14, None, None] * _peng(rows[:, 15:25], s2))
            f = f.astype(np.complex128)
            if req.absorp_n_i is not None:
                f = f + 1j * _absorptive(req.absorp_n_i[a0:a1], s2)
            out[k] += req.parameter * np.sum(rows[:, 2, None, None] * f * _phase(rows, kx, ky), axis=0)
    _add_correction(req, out)
    return out


def _add_correction(req, out):
    """Peng-extended correction rows (GetPotential4AllSlice_multicore_lotabo_peng_corr.m:13-60)."""
    cim = req.corr_info_matrix
    if cim is None or len(cim) == 0:
        return
    kx, ky, s2 = req.kx, req.ky, req.s2
    for series, rows_all, ion in ((req.series_n_corr, req.ele_n_corr, False),
                                  (req.series_n_i_corr, req.ele_n_i_corr, True)):
        if series is None or rows_all is None or len(series) == 0:
            continue
        beg = np.concatenate([[0], np.cumsum(series)]).astype(int)
        for k in range(min(len(series), out.shape[0])):
            for a in range(beg[k], beg[k + 1]):
                r = rows_all[a]
                if ion:
                    m = r[4] * cim[int(r[5]) - 1] + r[6] * cim[int(r[7]) - 1]
                else:
                    m = cim[int(r[4]) - 1]
                ph = np.exp(-2j * math.pi * (kx * r[0] + ky * r[1]))
                out[k] += req.parameter * r[3] * m * np.exp(-s2 * r[2]) * ph


def transmission(req, vg: np.ndarray | None = None) -> np.ndarray:
    """T_k = exp(i sigma/1000 * ifft2(ifftshift(V_k .* APERTURE)) * N^2)  (FP64)."""
    if vg is None:
        vg = potential_fourier(req)
    n = req.p_height * req.p_width
    v = sfft.ifft2(np.fft.ifftshift(vg * req.aper_true[None], axes=(-2, -1)), axes=(-2, -1)) * n
    return np.exp(1j * v * req.sigma / 1000.0)


# ----------------------------------------------------------------------------------------------
# STEM slice loop
# ----------------------------------------------------------------------------------------------

def _item(args):
    """One (probe, scan position): slice loop and detectors (cuda_STEM_CPU_Mcore...:60-77)."""
    (psi, T, r0, c0, prop, det_exit, det_mid, layer_of_slice, L) = args
    H, W = psi.shape
    A = det_exit.shape[0]
    mid = np.zeros((L, A))
    for k in range(T.shape[0]):
        psi = psi * T[k, r0:r0 + H, c0:c0 + W]
        psi = sfft.fft2(psi)
        psi = psi * prop
        oo = layer_of_slice.get(k + 1)
        if oo is not None:
            inten = np.abs(psi) ** 2
            mid[oo] = np.tensordot(det_mid, inten, axes=([1, 2], [0, 1]))
        psi = sfft.ifft2(psi)
    psi = sfft.fft2(psi)
    inten = np.abs(psi) ** 2
    return np.tensordot(det_exit, inten, axes=([1, 2], [0, 1])), mid


_POOL_STATE = {}


def _init_pool(T):
    _POOL_STATE["T"] = T


def _item_pooled(args):
    return _item((args[0], _POOL_STATE["T"]) + tuple(args[1:]))


def stem(req, T: np.ndarray | None = None, workers: int = 1, items=None):
    """Detector images in the MEX output layout.

    Returns ``(result, mid)`` with ``result[a * depth + pos]`` and
    ``mid[(layer * A + a) * depth + pos]`` -- the layouts of ``return_result`` and
    ``mid_layer_mat`` (cuda_source_lobato.cu:1510-1546).  ``items`` optionally restricts the scan
    positions computed (the rest stay zero); it is used to time a bounded CPU sample.
    """
    if T is None:
        T = transmission(req)
    rows, cols = _origins(req)
    det_exit = np.array([np.fft.ifftshift(a) for a in req.aper])
    det_mid = req.aper2
    mids = [int(m) for m in np.asarray(req.mid_layer).ravel()]
    layer_of_slice = {}
    for idx, m in enumerate(mids):
        layer_of_slice.setdefault(m, idx)
    L = len(mids)
    A = req.aper_num
    D = req.depth
    result = np.zeros((A, D))
    mid = np.zeros((L, A, D))
    positions = range(D) if items is None else items
    jobs = []
    for w in range(req.w_num):
        for pos in positions:
            jobs.append((w, pos, (req.probe[w], int(rows[pos]), int(cols[pos]), req.prop,
                                  det_exit, det_mid, layer_of_slice, L)))
    if workers > 1:
        ctx = mp.get_context("spawn")
        with ProcessPoolExecutor(workers, mp_context=ctx, initializer=_init_pool,
                                 initargs=(T,)) as ex:
            outs = list(ex.map(_item_pooled, [j[2] for j in jobs], chunksize=1))
    else:
        outs = [_item((j[2][0], T) + j[2][1:]) for j in jobs]
    for (w, pos, _), (r, m) in zip(jobs, outs):
        result[:, pos] += req.gfsf[w] * r
        mid[:, :, pos] += req.gfsf[w] * m
    return result.reshape(-1), mid.reshape(-1)


def _origins(req):
    pos = np.arange(req.depth)
    return (req.beginrow + (pos // req.width_red) * req.step,
            req.begincol + (pos % req.width_red) * req.step)


# ----------------------------------------------------------------------------------------------
# CBED: one probe position, the whole diffraction pattern (ToTEM_submit_v1.m:1478-1492)
# ----------------------------------------------------------------------------------------------

def cbed(req, T: np.ndarray | None = None) -> np.ndarray:
    """sum_n gfsf_n |fftshift(fft2(psi_n))|^2 over the defocus probes, psi_n propagated from the
    probe window at (beginrow, begincol) through every slice: psi .* T_k window, fft2, .* psf,
    ifft2 (the loop of ToTEM_submit_v1.m:1481-1491).  Returns the [H, W] pattern, zero frequency
    at the centre."""
    if T is None:
        T = transmission(req)
    r0, c0 = int(req.beginrow), int(req.begincol)
    out = np.zeros((req.height, req.width))
    for w in range(req.w_num):
        psi = np.asarray(req.probe[w], dtype=np.complex128)
        for k in range(T.shape[0]):
            psi = psi * T[k, r0:r0 + req.height, c0:c0 + req.width]
            psi = sfft.ifft2(sfft.fft2(psi) * req.prop)
        out += req.gfsf[w] * np.abs(np.fft.fftshift(sfft.fft2(psi))) ** 2
    return out


# ----------------------------------------------------------------------------------------------
# HRTEM plane-wave multislice (ToTEM_submit_v1.m:1320-1369)
# ----------------------------------------------------------------------------------------------

def hrtem_exit_wave(T: np.ndarray, prop_half: np.ndarray, wave: np.ndarray | None = None) -> np.ndarray:
    """Plane wave through all slices on the full grid; ``prop_half`` is the 1/2-limited propagator."""
    psi = np.ones(T.shape[1:], dtype=np.complex128) if wave is None else np.asarray(wave, dtype=np.complex128)
    for k in range(T.shape[0]):
        psi = psi * T[k]
        psi = sfft.fft2(psi)
        psi = psi * prop_half
        psi = sfft.ifft2(psi)
    return psi


def hrtem_image(exit_wave: np.ndarray, tcc: np.ndarray, ap: np.ndarray, gfsf) -> np.ndarray:
    """sum_n gfsf_n |ifft2(ifftshift(fftshift(fft2(psi)) .* tcc_n .* ap))|^2 (ToTEM_submit_v1.m:1364-1369)."""
    spec = np.fft.fftshift(sfft.fft2(exit_wave))
    out = np.zeros(exit_wave.shape)
    for g, t in zip(gfsf, tcc):
        out += g * np.abs(sfft.ifft2(np.fft.ifftshift(spec * t * ap))) ** 2
    return out


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1
