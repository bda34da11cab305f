"""A STEM / transmission request in the reference's MEX argument layout.

``StemRequest`` holds exactly the inputs ``myProjectfun`` receives (waveCuda.h:10-21) after
``cuda_stem.m`` has marshalled them: every 2-D array is row-major (C order) with the MATLAB row
index first, probe/aperture stacks are ``(count, H, W)``, coefficient rows are ``(atoms, ncol)``.
``beginrow``/``begincol`` are the 0-based values ``mexFunction`` passes on (waveCuda.cpp:99).

The ``build_*`` functions create the seeded synthetic workloads used by the tests and the bench.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Optional

import numpy as np

from . import optics, specimen

PENG = "p"
LOBATO = "l"


@dataclass
class StemRequest:
    param: str                        # 'p' (Peng, 13/25-column rows) or 'l' (Lobato, 14/26)
    probe: np.ndarray                 # (w_num, H, W) complex128
    aper: np.ndarray                  # (A, H, W) float64, centred masks
    aper2: np.ndarray                 # (A, H, W) float64, ifftshift(aper) (cuda_stem.m:34-39)
    ele_n: np.ndarray                 # (n, 13|14)
    series_n: np.ndarray              # (S,) float64 atom counts per slice
    ele_n_i: np.ndarray               # (m, 25|26)
    series_n_i: np.ndarray            # (S,)
    kx: np.ndarray                    # (P_H, P_W)
    ky: np.ndarray
    s2: np.ndarray
    prop: np.ndarray                  # (H, W) complex128, natural FFT order
    gfsf: np.ndarray                  # (w_num,)
    p_height: int
    p_width: int
    step: int
    beginrow: int                     # 0-based
    begincol: int
    width_red: int
    hight_red: int
    sigma: float
    parameter: float
    aper_true: np.ndarray             # (P_H, P_W)
    mid_layer: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int32))  # 1-based
    absorp_n: Optional[np.ndarray] = None      # (n, 10)
    absorp_n_i: Optional[np.ndarray] = None    # (m, 10)
    series_n_corr: Optional[np.ndarray] = None
    series_n_i_corr: Optional[np.ndarray] = None
    ele_n_corr: Optional[np.ndarray] = None    # (k, 5)
    ele_n_i_corr: Optional[np.ndarray] = None  # (k, 8)
    corr_info_matrix: Optional[np.ndarray] = None  # (cim_len, P_H, P_W)

    @property
    def height(self) -> int:
        return self.probe.shape[1]

    @property
    def width(self) -> int:
        return self.probe.shape[2]

    @property
    def depth(self) -> int:
        return self.width_red * self.hight_red

    @property
    def slices(self) -> int:
        return max(len(self.series_n), len(self.series_n_i))

    @property
    def w_num(self) -> int:
        return self.probe.shape[0]

    @property
    def aper_num(self) -> int:
        return self.aper.shape[0]

    @property
    def probe_slices(self) -> int:
        """Units of work: probes x defocus-spread probes x slices."""
        return self.depth * self.w_num * self.slices

    def padded_series(self):
        """Per-slice counts padded with zeros to ``slices`` entries (cuda_stem.m:1-21)."""
        S = self.slices

        def pad(a):
            out = np.zeros(S)
            if a is not None and len(a):
                out[: len(a)] = a
            return out
        return pad(self.series_n), pad(self.series_n_i)


def window_origins(req: StemRequest):
    """Top-left corner (row, col) of each probe window on the potential grid.

    ``pos`` runs row-major over the scan: row ``pos // width_red``, column ``pos % width_red``
    (cuda_source_lobato.cu:344-345).
    """
    pos = np.arange(req.depth)
    rows = req.beginrow + (pos // req.width_red) * req.step
    cols = req.begincol + (pos % req.width_red) * req.step
    return rows, cols


def validate(req: StemRequest):
    r, c = window_origins(req)
    if req.depth and (r.max() + req.height > req.p_height or c.max() + req.width > req.p_width
                      or r.min() < 0 or c.min() < 0):
        raise ValueError("probe windows leave the potential grid")


# ----------------------------------------------------------------------------------------------
# Workload builders
# ----------------------------------------------------------------------------------------------

def _stem_request(structure: specimen.Structure, flag: str, kv: float, sampling: float, n: int,
                  p: int, step: int, raster: tuple, begin: tuple, detectors_mrad, probe_spec,
                  mid_layer=(), dbmode: int = 0, multiceng: int = 0, engine_optics: bool = False,
                  optics_from: Optional[StemRequest] = None, native_slicing: bool = False) -> StemRequest:
    nuc, ion = specimen.potential_params(structure.atoms, flag)
    if native_slicing:  # the library's slicer (totem_slice_rows): same rows, O(atoms) instead of O(atoms x slices)
        from . import capi
        ele_n, ele_n_i, series_n, series_n_i = capi.slice_rows(
            nuc, ion, structure.slice_dz, structure.slicethick, multiceng, flag, dbmode)
    else:
        ele_n, ele_n_i, series_n, series_n_i = specimen.slice_rows(
            nuc, ion, structure.slice_dz, structure.slicethick, multiceng, flag, dbmode)
    kx, ky, s2 = optics.reciprocal_grids(p, p, sampling)
    if optics_from is not None:  # same probe, detectors and propagator (e.g. another phonon configuration)
        probe, gfsf, aper, aper2, prop = (optics_from.probe, optics_from.gfsf, optics_from.aper, optics_from.aper2,
                                          optics_from.prop)
    else:
        probe, gfsf = optics.stem_probes(probe_spec, n, sampling, engine=engine_optics)
        aper = optics.annular_detectors(n, sampling, kv, detectors_mrad)
        aper2 = np.array([np.fft.ifftshift(a) for a in aper])
        prop = optics.propagator(n, sampling, kv, structure.slice_dz, "2/3")
    S = structure.n_slices
    return StemRequest(
        param=flag, probe=probe, aper=aper, aper2=aper2,
        ele_n=ele_n, series_n=series_n if len(series_n) else np.zeros(S),
        ele_n_i=ele_n_i, series_n_i=series_n_i if len(series_n_i) else np.zeros(S),
        kx=kx, ky=ky, s2=s2, prop=prop, gfsf=gfsf, p_height=p, p_width=p, step=step,
        beginrow=begin[0], begincol=begin[1], width_red=raster[1], hight_red=raster[0],
        sigma=optics.interaction_sigma(kv), parameter=optics.potential_parameter(p, p, sampling),
        aper_true=np.ones((p, p)), mid_layer=np.asarray(mid_layer, dtype=np.int32))


def build_srtio3_stem(cells=(8, 8, 50), n: int = 512, sampling: float = 0.0625, step: int = 8,
                      raster=(64, 64), p: Optional[int] = None, flag: str = PENG, kv: float = 300.0,
                      semi_angle: float = 25.0, c3_um: float = -5.0, defocus_nm: float = 0.0,
                      detectors=((60.0, 200.0), (0.0, 10.0)), mid_layer=(),
                      phonon_seed: Optional[int] = None, rms=None, engine_optics: bool = False,
                      optics_from: Optional[StemRequest] = None, native_slicing: bool = False) -> StemRequest:
    """The SrTiO3 [001] STEM-ADF workload (8x8x50 cells, Peng, 300 kV, 512^2 window).

    The potential grid holds the scan plus one window: ``p = n + (raster-1)*step`` rounded up to a
    power of two, the block centred in it.  ``phonon_seed`` displaces atoms with per-element rms
    (Sr 0.089, Ti 0.075, O 0.088 Angstrom by default) drawn from ``numpy.random.default_rng(seed)``.
    ``engine_optics`` forms the probe's transfer functions on the GPU; ``optics_from`` reuses the
    probe, detectors and propagator of an earlier request of the same optics; ``native_slicing``
    slices with the library (``totem_slice_rows``) instead of NumPy.
    """
    need = n + (max(raster) - 1) * step
    if p is None:
        p = 1 << (need - 1).bit_length()
    begin = ((p - (n + (raster[0] - 1) * step)) // 2, (p - (n + (raster[1] - 1) * step)) // 2)
    rms = rms or {38: 0.089, 22: 0.075, 8: 0.088}
    dw = {z: specimen.b_from_rms(r) for z, r in rms.items()} if phonon_seed is not None else None
    st = specimen.srtio3_001(*cells, dw=dw)
    st = specimen.center_in_field(st, p * sampling, p * sampling)
    spec = optics.ProbeSpec(kv=kv, semi_angle_mrad=semi_angle,
                            aberrations=optics.Aberrations(focus=defocus_nm, Cs=c3_um * 1e3))
    if phonon_seed is not None:
        nuc, ion = specimen.potential_params(st.atoms, flag)
        rng = np.random.default_rng(phonon_seed)
        moved = specimen.frozen_phonon(nuc, st.slice_dz, st.slicethick, rng)
        atoms = st.atoms.copy()
        atoms[:, 1:4] = moved[:, 1:4]
        st = specimen.Structure(atoms, st.extent, st.slice_dz, st.n_slices)
    return _stem_request(st, flag, kv, sampling, n, p, step, raster, begin, detectors, spec,
                         mid_layer=mid_layer, engine_optics=engine_optics, optics_from=optics_from,
                         native_slicing=native_slicing)


def build_stem_on_structure(st: specimen.Structure, n: int = 512, sampling: float = 0.0625, step: int = 8,
                            raster=(64, 64), p: Optional[int] = None, flag: str = PENG, kv: float = 300.0,
                            semi_angle: float = 25.0, c3_um: float = -5.0, defocus_nm: float = 0.0,
                            detectors=((60.0, 200.0), (0.0, 10.0)), mid_layer=(),
                            native_slicing: bool = False, engine_optics: bool = False) -> StemRequest:
    """The STEM-ADF probe, detectors and scan of ``build_srtio3_stem`` on any specimen, centred
    on a potential grid of ``p`` (default: the scan plus one window, rounded up to a power of two)."""
    need = n + (max(raster) - 1) * step
    if p is None:
        p = 1 << (need - 1).bit_length()
    begin = ((p - (n + (raster[0] - 1) * step)) // 2, (p - (n + (raster[1] - 1) * step)) // 2)
    st = specimen.center_in_field(st, p * sampling, p * sampling)
    spec = optics.ProbeSpec(kv=kv, semi_angle_mrad=semi_angle,
                            aberrations=optics.Aberrations(focus=defocus_nm, Cs=c3_um * 1e3))
    return _stem_request(st, flag, kv, sampling, n, p, step, raster, begin, detectors, spec, mid_layer=mid_layer,
                         native_slicing=native_slicing, engine_optics=engine_optics)


def build_stem_from_table(atoms, eachthick: float, slicethick, n: int = 128, p: int = 256, sampling: float = 0.15,
                          step: int = 16, raster=(3, 3), flag: str = PENG, kv: float = 300.0,
                          semi_angle: float = 25.0, c3_um: float = -5.0, defocus_nm: float = 0.0,
                          detectors=((60.0, 200.0), (0.0, 10.0)), mid_layer=(), multiceng: int = 0,
                          native_slicing: bool = False) -> StemRequest:
    """A STEM request on a specimen given as ToTem's atom table (``allresul.x_new``: one row per
    atom ``Z x y z valence ionic-fraction B occupancy``, Angstrom) with its slicing (``eachthick``
    and the slice tops ``slicethick``, slicingdisplay.m:228-254), at the coordinates given (not
    re-centred).  The scan is centred on the ``p`` x ``p`` potential grid."""
    atoms = np.asarray(atoms, dtype=np.float64)
    slicethick = np.asarray(slicethick, dtype=np.float64)
    if not np.array_equal(slicethick, np.arange(len(slicethick)) * eachthick):
        raise ValueError("slice tops must be 0, eachthick, 2 eachthick, ... (as ToTem's slicing dialog writes them)")
    extent = tuple(float(v) for v in atoms[:, 1:4].max(axis=0)) if len(atoms) else (0.0, 0.0, 0.0)
    st = specimen.Structure(atoms, extent, float(eachthick), len(slicethick))
    spec = optics.ProbeSpec(kv=kv, semi_angle_mrad=semi_angle,
                            aberrations=optics.Aberrations(focus=defocus_nm, Cs=c3_um * 1e3))
    begin = ((p - (n + (raster[0] - 1) * step)) // 2, (p - (n + (raster[1] - 1) * step)) // 2)
    req = _stem_request(st, flag, kv, sampling, n, p, step, raster, begin, detectors, spec, mid_layer=mid_layer,
                        multiceng=multiceng, native_slicing=native_slicing)
    return req


def build_small_stem(n: int = 64, p: int = 128, raster=(3, 4), step: int = 5, slices: int = 6,
                     flag: str = PENG, kv: float = 200.0, sampling: float = 0.2,
                     detectors=((40.0, 150.0), (0.0, 15.0), (15.0, 40.0)), mid_layer=(2, 4),
                     focal_steps: int = 1, begin=None, seed: int = 0, cells: Optional[int] = None) -> StemRequest:
    """A small SrTiO3 case the FP64 oracle finishes in seconds (used by the parity tests).

    ``cells`` limits the crystal to ``cells x cells`` unit cells (default: fill the field).
    """
    a = 3.905
    field = p * sampling
    ncell = max(1, int(field // a) - 1) if cells is None else cells
    st = specimen.srtio3_001(ncell, ncell, max(1, slices // 2))
    st = specimen.center_in_field(st, field, field)
    st = specimen.Structure(st.atoms, st.extent, st.slice_dz, slices)
    rng = np.random.default_rng(seed)
    st.atoms[:, 1:3] += rng.uniform(-0.05, 0.05, size=(len(st.atoms), 2))
    spec = optics.ProbeSpec(kv=kv, semi_angle_mrad=20.0,
                            aberrations=optics.Aberrations(focus=-5.0, Cs=-2e3),
                            focal_spread_nm=3.0 if focal_steps > 1 else 0.0,
                            focal_steps=focal_steps)
    if begin is None:
        begin = ((p - (n + (raster[0] - 1) * step)) // 2, (p - (n + (raster[1] - 1) * step)) // 2)
    return _stem_request(st, flag, kv, sampling, n, p, step, raster, begin, detectors, spec,
                         mid_layer=mid_layer)


def with_absorption(req: StemRequest, seed: int = 1, scale: float = 0.05) -> StemRequest:
    """Attach synthetic absorptive coefficient rows (10 per atom) to a request (tests only)."""
    rng = np.random.default_rng(seed)

    def rows(n):
        c = np.empty((n, 10))
        c[:, 0::2] = rng.uniform(0.0, scale, size=(n, 5))
        c[:, 1::2] = rng.uniform(0.5, 20.0, size=(n, 5))
        return c
    return replace(req, absorp_n=rows(len(req.ele_n)) if len(req.ele_n) else None,
                   absorp_n_i=rows(len(req.ele_n_i)) if len(req.ele_n_i) else None)


def with_ionic_oxygen(req: StemRequest, every: int = 3, ion_fraction: float = 0.4) -> StemRequest:
    """Move every ``every``-th neutral row to the ionic table as partly ionised O (O2-: the ion
    fraction from the ionic Peng table, the rest neutral O), keeping per-slice counts (tests;
    Peng requests only)."""
    o2 = specimen.ion_params(8, -2)
    neutral_o = specimen.element_params(8, "p")
    rows = req.ele_n
    n = len(rows)
    ion_idx = np.arange(0, n, every)
    ion_rows = np.zeros((len(ion_idx), 25))
    ion_rows[:, 0:3] = rows[ion_idx, 0:3]
    ion_rows[:, 3] = ion_fraction
    ion_rows[:, 4:14:2], ion_rows[:, 5:14:2] = o2[:5], o2[5:]
    ion_rows[:, 14] = 1.0 - ion_fraction
    ion_rows[:, 15:25:2], ion_rows[:, 16:25:2] = neutral_o[:5], neutral_o[5:]
    keep = np.setdiff1d(np.arange(n), ion_idx)
    beg = np.concatenate([[0], np.cumsum(req.series_n)]).astype(int)
    sl = np.searchsorted(beg, np.arange(n), side="right") - 1
    series_n = np.bincount(sl[keep], minlength=req.slices).astype(float)
    series_i = np.bincount(sl[ion_idx], minlength=req.slices).astype(float)
    return replace(req, ele_n=rows[keep], series_n=series_n, ele_n_i=ion_rows, series_n_i=series_i)


def with_correction(req: StemRequest, seed: int = 2, every: int = 4, per_element: bool = False) -> StemRequest:
    """Attach synthetic Peng-extended correction rows to a request (tests only): two correction
    planes (cim) on the potential grid, a neutral row (x, y, B, amplitude, plane) at every
    ``every``-th atom and an ionic row (x, y, B, amplitude, w1, plane1, w2, plane2) at every
    ``2 every``-th, keeping the atoms' slices.  The values are drawn per row, or with
    ``per_element`` once per distinct coefficient row (element), as ToTem's rows are."""
    rng = np.random.default_rng(seed)
    if per_element:
        elem = np.unique(req.ele_n[:, 3:13], axis=0, return_inverse=True)[1].reshape(-1)
        ne = int(elem.max()) + 1 if len(elem) else 0
        table_n = [[rng.uniform(0.5, 5.0), rng.uniform(0.1, 1.0), 1 + e % 2] for e in range(ne)]
        table_i = [[rng.uniform(0.5, 5.0), rng.uniform(0.1, 1.0), rng.uniform(0, 1), 1, rng.uniform(0, 1), 2]
                   for _ in range(ne)]
    cim = np.stack([np.exp(-req.s2 * rng.uniform(0.5, 3.0)) * rng.uniform(0.5, 1.5, size=req.s2.shape)
                    for _ in range(2)])
    beg = np.concatenate([[0], np.cumsum(req.series_n)]).astype(int)
    n_rows, i_rows, n_cnt, i_cnt = [], [], np.zeros(req.slices), np.zeros(req.slices)
    for k in range(req.slices):
        for a in range(beg[k], beg[k + 1]):
            x, y = req.ele_n[a, 0], req.ele_n[a, 1]
            if a % every == 0:
                n_rows.append([x, y] + (table_n[elem[a]] if per_element else
                                        [rng.uniform(0.5, 5.0), rng.uniform(0.1, 1.0), 1 + a % 2]))
                n_cnt[k] += 1
            if a % (2 * every) == 1:
                i_rows.append([x, y] + (table_i[elem[a]] if per_element else
                                        [rng.uniform(0.5, 5.0), rng.uniform(0.1, 1.0), rng.uniform(0, 1), 1,
                                         rng.uniform(0, 1), 2]))
                i_cnt[k] += 1
    return replace(req, corr_info_matrix=cim, series_n_corr=n_cnt, series_n_i_corr=i_cnt,
                   ele_n_corr=np.asarray(n_rows, dtype=float).reshape(-1, 5),
                   ele_n_i_corr=np.asarray(i_rows, dtype=float).reshape(-1, 8))


def without_slice_atoms(req: StemRequest, slices) -> StemRequest:
    """The request with every atom of the given 0-based slices removed (vacuum slices; tests)."""
    drop = set(int(s) for s in slices)

    def cut(rows, counts, extra):
        if rows is None or len(rows) == 0:
            return rows, counts, extra
        beg = np.concatenate([[0], np.cumsum(counts)]).astype(int)
        keep = np.concatenate([np.arange(beg[s], beg[s + 1]) for s in range(len(counts)) if s not in drop]
                              + [np.zeros(0, dtype=int)]).astype(int)
        c = np.array([0.0 if s in drop else counts[s] for s in range(len(counts))])
        return rows[keep], c, (extra[keep] if extra is not None else None)
    ele_n, series_n, absorp_n = cut(req.ele_n, req.series_n, req.absorp_n)
    ele_n_i, series_n_i, absorp_n_i = cut(req.ele_n_i, req.series_n_i, req.absorp_n_i)
    return replace(req, ele_n=ele_n, series_n=series_n, absorp_n=absorp_n, ele_n_i=ele_n_i,
                   series_n_i=series_n_i, absorp_n_i=absorp_n_i)


# ----------------------------------------------------------------------------------------------
# HRTEM (the reference's HRTEMsimulation: *P transmission, then plane-wave multislice and TCC
# imaging in MATLAB, ToTEM_submit_v1.m:1259-1369)
# ----------------------------------------------------------------------------------------------

@dataclass
class HrtemSpec:
    """Inputs of the HRTEM step after the transmission."""
    prop: np.ndarray                       # (P, P) complex psf_fft, FFT order
    wave: Optional[np.ndarray] = None      # (P, P) incident wave; None = plane wave of ones
    tf: Optional[np.ndarray] = None        # (K, P, P) complex, FFT order: ifftshift(tcc_k .* aperture)
    weights: Optional[np.ndarray] = None   # (K,) gfsf


def specimen_request(structure: specimen.Structure, flag: str, kv: float, sampling: float, p: int) -> StemRequest:
    """Transmission-only request (the ``*P`` MEX inputs) of ``structure`` on a p x p grid."""
    nuc, ion = specimen.potential_params(structure.atoms, flag)
    ele_n, ele_n_i, series_n, series_n_i = specimen.slice_rows(
        nuc, ion, structure.slice_dz, structure.slicethick, 0, flag, 0)
    kx, ky, s2 = optics.reciprocal_grids(p, p, sampling)
    S = structure.n_slices
    return StemRequest(
        param=flag, probe=np.zeros((1, 2, 2), dtype=np.complex128), aper=np.zeros((0, 2, 2)),
        aper2=np.zeros((0, 2, 2)), ele_n=ele_n, series_n=series_n if len(series_n) else np.zeros(S),
        ele_n_i=ele_n_i, series_n_i=series_n_i if len(series_n_i) else np.zeros(S),
        kx=kx, ky=ky, s2=s2, prop=np.zeros((2, 2), dtype=np.complex128), gfsf=np.ones(1),
        p_height=p, p_width=p, step=0, beginrow=0, begincol=0, width_red=0, hight_red=0,
        sigma=optics.interaction_sigma(kv), parameter=optics.potential_parameter(p, p, sampling),
        aper_true=np.ones((p, p)))


def hrtem_spec(p: int, sampling: float, kv: float, dz: float, defocus_nm: float = 0.0, cs_mm: float = 0.0,
               aperture_mrad: Optional[float] = None, focal_spread_nm: float = 0.0, focal_steps: int = 1,
               image: bool = True) -> HrtemSpec:
    """Propagator with the HRTEM half-Nyquist limit (ToTEM_submit_v1.m:1330-1334) and, for the
    image, the transfer functions tf_k = ifftshift(tcc_k .* aperture) with their Gaussian focal
    weights (WholeTCC2D_newTEM, Gaussian_focal)."""
    prop = optics.propagator(p, sampling, kv, dz, "1/2")
    if not image:
        return HrtemSpec(prop=prop)
    spec = optics.ProbeSpec(kv=kv, semi_angle_mrad=aperture_mrad or 100.0,
                            aberrations=optics.Aberrations(focus=defocus_nm, Cs=cs_mm * 1e6),
                            focal_spread_nm=focal_spread_nm, focal_steps=focal_steps)
    tcc, w = optics.tcc_stack(spec, p, sampling)
    ap = np.ones((p, p))
    if aperture_mrad:
        lam_a = optics.wavelength_nm(kv) * 10
        ap = optics.aperture_mask(p, sampling, aperture_mrad * 1e-3 / lam_a)
    tf = np.fft.ifftshift(tcc * ap, axes=(-2, -1))
    return HrtemSpec(prop=prop, tf=tf, weights=np.asarray(w, dtype=np.float64))


def build_si_hrtem_001(cells=(4, 4, 20), p: int = 256, kv: float = 200.0, flag: str = LOBATO,
                       defocus_nm: float = -50.0, cs_mm: float = 1.2, aperture_mrad: float = 20.0,
                       slices: Optional[int] = None):
    """Si diamond [001], 4 x 4 x 20 cells, 256^2 (0.08486 Angstrom), 80 slices of 1.358
    Angstrom, Lobato, 200 kV, plane wave; image with Cs 1.2 mm, defocus -50 nm, 20 mrad.
    ``slices`` keeps only the first slices (small test cases).  Returns (specimen, HrtemSpec)."""
    st = specimen.si_001(*cells)
    if slices is not None:
        st = specimen.Structure(st.atoms, st.extent, st.slice_dz, slices)
    sampling = st.extent[0] / p
    req = specimen_request(st, flag, kv, sampling, p)
    return req, hrtem_spec(p, sampling, kv, st.slice_dz, defocus_nm, cs_mm, aperture_mrad)


def build_si_hrtem_110(repeats: int = 520, p: int = 1024, sampling: float = 0.05, kv: float = 200.0,
                       flag: str = LOBATO, defocus_nm: float = -50.0, cs_mm: float = 1.2,
                       aperture_mrad: float = 20.0, focal_spread_nm: float = 4.0, focal_steps: int = 11):
    """Si [110], ``repeats`` slices of a/sqrt2 (520: 200 nm), centred on a p x p grid; the image
    over ``focal_steps`` Gaussian-weighted defoci of rms ``focal_spread_nm``."""
    a = 5.431
    field = p * sampling
    nx, ny = max(1, int(field // a) - 1), max(1, int(field // (a / math.sqrt(2))) - 1)
    st = specimen.center_in_field(specimen.si_110(nx, ny, repeats), field, field)
    req = specimen_request(st, flag, kv, sampling, p)
    return req, hrtem_spec(p, sampling, kv, st.slice_dz, defocus_nm, cs_mm, aperture_mrad, focal_spread_nm,
                           focal_steps)

