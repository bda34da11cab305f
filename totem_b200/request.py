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
                  mid_layer=(), dbmode: int = 0, multiceng: int = 0) -> StemRequest:
    nuc, ion = specimen.potential_params(structure.atoms, flag)
    ele_n, ele_n_i, series_n, series_n_i = specimen.slice_rows(
        nuc, ion, structure.slice_dz, structure.slicethick, multiceng, flag, dbmode)
    kx, ky, s2 = optics.reciprocal_grids(p, p, sampling)
    probe, gfsf = optics.stem_probes(probe_spec, n, sampling)
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
                      phonon_seed: Optional[int] = None, rms=None) -> StemRequest:
    """The SrTiO3 [001] STEM-ADF workload (8x8x50 cells, Peng, 300 kV, 512^2 window).

    The potential grid holds the scan plus one window: ``p = n + (raster-1)*step`` rounded up to a
    power of two, the block centred in it.  ``phonon_seed`` displaces atoms with per-element rms
    (Sr 0.089, Ti 0.075, O 0.088 Angstrom by default) drawn from ``numpy.random.default_rng(seed)``.
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
                         mid_layer=mid_layer)


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
