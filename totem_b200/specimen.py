"""Specimen preparation: crystal builders, scattering-parameter rows, slicing, frozen phonons.

This is the host-side code that turns an atom list into the per-slice coefficient rows the
multislice engine consumes.  It restates, in NumPy:

  * ``getpotentialpara_lotabo_peng.m:1-86``        -> :func:`potential_params`
  * ``CommonPart_forsimulation_lobato_peng.m:88-116`` (Debye-Waller folded into Peng b) ->
    :func:`fold_debye_waller`
  * ``CalAllEquilent20210223_lobato_peng.m:23-228`` -> :func:`slice_rows`
  * ``randshiftpos.m:1-44`` (seeded instead of ``rng('shuffle')``) -> :func:`frozen_phonon`

Atom-table columns (``getpotentialpara_lotabo_peng.m:13-14``)::

    0 Z | 1 x | 2 y | 3 z | 4 valence | 5 ion fraction | 6 Debye-Waller B | 7 occupancy

Coefficient-row layouts produced for the engine (``CalAllEquilent20210223_lobato_peng.m:80-98``):

  * neutral Peng, 13 columns:  ``x y occ a1 b1 a2 b2 a3 b3 a4 b4 a5 b5``
  * neutral Lobato, 14 columns: the same followed by ``B * DBmode``
  * ion Peng, 25 columns: ``x y occ f_ion a1..b5(ion) f_atom a1..b5(atom)``
  * ion Lobato, 26 columns: the same followed by ``B * DBmode``
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np
from scipy.special import erf

_TABLES = None


def tables():
    """Scattering-factor tables parsed from the reference (see ``data/extract_tables.py``)."""
    global _TABLES
    if _TABLES is None:
        path = os.path.join(os.path.dirname(__file__), "data", "scattering_tables.npz")
        d = np.load(path)
        _TABLES = {k: d[k] for k in d.files}
    return _TABLES


def element_params(z: int, flag: str) -> np.ndarray:
    """``a1..a5 b1..b5`` for element ``z`` ('p'/'n' = Peng, 'l' = Lobato)."""
    t = tables()["lobato" if flag == "l" else "peng"]
    return t[int(z) - 1]


def ion_params(z: int, valence: int) -> np.ndarray:
    ions = tables()["peng_ion"]
    k = np.flatnonzero((ions[:, 0] == z) & (ions[:, 1] == valence))
    if k.size == 0:
        raise KeyError(f"no Peng ion parameters for Z={z} valence={valence}")
    return ions[k[0], 2:]


def _interleave(p: np.ndarray) -> np.ndarray:
    """a1..a5 b1..b5 -> a1 b1 a2 b2 ... a5 b5 (getpotentialpara_lotabo_peng.m:34-37)."""
    p = np.atleast_2d(p)
    out = np.empty_like(p)
    out[:, 0::2] = p[:, :5]
    out[:, 1::2] = p[:, 5:]
    return out


# ----------------------------------------------------------------------------------------------
# Crystal builders
# ----------------------------------------------------------------------------------------------

@dataclass
class Structure:
    atoms: np.ndarray          # (n, 8) atom table
    extent: tuple              # (lx, ly, lz) in Angstrom of the built block
    slice_dz: float            # slice thickness ("eachthick")
    n_slices: int

    @property
    def slicethick(self) -> np.ndarray:
        """Top of every slice (``allresul.slicethick``)."""
        return np.arange(self.n_slices, dtype=np.float64) * self.slice_dz


def _tile(basis, cell, reps):
    """Replicate a fractional basis [(Z, fx, fy, fz)] over ``reps`` cells of size ``cell``: rows
    ordered by cell z, then y, then x, then basis atom, with coordinates (i + fx) * ax etc."""
    nx, ny, nz = reps
    ax, ay, az = cell
    b = np.asarray(basis, dtype=np.float64)
    k, j, i = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                          np.arange(nx, dtype=np.float64), indexing="ij")
    out = np.empty((nz, ny, nx, len(b), 4))
    out[..., 0] = b[:, 0]
    out[..., 1] = (i[..., None] + b[:, 1]) * ax
    out[..., 2] = (j[..., None] + b[:, 2]) * ay
    out[..., 3] = (k[..., None] + b[:, 3]) * az
    return out.reshape(-1, 4)


def _table(zxyz, dw=None, occ=1.0, z_shift=0.0):
    """Atom table from (Z, x, y, z) rows.

    ``z_shift`` moves every atom off the slice boundaries (a quarter slice in the builders): an
    atom exactly on a boundary can otherwise land in two slices, because the slicing test
    ``top <= z < top + dz`` (CalAllEquilent20210223_lobato_peng.m:24) compares sums that round
    differently.
    """
    n = zxyz.shape[0]
    x = np.zeros((n, 8))
    x[:, 0:4] = zxyz
    x[:, 3] += z_shift
    x[:, 7] = occ
    if dw is not None:
        x[:, 6] = [dw.get(int(z), 0.0) for z in zxyz[:, 0]]
    return x


SRTIO3_BASIS = [(38, 0.0, 0.0, 0.0), (8, 0.5, 0.5, 0.0),
                (22, 0.5, 0.5, 0.5), (8, 0.5, 0.0, 0.5), (8, 0.0, 0.5, 0.5)]


def srtio3_001(nx: int, ny: int, nz: int, a: float = 3.905, slices_per_cell: int = 2,
               dw=None) -> Structure:
    """SrTiO3 perovskite viewed along [001]: SrO and TiO2 planes, ``slices_per_cell`` per cell."""
    zxyz = _tile(SRTIO3_BASIS, (a, a, a), (nx, ny, nz))
    dz = a / slices_per_cell
    return Structure(_table(zxyz, dw, z_shift=0.25 * dz), (nx * a, ny * a, nz * a), dz,
                     nz * slices_per_cell)


def _diamond_basis():
    fcc = [(0, 0, 0), (0, 0.5, 0.5), (0.5, 0, 0.5), (0.5, 0.5, 0)]
    out = []
    for f in fcc:
        out.append((14,) + f)
        out.append((14, f[0] + 0.25, f[1] + 0.25, f[2] + 0.25))
    return out


def si_001(nx: int, ny: int, nz: int, a: float = 5.431, slices_per_cell: int = 4,
           dw=None) -> Structure:
    """Diamond-cubic Si along [001]; 4 slices per cell puts each atomic plane in its own slice."""
    zxyz = _tile(_diamond_basis(), (a, a, a), (nx, ny, nz))
    dz = a / slices_per_cell
    return Structure(_table(zxyz, dw, z_shift=0.25 * dz), (nx * a, ny * a, nz * a), dz,
                     nz * slices_per_cell)


def si_110(nx: int, ny: int, nz: int, a: float = 5.431, slices_per_repeat: int = 1,
           dw=None) -> Structure:
    """Si viewed along [110]: orthogonal cell (a, a/sqrt2, a/sqrt2) with x=[001], y=[1-10], z=[110].

    ``nz`` counts [110] repeats of a/sqrt(2) (3.840 Angstrom).
    """
    b = a / math.sqrt(2)
    cart = []
    for zz, fx, fy, fz in _diamond_basis():
        # conventional cubic -> rotated frame: X=[001], Y=[1-10]/sqrt2, Z=[110]/sqrt2
        cx, cy, cz = fx * a, fy * a, fz * a
        cart.append((cz, (cx - cy) / math.sqrt(2), (cx + cy) / math.sqrt(2)))
    cart = np.array(cart)
    cell = np.array([a, b, b])
    frac = np.mod(cart / cell, 1.0)
    frac = np.round(frac * 1e9) / 1e9 % 1.0
    uniq = np.unique(frac, axis=0)
    basis = [(14, f[0], f[1], f[2]) for f in uniq]
    zxyz = _tile(basis, (a, b, b), (nx, ny, nz))
    dz = b / slices_per_repeat
    return Structure(_table(zxyz, dw, z_shift=0.25 * dz / slices_per_repeat), (nx * a, ny * b, nz * b), dz,
                     nz * slices_per_repeat)


def center_in_field(st: Structure, field_x: float, field_y: float) -> Structure:
    """Shift the block so it sits in the middle of a ``field_x`` x ``field_y`` potential grid."""
    x = st.atoms.copy()
    x[:, 1] += (field_x - st.extent[0]) / 2
    x[:, 2] += (field_y - st.extent[1]) / 2
    return Structure(x, st.extent, st.slice_dz, st.n_slices)


# ----------------------------------------------------------------------------------------------
# Parameter rows (getpotentialpara_lotabo_peng.m)
# ----------------------------------------------------------------------------------------------

def _per_species(keys: np.ndarray, rowfn) -> np.ndarray:
    """rowfn(key) for every row of ``keys`` (Z, or Z and valence), evaluated once per distinct key."""
    uniq, inv = np.unique(keys, axis=0, return_inverse=True)
    return np.array([rowfn(u) for u in uniq])[inv.reshape(-1)]


def potential_params(x: np.ndarray, flag: str):
    """Split atoms into the 16-column "nuclear" table and the 28-column "partly ionic" table.

    16 columns: ``Z x y z B occ a1 b1 .. a5 b5`` (neutral atoms, and fully ionised atoms with
    the Peng ion parameters).  28 columns: ``Z x y z B occ f_ion ion(a1 b1..a5 b5) f_atom
    atom(a1 b1..a5 b5)`` (getpotentialpara_lotabo_peng.m:26-84).
    """
    x = np.asarray(x, dtype=np.float64)
    nuc = []
    neutral = x[x[:, 5] == 0]
    if len(neutral):
        t = np.zeros((len(neutral), 16))
        t[:, 0] = neutral[:, 0]
        t[:, 1:4] = neutral[:, 1:4]
        t[:, 4] = neutral[:, 6]
        t[:, 5] = neutral[:, 7] * (1 - neutral[:, 5])
        t[:, 6:16] = _per_species(neutral[:, 0], lambda z: _interleave(element_params(int(z), flag))[0])
        nuc.append(t)
    full = x[x[:, 5] == 1]
    if len(full):
        t = np.zeros((len(full), 16))
        t[:, 0] = full[:, 0]
        t[:, 1:4] = full[:, 1:4]
        t[:, 4] = full[:, 6]
        t[:, 5] = full[:, 7] * full[:, 5]
        t[:, 6:16] = _per_species(full[:, [0, 4]], lambda zv: _interleave(ion_params(int(zv[0]), int(zv[1])))[0])
        nuc.append(t)
    all_nuclear = np.concatenate(nuc) if nuc else np.zeros((0, 16))
    part = x[(x[:, 5] > 0) & (x[:, 5] < 1)]
    if len(part):
        t = np.zeros((len(part), 28))
        t[:, 0] = part[:, 0]
        t[:, 1:4] = part[:, 1:4]
        t[:, 4] = part[:, 6]
        t[:, 5] = part[:, 7]
        t[:, 6] = part[:, 5]
        t[:, 7:17] = _per_species(part[:, [0, 4]], lambda zv: _interleave(ion_params(int(zv[0]), int(zv[1])))[0])
        t[:, 17] = 1 - part[:, 5]
        t[:, 18:28] = _per_species(part[:, 0], lambda z: _interleave(element_params(int(z), flag))[0])
        all_nuc_ion = t
    else:
        all_nuc_ion = np.zeros((0, 28))
    return all_nuclear, all_nuc_ion


def fold_debye_waller(all_nuclear, all_nuc_ion, flag: str):
    """Add B to every Peng ``b_i`` when a Debye-Waller envelope is requested.

    CommonPart_forsimulation_lobato_peng.m:88-110; Lobato keeps B separate (the engine
    multiplies by exp(-B s^2) instead).
    """
    if flag == "l":
        return all_nuclear, all_nuc_ion
    a = all_nuclear.copy()
    b = all_nuc_ion.copy()
    if len(a):
        a[:, 7:16:2] += a[:, 4:5]
    if len(b):
        b[:, 8:17:2] += b[:, 4:5]
        b[:, 19:28:2] += b[:, 4:5]
    return a, b


def _contribution(bcoef, z1, z2):
    """|erf(2 pi z2/sqrt(b))/2 - erf(2 pi z1/sqrt(b))/2| (CalAllEquilent20210223_lobato_peng.m:226)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.abs(0.5 * erf(2 * np.pi * z2 / np.sqrt(bcoef)) - 0.5 * erf(2 * np.pi * z1 / np.sqrt(bcoef)))
    return r


def _select(table, zcol, slicethick, eachthick, multiceng, i):
    top = slicethick[i]
    sel = np.flatnonzero((table[:, zcol] >= top - multiceng * eachthick)
                         & (table[:, zcol] < top + multiceng * eachthick + eachthick))
    z = table[sel, zcol]
    z1 = z - (top + eachthick)
    z2 = z - top
    if i == 0:
        z2 = np.full_like(z2, np.inf)
    if i == len(slicethick) - 1:
        z1 = np.full_like(z1, -np.inf)
    z2 = np.where(np.abs(z2) >= multiceng * eachthick, np.inf, z2)
    z1 = np.where(np.abs(z1) >= multiceng * eachthick, -np.inf, z1)
    return sel, z1[:, None], z2[:, None]


def slice_rows(all_nuclear, all_nuc_ion, eachthick: float, slicethick, multiceng: int,
               flag: str, dbmode: int = 0):
    """Assign atoms to slices and produce the engine's coefficient rows.

    Restates CalAllEquilent20210223_lobato_peng.m:23-228 (absorptive rows are not produced;
    the absorptive-potential fit is not part of this engine's host tools).
    Returns ``(ele_n, ele_n_i, series_n, series_n_i)``.
    """
    slicethick = np.asarray(slicethick, dtype=np.float64)
    S = len(slicethick)
    ele, series = [], []
    if len(all_nuclear):
        for i in range(S):
            sel, z1, z2 = _select(all_nuclear, 3, slicethick, eachthick, multiceng, i)
            rows = all_nuclear[sel].copy()
            rows[:, 6:16:2] *= _contribution(rows[:, 7:16:2], z1, z2)
            series.append(len(sel))
            ele.append(rows)
    ele_i, series_i = [], []
    if len(all_nuc_ion):
        for i in range(S):
            sel, z1, z2 = _select(all_nuc_ion, 3, slicethick, eachthick, multiceng, i)
            rows = all_nuc_ion[sel].copy()
            rows[:, 7:17:2] *= _contribution(rows[:, 8:17:2], z1, z2)
            rows[:, 18:28:2] *= _contribution(rows[:, 19:28:2], z1, z2)
            series_i.append(len(sel))
            ele_i.append(rows)

    def finish(blocks, ncol):
        if not blocks:
            return np.zeros((0, ncol - 3 + (1 if flag == "l" else 0)))
        t = np.concatenate(blocks)
        b = t[:, 4].copy()
        t = np.delete(t, [0, 3, 4], axis=1)  # drop Z, z, B
        if flag == "l":
            t = np.concatenate([t, (b * dbmode)[:, None]], axis=1)
        return t

    ele_n = finish(ele, 16)
    ele_n_i = finish(ele_i, 28)
    series_n = np.array(series, dtype=np.float64) if series else np.zeros(0)
    series_n_i = np.array(series_i, dtype=np.float64) if series_i else np.zeros(0)
    return ele_n, ele_n_i, series_n, series_n_i


def frozen_phonon(table: np.ndarray, eachthick: float, slicethick, rng: np.random.Generator,
                  zcol: int = 3, bcol: int = 4) -> np.ndarray:
    """Gaussian thermal displacement with sigma = sqrt(B / 8 pi^2) per axis (randshiftpos.m:1-14).

    Works on the 16/28-column tables (x, y, z at columns 1..3, B at column 4).  Atoms displaced
    out of the slab are re-drawn, as the reference does.  The stream comes from ``rng`` so a
    configuration is reproducible from its seed.
    """
    slicethick = np.asarray(slicethick)
    out = table.copy()
    sig = np.sqrt(table[:, bcol] / 8 / np.pi ** 2)[:, None]
    out[:, 1:4] = table[:, 1:4] + rng.standard_normal((len(table), 3)) * sig
    lo, hi = slicethick[0], slicethick[-1] + eachthick
    bad = np.flatnonzero((out[:, zcol] < lo) | (out[:, zcol] >= hi))
    while bad.size:
        out[bad, 1:4] = table[bad, 1:4] + rng.standard_normal((bad.size, 3)) * sig[bad]
        bad = bad[(out[bad, zcol] < lo) | (out[bad, zcol] >= hi)]
    return out


def b_from_rms(rms: float) -> float:
    """Debye-Waller B for an isotropic per-axis rms displacement (B = 8 pi^2 u^2)."""
    return 8 * math.pi ** 2 * rms * rms
