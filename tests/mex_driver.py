"""Test helper: call the reference's MEX shim (built by ``oracle/build_ref.py``) the way MATLAB's
``cuda_stem.m`` does, with 41 stand-in MATLAB arrays built from a ``StemRequest``.

Argument order and meaning follow cuda_stem.m:97-106 and waveCuda.cpp:18-99: every array is
handed over in the memory order ``cuda_stem.m`` produces by its transposes (row-major with the
MATLAB row index first, which is how ``StemRequest`` stores them), scalars are 1x1 doubles,
``beginRow`` / ``beginCol`` are 1-based (the shim subtracts one), the mid-layer list is uint32.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_OUT = os.path.join(ROOT, "oracle", "_ref")

MEX_NAMES = {("p", False): "waveCudaPengAndCorr", ("l", False): "waveCudalobato",
             ("p", True): "waveCudaPengAndCorrP", ("l", True): "waveCudalobatoP"}


def mex_library(param: str, transmission: bool, out_dir: str = REF_OUT) -> C.CDLL | None:
    path = os.path.join(out_dir, f"mex_{MEX_NAMES[(param, transmission)]}.so")
    if not os.path.exists(path):
        return None
    from totem_b200 import capi
    capi.load()  # the engine library first: the MEX builds link against it
    # local symbol scope, as MATLAB loads MEX files: the four shim libraries export the same
    # myProjectfun, and each MEX build must bind to the one it was linked against
    lib = C.CDLL(path, mode=C.RTLD_LOCAL)
    vp = C.c_void_p
    lib.mexFunction.argtypes = [C.c_int, C.POINTER(vp), C.c_int, C.POINTER(vp)]
    lib.mexFunction.restype = None
    lib.mex_stub_wrap.argtypes = [vp, C.c_size_t, C.c_size_t]
    lib.mex_stub_wrap.restype = vp
    lib.mex_stub_data.argtypes = [vp]
    lib.mex_stub_data.restype = vp
    lib.mex_stub_rows.argtypes = [vp]
    lib.mex_stub_rows.restype = C.c_size_t
    lib.mex_stub_cols.argtypes = [vp]
    lib.mex_stub_cols.restype = C.c_size_t
    lib.mex_stub_free.argtypes = [vp]
    lib.mex_stub_last_error.restype = C.c_char_p
    lib.mex_stub_error_count.restype = C.c_int
    return lib


class MexCall:
    """The 41 right-hand-side arrays of one MEX call, kept alive with their stand-in headers."""

    def __init__(self, lib, req, transmission: bool = False):
        self.lib = lib
        self.keep = []
        self.arrays = []
        series_n, series_n_i = req.padded_series()
        stem = not transmission

        def arr(a, dtype=np.float64):
            if a is None:
                return self._wrap(None, 0, 0)
            a = np.ascontiguousarray(a, dtype=dtype)
            self.keep.append(a)
            rows = a.shape[0] if a.ndim else 1
            return self._wrap(a, rows, a.size // max(rows, 1))

        def scalar(v):
            return arr(np.array([float(v)]))

        probe = req.probe if stem else np.zeros((1, 2, 2), complex)
        corr = req.corr_info_matrix is not None and len(req.corr_info_matrix)
        mids = np.asarray(req.mid_layer, dtype=np.uint32) if stem else np.zeros(0, np.uint32)
        rhs = [
            arr(probe.real), arr(probe.imag), arr(req.aper if stem else None),
            arr(series_n), arr(req.absorp_n), arr(series_n_i), arr(req.absorp_n_i),
            arr(req.ele_n if len(req.ele_n) else None), arr(req.ele_n_i if len(req.ele_n_i) else None),
            arr(req.kx), arr(req.ky), arr(req.s2),
            arr(req.prop.real if stem else None), arr(req.prop.imag if stem else None),
            arr(req.gfsf if stem else np.ones(1)),
            scalar(req.height if stem else 0), scalar(req.width if stem else 0), scalar(req.depth if stem else 0),
            scalar(req.p_height), scalar(req.p_width), scalar(req.slices), scalar(req.step if stem else 0),
            scalar(req.beginrow + 1 if stem else 1), scalar(req.begincol + 1 if stem else 1),
            scalar(req.width_red if stem else 0), scalar(req.sigma), scalar(req.w_num if stem else 1),
            scalar(req.aper_num if stem else 0), scalar(req.parameter), arr(req.aper_true),
            scalar(1 if req.absorp_n is not None else 0), scalar(1 if req.absorp_n_i is not None else 0),
            arr(mids if len(mids) else None, np.uint32), scalar(len(mids)), arr(req.aper2 if stem else None),
            arr(req.series_n_corr if corr else None), arr(req.series_n_i_corr if corr else None),
            arr(req.ele_n_corr if corr else None), arr(req.ele_n_i_corr if corr else None),
            arr(req.corr_info_matrix if corr else None), scalar(len(req.corr_info_matrix) if corr else 0),
        ]
        assert len(rhs) == 41
        self.prhs = (C.c_void_p * 41)(*rhs)

    def _wrap(self, a, rows, cols):
        h = self.lib.mex_stub_wrap(None if a is None else a.ctypes.data, rows, cols)
        self.arrays.append(h)
        return h

    def call(self, nlhs: int = 4, nrhs: int = 41):
        """mexFunction(nlhs, plhs, nrhs, prhs); returns the output arrays as NumPy copies (column-
        major MATLAB shapes flattened), or None where the shim created none."""
        plhs = (C.c_void_p * 4)()
        self.lib.mexFunction(nlhs, plhs, nrhs, self.prhs)
        outs = []
        for h in plhs:
            if not h:
                outs.append(None)
                continue
            m, n = self.lib.mex_stub_rows(h), self.lib.mex_stub_cols(h)
            p = self.lib.mex_stub_data(h)
            outs.append(np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(m * n,)).copy()
                        if m * n else np.zeros(0))
            self.lib.mex_stub_free(h)
        return outs

    def close(self):
        for h in self.arrays:
            self.lib.mex_stub_free(h)
        self.arrays = []
