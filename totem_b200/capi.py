"""ctypes binding of ``include/totem_b200.h`` (the engine's C ABI).

Loading fails loudly when the shared library is missing: there is no CPU or PyTorch fallback.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
CORE_PATH = os.path.join(LIB_DIR, "libtotem_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "totem_b200.h")
SHIM_LIBS = {("p", False): "libwaveCudaPeng.so", ("l", False): "libwaveCudaLobato.so",
             ("p", True): "libwaveCudaPengP.so", ("l", True): "libwaveCudaLobatoP.so"}

OK, ERR_INVALID_ARG, ERR_UNSUPPORTED, ERR_CUDA, ERR_CUFFT, ERR_OOM, ERR_NO_DEVICE, ERR_STATE, ERR_TIMEOUT = range(9)
SCHED_FIFO, SCHED_SHORTEST = 0, 1
REQ_QUEUED, REQ_PREPARING, REQ_RUNNING, REQ_DONE, REQ_FAILED = range(5)
PARAM_PENG, PARAM_LOBATO = 0, 1
PATH_FUSED, PATH_PLAIN, PATH_FUSED_ONLY = 0, 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class TotemStemArgs(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int), ("param", C.c_int),
        ("probe_re", _dp), ("probe_im", _dp), ("aper", _dp),
        ("atom_slice", _dp), ("absorp_n", _dp), ("atom_slice_i", _dp), ("absorp_n_i", _dp),
        ("proj_coff_mat", _dp), ("proj_coff_mat_i", _dp),
        ("kx", _dp), ("ky", _dp), ("s_2", _dp), ("prop_re", _dp), ("prop_im", _dp), ("gfsf", _dp),
        ("height", C.c_int), ("width", C.c_int), ("depth", C.c_int),
        ("p_height", C.c_int), ("p_width", C.c_int), ("slices", C.c_int), ("step", C.c_int),
        ("begin_row", C.c_int), ("begin_col", C.c_int), ("width_red", C.c_int),
        ("sigma", C.c_double), ("w_num", C.c_int), ("aper_num", C.c_int), ("parameter", C.c_double),
        ("aper_true", _dp), ("mid_layer", _ip), ("layer_len", C.c_int), ("aper2", _dp),
        ("series_n_corr", _dp), ("series_n_i_corr", _dp), ("ele_n_corr", _dp), ("ele_n_i_corr", _dp),
        ("corr_info_matrix", _dp), ("cim_len", C.c_int),
    ]


class TotemStemOut(C.Structure):
    _fields_ = [("result", _dp), ("mid_layer_mat", _dp), ("potential_re", _dp), ("potential_im", _dp)]


T_COMPLEX64, T_BF16 = 0, 1


class TotemRunOptions(C.Structure):
    _fields_ = [("path", C.c_int), ("batch", C.c_int), ("skip_transmission", C.c_int), ("profile", C.c_int),
                ("col_variant", C.c_int), ("t_storage", C.c_int), ("row_variant", C.c_int)]


class TotemHrtemArgs(C.Structure):
    _fields_ = [("struct_size", C.c_int), ("wave_re", _dp), ("wave_im", _dp), ("prop_re", _dp), ("prop_im", _dp),
                ("defoci", C.c_int), ("tf_re", _dp), ("tf_im", _dp), ("weights", _dp), ("t_storage", C.c_int)]


class TotemHrtemOut(C.Structure):
    _fields_ = [("exit_re", _dp), ("exit_im", _dp), ("image", _dp)]


class TotemTiming(C.Structure):
    _fields_ = [("transmission_ms", C.c_float), ("slice_loop_ms", C.c_float), ("total_ms", C.c_float),
                ("kernel_launches", C.c_int), ("batch", C.c_int),
                ("row_pass_ms", C.c_float), ("col_pass_ms", C.c_float),
                ("row_pass_launches", C.c_int), ("col_pass_launches", C.c_int),
                ("probe_slices", C.c_longlong), ("h2d_bytes", C.c_longlong), ("d2h_bytes", C.c_longlong),
                ("slice_path", C.c_int), ("tx_fft_path", C.c_int), ("tx_builder", C.c_int),
                ("row_variant", C.c_int), ("col_variant", C.c_int)]


class TotemServerOptions(C.Structure):
    _fields_ = [("struct_size", C.c_int), ("device", C.c_int), ("hbm_budget", C.c_ulonglong),
                ("wave_bytes", C.c_ulonglong), ("chunk_bytes", C.c_ulonglong), ("ticks_ahead", C.c_int),
                ("policy", C.c_int), ("prep_threads", C.c_int), ("mixed_windows", C.c_int)]


class TotemRequestInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("status", C.c_int), ("queued_ms", C.c_double), ("prepare_ms", C.c_double),
                ("run_ms", C.c_double), ("latency_ms", C.c_double), ("probe_slices", C.c_longlong)]


class TotemServerStats(C.Structure):
    _fields_ = [("ticks", C.c_longlong), ("probe_slices", C.c_longlong), ("launches", C.c_longlong),
                ("groups", C.c_longlong), ("requests_done", C.c_longlong), ("issue_ms", C.c_double),
                ("throttle_ms", C.c_double), ("idle_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TotemAberrations(C.Structure):
    _fields_ = [("struct_size", C.c_int)] + [(f, C.c_double) for f in (
        "focus", "A1", "phiA1", "A2", "phiA2", "B2", "phiB2", "Cs", "A3", "phiA3", "S3", "phiS3", "A4", "phiA4",
        "D4", "phiD4", "B4", "phiB4", "A5", "phiA5", "C5", "S5", "phiS5", "D5", "phiD5")]


class TotemError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"totem_b200 error {code}: {msg}")
        self.code = code


_LIB = None


def library_path() -> str:
    return CORE_PATH


def load() -> C.CDLL:
    """Load ``libtotem_b200.so`` (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(CORE_PATH):
        raise RuntimeError(f"{CORE_PATH} is missing: run `python -m totem_b200.build` "
                           "(this engine has no CPU fallback)")
    lib = C.CDLL(CORE_PATH)
    vp = C.c_void_p
    lib.totem_abi_version.restype = C.c_int
    lib.totem_status_string.restype = C.c_char_p
    lib.totem_status_string.argtypes = [C.c_int]
    lib.totem_last_error.restype = C.c_char_p
    lib.totem_session_create.argtypes = [C.c_int, vp, C.POINTER(vp)]
    lib.totem_session_destroy.argtypes = [vp]
    lib.totem_session_upload.argtypes = [vp, C.POINTER(TotemStemArgs)]
    lib.totem_session_run.argtypes = [vp, C.c_int, C.POINTER(TotemRunOptions)]
    lib.totem_session_download.argtypes = [vp, C.POINTER(TotemStemOut)]
    lib.totem_session_timing.argtypes = [vp, C.POINTER(TotemTiming)]
    lib.totem_session_transmission.argtypes = [vp, C.POINTER(vp)]
    lib.totem_stem_run.argtypes = [C.POINTER(TotemStemArgs), C.POINTER(TotemRunOptions), C.POINTER(TotemStemOut)]
    lib.totem_session_hrtem.argtypes = [vp, C.POINTER(TotemHrtemArgs), C.POINTER(TotemHrtemOut)]
    lib.totem_hrtem_run.argtypes = [C.POINTER(TotemStemArgs), C.POINTER(TotemHrtemArgs), C.POINTER(TotemHrtemOut)]
    lib.totem_transmission_run.argtypes = [C.POINTER(TotemStemArgs), C.POINTER(TotemStemOut)]
    lib.totem_stem_slices_noalloc.argtypes = ([vp, C.c_int, C.c_int, C.c_int, vp, C.c_int, vp, vp] + [C.c_int] * 9
                                              + [vp, vp])
    ull, ullp = C.c_ulonglong, C.POINTER(C.c_ulonglong)
    lib.totem_server_create.argtypes = [C.POINTER(TotemServerOptions), C.POINTER(vp)]
    lib.totem_server_submit.argtypes = [vp, C.POINTER(TotemStemArgs), C.POINTER(TotemStemOut), ullp]
    lib.totem_server_wait.argtypes = [vp, ull, C.c_int]
    lib.totem_server_info.argtypes = [vp, ull, C.POINTER(TotemRequestInfo)]
    lib.totem_server_destroy.argtypes = [vp]
    lib.totem_server_stats.argtypes = [vp, C.POINTER(TotemServerStats)]
    lib.totem_tcc_stack.argtypes = [C.POINTER(TotemAberrations), C.c_double, C.c_int, C.c_double, C.c_double,
                                    C.c_int, C.c_int, C.c_double, _dp, _dp]
    lib.totem_set_tx_builder.argtypes = [C.c_int, C.c_size_t]
    lib.totem_set_slice_graphs.argtypes = [C.c_int]
    lib.totem_set_band_skip.argtypes = [C.c_int]
    lib.totem_fp32_peak.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.totem_inject_failures.argtypes = [C.c_longlong, C.c_int]
    lib.totem_load_tuning.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
    lib.totem_tuned_config.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       C.POINTER(C.c_longlong)]
    llp = C.POINTER(C.c_longlong)
    lib.totem_slice_rows.argtypes = [C.c_int, _dp, C.c_int, _dp, C.c_int, C.c_double, _dp, C.c_int, C.c_int, C.c_int,
                                     _dp, C.c_longlong, _dp, C.c_longlong, _dp, _dp, llp, llp]
    lib.totem_fold_debye_waller.argtypes = [C.c_int, _dp, C.c_int, _dp, C.c_int]
    lib.totem_frozen_phonon.argtypes = [_dp, C.c_int, C.c_int, C.c_double, _dp, C.c_int, C.c_ulonglong, _dp]
    lib.totem_grid_batches.argtypes = [_ip, C.c_int, C.c_int, _ip, C.c_int, _ip]
    lib.totem_plan_simulate.argtypes = [C.c_int, _ip, C.POINTER(C.c_longlong), _ip, _ip, ull, ull, C.c_int, _ip, _ip,
                                        ullp]
    for name in ("totem_session_create", "totem_session_destroy", "totem_session_upload", "totem_session_run",
                 "totem_session_download", "totem_session_timing", "totem_session_transmission",
                 "totem_stem_run", "totem_transmission_run", "totem_stem_slices_noalloc", "totem_session_hrtem",
                 "totem_hrtem_run", "totem_session_cbed", "totem_cbed_run", "totem_server_create",
                 "totem_server_submit", "totem_server_wait", "totem_server_info", "totem_server_destroy",
                 "totem_server_stats", "totem_plan_simulate", "totem_tcc_stack", "totem_set_tx_builder",
                 "totem_grid_batches", "totem_set_slice_graphs", "totem_set_band_skip", "totem_fp32_peak", "totem_inject_failures", "totem_load_tuning", "totem_tuned_config", "totem_slice_rows", "totem_fold_debye_waller", "totem_frozen_phonon"):
        getattr(lib, name).restype = C.c_int
    _LIB = lib
    return lib


def check(rc: int):
    if rc != OK:
        lib = load()
        raise TotemError(rc, f"{lib.totem_status_string(rc).decode()}: {lib.totem_last_error().decode()}")


def header_functions() -> list[str]:
    """Names of the C functions declared in ``include/totem_b200.h``."""
    text = open(HEADER).read()
    c_part = text.split("#ifdef __cplusplus\n} /* extern \"C\" */")[0]
    return sorted(set(re.findall(r"\b(totem_[a-z_]+)\s*\(", c_part)))


# ----------------------------------------------------------------------------------------------
# numpy <-> struct marshalling
# ----------------------------------------------------------------------------------------------

def _d(a):
    if a is None:
        return None
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a, typ=_dp):
    if a is None:
        return C.cast(None, typ)
    return a.ctypes.data_as(typ)


class Marshalled:
    """Keeps the numpy buffers referenced by a TotemStemArgs alive."""

    def __init__(self, req, stem: bool = True):
        self.keep = []

        def k(a):
            a = _d(a)
            if a is not None:
                self.keep.append(a)
            return a
        series_n, series_n_i = req.padded_series()
        a = TotemStemArgs()
        a.struct_size = C.sizeof(TotemStemArgs)
        a.param = PARAM_LOBATO if req.param == "l" else PARAM_PENG
        if stem:
            a.probe_re = _ptr(k(req.probe.real))
            a.probe_im = _ptr(k(req.probe.imag))
            a.aper = _ptr(k(req.aper))
            a.prop_re = _ptr(k(req.prop.real))
            a.prop_im = _ptr(k(req.prop.imag))
            a.gfsf = _ptr(k(req.gfsf))
            a.aper2 = _ptr(k(req.aper2))
            a.height, a.width = req.height, req.width
            a.depth = req.depth
            a.step, a.begin_row, a.begin_col, a.width_red = req.step, req.beginrow, req.begincol, req.width_red
            a.w_num, a.aper_num = req.w_num, req.aper_num
            mid = np.ascontiguousarray(req.mid_layer, dtype=np.int32)
            self.keep.append(mid)
            a.mid_layer = mid.ctypes.data_as(_ip)
            a.layer_len = len(mid)
        else:
            a.w_num = 1
        a.atom_slice = _ptr(k(series_n))
        a.atom_slice_i = _ptr(k(series_n_i))
        a.absorp_n = _ptr(k(req.absorp_n))
        a.absorp_n_i = _ptr(k(req.absorp_n_i))
        a.proj_coff_mat = _ptr(k(req.ele_n if len(req.ele_n) else None))
        a.proj_coff_mat_i = _ptr(k(req.ele_n_i if len(req.ele_n_i) else None))
        a.kx, a.ky, a.s_2 = _ptr(k(req.kx)), _ptr(k(req.ky)), _ptr(k(req.s2))
        a.p_height, a.p_width, a.slices = req.p_height, req.p_width, req.slices
        a.sigma, a.parameter = req.sigma, req.parameter
        a.aper_true = _ptr(k(req.aper_true))
        if req.corr_info_matrix is not None and len(req.corr_info_matrix):
            a.series_n_corr = _ptr(k(req.series_n_corr))
            a.series_n_i_corr = _ptr(k(req.series_n_i_corr))
            a.ele_n_corr = _ptr(k(req.ele_n_corr))
            a.ele_n_i_corr = _ptr(k(req.ele_n_i_corr))
            a.corr_info_matrix = _ptr(k(req.corr_info_matrix))
            a.cim_len = len(req.corr_info_matrix)
        self.args = a


class Session:
    """A device session: inputs uploaded once, runs on the device, results fetched on demand."""

    def __init__(self, device: int = -1, stream: int | None = None):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.totem_session_create(device, C.c_void_p(stream) if stream else None, C.byref(h)))
        self.h = h
        self.req = None
        self._m = None

    def close(self):
        if self.h:
            self.lib.totem_session_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, req, stem: bool = True):
        self._m = Marshalled(req, stem)
        self.req = req
        check(self.lib.totem_session_upload(self.h, C.byref(self._m.args)))

    def run(self, what: int = 0, path: int = PATH_FUSED, batch: int = 0, skip_transmission: bool = False,
            profile: bool = False, col_variant: int = 0, t_storage: int = T_COMPLEX64, row_variant: int = 0):
        o = TotemRunOptions(path, batch, int(skip_transmission), int(profile), col_variant, t_storage, row_variant)
        check(self.lib.totem_session_run(self.h, what, C.byref(o)))

    def hrtem(self, spec, t_storage: int = T_COMPLEX64, exit_wave: bool = True, image: bool = True):
        """HRTEM on the uploaded specimen (``totem_session_hrtem``): (exit wave, image)."""
        h, out, ex, img = _hrtem_marshal(spec, self.req.p_height, self.req.p_width, t_storage, exit_wave, image)
        check(self.lib.totem_session_hrtem(self.h, C.byref(h.args), C.byref(out)))
        return ex(), img

    def cbed(self):
        """CBED pattern of the uploaded depth-1 request (``totem_session_cbed``)."""
        pat = np.zeros(self.req.height * self.req.width)
        check(self.lib.totem_session_cbed(self.h, _ptr(pat)))
        return pat.reshape(self.req.height, self.req.width)

    def download(self, want_transmission: bool = False):
        req = self.req
        out = TotemStemOut()
        res = mid = tre = tim = None
        if req.depth:
            res = np.zeros(req.aper_num * req.depth)
            mid = np.zeros(req.aper_num * req.depth * len(req.mid_layer))
            out.result = _ptr(res)
            out.mid_layer_mat = _ptr(mid)
        if want_transmission:
            n = req.p_height * req.p_width * req.slices
            tre, tim = np.zeros(n), np.zeros(n)
            out.potential_re, out.potential_im = _ptr(tre), _ptr(tim)
        check(self.lib.totem_session_download(self.h, C.byref(out)))
        t = None
        if want_transmission:
            t = (tre + 1j * tim).reshape(req.slices, req.p_height, req.p_width)
        return res, mid, t

    def timing(self) -> TotemTiming:
        t = TotemTiming()
        check(self.lib.totem_session_timing(self.h, C.byref(t)))
        return t

    def transmission_ptr(self) -> int:
        """Device address of the transmission stack built by the last run (complex64)."""
        p = C.c_void_p()
        check(self.lib.totem_session_transmission(self.h, C.byref(p)))
        return p.value


def stem_slices_noalloc(transmission: int, p_height: int, p_width: int, slices: int, probe: int, w_num: int,
                        propagator: int, masks: int, aper_num: int, n: int, step: int, begin_row: int,
                        begin_col: int, width_red: int, depth: int, item0: int, items: int, result: int,
                        stream: int | None = None):
    """``totem_stem_slices_noalloc``: every pointer is a device address owned by the caller."""
    lib = load()
    check(lib.totem_stem_slices_noalloc(transmission, p_height, p_width, slices, probe, w_num, propagator, masks,
                                        aper_num, n, step, begin_row, begin_col, width_red, depth, item0, items,
                                        result, stream))


class Server:
    """The serving scheduler (``totem_server_*``): submit requests, wait for them, read latencies.

    Every submitted request keeps its marshalled inputs and its output arrays referenced here
    until it is waited for, as the C API requires.
    """

    def __init__(self, device: int = -1, hbm_budget: int = 0, wave_bytes: int = 0, chunk_bytes: int = 0,
                 ticks_ahead: int = 0, policy: int = SCHED_SHORTEST, prep_threads: int = 0,
                 mixed_windows: bool = False):
        self.lib = load()
        o = TotemServerOptions(C.sizeof(TotemServerOptions), device, hbm_budget, wave_bytes, chunk_bytes,
                               ticks_ahead, policy, prep_threads, int(mixed_windows))
        h = C.c_void_p()
        check(self.lib.totem_server_create(C.byref(o), C.byref(h)))
        self.h = h
        self._live = {}

    def submit(self, req) -> int:
        m = Marshalled(req, True)
        res = np.zeros(req.aper_num * req.depth)
        mid = np.zeros(req.aper_num * req.depth * len(req.mid_layer))
        out = TotemStemOut(_ptr(res), _ptr(mid), None, None)
        t = C.c_ulonglong()
        check(self.lib.totem_server_submit(self.h, C.byref(m.args), C.byref(out), C.byref(t)))
        self._live[t.value] = (m, out, res, mid)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """Results (detector sums, mid-layer sums) of a finished request; raises on failure."""
        check(self.lib.totem_server_wait(self.h, ticket, timeout_ms))
        _, _, res, mid = self._live.pop(ticket)
        return res, mid

    def info(self, ticket: int) -> TotemRequestInfo:
        i = TotemRequestInfo()
        check(self.lib.totem_server_info(self.h, ticket, C.byref(i)))
        return i

    def stats(self) -> dict:
        st = TotemServerStats()
        check(self.lib.totem_server_stats(self.h, C.byref(st)))
        return st.as_dict()

    def close(self):
        if self.h:
            self.lib.totem_server_destroy(self.h)
            self.h = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def plan_simulate(n, items, slices, arrive, wave_bytes: int, chunk_bytes: int = 0, policy: int = SCHED_SHORTEST):
    """``totem_plan_simulate``: the scheduler's admission policy without a device.

    Returns (first_tick, done_tick, max_inflight_bytes)."""
    lib = load()
    cnt = len(n)
    n_ = np.ascontiguousarray(n, dtype=np.int32)
    it_ = np.ascontiguousarray(items, dtype=np.int64)
    sl_ = np.ascontiguousarray(slices, dtype=np.int32)
    ar_ = np.ascontiguousarray(arrive, dtype=np.int32)
    first = np.zeros(cnt, dtype=np.int32)
    done = np.zeros(cnt, dtype=np.int32)
    mx = C.c_ulonglong()
    check(lib.totem_plan_simulate(cnt, n_.ctypes.data_as(_ip), it_.ctypes.data_as(C.POINTER(C.c_longlong)),
                                  sl_.ctypes.data_as(_ip), ar_.ctypes.data_as(_ip), wave_bytes, chunk_bytes, policy,
                                  first.ctypes.data_as(_ip), done.ctypes.data_as(_ip), C.byref(mx)))
    return first, done, mx.value


class _HrtemMarshalled:
    """Keeps the numpy buffers referenced by a TotemHrtemArgs alive."""

    def __init__(self, spec, t_storage):
        self.keep = []

        def k(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            self.keep.append(a)
            return _ptr(a)
        a = TotemHrtemArgs()
        a.struct_size = C.sizeof(TotemHrtemArgs)
        if spec.wave is not None:
            a.wave_re, a.wave_im = k(spec.wave.real), k(spec.wave.imag)
        a.prop_re, a.prop_im = k(spec.prop.real), k(spec.prop.imag)
        if spec.tf is not None and len(spec.tf):
            a.defoci = len(spec.tf)
            a.tf_re, a.tf_im = k(spec.tf.real), k(spec.tf.imag)
            a.weights = k(spec.weights)
        a.t_storage = t_storage
        self.args = a


def _hrtem_marshal(spec, ph, pw, t_storage, exit_wave, image):
    h = _HrtemMarshalled(spec, t_storage)
    out = TotemHrtemOut()
    ere = eim = img = None
    if exit_wave:
        ere, eim = np.zeros((ph, pw)), np.zeros((ph, pw))
        out.exit_re, out.exit_im = _ptr(ere), _ptr(eim)
    if image and spec.tf is not None and len(spec.tf):
        img = np.zeros((ph, pw))
        out.image = _ptr(img)

    def ex():
        return None if ere is None else ere + 1j * eim
    return h, out, ex, img


def tcc_stack(ab, lambda_nm: float, n: int, sampling_a: float, alpha_mrad: float, with_gradient: bool, steps: int,
              delta_nm: float) -> np.ndarray:
    """``totem_tcc_stack``: the transfer functions (steps, n, n) complex128 on the centred grid,
    evaluated on the device in FP64.  ``ab`` is an ``optics.Aberrations``."""
    lib = load()
    a = TotemAberrations()
    a.struct_size = C.sizeof(TotemAberrations)
    for name, _ in TotemAberrations._fields_[1:]:
        setattr(a, name, float(getattr(ab, name)))
    re_ = np.zeros((steps, n, n))
    im_ = np.zeros((steps, n, n))
    check(lib.totem_tcc_stack(C.byref(a), lambda_nm, n, sampling_a, alpha_mrad, int(with_gradient), steps, delta_nm,
                              _ptr(re_), _ptr(im_)))
    return re_ + 1j * im_


def hrtem_run(specimen, spec, t_storage: int = T_COMPLEX64, exit_wave: bool = True, image: bool = True):
    """One-shot HRTEM (``totem_hrtem_run``): returns (exit wave [P_H, P_W] complex, image or None)."""
    lib = load()
    m = Marshalled(specimen, False)
    h, out, ex, img = _hrtem_marshal(spec, specimen.p_height, specimen.p_width, t_storage, exit_wave, image)
    check(lib.totem_hrtem_run(C.byref(m.args), C.byref(h.args), C.byref(out)))
    return ex(), img


def cbed_run(req):
    """One-shot CBED pattern (``totem_cbed_run``) of a depth-1 request: [height, width], zero
    frequency at the centre."""
    lib = load()
    m = Marshalled(req, True)
    pat = np.zeros(req.height * req.width)
    check(lib.totem_cbed_run(C.byref(m.args), _ptr(pat)))
    return pat.reshape(req.height, req.width)


def stem_run(req, path: int = PATH_FUSED, batch: int = 0):
    """One-shot STEM call through ``totem_stem_run`` (host buffers in, host buffers out)."""
    lib = load()
    m = Marshalled(req, True)
    res = np.zeros(req.aper_num * req.depth)
    mid = np.zeros(req.aper_num * req.depth * len(req.mid_layer))
    out = TotemStemOut(_ptr(res), _ptr(mid), None, None)
    opt = TotemRunOptions(path, batch, 0, 0, 0, T_COMPLEX64, 0)
    check(lib.totem_stem_run(C.byref(m.args), C.byref(opt), C.byref(out)))
    return res, mid


# ----------------------------------------------------------------------------------------------
# Specimen preparation in the library (host only)
# ----------------------------------------------------------------------------------------------

def _param(flag: str) -> int:
    return PARAM_LOBATO if flag == "l" else PARAM_PENG


def _table(t, ncol):
    t = np.ascontiguousarray(t, dtype=np.float64).reshape(-1, ncol)
    return t, t.ctypes.data_as(_dp)


def slice_rows(all_nuclear, all_nuc_ion, eachthick: float, slicethick, multiceng: int, flag: str, dbmode: int = 0):
    """``totem_slice_rows``: the same outputs as ``specimen.slice_rows`` (ele_n, ele_n_i,
    series_n, series_n_i; a kind without atoms gives an empty series)."""
    lib = load()
    nuc, nuc_p = _table(all_nuclear, 16)
    ion, ion_p = _table(all_nuc_ion, 28)
    st = np.ascontiguousarray(slicethick, dtype=np.float64)
    S = len(st)
    rn, ri = C.c_longlong(0), C.c_longlong(0)
    args = (_param(flag), nuc_p, len(nuc), ion_p, len(ion), float(eachthick), st.ctypes.data_as(_dp), S,
            int(multiceng), int(dbmode))
    check(lib.totem_slice_rows(*args, None, 0, None, 0, None, None, C.byref(rn), C.byref(ri)))
    extra = 1 if flag == "l" else 0
    ele_n = np.zeros((rn.value, 13 + extra))
    ele_i = np.zeros((ri.value, 25 + extra))
    sn, si = np.zeros(S), np.zeros(S)
    check(lib.totem_slice_rows(*args, ele_n.ctypes.data_as(_dp), rn.value, ele_i.ctypes.data_as(_dp), ri.value,
                               sn.ctypes.data_as(_dp), si.ctypes.data_as(_dp), C.byref(rn), C.byref(ri)))
    return ele_n, ele_i, (sn if len(nuc) else np.zeros(0)), (si if len(ion) else np.zeros(0))


def fold_debye_waller(all_nuclear, all_nuc_ion, flag: str):
    """``totem_fold_debye_waller`` on copies of the two tables."""
    nuc, nuc_p = _table(np.array(all_nuclear, dtype=np.float64, copy=True), 16)
    ion, ion_p = _table(np.array(all_nuc_ion, dtype=np.float64, copy=True), 28)
    check(load().totem_fold_debye_waller(_param(flag), nuc_p, len(nuc), ion_p, len(ion)))
    return nuc, ion


def frozen_phonon(table, eachthick: float, slicethick, seed: int) -> np.ndarray:
    """``totem_frozen_phonon``: one seeded thermal configuration of a 16/28-column table."""
    t = np.ascontiguousarray(table, dtype=np.float64)
    out = np.empty_like(t)
    st = np.ascontiguousarray(slicethick, dtype=np.float64)
    check(load().totem_frozen_phonon(t.ctypes.data_as(_dp), t.shape[0], t.shape[1], float(eachthick),
                                     st.ctypes.data_as(_dp), len(st), int(seed) & (2 ** 64 - 1),
                                     out.ctypes.data_as(_dp)))
    return out


TX_AUTO, TX_DIRECT, TX_GRIDDING, TX_ROWS = 0, 1, 2, 3


def load_tuning(path: str | None) -> int:
    """``totem_load_tuning``: replace the process's tuning table (None = no table); returns the
    number of entries."""
    n = C.c_int(0)
    check(load().totem_load_tuning(path.encode() if path else None, C.byref(n)))
    return n.value


def tuned_config(n: int, device: int = 0):
    """``totem_tuned_config``: (row_variant, col_variant, batch_bytes) a fused run with an n x n
    window would use on ``device`` by default."""
    r, c, b = C.c_int(0), C.c_int(0), C.c_longlong(0)
    check(load().totem_tuned_config(device, n, C.byref(r), C.byref(c), C.byref(b)))
    return r.value, c.value, b.value


TUNING_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "tuning.jsonl")


def inject_failures(alloc_after: int = -1, prepare_every: int = 0):
    """``totem_inject_failures``: make the next device allocation after ``alloc_after`` more fail
    once (-1 = off), and every ``prepare_every``-th server preparation fail (0 = off)."""
    check(load().totem_inject_failures(int(alloc_after), int(prepare_every)))


def fp32_peak(device: int = 0):
    """``totem_fp32_peak``: measured FP32 FMA throughput of a GPU in TFLOP/s, (scalar, packed)."""
    a, b = C.c_double(), C.c_double()
    check(load().totem_fp32_peak(int(device), C.byref(a), C.byref(b)))
    return a.value, b.value


def set_band_skip(enable: bool):
    """``totem_set_band_skip``: skip the wave columns the propagator zeroes (default on)."""
    check(load().totem_set_band_skip(1 if enable else 0))


def set_slice_graphs(enable: bool):
    """``totem_set_slice_graphs``: replay repeated fused slice loops as CUDA graphs (default on)."""
    check(load().totem_set_slice_graphs(1 if enable else 0))


def set_tx_builder(mode: int, scratch_bytes: int = 0):
    """Process-wide transmission builder for separable grids (``totem_set_tx_builder``):
    TX_AUTO (cost model), TX_DIRECT (sums over atoms at every pixel) or TX_GRIDDING (Gaussian
    gridding + FFT where the axes are uniform); ``scratch_bytes`` bounds the gridding work memory
    (0 = the library default)."""
    check(load().totem_set_tx_builder(int(mode), int(scratch_bytes)))


def grid_batches(job_beg, jobs_per_batch: int) -> np.ndarray:
    """The gridding builder's batch plan (``totem_grid_batches``): rows (s_lo, s_hi, j_lo, j_hi)."""
    lib = load()
    jb = np.ascontiguousarray(job_beg, dtype=np.int32)
    slices = len(jb) - 1
    cnt = C.c_int(0)
    cap = 2 * (int(jb[-1]) + slices) + 2
    out = np.zeros((cap, 4), dtype=np.int32)
    check(lib.totem_grid_batches(jb.ctypes.data_as(_ip), slices, int(jobs_per_batch),
                                 out.ctypes.data_as(_ip), cap, C.byref(cnt)))
    return out[:cnt.value]


@contextlib.contextmanager
def tx_builder(mode: int, scratch_bytes: int = 0):
    """``set_tx_builder`` for the duration of a ``with`` block, then back to TX_AUTO."""
    set_tx_builder(mode, scratch_bytes)
    try:
        yield
    finally:
        set_tx_builder(TX_AUTO, 0)


def transmission_run(req):
    """One-shot transmission (the ``*P`` MEX semantics) through ``totem_transmission_run``."""
    lib = load()
    m = Marshalled(req, False)
    n = req.p_height * req.p_width * req.slices
    tre, tim = np.zeros(n), np.zeros(n)
    out = TotemStemOut(None, None, _ptr(tre), _ptr(tim))
    check(lib.totem_transmission_run(C.byref(m.args), C.byref(out)))
    return (tre + 1j * tim).reshape(req.slices, req.p_height, req.p_width)


# ----------------------------------------------------------------------------------------------
# The reference's own entry point: myProjectfun (C++ linkage) from the MEX-flavour libraries
# ----------------------------------------------------------------------------------------------

MYPROJECTFUN_MANGLED = ("_Z12myProjectfunPdS_S_S_S_S_S_S_S_S_S_S_S_S_S_iiiiiiiiiidiidS_PiiS_S_S_S_S_S_iS_S_S_S_")


def myprojectfun_lib(param: str, transmission: bool) -> C.CDLL:
    load()  # the core library must be loadable first (the shims link against it)
    path = os.path.join(LIB_DIR, SHIM_LIBS[(param, transmission)])
    lib = C.CDLL(path)
    f = getattr(lib, MYPROJECTFUN_MANGLED)
    f.restype = None
    f.argtypes = [_dp] * 15 + [C.c_int] * 10 + [C.c_double, C.c_int, C.c_int, C.c_double, _dp, _ip, C.c_int,
                                                _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp]
    return lib


def call_myprojectfun(req, transmission: bool = False):
    """Call ``myProjectfun`` exactly as waveCuda.cpp does (beginRow/beginCol already 0-based)."""
    lib = myprojectfun_lib(req.param, transmission)
    f = getattr(lib, MYPROJECTFUN_MANGLED)
    m = Marshalled(req, not transmission)
    a = m.args
    res = np.zeros(max(1, req.aper_num * req.depth))
    mid = np.zeros(max(1, req.aper_num * req.depth * len(req.mid_layer)))
    n = req.p_height * req.p_width * req.slices
    px, py = np.zeros(max(n, 1)), np.zeros(max(n, 1))
    f(a.probe_re, a.probe_im, a.aper, a.atom_slice, a.absorp_n, a.atom_slice_i, a.absorp_n_i, a.proj_coff_mat,
      a.proj_coff_mat_i, a.kx, a.ky, a.s_2, a.prop_re, a.prop_im, a.gfsf, a.height, a.width, a.depth, a.p_height,
      a.p_width, a.slices, a.step, a.begin_row, a.begin_col, a.width_red, a.sigma, a.w_num, a.aper_num,
      a.parameter, a.aper_true, a.mid_layer, a.layer_len, a.aper2, a.series_n_corr, a.series_n_i_corr,
      a.ele_n_corr, a.ele_n_i_corr, a.corr_info_matrix, a.cim_len, _ptr(res), _ptr(mid), _ptr(px), _ptr(py))
    if transmission:
        return (px[:n] + 1j * py[:n]).reshape(req.slices, req.p_height, req.p_width)
    return res[: req.aper_num * req.depth], mid[: req.aper_num * req.depth * len(req.mid_layer)]
