"""The C ABI: the library loads, exports what the header declares, and its struct layouts match
the ctypes binding.  No GPU is needed; on a machine without one the entry points must fail with
TOTEM_ERR_NO_DEVICE and a message instead of crashing."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from totem_b200 import build, capi


@pytest.fixture(scope="module")
def lib():
    build.build()
    return capi.load()


def test_exports_every_header_function(lib):
    names = capi.header_functions()
    assert "totem_stem_run" in names and "totem_stem_slices_noalloc" in names
    for n in names:
        assert hasattr(lib, n), n


def test_myprojectfun_shims_export_reference_symbol(lib):
    for key, name in capi.SHIM_LIBS.items():
        path = os.path.join(capi.LIB_DIR, name)
        out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
        assert capi.MYPROJECTFUN_MANGLED in out, name
        l = capi.myprojectfun_lib(*key)
        assert getattr(l, capi.MYPROJECTFUN_MANGLED)


def test_mangled_name_is_the_reference_signature(tmp_path):
    # compile the reference's declaration (waveCuda.h:10-21, restated in include/totem_b200.h) and
    # check that g++ mangles it to the symbol the shims export
    src = tmp_path / "m.cpp"
    src.write_text('#include "totem_b200.h"\nvoid (*keep)(double*, double*, double*, double*, double*, double*, double*,'
                   ' double*, double*, double*, double*, double*, double*, double*, double*, int, int, int, int, int,'
                   ' int, int, int, int, int, double, int, int, double, double*, int*, int, double*, double*,'
                   ' double*, double*, double*, double*, int, double*, double*, double*, double*) = &myProjectfun;\n')
    obj = tmp_path / "m.o"
    subprocess.run(["g++", "-c", "-I", os.path.dirname(capi.HEADER), str(src), "-o", str(obj)], check=True)
    syms = subprocess.run(["nm", str(obj)], capture_output=True, text=True).stdout
    assert capi.MYPROJECTFUN_MANGLED in syms


def _c_layout(tmp_path, struct, fields):
    body = "\n".join(f'printf("%s %zu\\n", "{f}", offsetof({struct}, {f}));' for f in fields)
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "totem_b200.h"\nint main(void){\n'
                   f'printf("sizeof %zu\\n", sizeof({struct}));\n{body}\nreturn 0;}}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.dirname(capi.HEADER), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    return dict((ln.split()[0], int(ln.split()[1])) for ln in out if ln.strip())


@pytest.mark.parametrize("cls", [capi.TotemStemArgs, capi.TotemStemOut, capi.TotemRunOptions, capi.TotemTiming,
                                 capi.TotemServerOptions])
def test_struct_layout_matches_header(tmp_path, cls):
    names = [f[0] for f in cls._fields_]
    c = _c_layout(tmp_path, cls.__name__, names)
    assert c["sizeof"] == C.sizeof(cls)
    for n in names:
        assert c[n] == getattr(cls, n).offset, n


def test_status_strings(lib):
    for code in range(8):
        s = lib.totem_status_string(code).decode()
        assert s and s != "unknown status"
    assert lib.totem_status_string(99).decode() == "unknown status"
    assert lib.totem_abi_version() == 4


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the behaviour without a CUDA device")
def test_no_device_is_an_error_not_a_crash(lib):
    from totem_b200 import request
    req = request.build_small_stem(n=64, p=128, raster=(1, 2), slices=2)
    with pytest.raises(capi.TotemError) as e:
        capi.stem_run(req)
    assert e.value.code == capi.ERR_NO_DEVICE
    assert "device" in lib.totem_last_error().decode().lower()
    h = C.c_void_p()
    assert lib.totem_session_create(-1, None, C.byref(h)) == capi.ERR_NO_DEVICE
    a, b = C.c_double(), C.c_double()
    assert lib.totem_fp32_peak(0, C.byref(a), C.byref(b)) == capi.ERR_NO_DEVICE
    one = request.build_small_stem(n=64, p=128, raster=(1, 1), slices=2)
    with pytest.raises(capi.TotemError) as e:
        capi.cbed_run(one)
    assert e.value.code == capi.ERR_NO_DEVICE


def test_null_arguments_are_rejected(lib):
    assert lib.totem_session_create(0, None, None) == capi.ERR_INVALID_ARG
    assert lib.totem_fp32_peak(0, None, None) == capi.ERR_INVALID_ARG
    assert lib.totem_session_cbed(None, None) == capi.ERR_INVALID_ARG
    assert lib.totem_session_upload(None, None) == capi.ERR_INVALID_ARG
    assert lib.totem_session_run(None, 0, None) == capi.ERR_INVALID_ARG
    assert lib.totem_session_destroy(None) == capi.OK


def test_builder_choice_is_validated(lib):
    # a process-wide setting: no device needed
    assert lib.totem_set_tx_builder(7, 0) == capi.ERR_INVALID_ARG
    assert lib.totem_set_tx_builder(capi.TX_GRIDDING, 1 << 20) == capi.OK
    assert lib.totem_set_tx_builder(capi.TX_AUTO, 0) == capi.OK


def test_slice_graph_switch_is_validated(lib):
    assert lib.totem_set_slice_graphs(2) == capi.ERR_INVALID_ARG
    assert lib.totem_set_slice_graphs(0) == capi.OK
    assert lib.totem_set_slice_graphs(1) == capi.OK


def test_noalloc_rejects_2048_windows_before_any_device_call(lib):
    # one 2048^2 probe would need the whole fixed scratch array: refused while validating the
    # arguments, before the entry point touches a device (so this runs without a GPU)
    fake = C.c_void_p(256)
    rc = lib.totem_stem_slices_noalloc(fake, 4096, 4096, 2, fake, 1, fake, fake, 2, 2048, 8, 0, 0, 1, 1, 0, 1,
                                       fake, None)
    assert rc == capi.ERR_UNSUPPORTED
    assert "1024" in lib.totem_last_error().decode()


def test_failure_injection_arguments(lib):
    assert lib.totem_inject_failures(C.c_longlong(-2), 0) == capi.ERR_INVALID_ARG
    assert lib.totem_inject_failures(C.c_longlong(-1), -1) == capi.ERR_INVALID_ARG
    assert lib.totem_inject_failures(C.c_longlong(-1), 0) == capi.OK
