"""Build the engine's shared libraries in-tree with nvcc for sm_100a.

Outputs (``totem_b200/lib/``):
  * ``libtotem_b200.so``   -- kernels, runtime and the C ABI of ``include/totem_b200.h``
  * ``libwaveCudaPeng.so``, ``libwaveCudaLobato.so``, ``libwaveCudaPengP.so``,
    ``libwaveCudaLobatoP.so`` -- the reference's ``myProjectfun`` entry point (C++ linkage), one
    library per MEX flavour, each linked against ``libtotem_b200.so``.

Usage: ``python -m totem_b200.build [--force]``.  Objects are rebuilt when a source or header is
newer than them.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(LIB, "obj")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler",
                     "-fvisibility=hidden", "--expt-relaxed-constexpr", "-I", INCLUDE]
CU_SOURCES = ["util.cu", "transmission.cu", "multislice.cu", "rowpass.cu", "groups.cu",
              "windows_mr_a.cu", "windows_mr_b.cu", "windows_mr_c.cu", "windows_mr_d.cu", "hrtem.cu", "optics.cu", "plain.cu", "engine.cu",
              "noalloc.cu", "server.cu", "specimen.cpp"]
SHIMS = {  # library name -> (param flag, transmission flag)
    "libwaveCudaPeng.so": (0, 0),
    "libwaveCudaLobato.so": (1, 0),
    "libwaveCudaPengP.so": (0, 1),
    "libwaveCudaLobatoP.so": (1, 1),
}
CORE = os.path.join(LIB, "libtotem_b200.so")


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "totem_b200.h"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _compile(src, force, extra=()):
    obj = os.path.join(OBJ, os.path.splitext(os.path.basename(src))[0] + ".o")
    if force or _stale(obj, [src] + _headers()):
        _run([NVCC, *NVCC_FLAGS, *extra, "-c", src, "-o", obj])
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(CORE, objs):
        # static cudart: the library does not depend on which CUDA runtime the host process loaded
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", CORE, *objs,
              "-L", os.path.join(CUDA_HOME, "lib64"), "-lcufft", "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")])
    shim_src = os.path.join(CSRC, "myprojectfun.cpp")
    for name, (param, trans) in SHIMS.items():
        out = os.path.join(LIB, name)
        if force or _stale(out, [shim_src, CORE, os.path.join(INCLUDE, "totem_b200.h")]):
            _run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", f"-DTOTEM_SHIM_PARAM={param}",
                  f"-DTOTEM_SHIM_TRANSMISSION={trans}", "-I", INCLUDE, shim_src, "-o", out,
                  "-L", LIB, "-ltotem_b200", "-Wl,-rpath,$ORIGIN"])
    if verbose:
        print("built", CORE)
    return CORE


def ptxas_report() -> str:
    """Registers / spills / shared memory of every kernel (nvcc -Xptxas -v)."""
    out = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        r = subprocess.run([NVCC, *NVCC_FLAGS, "-Xptxas", "-v", "-c", src, "-o", os.devnull],
                           capture_output=True, text=True)
        out.append(r.stderr)
    return "\n".join(out)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true")
    ns = ap.parse_args()
    if ns.ptxas:
        print(ptxas_report())
    else:
        build(ns.force, verbose=True)
        sys.exit(0)
