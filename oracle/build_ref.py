"""Recipe: the reference's own MEX shim, compiled unchanged and linked to this repo's libraries.

TEST INFRASTRUCTURE ONLY.  ToTem builds four MEX files from one shim, ``waveCuda.cpp`` with
``waveCuda.h`` (mex_cuda.m:29-37): ``waveCudalobato_<v>``, ``waveCudaPengAndCorr_<v>`` and the
transmission-only ``waveCudalobatoP_<v>`` / ``waveCudaPengAndCorrP_<v>``, each linked to one
``cuda_source_*`` object that defines ``myProjectfun``.  This recipe compiles the same two
reference files, read where they lie in the reference tree and not copied, against the stand-in
``mex.h`` in ``tests/mex_stub`` and links each MEX build to the corresponding library of this
repo (``libwaveCuda{Lobato,Peng,LobatoP,PengP}.so``) instead of the reference's CUDA objects,
with ``--no-undefined``: every symbol the shim needs must come from this repo's libraries.

Outputs go to ``oracle/_ref/mex_<name>.so`` only.  Nothing in the product loads them; the tests
call their ``mexFunction`` with 41 stand-in MATLAB arrays.

    python -m oracle.build_ref [reference-dir]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
STUB = os.path.join(ROOT, "tests", "mex_stub")
LIB = os.path.join(ROOT, "totem_b200", "lib")
REFERENCE_DIR = "/root/reference"

# MEX name (mex_cuda.m:29-37) -> this repo's myProjectfun library
FLAVOURS = {
    "waveCudalobato": "libwaveCudaLobato.so",
    "waveCudaPengAndCorr": "libwaveCudaPeng.so",
    "waveCudalobatoP": "libwaveCudaLobatoP.so",
    "waveCudaPengAndCorrP": "libwaveCudaPengP.so",
}


def mex_path(name: str, out_dir: str = OUT) -> str:
    return os.path.join(out_dir, f"mex_{name}.so")


def build(ref_dir: str = REFERENCE_DIR, out_dir: str = OUT) -> list[str] | None:
    """Compile the four MEX builds; None when the reference's shim is not present."""
    src = os.path.join(ref_dir, "waveCuda.cpp")
    if not os.path.exists(src) or not os.path.exists(os.path.join(ref_dir, "waveCuda.h")):
        return None
    os.makedirs(out_dir, exist_ok=True)
    outs = []
    for name, lib in FLAVOURS.items():
        out = mex_path(name, out_dir)
        deps = [src, os.path.join(STUB, "mex.h"), os.path.join(STUB, "mex_stub.cpp"), os.path.join(LIB, lib)]
        if not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps):
            rel = os.path.relpath(LIB, out_dir)
            cmd = ["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-I", STUB, "-I", ref_dir, src,
                   os.path.join(STUB, "mex_stub.cpp"), "-o", out, "-L", LIB, f"-l:{lib}",
                   f"-Wl,-rpath,$ORIGIN/{rel}", "-Wl,--no-undefined"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("MEX shim build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        outs.append(out)
    return outs


if __name__ == "__main__":
    built = build(sys.argv[1] if len(sys.argv) > 1 else REFERENCE_DIR)
    print("\n".join(built) if built else "reference shim not found: nothing built")
