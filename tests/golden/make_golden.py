"""Generate the oracle's golden fixtures: ``python -m tests.golden.make_golden``.

Each fixture stores the inputs the oracle sees (probe, coefficient rows, propagator, masks), the
transmission stack and the detector outputs of one small seeded request.  They pin the oracle
and the input builders against unintended change; they are not reference outputs (the reference
publishes none and its MATLAB path cannot run here).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

CASES = {
    "peng_small": dict(flag="p", n=64, p=128, raster=(3, 4), step=5, slices=6, mid_layer=(2, 4)),
    "lobato_spread": dict(flag="l", n=64, p=128, raster=(2, 3), step=7, slices=4, mid_layer=(3,), focal_steps=3),
}


def build_case(kw):
    from totem_b200 import request
    return request.build_small_stem(**kw)


def main():
    from oracle import stem_oracle as so
    here = os.path.dirname(os.path.abspath(__file__))
    for name, kw in CASES.items():
        req = build_case(kw)
        T = so.transmission(req)
        res, mid = so.stem(req, T)
        np.savez_compressed(os.path.join(here, f"{name}.npz"), probe=req.probe, ele_n=req.ele_n, prop=req.prop,
                            aper=req.aper, T=T, result=res, mid=mid)
        print(name, res[:3])


if __name__ == "__main__":
    main()
