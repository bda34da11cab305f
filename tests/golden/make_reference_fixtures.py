"""Fixtures read from data files that ship with the reference (run where the reference tree is):

    python -m tests.golden.make_reference_fixtures [reference-dir]

* ``allresul_srtio3.npz`` from ``allresul.mat``: the specimen ToTem's slicing dialog saved
  (slicingdisplay.m:250-254: ``allresul.x_new``, ``eachthick``, ``slicethick``) and its STEM
  simulation loads (ToTEM_submit_v1.m:764-766): 791 atoms of a tilted SrTiO3 block, one row per
  atom ``Z x y z valence ionic-fraction B occupancy`` (the column meaning of
  getpotentialpara_lotabo_peng.m:13-14), slices of 0.823175 Angstrom, 41 slice tops.
* ``pydata_grid.npz`` from ``pydata.mat``: the reciprocal-space axes ``U`` (along columns) and
  ``V`` (along rows) of a 320 x 320 grid at 0.01 nm sampling that ToTem wrote for its batch
  HRTEM script, in nm^-1 (one row of ``U``, one column of ``V``; both arrays are meshgrids).

These are inputs the reference produced, not outputs of this repo's code; the tests feed them
through the slicing, the reciprocal-grid builder and the engine-vs-oracle comparison.
"""
import os
import sys

import numpy as np
import scipy.io as sio

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_dir: str):
    a = sio.loadmat(os.path.join(ref_dir, "allresul.mat"))["allresul"][0, 0]
    atoms = np.asarray(a["x_new"], dtype=np.float64)
    eachthick = float(np.asarray(a["eachthick"]).ravel()[0])
    slicethick = np.asarray(a["slicethick"], dtype=np.float64).ravel()
    np.savez(os.path.join(HERE, "allresul_srtio3.npz"), atoms=atoms, eachthick=eachthick, slicethick=slicethick)
    p = sio.loadmat(os.path.join(ref_dir, "pydata.mat"))
    U, V = np.asarray(p["U"], dtype=np.float64), np.asarray(p["V"], dtype=np.float64)
    assert np.array_equal(U, np.broadcast_to(U[0], U.shape)) and np.array_equal(V, np.broadcast_to(V[:, :1], V.shape))
    sampling_nm = float(np.asarray(p["para_part1"][0, 0]["sampling"]).ravel()[0])
    np.savez(os.path.join(HERE, "pydata_grid.npz"), u_axis=U[0], v_axis=V[:, 0], sampling_nm=sampling_nm)
    print(f"allresul: {atoms.shape[0]} atoms, eachthick {eachthick}, {len(slicethick)} slice tops; "
          f"pydata: {U.shape} grid at {sampling_nm} nm")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
