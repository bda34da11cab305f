"""Extract the scattering-factor parameter tables from the reference's MATLAB data files.

The reference keeps its tables as MATLAB source:
  * ``Lobato_para.m:4-316``  -- Lobato & Van Dyck (2014) neutral-atom parameters, Z = 1..103,
    two text rows per element (a1..a5, then b1..b5), assembled at ``Lobato_para.m:311-316``.
  * ``ABSFpara.m:5-222``     -- Peng et al. neutral-atom parameters, Z = 1..98, one row
    ``a1..a5 b1..b5`` per element.
  * ``ABSFpara.m:224-441``   -- Peng ionic parameters, rows ``Z valence a1..a5 b1..b5``.

This script parses those numbers (it does not retype them) and writes ``scattering_tables.npz``
next to itself.  It is run once, in a checkout that has the reference sources, with

    python -m totem_b200.data.extract_tables /path/to/reference

The generated ``.npz`` is committed because the GPU hosts that run the engine do not carry the
reference tree.
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

_NUM = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?")


def _strip_comment(line: str) -> str:
    i = line.find("%")
    return line if i < 0 else line[:i]


def _block(text: str, name: str) -> list[list[float]]:
    """Numbers of the MATLAB matrix literal ``name=[ ... ];`` as rows (one per text line)."""
    m = re.search(r"\b" + name + r"\s*=\s*\[", text)
    if m is None:
        raise ValueError(f"matrix {name} not found")
    start = m.end()
    end = text.index("]", start)
    rows = []
    for raw in text[start:end].splitlines():
        nums = _NUM.findall(_strip_comment(raw).replace("...", " "))
        if nums:
            rows.append([float(v) for v in nums])
    return rows


def parse_lobato(path: str) -> np.ndarray:
    text = open(path, encoding="latin-1").read()
    rows = _block(text, "para")
    if len(rows) % 2 or any(len(r) != 5 for r in rows):
        raise ValueError("unexpected Lobato table shape")
    a = np.array(rows[0::2])
    b = np.array(rows[1::2])
    return np.concatenate([a, b], axis=1)  # (Z, 10): a1..a5 b1..b5 (Lobato_para.m:313-314)


def parse_peng(path: str) -> tuple[np.ndarray, np.ndarray]:
    text = open(path, encoding="latin-1").read()
    neutral = np.array(_block(text, "PengPara"))
    ions = np.array(_block(text, "PengIon"))
    if neutral.shape[1] != 10 or ions.shape[1] != 12:
        raise ValueError("unexpected Peng table shape")
    return neutral, ions


def main(ref_dir: str) -> str:
    lobato = parse_lobato(os.path.join(ref_dir, "Lobato_para.m"))
    peng, peng_ion = parse_peng(os.path.join(ref_dir, "ABSFpara.m"))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scattering_tables.npz")
    np.savez(out, lobato=lobato, peng=peng, peng_ion=peng_ion)
    print(f"lobato {lobato.shape}  peng {peng.shape}  peng_ion {peng_ion.shape} -> {out}")
    return out


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python -m totem_b200.data.extract_tables <directory holding Lobato_para.m and ABSFpara.m>")
    main(sys.argv[1])
