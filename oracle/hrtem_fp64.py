"""FP64 re-run of the HRTEM propagation on the GPU -- TEST INFRASTRUCTURE ONLY.

The precision sweep compares the engine's FP32 propagation (complex64 or bfloat16 transmission)
with the same propagation in FP64 (torch complex128 FFTs), from the same transmission stack, so
that the difference measured is the one the storage and arithmetic precision make.  It follows
the HRTEM loop of ToTEM_submit_v1.m:1341-1369 like ``stem_oracle.hrtem_exit_wave``, which is the
CPU oracle for small grids.  Only ``tests/`` import this module.
"""
from __future__ import annotations

import numpy as np


class _DeviceArray:
    """A raw device buffer seen through the CUDA array interface (the tests only read it)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_complex64(ptr: int, shape):
    import torch
    return torch.as_tensor(_DeviceArray(ptr, shape, "<c8"), device="cuda")


def hrtem_fp64(T, prop: np.ndarray, tf: np.ndarray | None = None, weights=None):
    """Plane wave through T (a torch complex64 [S, P, P] tensor on the GPU) in complex128.
    Returns (exit wave, image or None) as numpy arrays."""
    import torch
    dev = T.device
    H = torch.as_tensor(prop, dtype=torch.complex128, device=dev)
    psi = torch.ones(T.shape[1:], dtype=torch.complex128, device=dev)
    for k in range(T.shape[0]):
        psi = torch.fft.ifft2(torch.fft.fft2(psi * T[k].to(torch.complex128)) * H)
    img = None
    if tf is not None:
        spec = torch.fft.fft2(psi)
        img = torch.zeros(psi.shape, dtype=torch.float64, device=dev)
        for w, t in zip(weights, tf):
            u = torch.fft.ifft2(spec * torch.as_tensor(t, dtype=torch.complex128, device=dev))
            img += float(w) * (u.real ** 2 + u.imag ** 2)
        img = img.cpu().numpy()
    return psi.cpu().numpy(), img
