"""The shared-memory Stockham FFT plans of ``totem_b200/csrc/fft.cuh``, checked on the CPU.

Every plan in the header (the power-of-two ``Plan<N>`` specialisations and the mixed-radix
``TOTEM_PLAN`` rows) is parsed and its schedule executed in NumPy exactly as ``StageLoop`` lays
it out: thread j holds v[m] = x[j + m T]; stage s reads x[b + r N/R_s] for b = j + q T, applies
W_{Ns R}^{r (b mod Ns)}, a radix-R DFT, and writes position (b / Ns) Ns R + b mod Ns + r Ns into the
padded exchange buffer (one pad slot after every R_0 elements); the last stage's outputs land in
the entry layout.  The result must be the DFT (forward and inverse) of random data, and every
launch-shape constraint the kernels rely on must hold.
"""
import os
import re

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FFT_CUH = os.path.join(os.path.dirname(HERE), "totem_b200", "csrc", "fft.cuh")


def _plans():
    src = open(FFT_CUH).read()
    plans = {}
    spec = re.compile(r"template <> struct Plan<(\d+)> \{ static constexpr int P = (\d+), S = (\d+); "
                      r"static constexpr int R\[3\] = \{(\d+), (\d+), (\d+)\}; \};")
    for m in spec.finditer(src):
        n, p, s, *r = map(int, m.groups())
        plans.setdefault(n, (p, r[:s]))  # the first of an #if / #else pair is the alternative
    for m in re.finditer(r"^TOTEM_PLAN\((\d+), (\d+), (\d+), (\d+), (\d+), (\d+)\)", src, re.M):
        n, p, s, *r = map(int, m.groups())
        plans[n] = (p, r[:s])
    # the default 2048 plan is the #else branch (32 points per thread)
    m = re.search(r"#else\ntemplate <> struct Plan<2048> \{ static constexpr int P = (\d+), S = (\d+); "
                  r"static constexpr int R\[3\] = \{(\d+), (\d+), (\d+)\}; \};", src)
    if m:
        p, s, *r = map(int, m.groups())
        plans[2048] = (p, r[:s])
    return plans


def _mr_windows():
    src = open(FFT_CUH).read()
    out = []
    for part in "ABCD":
        m = re.search(rf"#define TOTEM_MR_WINDOWS_{part}\(X\)(.*)", src)
        out += [int(v) for v in re.findall(r"X\((\d+)\)", m.group(1))]
    return out


PLANS = _plans()


def _dft(x, inv):
    r = len(x)
    k = np.arange(r)
    return np.exp((1j if inv else -1j) * 2 * np.pi * np.outer(k, k) / r) @ x


def _stockham(x, n, inv):
    p, radices = PLANS[n]
    t = n // p
    r0 = radices[0]
    pad = lambda q: q + q // r0  # noqa: E731
    ns = [1]
    for r in radices[:-1]:
        ns.append(ns[-1] * r)
    v = np.array([[x[j + m * t] for m in range(p)] for j in range(t)], dtype=complex)
    sm = np.full(n + n // r0, np.nan, dtype=complex)
    for s, r in enumerate(radices):
        q_n = p // r
        if s == 0 and q_n > 1:  # entry layout v[q + r Q] -> stage layout v[q R + r]
            v = np.stack([np.array([v[j][q + rr * q_n] for q in range(q_n) for rr in range(r)]) for j in range(t)])
        for j in range(t):
            for q in range(q_n):
                b = j + q * t
                if ns[s] > 1:
                    k = b % ns[s]
                    v[j, q * r + 1:(q + 1) * r] *= np.exp((1j if inv else -1j) * 2 * np.pi * k * np.arange(1, r)
                                                          / (ns[s] * r))
                v[j, q * r:(q + 1) * r] = _dft(v[j, q * r:(q + 1) * r], inv)
        if s == len(radices) - 1:
            out = np.empty(n, dtype=complex)
            for j in range(t):
                for q in range(q_n):
                    for rr in range(r):
                        out[j + t * (q + rr * q_n)] = v[j, q * r + rr]
            return out
        for j in range(t):
            for q in range(q_n):
                b = j + q * t
                base = (b // ns[s]) * ns[s] * r + b % ns[s]
                for rr in range(r):
                    sm[pad(base + rr * ns[s])] = v[j, q * r + rr]
        rn = radices[s + 1]
        v = np.stack([np.array([sm[pad(j + q * t + rr * (n // rn))] for q in range(p // rn) for rr in range(rn)])
                      for j in range(t)])
        assert not np.isnan(v).any()


def test_every_window_has_a_plan():
    mr = _mr_windows()
    assert len(mr) == len(set(mr)) == 16
    for n in [64, 128, 256, 512, 1024, 2048, 4096] + mr:
        assert n in PLANS, n
    for n in mr:
        assert n % 16 == 0 and n & (n - 1), n  # multiples of 16 that are not powers of two


@pytest.mark.parametrize("n", sorted(PLANS))
def test_plan_schedule_is_the_dft(n):
    p, radices = PLANS[n]
    assert int(np.prod(radices)) == n and all(p % r == 0 for r in radices) and len(radices) <= 3
    t = n // p
    # launch shapes (ColCfg): a column tile of G columns x T threads is whole warps (G = 16 up to
    # 512, 8 above; mixed-radix edges halve it when the tile exceeds 256 threads and the half tile
    # does not); transform groups that do not divide a warp evenly synchronise the whole CTA
    g = 16 if n <= 512 else (8 if n <= 2048 else 2)
    if n & (n - 1) and g * t > 256 and (g // 2) * t <= 256:
        g //= 2
    assert (g * t) % 32 == 0 and n % g == 0
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    scale = np.abs(ref).max()
    assert np.abs(_stockham(x, n, False) - ref).max() < 1e-11 * scale
    assert np.abs(_stockham(x, n, True) - np.fft.ifft(x) * n).max() < 1e-11 * scale
