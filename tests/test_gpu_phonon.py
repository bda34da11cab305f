"""Frozen-phonon STEM: configurations batched through the serving scheduler against one blocking
call per configuration (bit-identical sums) and against the FP64 oracle."""
import numpy as np
import pytest

from oracle import stem_oracle as so
from tests.conftest import rel_l2
from totem_b200 import phonon, request

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _configs(count):
    return [request.build_srtio3_stem(cells=(3, 3, 3), n=64, p=128, sampling=0.1, step=4, raster=(2, 3),
                                      mid_layer=(3,), phonon_seed=s) for s in range(count)]


def test_batched_configurations_equal_sequential_and_oracle(engine_lib):
    configs = _configs(3)
    res_b, mid_b = phonon.frozen_phonon(configs)
    res_s, mid_s = phonon.frozen_phonon_sequential(configs)
    assert np.array_equal(res_b, res_s) and np.array_equal(mid_b, mid_s)
    ref_res = ref_mid = 0
    for c in configs:
        r, m = so.stem(c, so.transmission(c))
        ref_res, ref_mid = ref_res + r, ref_mid + m
    assert rel_l2(res_b, ref_res) < TOL
    assert rel_l2(mid_b, ref_mid) < TOL


def test_configurations_differ(engine_lib):
    a, b = _configs(2)
    assert not np.array_equal(a.ele_n[:, :2], b.ele_n[:, :2])
