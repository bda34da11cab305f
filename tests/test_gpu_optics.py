"""Transfer functions on the device (``totem_tcc_stack``, FP64) against the NumPy restatement of
WholeTCC2D_newTEM, with every aberration coefficient non-zero so each term is exercised."""
import numpy as np
import pytest

from totem_b200 import optics

pytestmark = pytest.mark.gpu


def _spec(seed):
    rng = np.random.default_rng(seed)
    names = [f for f in optics.Aberrations.__dataclass_fields__]
    vals = {}
    for f in names:
        if f.startswith("phi"):
            vals[f] = float(rng.uniform(-180, 180))
        else:
            vals[f] = float(rng.uniform(-1, 1)) * {"focus": 20.0, "Cs": 2e4, "C5": 1e6}.get(f, 50.0)
    return optics.ProbeSpec(kv=200.0, semi_angle_mrad=25.0, aberrations=optics.Aberrations(**vals),
                            convergence_mrad=0.3, focal_spread_nm=3.0, focal_steps=5)


@pytest.mark.parametrize("seed,n,grad", [(0, 128, True), (1, 256, False), (2, 96, True)])
def test_tcc_stack_engine_matches_numpy(engine_lib, seed, n, grad):
    spec = _spec(seed)
    ref, w_ref = optics.tcc_stack(spec, n, 0.1, with_gradient=grad)
    got, w_got = optics.tcc_stack(spec, n, 0.1, with_gradient=grad, engine=True)
    assert np.array_equal(w_ref, w_got)
    assert np.max(np.abs(got - ref)) < 1e-7


def test_stem_probes_engine(engine_lib):
    spec = _spec(3)
    p_ref, _ = optics.stem_probes(spec, 128, 0.1)
    p_got, _ = optics.stem_probes(spec, 128, 0.1, engine=True)
    assert np.max(np.abs(p_got - p_ref)) < 1e-7
