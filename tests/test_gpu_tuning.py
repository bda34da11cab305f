"""The autotuner's table on the GPU: its pick is within 3 % of the best hand configuration
(the built-in defaults and the variants measured by hand) at 512^2, 1024^2 and 2048^2 windows,
and the engine applies the table to runs that leave the launch shapes at 0."""
import json

import pytest

from totem_b200 import capi, request, tune

pytestmark = pytest.mark.gpu

# hand configurations (row_variant, col_variant, batch MiB) tried before the tuner existed
HAND = {512: [(1, 1, 4096), (4, 1, 4096), (1, 5, 4096), (1, 2, 4096), (1, 6, 4096)],
        1024: [(1, 1, 4096), (5, 1, 4096), (1, 5, 4096), (1, 2, 4096)],
        2048: [(1, 1, 4096), (4, 1, 4096), (1, 5, 4096)]}


def _entry(n):
    name = tune.device_name(0)
    for line in open(capi.TUNING_FILE):
        d = json.loads(line)
        if d["device"] == name and d["n"] == n:
            return d
    pytest.skip(f"no tuning entry for {name} at {n}")


@pytest.mark.parametrize("n", [512, 1024, 2048])
def test_tuned_pick_within_3_percent_of_best_hand_configuration(engine_lib, n):
    e = _entry(n)
    assert capi.tuned_config(n) == (e["row_variant"], e["col_variant"], int(e["batch_mib"] * 2 ** 20))
    tm = tune.Timer(tune.workload(n), reps=3)
    try:
        hand = min(tm(*c) for c in HAND[n])
        pick = tm(e["row_variant"], e["col_variant"], e["batch_mib"])
    finally:
        tm.close()
    print(f"n={n}: tuned {pick:.4f} us, best hand {hand:.4f} us per probe*slice")
    assert pick <= 1.03 * hand, (pick, hand)


def test_engine_applies_the_table(engine_lib, tmp_path):
    req = request.build_small_stem(raster=(3, 3))
    path = tmp_path / "t.jsonl"
    # 1/16 MiB of waves: two 64^2 probes per batch (the 9 probes run in 5 batches of at most 2)
    path.write_text(json.dumps({"device": tune.device_name(0), "n": req.height, "row_variant": 4, "col_variant": 5,
                                "batch_mib": 0.0625}) + "\n")
    try:
        assert capi.load_tuning(str(path)) == 1
        s = capi.Session(device=0)
        s.upload(req)
        s.run()
        res, mid, _ = s.download()
        t = s.timing()
        assert (t.row_variant, t.col_variant) == (4, 5)
        assert t.batch == 2
        s.run(col_variant=1, batch=9)  # explicit options win
        t = s.timing()
        assert (t.row_variant, t.col_variant, t.batch) == (4, 1, 9)
        capi.load_tuning(None)
        s.run()
        res2, mid2, _ = s.download()
        assert s.timing().col_variant == 1
        s.close()
        # 8-column tiles regroup the FP64 detector sums: equal to rounding
        import numpy as np
        np.testing.assert_allclose(res, res2, rtol=1e-12)
        np.testing.assert_allclose(mid, mid2, rtol=1e-12)
    finally:
        capi.load_tuning(capi.TUNING_FILE)


def test_fp32_peak_is_measured(engine_lib):
    # B200: 148 SMs x 128 FP32 lanes x 2 flops at 1.3-2.0 GHz, i.e. about 50-75 TFLOP/s of scalar
    # FFMA; packed FFMA2 at most twice that
    ffma, ffma2 = capi.fp32_peak(0)
    assert 20.0 < ffma < 200.0, ffma
    assert 20.0 < ffma2 < 400.0, ffma2
    with pytest.raises(capi.TotemError) as e:
        capi.fp32_peak(99)
    assert e.value.code == capi.ERR_INVALID_ARG
