"""The gridding transmission builder's batch plan (``totem_grid_batches``), host logic only: on
random job tables every job runs exactly once, in order, and every slice is written once by the
batch holding its first job (or, for a slice without jobs, by exactly one batch) before any
batch adds to it."""
import numpy as np
import pytest

from totem_b200 import build, capi


@pytest.fixture(scope="module")
def lib():
    build.build()
    return capi.load()


def _check(job_beg, per_batch):
    b = capi.grid_batches(job_beg, per_batch)
    slices, total = len(job_beg) - 1, int(job_beg[-1])
    assert len(b) >= 1
    # job ranges partition [0, total) in order, none larger than per_batch
    assert b[0, 2] == 0 and b[-1, 3] == total
    assert np.all(b[1:, 2] == b[:-1, 3])
    assert np.all(b[:, 3] - b[:, 2] <= per_batch)
    # slice ranges advance, cover every slice, and overlap only in a continued slice
    assert b[0, 0] == 0 and b[-1, 1] == slices
    written = np.zeros(slices, dtype=int)
    seen_jobs = np.zeros(total, dtype=int)
    for s_lo, s_hi, j_lo, j_hi in b:
        assert s_lo < s_hi
        for s in range(s_lo, s_hi):
            lo, hi = max(job_beg[s], j_lo), min(job_beg[s + 1], j_hi)
            add = job_beg[s] < j_lo
            if add:
                assert written[s] == 1, "added to a slice before it was written"
            else:
                assert written[s] == 0, "slice written twice"
                written[s] = 1
            seen_jobs[lo:hi] += 1
    assert np.all(written == 1)
    assert np.all(seen_jobs == 1)


def test_plan_examples(lib):
    _check([0, 3, 6, 9], 1)            # every slice split, last one too
    _check([0, 3, 6, 9], 2)
    _check([0, 0, 2, 2, 5, 5], 1)      # vacuum slices between, before and after
    _check([0, 0, 0], 4)               # no jobs at all: one batch writes zeros
    _check([0, 7], 3)                  # one slice, three batches


def test_plan_random(lib):
    rng = np.random.default_rng(0)
    for _ in range(300):
        slices = int(rng.integers(1, 40))
        counts = rng.integers(0, 5, size=slices)
        counts[rng.random(slices) < 0.2] = 0
        job_beg = np.concatenate([[0], np.cumsum(counts)])
        _check(job_beg, int(rng.integers(1, 12)))


def test_plan_rejects_bad_tables(lib):
    with pytest.raises(capi.TotemError):
        capi.grid_batches([0, 3, 2], 2)
    with pytest.raises(capi.TotemError):
        capi.grid_batches([0, 1], 0)
