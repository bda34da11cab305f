"""Serving scheduler: the admission policy (``totem_plan_simulate``, no device needed) against a
plain-Python restatement of the same rules, plus its invariants and the API's error paths."""
import numpy as np
import pytest

from totem_b200 import capi


def _policy_model(n, items, slices, arrive, wave, chunk, policy):
    """The admission rules of the scheduler, restated: every tick, requests in arrival order (FIFO)
    or by least remaining work (SHORTEST) start up to ``chunk`` bytes of probes while the bytes in
    flight stay within ``wave``; FIFO does not let a later request overtake one that cannot start;
    a probe larger than ``wave`` starts alone."""
    cnt = len(n)
    chunk = chunk or wave // 4
    ib = [n[i] * n[i] * 8 for i in range(cnt)]
    order = sorted(range(cnt), key=lambda i: arrive[i])
    pending, active = [], []   # pending: [id, next]; active: (id, items, last_tick, bytes)
    first, done = [-1] * cnt, [-1] * cnt
    left = list(items)
    inflight = mx = 0
    added, remaining, tick = 0, cnt, 0
    while remaining:
        while added < cnt and arrive[order[added]] <= tick:
            i = order[added]
            added += 1
            if items[i] == 0:
                first[i] = done[i] = tick
                remaining -= 1
            else:
                pending.append([i, 0])
        visit = list(range(len(pending)))
        if policy == capi.SCHED_SHORTEST:
            visit.sort(key=lambda k: (items[pending[k][0]] - pending[k][1]) * slices[pending[k][0]])
        for k in visit:
            i, nxt = pending[k]
            free = max(wave - inflight, 0)
            if free >= ib[i]:
                cap = max(1, min(free, chunk) // ib[i])
            elif inflight == 0 and ib[i] > wave:
                cap = 1
            else:
                cap = 0
            take = min(cap, items[i] - nxt, 1 << 20)
            if take <= 0:
                if policy == capi.SCHED_FIFO:
                    break
                continue
            pending[k][1] += take
            active.append((i, take, tick + slices[i] - 1, take * ib[i]))
            inflight += take * ib[i]
            if first[i] < 0:
                first[i] = tick
        pending = [p for p in pending if p[1] < items[p[0]]]
        mx = max(mx, inflight)
        keep = []
        for g in active:
            if g[2] <= tick:
                inflight -= g[3]
                left[g[0]] -= g[1]
                if left[g[0]] == 0:
                    done[g[0]] = tick
                    remaining -= 1
            else:
                keep.append(g)
        active = keep
        tick += 1
    return np.array(first), np.array(done), mx


def _random_case(rng, count):
    n = rng.choice([64, 128, 256, 512], size=count)
    items = rng.integers(0, 300, size=count)
    slices = rng.integers(1, 40, size=count)
    arrive = np.sort(rng.integers(0, 60, size=count))
    return n, items, slices, arrive


@pytest.mark.parametrize("policy", [capi.SCHED_FIFO, capi.SCHED_SHORTEST])
@pytest.mark.parametrize("seed", range(4))
def test_policy_matches_restatement(policy, seed):
    rng = np.random.default_rng(seed)
    n, items, slices, arrive = _random_case(rng, 40)
    wave = int(rng.integers(40, 400)) * 256 * 256 * 8
    chunk = int(rng.integers(0, 3)) * wave // 8
    f, d, mx = capi.plan_simulate(n, items, slices, arrive, wave, chunk, policy)
    rf, rd, rmx = _policy_model(list(n), list(items), list(slices), list(arrive), wave, chunk, policy)
    np.testing.assert_array_equal(f, rf)
    np.testing.assert_array_equal(d, rd)
    assert mx == rmx


@pytest.mark.parametrize("policy", [capi.SCHED_FIFO, capi.SCHED_SHORTEST])
def test_invariants(policy):
    rng = np.random.default_rng(11)
    n, items, slices, arrive = _random_case(rng, 200)
    wave = 300 * 512 * 512 * 8
    f, d, mx = capi.plan_simulate(n, items, slices, arrive, wave, 0, policy)
    assert mx <= wave
    assert np.all(f >= arrive)
    nz = items > 0
    # every probe runs all its slices: a request lasts at least its slice count
    assert np.all(d[nz] - f[nz] >= slices[nz] - 1)
    assert np.all(d[~nz] == f[~nz])


def test_fifo_keeps_arrival_order():
    n = [256] * 6
    items = [50, 400, 3, 20, 1, 90]
    slices = [10, 30, 5, 8, 40, 3]
    arrive = [0, 0, 1, 1, 2, 2]
    f, d, _ = capi.plan_simulate(n, items, slices, arrive, 100 * 256 * 256 * 8, 0, capi.SCHED_FIFO)
    assert list(f) == sorted(f)


def test_shortest_lets_small_requests_through():
    # a large request occupies the waves; a 1-probe request arriving later finishes far earlier
    # under SHORTEST than under FIFO
    n, items, slices, arrive = [512, 512], [4000, 1], [100, 20], [0, 5]
    wave = 256 * 512 * 512 * 8
    _, d_fifo, _ = capi.plan_simulate(n, items, slices, arrive, wave, 0, capi.SCHED_FIFO)
    _, d_short, _ = capi.plan_simulate(n, items, slices, arrive, wave, 0, capi.SCHED_SHORTEST)
    assert d_short[1] < d_fifo[1]
    assert d_short[1] - arrive[1] < 200


def test_oversize_probe_runs_alone():
    f, d, mx = capi.plan_simulate([2048, 64], [2, 10], [5, 5], [0, 0], 1 << 20, 0, capi.SCHED_FIFO)
    assert mx == 2048 * 2048 * 8
    assert d[0] == 9 and f[1] == 10


def test_simulate_rejects_bad_input():
    with pytest.raises(capi.TotemError) as e:
        capi.plan_simulate([64], [1], [0], [0], 1 << 20)
    assert e.value.code == capi.ERR_INVALID_ARG
    with pytest.raises(capi.TotemError):
        capi.plan_simulate([64], [1], [1], [0], 1 << 20, policy=7)


def test_server_needs_a_device(engine_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    with pytest.raises(capi.TotemError) as e:
        capi.Server()
    assert e.value.code == capi.ERR_NO_DEVICE
