"""Serving layer on the host: the admission policy (FIFO within slots and an
HBM budget, continuous batching) on synthetic traces, the Philox block
function of the device generator, and the request byte estimate.  Needs
the library's host code only (no GPU)."""
import numpy as np
import pytest

import lowmachfhd_b200 as L


def _check_trace(slots, budget, arrive, nbytes, runtime, start):
    n = len(arrive)
    end = [s + r for s, r in zip(start, runtime)]
    for i in range(n):
        assert start[i] >= arrive[i] - 1e-12
        if i:
            assert start[i] >= start[i - 1] - 1e-12  # arrival order
    events = sorted(set(start) | set(end))
    for t in events:
        run = [i for i in range(n) if start[i] <= t < end[i]]
        assert len(run) <= slots
        assert sum(nbytes[i] for i in run) <= budget
    # work conservation: a request that waited started when it first could
    for i in range(n):
        t0 = max(arrive[i], start[i - 1] if i else 0.0)
        if start[i] > t0 + 1e-12:
            assert any(abs(start[i] - e) < 1e-12 for e in end)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_admission_policy(seed):
    rng = np.random.default_rng(seed)
    n, slots, budget = 200, 4, 1000
    arrive = np.cumsum(rng.exponential(0.05, n))
    nbytes = rng.integers(50, 600, n)
    runtime = rng.uniform(0.05, 0.5, n)
    start = L.sched_simulate(slots, budget, list(arrive), list(nbytes), list(runtime))
    _check_trace(slots, budget, list(arrive), list(nbytes), list(runtime), start)


def test_admission_small_trace():
    # 2 slots, 100 bytes: the second request waits for memory, the third
    # starts beside it, the fourth waits for a slot
    assert L.sched_simulate(2, 100, [0, 0, 0, 1], [60, 60, 30, 10], [1, 1, 1, 1]) == [0.0, 1.0, 1.0, 2.0]


def test_admission_refuses_oversized():
    with pytest.raises(L.FhdError):
        L.sched_simulate(2, 100, [0.0], [101], [1.0])


def _philox_py(ctr, key):
    """Philox-4x32-10 transcribed from Salmon et al., SC 2011"""
    M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    for _ in range(10):
        p0, p1 = M0 * c0, M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & 0xFFFFFFFF, p1 & 0xFFFFFFFF, ((p0 >> 32) ^ c3 ^ k1) & 0xFFFFFFFF, \
            p0 & 0xFFFFFFFF
        k0, k1 = (k0 + W0) & 0xFFFFFFFF, (k1 + W1) & 0xFFFFFFFF
    return [c0, c1, c2, c3]


def test_philox_block():
    rng = np.random.default_rng(5)
    for _ in range(200):
        ctr = [int(x) for x in rng.integers(0, 2 ** 32, 4, dtype=np.uint64)]
        key = [int(x) for x in rng.integers(0, 2 ** 32, 2, dtype=np.uint64)]
        assert L.philox4x32_10(ctr, key) == _philox_py(ctr, key)
    # uniformity of the words over consecutive counters
    words = np.array([L.philox4x32_10([j, 7, 3, 0], [11, 13]) for j in range(4000)], dtype=np.float64)
    u = words / 2.0 ** 32
    assert abs(u.mean() - 0.5) < 0.01
    assert abs(u.var() - 1.0 / 12) < 0.003


def test_request_bytes():
    small = L.Server.request_bytes(L.make_request(dim=3, n_cells=[32, 32, 32]))
    big = L.Server.request_bytes(L.make_request(dim=3, n_cells=[64, 64, 64]))
    fp64 = L.Server.request_bytes(L.make_request(dim=3, n_cells=[64, 64, 64], precision=L.FHD_PREC_FP64))
    assert small < big < fp64
    # about 8x the cells, plus a fixed reserve
    assert 6 * (small - (64 << 20)) < big - (64 << 20) < 10 * (small - (64 << 20))
