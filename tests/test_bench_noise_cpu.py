"""The bench's stochastic inputs.  Stochastic fields must be fresh every
step: replaying a ring of two noise sets makes the species densities drift
linearly in the step count instead of as a random walk, and at 256^3 the
tails of the 4-species workload then reach zero density within about 40
steps.  Checked on the CPU oracle at a small grid, plus the window
arithmetic of the end-to-end leg's host noise pool."""
import numpy as np
import pytest

import bench


def _spread(n, steps, ring):
    oc = bench.OracleCase(n)
    rho0 = np.array(oc.rho)
    if ring:
        # replay two noise sets, as an alternating two-set ring would
        fresh = oc.noise
        oc.noise = lambda k: fresh(1 + k % 2)
        oc.mass_noise = lambda k: bench.OracleCase.mass_noise(oc, 1 + k % 2)
    for k in range(1, steps + 1):
        oc.step(k)
    rho = np.array(oc.rho)
    return float(np.std(rho - rho0)), float(rho.min())


def test_two_set_ring_drifts_fresh_noise_diffuses():
    s_ring, _ = _spread(16, 24, ring=True)
    s_fresh, m_fresh = _spread(16, 24, ring=False)
    # linear against square-root growth: about sqrt(24/2) apart after 24 steps
    assert s_ring > 2.5 * s_fresh, (s_ring, s_fresh)
    assert m_fresh > 0.15


@pytest.mark.parametrize("n,steps", [(256, 25), (256, 200), (64, 60), (128, 20), (48, 30)])
def test_host_pool_windows_are_fresh(n, steps):
    """two (field, step) windows of the pool never start at offsets that
    differ, modulo the field size, by zero or by the offset of a periodic
    neighbour cell (x, y, z shifts in {-1, 0, 1}): no cell sees a pool element
    that it or a neighbour saw in another step or field"""
    nc = n ** 3
    stride = bench.pool_stride(n, steps)
    assert stride % 512 == 0  # 4 KiB-aligned windows
    near = bench.neighbour_shifts(n)
    for nf in (3, 3 + 3 * bench.NSPECIES):
        offs = [(f, i, f * nc + i * stride) for f in range(nf) for i in range(steps + 1)]
        for f, i, o in offs[:: max(1, len(offs) // 200)]:
            for g, j, o2 in offs:
                if i != j:  # one step's fields are disjoint windows
                    assert (o - o2) % nc not in near, (f, i, g, j)
