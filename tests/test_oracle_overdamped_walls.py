"""The oracle's overdamped step (advance_timestep_overdamped.f90:135-734) with
homogeneous walls: exact properties of the step, which the reference's stored
results (periodic or inhomogeneous walls) do not cover:
  * each species' total mass is conserved (no mass or advective flux through
    a wall face);
  * the normal velocity stays zero on the wall faces."""
import numpy as np
import pytest

import oracle as O
from tests.test_oracle_multispecies import mass_fields, mix, state
from tests.test_oracle_stoch_walls import edge_shape

NS, SL, PE = O.NO_SLIP_WALL, O.SLIP_WALL, -1


@pytest.fixture(autouse=True)
def periodic_afterwards():
    yield
    O.set_walls()


def inputs(dim, n, ns, bc_lo, seed=3):
    """seeded inputs of one overdamped step with walls: constant viscosity
    (visc_type 1), edge arrays with the high wall's planes, normal velocity
    zero on the wall faces"""
    nc = int(np.prod(n[:dim]))
    nE = 1 if dim == 2 else 3
    rng = np.random.default_rng(seed)
    ne = [int(np.prod(edge_shape(dim, n, e, bc_lo))) for e in range(nE)]
    shape = [n[d] for d in reversed(range(dim))]
    u = []
    for c in range(dim):
        a = (1e-2 * rng.standard_normal(nc)).reshape(shape)
        if bc_lo[c] != PE:
            idx = [slice(None)] * dim
            idx[dim - 1 - c] = 0
            a[tuple(idx)] = 0.0
        u.append(a.ravel())
    W_ed = []
    for r in range(2):
        for e in range(nE):
            a = rng.standard_normal(ne[e])
            W_ed += [a, a.copy()]
    mp = mix(ns) if ns > 1 else None
    return dict(
        u=u, rho=state(dim, n, ns) if ns > 1 else [np.ones(nc)], pi=1e-2 * rng.standard_normal(nc),
        eta=np.full(nc, 1.3), eta_ed=[np.full(m, 1.3) for m in ne], kappa=np.zeros(nc), T=np.ones(nc),
        T_ed=[np.ones(m) for m in ne], W_cc=[np.sqrt(2.0) * rng.standard_normal(nc) for _ in range(2 * dim)],
        W_ed=W_ed, W_m=mass_fields(dim, n, ns, seed=seed + 2, n_rngs=2) if ns > 1 else None, mp=mp,
        sp=O.StochParams(k_B=1e-3 if ns > 1 else 1.0, variance_coef_mom=1.0, dV=100.0 if ns > 1 else 1.0,
                         stoch_stress_form=1, filtering_width=0),
        dt=0.5 if ns > 1 else 0.1)


@pytest.mark.parametrize("bc_lo,bc_hi", [([PE, NS, PE], [PE, NS, PE]), ([SL, NS, PE], [NS, SL, PE])])
@pytest.mark.parametrize("ns", [1, 3])
def test_overdamped_walls_conserve_mass_and_keep_walls(bc_lo, bc_hi, ns):
    dim, n = 2, [16, 12]
    a = inputs(dim, n, ns, bc_lo)
    O.set_walls(bc_lo, bc_hi)
    m0 = [r.sum() for r in a["rho"]]
    rc, u, rho, pi, st = O.advance_overdamped(dim, n, 1.0, 1, O.default_params(gmres_rel_tol=1e-10), a["sp"],
                                              a["mp"], a["dt"], a["u"], a["rho"], a["pi"], a["eta"], a["eta_ed"],
                                              a["kappa"], a["T"], a["T_ed"], a["W_cc"], a["W_ed"], a["W_m"])
    assert rc in (0, 3)
    for s in range(ns):
        assert abs(rho[s].sum() - m0[s]) < 1e-12 * abs(m0[s])
    for c in range(dim):
        if bc_lo[c] != PE:
            a2 = u[c].reshape(n[1], n[0])
            assert np.all((a2[:, 0] if c == 0 else a2[0, :]) == 0.0)
    assert any(np.any(x != 0.0) for x in u)
