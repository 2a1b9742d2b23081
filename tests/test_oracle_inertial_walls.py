"""The oracle's inertial step (advance_timestep_inertial.f90:45-923) with
homogeneous walls: each species' mass is conserved and the normal velocity
stays zero on the wall faces.  The step's walls are those of its parts (the
Stokes solve, the fluxes, the zero pressure gradient on wall faces) and the
momentum advection's zero update on wall faces (mk_advective_m_fluxdiv.f90:
80-85)."""
import numpy as np
import pytest

import oracle as O
from tests.test_oracle_overdamped_walls import inputs

NS, SL, PE = O.NO_SLIP_WALL, O.SLIP_WALL, -1


@pytest.fixture(autouse=True)
def periodic_afterwards():
    yield
    O.set_walls()


def step(dim, n, ns, bc_lo, bc_hi):
    a = inputs(dim, n, ns, bc_lo)
    O.set_walls(bc_lo, bc_hi)
    params = O.default_params(gmres_rel_tol=1e-10)
    W_cc1 = a["W_cc"][:dim]
    W_ed1 = a["W_ed"][:len(a["W_ed"]) // 2]
    if ns == 1:
        rc, u, rho, pi, st = O.advance_inertial(dim, n, 1.0, 1, params, a["sp"], a["dt"], a["u"], a["rho"][0],
                                                a["pi"], a["eta"], a["eta_ed"], a["kappa"], a["T"], a["T_ed"],
                                                W_cc1, W_ed1)
        return a, rc, u, [rho], pi, None
    F0 = O.mass_fluxdiv(dim, n, 1.0, a["sp"], a["mp"], a["rho"], a["dt"], [1.0], a["W_m"][:dim * ns])
    rc, u, rho, pi, F, st = O.advance_inertial_ms(dim, n, 1.0, 1, params, a["sp"], a["mp"], a["dt"], a["u"],
                                                  a["rho"], a["pi"], F0, a["eta"], a["eta_ed"], a["kappa"], a["T"],
                                                  a["T_ed"], W_cc1, W_ed1, a["W_m"])
    return a, rc, u, rho, pi, F


@pytest.mark.parametrize("bc_lo,bc_hi", [([PE, NS, PE], [PE, NS, PE]), ([SL, NS, PE], [NS, SL, PE])])
@pytest.mark.parametrize("ns", [1, 3])
def test_inertial_walls_conserve_mass_and_keep_walls(bc_lo, bc_hi, ns):
    dim, n = 2, [16, 12]
    a, rc, u, rho, pi, F = step(dim, n, ns, bc_lo, bc_hi)
    assert rc in (0, 3)
    for s in range(ns):
        m0 = a["rho"][s].sum()
        assert abs(rho[s].sum() - m0) < 1e-12 * abs(m0)
    for c in range(dim):
        if bc_lo[c] != PE:
            a2 = u[c].reshape(n[1], n[0])
            assert np.all((a2[:, 0] if c == 0 else a2[0, :]) == 0.0)
    assert all(np.all(np.isfinite(x)) for x in u)
