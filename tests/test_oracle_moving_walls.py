"""Moving no-slip walls (wallspeed_lo / wallspeed_hi, the constant values of
inhomogeneous_bc_val.f90) in the oracle's overdamped and inertial steps.

Behind a moving no-slip wall the tangential ghost is 2 v_bc - u
(physbc_macvel_*_inhomogeneous, multifab_physbc_stag.f90:1118-1160), and the
steps take their diffusive_m_fluxdiv of the velocity with it: the solve is
then in delta form with homogeneous walls.  Known answers:
  * plane Couette flow: between walls moving at v_lo and v_hi the steady
    Stokes velocity is linear, v_lo + (v_hi - v_lo) y / L, exactly on the
    staggered grid (the ghost rule makes the wall value the mean of the
    ghost and the first face, which the linear profile satisfies).  One
    noise-free overdamped step from rest reaches it (each of its solves is
    a steady Stokes solve);
  * the same profile is a steady state of the inertial step (no pressure
    gradient, no advective flux: the velocity is uniform along the flow);
  * from rest, one inertial step drags the fluid beside each wall along it,
    antisymmetric in y for opposite wall speeds;
  * a speed on a slip wall is refused (there the value is a traction)."""
import numpy as np
import pytest

import oracle as O

NS, SL, PE = O.NO_SLIP_WALL, O.SLIP_WALL, -1
UNSUPPORTED = -5


@pytest.fixture(autouse=True)
def still_and_periodic_afterwards():
    yield
    O.set_walls()
    O.set_wall_speed()


def quiet_inputs(dim, n, bc_lo):
    """no noise (k_B = 0), unit density, constant viscosity 1.3"""
    nc = int(np.prod(n[:dim]))
    nE = 1 if dim == 2 else 3
    from tests.test_oracle_stoch_walls import edge_shape
    ne = [int(np.prod(edge_shape(dim, n, e, bc_lo))) for e in range(nE)]
    return dict(
        eta=np.full(nc, 1.3), eta_ed=[np.full(m, 1.3) for m in ne], kappa=np.zeros(nc), T=np.ones(nc),
        T_ed=[np.ones(m) for m in ne], W_cc=[np.zeros(nc) for _ in range(2 * dim)],
        W_ed=[np.zeros(ne[e % nE]) for e in range(4 * nE)], rho=np.ones(nc), pi=np.zeros(nc),
        sp=O.StochParams(k_B=0.0, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0))


def couette(dim, n, d, lo, hi):
    """the linear profile between walls normal to d, on the faces of a
    tangential component (face centres at (j + 1/2) / n[d] of the gap)"""
    shape = [n[q] for q in reversed(range(dim))]
    y = (np.arange(n[d]) + 0.5) / n[d]
    prof = lo + (hi - lo) * y
    sh = [1] * dim
    sh[dim - 1 - d] = n[d]
    return np.broadcast_to(prof.reshape(sh), shape).ravel().copy()


def speeds(dim, d, lo_t, hi_t):
    """wallspeed arrays (Fortran layout, [t + 2 d]) for the walls normal to d"""
    lo, hi = [0.0] * 6, [0.0] * 6
    for t, (a, b) in enumerate(zip(lo_t, hi_t)):
        lo[t + 2 * d], hi[t + 2 * d] = a, b
    return lo, hi


def overdamped(dim, n, a, u0, tol=1e-12):
    return O.advance_overdamped(dim, n, 1.0, 1, O.default_params(gmres_rel_tol=tol), a["sp"], None, 0.1, u0,
                                [a["rho"]], a["pi"], a["eta"], a["eta_ed"], a["kappa"], a["T"], a["T_ed"],
                                a["W_cc"], a["W_ed"], None)


def inertial(dim, n, a, u0, dt=0.05, tol=1e-12):
    return O.advance_inertial(dim, n, 1.0, 1, O.default_params(gmres_rel_tol=tol), a["sp"], dt, u0, a["rho"],
                              a["pi"], a["eta"], a["eta_ed"], a["kappa"], a["T"], a["T_ed"], a["W_cc"][:dim],
                              a["W_ed"][:len(a["W_ed"]) // 2])


@pytest.mark.parametrize("dim,n,d,lo_t,hi_t", [
    (2, [8, 16], 1, [-1.0], [1.0]),
    (2, [12, 8], 0, [0.5], [2.0]),
    (3, [8, 8, 12], 2, [-1.0, 0.25], [1.0, 0.75]),
])
def test_overdamped_step_reaches_couette_flow(dim, n, d, lo_t, hi_t):
    bc = [PE, PE, PE]
    bc[d] = NS
    O.set_walls(bc, bc)
    O.set_wall_speed(*speeds(dim, d, lo_t, hi_t))
    a = quiet_inputs(dim, n, bc)
    nc = int(np.prod(n[:dim]))
    rc, u, rho, pi, st = overdamped(dim, n, a, [np.zeros(nc) for _ in range(dim)])
    assert rc == 0
    t = 0
    for c in range(dim):
        if c == d:
            assert np.max(np.abs(u[c])) < 1e-10
            continue
        want = couette(dim, n, d, lo_t[t], hi_t[t])
        t += 1
        assert np.max(np.abs(u[c] - want)) < 1e-9 * np.max(np.abs(want))


def test_couette_flow_is_a_steady_state_of_the_inertial_step():
    dim, n, d = 2, [8, 16], 1
    bc = [PE, NS, PE]
    O.set_walls(bc, bc)
    O.set_wall_speed(*speeds(dim, d, [-1.0], [1.0]))
    a = quiet_inputs(dim, n, bc)
    u0 = [couette(dim, n, d, -1.0, 1.0), np.zeros(int(np.prod(n)))]
    rc, u, rho, pi, st = inertial(dim, n, a, u0)
    assert rc in (0, 3)
    assert np.max(np.abs(u[0] - u0[0])) < 1e-9
    assert np.max(np.abs(u[1])) < 1e-10


def test_inertial_step_drags_the_fluid_beside_the_walls():
    dim, n, d = 2, [8, 16], 1
    bc = [PE, NS, PE]
    O.set_walls(bc, bc)
    O.set_wall_speed(*speeds(dim, d, [-1.0], [1.0]))
    a = quiet_inputs(dim, n, bc)
    nc = int(np.prod(n))
    rc, u, rho, pi, st = inertial(dim, n, a, [np.zeros(nc), np.zeros(nc)])
    assert rc in (0, 3)
    ux = u[0].reshape(n[1], n[0])
    assert np.all(ux[0] < 0) and np.all(ux[-1] > 0)
    assert np.max(np.abs(ux + ux[::-1])) < 1e-12
    # the standing walls' step is the rest state
    O.set_wall_speed()
    rc, u, rho, pi, st = inertial(dim, n, a, [np.zeros(nc), np.zeros(nc)])
    assert np.max(np.abs(u[0])) == 0.0


def test_speed_on_a_slip_wall_is_refused():
    dim, n = 2, [8, 8]
    bc_lo, bc_hi = [PE, SL, PE], [PE, NS, PE]
    O.set_walls(bc_lo, bc_hi)
    O.set_wall_speed(*speeds(dim, 1, [1.0], [0.0]))
    a = quiet_inputs(dim, n, bc_lo)
    rc = overdamped(dim, n, a, [np.zeros(64), np.zeros(64)])[0]
    assert rc == UNSUPPORTED
    # the no-slip side may move
    O.set_wall_speed(*speeds(dim, 1, [0.0], [1.0]))
    assert overdamped(dim, n, a, [np.zeros(64), np.zeros(64)])[0] == 0


def test_speed_on_a_periodic_side_is_ignored():
    dim, n = 2, [8, 8]
    bc = [PE, NS, PE]
    O.set_walls(bc, bc)
    a = quiet_inputs(dim, n, bc)
    O.set_wall_speed(*speeds(dim, 0, [3.0], [3.0]))  # walls normal to x: none here
    rc, u, rho, pi, st = overdamped(dim, n, a, [np.zeros(64), np.zeros(64)])
    assert rc == 0 and np.max(np.abs(u[0])) == 0.0
