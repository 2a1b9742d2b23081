"""Wall rules of the stochastic fluxes in the oracle:
  * momentum (stochastic_m_fluxdiv.f90:363-451, mflux_bc_2d / _3d): edges on
    a no-slip wall times sqrt(2), on a slip wall zero; the high wall's edges
    are a plane of their own; the normal force on a wall face is zero
    (multifab_physbc_domainvel);
  * mass (stochastic_mass_fluxdiv.f90:216-368, stoch_mass_bc): no random
    flux through a wall face.

The reference stores no results for these, so the restatement is checked
against an independent numpy form of the 2D rules and by exact conservation
sums in 3D."""
import numpy as np
import pytest

import oracle as O

NS, SL, PE = O.NO_SLIP_WALL, O.SLIP_WALL, -1


@pytest.fixture(autouse=True)
def periodic_afterwards():
    yield
    O.set_walls()


def edge_shape(dim, n, e, bc_lo):
    """numpy shape (z, y, x) of edge set e with the high-wall planes"""
    dirs = (0, 1) if dim == 2 else [(0, 1), (0, 2), (1, 2)][e]
    m = [n[d] + (1 if (d in dirs and bc_lo[d] != PE) else 0) for d in range(dim)]
    return tuple(reversed(m))


def fields(dim, n, bc_lo, seed, n_rngs=2):
    rng = np.random.default_rng(seed)
    nc = int(np.prod(n[:dim]))
    nE = 1 if dim == 2 else 3
    eta = 1 + rng.random(nc)
    T = 1 + rng.random(nc)
    eta_ed = [1 + rng.random(int(np.prod(edge_shape(dim, n, e, bc_lo)))) for e in range(nE)]
    T_ed = [1 + rng.random(int(np.prod(edge_shape(dim, n, e, bc_lo)))) for e in range(nE)]
    W_cc = [rng.standard_normal(nc) for _ in range(n_rngs * dim)]
    W_ed = []
    for r in range(n_rngs):
        for e in range(nE):
            W_ed += [rng.standard_normal(int(np.prod(edge_shape(dim, n, e, bc_lo)))) for _ in range(2)]
    return eta, T, eta_ed, T_ed, W_cc, W_ed


SP = dict(k_B=2.0, variance_coef_mom=1.0, dV=0.125, stoch_stress_form=0, filtering_width=0)
W8 = [0.5, -0.25]


def scaled(dim, sp, dt, arr_w, weights, eta, T, n_rngs, idx, stride):
    """(variance * sum_r w_r W_r) * sqrt(eta T), in the oracle's order"""
    s = np.zeros_like(eta)
    for r in range(n_rngs):
        s = s + weights[r] * arr_w[r * stride + idx]
    var = np.sqrt(sp.variance_coef_mom * 2.0 * sp.k_B / (sp.dV * dt))
    return (var * s) * np.sqrt(eta * T)


def numpy_stoch_m_2d(n, dx, bc_lo, bc_hi, eta, T, eta_ed, T_ed, dt, W_cc, W_ed):
    """stoch_m_force_2d with mflux_bc_2d and the wall-face rule, in numpy"""
    sp = O.StochParams(**SP)
    nx, ny = n
    cc = [scaled(2, sp, dt, W_cc, W8, eta, T, 2, c, 2).reshape(ny, nx) for c in range(2)]
    sh = edge_shape(2, n, 0, bc_lo)
    nd = [scaled(2, sp, dt, W_ed, W8, eta_ed[0], T_ed[0], 2, comp, 2).reshape(sh) for comp in range(2)]
    for d, ax in ((0, 1), (1, 0)):  # x boundaries, then y
        if bc_lo[d] == PE:
            continue
        for side, idx in ((bc_lo[d], 0), (bc_hi[d], sh[ax] - 1)):
            sl = [slice(None), slice(None)]
            sl[ax] = idx
            for comp in range(2):
                nd[comp][tuple(sl)] = np.sqrt(2.0) * nd[comp][tuple(sl)] if side == NS else 0.0
    # node (i, j) with periodic wrap where periodic
    def N(comp, j, i):
        jj = j % ny if bc_lo[1] == PE else j
        ii = i % nx if bc_lo[0] == PE else i
        return nd[comp][jj, ii]
    out = [np.zeros((ny, nx)), np.zeros((ny, nx))]
    for j in range(ny):
        for i in range(nx):
            d0 = (cc[0][j, i] - cc[0][j, (i - 1) % nx]) / dx + (N(0, j + 1, i) - N(0, j, i)) / dx
            d1 = (N(1, j, i + 1) - N(1, j, i)) / dx + (cc[1][j, i] - cc[1][(j - 1) % ny, i]) / dx
            out[0][j, i] = 0.0 if (bc_lo[0] != PE and i == 0) else d0
            out[1][j, i] = 0.0 if (bc_lo[1] != PE and j == 0) else d1
    return [o.ravel() for o in out]


@pytest.mark.parametrize("bc_lo,bc_hi", [([PE, NS, PE], [PE, NS, PE]), ([SL, PE, PE], [SL, PE, PE]),
                                         ([NS, SL, PE], [SL, NS, PE]), ([NS, NS, PE], [NS, NS, PE])])
def test_stoch_m_2d_matches_numpy(bc_lo, bc_hi):
    n, dx, dt = [12, 8], 0.5, 0.1
    eta, T, eta_ed, T_ed, W_cc, W_ed = fields(2, n, bc_lo, 3)
    O.set_walls(bc_lo, bc_hi)
    got = O.stochastic_m_fluxdiv(2, n, dx, O.StochParams(**SP), eta, eta_ed, T, T_ed, dt, W8, W_cc, W_ed)
    ref = numpy_stoch_m_2d(n, dx, bc_lo, bc_hi, eta, T, eta_ed, T_ed, dt, W_cc, W_ed)
    for c in range(2):
        assert np.max(np.abs(got[c] - ref[c])) <= 1e-12 * np.max(np.abs(ref[c]))


@pytest.mark.parametrize("increment", [False, True])
def test_stoch_m_wall_faces_zero(increment):
    dim, n = 3, [8, 6, 4]
    bc = [NS, PE, SL]
    eta, T, eta_ed, T_ed, W_cc, W_ed = fields(dim, n, bc, 4)
    O.set_walls(bc, bc)
    force0 = [np.full(int(np.prod(n)), 7.0) for _ in range(dim)]
    got = O.stochastic_m_fluxdiv(dim, n, 1.0, O.StochParams(**SP), eta, eta_ed, T, T_ed, 0.1, W8, W_cc, W_ed,
                                 force=force0, increment=increment)
    u = got[0].reshape(4, 6, 8)
    w = got[2].reshape(4, 6, 8)
    assert np.all(u[:, :, 0] == 0.0) and np.all(w[0] == 0.0)
    assert np.all(u[:, :, 1:] != 0.0)


def test_stoch_m_momentum_balance_3d():
    """sum of the x force over all x faces = the edge fluxes through the y and
    z walls: the no-slip y walls pass sqrt(2) times theirs, the slip z walls
    none (x periodic telescopes)"""
    dim, n, dx, dt = 3, [6, 8, 4], 0.5, 0.1
    bc = [PE, NS, SL]
    eta, T, eta_ed, T_ed, W_cc, W_ed = fields(dim, n, bc, 5)
    O.set_walls(bc, bc)
    sp = O.StochParams(**SP)
    got = O.stochastic_m_fluxdiv(dim, n, dx, sp, eta, eta_ed, T, T_ed, dt, W8, W_cc, W_ed)
    xy = scaled(3, sp, dt, W_ed, W8, eta_ed[0], T_ed[0], 2, 0, 6).reshape(edge_shape(3, n, 0, bc))
    expect = np.sqrt(2.0) * (xy[:, -1, :].sum() - xy[:, 0, :].sum()) / dx
    assert abs(got[0].sum() - expect) < 1e-10 * np.abs(xy).sum() / dx
    # y momentum: the x direction is periodic and the z walls slip; the y wall
    # faces carry no force
    v = got[1].reshape(4, 8, 6)
    assert np.all(v[:, 0, :] == 0.0)


def test_stoch_mass_wall_faces_and_conservation():
    dim, n, ns = 3, [6, 4, 8], 3
    mp = O.mixture_params([1.0, 2.0, 3.0], [1.0, 0.5, 2.0])
    bc = [SL, PE, NS]
    rng = np.random.default_rng(6)
    nc = int(np.prod(n))
    sqrtL = [rng.standard_normal(nc) for _ in range(dim * ns * ns)]
    W_fc = [rng.standard_normal(nc) for _ in range(2 * dim * ns)]
    sp = O.StochParams(k_B=1.0, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    O.set_walls(bc, bc)
    div, flux = O.stochastic_mass_fluxdiv(dim, n, 1.0, sp, mp, sqrtL, 0.1, W8, W_fc, want_flux=True)
    for s in range(ns):
        fx = flux[0 * ns + s].reshape(8, 4, 6)
        fz = flux[2 * ns + s].reshape(8, 4, 6)
        assert np.all(fx[:, :, 0] == 0.0) and np.all(fz[0] == 0.0)
        assert np.any(flux[1 * ns + s] != 0.0)
        assert abs(div[s].sum()) < 1e-10 * np.abs(div[s]).sum()


def test_mass_fluxdiv_walls_zero_faces_and_conservation():
    """compute_mass_fluxdiv with walls: no diffusive or random flux through a
    wall face, and each species' divergence sums to zero"""
    from tests.test_oracle_multispecies import mass_fields, mix, state
    dim, n, ns = 3, [8, 6, 4], 3
    bc = [NS, PE, SL]
    mp = mix(ns)
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-2)
    W = mass_fields(dim, n, ns, n_rngs=1)
    O.set_walls(bc, bc)
    div, flux = O.mass_fluxdiv(dim, n, 1.0, sp, mp, rho, 0.05, [1.0], W, want_flux=True)
    for s in range(ns):
        assert np.all(flux[0 * ns + s].reshape(4, 6, 8)[:, :, 0] == 0.0)
        assert np.all(flux[2 * ns + s].reshape(4, 6, 8)[0] == 0.0)
        assert np.any(flux[0 * ns + s].reshape(4, 6, 8)[:, :, 1:] != 0.0)
        assert abs(div[s].sum()) < 1e-10 * np.abs(div[s]).sum()


def test_sqrtL_wall_faces_use_the_extrapolated_ghost():
    """on a wall face the factor is the periodic one with the wrapped
    neighbour replaced by the interior cell (first-order extrapolation);
    the other faces are unchanged"""
    from tests.test_oracle_multispecies import mix, state
    dim, n, ns = 2, [8, 6], 3
    mp = mix(ns)
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-2)
    O.set_walls([NS, PE, PE], [SL, PE, PE])
    got = O.sqrtLonsager_fc(dim, n, sp, mp, rho)
    O.set_walls()
    per = O.sqrtLonsager_fc(dim, n, sp, mp, rho)
    mod = [r.reshape(6, 8).copy() for r in rho]
    for r in mod:
        r[:, 7] = r[:, 0]  # the wrapped neighbour of face 0 becomes the interior cell
    ghost = O.sqrtLonsager_fc(dim, n, sp, mp, [r.ravel() for r in mod])
    for q in range(ns * ns):
        g = got[q].reshape(6, 8)
        assert np.array_equal(g[:, 0], ghost[q].reshape(6, 8)[:, 0])
        assert np.array_equal(g[:, 1:], per[q].reshape(6, 8)[:, 1:])
        assert np.array_equal(got[ns * ns + q], per[ns * ns + q])  # y faces: periodic
