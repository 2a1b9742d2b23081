"""Walls with visc_type 2 and 3 (constant coefficients; visc_type 2:
L = beta (lap u + grad div u), visc_type 3: beta lap u + (beta / 3 + gamma)
grad div u) in the oracle: the uniform stencil of stag_applyop_level on the ghost cells
of multifab_physbc_stag.f90, whose cross terms read the other velocity
components on and behind the walls.  Exact checks:
  * on a discretely divergence-free field the visc_type 2 operator equals the
    visc_type 1 one, face by face (its extra part is beta times the gradient
    of the cell divergence); fields built from a stream function that is
    zero on the wall nodes, so the normal velocity vanishes on the walls;
  * a field with divergence makes them differ (the cross terms are seen);
  * a slip wall is a mirror: the solve with slip walls equals the periodic
    solve on the doubled box;
  * plane Poiseuille flow (divergence-free) has the visc_type 1 profile."""
import numpy as np
import pytest

import oracle as O
from tests import problems as P
from tests.test_oracle_walls import doubled, half

NS, SL, PE = O.NO_SLIP_WALL, O.SLIP_WALL, -1


@pytest.fixture(autouse=True)
def periodic_afterwards():
    yield
    O.set_walls()


def stream_field(n, walls, seed):
    """2D staggered velocity from a node stream function psi (zero on the
    wall nodes): u_x = d psi / dy, u_y = -d psi / dx, discretely div-free"""
    nx, ny = n
    rng = np.random.default_rng(seed)
    psi = rng.standard_normal((ny + 1, nx + 1))
    if walls[0]:
        psi[:, 0] = psi[:, nx] = 0.0
    else:
        psi[:, nx] = psi[:, 0]
    if walls[1]:
        psi[0, :] = psi[ny, :] = 0.0
    else:
        psi[ny, :] = psi[0, :]
    ux = psi[1:, :nx] - psi[:ny, :nx]
    uy = -(psi[:ny, 1:] - psi[:ny, :nx])
    return [ux.ravel(), uy.ravel()]


def divergence(n, u, walls):
    nx, ny = n
    ux, uy = u[0].reshape(ny, nx), u[1].reshape(ny, nx)
    uxp = np.zeros_like(ux) if walls[0] else np.roll(ux, -1, axis=1)
    if walls[0]:
        uxp[:, :-1] = ux[:, 1:]
    uyp = np.zeros_like(uy) if walls[1] else np.roll(uy, -1, axis=0)
    if walls[1]:
        uyp[:-1, :] = uy[1:, :]
    return (uxp - ux) + (uyp - uy)


@pytest.mark.parametrize("bc_lo,bc_hi", [([PE, NS, PE], [PE, NS, PE]), ([SL, NS, PE], [NS, SL, PE]),
                                         ([NS, PE, PE], [SL, PE, PE])])
@pytest.mark.parametrize("visc", [2, 3])
def test_visc2_equals_visc1_on_divergence_free_fields(bc_lo, bc_hi, visc):
    """visc_type 3 too: its extra part is (beta / 3 + gamma) grad div u"""
    n = [12, 10]
    walls = [bc_lo[0] != PE, bc_lo[1] != PE]
    O.set_walls(bc_lo, bc_hi)
    u = stream_field(n, walls, 3)
    assert np.max(np.abs(divergence(n, u, walls))) < 1e-13
    p = np.zeros(120)
    pb1 = P.problem(2, n, 1, dx=0.5, seed=4)
    pb2 = P.problem(2, n, visc, dx=0.5, seed=4)
    assert pb1.beta[0] == pb2.beta[0]
    a1, _ = O.apply_matrix(pb1, 1.0, u, p)
    a2, _ = O.apply_matrix(pb2, 1.0, u, p)
    assert P.rel_inf(a2, a1) < 1e-13
    # with divergence the cross terms differ
    v = [x + 0.1 * np.random.default_rng(5).standard_normal(120) for x in u]
    for c in range(2):
        if walls[c]:
            v[c].reshape(10, 12)[(slice(None), 0) if c == 0 else (0, slice(None))] = 0.0
    b1, _ = O.apply_matrix(pb1, 1.0, v, p)
    b2, _ = O.apply_matrix(pb2, 1.0, v, p)
    assert P.rel_inf(b2, b1) > 1e-3


@pytest.mark.parametrize("dim,n,wall_dir", [(2, [16, 16], 1), (3, [8, 8, 8], 2)])
def test_slip_walls_mirror_the_periodic_solve_visc2(dim, n, wall_dir):
    rng = np.random.default_rng(6)
    nc = int(np.prod(n))
    b_u = [rng.standard_normal(nc) for _ in range(dim)]
    b_p = rng.standard_normal(nc)
    b_p -= b_p.mean()
    shape = [n[d] for d in reversed(range(dim))]
    a = b_u[wall_dir].reshape(shape)
    idx = [slice(None)] * dim
    idx[dim - 1 - wall_dir] = 0
    a[tuple(idx)] = 0.0
    b_u[wall_dir] = a.ravel()
    params = O.default_params(gmres_rel_tol=1e-12)
    bc = [-1] * 3
    bc[wall_dir] = SL
    O.set_walls(bc, bc)
    pb = P.problem(dim, n, 2, dx=1.0, seed=7)
    rc, x_u, x_p, _, st = O.gmres(pb, params, 2.0, b_u, b_p)
    assert rc in (0, 3)
    O.set_walls()
    n2 = list(n)
    n2[wall_dir] *= 2
    pb2 = P.problem(dim, n2, 2, dx=1.0, seed=7)
    assert pb2.beta[0] == pb.beta[0]
    bu2, bp2 = doubled(dim, n, wall_dir, b_u, b_p)
    rc2, y_u, y_p, _, _ = O.gmres(pb2, params, 2.0, bu2, bp2)
    assert rc2 in (0, 3)
    for c in range(dim):
        assert P.rel_inf([x_u[c]], [half(dim, n2, wall_dir, y_u[c])]) < 1e-8, c


def test_poiseuille_visc2_is_the_visc1_profile():
    n, nc = [8, 16], 128
    O.set_walls([-1, NS, -1], [-1, NS, -1])
    out = []
    for visc in (1, 2):
        pb = P.problem(2, n, visc, dx=1.0 / 16, seed=5)
        rc, x_u, x_p, _, st = O.gmres(pb, O.default_params(gmres_rel_tol=1e-12), 0.0,
                                      [np.ones(nc), np.zeros(nc)], np.zeros(nc))
        assert rc in (0, 3)
        out.append(x_u)
    assert P.rel_inf(out[1], out[0]) < 1e-9
