"""gmres_spatial_order = 4 (apply_matrix.f90:54-67, 124-135) through the C
ABI against the oracle: the fourth-order viscous operator and gradient of
k_stokes_apply4, GMRES with it (the preconditioner stays second order), the
visc_type restriction and the two-ghost-cell requirement of the host path."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_parity import dev, host, zeros

pytestmark = pytest.mark.gpu

SHAPES = [(2, [16, 16]), (2, [32, 16]), (3, [8, 8, 8]), (3, [16, 8, 12])]


@pytest.mark.parametrize("dim,n", SHAPES)
@pytest.mark.parametrize("theta", [0.0, 3.0])
def test_apply_matrix_order4(cuda, dim, n, theta):
    pb = P.problem(dim, n, 1, dx=0.5, seed=11)
    u, p = P.random_stokes(dim, n, seed=12)
    ref_u, ref_p = O.apply_matrix(pb, theta, u, p, order=4)
    with L.StokesSolver(dim, n, 0.5, 1, params=L.default_params(gmres_spatial_order=4)) as s:
        b_u, b_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_matrix(b_u, b_p, dev(u, cuda), dev(p, cuda), dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                       dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
    assert P.rel_inf(host(b_u), ref_u) < 1e-13
    assert P.rel_inf([host(b_p)], [ref_p]) < 1e-13
    # it is not the second-order operator
    o2_u, _ = O.apply_matrix(pb, theta, u, p)
    assert P.rel_inf(host(b_u), o2_u) > 1e-3


@pytest.mark.parametrize("dim,n,theta", [(2, [32, 32], 0.0), (2, [32, 16], 5.0), (3, [16, 16, 16], 0.0),
                                         (3, [16, 8, 16], 20.0)])
def test_gmres_order4(cuda, dim, n, theta):
    """GMRES on the fourth-order saddle-point operator with the second-order
    multigrid preconditioner: the oracle's iteration count and solution"""
    pb = P.problem(dim, n, 1, dx=1.0, seed=13)
    b_u, b_p = P.random_stokes(dim, n, seed=14)
    if theta == 0.0:
        b_u = [b - b.mean() for b in b_u]
    params = dict(gmres_rel_tol=1e-9, gmres_spatial_order=4)
    rc, ref_u, ref_p, npr_ref, st_ref = O.gmres(pb, O.default_params(**params), theta, b_u, b_p)
    # 0, or the true-residual warning (gmres.f90:286-289) that the coarser
    # second-order preconditioner can leave on the fourth-order system
    assert rc in (0, 3)
    with L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(**params)) as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        status, npr, st = s.gmres(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda),
                                  dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
    assert status == st_ref.status
    assert st["total_iters"] == st_ref.total_iters
    assert P.rel_inf(host(x_u), ref_u) < 1e-10
    assert P.rel_inf([host(x_p)], [ref_p]) < 1e-10


@pytest.mark.parametrize("visc", [-1, 2, 3])
def test_order4_needs_visc_type_one(cuda, visc):
    with pytest.raises(L.FhdError) as e:
        L.StokesSolver(2, [16, 16], 1.0, visc, params=L.default_params(gmres_spatial_order=4))
    assert e.value.status == L._capi.FHD_ERR_UNSUPPORTED


def test_order4_needs_two_ghost_cells(cuda):
    """x_u and x_p with one ghost cell are refused for order 4
    (apply_matrix.f90:61-67) and accepted with two"""
    dim, n = 2, [16, 16]
    pb = P.problem(dim, n, 1, dx=1.0, seed=15)
    u, p = P.random_stokes(dim, n, seed=16)
    nodal = [[1, 0], [0, 1]]
    fab = lambda x, nd, ng: L.fab_from_canonical(x, dim, n, nd, ng)
    with L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(gmres_spatial_order=4)) as s:
        def run(ng):
            b_u = [fab(np.zeros(pb.nc), nodal[c], 0) for c in range(dim)]
            b_p = fab(np.zeros(pb.nc), [0, 0], 0)
            s.apply_matrix_fab(b_u, b_p, [fab(u[c], nodal[c], ng) for c in range(dim)], fab(p, [0, 0], ng),
                               [fab(pb.alpha_fc[c], nodal[c], 0) for c in range(dim)], fab(pb.beta, [0, 0], 0),
                               [fab(pb.beta_ed[0], [1, 1], 0)], fab(pb.gamma, [0, 0], 0), 1.0)
            return b_u, b_p
        with pytest.raises(L.FhdError) as e:
            run(1)
        assert e.value.status == L._capi.FHD_ERR_BAD_GHOSTS
        b_u, b_p = run(2)
    ref_u, ref_p = O.apply_matrix(pb, 1.0, u, p, order=4)
    for c in range(dim):
        got = L.canonical_from_fab(b_u[c], dim, n)
        assert P.rel_inf([got], [ref_u[c]]) < 1e-13
