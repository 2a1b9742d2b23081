"""Homogeneous no-slip and slip walls (fhd_ctx_create_bc bc codes 100, 200)
through the C ABI against the oracle: apply_matrix, one staggered V-cycle,
apply_precon and GMRES in FP64 (same iteration counts), the mixed-precision
solve, and the options that refuse walls."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_parity import dev, host, zeros

pytestmark = pytest.mark.gpu

NS, SL, PE = L.FHD_BC_NO_SLIP_WALL, L.FHD_BC_SLIP_WALL, L.FHD_BC_PERIODIC

# (dim, n, bc_lo, bc_hi): channels, a box walled on every side, mixed kinds
CASES = [
    (2, [16, 16], [PE, NS, PE], [PE, NS, PE]),
    (2, [32, 16], [SL, PE, PE], [SL, PE, PE]),
    (2, [16, 16], [NS, SL, PE], [SL, NS, PE]),
    (3, [8, 8, 8], [PE, PE, NS], [PE, PE, NS]),
    (3, [16, 8, 8], [NS, SL, PE], [NS, SL, PE]),
    (3, [8, 8, 8], [NS, NS, NS], [NS, NS, NS]),
]


@pytest.fixture(autouse=True)
def periodic_afterwards():
    yield
    O.set_walls()


def wall_rhs(dim, n, bc_lo, seed, theta):
    """random Stokes rhs, zero on the wall faces; for theta = 0 without
    no-slip walls, the periodic components' means removed (consistent)"""
    b_u, b_p = P.random_stokes(dim, n, seed=seed)
    shape = [n[d] for d in reversed(range(dim))]
    for c in range(dim):
        if bc_lo[c] != PE:
            a = b_u[c].reshape(shape)
            idx = [slice(None)] * dim
            idx[dim - 1 - c] = 0
            a[tuple(idx)] = 0.0
            b_u[c] = a.ravel()
    if theta == 0.0 and NS not in bc_lo[:dim]:
        for c in range(dim):
            if bc_lo[c] == PE:
                b_u[c] = b_u[c] - b_u[c].mean()
    return b_u, b_p


def solver(dim, n, bc_lo, bc_hi, precision="fp64", **params):
    return L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(**params), precision=precision, bc_lo=bc_lo,
                          bc_hi=bc_hi)


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
@pytest.mark.parametrize("theta", [0.0, 3.0])
def test_apply_matrix_walls(cuda, dim, n, bc_lo, bc_hi, theta):
    O.set_walls(bc_lo, bc_hi)
    pb = P.problem(dim, n, 1, dx=1.0, seed=21)
    u, p = wall_rhs(dim, n, bc_lo, 22, 1.0)
    ref_u, ref_p = O.apply_matrix(pb, theta, u, p)
    with solver(dim, n, bc_lo, bc_hi) as s:
        b_u, b_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_matrix(b_u, b_p, dev(u, cuda), dev(p, cuda), dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                       dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
    assert P.rel_inf(host(b_u), ref_u) < 1e-13
    assert P.rel_inf([host(b_p)], [ref_p]) < 1e-13


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
def test_stag_mg_one_vcycle_walls(cuda, dim, n, bc_lo, bc_hi):
    O.set_walls(bc_lo, bc_hi)
    pb = P.problem(dim, n, 1, dx=1.0, seed=23)
    rhs, _ = wall_rhs(dim, n, bc_lo, 24, 1.0)
    params = O.default_params()
    ref = O.stag_mg_solver(pb, params, 0.7, rhs)
    with solver(dim, n, bc_lo, bc_hi) as s:
        phi = zeros(pb.nc, dim, cuda)
        s.stag_mg_solver(dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), 0.7,
                         phi, dev(rhs, cuda))
    assert P.rel_inf(host(phi), ref) < 1e-12


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
@pytest.mark.parametrize("theta", [0.0, 2.0])
def test_apply_precon_walls(cuda, dim, n, bc_lo, bc_hi, theta):
    O.set_walls(bc_lo, bc_hi)
    pb = P.problem(dim, n, 1, dx=1.0, seed=25)
    b_u, b_p = wall_rhs(dim, n, bc_lo, 26, theta)
    params = O.default_params()
    ref_u, ref_p = O.apply_precon(pb, params, theta, b_u, b_p)
    with solver(dim, n, bc_lo, bc_hi) as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_precon(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                       dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
    assert P.rel_inf(host(x_u), ref_u) < 1e-11
    assert P.rel_inf([host(x_p)], [ref_p]) < 1e-11


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
@pytest.mark.parametrize("theta", [0.0, 2.0])
def test_gmres_walls(cuda, dim, n, bc_lo, bc_hi, theta):
    O.set_walls(bc_lo, bc_hi)
    pb = P.problem(dim, n, 1, dx=1.0, seed=27)
    b_u, b_p = wall_rhs(dim, n, bc_lo, 28, theta)
    rc, ref_u, ref_p, npr_ref, st_ref = O.gmres(pb, O.default_params(gmres_rel_tol=1e-9), theta, b_u, b_p)
    assert rc == 0
    with solver(dim, n, bc_lo, bc_hi, gmres_rel_tol=1e-9) as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        status, npr, st = s.gmres(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda),
                                  dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
    assert status == 0
    assert st["total_iters"] == st_ref.total_iters
    assert P.rel_inf(host(x_u), ref_u) < 1e-10
    assert P.rel_inf([host(x_p)], [ref_p]) < 1e-10


def test_mixed_precision_walls(cuda):
    """FP32 multigrid with walls inside FP64 GMRES reaches the FP64 solution"""
    dim, n, bc_lo, bc_hi = 3, [16, 16, 16], [PE, NS, SL], [PE, NS, SL]
    O.set_walls(bc_lo, bc_hi)
    pb = P.problem(dim, n, 1, dx=1.0, seed=29)
    b_u, b_p = wall_rhs(dim, n, bc_lo, 30, 2.0)
    rc, ref_u, ref_p, _, st_ref = O.gmres(pb, O.default_params(gmres_rel_tol=1e-10), 2.0, b_u, b_p)
    assert rc == 0
    with solver(dim, n, bc_lo, bc_hi, precision="mixed", gmres_rel_tol=1e-10) as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        status, _, st = s.gmres(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda),
                                dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), 2.0)
    assert status == 0
    assert abs(st["total_iters"] - st_ref.total_iters) <= 2
    assert P.rel_inf(host(x_u), ref_u) < 1e-8
    assert P.rel_inf([host(x_p)], [ref_p]) < 1e-8


@pytest.mark.parametrize("kw", [dict(visc=-1), dict(visc=-2), dict(precon_type=2), dict(stag_mg_smoother=0),
                                dict(gmres_spatial_order=4), dict(code=102), dict(code=203)])
def test_unsupported_wall_options(cuda, kw):
    visc = kw.pop("visc", 1)
    code = kw.pop("code", NS)
    with pytest.raises(L.FhdError) as e:
        L.StokesSolver(2, [16, 16], 1.0, visc, params=L.default_params(**kw), bc_lo=[PE, code, PE],
                       bc_hi=[PE, code, PE])
    assert e.value.status == L._capi.FHD_ERR_UNSUPPORTED


def test_one_sided_periodic_is_refused(cuda):
    with pytest.raises(L.FhdError) as e:
        L.StokesSolver(2, [16, 16], 1.0, 1, bc_lo=[PE, NS, PE], bc_hi=[PE, PE, PE])
    assert e.value.status == L._capi.FHD_ERR_BAD_ARG
