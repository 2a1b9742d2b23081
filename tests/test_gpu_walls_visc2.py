"""Walls with visc_type 2 and 3 (constant coefficients) on the GPU against the
oracle: apply_matrix, one V-cycle of the staggered multigrid, GMRES (FP64,
same iteration count; mixed precision to the FP64 solution) and the
overdamped and inertial steps.  The wall stencil is the uniform one of
stag_applyop_level on ghost cells, the cross terms reading the other
components on and behind the walls."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_overdamped import _mix_kw
from tests.test_gpu_parity import dev, host, zeros
from tests.test_gpu_walls import CASES, wall_rhs
from tests.test_oracle_overdamped_walls import inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def periodic_afterwards():
    yield
    O.set_walls()


def solver(dim, n, bc_lo, bc_hi, precision="fp64", visc=2, **params):
    return L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(**params), precision=precision, bc_lo=bc_lo,
                          bc_hi=bc_hi)


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
@pytest.mark.parametrize("visc", [2, 3])
def test_apply_matrix_walls_visc2(cuda, dim, n, bc_lo, bc_hi, visc):
    O.set_walls(bc_lo, bc_hi)
    pb = P.problem(dim, n, visc, dx=1.0, seed=41)
    u, p = wall_rhs(dim, n, bc_lo, 42, 1.0)
    ref_u, ref_p = O.apply_matrix(pb, 2.0, u, p)
    with solver(dim, n, bc_lo, bc_hi, visc=visc) as s:
        b_u, b_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_matrix(b_u, b_p, dev(u, cuda), dev(p, cuda), dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                       dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), 2.0)
    assert P.rel_inf(host(b_u), ref_u) < 1e-13
    assert P.rel_inf([host(b_p)], [ref_p]) < 1e-13


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
def test_stag_mg_one_vcycle_walls_visc2(cuda, dim, n, bc_lo, bc_hi):
    O.set_walls(bc_lo, bc_hi)
    pb = P.problem(dim, n, 2, dx=1.0, seed=43)
    rhs, _ = wall_rhs(dim, n, bc_lo, 44, 1.0)
    params = O.default_params(stag_mg_max_vcycles=1)
    ref = O.stag_mg_solver(pb, params, 1.0, rhs)
    with solver(dim, n, bc_lo, bc_hi, stag_mg_max_vcycles=1) as s:
        phi = zeros(pb.nc, dim, cuda)
        s.stag_mg_solver(dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda),
                         1.0, phi, dev(rhs, cuda))
    assert P.rel_inf(host(phi), ref) < 1e-12


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
@pytest.mark.parametrize("theta,visc", [(0.0, 2), (2.0, 2), (2.0, 3)])
def test_gmres_walls_visc2(cuda, dim, n, bc_lo, bc_hi, theta, visc):
    O.set_walls(bc_lo, bc_hi)
    pb = P.problem(dim, n, visc, dx=1.0, seed=45)
    b_u, b_p = wall_rhs(dim, n, bc_lo, 46, theta)
    rc, ref_u, ref_p, npr_ref, st_ref = O.gmres(pb, O.default_params(gmres_rel_tol=1e-9), theta, b_u, b_p)
    assert rc == 0
    for precision, tol in (("fp64", 1e-10), ("mixed", 1e-7)):
        with solver(dim, n, bc_lo, bc_hi, precision=precision, visc=visc, gmres_rel_tol=1e-9) as s:
            x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
            status, npr, st = s.gmres(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda),
                                      dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
        assert status == 0
        if precision == "fp64":
            assert st["total_iters"] == st_ref.total_iters
        assert P.rel_inf(host(x_u), ref_u) < tol
        assert P.rel_inf([host(x_p)], [ref_p]) < tol


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", [CASES[0], CASES[4]])
@pytest.mark.parametrize("ns", [1, 3])
def test_overdamped_walls_visc2(cuda, dim, n, bc_lo, bc_hi, ns):
    a = inputs(dim, n, ns, bc_lo)
    O.set_walls(bc_lo, bc_hi)
    rc, u_r, rho_r, pi_r, st_r = O.advance_overdamped(dim, n, 1.0, 2, O.default_params(gmres_rel_tol=1e-10),
                                                      a["sp"], a["mp"], a["dt"], a["u"], a["rho"], a["pi"], a["eta"],
                                                      a["eta_ed"], a["kappa"], a["T"], a["T_ed"], a["W_cc"],
                                                      a["W_ed"], a["W_m"])
    assert rc in (0, 3)
    sp = L.StochParams(k_B=a["sp"].k_B, variance_coef_mom=1.0, dV=a["sp"].dV, stoch_stress_form=1, filtering_width=0)
    with solver(dim, n, bc_lo, bc_hi, gmres_rel_tol=1e-10) as s:
        u, rho, pi = dev(a["u"], cuda), dev(a["rho"], cuda), dev(a["pi"], cuda)
        mp_l = L.mixture_params(**_mix_kw(a["mp"])) if a["mp"] is not None else None
        s.advance_timestep_overdamped(sp, mp_l, a["dt"], u, rho, pi, dev(a["eta"], cuda), dev(a["eta_ed"], cuda),
                                      dev(a["kappa"], cuda), dev(a["T"], cuda), dev(a["T_ed"], cuda),
                                      dev(a["W_cc"], cuda), dev(a["W_ed"], cuda),
                                      dev(a["W_m"], cuda) if a["W_m"] is not None else None)
    assert P.rel_inf(host(u), u_r) < 1e-10
    for q in range(ns):
        assert np.abs(host(rho)[q] - rho_r[q]).max() < 1e-12 * np.abs(rho_r[q]).max()
