"""Reservoir boundaries (bc codes 101 NO_SLIP_RESERVOIR, 201 SLIP_RESERVOIR).

The reference treats them as no-slip and slip walls for the velocity and the
pressure (the NO_SLIP / SLIP ranges of define_bc_tower.f90:225-250,
301-355) and for the stochastic momentum flux (mflux_bc_2d / _3d,
stochastic_m_fluxdiv.f90:363-451).  So a context with reservoirs gives, bit
for bit, the results of the same context with walls in the Stokes solve,
the stochastic momentum flux and the single-fluid steps (whose mass flux is
zero, so no normal velocity is set at a reservoir).  The mass exchange of a
reservoir (Dirichlet concentrations, the sqrt(2) random flux through it) is
not built: the mass-flux entries and the multispecies steps refuse such a
context before any launch.  The closed and impermeable codes (102, 103,
202, 203) are refused at creation."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_overdamped import _mix_kw
from tests.test_gpu_parity import dev, host, zeros
from tests.test_gpu_walls import wall_rhs
from tests.test_oracle_overdamped_walls import inputs

pytestmark = pytest.mark.gpu

NS, SL, PE = L.FHD_BC_NO_SLIP_WALL, L.FHD_BC_SLIP_WALL, L.FHD_BC_PERIODIC
NR, SR = L.FHD_BC_NO_SLIP_RESERVOIR, L.FHD_BC_SLIP_RESERVOIR
AS_WALL = {NR: NS, SR: SL, NS: NS, SL: SL, PE: PE}

CASES = [
    (2, [32, 16], [PE, NR, PE], [PE, SR, PE]),
    (3, [16, 16, 8], [NR, SL, PE], [NS, SR, PE]),
]


def ctx(dim, n, bc_lo, bc_hi, walls):
    lo = [AS_WALL[b] for b in bc_lo] if walls else bc_lo
    hi = [AS_WALL[b] for b in bc_hi] if walls else bc_hi
    return L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(gmres_rel_tol=1e-10), bc_lo=lo, bc_hi=hi)


def both(run):
    """run(walls) on the wall context and on the reservoir context"""
    return run(True), run(False)


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
def test_gmres_with_reservoirs_is_gmres_with_walls(cuda, dim, n, bc_lo, bc_hi):
    pb = P.problem(dim, n, 1, dx=1.0, seed=31)
    b_u, b_p = wall_rhs(dim, n, [AS_WALL[b] for b in bc_lo], 32, 1.0)

    def run(walls):
        with ctx(dim, n, bc_lo, bc_hi, walls) as s:
            x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
            status, npr, st = s.gmres(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda),
                                      dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), 1.0)
            assert status == 0
            return host(x_u) + [host(x_p)], st["total_iters"]

    (a, ia), (b, ib) = both(run)
    assert ia == ib
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
def test_stochastic_fluxes_and_steps_with_reservoirs_are_those_with_walls(cuda, dim, n, bc_lo, bc_hi):
    a = inputs(dim, n, 1, bc_lo)

    def run(walls):
        out = []
        with ctx(dim, n, bc_lo, bc_hi, walls) as s:
            sp = L.StochParams(k_B=a["sp"].k_B, variance_coef_mom=1.0, dV=a["sp"].dV, stoch_stress_form=1,
                               filtering_width=0)
            f = dev([np.zeros(P.nc_of(dim, n)) for _ in range(dim)], cuda)
            s.stochastic_m_fluxdiv(sp, f, False, dev(a["eta"], cuda), dev(a["eta_ed"], cuda), dev(a["T"], cuda),
                                   dev(a["T_ed"], cuda), a["dt"], [1.0, 0.5], dev(a["W_cc"], cuda),
                                   dev(a["W_ed"], cuda))
            out += host(f)
            u, rho, pi = dev(a["u"], cuda), dev(a["rho"], cuda), dev(a["pi"], cuda)
            s.advance_timestep_overdamped(sp, None, a["dt"], u, rho, pi, dev(a["eta"], cuda), dev(a["eta_ed"], cuda),
                                          dev(a["kappa"], cuda), dev(a["T"], cuda), dev(a["T_ed"], cuda),
                                          dev(a["W_cc"], cuda), dev(a["W_ed"], cuda), None)
            out += host(u) + [host(pi)] + host(rho)
            u, r1, pi = dev(a["u"], cuda), dev(a["rho"][0], cuda), dev(a["pi"], cuda)
            s.advance_timestep_inertial(sp, a["dt"], u, r1, pi, dev(a["eta"], cuda), dev(a["eta_ed"], cuda),
                                        dev(a["kappa"], cuda), dev(a["T"], cuda), dev(a["T_ed"], cuda),
                                        dev(a["W_cc"][:dim], cuda), dev(a["W_ed"][:len(a["W_ed"]) // 2], cuda))
            out += host(u) + [host(pi), host(r1)]
        return out

    w, r = both(run)
    assert all(np.array_equal(x, y) for x, y in zip(w, r))
    assert any(np.any(x != 0.0) for x in r)


def test_mass_exchange_of_reservoirs_is_refused(cuda):
    dim, n, bc_lo, bc_hi = CASES[0]
    ns = 3
    a = inputs(dim, n, ns, bc_lo)
    O.set_walls([AS_WALL[b] for b in bc_lo], [AS_WALL[b] for b in bc_hi])
    try:
        F0 = O.mass_fluxdiv(dim, n, 1.0, a["sp"], a["mp"], a["rho"], a["dt"], [1.0], a["W_m"][:dim * ns])
    finally:
        O.set_walls()
    sp = L.StochParams(k_B=a["sp"].k_B, variance_coef_mom=1.0, dV=a["sp"].dV, stoch_stress_form=1, filtering_width=0)
    mp = L.mixture_params(**_mix_kw(a["mp"]))
    nc = P.nc_of(dim, n)
    with ctx(dim, n, bc_lo, bc_hi, False) as s:
        rho = dev(a["rho"], cuda)
        calls = {
            "compute_mass_fluxdiv": lambda: s.compute_mass_fluxdiv(
                mp, sp, rho, a["dt"], [1.0], dev(a["W_m"][:dim * ns], cuda),
                dev([np.zeros(nc) for _ in range(ns)], cuda)),
            "overdamped": lambda: s.advance_timestep_overdamped(
                sp, mp, a["dt"], dev(a["u"], cuda), rho, dev(a["pi"], cuda), dev(a["eta"], cuda),
                dev(a["eta_ed"], cuda), dev(a["kappa"], cuda), dev(a["T"], cuda), dev(a["T_ed"], cuda),
                dev(a["W_cc"], cuda), dev(a["W_ed"], cuda), dev(a["W_m"], cuda)),
            "inertial_ms": lambda: s.advance_timestep_inertial_multispecies(
                sp, mp, a["dt"], dev(a["u"], cuda), rho, dev(a["pi"], cuda), dev(F0, cuda), dev(a["eta"], cuda),
                dev(a["eta_ed"], cuda), dev(a["kappa"], cuda), dev(a["T"], cuda), dev(a["T_ed"], cuda),
                dev(a["W_cc"][:dim], cuda), dev(a["W_ed"][:len(a["W_ed"]) // 2], cuda), dev(a["W_m"], cuda)),
        }
        for name, call in calls.items():
            with pytest.raises(L.FhdError) as e:
                call()
            assert e.value.status == L._capi.FHD_ERR_UNSUPPORTED, name
            assert "reservoir" in e.value.detail, name


@pytest.mark.parametrize("code", [102, 103, 202, 203])
def test_closed_and_impermeable_codes_are_refused(cuda, code):
    with pytest.raises(L.FhdError) as e:
        L.StokesSolver(2, [16, 16], 1.0, 1, bc_lo=[PE, code, PE], bc_hi=[PE, code, PE])
    assert e.value.status == L._capi.FHD_ERR_UNSUPPORTED
