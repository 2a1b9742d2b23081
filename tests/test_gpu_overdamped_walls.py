"""The overdamped step (advance_timestep_overdamped.f90:135-734) in a box with
homogeneous walls (visc_type 1): GPU against the oracle on identical seeded
inputs, FP64 and mixed.  The step's walls are those of its parts: the Stokes
solve, the stochastic momentum flux (the high wall's edge planes), the mass
fluxes and the zero pressure gradient on wall faces; density advection
carries nothing through a wall face, where the normal velocity is zero."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_parity import dev, host
from tests.test_gpu_overdamped import _mix_kw
from tests.test_oracle_overdamped_walls import inputs

pytestmark = pytest.mark.gpu

NS, SL, PE = L.FHD_BC_NO_SLIP_WALL, L.FHD_BC_SLIP_WALL, L.FHD_BC_PERIODIC


@pytest.fixture(autouse=True)
def periodic_afterwards():
    yield
    O.set_walls()


def _run(cuda, dim, n, ns, bc_lo, bc_hi, precision="fp64"):
    a = inputs(dim, n, ns, bc_lo)
    O.set_walls(bc_lo, bc_hi)
    params = dict(gmres_rel_tol=1e-10)
    rc, u_r, rho_r, pi_r, st_r = O.advance_overdamped(dim, n, 1.0, 1, O.default_params(**params), a["sp"], a["mp"],
                                                      a["dt"], a["u"], a["rho"], a["pi"], a["eta"], a["eta_ed"],
                                                      a["kappa"], a["T"], a["T_ed"], a["W_cc"], a["W_ed"], a["W_m"])
    assert rc in (0, 3)
    with L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(**params), precision=precision, bc_lo=bc_lo,
                        bc_hi=bc_hi) as s:
        u, rho, pi = dev(a["u"], cuda), dev(a["rho"], cuda), dev(a["pi"], cuda)
        mp_l = L.mixture_params(**_mix_kw(a["mp"])) if a["mp"] is not None else None
        sp = a["sp"]
        sp_l = L.StochParams(k_B=sp.k_B, variance_coef_mom=1.0, dV=sp.dV, stoch_stress_form=1, filtering_width=0)
        status, stats = s.advance_timestep_overdamped(sp_l, mp_l, a["dt"], u, rho, pi, dev(a["eta"], cuda),
                                                      dev(a["eta_ed"], cuda), dev(a["kappa"], cuda),
                                                      dev(a["T"], cuda), dev(a["T_ed"], cuda), dev(a["W_cc"], cuda),
                                                      dev(a["W_ed"], cuda),
                                                      dev(a["W_m"], cuda) if a["W_m"] is not None else None)
    return (host(u), host(rho), host(pi), stats), (u_r, rho_r, pi_r, st_r)


CASES = [(2, [32, 32], [PE, NS, PE], [PE, NS, PE]), (2, [32, 16], [SL, NS, PE], [SL, NS, PE]),
         (3, [16, 16, 16], [PE, PE, NS], [PE, PE, NS]), (3, [16, 16, 16], [NS, SL, PE], [NS, SL, PE])]


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
@pytest.mark.parametrize("ns", [1, 3])
def test_overdamped_walls(cuda, dim, n, bc_lo, bc_hi, ns):
    (u, rho, pi, st), (u_r, rho_r, pi_r, st_r) = _run(cuda, dim, n, ns, bc_lo, bc_hi)
    assert [s["total_iters"] for s in st] == [st_r[0].total_iters, st_r[1].total_iters]
    assert P.rel_inf(u, u_r) < 1e-10
    assert P.rel_inf([pi - pi.mean()], [pi_r - pi_r.mean()]) < 1e-10
    for s in range(ns):
        assert np.abs(rho[s] - rho_r[s]).max() < 1e-12 * np.abs(rho_r[s]).max()


def test_overdamped_walls_mixed_precision(cuda):
    dim, n, bc_lo, bc_hi = 3, [16, 16, 16], [NS, SL, PE], [NS, SL, PE]
    (u, rho, pi, st), (u_r, rho_r, pi_r, st_r) = _run(cuda, dim, n, 3, bc_lo, bc_hi, precision="mixed")
    assert P.rel_inf(u, u_r) < 1e-5
    for s in range(3):
        assert np.abs(rho[s] - rho_r[s]).max() < 1e-6 * np.abs(rho_r[s]).max()
