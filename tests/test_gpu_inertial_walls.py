"""The inertial step (advance_timestep_inertial.f90:45-923) in a box with
homogeneous walls (visc_type 1), single fluid and a 3-species mixture: GPU
against the oracle on identical seeded inputs, FP64 with the same GMRES
iterations, and the mixed-precision step."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_overdamped import _mix_kw
from tests.test_gpu_parity import dev, host
from tests.test_oracle_inertial_walls import step

pytestmark = pytest.mark.gpu

NS, SL, PE = L.FHD_BC_NO_SLIP_WALL, L.FHD_BC_SLIP_WALL, L.FHD_BC_PERIODIC


@pytest.fixture(autouse=True)
def periodic_afterwards():
    yield
    O.set_walls()


def _run(cuda, dim, n, ns, bc_lo, bc_hi, precision="fp64"):
    a, rc, u_r, rho_r, pi_r, F_r = step(dim, n, ns, bc_lo, bc_hi)
    assert rc in (0, 3)
    sp = a["sp"]
    sp_l = L.StochParams(k_B=sp.k_B, variance_coef_mom=1.0, dV=sp.dV, stoch_stress_form=1, filtering_width=0)
    W_cc1 = a["W_cc"][:dim]
    W_ed1 = a["W_ed"][:len(a["W_ed"]) // 2]
    with L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(gmres_rel_tol=1e-10), precision=precision,
                        bc_lo=bc_lo, bc_hi=bc_hi) as s:
        u, pi = dev(a["u"], cuda), dev(a["pi"], cuda)
        common = (dev(a["eta"], cuda), dev(a["eta_ed"], cuda), dev(a["kappa"], cuda), dev(a["T"], cuda),
                  dev(a["T_ed"], cuda), dev(W_cc1, cuda), dev(W_ed1, cuda))
        if ns == 1:
            rho = dev(a["rho"][0], cuda)
            status, stats = s.advance_timestep_inertial(sp_l, a["dt"], u, rho, pi, *common)
            rho = [rho]
        else:
            rho = dev(a["rho"], cuda)
            mp_l = L.mixture_params(**_mix_kw(a["mp"]))
            O.set_walls(bc_lo, bc_hi)
            F0 = O.mass_fluxdiv(dim, n, 1.0, sp, a["mp"], a["rho"], a["dt"], [1.0], a["W_m"][:dim * ns])
            F = dev(F0, cuda)
            status, stats = s.advance_timestep_inertial_multispecies(sp_l, mp_l, a["dt"], u, rho, pi, F, *common[:5],
                                                                     *common[5:], dev(a["W_m"], cuda))
    return (host(u), host(rho), host(pi), stats), (u_r, rho_r, pi_r)


CASES = [(2, [32, 32], [PE, NS, PE], [PE, NS, PE]), (2, [32, 16], [SL, NS, PE], [SL, NS, PE]),
         (3, [16, 16, 16], [PE, PE, NS], [PE, PE, NS]), (3, [16, 16, 16], [NS, SL, PE], [NS, SL, PE])]


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
@pytest.mark.parametrize("ns", [1, 3])
def test_inertial_walls(cuda, dim, n, bc_lo, bc_hi, ns):
    (u, rho, pi, st), (u_r, rho_r, pi_r) = _run(cuda, dim, n, ns, bc_lo, bc_hi)
    assert P.rel_inf(u, u_r) < 1e-10
    assert P.rel_inf([pi - pi.mean()], [pi_r - pi_r.mean()]) < 1e-10
    for s in range(ns):
        assert np.abs(rho[s] - rho_r[s]).max() < 1e-12 * np.abs(rho_r[s]).max()


def test_inertial_walls_mixed_precision(cuda):
    (u, rho, pi, st), (u_r, rho_r, pi_r) = _run(cuda, 3, [16, 16, 16], 3, [NS, SL, PE], [NS, SL, PE],
                                                precision="mixed")
    assert P.rel_inf(u, u_r) < 1e-5
    for s in range(3):
        assert np.abs(rho[s] - rho_r[s]).max() < 1e-6 * np.abs(rho_r[s]).max()
