"""Moving no-slip walls (fhd_ctx_set_wall_speed: wallspeed_lo / wallspeed_hi)
in the device timesteps, against the oracle on identical seeded inputs:
overdamped, inertial and multispecies inertial, 2D and 3D, FP64 (and one
mixed case); at 128^2 the noise-free overdamped step against the exact
plane Couette profile; the refusal of a speed on a slip wall."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_overdamped import _mix_kw
from tests.test_gpu_parity import dev, host
from tests.test_oracle_inertial_walls import step
from tests.test_oracle_moving_walls import couette, quiet_inputs, speeds
from tests.test_oracle_overdamped_walls import inputs

pytestmark = pytest.mark.gpu

NS, SL, PE = L.FHD_BC_NO_SLIP_WALL, L.FHD_BC_SLIP_WALL, L.FHD_BC_PERIODIC


@pytest.fixture(autouse=True)
def still_and_periodic_afterwards():
    yield
    O.set_walls()
    O.set_wall_speed()


CASES = [
    (2, [32, 32], [PE, NS, PE], [PE, NS, PE], speeds(2, 1, [-0.02], [0.03])),
    (3, [16, 16, 16], [PE, PE, NS], [PE, PE, NS], speeds(3, 2, [0.01, -0.005], [0.02, 0.004])),
    (3, [16, 16, 16], [NS, SL, PE], [NS, SL, PE], speeds(3, 0, [0.002, 0.004], [-0.003, 0.001])),
]


def solver(dim, n, bc_lo, bc_hi, ws, precision="fp64"):
    s = L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(gmres_rel_tol=1e-10), precision=precision,
                       bc_lo=bc_lo, bc_hi=bc_hi)
    s.set_wall_speed(*ws)
    return s


def sp_of(sp):
    return L.StochParams(k_B=sp.k_B, variance_coef_mom=1.0, dV=sp.dV, stoch_stress_form=1, filtering_width=0)


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi,ws", CASES)
@pytest.mark.parametrize("ns", [1, 3])
def test_overdamped_moving_walls(cuda, dim, n, bc_lo, bc_hi, ws, ns):
    a = inputs(dim, n, ns, bc_lo)
    O.set_walls(bc_lo, bc_hi)
    O.set_wall_speed(*ws)
    rc, u_r, rho_r, pi_r, st_r = O.advance_overdamped(dim, n, 1.0, 1, O.default_params(gmres_rel_tol=1e-10),
                                                      a["sp"], a["mp"], a["dt"], a["u"], a["rho"], a["pi"], a["eta"],
                                                      a["eta_ed"], a["kappa"], a["T"], a["T_ed"], a["W_cc"],
                                                      a["W_ed"], a["W_m"])
    assert rc in (0, 3)
    with solver(dim, n, bc_lo, bc_hi, ws) as s:
        u, rho, pi = dev(a["u"], cuda), dev(a["rho"], cuda), dev(a["pi"], cuda)
        mp_l = L.mixture_params(**_mix_kw(a["mp"])) if a["mp"] is not None else None
        status, st = s.advance_timestep_overdamped(sp_of(a["sp"]), mp_l, a["dt"], u, rho, pi, dev(a["eta"], cuda),
                                                   dev(a["eta_ed"], cuda), dev(a["kappa"], cuda), dev(a["T"], cuda),
                                                   dev(a["T_ed"], cuda), dev(a["W_cc"], cuda), dev(a["W_ed"], cuda),
                                                   dev(a["W_m"], cuda) if a["W_m"] is not None else None)
    pi = host(pi)
    assert P.rel_inf(host(u), u_r) < 1e-10
    assert P.rel_inf([pi - pi.mean()], [pi_r - pi_r.mean()]) < 1e-10
    for q in range(ns):
        assert np.abs(host(rho)[q] - rho_r[q]).max() < 1e-12 * np.abs(rho_r[q]).max()
    assert [x["total_iters"] for x in st] == [st_r[0].total_iters, st_r[1].total_iters]


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi,ws", CASES)
@pytest.mark.parametrize("ns", [1, 3])
def test_inertial_moving_walls(cuda, dim, n, bc_lo, bc_hi, ws, ns):
    O.set_wall_speed(*ws)
    a, rc, u_r, rho_r, pi_r, F_r = step(dim, n, ns, bc_lo, bc_hi)
    assert rc in (0, 3)
    W_cc1 = a["W_cc"][:dim]
    W_ed1 = a["W_ed"][:len(a["W_ed"]) // 2]
    with solver(dim, n, bc_lo, bc_hi, ws) as s:
        u, pi = dev(a["u"], cuda), dev(a["pi"], cuda)
        common = (dev(a["eta"], cuda), dev(a["eta_ed"], cuda), dev(a["kappa"], cuda), dev(a["T"], cuda),
                  dev(a["T_ed"], cuda), dev(W_cc1, cuda), dev(W_ed1, cuda))
        if ns == 1:
            rho = dev(a["rho"][0], cuda)
            s.advance_timestep_inertial(sp_of(a["sp"]), a["dt"], u, rho, pi, *common)
            rho = [rho]
        else:
            rho = dev(a["rho"], cuda)
            F0 = O.mass_fluxdiv(dim, n, 1.0, a["sp"], a["mp"], a["rho"], a["dt"], [1.0], a["W_m"][:dim * ns])
            s.advance_timestep_inertial_multispecies(sp_of(a["sp"]), L.mixture_params(**_mix_kw(a["mp"])), a["dt"],
                                                     u, rho, pi, dev(F0, cuda), *common, dev(a["W_m"], cuda))
    assert P.rel_inf(host(u), u_r) < 1e-10
    pi = host(pi)
    assert P.rel_inf([pi - pi.mean()], [pi_r - pi_r.mean()]) < 1e-10
    for q in range(ns):
        assert np.abs(host(rho[q]) - rho_r[q]).max() < 1e-12 * np.abs(rho_r[q]).max()


def test_overdamped_moving_walls_mixed_precision(cuda):
    dim, n, bc_lo, bc_hi, ws = CASES[1]
    a = inputs(dim, n, 1, bc_lo)
    O.set_walls(bc_lo, bc_hi)
    O.set_wall_speed(*ws)
    rc, u_r, rho_r, pi_r, st_r = O.advance_overdamped(dim, n, 1.0, 1, O.default_params(gmres_rel_tol=1e-10),
                                                      a["sp"], None, a["dt"], a["u"], a["rho"], a["pi"], a["eta"],
                                                      a["eta_ed"], a["kappa"], a["T"], a["T_ed"], a["W_cc"],
                                                      a["W_ed"], None)
    with solver(dim, n, bc_lo, bc_hi, ws, precision="mixed") as s:
        u, rho, pi = dev(a["u"], cuda), dev(a["rho"], cuda), dev(a["pi"], cuda)
        s.advance_timestep_overdamped(sp_of(a["sp"]), None, a["dt"], u, rho, pi, dev(a["eta"], cuda),
                                      dev(a["eta_ed"], cuda), dev(a["kappa"], cuda), dev(a["T"], cuda),
                                      dev(a["T_ed"], cuda), dev(a["W_cc"], cuda), dev(a["W_ed"], cuda), None)
    assert P.rel_inf(host(u), u_r) < 1e-5


def test_couette_flow_at_128_squared(cuda):
    """noise-free overdamped step from rest between walls moving at -1 and
    +1: the exact linear profile (a size-independent known answer)"""
    dim, n, d = 2, [128, 128], 1
    bc = [PE, NS, PE]
    a = quiet_inputs(dim, n, bc)
    nc = 128 * 128
    with L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(gmres_rel_tol=1e-12), bc_lo=bc, bc_hi=bc) as s:
        s.set_wall_speed(*speeds(dim, d, [-1.0], [1.0]))
        u, rho, pi = dev([np.zeros(nc), np.zeros(nc)], cuda), dev([a["rho"]], cuda), dev(a["pi"], cuda)
        s.advance_timestep_overdamped(sp_of(a["sp"]), None, 0.1, u, rho, pi, dev(a["eta"], cuda),
                                      dev(a["eta_ed"], cuda), dev(a["kappa"], cuda), dev(a["T"], cuda),
                                      dev(a["T_ed"], cuda), dev(a["W_cc"], cuda), dev(a["W_ed"], cuda), None)
    want = couette(dim, n, d, -1.0, 1.0)
    got = host(u)
    assert np.max(np.abs(got[0] - want)) < 1e-8
    assert np.max(np.abs(got[1])) < 1e-8


def test_speed_on_a_slip_wall_is_refused(cuda):
    with L.StokesSolver(2, [16, 16], 1.0, 1, bc_lo=[PE, SL, PE], bc_hi=[PE, NS, PE]) as s:
        with pytest.raises(L.FhdError) as e:
            s.set_wall_speed(*speeds(2, 1, [1.0], [0.0]))
        assert e.value.status == L._capi.FHD_ERR_UNSUPPORTED
        s.set_wall_speed(*speeds(2, 1, [0.0], [1.0]))  # the no-slip side may move
