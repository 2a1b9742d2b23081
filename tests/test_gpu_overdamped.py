"""Parity of the overdamped step (advance_timestep_overdamped.f90:135-734)
between the sm_100a library and the oracle on identical seeded inputs."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_parity import dev, host
from tests.test_oracle_multispecies import mass_fields, mix, state

pytestmark = pytest.mark.gpu


def _run(cuda, dim, n, ns, precision="fp64", seed=3):
    nc = P.nc_of(dim, n)
    nE = 1 if dim == 2 else 3
    rng = np.random.default_rng(seed)
    one = np.ones(nc)
    eta = 1.0 + 0.1 * rng.random(nc)
    eta_ed = O.average_cc_to_edge(dim, n, eta)
    T = np.ones(nc)
    T_ed = [one] * nE
    kappa = np.zeros(nc)
    mp = mix(ns) if ns > 1 else None
    sp = O.StochParams(k_B=1e-3 if ns > 1 else 1.0, variance_coef_mom=1.0, dV=100.0 if ns > 1 else 1.0,
                       stoch_stress_form=1, filtering_width=0)
    u0 = [1e-2 * rng.standard_normal(nc) for _ in range(dim)]
    rho0 = state(dim, n, ns) if ns > 1 else [np.ones(nc)]
    pi0 = 1e-2 * rng.standard_normal(nc)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=seed + 1, n_rngs=2)
    W_m = mass_fields(dim, n, ns, seed=seed + 2, n_rngs=2) if ns > 1 else None
    dt = 0.5 if ns > 1 else 0.1
    params = dict(gmres_rel_tol=1e-10)
    rc, u_r, rho_r, pi_r, st_r = O.advance_overdamped(dim, n, 1.0, -1, O.default_params(**params), sp, mp, dt, u0,
                                                      rho0, pi0, eta, eta_ed, kappa, T, T_ed, W_cc, W_ed, W_m)
    assert rc in (0, 3)
    with L.StokesSolver(dim, n, 1.0, -1, params=L.default_params(**params), precision=precision) as s:
        u, rho, pi = dev(u0, cuda), dev(rho0, cuda), dev(pi0, cuda)
        mp_l = L.mixture_params(**_mix_kw(mp)) if mp is not None else None
        sp_l = L.StochParams(k_B=sp.k_B, variance_coef_mom=1.0, dV=sp.dV, stoch_stress_form=1, filtering_width=0)
        status, stats = s.advance_timestep_overdamped(sp_l, mp_l, dt, u, rho, pi, dev(eta, cuda), dev(eta_ed, cuda),
                                                      dev(kappa, cuda), dev(T, cuda), dev(T_ed, cuda),
                                                      dev(W_cc, cuda), dev(W_ed, cuda),
                                                      dev(W_m, cuda) if W_m is not None else None)
    return (host(u), host(rho), host(pi), stats), (u_r, rho_r, pi_r, st_r)


def _mix_kw(mp):
    ns = mp.nspecies
    return dict(molmass=list(mp.molmass[:ns]), Dbar=list(mp.Dbar[:ns * (ns - 1) // 2]),
                rhobar=list(mp.rhobar[:ns]), variance_coef_mass=mp.variance_coef_mass)


@pytest.mark.parametrize("dim,n", [(2, [32, 32]), (3, [16, 16, 16])])
def test_overdamped_single_fluid(cuda, dim, n):
    (u, rho, pi, st), (u_r, rho_r, pi_r, st_r) = _run(cuda, dim, n, 1)
    assert [s["total_iters"] for s in st] == [st_r[0].total_iters, st_r[1].total_iters]
    assert P.rel_inf(u, u_r) < 1e-10
    assert P.rel_inf([pi], [pi_r]) < 1e-10
    assert np.abs(rho[0] - rho_r[0]).max() < 1e-12


@pytest.mark.parametrize("dim,n", [(2, [32, 32]), (3, [16, 16, 16])])
def test_overdamped_mixture(cuda, dim, n):
    (u, rho, pi, st), (u_r, rho_r, pi_r, st_r) = _run(cuda, dim, n, 3)
    assert P.rel_inf(u, u_r) < 1e-10
    assert P.rel_inf([pi], [pi_r]) < 1e-10
    for s in range(3):
        assert np.abs(rho[s] - rho_r[s]).max() < 1e-12 * np.abs(rho_r[s]).max()


def test_overdamped_mixture_mixed_precision(cuda):
    (u, rho, pi, st), (u_r, rho_r, pi_r, st_r) = _run(cuda, 3, [16, 16, 16], 3, precision="mixed")
    # FP32 preconditioner and stochastic fluxes, FP64 outer solve at 1e-10
    assert P.rel_inf(u, u_r) < 1e-5
    for s in range(3):
        assert np.abs(rho[s] - rho_r[s]).max() < 1e-6 * np.abs(rho_r[s]).max()
