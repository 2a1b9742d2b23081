"""Parity of the sm_100a multispecies mass fluxes and step with the oracle."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_oracle_multispecies import mass_fields, mix, state

pytestmark = pytest.mark.gpu


def dev(a, device):
    import torch
    if isinstance(a, (list, tuple)):
        return [dev(x, device) for x in a]
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(device)


def host(t):
    if isinstance(t, (list, tuple)):
        return [host(x) for x in t]
    return t.detach().cpu().numpy()


def lmix(ns, seed=0, var=1.0):
    m = mix(ns, seed, var)
    return L.mixture_params([m.molmass[i] for i in range(ns)], [m.Dbar[i] for i in range(ns * (ns - 1) // 2)],
                            rhobar=[1.0] * ns, variance_coef_mass=var)


@pytest.mark.parametrize("dim,n,ns", [(2, [16, 24], 2), (2, [16, 16], 3), (3, [8, 8, 8], 4), (3, [8, 12, 8], 5)])
@pytest.mark.parametrize("avg", [1, 10])
def test_mass_fluxdiv(cuda, dim, n, ns, avg):
    mp = mix(ns)
    mp.avg_type = avg
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-2)
    W = mass_fields(dim, n, ns, n_rngs=2)
    ref = O.mass_fluxdiv(dim, n, 1.0, sp, mp, rho, 0.05, [0.7, -0.3], W)
    lm = lmix(ns)
    lm.avg_type = avg
    lsp = L.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    import torch
    with L.StokesSolver(dim, n, 1.0, 1) as s:
        out = [torch.zeros(P.nc_of(dim, n), dtype=torch.float64, device=cuda) for _ in range(ns)]
        s.compute_mass_fluxdiv(lm, lsp, dev(rho, cuda), 0.05, [0.7, -0.3], dev(W, cuda), out)
    assert P.rel_inf(host(out), ref) < 1e-12


def test_mass_fluxdiv_mixed_precision(cuda):
    dim, n, ns = 3, [16, 16, 16], 4
    mp = mix(ns)
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-3)
    W = mass_fields(dim, n, ns)
    ref = O.mass_fluxdiv(dim, n, 1.0, sp, mp, rho, 0.05, [1.0], W)
    import torch
    with L.StokesSolver(dim, n, 1.0, 1, precision="mixed") as s:
        out = [torch.zeros(P.nc_of(dim, n), dtype=torch.float64, device=cuda) for _ in range(ns)]
        s.compute_mass_fluxdiv(lmix(ns), L.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1,
                                                       filtering_width=0), dev(rho, cuda), 0.05, [1.0], dev(W, cuda),
                               out)
    err = P.rel_inf(host(out), ref)
    assert err < 2e-3, err  # FP32 chi iteration and Cholesky


def test_multispecies_step(cuda):
    dim, n, ns = 3, [16, 16, 16], 4
    nc = P.nc_of(dim, n)
    mp = mix(ns)
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-3)
    rng = np.random.default_rng(3)
    umac = [1e-3 * rng.standard_normal(nc) for _ in range(dim)]
    eta = np.ones(nc)
    ee = O.average_cc_to_edge(dim, n, eta)
    W0 = mass_fields(dim, n, ns, seed=4)
    F0 = O.mass_fluxdiv(dim, n, 1.0, sp, mp, rho, 0.05, [1.0], W0)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=5)
    W_mass = W0 + mass_fields(dim, n, ns, seed=6)
    params = O.default_params(gmres_rel_tol=1e-9)
    rc, ru, rr, rp, rF, rst = O.advance_inertial_ms(dim, n, 1.0, 1, params, sp, mp, 0.05, umac, rho, np.zeros(nc), F0,
                                                    eta, ee, np.zeros(nc), np.ones(nc), ee, W_cc, W_ed, W_mass)
    assert rc == 0
    lsp = L.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    with L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(gmres_rel_tol=1e-9)) as s:
        u, r, p, F = dev(umac, cuda), dev(rho, cuda), dev(np.zeros(nc), cuda), dev(F0, cuda)
        status, st = s.advance_timestep_inertial_multispecies(lsp, lmix(ns), 0.05, u, r, p, F, dev(eta, cuda),
                                                              dev(ee, cuda), dev(np.zeros(nc), cuda),
                                                              dev(np.ones(nc), cuda), dev(ee, cuda), dev(W_cc, cuda),
                                                              dev(W_ed, cuda), dev(W_mass, cuda))
    assert status == 0
    assert [x["total_iters"] for x in st] == [rst[0].total_iters, rst[1].total_iters]
    for c in range(dim):
        assert P.rel_inf([host(u[c])], [ru[c]]) < 1e-10
    assert P.rel_inf(host(r), rr) < 1e-12
    assert P.rel_inf(host(F), rF) < 1e-10
    assert P.rel_inf([host(p)], [rp]) < 1e-10
