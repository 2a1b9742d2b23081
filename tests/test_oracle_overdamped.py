"""The oracle's overdamped timestep (advance_timestep_overdamped.f90:135-734):
identities the reference scheme guarantees on a periodic box."""
import numpy as np
import pytest

import oracle as O
from tests import problems as P
from tests.test_oracle_multispecies import mass_fields, mix, state


def _coef(dim, n):
    nc = P.nc_of(dim, n)
    nE = 1 if dim == 2 else 3
    one = np.ones(nc)
    return nc, one, [one] * nE, np.zeros(nc), one, [one] * nE


def _div(dim, n, dx, u):
    """discrete divergence of face velocities (low-side faces), periodic"""
    shape = tuple(reversed(n[:dim]))
    d = np.zeros(shape)
    for c in range(dim):
        a = u[c].reshape(shape)
        d += (np.roll(a, -1, axis=dim - 1 - c) - a) / dx
    return d


def test_quiescent_state_stays_quiescent():
    dim, n = 2, [16, 16]
    nc, eta, eta_ed, kappa, T, T_ed = _coef(dim, n)
    sp = O.StochParams(k_B=1.0, variance_coef_mom=0.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=1, n_rngs=2)
    rc, u, rho, pi, st = O.advance_overdamped(dim, n, 1.0, 1, O.default_params(gmres_rel_tol=1e-10), sp, None, 0.1,
                                              [np.zeros(nc) for _ in range(dim)], [np.ones(nc)], np.zeros(nc), eta,
                                              eta_ed, kappa, T, T_ed, W_cc, W_ed)
    assert rc == 0
    assert max(np.abs(x).max() for x in u) == 0.0
    assert np.abs(pi).max() == 0.0
    assert np.array_equal(rho[0], np.ones(nc))


@pytest.mark.parametrize("dim,n", [(2, [32, 32]), (3, [8, 8, 8])])
def test_single_fluid_step_is_divergence_free(dim, n):
    nc, eta, eta_ed, kappa, T, T_ed = _coef(dim, n)
    sp = O.StochParams(k_B=1.0, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=3, n_rngs=2)
    rc, u, rho, pi, st = O.advance_overdamped(dim, n, 1.0, 1, O.default_params(gmres_rel_tol=1e-10), sp, None, 0.1,
                                              [np.zeros(nc) for _ in range(dim)], [np.ones(nc)], np.zeros(nc), eta,
                                              eta_ed, kappa, T, T_ed, W_cc, W_ed)
    assert rc in (0, 3)
    assert st[0].total_iters >= 1 and st[1].total_iters >= 1
    umax = max(np.abs(x).max() for x in u)
    assert umax > 0
    # the corrector solves D u = 0 to the GMRES tolerance
    assert np.abs(_div(dim, n, 1.0, u)).max() < 1e-7 * umax
    # a divergence-free velocity carries a uniform density unchanged
    assert np.abs(rho[0] - 1.0).max() < 1e-6


def test_mixture_step_conserves_every_species():
    dim, n, ns = 2, [16, 16], 3
    nc, eta, eta_ed, kappa, T, T_ed = _coef(dim, n)
    mp = mix(ns)
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=100.0, stoch_stress_form=1, filtering_width=0)
    rho0 = state(dim, n, ns)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=4, n_rngs=2)
    W_m = mass_fields(dim, n, ns, seed=5, n_rngs=2)
    rc, u, rho, pi, st = O.advance_overdamped(dim, n, 1.0, 1, O.default_params(gmres_rel_tol=1e-10), sp, mp, 0.5,
                                              [np.zeros(nc) for _ in range(dim)], rho0, np.zeros(nc), eta, eta_ed,
                                              kappa, T, T_ed, W_cc, W_ed, W_m)
    assert rc in (0, 3)
    for s in range(ns):
        assert abs(rho[s].sum() - rho0[s].sum()) < 1e-12 * nc
        assert not np.array_equal(rho[s], rho0[s])
