"""The CPU oracle against the reference's own stored results.

* Discretisation-error KAT: exec/stokes_preconditioner/test_gmres/run_result/
  Accuracy_tests/{2d,3d}_dis_accuracy.dat (main_driver.f90 test_type = 0),
  extracted into tests/golden/accuracy_kat.json by make_accuracy_kat.py.
* Staggered multigrid residual history shape: run_result/
  Mg_StagMg_performance/3d_periodic_precon_finegridGS_8botsmooth_vel.dat
  (per-V-cycle reduction 0.045 .. 0.097, 3D periodic, GS, 8 bottom smooths).
* Pressure multigrid residual history: run_result/Mg_StagMg_performance/
  3d_periodic_precon_finegridGS_pre.dat (64^3 periodic, GS; per-V-cycle
  reduction 0.035 .. 0.080, settling near 0.08).
* GMRES iteration counts for periodic constant-coefficient Stokes
  (doc/Stokes_Preconditioners.tex:408-429: 1-2 iterations).
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from tests import problems as P

GOLD = os.path.join(os.path.dirname(__file__), "golden", "accuracy_kat.json")
ROWS = json.load(open(GOLD))


def _id(r):
    return f"{r['dim']}d-n{r['n']}-c{r['prob_coeff']}-s{r['prob_sol']}-v{r['visc_type']}"


@pytest.mark.parametrize("row", [r for r in ROWS if r["n"] <= (64 if r["dim"] == 3 else 128)], ids=_id)
def test_accuracy_kat(row):
    err = O.accuracy_test(row["dim"], row["n"], row["prob_coeff"], row["prob_sol"], row["visc_type"])
    keys = ["U", "V", "W"][: row["dim"]] + ["P"]
    for i, k in enumerate(keys):
        if k not in row["errors"]:
            continue
        ref = row["errors"][k]
        # roundoff of the O(1/dx^2) stencil sums: ~1e-9 relative at 128^2
        assert abs(err[i] - ref) <= 1e-8 * abs(ref), (k, err[i], ref)


def test_accuracy_second_order():
    e = [O.accuracy_test(2, n, 1, 31, 1)[0] for n in (32, 64, 128)]
    assert 3.9 < e[0] / e[1] < 4.1 and 3.9 < e[1] / e[2] < 4.1


def test_nlevs_mg():
    # stag_mg_layout.f90:202-208: coarsen while even and length/minwidth != 1
    assert O.compute_nlevs_mg(2, [64, 64]) == 6
    assert O.compute_nlevs_mg(3, [128, 128, 128]) == 7
    assert O.compute_nlevs_mg(3, [256, 256, 256]) == 8
    assert O.compute_nlevs_mg(2, [96, 96]) == 6  # 96,48,24,12,6,3
    assert O.compute_nlevs_mg(3, [64, 64, 64], 4) == 5


def test_stag_mg_history_shape():
    dim, n = 3, [32, 32, 32]
    nc = P.nc_of(dim, n)
    pb = O.Problem(dim, n, 1.0, 1, [np.ones(nc)] * 3, np.ones(nc), [np.ones(nc)] * 3, np.zeros(nc))
    rng = np.random.default_rng(10)
    rhs = [rng.uniform(size=nc) for _ in range(3)]
    rhs = [r - r.mean() for r in rhs]
    p = O.default_params(stag_mg_max_vcycles=8, stag_mg_minwidth=4, stag_mg_rel_tol=1e-14)
    h = O.stag_mg_history(pb, p, 0.0, rhs)
    rates = h[1:] / h[:-1]
    assert h[0] < 0.05
    assert np.all(rates > 0.03) and np.all(rates < 0.15), rates


# per-V-cycle reductions of the stored 64^3 periodic pressure history
PRES_REF = [0.0346, 0.0665, 0.0642, 0.0741, 0.0717, 0.0743, 0.0745, 0.0759, 0.0794, 0.0795]


def test_pressure_mg_history_matches_the_reference_rate():
    """the pressure multigrid (macproject.f90, the reference's settings:
    2 + 2 red-black GS sweeps, 8 bottom smooths) on the 64^3 periodic
    constant-coefficient Poisson problem: the per-V-cycle reduction settles
    where the reference's stored history does (0.08); the first cycles depend
    on the right-hand side, which the stored run does not record"""
    dim, n = 3, [64, 64, 64]
    nc = 64 ** 3
    rng = np.random.default_rng(10)
    rhs = rng.uniform(size=nc)
    rhs -= rhs.mean()
    h = O.macproject_history(dim, n, 1.0, O.default_params(mg_max_vcycles=11), [np.ones(nc)] * 3, rhs)
    rates = h[1:] / h[:-1]
    assert np.all(rates > 0.03) and np.all(rates < 0.09), rates
    asym, ref = rates[-4:].mean(), np.mean(PRES_REF[-4:])
    assert abs(asym - ref) < 0.1 * ref, (asym, ref)


@pytest.mark.parametrize("precon,iters", [(1, 1), (-1, 1), (2, 2), (5, 1)])
def test_gmres_periodic_iterations_exact_inner(precon, iters):
    """Stokes_Preconditioners.tex:385-429 (Test 1, BC=4, rho=1, mu=1, h=1,
    dt=0.5): with exact inner solves the projection preconditioner takes 1
    iteration and the lower-triangular one 2 on a periodic box."""
    dim, n = 2, [64, 64]
    pb = P.problem(dim, n, 1, dx=1.0)
    for c in range(dim):
        pb.alpha_fc[c][:] = 1.0
    pb.beta[:] = 1.0
    pb.beta_ed[0][:] = 1.0
    pb.gamma[:] = 0.0
    u, p = P.random_stokes(dim, n, seed=3)
    theta = 2.0
    b_u, b_p = O.apply_matrix(pb, theta, u, p)
    params = O.default_params(precon_type=precon, stag_mg_max_vcycles=100, stag_mg_rel_tol=1e-13,
                              mg_max_vcycles=100, mg_rel_tol=1e-13, gmres_rel_tol=1e-8)
    rc, xu, xp, npr, st = O.gmres(pb, params, theta, b_u, b_p)
    assert rc == 0
    assert st.total_iters == iters
    assert P.rel_inf(xu, u) < 1e-6


@pytest.mark.parametrize("precon", [1, -1, 2, -2, 3, -3, 4, -4, 5])
def test_gmres_all_precon_types_converge(precon):
    dim, n = 2, [32, 32]
    pb = P.problem(dim, n, -1, dx=1.0 / 32)
    u, p = P.random_stokes(dim, n, seed=3)
    b_u, b_p = O.apply_matrix(pb, 1.0, u, p)
    rc, xu, xp, npr, st = O.gmres(pb, O.default_params(precon_type=precon), 1.0, b_u, b_p)
    assert rc in (0, 3) and st.total_iters <= 40  # 3: true-residual warning only
    assert P.rel_inf(xu, u) < 1e-6


def test_gmres_overdamped_stochastic():
    # configuration 1: 2D 64^2 periodic, overdamped, stochastic forcing
    dim, n = 2, [64, 64]
    pb = P.problem(dim, n, 1, variable=False)
    pb.beta[:] = 1.0
    pb.beta_ed[0][:] = 1.0
    pb.gamma[:] = 0.0
    for c in range(dim):
        pb.alpha_fc[c][:] = 1.0
    sp = O.StochParams(k_B=1.0, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=1)
    ones = np.ones(P.nc_of(dim, n))
    f = O.stochastic_m_fluxdiv(dim, n, 1.0, sp, ones, [ones], ones, [ones], 0.1, [1.0], W_cc, W_ed)
    params = O.default_params(gmres_rel_tol=1e-9)
    rc, xu, xp, npr, st = O.gmres(pb, params, 0.0, f, np.zeros(P.nc_of(dim, n)))
    assert rc == 0
    assert st.norm_resid <= 1e-9 * min(st.norm_pre_b, st.norm_init_resid)
    # the velocity is divergence free and mean free
    b_u, b_p = O.apply_matrix(pb, 0.0, xu, xp)
    assert np.max(np.abs(b_p)) < 1e-7 * np.max(np.abs(xu[0]))
    assert abs(xu[0].mean()) < 1e-12 and abs(xu[1].mean()) < 1e-12


def test_stochastic_flux_sums_to_zero():
    # a divergence on a periodic box has zero sum in every component
    for dim, n in ((2, [16, 24]), (3, [8, 8, 12])):
        sp = O.StochParams(k_B=1.0, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
        W_cc, W_ed = P.stochastic_fields(dim, n, seed=5, n_rngs=2)
        nc = P.nc_of(dim, n)
        rng = np.random.default_rng(2)
        eta = 1 + rng.random(nc)
        T = 1 + rng.random(nc)
        f = O.stochastic_m_fluxdiv(dim, n, 0.5, sp, eta, O.average_cc_to_edge(dim, n, eta), T,
                                   O.average_cc_to_edge(dim, n, T), 0.1, [0.5, -0.25], W_cc, W_ed)
        for c in range(dim):
            assert abs(f[c].sum()) < 1e-10 * np.abs(f[c]).sum()


def test_precon_mean_free():
    dim, n = 3, [8, 8, 8]
    pb = P.problem(dim, n, -2)
    u, p = P.random_stokes(dim, n, seed=4, zero_mean_p=False)
    for theta in (0.0, 2.0):
        xu, xp = O.apply_precon(pb, O.default_params(), theta, u, p)
        assert abs(xp.mean()) < 1e-13
        if theta == 0.0:
            assert max(abs(x.mean()) for x in xu) < 1e-13


def test_inertial_step_runs():
    dim, n = 3, [8, 8, 8]
    nc = P.nc_of(dim, n)
    rng = np.random.default_rng(0)
    umac = [0.01 * rng.standard_normal(nc) for _ in range(dim)]
    rho = np.ones(nc)
    pi = np.zeros(nc)
    eta = np.ones(nc)
    eta_ed = O.average_cc_to_edge(dim, n, eta)
    T = np.ones(nc)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=9)
    sp = O.StochParams(k_B=1e-3, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rc, u2, r2, p2, st = O.advance_inertial(dim, n, 1.0, 1, O.default_params(), sp, 0.05, umac, rho, pi,
                                            eta, eta_ed, np.zeros(nc), T, eta_ed, W_cc, W_ed)
    assert rc == 0
    assert st[0].total_iters >= 1 and st[1].total_iters >= 1
    assert abs(r2.sum() - rho.sum()) < 1e-10 * rho.sum()
