"""The oracle's multispecies mass fluxes (src_multiSpec of LowMachFHD):
structural identities the reference guarantees and a fluctuation-
dissipation check of the stochastic flux."""
import numpy as np
import pytest

import oracle as O
from tests import problems as P

MOLMASS = [1.0, 2.0, 3.0, 4.0, 5.0]


def mix(ns=4, seed=0, var=1.0):
    rng = np.random.default_rng(seed)
    D = rng.uniform(0.5, 2.0, ns * (ns - 1) // 2) * 1e-2
    return O.mixture_params(MOLMASS[:ns], list(D), rhobar=[1.0] * ns, variance_coef_mass=var)


def state(dim, n, ns, seed=1, amp=1e-3):
    rng = np.random.default_rng(seed)
    nc = P.nc_of(dim, n)
    w = 1.0 / ns + amp * rng.standard_normal((ns, nc))
    w /= w.sum(axis=0)
    return [np.ascontiguousarray(w[i]) for i in range(ns)]


def mass_fields(dim, n, ns, seed=2, n_rngs=1):
    rng = np.random.default_rng(seed)
    nc = P.nc_of(dim, n)
    return [rng.standard_normal(nc) for _ in range(n_rngs * dim * ns)]


@pytest.mark.parametrize("ns", [2, 3, 4])
def test_onsager_cholesky(ns):
    mp = mix(ns)
    rho = np.array(state(3, [2, 2, 2], ns)).T[0]
    kB = 1e-4
    rc, chi, L = O.mixture_local(mp, kB, rho)
    assert rc == 0
    assert np.allclose(chi, chi.T, atol=1e-14 * np.abs(chi).max())
    rt = rho.sum()
    W = rho / rt
    mtot = 1.0 / np.sum(W / np.array(MOLMASS[:ns]))
    onsager = mtot * rt * np.outer(W, W) * chi / kB
    assert np.allclose(L @ L.T, onsager, rtol=1e-8, atol=1e-10 * np.abs(onsager).max())
    assert np.all(np.triu(L, 1) == 0)


@pytest.mark.parametrize("dim,n,ns", [(2, [16, 12], 3), (3, [8, 8, 8], 4)])
def test_mass_fluxdiv_conservation(dim, n, ns):
    mp = mix(ns)
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-2)
    W = mass_fields(dim, n, ns)
    div, flux = O.mass_fluxdiv(dim, n, 1.0, sp, mp, rho, 0.05, [1.0], W, want_flux=True)
    # corrected fluxes sum to zero over species on every face
    for d in range(dim):
        s = sum(flux[d * ns + i] for i in range(ns))
        assert np.max(np.abs(s)) <= 1e-12 * max(np.max(np.abs(f)) for f in flux)
    # every species' divergence sums to zero over the periodic box
    for i in range(ns):
        assert abs(div[i].sum()) <= 1e-10 * np.abs(div[i]).sum()


def test_stochastic_mass_flux_covariance():
    """fluctuation-dissipation: on a uniform state the stochastic flux on a
    face has covariance variance^2 * L (stochastic_mass_fluxdiv.f90:70-88)"""
    dim, n, ns = 3, [24, 24, 24], 3
    mp = mix(ns)
    # dV large enough that the C0-smoothed Heaviside of compute_nonnegative_rho_av
    # (min(dV*rho/m, 1)) is inactive, so rho_av equals rho
    kB, dV, dt = 1e-4, 100.0, 0.05
    sp = O.StochParams(k_B=kB, variance_coef_mom=1.0, dV=dV, stoch_stress_form=1, filtering_width=0)
    nc = P.nc_of(dim, n)
    w0 = np.array([0.2, 0.35, 0.45])
    rho = [np.full(nc, w0[i]) for i in range(ns)]
    W = mass_fields(dim, n, ns, seed=7)
    _, flux = O.mass_fluxdiv(dim, n, 1.0, sp, mp, rho, dt, [1.0], W, want_flux=True)
    samples = np.concatenate([np.stack([flux[d * ns + i] for i in range(ns)]) for d in range(dim)], axis=1)
    cov = samples @ samples.T / samples.shape[1]
    rc, chi, L = O.mixture_local(mp, kB, w0)
    expect = (2.0 * kB / (dV * dt)) * (L @ L.T)
    # 3*24^3 samples: relative standard error ~ 0.5 %
    assert np.allclose(cov, expect, rtol=0.03, atol=0.03 * np.abs(expect).max())


def test_multispecies_step_conserves_mass():
    dim, n, ns = 3, [8, 8, 8], 4
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
    rc, u, r, p, F1, st = O.advance_inertial_ms(dim, n, 1.0, 1, O.default_params(gmres_rel_tol=1e-9), sp, mp, 0.05,
                                                umac, rho, np.zeros(nc), F0, eta, ee, np.zeros(nc), np.ones(nc), ee,
                                                W_cc, W_ed, W_mass)
    assert rc == 0
    for i in range(ns):
        assert abs(r[i].sum() - rho[i].sum()) <= 1e-12 * rho[i].sum()
    assert st[0].total_iters >= 1 and st[1].total_iters >= 1


BASE = np.array([0.2, 0.35, 0.45, 0.3, 0.25])


@pytest.mark.parametrize("ns", [3, 4, 5])
@pytest.mark.parametrize("trace", [(0,), (1,), ("last",), (0, 2)])
def test_trace_species_limit(ns, trace):
    """The trace-species subsystem (compute_chi_sub and
    compute_sqrtLonsager_sub, mass_flux_utilities.f90:654-739, 1425-1502) is
    the limit of the full system as the trace mass fractions go to zero: rho W
    chi to the truncation of the 10-step chi iteration, the Cholesky factor at
    the rate sqrt(w) (its trace pivot is O(w))."""
    idx = [ns - 1 if t == "last" else t for t in trace]
    if len(idx) >= ns - 1:
        pytest.skip("all but one trace: zero by definition")
    mp = mix(ns)
    r_small, r_zero = BASE[:ns].copy(), BASE[:ns].copy()
    r_small[idx] = 1e-12
    r_zero[idx] = 0.0
    a1, L1 = O.mixture_trace_local(mp, 1e-4, r_small)
    a0, L0 = O.mixture_trace_local(mp, 1e-4, r_zero)
    assert np.all(np.isfinite(a0)) and np.all(np.isfinite(L0))
    assert np.abs(a1 - a0).max() <= 5e-6 * np.abs(a0).max()
    assert np.abs(L1 - L0).max() <= 1e-5 * np.abs(L0).max()
    # the subsystem factor is expanded with zero rows and columns
    assert np.all(L0[idx, :] == 0.0) and np.all(L0[:, idx] == 0.0)
    assert np.all(np.triu(L0, 1) == 0.0)
    # rho W chi of a trace species: zero rows except the diagonal entry
    for k in idx:
        row = a0[k].copy()
        assert row[k] > 0.0
        row[k] = 0.0
        assert np.all(row == 0.0)


@pytest.mark.parametrize("ns", [2, 3, 4])
def test_all_but_one_trace(ns):
    mp = mix(ns)
    r = np.zeros(ns)
    r[1 % ns] = 0.9
    a, L = O.mixture_trace_local(mp, 1e-4, r)
    assert np.all(a == 0.0) and np.all(L == 0.0)


def test_mass_fluxdiv_with_trace_cells():
    """A state where species densities vanish on some cells (faces with one,
    two and all-but-one trace species): the fluxes stay finite and
    conservative."""
    dim, n, ns = 3, [8, 8, 8], 4
    mp = mix(ns)
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = trace_state(dim, n, ns)
    W = mass_fields(dim, n, ns)
    div, flux = O.mass_fluxdiv(dim, n, 1.0, sp, mp, rho, 0.05, [1.0], W, want_flux=True)
    assert all(np.all(np.isfinite(d)) for d in div)
    for d in range(dim):
        s = sum(flux[d * ns + i] for i in range(ns))
        assert np.max(np.abs(s)) <= 1e-12 * max(np.max(np.abs(f)) for f in flux)
    for i in range(ns):
        assert abs(div[i].sum()) <= 1e-10 * np.abs(div[i]).sum()


def trace_state(dim, n, ns, seed=5, amp=1e-2):
    """mass fractions near 1/ns with seeded cells where one species, two
    species or every species but one has zero density.  The modified cells
    are on one colour of the checkerboard, so no two share a face: a face
    between cells of disjoint species support would have a zero averaged
    density (0/0 in compute_sqrtLonsager_local, as in the reference)."""
    rho = state(dim, n, ns, seed=seed, amp=amp)
    rng = np.random.default_rng(seed + 100)
    nn = list(n) + [1] * (3 - dim)
    i, j, k = np.meshgrid(*[np.arange(m) for m in nn], indexing="ij")
    even = ((i + j + k) % 2 == 0).transpose(2, 1, 0).reshape(-1)  # x fastest
    cells = rng.permutation(np.flatnonzero(even))
    q = len(cells) // 4
    for c in cells[:q]:                      # one trace species
        rho[int(rng.integers(ns))][c] = 0.0
    for c in cells[q:2 * q]:                 # two trace species (never all of them)
        for s in rng.choice(ns, min(2, ns - 1), replace=False):
            rho[int(s)][c] = 0.0
    for c in cells[2 * q:3 * q]:             # all but one
        keep = int(rng.integers(ns))
        for s in range(ns):
            if s != keep:
                rho[s][c] = 0.0
    return rho


@pytest.mark.parametrize("dim,n,ns", [(2, [16, 12], 3), (3, [8, 8, 8], 4)])
def test_split_stochastic_mass_flux_matches_combined(dim, n, ns):
    """compute_sqrtLonsager_fc + stochastic_mass_fluxdiv (the drop-in
    boundary's split form) equal the stochastic part of the fused
    compute_mass_fluxdiv: total minus the diffusive-only flux"""
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = trace_state(dim, n, ns)
    W = mass_fields(dim, n, ns, n_rngs=2)
    mp = mix(ns)
    sqL = O.sqrtLonsager_fc(dim, n, sp, mp, rho)
    _, flux = O.stochastic_mass_fluxdiv(dim, n, 1.0, sp, mp, sqL, 0.05, [0.7, -0.3], W, want_flux=True)
    _, f_all = O.mass_fluxdiv(dim, n, 1.0, sp, mp, rho, 0.05, [0.7, -0.3], W, want_flux=True)
    _, f_dif = O.mass_fluxdiv(dim, n, 1.0, sp, mix(ns, var=0.0), rho, 0.05, [0.7, -0.3], W, want_flux=True)
    scale = max(np.abs(f).max() for f in flux)
    assert max(np.abs((a - b) - c).max() for a, b, c in zip(f_all, f_dif, flux)) <= 1e-13 * scale
