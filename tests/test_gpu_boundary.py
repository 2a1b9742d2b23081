"""The host BoxLib-fab entry points a Fortran driver binds for the
staggered multigrid and the split stochastic mass flux:
fhd_stag_mg_solve (stag_mg_solver.f90:37-50), fhd_compute_sqrtLonsager_fc
(mass_flux_utilities.f90:1096-1229) and fhd_stochastic_mass_fluxdiv
(stochastic_mass_fluxdiv.f90:37-51), with one and two boxes per multifab,
against the oracle; and their device-pointer forms."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_multispecies import dev, host, lmix
from tests.test_oracle_multispecies import mass_fields, mix, state, trace_state

pytestmark = pytest.mark.gpu


def boxes(dim, n, nboxes):
    """lo/hi of the boxes of a level split along x"""
    if nboxes == 1:
        return [([0] * dim, [k - 1 for k in n[:dim]])]
    half = n[0] // 2
    return [([0] + [0] * (dim - 1), [half - 1] + [k - 1 for k in n[1:dim]]),
            ([half] + [0] * (dim - 1), [n[0] - 1] + [k - 1 for k in n[1:dim]])]


def mf(xs, dim, n, nodal, ng, nboxes):
    """a multifab of the canonical arrays xs (one per component)"""
    xs = xs if isinstance(xs, (list, tuple)) else [xs]
    return [L.fab_from_components(xs, dim, n, nodal, ng, lo=lo, hi=hi) for lo, hi in boxes(dim, n, nboxes)]


def assert_mf(got, xs, dim, n, nodal, ng, nboxes, tol):
    want = mf(xs, dim, n, nodal, ng, nboxes)
    scale = max(float(np.max(np.abs(x))) for x in (xs if isinstance(xs, (list, tuple)) else [xs]))
    for g, w in zip(got, want):
        assert g.data.shape == w.data.shape
        assert np.max(np.abs(g.data - w.data)) <= tol * scale


def face_nodal(dim, d):
    return [1 if k == d else 0 for k in range(dim)]


@pytest.mark.parametrize("dim,n,visc", [(2, [32, 24], 1), (3, [16, 16, 8], -1), (3, [16, 8, 16], 2)])
@pytest.mark.parametrize("nboxes", [1, 2])
def test_stag_mg_solve_fab(cuda, dim, n, visc, nboxes):
    pb = P.problem(dim, n, visc, dx=1.0, seed=3)
    rhs, _ = P.random_stokes(dim, n, seed=4)
    rng = np.random.default_rng(5)
    phi0 = [rng.standard_normal(pb.nc) for _ in range(dim)]
    theta = 0.7
    ref = O.stag_mg_solver(pb, O.default_params(), theta, rhs, phi0)
    ne = 1 if dim == 2 else 3
    ed_nodal = [[1, 1]] if dim == 2 else [[1, 1, 0], [1, 0, 1], [0, 1, 1]]
    alpha = [mf(pb.alpha_fc[c], dim, n, face_nodal(dim, c), 0, nboxes) for c in range(dim)]
    beta = mf(pb.beta, dim, n, [0] * dim, 1, nboxes)
    beta_ed = [mf(pb.beta_ed[e], dim, n, ed_nodal[e], 0, nboxes) for e in range(ne)]
    gamma = mf(pb.gamma, dim, n, [0] * dim, 1, nboxes)
    phi = [mf(phi0[c], dim, n, face_nodal(dim, c), 1, nboxes) for c in range(dim)]
    rhs_f = [mf(rhs[c], dim, n, face_nodal(dim, c), 0, nboxes) for c in range(dim)]
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params()) as s:
        s.stag_mg_solver_fab(alpha, beta, beta_ed, gamma, theta, phi, rhs_f)
    for c in range(dim):
        assert_mf(phi[c], ref[c], dim, n, face_nodal(dim, c), 1, nboxes, 1e-12)


def test_stag_mg_solve_fab_needs_ghosts(cuda):
    dim, n = 2, [16, 16]
    pb = P.problem(dim, n, 1, seed=3)
    rhs, _ = P.random_stokes(dim, n, seed=4)
    fab = lambda x, nd, ng: mf(x, dim, n, nd, ng, 1)
    with L.StokesSolver(dim, n, 1.0, 1) as s:
        with pytest.raises(L.FhdError) as e:
            s.stag_mg_solver_fab([fab(pb.alpha_fc[c], face_nodal(dim, c), 0) for c in range(dim)],
                                 fab(pb.beta, [0, 0], 0), [fab(pb.beta_ed[0], [1, 1], 0)], fab(pb.gamma, [0, 0], 0),
                                 1.0, [fab(np.zeros(pb.nc), face_nodal(dim, c), 0) for c in range(dim)],
                                 [fab(rhs[c], face_nodal(dim, c), 0) for c in range(dim)])
        assert e.value.status == -2  # FHD_ERR_BAD_GHOSTS


def _mix_case(dim, n, ns, traced):
    mp = mix(ns)
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = trace_state(dim, n, ns) if traced else state(dim, n, ns, amp=1e-2)
    lsp = L.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    return mp, sp, rho, lmix(ns), lsp


@pytest.mark.parametrize("dim,n,ns", [(2, [16, 12], 2), (2, [16, 16], 3), (3, [8, 8, 8], 4), (3, [8, 12, 8], 5)])
@pytest.mark.parametrize("traced", [False, True])
def test_sqrtLonsager_fc(cuda, dim, n, ns, traced):
    import torch
    mp, sp, rho, lm, lsp = _mix_case(dim, n, ns, traced)
    ref = O.sqrtLonsager_fc(dim, n, sp, mp, rho)
    nc = P.nc_of(dim, n)
    with L.StokesSolver(dim, n, 1.0, 1) as s:
        out = [torch.zeros(nc, dtype=torch.float64, device=cuda) for _ in range(dim * ns * ns)]
        r = dev(rho, cuda)
        torch.cuda.synchronize()  # the context launches on its own stream
        s.compute_sqrtLonsager_fc(lm, lsp, r, out)
    assert P.rel_inf(host(out), ref) < 1e-12


@pytest.mark.parametrize("nboxes", [1, 2])
@pytest.mark.parametrize("dim,n,ns", [(2, [16, 12], 3), (3, [8, 8, 8], 4)])
def test_sqrtLonsager_fc_fab(cuda, dim, n, ns, nboxes):
    mp, sp, rho, lm, lsp = _mix_case(dim, n, ns, True)
    ref = O.sqrtLonsager_fc(dim, n, sp, mp, rho)
    nc = P.nc_of(dim, n)
    rho_f = mf(rho, dim, n, [0] * dim, 1, nboxes)
    rt_f = mf(sum(rho), dim, n, [0] * dim, 1, nboxes)
    L_f = [mf([np.zeros(nc)] * (ns * ns), dim, n, face_nodal(dim, d), 0, nboxes) for d in range(dim)]
    with L.StokesSolver(dim, n, 1.0, 1) as s:
        s.compute_sqrtLonsager_fc_fab(lm, lsp, rho_f, rt_f, L_f)
    for d in range(dim):
        assert_mf(L_f[d], ref[d * ns * ns:(d + 1) * ns * ns], dim, n, face_nodal(dim, d), 0, nboxes, 1e-12)


@pytest.mark.parametrize("dim,n,ns", [(2, [16, 12], 2), (3, [8, 8, 8], 4), (3, [8, 12, 8], 5)])
@pytest.mark.parametrize("increment", [False, True])
def test_stochastic_mass_fluxdiv(cuda, dim, n, ns, increment):
    import torch
    mp, sp, rho, lm, lsp = _mix_case(dim, n, ns, True)
    nc = P.nc_of(dim, n)
    sqL = O.sqrtLonsager_fc(dim, n, sp, mp, rho)
    W = mass_fields(dim, n, ns, n_rngs=2)
    rng = np.random.default_rng(9)
    div0 = [rng.standard_normal(nc) for _ in range(ns)]
    ref_div, ref_flux = O.stochastic_mass_fluxdiv(dim, n, 1.0, sp, mp, sqL, 0.05, [0.7, -0.3], W,
                                                  increment=increment, div0=div0, want_flux=True)
    # the corrected fluxes sum to zero over the species
    for d in range(dim):
        assert np.max(np.abs(sum(ref_flux[d * ns:(d + 1) * ns]))) <= 1e-13 * np.max(np.abs(ref_flux[d * ns]))
    with L.StokesSolver(dim, n, 1.0, 1) as s:
        div = dev(div0, cuda)
        flux = [torch.zeros(nc, dtype=torch.float64, device=cuda) for _ in range(dim * ns)]
        args = dev(sqL, cuda), dev(W, cuda)
        torch.cuda.synchronize()  # the context launches on its own stream
        s.stochastic_mass_fluxdiv(lm, lsp, args[0], 0.05, [0.7, -0.3], args[1], div, flux, increment=increment)
        out_div, out_flux = host(div), host(flux)
        # without the flux output the divergence is the same
        div2 = dev(div0, cuda)
        torch.cuda.synchronize()
        s.stochastic_mass_fluxdiv(lm, lsp, args[0], 0.05, [0.7, -0.3], args[1], div2, None, increment=increment)
        out_div2 = host(div2)
    assert P.rel_inf(out_div, ref_div) < 1e-12
    assert P.rel_inf(out_flux, ref_flux) < 1e-12
    assert P.rel_inf(out_div2, ref_div) < 1e-12


@pytest.mark.parametrize("nboxes", [1, 2])
def test_stochastic_mass_fluxdiv_fab(cuda, nboxes):
    dim, n, ns = 3, [8, 8, 8], 4
    mp, sp, rho, lm, lsp = _mix_case(dim, n, ns, True)
    nc = P.nc_of(dim, n)
    sqL = O.sqrtLonsager_fc(dim, n, sp, mp, rho)
    W = mass_fields(dim, n, ns, n_rngs=2)
    rng = np.random.default_rng(9)
    div0 = [rng.standard_normal(nc) for _ in range(ns)]
    ref_div, ref_flux = O.stochastic_mass_fluxdiv(dim, n, 1.0, sp, mp, sqL, 0.05, [0.7, -0.3], W, increment=True,
                                                  div0=div0, want_flux=True)
    L_f = [mf(sqL[d * ns * ns:(d + 1) * ns * ns], dim, n, face_nodal(dim, d), 0, nboxes) for d in range(dim)]
    W_f = [mf(W[q * ns:(q + 1) * ns], dim, n, face_nodal(dim, q % dim), 0, nboxes) for q in range(2 * dim)]
    div_f = mf(div0, dim, n, [0] * dim, 1, nboxes)
    flux_f = [mf([np.zeros(nc)] * ns, dim, n, face_nodal(dim, d), 0, nboxes) for d in range(dim)]
    rho_f = mf(rho, dim, n, [0] * dim, 1, nboxes)
    with L.StokesSolver(dim, n, 1.0, 1) as s:
        s.stochastic_mass_fluxdiv_fab(lm, lsp, rho_f, None, L_f, div_f, flux_f, 0.05, [0.7, -0.3], W_f,
                                      increment=True)
    assert_mf(div_f, ref_div, dim, n, [0] * dim, 1, nboxes, 1e-12)
    for d in range(dim):
        assert_mf(flux_f[d], ref_flux[d * ns:(d + 1) * ns], dim, n, face_nodal(dim, d), 0, nboxes, 1e-12)
