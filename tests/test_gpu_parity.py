"""Parity of the sm_100a library (called through its C ABI) with the CPU
oracle on identical seeded inputs.  FP64 tolerances: the stencils are
evaluated in the same order as the oracle (no FMA contraction), so they
agree to roundoff; reductions are summed in a different order, which GMRES
propagates to ~1e-13.  The bar is 1e-10 relative in every component."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P

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


def zeros(nc, k, device):
    import torch
    return [torch.zeros(nc, dtype=torch.float64, device=device) for _ in range(k)]


SHAPES = [(2, [16, 16]), (2, [32, 16]), (3, [8, 8, 8]), (3, [16, 8, 8])]
VISCS = [1, -1, 2, -2, 3, -3]


@pytest.mark.parametrize("dim,n", SHAPES)
@pytest.mark.parametrize("visc", VISCS)
def test_apply_matrix(cuda, dim, n, visc):
    pb = P.problem(dim, n, visc, dx=0.5, seed=visc + 7)
    u, p = P.random_stokes(dim, n, seed=2)
    theta = 3.0
    ref_u, ref_p = O.apply_matrix(pb, theta, u, p)
    with L.StokesSolver(dim, n, 0.5, visc) as s:
        b_u, b_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_matrix(b_u, b_p, dev(u, cuda), dev(p, cuda), dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                       dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
        assert s.kernel_launches >= 1
    assert P.rel_inf(host(b_u), ref_u) < 1e-13
    assert P.rel_inf([host(b_p)], [ref_p]) < 1e-13


@pytest.mark.parametrize("dim,n", SHAPES)
@pytest.mark.parametrize("visc", VISCS)
def test_stag_mg_one_vcycle(cuda, dim, n, visc):
    pb = P.problem(dim, n, visc, dx=1.0, seed=3)
    rhs, _ = P.random_stokes(dim, n, seed=4)
    params = O.default_params()
    theta = 0.7
    ref = O.stag_mg_solver(pb, params, theta, rhs)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params()) as s:
        phi = zeros(pb.nc, dim, cuda)
        s.stag_mg_solver(dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda),
                         theta, phi, dev(rhs, cuda))
    assert P.rel_inf(host(phi), ref) < 1e-12


# grids whose finest levels span several x-y tiles and z runs of the fused
# red-black smoothers (64x16 tiles; 96 -> 48-wide, 40 -> 10-high tiles), with
# uncoupled and coupled viscous operators, through one V-cycle and through
# the preconditioner (which adds the pressure multigrid)
TILED = [(1, [128, 32, 64]), (-1, [96, 40, 24]), (2, [64, 48, 32]), (-3, [96, 40, 24]),
         # above 96^3 cells the colour sweeps update two z-planes per thread
         (1, [96, 96, 96]), (-1, [128, 96, 80])]


@pytest.mark.parametrize("visc,n", TILED)
def test_stag_mg_tiled(cuda, visc, n):
    dim = 3
    pb = P.problem(dim, n, visc, dx=1.0, seed=8)
    rhs, _ = P.random_stokes(dim, n, seed=9)
    ref = O.stag_mg_solver(pb, O.default_params(), 0.7, rhs)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params()) as s:
        phi = zeros(pb.nc, dim, cuda)
        s.stag_mg_solver(dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda),
                         0.7, phi, dev(rhs, cuda))
    assert P.rel_inf(host(phi), ref) < 1e-12


@pytest.mark.parametrize("visc,n", TILED[:2] + TILED[4:5])
def test_apply_precon_tiled(cuda, visc, n):
    dim = 3
    pb = P.problem(dim, n, visc, dx=1.0, seed=10)
    b_u, b_p = P.random_stokes(dim, n, seed=11, zero_mean_p=False)
    ref_u, ref_p = O.apply_precon(pb, O.default_params(), 1.5, b_u, b_p)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params()) as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_precon(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                       dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), 1.5)
    assert P.rel_inf(host(x_u), ref_u) < 1e-11
    assert P.rel_inf([host(x_p)], [ref_p]) < 1e-11


@pytest.mark.parametrize("case", ["vcycles3", "jacobi", "odd24", "odd12x20", "minwidth4"])
def test_stag_mg_options(cuda, case):
    dim, n, kw, visc = 2, [32, 32], {}, -1
    if case == "vcycles3":
        kw = dict(stag_mg_max_vcycles=3, stag_mg_rel_tol=1e-14)
    elif case == "jacobi":
        kw = dict(stag_mg_smoother=0, stag_mg_omega=0.6)
    elif case == "odd24":
        n = [24, 24]
    elif case == "odd12x20":
        dim, n = 3, [12, 20, 8]
    elif case == "minwidth4":
        dim, n, kw = 3, [16, 16, 16], dict(stag_mg_minwidth=4)
    pb = P.problem(dim, n, visc, dx=1.0, seed=3)
    rhs, _ = P.random_stokes(dim, n, seed=4)
    ref = O.stag_mg_solver(pb, O.default_params(**kw), 1.0, rhs)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(**kw)) as s:
        phi = zeros(pb.nc, dim, cuda)
        s.stag_mg_solver(dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda),
                         1.0, phi, dev(rhs, cuda))
    assert P.rel_inf(host(phi), ref) < 1e-12


@pytest.mark.parametrize("dim,n", [(2, [32, 32]), (3, [16, 16, 16])])
@pytest.mark.parametrize("precon", [1, -1, 2, -2, 3, -3, 4, -4, 5])
@pytest.mark.parametrize("theta", [0.0, 2.0])
def test_apply_precon(cuda, dim, n, precon, theta):
    visc = -2 if dim == 3 else 3
    pb = P.problem(dim, n, visc, dx=1.0, seed=5)
    b_u, b_p = P.random_stokes(dim, n, seed=6, zero_mean_p=False)
    params = O.default_params(precon_type=precon)
    ref_u, ref_p = O.apply_precon(pb, params, theta, b_u, b_p)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(precon_type=precon)) as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_precon(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                       dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
    assert P.rel_inf(host(x_u), ref_u) < 1e-11
    assert P.rel_inf([host(x_p)], [ref_p]) < 1e-11


@pytest.mark.parametrize("dim,n,visc", [(2, [32, 32], -1), (3, [16, 16, 16], -2), (3, [16, 8, 16], 1),
                                        (2, [32, 16], 2)])
@pytest.mark.parametrize("precon", [1, 2, -2, 3, 4, 5])
@pytest.mark.parametrize("theta", [0.0, 2.0])
def test_apply_precon_bfbt(cuda, dim, n, visc, precon, theta):
    """visc_schur_approx = 1: the BFBt Schur complement
    (visc_schur_complement, apply_precon.f90:538-685) against the oracle"""
    pb = P.problem(dim, n, visc, dx=1.0, seed=15)
    b_u, b_p = P.random_stokes(dim, n, seed=16, zero_mean_p=False)
    ref_u, ref_p = O.apply_precon(pb, O.default_params(precon_type=precon, visc_schur_approx=1), theta, b_u, b_p)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(precon_type=precon, visc_schur_approx=1)) as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_precon(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                       dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
    assert P.rel_inf(host(x_u), ref_u) < 1e-11
    assert P.rel_inf([host(x_p)], [ref_p]) < 1e-11


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gmres_bfbt(cuda, precision):
    """GMRES with the BFBt preconditioner on a variable-viscosity 3D problem:
    FP64 takes the oracle's iterations and matches it to 1e-10; the mixed
    preconditioner reaches the same 1e-9 residual"""
    dim, n, visc = 3, [16, 16, 16], -1
    pb = P.problem(dim, n, visc, dx=1.0, seed=17)
    b_u, b_p = P.random_stokes(dim, n, seed=18)
    theta = 2.0
    rc, ref_u, ref_p, _, st_ref = O.gmres(pb, O.default_params(gmres_rel_tol=1e-9, visc_schur_approx=1), theta,
                                          b_u, b_p)
    assert rc == 0
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(gmres_rel_tol=1e-9, visc_schur_approx=1),
                        precision=precision) as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        status, _, st = s.gmres(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                                dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
    assert status == 0
    if precision == "fp64":
        assert st["total_iters"] == st_ref.total_iters
        assert P.rel_inf(host(x_u) + [host(x_p)], ref_u + [ref_p]) < 1e-10
    else:
        assert st["norm_resid"] <= 1e-9 * min(st["norm_pre_b"], st["norm_init_resid"])
        assert abs(st["total_iters"] - st_ref.total_iters) <= 2
        assert P.rel_inf(host(x_u) + [host(x_p)], ref_u + [ref_p]) < 1e-6


def _config1():
    """2D periodic 64^2, dx=1, rho=1, eta=1, kT=1, dt=0.1, overdamped
    (theta=0), visc_type 1, stochastic momentum forcing from seed-1 fields."""
    dim, n = 2, [64, 64]
    nc = P.nc_of(dim, n)
    ones = np.ones(nc)
    pb = O.Problem(dim, n, 1.0, 1, [ones, ones], ones, [ones], np.zeros(nc))
    sp = O.StochParams(k_B=1.0, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=1)
    f = O.stochastic_m_fluxdiv(dim, n, 1.0, sp, ones, [ones], ones, [ones], 0.1, [1.0], W_cc, W_ed)
    return pb, f, np.zeros(nc)


def test_gmres_config1(cuda):
    pb, f, bp = _config1()
    params = O.default_params(gmres_rel_tol=1e-9)
    rc, ref_u, ref_p, npr_ref, st_ref = O.gmres(pb, params, 0.0, f, bp)
    assert rc == 0
    with L.StokesSolver(2, pb.n, 1.0, 1, params=L.default_params(gmres_rel_tol=1e-9)) as s:
        x_u, x_p = zeros(pb.nc, 2, cuda), zeros(pb.nc, 1, cuda)[0]
        status, npr, st = s.gmres(dev(f, cuda), dev(bp, cuda), x_u, x_p, dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                                  dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), 0.0)
    assert status == 0
    assert st["total_iters"] == st_ref.total_iters
    for c in range(2):
        assert P.rel_inf([host(x_u[c])], [ref_u[c]]) < 1e-10
    assert P.rel_inf([host(x_p)], [ref_p]) < 1e-10
    assert abs(npr - npr_ref) <= 1e-12 * npr_ref


@pytest.mark.parametrize("dim,n,visc,theta", [(2, [32, 32], 1, 0.0), (3, [16, 16, 16], -1, 20.0),
                                                (3, [16, 8, 16], 2, 20.0)])
@pytest.mark.parametrize("sf", [2.5, 1e-3])
def test_gmres_scale_factor(cuda, dim, n, visc, theta, sf):
    """scale_factor != 1 (gmres.f90:118-135, 442-459): the solve for
    scale*x_p with scaled theta_alpha, rhs and viscosities, and a nonzero
    initial pressure guess, matches the oracle; the caller's operands are
    left as they were"""
    pb = P.problem(dim, n, visc, dx=1.0, seed=21)
    b_u, b_p = P.random_stokes(dim, n, seed=22)
    rng = np.random.default_rng(23)
    xp0 = rng.standard_normal(pb.nc)
    xp0 -= xp0.mean()
    params = O.default_params(gmres_rel_tol=1e-9, scale_factor=sf)
    rc, ref_u, ref_p, npr_ref, st_ref = O.gmres(pb, params, theta, b_u, b_p, x_p0=xp0)
    assert rc >= 0
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(gmres_rel_tol=1e-9, scale_factor=sf)) as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), dev(xp0, cuda)
        bu, beta = dev(b_u, cuda), dev(pb.beta, cuda)
        status, npr, st = s.gmres(bu, dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda), beta,
                                  dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
        assert np.array_equal(host(bu[0]), b_u[0]) and np.array_equal(host(beta), pb.beta)
    assert status == rc
    assert st["total_iters"] == st_ref.total_iters
    for c in range(dim):
        assert P.rel_inf([host(x_u[c])], [ref_u[c]]) < 1e-10
    assert P.rel_inf([host(x_p)], [ref_p]) < 1e-10


@pytest.mark.parametrize("visc", [1, -1, -2, 3])
def test_gmres_3d_inertial(cuda, visc):
    dim, n = 3, [16, 16, 16]
    pb = P.problem(dim, n, visc, dx=1.0, seed=11)
    b_u, b_p = P.random_stokes(dim, n, seed=12)
    theta = 1.0 / 0.05
    params = O.default_params(gmres_rel_tol=1e-9)
    rc, ref_u, ref_p, _, st_ref = O.gmres(pb, params, theta, b_u, b_p)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(gmres_rel_tol=1e-9)) as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        status, _, st = s.gmres(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                                dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
    assert status == rc
    assert st["total_iters"] == st_ref.total_iters
    for c in range(dim):
        assert P.rel_inf([host(x_u[c])], [ref_u[c]]) < 1e-10
    assert P.rel_inf([host(x_p)], [ref_p]) < 1e-10


@pytest.mark.parametrize("dim,n", [(2, [16, 24]), (3, [8, 12, 8])])
@pytest.mark.parametrize("increment", [False, True])
def test_stochastic_m_fluxdiv(cuda, dim, n, increment):
    nc = P.nc_of(dim, n)
    rng = np.random.default_rng(8)
    eta = 1 + rng.random(nc)
    T = 1 + rng.random(nc)
    eta_ed = O.average_cc_to_edge(dim, n, eta)
    T_ed = O.average_cc_to_edge(dim, n, T)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=5, n_rngs=2, symmetric=False)
    force0 = [rng.standard_normal(nc) for _ in range(dim)]
    sp = O.StochParams(k_B=2.0, variance_coef_mom=1.0, dV=0.125, stoch_stress_form=0, filtering_width=0)
    ref = O.stochastic_m_fluxdiv(dim, n, 0.5, sp, eta, eta_ed, T, T_ed, 0.1, [0.5, -0.25], W_cc, W_ed,
                                 force=force0, increment=increment)
    with L.StokesSolver(dim, n, 0.5, 1) as s:
        spd = L.StochParams(k_B=2.0, variance_coef_mom=1.0, dV=0.125, stoch_stress_form=0, filtering_width=0)
        f = dev(force0, cuda)
        s.stochastic_m_fluxdiv(spd, f, increment, dev(eta, cuda), dev(eta_ed, cuda), dev(T, cuda), dev(T_ed, cuda),
                               0.1, [0.5, -0.25], dev(W_cc, cuda), dev(W_ed, cuda))
    assert P.rel_inf(host(f), ref) < 1e-13


def test_inertial_step(cuda):
    dim, n = 3, [16, 16, 16]
    nc = P.nc_of(dim, n)
    rng = np.random.default_rng(0)
    umac = [0.05 * rng.standard_normal(nc) for _ in range(dim)]
    rho = 1.0 + 0.01 * rng.standard_normal(nc)
    pi = 0.01 * rng.standard_normal(nc)
    eta = np.ones(nc)
    eta_ed = O.average_cc_to_edge(dim, n, eta)
    T = np.ones(nc)
    kappa = np.zeros(nc)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=9)
    sp = O.StochParams(k_B=1e-3, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    params = O.default_params(gmres_rel_tol=1e-9)
    rc, ru, rr, rp, rst = O.advance_inertial(dim, n, 1.0, 1, params, sp, 0.05, umac, rho, pi, eta, eta_ed, kappa,
                                             T, eta_ed, W_cc, W_ed)
    assert rc == 0
    with L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(gmres_rel_tol=1e-9)) as s:
        spd = L.StochParams(k_B=1e-3, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
        u, r_, p_ = dev(umac, cuda), dev(rho, cuda), dev(pi, cuda)
        status, st = s.advance_timestep_inertial(spd, 0.05, u, r_, p_, dev(eta, cuda), dev(eta_ed, cuda),
                                                 dev(kappa, cuda), dev(T, cuda), dev(eta_ed, cuda), dev(W_cc, cuda),
                                                 dev(W_ed, cuda))
    assert status == 0
    assert [x["total_iters"] for x in st] == [rst[0].total_iters, rst[1].total_iters]
    for c in range(dim):
        assert P.rel_inf([host(u[c])], [ru[c]]) < 1e-10
    assert P.rel_inf([host(r_)], [rr]) < 1e-12
    assert P.rel_inf([host(p_)], [rp]) < 1e-10


@pytest.mark.parametrize("nboxes", [1, 2])
def test_gmres_fab_boundary(cuda, nboxes):
    """The drop-in host path: BoxLib fabs with ghost cells and duplicated
    periodic faces in, solution written back over valid and ghost cells."""
    pb, f, bp = _config1()
    dim, n = 2, pb.n
    params = O.default_params(gmres_rel_tol=1e-9)
    rc, ref_u, ref_p, _, _ = O.gmres(pb, params, 0.0, f, bp)

    def mf(x, nodal, ng):
        if nboxes == 1:
            return L.fab_from_canonical(x, dim, n, nodal, ng)
        half = n[0] // 2
        return [L.fab_from_canonical(x, dim, n, nodal, ng, lo=[0, 0], hi=[half - 1, n[1] - 1]),
                L.fab_from_canonical(x, dim, n, nodal, ng, lo=[half, 0], hi=[n[0] - 1, n[1] - 1])]

    nodal = [[1, 0], [0, 1]]
    b_u = [mf(f[c], nodal[c], 0) for c in range(dim)]
    b_p = mf(bp, [0, 0], 0)
    x_u = [mf(np.zeros(pb.nc), nodal[c], 1) for c in range(dim)]
    x_p = mf(np.zeros(pb.nc), [0, 0], 1)
    alpha = [mf(pb.alpha_fc[c], nodal[c], 0) for c in range(dim)]
    beta = mf(pb.beta, [0, 0], 1)
    beta_ed = [mf(pb.beta_ed[0], [1, 1], 0)]
    gamma = mf(pb.gamma, [0, 0], 1)
    with L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(gmres_rel_tol=1e-9)) as s:
        status, npr, st = s.gmres_fab(b_u, b_p, x_u, x_p, alpha, beta, beta_ed, gamma, 0.0)
    assert status == 0
    for c in range(dim):
        fa = x_u[c] if nboxes == 1 else x_u[c][0]
        full = L.fab_from_canonical(ref_u[c], dim, n, nodal[c], 1,
                                    lo=fa.lo[:2], hi=fa.hi[:2])
        assert np.max(np.abs(fa.data - full.data)) < 1e-10 * np.max(np.abs(ref_u[c]))
    fa = x_p if nboxes == 1 else x_p[1]
    full = L.fab_from_canonical(ref_p, dim, n, [0, 0], 1, lo=fa.lo[:2], hi=fa.hi[:2])
    assert np.max(np.abs(fa.data - full.data)) < 1e-10 * np.max(np.abs(ref_p))


def test_bad_ghosts_rejected(cuda):
    pb, f, bp = _config1()
    dim, n = 2, pb.n
    nodal = [[1, 0], [0, 1]]
    fab = lambda x, nd, ng: L.fab_from_canonical(x, dim, n, nd, ng)
    with L.StokesSolver(dim, n, 1.0, 1) as s:
        with pytest.raises(L.FhdError) as e:
            s.gmres_fab([fab(f[c], nodal[c], 0) for c in range(dim)], fab(bp, [0, 0], 0),
                        [fab(np.zeros(pb.nc), nodal[c], 0) for c in range(dim)], fab(np.zeros(pb.nc), [0, 0], 0),
                        [fab(pb.alpha_fc[c], nodal[c], 0) for c in range(dim)], fab(pb.beta, [0, 0], 0),
                        [fab(pb.beta_ed[0], [1, 1], 0)], fab(pb.gamma, [0, 0], 0), 0.0)
        assert e.value.status == L._capi.FHD_ERR_BAD_GHOSTS


def test_mixed_precision_solve(cuda):
    """FP32 multigrid preconditioner inside FP64 GMRES reaches the same
    1e-8 relative residual; the solution's error against the FP64 oracle is
    reported and bounded by the solver tolerance."""
    dim, n = 3, [32, 32, 32]
    pb = P.problem(dim, n, -1, dx=1.0, seed=13)
    b_u, b_p = P.random_stokes(dim, n, seed=14)
    theta = 20.0
    rc, ref_u, ref_p, _, st_ref = O.gmres(pb, O.default_params(gmres_rel_tol=1e-8), theta, b_u, b_p)
    with L.StokesSolver(dim, n, 1.0, -1, params=L.default_params(gmres_rel_tol=1e-8), precision="mixed") as s:
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        status, _, st = s.gmres(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda), dev(pb.beta, cuda),
                                dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
    assert status == 0
    assert st["norm_resid"] <= 1e-8 * min(st["norm_pre_b"], st["norm_init_resid"])
    assert st["total_iters"] <= st_ref.total_iters + 3
    assert P.rel_inf(host(x_u), ref_u) < 1e-6
