"""Parity of the sm_100a multispecies mass fluxes and step with the oracle."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_oracle_multispecies import mass_fields, mix, state, trace_state

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


# FP32 error budget of the mixed-precision mass fluxes (relative to the
# largest divergence):
#  * diffusive part: the molar concentrations x are rounded to FP32 (eps
#    6e-8 relative to x) and differenced between neighbouring cells, which
#    differ by about amp * x; the gradient then carries eps / amp relative
#    error: 6e-5 at amp = 1e-3 (measured 1e-5 to 2e-5);
#  * stochastic part: eps times the growth of the 10-step chi iteration and
#    the Cholesky factorisation, a few 1e-7 measured; the full flux is
#    dominated by it, so its error stays below 1e-5.
#  (A subsystem of non-trace species factorises in FP64 even in this mode:
#  its singular Onsager matrix leaves a roundoff pivot whose square root
#  would be sqrt(eps) = 2.4e-4 in FP32.)
MIXED_DIFFUSIVE_TOL = 6e-8 / 1e-3
MIXED_FULL_TOL = 1e-5


@pytest.mark.parametrize("var,tol", [(1.0, MIXED_FULL_TOL), (0.0, MIXED_DIFFUSIVE_TOL)])
def test_mass_fluxdiv_mixed_precision(cuda, var, tol):
    import torch
    dim, n, ns = 3, [16, 16, 16], 4
    mp = mix(ns, var=var)
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-3)
    W = mass_fields(dim, n, ns)
    ref = O.mass_fluxdiv(dim, n, 1.0, sp, mp, rho, 0.05, [1.0], W)
    with L.StokesSolver(dim, n, 1.0, 1, precision="mixed") as s:
        out = [torch.zeros(P.nc_of(dim, n), dtype=torch.float64, device=cuda) for _ in range(ns)]
        args = dev(rho, cuda), dev(W, cuda)
        torch.cuda.synchronize()  # the context launches on its own stream
        s.compute_mass_fluxdiv(lmix(ns, var=var), L.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0,
                                                               stoch_stress_form=1, filtering_width=0),
                               args[0], 0.05, [1.0], args[1], out)
    err = P.rel_inf(host(out), ref)
    assert err < tol, err


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


@pytest.mark.parametrize("dim,n,ns", [(2, [16, 24], 3), (3, [8, 8, 8], 4), (3, [8, 12, 8], 5)])
@pytest.mark.parametrize("avg", [1, 10])
def test_mass_fluxdiv_trace_species(cuda, dim, n, ns, avg):
    """cells with one, two and all-but-one zero species densities: the
    subsystem of non-trace species (compute_chi_sub,
    compute_sqrtLonsager_sub) on the faces and cells that have them"""
    mp = mix(ns)
    mp.avg_type = avg
    sp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = trace_state(dim, n, ns)
    W = mass_fields(dim, n, ns, n_rngs=2)
    ref = O.mass_fluxdiv(dim, n, 1.0, sp, mp, rho, 0.05, [0.7, -0.3], W)
    lm = lmix(ns)
    lm.avg_type = avg
    lsp = L.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    import torch
    for precision, tol in (("fp64", 1e-12), ("mixed", MIXED_FULL_TOL)):
        with L.StokesSolver(dim, n, 1.0, 1, precision=precision) as s:
            out = [torch.zeros(P.nc_of(dim, n), dtype=torch.float64, device=cuda) for _ in range(ns)]
            args = dev(rho, cuda), dev(W, cuda)
            torch.cuda.synchronize()  # the context launches on its own stream
            s.compute_mass_fluxdiv(lm, lsp, args[0], 0.05, [0.7, -0.3], args[1], out)
        assert P.rel_inf(host(out), ref) < tol, precision


def _c3_case(cuda, n, precision, seed=7):
    """the 4-species bench workload (masses 1-4, D_ij ~ U[0.5, 2]*1e-2,
    w = 0.25 + 1e-3 N(0,1), dx = 10, dt = 5, k_B T = 1e-4, GMRES 1e-8) on an
    n^3 grid, with fresh device noise every step"""
    import torch
    nc = n ** 3
    g = torch.Generator().manual_seed(seed)
    f64 = dict(dtype=torch.float64)
    umac = [(1e-3 * torch.randn(nc, generator=g, **f64)).to(cuda) for _ in range(3)]
    w = 0.25 + 1e-3 * torch.randn(4, nc, generator=g, **f64)
    w = w / w.sum(dim=0, keepdim=True)
    rho = [w[i].contiguous().to(cuda) for i in range(4)]
    rng = np.random.default_rng(11)
    D = list(rng.uniform(0.5, 2.0, 6) * 1e-2)
    mp = L.mixture_params([1.0, 2.0, 3.0, 4.0], D, rhobar=[1.0] * 4, variance_coef_mass=1.0)
    sp = L.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1000.0, stoch_stress_form=1, filtering_width=0)
    s = L.StokesSolver(3, [n] * 3, 10.0, 1, params=L.default_params(gmres_rel_tol=1e-8), precision=precision)
    noise = L.StepNoise(3, [n] * 3, 4, seed, cuda, s.stream)
    one = lambda: torch.ones(nc, device=cuda, **f64)
    state = dict(umac=umac, rho=rho, pi=torch.zeros(nc, device=cuda, **f64),
                 F=[torch.zeros(nc, device=cuda, **f64) for _ in range(4)], eta=one(), eta_ed=[one() for _ in range(3)],
                 kappa=torch.zeros(nc, device=cuda, **f64), T=one(), T_ed=[one() for _ in range(3)])
    torch.cuda.synchronize()  # the context launches on its own stream
    noise.draw_mass(0)
    s.compute_mass_fluxdiv(mp, sp, rho, 5.0, [1.0], noise.mass(0), state["F"])
    return s, noise, mp, sp, state


def _c3_step(s, noise, mp, sp, st, k):
    noise.draw(k)
    W_cc, W_ed, W_m = noise.inertial_args(k)
    return s.advance_timestep_inertial_multispecies(sp, mp, 5.0, st["umac"], st["rho"], st["pi"], st["F"], st["eta"],
                                                    st["eta_ed"], st["kappa"], st["T"], st["T_ed"], W_cc, W_ed, W_m)


def test_bench_workload_survives_many_steps(cuda):
    """the mixed-precision 4-species workload at 64^3 for 60 steps with
    fresh noise: every step succeeds, the fields stay finite and every
    density positive"""
    import torch
    s, noise, mp, sp, st = _c3_case(cuda, 64, "mixed")
    with s:
        for k in range(1, 61):
            status, stats = _c3_step(s, noise, mp, sp, st, k)
            assert status == 0, (k, stats)
        torch.cuda.synchronize()
        for a in st["umac"] + st["rho"] + [st["pi"]]:
            assert bool(torch.isfinite(a).all())
        assert min(float(r.min()) for r in st["rho"]) > 0.1
        assert max(float(u.abs().max()) for u in st["umac"]) < 1e-1


def test_step_noise_is_fresh_every_step(cuda):
    """no two steps of StepNoise draw the same fields, and the same seed
    draws the same fields again"""
    import torch
    a = L.StepNoise(3, [16] * 3, 4, 5, cuda)
    b = L.StepNoise(3, [16] * 3, 4, 5, cuda)
    a.draw_mass(0)  # M_0, which the first step's predictor reads
    b.draw_mass(0)
    seen = []
    for k in range(1, 5):
        a.draw(k)
        b.draw(k)
        wc, we, wm = a.inertial_args(k)
        wc2, we2, wm2 = b.inertial_args(k)
        for x, y in zip(wc + we + wm, wc2 + we2 + wm2):
            assert torch.equal(x, y)
        assert we[0] is we[1]
        cur = torch.stack([w.clone() for w in wc + we[::2] + a.mass(k)])
        for old in seen:
            assert float((cur - old).abs().min()) > 0.0
        seen.append(cur)
        # variance 2 on cells, 1 on edges and mass faces
        assert abs(float(wc[0].var()) - 2.0) < 0.2 and abs(float(a.mass(k)[0].var()) - 1.0) < 0.1


def test_multispecies_step_128cube_fp64(cuda):
    """one FP64 4-species inertial step of the bench workload at 128^3
    against the oracle"""
    n = 128
    nc = n ** 3
    s, noise, mp, sp, st = _c3_case(cuda, n, "fp64")
    init = {k: host(v) for k, v in st.items()}
    with s:
        status, stats = _c3_step(s, noise, mp, sp, st, 1)
        assert status == 0
        W_cc, W_ed, W_m = (host(x) for x in noise.inertial_args(1))
        out = {k: host(st[k]) for k in ("umac", "rho", "pi", "F")}
    rng = np.random.default_rng(11)
    D = list(rng.uniform(0.5, 2.0, 6) * 1e-2)
    omp = O.mixture_params([1.0, 2.0, 3.0, 4.0], D, rhobar=[1.0] * 4, variance_coef_mass=1.0)
    osp = O.StochParams(k_B=1e-4, variance_coef_mom=1.0, dV=1000.0, stoch_stress_form=1, filtering_width=0)
    ee = [np.ones(nc)] * 3
    rc, ru, rr, rp, rF, rst = O.advance_inertial_ms(3, [n] * 3, 10.0, 1, O.default_params(gmres_rel_tol=1e-8), osp,
                                                    omp, 5.0, init["umac"], init["rho"], init["pi"], init["F"],
                                                    np.ones(nc), ee, np.zeros(nc), np.ones(nc), ee, W_cc, W_ed, W_m)
    assert rc == 0
    assert [x["total_iters"] for x in stats] == [rst[0].total_iters, rst[1].total_iters]
    for c in range(3):
        assert P.rel_inf([out["umac"][c]], [ru[c]]) < 1e-10
    assert P.rel_inf(out["rho"], rr) < 1e-12
    assert P.rel_inf(out["F"], rF) < 1e-10
    assert P.rel_inf([out["pi"]], [rp]) < 1e-10
