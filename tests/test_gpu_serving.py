"""Device random numbers and the serving layer on the GPU: the generator's
statistics and determinism, results of served requests that do not depend
on what runs beside them, and a served request that equals the same steps
through the public per-call API."""
import math

import numpy as np
import pytest

import lowmachfhd_b200 as L

pytestmark = pytest.mark.gpu

GB = 1 << 30


def test_fill_normal(cuda):
    import torch
    n = 2_000_001
    x = torch.empty(n, dtype=torch.float64, device=cuda)
    L.fill_normal(x, seed=123, field=4, stream_a=9)
    torch.cuda.synchronize()
    assert abs(float(x.mean())) < 5e-3
    assert abs(float(x.var()) - 1.0) < 5e-3
    assert abs(float((x[1:] * x[:-1]).mean())) < 5e-3
    y = torch.empty_like(x)
    L.fill_normal(y, seed=123, field=4, stream_a=9)
    z = torch.empty_like(x)
    L.fill_normal(z, seed=123, field=5, stream_a=9)
    torch.cuda.synchronize()
    assert torch.equal(x, y)
    assert not torch.equal(x, z)
    # the first pair is the Box-Muller transform of the block at counter
    # (0, field, stream_a, stream_b)
    r = L.philox4x32_10([0, 4, 9, 0], [123, 0])
    a, b = (r[0] << 32) | r[1], (r[2] << 32) | r[3]
    u1, u2 = ((a >> 11) + 1) * 2.0 ** -53, (b >> 11) * 2.0 ** -53
    rad = math.sqrt(-2.0 * math.log(u1))
    assert abs(float(x[0]) - rad * math.cos(2 * math.pi * u2)) < 1e-13
    assert abs(float(x[1]) - rad * math.sin(2 * math.pi * u2)) < 1e-13


def _mix(ns, seed=0):
    rng = np.random.default_rng(seed)
    D = list(rng.uniform(0.5, 2.0, ns * (ns - 1) // 2) * 1e-2)
    return L.mixture_params([1.0, 2.0, 3.0, 4.0][:ns], D, rhobar=[1.0] * ns, variance_coef_mass=1.0)


def _requests():
    P = L.default_params
    R = L.make_request
    OD, IN = L.FHD_REQ_OVERDAMPED, L.FHD_REQ_INERTIAL
    return [
        R(kind=OD, dim=2, n_cells=[64, 64], steps=3, seed=1, dt=0.1, params=P(gmres_rel_tol=1e-9)),
        R(kind=OD, dim=2, n_cells=[96, 64], steps=2, seed=2, dt=0.1, eta=2.0, params=P(gmres_rel_tol=1e-9),
          precision=L.FHD_PREC_FP64),
        R(kind=IN, dim=3, n_cells=[32, 32, 32], steps=2, seed=3, dt=0.05, kT=1e-3, params=P(gmres_rel_tol=1e-9)),
        R(kind=OD, dim=3, n_cells=[32, 32, 16], steps=2, seed=4, dt=0.5, dx=10.0, kT=1e-4, nspecies=3, mix=_mix(3),
          params=P(gmres_rel_tol=1e-9)),
        R(kind=IN, dim=2, n_cells=[64, 64], steps=3, seed=5, dt=0.1, kT=1e-3, cell_depth=100.0, nspecies=2,
          mix=_mix(2, 1), params=P(gmres_rel_tol=1e-9), precision=L.FHD_PREC_FP64),
        R(kind=IN, dim=3, n_cells=[48, 32, 32], steps=2, seed=6, dt=0.05, kT=1e-3, visc_type=-1,
          params=P(gmres_rel_tol=1e-9)),
    ]


def _nc(r):
    return int(np.prod(list(r.n_cells)[: r.dim]))


def _serve(reqs, slots):
    outs = [(np.zeros(r.dim * _nc(r)), np.zeros(r.nspecies * _nc(r))) for r in reqs]
    with L.Server(slots, 16 * GB) as srv:
        ids = [srv.submit(r, u, rho) for r, (u, rho) in zip(reqs, outs)]
        res = [srv.wait(i) for i in ids]
    return res, outs


def test_served_results_do_not_depend_on_the_mix(cuda):
    reqs = _requests()
    alone = []
    for r in reqs:
        res, out = _serve([r], 1)
        alone.append((res[0], out[0]))
    mixed_res, mixed_out = _serve(reqs, 4)
    for (ra, (ua, rhoa)), rm, (um, rhom) in zip(alone, mixed_res, mixed_out):
        assert ra["status"] in (0, 3) and rm["status"] in (0, 3)
        assert ra["gmres_iters"] == rm["gmres_iters"] > 0
        assert ra["u_sumsq"] == rm["u_sumsq"] > 0
        assert np.array_equal(ua, um)
        assert np.array_equal(rhoa, rhom)
    # the requests overlapped on the device
    starts = sorted(r["t_start"] for r in mixed_res)
    ends = sorted(r["t_end"] for r in mixed_res)
    assert starts[1] < ends[0]


def test_served_request_equals_direct_steps(cuda):
    import torch
    dim, n, steps, seed = 2, [64, 48], 3, 17
    nc = n[0] * n[1]
    req = L.make_request(kind=L.FHD_REQ_OVERDAMPED, dim=dim, n_cells=n, steps=steps, seed=seed, dt=0.1, eta=1.5,
                         kT=0.5, params=L.default_params(gmres_rel_tol=1e-9), precision=L.FHD_PREC_FP64)
    (res,), ((u_served, _),) = _serve([req], 1)
    f64 = dict(dtype=torch.float64, device=cuda)
    u = [torch.zeros(nc, **f64) for _ in range(dim)]
    rho = [torch.ones(nc, **f64)]
    pi = torch.zeros(nc, **f64)
    eta = torch.full((nc,), 1.5, **f64)
    eta_ed = [torch.full((nc,), 1.5, **f64)]
    kappa = torch.zeros(nc, **f64)
    T = torch.ones(nc, **f64)
    T_ed = [torch.ones(nc, **f64)]
    sp = L.StochParams(k_B=0.5, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    with L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(gmres_rel_tol=1e-9)) as s:
        for k in range(1, steps + 1):
            # the server's field numbering: cell stages, then edge stages
            W_cc = [torch.empty(nc, **f64) for _ in range(2 * dim)]
            for i, w in enumerate(W_cc):
                L.fill_normal(w, seed, field=i, stream_a=k, stream_b=0x5EED, scale=math.sqrt(2.0))
            W_ed = []
            for i in range(2):
                w = torch.empty(nc, **f64)
                L.fill_normal(w, seed, field=2 * dim + i, stream_a=k, stream_b=0x5EED)
                W_ed += [w, w]
            torch.cuda.synchronize()
            s.advance_timestep_overdamped(sp, None, 0.1, u, rho, pi, eta, eta_ed, kappa, T, T_ed, W_cc, W_ed)
    direct = torch.cat(u).cpu().numpy()
    assert np.array_equal(direct, u_served)
