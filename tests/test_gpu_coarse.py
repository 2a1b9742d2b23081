"""The coarse end of both multigrid V-cycles as one single-block kernel
(fhd_ctx_set_coarse) against the per-level launch sequence on the same
inputs.  FP64: bit-identical (the same stencil, smoother, restriction and
prolongation expressions evaluated in the same order).  Mixed precision:
the FP32 levels agree to FP32 roundoff and GMRES takes the same number of
iterations.  Parity with the oracle on hierarchies the coarse kernel takes
over entirely is covered by the small-grid cases of test_gpu_parity.py,
which run with the coarse kernel on (the default)."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_parity import dev, host, zeros

pytestmark = pytest.mark.gpu

# (dim, n, visc, params): even hierarchies down to 2 cells, odd bottoms
# (24 -> 3, 12x20x8 -> 3x5x2), the Jacobi smoother, several V-cycles
CASES = [
    (3, [16, 16, 16], 1, {}),
    (3, [32, 32, 32], -1, {}),
    (3, [64, 32, 32], 1, {}),
    (3, [24, 24, 24], 2, {}),
    (3, [12, 20, 8], -2, {}),
    (3, [16, 16, 16], -3, {}),
    (2, [64, 64], -3, {}),
    (2, [24, 24], 3, dict(stag_mg_smoother=0, stag_mg_omega=0.6)),
    (2, [32, 32], -1, dict(stag_mg_max_vcycles=3, stag_mg_rel_tol=1e-14, mg_max_vcycles=3, mg_rel_tol=1e-14)),
]


def _run(cuda, dim, n, visc, kw, coarse, precision="fp64", seed=21):
    pb = P.problem(dim, n, visc, dx=1.0, seed=seed)
    rhs, _ = P.random_stokes(dim, n, seed=seed + 1)
    b_u, b_p = P.random_stokes(dim, n, seed=seed + 2, zero_mean_p=False)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(**kw), precision=precision) as s:
        s.set_coarse(coarse)
        coef = (dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda))
        phi = zeros(pb.nc, dim, cuda)
        s.stag_mg_solver(*coef, 0.7, phi, dev(rhs, cuda))
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_precon(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, *coef, 1.5)
        launches = s.kernel_launches
    return host(phi), host(x_u) + [host(x_p)], launches


@pytest.mark.parametrize("dim,n,visc,kw", CASES)
def test_coarse_kernel_bitwise_fp64(cuda, dim, n, visc, kw):
    phi1, x1, n1 = _run(cuda, dim, n, visc, kw, 1)
    phi0, x0, n0 = _run(cuda, dim, n, visc, kw, 0)
    for a, b in zip(phi1 + x1, phi0 + x0):
        assert np.array_equal(a, b)
    assert n1 < n0


@pytest.mark.parametrize("dim,n,visc", [(3, [32, 32, 32], 1), (3, [64, 64, 64], -1), (2, [128, 128], 2)])
def test_coarse_kernel_mixed(cuda, dim, n, visc):
    phi1, x1, _ = _run(cuda, dim, n, visc, {}, 1, precision="mixed")
    phi0, x0, _ = _run(cuda, dim, n, visc, {}, 0, precision="mixed")
    assert P.rel_inf(phi1, phi0) < 1e-5
    assert P.rel_inf(x1, x0) < 1e-5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_coarse_kernel_gmres(cuda, precision):
    """GMRES at 1e-8 with the coarse kernel on and off: same iterations,
    solutions agree to the solver tolerance, and both match the oracle."""
    dim, n, visc = 3, [32, 32, 32], -1
    pb = P.problem(dim, n, visc, dx=1.0, seed=31)
    b_u, b_p = P.random_stokes(dim, n, seed=32)
    theta = 20.0
    _, ref_u, ref_p, _, st_ref = O.gmres(pb, O.default_params(gmres_rel_tol=1e-8), theta, b_u, b_p)
    out = {}
    for coarse in (1, 0):
        with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(gmres_rel_tol=1e-8),
                            precision=precision) as s:
            s.set_coarse(coarse)
            x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
            status, _, st = s.gmres(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda),
                                    dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), theta)
            assert status == 0
            out[coarse] = (host(x_u), st["total_iters"])
    assert out[1][1] == out[0][1]
    assert abs(out[1][1] - st_ref.total_iters) <= (0 if precision == "fp64" else 3)
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert P.rel_inf(out[1][0], ref_u) < tol
    assert P.rel_inf(out[1][0], out[0][0]) < tol


def test_unaligned_user_arrays(cuda):
    """Caller arrays one element off a 16-byte boundary: the prolongation's
    pair accesses fall back to scalars (and the fused smoothers to the colour
    sweeps); the result equals the aligned run bit for bit."""
    import torch
    dim, n, visc = 3, [64, 32, 32], 1
    pb = P.problem(dim, n, visc, dx=1.0, seed=41)
    rhs, _ = P.random_stokes(dim, n, seed=42)
    out = []
    for shift in (0, 1):
        with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params()) as s:
            phi = [torch.zeros(pb.nc + shift, dtype=torch.float64, device=cuda)[shift:] for _ in range(dim)]
            r = []
            for a in rhs:
                t = torch.zeros(pb.nc + shift, dtype=torch.float64, device=cuda)[shift:]
                t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
                r.append(t)
            assert all((x.data_ptr() % 16 != 0) == bool(shift) for x in phi)
            s.stag_mg_solver(dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda),
                             0.7, phi, r)
            out.append(host(phi))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
    ref = O.stag_mg_solver(pb, O.default_params(), 0.7, rhs)
    assert P.rel_inf(out[1], ref) < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gmres_graph_modes_bitwise(cuda, precision):
    """GMRES with no graphs, preconditioner graphs and whole-iteration graphs
    (modes 0, 1, 2): each solve twice (the second replays the captured
    graphs); every solution is bitwise the same, with the same iterations."""
    dim, n, visc = 3, [32, 32, 16], -1
    pb = P.problem(dim, n, visc, dx=1.0, seed=81)
    b_u, b_p = P.random_stokes(dim, n, seed=82)
    out = []
    for mode in (0, 1, 2):
        with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(gmres_rel_tol=1e-8),
                            precision=precision) as s:
            s.set_graphs(mode)
            coef = (dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda))
            bu, bp = dev(b_u, cuda), dev(b_p, cuda)
            for _ in range(2):
                x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
                status, _, st = s.gmres(bu, bp, x_u, x_p, *coef, 5.0)
                assert status == 0
                out.append((host(x_u) + [host(x_p)], st["total_iters"]))
    for xs, it in out[1:]:
        assert it == out[0][1]
        for a, b in zip(xs, out[0][0]):
            assert np.array_equal(a, b)
