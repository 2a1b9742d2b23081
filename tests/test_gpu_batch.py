"""The batched solver (fhd_batch_*): many 2D periodic boxes of uneven size,
one launch per multigrid level and operation for all of them.  Each box's
GMRES solve must equal the single-box solver's on the same inputs, a box's
result must not depend on the other boxes of the batch, and the overdamped
step must equal the oracle's per box."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_multispecies import dev, host

pytestmark = pytest.mark.gpu

# levels above the coarse kernel (128, 96), a whole hierarchy in one CTA
# (40x24 -> 5x3, odd bottom), non-square and power-of-two boxes
SIZES = [(32, 32), (128, 128), (96, 96), (40, 24), (64, 32), (48, 80)]
ETAS = [1.0, 3.7, 0.6, 2.2, 1.4, 4.9]


def packed(arrs_per_box):
    """concatenate per-box arrays (a list per box of 3 components) into 3
    packed component arrays"""
    return [np.concatenate([a[c] for a in arrs_per_box]) for c in range(3)]


def rhs(sizes, seed):
    out = []
    for k, (nx, ny) in enumerate(sizes):
        b_u, b_p = P.random_stokes(2, [nx, ny], seed=seed + k)
        out.append([b_u[0], b_u[1], b_p])
    return out


def single(cuda, nx, ny, eta, b, precision, theta, params):
    nc = nx * ny
    one = np.ones(nc)
    with L.StokesSolver(2, [nx, ny], 1.0, 1, params=L.default_params(**params), precision=precision) as s:
        x_u = [dev(np.zeros(nc), cuda) for _ in range(2)]
        x_p = dev(np.zeros(nc), cuda)
        a = dev([b[0], b[1]], cuda), dev(b[2], cuda), dev([one, one], cuda), dev(eta * one, cuda), \
            dev([eta * one], cuda), dev(np.zeros(nc), cuda)
        import torch
        torch.cuda.synchronize()
        status, _, st = s.gmres(a[0], a[1], x_u, x_p, a[2], a[3], a[4], a[5], theta)
    return status, [host(x_u[0]), host(x_u[1]), host(x_p)], st


def batched(cuda, sizes, etas, bs, precision, theta, params):
    import torch
    with L.Batch(sizes, 1.0, params=L.default_params(**params), precision=precision) as B:
        bp = dev(packed(bs), cuda)
        x = [torch.zeros(B.total, dtype=torch.float64, device=cuda) for _ in range(3)]
        torch.cuda.synchronize()
        status, stats = B.gmres(bp, x, etas, theta)
        xs = [[host(B.box(x[c], k)) for c in range(3)] for k in range(len(sizes))]
        launches = B.kernel_launches
    return status, xs, stats, launches


@pytest.mark.parametrize("theta", [0.0, 5.0])
def test_batched_gmres_equals_single_box_fp64(cuda, theta):
    params = dict(gmres_rel_tol=1e-9)
    bs = rhs(SIZES, 10)
    status, xs, stats, _ = batched(cuda, SIZES, ETAS, bs, "fp64", theta, params)
    for k, (nx, ny) in enumerate(SIZES):
        st1, x1, s1 = single(cuda, nx, ny, ETAS[k], bs[k], "fp64", theta, params)
        assert stats[k]["total_iters"] == s1["total_iters"], k
        assert stats[k]["status"] == st1
        assert P.rel_inf(xs[k][:2], x1[:2]) < 1e-10, k
        assert P.rel_inf(xs[k][2:], x1[2:]) < 1e-10, k


def test_batched_gmres_mixed_precision(cuda):
    """FP32 multigrid inside FP64 GMRES: the batched and the single-box
    mixed solves take the same number of iterations (+-2: their FP32
    roundings differ) and both reach the FP64 solution to the Krylov
    tolerance.  At theta = 0 the rhs is made consistent (velocity means
    removed): with a mean left in b_u the FP32 V-cycle rounds relative to
    that unreachable constant and the preconditioned residual levels off
    near 1e-6 (FHD_WARN_NOT_CONVERGED_OUTER), where FP64 reports
    FHD_WARN_TRUE_RESID."""
    params = dict(gmres_rel_tol=1e-10)
    bs = [[b[0] - b[0].mean(), b[1] - b[1].mean(), b[2]] for b in rhs(SIZES, 30)]
    status, xs, stats, _ = batched(cuda, SIZES, ETAS, bs, "mixed", 0.0, params)
    assert status == 0
    for k, (nx, ny) in enumerate(SIZES):
        st1, x1, s1 = single(cuda, nx, ny, ETAS[k], bs[k], "mixed", 0.0, params)
        st6, x64, _ = single(cuda, nx, ny, ETAS[k], bs[k], "fp64", 0.0, params)
        assert st1 == 0 and st6 == 0 and stats[k]["status"] == 0, k
        assert abs(stats[k]["total_iters"] - s1["total_iters"]) <= 2, k
        for a in (xs[k], x1):
            assert P.rel_inf(a[:2], x64[:2]) < 1e-8, k
            assert P.rel_inf(a[2:], x64[2:]) < 1e-8, k


def test_box_result_does_not_depend_on_the_batch(cuda):
    """a box solved in a batch of six gives bitwise the result it gives
    alone: per-box reductions in a fixed order, masked slots"""
    params = dict(gmres_rel_tol=1e-9)
    bs = rhs(SIZES, 50)
    for precision in ("fp64", "mixed"):
        _, xs, stats, _ = batched(cuda, SIZES, ETAS, bs, precision, 0.0, params)
        for k in (1, 3):
            _, x1, s1, _ = batched(cuda, [SIZES[k]], [ETAS[k]], [bs[k]], precision, 0.0, params)
            assert stats[k]["total_iters"] == s1[0]["total_iters"]
            for c in range(3):
                assert np.array_equal(xs[k][c], x1[0][c]), (precision, k, c)


def test_launches_do_not_grow_with_the_box_count(cuda):
    params = dict(gmres_rel_tol=1e-9)
    sizes = [(64, 64)] * 4
    bs = rhs(sizes, 70)
    _, _, st4, n4 = batched(cuda, sizes, [1.0] * 4, bs, "mixed", 0.0, params)
    sizes16 = [(64, 64)] * 16
    bs16 = rhs(sizes16, 70)
    _, _, st16, n16 = batched(cuda, sizes16, [1.0] * 16, bs16, "mixed", 0.0, params)
    if max(s["total_iters"] for s in st4) == max(s["total_iters"] for s in st16):
        assert n16 == n4


def test_batched_overdamped_step_equals_oracle(cuda):
    """one noise-free overdamped step per box (k_B T = 0) against the
    oracle's advance_overdamped (single fluid, density 1)"""
    import torch
    sizes = [(32, 32), (64, 48), (40, 24)]
    etas = [1.0, 2.5, 0.7]
    dt = 0.1
    params = dict(gmres_rel_tol=1e-10)
    rng = np.random.default_rng(4)
    u0 = [[1e-2 * rng.standard_normal(nx * ny) for _ in range(2)] for nx, ny in sizes]
    p0 = [1e-2 * rng.standard_normal(nx * ny) for nx, ny in sizes]
    with L.Batch(sizes, 1.0, params=L.default_params(**params), precision="fp64") as B:
        u = [dev(np.concatenate([a[c] for a in u0]), cuda) for c in range(2)]
        pi = dev(np.concatenate(p0), cuda)
        torch.cuda.synchronize()
        status, iters = B.overdamped(u, pi, etas, [0.0] * len(sizes), dt, 1, seed=3)
        ub = [[host(B.box(u[c], k)) for c in range(2)] for k in range(len(sizes))]
        pb = [host(B.box(pi, k)) for k in range(len(sizes))]
    assert status in (0, 3)
    sp = O.StochParams(k_B=0.0, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    for k, (nx, ny) in enumerate(sizes):
        n = [nx, ny]
        nc = nx * ny
        eta = etas[k] * np.ones(nc)
        W_cc, W_ed = P.stochastic_fields(2, n, seed=9, n_rngs=2)
        rc, u_r, rho_r, pi_r, st_r = O.advance_overdamped(2, n, 1.0, 1, O.default_params(**params), sp, None, dt,
                                                          u0[k], [np.ones(nc)], p0[k], eta, [eta], np.zeros(nc),
                                                          np.ones(nc), [np.ones(nc)], W_cc, W_ed, None)
        assert rc in (0, 3)
        assert P.rel_inf(ub[k], u_r) < 1e-8, k
        assert P.rel_inf([pb[k]], [pi_r]) < 1e-8, k
        assert iters[k] == st_r[0].total_iters + st_r[1].total_iters


def test_batched_overdamped_noise(cuda):
    """from rest, one step's velocity is linear in the noise amplitude
    sqrt(k_B T); the same seed repeats, another seed differs"""
    import torch
    sizes = [(32, 32), (48, 48)]

    def run(kT, seed):
        with L.Batch(sizes, 1.0, params=L.default_params(gmres_rel_tol=1e-10), precision="fp64") as B:
            u = [torch.zeros(B.total, dtype=torch.float64, device=cuda) for _ in range(2)]
            pi = torch.zeros(B.total, dtype=torch.float64, device=cuda)
            torch.cuda.synchronize()
            B.overdamped(u, pi, [1.0, 2.0], [kT, kT], 0.1, 1, seed=seed)
            return [host(x) for x in u]

    a, b, c, d = run(1.0, 5), run(4.0, 5), run(1.0, 5), run(1.0, 6)
    assert np.all(np.isfinite(a[0])) and np.abs(a[0]).max() > 0
    for x, y in zip(a, b):
        assert np.allclose(2.0 * x, y, rtol=1e-7, atol=1e-12 * np.abs(y).max())
    assert all(np.array_equal(x, y) for x, y in zip(a, c))
    assert not np.allclose(a[0], d[0])
