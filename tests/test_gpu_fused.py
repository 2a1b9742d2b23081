"""The row-tile fused smoother of the large FP32 levels (visc_type 1,
fhd_ctx_set_fused) against the colour-by-colour sweeps on the same inputs,
and against the oracle.  Both evaluate the same stencil expression in the
same colour order on the same operands; the FP32 results agree to FP32
roundoff (the fused smooth is out of place, so no value differs in its
inputs), and GMRES takes the same number of iterations."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_parity import dev, host, zeros

pytestmark = pytest.mark.gpu

# level 0 above 64^3 cells with an x extent of 64..256 (the fused smoother's
# range): 16-row tiles on 128x64x64, 8-row tiles on 256x64x32, 32-row tiles
# and z-runs of a non-power-of-two depth on 64x128x48
GRIDS = [[128, 64, 64], [256, 64, 32], [64, 128, 48]]


def _vcycle_and_precon(cuda, n, fused, seed=51):
    dim, visc = 3, 1
    pb = P.problem(dim, n, visc, dx=1.0, seed=seed)
    rhs, _ = P.random_stokes(dim, n, seed=seed + 1)
    b_u, b_p = P.random_stokes(dim, n, seed=seed + 2, zero_mean_p=False)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(), precision="mixed") as s:
        s.set_fused(fused)
        s.set_tune(0)  # the fixed size rules: fused where the level allows
        coef = (dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda))
        phi = zeros(pb.nc, dim, cuda)
        s.stag_mg_solver(*coef, 0.7, phi, dev(rhs, cuda))
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_precon(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, *coef, 1.5)
        launches = s.kernel_launches
    return pb, rhs, host(phi), host(x_u) + [host(x_p)], launches


@pytest.mark.parametrize("n", GRIDS)
def test_fused_matches_colour_sweeps(cuda, n):
    pb, rhs, phi1, x1, n1 = _vcycle_and_precon(cuda, n, 1)
    _, _, phi0, x0, n0 = _vcycle_and_precon(cuda, n, 0)
    assert n1 < n0  # the fused launches replaced colour launches
    assert P.rel_inf(phi1, phi0) < 1e-5
    assert P.rel_inf(x1, x0) < 1e-5


def test_fused_vcycle_against_oracle(cuda):
    """One FP32 V-cycle through the fused smoother against the oracle's FP64
    V-cycle on the same inputs: FP32 roundoff apart."""
    n = [128, 64, 64]
    pb, rhs, phi, _, _ = _vcycle_and_precon(cuda, n, 1)
    ref = O.stag_mg_solver(pb, O.default_params(), 0.7, rhs)
    assert P.rel_inf(phi, ref) < 1e-4


def test_fused_gmres(cuda):
    """Mixed-precision GMRES at 1e-8 with the fused smoother on and off:
    the same iteration count and solutions that agree to the tolerance."""
    import torch
    dim, n, visc = 3, [128, 64, 64], 1
    pb = P.problem(dim, n, visc, dx=1.0, seed=61)
    b_u, b_p = P.random_stokes(dim, n, seed=62)
    out = {}
    for fused in (1, 0):
        with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(gmres_rel_tol=1e-8),
                            precision="mixed") as s:
            s.set_fused(fused)
            s.set_tune(0)
            x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
            status, _, st = s.gmres(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, dev(pb.alpha_fc, cuda),
                                    dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), 20.0)
            assert status == 0
            assert st["norm_resid"] <= 1e-8 * min(st["norm_pre_b"], st["norm_init_resid"])
            out[fused] = (host(x_u) + [host(x_p)], st["total_iters"])
    assert abs(out[1][1] - out[0][1]) <= 1
    assert P.rel_inf(out[1][0], out[0][0]) < 1e-6
    del torch
