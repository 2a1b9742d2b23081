"""Contexts made with the driver's box layout (fhd_ctx_create_bc,
max_grid_size): the staggered multigrid with several boxes, with and without
the fancy nested bottom solve, against the oracle with the same layout."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_multispecies import dev, host

pytestmark = pytest.mark.gpu


@pytest.fixture
def layout():
    yield O.set_max_grid_size
    O.set_max_grid_size(None)


CASES = [(3, [32, 32, 32], [8, 8, 8], -1), (2, [64, 32], [16, 16], 1), (3, [32, 16, 32], [16, 8, 8], 2)]
OPTS = [dict(), dict(stag_mg_bottom_solver=0), dict(stag_mg_max_vcycles=3, stag_mg_rel_tol=1e-12),
        dict(stag_mg_bottom_solver=0, stag_mg_max_vcycles=3, stag_mg_rel_tol=1e-12)]


@pytest.mark.parametrize("dim,n,mgs,visc", CASES)
@pytest.mark.parametrize("opt", range(len(OPTS)))
def test_stag_mg_box_layout(cuda, layout, dim, n, mgs, visc, opt):
    import torch
    kw = OPTS[opt]
    pb = P.problem(dim, n, visc, seed=3)
    rhs, _ = P.random_stokes(dim, n, seed=4)
    layout(mgs)
    ref = O.stag_mg_solver(pb, O.default_params(**kw), 0.7, rhs)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(**kw), max_grid_size=mgs) as s:
        phi = [torch.zeros(pb.nc, dtype=torch.float64, device=cuda) for _ in range(dim)]
        args = dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda), dev(rhs, cuda)
        torch.cuda.synchronize()  # the context launches on its own stream
        s.stag_mg_solver(args[0], args[1], args[2], args[3], 0.7, phi, args[4])
    assert P.rel_inf(host(phi), ref) < 1e-12


@pytest.mark.parametrize("mixed", [False, True])
def test_gmres_box_layout(cuda, layout, mixed):
    """GMRES with a multi-box layout whose fancy bottom nests two V-cycles"""
    import torch
    dim, n, mgs, visc = 3, [32, 32, 32], [16, 16, 16], 1
    kw = dict(gmres_rel_tol=1e-9, stag_mg_max_vcycles=2, stag_mg_rel_tol=1e-12)
    pb = P.problem(dim, n, visc, seed=11)
    b_u, b_p = P.random_stokes(dim, n, seed=12)
    layout(mgs)
    rc, ref_u, ref_p, _, st_ref = O.gmres(pb, O.default_params(**kw), 20.0, b_u, b_p)
    assert rc >= 0  # 0, or one of the reference's non-convergence warnings
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(**kw), max_grid_size=mgs,
                        precision="mixed" if mixed else "fp64") as s:
        x_u = [torch.zeros(pb.nc, dtype=torch.float64, device=cuda) for _ in range(dim)]
        x_p = torch.zeros(pb.nc, dtype=torch.float64, device=cuda)
        a = [dev(x, cuda) for x in (b_u, b_p, pb.alpha_fc, pb.beta, pb.beta_ed, pb.gamma)]
        torch.cuda.synchronize()
        status, _, st = s.gmres(a[0], a[1], x_u, x_p, a[2], a[3], a[4], a[5], 20.0)
    tol = 1e-7 if mixed else 1e-10
    if not mixed:
        assert status == rc
        assert st["total_iters"] == st_ref.total_iters
        # the true (unpreconditioned) residual GMRES reports survives the
        # multigrids' own convergence checks inside the preconditioner
        assert abs(st["norm_resid_Stokes"] - st_ref.norm_resid_Stokes) <= 1e-6 * st_ref.norm_resid_Stokes
        assert abs(st["norm_init_Stokes"] - st_ref.norm_init_Stokes) <= 1e-12 * st_ref.norm_init_Stokes
    else:
        assert status >= 0
    for c in range(dim):
        assert P.rel_inf([host(x_u[c])], [ref_u[c]]) < tol
    assert P.rel_inf([host(x_p)], [ref_p]) < tol
