"""The allocation-free staggered multigrid entry point.

Callers that cannot allocate device memory (device memory owned by another
runtime, fixed pools, regions where an allocation would synchronise) use
fhd_dev_stag_mg_solver_noalloc.  It must give the result of the regular
fhd_dev_stag_mg_solver, call after call, although its work arrays are one
static device array that keeps the previous call's contents.  This file runs
last so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

import lowmachfhd_b200 as L
from tests import problems as P

pytestmark = pytest.mark.gpu


def _dev(a, device):
    import torch
    if isinstance(a, (list, tuple)):
        return [_dev(x, device) for x in a]
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(device)


@pytest.mark.parametrize("dim,n,visc,kw", [(3, [16, 16, 16], -1, {}),
                                           (2, [64, 32], 2, {}),
                                           (3, [16, 16, 8], 1, {"stag_mg_max_vcycles": 3, "stag_mg_rel_tol": 1e-14})])
def test_noalloc_matches_stag_mg_solver_twice(cuda, dim, n, visc, kw):
    import torch
    pb = P.problem(dim, n, visc, dx=1.0, seed=21)
    coeffs = (_dev(pb.alpha_fc, cuda), _dev(pb.beta, cuda), _dev(pb.beta_ed, cuda), _dev(pb.gamma, cuda))
    params = L.default_params(**kw)
    theta = 1.5
    with L.StokesSolver(dim, n, 1.0, visc, params=params) as s:
        for call in range(2):
            rhs, _ = P.random_stokes(dim, n, seed=30 + call)
            rhs_d = _dev(rhs, cuda)
            ref = [torch.zeros(pb.nc, dtype=torch.float64, device=cuda) for _ in range(dim)]
            s.stag_mg_solver(*coeffs, theta, ref, rhs_d)
            out = [torch.zeros(pb.nc, dtype=torch.float64, device=cuda) for _ in range(dim)]
            torch.cuda.synchronize()
            L.stag_mg_solver_noalloc(dim, n, 1.0, visc, params, *coeffs, theta, out, rhs_d)
            for c in range(dim):
                a, b = out[c].cpu().numpy(), ref[c].cpu().numpy()
                assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b)), (call, c)


def test_noalloc_rejects_oversized_grid(cuda):
    import torch
    dim, n = 3, [128, 128, 128]
    nc = int(np.prod(n))
    z = [torch.zeros(1, dtype=torch.float64, device=cuda) for _ in range(3)]
    with pytest.raises(L.FhdError) as e:
        L.stag_mg_solver_noalloc(dim, n, 1.0, 1, L.default_params(), z, z[0], z, z[0], 1.0, z, z)
    assert e.value.status == L._capi.FHD_ERR_BAD_ARG
    assert b"static scratch" in L.lib().fhd_last_error()
