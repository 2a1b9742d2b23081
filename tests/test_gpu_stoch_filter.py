"""The stochastic stress filter (filtering_width 1, 2, 4; filter_stoch_m_flux,
stochastic_m_fluxdiv.f90:604-778) through the C ABI: the device entry
against the oracle (FP64 and mixed, both stress forms, overwrite and
increment), the host-fab entry, an inertial step with the filter, the
refusals, and at 128^3 the size-independent identity that the filtered
divergence is the filter of the unfiltered one (both operators are
constant-coefficient stencils on the periodic box, so they commute)."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_parity import dev, host
from tests.test_gpu_stoch_walls import edge_fab
from tests.test_oracle_stoch_filter import TAPS, inputs

pytestmark = pytest.mark.gpu

W2 = [0.5, -0.25]


def sp_pair(form, width):
    kw = dict(k_B=2.0, variance_coef_mom=1.0, dV=0.125, stoch_stress_form=form, filtering_width=width)
    return O.StochParams(**kw), L.StochParams(**kw)


def device_force(cuda, dim, n, spd, eta, eta_ed, T, T_ed, W_cc, W_ed, force0=None, increment=False,
                 precision="fp64"):
    nc = P.nc_of(dim, n)
    f = dev(force0 if force0 is not None else [np.zeros(nc) for _ in range(dim)], cuda)
    with L.StokesSolver(dim, n, 0.5, 1, precision=precision) as s:
        s.stochastic_m_fluxdiv(spd, f, increment, dev(eta, cuda), dev(eta_ed, cuda), dev(T, cuda),
                               dev(T_ed, cuda), 0.1, W2, dev(W_cc, cuda), dev(W_ed, cuda))
    return f


@pytest.mark.parametrize("dim,n", [(2, [32, 24]), (3, [16, 12, 8])])
@pytest.mark.parametrize("width", [1, 2, 4])
@pytest.mark.parametrize("form,increment", [(0, False), (1, True)])
def test_filtered_stochastic_m_fluxdiv(cuda, dim, n, width, form, increment):
    eta, eta_ed, T, T_ed, W_cc, W_ed = inputs(dim, n, 21, form)
    force0 = [np.random.default_rng(22).standard_normal(P.nc_of(dim, n)) for _ in range(dim)]
    osp, lsp = sp_pair(form, width)
    ref = O.stochastic_m_fluxdiv(dim, n, 0.5, osp, eta, eta_ed, T, T_ed, 0.1, W2, W_cc, W_ed, force=force0,
                                 increment=increment)
    f = device_force(cuda, dim, n, lsp, eta, eta_ed, T, T_ed, W_cc, W_ed, force0, increment)
    assert P.rel_inf(host(f), ref) < 1e-13


@pytest.mark.parametrize("dim,n", [(2, [32, 24]), (3, [16, 12, 8])])
def test_filtered_stochastic_m_fluxdiv_mixed(cuda, dim, n):
    """FP32 stresses, filter passes and divergence: the relative error is a
    few FP32 roundings of the summed terms"""
    eta, eta_ed, T, T_ed, W_cc, W_ed = inputs(dim, n, 23, 1)
    osp, lsp = sp_pair(1, 4)
    ref = O.stochastic_m_fluxdiv(dim, n, 0.5, osp, eta, eta_ed, T, T_ed, 0.1, W2, W_cc, W_ed)
    f = device_force(cuda, dim, n, lsp, eta, eta_ed, T, T_ed, W_cc, W_ed, precision="mixed")
    assert P.rel_inf(host(f), ref) < 1e-5


def torch_filter(x, dim, n, width):
    import torch
    a = x.reshape([n[d] for d in reversed(range(dim))])
    w = TAPS[width]
    for d in range(dim):
        ax = dim - 1 - d
        y = w[0] * a
        for s in range(1, width + 1):
            y = y + w[s] * (torch.roll(a, s, dims=ax) + torch.roll(a, -s, dims=ax))
        a = y
    return a.reshape(-1)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 1e-5)])
def test_filter_commutes_with_the_divergence_at_128cube(cuda, precision, tol):
    dim, n, width = 3, [128, 128, 128], 4
    eta, eta_ed, T, T_ed, W_cc, W_ed = inputs(dim, n, 25, 1)
    _, plain = sp_pair(1, 0)
    _, filt = sp_pair(1, width)
    a = device_force(cuda, dim, n, plain, eta, eta_ed, T, T_ed, W_cc, W_ed, precision=precision)
    b = device_force(cuda, dim, n, filt, eta, eta_ed, T, T_ed, W_cc, W_ed, precision=precision)
    for c in range(dim):
        want = torch_filter(a[c], dim, n, width)
        err = float((b[c] - want).abs().max()) / float(want.abs().max())
        assert err < tol, (c, err)


def test_filtered_host_fab_entry(cuda):
    dim, n, width, PE = 2, [16, 8], 2, L.FHD_BC_PERIODIC
    eta, eta_ed, T, T_ed, W_cc, W_ed = inputs(dim, n, 27, 0)
    osp, lsp = sp_pair(0, width)
    ref = O.stochastic_m_fluxdiv(dim, n, 0.5, osp, eta, eta_ed, T, T_ed, 0.1, W2, W_cc, W_ed)
    cell, ng, bc = [0] * dim, 1, [PE, PE, PE]
    nc = P.nc_of(dim, n)
    force = [L.fab_from_canonical(np.zeros(nc), dim, n, [int(d == c) for d in range(dim)], 0) for c in range(dim)]
    with L.StokesSolver(dim, n, 0.5, 1) as s:
        s.stochastic_m_fluxdiv_fab(
            lsp, force, False, L.fab_from_canonical(eta, dim, n, cell, ng), [edge_fab([eta_ed[0]], dim, n, 0, bc, ng)],
            L.fab_from_canonical(T, dim, n, cell, ng), [edge_fab([T_ed[0]], dim, n, 0, bc, ng)], 0.1, W2,
            [L.fab_from_components(W_cc[r * dim:(r + 1) * dim], dim, n, cell, ng) for r in range(2)],
            [edge_fab(W_ed[2 * r:2 * r + 2], dim, n, 0, bc, ng) for r in range(2)])
    got = [L.canonical_from_fab(f, dim, n) for f in force]
    assert P.rel_inf(got, ref) < 1e-13


def test_inertial_step_with_the_filter(cuda):
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
    kw = dict(k_B=1e-3, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=2)
    params = O.default_params(gmres_rel_tol=1e-9)
    rc, ru, rr, rp, rst = O.advance_inertial(dim, n, 1.0, 1, params, O.StochParams(**kw), 0.05, umac, rho, pi, eta,
                                             eta_ed, kappa, T, eta_ed, W_cc, W_ed)
    assert rc == 0
    with L.StokesSolver(dim, n, 1.0, 1, params=L.default_params(gmres_rel_tol=1e-9)) as s:
        u, r_, p_ = dev(umac, cuda), dev(rho, cuda), dev(pi, cuda)
        status, st = s.advance_timestep_inertial(L.StochParams(**kw), 0.05, u, r_, p_, dev(eta, cuda),
                                                 dev(eta_ed, cuda), dev(kappa, cuda), dev(T, cuda),
                                                 dev(eta_ed, cuda), dev(W_cc, cuda), dev(W_ed, cuda))
    assert status == 0
    assert [x["total_iters"] for x in st] == [rst[0].total_iters, rst[1].total_iters]
    for c in range(dim):
        assert P.rel_inf([host(u[c])], [ru[c]]) < 1e-10
    assert P.rel_inf([host(p_)], [rp]) < 1e-10


@pytest.mark.parametrize("width,n,bc,want", [
    (3, [16, 16], None, L._capi.FHD_ERR_BAD_ARG),
    (4, [16, 2], None, L._capi.FHD_ERR_BAD_ARG),
    (1, [16, 16], "walls", L._capi.FHD_ERR_UNSUPPORTED),
])
def test_filter_refusals(cuda, width, n, bc, want):
    """checked on the host before any launch"""
    dim = 2
    nc = P.nc_of(dim, n)
    _, lsp = sp_pair(0, width)
    kw = {}
    if bc:
        kw = dict(bc_lo=[L.FHD_BC_PERIODIC, L.FHD_BC_NO_SLIP_WALL, L.FHD_BC_PERIODIC],
                  bc_hi=[L.FHD_BC_PERIODIC, L.FHD_BC_NO_SLIP_WALL, L.FHD_BC_PERIODIC])
    ne = nc + (n[0] if bc else 0)
    one, one_ed = dev(np.ones(nc), cuda), [dev(np.ones(ne), cuda)]
    f = dev([np.zeros(nc) for _ in range(dim)], cuda)
    with L.StokesSolver(dim, n, 0.5, 1, **kw) as s:
        with pytest.raises(L.FhdError) as e:
            s.stochastic_m_fluxdiv(lsp, f, False, one, one_ed, one, one_ed, 0.1, [1.0],
                                   [dev(np.ones(nc), cuda) for _ in range(dim)],
                                   [dev(np.ones(ne), cuda) for _ in range(2)])
    assert e.value.status == want
