"""Walls in the stochastic and mass fluxes through the C ABI against the
oracle: fhd_dev_stochastic_m_fluxdiv (mflux_bc_2d / _3d,
stochastic_m_fluxdiv.f90:363-451, the high wall's edge planes, zero normal
force on wall faces), fhd_dev_stochastic_mass_fluxdiv (stoch_mass_bc,
stochastic_mass_fluxdiv.f90:216-368), fhd_dev_compute_mass_fluxdiv and
fhd_dev_compute_sqrtLonsager_fc (first-order extrapolated concentrations at
walls, scalar_bc), FP64 and mixed; the host-fab fhd_stochastic_m_fluxdiv
(the high wall's edge planes taken from the nodal fabs) and
fhd_stochastic_mass_fluxdiv (the high wall face of a flux fab is zero, as
the periodic scatter writes it), and the host-fab
fhd_compute_sqrtLonsager_fc (the high wall face written from its own plane)."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
import oracle as O
from tests import problems as P
from tests.test_gpu_parity import dev, host
from tests.test_oracle_stoch_walls import SP, W8, fields

pytestmark = pytest.mark.gpu

NS, SL, PE = L.FHD_BC_NO_SLIP_WALL, L.FHD_BC_SLIP_WALL, L.FHD_BC_PERIODIC

CASES = [
    (2, [16, 8], [PE, NS, PE], [PE, NS, PE]),
    (2, [8, 16], [SL, PE, PE], [NS, PE, PE]),
    (2, [16, 16], [NS, SL, PE], [SL, NS, PE]),
    (3, [8, 8, 8], [PE, PE, NS], [PE, PE, NS]),
    (3, [16, 8, 8], [NS, SL, PE], [NS, SL, PE]),
    (3, [8, 8, 8], [NS, NS, SL], [SL, NS, NS]),
]


@pytest.fixture(autouse=True)
def periodic_afterwards():
    yield
    O.set_walls()


def solver(dim, n, bc_lo, bc_hi, precision="fp64"):
    return L.StokesSolver(dim, n, 0.5, 1, precision=precision, bc_lo=bc_lo, bc_hi=bc_hi)


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", CASES)
@pytest.mark.parametrize("increment", [False, True])
def test_stochastic_m_fluxdiv_walls(cuda, dim, n, bc_lo, bc_hi, increment):
    nc = P.nc_of(dim, n)
    eta, T, eta_ed, T_ed, W_cc, W_ed = fields(dim, n, bc_lo, 11)
    force0 = [np.random.default_rng(12).standard_normal(nc) for _ in range(dim)]
    O.set_walls(bc_lo, bc_hi)
    ref = O.stochastic_m_fluxdiv(dim, n, 0.5, O.StochParams(**SP), eta, eta_ed, T, T_ed, 0.1, W8, W_cc, W_ed,
                                 force=force0, increment=increment)
    with solver(dim, n, bc_lo, bc_hi) as s:
        f = dev(force0, cuda)
        s.stochastic_m_fluxdiv(L.StochParams(**SP), f, increment, dev(eta, cuda), dev(eta_ed, cuda), dev(T, cuda),
                               dev(T_ed, cuda), 0.1, W8, dev(W_cc, cuda), dev(W_ed, cuda))
    assert P.rel_inf(host(f), ref) < 1e-13


def test_stochastic_m_fluxdiv_walls_mixed(cuda):
    """the FP32 arithmetic of a mixed-precision context: relative error of
    FP32 roundoff on the summed stress"""
    dim, n, bc_lo, bc_hi = 3, [16, 8, 8], [NS, SL, PE], [NS, SL, PE]
    nc = P.nc_of(dim, n)
    eta, T, eta_ed, T_ed, W_cc, W_ed = fields(dim, n, bc_lo, 13)
    O.set_walls(bc_lo, bc_hi)
    ref = O.stochastic_m_fluxdiv(dim, n, 0.5, O.StochParams(**SP), eta, eta_ed, T, T_ed, 0.1, W8, W_cc, W_ed)
    with solver(dim, n, bc_lo, bc_hi, precision="mixed") as s:
        f = dev([np.zeros(nc) for _ in range(dim)], cuda)
        s.stochastic_m_fluxdiv(L.StochParams(**SP), f, False, dev(eta, cuda), dev(eta_ed, cuda), dev(T, cuda),
                               dev(T_ed, cuda), 0.1, W8, dev(W_cc, cuda), dev(W_ed, cuda))
    got = host(f)
    assert P.rel_inf(got, ref) < 1e-5
    for c in range(2):  # the wall faces stay exactly zero
        a = got[c].reshape(8, 8, 16)
        assert np.all((a[:, :, 0] if c == 0 else a[:, 0, :]) == 0.0)


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", [CASES[0], CASES[2], CASES[4], CASES[5]])
def test_stochastic_mass_fluxdiv_walls(cuda, dim, n, bc_lo, bc_hi):
    ns = 3
    nc = P.nc_of(dim, n)
    rng = np.random.default_rng(14)
    sqrtL = [rng.standard_normal(nc) for _ in range(dim * ns * ns)]
    W_fc = [rng.standard_normal(nc) for _ in range(2 * dim * ns)]
    div0 = [rng.standard_normal(nc) for _ in range(ns)]
    spk = dict(k_B=1.0, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    O.set_walls(bc_lo, bc_hi)
    ref_div, ref_flux = O.stochastic_mass_fluxdiv(dim, n, 0.5, O.StochParams(**spk),
                                                  O.mixture_params([1.0, 2.0, 3.0], [1.0, 0.5, 2.0]), sqrtL, 0.1,
                                                  W8, W_fc, increment=True, div0=div0, want_flux=True)
    with solver(dim, n, bc_lo, bc_hi) as s:
        div = dev(div0, cuda)
        flux = dev([np.zeros(nc) for _ in range(dim * ns)], cuda)
        s.stochastic_mass_fluxdiv(L.mixture_params([1.0, 2.0, 3.0], [1.0, 0.5, 2.0]), L.StochParams(**spk),
                                  dev(sqrtL, cuda), 0.1, W8, dev(W_fc, cuda), div, flux, increment=True)
    assert P.rel_inf(host(div), ref_div) < 1e-12
    assert P.rel_inf(host(flux), ref_flux) < 1e-12


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", [CASES[2], CASES[4], CASES[5]])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_compute_mass_fluxdiv_walls(cuda, dim, n, bc_lo, bc_hi, precision, tol):
    from tests.test_gpu_multispecies import lmix
    from tests.test_oracle_multispecies import mass_fields, mix, state
    ns = 3
    sp = dict(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-2)
    W = mass_fields(dim, n, ns, n_rngs=2)
    O.set_walls(bc_lo, bc_hi)
    ref = O.mass_fluxdiv(dim, n, 1.0, O.StochParams(**sp), mix(ns), rho, 0.05, [0.7, -0.3], W)
    with L.StokesSolver(dim, n, 1.0, 1, precision=precision, bc_lo=bc_lo, bc_hi=bc_hi) as s:
        out = dev([np.zeros(P.nc_of(dim, n)) for _ in range(ns)], cuda)
        s.compute_mass_fluxdiv(lmix(ns), L.StochParams(**sp), dev(rho, cuda), 0.05, [0.7, -0.3], dev(W, cuda), out)
    assert P.rel_inf(host(out), ref) < tol


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", [CASES[0], CASES[4]])
def test_compute_sqrtLonsager_fc_walls(cuda, dim, n, bc_lo, bc_hi):
    from tests.test_gpu_multispecies import lmix
    from tests.test_oracle_multispecies import mix, state
    ns = 3
    sp = dict(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-2)
    O.set_walls(bc_lo, bc_hi)
    ref = O.sqrtLonsager_fc(dim, n, O.StochParams(**sp), mix(ns), rho)
    with solver(dim, n, bc_lo, bc_hi) as s:
        out = dev([np.zeros(P.nc_of(dim, n)) for _ in range(dim * ns * ns)], cuda)
        s.compute_sqrtLonsager_fc(lmix(ns), L.StochParams(**sp), dev(rho, cuda), out)
    assert P.rel_inf(host(out), ref) < 1e-12


def edge_fab(xs, dim, n, e, bc_lo, ng):
    """wall-extended edge arrays of set e (one per component) -> one
    whole-domain nodal fab: in a wall direction of the set the nodal plane
    hi+1 is the high wall's, elsewhere the duplicated plane wraps"""
    dirs = (0, 1) if dim == 2 else [(0, 1), (0, 2), (1, 2)][e]
    nodal = [1 if d in dirs else 0 for d in range(dim)]
    shape = tuple(reversed([n[d] + (1 if (d in dirs and bc_lo[d] != PE) else 0) for d in range(dim)]))
    idx = []
    for d in range(dim):
        r = np.arange(-ng, n[d] + nodal[d] + ng)
        idx.append(np.clip(r, 0, shape[dim - 1 - d] - 1) if bc_lo[d] != PE else np.mod(r, n[d]))
    comps = []
    for x in xs:
        a = x.reshape(shape)
        sub = a[np.ix_(idx[1], idx[0])] if dim == 2 else a[np.ix_(idx[2], idx[1], idx[0])]
        comps.append(np.asfortranarray(sub.T))
    data = np.asfortranarray(np.stack(comps, axis=-1)) if len(comps) > 1 else comps[0]
    pad = [0] * (3 - dim)
    return L.FabArray(data, [0] * dim + pad, [k - 1 for k in n[:dim]] + pad, nodal + pad, ng, ncomp=len(xs))


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", [CASES[0], CASES[4], CASES[5]])
def test_stochastic_m_fluxdiv_host_fabs_walls(cuda, dim, n, bc_lo, bc_hi):
    nE = 1 if dim == 2 else 3
    eta, T, eta_ed, T_ed, W_cc, W_ed = fields(dim, n, bc_lo, 15)
    rng = np.random.default_rng(16)
    force0 = [rng.standard_normal(P.nc_of(dim, n)) for _ in range(dim)]
    O.set_walls(bc_lo, bc_hi)
    ref = O.stochastic_m_fluxdiv(dim, n, 0.5, O.StochParams(**SP), eta, eta_ed, T, T_ed, 0.1, W8, W_cc, W_ed,
                                 force=force0, increment=True)
    ng = 1
    cell = [0] * dim
    force = [L.fab_from_canonical(force0[c], dim, n, [int(d == c) for d in range(dim)], 0) for c in range(dim)]
    with solver(dim, n, bc_lo, bc_hi) as s:
        s.stochastic_m_fluxdiv_fab(
            L.StochParams(**SP), force, True, L.fab_from_canonical(eta, dim, n, cell, ng),
            [edge_fab([eta_ed[e]], dim, n, e, bc_lo, ng) for e in range(nE)],
            L.fab_from_canonical(T, dim, n, cell, ng), [edge_fab([T_ed[e]], dim, n, e, bc_lo, ng) for e in range(nE)],
            0.1, W8, [L.fab_from_components(W_cc[r * dim:(r + 1) * dim], dim, n, cell, ng) for r in range(2)],
            [edge_fab(W_ed[(r * nE + e) * 2:(r * nE + e) * 2 + 2], dim, n, e, bc_lo, ng)
             for r in range(2) for e in range(nE)])
    got = [L.canonical_from_fab(f, dim, n) for f in force]
    assert P.rel_inf(got, ref) < 1e-13


def test_stochastic_m_fluxdiv_host_fabs_walls_checks_the_edge_fabs(cuda):
    """with walls an edge multifab must be one whole-domain fab, nodal in its
    set's directions (else its high-wall plane is not there)"""
    dim, n, bc_lo, bc_hi = CASES[0]
    eta, T, eta_ed, T_ed, W_cc, W_ed = fields(dim, n, bc_lo, 17)
    cell = [0, 0]
    nc = P.nc_of(dim, n)
    force = [L.fab_from_canonical(np.zeros(nc), dim, n, [int(d == c) for d in range(dim)], 0) for c in range(dim)]
    wrong = L.fab_from_canonical(np.ones(nc), dim, n, cell, 1)  # a cell fab where a node fab belongs
    with solver(dim, n, bc_lo, bc_hi) as s:
        with pytest.raises(L.FhdError) as e:
            s.stochastic_m_fluxdiv_fab(
                L.StochParams(**SP), force, False, L.fab_from_canonical(eta, dim, n, cell, 1), [wrong],
                L.fab_from_canonical(T, dim, n, cell, 1), [edge_fab([T_ed[0]], dim, n, 0, bc_lo, 1)], 0.1, W8,
                [L.fab_from_components(W_cc[r * 2:(r + 1) * 2], dim, n, cell, 1) for r in range(2)],
                [edge_fab(W_ed[2 * r:2 * r + 2], dim, n, 0, bc_lo, 1) for r in range(2)])
        assert e.value.status == L._capi.FHD_ERR_BAD_ARG


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", [CASES[2], CASES[4]])
def test_stochastic_mass_fluxdiv_host_fabs_walls(cuda, dim, n, bc_lo, bc_hi):
    from tests.test_gpu_boundary import assert_mf, face_nodal, mf
    from tests.test_gpu_multispecies import lmix
    from tests.test_oracle_multispecies import mass_fields, mix, state
    ns = 3
    nc = P.nc_of(dim, n)
    sp = dict(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-2)
    W = mass_fields(dim, n, ns, n_rngs=2)
    div0 = [np.random.default_rng(18).standard_normal(nc) for _ in range(ns)]
    O.set_walls(bc_lo, bc_hi)
    sqL = O.sqrtLonsager_fc(dim, n, O.StochParams(**sp), mix(ns), rho)
    ref_div, ref_flux = O.stochastic_mass_fluxdiv(dim, n, 1.0, O.StochParams(**sp), mix(ns), sqL, 0.05, [0.7, -0.3],
                                                  W, increment=True, div0=div0, want_flux=True)
    L_f = [mf(sqL[d * ns * ns:(d + 1) * ns * ns], dim, n, face_nodal(dim, d), 0, 1) for d in range(dim)]
    W_f = [mf(W[q * ns:(q + 1) * ns], dim, n, face_nodal(dim, q % dim), 0, 1) for q in range(2 * dim)]
    div_f = mf(div0, dim, n, [0] * dim, 1, 1)
    flux_f = [mf([np.zeros(nc)] * ns, dim, n, face_nodal(dim, d), 0, 1) for d in range(dim)]
    with L.StokesSolver(dim, n, 1.0, 1, bc_lo=bc_lo, bc_hi=bc_hi) as s:
        s.stochastic_mass_fluxdiv_fab(lmix(ns), L.StochParams(**sp), mf(rho, dim, n, [0] * dim, 1, 1), None, L_f,
                                      div_f, flux_f, 0.05, [0.7, -0.3], W_f, increment=True)
    assert_mf(div_f, ref_div, dim, n, [0] * dim, 1, 1, 1e-12)
    for d in range(dim):
        assert_mf(flux_f[d], ref_flux[d * ns:(d + 1) * ns], dim, n, face_nodal(dim, d), 0, 1, 1e-12)


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", [CASES[0], CASES[4]])
def test_compute_sqrtLonsager_fc_host_fabs_walls(cuda, dim, n, bc_lo, bc_hi):
    """faces 0 .. n-1 as the device entry, and the fab's nodal plane hi+1 of
    a wall direction the high wall's own factor: the last cell with its
    extrapolated ghost, which is face 0 of the density flipped along d"""
    from tests.test_gpu_boundary import face_nodal, mf
    from tests.test_gpu_multispecies import lmix
    from tests.test_oracle_multispecies import mix, state
    ns = 3
    sp = dict(k_B=1e-4, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    rho = state(dim, n, ns, amp=1e-2)
    shape = [n[k] for k in reversed(range(dim))]
    O.set_walls(bc_lo, bc_hi)
    ref = O.sqrtLonsager_fc(dim, n, O.StochParams(**sp), mix(ns), rho)
    out = [mf([np.zeros(P.nc_of(dim, n))] * (ns * ns), dim, n, face_nodal(dim, d), 0, 1) for d in range(dim)]
    with solver(dim, n, bc_lo, bc_hi) as s:
        s.compute_sqrtLonsager_fc_fab(lmix(ns), L.StochParams(**sp), mf(rho, dim, n, [0] * dim, 1, 1), None, out)
    scale = max(float(np.max(np.abs(x))) for x in ref)
    for d in range(dim):
        data = out[d][0].data
        flip = None
        if bc_lo[d] != PE:
            ax = dim - 1 - d
            flip = O.sqrtLonsager_fc(dim, n, O.StochParams(**sp), mix(ns),
                                     [np.flip(r.reshape(shape), axis=ax).ravel() for r in rho])
        for q in range(ns * ns):
            arr = data[..., q]
            got = arr[tuple(slice(0, n[k]) for k in range(dim))].T.ravel()
            assert np.max(np.abs(got - ref[d * ns * ns + q])) <= 1e-12 * scale
            if flip is not None:
                hi_plane = np.take(arr, n[d], axis=d)  # Fortran axes: x, y, (z) without d
                want = np.take(flip[d * ns * ns + q].reshape(shape), 0, axis=dim - 1 - d).T
                assert np.max(np.abs(hi_plane - want)) <= 1e-12 * scale
