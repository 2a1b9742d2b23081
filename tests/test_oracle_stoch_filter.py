"""The stochastic stress filter (filtering_width 1, 2, 4; filter_stoch_m_flux,
stochastic_m_fluxdiv.f90:604-778) in the oracle.

The filter smooths the scaled random stresses before their divergence
(stochastic_m_fluxdiv.f90:172-174, 226-230): one pass along x, then y, then
z, each a symmetric stencil over the periodic images.  On a periodic box
both the filter and the divergence are constant-coefficient difference
operators, so they commute: the filtered divergence equals the filter
applied to the unfiltered divergence on each face array.  The tests check
that identity against a numpy statement of the stencil weights, the
weights themselves (unit response at wavenumber 0, zero at the grid
Nyquist wavenumber, flat to order 2 * width at 0), and the refusals."""
import numpy as np
import pytest

import oracle as O
from tests import problems as P

BAD_ARG, UNSUPPORTED = -1, -5  # FHD_ERR_BAD_ARG, FHD_ERR_UNSUPPORTED

# taps of filter_stoch_m_flux, offset 0..width (symmetric)
TAPS = {1: [1 / 2, 1 / 4],
        2: [5 / 8, 1 / 4, -1 / 16],
        4: [93 / 128, 7 / 32, -7 / 64, 1 / 32, -1 / 256]}


def filt_np(dim, n, a, width):
    """the separable periodic filter of one array in the canonical layout
    (x fastest)"""
    shape = [n[d] for d in reversed(range(dim))]
    x = a.reshape(shape)
    for d in range(dim):
        ax = dim - 1 - d
        w = TAPS[width]
        y = w[0] * x
        for s in range(1, width + 1):
            y = y + w[s] * (np.roll(x, s, axis=ax) + np.roll(x, -s, axis=ax))
        x = y
    return x.ravel()


def inputs(dim, n, seed, form):
    nc = P.nc_of(dim, n)
    rng = np.random.default_rng(seed)
    eta = 1 + rng.random(nc)
    T = 1 + rng.random(nc)
    eta_ed = O.average_cc_to_edge(dim, n, eta)
    T_ed = O.average_cc_to_edge(dim, n, T)
    W_cc, W_ed = P.stochastic_fields(dim, n, seed=seed + 1, n_rngs=2, symmetric=form == 1)
    return eta, eta_ed, T, T_ed, W_cc, W_ed


def sp_of(form, width):
    return O.StochParams(k_B=2.0, variance_coef_mom=1.0, dV=0.125, stoch_stress_form=form,
                         filtering_width=width)


@pytest.mark.parametrize("width", [1, 2, 4])
def test_taps_sum_to_one_and_vanish_at_nyquist(width):
    w = TAPS[width]
    k = np.linspace(0, np.pi, 9)
    sym = w[0] + 2 * sum(w[s] * np.cos(s * k) for s in range(1, width + 1))
    assert abs(sym[0] - 1) < 1e-15 and abs(sym[-1]) < 1e-15
    assert np.all(sym >= -1e-15) and np.all(sym <= 1 + 1e-15)
    # flat at k = 0: the moments sum_s s^(2m) w_s vanish for 1 <= m < width
    for m in range(1, width):
        assert abs(sum(w[s] * s ** (2 * m) for s in range(1, width + 1))) < 1e-15


@pytest.mark.parametrize("dim,n", [(2, [8, 6]), (3, [6, 4, 8])])
@pytest.mark.parametrize("width", [1, 2, 4])
@pytest.mark.parametrize("form", [0, 1])
def test_filtered_divergence_is_the_filtered_force(dim, n, width, form):
    eta, eta_ed, T, T_ed, W_cc, W_ed = inputs(dim, n, 3, form)
    plain = O.stochastic_m_fluxdiv(dim, n, 0.5, sp_of(form, 0), eta, eta_ed, T, T_ed, 0.1, [0.5, -0.25],
                                   W_cc, W_ed)
    filt = O.stochastic_m_fluxdiv(dim, n, 0.5, sp_of(form, width), eta, eta_ed, T, T_ed, 0.1, [0.5, -0.25],
                                  W_cc, W_ed)
    want = [filt_np(dim, n, f, width) for f in plain]
    assert P.rel_inf(filt, want) < 1e-13
    # the filter does something
    assert P.rel_inf(filt, plain) > 0.1


def test_increment_adds_the_filtered_divergence():
    dim, n, width = 3, [4, 4, 4], 4
    eta, eta_ed, T, T_ed, W_cc, W_ed = inputs(dim, n, 5, 1)
    rng = np.random.default_rng(2)
    f0 = [rng.standard_normal(P.nc_of(dim, n)) for _ in range(dim)]
    sp = sp_of(1, width)
    alone = O.stochastic_m_fluxdiv(dim, n, 0.5, sp, eta, eta_ed, T, T_ed, 0.1, [1.0, 0.5], W_cc, W_ed)
    inc = O.stochastic_m_fluxdiv(dim, n, 0.5, sp, eta, eta_ed, T, T_ed, 0.1, [1.0, 0.5], W_cc, W_ed,
                                 force=f0, increment=True)
    assert P.rel_inf(inc, [a + b for a, b in zip(f0, alone)]) < 1e-14


@pytest.fixture
def walls_afterwards():
    yield
    O.set_walls()


@pytest.mark.parametrize("width,n,want", [(3, [8, 8], BAD_ARG), (4, [8, 3], BAD_ARG),
                                          (4, [3, 8], BAD_ARG)])
def test_bad_widths_are_refused(width, n, want):
    dim = 2
    eta, eta_ed, T, T_ed, W_cc, W_ed = inputs(dim, n, 1, 0)
    rc, _ = O.stochastic_m_fluxdiv(dim, n, 0.5, sp_of(0, width), eta, eta_ed, T, T_ed, 0.1, [0.5, -0.25],
                                   W_cc, W_ed, status=True)
    assert rc == want


def test_filter_with_walls_is_unsupported(walls_afterwards):
    dim, n = 2, [8, 8]
    O.set_walls([-1, O.NO_SLIP_WALL, -1], [-1, O.NO_SLIP_WALL, -1])
    eta, eta_ed, T, T_ed, W_cc, W_ed = inputs(dim, n, 1, 0)
    W_ed = [np.concatenate([w, w[:n[0]]]) for w in W_ed]  # the high-wall row of nodes
    ext = [np.concatenate([e, e[:n[0]]]) for e in eta_ed]
    rc, _ = O.stochastic_m_fluxdiv(dim, n, 0.5, sp_of(0, 1), eta, ext, T, ext, 0.1, [0.5, -0.25],
                                   W_cc, W_ed, status=True)
    assert rc == UNSUPPORTED
