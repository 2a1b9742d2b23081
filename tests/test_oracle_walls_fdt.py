"""Fluctuation-dissipation balance of the discrete operators, with walls and
periodic.

With eta = T = 1, unit variance and the non-symmetric stress (stoch_stress_form
0), the stochastic momentum flux divergence (stochastic_m_fluxdiv.f90:42-602)
is a linear map D of independent unit normals.  Its covariance D D^T must
equal -L, the visc_type 1 viscous operator with the same walls
(stag_applyop.f90 with the ghost rules of multifab_physbc_stag.f90): the
discrete fluctuation-dissipation balance.  Next to a no-slip wall the
Laplacian's diagonal gains 2 from the mirrored ghost (-u), which the wall
edge's noise supplies only when scaled by sqrt(2); at a slip wall the ghost
(+u) cancels, and the wall edge must carry no noise (mflux_bc_2d / _3d,
stochastic_m_fluxdiv.f90:363-451).  So the identity pins those rules
independently of the restatement that implements them.  It holds on the
velocity unknowns: the wall faces are held at zero and are not unknowns."""
import numpy as np
import pytest

import oracle as O
from tests import problems as P
from tests.test_oracle_stoch_walls import edge_shape

NS, SL, PE = O.NO_SLIP_WALL, O.SLIP_WALL, -1


@pytest.fixture(autouse=True)
def periodic_afterwards():
    yield
    O.set_walls()


def stochastic_map(dim, n, bc_lo, form=0):
    """the columns of D: the divergence for each unit noise entry (form 1:
    the symmetric stress, cell noise of variance 2 and one noise shared by
    both components of an edge, as fill_m_stochastic draws them)"""
    nc = int(np.prod(n[:dim]))
    nE = 1 if dim == 2 else 3
    ne = [int(np.prod(edge_shape(dim, n, e, bc_lo))) for e in range(nE)]
    # variance sqrt(vc 2 k_B / (dV dt)) = 1
    sp = O.StochParams(k_B=0.5, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=form, filtering_width=0)
    one = np.ones(nc)
    one_ed = [np.ones(m) for m in ne]
    W_cc0 = [np.zeros(nc) for _ in range(dim)]
    W_ed0 = [np.zeros(ne[e // 2]) for e in range(2 * nE)]
    cols = []

    def apply(W_cc, W_ed):
        f = O.stochastic_m_fluxdiv(dim, n, 1.0, sp, one, one_ed, one, one_ed, 1.0, [1.0], W_cc, W_ed)
        cols.append(np.concatenate(f))

    for c in range(dim):
        for i in range(nc):
            W = [w.copy() for w in W_cc0]
            W[c][i] = np.sqrt(2.0) if form == 1 else 1.0
            apply(W, W_ed0)
    for q in range(2 * nE):
        if form == 1 and q % 2 == 1:
            continue  # the second component carries the first one's noise
        for i in range(ne[q // 2]):
            W = [w.copy() for w in W_ed0]
            W[q][i] = 1.0
            if form == 1:
                W[q + 1][i] = 1.0
            apply(W_cc0, W)
    return np.array(cols).T


def minus_viscous(dim, n, visc=1):
    """the matrix of -L u (apply_matrix with theta 0 and zero pressure),
    eta = 1"""
    nc = int(np.prod(n[:dim]))
    pb = P.problem(dim, n, visc, dx=1.0, seed=1)
    pb.beta[:] = 1.0
    for e in pb.beta_ed:
        e[:] = 1.0
    pb.gamma[:] = 0.0
    cols = []
    for c in range(dim):
        for i in range(nc):
            u = [np.zeros(nc) for _ in range(dim)]
            u[c][i] = 1.0
            b_u, _ = O.apply_matrix(pb, 0.0, u, np.zeros(nc))
            cols.append(np.concatenate(b_u))
    return np.array(cols).T


def interior(dim, n, bc_lo):
    """indices of the velocity unknowns: every face but the wall faces,
    which the solve holds at zero"""
    shape = [n[d] for d in reversed(range(dim))]
    keep = []
    for c in range(dim):
        m = np.ones(shape, dtype=bool)
        if bc_lo[c] != PE:
            idx = [slice(None)] * dim
            idx[dim - 1 - c] = 0
            m[tuple(idx)] = False
        keep.append(m.ravel())
    return np.flatnonzero(np.concatenate(keep))


@pytest.mark.parametrize("dim,n,bc_lo,bc_hi", [
    (2, [6, 6], [PE, NS, PE], [PE, NS, PE]),
    (2, [6, 4], [SL, PE, PE], [SL, PE, PE]),
    (2, [4, 6], [NS, SL, PE], [SL, NS, PE]),
    (3, [4, 4, 4], [NS, SL, PE], [NS, SL, PE]),
])
def test_stochastic_covariance_is_the_viscous_operator(dim, n, bc_lo, bc_hi):
    O.set_walls(bc_lo, bc_hi)
    keep = interior(dim, n, bc_lo)
    D = stochastic_map(dim, n, bc_lo)[keep]
    A = minus_viscous(dim, n)[np.ix_(keep, keep)]
    C = D @ D.T
    assert np.max(np.abs(C - A)) < 1e-12 * np.max(np.abs(A))


def test_the_balance_fails_without_the_wall_factor():
    """the same identity with the no-slip wall edges unscaled does not hold:
    the test sees the sqrt(2)"""
    dim, n, bc = 2, [6, 6], [PE, NS, PE]
    O.set_walls(bc, bc)
    keep = interior(dim, n, bc)
    D = stochastic_map(dim, n, bc)
    A = minus_viscous(dim, n)[np.ix_(keep, keep)]
    nc = 36
    ne = int(np.prod(edge_shape(dim, n, 0, bc)))
    # the columns of the wall nodes (y = 0 and y = n) of both edge components
    Dm = D.copy()
    for comp in range(2):
        for idx in range(ne):
            j = idx // n[0]
            if j == 0 or j == n[1]:
                Dm[:, 2 * nc + comp * ne + idx] /= np.sqrt(2.0)
    Dm = Dm[keep]
    assert np.max(np.abs(Dm @ Dm.T - A)) > 0.1 * np.max(np.abs(A))


@pytest.mark.parametrize("dim,n", [(2, [6, 4]), (3, [4, 4, 4])])
@pytest.mark.parametrize("form,visc", [(0, 1), (1, 2)])
def test_periodic_covariance_is_the_viscous_operator(dim, n, form, visc):
    """periodic box: the non-symmetric stress balances visc_type 1 (eta
    Lap u), the symmetric one visc_type 2 (div eta (grad u + grad u^T))"""
    D = stochastic_map(dim, n, [PE, PE, PE], form)
    A = minus_viscous(dim, n, visc)
    assert np.max(np.abs(D @ D.T - A)) < 1e-12 * np.max(np.abs(A))
