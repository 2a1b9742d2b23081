"""gmres_spatial_order = 4 in the oracle (apply_matrix.f90:54-67, 124-135).

The reference holds no stored results for this option, so the restatement is
checked by the properties of its formulas on smooth periodic fields:
  * the viscous operator of stag_applyop_4o (stag_applyop.f90:1262-1510)
    converges at fourth order;
  * the gradient of compute_grad_4o (div_and_grad.f90:804-880) converges at
    second order: its weights -1, 15, -15, 1 over 12 dx leave -h^2/24 of the
    third derivative, the same leading error as the two-point difference;
  * order 2 is unchanged by the order argument;
  * visc_type other than 1 is refused, as stag_applyop_4o refuses it.
"""
import numpy as np
import pytest

import oracle as O
from tests import problems as P


def face_coords(dim, n, c):
    """coordinates of the faces of component c on [0, 1]^dim"""
    h = 1.0 / n
    axes = [(np.arange(n) + (0.0 if d == c else 0.5)) * h for d in range(dim)]
    grids = np.meshgrid(*axes, indexing="ij")
    # canonical layout: x fastest
    return [g.transpose(tuple(range(dim))[::-1]).ravel() for g in grids]


def cell_coords(dim, n):
    h = 1.0 / n
    axes = [(np.arange(n) + 0.5) * h for _ in range(dim)]
    grids = np.meshgrid(*axes, indexing="ij")
    return [g.transpose(tuple(range(dim))[::-1]).ravel() for g in grids]


def viscous_error(dim, n, order):
    """max |A u - beta (-lap u)| for u_c = prod_d sin(2 pi x_d), p = 0,
    theta = 0"""
    nn = [n] * dim
    pb = P.problem(dim, nn, 1, dx=1.0 / n, seed=1)
    k = 2.0 * np.pi
    u = []
    for c in range(dim):
        X = face_coords(dim, n, c)
        u.append(np.prod([np.sin(k * x) for x in X], axis=0))
    b_u, _ = O.apply_matrix(pb, 0.0, u, np.zeros(pb.nc), order=order)
    beta = pb.beta[0]
    return max(np.max(np.abs(b_u[c] - beta * dim * k * k * u[c])) for c in range(dim))


def gradient_error(dim, n, order):
    """max |A (0, p) - grad p| for p = cos(2 pi x)"""
    nn = [n] * dim
    pb = P.problem(dim, nn, 1, dx=1.0 / n, seed=1)
    k = 2.0 * np.pi
    p = np.cos(k * cell_coords(dim, n)[0])
    b_u, _ = O.apply_matrix(pb, 0.0, [np.zeros(pb.nc) for _ in range(dim)], p, order=order)
    exact = -k * np.sin(k * face_coords(dim, n, 0)[0])
    return np.max(np.abs(b_u[0] - exact))


@pytest.mark.parametrize("dim,n0", [(2, 16), (3, 16)])
def test_viscous_operator_is_fourth_order(dim, n0):
    e1, e2 = viscous_error(dim, n0, 4), viscous_error(dim, 2 * n0, 4)
    assert 13.0 < e1 / e2 < 17.0
    # and second order with the default stencil
    f1, f2 = viscous_error(dim, n0, 2), viscous_error(dim, 2 * n0, 2)
    assert 3.5 < f1 / f2 < 4.5


@pytest.mark.parametrize("dim,n0", [(2, 16), (3, 8)])
def test_gradient_is_second_order(dim, n0):
    e1, e2 = gradient_error(dim, n0, 4), gradient_error(dim, 2 * n0, 4)
    assert 3.5 < e1 / e2 < 4.5
    # the leading error: -h^2/24 of the third derivative, k^3 h^2 / 24 at most
    h = 1.0 / (2 * n0)
    k = 2.0 * np.pi
    assert abs(e2 - k ** 3 * h * h / 24.0) < 0.1 * e2


def test_order_two_is_unchanged():
    pb = P.problem(2, [16, 8], 1, dx=0.5, seed=3)
    u, p = P.random_stokes(2, [16, 8], seed=4)
    a = O.apply_matrix(pb, 2.0, u, p)
    b = O.apply_matrix(pb, 2.0, u, p, order=2)
    assert all(np.array_equal(x, y) for x, y in zip(a[0], b[0]))
    assert np.array_equal(a[1], b[1])


@pytest.mark.parametrize("visc", [-1, 2, -2, 3, -3])
def test_order_four_needs_visc_type_one(visc):
    pb = P.problem(2, [8, 8], visc, dx=1.0, seed=5)
    u, p = P.random_stokes(2, [8, 8], seed=6)
    with pytest.raises(AssertionError):
        O.apply_matrix(pb, 1.0, u, p, order=4)


def test_divergence_stays_second_order():
    """the pressure row is -D u with the second-order divergence for both
    orders (apply_matrix.f90:143-147)"""
    pb = P.problem(3, [8, 8, 8], 1, dx=0.25, seed=7)
    u, p = P.random_stokes(3, [8, 8, 8], seed=8)
    _, bp2 = O.apply_matrix(pb, 0.0, u, p, order=2)
    _, bp4 = O.apply_matrix(pb, 0.0, u, p, order=4)
    assert np.array_equal(bp2, bp4)
