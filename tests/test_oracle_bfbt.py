"""The oracle's BFBt Schur complement (visc_schur_approx = 1,
visc_schur_complement, apply_precon.f90:538-685, with inverse_diag_lap.f90):
GMRES converges with it for every precon_type and supported visc_type, it
needs no more iterations than the simple Schur complement where the
viscosity varies (the case it exists for), and |visc_type| = 3 is refused as
inverse_diag_lap refuses it."""
import pytest

import oracle as O
from tests import problems as P


@pytest.mark.parametrize("dim,n,visc", [(2, [32, 32], -1), (3, [16, 16, 16], -1), (2, [32, 16], -2),
                                        (3, [16, 8, 16], -2)])
def test_bfbt_converges_and_helps_variable_viscosity(dim, n, visc):
    pb = P.problem(dim, n, visc, seed=3)
    b_u, b_p = P.random_stokes(dim, n, seed=4)
    its = {}
    for vs in (0, 1):
        rc, _, _, _, st = O.gmres(pb, O.default_params(visc_schur_approx=vs, gmres_rel_tol=1e-9), 2.0, b_u, b_p)
        assert rc == 0
        its[vs] = st.total_iters
    assert its[1] <= its[0]


@pytest.mark.parametrize("precon", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("visc", [2, -1])
def test_bfbt_every_precon_type(precon, visc):
    dim, n = 2, [16, 16]
    pb = P.problem(dim, n, visc, seed=7)
    b_u, b_p = P.random_stokes(dim, n, seed=8)
    prm = O.default_params(visc_schur_approx=1, precon_type=precon, gmres_rel_tol=1e-9, gmres_max_iter=200)
    rc, u, p, _, st = O.gmres(pb, prm, 5.0, b_u, b_p)
    assert rc == 0, (rc, st.total_iters)


def test_bfbt_rejects_visc_type_3():
    dim, n = 2, [8, 8]
    pb = P.problem(dim, n, 3, seed=1)
    b_u, b_p = P.random_stokes(dim, n, seed=2)
    with pytest.raises(AssertionError):
        O.apply_precon(pb, O.default_params(visc_schur_approx=1), 1.0, b_u, b_p)
