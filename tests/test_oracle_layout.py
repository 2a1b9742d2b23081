"""The staggered multigrid's box layout (probin_common max_grid_size) in
the oracle: with several boxes the hierarchy stops at the boxes' depth
(compute_nlevs_mg over the boxes), and with stag_mg_bottom_solver = 4 its
bottom is the "fancy" nested stag_mg_solver over the deeper levels of the
domain (stag_mg_solver.f90:447-555, stag_mg_layout.f90:96-107)."""
import numpy as np
import pytest

import oracle as O
from tests import problems as P


@pytest.fixture
def layout():
    yield O.set_max_grid_size
    O.set_max_grid_size(None)


def solve(dim, n, mgs, set_mgs, **kw):
    pb = P.problem(dim, n, -1, seed=3)
    rhs, _ = P.random_stokes(dim, n, seed=4)
    set_mgs(mgs)
    return O.stag_mg_solver(pb, O.default_params(**kw), 0.7, rhs)


@pytest.mark.parametrize("dim,n,mgs", [(3, [32, 32, 32], [8, 8, 8]), (2, [64, 32], [16, 16])])
def test_fancy_bottom_with_one_vcycle_is_the_domain_hierarchy(layout, dim, n, mgs):
    """the nested solve's one V-cycle smooths the shared level before and
    after it, as the domain hierarchy smooths an intermediate level"""
    one = solve(dim, n, None, layout)
    fancy = solve(dim, n, mgs, layout)
    for a, b in zip(one, fancy):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("dim,n,mgs", [(3, [32, 32, 32], [8, 8, 8]), (2, [64, 32], [16, 16])])
def test_boxes_without_fancy_bottom_stop_at_the_box_depth(layout, dim, n, mgs):
    one = solve(dim, n, None, layout, stag_mg_bottom_solver=0)
    boxes = solve(dim, n, mgs, layout, stag_mg_bottom_solver=0)
    assert not all(np.array_equal(a, b) for a, b in zip(one, boxes))
    # a box hierarchy with 8 bottom smooths still solves: the residual of a
    # few V-cycles falls well below the right-hand side
    pb = P.problem(dim, n, -1, seed=3)
    rhs, _ = P.random_stokes(dim, n, seed=4)
    layout(mgs)
    hist = O.stag_mg_history(pb, O.default_params(stag_mg_bottom_solver=0, stag_mg_max_vcycles=6,
                                                  stag_mg_rel_tol=1e-30), 0.7, rhs)
    assert hist[-1] < 1e-3


def test_fancy_bottom_with_several_vcycles_nests(layout):
    dim, n, mgs = 3, [32, 32, 32], [8, 8, 8]
    kw = dict(stag_mg_max_vcycles=3, stag_mg_rel_tol=1e-12)
    one = solve(dim, n, None, layout, **kw)
    fancy = solve(dim, n, mgs, layout, **kw)
    # the nested bottom solve takes up to 3 V-cycles of its own per outer one
    assert not all(np.array_equal(a, b) for a, b in zip(one, fancy))
    rel = max(np.abs(a - b).max() for a, b in zip(one, fancy)) / max(np.abs(a).max() for a in one)
    assert rel < 1e-2  # both are converging to the same solution
