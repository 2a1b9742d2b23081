"""CPU-side checks of the product library: it loads without a GPU, exports
every function include/fhd_b200.h declares, reports a missing device as an
error code, and the host fab helpers round-trip."""
import ctypes as C
import os

import numpy as np
import pytest

import lowmachfhd_b200 as L
from lowmachfhd_b200 import _capi


def test_library_exists():
    assert os.path.exists(_capi.LIB_PATH), "run lowmachfhd_b200/build.py"


def test_exports_every_header_symbol():
    names = _capi.header_functions()
    assert len(names) >= 15
    lib = C.CDLL(_capi.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_default_matches_probin():
    p = L.default_params()
    assert (p.precon_type, p.stag_mg_nsmooths_down, p.stag_mg_nsmooths_bottom, p.gmres_max_inner) == (1, 2, 8, 5)
    assert p.gmres_rel_tol == 1e-9 and p.stag_mg_smoother == 1 and p.mg_max_vcycles == 1


def test_status_strings():
    assert b"orthogonalization" in _capi.lib().fhd_status_string(_capi.FHD_ERR_ORTHO_BREAKDOWN)


def test_bad_arguments_rejected_before_device():
    lib = _capi.lib()
    h = C.c_void_p()
    p = L.default_params()
    n = (C.c_int * 3)(16, 16, 1)
    rc = lib.fhd_ctx_create(2, n, (C.c_double * 3)(1.0, 2.0, 1.0), 1, C.byref(p), 0, C.byref(h))
    assert rc == _capi.FHD_ERR_DX_NOT_ISOTROPIC
    rc = lib.fhd_ctx_create(4, n, (C.c_double * 3)(1.0, 1.0, 1.0), 1, C.byref(p), 0, C.byref(h))
    assert rc == _capi.FHD_ERR_BAD_ARG
    rc = lib.fhd_ctx_create(2, n, (C.c_double * 3)(1.0, 1.0, 1.0), 7, C.byref(p), 0, C.byref(h))
    assert rc == _capi.FHD_ERR_BAD_ARG


def test_no_device_is_an_error_code():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(L.FhdError) as e:
        L.StokesSolver(2, [16, 16], 1.0, 1)
    assert e.value.status == _capi.FHD_ERR_NO_DEVICE


@pytest.mark.parametrize("dim,n,nodal,ng", [(2, [6, 4], [1, 0], 1), (3, [4, 6, 2], [0, 1, 1], 2),
                                            (2, [5, 5], [0, 0], 0)])
def test_fab_roundtrip(dim, n, nodal, ng):
    x = np.arange(int(np.prod(n)), dtype=np.float64)
    fa = L.fab_from_canonical(x, dim, n, nodal, ng)
    ext = [n[d] + nodal[d] + 2 * ng for d in range(dim)]
    assert list(fa.data.shape) == ext
    assert np.array_equal(L.canonical_from_fab(fa, dim, n), x)
    # periodic duplicate plane equals the low plane
    if nodal[0]:
        assert np.array_equal(fa.data[ng + n[0]], fa.data[ng])


def test_layout_context_rejects_walls_and_uneven_boxes_before_device():
    """fhd_ctx_create_bc takes the driver's max_grid_size, bc_lo and bc_hi:
    periodic, no-slip (100) and slip (200) codes, a direction periodic on
    both sides or on neither, walls with one box only, boxes that divide the
    domain; reservoirs (101, 201) are accepted as walls, the closed and
    impermeable codes are not built"""
    lib = _capi.lib()
    h = C.c_void_p()
    p = L.default_params()
    n = (C.c_int * 3)(32, 32, 32)
    dx = (C.c_double * 3)(1.0, 1.0, 1.0)
    per = (C.c_int * 3)(-1, -1, -1)
    wall = (C.c_int * 3)(-1, 100, -1)
    closed = (C.c_int * 3)(-1, 102, -1)
    mgs = (C.c_int * 3)(16, 16, 16)
    one = (C.c_int * 3)(32, 32, 32)
    assert lib.fhd_ctx_create_bc(3, n, one, wall, per, dx, 1, C.byref(p), 0, C.byref(h)) == _capi.FHD_ERR_BAD_ARG
    assert lib.fhd_ctx_create_bc(3, n, one, closed, closed, dx, 1, C.byref(p), 0,
                                 C.byref(h)) == _capi.FHD_ERR_UNSUPPORTED
    assert b"other codes are not" in lib.fhd_last_error()
    assert lib.fhd_ctx_create_bc(3, n, mgs, wall, wall, dx, 1, C.byref(p), 0, C.byref(h)) == _capi.FHD_ERR_UNSUPPORTED
    assert b"one box" in lib.fhd_last_error()
    assert lib.fhd_ctx_create_bc(3, n, one, wall, wall, dx, -1, C.byref(p), 0, C.byref(h)) == _capi.FHD_ERR_UNSUPPORTED
    uneven = (C.c_int * 3)(12, 16, 16)
    assert lib.fhd_ctx_create_bc(3, n, uneven, per, per, dx, 1, C.byref(p), 0, C.byref(h)) == _capi.FHD_ERR_UNSUPPORTED
    zero = (C.c_int * 3)(0, 16, 16)
    assert lib.fhd_ctx_create_bc(3, n, zero, per, per, dx, 1, C.byref(p), 0, C.byref(h)) == _capi.FHD_ERR_BAD_ARG
    assert not h.value
