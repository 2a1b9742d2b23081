"""TEST INFRASTRUCTURE ONLY: ctypes bindings of the CPU FP64 oracle.

The oracle (fhd_oracle.cpp) restates LowMachFHD's staggered Stokes solver and
stochastic momentum flux on the CPU.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg import this module; the product library
never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class GmresParams(C.Structure):
    _fields_ = [
        ("precon_type", C.c_int), ("visc_schur_approx", C.c_int),
        ("p_norm_weight", C.c_double), ("scale_factor", C.c_double),
        ("mg_verbose", C.c_int), ("cg_verbose", C.c_int),
        ("mg_max_vcycles", C.c_int), ("mg_minwidth", C.c_int), ("mg_bottom_solver", C.c_int),
        ("mg_nsmooths_down", C.c_int), ("mg_nsmooths_up", C.c_int), ("mg_nsmooths_bottom", C.c_int),
        ("mg_max_bottom_nlevels", C.c_int),
        ("mg_rel_tol", C.c_double), ("mg_abs_tol", C.c_double),
        ("stag_mg_verbosity", C.c_int), ("stag_mg_max_vcycles", C.c_int), ("stag_mg_minwidth", C.c_int),
        ("stag_mg_bottom_solver", C.c_int),
        ("stag_mg_nsmooths_down", C.c_int), ("stag_mg_nsmooths_up", C.c_int),
        ("stag_mg_nsmooths_bottom", C.c_int), ("stag_mg_max_bottom_nlevels", C.c_int),
        ("stag_mg_omega", C.c_double), ("stag_mg_smoother", C.c_int), ("stag_mg_rel_tol", C.c_double),
        ("gmres_rel_tol", C.c_double), ("gmres_abs_tol", C.c_double),
        ("gmres_verbose", C.c_int), ("gmres_max_outer", C.c_int), ("gmres_max_inner", C.c_int),
        ("gmres_max_iter", C.c_int), ("gmres_min_iter", C.c_int), ("gmres_spatial_order", C.c_int),
    ]


def default_params(**kw) -> GmresParams:
    """Defaults of probin_gmres_init (probin_gmres.f90:122-163)."""
    p = GmresParams(
        precon_type=1, visc_schur_approx=0, p_norm_weight=1.0, scale_factor=1.0,
        mg_verbose=0, cg_verbose=0, mg_max_vcycles=1, mg_minwidth=2, mg_bottom_solver=4,
        mg_nsmooths_down=2, mg_nsmooths_up=2, mg_nsmooths_bottom=8, mg_max_bottom_nlevels=10,
        mg_rel_tol=1e-9, mg_abs_tol=1e-14,
        stag_mg_verbosity=0, stag_mg_max_vcycles=1, stag_mg_minwidth=2, stag_mg_bottom_solver=4,
        stag_mg_nsmooths_down=2, stag_mg_nsmooths_up=2, stag_mg_nsmooths_bottom=8,
        stag_mg_max_bottom_nlevels=10, stag_mg_omega=1.0, stag_mg_smoother=1, stag_mg_rel_tol=1e-9,
        gmres_rel_tol=1e-9, gmres_abs_tol=0.0, gmres_verbose=1, gmres_max_outer=20,
        gmres_max_inner=5, gmres_max_iter=100, gmres_min_iter=1, gmres_spatial_order=2)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class StochParams(C.Structure):
    _fields_ = [("k_B", C.c_double), ("variance_coef_mom", C.c_double), ("dV", C.c_double),
                ("stoch_stress_form", C.c_int), ("filtering_width", C.c_int)]


class MixtureParams(C.Structure):
    """fhd_mixture_params (probin_multispecies.f90:100-140), ideal mixture."""
    _fields_ = [("nspecies", C.c_int), ("molmass", C.c_double * 8), ("Dbar", C.c_double * 28),
                ("rhobar", C.c_double * 8), ("variance_coef_mass", C.c_double), ("chi_iterations", C.c_int),
                ("fraction_tolerance", C.c_double), ("correct_flux", C.c_int), ("avg_type", C.c_int)]


def mixture_params(molmass, Dbar, rhobar=None, variance_coef_mass=1.0, chi_iterations=10,
                   fraction_tolerance=1e-14, correct_flux=1, avg_type=1):
    ns = len(molmass)
    m = MixtureParams()
    m.nspecies = ns
    for i, v in enumerate(molmass):
        m.molmass[i] = v
    assert len(Dbar) == ns * (ns - 1) // 2
    for i, v in enumerate(Dbar):
        m.Dbar[i] = v
    for i, v in enumerate(rhobar if rhobar is not None else [1.0] * ns):
        m.rhobar[i] = v
    m.variance_coef_mass = variance_coef_mass
    m.chi_iterations = chi_iterations
    m.fraction_tolerance = fraction_tolerance
    m.correct_flux = correct_flux
    m.avg_type = avg_type
    return m


class SolveStats(C.Structure):
    _fields_ = [("outer_iters", C.c_int), ("total_iters", C.c_int), ("vcycles", C.c_int),
                ("status", C.c_int),
                ("norm_b", C.c_double), ("norm_pre_b", C.c_double), ("norm_init_resid", C.c_double),
                ("norm_resid", C.c_double), ("norm_resid_Stokes", C.c_double),
                ("norm_init_Stokes", C.c_double), ("norm_resid_est", C.c_double)]


def build() -> str:
    """Compile the oracle with its Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
    return _lib


# ----------------------------------------------------------------------
# array helpers
# ----------------------------------------------------------------------
_DP = C.POINTER(C.c_double)


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def _pp(arrs):
    """array of double* from a list of float64 arrays"""
    arr = (_DP * max(1, len(arrs)))()
    for i, a in enumerate(arrs):
        arr[i] = _p(a)
    return arr


def _n3(n):
    n = list(n) + [1] * (3 - len(n))
    return (C.c_int * 3)(*n)


def nedge(dim):
    return 1 if dim == 2 else 3


class Problem:
    """Grid + coefficients of one Stokes problem (canonical layout; flat
    arrays of nx*ny*nz, x fastest)."""

    def __init__(self, dim, n, dx, visc_type, alpha_fc, beta, beta_ed, gamma):
        self.dim, self.n, self.dx, self.visc_type = dim, list(n), float(dx), visc_type
        self.alpha_fc = [np.ascontiguousarray(a, np.float64) for a in alpha_fc]
        self.beta = np.ascontiguousarray(beta, np.float64)
        self.beta_ed = [np.ascontiguousarray(a, np.float64) for a in beta_ed]
        self.gamma = np.ascontiguousarray(gamma, np.float64)

    @property
    def nc(self):
        return int(np.prod(self.n[: self.dim]))


def stag_applyop(pb: Problem, phi, color=0, theta=1.0):
    Lphi = [np.zeros(pb.nc) for _ in range(pb.dim)]
    alpha = [a * theta for a in pb.alpha_fc]
    lib().or_stag_applyop(pb.dim, _n3(pb.n), C.c_double(pb.dx), pb.visc_type, _pp(phi), _pp(Lphi),
                          _pp(alpha), _p(pb.beta), _pp(pb.beta_ed), _p(pb.gamma), color)
    return Lphi


def stag_mg_solver(pb: Problem, params, theta, rhs, phi0=None):
    phi = [np.zeros(pb.nc) if phi0 is None else phi0[d].copy() for d in range(pb.dim)]
    rc = lib().or_stag_mg_solver(pb.dim, _n3(pb.n), C.c_double(pb.dx), pb.visc_type, C.byref(params),
                                 _pp(pb.alpha_fc), _p(pb.beta), _pp(pb.beta_ed), _p(pb.gamma),
                                 C.c_double(theta), _pp(phi), _pp(rhs))
    assert rc == 0, rc
    return phi


def macproject(dim, n, dx, params, alphainv, rhs):
    phi = np.zeros(int(np.prod(n[:dim])))
    lib().or_macproject(dim, _n3(n), C.c_double(dx), C.byref(params), _p(phi), _pp(alphainv), _p(rhs))
    return phi


def macproject_history(dim, n, dx, params, alphainv, rhs):
    """per-V-cycle L2 residual ratios of the pressure multigrid from a zero
    guess (mg_max_vcycles cycles, no stopping test)"""
    phi = np.zeros(int(np.prod(n[:dim])))
    hist = np.zeros(params.mg_max_vcycles)
    rc = lib().or_macproject_history(dim, _n3(n), C.c_double(dx), C.byref(params), _p(phi), _pp(alphainv), _p(rhs),
                                     _p(hist))
    assert rc == 0
    return hist


def apply_matrix(pb: Problem, theta, x_u, x_p, order=2):
    """apply_matrix.f90:24-157; order = gmres_spatial_order (2, or 4 with
    visc_type 1)"""
    b_u = [np.zeros(pb.nc) for _ in range(pb.dim)]
    b_p = np.zeros(pb.nc)
    rc = lib().or_apply_matrix_order(pb.dim, _n3(pb.n), C.c_double(pb.dx), pb.visc_type, _pp(b_u), _p(b_p),
                                     _pp(x_u), _p(x_p), _pp(pb.alpha_fc), _p(pb.beta), _pp(pb.beta_ed),
                                     _p(pb.gamma), C.c_double(theta), int(order))
    assert rc == 0, rc
    return b_u, b_p


def apply_precon(pb: Problem, params, theta, b_u, b_p):
    x_u = [np.zeros(pb.nc) for _ in range(pb.dim)]
    x_p = np.zeros(pb.nc)
    rc = lib().or_apply_precon(pb.dim, _n3(pb.n), C.c_double(pb.dx), pb.visc_type, C.byref(params),
                               _pp(b_u), _p(b_p), _pp(x_u), _p(x_p), _pp(pb.alpha_fc), _p(pb.beta),
                               _pp(pb.beta_ed), _p(pb.gamma), C.c_double(theta))
    assert rc == 0, rc
    return x_u, x_p


def gmres(pb: Problem, params, theta, b_u, b_p, x_u0=None, x_p0=None):
    x_u = [np.zeros(pb.nc) if x_u0 is None else x_u0[d].copy() for d in range(pb.dim)]
    x_p = np.zeros(pb.nc) if x_p0 is None else x_p0.copy()
    npr = C.c_double(0.0)
    st = SolveStats()
    rc = lib().or_gmres(pb.dim, _n3(pb.n), C.c_double(pb.dx), pb.visc_type, C.byref(params),
                        _pp(b_u), _p(b_p), _pp(x_u), _p(x_p), _pp(pb.alpha_fc), _p(pb.beta),
                        _pp(pb.beta_ed), _p(pb.gamma), C.c_double(theta), C.byref(npr), C.byref(st))
    return rc, x_u, x_p, npr.value, st


def stochastic_m_fluxdiv(dim, n, dx, sp, eta, eta_ed, temp, temp_ed, dt, weights, W_cc, W_ed,
                         force=None, increment=False, status=False):
    """the divergence on the faces; with status=True the pair (status,
    force) instead of asserting status 0"""
    nc = int(np.prod(n[:dim]))
    force = [np.zeros(nc) for _ in range(dim)] if force is None else [f.copy() for f in force]
    w = np.ascontiguousarray(weights, np.float64)
    rc = lib().or_stochastic_m_fluxdiv(dim, _n3(n), C.c_double(dx), C.byref(sp), _pp(force),
                                       int(increment), _p(eta), _pp(eta_ed), _p(temp), _pp(temp_ed),
                                       C.c_double(dt), _p(w), len(weights), _pp(W_cc), _pp(W_ed))
    if status:
        return rc, force
    assert rc == 0, rc
    return force


def average_cc_to_edge(dim, n, cc):
    nc = int(np.prod(n[:dim]))
    ed = [np.zeros(nc) for _ in range(nedge(dim))]
    lib().or_average_cc_to_edge(dim, _n3(n), _p(cc), _pp(ed))
    return ed


def average_cc_to_face(dim, n, cc):
    nc = int(np.prod(n[:dim]))
    fc = [np.zeros(nc) for _ in range(dim)]
    lib().or_average_cc_to_face(dim, _n3(n), _p(cc), _pp(fc))
    return fc


def advance_inertial(dim, n, dx, visc_type, params, sp, dt, umac, rho, pi, eta, eta_ed, kappa,
                     temp, temp_ed, W_cc, W_ed):
    umac = [u.copy() for u in umac]
    rho, pi = rho.copy(), pi.copy()
    st = (SolveStats * 2)()
    rc = lib().or_advance_inertial(dim, _n3(n), C.c_double(dx), visc_type, C.byref(params), C.byref(sp),
                                   C.c_double(dt), _pp(umac), _p(rho), _p(pi), _p(eta), _pp(eta_ed),
                                   _p(kappa), _p(temp), _pp(temp_ed), _pp(W_cc), _pp(W_ed), st)
    return rc, umac, rho, pi, st


def accuracy_test(dim, n, prob_coeff, prob_sol, visc_type, order=2):
    err = np.zeros(4)
    rc = lib().or_accuracy_test_order(dim, n, prob_coeff, prob_sol, visc_type, int(order), _p(err))
    assert rc == 0
    return err[: dim + 1]


PERIODIC, NO_SLIP_WALL, SLIP_WALL = -1, 100, 200


def set_walls(bc_lo=(PERIODIC,) * 3, bc_hi=(PERIODIC,) * 3):
    """boundary codes of the grids later calls build (bc.f90 codes)"""
    lo = (C.c_int * 3)(*[int(b) for b in bc_lo])
    hi = (C.c_int * 3)(*[int(b) for b in bc_hi])
    rc = lib().or_set_walls(lo, hi)
    assert rc == 0, rc


def set_wall_speed(lo=None, hi=None):
    """wallspeed_lo / wallspeed_hi (probin_common) for the steps: six values
    each, speed (t, d) of the t-th tangential component on the wall normal
    to d at [t + 2 d]; None is all zero"""
    a = (C.c_double * 6)(*([0.0] * 6 if lo is None else [float(x) for x in lo]))
    b = (C.c_double * 6)(*([0.0] * 6 if hi is None else [float(x) for x in hi]))
    lib().or_set_wall_speed(a, b)


def compute_nlevs_mg(dim, n, minwidth=2):
    return lib().or_compute_nlevs_mg(dim, _n3(n), minwidth)


def num_threads():
    return lib().or_num_threads()


def stag_mg_history(pb: Problem, params, theta, rhs):
    """per-V-cycle L2 residual ratios of stag_mg_solver from a zero guess"""
    phi = [np.zeros(pb.nc) for _ in range(pb.dim)]
    hist = np.zeros(params.stag_mg_max_vcycles)
    rc = lib().or_stag_mg_history(pb.dim, _n3(pb.n), C.c_double(pb.dx), pb.visc_type, C.byref(params),
                                  _pp(pb.alpha_fc), _p(pb.beta), _pp(pb.beta_ed), _p(pb.gamma),
                                  C.c_double(theta), _pp(phi), _pp(rhs), _p(hist))
    assert rc == 0
    return hist


def mass_fluxdiv(dim, n, dx, sp, mp, rho, dt, weights, W_fc, want_flux=False):
    nc = int(np.prod(n[:dim]))
    ns = mp.nspecies
    out = [np.zeros(nc) for _ in range(ns)]
    flux = [np.zeros(nc) for _ in range(dim * ns)] if want_flux else None
    w = np.ascontiguousarray(weights, np.float64)
    rc = lib().or_mass_fluxdiv(dim, _n3(n), C.c_double(dx), C.byref(sp), C.byref(mp), _pp(rho), C.c_double(dt),
                               _p(w), len(weights), _pp(W_fc), _pp(out), _pp(flux) if want_flux else None)
    assert rc == 0, rc
    return (out, flux) if want_flux else out


def advance_overdamped(dim, n, dx, visc_type, params, sp, mp, dt, umac, rho, pi, eta, eta_ed, kappa, temp,
                       temp_ed, W_cc, W_ed, W_mass=None):
    """advance_timestep_overdamped (advance_timestep_overdamped.f90:135-734).
    rho: list of species arrays (one array and mp=None for a single fluid).
    W_cc: 2*dim cell fields, W_ed: 2*2*nE node/edge fields, W_mass:
    2*dim*ns face fields (two random stages)."""
    umac = [u.copy() for u in umac]
    rho = [r.copy() for r in rho]
    pi = pi.copy()
    st = (SolveStats * 2)()
    rc = lib().or_advance_overdamped(dim, _n3(n), C.c_double(dx), visc_type, C.byref(params), C.byref(sp),
                                     C.byref(mp) if mp is not None else None, C.c_double(dt), _pp(umac), _pp(rho),
                                     _p(pi), _p(eta), _pp(eta_ed), _p(kappa), _p(temp), _pp(temp_ed), _pp(W_cc),
                                     _pp(W_ed), _pp(W_mass) if W_mass is not None else None, st)
    return rc, umac, rho, pi, st


def advance_inertial_ms(dim, n, dx, visc_type, params, sp, mp, dt, umac, rho, pi, fluxdiv, eta, eta_ed, kappa,
                        temp, temp_ed, W_cc, W_ed, W_mass):
    umac = [u.copy() for u in umac]
    rho = [r.copy() for r in rho]
    fluxdiv = [f.copy() for f in fluxdiv]
    pi = pi.copy()
    st = (SolveStats * 2)()
    rc = lib().or_advance_inertial_ms(dim, _n3(n), C.c_double(dx), visc_type, C.byref(params), C.byref(sp),
                                      C.byref(mp), C.c_double(dt), _pp(umac), _pp(rho), _p(pi), _pp(fluxdiv),
                                      _p(eta), _pp(eta_ed), _p(kappa), _p(temp), _pp(temp_ed), _pp(W_cc),
                                      _pp(W_ed), _pp(W_mass), st)
    return rc, umac, rho, pi, fluxdiv, st


def mixture_local(mp, k_B, rho):
    ns = mp.nspecies
    chi = np.zeros(ns * ns)
    L = np.zeros(ns * ns)
    rc = lib().or_mixture_local(C.byref(mp), C.c_double(k_B), _p(np.ascontiguousarray(rho, np.float64)), _p(chi),
                                _p(L))
    return rc, chi.reshape(ns, ns), L.reshape(ns, ns)


def mixture_trace_local(mp, k_B, rho):
    """rho W chi and the Cholesky factor of the Onsager matrix at one state
    (compute_rhoWchi_local, compute_sqrtLonsager_local), trace species
    included"""
    ns = mp.nspecies
    a = np.zeros(ns * ns)
    L = np.zeros(ns * ns)
    lib().or_mixture_trace_local(C.byref(mp), C.c_double(k_B), _p(np.ascontiguousarray(rho, np.float64)), _p(a),
                                 _p(L))
    return a.reshape(ns, ns), L.reshape(ns, ns)


def sqrtLonsager_fc(dim, n, sp, mp, rho):
    """compute_sqrtLonsager_fc: list of dim*ns*ns face arrays, entry (r, c)
    of direction d at index d*ns*ns + r + ns*c"""
    ns = mp.nspecies
    nc = int(np.prod(list(n)[:dim]))
    out = [np.zeros(nc) for _ in range(dim * ns * ns)]
    lib().or_sqrtLonsager_fc(dim, _n3(n), C.byref(sp), C.byref(mp), _pp(rho), _pp(out))
    return out


def stochastic_mass_fluxdiv(dim, n, dx, sp, mp, sqrtL, dt, weights, W_fc, increment=False, div0=None,
                            want_flux=False):
    """stochastic_mass_fluxdiv with given face factors: (div, flux|None)"""
    ns = mp.nspecies
    nc = int(np.prod(list(n)[:dim]))
    div = [np.array(d, dtype=np.float64) for d in div0] if div0 is not None else [np.zeros(nc) for _ in range(ns)]
    flux = [np.zeros(nc) for _ in range(dim * ns)] if want_flux else None
    w = (C.c_double * len(weights))(*weights)
    lib().or_stochastic_mass_fluxdiv(dim, _n3(n), C.c_double(dx), C.byref(sp), C.byref(mp), _pp(sqrtL),
                                     C.c_double(dt), C.cast(w, _DP), len(weights), _pp(W_fc), int(bool(increment)),
                                     _pp(div), _pp(flux) if flux is not None else None)
    return div, flux


def set_max_grid_size(mgs=None):
    """probin_common max_grid_size of the staggered multigrid's box layout
    (module state of the oracle); None: one box"""
    a = (C.c_int * 3)(*((list(mgs) + [0] * 3)[:3] if mgs else [0, 0, 0]))
    lib().or_set_max_grid_size(a)
