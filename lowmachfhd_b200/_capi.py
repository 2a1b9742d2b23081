"""ctypes declarations of the C ABI in include/fhd_b200.h.

The product path: every call goes to the sm_100a library _fhd_b200.so built
in this directory.  There is no fallback; a missing library raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_fhd_b200.so")
HEADER = os.path.join(HERE, "..", "include", "fhd_b200.h")

FHD_OK = 0
FHD_WARN_NOT_CONVERGED_MAXITER = 1
FHD_WARN_NOT_CONVERGED_OUTER = 2
FHD_WARN_TRUE_RESID = 3
FHD_ERR_BAD_ARG = -1
FHD_ERR_BAD_GHOSTS = -2
FHD_ERR_DX_NOT_ISOTROPIC = -3
FHD_ERR_ORTHO_BREAKDOWN = -4
FHD_ERR_UNSUPPORTED = -5
FHD_ERR_NONFINITE = -6
FHD_ERR_OOM = -7
FHD_ERR_CUDA = -8
FHD_ERR_NO_DEVICE = -9

FHD_PREC_FP64 = 0
FHD_PREC_MIXED = 1

# boundary codes of fhd_ctx_create_bc (bc.f90:24-44)
FHD_BC_PERIODIC = -1
FHD_BC_NO_SLIP_WALL = 100
FHD_BC_SLIP_WALL = 200
FHD_BC_NO_SLIP_RESERVOIR = 101
FHD_BC_SLIP_RESERVOIR = 201


class GmresParams(C.Structure):
    """fhd_gmres_params: mirror of namelist probin_gmres (probin_gmres.f90:12-163)."""
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


class StochParams(C.Structure):
    """fhd_stoch_params (stochastic_m_fluxdiv.f90:137)."""
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


FHD_REQ_OVERDAMPED = 0
FHD_REQ_INERTIAL = 1


class Request(C.Structure):
    """fhd_request: one served problem (include/fhd_b200.h)."""
    _fields_ = [("kind", C.c_int), ("dim", C.c_int), ("n_cells", C.c_int * 3), ("dx", C.c_double),
                ("cell_depth", C.c_double), ("visc_type", C.c_int), ("precision", C.c_int), ("nspecies", C.c_int),
                ("mix", MixtureParams), ("rho0", C.c_double), ("eta", C.c_double), ("kT", C.c_double),
                ("dt", C.c_double), ("steps", C.c_int), ("seed", C.c_ulonglong), ("params", GmresParams),
                ("out_umac", C.POINTER(C.c_double)), ("out_rho", C.POINTER(C.c_double))]


class RequestResult(C.Structure):
    _fields_ = [("id", C.c_longlong), ("status", C.c_int), ("gmres_iters", C.c_int), ("launches", C.c_longlong),
                ("t_submit", C.c_double), ("t_start", C.c_double), ("t_end", C.c_double), ("u_sumsq", C.c_double),
                ("bytes", C.c_ulonglong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SolveStats(C.Structure):
    _fields_ = [("outer_iters", C.c_int), ("total_iters", C.c_int), ("vcycles", C.c_int),
                ("status", C.c_int),
                ("norm_b", C.c_double), ("norm_pre_b", C.c_double), ("norm_init_resid", C.c_double),
                ("norm_resid", C.c_double), ("norm_resid_Stokes", C.c_double),
                ("norm_init_Stokes", C.c_double), ("norm_resid_est", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Fab(C.Structure):
    """fhd_fab: one Fortran column-major box (lo-ng : hi+nodal+ng, ..., ncomp)."""
    _fields_ = [("data", C.POINTER(C.c_double)), ("lo", C.c_int * 3), ("hi", C.c_int * 3),
                ("nodal", C.c_int * 3), ("ng", C.c_int), ("ncomp", C.c_int)]


class Multifab(C.Structure):
    _fields_ = [("nfabs", C.c_int), ("fabs", C.POINTER(Fab))]


_DP = C.POINTER(C.c_double)
_PP = C.POINTER(_DP)
_VP = C.c_void_p

_PROTOS = {
    "fhd_gmres_params_default": (None, [C.POINTER(GmresParams)]),
    "fhd_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int,
                                 C.POINTER(GmresParams), C.c_int, C.POINTER(_VP)]),
    "fhd_ctx_create_bc": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int, C.POINTER(GmresParams),
                                    C.c_int, C.POINTER(_VP)]),
    "fhd_ctx_destroy": (C.c_int, [_VP]),
    "fhd_batch_create": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.c_double, C.POINTER(GmresParams), C.c_int,
                                   C.POINTER(_VP)]),
    "fhd_batch_destroy": (C.c_int, [_VP]),
    "fhd_batch_box_offset": (C.c_longlong, [_VP, C.c_int]),
    "fhd_batch_kernel_launches": (C.c_longlong, [_VP]),
    "fhd_batch_gmres": (C.c_int, [_VP, _PP, _PP, _DP, C.c_double, C.POINTER(SolveStats)]),
    "fhd_batch_overdamped": (C.c_int, [_VP, _PP, _DP, _DP, _DP, C.c_double, C.c_int, C.c_ulonglong, C.c_int,
                                       C.POINTER(C.c_int)]),
    "fhd_ctx_stream": (_VP, [_VP]),
    "fhd_ctx_set_stream": (C.c_int, [_VP, _VP]),
    "fhd_ctx_kernel_launches": (C.c_longlong, [_VP]),
    "fhd_ctx_set_graphs": (C.c_int, [_VP, C.c_int]),
    "fhd_ctx_set_coarse": (C.c_int, [_VP, C.c_int]),
    "fhd_ctx_set_fused": (C.c_int, [_VP, C.c_int]),
    "fhd_ctx_set_tune": (C.c_int, [_VP, C.c_int]),
    "fhd_ctx_set_wall_speed": (C.c_int, [_VP, _DP, _DP]),
    "fhd_tune_export": (C.c_longlong, [C.c_char_p, C.c_longlong]),
    "fhd_tune_import": (C.c_int, [C.c_char_p]),
    "fhd_tune_key": (C.c_longlong, [C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_int, C.c_char_p, C.c_longlong]),
    "fhd_tune_candidates": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.POINTER(C.c_int), C.c_int]),
    "fhd_sk_create": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.c_double, C.c_int, C.POINTER(C.c_int), C.c_int,
                                C.POINTER(C.c_int), C.POINTER(_VP)]),
    "fhd_sk_update": (C.c_int, [_VP, C.POINTER(C.POINTER(C.c_double)), _VP]),
    "fhd_sk_read": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                              C.POINTER(C.c_longlong)]),
    "fhd_sk_modes": (C.c_longlong, [_VP]),
    "fhd_sk_destroy": (C.c_int, [_VP]),
    "fhd_ctx_tune_info": (C.c_int, [_VP, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "fhd_ctx_device_bytes": (C.c_ulonglong, [_VP]),
    "fhd_ctx_profile": (C.c_int, [_VP, C.c_int]),
    "fhd_ctx_profile_read": (C.c_int, [_VP, C.POINTER(C.c_longlong), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double)]),
    "fhd_status_string": (C.c_char_p, [C.c_int]),
    "fhd_last_error": (C.c_char_p, []),
    "fhd_dev_apply_matrix": (C.c_int, [_VP, _PP, _DP, _PP, _DP, _PP, _DP, _PP, _DP, C.c_double]),
    "fhd_dev_apply_precon": (C.c_int, [_VP, _PP, _DP, _PP, _DP, _PP, _DP, _PP, _DP, C.c_double]),
    "fhd_dev_stag_mg_solver": (C.c_int, [_VP, _PP, _DP, _PP, _DP, C.c_double, _PP, _PP]),
    "fhd_dev_gmres": (C.c_int, [_VP, _PP, _DP, _PP, _DP, _PP, _DP, _PP, _DP, C.c_double, _DP,
                                C.POINTER(SolveStats)]),
    "fhd_dev_stochastic_m_fluxdiv": (C.c_int, [_VP, C.POINTER(StochParams), _PP, C.c_int, _DP, _PP, _DP, _PP,
                                               C.c_double, _DP, C.c_int, _PP, _PP]),
    "fhd_dev_advance_inertial": (C.c_int, [_VP, C.POINTER(StochParams), C.c_double, _PP, _DP, _DP, _DP, _PP,
                                           _DP, _DP, _PP, _PP, _PP, C.POINTER(SolveStats)]),
    "fhd_dev_stag_mg_solver_noalloc": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.c_double, C.c_int,
                                                 C.POINTER(GmresParams), _PP, _DP, _PP, _DP, C.c_double, _PP,
                                                 _PP, _VP]),
    "fhd_dev_compute_mass_fluxdiv": (C.c_int, [_VP, C.POINTER(MixtureParams), C.POINTER(StochParams), _PP,
                                               C.c_double, _DP, C.c_int, _PP, _PP]),
    "fhd_dev_advance_inertial_multispecies": (C.c_int, [_VP, C.POINTER(StochParams), C.POINTER(MixtureParams),
                                                        C.c_double, _PP, _PP, _DP, _PP, _DP, _PP, _DP, _DP, _PP,
                                                        _PP, _PP, _PP, C.POINTER(SolveStats)]),
    "fhd_dev_advance_overdamped": (C.c_int, [_VP, C.POINTER(StochParams), C.POINTER(MixtureParams), C.c_double,
                                             _PP, _PP, _DP, _DP, _PP, _DP, _DP, _PP, _PP, _PP, _PP,
                                             C.POINTER(SolveStats)]),
    "fhd_dev_fill_normal": (C.c_int, [_VP, C.c_longlong, C.c_ulonglong, C.c_uint, C.c_uint, C.c_uint, C.c_double,
                                      _VP]),
    "fhd_philox4x32_10": (None, [C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.POINTER(C.c_uint)]),
    "fhd_request_default": (None, [C.POINTER(Request)]),
    "fhd_request_bytes": (C.c_ulonglong, [C.POINTER(Request)]),
    "fhd_server_create": (C.c_int, [C.c_int, C.c_ulonglong, C.POINTER(_VP)]),
    "fhd_server_submit": (C.c_int, [_VP, C.POINTER(Request), C.POINTER(C.c_longlong)]),
    "fhd_server_wait": (C.c_int, [_VP, C.c_longlong, C.POINTER(RequestResult)]),
    "fhd_server_clock": (C.c_double, [_VP]),
    "fhd_server_destroy": (C.c_int, [_VP]),
    "fhd_sched_simulate": (C.c_int, [C.c_int, C.c_ulonglong, C.c_int, _DP, C.POINTER(C.c_ulonglong), _DP, _DP]),
    "fhd_dev_compute_sqrtLonsager_fc": (C.c_int, [_VP, C.POINTER(MixtureParams), C.POINTER(StochParams), _PP, _PP]),
    "fhd_dev_stochastic_mass_fluxdiv": (C.c_int, [_VP, C.POINTER(MixtureParams), C.POINTER(StochParams), _PP,
                                                  C.c_double, _DP, C.c_int, _PP, C.c_int, _PP, _PP]),
    "fhd_stag_mg_solve": (C.c_int, [_VP] + [C.POINTER(Multifab)] * 4 + [C.c_double] + [C.POINTER(Multifab)] * 2),
    "fhd_compute_sqrtLonsager_fc": (C.c_int, [_VP, C.POINTER(MixtureParams), C.POINTER(StochParams)]
                                    + [C.POINTER(Multifab)] * 3),
    "fhd_stochastic_mass_fluxdiv": (C.c_int, [_VP, C.POINTER(MixtureParams), C.POINTER(StochParams)]
                                    + [C.POINTER(Multifab)] * 5 + [C.c_double, _DP, C.c_int, C.POINTER(Multifab),
                                                                   C.c_int]),
    "fhd_gmres": (C.c_int, [_VP] + [C.POINTER(Multifab)] * 8 + [_DP, _DP, C.POINTER(SolveStats)]),
    "fhd_apply_precon": (C.c_int, [_VP] + [C.POINTER(Multifab)] * 8 + [C.c_double]),
    "fhd_apply_matrix": (C.c_int, [_VP] + [C.POINTER(Multifab)] * 8 + [C.c_double]),
    "fhd_stochastic_m_fluxdiv": (C.c_int, [_VP, C.POINTER(StochParams), C.POINTER(Multifab), C.c_int,
                                           C.POINTER(Multifab), C.POINTER(Multifab), C.POINTER(Multifab),
                                           C.POINTER(Multifab), C.c_double, _DP, C.c_int, C.POINTER(Multifab),
                                           C.POINTER(Multifab)]),
}

_lib = None


def header_functions(path: str = HEADER) -> list[str]:
    """Names of the functions include/fhd_b200.h declares."""
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(fhd_[a-z0-9_]+)\s*\(", src)
    out = []
    for n in names:
        if n not in out:
            out.append(n)
    return out


def lib() -> C.CDLL:
    """Load the sm_100a library; raise if it was never built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"lowmachfhd_b200: {LIB_PATH} is missing -- run lowmachfhd_b200/build.py "
                          "(nvcc, sm_100a); there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class FhdError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib().fhd_status_string(status).decode()
        # the library's own message names the site that failed
        detail = (lib().fhd_last_error() or b"").decode(errors="replace")
        super().__init__(f"{where}: status {status}: {msg}" + (f" ({detail})" if detail else ""))
        self.status = status
        self.detail = detail


def check(status: int, where: str) -> int:
    if status < 0:
        raise FhdError(status, where)
    return status
