"""lowmachfhd_b200 -- B200 (sm_100a) implementation of LowMachFHD's implicit
staggered-grid Stokes solve and stochastic momentum flux.

Python mirror of the reference interface (staggered_grid/src_gmres and
src_lowMach of LowMachFHD): the same routine names and argument meaning as
gmres, apply_precon, apply_matrix, stag_mg_solver, stochastic_m_fluxdiv and
advance_timestep_inertial.  Every call goes through the C ABI of the CUDA
library (include/fhd_b200.h); torch tensors serve only as device memory.

Device arrays are flat float64 CUDA tensors in the canonical periodic layout
(x fastest; face arrays hold the low face of each cell; see the header).
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _capi
from ._capi import (FHD_BC_NO_SLIP_RESERVOIR, FHD_BC_NO_SLIP_WALL, FHD_BC_PERIODIC, FHD_BC_SLIP_RESERVOIR, FHD_BC_SLIP_WALL, FHD_PREC_FP64, FHD_PREC_MIXED, FHD_REQ_INERTIAL, FHD_REQ_OVERDAMPED, Fab, FhdError,
                    GmresParams, MixtureParams, Multifab, Request, RequestResult, SolveStats, StochParams, check, lib,
                    mixture_params)

__all__ = ["StokesSolver", "GmresParams", "StochParams", "SolveStats", "MixtureParams", "mixture_params",
           "Server", "Batch", "StructureFactor", "tune_candidates", "tune_export", "tune_import", "tune_key", "Request", "RequestResult", "make_request", "fill_normal", "StepNoise", "philox4x32_10", "sched_simulate",
           "FHD_REQ_OVERDAMPED", "FHD_REQ_INERTIAL",
           "default_params", "FhdError",
           "FHD_PREC_FP64", "FHD_PREC_MIXED", "FHD_BC_PERIODIC", "FHD_BC_NO_SLIP_WALL", "FHD_BC_SLIP_WALL", "FHD_BC_NO_SLIP_RESERVOIR", "FHD_BC_SLIP_RESERVOIR", "lib", "fab_from_canonical", "fab_from_components", "canonical_from_fab", "FabArray"]


def default_params(**overrides) -> GmresParams:
    """probin_gmres defaults (probin_gmres.f90:122-163) with overrides."""
    p = GmresParams()
    lib().fhd_gmres_params_default(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(f"probin_gmres has no parameter {k}")
        setattr(p, k, v)
    return p


_DP = C.POINTER(C.c_double)


def _dptr(t) -> _DP:
    """device pointer of a contiguous float64 CUDA tensor"""
    if t is None:
        return None
    if not (t.is_cuda and t.dtype.itemsize == 8 and t.is_contiguous()):
        raise TypeError("expected a contiguous float64 CUDA tensor")
    return C.cast(C.c_void_p(t.data_ptr()), _DP)


def _dpp(ts: Sequence) -> C.Array:
    arr = (_DP * max(1, len(ts)))()
    for i, t in enumerate(ts):
        arr[i] = _dptr(t)
    return arr


class StokesSolver:
    """One periodic box and its solver state (the fhd_ctx of the C ABI):
    multigrid hierarchies (stag_mg_layout_build, mgt_macproj_precon_build),
    Krylov storage and a CUDA stream."""

    def __init__(self, dim: int, n_cells: Sequence[int], dx: float | Sequence[float], visc_type: int,
                 params: GmresParams | None = None, precision: str = "fp64", max_grid_size=None, bc_lo=None,
                 bc_hi=None):
        self.dim = int(dim)
        n = list(n_cells) + [1] * (3 - len(n_cells))
        self.n_cells = n[:3]
        dxs = [float(dx)] * 3 if np.isscalar(dx) else list(dx) + [float(dx[0])] * (3 - len(dx))
        self.dx = dxs[0]
        self.visc_type = int(visc_type)
        self.params = params if params is not None else default_params()
        self.precision = precision
        mode = FHD_PREC_MIXED if precision == "mixed" else FHD_PREC_FP64
        h = C.c_void_p()
        if max_grid_size is None and bc_lo is None and bc_hi is None:
            st = lib().fhd_ctx_create(self.dim, (C.c_int * 3)(*self.n_cells), (C.c_double * 3)(*dxs),
                                      self.visc_type, C.byref(self.params), mode, C.byref(h))
            check(st, "fhd_ctx_create")
        else:
            # the driver's layout: max_grid_size and the BoxLib boundary codes
            # (-1 periodic), as fhd_ctx_create_bc takes them
            i3 = lambda v, dflt: (C.c_int * 3)(*((list(v) if v is not None else [dflt] * 3) + [dflt] * 3)[:3])
            st = lib().fhd_ctx_create_bc(self.dim, (C.c_int * 3)(*self.n_cells), i3(max_grid_size, 1 << 30),
                                         i3(bc_lo, -1), i3(bc_hi, -1), (C.c_double * 3)(*dxs), self.visc_type,
                                         C.byref(self.params), mode, C.byref(h))
            check(st, "fhd_ctx_create_bc")
        self._h = h

    # ----------------------------------------------------------------
    @property
    def nc(self) -> int:
        return int(np.prod(self.n_cells[: self.dim]))

    @property
    def nedge(self) -> int:
        return 1 if self.dim == 2 else 3

    @property
    def kernel_launches(self) -> int:
        return int(lib().fhd_ctx_kernel_launches(self._h))

    @property
    def device_bytes(self) -> int:
        return int(lib().fhd_ctx_device_bytes(self._h))

    @property
    def stream(self) -> int:
        return int(lib().fhd_ctx_stream(self._h) or 0)

    def set_stream(self, stream_handle: int | None):
        check(lib().fhd_ctx_set_stream(self._h, C.c_void_p(stream_handle or 0)), "fhd_ctx_set_stream")

    def set_graphs(self, mode: int):
        """preconditioner applications inside GMRES as CUDA graphs: 1 on,
        0 off, -1 default"""
        check(lib().fhd_ctx_set_graphs(self._h, int(mode)), "fhd_ctx_set_graphs")

    def set_coarse(self, mode: int):
        """coarse multigrid levels in one single-block kernel per V-cycle: 1
        or -1 (default) on, 0 one launch per smoother colour and transfer"""
        check(lib().fhd_ctx_set_coarse(self._h, int(mode)), "fhd_ctx_set_coarse")

    def set_fused(self, mode: int):
        """whole smooths of the large FP32 levels as one bulk-copy-staged
        launch each: 1 or -1 (default) on, 0 one launch per colour"""
        check(lib().fhd_ctx_set_fused(self._h, int(mode)), "fhd_ctx_set_fused")

    def set_wall_speed(self, wallspeed_lo=None, wallspeed_hi=None):
        """moving no-slip walls for the timesteps: wallspeed_lo / wallspeed_hi
        of probin_common, six values each in the Fortran layout (speed of the
        t-th tangential component on the wall normal to d at [t + 2 d]);
        None is all zero (standing walls)"""
        a = (C.c_double * 6)(*([0.0] * 6 if wallspeed_lo is None else [float(x) for x in wallspeed_lo]))
        b = (C.c_double * 6)(*([0.0] * 6 if wallspeed_hi is None else [float(x) for x in wallspeed_hi]))
        check(lib().fhd_ctx_set_wall_speed(self._h, C.cast(a, _DP), C.cast(b, _DP)), "fhd_ctx_set_wall_speed")

    def set_tune(self, mode: int):
        """smoother autotuner: 1 or -1 (default) time the candidate plans of
        each level shape once per process and keep the fastest, 0 the fixed
        size rules, 2 + k force candidate k of every level (tests)"""
        check(lib().fhd_ctx_set_tune(self._h, int(mode)), "fhd_ctx_set_tune")

    def tune_info(self, which: str = "stag", level: int = 0) -> dict:
        """plan of one level after the last solve call: kind (-1 fixed rules,
        0 colour launches, 1 tiled fused, 2 row-tile), candidates considered,
        measured time of a smooth pair, block or tile shape"""
        kind, nc, us = C.c_int(0), C.c_int(0), C.c_double(0)
        shape = (C.c_int * 5)()
        check(lib().fhd_ctx_tune_info(self._h, 0 if which == "stag" else 1, int(level), C.byref(kind),
                                      C.byref(nc), C.byref(us), shape), "fhd_ctx_tune_info")
        names = {-1: "rules", 0: "colour", 1: "tiled", 2: "rowtile"}
        return {"kind": names[kind.value], "candidates": nc.value, "pair_us": us.value, "shape": list(shape)}

    def profile(self, enable: bool = True):
        """time the finest-level smoother launches with CUDA events"""
        check(lib().fhd_ctx_profile(self._h, int(enable)), "fhd_ctx_profile")

    def profile_read(self):
        """(launches, device ms, algorithmic bytes) since profile(True)"""
        n, ms, b = C.c_longlong(0), C.c_double(0), C.c_double(0)
        check(lib().fhd_ctx_profile_read(self._h, C.byref(n), C.byref(ms), C.byref(b)), "fhd_ctx_profile_read")
        return n.value, ms.value, b.value

    def close(self):
        if getattr(self, "_h", None):
            lib().fhd_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ----------------------------------------------------------------
    # device-pointer mirror of the reference routines
    # ----------------------------------------------------------------
    def apply_matrix(self, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha):
        """apply_matrix (apply_matrix.f90:24-157): b = A x."""
        return check(lib().fhd_dev_apply_matrix(self._h, _dpp(b_u), _dptr(b_p), _dpp(x_u), _dptr(x_p),
                                                _dpp(alpha_fc), _dptr(beta), _dpp(beta_ed), _dptr(gamma),
                                                float(theta_alpha)), "apply_matrix")

    def apply_precon(self, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha):
        """apply_precon (apply_precon.f90:29-475): x = M^{-1} b."""
        return check(lib().fhd_dev_apply_precon(self._h, _dpp(b_u), _dptr(b_p), _dpp(x_u), _dptr(x_p),
                                                _dpp(alpha_fc), _dptr(beta), _dpp(beta_ed), _dptr(gamma),
                                                float(theta_alpha)), "apply_precon")

    def stag_mg_solver(self, alpha_fc, beta_cc, beta_ed, gamma_cc, theta_alpha, phi_fc, rhs_fc):
        """stag_mg_solver (stag_mg_solver.f90:37-863); phi_fc in/out."""
        return check(lib().fhd_dev_stag_mg_solver(self._h, _dpp(alpha_fc), _dptr(beta_cc), _dpp(beta_ed),
                                                  _dptr(gamma_cc), float(theta_alpha), _dpp(phi_fc),
                                                  _dpp(rhs_fc)), "stag_mg_solver")

    def gmres(self, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha):
        """gmres (gmres.f90:32-491).  x_u/x_p: initial guess in, solution
        out.  Returns (status, norm_pre_rhs, stats dict); status > 0 is a
        non-convergence warning as printed by the reference."""
        npr = C.c_double(0.0)
        st = SolveStats()
        status = check(lib().fhd_dev_gmres(self._h, _dpp(b_u), _dptr(b_p), _dpp(x_u), _dptr(x_p),
                                           _dpp(alpha_fc), _dptr(beta), _dpp(beta_ed), _dptr(gamma),
                                           float(theta_alpha), C.byref(npr), C.byref(st)), "gmres")
        return status, npr.value, st.as_dict()

    def stochastic_m_fluxdiv(self, sp: StochParams, stoch_m_force, increment, eta, eta_ed, temperature,
                             temperature_ed, dt, weights, W_cc, W_ed):
        """stochastic_m_fluxdiv (stochastic_m_fluxdiv.f90:42-778), with the
        stress filter of sp.filtering_width 1, 2 or 4 on periodic boxes.
        W_cc: n_rngs*dim cell tensors, W_ed: n_rngs*2*nE node/edge tensors."""
        w = (C.c_double * len(weights))(*[float(x) for x in weights])
        return check(lib().fhd_dev_stochastic_m_fluxdiv(self._h, C.byref(sp), _dpp(stoch_m_force),
                                                        int(bool(increment)), _dptr(eta), _dpp(eta_ed),
                                                        _dptr(temperature), _dpp(temperature_ed), float(dt),
                                                        C.cast(w, _DP), len(weights), _dpp(W_cc), _dpp(W_ed)),
                     "stochastic_m_fluxdiv")

    def advance_timestep_inertial(self, sp: StochParams, dt, umac, rho, pi, eta, eta_ed, kappa, temperature,
                                  temperature_ed, W_cc, W_ed):
        """One single-species inertial step (advance_timestep_inertial.f90)
        in place on umac, rho, pi.  Returns (status, [stats_pred, stats_corr])."""
        st = (SolveStats * 2)()
        status = check(lib().fhd_dev_advance_inertial(self._h, C.byref(sp), float(dt), _dpp(umac), _dptr(rho),
                                                      _dptr(pi), _dptr(eta), _dpp(eta_ed), _dptr(kappa),
                                                      _dptr(temperature), _dpp(temperature_ed), _dpp(W_cc),
                                                      _dpp(W_ed), st), "advance_timestep_inertial")
        return status, [st[0].as_dict(), st[1].as_dict()]

    def compute_mass_fluxdiv(self, mp: MixtureParams, sp: StochParams, rho, dt, weights, W_fc, mass_fluxdiv):
        """compute_mass_fluxdiv (compute_mass_fluxdiv.f90:29-183), ideal
        isothermal mixture: mass_fluxdiv = div(diffusive + stochastic flux).
        W_fc[(r*dim+d)*nspecies+i]: N(0,1) face fields."""
        w = (C.c_double * len(weights))(*[float(x) for x in weights])
        return check(lib().fhd_dev_compute_mass_fluxdiv(self._h, C.byref(mp), C.byref(sp), _dpp(rho), float(dt),
                                                        C.cast(w, _DP), len(weights), _dpp(W_fc),
                                                        _dpp(mass_fluxdiv)), "compute_mass_fluxdiv")

    def compute_sqrtLonsager_fc(self, mp: MixtureParams, sp: StochParams, rho, sqrtLonsager_fc):
        """compute_sqrtLonsager_fc (mass_flux_utilities.f90:1096-1229):
        sqrtLonsager_fc[d*ns*ns + r + ns*c] = entry (r, c) of the face
        Cholesky factors of direction d"""
        return check(lib().fhd_dev_compute_sqrtLonsager_fc(self._h, C.byref(mp), C.byref(sp), _dpp(rho),
                                                           _dpp(sqrtLonsager_fc)), "compute_sqrtLonsager_fc")

    def stochastic_mass_fluxdiv(self, mp: MixtureParams, sp: StochParams, sqrtLonsager_fc, dt, weights, W_fc,
                                stoch_mass_fluxdiv, stoch_mass_flux=None, increment=False):
        """stochastic_mass_fluxdiv (stochastic_mass_fluxdiv.f90:37-116) with
        the face factors of compute_sqrtLonsager_fc"""
        w = (C.c_double * len(weights))(*[float(x) for x in weights])
        return check(lib().fhd_dev_stochastic_mass_fluxdiv(
            self._h, C.byref(mp), C.byref(sp), _dpp(sqrtLonsager_fc), float(dt), C.cast(w, _DP), len(weights),
            _dpp(W_fc), int(bool(increment)), _dpp(stoch_mass_fluxdiv),
            _dpp(stoch_mass_flux) if stoch_mass_flux is not None else None), "stochastic_mass_fluxdiv")

    def advance_timestep_overdamped(self, sp: StochParams, mp, dt, umac, rho, pi, eta, eta_ed, kappa, temperature,
                                    temperature_ed, W_cc, W_ed, W_mass=None):
        """One overdamped step (advance_timestep_overdamped.f90:135-734) in
        place on umac, rho (list of species arrays; one array and mp=None
        for a single fluid) and pi.  W_cc/W_ed/W_mass hold the step's two
        random stages.  Returns (status, [stats_pred, stats_corr])."""
        st = (SolveStats * 2)()
        status = check(lib().fhd_dev_advance_overdamped(
            self._h, C.byref(sp), C.byref(mp) if mp is not None else None, float(dt), _dpp(umac), _dpp(rho),
            _dptr(pi), _dptr(eta), _dpp(eta_ed), _dptr(kappa), _dptr(temperature), _dpp(temperature_ed),
            _dpp(W_cc), _dpp(W_ed), _dpp(W_mass) if W_mass is not None else None, st), "advance_timestep_overdamped")
        return status, [st[0].as_dict(), st[1].as_dict()]

    def advance_timestep_inertial_multispecies(self, sp: StochParams, mp: MixtureParams, dt, umac, rho, pi,
                                               mass_fluxdiv, eta, eta_ed, kappa, temperature, temperature_ed,
                                               W_cc, W_ed, W_mass):
        """One inertial step of an ideal isothermal mixture
        (advance_timestep_inertial.f90) in place on umac, rho (species
        list), pi and mass_fluxdiv (F^n in, F^{n+1} out).  W_mass: the
        previous corrector's dim*nspecies face fields, then the new ones."""
        st = (SolveStats * 2)()
        status = check(lib().fhd_dev_advance_inertial_multispecies(
            self._h, C.byref(sp), C.byref(mp), float(dt), _dpp(umac), _dpp(rho), _dptr(pi), _dpp(mass_fluxdiv),
            _dptr(eta), _dpp(eta_ed), _dptr(kappa), _dptr(temperature), _dpp(temperature_ed), _dpp(W_cc),
            _dpp(W_ed), _dpp(W_mass), st), "advance_timestep_inertial_multispecies")
        return status, [st[0].as_dict(), st[1].as_dict()]

    # ----------------------------------------------------------------
    # host BoxLib-fab mirror (the drop-in boundary)
    # ----------------------------------------------------------------
    def gmres_fab(self, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha):
        """gmres on host FabArray multifabs (lists of FabArray per multifab)."""
        keep = []
        mfs = [_mf_vec(v, keep) for v in (b_u,)] + [_mf(b_p, keep)] + [_mf_vec(x_u, keep)] + [_mf(x_p, keep)]
        mfs += [_mf_vec(alpha_fc, keep), _mf(beta, keep), _mf_vec(beta_ed, keep), _mf(gamma, keep)]
        th = C.c_double(theta_alpha)
        npr = C.c_double(0.0)
        st = SolveStats()
        status = check(lib().fhd_gmres(self._h, *mfs, C.byref(th), C.byref(npr), C.byref(st)), "fhd_gmres")
        return status, npr.value, st.as_dict()

    def apply_matrix_fab(self, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha):
        keep = []
        mfs = [_mf_vec(b_u, keep), _mf(b_p, keep), _mf_vec(x_u, keep), _mf(x_p, keep),
               _mf_vec(alpha_fc, keep), _mf(beta, keep), _mf_vec(beta_ed, keep), _mf(gamma, keep)]
        return check(lib().fhd_apply_matrix(self._h, *mfs, float(theta_alpha)), "fhd_apply_matrix")

    def apply_precon_fab(self, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha):
        keep = []
        mfs = [_mf_vec(b_u, keep), _mf(b_p, keep), _mf_vec(x_u, keep), _mf(x_p, keep),
               _mf_vec(alpha_fc, keep), _mf(beta, keep), _mf_vec(beta_ed, keep), _mf(gamma, keep)]
        return check(lib().fhd_apply_precon(self._h, *mfs, float(theta_alpha)), "fhd_apply_precon")

    def stag_mg_solver_fab(self, alpha_fc, beta_cc, beta_ed, gamma_cc, theta_alpha, phi_fc, rhs_fc):
        """stag_mg_solver on host multifabs; phi_fc (>= 1 ghost cell) in/out"""
        keep = []
        return check(lib().fhd_stag_mg_solve(self._h, _mf_vec(alpha_fc, keep), _mf(beta_cc, keep),
                                             _mf_vec(beta_ed, keep), _mf(gamma_cc, keep), float(theta_alpha),
                                             _mf_vec(phi_fc, keep), _mf_vec(rhs_fc, keep)), "fhd_stag_mg_solve")

    def compute_sqrtLonsager_fc_fab(self, mp: MixtureParams, sp: StochParams, rho, rhotot, sqrtLonsager_fc):
        """compute_sqrtLonsager_fc on host multifabs: rho (nspecies
        components, >= 1 ghost cell), sqrtLonsager_fc (dim face multifabs of
        nspecies^2 components, written)"""
        keep = []
        return check(lib().fhd_compute_sqrtLonsager_fc(self._h, C.byref(mp), C.byref(sp), _mf(rho, keep),
                                                       _mf(rhotot, keep) if rhotot is not None else None,
                                                       _mf_vec(sqrtLonsager_fc, keep)), "fhd_compute_sqrtLonsager_fc")

    def stochastic_mass_fluxdiv_fab(self, mp: MixtureParams, sp: StochParams, rho, rhotot, sqrtLonsager_fc,
                                    stoch_mass_fluxdiv, stoch_mass_flux, dt, weights, W_fc, increment=False):
        """stochastic_mass_fluxdiv on host multifabs; W_fc[r*dim+d]: the
        nspecies-component N(0,1) face multifab of stage r, direction d"""
        keep = []
        w = (C.c_double * len(weights))(*[float(x) for x in weights])
        return check(lib().fhd_stochastic_mass_fluxdiv(
            self._h, C.byref(mp), C.byref(sp), _mf(rho, keep) if rho is not None else None,
            _mf(rhotot, keep) if rhotot is not None else None, _mf_vec(sqrtLonsager_fc, keep),
            _mf(stoch_mass_fluxdiv, keep), _mf_vec(stoch_mass_flux, keep) if stoch_mass_flux is not None else None,
            float(dt), C.cast(w, _DP), len(weights), _mf_vec(W_fc, keep), int(bool(increment))),
            "fhd_stochastic_mass_fluxdiv")

    def stochastic_m_fluxdiv_fab(self, sp: StochParams, stoch_m_force, increment, eta, eta_ed, temperature,
                                 temperature_ed, dt, weights, W_cc, W_ed):
        """stochastic_m_fluxdiv on host multifabs: stoch_m_force (dim face
        multifabs, in/out), eta and temperature cell multifabs, eta_ed and
        temperature_ed node (2D) or edge (3D) multifabs, W_cc[r] the
        dim-component cell multifab of stage r, W_ed[r*nE+e] the 2-component
        node/edge multifab of stage r and edge set e"""
        keep = []
        w = (C.c_double * len(weights))(*[float(x) for x in weights])
        return check(lib().fhd_stochastic_m_fluxdiv(
            self._h, C.byref(sp), _mf_vec(stoch_m_force, keep), int(bool(increment)), _mf(eta, keep),
            _mf_vec(eta_ed, keep), _mf(temperature, keep), _mf_vec(temperature_ed, keep), float(dt),
            C.cast(w, _DP), len(weights), _mf_vec(W_cc, keep), _mf_vec(W_ed, keep)), "fhd_stochastic_m_fluxdiv")


def stag_mg_solver_noalloc(dim, n_cells, dx, visc_type, params, alpha_fc, beta_cc, beta_ed, gamma_cc,
                           theta_alpha, phi_fc, rhs_fc, stream=None):
    """stag_mg_solver that allocates no device memory (no context needed):
    for callers that cannot call cudaMalloc.  Work arrays live in the
    library's static device array; grids beyond its size are rejected and
    calls that overlap on the GPU race on it."""
    n = list(n_cells) + [1] * (3 - len(n_cells))
    return check(lib().fhd_dev_stag_mg_solver_noalloc(int(dim), (C.c_int * 3)(*n[:3]), float(dx), int(visc_type),
                                                      C.byref(params), _dpp(alpha_fc), _dptr(beta_cc),
                                                      _dpp(beta_ed), _dptr(gamma_cc), float(theta_alpha),
                                                      _dpp(phi_fc), _dpp(rhs_fc), C.c_void_p(stream or 0)),
                 "stag_mg_solver_noalloc")


# ----------------------------------------------------------------------
# host fab helpers (BoxLib layout <-> canonical layout, numpy)
# ----------------------------------------------------------------------
class FabArray:
    """One BoxLib fab: Fortran-ordered float64 array covering
    lo-ng .. hi+nodal+ng in each direction (component 0)."""

    def __init__(self, data: np.ndarray, lo, hi, nodal, ng: int, ncomp: int = 1):
        self.data = data
        self.lo, self.hi, self.nodal, self.ng, self.ncomp = list(lo), list(hi), list(nodal), int(ng), int(ncomp)

    def fab(self) -> Fab:
        f = Fab()
        assert self.data.dtype == np.float64 and self.data.flags.f_contiguous
        f.data = self.data.ctypes.data_as(_DP)
        for d in range(3):
            f.lo[d] = self.lo[d] if d < len(self.lo) else 0
            f.hi[d] = self.hi[d] if d < len(self.hi) else 0
            f.nodal[d] = self.nodal[d] if d < len(self.nodal) else 0
        f.ng = self.ng
        f.ncomp = self.ncomp
        return f


def _mf(fa, keep):
    boxes = fa if isinstance(fa, (list, tuple)) else [fa]
    arr = (Fab * len(boxes))(*[b.fab() for b in boxes])
    keep.append(arr)
    mf = Multifab(len(boxes), C.cast(arr, C.POINTER(Fab)))
    keep.append(mf)
    return C.byref(mf)


def _mf_vec(fas, keep):
    mfs = []
    for fa in fas:
        boxes = fa if isinstance(fa, (list, tuple)) else [fa]
        arr = (Fab * len(boxes))(*[b.fab() for b in boxes])
        keep.append(arr)
        mfs.append(Multifab(len(boxes), C.cast(arr, C.POINTER(Fab))))
    a = (Multifab * len(mfs))(*mfs)
    keep.append(a)
    return C.cast(a, C.POINTER(Multifab))


def fab_from_canonical(x: np.ndarray, dim: int, n_cells, nodal, ng: int, lo=None, hi=None) -> FabArray:
    """Periodic canonical array -> one fab over box lo..hi (default the
    whole domain), ghost cells and the duplicated nodal plane filled."""
    n = list(n_cells)[:dim]
    lo = list(lo) if lo is not None else [0] * dim
    hi = list(hi) if hi is not None else [k - 1 for k in n]
    nodal = list(nodal)[:dim]
    idx = []
    for d in range(dim):
        rng = np.arange(lo[d] - ng, hi[d] + nodal[d] + ng + 1)
        idx.append(np.mod(rng, n[d]))
    can = x.reshape([n[d] for d in reversed(range(dim))])  # (z, y, x) C order
    if dim == 2:
        sub = can[np.ix_(idx[1], idx[0])]
    else:
        sub = can[np.ix_(idx[2], idx[1], idx[0])]
    data = np.asfortranarray(sub.T)
    return FabArray(data, lo + [0] * (3 - dim), hi + [0] * (3 - dim), nodal + [0] * (3 - dim), ng)


def fab_from_components(xs, dim: int, n_cells, nodal, ng: int, lo=None, hi=None) -> FabArray:
    """Periodic canonical arrays, one per component -> one multi-component
    fab (Fortran order, the component index slowest)."""
    fabs = [fab_from_canonical(x, dim, n_cells, nodal, ng, lo, hi) for x in xs]
    data = np.asfortranarray(np.stack([f.data for f in fabs], axis=-1))
    f0 = fabs[0]
    return FabArray(data, f0.lo, f0.hi, f0.nodal, ng, ncomp=len(xs))


def canonical_from_fab(fa: FabArray, dim: int, n_cells) -> np.ndarray:
    """Valid cells lo..hi of one whole-domain fab -> canonical array."""
    n = list(n_cells)[:dim]
    g = fa.ng
    sl = tuple(slice(g, g + fa.hi[d] - fa.lo[d] + 1) for d in range(dim))
    return np.ascontiguousarray(fa.data[sl].T).reshape(-1)


# ----------------------------------------------------------------------
# device random numbers and serving
# ----------------------------------------------------------------------
def fill_normal(out, seed: int, field: int = 0, stream_a: int = 0, stream_b: int = 0, scale: float = 1.0,
                stream: int | None = None):
    """out (contiguous float64 CUDA tensor) = scale * N(0,1) from the
    device Philox-4x32-10 generator (fill_m_stochastic's role)."""
    check(lib().fhd_dev_fill_normal(C.c_void_p(out.data_ptr()), out.numel(), int(seed), int(field), int(stream_a),
                                    int(stream_b), float(scale), C.c_void_p(stream or 0)), "fill_normal")


def philox4x32_10(ctr, key):
    """the Philox-4x32-10 block function (host side of the device generator)"""
    c = (C.c_uint * 4)(*[int(x) & 0xFFFFFFFF for x in ctr])
    k = (C.c_uint * 2)(*[int(x) & 0xFFFFFFFF for x in key])
    o = (C.c_uint * 4)()
    lib().fhd_philox4x32_10(c, k, o)
    return list(o)


class StepNoise:
    """Fresh N(0,1) stochastic fields for every inertial step, drawn on the
    device by the Philox generator: the work of fill_m_stochastic
    (stochastic_m_fluxdiv.f90:781-860, symmetric stress form: cell entries
    with variance 2, the two components of a node/edge equal) and
    fill_mass_stochastic (stochastic_mass_fluxdiv.f90:182-214).

    The counters follow the server's: momentum field c counted by the step,
    mass field 1000 + d*ns + i counted by the noise index.  Step k of
    advance_timestep_inertial reads the mass noise M_{k-1} (predictor) and M_k
    (corrector); F^0 comes from M_0.  So two runs with the same seed (say
    mixed precision and FP64) see the same fields, and no two steps do."""

    def __init__(self, dim: int, n_cells, nspecies: int, seed: int, device, stream: int | None = None):
        import torch
        self.dim, self.ns, self.seed, self.stream = dim, nspecies, int(seed), stream
        nc = int(np.prod(list(n_cells)[:dim]))
        ne = 1 if dim == 2 else 3
        z = lambda: torch.empty(nc, dtype=torch.float64, device=device)
        self.W_cc = [z() for _ in range(dim)]
        self._ed = [z() for _ in range(ne)]
        # both components of a node/edge point at the same field
        self.W_ed = [e for e in self._ed for _ in range(2)]
        self._mass = [[z() for _ in range(dim * nspecies)] for _ in range(2)] if nspecies > 1 else None

    def _fill(self, out, field, count, scale=1.0):
        fill_normal(out, self.seed, field, count, 0x5EED, scale, self.stream)

    def draw_mass(self, j: int):
        """mass noise M_j into its ring slot"""
        for i, w in enumerate(self._mass[j % 2]):
            self._fill(w, 1000 + i, j)

    def mass(self, j: int):
        return self._mass[j % 2]

    def draw(self, step: int):
        """the fields of inertial step `step` (>= 1): momentum, and M_step"""
        for c, w in enumerate(self.W_cc):
            self._fill(w, c, step, 2.0 ** 0.5)
        for e, w in enumerate(self._ed):
            self._fill(w, self.dim + e, step)
        if self._mass is not None:
            self.draw_mass(step)

    def launches_per_draw(self) -> int:
        return len(self.W_cc) + len(self._ed) + (len(self._mass[0]) if self._mass is not None else 0)

    def inertial_args(self, step: int):
        """(W_cc, W_ed, W_mass) of step `step` as the multispecies inertial
        step takes them: W_mass = M_{step-1} followed by M_step"""
        wm = (list(self.mass(step - 1)) + list(self.mass(step))) if self._mass is not None else None
        return self.W_cc, self.W_ed, wm


def make_request(**kw) -> Request:
    """an fhd_request with the library defaults, fields overridden by kw
    (n_cells as a list; params as a GmresParams; mix as MixtureParams)"""
    r = Request()
    lib().fhd_request_default(C.byref(r))
    for k, v in kw.items():
        if k == "n_cells":
            n = list(v) + [1] * (3 - len(v))
            r.n_cells = (C.c_int * 3)(*n)
        elif not hasattr(r, k):
            raise AttributeError(f"fhd_request has no field {k}")
        else:
            setattr(r, k, v)
    return r


def sched_simulate(slots: int, budget: int, arrive, nbytes, runtime):
    """start times the server's admission policy gives a synthetic trace"""
    n = len(arrive)
    a = (C.c_double * max(1, n))(*arrive)
    b = (C.c_ulonglong * max(1, n))(*[int(x) for x in nbytes])
    r = (C.c_double * max(1, n))(*runtime)
    s = (C.c_double * max(1, n))()
    check(lib().fhd_sched_simulate(int(slots), int(budget), n, C.cast(a, _DP), b, C.cast(r, _DP), C.cast(s, _DP)),
          "sched_simulate")
    return list(s)[:n]


def tune_candidates(which: str, dim: int, n_cells, precision: str = "mixed", visc_type: int = 1, sms: int = 148,
                    smem_optin: int = 232448, smem_sm: int = 233472) -> list[dict]:
    """the smoother plans the autotuner would time for one level (host
    only); defaults: the B200's 148 SMs and shared-memory limits"""
    n = (C.c_int * 3)(*(list(n_cells) + [1] * (3 - len(n_cells))))
    prec = FHD_PREC_MIXED if precision == "mixed" else FHD_PREC_FP64
    out = (C.c_int * (7 * 64))()
    k = check(lib().fhd_tune_candidates(0 if which == "stag" else 1, int(dim), n, prec, int(visc_type), int(sms),
                                        int(smem_optin), int(smem_sm), out, 64), "fhd_tune_candidates")
    names = {0: "colour", 1: "tiled", 2: "rowtile"}
    return [dict(kind=names[out[7 * i]], x=out[7 * i + 1], y=out[7 * i + 2], zruns=out[7 * i + 3],
                 per_sm=out[7 * i + 4], smem=out[7 * i + 5], threads=out[7 * i + 6]) for i in range(min(k, 64))]


def tune_export() -> str:
    """the autotuner's table as text (fhd_tune_export)"""
    need = int(lib().fhd_tune_export(None, 0))
    buf = C.create_string_buffer(need)
    lib().fhd_tune_export(buf, need)
    return buf.value.decode()


def tune_import(text: str) -> int:
    """add plans from text written by tune_export (fhd_tune_import)"""
    return check(lib().fhd_tune_import(text.encode()), "fhd_tune_import")


def tune_key(which: str, dim: int, n_cells, precision: str = "mixed", visc_type: int = 1, sms: int = 148,
             smem_optin: int = 232448, smem_sm: int = 233472, device: int = 0) -> str:
    """the autotuner's table key of one level shape (fhd_tune_key; host
    only); defaults: device 0 with the B200's 148 SMs and shared-memory
    limits"""
    n = (C.c_int * 3)(*(list(n_cells) + [1] * (3 - len(n_cells))))
    prec = FHD_PREC_MIXED if precision == "mixed" else FHD_PREC_FP64
    args = (0 if which == "stag" else 1, int(dim), n, prec, int(visc_type), int(sms), int(smem_optin), int(smem_sm),
            int(device))
    need = check(int(lib().fhd_tune_key(*args, None, 0)), "fhd_tune_key")
    buf = C.create_string_buffer(need)
    lib().fhd_tune_key(*args, buf, need)
    return buf.value.decode()


class StructureFactor:
    """Static structure factors on the device (fhd_sk_*; HydroGrid's
    updateStructureFactors, HydroGrid/HydroGridModule.f90:1077-1180): per
    update, the DFT of each of `nvars` fields, the staggered phase shift of
    velocity component d when shift[d] is +1 or -1, and the running mean of
    Ua conj(Ub) for every pair (a, b); read(p) returns pair p times dV/N_c
    on the half spectrum as a complex array of shape (nz, ny, nx//2+1) (2D:
    (ny, nx//2+1))."""

    def __init__(self, dim: int, n_cells: Sequence[int], dV: float, nvars: int, pairs, shift=None):
        n = (C.c_int * 3)(*(list(n_cells) + [1] * (3 - len(n_cells))))
        pr = [int(x) for p in pairs for x in p]
        parr = (C.c_int * len(pr))(*pr)
        sarr = (C.c_int * nvars)(*[int(x) for x in shift]) if shift is not None else None
        h = C.c_void_p()
        check(lib().fhd_sk_create(int(dim), n, float(dV), int(nvars), sarr, len(pairs), parr, C.byref(h)),
              "fhd_sk_create")
        self._h = h
        self.dim = dim
        self.n = list(n_cells)
        self.npairs = len(pairs)

    def update(self, fields, stream_handle: int | None = None):
        check(lib().fhd_sk_update(self._h, _dpp(fields), C.c_void_p(stream_handle or 0)), "fhd_sk_update")

    def read(self, pair: int):
        nm = int(lib().fhd_sk_modes(self._h))
        re, im = np.empty(nm), np.empty(nm)
        ns = C.c_longlong()
        check(lib().fhd_sk_read(self._h, int(pair), re.ctypes.data_as(_DP), im.ctypes.data_as(_DP), C.byref(ns)),
              "fhd_sk_read")
        shape = ([self.n[2]] if self.dim == 3 else []) + [self.n[1], self.n[0] // 2 + 1]
        return (re + 1j * im).reshape(shape), ns.value

    def close(self):
        if getattr(self, "_h", None):
            lib().fhd_sk_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent 2D periodic boxes of uneven size solved together
    (fhd_batch_*): one launch per multigrid level and operation covers all
    boxes, GMRES's scalar control runs on the device per box.  Vectors are
    flat float64 CUDA tensors of all boxes' cells concatenated in box order
    (offset(b) is box b's first element)."""

    def __init__(self, n_cells, dx: float = 1.0, params: GmresParams | None = None, precision: str = "mixed"):
        sizes = [(int(a), int(b)) for a, b in n_cells]
        self.n_cells = sizes
        self.params = params if params is not None else default_params()
        arr = (C.c_int * (2 * len(sizes)))(*[v for ab in sizes for v in ab])
        h = C.c_void_p()
        mode = FHD_PREC_MIXED if precision == "mixed" else FHD_PREC_FP64
        check(lib().fhd_batch_create(len(sizes), arr, float(dx), C.byref(self.params), mode, C.byref(h)),
              "fhd_batch_create")
        self._h = h

    @property
    def nboxes(self) -> int:
        return len(self.n_cells)

    def offset(self, box: int) -> int:
        return int(lib().fhd_batch_box_offset(self._h, int(box)))

    @property
    def total(self) -> int:
        return self.offset(self.nboxes)

    @property
    def kernel_launches(self) -> int:
        return int(lib().fhd_batch_kernel_launches(self._h))

    def box(self, t, b: int):
        """box b's part of a packed vector t"""
        return t[self.offset(b):self.offset(b + 1)]

    def gmres(self, b, x, eta, theta_alpha: float = 0.0):
        """gmres of every box: b and x lists of 3 packed tensors (u_x, u_y,
        p); x in/out; eta per box.  Returns (worst status, per-box stats)."""
        e = (C.c_double * self.nboxes)(*[float(v) for v in eta])
        st = (SolveStats * self.nboxes)()
        status = check(lib().fhd_batch_gmres(self._h, _dpp(b), _dpp(x), C.cast(e, _DP), float(theta_alpha), st),
                       "fhd_batch_gmres")
        return status, [st[i].as_dict() for i in range(self.nboxes)]

    def overdamped(self, umac, pi, eta, kT, dt: float, steps: int, seed: int = 1, step0: int = 0):
        """`steps` overdamped steps of every box in place (umac: 2 packed face
        tensors, pi packed); returns (worst status, GMRES iterations per box)"""
        e = (C.c_double * self.nboxes)(*[float(v) for v in eta])
        k = (C.c_double * self.nboxes)(*[float(v) for v in kT])
        it = (C.c_int * self.nboxes)()
        status = check(lib().fhd_batch_overdamped(self._h, _dpp(umac), _dptr(pi), C.cast(e, _DP), C.cast(k, _DP),
                                                  float(dt), int(steps), int(seed), int(step0), it),
                       "fhd_batch_overdamped")
        return status, list(it)

    def close(self):
        if getattr(self, "_h", None):
            lib().fhd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Server:
    """Many device-resident problems on one GPU (fhd_server_*): `slots`
    worker threads with a CUDA stream each, admission in arrival order
    within an HBM byte budget."""

    def __init__(self, slots: int, hbm_budget_bytes: int):
        h = C.c_void_p()
        check(lib().fhd_server_create(int(slots), int(hbm_budget_bytes), C.byref(h)), "fhd_server_create")
        self._h = h
        self._keep = {}

    @staticmethod
    def request_bytes(req: Request) -> int:
        return int(lib().fhd_request_bytes(C.byref(req)))

    def clock(self) -> float:
        return float(lib().fhd_server_clock(self._h))

    def submit(self, req: Request, out_umac=None, out_rho=None) -> int:
        """queue a copy of req; out_umac / out_rho: optional float64 numpy
        arrays (dim*Nc, nspecies*Nc) that receive the final state"""
        r = Request.from_buffer_copy(req)
        if out_umac is not None:
            r.out_umac = out_umac.ctypes.data_as(_DP)
        if out_rho is not None:
            r.out_rho = out_rho.ctypes.data_as(_DP)
        rid = C.c_longlong()
        check(lib().fhd_server_submit(self._h, C.byref(r), C.byref(rid)), "fhd_server_submit")
        self._keep[rid.value] = (out_umac, out_rho)
        return rid.value

    def wait(self, rid: int) -> dict:
        res = RequestResult()
        check(lib().fhd_server_wait(self._h, int(rid), C.byref(res)), "fhd_server_wait")
        self._keep.pop(rid, None)
        return res.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            lib().fhd_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
