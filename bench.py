"""Benchmark: LowMachFHD inertial low-Mach timesteps on a 3D 256^3 periodic
grid, mixed precision (FP32 multigrid preconditioner and stochastic flux
inside FP64 GMRES) against the plain FP64 path on the same B200, GMRES
relative residual 1e-8.

A step is one Crank-Nicolson predictor-corrector step of
advance_timestep_inertial (two preconditioned GMRES Stokes solves plus the
stochastic momentum flux, advection and viscous terms) through the
device-resident step entry point of the C ABI.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank runs an independent replica (the path does not
shard: "replicas only"); value = steps of all ranks / max-over-ranks time.
Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "3D 256³ steps/s: mixed vs FP64 (same B200, 1e-8 resid); served p50/p99 latency"
N_CELLS = 256
DX = 10.0
DT = 5.0
KT = 1e-4
REL_TOL = 1e-8
NSPECIES = 4
MOLMASS = [1.0, 2.0, 3.0, 4.0]
WORKLOAD = "lowmach_inertial_step_3d_256cube_periodic_4species"


def mixture(seed=11):
    """4-species ideal mixture: masses 1..4, Maxwell-Stefan coefficients
    D_ij ~ U[0.5, 2] * 1e-2 (seeded, symmetric), rhobar = 1"""
    import numpy as np
    rng = np.random.default_rng(seed)
    D = list(rng.uniform(0.5, 2.0, NSPECIES * (NSPECIES - 1) // 2) * 1e-2)
    return dict(molmass=MOLMASS, Dbar=D, rhobar=[1.0] * NSPECIES, variance_coef_mass=1.0)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_CELLS, help="cells per direction")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-n", type=int, default=128)
    ap.add_argument("--only", choices=["mixed", "fp64"], default=None, help="run one precision only")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving and batched legs")
    ap.add_argument("--probe", choices=["stagmg", "gmres", "stochm", "batch"], default=None,
                    help="profiling probe on one single-fluid 3D grid: K stag_mg_solver calls (one V-cycle "
                         "each), K GMRES solves (theta 20, 1e-8), or K stochastic_m_fluxdiv calls; or (batch) "
                         "K batched overdamped steps of the 512 2D realizations after one warm-up step")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="fp64", help="precision of --probe")
    ap.add_argument("--tune", type=int, default=-1,
                    help="smoother autotuner mode of --probe (fhd_ctx_set_tune: -1 tune, 0 fixed rules, 2+k "
                         "candidate k on every level)")
    return ap.parse_args()


def run_probe(args):
    """K staggered multigrid solves, GMRES solves or stochastic momentum
    flux evaluations on random single-fluid data (small, self-contained
    workloads for kernel captures)."""
    import torch

    import lowmachfhd_b200 as L
    dev = torch.device("cuda:0")
    if args.probe == "batch":
        r = run_batch_solver(L, torch, dev, count=BATCH_REALIZATIONS, steps=args.steps)
        print(json.dumps({"probe": "batch", **r}))
        return 0
    n = args.n
    nc = n ** 3
    s = L.StokesSolver(3, [n, n, n], 1.0, 1, params=L.default_params(gmres_max_inner=1),
                       precision=args.precision)
    s.set_tune(args.tune)
    g = torch.Generator().manual_seed(3)
    f64 = dict(dtype=torch.float64)
    alpha = [(1.0 + 1e-3 * torch.randn(nc, generator=g, **f64)).to(dev) for _ in range(3)]
    one = torch.ones(nc, device=dev, **f64)
    rhs = [torch.randn(nc, generator=g, **f64).to(dev) for _ in range(3)]
    phi = [torch.zeros(nc, device=dev, **f64) for _ in range(3)]
    zero = torch.zeros(nc, device=dev, **f64)
    if args.probe == "gmres":
        s.close()
        s = L.StokesSolver(3, [n, n, n], 1.0, 1, params=L.default_params(gmres_rel_tol=REL_TOL),
                           precision=args.precision)
        s.set_tune(args.tune)
        bp = torch.randn(nc, generator=g, **f64)
        bp = (bp - bp.mean()).to(dev)
        x_p = torch.zeros(nc, device=dev, **f64)

        def call():
            for c in range(3):
                phi[c].zero_()
            x_p.zero_()
            s.gmres(rhs, bp, phi, x_p, alpha, one, [one, one, one], zero, 20.0)
    elif args.probe == "stochm":
        sp = L.StochParams(k_B=KT, variance_coef_mom=1.0, dV=DX ** 3, stoch_stress_form=1, filtering_width=0)
        W_cc = [torch.randn(nc, generator=g, **f64).to(dev) for _ in range(3)]
        W_ed = [torch.randn(nc, generator=g, **f64).to(dev) for _ in range(6)]

        def call():
            s.stochastic_m_fluxdiv(sp, phi, False, one, [one, one, one], one, [one, one, one], DT, [1.0],
                                   W_cc, W_ed)
    else:
        def call():
            s.stag_mg_solver(alpha, one, [one, one, one], zero, 20.0, phi, rhs)
    # the warm-up calls pick the smoother plans (autotuner); the NVTX range
    # "probe" holds only the measured calls, so that a profiler can be
    # restricted to them (ncu --nvtx --nvtx-include "probe/")
    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("probe")
    for _ in range(args.steps):
        call()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"probe": args.probe, "n": n, "precision": args.precision, "calls": args.warmup + args.steps,
                      "launches": s.kernel_launches, "plan_level0": s.tune_info("stag", 0)}))
    s.close()
    return 0


# ----------------------------------------------------------------------
# serving: a Poisson stream of Stokes / timestep requests of mixed sizes
# ----------------------------------------------------------------------
SERVE_RATE = 10.0      # requests per second (below the capacity of the mix)
SERVE_REQUESTS = 120
SERVE_SLOTS = 8
SERVE_BUDGET = 96 << 30


def serve_requests(L, count, seed, precision):
    """Requests of the serving configuration: 2D 64^2-512^2 overdamped and
    3D 32^3-192^3 inertial problems (sides log-uniform, multiples of 8),
    1-4 species, eta ~ U[0.5, 5], k_B T ~ U[1e-4, 1e-3], 4 steps each,
    seeded.  Mixtures use a cell volume of 1000 (dx = 10 in 3D, depth 1000
    in 2D)."""
    import numpy as np
    reqs = []
    for i in range(count):
        rng = np.random.default_rng(seed + i)
        dim = int(rng.integers(2, 4))
        lo, hi = (64, 512) if dim == 2 else (32, 192)
        side = max(lo, min(hi, int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))) / 8)) * 8))
        ns = int(rng.integers(1, 5))
        eta = float(rng.uniform(0.5, 5.0))
        kT = float(rng.uniform(1e-4, 1e-3))
        D = list(rng.uniform(0.5, 2.0, max(1, ns * (ns - 1) // 2)) * 1e-2)
        kw = dict(dim=dim, n_cells=[side] * dim, nspecies=ns, eta=eta, kT=kT, steps=4, seed=1000 + i,
                  precision=L.FHD_PREC_MIXED if precision == "mixed" else L.FHD_PREC_FP64,
                  params=L.default_params(gmres_rel_tol=REL_TOL))
        if dim == 2:
            kw.update(kind=L.FHD_REQ_OVERDAMPED, dx=1.0, cell_depth=1000.0, dt=0.1)
        else:
            kw.update(kind=L.FHD_REQ_INERTIAL, dx=10.0, dt=0.05 * 100.0 / eta)
        if ns > 1:
            kw["mix"] = L.mixture_params([1.0, 2.0, 3.0, 4.0][:ns], D[: ns * (ns - 1) // 2], rhobar=[1.0] * ns,
                                         variance_coef_mass=1.0)
        reqs.append(L.make_request(**kw))
    return reqs


def serve_warmup(L, srv, precision, shapes=()):
    """one tiny request per (dimension, species count, kind) so that the
    first launch of every kernel the mix uses is not inside the measurement;
    then one one-step request per grid shape in `shapes`, which fills the
    autotuner's table for those shapes (the smoother plans are picked once
    per process and shape, as a deployed server would load its table)"""
    ids = []
    for dim, side in sorted(set(shapes)):
        kw = dict(dim=dim, n_cells=[side] * dim, nspecies=1, steps=1, kT=1e-4,
                  precision=L.FHD_PREC_MIXED if precision == "mixed" else L.FHD_PREC_FP64,
                  kind=L.FHD_REQ_OVERDAMPED if dim == 2 else L.FHD_REQ_INERTIAL,
                  dx=1.0 if dim == 2 else 10.0, cell_depth=1000.0, dt=0.1 if dim == 2 else 5.0,
                  params=L.default_params(gmres_rel_tol=REL_TOL, gmres_max_iter=2))
        ids.append(srv.submit(L.make_request(**kw)))
    for i in ids:
        srv.wait(i)
    ids = []
    for dim in (2, 3):
        for ns in (1, 2, 3, 4):
            kw = dict(dim=dim, n_cells=[16] * dim if dim == 2 else [8] * 3, nspecies=ns, steps=1, kT=1e-4,
                      precision=L.FHD_PREC_MIXED if precision == "mixed" else L.FHD_PREC_FP64,
                      kind=L.FHD_REQ_OVERDAMPED if dim == 2 else L.FHD_REQ_INERTIAL,
                      dx=1.0 if dim == 2 else 10.0, cell_depth=1000.0, dt=0.1 if dim == 2 else 5.0)
            if ns > 1:
                kw["mix"] = L.mixture_params([1.0, 2.0, 3.0, 4.0][:ns], [1e-2] * (ns * (ns - 1) // 2),
                                             rhobar=[1.0] * ns)
            ids.append(srv.submit(L.make_request(**kw)))
    for i in ids:
        srv.wait(i)


def run_serving(L, slots, precision, rate, count, seed=7):
    """Poisson arrivals at `rate` (seeded; rate None: all at once, the
    saturation throughput); returns latency percentiles (submit to result)
    and completed requests per second."""
    import numpy as np
    reqs = serve_requests(L, count, seed, precision)
    if rate:
        gaps = np.random.default_rng(seed).exponential(1.0 / rate, count)
        arrive = np.cumsum(gaps) - gaps[0]
    else:
        arrive = np.zeros(count)
    with L.Server(slots, SERVE_BUDGET) as srv:
        serve_warmup(L, srv, precision, shapes=[(r.dim, r.n_cells[0]) for r in reqs])
        t0 = time.perf_counter()
        ids = []
        for r, a in zip(reqs, arrive):
            d = a - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            ids.append(srv.submit(r))
        res = [srv.wait(i) for i in ids]
    lat = np.array([r["t_end"] - r["t_submit"] for r in res]) * 1e3
    span = max(r["t_end"] for r in res) - min(r["t_submit"] for r in res)
    bad = [r["status"] for r in res if r["status"] < 0]
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "solves_per_s": count / span, "requests": count, "errors": len(bad),
            "gmres_iters": int(sum(r["gmres_iters"] for r in res))}


# ----------------------------------------------------------------------
# batched: many independent 2D realizations of uneven size
# ----------------------------------------------------------------------
BATCH_REALIZATIONS = 512
BATCH_STEPS = 20
BATCH_SLOTS = 16


def batch_realizations(count, seed):
    """sides log-uniform in [32, 256] rounded to multiples of 8, eta ~
    U[0.5, 5] (seeded)"""
    import numpy as np
    rng = np.random.default_rng(seed)
    sides = np.clip(np.round(np.exp(rng.uniform(math.log(32), math.log(256), count)) / 8) * 8, 32, 256).astype(int)
    return sides, rng.uniform(0.5, 5.0, count)


def run_batch_solver(L, torch, dev, count=BATCH_REALIZATIONS, steps=BATCH_STEPS, seed=1):
    """the same realizations through the batched solver (fhd_batch_*): every
    box advanced together, one launch per multigrid level and operation for
    all 512 boxes.  The call synchronises its own stream once per GMRES
    cycle, so the time is host wall time around the synchronous call, after
    one untimed warm-up step."""
    sides, etas = batch_realizations(count, seed)
    sizes = [(int(n), int(n)) for n in sides]
    params = L.default_params(gmres_rel_tol=REL_TOL)
    with L.Batch(sizes, 1.0, params=params, precision="mixed") as B:
        u = [torch.zeros(B.total, dtype=torch.float64, device=dev) for _ in range(2)]
        pi = torch.zeros(B.total, dtype=torch.float64, device=dev)
        kT = [1.0] * count
        torch.cuda.synchronize()
        B.overdamped(u, pi, etas, kT, 0.1, 1, seed=seed, step0=0)
        n0 = B.kernel_launches
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        status, iters = B.overdamped(u, pi, etas, kT, 0.1, steps, seed=seed, step0=1)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        launches = B.kernel_launches - n0
        finite = bool(torch.isfinite(u[0]).all().item() and torch.isfinite(pi).all().item())
        cells = B.total
    return {"realizations": count, "steps_each": steps, "cells": cells,
            "realization_steps_per_s": count * steps / wall, "wall_s": wall,
            "timing": "host wall time around the synchronous call (one sync per GMRES cycle inside)",
            "gmres_iters": int(sum(iters)), "gmres_iters_max_box": int(max(iters)),
            "kernel_launches": launches, "launches_per_step": launches / steps,
            "status": status, "finite": finite}


def run_batched(L, count=BATCH_REALIZATIONS, steps=BATCH_STEPS, slots=BATCH_SLOTS, seed=1):
    """count 2D periodic realizations, sides log-uniform in [32, 256] rounded
    to multiples of 8 (seeded), eta ~ U[0.5, 5], `steps` overdamped steps
    each, FP32 preconditioner inside FP64 GMRES at 1e-8; all submitted at
    once to one server.  Returns realization-steps per second."""
    sides, etas = batch_realizations(count, seed)
    reqs = [L.make_request(kind=L.FHD_REQ_OVERDAMPED, dim=2, n_cells=[int(n), int(n)], eta=float(e), kT=1.0,
                           dt=0.1, steps=steps, seed=5000 + i, precision=L.FHD_PREC_MIXED,
                           params=L.default_params(gmres_rel_tol=REL_TOL))
            for i, (n, e) in enumerate(zip(sides, etas))]
    with L.Server(slots, SERVE_BUDGET) as srv:
        serve_warmup(L, srv, "mixed")
        t0 = time.perf_counter()
        ids = [srv.submit(r) for r in reqs]
        res = [srv.wait(i) for i in ids]
        wall = time.perf_counter() - t0
    return {"realizations": count, "steps_each": steps, "slots": slots,
            "sides": f"log-uniform 32-256, multiples of 8 (seed {seed})", "eta": "U[0.5, 5]",
            "realization_steps_per_s": count * steps / wall, "wall_s": wall,
            "gmres_iters": int(sum(r["gmres_iters"] for r in res)),
            "errors": sum(1 for r in res if r["status"] < 0)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------
class Clocks:
    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thr = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return

        def rd():
            for line in self.proc.stdout:
                self.rows.append([x.strip() for x in line.split(",")])
        self.thr = threading.Thread(target=rd, daemon=True)
        self.thr.start()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thr:
            self.thr.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                pass
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------
# problem set-up (seeded synthetic inputs; no dataset involved)
# ----------------------------------------------------------------------
NOISE_SEED = 20261204


def neighbour_shifts(n):
    """offsets, modulo the n^3 field size, from a cell to its periodic
    neighbours (shifts of -1, 0, 1 in x, y and z) and to itself"""
    nc = n ** 3
    sh = {0, 1, -1, n - 1, 1 - n}
    return {(a + n * b + n * n * c) % nc for a in sh for b in sh for c in sh}


def pool_stride(n, steps):
    """Stride between steps in the end-to-end leg's host noise pools: step i
    reads field f from the window starting at f*nc + i*stride.  Two windows
    of different steps i, j differ in offset, modulo nc, by (i - j)*stride;
    the stride is the first odd multiple of 512 (4 KiB-aligned windows) near
    nc/16 for which no step difference up to `steps` gives zero or a
    neighbour's offset, so no cell or neighbour sees a pool element twice."""
    nc = n ** 3
    near = neighbour_shifts(n)
    q = max(1, nc // (16 * 512)) | 1
    while True:
        s = 512 * q
        if all((k * s) % nc not in near for k in range(1, steps + 1)):
            return s
        q += 2


class HostNoisePool:
    """pinned host N(0,1) pools from which every step of the end-to-end leg
    uploads fields no earlier step used: the cell fields of the symmetric
    momentum stress (variance 2), and the unit-variance edge and mass-face
    fields"""

    def __init__(self, torch, n, steps, seed):
        g = torch.Generator().manual_seed(seed)
        nc = n ** 3
        self.stride = pool_stride(n, steps)
        span = (steps + 1) * self.stride
        self.nc = nc
        self.cc = (torch.randn(3 * nc + span, generator=g, dtype=torch.float64) * 2.0 ** 0.5).pin_memory()
        self.unit = torch.randn((3 + 3 * NSPECIES) * nc + span, generator=g, dtype=torch.float64).pin_memory()

    def fields(self, i):
        """(W_cc[3], W_ed[3] distinct, W_mass[3*ns]) host views of step i"""
        o, nc = i * self.stride, self.nc
        cc = [self.cc[c * nc + o: (c + 1) * nc + o] for c in range(3)]
        un = [self.unit[f * nc + o: (f + 1) * nc + o] for f in range(3 + 3 * NSPECIES)]
        return cc, un[:3], un[3:]


class Case:
    """the bench state: velocity, species densities, pressure and the mass
    flux divergence of one 256^3 periodic box, in place"""

    def __init__(self, L, torch, dev, n, precision, seed=7):
        self.torch, self.dev, self.n = torch, dev, n
        nc = n ** 3
        self.nc = nc
        params = L.default_params(gmres_rel_tol=REL_TOL)
        self.s = L.StokesSolver(3, [n, n, n], DX, 1, params=params, precision=precision)
        g = torch.Generator(device="cpu").manual_seed(seed)
        f64 = dict(dtype=torch.float64)
        self.umac = [(1e-3 * torch.randn(nc, generator=g, **f64)).to(dev) for _ in range(3)]
        # mass fractions 0.25 + 1e-3 N(0,1), renormalised; total density 1
        w = 0.25 + 1e-3 * torch.randn(NSPECIES, nc, generator=g, **f64)
        w = w / w.sum(dim=0, keepdim=True)
        self.rho = [w[i].contiguous().to(dev) for i in range(NSPECIES)]
        self.F = [torch.zeros(nc, device=dev, **f64) for _ in range(NSPECIES)]
        self.mp = L.mixture_params(**mixture())
        self.pi = torch.zeros(nc, device=dev, **f64)
        self.eta = torch.ones(nc, device=dev, **f64)
        self.eta_ed = [torch.ones(nc, device=dev, **f64) for _ in range(3)]
        self.kappa = torch.zeros(nc, device=dev, **f64)
        self.T = torch.ones(nc, device=dev, **f64)
        self.T_ed = [torch.ones(nc, device=dev, **f64) for _ in range(3)]
        self.sp = L.StochParams(k_B=KT, variance_coef_mom=1.0, dV=DX ** 3, stoch_stress_form=1, filtering_width=0)
        torch.cuda.synchronize()  # the context launches on its own stream

    def init_fluxes(self, W_m0):
        """F^0 = compute_mass_fluxdiv at the initial state (main_driver.f90
        start-up, before the time loop)"""
        self.s.compute_mass_fluxdiv(self.mp, self.sp, self.rho, DT, [1.0], W_m0, self.F)

    def step(self, W_cc, W_ed, W_mass):
        return self.s.advance_timestep_inertial_multispecies(
            self.sp, self.mp, DT, self.umac, self.rho, self.pi, self.F, self.eta, self.eta_ed, self.kappa, self.T,
            self.T_ed, W_cc, W_ed, W_mass)

    def snapshot(self):
        return [t.clone() for t in self.umac + self.rho + [self.pi]]


def mixed_vs_fp64(mix, f64, rho0):
    """relative infinity-norm differences of the mixed run's final fields
    from the FP64 run's (same inputs, same noise, same step count): velocity
    components and pressure against the FP64 field's largest magnitude, each
    species density against the FP64 run's largest change of that density
    over the run"""
    out = {}
    for c in range(3):
        out[f"u{c}"] = float((mix[c] - f64[c]).abs().max() / f64[c].abs().max())
    for i in range(NSPECIES):
        d = (mix[3 + i] - f64[3 + i]).abs().max()
        out[f"rho{i}_vs_change"] = float(d / (f64[3 + i] - rho0[i]).abs().max())
        out[f"rho{i}"] = float(d / f64[3 + i].abs().max())
    out["pi"] = float((mix[-1] - f64[-1]).abs().max() / f64[-1].abs().max())
    return out


def dist_init(args):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(ws, v, torch, dev):
    if ws == 1:
        return v
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------
# CPU baseline: the oracle (C++ FP64 restatement, OpenMP on all host
# threads) on a bounded sample of the workload
# ----------------------------------------------------------------------
class OracleCase:
    """the bench workload on the CPU oracle at n^3 (a sample of the 256^3
    step: the same mixture, scales and tolerances, 1/8 of the cells at
    128^3), stepped with fresh host noise every step"""

    def __init__(self, n):
        import numpy as np

        import oracle as O
        O.build()
        self.O, self.np, self.n = O, np, n
        nc = n ** 3
        self.nc = nc
        rng = np.random.default_rng(7)
        self.umac = [1e-3 * rng.standard_normal(nc) for _ in range(3)]
        w = 0.25 + 1e-3 * rng.standard_normal((NSPECIES, nc))
        w /= w.sum(axis=0)
        self.rho = [np.ascontiguousarray(w[i]) for i in range(NSPECIES)]
        self.pi = np.zeros(nc)
        self.ones = np.ones(nc)
        self.sp = O.StochParams(k_B=KT, variance_coef_mom=1.0, dV=DX ** 3, stoch_stress_form=1, filtering_width=0)
        self.mp = O.mixture_params(**mixture())
        self.params = O.default_params(gmres_rel_tol=REL_TOL)
        self.W_prev = self.mass_noise(0)
        self.F = O.mass_fluxdiv(3, [n] * 3, DX, self.sp, self.mp, self.rho, DT, [1.0], self.W_prev)

    def mass_noise(self, k):
        r = self.np.random.default_rng(1000 + k)
        return [r.standard_normal(self.nc) for _ in range(3 * NSPECIES)]

    def noise(self, k):
        r = self.np.random.default_rng(5000 + k)
        W_cc = [r.standard_normal(self.nc) * 2 ** 0.5 for _ in range(3)]
        W_ed = []
        for _ in range(3):
            a = r.standard_normal(self.nc)
            W_ed += [a, a]
        return W_cc, W_ed, self.mass_noise(k)

    def step(self, k):
        """one timed inertial step k (its noise is drawn before the clock
        starts); returns the seconds it took"""
        W_cc, W_ed, W_new = self.noise(k)
        t0 = time.perf_counter()
        rc, self.umac, self.rho, self.pi, self.F, _ = self.O.advance_inertial_ms(
            3, [self.n] * 3, DX, 1, self.params, self.sp, self.mp, DT, self.umac, self.rho, self.pi, self.F,
            self.ones, [self.ones] * 3, self.np.zeros(self.nc), self.ones, [self.ones] * 3, W_cc, W_ed,
            list(self.W_prev) + list(W_new))
        sec = time.perf_counter() - t0
        if rc < 0:
            raise RuntimeError(f"oracle step failed: {rc}")
        self.W_prev = W_new
        return sec


def sample_text(n_sample, n_full, sec):
    scale = (n_full / n_sample) ** 3
    return (f"FP64 4-species inertial steps of this workload at {n_sample}^3 (1/{scale:g} of the {n_full}^3 cells; "
            f"{sec:.2f} s each) on the CPU oracle, OpenMP on all host threads; value = 1 / ({scale:g} x seconds "
            f"per {n_sample}^3 step), since the GMRES iteration count does not grow with the grid under multigrid "
            f"preconditioning")


def cpu_sample(n_sample: int, n_full: int):
    oc = OracleCase(n_sample)
    sec = oc.step(1)
    scale = (n_full / n_sample) ** 3
    return {"value": 1.0 / (sec * scale), "unit": "steps/s", "cores": oc.O.num_threads(), "kind": "port",
            "sample": "one of the " + sample_text(n_sample, n_full, sec)}


def run_reference(args):
    """the reference arm: the CPU oracle (the reference itself cannot be
    built here: Fortran on FBoxLib) on W untimed and K timed sample steps of
    the workload; rank 0 only"""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    n_s = args.cpu_sample_n
    oc = OracleCase(n_s)
    secs = []
    for k in range(1, args.warmup + args.steps + 1):
        sec = oc.step(k)
        if k > args.warmup:
            secs.append(sec)
    sec = sum(secs) / len(secs)
    scale = (args.n / n_s) ** 3
    v = 1.0 / (sec * scale)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": 0,
            "steps": len(secs), "warmup": args.warmup, "ms_per_step": sec * 1e3,
            "value_from_ms_per_step": f"value = 1 / ({scale:g} x ms_per_step / 1000): each timed step is a {n_s}^3 "
                                      f"step, 1/{scale:g} of the {args.n}^3 step's cells",
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded N(0,1) fields)",
            "config": {"workload": WORKLOAD, "n_cells": [args.n] * 3, "dx": DX, "dt": DT, "k_B": KT,
                       "gmres_rel_tol": REL_TOL, "visc_type": 1, "species": NSPECIES, "molmass": MOLMASS,
                       "sample_n_cells": [n_s] * 3},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": oc.O.num_threads(), "kind": "port",
                             "sample": sample_text(n_s, args.n, sec)},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# finest-level smoother kernel by the kind of plan the autotuner picked
SMOOTHER_KERNEL = {
    "rowtile": "k_stag_rbx (finest-level row-tile fused red-black smooth of all three components)",
    "tiled": "k_stag_rb (finest-level tiled fused red-black smooth)",
    "colour": "k_stag_gs (finest-level colour sweep)",
    "rules": "finest-level smoother of the fixed size rules",
}


def run_leg(L, torch, dev, args, precision, rank, ws, e2e):
    """W warm-up and K timed steps of one precision with fresh device noise
    every step (drawn inside the timed region); then, if e2e, K more steps
    through the same public call with every step's noise uploaded from
    pinned host memory inside the timed region"""
    n, K, W = args.n, args.steps, args.warmup
    nc = n ** 3
    case = Case(L, torch, dev, n, precision)
    # the context launches on a torch-owned stream so that torch's
    # pinned-memory and caching allocators never see a destroyed stream
    stream = torch.cuda.Stream(device=dev)
    case.s.set_stream(stream.cuda_stream)
    noise = L.StepNoise(3, [n] * 3, NSPECIES, NOISE_SEED + rank, dev, stream.cuda_stream)
    torch.cuda.synchronize()
    noise.draw_mass(0)
    case.init_fluxes(noise.mass(0))
    rho0 = [r.clone() for r in case.rho]

    def step(k):
        noise.draw(k)
        return case.step(*noise.inertial_args(k))

    for k in range(1, W + 1):
        step(k)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = Clocks(dev.index or 0)
    if precision == "mixed":
        clocks.start()
    launches0 = case.s.kernel_launches
    case.s.profile(True)
    iters = []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    # an NVTX range around the timed steps, so that a profiler can be
    # restricted to them (ncu --nvtx --nvtx-include "timed_mixed/")
    torch.cuda.nvtx.range_push(f"timed_{precision}")
    ev0.record(stream)
    for k in range(W + 1, W + K + 1):
        st, stats = step(k)
        iters.append([x["total_iters"] for x in stats])
    ev1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    ms = ev0.elapsed_time(ev1)
    barrier(ws)
    prof = case.s.profile_read()
    case.s.profile(False)
    # the smoother plans the autotuner picked for the finest levels
    plan = {"stag_level0": case.s.tune_info("stag", 0), "cc_level0": case.s.tune_info("cc", 0)}
    launches = case.s.kernel_launches - launches0 + K * noise.launches_per_draw()
    clk = clocks.stop() if precision == "mixed" else None
    res = dict(ms=allmax(ws, ms, torch, dev), iters=iters, prof=prof, launches=launches, clocks=clk, plan=plan,
               resid=stats[-1]["norm_resid"] / max(stats[0]["norm_pre_b"], 1e-300), final=case.snapshot(),
               rho0=rho0, rho_min=min(float(r.min()) for r in case.rho))
    if e2e:
        res["e2e"] = run_e2e(torch, dev, case, stream, noise.mass(W + K), K, rank, ws)
    case.s.close()
    del case
    torch.cuda.empty_cache()
    return res


def run_e2e(torch, dev, case, stream, mass_prev, K, rank, ws):
    """K steps through the public step call, each step's N(0,1) fields
    copied from pinned host memory inside the timed region (18 fields of
    nc doubles: 3 cell, 3 edge, 12 mass-face), overlapped with the previous
    step on a copy stream, and each step's solver diagnostics read back"""
    nc = case.nc
    pool = HostNoisePool(torch, case.n, K, NOISE_SEED + 7919 * (rank + 1))
    h2d = (3 + 3 + 3 * NSPECIES) * nc * 8
    # three staging sets: step i computes on set i%3 (and reads the previous
    # step's mass noise from set (i-1)%3) while a copy stream uploads step
    # i+1's fields into set (i+1)%3, which the step before last finished with
    NS = 3
    mk = lambda m: [torch.empty(nc, dtype=torch.float64, device=dev) for _ in range(m)]
    stage = [(mk(3), mk(3), mk(3 * NSPECIES)) for _ in range(NS)]
    # the mass noise of the device-noise run's last step is the first e2e
    # step's previous-step noise
    for d_, s_ in zip(stage[NS - 1][2], mass_prev):
        d_.copy_(s_)
    torch.cuda.synchronize()
    barrier(ws)
    cs = torch.cuda.Stream(device=dev)
    copied = [torch.cuda.Event() for _ in range(K)]
    stepped = [torch.cuda.Event() for _ in range(K)]

    def upload(i):
        with torch.cuda.stream(cs):
            if i >= 2:
                cs.wait_event(stepped[i - 2])
            for part_d, part_h in zip(stage[i % NS], pool.fields(i)):
                for d_, h_ in zip(part_d, part_h):
                    d_.copy_(h_, non_blocking=True)
            copied[i].record(cs)

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    cs.wait_stream(stream)
    upload(0)
    with torch.cuda.stream(stream):
        for i in range(K):
            if i + 1 < K:
                upload(i + 1)
            stream.wait_event(copied[i])
            cur, prev = stage[i % NS], stage[(i - 1) % NS]
            W_ed = [e for e in cur[1] for _ in range(2)]
            case.step(cur[0], W_ed, list(prev[2]) + list(cur[2]))
            stepped[i].record(stream)
    stream.wait_stream(cs)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = allmax(ws, e0.elapsed_time(e1), torch, dev)
    del stage, pool
    return dict(ms=ms, h2d=h2d, d2h=2 * 80)  # the two solves' fhd_solve_stats per step


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.probe:
        return run_probe(args)
    import torch

    import lowmachfhd_b200 as L

    ws, rank, local = dist_init(args)
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    n = args.n
    hbm, peak_kind = peaks()

    results = {}
    for precision in ((args.only,) if args.only else ("mixed", "fp64")):
        results[precision] = run_leg(L, torch, dev, args, precision, rank, ws,
                                     e2e=(precision == "mixed" and not args.no_e2e))

    if args.only or args.no_e2e:
        if rank == 0:
            print(json.dumps({"partial_run": True, "only": args.only, "n": n, "steps": args.steps,
                              **{k: {"ms_per_step": v["ms"] / args.steps, "gpu_launches": v["launches"],
                                     "rho_min": v["rho_min"],
                                     "gmres_iters_per_step": [sum(x) for x in v["iters"]]}
                                 for k, v in results.items()}}), flush=True)
        return 0
    mixed, fp64 = results["mixed"], results["fp64"]
    errs = mixed_vs_fp64(mixed.pop("final"), fp64.pop("final"), fp64["rho0"])
    K = args.steps
    value = ws * K / (mixed["ms"] / 1e3)
    fp64_value = ws * K / (fp64["ms"] / 1e3)
    n_l, ms_l, bytes_l = mixed["prof"]
    achieved = (bytes_l / n_l) / ((ms_l / n_l) / 1e3) / 1e9 if n_l else None
    n64, ms64, b64 = fp64["prof"]
    achieved64 = (b64 / n64) / ((ms64 / n64) / 1e3) / 1e9 if n64 else None
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": K, "warmup": args.warmup,
        "ms_per_step": mixed["ms"] / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 multigrid / f64 Krylov",
        "data": "synthetic: seeded initial state; fresh N(0,1) stochastic fields every step",
        "config": {"workload": WORKLOAD, "n_cells": [n] * 3, "dx": DX, "dt": DT, "k_B": KT, "rho_total": 1.0,
                   "eta": 1.0, "visc_type": 1, "precon_type": 1, "gmres_rel_tol": REL_TOL, "species": NSPECIES,
                   "molmass": MOLMASS, "Dbar": "U[0.5,2]*1e-2 seeded", "w0": "0.25 + 1e-3 N(0,1), renormalised",
                   "noise": "drawn on the device every step inside the timed region (Philox-4x32-10, "
                            "18 fields of 16.8M doubles); e2e: uploaded from pinned host memory every step",
                   "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (each 256^3 field is 134 MB)"},
        "fp64": {"value": fp64_value, "unit": "steps/s", "ms_per_step": fp64["ms"] / K,
                 "gmres_iters_per_step": [sum(x) for x in fp64["iters"]]},
        "mixed_over_fp64": value / fp64_value,
        "mixed_vs_fp64": dict(errs, steps=args.warmup + K,
                              note="relative inf-norm differences of the mixed run's final fields from the FP64 "
                                   "run's; same initial state and noise"),
        "gmres_iters_per_step": [sum(x) for x in mixed["iters"]],
        "gmres_iters_per_s": ws * sum(sum(x) for x in mixed["iters"]) / (mixed["ms"] / 1e3),
        "corrector_resid_over_pre_rhs": mixed["resid"],
        "rho_min_final": mixed["rho_min"],
        "gpu_launches": mixed["launches"],
        "autotuned_plans": {"mixed": mixed["plan"], "fp64": fp64["plan"]},
        "roofline": {"kernel": SMOOTHER_KERNEL[mixed["plan"]["stag_level0"]["kind"]],
                     "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (achieved / hbm) if achieved else None,
                     # ncu DRAM read + write of one launch of the same kernel
                     # on the 256^3 finest level (635.5 + 181.4 MB)
                     "traffic": (635.5 + 181.4) * 1e6,
                     "traffic_source": "ncu capture of one 256^3 launch",
                     "peak_kind": peak_kind, "launches_timed": n_l,
                     "avg_launch_us": (ms_l / n_l * 1e3) if n_l else None,
                     "bytes_per_launch": (bytes_l / n_l) if n_l else None,
                     "fp64_kernel": SMOOTHER_KERNEL[fp64["plan"]["stag_level0"]["kind"]],
                     "fp64_achieved": achieved64},
        "clocks": mixed["clocks"],
        "e2e": {"value": ws * K / (mixed["e2e"]["ms"] / 1e3), "unit": "steps/s",
                "h2d_bytes_per_step": mixed["e2e"]["h2d"], "d2h_bytes_per_step": mixed["e2e"]["d2h"]},
    }
    if rank == 0 and not args.no_serve:
        served = run_serving(L, SERVE_SLOTS, "mixed", SERVE_RATE, SERVE_REQUESTS)
        saturated = run_serving(L, SERVE_SLOTS, "mixed", None, SERVE_REQUESTS)
        plain = run_serving(L, 1, "fp64", SERVE_RATE, SERVE_REQUESTS)
        line["served"] = {
            "config": {"arrivals": f"Poisson {SERVE_RATE:g}/s, seeded", "requests": SERVE_REQUESTS,
                       "sizes": "2D 64^2-512^2 overdamped, 3D 32^3-192^3 inertial, log-uniform, 1-4 species",
                       "steps_per_request": 4, "slots": SERVE_SLOTS, "hbm_budget_gb": SERVE_BUDGET >> 30,
                       "latency": "submit to result, after one warm-up request per kind and one per grid shape (autotuner table)"},
            "p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"],
            "mixed_continuous": served,
            "mixed_continuous_saturated": saturated,
            "fp64_one_at_a_time": plain,
        }
        line["batched"] = run_batched(L)
        line["batched"]["one_launch_per_level"] = run_batch_solver(L, torch, dev)
    if ws > 1:
        barrier(ws)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_sample(args.cpu_sample_n, n)
        except Exception as e:  # the baseline never decides the run
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
