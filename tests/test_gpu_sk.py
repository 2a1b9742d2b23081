"""Static structure factor of the velocity in the 3D inertial scheme
(advance_timestep_inertial.f90:45-923): with equilibrium initial
fluctuations (the variance k_B T/(rho dV) per face of
stochastic_m_fluxdiv.f90:964-968, projected onto discretely divergence-free
fields) the centred Crank-Nicolson scheme with its consistent noise keeps
S(k) = sum_i <|u_i(k)|^2> / (N_c (d-1)) at k_B T/(rho dV) for every mode.
The configuration is 3D periodic 128^3, rho = eta = 1, k_B T = 1e-3,
dt = 0.05, 100 steps in FP64; the check is the time average over steps
20-100, shell by shell, within 2 %.  FFTs and random fields are test
harness (torch); every step goes through the C ABI."""
import math

import numpy as np
import pytest

import lowmachfhd_b200 as L

pytestmark = pytest.mark.gpu


def _projected_fluctuations(torch, n, var, gen, dev):
    """N(0, var) face velocities projected onto the kernel of the discrete
    divergence of the MAC grid (low-side faces: div u = sum_d (u_d(i+e_d) -
    u_d(i))/dx, Fourier symbol exp(i k_d) - 1)"""
    shape = (n, n, n)  # (z, y, x)
    u = [torch.randn(shape, generator=gen, device=dev, dtype=torch.float64) * math.sqrt(var) for _ in range(3)]
    U = [torch.fft.fftn(x) for x in u]
    k = 2 * math.pi * torch.fft.fftfreq(n, device=dev, dtype=torch.float64)
    kz, ky, kx = torch.meshgrid(k, k, k, indexing="ij")
    g = [torch.exp(1j * kk) - 1 for kk in (kx, ky, kz)]
    gg = sum((gi.conj() * gi).real for gi in g)
    gg[0, 0, 0] = 1.0
    dot = sum(gi * Ui for gi, Ui in zip(g, U))
    U = [Ui - gi.conj() * dot / gg for gi, Ui in zip(g, U)]
    return [torch.fft.ifftn(Ui).real.contiguous().reshape(-1) for Ui in U]


def test_velocity_structure_factor_flat(cuda):
    import torch
    n, dt, kT, steps, first = 128, 0.05, 1e-3, 100, 20
    nc = n ** 3
    dev = cuda
    gen = torch.Generator(device=dev).manual_seed(2024)
    f64 = dict(dtype=torch.float64, device=dev)
    var = kT / (1.0 * 1.0)  # k_B T / (rho dV), dV = 1
    u = _projected_fluctuations(torch, n, var, gen, dev)
    rho = torch.ones(nc, **f64)
    pi = torch.zeros(nc, **f64)
    eta = torch.ones(nc, **f64)
    eta_ed = [torch.ones(nc, **f64) for _ in range(3)]
    kappa = torch.zeros(nc, **f64)
    T = torch.ones(nc, **f64)
    T_ed = [torch.ones(nc, **f64) for _ in range(3)]
    sp = L.StochParams(k_B=kT, variance_coef_mom=1.0, dV=1.0, stoch_stress_form=1, filtering_width=0)
    kk = torch.fft.fftfreq(n, d=1.0 / n, device=dev)
    kz, ky, kx = torch.meshgrid(kk, kk, kk, indexing="ij")
    shell = torch.sqrt(kx ** 2 + ky ** 2 + kz ** 2).round().long().reshape(-1)
    nshell = int(shell.max()) + 1
    counts = torch.bincount(shell, minlength=nshell).double()
    acc = torch.zeros(nshell, **f64)
    samples = 0
    # the library's device structure factor of the same samples (HydroGrid's
    # S_ii, no phase shift: |u_i(k)|^2 does not depend on it)
    sk = L.StructureFactor(3, [n, n, n], 1.0, 3, [(0, 0), (1, 1), (2, 2)])
    with L.StokesSolver(3, [n, n, n], 1.0, 1, params=L.default_params(gmres_rel_tol=1e-9)) as s:
        for step in range(1, steps + 1):
            W_cc = [torch.randn(nc, generator=gen, **f64) * math.sqrt(2.0) for _ in range(3)]
            W_ed = []
            for _ in range(3):
                a = torch.randn(nc, generator=gen, **f64)
                W_ed += [a, a]
            status, stats = s.advance_timestep_inertial(sp, dt, u, rho, pi, eta, eta_ed, kappa, T, T_ed, W_cc, W_ed)
            assert status in (0, 3)
            if step > first:
                S = sum((torch.fft.fftn(x.reshape(n, n, n)).abs() ** 2) for x in u).reshape(-1) / (nc * 2)
                acc += torch.bincount(shell, weights=S, minlength=nshell)
                samples += 1
                sk.update(u)
    acc = acc.cpu().numpy()
    counts = counts.cpu().numpy()
    # device S(k): half spectrum, modes 0 < kx < n/2 stand for their mirror
    # images too; shell sums of the running mean times the samples must equal
    # the shell sums of the torch spectra above
    dev_sk = sum(sk.read(p)[0].real for p in range(3)) / 2.0
    sk.close()
    w = np.full(n // 2 + 1, 2.0)
    w[0] = w[n // 2] = 1.0
    half = shell.reshape(n, n, n)[:, :, : n // 2 + 1].cpu().numpy().reshape(-1)
    dev_acc = np.bincount(half, weights=(dev_sk * w[None, None, :]).reshape(-1), minlength=nshell) * samples
    assert np.max(np.abs(dev_acc[:nshell] - acc)) <= 1e-10 * np.max(np.abs(acc))
    ref = kT
    # flatness: bands of 8 shells from |k| = 8 to 64 (each > 1e4 modes, so
    # the sampling error is well below the 2 % bar; the lowest shells hold
    # a handful of slowly decorrelating modes and enter only the mean)
    bands = [(lo, lo + 8) for lo in range(8, 64, 8)]
    ratios = [acc[lo:hi].sum() / (counts[lo:hi].sum() * samples) / ref for lo, hi in bands]
    mean = acc[1:64].sum() / (counts[1:64].sum() * samples) / ref
    print("S(k)/(kT/(rho dV)) by |k| band:", {f"{lo}-{hi}": round(float(r), 4) for (lo, hi), r in zip(bands, ratios)},
          "mean", round(float(mean), 4))
    for (lo, hi), r in zip(bands, ratios):
        assert abs(r - 1.0) < 0.02, (lo, hi, r)
    assert abs(mean - 1.0) < 0.01, mean
