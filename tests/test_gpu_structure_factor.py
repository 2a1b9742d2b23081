"""Device static structure factors (fhd_sk_*) against a numpy restatement of
HydroGrid's updateStructureFactors (HydroGrid/HydroGridModule.f90:
1077-1180) and writeStructureFactors' normalisation (1862-1868): per sample
the unnormalised DFT of each field, the staggered phase shift exp(i s k_d
pi / N_d) of velocity component d (1119-1141), the running mean of
Ua conj(Ub), times dV / N_cells.  Different FFT algorithms, so the bar is
1e-12 of the largest mode."""
import numpy as np
import pytest

import lowmachfhd_b200 as L

pytestmark = pytest.mark.gpu


def _reference(fields, dim, n, dV, pairs, shift):
    """numpy restatement: fields is a list of samples, each a list of
    flat arrays in the canonical layout (x fastest)"""
    shape = tuple(reversed(n[:dim]))  # (nz,) ny, nx
    # integer wavenumbers in FFT order with the Nyquist mode positive, as
    # HydroGrid orders them (0 1 2 3 -2 -1 for N = 6)
    def wavenumbers(N):
        k = np.arange(N)
        return np.where(k > N // 2, k - N, k)
    waves = [np.arange(n[0] // 2 + 1)] + [wavenumbers(n[d]) for d in range(1, dim)]
    grids = np.meshgrid(*reversed(waves), indexing="ij")  # (kz,) ky, kx
    kd = list(reversed(grids))  # kx, ky, (kz)
    acc = [np.zeros(grids[0].shape, complex) for _ in pairs]
    for it, sample in enumerate(fields, start=1):
        U = []
        for v, f in enumerate(sample):
            u = np.fft.rfftn(f.reshape(shape))
            s = shift[v] if shift is not None else 0
            if s:
                u = u * np.exp(1j * s * kd[v] * np.pi / n[v])
            U.append(u)
        for p, (a, b) in enumerate(pairs):
            acc[p] = ((it - 1) * acc[p] + U[a] * np.conj(U[b])) / it
    nc = int(np.prod(n[:dim]))
    return [a * dV / nc for a in acc]


@pytest.mark.parametrize("dim,n,shift", [(3, [32, 24, 16], [1, -1, 1, 0]), (2, [48, 32], [1, 1, 0]),
                                         (3, [16, 16, 16], None)])
def test_structure_factor_matches_numpy(cuda, dim, n, shift):
    import torch
    nvars = 4 if dim == 3 else 3
    pairs = [(0, 0), (1, 1), (0, 1), (nvars - 1, nvars - 1), (1, nvars - 1)]
    dV = 0.37
    rng = np.random.default_rng(5)
    nc = int(np.prod(n))
    samples = [[rng.standard_normal(nc) for _ in range(nvars)] for _ in range(3)]
    ref = _reference(samples, dim, n, dV, pairs, shift)
    with L.StructureFactor(dim, n, dV, nvars, pairs, shift) as sk:
        for sample in samples:
            sk.update([torch.from_numpy(f).to(cuda) for f in sample])
        for p in range(len(pairs)):
            got, ns = sk.read(p)
            assert ns == 3
            assert got.shape == ref[p].shape
            scale = np.max(np.abs(ref[p]))
            assert np.max(np.abs(got - ref[p])) <= 1e-12 * scale, p


def test_structure_factor_rejects_bad_pairs(cuda):
    with pytest.raises(L.FhdError):
        L.StructureFactor(3, [8, 8, 8], 1.0, 2, [(0, 2)])
    with pytest.raises(L.FhdError):
        L.StructureFactor(2, [8, 8], 1.0, 3, [(0, 0)], shift=[0, 0, 1])
