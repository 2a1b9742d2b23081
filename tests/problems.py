"""Seeded synthetic problems in the canonical periodic layout, shared by the
oracle tests and the GPU parity tests (numpy on the host)."""
import numpy as np

import oracle as O


def nc_of(dim, n):
    return int(np.prod(n[:dim]))


def coefficients(dim, n, visc_type, seed=0, variable=None):
    """alpha_fc (faces), beta (cells), beta_ed (nodes/edges from
    average_cc_to_node/edge), gamma (cells).  Variable coefficients for
    visc_type < 0, constants otherwise (as the constant-coefficient stencils
    read beta, gamma of the first cell)."""
    rng = np.random.default_rng(seed)
    nc = nc_of(dim, n)
    variable = (visc_type < 0) if variable is None else variable
    if variable:
        beta = 1.0 + 0.5 * rng.random(nc)
        gamma = 0.5 + 0.5 * rng.random(nc)
        rho = 1.0 + 0.3 * rng.random(nc)
    else:
        beta = np.full(nc, 1.3)
        gamma = np.full(nc, 0.7)
        rho = np.ones(nc)
    alpha_fc = O.average_cc_to_face(dim, n, rho)
    beta_ed = O.average_cc_to_edge(dim, n, beta)
    return alpha_fc, beta, beta_ed, gamma


def problem(dim, n, visc_type, dx=1.0, seed=0, variable=None):
    a, b, be, g = coefficients(dim, n, visc_type, seed, variable)
    return O.Problem(dim, n, dx, visc_type, a, b, be, g)


def random_stokes(dim, n, seed=1, zero_mean_p=True):
    rng = np.random.default_rng(seed)
    nc = nc_of(dim, n)
    u = [rng.standard_normal(nc) for _ in range(dim)]
    p = rng.standard_normal(nc)
    if zero_mean_p:
        p -= p.mean()
    return u, p


def stochastic_fields(dim, n, seed=1, n_rngs=1, symmetric=True):
    """N(0,1) fields as fill_m_stochastic prepares them
    (stochastic_m_fluxdiv.f90:781-860): cell entries with variance 2 and
    equal edge components for the symmetric form."""
    rng = np.random.default_rng(seed)
    nc = nc_of(dim, n)
    nE = 1 if dim == 2 else 3
    W_cc, W_ed = [], []
    for r in range(n_rngs):
        for c in range(dim):
            w = rng.standard_normal(nc)
            W_cc.append(w * np.sqrt(2.0) if symmetric else w)
        for e in range(nE):
            a = rng.standard_normal(nc)
            b = a.copy() if symmetric else rng.standard_normal(nc)
            W_ed += [a, b]
    return W_cc, W_ed


def rel_inf(a, b):
    """max |a-b| / max |b| over a list of arrays"""
    num = max(float(np.max(np.abs(x - y))) for x, y in zip(a, b))
    den = max(float(np.max(np.abs(y))) for y in b)
    return num / den if den > 0 else num
