"""The smoother autotuner (fhd_ctx_set_tune): every candidate plan it may
pick -- colour launches with each thread-block shape, the tiled fused smooth
with each tile, the row-tile smooth with each tile height -- forced on every
level in turn, against the fixed size rules on the same inputs.  FP64 plans
evaluate the same expression on the same operands, so they agree bitwise;
FP32 plans agree to FP32 roundoff, the bar of the fused-smoother tests.  Then
the tuned choice itself: timed once per level shape, cached for the process,
and the same solution."""
import numpy as np
import pytest

import lowmachfhd_b200 as L
from tests import problems as P
from tests.test_gpu_parity import dev, host, zeros

pytestmark = pytest.mark.gpu

# (dim, n, visc_type, precision): row-tile, tiled and colour candidates on
# FP32 visc_type 1; tiled and colour on FP64 with variable and coupled
# viscosity; colour block shapes only in 2D
# (every finest level here is too large for the single-CTA coarse kernel,
# so the finest levels of both multigrids smooth through launches)
CASES = [(3, [128, 64, 64], 1, "mixed"), (3, [32, 32, 32], -1, "fp64"), (3, [32, 16, 32], 2, "fp64"),
         (2, [128, 128], 1, "mixed"), (2, [256, 128], -1, "fp64"), (3, [256, 32, 32], 1, "mixed")]


def _run(cuda, dim, n, visc, precision, tune, seed=71):
    pb = P.problem(dim, n, visc, dx=1.0, seed=seed, variable=(visc < 0) or None)
    rhs, _ = P.random_stokes(dim, n, seed=seed + 1)
    b_u, b_p = P.random_stokes(dim, n, seed=seed + 2, zero_mean_p=False)
    with L.StokesSolver(dim, n, 1.0, visc, params=L.default_params(), precision=precision) as s:
        s.set_tune(tune)
        coef = (dev(pb.alpha_fc, cuda), dev(pb.beta, cuda), dev(pb.beta_ed, cuda), dev(pb.gamma, cuda))
        phi = zeros(pb.nc, dim, cuda)
        s.stag_mg_solver(*coef, 0.7, phi, dev(rhs, cuda))
        x_u, x_p = zeros(pb.nc, dim, cuda), zeros(pb.nc, 1, cuda)[0]
        s.apply_precon(dev(b_u, cuda), dev(b_p, cuda), x_u, x_p, *coef, 1.5)
        info = (s.tune_info("stag", 0), s.tune_info("cc", 0))
    return host(phi) + host(x_u) + [host(x_p)], info


def _agree(a, b, precision):
    if precision == "fp64":
        return all(np.array_equal(x, y) for x, y in zip(a, b))
    return P.rel_inf(a, b) < 1e-5


@pytest.mark.parametrize("dim,n,visc,precision", CASES)
def test_every_candidate_matches_the_rules(cuda, dim, n, visc, precision):
    ref, info0 = _run(cuda, dim, n, visc, precision, 0)
    assert info0[0]["kind"] == "rules"
    _, info = _run(cuda, dim, n, visc, precision, 2)
    ncand = max(info[0]["candidates"], info[1]["candidates"])
    assert ncand >= (2 if dim == 2 else 4)
    kinds = set()
    for k in range(ncand):
        out, info = _run(cuda, dim, n, visc, precision, 2 + k)
        kinds.update(i["kind"] for i in info)
        assert _agree(out, ref, precision), (k, info)
    expect = {"colour"} if dim == 2 else {"colour", "tiled"}
    if dim == 3 and visc == 1 and precision == "mixed":
        expect.add("rowtile")
    assert expect <= kinds


@pytest.mark.parametrize("dim,n,visc,precision", [CASES[0], CASES[1], CASES[3]])
def test_tuned_plan_is_timed_cached_and_equal(cuda, dim, n, visc, precision):
    ref, _ = _run(cuda, dim, n, visc, precision, 0)
    out1, info1 = _run(cuda, dim, n, visc, precision, -1)
    out2, info2 = _run(cuda, dim, n, visc, precision, 1)
    for info in (info1, info2):
        for lv in info:
            assert lv["kind"] in ("colour", "tiled", "rowtile")
            assert lv["candidates"] >= 1 and lv["pair_us"] > 0
    # the second context reuses the first one's measurement
    assert info1 == info2
    assert _agree(out1, ref, precision)
    assert _agree(out2, out1, "fp64")


def test_imported_plan_is_used_untimed(cuda):
    """a plan imported as text (fhd_tune_import) is taken, untimed, by the
    first solve of its shape, and gives the rules' result"""
    dim, n, visc, precision = 3, [64, 64, 32], 1, "mixed"  # a shape no other test tunes
    cands = L.tune_candidates("stag", dim, n, precision, visc)
    idx = next(i for i, c in enumerate(cands) if c["kind"] == "tiled")
    import torch
    pr = torch.cuda.get_device_properties(cuda)
    key = L.tune_key("stag", dim, n, precision, visc, sms=pr.multi_processor_count,
                     smem_optin=pr.shared_memory_per_block_optin, smem_sm=pr.shared_memory_per_multiprocessor,
                     device=cuda.index or 0)
    line = f"{key} {idx}"
    assert L.tune_import(line + "\n") == 1
    ref, _ = _run(cuda, dim, n, visc, precision, 0)
    out, info = _run(cuda, dim, n, visc, precision, -1)
    st = info[0]
    assert st["kind"] == "tiled" and st["pair_us"] == 0 and st["candidates"] == len(cands)
    assert st["shape"][:2] == [cands[idx]["x"], cands[idx]["y"]]
    assert _agree(out, ref, precision)
    assert line in L.tune_export().splitlines()
