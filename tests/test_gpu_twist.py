"""The two-ended ("twisted") line solve against the oracle.

Kinds "fp64-twist" (FP64 fields and elimination with FMA: fast FP64 contexts,
and a filter candidate of the mixed path), "fp32-twist" (FP32 derivative
fields) and "fp64-tile/fp32-twist" (filter of the FP64 state with an FP32
elimination) run two warps per tile of 32 lines: one eliminates from the
line's first row, the other from its last row (the factors of the system with
its ends swapped), and the four unknowns where they meet come from a 4 x 4
inverse. Lines of at least 32 points. Bounds: a few FP64 ulps of the field's
scale for the FP64 unit solves, FP32 rounding for the FP32 ones, and the
specification's 1e-10 / 1e-5 after 12 steps.
"""
import numpy as np
import pytest

import pyoracle as po
from canard_b200 import api, cases
from test_gpu_mixed import rel_l2, state_errors

pytestmark = pytest.mark.gpu

DIRS = ("xi", "eta", "zeta")


def noise_fields(cs, nn, n):
    blk = cs.blocks[0]
    rng = np.random.default_rng(20261204)
    pos = np.arange(n + 1)
    ax = {1: 2, 2: 1, 3: 0}[nn]
    modes = sum(np.sin(2 * np.pi * k * pos / n) for k in range(1, 33))
    bshape = [1, 1, 1]
    bshape[ax] = n + 1
    return np.stack([rng.standard_normal(blk.shape) + modes.reshape(bshape) for _ in range(5)])


@pytest.mark.parametrize("nn", [1, 2, 3])
@pytest.mark.parametrize("op,prec,kind,tol", [
    (0, api.FP64_FAST, "fp64-twist", 1e-13),
    (1, api.FP64_FAST, "fp64-twist", 1e-13),
    (0, api.FP32_MIXED, "fp32-twist", 5e-6),
    (1, api.FP32_MIXED, "fp64-tile/fp32-twist", 1e-7),
    (1, api.FP32_MIXED, "fp64-twist", 1e-13),
])
def test_twist_line_bench_five_noise_fields(nn, op, prec, kind, tol):
    """Five fields of N(0,1) noise plus sin(k x), k = 1..32, along a 257-point
    direction (the other two directions short): one launch of the two-ended
    kind against the oracle's deriv / filte of each field."""
    n = 256
    cs = cases.tgv(nx=n if nn == 1 else 24, ny=n if nn == 2 else 20, nz=n if nn == 3 else 16)
    fields = noise_fields(cs, nn, n)
    g = api.Context(cs, precision=prec, setup=False, upload_state=False)
    g.set_line_kind("flux" if op == 0 else "filter", DIRS[nn - 1], kind)
    out, _ = g.line_bench(op, nn, fields, reps=1)
    o = po.Oracle(cs, setup=False)
    inn = {2: 1, 3: 2, 1: 3}[nn]
    for k in range(5):
        f = fields[k].ravel().copy()
        if op == 0:
            o.mpigo([f], 0, 1, 0, 1, 1)
            d = np.zeros_like(f)
            o.deriv(0, f, d, nn, 1)
            ref = d
        else:
            o.mpigo([f], 1, 1, 0, k + 1, k + 1)
            o.filte(0, f, inn, k + 1)
            ref = f
        err = rel_l2(out[k].ravel(), ref)
        assert err <= tol, (nn, op, kind, k, err)


@pytest.mark.parametrize("L", [32, 33, 47])
def test_twist_short_and_odd_lines(L):
    """The shortest lines the kind takes (halves of 16 rows), and odd lengths:
    derivative and filter along eta against the oracle."""
    cs = cases.tgv(nx=20, ny=L - 1, nz=18)
    fields = noise_fields(cs, 2, L - 1)
    for op, tol in ((0, 1e-13), (1, 1e-13)):
        g = api.Context(cs, precision=api.FP64_FAST, setup=False, upload_state=False)
        g.set_line_kind("flux" if op == 0 else "filter", "eta", "fp64-twist")
        out, _ = g.line_bench(op, 2, fields, reps=1)
        o = po.Oracle(cs, setup=False)
        for k in range(5):
            f = fields[k].ravel().copy()
            if op == 0:
                o.mpigo([f], 0, 1, 0, 1, 1)
                d = np.zeros_like(f)
                o.deriv(0, f, d, 2, 1)
                ref = d
            else:
                o.mpigo([f], 1, 1, 0, k + 1, k + 1)
                o.filte(0, f, 1, k + 1)
                ref = f
            err = rel_l2(out[k].ravel(), ref)
            assert err <= tol, (L, op, k, err)
        g.close()


def test_twist_kind_rejected_on_short_lines():
    cs = cases.tgv(nx=24, ny=20, nz=16)
    g = api.Context(cs, precision=api.FP64_FAST, setup=False, upload_state=False)
    with pytest.raises(api.CanardError):
        g.set_line_kind("flux", "xi", "fp64-twist")


def twist_cases():
    return {
        "periodic": lambda: cases.tgv(nx=40, ny=36, nz=32),
        "multiblock": lambda: cases.curvilinear_4block(40, 32, 31),
    }


@pytest.mark.parametrize("name", list(twist_cases()))
@pytest.mark.parametrize("prec,kinds,tol", [
    (api.FP64_FAST, ("fp64-twist", "fp64-twist"), 1e-10),
    (api.FP32_MIXED, ("fp64-tile/fp32-twist", "fp32-twist"), 1e-5),
])
def test_twist_steps_within_tolerance(name, prec, kinds, tol):
    """Every line group in every direction pinned to the two-ended kinds
    (periodic lines with the in-kernel contraction; block interfaces, GCBC
    faces and sponge on the 4-block grid): 12 steps against the oracle."""
    cs = twist_cases()[name]()
    o = po.Oracle(cs)
    g = api.Context(cs, precision=prec)
    for d in DIRS:
        g.set_line_kind("filter", d, kinds[0])
        g.set_line_kind("viscous", d, kinds[1])
        g.set_line_kind("flux", d, kinds[1])
    o.step(12)
    g.step(12)
    uref = 0.1 if name == "periodic" else 0.4
    for b in range(len(cs.blocks)):
        errs = state_errors(g.state(b), o.state(b), uref)
        assert max(errs) <= tol, (name, b, errs)
