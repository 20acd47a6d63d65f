"""The quad split derivative (four lanes per line) against the oracle.

Kinds "fp64-quad" (FP64 fields, fast FP64 contexts) and "fp32-quad" (FP32
fields, mixed-precision contexts) solve each derivative line in four segments
joined by the homogeneous recurrences; they apply to lines long enough for four
segments that each outlast the recurrences' decay (about 4 x 60 points in FP64,
4 x 40 in FP32). Bounds: a few FP64 ulps of the field's scale for the FP64 unit
solves, FP32 rounding for the FP32 ones, and the specification's 1e-10 / 1e-5
after 12 steps.
"""
import numpy as np
import pytest

import pyoracle as po
from canard_b200 import api, cases
from test_gpu_mixed import rel_l2, state_errors

pytestmark = pytest.mark.gpu


def noise_case(nn, n=256):
    return cases.tgv(nx=n if nn == 1 else 24, ny=n if nn == 2 else 20, nz=n if nn == 3 else 16)


@pytest.mark.parametrize("nn", [1, 2, 3])
@pytest.mark.parametrize("prec,kind,tol", [(api.FP64_FAST, "fp64-quad", 1e-13), (api.FP32_MIXED, "fp32-quad", 5e-6)])
def test_quad_line_bench_five_noise_fields(nn, prec, kind, tol):
    """Five fields of N(0,1) noise plus sin(k x), k = 1..32, along a 257-point
    direction: one launch of the quad kind against the oracle's deriv."""
    cs = noise_case(nn)
    blk = cs.blocks[0]
    rng = np.random.default_rng(20261203)
    n = 256
    pos = np.arange(n + 1)
    ax = {1: 2, 2: 1, 3: 0}[nn]
    modes = sum(np.sin(2 * np.pi * k * pos / n) for k in range(1, 33))
    bshape = [1, 1, 1]
    bshape[ax] = n + 1
    fields = np.stack([rng.standard_normal(blk.shape) + modes.reshape(bshape) for _ in range(5)])
    g = api.Context(cs, precision=prec, setup=False, upload_state=False)
    g.set_line_kind("flux", "xi eta zeta".split()[nn - 1], kind)
    out, _ = g.line_bench(0, nn, fields, reps=1)
    o = po.Oracle(cs, setup=False)
    for k in range(5):
        f = fields[k].ravel().copy()
        o.mpigo([f], 0, 1, 0, 1, 1)
        d = np.zeros_like(f)
        o.deriv(0, f, d, nn, 1)
        err = rel_l2(out[k].ravel(), d)
        assert err <= tol, (nn, kind, k, err)


def test_quad_kind_rejected_on_short_lines():
    cs = cases.tgv(nx=24, ny=20, nz=16)
    g = api.Context(cs, precision=api.FP64_FAST, setup=False, upload_state=False)
    with pytest.raises(api.CanardError):
        g.set_line_kind("flux", "xi", "fp64-quad")


@pytest.mark.parametrize("prec,kind,tol", [(api.FP64_FAST, "fp64-quad", 1e-10), (api.FP32_MIXED, "fp32-quad", 1e-5)])
def test_quad_steps_within_tolerance(prec, kind, tol):
    """A Taylor-Green block with 257-point xi lines, the viscous gradients and
    flux derivatives along xi pinned to the quad kind: 12 steps against the
    oracle."""
    cs = cases.tgv(nx=256, ny=20, nz=16)
    o = po.Oracle(cs)
    g = api.Context(cs, precision=prec)
    g.set_line_kind("viscous", "xi", kind)
    g.set_line_kind("flux", "xi", kind)
    o.step(12)
    g.step(12)
    errs = state_errors(g.state(0), o.state(0), 0.1)
    assert max(errs) <= tol, errs
