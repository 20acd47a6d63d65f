"""The fast FP64 mode (CANARD_FP64_FAST) against the FP64 oracle.

A fast FP64 context keeps every value in FP64 but solves each compact line in
two halves: the derivatives with two lanes per line, the halves joined by the
homogeneous solutions, and the filter (on lines of at least 32 points) with the
two-ended solve, one warp eliminating from each end; both with FMA contraction
in the eliminations. It filters the five fields direction by direction. Its results therefore differ from the
reference's operation order at the rounding level only. The bound its steps
are held to is the specification's: relative L2 error <= 1e-10 per conserved
variable after 10-12 steps (momenta against ||rho|| * U_ref where that exceeds
their own norm, as in the mixed-precision tests). Unit line solves are checked
at a few FP64 ulps of the field's scale.
"""
import numpy as np
import pytest

import pyoracle as po
from canard_b200 import api, cases
from test_gpu_mixed import CASES, UREF, rel_l2, smooth_fields, state_errors

pytestmark = pytest.mark.gpu

TOL_STEPS = 1e-10


@pytest.mark.parametrize("name", list(CASES))
def test_unit_deriv_fast64(name):
    cs = CASES[name]()
    o = po.Oracle(cs, setup=False)
    g = api.Context(cs, precision=api.FP64_FAST, setup=False, upload_state=False)
    f = smooth_fields(cs, 3)
    o.mpigo([x.copy() for x in f], 0, 1, 0, 1, 1)
    g.mpigo([x.copy() for x in f], 0, 1, 0, 1, 1)
    for b, blk in enumerate(cs.blocks):
        for nn in (1, 2, 3):
            a = np.zeros(blk.npts)
            c = np.zeros(blk.npts)
            o.deriv(b, f[b], a, nn, 1)
            g.deriv(b, f[b], c, nn, 1)
            err = rel_l2(c, a)
            assert err <= 1e-13, (name, b, nn, err)


@pytest.mark.parametrize("name", list(CASES))
def test_unit_filter_fast64(name):
    cs = CASES[name]()
    o = po.Oracle(cs, setup=False)
    g = api.Context(cs, precision=api.FP64_FAST, setup=False, upload_state=False)
    fo = smooth_fields(cs, 5)
    fg = [x.copy() for x in fo]
    for m in (1, 2):
        for inn in (1, 2, 3):
            o.mpigo(fo, 1, 1, 0, 3 * (m - 1) + inn, m)
            g.mpigo(fg, 1, 1, 0, 3 * (m - 1) + inn, m)
            for b in range(len(cs.blocks)):
                o.filte(b, fo[b], inn, m)
                g.filte(b, fg[b], inn, m)
                assert rel_l2(fg[b], fo[b]) <= 1e-14, (name, m, inn, b, rel_l2(fg[b], fo[b]))


@pytest.mark.parametrize("op", [0, 1])
@pytest.mark.parametrize("nn", [1, 2, 3])
def test_line_bench_five_noise_fields(nn, op):
    """Five fields of N(0,1) noise plus sin(k x) modes, k = 1..32, on a
    257-point line direction: one launch of the split FP64 solve against the
    oracle's deriv / filte of each field."""
    n = 256
    cs = cases.tgv(nx=n if nn == 1 else 24, ny=n if nn == 2 else 20, nz=n if nn == 3 else 16)
    blk = cs.blocks[0]
    rng = np.random.default_rng(20261203)
    pos = np.arange(n + 1)
    shape = blk.shape
    ax = {1: 2, 2: 1, 3: 0}[nn]
    modes = sum(np.sin(2 * np.pi * k * pos / n) for k in range(1, 33))
    bshape = [1, 1, 1]
    bshape[ax] = n + 1
    fields = np.stack([rng.standard_normal(shape) + modes.reshape(bshape) for _ in range(5)])
    g = api.Context(cs, precision=api.FP64_FAST, setup=False, upload_state=False)
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
        assert err <= 1e-13, (nn, op, k, err)


@pytest.mark.parametrize("name", list(CASES))
def test_steps_fast64_within_1e_10(name):
    cs = CASES[name]()
    o = po.Oracle(cs)
    g = api.Context(cs, precision=api.FP64_FAST)
    o.step(12)
    g.step(12)
    np.testing.assert_array_equal(g.time()[:2], o.time()[:2])
    for b in range(len(cs.blocks)):
        errs = state_errors(g.state(b), o.state(b), UREF[name])
        print(name, b, ["%.2e" % e for e in errs])
        assert max(errs) <= TOL_STEPS, (name, b, errs)


def test_tgv64_fast64_ten_steps():
    cs = cases.tgv(64)
    o = po.Oracle(cs)
    g = api.Context(cs, precision=api.FP64_FAST)
    o.step(10)
    g.step(10)
    errs = state_errors(g.state(0), o.state(0), 0.1)
    print("tgv64", ["%.2e" % e for e in errs])
    assert max(errs) <= TOL_STEPS, errs


def test_autotuned_fast64_within_1e_10():
    cs = CASES["multiblock"]()
    g = api.Context(cs, precision=api.FP64_FAST)
    rep = g.autotune(reps=2)
    assert len(rep) == 9
    o = po.Oracle(cs)
    g.step(12)
    o.step(12)
    for b in range(len(cs.blocks)):
        errs = state_errors(g.state(b), o.state(b), UREF["multiblock"])
        assert max(errs) <= TOL_STEPS, (b, errs, rep)


def test_split_kind_in_a_bit_exact_context_stays_within_rounding():
    """The split FP64 kind pinned for one group of a plain FP64 context: its
    12 steps stay within the tolerance of the bit-exact run."""
    cs = CASES["nonperiodic"]()
    a = api.Context(cs)
    b = api.Context(cs)
    for d in ("xi", "eta", "zeta"):
        b.set_line_kind("flux", d, "fp64-split")
    a.step(12)
    b.step(12)
    errs = state_errors(b.state(0), a.state(0), UREF["nonperiodic"])
    assert max(errs) <= TOL_STEPS, errs
